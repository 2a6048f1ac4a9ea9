/*
 * ocfd_oracle.h -- CPU FP64 oracle for the OpenCFD-SCU per-RK-stage RHS path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * algorithm (OpenCFD-SCU, src/OCFD_*.cu) used as the checker for the CUDA
 * product in opencfd-scu_b200/.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py may load it.  Nothing in the
 * product links against it.
 *
 * Layout follows the reference so that golden files written by the reference
 * build compare index-for-index:
 *   - primitive and metric fields live on the LAP box, LAP = 4,
 *     f[(k)*(ny+8)*(nx+8) + (j)*(nx+8) + (i)], i,j,k in [0, n+8)
 *     (head/cuda_utility.h:16-17, get_Field_LAP);
 *   - conserved f, fn, du are SoA without ghosts, [5][nz][ny][nx]
 *     (head/cuda_utility.h:25, get_SoA).
 *
 * Parity is pinned against the reference's own CUDA build run on a B200
 * (oracle/ref.mk builds it; tests/golden/ holds its outputs).
 */
#ifndef OCFD_ORACLE_H
#define OCFD_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define ORO_LAP 4

typedef struct oro_config {
    int nx, ny, nz;            /* interior cells (single rank: NX_GLOBAL...)   */
    int iperiodic[3];          /* IPERIODIC                                     */
    int jac_bound[3];          /* JAC_BOUND                                     */
    int d0_bound[6];           /* DIF_BOUND                                     */
    int non_ref[6];            /* NON_REFLETION                                 */
    int scheme_invis;          /* 301 UP7 .. 310 SCHEME_HYBRIDAUTO              */
    int scheme_vis;            /* 203 CD6, 204 CD8                              */
    int charteric;             /* CHARTERIC                                     */
    int hy_style;              /* HY_STYLE (2 = Jameson sensor)                 */
    double hy_dp_intv[2];      /* HY_DP_INTV                                    */
    double re, ama, gamma, pr, t_ref, epsl_sw, dt;
    double weno_tv_limiter;    /* src/parameters.c:75 (5.0)                     */
    double weno_tv_max;        /* src/parameters.c:76 (0.2)                     */
    int nthreads;              /* OpenMP threads (<=0: runtime default)         */
    int hy_nochar_fixed;       /* CHARTERIC=0 hybrid, components 1-4: 0 = use the
                                  face flag (intent); 1/2/3 = force that flag
                                  (what an uninitialised register yields)       */
    int ibc;                   /* IBC: 0 none, 108 compression corner           */
    int bc_npara[4];           /* 108: MZMAX MTMAX INLET_BOUNDARY IFLAG_WALL_NOT_NORMAL */
    double bc_rpara[8];        /* 108: TW EPSL X_DIST_BEGIN X_DIST_END BETA
                                  X_WALL_BEGIN X_UP_BOUNDARY_BEGIN SLZ          */
    int nfilter;               /* number of FILTER_NPARA<n> entries (<= 8)      */
    int filter_ipara[8][11];   /* ntime, fx, fy, fz, ib, ie, jb, je, kb, ke, scheme */
    double filter_rpara[8][3]; /* s0, rth, time limit                           */
} oro_config;

typedef struct oro_state oro_state;

oro_state *oro_create(const oro_config *cfg);
void oro_destroy(oro_state *s);

/* Metric fields, interior values, 13 records in the order of
 * OCFD3d-Jacobi.dat: Axx Ayy Azz Akx Aky Akz Aix Aiy Aiz Asx Asy Asz Ajac,
 * each [nz][ny][nx].  Ghosts follow Init_Jacobian3d
 * (src/OCFD_Comput_Jacobian3d.cu:32-218): 1.0 everywhere, then periodic
 * exchange in the periodic directions. */
void oro_set_metrics(oro_state *s, const double *fields13);
/* Mesh coordinates x,y,z, interior [3][nz][ny][nx] (OCFD3d-Mesh.dat): the
 * metrics are computed as Comput_Jacobian3d does
 * (src/OCFD_Comput_Jacobian3d.cu:221-424); JAC_BOUND selects the one-sided
 * derivative closures at both ends of a direction. */
void oro_set_mesh(oro_state *s, const double *xyz3);
/* 1 when a Jacobian on the LAP box is negative (ana_Jac, src/OCFD_ana.cu:24-48). */
int oro_negative_jacobian(const oro_state *s);
/* The 13 metric fields, interior, in OCFD3d-Jacobi.dat order. */
void oro_get_metrics(const oro_state *s, double *fields13);

/* Initial primitives d,u,v,w,T, interior [5][nz][ny][nx] (opencfd.dat).
 * Mirrors init() (src/OCFD_init.cu:26-131): ghosts zero, pri_to_cons. */
void oro_set_primitives(oro_state *s, const double *prim5, int istep, double tt);

/* Inlet profile of IBC 108 (flow1d-inlet.dat columns d,u,v,T), [4][ny];
 * without it (INLET_BOUNDARY = 0) the profile is d=u=T=1, v=0. */
void oro_set_inlet(oro_state *s, const double *ub1);

/* Pre-loop of NS_solver_real (src/OCFD_NS_Solver.cu:45-53). */
void oro_prepare(oro_state *s);

/* Per-stage API (same names and order as the reference driver). */
void oro_du_comput(oro_state *s, int krk);       /* src/OCFD_Stream.cu:28  */
void oro_time_advance(oro_state *s, int krk);    /* src/OCFD_time.cu:96    */
void oro_get_duvwT(oro_state *s);                /* src/commen_kernel.cu:111 */
void oro_bc(oro_state *s);                       /* src/OCFD_boundary.cu:18  */
void oro_get_amu(oro_state *s);                  /* src/commen_kernel.cu:133 */
void oro_swap_time_levels(oro_state *s);         /* src/OCFD_NS_Solver.cu:63-73 */

/* nsteps full RK3 steps (swap + 3 stages, Istep++, filtering),
 * src/OCFD_NS_Solver.cu:63-95. */
void oro_step(oro_state *s, int nsteps);
/* filtering() (src/OCFD_filtering.cu:75-183) at the current Istep / tt. */
void oro_filtering(oro_state *s);

/* Read-back helpers (interior only). */
void oro_get_primitives(const oro_state *s, double *prim5);   /* d u v w T  */
void oro_get_pressure(const oro_state *s, double *p);
void oro_get_conserved(const oro_state *s, double *f5);
void oro_get_conserved_n(const oro_state *s, double *f5);
void oro_get_du(const oro_state *s, double *du5);
void oro_get_flags(const oro_state *s, int *sx, int *sy, int *sz);
/* Q criterion of the current primitives, interior [nz][ny][nx]: get_Q
 * (src/OCFD_ana.cu:317-456) after the ghost exchange of u, v, w. */
void oro_q_criterion(oro_state *s, double *q);
/* the first n draws of the C library's rand() from its initial state */
void oro_libc_rand(int n, int *out);
int  oro_istep(const oro_state *s);
double oro_tt(const oro_state *s);

/* Point kernels exposed for unit tests (reference formulas, stencils as in
 * the reference: P side stencil[k] = f(i-3+k), k=0..7; M side f(i-4+k)). */
double oro_weno7_p(const double *s7);
double oro_weno7_m(const double *s7);
double oro_weno5_p(const double *s5);
double oro_weno5_m(const double *s5);
double oro_up7_p(const double *s8);
double oro_up7_m(const double *s8);
double oro_omp6_p(int flag, const double *s8);
double oro_omp6_m(int flag, const double *s8);
double oro_nnd2_p(const double *s3);
double oro_nnd2_m(const double *s3);
double oro_weno7_symbo_p(int lmt, double tv_lim, double tv_max, const double *s8);
double oro_weno7_symbo_m(int lmt, double tv_lim, double tv_max, const double *s8);
double oro_cd6(const double *s7);
double oro_cd8(const double *s9);
/* Steger-Warming split of one point: out[0..4] = f+, out[5..9] = f-. */
void oro_sw_split(double d, double u, double v, double w, double cc,
                  double a1, double a2, double a3, double gamma, double epsl_sw,
                  double *out10);
/* Characteristic matrices at a face: L (5x5 row-major) and R (5x5 row-major). */
void oro_char_matrices(double u1, double v1, double w1, double c1,
                       double a1, double a2, double a3, double gamma,
                       double *L25, double *R25);

#ifdef __cplusplus
}
#endif
#endif
