/*
 * ocfd_oracle.c -- CPU FP64 oracle for the OpenCFD-SCU per-RK-stage RHS path.
 *
 * TEST INFRASTRUCTURE ONLY (see ocfd_oracle.h).  Every function restates the
 * reference algorithm and cites the reference file:line it follows.  Formula
 * order is kept as written in the reference so that results agree to the
 * last few ulps; the build uses -ffp-contract=off so no FMA is introduced.
 *
 * Reference quirks replicated (default behaviour of the reference build):
 *   - ghost cells are filled only for the interior range of the two other
 *     directions; edge/corner ghosts of the primitive fields stay 0
 *     (src/OCFD_mpi_dev.cu:186-310, src/OCFD_init.cu:37-40);
 *   - the hybrid sensor at KRK=1 reads ghost values of d,T from the previous
 *     exchange, i.e. one stage old (src/OCFD_Stream.cu:34 precedes :291);
 *   - conserved variables are re-projected from the primitives on all six
 *     faces every stage (src/OCFD_boundary.cu:40-91);
 *   - du is accumulated in kernel order x+,x-,y+,y-,z+,z-,vis x,y,z
 *     (src/OCFD_Stream.cu:289-335), here by a single writer.
 */
#include "ocfd_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define LAP ORO_LAP

struct oro_state {
    oro_config c;
    int nx, ny, nz;
    int nx2, ny2, nz2;          /* n + 2*LAP */
    size_t nlap;                /* LAP box size */
    size_t nin;                 /* interior size */
    /* derived constants, src/OCFD_init.cu:381-399, :29-31 */
    double hx, hy, hz;
    double Cv, Cp, Tsb, amu_C0, tmp0, split_C1, split_C3, vis_flux_init_c;
    /* LAP-box fields */
    double *d, *u, *v, *w, *T, *P, *cc;
    double *A[13];              /* Axx Ayy Azz Akx Aky Akz Aix Aiy Aiz Asx Asy Asz Ajac */
    double *psens;              /* Comput_P output (sensor input) */
    double *fp[3], *fm[3];      /* split fluxes [5][LAP box] per direction */
    double *ev[4];              /* viscous Ev1..4, LAP box */
    /* interior fields */
    double *amu;
    double *grad[12];           /* uk ui us vk vi vs wk wi ws Tk Ti Ts */
    double *vis[4];
    double *f, *fn, *du;        /* [5][nz][ny][nx] */
    int *sch[3];                /* hybrid flags: (nx+1)ny nz, nx(ny+1)nz, nx ny(nz+1) */
    int istep;
    double tt;
    /* filtering: pf_lap (U after the stage-3 RK update, before the face
     * re-projection) and the ranges as set_para_filtering leaves them */
    double *flap;               /* [5][LAP box] */
    int fpar[8][11];
    int fjudge[3];
    /* IBC 108 (bc_user_Compression_conner_init, src/OCFD_boundary_init.c:376-438) */
    int bc_ready, x_begin;
    double *ub1;                /* [4][ny] d u v T */
    double *bfx, *bgz;          /* [nx], [nz] blowing shapes */
    double TM[64];
};

enum { AXX = 0, AYY, AZZ, AKX, AKY, AKZ, AIX, AIY, AIZ, ASX, ASY, ASZ, AJAC };

static inline size_t L(const oro_state *s, int i, int j, int k) {
    return (size_t)i + (size_t)s->nx2 * ((size_t)j + (size_t)s->ny2 * (size_t)k);
}
static inline size_t I(const oro_state *s, int i, int j, int k) {
    return (size_t)i + (size_t)s->nx * ((size_t)j + (size_t)s->ny * (size_t)k);
}

static double *xcalloc(size_t n) {
    double *p = (double *)calloc(n ? n : 1, sizeof(double));
    if (!p) { fprintf(stderr, "oracle: out of memory\n"); abort(); }
    return p;
}

/* ------------------------------------------------------------------------ */
/* construction                                                              */
/* ------------------------------------------------------------------------ */

oro_state *oro_create(const oro_config *cfg) {
    oro_state *s = (oro_state *)calloc(1, sizeof(oro_state));
    s->c = *cfg;
    if (s->c.weno_tv_limiter == 0.0) s->c.weno_tv_limiter = 5.0;   /* src/parameters.c:75 */
    if (s->c.weno_tv_max == 0.0) s->c.weno_tv_max = 0.2;           /* src/parameters.c:76 */
    if (s->c.t_ref <= 0) s->c.t_ref = 288.15;                      /* src/parameters.c:497 */
    s->nx = cfg->nx; s->ny = cfg->ny; s->nz = cfg->nz;
    s->nx2 = s->nx + 2 * LAP; s->ny2 = s->ny + 2 * LAP; s->nz2 = s->nz + 2 * LAP;
    s->nlap = (size_t)s->nx2 * s->ny2 * s->nz2;
    s->nin = (size_t)s->nx * s->ny * s->nz;
#ifdef _OPENMP
    if (cfg->nthreads > 0) omp_set_num_threads(cfg->nthreads);
#endif
    /* init(): hx = 1/(NX_GLOBAL-1)  (src/OCFD_init.cu:29-31) */
    s->hx = 1.0 / (s->nx - 1.0);
    s->hy = 1.0 / (s->ny - 1.0);
    s->hz = 1.0 / (s->nz - 1.0);
    /* opencfd_para_init (src/OCFD_init.cu:381-399) */
    double G = s->c.gamma, Ma = s->c.ama;
    s->Cv = 1.0 / (G * (G - 1.0) * Ma * Ma);
    s->Cp = 1.0 / ((G - 1.0) * Ma * Ma);
    s->Tsb = 110.4 / s->c.t_ref;
    s->amu_C0 = 1.0 / s->c.re * (1.0 + 110.4 / s->c.t_ref);
    s->tmp0 = 1.0 / (2.0 * G);
    s->split_C1 = 2.0 * (G - 1.0);
    s->split_C3 = (3.0 - G) / (2.0 * (G - 1.0));
    s->vis_flux_init_c = s->Cp / s->c.pr;

    s->d = xcalloc(s->nlap); s->u = xcalloc(s->nlap); s->v = xcalloc(s->nlap);
    s->w = xcalloc(s->nlap); s->T = xcalloc(s->nlap); s->P = xcalloc(s->nlap);
    /* one pressure field, as pP_d: Comput_P fills the LAP box at the first
     * stage of a step (sensor input), cons_to_pri_kernel rewrites the
     * interior each stage, the filter reads it after the step */
    s->cc = xcalloc(s->nlap); s->psens = s->P;
    for (int m = 0; m < 13; m++) {
        s->A[m] = xcalloc(s->nlap);
        for (size_t q = 0; q < s->nlap; q++) s->A[m][q] = 1.0;   /* Init_Jacobian3d :36-64 */
    }
    for (int dir = 0; dir < 3; dir++) { s->fp[dir] = xcalloc(5 * s->nlap); s->fm[dir] = xcalloc(5 * s->nlap); }
    for (int m = 0; m < 4; m++) { s->ev[m] = xcalloc(s->nlap); s->vis[m] = xcalloc(s->nin); }
    s->amu = xcalloc(s->nin);
    for (int m = 0; m < 12; m++) s->grad[m] = xcalloc(s->nin);
    s->f = xcalloc(5 * s->nin); s->fn = xcalloc(5 * s->nin); s->du = xcalloc(5 * s->nin);
    s->sch[0] = (int *)calloc((size_t)(s->nx + 1) * s->ny * s->nz, sizeof(int));
    s->sch[1] = (int *)calloc((size_t)s->nx * (s->ny + 1) * s->nz, sizeof(int));
    s->sch[2] = (int *)calloc((size_t)s->nx * s->ny * (s->nz + 1), sizeof(int));
    /* set_para_filtering (src/OCFD_filtering.cu:20-73) on a single rank:
     * ranges [ib, ie) etc. (0-based, without LAP), kept 6 cells away from
     * a non-periodic lower face and 5 from an upper one */
    s->flap = NULL;
    if (s->c.nfilter > 8) s->c.nfilter = 8;
    int nn[3] = { s->nx, s->ny, s->nz };
    for (int k = 0; k < s->c.nfilter; k++) {
        for (int t = 0; t < 11; t++) s->fpar[k][t] = s->c.filter_ipara[k][t];
        for (int d = 0; d < 3; d++) {
            if (s->fpar[k][1 + d] == 1) s->fjudge[d] = 1;
            if (s->c.iperiodic[d] != 1) {
                if (s->fpar[k][4 + 2 * d] < 6) s->fpar[k][4 + 2 * d] = 6;
                if (s->fpar[k][5 + 2 * d] > nn[d] - 5) s->fpar[k][5 + 2 * d] = nn[d] - 5;
            }
        }
    }
    if (s->c.nfilter > 0) s->flap = xcalloc(5 * s->nlap);
    s->bc_ready = 0;
    s->ub1 = xcalloc(4 * (size_t)s->ny);
    for (int j = 0; j < s->ny; j++) { s->ub1[j] = 1.0; s->ub1[s->ny + j] = 1.0; s->ub1[2 * s->ny + j] = 0.0; s->ub1[3 * s->ny + j] = 1.0; }
    s->bfx = xcalloc(s->nx); s->bgz = xcalloc(s->nz);
    return s;
}

void oro_set_inlet(oro_state *s, const double *ub1) {
    memcpy(s->ub1, ub1, 4 * (size_t)s->ny * sizeof(double));
}

/* rand() of the GNU C library from its initial state (srand(1)): a table
 * t[0] = 1, t[i] = 16807 t[i-1] mod 2147483647 (i < 31), t[31..33] =
 * t[0..2], then t[i] = t[i-3] + t[i-31] mod 2^32; draws are t[i] >> 1 for
 * i >= 344.  A ring of the last 34 values is enough. */
void oro_libc_rand(int n, int *out) {
    uint32_t t[34];
    t[0] = 1u;
    for (int i = 1; i < 31; i++) t[i] = (uint32_t)((16807ULL * t[i - 1]) % 2147483647ULL);
    for (int i = 31; i < 34; i++) t[i] = t[i - 31];
    int got = 0;
    for (long i = 34; got < n; i++) {
        uint32_t v = t[(i - 31) % 34] + t[(i - 3) % 34];
        t[i % 34] = v;
        if (i >= 344) out[got++] = (int)(v >> 1);
    }
}

/* x_begin, the blowing shapes fx (x) and gz (z) and the frequency weights TM,
 * from the wall and top coordinates (get_xs_blow_suction_multiwave,
 * get_fait_multifrequancy, src/OCFD_boundary_init.c:376-521).  MZMAX > 0
 * takes its MZMAX phases from the first rand() draws of the C library in its
 * initial state (nothing seeds it before, :444-499), restated by
 * oro_libc_rand. */
static void bc108_init(oro_state *s) {
    const double PI = 3.14159265358979323846;
    const double *Axx = s->A[AXX], *Azz = s->A[AZZ];
    double DB = s->c.bc_rpara[2], DE = s->c.bc_rpara[3], SL = s->c.bc_rpara[7], XUP = s->c.bc_rpara[6];
    int MZ = s->c.bc_npara[0], MT = s->c.bc_npara[1];
    s->x_begin = 0;
    for (int i = 0; i < s->nx; i++)
        if (Axx[L(s, i + LAP, s->ny + LAP - 1, LAP)] <= XUP) s->x_begin = i;
    for (int i = 0; i < s->nx; i++) {
        double xa = Axx[L(s, i + LAP, LAP, LAP)];
        if (xa >= DB && xa <= DE) {
            double seta = 10. * PI * (xa - DB)/(DB - DE);
            s->bfx[i] = 4. / sqrt(27.) * sin(seta) * (1. - cos(seta));
        } else {
            s->bfx[i] = 0.;
        }
    }
    double *faiz = NULL, *zl = NULL;
    if (MZ > 0) {
        int *draw = (int *)malloc(sizeof(int) * (size_t)MZ);
        faiz = (double *)malloc(sizeof(double) * (size_t)MZ);
        zl = (double *)malloc(sizeof(double) * (size_t)MZ);
        oro_libc_rand(MZ, draw);
        double ztmp = 0.;
        for (int m = 0; m < MZ; m++) {
            faiz[m] = draw[m] / (double)2147483647;     /* RAND_MAX */
            zl[m] = m == 0 ? 1. : zl[m - 1] / 1.25;
            ztmp += zl[m];
        }
        for (int m = 0; m < MZ; m++) zl[m] = zl[m] / ztmp;
        free(draw);
    }
    for (int k = 0; k < s->nz; k++) {
        double za = Azz[L(s, LAP, LAP, k + LAP)];
        double seta = za / SL;
        if (MZ > 0) {
            s->bgz[k] = 0.;
            for (int m = 0; m < MZ; m++) s->bgz[k] = s->bgz[k] + zl[m] * sin(2. * PI * (m + 1) * (seta + faiz[m]));
        } else if (MZ == 0) {
            s->bgz[k] = 1.;
        } else {
            s->bgz[k] = sin(-2. * PI * MZ * seta);
        }
    }
    free(faiz);
    free(zl);
    double Ttmp = 0.;
    for (int k = 0; k < MT && k < 64; k++) {
        s->TM[0] = 1.;
        if (k > 0) s->TM[k] = s->TM[k - 1] / 1.25;
        Ttmp = Ttmp + s->TM[k];
    }
    for (int k = 0; k < MT && k < 64; k++) s->TM[k] = s->TM[k] / Ttmp;
    s->bc_ready = 1;
}

/* bc_user_Compression_conner (src/OCFD_boundary_compression_conner.cu:122-180) */
static void bc108(oro_state *s) {
    if (!s->bc_ready) bc108_init(s);
    int nx = s->nx, ny = s->ny, nz = s->nz;
    const double *ub1 = s->ub1;
    /* inlet, i = 1: the ghost columns and the first column take the profile */
    for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i <= LAP; i++) {
                size_t q = L(s, i, j + LAP, k + LAP);
                s->d[q] = ub1[j]; s->u[q] = ub1[ny + j]; s->v[q] = ub1[2 * ny + j];
                s->w[q] = 0.; s->T[q] = ub1[3 * ny + j];
            }
    /* upper boundary from x_begin on */
    for (int k = 0; k < nz; k++)
        for (int i = s->x_begin; i < nx; i++) {
            size_t q = L(s, i + LAP, ny + LAP - 1, k + LAP);
            s->d[q] = ub1[ny - 1]; s->u[q] = ub1[ny + ny - 1]; s->v[q] = ub1[2 * ny + ny - 1];
            s->w[q] = 0.; s->T[q] = ub1[3 * ny + ny - 1];
        }
    double BETA = s->c.bc_rpara[4], EPSL = s->c.bc_rpara[1], TW = s->c.bc_rpara[0];
    double ht = 0.;
    if (BETA > 0.) {
        for (int m = 0; m < s->c.bc_npara[1] && m < 64; m++) ht = ht + s->TM[m] * sin((m + 1)*BETA*s->tt);
    } else {
        ht = 1.;
    }
    /* wall, j = 1: no slip with blowing, then the wall temperature */
    for (int k = 0; k < nz; k++)
        for (int i = 0; i < nx; i++) {
            size_t q = L(s, i + LAP, LAP, k + LAP);
            s->u[q] = 0.;
            s->v[q] = EPSL * s->bfx[i] * s->bgz[k] * ht;
            s->w[q] = 0.;
        }
    if (s->c.bc_npara[3] != 0) return;           /* "non-normal wall is not supported" */
    size_t sy = (size_t)s->nx2;
    for (int k = 0; k < nz; k++)
        for (int i = 0; i < nx; i++) {
            size_t q = L(s, i + LAP, LAP, k + LAP);
            double pw;
            if (TW > 0) {
                pw = (18. * s->d[q + sy] * s->T[q + sy] - 9. * s->d[q + 2 * sy] * s->T[q + 2 * sy]
                      + 2. * s->d[q + 3 * sy] * s->T[q + 3 * sy]) / 11.;
                s->T[q] = TW;
                s->d[q] = pw / s->T[q];
                for (int g = 0; g < LAP; g++) {
                    size_t qg = L(s, i + LAP, g, k + LAP), qm = L(s, i + LAP, 2 * LAP - g, k + LAP);
                    s->d[qg] = s->d[qm]; s->u[qg] = -s->u[qm]; s->v[qg] = -s->v[qm];
                    s->w[qg] = -s->w[qm]; s->T[qg] = s->T[qm];
                }
            } else {
                s->T[q] = (18. * s->T[q + sy] - 9. * s->T[q + 2 * sy] + 2. * s->T[q + 3 * sy]) / 11.;
                pw = (18. * s->d[q + sy] * s->T[q + sy] - 9. * s->d[q + 2 * sy] * s->T[q + 2 * sy]
                      + 2. * s->d[q + 3 * sy] * s->T[q + 3 * sy]) / 11.;
                s->d[q] = pw / s->T[q];
            }
        }
}

void oro_destroy(oro_state *s) {
    if (!s) return;
    free(s->d); free(s->u); free(s->v); free(s->w); free(s->T); free(s->P); free(s->cc);
    free(s->flap); free(s->ub1); free(s->bfx); free(s->bgz);
    for (int m = 0; m < 13; m++) free(s->A[m]);
    for (int dir = 0; dir < 3; dir++) { free(s->fp[dir]); free(s->fm[dir]); }
    for (int m = 0; m < 4; m++) { free(s->ev[m]); free(s->vis[m]); }
    free(s->amu);
    for (int m = 0; m < 12; m++) free(s->grad[m]);
    free(s->f); free(s->fn); free(s->du);
    for (int m = 0; m < 3; m++) free(s->sch[m]);
    free(s);
}

/* ------------------------------------------------------------------------ */
/* ghost exchange (single rank)                                              */
/* exchange_boundary_{x,y,z}_packed_dev, src/OCFD_mpi_dev.cu:186-310: the    */
/* x exchange covers y,z in the interior only, etc.  Non-periodic single     */
/* rank: the neighbour is MPI_PROC_NULL and nothing is written.              */
/* ------------------------------------------------------------------------ */

static void exchange_x(oro_state *s, double *f) {
    if (!s->c.iperiodic[0]) return;
    int nx = s->nx;
#pragma omp parallel for
    for (int k = LAP; k < s->nz + LAP; k++)
        for (int j = LAP; j < s->ny + LAP; j++)
            for (int i = 0; i < LAP; i++) {
                f[L(s, nx + LAP + i, j, k)] = f[L(s, LAP + i, j, k)];
                f[L(s, i, j, k)] = f[L(s, nx + i, j, k)];
            }
}
static void exchange_y(oro_state *s, double *f) {
    if (!s->c.iperiodic[1]) return;
    int ny = s->ny;
#pragma omp parallel for
    for (int k = LAP; k < s->nz + LAP; k++)
        for (int j = 0; j < LAP; j++)
            for (int i = LAP; i < s->nx + LAP; i++) {
                f[L(s, i, ny + LAP + j, k)] = f[L(s, i, LAP + j, k)];
                f[L(s, i, j, k)] = f[L(s, i, ny + j, k)];
            }
}
static void exchange_z(oro_state *s, double *f) {
    if (!s->c.iperiodic[2]) return;
    int nz = s->nz;
#pragma omp parallel for
    for (int k = 0; k < LAP; k++)
        for (int j = LAP; j < s->ny + LAP; j++)
            for (int i = LAP; i < s->nx + LAP; i++) {
                f[L(s, i, j, nz + LAP + k)] = f[L(s, i, j, LAP + k)];
                f[L(s, i, j, k)] = f[L(s, i, j, nz + k)];
            }
}
static void exchange_xyz(oro_state *s, double *f) {
    exchange_x(s, f); exchange_y(s, f); exchange_z(s, f);
}

/* ------------------------------------------------------------------------ */
/* set-up                                                                    */
/* ------------------------------------------------------------------------ */

void oro_set_metrics(oro_state *s, const double *fields13) {
    /* read_3d1 into the interior, then exchange_boundary_xyz
     * (src/OCFD_Comput_Jacobian3d.cu:142-201). */
    for (int m = 0; m < 13; m++) {
        const double *src = fields13 + (size_t)m * s->nin;
        for (int k = 0; k < s->nz; k++)
            for (int j = 0; j < s->ny; j++)
                for (int i = 0; i < s->nx; i++)
                    s->A[m][L(s, i + LAP, j + LAP, k + LAP)] = src[I(s, i, j, k)];
        exchange_xyz(s, s->A[m]);
    }
}

/* d(coordinate)/d(index) along dir for metrics: OCFD_d{x,y,z}0_CD6_kernel
 * (src/OCFD_Schemes.cu:1236-1304) over the interior, then, when JAC_BOUND of
 * the direction is non-zero, OCFD_D{x,y,z}0_bound_kernel_{m,p}
 * (src/OCFD_bound_Scheme.cu:189-349) on the four points at each end, with
 * each direction's own grouping of the terms. */
static void jac_d0(oro_state *s, const double *f, double *out, int dir) {
    size_t st[3] = { 1, (size_t)s->nx2, (size_t)s->nx2 * s->ny2 };
    long sd = (long)st[dir];
    double h = dir == 0 ? s->hx : (dir == 1 ? s->hy : s->hz);
    int n = dir == 0 ? s->nx : (dir == 1 ? s->ny : s->nz);
    int bound = s->c.jac_bound[dir] != 0;
#pragma omp parallel for
    for (int k = 0; k < s->nz; k++)
        for (int j = 0; j < s->ny; j++)
            for (int i = 0; i < s->nx; i++) {
                size_t q = L(s, i + LAP, j + LAP, k + LAP);
                const double *c = f + q;            /* c[t*sd] = f(X+t) */
#define F_(t) c[(long)(t) * sd]
                int X = dir == 0 ? i : (dir == 1 ? j : k);
                double v = (45.0*(F_(1) - F_(-1)) - 9.0*(F_(2) - F_(-2)) + (F_(3) - F_(-3)))/(60.0*h);
                if (bound) {
                    /* lower end: same grouping in x, y, z (points 0..6 of the line) */
                    if (X == 0) v = (F_(1) - F_(0))/h;
                    else if (X == 1) v = (F_(1) - F_(-1))*0.5/h;
                    else if (X == 2) v = (F_(-2) - 8.0*F_(-1) + 8.0*F_(1) - F_(2))/(12.0*h);
                    else if (X == 3) v = (F_(3) - F_(-3) - 9.0*(F_(2) - F_(-2)) + 45.0*(F_(1) - F_(-1)))/(60.0*h);
                    /* upper end, t = n-1 */
                    int u = X - (n - 1);
                    if (dir != 1) {
                        if (u == 0) v = (F_(0) - F_(-1))/h;
                        else if (u == -1) v = (F_(1) - F_(-1))*0.5/h;
                        else if (u == -2) v = (F_(-2) - 8.0*F_(-1) + 8.0*F_(1) - F_(2))/(12.0*h);
                        else if (u == -3) v = (F_(3) - F_(-3) - 9.0*(F_(2) - F_(-2)) + 45.0*(F_(1) - F_(-1)))/(60.0*h);
                    } else {
                        if (u == 0) v = -(F_(-1) - F_(0))/h;
                        else if (u == -1) v = -(F_(-1) - F_(1))*0.5/h;
                        else if (u == -2) v = -(F_(2) - 8.0*F_(1) + 8.0*F_(-1) - F_(-2))/(12.0*h);
                        else if (u == -3) v = -(F_(-3) - F_(3) - 9.0*(F_(-2) - F_(2)) + 45.0*(F_(-1) - F_(1)))/(60.0*h);
                    }
                }
#undef F_
                out[I(s, i, j, k)] = v;
            }
}

void oro_set_mesh(oro_state *s, const double *xyz3) {
    /* Init_Jacobian3d (src/OCFD_Comput_Jacobian3d.cu:32-141): every metric
     * field 1.0 on the LAP box, coordinates into Axx, Ayy, Azz, periodic
     * exchange of those three, then Comput_Jacobian3d (:221-246). */
    for (int m = 0; m < 13; m++)
        for (size_t q = 0; q < s->nlap; q++) s->A[m][q] = 1.0;
    for (int m = 0; m < 3; m++) {
        const double *src = xyz3 + (size_t)m * s->nin;
        for (int k = 0; k < s->nz; k++)
            for (int j = 0; j < s->ny; j++)
                for (int i = 0; i < s->nx; i++)
                    s->A[m][L(s, i + LAP, j + LAP, k + LAP)] = src[I(s, i, j, k)];
        exchange_xyz(s, s->A[m]);
    }
    /* comput_Jac3d (:393-424): xi..zk = d(x,y,z)/d(i,j,k) */
    double **D = s->grad;   /* scratch: D[3*dir + c] = d coord c / d index dir */
    for (int dir = 0; dir < 3; dir++)
        for (int c = 0; c < 3; c++) jac_d0(s, s->A[AXX + c], D[3 * dir + c], dir);
    /* comput_Jac3d_kernal (:250-391) */
    int nx = s->nx, ny = s->ny, nz = s->nz;
#pragma omp parallel for
    for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                size_t c = I(s, i, j, k), q = L(s, i + LAP, j + LAP, k + LAP);
                double xi1 = D[0][c], yi1 = D[1][c], zi1 = D[2][c];
                double xj1 = D[3][c], yj1 = D[4][c], zj1 = D[5][c];
                double xk1 = D[6][c], yk1 = D[7][c], zk1 = D[8][c];
                double Jac1 = 1.0 / (xi1 * yj1 * zk1 + yi1 * zj1 * xk1 + zi1 * xj1 * yk1
                                     - zi1 * yj1 * xk1 - yi1 * xj1 * zk1 - xi1 * zj1 * yk1);
                s->A[AJAC][q] = Jac1;
                s->A[AKX][q] = (yj1 * zk1 - zj1 * yk1);
                s->A[AKY][q] = (zj1 * xk1 - xj1 * zk1);
                s->A[AKZ][q] = (xj1 * yk1 - yj1 * xk1);
                s->A[AIX][q] = (yk1 * zi1 - zk1 * yi1);
                s->A[AIY][q] = (zk1 * xi1 - xk1 * zi1);
                s->A[AIZ][q] = (xk1 * yi1 - yk1 * xi1);
                s->A[ASX][q] = (yi1 * zj1 - zi1 * yj1);
                s->A[ASY][q] = (zi1 * xj1 - xi1 * zj1);
                s->A[ASZ][q] = (xi1 * yj1 - yi1 * xj1);
            }
    /* constant extrapolation into the ghost slabs of the 10 computed fields
     * (x ghosts for interior y,z; y ghosts for interior x,z; z ghosts for
     * interior x,y), then the periodic exchange overwrites periodic sides */
    for (int m = AKX; m <= AJAC; m++) {
        double *A = s->A[m];
        for (int k = 0; k < nz; k++)
            for (int j = 0; j < ny; j++)
                for (int g = 0; g < LAP; g++) {
                    A[L(s, g, j + LAP, k + LAP)] = A[L(s, LAP, j + LAP, k + LAP)];
                    A[L(s, nx + LAP + g, j + LAP, k + LAP)] = A[L(s, nx - 1 + LAP, j + LAP, k + LAP)];
                }
        for (int k = 0; k < nz; k++)
            for (int g = 0; g < LAP; g++)
                for (int i = 0; i < nx; i++) {
                    A[L(s, i + LAP, g, k + LAP)] = A[L(s, i + LAP, LAP, k + LAP)];
                    A[L(s, i + LAP, ny + LAP + g, k + LAP)] = A[L(s, i + LAP, ny - 1 + LAP, k + LAP)];
                }
        for (int g = 0; g < LAP; g++)
            for (int j = 0; j < ny; j++)
                for (int i = 0; i < nx; i++) {
                    A[L(s, i + LAP, j + LAP, g)] = A[L(s, i + LAP, j + LAP, LAP)];
                    A[L(s, i + LAP, j + LAP, nz + LAP + g)] = A[L(s, i + LAP, j + LAP, nz - 1 + LAP)];
                }
        exchange_xyz(s, A);
    }
}

int oro_negative_jacobian(const oro_state *s) {
    /* ana_Jac (src/OCFD_ana.cu:24-48): any Ajac < 0 on the LAP box */
    for (size_t q = 0; q < s->nlap; q++)
        if (s->A[AJAC][q] < 0) return 1;
    return 0;
}

void oro_get_metrics(const oro_state *s, double *fields13) {
    for (int m = 0; m < 13; m++) {
        double *dst = fields13 + (size_t)m * s->nin;
        for (int k = 0; k < s->nz; k++)
            for (int j = 0; j < s->ny; j++)
                for (int i = 0; i < s->nx; i++)
                    dst[I(s, i, j, k)] = s->A[m][L(s, i + LAP, j + LAP, k + LAP)];
    }
}

/* pri_to_cons_kernel (src/commen_kernel.cu:32-66) for one interior cell. */
static inline void p2c_cell(oro_state *s, int i, int j, int k) {
    size_t q = L(s, i + LAP, j + LAP, k + LAP), n = s->nin, c = I(s, i, j, k);
    double d = s->d[q], u = s->u[q], v = s->v[q], w = s->w[q], T = s->T[q];
    s->f[c] = d;
    s->f[c + n] = u * d;
    s->f[c + 2 * n] = v * d;
    s->f[c + 3 * n] = w * d;
    s->f[c + 4 * n] = d * ((u * u + v * v + w * w) * 0.5 + s->Cv * T);
}

void oro_set_primitives(oro_state *s, const double *prim5, int istep, double tt) {
    double *dst[5] = { s->d, s->u, s->v, s->w, s->T };
    for (int m = 0; m < 5; m++) {
        memset(dst[m], 0, s->nlap * sizeof(double));
        const double *src = prim5 + (size_t)m * s->nin;
        for (int k = 0; k < s->nz; k++)
            for (int j = 0; j < s->ny; j++)
                for (int i = 0; i < s->nx; i++)
                    dst[m][L(s, i + LAP, j + LAP, k + LAP)] = src[I(s, i, j, k)];
    }
    memset(s->P, 0, s->nlap * sizeof(double));
    memset(s->cc, 0, s->nlap * sizeof(double));
    memset(s->f, 0, 5 * s->nin * sizeof(double));
    memset(s->fn, 0, 5 * s->nin * sizeof(double));
    memset(s->du, 0, 5 * s->nin * sizeof(double));
#pragma omp parallel for
    for (int k = 0; k < s->nz; k++)
        for (int j = 0; j < s->ny; j++)
            for (int i = 0; i < s->nx; i++) p2c_cell(s, i, j, k);
    s->istep = istep;
    s->tt = tt;
}

/* ------------------------------------------------------------------------ */
/* common kernels                                                            */
/* ------------------------------------------------------------------------ */

/* get_Amu_kernal, src/commen_kernel.cu:122-132 */
void oro_get_amu(oro_state *s) {
#pragma omp parallel for
    for (int k = 0; k < s->nz; k++)
        for (int j = 0; j < s->ny; j++)
            for (int i = 0; i < s->nx; i++) {
                double t = s->T[L(s, i + LAP, j + LAP, k + LAP)];
                s->amu[I(s, i, j, k)] = s->amu_C0 * sqrt(t * t * t) / (s->Tsb + t);
            }
}

/* cons_to_pri_kernel, src/commen_kernel.cu:77-109 */
void oro_get_duvwT(oro_state *s) {
    size_t n = s->nin;
    double G = s->c.gamma, Ma = s->c.ama, Cv = s->Cv;
#pragma omp parallel for
    for (int k = 0; k < s->nz; k++)
        for (int j = 0; j < s->ny; j++)
            for (int i = 0; i < s->nx; i++) {
                size_t c = I(s, i, j, k), q = L(s, i + LAP, j + LAP, k + LAP);
                double d1 = s->f[c];
                double u1 = s->f[c + n] / d1;
                double v1 = s->f[c + 2 * n] / d1;
                double w1 = s->f[c + 3 * n] / d1;
                double T1 = s->f[c + 4 * n];
                double T2 = (T1 - 0.5 * d1 * (u1 * u1 + v1 * v1 + w1 * w1)) / (d1 * Cv);
                s->d[q] = d1; s->u[q] = u1; s->v[q] = v1; s->w[q] = w1; s->T[q] = T2;
                s->P[q] = T2 * d1 / (G * Ma * Ma);
            }
}

/* OCFD_bc (src/OCFD_boundary.cu:18-92): the IBC 108 boundary values, then
 * the face re-projection of all six faces. */
void oro_bc(oro_state *s) {
    if (s->c.ibc == 108) bc108(s);
    int nx = s->nx, ny = s->ny, nz = s->nz;
    for (int k = 0; k < nz; k++) for (int j = 0; j < ny; j++) { p2c_cell(s, 0, j, k); p2c_cell(s, nx - 1, j, k); }
    for (int k = 0; k < nz; k++) for (int i = 0; i < nx; i++) { p2c_cell(s, i, 0, k); p2c_cell(s, i, ny - 1, k); }
    for (int j = 0; j < ny; j++) for (int i = 0; i < nx; i++) { p2c_cell(s, i, j, 0); p2c_cell(s, i, j, nz - 1); }
}

void oro_prepare(oro_state *s) {
    /* src/OCFD_NS_Solver.cu:45-53 */
    exchange_xyz(s, s->d); exchange_xyz(s, s->u); exchange_xyz(s, s->v);
    exchange_xyz(s, s->w); exchange_xyz(s, s->T);
    oro_bc(s);
    oro_get_amu(s);
}

/* ------------------------------------------------------------------------ */
/* Steger-Warming splitting, src/OCFD_split.cu:92-142 (per direction),       */
/* called with tmp0 = d/(2 gamma) (:160).                                    */
/* ------------------------------------------------------------------------ */

static inline void sw_point(double tmp0, double u, double v, double w, double cc,
                            double A1, double A2, double A3, double G, double eps,
                            double split_C1, double split_C3, double *fp, double *fm) {
    double ss, E1, E2, E3, E1P, E2P, E3P, E1M, E2M, E3M;
    double uc1, uc2, vc1, vc2, wc1, wc2, vvc1, vvc2, vv, W2;
    ss = sqrt(A1 * A1 + A2 * A2 + A3 * A3);
    E1 = A1 * u + A2 * v + A3 * w;
    E2 = E1 - cc * ss;
    E3 = E1 + cc * ss;
    ss = 1.0 / ss;
    A1 *= ss; A2 *= ss; A3 *= ss;
    E1P = (E1 + sqrt(E1 * E1 + eps * eps)) * 0.50;
    E2P = (E2 + sqrt(E2 * E2 + eps * eps)) * 0.50;
    E3P = (E3 + sqrt(E3 * E3 + eps * eps)) * 0.50;
    E1M = E1 - E1P; E2M = E2 - E2P; E3M = E3 - E3P;
    uc1 = u - cc * A1; uc2 = u + cc * A1;
    vc1 = v - cc * A2; vc2 = v + cc * A2;
    wc1 = w - cc * A3; wc2 = w + cc * A3;
    vvc1 = (uc1 * uc1 + vc1 * vc1 + wc1 * wc1) * 0.50;
    vvc2 = (uc2 * uc2 + vc2 * vc2 + wc2 * wc2) * 0.50;
    vv = (G - 1.0) * (u * u + v * v + w * w);
    W2 = split_C3 * cc * cc;
    fp[0] = tmp0 * (split_C1 * E1P + E2P + E3P);
    fp[1] = tmp0 * (split_C1 * E1P * u + E2P * uc1 + E3P * uc2);
    fp[2] = tmp0 * (split_C1 * E1P * v + E2P * vc1 + E3P * vc2);
    fp[3] = tmp0 * (split_C1 * E1P * w + E2P * wc1 + E3P * wc2);
    fp[4] = tmp0 * (E1P * vv + E2P * vvc1 + E3P * vvc2 + W2 * (E2P + E3P));
    fm[0] = tmp0 * (split_C1 * E1M + E2M + E3M);
    fm[1] = tmp0 * (split_C1 * E1M * u + E2M * uc1 + E3M * uc2);
    fm[2] = tmp0 * (split_C1 * E1M * v + E2M * vc1 + E3M * vc2);
    fm[3] = tmp0 * (split_C1 * E1M * w + E2M * wc1 + E3M * wc2);
    fm[4] = tmp0 * (E1M * vv + E2M * vvc1 + E3M * vvc2 + W2 * (E2M + E3M));
}

void oro_sw_split(double d, double u, double v, double w, double cc,
                  double a1, double a2, double a3, double gamma, double epsl_sw,
                  double *out10) {
    double tmp0 = d * (1.0 / (2.0 * gamma));
    sw_point(tmp0, u, v, w, cc, a1, a2, a3, gamma, epsl_sw, 2.0 * (gamma - 1.0),
             (3.0 - gamma) / (2.0 * (gamma - 1.0)), out10, out10 + 5);
}

/* sound_speed_kernel (src/commen_kernel.cu:144-153) + Stager_Warming
 * (src/OCFD_split.cu:144-198) over the whole LAP box. */
static void split_all(oro_state *s) {
    double G = s->c.gamma, eps = s->c.epsl_sw, Ma = s->c.ama;
    size_t nl = s->nlap;
#pragma omp parallel for
    for (long q = 0; q < (long)nl; q++) {
        s->cc[q] = sqrt(s->T[q]) / Ma;
    }
#pragma omp parallel for
    for (long q = 0; q < (long)nl; q++) {
        double tmp0 = s->d[q] * s->tmp0;
        double u = s->u[q], v = s->v[q], w = s->w[q], cc = s->cc[q];
        double fp[5], fm[5];
        for (int dir = 0; dir < 3; dir++) {
            int a = AKX + 3 * dir;
            sw_point(tmp0, u, v, w, cc, s->A[a][q], s->A[a + 1][q], s->A[a + 2][q], G, eps,
                     s->split_C1, s->split_C3, fp, fm);
            for (int m = 0; m < 5; m++) {
                s->fp[dir][(size_t)m * nl + q] = fp[m];
                s->fm[dir][(size_t)m * nl + q] = fm[m];
            }
        }
    }
}

/* ------------------------------------------------------------------------ */
/* reconstruction point kernels, src/OCFD_Schemes.cu                         */
/* ------------------------------------------------------------------------ */

/* OCFD_weno7_kernel_P, src/OCFD_Schemes.cu:616-663; s[0..6] = f(i-3..i+3) */
double oro_weno7_p(const double *s) {
    double S0 = 0.0, S1 = 0.0, S2 = 0.0, S3 = 0.0, tmp, tmp1, tmp2;
    tmp  = -2.0*s[0] +  9.0*s[1] - 18.0*s[2] + 11.0*s[3]; S0 += 960*tmp*tmp;
    tmp1 = -6.0*s[0] + 24.0*s[1] - 30.0*s[2] + 12.0*s[3]; S0 += (1040.0)*tmp1*tmp1;
    tmp2 = -6.0*s[0] + 18.0*( s[1] - s[2] ) + 6.0*s[3];   S0 += (1043.0)*tmp2*tmp2;
    tmp  = tmp * tmp2; S0 += 80.0*tmp;

    tmp  =      s[1] - 6.0*s[2] +  3.0*s[3] + 2.0*s[4]; S1 += 960*tmp*tmp;
    tmp1 =                   6.0*s[2] - 12.0*s[3] + 6.0*s[4]; S1 += (1040.0)*tmp1*tmp1;
    tmp2 = -6.0*s[1] + 18.0*( s[2] - s[3] ) + 6.0*s[4]; S1 += (1043.0)*tmp2*tmp2;
    tmp  = tmp * tmp2; S1 += 80.0*tmp;

    tmp  = -2.0*s[2] - 3.0*s[3] +  6.0*s[4] -   s[5]; S2 += 960*tmp*tmp;
    tmp1 =                 6.0*s[3] - 12.0*s[4] + 6.0*s[5]; S2 += (1040.0)*tmp1*tmp1;
    tmp2 = -6.0*s[2] + 18.0*(s[3] - s[4]) + 6.0*s[5]; S2 += (1043.0)*tmp2*tmp2;
    tmp  = tmp * tmp2; S2 += 80.0*tmp;

    tmp  = -11.0*s[3] + 18.0*s[4] -  9.0*s[5] + 2.0*s[6]; S3 += 960*tmp*tmp;
    tmp1 =  12.0*s[3] - 30.0*s[4] + 24.0*s[5] - 6.0*s[6]; S3 += (1040.0)*tmp1*tmp1;
    tmp2 =  -6.0*s[3] + 18.0*( s[4] -  s[5] ) + 6.0*s[6];  S3 += (1043.0)*tmp2*tmp2;
    tmp  =  tmp * tmp2; S3 += 80.0*tmp;

    tmp  =        ((3.456e-4+S1)*(3.456e-4+S1))*((3.456e-4+S2)*(3.456e-4+S2))*((3.456e-4+S3)*(3.456e-4+S3));
    tmp1 = (12.0)*((3.456e-4+S0)*(3.456e-4+S0))*((3.456e-4+S2)*(3.456e-4+S2))*((3.456e-4+S3)*(3.456e-4+S3));
    tmp2 = (18.0)*((3.456e-4+S0)*(3.456e-4+S0))*((3.456e-4+S1)*(3.456e-4+S1))*((3.456e-4+S3)*(3.456e-4+S3));
    S3   =  (4.0)*((3.456e-4+S0)*(3.456e-4+S0))*((3.456e-4+S1)*(3.456e-4+S1))*((3.456e-4+S2)*(3.456e-4+S2));
    S2 = tmp2; S1 = tmp1; S0 = tmp;

    double am = S0 + S1 + S2 + S3;
    tmp1 = 0.0;
    tmp = -3.0*s[0] + 13.0*s[1] - 23.0*s[2] + 25.0*s[3]; tmp1 += S0*tmp;
    tmp =      s[1] -  5.0*s[2] + 13.0*s[3] +  3.0*s[4]; tmp1 += S1*tmp;
    tmp =     -s[2] +  7.0*s[3] +  7.0*s[4] -      s[5]; tmp1 += S2*tmp;
    tmp =  3.0*s[3] + 13.0*s[4] -  5.0*s[5] +      s[6]; tmp1 += S3*tmp;
    tmp1 /= (12.0*am);
    return tmp1;
}

/* OCFD_weno7_kernel_M, src/OCFD_Schemes.cu:691-741; s[0..6] = f(i-3..i+3), face i-1/2 */
double oro_weno7_m(const double *s) {
    double S0 = 0.0, S1 = 0.0, S2 = 0.0, S3 = 0.0, tmp, tmp1, tmp2;
    tmp  = -2.0*s[6] +  9.0*s[5] - 18.0*s[4] + 11.0*s[3]; S0 += 960*tmp*tmp;
    tmp1 = -6.0*s[6] + 24.0*s[5] - 30.0*s[4] + 12.0*s[3]; S0 += (1040.0)*tmp1*tmp1;
    tmp2 = -6.0*s[6] + 18.0*( s[5] -  s[4] ) + 6.0*s[3];  S0 += (1043.0)*tmp2*tmp2;
    tmp  = tmp * tmp2; S0 += (80.0) * tmp;

    tmp  =      s[5] -  6.0* s[4] + 3.0*s[3] + 2.0*s[2]; S1 += 960*tmp*tmp;
    tmp1 =                  6.0*s[4] - 12.0* s[3] +  6.0*s[2]; S1 += (1040.0)*tmp1*tmp1;
    tmp2 = -6.0*s[5] + 18.0*( s[4] -  s[3]) + 6.0*s[2];  S1 += (1043.0)*tmp2*tmp2;
    tmp  = tmp *tmp2; S1 += (80.0) * tmp;

    tmp  =    -2.0*s[4] - 3.0*s[3] + 6.0*s[2] - s[1]; S2 += 960*tmp*tmp;
    tmp1 =                 6.0*s[3] - 12.0*s[2] + 6.0*s[1]; S2 += (1040.0)*tmp1*tmp1;
    tmp2 = -6.0*s[4] + 18.0*(s[3] - s[2]) + 6.0*s[1]; S2 += (1043.0)*tmp2*tmp2;
    tmp  = tmp *tmp2; S2 += (80.0) * tmp;

    tmp  = -11.0*s[3] + 18.0*s[2] -  9.0*s[1] + 2.0*s[0]; S3 += 960*tmp*tmp;
    tmp1 =  12.0*s[3] - 30.0*s[2] + 24.0*s[1] - 6.0*s[0]; S3 += (1040.0)*tmp1*tmp1;
    tmp2 =  -6.0*s[3] + 18.0*( s[2] -  s[1] ) + 6.0*s[0]; S3 += (1043.0)*tmp2*tmp2;
    tmp  =  tmp *tmp2; S3 += (80.0) * tmp;

    tmp  =        ((3.456e-4+S1)*(3.456e-4+S1))*((3.456e-4+S2)*(3.456e-4+S2))*((3.456e-4+S3)*(3.456e-4+S3));
    tmp1 = (12.0)*((3.456e-4+S0)*(3.456e-4+S0))*((3.456e-4+S2)*(3.456e-4+S2))*((3.456e-4+S3)*(3.456e-4+S3));
    tmp2 = (18.0)*((3.456e-4+S0)*(3.456e-4+S0))*((3.456e-4+S1)*(3.456e-4+S1))*((3.456e-4+S3)*(3.456e-4+S3));
    S3   =  (4.0)*((3.456e-4+S0)*(3.456e-4+S0))*((3.456e-4+S1)*(3.456e-4+S1))*((3.456e-4+S2)*(3.456e-4+S2));
    S2 = tmp2; S1 = tmp1; S0 = tmp;

    double am = S0 + S1 + S2 + S3;
    tmp1 = 0.0;
    tmp = -3.0*s[6] + 13.0*s[5] - 23.0*s[4] + 25.0*s[3]; tmp1 += S0*tmp;
    tmp =      s[5] -  5.0*s[4] + 13.0*s[3] +  3.0*s[2]; tmp1 += S1*tmp;
    tmp =     -s[4] +  7.0*s[3] +  7.0*s[2] -      s[1]; tmp1 += S2*tmp;
    tmp =  3.0*s[3] + 13.0*s[2] -  5.0*s[1] +      s[0]; tmp1 += S3*tmp;
    tmp1 /= (12.0*am);
    return tmp1;
}

/* OCFD_weno5_kernel_P, src/OCFD_Schemes.cu:1118-1151; s[0..4] = f(i-2..i+2) */
double oro_weno5_p(const double *s) {
    double S0 = 0.0, S1 = 0.0, S2 = 0.0, tmp, ep = 1e-6;
    tmp =     s[2] - 2.0*s[3] + s[4]; S0 += 13*tmp*tmp;
    tmp = 3.0*s[2] - 4.0*s[3] + s[4]; S0 +=  3*tmp*tmp;
    double q03 = (2.0*s[2] + 5.0*s[3] - s[4]);
    tmp = s[1] - 2.0*s[2] + s[3]; S1 += 13*tmp*tmp;
    tmp =                  s[1] - s[3]; S1 +=  3*tmp*tmp;
    double q13 = (-s[1] + 5.0*s[2] + 2.0*s[3]);
    tmp = s[0] - 2.0*s[1] +     s[2]; S2 += 13*tmp*tmp;
    tmp = s[0] - 4.0*s[1] + 3.0*s[2]; S2 +=  3*tmp*tmp;
    double q23 = (2.0*s[0] - 7.0*s[1] + 11.0*s[2]);
    double a0 = 3.0*((12.0*ep + S1)*(12.0*ep + S1))*((12.0*ep + S2)*(12.0*ep + S2));
    double a1 = 6.0*((12.0*ep + S0)*(12.0*ep + S0))*((12.0*ep + S2)*(12.0*ep + S2));
    double a2 =     ((12.0*ep + S0)*(12.0*ep + S0))*((12.0*ep + S1)*(12.0*ep + S1));
    tmp = (a0*q03 + a1*q13 + a2*q23)/(6.0*(a0 + a1 + a2));
    return tmp;
}

/* OCFD_weno5_kernel_M, src/OCFD_Schemes.cu:1176-1208; s[0..4] = f(i-2..i+2), face i-1/2 */
double oro_weno5_m(const double *s) {
    double S0 = 0.0, S1 = 0.0, S2 = 0.0, tmp, ep = 1e-6;
    tmp =     s[2] - 2.0*s[1] + s[0]; S0 += 13*tmp*tmp;
    tmp = 3.0*s[2] - 4.0*s[1] + s[0]; S0 +=  3*tmp*tmp;
    double q03 = (2.0*s[2] + 5.0*s[1] - s[0]);
    tmp = s[3] - 2.0*s[2] + s[1]; S1 += 13*tmp*tmp;
    tmp =                  s[3] - s[1]; S1 +=  3*tmp*tmp;
    double q13 = (-s[3] + 5.0*s[2] + 2.0*s[1]);
    tmp = s[4] - 2.0*s[3] +     s[2]; S2 += 13*tmp*tmp;
    tmp = s[4] - 4.0*s[3] + 3.0*s[2]; S2 +=  3*tmp*tmp;
    double q23 = (2.0*s[4] - 7.0*s[3] + 11.0*s[2]);
    double a0 = 3.0*((12.0*ep + S1)*(12.0*ep + S1))*((12.0*ep + S2)*(12.0*ep + S2));
    double a1 = 6.0*((12.0*ep + S0)*(12.0*ep + S0))*((12.0*ep + S2)*(12.0*ep + S2));
    double a2 =     ((12.0*ep + S0)*(12.0*ep + S0))*((12.0*ep + S1)*(12.0*ep + S1));
    tmp = (a0*q03 + a1*q13 + a2*q23)/(6.0*(a0 + a1 + a2));
    return tmp;
}

/* OCFD_UP7_kernel_P, src/OCFD_Schemes.cu:865-873; s[0..6] = f(i-3..i+3) */
double oro_up7_p(const double *s) {
    return (-3.0*s[0] + 25.0*s[1] - 101.0*s[2] + 319.0*s[3] + 214.0*s[4]
            - 38.0*s[5] + 4.0*s[6])/420.0;
}
/* OCFD_UP7_kernel_M, src/OCFD_Schemes.cu:899-907; s[0..7] = f(i-4..i+3), face i-1/2 */
double oro_up7_m(const double *s) {
    return (-3.0*s[7] + 25.0*s[6] - 101.0*s[5] + 319.0*s[4] + 214.0*s[3]
            - 38.0*s[2] + 4.0*s[1])/420.0;
}

/* sign / minmod2 / minmod4, src/OCFD_Schemes.cu:766-797 (minmod4 keeps the
 * reference's fmin of signed arguments) */
static inline double sgn_(double x1, double x2) { return x2 >= 0 ? fabs(x1) : -fabs(x1); }
static inline double minmod2(double x1, double x2) {
    return 0.5*(sgn_(1.0, x1) + sgn_(1.0, x2))*fmin(fabs(x1), fabs(x2));
}
static inline double minmod4(double x1, double x2, double x3, double x4) {
    double m = 0.5*(sgn_(1.0, x1) + sgn_(1.0, x2));
    m = m*fabs(0.5*(sgn_(1.0, x1) + sgn_(1.0, x3)));
    m = m*fabs(0.5*(sgn_(1.0, x1) + sgn_(1.0, x4)));
    double tmp = fmin(x1, x2), tmp1 = fmin(x3, x4);
    tmp = fmin(tmp, tmp1);
    return m*tmp;
}

/* OCFD_NND2_kernel_P/M, src/OCFD_Schemes.cu:800-837; s[0..2] = f(i-1..i+1) */
double oro_nnd2_p(const double *s) { return s[1] + 0.5*minmod2(s[2] - s[1], s[1] - s[0]); }
double oro_nnd2_m(const double *s) { return s[1] + 0.5*minmod2(s[0] - s[1], s[1] - s[2]); }

/* OCFD_OMP6_kernel_P, src/OCFD_Schemes.cu:936-1008; s[0..7] = f(i-3..i+4) */
double oro_omp6_p(int flag, const double *s) {
    double m, n;
    if (flag == 1) { m = 0.001; n = 0.0; }
    else if (flag == 2) { m = 0.0; n = -1.0/140.0; }
    else { m = 0.015; n = 0.0; }
    double mid_nf = 0.5*(m + n); m = 0.5*(m - n);
    mid_nf =             ( 60.0*mid_nf  * s[7] +
      ( 1.0 -   60.0*m -  360.0*mid_nf) * s[6] +
      (-8.0 +  360.0*m +  900.0*mid_nf) * s[5] +
      (37.0 -  900.0*m - 1200.0*mid_nf) * s[4] +
      (37.0 + 1200.0*m +  900.0*mid_nf) * s[3] +
      (-8.0 -  900.0*m -  360.0*mid_nf) * s[2] +
      (1.0  +  360.0*m +   60.0*mid_nf) * s[1] -
                                 60.0*m * s[0])/60.0;
    m = s[3] + minmod2((s[4] - s[3]), (s[3] - s[2]));
    if ((mid_nf - s[3])*(mid_nf - m) >= 1.e-10) {
        double tmp, tmp1;
        m = s[2] + s[4] - 2.0*s[3];
        n = s[3] + s[5] - 2.0*s[4];
        tmp = 4.0*m - n;
        tmp1 = 4.0*n - m;
        tmp = 0.5*(s[3] + s[4]) - 0.5*minmod4(tmp, tmp1, n, m);
        n = s[1] + s[3] - 2.0*s[2];
        tmp1 = s[3] + 0.5*(s[3] - s[2]) + 4.0*minmod4(4*n - m, 4*m - n, m, n)/3.0;
        {
            m = fmin(s[3], s[4]);
            m = fmin(m, tmp);
            n = s[3] + 4.0*(s[3] - s[2]);
            n = fmin(s[3], n);
            n = fmin(n, tmp1);
            m = fmax(m, n);
        }
        {
            tmp = fmax(s[3], tmp);
            tmp = fmax(s[4], tmp);
            n = s[3] + 4.0*(s[3] - s[2]);
            n = fmax(s[3], n);
            n = fmax(n, tmp1);
            n = fmin(tmp, n);
        }
        mid_nf = mid_nf + minmod2(n - mid_nf, m - mid_nf);
    }
    return mid_nf;
}

/* OCFD_OMP6_kernel_M, src/OCFD_Schemes.cu:1037-1095; s[0..7] = f(i-4..i+3), face i-1/2 */
double oro_omp6_m(int flag, const double *s) {
    double m, n;
    if (flag == 1) { m = 0.001; n = 0.0; }
    else if (flag == 2) { m = 0.0; n = -1.0/140.0; }
    else { m = 0.015; n = 0.0; }
    double mid_nf = 0.5*(m + n); m = 0.5*(m - n);
    mid_nf =            (  60.0*mid_nf  * s[0] +
       (1.0 -   60.0*m -  360.0*mid_nf) * s[1] +
      (-8.0 +  360.0*m +  900.0*mid_nf) * s[2] +
      (37.0 -  900.0*m - 1200.0*mid_nf) * s[3] +
      (37.0 + 1200.0*m +  900.0*mid_nf) * s[4]  +
      (-8.0 -  900.0*m -  360.0*mid_nf) * s[5]  +
       (1.0 +  360.0*m +   60.0*mid_nf) * s[6]  -
                                 60.0*m * s[7])/60.0;
    m = s[4] + minmod2((s[3] - s[4]), (s[4] - s[5]));
    if ((mid_nf - s[4])*(mid_nf - m) >= 1.e-10) {
        double tmp, tmp1;
        m = s[5] + s[3] - 2.0*s[4];
        n = s[4] + s[2] - 2.0*s[3];
        tmp = 4.0*m - n;
        tmp1 = 4.0*n - m;
        tmp = 0.5*(s[4] + s[3]) - 0.5*minmod4(tmp, tmp1, n, m);
        n = s[6] + s[4] - 2.0*s[5];
        tmp1 = s[4] + 0.5*(s[4] - s[3]) + 4.0*minmod4(4*n - m, 4*m - n, m, n)/3.0;
        {
            m = fmin(s[5], s[3]);
            m = fmin(m, tmp);
            n = s[4] + 4.0*(s[4] - s[5]);
            n = fmin(s[4], n);
            n = fmin(n, tmp1);
            m = fmax(m, n);
        }
        {
            tmp = fmax(s[4], tmp);
            tmp = fmax(s[3], tmp);
            n = s[4] + 4.0*(s[4] - s[5]);
            n = fmax(s[4], n);
            n = fmax(n, tmp1);
            n = fmin(tmp, n);
        }
        mid_nf = mid_nf + minmod2(n - mid_nf, m - mid_nf);
    }
    return mid_nf;
}

/* OCFD_weno7_SYMBO_kernel_P, src/OCFD_Schemes.cu:391-478; s[0..7] = f(i-3..i+4) */
double oro_weno7_symbo_p(int lmt, double tv_lim, double tv_max, const double *s) {
    double S0, S1, S2, S3, S4, tmp, tmp1, TVmin = 0, TVmax = 1;
    if (lmt == 1) {
        S0 = fabs(s[1] - s[0]) + fabs(s[2] - s[1]) + fabs(s[3] - s[2]);
        S1 = fabs(s[2] - s[1]) + fabs(s[3] - s[2]) + fabs(s[4] - s[3]);
        S2 = fabs(s[3] - s[2]) + fabs(s[4] - s[3]) + fabs(s[5] - s[4]);
        S3 = fabs(s[4] - s[3]) + fabs(s[5] - s[4]) + fabs(s[6] - s[5]);
        S4 = fabs(s[5] - s[4]) + fabs(s[6] - s[5]) + fabs(s[7] - s[6]);
        tmp = fmin(S0, S1); tmp1 = fmin(S2, S3); tmp = fmin(tmp, tmp1); TVmin = fmin(tmp, S4);
        tmp = fmax(S0, S1); tmp1 = fmax(S2, S3); tmp = fmax(tmp, tmp1); TVmax = fmax(tmp, S4);
    }
    if (TVmax < tv_lim*TVmin && TVmax < tv_max) {
        S0 = 0.0401954833730; S1 = 0.2493800006710; S2 = 0.4802686256260;
        S3 = 0.2009775476730; S4 = 0.0291783426580;
    } else {
        S0 = 0.0; S1 = 0.0; S2 = 0.0; S3 = 0.0; S4 = 0.0;
        tmp =  -2.0*s[0] +  9.0*s[1] - 18.0*s[2] + 11.0*s[3]; S0 += 720.0*tmp*tmp;
        tmp =       s[1] -  6.0*s[2] +  3.0*s[3] +  2.0*s[4]; S1 += 720.0*tmp*tmp;
        tmp =  -2.0*s[2] -  3.0*s[3] +  6.0*s[4] -      s[5]; S2 += 720.0*tmp*tmp;
        tmp = -11.0*s[3] + 18.0*s[4] -  9.0*s[5] +  2.0*s[6]; S3 += 720.0*tmp*tmp;
        tmp = -26.0*s[4] + 57.0*s[5] - 42.0*s[6] + 11.0*s[7]; S4 += 720.0*tmp*tmp;

        tmp = -6.0*s[0] + 24.0*s[1] - 30.0*s[2] + 12.0*s[3]; S0 += 780.0*tmp*tmp;
        tmp =                    6.0*s[2] - 12.0*s[3] +  6.0*s[4]; S1 += 780.0*tmp*tmp;
        tmp =                    6.0*s[3] - 12.0*s[4] +  6.0*s[5]; S2 += 780.0*tmp*tmp;
        tmp = 12.0*s[3] - 30.0*s[4] + 24.0*s[5] -  6.0*s[6]; S3 += 780.0*tmp*tmp;
        tmp = 18.0*s[4] - 48.0*s[5] + 42.0*s[6] - 12.0*s[7]; S4 += 780.0*tmp*tmp;

        tmp = -6.0*s[0] + 18.0*( s[1] - s[2] ) + 6.0*s[3]; S0 += 781.0*tmp*tmp;
        tmp = -6.0*s[1] + 18.0*( s[2] - s[3] ) + 6.0*s[4]; S1 += 781.0*tmp*tmp;
        tmp = -6.0*s[2] + 18.0*( s[3] - s[4] ) + 6.0*s[5]; S2 += 781.0*tmp*tmp;
        tmp = -6.0*s[3] + 18.0*( s[4] - s[5] ) + 6.0*s[6]; S3 += 781.0*tmp*tmp;
        tmp = -6.0*s[4] + 18.0*( s[5] - s[6] ) + 6.0*s[7]; S4 += 781.0*tmp*tmp;
        {
            tmp = fmax(S0, S1); tmp1 = fmax(S2, S3); tmp = fmax(tmp, tmp1); S4 = fmax(tmp, S4);
        }
        {
            double tmp2, tmp3;
            tmp =  (0.0401954833730)*(2.592e-6+S1)*(2.592e-6+S2)*(2.592e-6+S3)*(2.592e-6+S4);
            tmp1 = (0.2493800006710)*(2.592e-6+S0)*(2.592e-6+S2)*(2.592e-6+S3)*(2.592e-6+S4);
            tmp2 = (0.4802686256260)*(2.592e-6+S0)*(2.592e-6+S1)*(2.592e-6+S3)*(2.592e-6+S4);
            tmp3 = (0.2009775476730)*(2.592e-6+S0)*(2.592e-6+S1)*(2.592e-6+S2)*(2.592e-6+S4);
            S4 =   (0.0291783426580)*(2.592e-6+S0)*(2.592e-6+S1)*(2.592e-6+S2)*(2.592e-6+S3);
            S3 = tmp3; S2 = tmp2; S1 = tmp1; S0 = tmp;
        }
    }
    double am = S0 + S1 + S2 + S3 + S4;
    tmp1 = 0.0;
    tmp = -3.0*s[0] + 13.0*s[1] - 23.0*s[2] + 25.0*s[3]; tmp1 += S0*tmp;
    tmp =      s[1] -  5.0*s[2] + 13.0*s[3] +  3.0*s[4]; tmp1 += S1*tmp;
    tmp =     -s[2] +  7.0*s[3] +  7.0*s[4] -      s[5]; tmp1 += S2*tmp;
    tmp =  3.0*s[3] + 13.0*s[4] -  5.0*s[5] +      s[6]; tmp1 += S3*tmp;
    tmp = 25.0*s[4] - 23.0*s[5] + 13.0*s[6] -  3.0*s[7]; tmp1 += S4*tmp;
    tmp1 /= (12.0*am);
    return tmp1;
}

/* OCFD_weno7_SYMBO_kernel_M, src/OCFD_Schemes.cu:506-590; s[0..7] = f(i-4..i+3).
 * The reference never computes TVmin on this side (quirk), so the linear
 * branch cannot fire; TVmax uses fmin for the first pairs as written. */
double oro_weno7_symbo_m(int lmt, double tv_lim, double tv_max, const double *s) {
    double S0, S1, S2, S3, S4, tmp, tmp1, TVmin = 0, TVmax = 1;
    if (lmt == 1) {
        S0 = fabs(s[7] - s[6]) + fabs(s[6] - s[5]) + fabs(s[5] - s[4]);
        S1 = fabs(s[6] - s[5]) + fabs(s[5] - s[4]) + fabs(s[4] - s[3]);
        S2 = fabs(s[5] - s[4]) + fabs(s[4] - s[3]) + fabs(s[3] - s[2]);
        S3 = fabs(s[4] - s[3]) + fabs(s[3] - s[2]) + fabs(s[2] - s[1]);
        S4 = fabs(s[3] - s[2]) + fabs(s[2] - s[1]) + fabs(s[1] - s[0]);
        tmp = fmin(S0, S1); tmp1 = fmin(S2, S3); tmp = fmax(tmp, tmp1); TVmax = fmax(tmp, S4);
    }
    if (TVmax < tv_lim*TVmin && TVmax < tv_max) {
        S0 = 0.0401954833730; S1 = 0.2493800006710; S2 = 0.4802686256260;
        S3 = 0.2009775476730; S4 = 0.0291783426580;
    } else {
        S0 = 0.0; S1 = 0.0; S2 = 0.0; S3 = 0.0; S4 = 0.0;
        tmp =  -2.0*s[7] +  9.0*s[6] - 18.0*s[5] + 11.0*s[4]; S0 += 720.0*tmp*tmp;
        tmp =       s[6] -  6.0*s[5] +  3.0*s[4] +  2.0*s[3]; S1 += 720.0*tmp*tmp;
        tmp =  -2.0*s[5] -  3.0*s[4] +  6.0*s[3] -      s[2]; S2 += 720.0*tmp*tmp;
        tmp = -11.0*s[4] + 18.0*s[3] -  9.0*s[2] +  2.0*s[1]; S3 += 720.0*tmp*tmp;
        tmp = -26.0*s[3] + 57.0*s[2] - 42.0*s[1] + 11.0*s[0]; S4 += 720.0*tmp*tmp;

        tmp = -6.0*s[7] + 24.0*s[6] - 30.0*s[5] + 12.0*s[4]; S0 += 780.0*tmp*tmp;
        tmp =                    6.0*s[5] - 12.0*s[4] +  6.0*s[3]; S1 += 780.0*tmp*tmp;
        tmp =                    6.0*s[4] - 12.0*s[3] +  6.0*s[2]; S2 += 780.0*tmp*tmp;
        tmp = 12.0*s[4] - 30.0*s[3] + 24.0*s[2] -  6.0*s[1]; S3 += 780.0*tmp*tmp;
        tmp = 18.0*s[3] - 48.0*s[2] + 42.0*s[1] - 12.0*s[0]; S4 += 780.0*tmp*tmp;

        tmp = -6.0*s[7] + 18.0*( s[6] - s[5] ) + 6.0*s[4]; S0 += 781.0*tmp*tmp;
        tmp = -6.0*s[6] + 18.0*( s[5] - s[4] ) + 6.0*s[3]; S1 += 781.0*tmp*tmp;
        tmp = -6.0*s[5] + 18.0*( s[4] - s[3] ) + 6.0*s[2]; S2 += 781.0*tmp*tmp;
        tmp = -6.0*s[4] + 18.0*( s[3] - s[2] ) + 6.0*s[1]; S3 += 781.0*tmp*tmp;
        tmp = -6.0*s[3] + 18.0*( s[2] - s[1] ) + 6.0*s[0]; S4 += 781.0*tmp*tmp;
        {
            tmp = fmax(S0, S1); tmp1 = fmax(S2, S3); tmp = fmax(tmp, tmp1); S4 = fmax(tmp, S4);
        }
        {
            double tmp2, tmp3;
            tmp =  (0.0401954833730)*(2.592e-6+S1)*(2.592e-6+S2)*(2.592e-6+S3)*(2.592e-6+S4);
            tmp1 = (0.2493800006710)*(2.592e-6+S0)*(2.592e-6+S2)*(2.592e-6+S3)*(2.592e-6+S4);
            tmp2 = (0.4802686256260)*(2.592e-6+S0)*(2.592e-6+S1)*(2.592e-6+S3)*(2.592e-6+S4);
            tmp3 = (0.2009775476730)*(2.592e-6+S0)*(2.592e-6+S1)*(2.592e-6+S2)*(2.592e-6+S4);
            S4 =   (0.0291783426580)*(2.592e-6+S0)*(2.592e-6+S1)*(2.592e-6+S2)*(2.592e-6+S3);
            S3 = tmp3; S2 = tmp2; S1 = tmp1; S0 = tmp;
        }
    }
    double am = S0 + S1 + S2 + S3 + S4;
    tmp1 = 0.0;
    tmp = -3.0*s[7] + 13.0*s[6] - 23.0*s[5] + 25.0*s[4]; tmp1 += S0*tmp;
    tmp =      s[6] -  5.0*s[5] + 13.0*s[4] +  3.0*s[3]; tmp1 += S1*tmp;
    tmp =    - s[5] +  7.0*s[4] +  7.0*s[3] -      s[2]; tmp1 += S2*tmp;
    tmp =  3.0*s[4] + 13.0*s[3] -  5.0*s[2] +      s[1]; tmp1 += S3*tmp;
    tmp = 25.0*s[3] - 23.0*s[2] + 13.0*s[1] -  3.0*s[0]; tmp1 += S4*tmp;
    tmp1 /= (12.0*am);
    return tmp1;
}

/* OCFD_kernel_CD6 / CD8, src/OCFD_Schemes.cu:96-126 */
double oro_cd6(const double *s) {
    return (45.0*(s[4] - s[2]) - 9.0*(s[5] - s[1]) + (s[6] - s[0]))/60.0;
}
double oro_cd8(const double *s) {
    return (672.0*(s[5] - s[3]) - 168.0*(s[6] - s[2]) + 32.0*(s[7] - s[1]) - 3.0*(s[8] - s[0]))/840.0;
}

/* ------------------------------------------------------------------------ */
/* characteristic projection, src/OCFD_flux_charteric.cu:321-752             */
/* ------------------------------------------------------------------------ */

typedef struct { double u1, v1, w1, c1, n1, n2, n3, l1, l2, l3, m1, m2, m3, KK; } char_para;

/* get_para_charteric_{p,m}_kernel body, :330-418 (face averages given). */
static inline void char_para_make(double u1, double v1, double w1, double c1,
                                  double a1, double a2, double a3, double G, char_para *p) {
    double ss, n1, n2, n3, l1, l2, l3;
    ss = sqrt(a1*a1 + a2*a2 + a3*a3);
    n1 = a1/ss; n2 = a2/ss; n3 = a3/ss;
    if (fabs(n3) <= fabs(n2)) {
        ss = sqrt(n1*n1 + n2*n2);
        l1 = -n2/ss; l2 = n1/ss; l3 = 0.0;
    } else {
        ss = sqrt(n1*n1 + n3*n3);
        l1 = -n3/ss; l2 = 0.0; l3 = n1/ss;
    }
    p->u1 = u1; p->v1 = v1; p->w1 = w1; p->c1 = c1;
    p->n1 = n1; p->n2 = n2; p->n3 = n3; p->l1 = l1; p->l2 = l2; p->l3 = l3;
    p->m1 = n2*l3 - n3*l2; p->m2 = n3*l1 - n1*l3; p->m3 = n1*l2 - n2*l1;
    p->KK = (G - 1.0)/(c1*c1);
}

/* flux_charteric_ptoc_kernel, :617-676 -- left matrix rows */
static inline void char_L(const char_para *p, double S[25]) {
    double u1 = p->u1, v1 = p->v1, w1 = p->w1, c1 = p->c1, n1 = p->n1, n2 = p->n2, n3 = p->n3;
    double l1 = p->l1, l2 = p->l2, l3 = p->l3, m1 = p->m1, m2 = p->m2, m3 = p->m3, KK = p->KK;
    double X1 = 1.0/(2.0*c1);
    double un = u1*n1 + v1*n2 + w1*n3;
    double v2 = (u1*u1 + v1*v1 + w1*w1)*0.5;
    S[0] = 1.0 - KK*v2; S[1] = KK*u1; S[2] = KK*v1; S[3] = KK*w1; S[4] = -KK;
    S[5] = -(u1*l1 + v1*l2 + w1*l3); S[6] = l1; S[7] = l2; S[8] = l3; S[9] = 0.0;
    S[10] = -(u1*m1 + v1*m2 + w1*m3); S[11] = n2*l3 - n3*l2; S[12] = n3*l1 - n1*l3; S[13] = n1*l2 - n2*l1; S[14] = 0.0;
    S[15] = KK*v2*0.5 + X1*un; S[16] = -X1*n1 - KK*u1*0.5; S[17] = -X1*n2 - KK*v1*0.5; S[18] = -X1*n3 - KK*w1*0.5; S[19] = KK*0.5;
    S[20] = S[15] - 2*X1*un; S[21] = 2*X1*n1 + S[16]; S[22] = 2*X1*n2 + S[17]; S[23] = 2*X1*n3 + S[18]; S[24] = S[19];
}

/* flux_charteric_ctop_kernel, :678-752 -- right matrix rows */
static inline void char_R(const char_para *p, double S[25]) {
    double u1 = p->u1, v1 = p->v1, w1 = p->w1, c1 = p->c1, n1 = p->n1, n2 = p->n2, n3 = p->n3;
    double l1 = p->l1, l2 = p->l2, l3 = p->l3, m1 = p->m1, m2 = p->m2, m3 = p->m3, KK = p->KK;
    S[0] = 1.0; S[1] = 0.0; S[2] = 0.0; S[3] = 1.0; S[4] = 1.0;
    S[5] = u1; S[6] = l1; S[7] = n2*l3 - n3*l2; S[8] = u1 - c1*n1; S[9] = 2*u1 - S[8];
    S[10] = v1; S[11] = l2; S[12] = n3*l1 - n1*l3; S[13] = v1 - c1*n2; S[14] = 2*v1 - S[13];
    S[15] = w1; S[16] = l3; S[17] = n1*l2 - n2*l1; S[18] = w1 - c1*n3; S[19] = 2*w1 - S[18];
    S[20] = (u1*u1 + v1*v1 + w1*w1)*0.5;
    double H = S[20] + 1.0/KK;
    S[21] = u1*l1 + v1*l2 + w1*l3; S[22] = u1*m1 + v1*m2 + w1*m3;
    S[23] = H - c1*(u1*n1 + v1*n2 + w1*n3); S[24] = 2*H - S[23];
}

static inline void mat5_apply(const double S[25], double x[5]) {
    double y[5];
    for (int r = 0; r < 5; r++)
        y[r] = S[5*r]*x[0] + S[5*r+1]*x[1] + S[5*r+2]*x[2] + S[5*r+3]*x[3] + S[5*r+4]*x[4];
    for (int r = 0; r < 5; r++) x[r] = y[r];
}

void oro_char_matrices(double u1, double v1, double w1, double c1,
                       double a1, double a2, double a3, double gamma,
                       double *L25, double *R25) {
    char_para p;
    char_para_make(u1, v1, w1, c1, a1, a2, a3, gamma, &p);
    char_L(&p, L25);
    char_R(&p, R25);
}

/* ------------------------------------------------------------------------ */
/* hybrid sensor, style 2 (Jameson), src/OCFD_Schemes_hybrid_auto.cu         */
/* ------------------------------------------------------------------------ */

/* Comput_P (:48-68) over the LAP box, then Comput_Scheme_point_Jameson (:680-703). */
static void set_scheme_hybrid(oro_state *s) {
    double p00 = 1.0/(s->c.gamma*s->c.ama*s->c.ama);
#pragma omp parallel for
    for (long q = 0; q < (long)s->nlap; q++) s->psens[q] = p00 * s->d[q] * s->T[q];
    const double *P = s->psens;
    double t1 = s->c.hy_dp_intv[0], t2 = s->c.hy_dp_intv[1];
    size_t sx = s->nx2, sy = (size_t)s->nx2 * s->ny2;
    int nx = s->nx, ny = s->ny, nz = s->nz;
    for (int dir = 0; dir < 3; dir++) {
        int ex = nx + (dir == 0), ey = ny + (dir == 1), ez = nz + (dir == 2);
        int *out = s->sch[dir];
#pragma omp parallel for
        for (int k = 0; k < ez; k++)
            for (int j = 0; j < ey; j++)
                for (int i = 0; i < ex; i++) {
                    /* flag index q corresponds to cell q-1 along dir */
                    int ci = i + LAP - (dir == 0), cj = j + LAP - (dir == 1), ck = k + LAP - (dir == 2);
                    size_t q = L(s, ci, cj, ck);
                    double dp0 = fabs(-P[q - 1] + 2*P[q] - P[q + 1])/(P[q - 1] + 2*P[q] + P[q + 1]);
                    dp0 += fabs(-P[q - sx] + 2*P[q] - P[q + sx])/(P[q - sx] + 2*P[q] + P[q + sx]);
                    dp0 += fabs(-P[q - sy] + 2*P[q] - P[q + sy])/(P[q - sy] + 2*P[q] + P[q + sy]);
                    int kp = 1;
                    if (dp0 > t1) kp += 1;
                    if (dp0 > t2) kp += 1;
                    out[(size_t)i + (size_t)ex * ((size_t)j + (size_t)ey * k)] = kp;
                }
    }
}

/* flag of the face F+1/2 (left cell F), both sides:
 * get_Hyscheme_flag_p_kernel (:832-859) / get_Hyscheme_flag_m_kernel (:928-955) */
static inline int face_flag(const oro_state *s, int dir, int i, int j, int k) {
    int ex = s->nx + (dir == 0), ey = s->ny + (dir == 1);
    int fi = i + (dir == 0), fj = j + (dir == 1), fk = k + (dir == 2);
    return s->sch[dir][(size_t)fi + (size_t)ex * ((size_t)fj + (size_t)ey * fk)];
}

/* ------------------------------------------------------------------------ */
/* inviscid sweeps                                                           */
/* ------------------------------------------------------------------------ */

/* ------------------------------------------------------------------------ */
/* boundary closures on non-periodic directions, src/OCFD_bound_Scheme.cu    */
/* ------------------------------------------------------------------------ */

/* one-sided WENO5 candidates, :554-745; s[0..4] = f(i-2..i+2) (P) */
static double w5_p_left(const double *s) {
    double S0 = 0.0, tmp, ep = 1e-6;
    tmp =     s[2] - 2.0*s[3] + s[4]; S0 += 13*tmp*tmp;
    tmp = 3.0*s[2] - 4.0*s[3] + s[4]; S0 +=  3*tmp*tmp;
    double a0 = 1.0/((12.0*ep + S0)*(12.0*ep + S0));
    double q03 = (2.0*s[2] + 5.0*s[3] - s[4]);
    return a0*q03/(6.0*a0);
}
static double w5_m_left(const double *s) {
    double S2 = 0.0, tmp, ep = 1e-6;
    tmp = s[4] - 2.0*s[3] +     s[2]; S2 += 13*tmp*tmp;
    tmp = s[4] - 4.0*s[3] + 3.0*s[2]; S2 +=  3*tmp*tmp;
    double a2 = 1.0/((12.0*ep + S2)*(12.0*ep + S2));
    double q23 = (2.0*s[4] - 7.0*s[3] + 11.0*s[2]);
    return a2*q23/(6.0*a2);
}
static double w5_p_right_plus(const double *s) {
    double S1 = 0.0, S2 = 0.0, tmp, ep = 1e-6;
    tmp = s[1] - 2.0*s[2] + s[3]; S1 += 13*tmp*tmp;
    tmp =             s[1] - s[3]; S1 +=  3*tmp*tmp;
    double a1 = 6.0/((12.0*ep + S1)*(12.0*ep + S1));
    double q13 = (-s[1] + 5.0*s[2] + 2.0*s[3]);
    tmp = s[0] - 2.0*s[1] +     s[2]; S2 += 13*tmp*tmp;
    tmp = s[0] - 4.0*s[1] + 3.0*s[2]; S2 +=  3*tmp*tmp;
    double a2 = 1.0/((12.0*ep + S2)*(12.0*ep + S2));
    double q23 = (2.0*s[0] - 7.0*s[1] + 11.0*s[2]);
    return (a1*q13 + a2*q23)/(6.0*(a1 + a2));
}
static double w5_p_left_plus(const double *s) {
    double S0 = 0.0, S1 = 0.0, tmp, ep = 1e-6;
    tmp =     s[2] - 2.0*s[3] + s[4]; S0 += 13*tmp*tmp;
    tmp = 3.0*s[2] - 4.0*s[3] + s[4]; S0 +=  3*tmp*tmp;
    double a0 = 3.0/((12.0*ep + S0)*(12.0*ep + S0));
    double q03 = (2.0*s[2] + 5.0*s[3] - s[4]);
    tmp = s[1] - 2.0*s[2] + s[3]; S1 += 13*tmp*tmp;
    tmp =             s[1] - s[3]; S1 +=  3*tmp*tmp;
    double a1 = 6.0/((12.0*ep + S1)*(12.0*ep + S1));
    double q13 = (-s[1] + 5.0*s[2] + 2.0*s[3]);
    return (a0*q03 + a1*q13)/(6.0*(a0 + a1));
}
static double w5_m_right_plus(const double *s) {
    double S0 = 0.0, S1 = 0.0, tmp, ep = 1e-6;
    tmp =     s[2] - 2.0*s[1] + s[0]; S0 += 13*tmp*tmp;
    tmp = 3.0*s[2] - 4.0*s[1] + s[0]; S0 +=  3*tmp*tmp;
    double a0 = 3.0/((12.0*ep + S0)*(12.0*ep + S0));
    double q03 = (2.0*s[2] + 5.0*s[1] - s[0]);
    tmp = s[3] - 2.0*s[2] + s[1]; S1 += 13*tmp*tmp;
    tmp =             s[3] - s[1]; S1 +=  3*tmp*tmp;
    double a1 = 6.0/((12.0*ep + S1)*(12.0*ep + S1));
    double q13 = (-s[3] + 5.0*s[2] + 2.0*s[1]);
    return (a0*q03 + a1*q13)/(6.0*(a0 + a1));
}
static double w5_m_left_plus(const double *s) {
    double S1 = 0.0, S2 = 0.0, tmp, ep = 1e-6;
    tmp = s[3] - 2.0*s[2] + s[1]; S1 += 13*tmp*tmp;
    tmp =             s[3] - s[1]; S1 +=  3*tmp*tmp;
    double a1 = 6.0/((12.0*ep + S1)*(12.0*ep + S1));
    double q13 = (-s[3] + 5.0*s[2] + 2.0*s[1]);
    tmp = s[4] - 2.0*s[3] +     s[2]; S2 += 13*tmp*tmp;
    tmp = s[4] - 4.0*s[3] + 3.0*s[2]; S2 +=  3*tmp*tmp;
    double a2 = 1.0/((12.0*ep + S2)*(12.0*ep + S2));
    double q23 = (2.0*s[4] - 7.0*s[3] + 11.0*s[2]);
    return (a1*q13 + a2*q23)/(6.0*(a1 + a2));
}

/* Stencil extents (-ia1, ib1) of the reference kernels, which decide how far
 * the closures reach: P kernels and M kernels of each scheme. */
static void closure_extent(int scheme, int chart, int *kap, int *kbp, int *kam, int *kbm) {
    if (chart) { *kap = 3; *kbp = 4; *kam = 4; *kbm = 3; return; }
    switch (scheme) {
    case 302: case 306: *kap = 2; *kbp = 2; *kam = 2; *kbm = 2; break;   /* WENO5, NND2 */
    case 303: *kap = 3; *kbp = 3; *kam = 3; *kbm = 3; break;             /* WENO7 */
    default:  *kap = 3; *kbp = 4; *kam = 4; *kbm = 3; break;             /* UP7, SYMBO, OMP6, hybrid */
    }
}

/* P-side closure of face F+1/2 on a line of n cells, s8[t] = f(F-3+t):
 * OCFD_bound_scheme_kernel_p with boundp1 / boundp2 (:748-848).
 * Returns 1 when the closure replaces the interior scheme. */
static int closure_p(int lo, int hi, int KA, int KB, int F, int n, const double *s8, double *out) {
    int c = F + 1;
    if (lo && c <= KA) {
        if (c == 0) *out = s8[4];
        if (c == 1) *out = w5_p_left(s8 + 1);
        if (c == 2) *out = w5_p_left_plus(s8 + 1);
        if (c == 3) *out = oro_weno5_p(s8 + 1);
        return 1;
    }
    if (hi) {
        int t = c - (n + 1);
        if (t >= -KB) {
            if (t == -1) *out = s8[3] + 0.5*minmod2(s8[3] - s8[2], s8[3] - s8[2]);
            if (t == -2) *out = w5_p_right_plus(s8 + 1);
            if (t <= -3) *out = oro_weno5_p(s8 + 1);
            return 1;
        }
    }
    return 0;
}

/* M-side closure, OCFD_bound_scheme_kernel_m with boundm1 / boundm2 (:850-944) */
static int closure_m(int lo, int hi, int KA, int KB, int F, int n, const double *s8, double *out) {
    int c = F + 1;
    if (lo && c < KA) {
        if (c == 0) *out = w5_m_left(s8 + 2);
        if (c == 1) *out = w5_m_left_plus(s8 + 2);
        if (c >= 2) *out = oro_weno5_m(s8 + 2);
        return 1;
    }
    if (hi) {
        int t = c - (n + 1);
        if (t >= -KB - 1) {
            if (t == -1) *out = s8[3];
            if (t == -2) *out = s8[4] - 0.5*minmod2(s8[4] - s8[3], s8[4] - s8[3]);
            if (t == -3) *out = w5_m_right_plus(s8 + 2);
            if (t == -4) *out = oro_weno5_m(s8 + 2);
            return 1;
        }
    }
    return 0;
}

/* face flux of one component from the 8-point stencil s8[k] = f(F-3+k) */
static double face_p(const oro_state *s, int scheme, int hflag, const double *s8) {
    switch (scheme) {
    case 301: return oro_up7_p(s8);
    case 302: return oro_weno5_p(s8 + 1);
    case 303: return oro_weno7_p(s8);
    case 304: return oro_weno7_symbo_p(0, s->c.weno_tv_limiter, s->c.weno_tv_max, s8);
    case 305: return oro_weno7_symbo_p(1, s->c.weno_tv_limiter, s->c.weno_tv_max, s8);
    case 306: return oro_nnd2_p(s8 + 2);
    case 307: return oro_omp6_p(0, s8);
    case 308: return oro_omp6_p(1, s8);
    case 309: return oro_omp6_p(2, s8);
    case 310: /* style 2: OCFD_HybridAuto_P_Jameson_kernel :895-925 */
        if (hflag == 1) return oro_up7_p(s8);
        if (hflag == 2) return oro_weno7_p(s8);
        return oro_weno5_p(s8 + 1);
    }
    return 0.0;
}
static double face_m(const oro_state *s, int scheme, int hflag, const double *s8) {
    switch (scheme) {
    case 301: return oro_up7_m(s8);
    case 302: return oro_weno5_m(s8 + 2);
    case 303: return oro_weno7_m(s8 + 1);
    case 304: return oro_weno7_symbo_m(0, s->c.weno_tv_limiter, s->c.weno_tv_max, s8);
    case 305: return oro_weno7_symbo_m(1, s->c.weno_tv_limiter, s->c.weno_tv_max, s8);
    case 306: return oro_nnd2_m(s8 + 3);
    case 307: return oro_omp6_m(0, s8);
    case 308: return oro_omp6_m(1, s8);
    case 309: return oro_omp6_m(2, s8);
    case 310: /* OCFD_HybridAuto_M_Jameson_kernel :992-1023 */
        if (hflag == 1) return oro_up7_m(s8);
        if (hflag == 2) return oro_weno7_m(s8 + 1);
        return oro_weno5_m(s8 + 2);
    }
    return 0.0;
}

/* One direction, both signs: OCFD_d{x,y,z}1 and OCFD_d{x,y,z}2
 * (src/OCFD_Schemes_Choose.cu:88-764) on a single-rank domain, with the
 * boundary closures of faces whose DIF_BOUND is 1.
 * du(X) += -Ajac(X)*(F+(X+1/2) - F+(X-1/2))/h, then the same for F-. */
static void invis_sweep(oro_state *s, int dir) {
    int n[3] = { s->nx, s->ny, s->nz };
    size_t st[3] = { 1, (size_t)s->nx2, (size_t)s->nx2 * s->ny2 };
    size_t sdir = st[dir];
    int len = n[dir];
    int o1 = (dir == 0) ? 1 : 0, o2 = (dir == 2) ? 1 : 2;   /* the two other directions */
    double h = dir == 0 ? s->hx : (dir == 1 ? s->hy : s->hz);
    size_t nl = s->nlap, nin = s->nin;
    int scheme = s->c.scheme_invis, chart = s->c.charteric;
    double G = s->c.gamma;
    const double *Aj = s->A[AJAC];
    const double *Ax = s->A[AKX + 3 * dir], *Ay = s->A[AKX + 3 * dir + 1], *Az = s->A[AKX + 3 * dir + 2];
    /* boundary handling of this direction (OCFD_bound / OCFD_bound_non_ref,
     * src/OCFD_bound_Scheme.cu:352-469): flagxyzb.y is LOWER, UPPER or both
     * (7/8/9) when DIF_BOUND of the face is 1; flagxyzb.z is NON_REFLETION */
    const int lo = s->c.d0_bound[2 * dir] == 1, hi = s->c.d0_bound[2 * dir + 1] == 1;
    const int LOWER = 1 + dir, UPPER = 4 + dir;
    const int flagy = lo ? (hi ? 7 + dir : LOWER) : (hi ? UPPER : 0);
    const int nr_lo = s->c.non_ref[2 * dir], nr_hi = s->c.non_ref[2 * dir + 1];
    /* the characteristic kernels (304, 305, 310 with CHARTERIC=1) */
    const int char_kernel = chart && (scheme == 304 || scheme == 305 || scheme == 310);
    int kap, kbp, kam, kbm;
    closure_extent(scheme, char_kernel, &kap, &kbp, &kam, &kbm);

#pragma omp parallel
    {
        double *fpp = (double *)malloc(sizeof(double) * 5 * (len + 1));
        double *fmm = (double *)malloc(sizeof(double) * 5 * (len + 1));
#pragma omp for collapse(2)
        for (int b = 0; b < n[o2]; b++)
            for (int a = 0; a < n[o1]; a++) {
                int idx[3];
                idx[o1] = a + LAP; idx[o2] = b + LAP;
                /* faces F+1/2, F = -1 .. len-1 (interior-relative) */
                for (int F = -1; F < len; F++) {
                    idx[dir] = F + LAP;
                    size_t q = L(s, idx[0], idx[1], idx[2]);
                    double s8p[5][8], s8m[5][8];
                    for (int m = 0; m < 5; m++)
                        for (int t = 0; t < 8; t++) {
                            size_t qq = q + (size_t)((long)(t - 3) * (long)sdir);
                            s8p[m][t] = s->fp[dir][(size_t)m * nl + qq];
                            s8m[m][t] = s->fm[dir][(size_t)m * nl + qq];
                        }
                    int hflag = 0;
                    if (scheme == 310) {
                        int fi[3] = { idx[0] - LAP, idx[1] - LAP, idx[2] - LAP };
                        hflag = face_flag(s, dir, fi[0], fi[1], fi[2]);
                    }
                    double outp[5], outm[5];
                    int use_char = chart && (scheme == 304 || scheme == 305 || (scheme == 310 && hflag != 1));
                    if (chart && scheme != 304 && scheme != 305 && scheme != 310) {
                        /* the reference prints "does not support" and adds nothing */
                        for (int m = 0; m < 5; m++) { outp[m] = 0.0; outm[m] = 0.0; }
                    } else if (use_char) {
                        /* characteristic kernels, src/OCFD_flux_charteric.cu:754-906, :1000-1268 */
                        size_t q1 = q + sdir;
                        double u1 = (s->u[q] + s->u[q1])*0.5, v1 = (s->v[q] + s->v[q1])*0.5;
                        double w1 = (s->w[q] + s->w[q1])*0.5, c1 = (s->cc[q] + s->cc[q1])*0.5;
                        double a1 = (Ax[q] + Ax[q1])*0.5, a2 = (Ay[q] + Ay[q1])*0.5, a3 = (Az[q] + Az[q1])*0.5;
                        char_para p; double Lm[25], Rm[25];
                        char_para_make(u1, v1, w1, c1, a1, a2, a3, G, &p);
                        char_L(&p, Lm); char_R(&p, Rm);
                        for (int t = 0; t < 8; t++) {
                            double xp[5], xm[5];
                            for (int m = 0; m < 5; m++) { xp[m] = s8p[m][t]; xm[m] = s8m[m][t]; }
                            mat5_apply(Lm, xp); mat5_apply(Lm, xm);
                            for (int m = 0; m < 5; m++) { s8p[m][t] = xp[m]; s8m[m][t] = xm[m]; }
                        }
                        /* closures act on the characteristic stencils (the
                         * kernels call OCFD_bound_scheme_kernel_{p,m} after ptoc) */
                        for (int m = 0; m < 5; m++) {
                            if (!closure_p(lo, hi, kap, kbp, F, len, s8p[m], &outp[m])) {
                                if (scheme == 310) outp[m] = face_p(s, 310, hflag, s8p[m]);
                                else outp[m] = oro_weno7_symbo_p(scheme == 305, s->c.weno_tv_limiter, s->c.weno_tv_max, s8p[m]);
                            }
                            if (!closure_m(lo, hi, kam, kbm, F, len, s8m[m], &outm[m])) {
                                if (scheme == 310) outm[m] = face_m(s, 310, hflag, s8m[m]);
                                else outm[m] = oro_weno7_symbo_m(scheme == 305, s->c.weno_tv_limiter, s->c.weno_tv_max, s8m[m]);
                            }
                        }
                        mat5_apply(Rm, outp); mat5_apply(Rm, outm);
                    } else {
                        for (int m = 0; m < 5; m++) {
                            int hf = hflag;
                            if (scheme == 310 && !chart && m > 0 && s->c.hy_nochar_fixed) hf = s->c.hy_nochar_fixed;
                            if (!closure_p(lo, hi, kap, kbp, F, len, s8p[m], &outp[m]))
                                outp[m] = face_p(s, scheme, hf, s8p[m]);
                            if (!closure_m(lo, hi, kam, kbm, F, len, s8m[m], &outm[m]))
                                outm[m] = face_m(s, scheme, hf, s8m[m]);
                        }
                    }
                    for (int m = 0; m < 5; m++) {
                        fpp[(size_t)m * (len + 1) + (F + 1)] = outp[m];
                        fmm[(size_t)m * (len + 1) + (F + 1)] = outm[m];
                    }
                }
                for (int X = 0; X < len; X++) {
                    idx[dir] = X + LAP;
                    size_t q = L(s, idx[0], idx[1], idx[2]);
                    int ci[3] = { idx[0] - LAP, idx[1] - LAP, idx[2] - LAP };
                    size_t c = I(s, ci[0], ci[1], ci[2]);
                    double aj = Aj[q];
                    /* put_du_p_kernel (src/OCFD_Schemes.cu:293-338) and
                     * put_du_character_p_kernel (src/OCFD_flux_charteric.cu:16-64) */
                    for (int m = 0; m < 5; m++) {
                        double r = fpp[(size_t)m * (len + 1) + X + 1], l = fpp[(size_t)m * (len + 1) + X];
                        double *du = &s->du[(size_t)m * nin + c];
                        if (!char_kernel) {
                            if (X == 0 && nr_lo == 1) *du += 0.0;
                            else *du += -aj*(r - l)/h;
                        } else if (flagy == LOWER && nr_lo == 1 && X == 0) {
                            *du += 0.0;
                        } else if ((flagy == LOWER && X == 0) || (flagy == UPPER && X == len - 1)) {
                            /* OCFD_bound_character_kernel_p (:121-210) on the split fluxes */
                            const double *fl = s->fp[dir] + (size_t)m * nl;
                            size_t q0 = q;
                            double tmp;
                            if (X == 0) {
                                tmp = (fl[q0 + sdir] - fl[q0]);
                            } else {
                                double f0 = fl[q0], f1 = fl[q0 - sdir], f2 = fl[q0 - 2 * sdir];
                                double tr = f0 + 0.5*minmod2(f0 - f1, f0 - f1);
                                double tl = f1 + 0.5*minmod2(f0 - f1, f1 - f2);
                                tmp = tr - tl;
                            }
                            *du += -aj*tmp/h;
                        } else {
                            *du += -aj*(r - l)/h;
                        }
                    }
                    /* put_du_m_kernel (:340-381) and put_du_character_m_kernel
                     * (:67-118; its y case tests flag 3, so the lower special
                     * never applies on y) */
                    const int mlower = dir == 1 ? 3 : LOWER;
                    for (int m = 0; m < 5; m++) {
                        double r = fmm[(size_t)m * (len + 1) + X + 1], l = fmm[(size_t)m * (len + 1) + X];
                        double *du = &s->du[(size_t)m * nin + c];
                        if (!char_kernel) {
                            if (X == len - 1 && nr_hi == 1) *du += 0.0;
                            else *du += -aj*(r - l)/h;
                        } else if (flagy == UPPER && nr_hi == 1 && X == len - 1) {
                            *du += 0.0;
                        } else if ((flagy == mlower && X == 0) || (flagy == UPPER && X == len - 1)) {
                            /* OCFD_bound_character_kernel_m (:214-319) */
                            const double *fl = s->fm[dir] + (size_t)m * nl;
                            double tmp;
                            if (X == 0) {
                                double f0 = fl[q], f1 = fl[q + sdir], f2 = fl[q + 2 * sdir];
                                double tr = f1 - 0.5*minmod2(f2 - f1, f1 - f0);
                                double tl = f0 - 0.5*minmod2(f1 - f0, f1 - f0);
                                tmp = tr - tl;
                            } else {
                                tmp = (fl[q] - fl[q - sdir]);
                            }
                            *du += -aj*tmp/h;
                        } else {
                            *du += -aj*(r - l)/h;
                        }
                    }
                }
            }
        free(fpp); free(fmm);
    }
}

/* The per-cell order of the reference is x+ (all comps), x-, y+, y-, ...; the
 * sweep above adds x+ then x- per component, which for one address is the
 * same sequence of additions. */

/* ------------------------------------------------------------------------ */
/* viscous terms, src/OCFD_NS_Jacobian3d.cu:58-440                            */
/* ------------------------------------------------------------------------ */

/* Derivative closures of OCFD_D0bound_scheme_kernel (src/OCFD_bound_Scheme.cu:79-186)
 * for point i of a line of n cells, c[k] = f(i+k).  lo / hi: DIF_BOUND of the
 * lower / upper face is 1 (OCFD_bound, :436-469).  The lower closure is tried
 * first, as in the reference's case 7/8/9.  Returns 1 when a closure applies. */
static int d0_closure(int lo, int hi, int i, int n, const double *c, double *out) {
    if (lo) {
        if (i == 0) { *out = (c[1] - c[0]); return 1; }
        if (i == 1) { *out = (c[1] - c[-1])*0.5; return 1; }
        if (i == 2) { *out = (c[-2] - 8.0*c[-1] + 8.0*c[1] - c[2])/12.0; return 1; }
        if (i == 3) { *out = (c[3] - c[-3] - 9.0*(c[2] - c[-2]) + 45.0*(c[1] - c[-1]))/60.0; return 1; }
    }
    if (hi) {
        int t = i - n;
        if (t == -1) { *out = (c[0] - c[-1]); return 1; }
        if (t == -2) { *out = (c[1] - c[-1])*0.5; return 1; }
        if (t == -3) { *out = (c[-2] - 8.0*c[-1] + 8.0*c[1] - c[2])/12.0; return 1; }
        if (t == -4) { *out = (c[3] - c[-3] - 9.0*(c[2] - c[-2]) + 45.0*(c[1] - c[-1]))/60.0; return 1; }
    }
    return 0;
}

/* OCFD_d{x,y,z}0 (src/OCFD_Schemes_Choose.cu:19-84) with CD6/CD8 over the
 * interior of a LAP field, closures on faces whose DIF_BOUND is 1. */
static void d0(oro_state *s, const double *f, double *out, int dir) {
    size_t st[3] = { 1, (size_t)s->nx2, (size_t)s->nx2 * s->ny2 };
    size_t sd = st[dir];
    double h = dir == 0 ? s->hx : (dir == 1 ? s->hy : s->hz);
    int cd8 = s->c.scheme_vis == 204;
    int n = dir == 0 ? s->nx : (dir == 1 ? s->ny : s->nz);
    int lo = s->c.d0_bound[2 * dir] == 1, hi = s->c.d0_bound[2 * dir + 1] == 1;
#pragma omp parallel for
    for (int k = 0; k < s->nz; k++)
        for (int j = 0; j < s->ny; j++)
            for (int i = 0; i < s->nx; i++) {
                size_t q = L(s, i + LAP, j + LAP, k + LAP);
                int X = dir == 0 ? i : (dir == 1 ? j : k);
                double st9[9], tmp;
                for (int t = 0; t < 9; t++) st9[t] = f[q + (size_t)((long)(t - 4) * (long)sd)];
                if (!d0_closure(lo, hi, X, n, st9 + 4, &tmp))
                    tmp = cd8 ? oro_cd8(st9) : oro_cd6(st9 + 1);
                out[I(s, i, j, k)] = tmp/h;   /* put_d0_kernel :75-94 */
            }
}

/* get_Q (src/OCFD_ana.cu:317-456): the derivatives of u, v, w along the
 * three grid directions (OCFD_d{x,y,z}0 with the D0_bound closures), the
 * velocity gradient through the metrics (get_Q_kernal :317-389) and
 * Q = (ux vy + ux wz + vy wz - uy vx - uz wx - vz wy) Ajac^2 at every
 * interior cell.  (The reference kernel stores Q at LAP offsets into a field
 * allocated without ghosts; this is the interior value it computes.)  The
 * ghosts of u, v, w are exchanged first. */
void oro_q_criterion(oro_state *s, double *q) {
    exchange_xyz(s, s->u);
    exchange_xyz(s, s->v);
    exchange_xyz(s, s->w);
    const double *pr[3] = { s->u, s->v, s->w };
    for (int m = 0; m < 3; m++)
        for (int dir = 0; dir < 3; dir++) d0(s, pr[m], s->grad[3 * m + dir], dir);
#pragma omp parallel for
    for (int k = 0; k < s->nz; k++)
        for (int j = 0; j < s->ny; j++)
            for (int i = 0; i < s->nx; i++) {
                size_t p = L(s, i + LAP, j + LAP, k + LAP), c = I(s, i, j, k);
                double Akx = s->A[AKX][p], Aix = s->A[AIX][p], Asx = s->A[ASX][p];
                double Aky = s->A[AKY][p], Aiy = s->A[AIY][p], Asy = s->A[ASY][p];
                double Akz = s->A[AKZ][p], Aiz = s->A[AIZ][p], Asz = s->A[ASZ][p];
                double uk = s->grad[0][c], ui = s->grad[1][c], us = s->grad[2][c];
                double vk = s->grad[3][c], vi = s->grad[4][c], vs = s->grad[5][c];
                double wk = s->grad[6][c], wi = s->grad[7][c], ws = s->grad[8][c];
                double ux = uk*Akx + ui*Aix + us*Asx;
                double vx = vk*Akx + vi*Aix + vs*Asx;
                double wx = wk*Akx + wi*Aix + ws*Asx;
                double uy = uk*Aky + ui*Aiy + us*Asy;
                double vy = vk*Aky + vi*Aiy + vs*Asy;
                double wy = wk*Aky + wi*Aiy + ws*Asy;
                double uz = uk*Akz + ui*Aiz + us*Asz;
                double vz = vk*Akz + vi*Aiz + vs*Asz;
                double wz = wk*Akz + wi*Aiz + ws*Asz;
                double aj = s->A[AJAC][p];
                q[c] = (ux*vy + ux*wz + vy*wz - uy*vx - uz*wx - vz*wy) * aj * aj;
            }
}

static void viscous(oro_state *s) {
    /* du_viscous_Jacobian3d_init (:58-77) */
    const double *pr[4] = { s->u, s->v, s->w, s->T };
    for (int m = 0; m < 4; m++)
        for (int dir = 0; dir < 3; dir++) d0(s, pr[m], s->grad[3 * m + dir], dir);
    size_t nin = s->nin;
    for (int dir = 0; dir < 3; dir++) {
        /* vis_flux_ker (:80-236) with (Ax,Ay,Az) of this direction */
        const double *Ax = s->A[AKX + 3 * dir], *Ay = s->A[AKX + 3 * dir + 1], *Az = s->A[AKX + 3 * dir + 2];
#pragma omp parallel for
        for (int k = 0; k < s->nz; k++)
            for (int j = 0; j < s->ny; j++)
                for (int i = 0; i < s->nx; i++) {
                    size_t q = L(s, i + LAP, j + LAP, k + LAP), c = I(s, i, j, k);
                    double Akx = s->A[AKX][q], Aix = s->A[AIX][q], Asx = s->A[ASX][q];
                    double Aky = s->A[AKY][q], Aiy = s->A[AIY][q], Asy = s->A[ASY][q];
                    double Akz = s->A[AKZ][q], Aiz = s->A[AIZ][q], Asz = s->A[ASZ][q];
                    double Amu = s->amu[c];
                    double uk = s->grad[0][c], ui = s->grad[1][c], us = s->grad[2][c];
                    double vk = s->grad[3][c], vi = s->grad[4][c], vs = s->grad[5][c];
                    double wk = s->grad[6][c], wi = s->grad[7][c], ws = s->grad[8][c];
                    double Tk = s->grad[9][c], Ti = s->grad[10][c], Ts = s->grad[11][c];
                    double ux, vx, wx, uy, vy, wy, uz, vz, wz, div;
                    double s11, s12, s13, s22, s23, s33, E1, E2, E3, Tx, Ty, Tz, Amuk;
                    /* vis_flux_s_ker :24-78 */
                    ux = uk*Akx + ui*Aix + us*Asx;
                    vx = vk*Akx + vi*Aix + vs*Asx;
                    wx = wk*Akx + wi*Aix + ws*Asx;
                    uy = uk*Aky + ui*Aiy + us*Asy;
                    vy = vk*Aky + vi*Aiy + vs*Asy;
                    wy = wk*Aky + wi*Aiy + ws*Asy;
                    uz = uk*Akz + ui*Aiz + us*Asz;
                    vz = vk*Akz + vi*Aiz + vs*Asz;
                    wz = wk*Akz + wi*Aiz + ws*Asz;
                    div = ux + vy + wz;
                    s11 = (2.0*ux - 2.0/3.0*div) * Amu;
                    s22 = (2.0*vy - 2.0/3.0*div) * Amu;
                    s33 = (2.0*wz - 2.0/3.0*div) * Amu;
                    s12 = (uy + vx) * Amu;
                    s13 = (uz + wx) * Amu;
                    s23 = (vz + wy) * Amu;
                    /* vis_flux_e_ker :81-132 */
                    double u = s->u[q], v = s->v[q], w = s->w[q];
                    Amuk = Amu * s->vis_flux_init_c;
                    Tx = Tk*Akx + Ti*Aix + Ts*Asx;
                    Ty = Tk*Aky + Ti*Aiy + Ts*Asy;
                    Tz = Tk*Akz + Ti*Aiz + Ts*Asz;
                    E1 = u*s11 + v*s12 + w*s13 + Amuk*Tx;
                    E2 = u*s12 + v*s22 + w*s23 + Amuk*Ty;
                    E3 = u*s13 + v*s23 + w*s33 + Amuk*Tz;
                    /* vis_flus_ev_ker :135-174 */
                    double Aj1 = s->A[AJAC][q];
                    double akx = Ax[q]*Aj1, aky = Ay[q]*Aj1, akz = Az[q]*Aj1;
                    s->ev[0][q] = (akx*s11 + aky*s12 + akz*s13);
                    s->ev[1][q] = (akx*s12 + aky*s22 + akz*s23);
                    s->ev[2][q] = (akx*s13 + aky*s23 + akz*s33);
                    s->ev[3][q] = (akx*E1 + aky*E2 + akz*E3);
                }
        /* Ev ghost exchange in this direction (src/OCFD_Stream.cu:313-331) */
        for (int m = 0; m < 4; m++) {
            if (dir == 0) exchange_x(s, s->ev[m]);
            else if (dir == 1) exchange_y(s, s->ev[m]);
            else exchange_z(s, s->ev[m]);
        }
        /* du_viscous_Jacobian3d_{x,y,z}_final (:248-440): derivative + YF_Pe_XF */
        for (int m = 0; m < 4; m++) d0(s, s->ev[m], s->vis[m], dir);
#pragma omp parallel for
        for (int k = 0; k < s->nz; k++)
            for (int j = 0; j < s->ny; j++)
                for (int i = 0; i < s->nx; i++) {
                    size_t c = I(s, i, j, k);
                    double ajac = s->A[AJAC][L(s, i + LAP, j + LAP, k + LAP)];
                    for (int m = 0; m < 4; m++) s->du[(size_t)(m + 1) * nin + c] += ajac * s->vis[m][c];
                }
    }
}

/* ------------------------------------------------------------------------ */
/* stage orchestration                                                       */
/* ------------------------------------------------------------------------ */

void oro_du_comput(oro_state *s, int krk) {
    /* src/OCFD_Stream.cu:28-54, Stream_MODE 0 */
    if (s->c.scheme_invis == 310 && krk == 1) set_scheme_hybrid(s);
    memset(s->du, 0, 5 * s->nin * sizeof(double));
    /* du_invis_Jacobian3d (:289-305) */
    exchange_xyz(s, s->d); exchange_xyz(s, s->u); exchange_xyz(s, s->v);
    exchange_xyz(s, s->w); exchange_xyz(s, s->T);
    split_all(s);
    for (int dir = 0; dir < 3; dir++) invis_sweep(s, dir);
    /* du_vis_Jacobian3d (:307-335) */
    viscous(s);
}

/* OCFD_time_advance_ker{1,2,3}, src/OCFD_time.cu:44-94 */
void oro_time_advance(oro_state *s, int krk) {
    size_t n5 = 5 * s->nin;
    double dt = s->c.dt;
    double *f = s->f, *fn = s->fn, *du = s->du;
    if (krk == 1) {
#pragma omp parallel for
        for (long q = 0; q < (long)n5; q++) f[q] = fn[q] + dt*du[q];
    } else if (krk == 2) {
        double tmp1 = 3.0/4.0, tmp2 = 1.0/4.0;
#pragma omp parallel for
        for (long q = 0; q < (long)n5; q++) f[q] = tmp1*fn[q] + tmp2*(f[q] + dt*du[q]);
    } else {
        double tmp1 = 1.0/3.0, tmp2 = 2.0/3.0;
#pragma omp parallel for
        for (long q = 0; q < (long)n5; q++) f[q] = tmp1*fn[q] + tmp2*(f[q] + dt*du[q]);
        /* OCFD_time_advance_ker3 also writes pf_lap (:78-92) */
        if (s->flap) {
            for (int m = 0; m < 5; m++)
                for (int k = 0; k < s->nz; k++)
                    for (int j = 0; j < s->ny; j++)
                        for (int i = 0; i < s->nx; i++)
                            s->flap[(size_t)m * s->nlap + L(s, i + LAP, j + LAP, k + LAP)] = f[(size_t)m * s->nin + I(s, i, j, k)];
        }
    }
}

/* ------------------------------------------------------------------------ */
/* shock-capturing filter, src/OCFD_filtering.cu:363-606                     */
/* ------------------------------------------------------------------------ */

/* sigma of filter_{x,y}3d_shock_kernel at LAP point q along stride sd */
static double filter_sigma(const double *P, size_t q, long sd, double rth) {
    double p_m2 = P[q - 2 * sd], p_m1 = P[q - sd], p_00 = P[q], p_p1 = P[q + sd], p_p2 = P[q + 2 * sd];
    double dp0 = 0.25 * (-p_p1 + 2.0 * p_00 - p_m1);
    double dp1 = 0.25 * (-p_p2 + 2.0 * p_p1 - p_00);
    double dp2 = 0.25 * (-p_00 + 2.0 * p_m1 - p_m2);
    double ri = 0.5 * ((dp0 - dp1) * (dp0 - dp1) + (dp0 - dp2) * (dp0 - dp2)) / (p_00 * p_00) + 1e-16;
    ri = 1.0 - rth / ri;
    return 0.5 * (ri + fabs(ri));
}

/* One pass along dir over cells [b, e-1) along dir and [b, e) across it
 * (the kernels' coverage); U = pf_lap - filter(pf_lap), written to f.
 * jcap (>= 0): last covered index + 1 along y, for the z pass that the
 * reference launches as the y kernel on an (8, 8, 4+2) block (A-3). */
static void filter_pass(oro_state *s, int dir, const int *r, double s0, double rth, int jcap) {
    const double c1 = -0.2103830, c2 = 0.0396170;
    size_t st[3] = { 1, (size_t)s->nx2, (size_t)s->nx2 * s->ny2 };
    long sd = (long)st[dir];
    int lo[3] = { r[0], r[2], r[4] }, hi[3] = { r[1], r[3], r[5] };
    hi[dir] -= 1;
    if (jcap >= 0 && hi[1] > jcap) hi[1] = jcap;
#pragma omp parallel for collapse(2)
    for (int k = lo[2]; k < hi[2]; k++)
        for (int j = lo[1]; j < hi[1]; j++)
            for (int i = lo[0]; i < hi[0]; i++) {
                size_t q = L(s, i + LAP, j + LAP, k + LAP);
                double hm = filter_sigma(s->psens, q - sd, sd, rth);
                double h0 = filter_sigma(s->psens, q, sd, rth);
                double hp = filter_sigma(s->psens, q + sd, sd, rth);
                double Sc1 = 0.5 * (h0 + hp) * s0;
                double Sc2 = 0.5 * (h0 + hm) * s0;
                for (int m = 0; m < 5; m++) {
                    const double *fl = s->flap + (size_t)m * s->nlap;
                    s->f[(size_t)m * s->nin + I(s, i, j, k)] = fl[q] - (
                        Sc1 * (c1 * (fl[q + sd] - fl[q]) + c2 * (fl[q + 2 * sd] - fl[q - sd]))
                      - Sc2 * (c1 * (fl[q] - fl[q - sd]) + c2 * (fl[q + sd] - fl[q - 2 * sd])));
                }
            }
}

void oro_filtering(oro_state *s) {
    if (!s->c.nfilter) return;
    int any = 0;
    for (int m = 0; m < s->c.nfilter; m++)
        if (s->istep % s->fpar[m][0] == 0) any = 1;
    if (!any) return;
    /* exchange p and the five pf_lap fields in the directions any filter uses */
    void (*ex[3])(oro_state *, double *) = { exchange_x, exchange_y, exchange_z };
    for (int d = 0; d < 3; d++) {
        if (!s->fjudge[d]) continue;
        ex[d](s, s->psens);
        for (int m = 0; m < 5; m++) ex[d](s, s->flap + (size_t)m * s->nlap);
    }
    for (int m = 0; m < s->c.nfilter; m++) {
        if (!(s->tt <= s->c.filter_rpara[m][2])) continue;
        if (s->istep % s->fpar[m][0] != 0) continue;
        if (s->fpar[m][10] != 2) continue;          /* only the shock filter exists */
        double s0 = s->c.filter_rpara[m][0], rth = s->c.filter_rpara[m][1];
        const int *r = &s->fpar[m][4];
        if (s->fpar[m][1] == 1) filter_pass(s, 0, r, s0, rth, -1);
        if (s->fpar[m][2] == 1) filter_pass(s, 1, r, s0, rth, -1);
        if (s->fpar[m][3] == 1) {
            /* filter_z3d_shock launches the y kernel with blockdim (8, 8, 6)
             * on the grid for (8, 8, 4): y rows advance by 6 per block, so
             * only jb + 6*ceil((je-jb)/8) rows are reached */
            int jb = r[2], je = r[3];
            int gy = (je - jb + 7) / 8;
            filter_pass(s, 1, r, s0, rth, jb + 6 * gy);
        }
    }
}

void oro_swap_time_levels(oro_state *s) {
    double *t = s->f; s->f = s->fn; s->fn = t;
}

void oro_step(oro_state *s, int nsteps) {
    for (int n = 0; n < nsteps; n++) {
        oro_swap_time_levels(s);
        for (int krk = 1; krk <= 3; krk++) {
            oro_du_comput(s, krk);
            oro_time_advance(s, krk);
            oro_get_duvwT(s);
            oro_bc(s);
            oro_get_amu(s);
        }
        s->istep++;
        s->tt += s->c.dt;
        oro_filtering(s);
    }
}

/* ------------------------------------------------------------------------ */
/* read-back                                                                 */
/* ------------------------------------------------------------------------ */

static void copy_interior(const oro_state *s, const double *src, double *dst) {
    for (int k = 0; k < s->nz; k++)
        for (int j = 0; j < s->ny; j++)
            for (int i = 0; i < s->nx; i++)
                dst[I(s, i, j, k)] = src[L(s, i + LAP, j + LAP, k + LAP)];
}
void oro_get_primitives(const oro_state *s, double *prim5) {
    const double *src[5] = { s->d, s->u, s->v, s->w, s->T };
    for (int m = 0; m < 5; m++) copy_interior(s, src[m], prim5 + (size_t)m * s->nin);
}
void oro_get_pressure(const oro_state *s, double *p) { copy_interior(s, s->P, p); }
void oro_get_conserved(const oro_state *s, double *f5) { memcpy(f5, s->f, 5 * s->nin * sizeof(double)); }
void oro_get_conserved_n(const oro_state *s, double *f5) { memcpy(f5, s->fn, 5 * s->nin * sizeof(double)); }
void oro_get_du(const oro_state *s, double *du5) { memcpy(du5, s->du, 5 * s->nin * sizeof(double)); }
void oro_get_flags(const oro_state *s, int *sx, int *sy, int *sz) {
    memcpy(sx, s->sch[0], sizeof(int) * (size_t)(s->nx + 1) * s->ny * s->nz);
    memcpy(sy, s->sch[1], sizeof(int) * (size_t)s->nx * (s->ny + 1) * s->nz);
    memcpy(sz, s->sch[2], sizeof(int) * (size_t)s->nx * s->ny * (s->nz + 1));
}
int oro_istep(const oro_state *s) { return s->istep; }
double oro_tt(const oro_state *s) { return s->tt; }
