/*
 * ocfd_b200.h -- C ABI of the B200 (sm_100a) implementation of the
 * OpenCFD-SCU per-RK-stage right-hand-side path.
 *
 * Two layers:
 *
 *  1. A context API (ocfd_b200_*): explicit handle, int status codes (0 ok,
 *     negative on error, never aborts), caller-owned host buffers,
 *     library-owned device buffers, one CUDA stream per context.
 *
 *  2. Reference-named entry points (du_comput, OCFD_time_advance, get_duvwT,
 *     get_Amu, OCFD_bc, Set_Scheme_HybridAuto) acting on a context bound with
 *     ocfd_b200_compat_bind().  These replace the reference's own objects for
 *     the RHS path; the reference's driver, configuration reader and I/O link
 *     against them unchanged apart from its f/fn pointer swap.
 *
 * Arrays crossing the ABI are FP64, C order [nvar][nz][ny][nx] (x fastest),
 * interior cells only -- the order of the reference's record files
 * (src/OCFD_IO.c:157-228).  Primitive order is d,u,v,w,T; conserved order
 * is rho, rho u, rho v, rho w, E; metric order is
 * Axx Ayy Azz Akx Aky Akz Aix Aiy Aiz Asx Asy Asz Ajac
 * (src/OCFD_Comput_Jacobian3d.cu:142-181).
 */
#ifndef OCFD_B200_H
#define OCFD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OCFD_B200_ABI_VERSION 1

/* status codes */
#define OCFD_OK               0
#define OCFD_ERR_ARG         -1   /* bad argument or size                   */
#define OCFD_ERR_UNSUPPORTED -2   /* configuration outside what is built    */
#define OCFD_ERR_CUDA        -3   /* CUDA runtime error (see last_error)     */
#define OCFD_ERR_NOMEM       -4   /* device allocation failed                */
#define OCFD_ERR_STATE       -5   /* call out of order (e.g. no metrics yet) */
#define OCFD_ERR_NODEVICE    -6   /* no usable CUDA device                   */

typedef struct ocfd_b200_ctx ocfd_b200_ctx;

/* Replaces the globals that read_parameters() fills from opencfd-scu.in
 * (src/parameters.c:197-345) for the keys the RHS path consumes. */
typedef struct ocfd_b200_config {
    int nx, ny, nz;            /* GRID_3D (single GPU holds the whole grid)      */
    int iperiodic[3];          /* IPERIODIC                                       */
    int jac_bound[3];          /* JAC_BOUND                                       */
    int dif_bound[6];          /* DIF_BOUND                                       */
    int non_reflection[6];     /* NON_REFLETION                                   */
    int scheme_invis;          /* SCHEME_INVIS id: 301 UP7 .. 310 HYBRIDAUTO      */
    int scheme_vis;            /* SCHEME_VIS id: 203 CD6, 204 CD8                 */
    int charteric;             /* CHARTERIC                                       */
    int hy_style;              /* HY_STYLE (2 = Jameson pressure sensor)          */
    double hy_dp_intv[2];      /* HY_DP_INTV                                      */
    double re, ama, gamma, pr, t_ref, epsl_sw, dt;   /* RE AMA GAMMA PR T_REF EPSL_SW DT */
    int device;                /* CUDA device ordinal                             */
    /* SCHEME_HYBRIDAUTO with CHARTERIC = 0: the reference's per-component
     * kernels read an uninitialised scheme flag for components 1-4
     * (src/OCFD_Schemes_hybrid_auto.cu:907,1005); its sm_100a build then
     * uses WENO5 there.  0 (default) reproduces that build; 1 gives every
     * component the face's flag. */
    int hybrid_nochar_same_flag;
} ocfd_b200_config;

int  ocfd_b200_abi_version(void);
const char *ocfd_b200_status_string(int status);
/* Last error message of a context (or of the last failed create when ctx is NULL). */
const char *ocfd_b200_last_error(const ocfd_b200_ctx *ctx);

/* Allocate device state for one grid.  Replaces opencfd_mem_init_all()
 * (src/OCFD_init.cu:134-235) and opencfd_para_init[_dev]()
 * (src/OCFD_init.cu:381-410, :580-616). */
int ocfd_b200_create(const ocfd_b200_config *cfg, ocfd_b200_ctx **out);
int ocfd_b200_destroy(ocfd_b200_ctx *ctx);

/* Use the caller's CUDA stream (cudaStream_t passed as void*); NULL = the
 * context's own stream. */
int ocfd_b200_set_stream(ocfd_b200_ctx *ctx, void *stream);
void *ocfd_b200_get_stream(const ocfd_b200_ctx *ctx);
/* Waits for the context's stream, then reads the kernels' error word: a
 * wait on a staged tile or on a tensor-core product that ran out of its
 * bound (the kernel stopped; the step's result is invalid), or, in the
 * bounds-checked build, an index outside its array, returns OCFD_ERR_CUDA
 * with the cause in ocfd_b200_last_error and clears the word.  The hybrid
 * scheme's per-step read-back checks the same word. */
int ocfd_b200_synchronize(ocfd_b200_ctx *ctx);

/* Grid metrics, 13 interior fields (host or device memory).  Replaces the
 * OCFD3d-Jacobi.dat branch of Init_Jacobian3d()
 * (src/OCFD_Comput_Jacobian3d.cu:32-218): ghosts start at 1.0 and are
 * filled periodically in periodic directions. */
int ocfd_b200_set_metrics(ocfd_b200_ctx *ctx, const double *metrics13);
/* Metric storage: 0 (default) detects grids whose conservative metrics and
 * Jacobian are single values and keeps those in registers instead of
 * reading 10 fields (same arithmetic); 1 always reads the fields.  Takes
 * effect at the next set_metrics.  uniform_metrics reports the choice. */
int ocfd_b200_set_metric_mode(ocfd_b200_ctx *ctx, int mode);
int ocfd_b200_uniform_metrics(const ocfd_b200_ctx *ctx);
/* Inviscid sweep kernel variant: 4 (default) no block barriers: each warp
 * walks its own lines (one x row, or 8 y or z lines) through a ring of
 * split values in shared memory.  For UP7 the loop makes no calls and the
 * cells at bounded line ends are finished by a second kernel with the same
 * arithmetic; for WENO7 and the characteristic hybrid scheme every face,
 * closure and line-end rule is formed in the walk (variant 6), except that a
 * hybrid direction whose sensor pass marked almost every face UP7 takes the
 * UP7 walk with its few other cells deferred (the choice is read back once
 * per step, after the sensor); in the precision form the y and z UP7 walks
 * run as per-lane marches over pencil tiles staged in shared memory by the
 * tensor copy engine, each lane keeping its face window in registers.
 * 5: the walk with every face through one in-loop dispatch (the path of the
 * schemes other than UP7, WENO7 and the hybrid scheme in variant 4 too);
 * 6: the in-line walk alone (characteristic hybrid scheme and WENO7 only);
 * 7: as 4 with every UP7 walk through the shared-memory ring; 8: as 4 with
 * the y and z marches in FP64 as well (as fast as the ring there).  All
 * agree to the parity bound (WENO weights amplify the different multiply-add
 * contractions); 4, 7 and 8 agree bit for bit.  Other values: OCFD_ERR_ARG. */
int ocfd_b200_set_sweep_impl(ocfd_b200_ctx *ctx, int impl);
/* Arithmetic form of the stencils.  0 (default): FP64 throughout, the
 * reference's own arithmetic.  1, the precision form: the Steger-Warming
 * split, characteristic projection, reconstruction, sensor and viscous
 * stencils run in FP32 on FP32 copies of the primitives, with the stage
 * RHS and the viscous fluxes stored in FP32; the conserved state, the RK3
 * update, cons->prim, the grid metrics and the reductions stay FP64.
 * With a boundary-condition family its values are formed in FP64 (and
 * copied to the FP32 primitives); the shock filter forms its weights from an
 * FP32 pressure and updates U in FP64.  Covers the characteristic hybrid
 * scheme and WENO7 (OCFD_ERR_UNSUPPORTED otherwise); whole steps only
 * (ocfd_b200_step).  Switching back recomputes the FP64 primitives from the
 * conserved state. */
int ocfd_b200_set_precision(ocfd_b200_ctx *ctx, int form);
/* HybridAuto_scheme_Proportion (src/OCFD_Schemes_hybrid_auto.cu:745-829):
 * frac[3*d + t], the share of direction d's flag entries that are 1 (t=0),
 * 2 (t=1) or any other value (t=2), for the flags the last sensor pass
 * wrote. */
int ocfd_b200_scheme_proportion(ocfd_b200_ctx *ctx, double frac[9]);
/* get_Q (src/OCFD_ana.cu:317-456): the Q criterion
 * Q = (ux vy + ux wz + vy wz - uy vx - uz wx - vz wy) Ajac^2 of the current
 * primitives, the velocity derivatives by the viscous scheme's central
 * differences (with the DIF_BOUND closures) through the metrics, into a host
 * array [nz][ny][nx].  The reference's kernel stores Q at ghost offsets in a
 * field allocated without ghosts; this is the interior value it computes. */
int ocfd_b200_q_criterion(ocfd_b200_ctx *ctx, double *q);
/* init_time_average / ana_time_average (src/OCFD_ana.cu:224-316): reset != 0
 * zeroes the running means of d, u, v, w, T; reset = 0 adds the current
 * primitives as one more sample, m = (n m + x) / (n + 1).  get_time_average
 * copies the means to a host array [5][nz][ny][nx] (mean5 may be NULL) and
 * the number of samples to *count. */
int ocfd_b200_time_average(ocfd_b200_ctx *ctx, int reset);
int ocfd_b200_get_time_average(ocfd_b200_ctx *ctx, double *mean5, int *count);
/* Learned scheme switch (hybrid scheme).  A 14 -> 32 -> 32 -> 1 ReLU network
 * over normalised pressure and density differences on the sensor's 7-point
 * stencil takes the place of the plain sensor's choice
 * (Comput_Scheme_point_Jameson, src/OCFD_Schemes_hybrid_auto.cu:611-703) and
 * writes the same flag arrays: a cell whose confidence max(s, 1 - s),
 * s = sigmoid(output), reaches `confidence` gets flag 1 (s < 1/2) or the
 * larger of 2 and the plain flag (s >= 1/2); any other cell keeps the plain
 * flag.  Inference: BF16 tensor-core products, FP32 accumulation.  The
 * parameter vector (ocfd_b200_mlp_nparam() floats) is mu[14] sigma[14]
 * W1[32][14] b1[32] W2[32][32] b2[32] W3[32] b3, features standardised as
 * (f - mu) / sigma.  params = NULL switches back to the plain sensor. */
int ocfd_b200_mlp_nparam(void);
int ocfd_b200_set_switch(ocfd_b200_ctx *ctx, const float *params, int nparam, double confidence);
/* Cells decided by the network, cells left to the plain flag, and network
 * flags that differ from the plain flag, summed over sensor passes since
 * the last ocfd_b200_set_switch. */
int ocfd_b200_switch_stats(ocfd_b200_ctx *ctx, long long counts[3]);
/* Features (count x 14, FP32) and labels (1 where the plain flag is 2 or
 * 3) of interior cells first .. first+count-1 (x fastest) of the current
 * state, into host arrays: the training data of the switch. */
int ocfd_b200_switch_features(ocfd_b200_ctx *ctx, long long first, long long count, float *feat, float *label);
/* Stand-alone network kernels on the current device (host arrays in and
 * out): logits of n feature rows through the tensor-core path; the FP32
 * gradient (network part, from W1 on) and loss of the summed binary
 * cross-entropy over n rows with positives weighted pos_w; Adam training
 * over shuffled mini-batches (params in/out, mean loss per epoch out). */
const char *ocfd_b200_mlp_last_error(void);
int ocfd_b200_mlp_infer(const float *params, const float *feat, long long n, float *logit);
int ocfd_b200_mlp_grad(const float *params, const float *feat, const float *label, long long n, float pos_w,
                       float *grad, double *loss);
int ocfd_b200_mlp_train(float *params, const float *feat, const float *label, long long n, int epochs, int batch,
                        float lr, float pos_w, unsigned long long seed, double *epoch_loss);
/* Bit d set: direction d currently takes the walk that forms every face in
 * line (variant 4 after the last sensor pass, or variant 6). */
int ocfd_b200_sweep_walks(const ocfd_b200_ctx *ctx);
/* Share of a direction's cells that the UP7 walk would defer (2 x its
 * non-UP7 faces, plus closed line ends) above which variant 4 takes the
 * in-line walk for that direction; default 0.002.  3 or more keeps the
 * UP7 walk whatever the sensor marks (every other cell then goes to the fix-up
 * kernel).  No reference counterpart (a tuning knob of this library). */
int ocfd_b200_set_walk_threshold(ocfd_b200_ctx *ctx, double frac);
/* Kernel of the viscous divergence + RK stage of whole steps: 2 stages the
 * Ev tiles of each plane (x and y with their halos, z in a ring of planes)
 * in shared memory by bulk tensor copies while the block marches along z;
 * 1 reads every Ev value through the L1/L2 caches; 0 (default) the staged
 * kernel in the precision form and the cached one in FP64, each the faster
 * of the two there.  The same arithmetic (results equal bit for bit).  No reference counterpart
 * (du_viscous_Jacobian3d_*_final, src/OCFD_NS_Jacobian3d.cu:80-440, is the
 * computation both replace). */
int ocfd_b200_set_viscous_impl(ocfd_b200_ctx *ctx, int impl);
int ocfd_b200_set_metrics_device(ocfd_b200_ctx *ctx, const double *metrics13_dev);
/* Mesh coordinates x,y,z, 3 interior fields (host or device memory), from
 * which the 13 metric fields are computed on the GPU.  Replaces the
 * OCFD3d-Mesh.dat branch of Init_Jacobian3d
 * (src/OCFD_Comput_Jacobian3d.cu:119-141) and Comput_Jacobian3d (:221-246):
 * CD6 derivatives of the coordinates, one-sided closures at both ends of a
 * direction whose JAC_BOUND is non-zero, cross products and the inverse
 * determinant, constant extrapolation into the ghosts, periodic exchange.
 * Returns OCFD_ERR_ARG on a negative Jacobian (ana_Jac, src/OCFD_ana.cu:24-48). */
int ocfd_b200_set_mesh(ocfd_b200_ctx *ctx, const double *xyz3);
int ocfd_b200_set_mesh_device(ocfd_b200_ctx *ctx, const double *xyz3_dev);
/* The 13 metric fields the kernels use, interior, OCFD3d-Jacobi.dat order
 * (synchronous; metrics must be set). */
int ocfd_b200_get_metrics(ocfd_b200_ctx *ctx, double *metrics13);

/* Initial primitives d,u,v,w,T (host or device).  Replaces the
 * INIT_STAT=1 part of init() (src/OCFD_init.cu:88-115): ghosts zero, then
 * pri_to_cons; followed by the pre-loop of NS_solver_real
 * (src/OCFD_NS_Solver.cu:45-53). */
int ocfd_b200_set_primitives(ocfd_b200_ctx *ctx, const double *prim5, int istep, double tt);
int ocfd_b200_set_primitives_device(ocfd_b200_ctx *ctx, const double *prim5_dev, int istep, double tt);

/* Whole steps as CUDA graphs (no counterpart in the reference; default on):
 * a step whose stages need nothing from the host -- no kernel timing, no
 * boundary-condition family, no z split -- is captured once per time-level
 * parity and replayed, which removes the per-kernel launch cost on small
 * grids.  With the hybrid scheme's automatic walk choice the first sensor
 * pass and its read-back run first and the graph holds the rest of the step
 * for the walks chosen.  Any change of the parameters, the stream or the switch
 * captures it again.  On a stream the caller is capturing, the kernels go
 * into the caller's graph; on a stream that cannot be captured (the legacy
 * default stream) steps launch one by one.  0 turns it off (every kernel
 * launched one by one). */
int ocfd_b200_set_graphs(ocfd_b200_ctx *ctx, int enabled);
/* Step graphs captured so far (a replayed step adds none). */
long long ocfd_b200_graph_captures(const ocfd_b200_ctx *ctx);
/* nsteps full SSP-RK3 steps (time-level swap + 3 stages each),
 * src/OCFD_NS_Solver.cu:63-89.  Asynchronous on the context stream. */
int ocfd_b200_step(ocfd_b200_ctx *ctx, int nsteps);

/* End-to-end call with host buffers: copy prim5_in to the device, run
 * nsteps, copy the primitives back into prim5_out (may alias prim5_in).
 * Metrics must be set.  Synchronous. */
int ocfd_b200_advance_host(ocfd_b200_ctx *ctx, const double *prim5_in, double *prim5_out,
                           int nsteps);

/* Boundary-condition family IBC with BC_NPARA / BC_RPARA (bc_parameter,
 * src/OCFD_boundary_init.c:50-93).  0: none; 108: compression corner
 * (src/OCFD_boundary_compression_conner.cu:122-180) with npara = MZMAX, MTMAX,
 * INLET_BOUNDARY, IFLAG_WALL_NOT_NORMAL and rpara = TW, EPSL, X_DIST_BEGIN,
 * X_DIST_END, BETA, X_WALL_BEGIN, X_UP_BOUNDARY_BEGIN, SLZ; inlet4 is the
 * flow1d-inlet.dat profile [4][ny] (d,u,v,T), needed when INLET_BOUNDARY = 1.
 * Call after the metrics (the wall and top coordinates are read from them)
 * and before set_primitives.  MZMAX > 0 sums MZMAX spanwise modes whose
 * phases are the first MZMAX draws of the C library's rand() from its initial
 * state, as the reference's set-up takes them (it seeds nothing first,
 * src/OCFD_boundary_init.c:444-499); MZMAX <= 4096. */
int ocfd_b200_set_bc(ocfd_b200_ctx *ctx, int ibc, const int *npara, int nnpara, const double *rpara,
                     int nrpara, const double *inlet4);

/* Shock-capturing filter n (0..7): FILTER_NPARA<n+1> = ntime, filter_x,
 * filter_y, filter_z, ib, ie, jb, je, kb, ke, scheme (2) and FILTER_RPARA<n+1>
 * = s0, rth, time limit (src/parameters.c:305-325); ranges clamped as
 * set_para_filtering (src/OCFD_filtering.cu:20-73).  step() then runs
 * filtering() (:75-183) after every step whose Istep is a multiple of ntime
 * while tt <= the time limit.  It reads the pressure the hybrid sensor
 * forms, so it is meaningful with SCHEME_HYBRIDAUTO only (as in the
 * reference, whose pressure field is otherwise zero). */
int ocfd_b200_set_filter(ocfd_b200_ctx *ctx, int n, const int npara[11], const double rpara[3]);
/* filtering() at the context's Istep and tt (src/OCFD_NS_Solver.cu:95). */
int ocfd_b200_filtering(ocfd_b200_ctx *ctx);
/* The driver's Istep and tt, which the per-stage calls do not advance. */
int ocfd_b200_set_time(ocfd_b200_ctx *ctx, int istep, double tt);

/* Per-stage pieces, same semantics as the reference calls of one stage. */
int ocfd_b200_swap_time_levels(ocfd_b200_ctx *ctx);        /* src/OCFD_NS_Solver.cu:65-73 */
int ocfd_b200_du_comput(ocfd_b200_ctx *ctx, int krk);      /* src/OCFD_Stream.cu:28-54    */
int ocfd_b200_time_advance(ocfd_b200_ctx *ctx, int krk);   /* src/OCFD_time.cu:96-123     */
int ocfd_b200_get_duvwT(ocfd_b200_ctx *ctx);               /* src/commen_kernel.cu:111-118 */
int ocfd_b200_bc(ocfd_b200_ctx *ctx);                      /* src/OCFD_boundary.cu:18-92  */

/* ---- the grid split in z across GPUs (one z slab per process) --------- */
/* Replaces the reference's z decomposition (part3d with NPX0 = NPY0 = 1,
 * src/OCFD_mpi.c:120-190) and its z halo exchange
 * (exchange_boundary_z_packed_dev, src/OCFD_mpi_dev.cu:271-310, host-staged
 * MPI_Sendrecv there): the ghost planes of each slab come from its
 * neighbours' interior planes over NCCL, device to device, wherever the
 * single-GPU path wraps z.  The context's nz is the slab's plane count.
 * ocfd_b200_slab_unique_id: one rank makes the id (NCCL's unique id) and
 * hands it to the others (e.g. over torch.distributed).
 * ocfd_b200_set_slab: call on every rank, right after create and before the
 * filters, metrics and state (collective: it returns once all nranks have
 * joined); rank_lo / rank_hi are the ranks holding the planes below / above
 * (ID_ZM1 / ID_ZP1, src/OCFD_mpi.c:183-189), z_offset this slab's first
 * global plane (k_offset).  Requires IPERIODIC z = 1 and at least 4 planes
 * per slab.  ana_residual, check_state and scheme_proportion then return
 * whole-grid values on every rank; the per-step walk choice uses the whole
 * grid's flag counts.  OCFD_ERR_UNSUPPORTED when NCCL cannot be loaded. */
#define OCFD_SLAB_ID_BYTES 128
int ocfd_b200_slab_unique_id(unsigned char id[OCFD_SLAB_ID_BYTES]);
int ocfd_b200_set_slab(ocfd_b200_ctx *ctx, int nranks, int rank, int rank_lo, int rank_hi, int z_offset,
                       int nz_global, const unsigned char id[OCFD_SLAB_ID_BYTES]);
/* The same split with the exchange carried by the caller instead of NCCL,
 * as the reference carries it through host memory and MPI_Sendrecv
 * (exchange_boundary_z_packed_dev, src/OCFD_mpi_dev.cu:271-310): a driver
 * with its own MPI between ranks whose GPUs have no NCCL path, or several
 * slab processes sharing one GPU (no kernel of one waits on another's).
 * The library packs the ghost planes, copies them to pinned host memory and
 * calls fn(user, 0, send, recv, count, type): send holds count elements for
 * rank_lo (this slab's lowest interior planes) then count for rank_hi (its
 * highest); fn must fill recv with rank_lo's count (that rank's highest
 * planes) then rank_hi's (its lowest), pairing the transfers as two
 * Sendrecv would.  The analysis sums call fn(user, 1, buf, buf, count,
 * type): sum buf over all ranks in place.  type: 0 FP64, 1 uint64, 2 uint32,
 * 3 FP32.  fn returns 0 on success.  Whole steps then run launched (no step
 * graph). */
typedef int (*ocfd_b200_slab_transport)(void *user, int op, void *send, void *recv, size_t count, int type);
int ocfd_b200_set_slab_host(ocfd_b200_ctx *ctx, int nranks, int rank, int rank_lo, int rank_hi, int z_offset,
                            int nz_global, ocfd_b200_slab_transport fn, void *user);

/* Read-back (synchronous). */
int ocfd_b200_get_primitives(ocfd_b200_ctx *ctx, double *prim5);
int ocfd_b200_get_primitives_device(ocfd_b200_ctx *ctx, double *prim5_dev);
int ocfd_b200_get_conserved(ocfd_b200_ctx *ctx, double *cons5);
int ocfd_b200_get_du(ocfd_b200_ctx *ctx, double *du5);
int ocfd_b200_get_flags(ocfd_b200_ctx *ctx, int8_t *flag_x, int8_t *flag_y, int8_t *flag_z);
int ocfd_b200_get_time(const ocfd_b200_ctx *ctx, int *istep, double *tt);

/* FP64 interior mean of E (which = 0) or T (which = 1); replaces
 * ana_residual() (src/OCFD_ana.cu:76-105), deterministic on any warp width. */
int ocfd_b200_ana_residual(ocfd_b200_ctx *ctx, int which, double *mean);
/* Counts cells with a NaN in d,u,v,w,T and cells with T < 0 (the checks of
 * ana_NAN_and_NT, src/OCFD_ana.cu:107-222) and returns the mean T. */
int ocfd_b200_check_state(ocfd_b200_ctx *ctx, long long *n_nan, long long *n_neg_t, double *mean_t);

/* Kernel timing: when enabled, step() brackets each kernel family with CUDA
 * events on the context stream.  get_timing returns accumulated device
 * milliseconds and launch counts per family (names by index). */
#define OCFD_TIMER_COUNT 8
int ocfd_b200_set_timing(ocfd_b200_ctx *ctx, int enabled);
int ocfd_b200_get_timing(ocfd_b200_ctx *ctx, double *ms, long long *launches, int n);
const char *ocfd_b200_timer_name(int index);
/* number of kernel launches issued by the library so far */
long long ocfd_b200_launch_count(const ocfd_b200_ctx *ctx);

/* ---- allocation-free field means (no counterpart in the reference) ---- */
/* FP64 means of nfield dense fields of n doubles each, laid out one after
 * another at `fields`; means[f] = sum(field f) / n.  Both pointers are
 * device memory on the calling thread's current device; the call is
 * asynchronous on `stream` (a cudaStream_t, NULL = legacy default stream).
 * It allocates nothing, for callers that keep their fields in their own
 * device buffers and may not allocate between steps (no context is
 * created; no cudaMalloc/cudaFree and their implicit synchronisation).
 * Partial sums go to one fixed device array shared by every call on a
 * device: at most OCFD_NOALLOC_MAX_FIELDS fields x 592 partials (37,888
 * bytes); nfield above the maximum returns OCFD_ERR_ARG with the reason in
 * ocfd_b200_last_error(NULL).  Every call looks up that array's address on
 * the current device (no allocation); the first call on a device can load
 * the library's device code there, so make it before any stream capture on
 * that device.
 * Calls that overlap in time on one device (other streams, other threads)
 * race on the shared array; order them.  For the same values the mean is
 * bitwise that of ocfd_b200_ana_residual. */
#define OCFD_NOALLOC_MAX_FIELDS 8
int ocfd_b200_field_means_noalloc(const double *fields, int nfield, long long n, double *means,
                                  void *stream);

/* ---- reference-named entry points (act on the bound context) ---------- */
int  ocfd_b200_compat_bind(ocfd_b200_ctx *ctx);
/* A translation unit that also includes the reference's own headers, which
 * declare these names with the reference's types, defines
 * OCFD_B200_NO_REFERENCE_NAMES before including this header. */
#ifndef OCFD_B200_NO_REFERENCE_NAMES
void du_comput(int KRK);                    /* head/OCFD_Stream.h:10           */
void OCFD_time_advance(int KRK);            /* src/OCFD_time.cu:96             */
void get_duvwT(void);                       /* head/commen_kernel.h:17         */
void get_Amu(void);                         /* head/commen_kernel.h:20         */
void OCFD_bc(void);                         /* src/OCFD_boundary.cu:18         */
void Set_Scheme_HybridAuto(void *stream);   /* head/OCFD_Schemes_hybrid_auto.h:24 (cudaStream_t*) */
void filtering(double *pf, double *pf_lap, double *pp);   /* src/OCFD_filtering.cu:75 */
#endif

#ifdef __cplusplus
}
#endif
#endif
