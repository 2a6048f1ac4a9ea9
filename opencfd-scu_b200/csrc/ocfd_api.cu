// ocfd_api.cu -- C ABI (include/ocfd_b200.h) over the sm_100a kernels.
//
// State ownership follows the reference's process-global device buffers
// (head/parameters_d.h:24-80) but lives in an explicit context: primitive
// and metric fields on the LAP box (LAP = 4 ghost layers), conserved
// variables f, fn and du without ghosts, hybrid flags as int8.
#include "ocfd_b200.h"
#include "ocfd_device.cuh"

#include <cuda.h>
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace ocfd {
cudaError_t launch_sensor(const Params &p, cudaStream_t st);
cudaError_t launch_q_criterion(const Params &p, double *q, cudaStream_t st);
cudaError_t launch_time_average(const Params &p, double *mean5, int n, cudaStream_t st);
bool march_tensor_map(const Params &p, const void *base, int elem_bytes, int dir, CUtensorMap *out);
bool march_supported(const Params &p, int dir);
cudaError_t march_prepare();
cudaError_t vdiv_prepare();
cudaError_t launch_march_dir(const Params &p, const CUtensorMap &tm, int dir, cudaStream_t st);
cudaError_t launch_ghost(const Params &p, double *const *fields, const int *dirmask, int nf, cudaStream_t st);
cudaError_t launch_ghost32(const Params &p, float *const *fields, const int *dirmask, int nf, cudaStream_t st);
cudaError_t launch_prims_to_fp32(const Params &p, cudaStream_t st);
cudaError_t launch_flag_hist(const Params &p, unsigned long long *counts, cudaStream_t st);
cudaError_t launch_vis_ev(const Params &p, cudaStream_t st);
cudaError_t launch_vis_div(const Params &p, int krk, int k0, int k1, cudaStream_t st);
void ev_ghost_fields(const Params &p, void *fields[12], int dirmask[12]);
cudaError_t launch_rk(const Params &p, int krk, cudaStream_t st);
cudaError_t launch_rk_only(const Params &p, int krk, cudaStream_t st);
cudaError_t launch_c2p(const Params &p, cudaStream_t st);
cudaError_t launch_bc_faces(const Params &p, cudaStream_t st);
cudaError_t launch_p2c(const Params &p, double *out, cudaStream_t st);
cudaError_t launch_scatter(const Params &p, const double *src, double *dst_lap, cudaStream_t st);
cudaError_t launch_gather(const Params &p, const double *src_lap, double *dst, cudaStream_t st);
cudaError_t launch_fill(double *f, long long n, double v, cudaStream_t st);
cudaError_t launch_mean(const Params &p, int which, double *scratch, unsigned long long *counts, double ncell,
                        cudaStream_t st);
struct Slab;
int slab_unique_id(unsigned char id[128], std::string &err);
Slab *slab_create(const Params &p, int nranks, int rank, int lo, int hi, const unsigned char id[128],
                  std::string &err);
void slab_destroy(Slab *s);
int slab_exchange(Slab *s, const Params &p, double *const *f, int nf, cudaStream_t st, std::string &err);
int slab_exchange32(Slab *s, const Params &p, float *const *f, int nf, cudaStream_t st, std::string &err);
int slab_allreduce(Slab *s, void *buf, size_t count, int type, cudaStream_t st, std::string &err);
Slab *slab_create_host(const Params &p, int nranks, int rank, int lo, int hi, SlabTransport fn, void *user,
                       std::string &err);
int slab_launches_per_exchange();
int reduce_scratch_doubles();
cudaError_t launch_sweeps3(const Params &p, cudaStream_t st);
cudaError_t launch_sweeps4(const Params &p, cudaStream_t st);
bool sweeps4_supported(const Params &p);
cudaError_t launch_sweep4_dir(const Params &p, int dir, cudaStream_t st);
cudaError_t launch_sweep3_dir(const Params &p, int dir, cudaStream_t st);
bool sweeps3_defers(const Params &p);
cudaError_t launch_mesh_metrics(const Params &p, const int jac_bound[3], double *scratch, cudaStream_t st);
cudaError_t launch_negative_jacobian(const Params &p, unsigned *flag, cudaStream_t st);
cudaError_t launch_filter_pass(const Params &p, int dir, const int box[6], double s0, double rth, cudaStream_t st);
cudaError_t launch_bc108(const Params &p, double ht, cudaStream_t st);
int sweeps3_kernels(const Params &p);
cudaError_t compute_dirconst(Params &p, DirConst *dev_scratch, cudaStream_t st);
int mlp_nparam();
int mlp_nnet();
int mlp_grad_blocks(long long n);
cudaError_t launch_switch_features(const Params &p, long long first, long long count, float *feat, float *label,
                                   cudaStream_t st);
cudaError_t launch_switch_infer(const Params &p, const float *w, float conf_logit, unsigned long long *stats,
                                cudaStream_t st);
cudaError_t launch_mlp_infer(const float *w, const float *feat, long long n, float *logit, int *err,
                             cudaStream_t st);
cudaError_t launch_mlp_grad(const float *w, const float *feat, const float *label, const int *idx, long long n,
                            float pos_w, float *part, float *lpart, float *grad, double *loss, cudaStream_t st);
cudaError_t launch_mlp_adam(float *w, const float *grad, float *m1, float *m2, float scale, float lr, int t,
                            cudaStream_t st);
}  // namespace ocfd

using ocfd::Params;

namespace {

enum Timer { T_SENSOR = 0, T_GHOST, T_SWEEP, T_VIS, T_RK, T_OTHER1, T_OTHER2, T_OTHER3 };
const char *kTimerNames[OCFD_TIMER_COUNT] = {
    "sensor", "ghost_fill", "inviscid_sweeps", "viscous_rk_update", "rk_update", "-", "-", "-"};

thread_local std::string g_create_error;

}  // namespace

struct ocfd_b200_ctx {
    ocfd_b200_config cfg;
    Params p;
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    // allocations
    double *prim_buf = nullptr;   // 5 LAP fields
    double *met_buf = nullptr;    // 13 LAP fields
    double *cons_buf = nullptr;   // f, fn, du: 15 interior fields
    double *ev_buf = nullptr;     // 12 LAP fields
    int8_t *flag_buf = nullptr;
    double *stage_buf = nullptr;  // 5 interior fields for host transfers
    double *red_buf = nullptr;    // reduction partials + result, then 16 words of counters
    unsigned *defer_buf = nullptr;  // three counters (padded to 256 B), then 3 deferred-cell lists
    double *filter_buf = nullptr;   // pf_lap (5 LAP fields) and the pressure (1 LAP field)
    // FILTER_NPARA / FILTER_RPARA as set_para_filtering leaves them
    int nfilter = 0;
    int fpar[8][11] = {};
    double frpar[8][3] = {};
    int fjudge[3] = {0, 0, 0};
    // IBC 108: device profile/shape arrays and the wall-blowing time law
    double *bc_buf = nullptr;
    double bc_beta = 0.0;
    int bc_mtmax = 0;
    double bc_TM[64] = {};
    double *pinned = nullptr;     // host staging for advance_host
    size_t pinned_bytes = 0;
    // hybrid scheme, variant 4: per direction, 1 = the walk that forms every
    // face in line, 0 = the UP7 walk with deferred cells; chosen after each
    // sensor pass from its count of non-UP7 faces
    unsigned *h_flag_count = nullptr;   // pinned
    // precision form: FP32 primitives (5 LAP fields), stage RHS (5 interior
    // fields) and viscous fluxes (12 LAP fields); the FP64 primitives are
    // brought up to date from the conserved state before they are read
    // (with a filter the last stage has written their interior: only the
    // ghosts are stale)
    float *prec_buf = nullptr;
    bool prims64_stale = false;
    bool prims64_interior_ok = false;
    // learned scheme switch: parameter vector on the device, the confidence
    // threshold as a logit, decision counters
    float *sw_w = nullptr;
    unsigned long long *sw_stats = nullptr;
    bool sw_on = false;
    float sw_conf_logit = 0.0f;
    int walk4[3] = {1, 1, 1};
    double walk4_threshold = 0.002;     // deferred cells per cell above which the inline walk is used
    // the UP7 walk of the y and z sweeps as per-lane marches over staged
    // pencil tiles (ocfd_march.cu): tensor maps of the FP64 and FP32
    // primitives per direction (y, z).  march: 0 the shared-memory ring walk
    // everywhere (sweep variant 7), 1 the march in the precision form only
    // (default: in FP64 the ring walk measured as fast), 2 the march in both
    // forms (variant 8)
    CUtensorMap tm64[2];
    CUtensorMap tm32[2];
    bool tm64_ok = false, tm32_ok = false;
    bool vdiv_ok = true;        // the staged divergence kernel can be launched
    // running time averages of d, u, v, w, T (5 interior fields, allocated on
    // first use) and the number of samples in them
    double *avg_buf = nullptr;
    int avg_n = 0;
    int march = 1;
    // the grid split in z across GPUs: this rank's slab starts at global
    // plane z_offset of nz_global; ghost planes in z come from the
    // neighbouring slabs (null: one GPU holds the grid)
    ocfd::Slab *slab = nullptr;
    int z_offset = 0, nz_global = 0, slab_count = 1;
    // the primitives' z exchange runs on its own stream while the x and y
    // sweeps (which read no z ghosts) run; the z sweep waits for it
    cudaStream_t xstream = nullptr;
    cudaEvent_t xev[2] = {nullptr, nullptr};
    // single-GPU steps: the viscous fluxes (they read only the primitives)
    // run on vstream beside the inviscid sweeps; vev fork and join it
    cudaStream_t vstream = nullptr;
    cudaEvent_t vev[2] = {nullptr, nullptr};
    bool x_pending = false;
    bool have_metrics = false;
    int metric_mode = 0;          // 0 auto-detect uniform grids, 1 always read the fields
    bool have_state = false;
    int istep = 0;
    double tt = 0.0;
    long long launches = 0;
    // timing
    bool timing = false;
    // whole RK3 steps replayed from CUDA graphs (one per time-level parity,
    // captured on first use and again whenever the parameter block, the
    // stream or the switch set-up differs from the captured one)
    struct StepGraph {
        cudaGraphExec_t exec = nullptr;
        Params key;
        cudaStream_t stream = nullptr;
        bool sw_on = false;
        float sw_conf = 0.0f;
        long long launches = 0;
        int walk = -1;          // the walks chosen by the sensor pass before it (-1: none)
        int march = 1;
    } graph[2];
    bool graphs_on = true;
    long long graph_captures = 0;       // step graphs captured so far
    cudaEvent_t ev[2] = {nullptr, nullptr};
    double t_ms[OCFD_TIMER_COUNT] = {0};
    long long t_n[OCFD_TIMER_COUNT] = {0};
    std::string err;
};

// interior cells of the whole grid
static double global_cells(const ocfd_b200_ctx *c) {
    return c->slab ? (double)c->p.nx * c->p.ny * c->nz_global : (double)c->p.N;
}

static int fail(ocfd_b200_ctx *c, int code, const std::string &msg) {
    if (c) c->err = msg; else g_create_error = msg;
    return code;
}

static int cuda_fail(ocfd_b200_ctx *c, cudaError_t e, const char *where) {
    std::string m = std::string(where) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    return fail(c, OCFD_ERR_CUDA, m);
}

#define CK(call, where)                                     \
    do {                                                    \
        cudaError_t _e = (call);                            \
        if (_e != cudaSuccess) return cuda_fail(ctx, _e, where); \
    } while (0)

extern "C" int ocfd_b200_abi_version(void) { return OCFD_B200_ABI_VERSION; }

extern "C" const char *ocfd_b200_status_string(int s) {
    switch (s) {
    case OCFD_OK: return "ok";
    case OCFD_ERR_ARG: return "invalid argument";
    case OCFD_ERR_UNSUPPORTED: return "unsupported configuration";
    case OCFD_ERR_CUDA: return "CUDA error";
    case OCFD_ERR_NOMEM: return "device out of memory";
    case OCFD_ERR_STATE: return "call out of order";
    case OCFD_ERR_NODEVICE: return "no CUDA device";
    }
    return "unknown status";
}

extern "C" const char *ocfd_b200_last_error(const ocfd_b200_ctx *ctx) {
    return ctx ? ctx->err.c_str() : g_create_error.c_str();
}

static void free_all(ocfd_b200_ctx *c) {
    cudaFree(c->prim_buf); cudaFree(c->met_buf); cudaFree(c->cons_buf);
    cudaFree(c->ev_buf); cudaFree(c->flag_buf); cudaFree(c->stage_buf);
    cudaFree(c->avg_buf);
    cudaFree(c->red_buf); cudaFree(c->defer_buf); cudaFree(c->filter_buf); cudaFree(c->bc_buf);
    if (c->pinned) cudaFreeHost(c->pinned);
    if (c->h_flag_count) cudaFreeHost(c->h_flag_count);
    cudaFree(c->prec_buf);
    cudaFree(c->sw_w);
    cudaFree(c->sw_stats);
    for (auto &g : c->graph) if (g.exec) { cudaGraphExecDestroy(g.exec); g.exec = nullptr; }
    if (c->xstream) cudaStreamSynchronize(c->xstream);
    ocfd::slab_destroy(c->slab);
    c->slab = nullptr;
    for (auto &e : c->xev) if (e) cudaEventDestroy(e);
    if (c->xstream) cudaStreamDestroy(c->xstream);
    if (c->vstream) cudaStreamSynchronize(c->vstream);
    for (auto &e : c->vev) if (e) cudaEventDestroy(e);
    if (c->vstream) cudaStreamDestroy(c->vstream);
    for (auto &e : c->ev) if (e) cudaEventDestroy(e);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
}

extern "C" int ocfd_b200_create(const ocfd_b200_config *cfg, ocfd_b200_ctx **out) {
    ocfd_b200_ctx *ctx = nullptr;
    if (!cfg || !out) return fail(nullptr, OCFD_ERR_ARG, "null argument");
    *out = nullptr;
    if (cfg->nx < 8 || cfg->ny < 8 || cfg->nz < 8)
        return fail(nullptr, OCFD_ERR_ARG, "each grid dimension must be >= 8 (LAP = 4 on both sides)");
    long long N = (long long)cfg->nx * cfg->ny * cfg->nz;
    if (N > (1LL << 34)) return fail(nullptr, OCFD_ERR_ARG, "grid too large");
    int si = cfg->scheme_invis;
    if (si < 301 || si > 310) return fail(nullptr, OCFD_ERR_UNSUPPORTED, "SCHEME_INVIS id must be 301..310");
    if (cfg->scheme_vis != 203 && cfg->scheme_vis != 204)
        return fail(nullptr, OCFD_ERR_UNSUPPORTED, "SCHEME_VIS id must be 203 (CD6) or 204 (CD8)");
    if (si == 310 && cfg->hy_style != 2)
        return fail(nullptr, OCFD_ERR_UNSUPPORTED, "SCHEME_HYBRIDAUTO is built for HY_STYLE = 2 (Jameson sensor)");
    if (!(cfg->ama > 0) || !(cfg->gamma > 1) || !(cfg->re > 0) || !(cfg->pr > 0))
        return fail(nullptr, OCFD_ERR_ARG, "AMA, GAMMA, RE, PR out of range");

    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(nullptr, OCFD_ERR_NODEVICE, "no CUDA device");
    if (cfg->device < 0 || cfg->device >= ndev) return fail(nullptr, OCFD_ERR_ARG, "device ordinal out of range");

    ctx = new ocfd_b200_ctx();
    ctx->cfg = *cfg;
    ctx->device = cfg->device;
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) { int r = cuda_fail(nullptr, e, "cudaSetDevice"); delete ctx; return r; }

    Params &p = ctx->p;
    memset(&p, 0, sizeof(p));
    p.nx = cfg->nx; p.ny = cfg->ny; p.nz = cfg->nz;
    int nx2 = p.nx + 2 * OCFD_LAP, ny2 = p.ny + 2 * OCFD_LAP, nz2 = p.nz + 2 * OCFD_LAP;
    p.pitch = (nx2 + 7) / 8 * 8;                 // 64-byte rows
    p.ys = p.pitch;
    p.zs = (long long)p.pitch * ny2;
    p.lapN = p.zs * nz2;
    p.N = N;
    // init() and opencfd_para_init() (src/OCFD_init.cu:29-31, :381-399)
    p.hx = 1.0 / (p.nx - 1.0);
    p.hy = 1.0 / (p.ny - 1.0);
    p.hz = 1.0 / (p.nz - 1.0);
    double G = cfg->gamma, Ma = cfg->ama;
    double t_ref = cfg->t_ref > 0 ? cfg->t_ref : 288.15;
    p.Ama = Ma; p.Gamma = G; p.epsl_sw = cfg->epsl_sw;
    p.Cv = 1.0 / (G * (G - 1.0) * Ma * Ma);
    double Cp = 1.0 / ((G - 1.0) * Ma * Ma);
    p.Tsb = 110.4 / t_ref;
    p.amu_C0 = 1.0 / cfg->re * (1.0 + 110.4 / t_ref);
    p.tmp0 = 1.0 / (2.0 * G);
    p.split_C1 = 2.0 * (G - 1.0);
    p.split_C3 = (3.0 - G) / (2.0 * (G - 1.0));
    p.vis_c = Cp / cfg->pr;
    p.dt = cfg->dt;
    p.p00 = 1.0 / (G * Ma * Ma);                 // Comput_P (src/OCFD_Schemes_hybrid_auto.cu:64)
    p.tv_lim = 5.0; p.tv_max = 0.2;              // src/parameters.c:75-76
    p.dp1 = cfg->hy_dp_intv[0]; p.dp2 = cfg->hy_dp_intv[1];
    p.scheme_invis = si; p.scheme_vis = cfg->scheme_vis; p.charteric = cfg->charteric;
    p.nochar_comp_flag = cfg->hybrid_nochar_same_flag ? 0 : 3;
    p.sweep_impl = 4;
    p.inv_h[0] = 1.0 / p.hx; p.inv_h[1] = 1.0 / p.hy; p.inv_h[2] = 1.0 / p.hz;
    p.inv_Ama = 1.0 / Ma;
    for (int d = 0; d < 3; d++) p.periodic[d] = cfg->iperiodic[d];
    p.zface_lo = p.zface_hi = 1;
    p.has_bnd = 0;
    for (int d = 0; d < 3; d++) {
        p.bnd_lo[d] = cfg->dif_bound[2 * d] == 1;
        p.bnd_hi[d] = cfg->dif_bound[2 * d + 1] == 1;
        p.nonref_lo[d] = cfg->non_reflection[2 * d];
        p.nonref_hi[d] = cfg->non_reflection[2 * d + 1];
        p.has_bnd |= p.bnd_lo[d] | p.bnd_hi[d] | (p.nonref_lo[d] == 1) | (p.nonref_hi[d] == 1);
    }

    size_t lapB = sizeof(double) * (size_t)p.lapN, inB = sizeof(double) * (size_t)N;
    size_t flagN = (size_t)(p.nx + 1) * p.ny * p.nz + (size_t)p.nx * (p.ny + 1) * p.nz + (size_t)p.nx * p.ny * (p.nz + 1);
    auto alloc = [&](void **ptr, size_t bytes, const char *what) -> int {
        cudaError_t ae = cudaMalloc(ptr, bytes);
        if (ae != cudaSuccess) {
            cudaGetLastError();
            ctx->err = std::string("cudaMalloc(") + what + "): " + cudaGetErrorString(ae);
            return ae == cudaErrorMemoryAllocation ? OCFD_ERR_NOMEM : OCFD_ERR_CUDA;
        }
        return OCFD_OK;
    };
    int rc;
    if ((rc = alloc((void **)&ctx->prim_buf, 5 * lapB, "primitives")) ||
        (rc = alloc((void **)&ctx->met_buf, 13 * lapB, "metrics")) ||
        (rc = alloc((void **)&ctx->cons_buf, 15 * inB, "conserved")) ||
        (rc = alloc((void **)&ctx->ev_buf, 12 * lapB, "viscous fluxes")) ||
        (rc = alloc((void **)&ctx->flag_buf, flagN, "flags")) ||
        (rc = alloc((void **)&ctx->stage_buf, 5 * inB, "staging")) ||
        (rc = alloc((void **)&ctx->red_buf, sizeof(double) * (ocfd::reduce_scratch_doubles() + 16), "reduction")) ||
        // deferred-cell lists of the call-free sweep (cell indices fit 32 bits)
        (N < (1LL << 32) && (rc = alloc((void **)&ctx->defer_buf, sizeof(unsigned) * (64 + 3 * (size_t)N),
                                        "deferred cells")))) {
        g_create_error = ctx->err;
        free_all(ctx);
        delete ctx;
        return rc;
    }
    for (int m = 0; m < 5; m++) p.prim[m] = ctx->prim_buf + (size_t)m * p.lapN;
    for (int m = 0; m < 13; m++) p.met[m] = ctx->met_buf + (size_t)m * p.lapN;
    p.f = ctx->cons_buf; p.fn = ctx->cons_buf + 5 * N; p.du = ctx->cons_buf + 10 * N;
    p.ev = ctx->ev_buf;
    p.flag[0] = ctx->flag_buf;
    p.flag[1] = ctx->flag_buf + (size_t)(p.nx + 1) * p.ny * p.nz;
    p.flag[2] = p.flag[1] + (size_t)p.nx * (p.ny + 1) * p.nz;
    p.defer_count = ctx->defer_buf;
    for (int d = 0; d < 3; d++) p.defer[d] = ctx->defer_buf ? ctx->defer_buf + 64 + (size_t)d * N : nullptr;
    p.flag_count = nullptr;
    if (ctx->defer_buf && cudaHostAlloc((void **)&ctx->h_flag_count, 64, cudaHostAllocDefault) == cudaSuccess)
        p.flag_count = ctx->defer_buf + 8;
    // word 16 of the counter block: the kernels' error word
    p.kerr = ctx->defer_buf ? reinterpret_cast<int *>(ctx->defer_buf + 16) : nullptr;
    if (p.kerr && (e = cudaMemset(p.kerr, 0, sizeof(int))) != cudaSuccess) {
        cuda_fail(nullptr, e, "error word");
        free_all(ctx); delete ctx;
        return OCFD_ERR_CUDA;
    }
    // the staged divergence kernel is used only when its shared-memory size is set
    if (ocfd::vdiv_prepare() != cudaSuccess) { cudaGetLastError(); p.vis_impl = 1; ctx->vdiv_ok = false; }
    ctx->tm64_ok = ocfd::march_prepare() == cudaSuccess &&
                   ocfd::march_tensor_map(p, ctx->prim_buf, 8, 1, &ctx->tm64[0]) &&
                   ocfd::march_tensor_map(p, ctx->prim_buf, 8, 2, &ctx->tm64[1]);
    cudaGetLastError();

    if ((e = cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreate(&ctx->ev[0])) != cudaSuccess || (e = cudaEventCreate(&ctx->ev[1])) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&ctx->vstream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&ctx->vev[0], cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&ctx->vev[1], cudaEventDisableTiming)) != cudaSuccess) {
        cuda_fail(nullptr, e, "stream/event create");
        free_all(ctx); delete ctx;
        return OCFD_ERR_CUDA;
    }
    ctx->stream = ctx->own_stream;
    // Init_Jacobian3d: metrics 1.0 everywhere; init(): primitives and du zero
    if ((e = ocfd::launch_fill(ctx->met_buf, 13 * p.lapN, 1.0, ctx->stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(ctx->prim_buf, 0, 5 * lapB, ctx->stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(ctx->cons_buf, 0, 15 * inB, ctx->stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(ctx->ev_buf, 0, 12 * lapB, ctx->stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(ctx->flag_buf, 0, flagN, ctx->stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) {
        cuda_fail(nullptr, e, "initialisation");
        free_all(ctx); delete ctx;
        return OCFD_ERR_CUDA;
    }
    *out = ctx;
    return OCFD_OK;
}

extern "C" int ocfd_b200_destroy(ocfd_b200_ctx *ctx) {
    if (!ctx) return OCFD_ERR_ARG;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    free_all(ctx);
    delete ctx;
    return OCFD_OK;
}

extern "C" int ocfd_b200_set_stream(ocfd_b200_ctx *ctx, void *stream) {
    if (!ctx) return OCFD_ERR_ARG;
    ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
    return OCFD_OK;
}
extern "C" void *ocfd_b200_get_stream(const ocfd_b200_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

// a kernel whose wait on a staged copy ran out leaves 1 in the error word
static int check_kerr(ocfd_b200_ctx *ctx, int word) {
    if (word == 0) return OCFD_OK;
    int zero = 0;
    cudaMemcpy(ctx->p.kerr, &zero, sizeof(int), cudaMemcpyHostToDevice);
    if (word == 3) {
        int at[3] = {0, 0, 0};
        cudaMemcpy(at, ctx->p.kerr + 1, sizeof(at), cudaMemcpyDeviceToHost);
        const long long v = (long long)(unsigned)at[1] | (long long)at[2] << 32;
        return fail(ctx, OCFD_ERR_CUDA, "bounds-checked build: a kernel formed an index outside its array "
                                        "(check at source line " + std::to_string(at[0]) + ", value " +
                                        std::to_string(v) + "; the access was redirected, the result is invalid)");
    }
    return fail(ctx, OCFD_ERR_CUDA, word == 2 ? "the learned switch gave up waiting for a tensor-core product "
                                                 "(the step's result is invalid)"
                                               : "a kernel gave up waiting for a staged tile (the step's result is invalid)");
}

extern "C" int ocfd_b200_synchronize(ocfd_b200_ctx *ctx) {
    if (!ctx) return OCFD_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->stream), "synchronize");
    if (ctx->p.kerr) {
        int w = 0;
        CK(cudaMemcpy(&w, ctx->p.kerr, sizeof(int), cudaMemcpyDeviceToHost), "error word");
        return check_kerr(ctx, w);
    }
    return OCFD_OK;
}

// ---------------------------------------------------------------------------
// internal helpers
// ---------------------------------------------------------------------------

static cudaError_t ghost_launch(const Params &p, double *const *f, const int *mask, int n, cudaStream_t st) {
    return ocfd::launch_ghost(p, f, mask, n, st);
}
static cudaError_t ghost_launch(const Params &p, float *const *f, const int *mask, int n, cudaStream_t st) {
    return ocfd::launch_ghost32(p, f, mask, n, st);
}
static int slab_exchange(ocfd_b200_ctx *ctx, double *const *f, int n, cudaStream_t st, std::string &err) {
    return ocfd::slab_exchange(ctx->slab, ctx->p, f, n, st, err);
}
static int slab_exchange(ocfd_b200_ctx *ctx, float *const *f, int n, cudaStream_t st, std::string &err) {
    return ocfd::slab_exchange32(ctx->slab, ctx->p, f, n, st, err);
}

// the solver stream waits for a z exchange left running on its own stream
static int join_z(ocfd_b200_ctx *ctx) {
    if (!ctx->x_pending) return OCFD_OK;
    ctx->x_pending = false;
    CK(cudaStreamWaitEvent(ctx->stream, ctx->xev[1], 0), "z exchange join");
    return OCFD_OK;
}

// Ghost fill of LAP-box fields, mask bit d for direction d: the periodic
// wrap on one GPU; with the grid split in z, the x and y wraps here and the
// z ghost planes from the neighbouring slabs (the reference's
// exchange_boundary_{x,y,z}_packed_dev order, src/OCFD_mpi_dev.cu:186-310)
// defer_z: the z exchange runs on the exchange stream; join_z before
// anything reads the z ghosts
template <typename T>
static int fill_ghosts(ocfd_b200_ctx *ctx, T *const *f, const int *mask, int n, const char *what,
                       bool defer_z = false) {
    if (!ctx->slab) {
        CK(ghost_launch(ctx->p, f, mask, n, ctx->stream), what);
        ctx->launches += 1;
        return OCFD_OK;
    }
    int mxy[16];
    T *fz[16];
    int nz = 0;
    bool xy = false;
    for (int m = 0; m < n; m++) {
        mxy[m] = mask[m] & 3;
        xy = xy || mxy[m];
        if (mask[m] & 4) fz[nz++] = f[m];
    }
    if (xy) {
        CK(ghost_launch(ctx->p, f, mxy, n, ctx->stream), what);
        ctx->launches += 1;
    }
    if (nz) {
        std::string err;
        cudaStream_t st = ctx->stream;
        if (defer_z && ctx->xstream) {
            int rc = join_z(ctx);
            if (rc) return rc;
            CK(cudaEventRecord(ctx->xev[0], ctx->stream), "z exchange fork");
            CK(cudaStreamWaitEvent(ctx->xstream, ctx->xev[0], 0), "z exchange fork");
            st = ctx->xstream;
        }
        if (slab_exchange(ctx, fz, nz, st, err)) return fail(ctx, OCFD_ERR_CUDA, std::string(what) + ": " + err);
        ctx->launches += ocfd::slab_launches_per_exchange();
        if (st != ctx->stream) {
            CK(cudaEventRecord(ctx->xev[1], st), "z exchange done");
            ctx->x_pending = true;
        }
    }
    return OCFD_OK;
}

static int ghost_prims64(ocfd_b200_ctx *ctx) {
    double *f[5]; int mask[5];
    for (int m = 0; m < 5; m++) { f[m] = ctx->p.prim[m]; mask[m] = 7; }
    return fill_ghosts(ctx, f, mask, 5, "ghost fill");
}

// the primitives the stencils read: FP64, or FP32 in the precision form
static int ghost_prims(ocfd_b200_ctx *ctx, bool defer_z = false) {
    if (!ctx->p.mixed) {
        double *f[5]; int mask[5];
        for (int m = 0; m < 5; m++) { f[m] = ctx->p.prim[m]; mask[m] = 7; }
        return fill_ghosts(ctx, f, mask, 5, "ghost fill", defer_z);
    }
    float *f[5]; int mask[5];
    for (int m = 0; m < 5; m++) { f[m] = ctx->p.prim32[m]; mask[m] = 7; }
    return fill_ghosts(ctx, f, mask, 5, "ghost fill", defer_z);
}

// precision form: FP64 primitives (interior and ghosts) from the FP64
// conserved state, before anything reads them
static int refresh_prims64(ocfd_b200_ctx *ctx) {
    if (!ctx->prims64_stale) return OCFD_OK;
    if (!ctx->prims64_interior_ok) {
        CK(ocfd::launch_c2p(ctx->p, ctx->stream), "cons_to_pri");
        ctx->launches += 1;
    }
    int rc = ghost_prims64(ctx);
    if (rc) return rc;
    ctx->prims64_stale = false;
    return OCFD_OK;
}

static int ghost_metrics(ocfd_b200_ctx *ctx) {
    double *f[12]; int mask[12];
    for (int m = 0; m < 12; m++) { f[m] = const_cast<double *>(ctx->p.met[m]); mask[m] = 7; }
    int rc = fill_ghosts(ctx, f, mask, 12, "metric ghost fill");
    if (rc) return rc;
    double *fj[1] = { const_cast<double *>(ctx->p.met[12]) }; int mj[1] = { 7 };
    return fill_ghosts(ctx, fj, mj, 1, "metric ghost fill");
}

// A kernel family of one stage: an NVTX range named for it (seen by a
// profiler attached to the process, free otherwise) and, with timing on,
// CUDA events around it on the solver stream.
struct TimerScope {
    ocfd_b200_ctx *c; int which; bool on;
    TimerScope(ocfd_b200_ctx *cc, int w) : c(cc), which(w), on(cc->timing) {
        nvtxRangePushA(kTimerNames[w]);
        if (on) cudaEventRecord(c->ev[0], c->stream);
    }
    ~TimerScope() {
        nvtxRangePop();
        if (!on) return;
        cudaEventRecord(c->ev[1], c->stream);
        if (cudaEventSynchronize(c->ev[1]) == cudaSuccess) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
            c->t_ms[which] += ms;
            c->t_n[which] += 1;
        }
    }
};

// One stage's RHS.  fused_rk = 0: du_comput semantics (du complete on
// return).  fused_rk = KRK: the viscous divergence kernel also applies the
// RK stage, cons->prim and the face re-projection (step() path).
// the boundary-condition family's values on the primitives
// (bc_user_Compression_conner, src/OCFD_boundary_compression_conner.cu:122-180)
static int apply_bc(ocfd_b200_ctx *ctx) {
    if (ctx->p.ibc != 108) return OCFD_OK;
    double ht = 0.;
    if (ctx->bc_beta > 0.) {
        for (int m = 0; m < ctx->bc_mtmax && m < 64; m++)
            ht = ht + ctx->bc_TM[m] * sin((m + 1) * ctx->bc_beta * ctx->tt);
    } else {
        ht = 1.;
    }
    CK(ocfd::launch_bc108(ctx->p, ht, ctx->stream), "boundary conditions");
    ctx->launches += 3;
    return OCFD_OK;
}

// Which walk each direction takes under variant 4 for the hybrid scheme.
// The UP7 walk leaves the two cells beside every non-UP7 face, and the ~10
// cells at each bounded end of a line, to a per-cell fix-up kernel that
// costs about as much as 80 cells of the walk; above a small fraction of
// such cells the walk that forms every face in line is faster.
static bool walk4_wanted(const ocfd_b200_ctx *ctx, int d, unsigned nonup7) {
    const Params &p = ctx->p;
    // flag entries the count covers (with the grid split in z, the counts are
    // summed over the slabs, each with its own nz + 1 entries in z)
    const long long nzc = ctx->slab ? (long long)ctx->nz_global + (d == 2) * (ctx->slab_count - 1) : p.nz;
    const long long nf = (long long)(p.nx + (d == 0)) * (p.ny + (d == 1)) * (nzc + (d == 2));
    const int n = d == 0 ? p.nx : (d == 1 ? p.ny : p.nz);
    const bool ends = p.bnd_lo[d] || p.bnd_hi[d] || p.nonref_lo[d] == 1 || p.nonref_hi[d] == 1;
    const double deferred = 2.0 * (double)nonup7 / (double)nf + (ends ? 10.0 / n : 0.0);
    return deferred > ctx->walk4_threshold;
}

static int sweeps_auto(ocfd_b200_ctx *ctx) {
    const Params &p = ctx->p;
    const bool hyb = p.scheme_invis == 310;
    int w[3];
    for (int d = 0; d < 3; d++) w[d] = (hyb && p.sweep_impl != 6) ? ctx->walk4[d] : 1;
    if ((!w[0] || !w[1] || !w[2]) && ocfd::sweeps3_defers(p))
        CK(cudaMemsetAsync(p.defer_count, 0, 3 * sizeof(unsigned), ctx->stream), "deferred counters");
    for (int d = 0; d < 3; d++) {
        if (d == 2) {
            int rc = join_z(ctx);
            if (rc) return rc;
        }
        if (w[d]) {
            CK(ocfd::launch_sweep4_dir(p, d, ctx->stream), "inviscid sweeps");
            ctx->launches += 1;
        } else if (d > 0 && ctx->march > (p.mixed ? 0 : 1) && ocfd::march_supported(p, d) &&
                   (p.mixed ? ctx->tm32_ok : ctx->tm64_ok)) {
            CK(ocfd::launch_march_dir(p, p.mixed ? ctx->tm32[d - 1] : ctx->tm64[d - 1], d, ctx->stream),
               "inviscid sweeps");
            ctx->launches += 2;
        } else {
            CK(ocfd::launch_sweep3_dir(p, d, ctx->stream), "inviscid sweeps");
            ctx->launches += ocfd::sweeps3_defers(p) ? 2 : 1;
        }
    }
    return OCFD_OK;
}

// the hybrid scheme's sensor (or learned switch) pass of the first stage,
// with the per-step read-back of its non-UP7 counts that picks the walks
static bool needs_readback(const ocfd_b200_ctx *ctx) {
    const Params &p = ctx->p;
    return p.scheme_invis == 310 && (p.sweep_impl == 4 || p.mixed) && ocfd::sweeps4_supported(p) && p.flag_count;
}

static int rhs_sensor(ocfd_b200_ctx *ctx) {
    const Params &p = ctx->p;
    {
        TimerScope ts(ctx, T_SENSOR);
        if (ctx->sw_on) CK(ocfd::launch_switch_infer(p, ctx->sw_w, ctx->sw_conf_logit, ctx->sw_stats, ctx->stream),
                           "learned switch");
        else            CK(ocfd::launch_sensor(p, ctx->stream), "sensor");
        ctx->launches += 1;
        if (needs_readback(ctx)) {
            // the choice follows this pass's flags: one small read-back per step
            if (ctx->slab) {        // every slab takes the same walk: counts of the whole grid
                std::string err;
                if (ocfd::slab_allreduce(ctx->slab, p.flag_count, 3, 2, ctx->stream, err))
                    return fail(ctx, OCFD_ERR_CUDA, err);
            }
            // the three counts and, 8 words on, the kernels' error word
            CK(cudaMemcpyAsync(ctx->h_flag_count, p.flag_count, 9 * sizeof(unsigned), cudaMemcpyDeviceToHost,
                               ctx->stream), "flag counts");
            CK(cudaStreamSynchronize(ctx->stream), "flag counts");
            if (int rc = check_kerr(ctx, (int)ctx->h_flag_count[8])) return rc;
            for (int d = 0; d < 3; d++) ctx->walk4[d] = walk4_wanted(ctx, d, ctx->h_flag_count[d]);
        }
    }
    return OCFD_OK;
}

// skip_sensor: the first stage's sensor pass has run already (step graphs)
static int rhs(ocfd_b200_ctx *ctx, int krk, int fused_rk, bool skip_sensor = false) {
    const Params &p = ctx->p;
    if (p.scheme_invis == 310 && krk == 1 && !skip_sensor) {
        int rc = rhs_sensor(ctx);
        if (rc) return rc;
    }
    {
        TimerScope ts(ctx, T_GHOST);
        int rc = ghost_prims(ctx, true);      // the z planes arrive while the x and y sweeps run
        if (rc) return rc;
    }
    // On one GPU the viscous fluxes and their ghost fill (they read the
    // primitives only) go to a second stream beside the inviscid sweeps; the
    // divergence kernel waits for both.  Timed runs keep the families apart.
    const bool side = ctx->vstream && !ctx->slab && !ctx->timing;
    void *evf[12]; int evmask[12];
    ocfd::ev_ghost_fields(p, evf, evmask);
    if (side) {
        CK(cudaEventRecord(ctx->vev[0], ctx->stream), "viscous fork");
        CK(cudaStreamWaitEvent(ctx->vstream, ctx->vev[0], 0), "viscous fork");
        CK(ocfd::launch_vis_ev(p, ctx->vstream), "viscous fluxes");
        CK(p.mixed ? ghost_launch(p, reinterpret_cast<float *const *>(evf), evmask, 12, ctx->vstream)
                   : ghost_launch(p, reinterpret_cast<double *const *>(evf), evmask, 12, ctx->vstream),
           "Ev ghost fill");
        CK(cudaEventRecord(ctx->vev[1], ctx->vstream), "viscous join");
        ctx->launches += 2;
    }
    {
        TimerScope ts(ctx, T_SWEEP);
        if (p.sweep_impl == 6 && !ocfd::sweeps4_supported(p))
            return fail(ctx, OCFD_ERR_UNSUPPORTED, "sweep variant 6 covers the characteristic hybrid scheme and WENO7");
        if (p.mixed || (p.sweep_impl == 4 && ocfd::sweeps4_supported(p))) {
            int rc = sweeps_auto(ctx);
            if (rc) return rc;
        } else {            // the other variants launch the three directions together
            int rc = join_z(ctx);
            if (rc) return rc;
            if (p.sweep_impl == 6) CK(ocfd::launch_sweeps4(p, ctx->stream), "inviscid sweeps");
            else                   CK(ocfd::launch_sweeps3(p, ctx->stream), "inviscid sweeps");
            ctx->launches += p.sweep_impl == 6 ? 3 : ocfd::sweeps3_kernels(p);
        }
    }
    {
        TimerScope ts(ctx, T_VIS);
        if (side) {
            CK(cudaStreamWaitEvent(ctx->stream, ctx->vev[1], 0), "viscous join");
        } else {
            CK(ocfd::launch_vis_ev(p, ctx->stream), "viscous fluxes");
            // (forming the planes away from the slab faces while the Ev_z planes
            // travel, and the two bands next to the faces after, measured slower
            // than one launch after the exchange: the small band launches and the
            // extra tail cost more than the exchange they hide)
            int rc = p.mixed ? fill_ghosts(ctx, reinterpret_cast<float *const *>(evf), evmask, 12, "Ev ghost fill")
                             : fill_ghosts(ctx, reinterpret_cast<double *const *>(evf), evmask, 12, "Ev ghost fill");
            if (rc) return rc;
            ctx->launches += 1;
        }
        CK(ocfd::launch_vis_div(p, fused_rk, 0, p.nz, ctx->stream), "viscous divergence");
        ctx->launches += 1;
    }
    if (fused_rk && p.ibc) {        // OCFD_bc: boundary values, then the faces
        int rc = apply_bc(ctx);
        if (rc) return rc;
        CK(ocfd::launch_bc_faces(p, ctx->stream), "face re-projection");
        ctx->launches += 1;
    }
    return OCFD_OK;
}

static int check_ready(ocfd_b200_ctx *ctx) {
    if (!ctx) return OCFD_ERR_ARG;
    if (!ctx->have_metrics) return fail(ctx, OCFD_ERR_STATE, "metrics not set");
    if (!ctx->have_state) return fail(ctx, OCFD_ERR_STATE, "primitives not set");
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
    return OCFD_OK;
}

// ---------------------------------------------------------------------------
// set-up
// ---------------------------------------------------------------------------

// A grid whose nine conservative metrics and Jacobian are each one value
// everywhere (uniform Cartesian) lets the kernels take them from the
// parameter block; the arithmetic is the same as reading the fields.
static void detect_uniform(ocfd_b200_ctx *ctx, const double *host13) {
    Params &p = ctx->p;
    // ghosts of a non-periodic direction keep the initial 1.0, which the
    // characteristic record of a boundary face averages in: field path
    bool uni = ctx->metric_mode == 0 && p.periodic[0] && p.periodic[1] && p.periodic[2];
    for (int m = 0; m < 13 && uni; m++) {
        const double *f = host13 + (size_t)m * p.N;
        p.mc[m] = f[0];
        if (m < ocfd::M_AKX) continue;          // coordinates are not read by the RHS
        for (long long q = 1; q < p.N; q++)
            if (f[q] != f[0]) { uni = false; break; }
    }
    p.uniform_metrics = uni ? 1 : 0;
}

static int set_metrics_impl(ocfd_b200_ctx *ctx, const double *src, cudaMemcpyKind kind) {
    if (!ctx || !src) return OCFD_ERR_ARG;
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    const Params &p = ctx->p;
    size_t inB = sizeof(double) * (size_t)p.N;
    if (kind == cudaMemcpyHostToDevice) {
        detect_uniform(ctx, src);
    } else {
        double *h = (double *)malloc(13 * inB);
        if (!h) return fail(ctx, OCFD_ERR_NOMEM, "host buffer for metric check");
        cudaError_t e = cudaMemcpy(h, src, 13 * inB, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) { free(h); return cuda_fail(ctx, e, "metric read-back"); }
        detect_uniform(ctx, h);
        free(h);
    }
    // Init_Jacobian3d starts every metric field at 1.0, ghosts included
    CK(ocfd::launch_fill(ctx->met_buf, 13 * p.lapN, 1.0, ctx->stream), "metric init");
    ctx->launches += 1;
    for (int m = 0; m < 13; m++) {
        CK(cudaMemcpyAsync(ctx->stage_buf, src + (size_t)m * p.N, inB, kind, ctx->stream), "metric copy");
        CK(ocfd::launch_scatter(p, ctx->stage_buf, const_cast<double *>(p.met[m]), ctx->stream), "metric scatter");
        ctx->launches += 1;
    }
    int rc = ghost_metrics(ctx);
    if (rc) return rc;
    if (ctx->p.uniform_metrics)
        CK(ocfd::compute_dirconst(ctx->p, reinterpret_cast<ocfd::DirConst *>(ctx->red_buf), ctx->stream),
           "direction constants");
    CK(cudaStreamSynchronize(ctx->stream), "set_metrics");
    ctx->have_metrics = true;
    return OCFD_OK;
}

extern "C" int ocfd_b200_set_metric_mode(ocfd_b200_ctx *ctx, int mode) {
    if (!ctx || mode < 0 || mode > 1) return OCFD_ERR_ARG;
    ctx->metric_mode = mode;
    if (mode == 1) ctx->p.uniform_metrics = 0;
    return OCFD_OK;
}
extern "C" int ocfd_b200_uniform_metrics(const ocfd_b200_ctx *ctx) { return ctx ? ctx->p.uniform_metrics : 0; }

// ---------------------------------------------------------------------------
// the grid split in z across GPUs (part3d with NPX0 = NPY0 = 1,
// src/OCFD_mpi.c:120-190)
// ---------------------------------------------------------------------------
extern "C" int ocfd_b200_slab_unique_id(unsigned char id[OCFD_SLAB_ID_BYTES]) {
    if (!id) return fail(nullptr, OCFD_ERR_ARG, "id is null");
    std::string err;
    if (ocfd::slab_unique_id(id, err)) return fail(nullptr, OCFD_ERR_UNSUPPORTED, err);
    return OCFD_OK;
}

static int set_slab_impl(ocfd_b200_ctx *ctx, int nranks, int rank, int rank_lo, int rank_hi, int z_offset,
                         int nz_global, const unsigned char *id, ocfd::SlabTransport fn, void *user) {
    if (!ctx || (!id && !fn)) return OCFD_ERR_ARG;
    Params &p = ctx->p;
    if (ctx->slab) return fail(ctx, OCFD_ERR_STATE, "the slab is already set");
    if (ctx->have_metrics || ctx->have_state || ctx->nfilter)
        return fail(ctx, OCFD_ERR_STATE, "set the slab before the filters, metrics and state");
    if (nranks < 1 || rank < 0 || rank >= nranks || rank_lo < 0 || rank_lo >= nranks || rank_hi < 0 ||
        rank_hi >= nranks)
        return fail(ctx, OCFD_ERR_ARG, "rank, neighbour ranks and rank count out of range");
    if (!p.periodic[2])
        return fail(ctx, OCFD_ERR_UNSUPPORTED, "the z split needs a periodic z direction (IPERIODIC z = 1)");
    if (p.nz < OCFD_LAP) return fail(ctx, OCFD_ERR_ARG, "a slab needs at least 4 z planes");
    if (z_offset < 0 || nz_global < p.nz || z_offset + p.nz > nz_global)
        return fail(ctx, OCFD_ERR_ARG, "slab planes outside the grid");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    // the exchange stream and its events first, so that a failure leaves the
    // context as it was (a stream or event made here is released at destroy)
    if ((!ctx->xstream && cudaStreamCreateWithFlags(&ctx->xstream, cudaStreamNonBlocking) != cudaSuccess) ||
        (!ctx->xev[0] && cudaEventCreateWithFlags(&ctx->xev[0], cudaEventDisableTiming) != cudaSuccess) ||
        (!ctx->xev[1] && cudaEventCreateWithFlags(&ctx->xev[1], cudaEventDisableTiming) != cudaSuccess)) {
        cudaGetLastError();
        return fail(ctx, OCFD_ERR_CUDA, "exchange stream");
    }
    std::string err;
    ctx->slab = fn ? ocfd::slab_create_host(p, nranks, rank, rank_lo, rank_hi, fn, user, err)
                   : ocfd::slab_create(p, nranks, rank, rank_lo, rank_hi, id, err);
    if (!ctx->slab) return fail(ctx, OCFD_ERR_CUDA, err);
    ctx->z_offset = z_offset;
    ctx->nz_global = nz_global;
    ctx->slab_count = nranks;
    // hz = 1/(NZ_GLOBAL - 1) (src/OCFD_init.cu:29-31); OCFD_bc re-projects
    // only the faces of the whole grid (src/OCFD_boundary.cu:78-95)
    p.hz = 1.0 / (nz_global - 1.0);
    p.inv_h[2] = 1.0 / p.hz;
    p.zface_lo = z_offset == 0;
    p.zface_hi = z_offset + p.nz == nz_global;
    // z closures (DIF_BOUND, NON_REFLETION) act at the faces of the whole
    // grid only, as the reference's npz == 0 / NPZ0-1 checks have them
    if (!p.zface_lo) { p.bnd_lo[2] = 0; p.nonref_lo[2] = 0; }
    if (!p.zface_hi) { p.bnd_hi[2] = 0; p.nonref_hi[2] = 0; }
    p.has_bnd = 0;
    for (int d = 0; d < 3; d++)
        p.has_bnd |= p.bnd_lo[d] | p.bnd_hi[d] | (p.nonref_lo[d] == 1) | (p.nonref_hi[d] == 1);
    return OCFD_OK;
}

extern "C" int ocfd_b200_set_slab(ocfd_b200_ctx *ctx, int nranks, int rank, int rank_lo, int rank_hi, int z_offset,
                                  int nz_global, const unsigned char id[OCFD_SLAB_ID_BYTES]) {
    if (!id) return OCFD_ERR_ARG;
    return set_slab_impl(ctx, nranks, rank, rank_lo, rank_hi, z_offset, nz_global, id, nullptr, nullptr);
}

// the same with the caller's host transport in place of NCCL
extern "C" int ocfd_b200_set_slab_host(ocfd_b200_ctx *ctx, int nranks, int rank, int rank_lo, int rank_hi,
                                       int z_offset, int nz_global, ocfd_b200_slab_transport fn, void *user) {
    if (!fn) return OCFD_ERR_ARG;
    return set_slab_impl(ctx, nranks, rank, rank_lo, rank_hi, z_offset, nz_global, nullptr, fn, user);
}

extern "C" int ocfd_b200_set_precision(ocfd_b200_ctx *ctx, int form) {
    if (!ctx || form < 0 || form > 1) return OCFD_ERR_ARG;
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    Params &p = ctx->p;
    if (form == 0) {
        if (!p.mixed) return OCFD_OK;
        if (int rc = refresh_prims64(ctx)) return rc;
        p.mixed = 0;
        CK(cudaStreamSynchronize(ctx->stream), "set_precision");
        return OCFD_OK;
    }
    if (p.mixed) return OCFD_OK;
    if (!ocfd::sweeps4_supported(p))
        return fail(ctx, OCFD_ERR_UNSUPPORTED, "the precision form covers the characteristic hybrid scheme and WENO7");
    if (!ctx->prec_buf) {
        const size_t n = 18 * (size_t)p.lapN + 5 * (size_t)p.N;
        cudaError_t e = cudaMalloc((void **)&ctx->prec_buf, n * sizeof(float));
        if (e != cudaSuccess) { ctx->prec_buf = nullptr; return cuda_fail(ctx, e, "precision-form buffers"); }
        CK(cudaMemsetAsync(ctx->prec_buf, 0, n * sizeof(float), ctx->stream), "memset");
    }
    for (int m = 0; m < 5; m++) p.prim32[m] = ctx->prec_buf + (size_t)m * p.lapN;
    p.ev32 = ctx->prec_buf + 5 * (size_t)p.lapN;
    p.pfil32 = ctx->prec_buf + 17 * (size_t)p.lapN;
    p.du32 = ctx->prec_buf + 18 * (size_t)p.lapN;
    ctx->tm32_ok = ocfd::march_tensor_map(p, ctx->prec_buf, 4, 1, &ctx->tm32[0]) &&
                   ocfd::march_tensor_map(p, ctx->prec_buf, 4, 2, &ctx->tm32[1]);
    p.mixed = 1;
    if (ctx->have_state) {
        CK(ocfd::launch_prims_to_fp32(p, ctx->stream), "FP32 primitives");
        ctx->launches += 1;
    }
    CK(cudaStreamSynchronize(ctx->stream), "set_precision");
    return OCFD_OK;
}

// ---------------------------------------------------------------------------
// learned scheme switch
// ---------------------------------------------------------------------------
extern "C" int ocfd_b200_mlp_nparam(void) { return ocfd::mlp_nparam(); }

extern "C" int ocfd_b200_set_switch(ocfd_b200_ctx *ctx, const float *params, int nparam, double confidence) {
    if (!ctx) return OCFD_ERR_ARG;
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    if (!params) { ctx->sw_on = false; return OCFD_OK; }
    if (nparam != ocfd::mlp_nparam() || !(confidence > 0.5 && confidence < 1.0))
        return fail(ctx, OCFD_ERR_ARG, "switch: parameter count or confidence (0.5, 1) wrong");
    for (int i = 0; i < 14; i++)
        if (!(params[14 + i] > 0.0f)) return fail(ctx, OCFD_ERR_ARG, "switch: feature scales must be > 0");
    if (!ctx->sw_w) {
        CK(cudaMalloc((void **)&ctx->sw_w, sizeof(float) * nparam), "switch parameters");
        CK(cudaMalloc((void **)&ctx->sw_stats, 4 * sizeof(unsigned long long)), "switch counters");
    }
    CK(cudaMemcpyAsync(ctx->sw_w, params, sizeof(float) * nparam, cudaMemcpyHostToDevice, ctx->stream),
       "switch parameters");
    CK(cudaMemsetAsync(ctx->sw_stats, 0, 4 * sizeof(unsigned long long), ctx->stream), "switch counters");
    CK(cudaStreamSynchronize(ctx->stream), "set_switch");
    ctx->sw_conf_logit = (float)log(confidence / (1.0 - confidence));
    ctx->sw_on = true;
    return OCFD_OK;
}

extern "C" int ocfd_b200_switch_stats(ocfd_b200_ctx *ctx, long long counts[3]) {
    if (!ctx || !counts) return OCFD_ERR_ARG;
    unsigned long long h[4] = {0, 0, 0, 0};
    if (ctx->sw_stats) {
        CK(cudaMemcpyAsync(h, ctx->sw_stats, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream), "switch counters");
        CK(cudaStreamSynchronize(ctx->stream), "switch counters");
    }
    for (int i = 0; i < 3; i++) counts[i] = (long long)h[i];
    return OCFD_OK;
}

extern "C" int ocfd_b200_switch_features(ocfd_b200_ctx *ctx, long long first, long long count, float *feat,
                                         float *label) {
    int rc = check_ready(ctx);
    if (rc) return rc;
    if (!feat || !label || first < 0 || count < 0 || first + count > ctx->p.N)
        return fail(ctx, OCFD_ERR_ARG, "switch_features: range outside the interior");
    if (count == 0) return OCFD_OK;
    if ((rc = refresh_prims64(ctx))) return rc;
    float *buf = nullptr;
    CK(cudaMalloc((void **)&buf, sizeof(float) * 15 * (size_t)count), "feature buffer");
    cudaError_t e = ocfd::launch_switch_features(ctx->p, first, count, buf, buf + 14 * (size_t)count, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(feat, buf, sizeof(float) * 14 * (size_t)count, cudaMemcpyDeviceToHost,
                                              ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(label, buf + 14 * (size_t)count, sizeof(float) * (size_t)count,
                                              cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(buf);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "switch_features");
    ctx->launches += 1;
    return OCFD_OK;
}

// stand-alone network entry points (no solver context; current device)
namespace {
struct DevBuf {
    void *p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
    cudaError_t alloc(size_t b) { return cudaMalloc(&p, b); }
    template <typename T> T *as() const { return static_cast<T *>(p); }
};
thread_local std::string g_mlp_err;
int mlp_fail(cudaError_t e, const char *where) {
    g_mlp_err = std::string(where) + ": " + cudaGetErrorString(e);
    return OCFD_ERR_CUDA;
}
#define MCK(call, where) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) return mlp_fail(e_, where); } while (0)
}  // namespace

extern "C" const char *ocfd_b200_mlp_last_error(void) { return g_mlp_err.c_str(); }

extern "C" int ocfd_b200_mlp_infer(const float *params, const float *feat, long long n, float *logit) {
    if (!params || !feat || !logit || n < 0) return OCFD_ERR_ARG;
    if (n == 0) return OCFD_OK;
    const int np = ocfd::mlp_nparam();
    DevBuf w, f, z, err;
    MCK(w.alloc(sizeof(float) * np), "alloc");
    MCK(f.alloc(sizeof(float) * 14 * (size_t)n), "alloc");
    MCK(z.alloc(sizeof(float) * (size_t)n), "alloc");
    MCK(err.alloc(sizeof(int)), "alloc");
    MCK(cudaMemset(err.p, 0, sizeof(int)), "memset");
    MCK(cudaMemcpy(w.p, params, sizeof(float) * np, cudaMemcpyHostToDevice), "copy");
    MCK(cudaMemcpy(f.p, feat, sizeof(float) * 14 * (size_t)n, cudaMemcpyHostToDevice), "copy");
    MCK(ocfd::launch_mlp_infer(w.as<float>(), f.as<float>(), n, z.as<float>(), err.as<int>(), 0), "mlp_infer");
    MCK(cudaMemcpy(logit, z.p, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost), "copy");
    int ew = 0;
    MCK(cudaMemcpy(&ew, err.p, sizeof(int), cudaMemcpyDeviceToHost), "copy");
    if (ew) {
        g_mlp_err = "mlp_infer: a tensor-core product did not complete within the wait limit";
        return OCFD_ERR_CUDA;
    }
    return OCFD_OK;
}

// gradient of the summed loss over rows 0..n-1 (network part of the
// parameter vector, from W1 on) and the summed loss
extern "C" int ocfd_b200_mlp_grad(const float *params, const float *feat, const float *label, long long n,
                                  float pos_w, float *grad, double *loss) {
    if (!params || !feat || !label || !grad || !loss || n <= 0) return OCFD_ERR_ARG;
    const int np = ocfd::mlp_nparam(), nn = ocfd::mlp_nnet(), nb = ocfd::mlp_grad_blocks(n);
    DevBuf w, f, y, part, lpart, g, l;
    MCK(w.alloc(sizeof(float) * np), "alloc");
    MCK(f.alloc(sizeof(float) * 14 * (size_t)n), "alloc");
    MCK(y.alloc(sizeof(float) * (size_t)n), "alloc");
    MCK(part.alloc(sizeof(float) * (size_t)nb * nn), "alloc");
    MCK(lpart.alloc(sizeof(float) * (size_t)nb), "alloc");
    MCK(g.alloc(sizeof(float) * nn), "alloc");
    MCK(l.alloc(sizeof(double)), "alloc");
    MCK(cudaMemcpy(w.p, params, sizeof(float) * np, cudaMemcpyHostToDevice), "copy");
    MCK(cudaMemcpy(f.p, feat, sizeof(float) * 14 * (size_t)n, cudaMemcpyHostToDevice), "copy");
    MCK(cudaMemcpy(y.p, label, sizeof(float) * (size_t)n, cudaMemcpyHostToDevice), "copy");
    MCK(cudaMemset(l.p, 0, sizeof(double)), "memset");
    MCK(ocfd::launch_mlp_grad(w.as<float>(), f.as<float>(), y.as<float>(), nullptr, n, pos_w, part.as<float>(),
                              lpart.as<float>(), g.as<float>(), l.as<double>(), 0), "mlp_grad");
    MCK(cudaMemcpy(grad, g.p, sizeof(float) * nn, cudaMemcpyDeviceToHost), "copy");
    MCK(cudaMemcpy(loss, l.p, sizeof(double), cudaMemcpyDeviceToHost), "copy");
    return OCFD_OK;
}

// Adam over shuffled mini-batches of mean loss; params (in/out) is the
// full parameter vector (mu and sigma are kept); epoch_loss[e] = mean loss
// of epoch e
extern "C" int ocfd_b200_mlp_train(float *params, const float *feat, const float *label, long long n, int epochs,
                                   int batch, float lr, float pos_w, unsigned long long seed, double *epoch_loss) {
    if (!params || !feat || !label || n <= 0 || epochs < 0 || batch <= 0 || n > 0x7fffffffLL) return OCFD_ERR_ARG;
    const int np = ocfd::mlp_nparam(), nn = ocfd::mlp_nnet(), nbmax = ocfd::mlp_grad_blocks(batch);
    DevBuf w, f, y, part, lpart, g, l, m1, m2, perm;
    MCK(w.alloc(sizeof(float) * np), "alloc");
    MCK(f.alloc(sizeof(float) * 14 * (size_t)n), "alloc");
    MCK(y.alloc(sizeof(float) * (size_t)n), "alloc");
    MCK(part.alloc(sizeof(float) * (size_t)nbmax * nn), "alloc");
    MCK(lpart.alloc(sizeof(float) * (size_t)nbmax), "alloc");
    MCK(g.alloc(sizeof(float) * nn), "alloc");
    MCK(l.alloc(sizeof(double)), "alloc");
    MCK(m1.alloc(sizeof(float) * nn), "alloc");
    MCK(m2.alloc(sizeof(float) * nn), "alloc");
    MCK(perm.alloc(sizeof(int) * (size_t)n), "alloc");
    MCK(cudaMemcpy(w.p, params, sizeof(float) * np, cudaMemcpyHostToDevice), "copy");
    MCK(cudaMemcpy(f.p, feat, sizeof(float) * 14 * (size_t)n, cudaMemcpyHostToDevice), "copy");
    MCK(cudaMemcpy(y.p, label, sizeof(float) * (size_t)n, cudaMemcpyHostToDevice), "copy");
    MCK(cudaMemset(m1.p, 0, sizeof(float) * nn), "memset");
    MCK(cudaMemset(m2.p, 0, sizeof(float) * nn), "memset");
    std::vector<int> order((size_t)n);
    for (long long i = 0; i < n; i++) order[(size_t)i] = (int)i;
    unsigned long long state = seed ? seed : 0x9E3779B97F4A7C15ULL;
    auto next = [&state]() {           // splitmix64
        unsigned long long z = (state += 0x9E3779B97F4A7C15ULL);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        return z ^ (z >> 31);
    };
    int t = 0;
    for (int ep = 0; ep < epochs; ep++) {
        for (long long i = n - 1; i > 0; i--) std::swap(order[(size_t)i], order[(size_t)(next() % (unsigned long long)(i + 1))]);
        MCK(cudaMemcpy(perm.p, order.data(), sizeof(int) * (size_t)n, cudaMemcpyHostToDevice), "copy");
        MCK(cudaMemset(l.p, 0, sizeof(double)), "memset");
        for (long long b0 = 0; b0 < n; b0 += batch) {
            const long long nb = std::min<long long>(batch, n - b0);
            MCK(ocfd::launch_mlp_grad(w.as<float>(), f.as<float>(), y.as<float>(), perm.as<int>() + b0, nb, pos_w,
                                      part.as<float>(), lpart.as<float>(), g.as<float>(), l.as<double>(), 0),
                "mlp_grad");
            MCK(ocfd::launch_mlp_adam(w.as<float>(), g.as<float>(), m1.as<float>(), m2.as<float>(),
                                      1.0f / (float)nb, lr, ++t, 0), "mlp_adam");
        }
        double ls = 0.0;
        MCK(cudaMemcpy(&ls, l.p, sizeof(double), cudaMemcpyDeviceToHost), "copy");
        if (epoch_loss) epoch_loss[ep] = ls / (double)n;
    }
    MCK(cudaMemcpy(params, w.p, sizeof(float) * np, cudaMemcpyDeviceToHost), "copy");
    return OCFD_OK;
}

extern "C" int ocfd_b200_sweep_walks(const ocfd_b200_ctx *ctx) {
    if (!ctx) return OCFD_ERR_ARG;
    const Params &p = ctx->p;
    if (p.sweep_impl == 6) return 7;
    if (p.sweep_impl != 4 || !ocfd::sweeps4_supported(p)) return 0;
    if (p.scheme_invis != 310) return 7;
    return ctx->walk4[0] | (ctx->walk4[1] << 1) | (ctx->walk4[2] << 2);
}

extern "C" int ocfd_b200_set_viscous_impl(ocfd_b200_ctx *ctx, int impl) {
    if (!ctx || impl < 0 || impl > 2) return OCFD_ERR_ARG;
    ctx->p.vis_impl = ctx->vdiv_ok ? impl : 1;
    return OCFD_OK;
}

extern "C" int ocfd_b200_set_walk_threshold(ocfd_b200_ctx *ctx, double frac) {
    if (!ctx || !(frac >= 0.0)) return OCFD_ERR_ARG;
    ctx->walk4_threshold = frac;
    return OCFD_OK;
}

extern "C" int ocfd_b200_set_sweep_impl(ocfd_b200_ctx *ctx, int impl) {
    if (!ctx || impl < 4 || impl > 8) return OCFD_ERR_ARG;
    ctx->march = impl == 7 ? 0 : (impl == 8 ? 2 : 1);
    ctx->p.sweep_impl = impl >= 7 ? 4 : impl;
    return OCFD_OK;
}

extern "C" int ocfd_b200_set_metrics(ocfd_b200_ctx *ctx, const double *m) {
    return set_metrics_impl(ctx, m, cudaMemcpyHostToDevice);
}
extern "C" int ocfd_b200_set_metrics_device(ocfd_b200_ctx *ctx, const double *m) {
    return set_metrics_impl(ctx, m, cudaMemcpyDeviceToDevice);
}

// The OCFD3d-Mesh.dat branch of Init_Jacobian3d (src/OCFD_Comput_Jacobian3d.cu:119-141)
// followed by Comput_Jacobian3d (:221-246) and ana_Jac (src/OCFD_ana.cu:24-48).
static int set_mesh_impl(ocfd_b200_ctx *ctx, const double *src, cudaMemcpyKind kind) {
    if (!ctx || !src) return OCFD_ERR_ARG;
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    Params &p = ctx->p;
    size_t inB = sizeof(double) * (size_t)p.N;
    CK(ocfd::launch_fill(ctx->met_buf, 13 * p.lapN, 1.0, ctx->stream), "metric init");
    ctx->launches += 1;
    for (int m = 0; m < 3; m++) {
        CK(cudaMemcpyAsync(ctx->stage_buf, src + (size_t)m * p.N, inB, kind, ctx->stream), "mesh copy");
        CK(ocfd::launch_scatter(p, ctx->stage_buf, const_cast<double *>(p.met[m]), ctx->stream), "mesh scatter");
        ctx->launches += 1;
    }
    {   // periodic exchange of the coordinates
        double *f[3]; int mask[3];
        for (int m = 0; m < 3; m++) { f[m] = const_cast<double *>(p.met[m]); mask[m] = 7; }
        int rc = fill_ghosts(ctx, f, mask, 3, "mesh ghost fill");
        if (rc) return rc;
    }
    // the Ev scratch (12 LAP fields) holds the nine coordinate derivatives
    CK(ocfd::launch_mesh_metrics(p, ctx->cfg.jac_bound, ctx->ev_buf, ctx->stream), "metrics from mesh");
    ctx->launches += 10;
    {   // periodic exchange of the ten computed fields
        double *f[10]; int mask[10];
        for (int m = 0; m < 10; m++) { f[m] = const_cast<double *>(p.met[ocfd::M_AKX + m]); mask[m] = 7; }
        int rc = fill_ghosts(ctx, f, mask, 10, "metric ghost fill");
        if (rc) return rc;
    }
    unsigned *flag = reinterpret_cast<unsigned *>(ctx->red_buf);
    CK(ocfd::launch_negative_jacobian(p, flag, ctx->stream), "Jacobian check");
    ctx->launches += 1;
    unsigned neg = 0;
    CK(cudaMemcpyAsync(&neg, flag, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream), "Jacobian check");
    CK(cudaStreamSynchronize(ctx->stream), "set_mesh");
    if (neg) return fail(ctx, OCFD_ERR_ARG, "negative Jacobian computed from the mesh (the reference stops here)");
    p.uniform_metrics = 0;          // metrics vary; kernels read the fields
    ctx->have_metrics = true;
    return OCFD_OK;
}

// the 13 metric fields as the kernels read them (interior), e.g. to write
// OCFD3d-Jacobi.dat after a mesh was given
extern "C" int ocfd_b200_get_metrics(ocfd_b200_ctx *ctx, double *metrics13) {
    int rc = check_ready(ctx);
    if (rc) return rc;
    if (!metrics13) return OCFD_ERR_ARG;
    const Params &p = ctx->p;
    size_t inB = sizeof(double) * (size_t)p.N;
    for (int m = 0; m < 13; m++) {
        CK(ocfd::launch_gather(p, p.met[m], ctx->stage_buf, ctx->stream), "metric gather");
        ctx->launches += 1;
        CK(cudaMemcpyAsync(metrics13 + (size_t)m * p.N, ctx->stage_buf, inB, cudaMemcpyDeviceToHost, ctx->stream),
           "metric read-back");
    }
    CK(cudaStreamSynchronize(ctx->stream), "get_metrics");
    return OCFD_OK;
}

extern "C" int ocfd_b200_set_mesh(ocfd_b200_ctx *ctx, const double *xyz3) {
    return set_mesh_impl(ctx, xyz3, cudaMemcpyHostToDevice);
}
extern "C" int ocfd_b200_set_mesh_device(ocfd_b200_ctx *ctx, const double *xyz3_dev) {
    return set_mesh_impl(ctx, xyz3_dev, cudaMemcpyDeviceToDevice);
}

static int upload_prims(ocfd_b200_ctx *ctx, const double *src, cudaMemcpyKind kind) {
    const Params &p = ctx->p;
    size_t inB = sizeof(double) * (size_t)p.N;
    CK(cudaMemcpyAsync(ctx->stage_buf, src, 5 * inB, kind, ctx->stream), "primitive copy");
    for (int m = 0; m < 5; m++) {
        CK(ocfd::launch_scatter(p, ctx->stage_buf + (size_t)m * p.N, p.prim[m], ctx->stream), "scatter");
        ctx->launches += 1;
    }
    return OCFD_OK;
}

static int set_prims_impl(ocfd_b200_ctx *ctx, const double *src, cudaMemcpyKind kind, int istep, double tt) {
    if (!ctx || !src) return OCFD_ERR_ARG;
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    const Params &p = ctx->p;
    // init(): ghosts of d,u,v,w,T zero (src/OCFD_init.cu:37-41), f/fn/du zero
    CK(cudaMemsetAsync(ctx->prim_buf, 0, 5 * sizeof(double) * (size_t)p.lapN, ctx->stream), "memset");
    CK(cudaMemsetAsync(ctx->cons_buf, 0, 15 * sizeof(double) * (size_t)p.N, ctx->stream), "memset");
    int rc = upload_prims(ctx, src, kind);
    if (rc) return rc;
    CK(ocfd::launch_p2c(p, p.f, ctx->stream), "pri_to_cons");
    ctx->launches += 1;
    // NS_solver_real pre-loop: exchange, OCFD_bc (the boundary family's
    // values, then the faces of f re-projected: without a family no change),
    // get_Amu (formed on the fly)
    rc = ghost_prims64(ctx);
    if (rc) return rc;
    ctx->tt = tt;
    if (p.ibc) {
        if ((rc = apply_bc(ctx))) return rc;
        CK(ocfd::launch_bc_faces(p, ctx->stream), "face re-projection");
        ctx->launches += 1;
    }
    if (p.mixed) {
        CK(ocfd::launch_prims_to_fp32(p, ctx->stream), "FP32 primitives");
        ctx->launches += 1;
    }
    ctx->prims64_stale = false;
    CK(cudaStreamSynchronize(ctx->stream), "set_primitives");
    ctx->istep = istep;
    ctx->tt = tt;
    ctx->have_state = true;
    return OCFD_OK;
}

extern "C" int ocfd_b200_set_primitives(ocfd_b200_ctx *ctx, const double *prim5, int istep, double tt) {
    return set_prims_impl(ctx, prim5, cudaMemcpyHostToDevice, istep, tt);
}
extern "C" int ocfd_b200_set_primitives_device(ocfd_b200_ctx *ctx, const double *prim5, int istep, double tt) {
    return set_prims_impl(ctx, prim5, cudaMemcpyDeviceToDevice, istep, tt);
}

// ---------------------------------------------------------------------------
// time stepping
// ---------------------------------------------------------------------------

extern "C" int ocfd_b200_swap_time_levels(ocfd_b200_ctx *ctx) {
    if (!ctx) return OCFD_ERR_ARG;
    double *t = ctx->p.f; ctx->p.f = ctx->p.fn; ctx->p.fn = t;
    return OCFD_OK;
}

// filtering() (src/OCFD_filtering.cu:75-183) at the context's Istep and tt
static int run_filters(ocfd_b200_ctx *ctx) {
    if (!ctx->nfilter) return OCFD_OK;
    bool any = false;
    for (int m = 0; m < ctx->nfilter; m++)
        if (ctx->istep % ctx->fpar[m][0] == 0) any = true;
    if (!any) return OCFD_OK;
    const Params &p = ctx->p;
    {   // periodic exchange of p and pf_lap in the directions any filter uses
        double *f[6]; int mask[6];
        const int dm = (ctx->fjudge[0] ? 1 : 0) | (ctx->fjudge[1] ? 2 : 0) | (ctx->fjudge[2] ? 4 : 0);
        int n = 0;
        if (!p.mixed) { f[n] = p.pfil; mask[n++] = dm; }
        for (int m = 0; m < 5; m++) { f[n] = p.flap + (size_t)m * p.lapN; mask[n++] = dm; }
        int rc = fill_ghosts(ctx, f, mask, n, "filter ghost fill");
        if (rc) return rc;
        if (p.mixed) {      // the precision form's FP32 pressure
            float *f32[1] = { p.pfil32 };
            if ((rc = fill_ghosts(ctx, f32, mask, 1, "filter ghost fill"))) return rc;
        }
    }
    for (int m = 0; m < ctx->nfilter; m++) {
        if (!(ctx->tt <= ctx->frpar[m][2]) || ctx->istep % ctx->fpar[m][0] != 0) continue;
        const double s0 = ctx->frpar[m][0], rth = ctx->frpar[m][1];
        int box[6];
        for (int t = 0; t < 6; t++) box[t] = ctx->fpar[m][4 + t];
        if (ctx->fpar[m][1] == 1) { CK(ocfd::launch_filter_pass(p, 0, box, s0, rth, ctx->stream), "filter x"); ctx->launches += 1; }
        if (ctx->fpar[m][2] == 1) { CK(ocfd::launch_filter_pass(p, 1, box, s0, rth, ctx->stream), "filter y"); ctx->launches += 1; }
        if (ctx->fpar[m][3] == 1) {
            // filter_z3d_shock launches the y kernel on an (8, 8, 4+2) block:
            // it filters along y, and its y rows reach only jb + 6*ceil((je-jb)/8)
            int zb[6];
            for (int t = 0; t < 6; t++) zb[t] = box[t];
            const int gy = (box[3] - box[2] + 7) / 8;
            if (zb[3] > box[2] + 6 * gy + 1) zb[3] = box[2] + 6 * gy + 1;
            CK(ocfd::launch_filter_pass(p, 1, zb, s0, rth, ctx->stream), "filter z");
            ctx->launches += 1;
        }
    }
    return OCFD_OK;
}

// A step runs from a CUDA graph unless something in it goes to the host: no
// kernel timing, no boundary-condition family (its wall law takes the time
// of each stage), no slab exchange.  The hybrid scheme's flag-count
// read-back comes before the graph; the filters run after the step.
static bool step_graph_ok(const ocfd_b200_ctx *ctx) {
    return ctx->graphs_on && !ctx->timing && !ctx->p.ibc && !ctx->slab;
}

// the three stages of one step, time levels already swapped (skip_sensor:
// the first stage's sensor pass has run)
static int step_launched(ocfd_b200_ctx *ctx, bool skip_sensor) {
    for (int krk = 1; krk <= 3; krk++) {
        int rc = rhs(ctx, krk, krk, skip_sensor);
        if (rc) return rc;
    }
    return OCFD_OK;
}

// The same from the graph of this parity, captured first if it is missing or
// stale.  With the hybrid scheme's per-step read-back the sensor pass runs
// first, outside the graph, and the graph holds the rest of the step for the
// walks that pass chose.
static int step_graph(ocfd_b200_ctx *ctx) {
    const bool skip = needs_readback(ctx);
    if (skip) {
        int rc = rhs_sensor(ctx);
        if (rc) return rc;
    }
    // a stream that the caller is capturing already takes the launches into
    // the caller's graph
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(ctx->stream, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
        cudaGetLastError();
        return step_launched(ctx, skip);
    }
    const int walk = skip ? ctx->walk4[0] | ctx->walk4[1] << 1 | ctx->walk4[2] << 2 : -1;
    auto &G = ctx->graph[ctx->p.f == ctx->cons_buf ? 0 : 1];
    const bool fresh = G.exec && G.stream == ctx->stream && G.sw_on == ctx->sw_on && G.walk == walk &&
                       G.march == ctx->march && G.sw_conf == ctx->sw_conf_logit && memcmp(&G.key, &ctx->p, sizeof(Params)) == 0;
    if (fresh) {
        CK(cudaGraphLaunch(G.exec, ctx->stream), "step graph");
        ctx->launches += G.launches;
        return OCFD_OK;
    }
    if (G.exec) { cudaGraphExecDestroy(G.exec); G.exec = nullptr; }
    if (cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        // a stream that cannot be captured (the legacy default stream):
        // launch one by one from now on
        cudaGetLastError();
        ctx->graphs_on = false;
        return step_launched(ctx, skip);
    }
    const long long l0 = ctx->launches;
    ctx->graph_captures += 1;
    int rc = OCFD_OK;
    for (int krk = 1; krk <= 3 && !rc; krk++) rc = rhs(ctx, krk, krk, skip);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
    if (rc || e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        if (rc) return rc;
        return cuda_fail(ctx, e, "step graph capture");
    }
    e = cudaGraphInstantiate(&G.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) { G.exec = nullptr; return cuda_fail(ctx, e, "step graph instantiate"); }
    memcpy(&G.key, &ctx->p, sizeof(Params));
    G.stream = ctx->stream;
    G.march = ctx->march;
    G.sw_on = ctx->sw_on;
    G.sw_conf = ctx->sw_conf_logit;
    G.walk = walk;
    G.launches = ctx->launches - l0;
    CK(cudaGraphLaunch(G.exec, ctx->stream), "step graph");
    return OCFD_OK;
}

extern "C" int ocfd_b200_set_graphs(ocfd_b200_ctx *ctx, int enabled) {
    if (!ctx) return OCFD_ERR_ARG;
    ctx->graphs_on = enabled != 0;
    return OCFD_OK;
}
extern "C" long long ocfd_b200_graph_captures(const ocfd_b200_ctx *ctx) { return ctx ? ctx->graph_captures : 0; }

extern "C" int ocfd_b200_step(ocfd_b200_ctx *ctx, int nsteps) {
    int rc = check_ready(ctx);
    if (rc) return rc;
    if (nsteps < 0) return fail(ctx, OCFD_ERR_ARG, "nsteps < 0");
    if (ctx->p.mixed && nsteps > 0) {
        ctx->prims64_stale = true;
        ctx->prims64_interior_ok = ctx->p.flap != nullptr;
    }
    for (int n = 0; n < nsteps; n++) {
        nvtxRangePushA("ocfd_b200_step");
        ocfd_b200_swap_time_levels(ctx);
        rc = step_graph_ok(ctx) ? step_graph(ctx) : step_launched(ctx, false);
        if (!rc) {
            ctx->istep++;
            ctx->tt += ctx->p.dt;
            rc = run_filters(ctx);
        }
        nvtxRangePop();
        if (rc) return rc;
    }
    return OCFD_OK;
}

extern "C" int ocfd_b200_filtering(ocfd_b200_ctx *ctx) {
    int rc = check_ready(ctx);
    if (rc) return rc;
    return run_filters(ctx);
}

extern "C" int ocfd_b200_set_time(ocfd_b200_ctx *ctx, int istep, double tt) {
    if (!ctx) return OCFD_ERR_ARG;
    ctx->istep = istep;
    ctx->tt = tt;
    return OCFD_OK;
}

// The first n values of the C library's rand() in its initial state (as
// after srand(1)): the additive generator r[i] = r[i-3] + r[i-31] mod 2^32
// over a table filled by r[i] = 16807 r[i-1] mod (2^31 - 1) from r[0] = 1,
// r[31..33] = r[0..2], the values up to r[343] discarded, each output
// r[i] >> 1 (the published description of the GNU C library's TYPE_3
// random()).
static std::vector<int> libc_rand_initial(int n) {
    std::vector<unsigned> r((size_t)344 + n);
    r[0] = 1u;
    for (int i = 1; i < 31; i++) {
        long long w = (16807LL * (long long)r[i - 1]) % 2147483647LL;
        if (w < 0) w += 2147483647LL;
        r[i] = (unsigned)w;
    }
    for (int i = 31; i < 34; i++) r[i] = r[i - 31];
    std::vector<int> out((size_t)n);
    for (int i = 34; i < 344 + n; i++) {
        r[i] = r[i - 31] + r[i - 3];
        if (i >= 344) out[i - 344] = (int)(r[i] >> 1);
    }
    return out;
}

// IBC and BC_NPARA / BC_RPARA (bc_parameter, src/OCFD_boundary_init.c:50-93)
// with the set-up of bc_user_Compression_conner_init (:376-438)
extern "C" int ocfd_b200_set_bc(ocfd_b200_ctx *ctx, int ibc, const int *npara, int nnpara, const double *rpara,
                                int nrpara, const double *inlet4) {
    if (!ctx) return OCFD_ERR_ARG;
    Params &p = ctx->p;
    if (ibc == 0) { p.ibc = 0; return OCFD_OK; }
    if (ibc != 108)
        return fail(ctx, OCFD_ERR_UNSUPPORTED, "IBC " + std::to_string(ibc) + " is not built (0 or 108)");
    if (!npara || !rpara || nnpara < 4 || nrpara < 8)
        return fail(ctx, OCFD_ERR_ARG, "IBC 108 needs 4 BC_NPARA and 8 BC_RPARA values");
    if (!ctx->have_metrics) return fail(ctx, OCFD_ERR_STATE, "set the metrics or mesh before the boundary conditions");
    const int MZ = npara[0], MT = npara[1], inlet_file = npara[2], not_normal = npara[3];
    if (MZ > 4096) return fail(ctx, OCFD_ERR_ARG, "MZMAX must be <= 4096");
    if (MT > 64) return fail(ctx, OCFD_ERR_ARG, "MTMAX must be <= 64");
    if (inlet_file == 1 && !inlet4) return fail(ctx, OCFD_ERR_ARG, "INLET_BOUNDARY = 1 needs the inflow profile");
    const double TW = rpara[0], EPSL = rpara[1], DB = rpara[2], DE = rpara[3], BETA = rpara[4];
    const double XUP = rpara[6], SL = rpara[7];
    const double PI = 3.14159265358979323846;
    // wall and top coordinates from the x and z metric records
    const size_t inB = sizeof(double) * (size_t)p.N;
    std::string err;
    double *hx = (double *)malloc(inB), *hz = (double *)malloc(inB);
    if (!hx || !hz) { free(hx); free(hz); return fail(ctx, OCFD_ERR_NOMEM, "host buffers for the boundary set-up"); }
    cudaError_t e = ocfd::launch_gather(p, p.met[0], ctx->stage_buf, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hx, ctx->stage_buf, inB, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = ocfd::launch_gather(p, p.met[2], ctx->stage_buf, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hz, ctx->stage_buf, inB, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) { free(hx); free(hz); return cuda_fail(ctx, e, "boundary set-up read-back"); }
    const int nx = p.nx, ny = p.ny, nz = p.nz;
    std::vector<double> host((size_t)4 * ny + nx + nz);
    double *ub1 = host.data(), *fx = ub1 + 4 * ny, *gz = fx + nx;
    for (int j = 0; j < ny; j++) {
        if (inlet_file == 1) for (int c = 0; c < 4; c++) ub1[c * ny + j] = inlet4[c * ny + j];
        else { ub1[j] = 1.; ub1[ny + j] = 1.; ub1[2 * ny + j] = 0.; ub1[3 * ny + j] = 1.; }
    }
    int x_begin = 0;
    for (int i = 0; i < nx; i++) {
        if (hx[i + (size_t)nx * (ny - 1)] <= XUP) x_begin = i;         // top row, first z plane
        const double xa = hx[i];                                        // wall row, first z plane
        if (xa >= DB && xa <= DE) {
            const double seta = 10. * PI * (xa - DB) / (DB - DE);
            fx[i] = 4. / sqrt(27.) * sin(seta) * (1. - cos(seta));
        } else {
            fx[i] = 0.;
        }
    }
    // MZMAX > 0: MZMAX spanwise modes of weights 1, 1/1.25, ... (normalised)
    // and phases rand() / RAND_MAX, the first draws of the C library's
    // generator in its initial state -- the reference seeds nothing before
    // (get_xs_blow_suction_multiwave, src/OCFD_boundary_init.c:444-499)
    std::vector<double> faiz, zl;
    if (MZ > 0) {
        std::vector<int> draws = libc_rand_initial(MZ);
        faiz.resize(MZ);
        zl.resize(MZ);
        double ztmp = 0.;
        for (int m = 0; m < MZ; m++) {
            faiz[m] = draws[m] / 2147483647.0;
            zl[m] = m == 0 ? 1. : zl[m - 1] / 1.25;
            ztmp = ztmp + zl[m];
        }
        for (int m = 0; m < MZ; m++) zl[m] = zl[m] / ztmp;
    }
    for (int k = 0; k < nz; k++) {
        const double za = hz[(size_t)nx * ny * k];                      // x = 0, y = 0
        const double seta = za / SL;
        if (MZ > 0) {
            gz[k] = 0.;
            for (int m = 0; m < MZ; m++) gz[k] = gz[k] + zl[m] * sin(2. * PI * (m + 1) * (seta + faiz[m]));
        } else {
            gz[k] = MZ == 0 ? 1. : sin(-2. * PI * MZ * seta);
        }
    }
    free(hx); free(hz);
    double Ttmp = 0.;
    for (int k = 0; k < MT; k++) {
        ctx->bc_TM[0] = 1.;
        if (k > 0) ctx->bc_TM[k] = ctx->bc_TM[k - 1] / 1.25;
        Ttmp = Ttmp + ctx->bc_TM[k];
    }
    for (int k = 0; k < MT; k++) ctx->bc_TM[k] = ctx->bc_TM[k] / Ttmp;
    if (!ctx->bc_buf) {
        e = cudaMalloc(&ctx->bc_buf, sizeof(double) * host.size());
        if (e != cudaSuccess) { cudaGetLastError(); return fail(ctx, OCFD_ERR_NOMEM, "boundary arrays"); }
    }
    CK(cudaMemcpyAsync(ctx->bc_buf, host.data(), sizeof(double) * host.size(), cudaMemcpyHostToDevice, ctx->stream),
       "boundary arrays");
    CK(cudaStreamSynchronize(ctx->stream), "set_bc");
    p.bc_ub1 = ctx->bc_buf; p.bc_fx = ctx->bc_buf + 4 * ny; p.bc_gz = p.bc_fx + nx;
    p.bc_xbegin = x_begin;
    p.bc_wall_mode = not_normal != 0 ? 0 : (TW > 0 ? 1 : 2);
    p.bc_tw = TW; p.bc_epsl = EPSL;
    ctx->bc_beta = BETA; ctx->bc_mtmax = MT;
    p.ibc = 108;
    return OCFD_OK;
}

// FILTER_NPARA<n+1> / FILTER_RPARA<n+1>, clamped as set_para_filtering does
// on one rank (src/OCFD_filtering.cu:20-73)
extern "C" int ocfd_b200_set_filter(ocfd_b200_ctx *ctx, int n, const int npara[11], const double rpara[3]) {
    if (!ctx || !npara || !rpara) return OCFD_ERR_ARG;
    if (n < 0 || n >= 8) return fail(ctx, OCFD_ERR_ARG, "filter index must be 0..7");
    if (npara[0] < 1) return fail(ctx, OCFD_ERR_ARG, "filter step interval must be >= 1");
    if (npara[10] != 2)
        return fail(ctx, OCFD_ERR_UNSUPPORTED, "only the shock-capturing filter (scheme 2) is built; "
                                                "the reference's 9-point filter aborts");
    Params &p = ctx->p;
    if (!ctx->filter_buf) {
        cudaError_t e = cudaMalloc(&ctx->filter_buf, sizeof(double) * 6 * (size_t)p.lapN);
        if (e != cudaSuccess) { cudaGetLastError(); return fail(ctx, OCFD_ERR_NOMEM, "filter buffers"); }
        CK(cudaMemsetAsync(ctx->filter_buf, 0, sizeof(double) * 6 * (size_t)p.lapN, ctx->stream), "filter init");
        p.flap = ctx->filter_buf;
        p.pfil = ctx->filter_buf + 5 * (size_t)p.lapN;
    }
    const int nn[3] = { p.nx, p.ny, p.nz };
    int kb = npara[8], ke = npara[9];
    if (ctx->slab) {
        // set_para_filtering (src/OCFD_filtering.cu:56-61) on this slab:
        // k ranges are global; a slab that holds none of the range would
        // filter rows of another slab's local numbering there, so such a
        // range is refused
        const int k0 = ctx->z_offset, k1 = ctx->z_offset + p.nz;
        if (kb >= k1 || ke <= k0)
            return fail(ctx, OCFD_ERR_UNSUPPORTED, "with the grid split in z, a filter's k range must reach every slab");
        kb = kb < k0 ? 0 : kb - k0;
        ke = ke >= k1 ? p.nz : ke - k0;
    }
    for (int t = 0; t < 11; t++) ctx->fpar[n][t] = npara[t];
    ctx->fpar[n][8] = kb;
    ctx->fpar[n][9] = ke;
    for (int d = 0; d < 3; d++) {
        if (npara[1 + d] == 1) ctx->fjudge[d] = 1;
        if (!p.periodic[d]) {
            if (ctx->fpar[n][4 + 2 * d] < 6) ctx->fpar[n][4 + 2 * d] = 6;
            if (ctx->fpar[n][5 + 2 * d] > nn[d] - 5) ctx->fpar[n][5 + 2 * d] = nn[d] - 5;
        }
        // a range past the grid (e.g. 0 .. 100000 for "everything") ends at
        // the grid, so no pass reaches beyond the fields
        if (ctx->fpar[n][4 + 2 * d] < 0) ctx->fpar[n][4 + 2 * d] = 0;
        if (ctx->fpar[n][5 + 2 * d] > nn[d]) ctx->fpar[n][5 + 2 * d] = nn[d];
    }
    for (int t = 0; t < 3; t++) ctx->frpar[n][t] = rpara[t];
    if (n + 1 > ctx->nfilter) ctx->nfilter = n + 1;
    return OCFD_OK;
}

extern "C" int ocfd_b200_du_comput(ocfd_b200_ctx *ctx, int krk) {
    int rc = check_ready(ctx);
    if (rc) return rc;
    if (ctx->p.mixed) return fail(ctx, OCFD_ERR_UNSUPPORTED, "the precision form runs whole steps only");
    if (krk < 1 || krk > 3) return fail(ctx, OCFD_ERR_ARG, "KRK must be 1..3");
    return rhs(ctx, krk, 0);
}

extern "C" int ocfd_b200_time_advance(ocfd_b200_ctx *ctx, int krk) {
    int rc = check_ready(ctx);
    if (rc) return rc;
    if (ctx->p.mixed) return fail(ctx, OCFD_ERR_UNSUPPORTED, "the precision form runs whole steps only");
    if (krk < 1 || krk > 3) return fail(ctx, OCFD_ERR_ARG, "KRK must be 1..3");
    CK(ocfd::launch_rk_only(ctx->p, krk, ctx->stream), "time advance");
    ctx->launches += 1;
    return OCFD_OK;
}

extern "C" int ocfd_b200_get_duvwT(ocfd_b200_ctx *ctx) {
    int rc = check_ready(ctx);
    if (rc) return rc;
    if (ctx->p.mixed) return fail(ctx, OCFD_ERR_UNSUPPORTED, "the precision form runs whole steps only");
    CK(ocfd::launch_c2p(ctx->p, ctx->stream), "cons_to_pri");
    ctx->launches += 1;
    return OCFD_OK;
}

extern "C" int ocfd_b200_bc(ocfd_b200_ctx *ctx) {
    int rc = check_ready(ctx);
    if (rc) return rc;
    if (ctx->p.mixed) return fail(ctx, OCFD_ERR_UNSUPPORTED, "the precision form runs whole steps only");
    if ((rc = apply_bc(ctx))) return rc;
    CK(ocfd::launch_bc_faces(ctx->p, ctx->stream), "face re-projection");
    ctx->launches += 1;
    return OCFD_OK;
}

// ---------------------------------------------------------------------------
// read-back
// ---------------------------------------------------------------------------

extern "C" int ocfd_b200_get_primitives_device(ocfd_b200_ctx *ctx, double *out) {
    if (!ctx || !out) return OCFD_ERR_ARG;
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    if (int rc = refresh_prims64(ctx)) return rc;
    for (int m = 0; m < 5; m++) {
        CK(ocfd::launch_gather(ctx->p, ctx->p.prim[m], out + (size_t)m * ctx->p.N, ctx->stream), "gather");
        ctx->launches += 1;
    }
    CK(cudaStreamSynchronize(ctx->stream), "get_primitives");
    return OCFD_OK;
}

extern "C" int ocfd_b200_get_primitives(ocfd_b200_ctx *ctx, double *out) {
    if (!ctx || !out) return OCFD_ERR_ARG;
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    if (int rc = refresh_prims64(ctx)) return rc;
    for (int m = 0; m < 5; m++) {
        CK(ocfd::launch_gather(ctx->p, ctx->p.prim[m], ctx->stage_buf + (size_t)m * ctx->p.N, ctx->stream), "gather");
        ctx->launches += 1;
    }
    CK(cudaMemcpyAsync(out, ctx->stage_buf, 5 * sizeof(double) * (size_t)ctx->p.N, cudaMemcpyDeviceToHost,
                       ctx->stream), "primitive copy");
    CK(cudaStreamSynchronize(ctx->stream), "get_primitives");
    return OCFD_OK;
}

static int get_interior5(ocfd_b200_ctx *ctx, const double *src, double *out, const char *what) {
    if (!ctx || !out) return OCFD_ERR_ARG;
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    CK(cudaMemcpyAsync(out, src, 5 * sizeof(double) * (size_t)ctx->p.N, cudaMemcpyDeviceToHost, ctx->stream), what);
    CK(cudaStreamSynchronize(ctx->stream), what);
    return OCFD_OK;
}

extern "C" int ocfd_b200_get_conserved(ocfd_b200_ctx *ctx, double *out) {
    return ctx ? get_interior5(ctx, ctx->p.f, out, "get_conserved") : OCFD_ERR_ARG;
}
extern "C" int ocfd_b200_get_du(ocfd_b200_ctx *ctx, double *out) {
    if (ctx && ctx->p.mixed) return fail(ctx, OCFD_ERR_UNSUPPORTED, "the precision form keeps du in FP32");
    return ctx ? get_interior5(ctx, ctx->p.du, out, "get_du") : OCFD_ERR_ARG;
}

extern "C" int ocfd_b200_get_flags(ocfd_b200_ctx *ctx, int8_t *fx, int8_t *fy, int8_t *fz) {
    if (!ctx || !fx || !fy || !fz) return OCFD_ERR_ARG;
    const Params &p = ctx->p;
    size_t nxf = (size_t)(p.nx + 1) * p.ny * p.nz, nyf = (size_t)p.nx * (p.ny + 1) * p.nz,
           nzf = (size_t)p.nx * p.ny * (p.nz + 1);
    CK(cudaMemcpyAsync(fx, p.flag[0], nxf, cudaMemcpyDeviceToHost, ctx->stream), "flags");
    CK(cudaMemcpyAsync(fy, p.flag[1], nyf, cudaMemcpyDeviceToHost, ctx->stream), "flags");
    CK(cudaMemcpyAsync(fz, p.flag[2], nzf, cudaMemcpyDeviceToHost, ctx->stream), "flags");
    CK(cudaStreamSynchronize(ctx->stream), "flags");
    return OCFD_OK;
}

// ana_residual (src/OCFD_ana.cu:76-105): mean of E (which = 0) or T (which = 1)
extern "C" int ocfd_b200_ana_residual(ocfd_b200_ctx *ctx, int which, double *mean) {
    int rc = check_ready(ctx);
    if (rc) return rc;
    if ((rc = refresh_prims64(ctx))) return rc;
    if (!mean || which < 0 || which > 1) return fail(ctx, OCFD_ERR_ARG, "which must be 0 (E) or 1 (T)");
    CK(ocfd::launch_mean(ctx->p, which, ctx->red_buf, nullptr, global_cells(ctx), ctx->stream), "reduction");
    ctx->launches += 2;
    if (ctx->slab) {
        std::string err;
        if (ocfd::slab_allreduce(ctx->slab, ctx->red_buf + ocfd::reduce_scratch_doubles() - 1, 1, 0, ctx->stream, err))
            return fail(ctx, OCFD_ERR_CUDA, err);
    }
    CK(cudaMemcpyAsync(mean, ctx->red_buf + ocfd::reduce_scratch_doubles() - 1, sizeof(double),
                       cudaMemcpyDeviceToHost, ctx->stream), "reduction read-back");
    CK(cudaStreamSynchronize(ctx->stream), "reduction");
    return OCFD_OK;
}

// ana_NAN_and_NT (src/OCFD_ana.cu:107-222) as counts: cells with a NaN in
// d,u,v,w,T and cells with T < 0; the mean of T is returned alongside.
extern "C" int ocfd_b200_check_state(ocfd_b200_ctx *ctx, long long *n_nan, long long *n_neg_t, double *mean_t) {
    int rc = check_ready(ctx);
    if (rc) return rc;
    if ((rc = refresh_prims64(ctx))) return rc;
    int nd = ocfd::reduce_scratch_doubles();
    unsigned long long *counts = reinterpret_cast<unsigned long long *>(ctx->red_buf + nd);
    CK(ocfd::launch_mean(ctx->p, 1, ctx->red_buf, counts, global_cells(ctx), ctx->stream), "state check");
    ctx->launches += 2;
    if (ctx->slab) {
        std::string err;
        if (ocfd::slab_allreduce(ctx->slab, ctx->red_buf + nd - 1, 1, 0, ctx->stream, err) ||
            ocfd::slab_allreduce(ctx->slab, counts, 2, 1, ctx->stream, err))
            return fail(ctx, OCFD_ERR_CUDA, err);
    }
    double host[3];
    CK(cudaMemcpyAsync(host, ctx->red_buf + nd - 1, 3 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream),
       "state check read-back");
    CK(cudaStreamSynchronize(ctx->stream), "state check");
    unsigned long long c[2];
    memcpy(c, host + 1, sizeof(c));
    if (n_nan) *n_nan = (long long)c[0];
    if (n_neg_t) *n_neg_t = (long long)c[1];
    if (mean_t) *mean_t = host[0];
    return OCFD_OK;
}

// get_Q (src/OCFD_ana.cu:317-456) of the current primitives, ghosts filled
// first; q: host array [nz][ny][nx]
extern "C" int ocfd_b200_q_criterion(ocfd_b200_ctx *ctx, double *q) {
    int rc = check_ready(ctx);
    if (rc) return rc;
    if (!q) return fail(ctx, OCFD_ERR_ARG, "null output");
    if ((rc = refresh_prims64(ctx))) return rc;
    if ((rc = ghost_prims64(ctx))) return rc;
    CK(ocfd::launch_q_criterion(ctx->p, ctx->stage_buf, ctx->stream), "Q criterion");
    ctx->launches += 1;
    CK(cudaMemcpyAsync(q, ctx->stage_buf, sizeof(double) * (size_t)ctx->p.N, cudaMemcpyDeviceToHost, ctx->stream),
       "Q read-back");
    CK(cudaStreamSynchronize(ctx->stream), "Q criterion");
    return OCFD_OK;
}

// init_time_average / ana_time_average (src/OCFD_ana.cu:224-316): reset the
// running means, or add the current primitives as one more sample
extern "C" int ocfd_b200_time_average(ocfd_b200_ctx *ctx, int reset) {
    int rc = check_ready(ctx);
    if (rc) return rc;
    const size_t bytes = 5 * sizeof(double) * (size_t)ctx->p.N;
    if (!ctx->avg_buf) {
        cudaError_t e = cudaMalloc((void **)&ctx->avg_buf, bytes);
        if (e != cudaSuccess) { ctx->avg_buf = nullptr; cudaGetLastError(); return fail(ctx, OCFD_ERR_NOMEM, "time averages"); }
        reset = 1;
    }
    if (reset) {
        CK(cudaMemsetAsync(ctx->avg_buf, 0, bytes, ctx->stream), "time averages");
        ctx->avg_n = 0;
        return OCFD_OK;
    }
    if ((rc = refresh_prims64(ctx))) return rc;
    CK(ocfd::launch_time_average(ctx->p, ctx->avg_buf, ctx->avg_n, ctx->stream), "time average");
    ctx->launches += 1;
    ctx->avg_n += 1;
    return OCFD_OK;
}

// the running means of d, u, v, w, T (host [5][nz][ny][nx]) and their sample count
extern "C" int ocfd_b200_get_time_average(ocfd_b200_ctx *ctx, double *mean5, int *count) {
    int rc = check_ready(ctx);
    if (rc) return rc;
    if (count) *count = ctx->avg_n;
    if (!mean5) return OCFD_OK;
    if (!ctx->avg_buf) return fail(ctx, OCFD_ERR_STATE, "no time averages taken");
    CK(cudaMemcpyAsync(mean5, ctx->avg_buf, 5 * sizeof(double) * (size_t)ctx->p.N, cudaMemcpyDeviceToHost,
                       ctx->stream), "time average read-back");
    CK(cudaStreamSynchronize(ctx->stream), "time average");
    return OCFD_OK;
}

// HybridAuto_scheme_Proportion (src/OCFD_Schemes_hybrid_auto.cu:745-829):
// frac[3 * dir + t] = share of direction dir's flag entries of type t (flag
// 1, flag 2, any other value), as the reference prints them
extern "C" int ocfd_b200_scheme_proportion(ocfd_b200_ctx *ctx, double frac[9]) {
    int rc = check_ready(ctx);
    if (rc) return rc;
    if (!frac) return fail(ctx, OCFD_ERR_ARG, "frac is null");
    const Params &p = ctx->p;
    unsigned long long *counts = reinterpret_cast<unsigned long long *>(ctx->red_buf + ocfd::reduce_scratch_doubles());
    CK(ocfd::launch_flag_hist(p, counts, ctx->stream), "scheme proportion");
    ctx->launches += 1;
    if (ctx->slab) {
        std::string err;
        if (ocfd::slab_allreduce(ctx->slab, counts, 9, 1, ctx->stream, err)) return fail(ctx, OCFD_ERR_CUDA, err);
    }
    unsigned long long h[9];
    CK(cudaMemcpyAsync(h, counts, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream), "scheme proportion");
    CK(cudaStreamSynchronize(ctx->stream), "scheme proportion");
    const double nzg = ctx->slab ? ctx->nz_global : p.nz;      // the whole grid's flag entries
    const double n[3] = {(double)(p.nx + 1) * p.ny * nzg, (double)p.nx * (p.ny + 1) * nzg,
                         (double)p.nx * p.ny * (nzg + (ctx->slab ? ctx->slab_count : 1))};
    for (int i = 0; i < 9; i++) frac[i] = (double)h[i] / n[i / 3];
    return OCFD_OK;
}

extern "C" int ocfd_b200_get_time(const ocfd_b200_ctx *ctx, int *istep, double *tt) {
    if (!ctx) return OCFD_ERR_ARG;
    if (istep) *istep = ctx->istep;
    if (tt) *tt = ctx->tt;
    return OCFD_OK;
}

extern "C" int ocfd_b200_advance_host(ocfd_b200_ctx *ctx, const double *in, double *out, int nsteps) {
    if (!ctx || !in || !out) return OCFD_ERR_ARG;
    if (!ctx->have_metrics) return fail(ctx, OCFD_ERR_STATE, "metrics not set");
    int rc = ocfd_b200_set_primitives(ctx, in, ctx->istep, ctx->tt);
    if (rc) return rc;
    if ((rc = ocfd_b200_step(ctx, nsteps))) return rc;
    return ocfd_b200_get_primitives(ctx, out);
}

// ---------------------------------------------------------------------------
// timing
// ---------------------------------------------------------------------------

extern "C" int ocfd_b200_set_timing(ocfd_b200_ctx *ctx, int enabled) {
    if (!ctx) return OCFD_ERR_ARG;
    ctx->timing = enabled != 0;
    for (int i = 0; i < OCFD_TIMER_COUNT; i++) { ctx->t_ms[i] = 0; ctx->t_n[i] = 0; }
    return OCFD_OK;
}
extern "C" int ocfd_b200_get_timing(ocfd_b200_ctx *ctx, double *ms, long long *n, int cnt) {
    if (!ctx) return OCFD_ERR_ARG;
    for (int i = 0; i < cnt && i < OCFD_TIMER_COUNT; i++) {
        if (ms) ms[i] = ctx->t_ms[i];
        if (n) n[i] = ctx->t_n[i];
    }
    return OCFD_OK;
}
extern "C" const char *ocfd_b200_timer_name(int i) {
    return (i >= 0 && i < OCFD_TIMER_COUNT) ? kTimerNames[i] : "";
}
extern "C" long long ocfd_b200_launch_count(const ocfd_b200_ctx *ctx) { return ctx ? ctx->launches : 0; }

// ---------------------------------------------------------------------------
// reference-named entry points
// ---------------------------------------------------------------------------
static ocfd_b200_ctx *g_bound = nullptr;

extern "C" int ocfd_b200_compat_bind(ocfd_b200_ctx *ctx) { g_bound = ctx; return OCFD_OK; }

static void compat_report(int rc, const char *what) {
    if (rc != OCFD_OK)
        fprintf(stderr, "ocfd_b200: %s failed: %s (%s)\n", what, ocfd_b200_status_string(rc),
                ocfd_b200_last_error(g_bound));
}

extern "C" void du_comput(int KRK) { compat_report(g_bound ? ocfd_b200_du_comput(g_bound, KRK) : OCFD_ERR_STATE, "du_comput"); }
extern "C" void OCFD_time_advance(int KRK) { compat_report(g_bound ? ocfd_b200_time_advance(g_bound, KRK) : OCFD_ERR_STATE, "OCFD_time_advance"); }
extern "C" void get_duvwT(void) { compat_report(g_bound ? ocfd_b200_get_duvwT(g_bound) : OCFD_ERR_STATE, "get_duvwT"); }
// viscosity is formed from T inside the viscous kernel; nothing to store
extern "C" void get_Amu(void) { compat_report(g_bound ? OCFD_OK : OCFD_ERR_STATE, "get_Amu"); }
extern "C" void OCFD_bc(void) { compat_report(g_bound ? ocfd_b200_bc(g_bound) : OCFD_ERR_STATE, "OCFD_bc"); }
extern "C" void Set_Scheme_HybridAuto(void *stream) {
    (void)stream;
    if (!g_bound) { compat_report(OCFD_ERR_STATE, "Set_Scheme_HybridAuto"); return; }
    cudaError_t e = ocfd::launch_sensor(g_bound->p, g_bound->stream);
    compat_report(e == cudaSuccess ? OCFD_OK : OCFD_ERR_CUDA, "Set_Scheme_HybridAuto");
}
// the library keeps pf_lap and p itself; the arguments are the reference's
// own buffers and are not read
extern "C" void filtering(double *pf, double *pf_lap, double *pp) {
    (void)pf; (void)pf_lap; (void)pp;
    compat_report(g_bound ? ocfd_b200_filtering(g_bound) : OCFD_ERR_STATE, "filtering");
}

// ---------------------------------------------------------------------------
// Allocation-free field means (no counterpart in the reference).
//
// For callers that own their device arrays and cannot allocate: a host code
// that keeps its fields in its own device buffers (the reference sizes its
// arrays to the whole GPU) and wants the FP64 residual means between steps
// without creating a solver context, which allocates the whole state, and
// without cudaMalloc/cudaFree, whose implicit device synchronisation would
// stall its pipeline.  The partial sums live in one file-scope device array
// that every call on a device shares; nothing is allocated per call.
//
// Same blocks, same per-thread order and same tree as the context reduction
// (launch_mean), so the mean of a field equals ocfd_b200_ana_residual's to
// the last bit when it is given the same values.
// ---------------------------------------------------------------------------
namespace {

constexpr int NA_BLOCKS = 592;        // partial sums per field (4 x 148 SMs)
constexpr int NA_THREADS = 256;
constexpr int NA_MAX_FIELDS = OCFD_NOALLOC_MAX_FIELDS;

// 8 fields x 592 partials x 8 bytes = 37,888 bytes per device.  Host code
// never passes this array's name to a kernel; it passes the address that
// cudaGetSymbolAddress returns on the current device.
static __device__ __align__(256) double g_mean_scratch[NA_MAX_FIELDS * NA_BLOCKS];

__global__ void __launch_bounds__(NA_THREADS) k_field_mean_partial(const double *fields, long long n,
                                                                  double *partial) {
    __shared__ double sh[NA_THREADS];
    const double *src = fields + (long long)blockIdx.y * n;
    double acc = 0.0;
    long long stride = (long long)gridDim.x * blockDim.x;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += stride) acc += src[q];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int h = NA_THREADS / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) sh[threadIdx.x] += sh[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.y * NA_BLOCKS + blockIdx.x] = sh[0];
}

__global__ void __launch_bounds__(NA_THREADS) k_field_mean_final(const double *partial, long long n,
                                                                double *means) {
    __shared__ double sh[NA_THREADS];
    const double *src = partial + blockIdx.x * NA_BLOCKS;
    double acc = 0.0;
    for (int q = threadIdx.x; q < NA_BLOCKS; q += blockDim.x) acc += src[q];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int h = NA_THREADS / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) sh[threadIdx.x] += sh[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) means[blockIdx.x] = sh[0] / (double)n;
}

// Address of the current device's copy of g_mean_scratch.  Looked up on every
// call (the lookup allocates nothing): a cached address would go stale if the
// caller reset the device or released its primary context, after which the
// library's device code is loaded again and the array may sit elsewhere.
int noalloc_scratch(double **out) {
    double *ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void **)&ptr, g_mean_scratch);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "field_means_noalloc: cudaGetSymbolAddress");
    *out = ptr;
    return OCFD_OK;
}

}  // namespace

extern "C" int ocfd_b200_field_means_noalloc(const double *fields, int nfield, long long n, double *means,
                                             void *stream) {
    if (!fields || !means) return fail(nullptr, OCFD_ERR_ARG, "field_means_noalloc: null fields or means");
    if (nfield < 1 || nfield > NA_MAX_FIELDS)
        return fail(nullptr, OCFD_ERR_ARG,
                    "field_means_noalloc: nfield = " + std::to_string(nfield) + " is outside 1.." +
                        std::to_string(NA_MAX_FIELDS) + " (the fixed scratch holds " +
                        std::to_string(NA_MAX_FIELDS) + " x " + std::to_string(NA_BLOCKS) + " partial sums)");
    if (n < 1 || n > (1LL << 40))
        return fail(nullptr, OCFD_ERR_ARG, "field_means_noalloc: n = " + std::to_string(n) + " is outside 1..2^40");
    double *scratch = nullptr;
    int rc = noalloc_scratch(&scratch);
    cudaError_t e;
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // every partial slot the final kernel reads is written by the first
    // kernel of the same call, so nothing in the scratch needs clearing
    k_field_mean_partial<<<dim3(NA_BLOCKS, nfield), NA_THREADS, 0, st>>>(fields, n, scratch);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "field_means_noalloc: partial sums");
    k_field_mean_final<<<nfield, NA_THREADS, 0, st>>>(scratch, n, means);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "field_means_noalloc: final sums");
    return OCFD_OK;
}
