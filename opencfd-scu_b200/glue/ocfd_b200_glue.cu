/*
 * ocfd_b200_glue.cu -- the reference driver's RHS-path calls served by
 * libocfd_b200.
 *
 * The reference's main program, parameter reader, initialisation, I/O and
 * analysis stay as they are (opencfd.c, src/OCFD_NS_Solver.cu:39-177 and the
 * rest); this file defines the six functions its time loop calls for the
 * RHS path:
 *
 *   OCFD_bc()             src/OCFD_boundary.cu:18
 *   du_comput(int)        src/OCFD_Stream.cu:28
 *   OCFD_time_advance(int) src/OCFD_time.cu:96
 *   get_duvwT()           src/commen_kernel.cu:111
 *   get_Amu()             src/commen_kernel.cu:133
 *   filtering(pf, pf_lap, pP)  src/OCFD_filtering.cu:75
 *
 * and forwards them to one library context.  The reference's own
 * definitions of these six are renamed in its objects at link time (the
 * recipe oracle/dropin.mk does it with objcopy), so its driver needs no
 * edit at all, not even the pf/pfn swap: the swap the driver makes of its
 * own pointers at the top of each step is mirrored by swapping the
 * context's time levels in du_comput(1).
 *
 * The context is made on the first OCFD_bc() call, which NS_solver_real
 * makes after init() and before the time loop: the configuration comes from
 * the globals read_parameters() filled, the metrics and the primitives from
 * the reference's device fields as init() left them, the filters from
 * set_para_filtering()'s tables.  After each step (in filtering(), which the
 * driver calls once per step, after the RK stages and before its analysis
 * and saves) the library's primitives are copied back into the reference's
 * device fields, so that its own output files and prints read them.
 *
 * Compiled against the reference's headers (parameters.h, parameters_d.h,
 * cuda_commen.h) and include/ocfd_b200.h.
 */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "parameters.h"
#include "parameters_d.h"
#include "cuda_commen.h"
#include "cuda_utility.h"

#define OCFD_B200_NO_REFERENCE_NAMES
#include "ocfd_b200.h"

extern "C" {
extern int IF_CHARTERIC;        /* src/parameters.c:162 */
}

namespace {

ocfd_b200_ctx *g_ctx = nullptr;
bool g_failed = false;

void check(int rc, const char *what) {
    if (rc != OCFD_OK) {
        fprintf(stderr, "ocfd_b200 glue: %s failed: %s (%s)\n", what, ocfd_b200_status_string(rc),
                ocfd_b200_last_error(g_ctx));
        g_failed = true;
    }
}

// interior of a reference LAP-box device field into a dense [nz][ny][nx] host array
void gather_field(const cudaField *f, double *dense, std::vector<double> &lap) {
    memcpy_All(lap.data(), f->ptr, f->pitch, D2H, nx_2lap, ny_2lap, nz_2lap);
    for (unsigned k = 0; k < nz; k++)
        for (unsigned j = 0; j < ny; j++)
            memcpy(dense + ((size_t)k * ny + j) * nx,
                   lap.data() + (((size_t)(k + LAP) * ny_2lap) + (j + LAP)) * nx_2lap + LAP, nx * sizeof(double));
}

// a dense [nz][ny][nx] host array into the interior of a reference device field
void scatter_field(const double *dense, REAL *host_lap, const cudaField *f) {
    for (unsigned k = 0; k < nz; k++)
        for (unsigned j = 0; j < ny; j++)
            memcpy(host_lap + (((size_t)(k + LAP) * ny_2lap) + (j + LAP)) * nx_2lap + LAP,
                   dense + ((size_t)k * ny + j) * nx, nx * sizeof(double));
    memcpy_inner(host_lap, f->ptr, f->pitch, H2D, nx_2lap, ny_2lap, nz_2lap);
}

void make_context() {
    ocfd_b200_config c;
    memset(&c, 0, sizeof(c));
    c.nx = (int)nx; c.ny = (int)ny; c.nz = (int)nz;
    for (int i = 0; i < 3; i++) { c.iperiodic[i] = Iperiodic[i]; c.jac_bound[i] = Jacbound[i]; }
    for (int i = 0; i < 6; i++) { c.dif_bound[i] = D0_bound[i]; c.non_reflection[i] = Non_ref[i]; }
    c.scheme_invis = Scheme_invis_ID;
    c.scheme_vis = Scheme_vis_ID;
    c.charteric = IF_CHARTERIC;
    if (Scheme_invis_ID == 310) {
        c.hy_style = HybridAuto.Style;
        c.hy_dp_intv[0] = HybridAuto.P_intvs[0];
        c.hy_dp_intv[1] = HybridA_Stage > 2 ? HybridAuto.P_intvs[1] : HybridAuto.P_intvs[0];
    }
    c.re = Re; c.ama = Ama; c.gamma = Gamma; c.pr = Pr; c.t_ref = Ref_T; c.epsl_sw = epsl_SW; c.dt = dt;
    int dev = 0;
    cudaGetDevice(&dev);
    c.device = dev;
    check(ocfd_b200_create(&c, &g_ctx), "create");
    if (g_failed) return;

    const size_t N = (size_t)nx * ny * nz;
    std::vector<double> lap((size_t)nx_2lap * ny_2lap * nz_2lap);
    // the metrics init() computed or read (Axx .. Ajac, the order of the ABI)
    std::vector<double> met(13 * N);
    const cudaField *mf[13] = { pAxx_d, pAyy_d, pAzz_d, pAkx_d, pAky_d, pAkz_d, pAix_d, pAiy_d, pAiz_d,
                                pAsx_d, pAsy_d, pAsz_d, pAjac_d };
    for (int m = 0; m < 13; m++) gather_field(mf[m], met.data() + m * N, lap);
    check(ocfd_b200_set_metrics(g_ctx, met.data()), "set_metrics");
    // the filters set_para_filtering() tabulated
    for (int n = 0; n < NFiltering && !g_failed; n++)
        check(ocfd_b200_set_filter(g_ctx, n, Filter_para[n], Filter_rpara[n]), "set_filter");
    // the state init() left
    std::vector<double> prim(5 * N);
    const cudaField *pf5[5] = { pd_d, pu_d, pv_d, pw_d, pT_d };
    for (int m = 0; m < 5; m++) gather_field(pf5[m], prim.data() + m * N, lap);
    if (!g_failed) check(ocfd_b200_set_primitives(g_ctx, prim.data(), Istep, tt), "set_primitives");
}

// the library's primitives into the reference's device fields (interior)
void publish_state() {
    const size_t N = (size_t)nx * ny * nz;
    std::vector<double> prim(5 * N);
    check(ocfd_b200_get_primitives(g_ctx, prim.data()), "get_primitives");
    REAL *hl[5] = { pd, pu, pv, pw, pT };
    const cudaField *pf5[5] = { pd_d, pu_d, pv_d, pw_d, pT_d };
    for (int m = 0; m < 5; m++) scatter_field(prim.data() + m * N, hl[m], pf5[m]);
}

bool ready() {
    if (!g_ctx && !g_failed) make_context();
    return g_ctx && !g_failed;
}

}  // namespace

extern "C" {

void OCFD_bc() {
    if (ready()) check(ocfd_b200_bc(g_ctx), "OCFD_bc");
}

void du_comput(int KRK) {
    if (!ready()) return;
    // the driver has just swapped pf and pfn for the new step
    if (KRK == 1) check(ocfd_b200_swap_time_levels(g_ctx), "swap_time_levels");
    check(ocfd_b200_du_comput(g_ctx, KRK), "du_comput");
}

void OCFD_time_advance(int KRK) {
    if (ready()) check(ocfd_b200_time_advance(g_ctx, KRK), "OCFD_time_advance");
}

void get_duvwT() {
    if (ready()) check(ocfd_b200_get_duvwT(g_ctx), "get_duvwT");
}

// the viscosity is formed from T inside the library's viscous kernel
void get_Amu() {}

void filtering(REAL *pf_unused, REAL *pf_lap_unused, REAL *pP_unused) {
    (void)pf_unused; (void)pf_lap_unused; (void)pP_unused;
    if (!ready()) return;
    check(ocfd_b200_set_time(g_ctx, Istep, tt), "set_time");
    check(ocfd_b200_filtering(g_ctx), "filtering");
    publish_state();
    if (g_failed) {
        fprintf(stderr, "ocfd_b200 glue: stopping\n");
        exit(3);
    }
}

}  // extern "C"
