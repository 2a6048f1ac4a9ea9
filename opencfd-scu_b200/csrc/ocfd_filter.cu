// ocfd_filter.cu -- shock-capturing filter after each step (sm_100a, FP64).
//
// Replaces filtering() / filter_{x,y,z}3d_shock (src/OCFD_filtering.cu:75-183,
// :363-606; Bogey, de Cacqueray & Bailly's shock-capturing filter): for each
// cell of a pass along direction d,
//   r_i    = 1/2 ((dp0-dp1)^2 + (dp0-dp2)^2) / p_i^2 + 1e-16,
//   sigma_i = max(0, 1 - rth / r_i),
//   U_i    = Ul_i - [ s0 sigma_{i+1/2} (c1 (Ul_{i+1}-Ul_i) + c2 (Ul_{i+2}-Ul_{i-1}))
//                   - s0 sigma_{i-1/2} (c1 (Ul_i-Ul_{i-1}) + c2 (Ul_{i+1}-Ul_{i-2})) ],
// sigma_{i+-1/2} the mean of the two cell values, dp the second differences of
// the pressure p as cons_to_pri leaves it after the step's last stage and Ul
// the state after the stage-3 update before the face re-projection.  Every
// pass reads Ul and writes U, so where passes overlap the last one stands.
// In the precision form sigma is formed from an FP32 pressure; Ul and the
// update of U stay FP64.
#include "ocfd_device.cuh"

#include <cuda_runtime.h>

namespace ocfd {

namespace {

constexpr double FC1 = -0.2103830, FC2 = 0.0396170;

// sigma_i from the pressure stencil, in the pressure's precision (FP64, or
// FP32 in the precision form)
template <typename R>
__device__ __forceinline__ R filter_sigma(const R *__restrict__ P, long long q, long long sd, R rth) {
    const R p_m2 = P[q - 2 * sd], p_m1 = P[q - sd], p_00 = P[q], p_p1 = P[q + sd], p_p2 = P[q + 2 * sd];
    const R dp0 = (R)0.25 * (-p_p1 + (R)2.0 * p_00 - p_m1);
    const R dp1 = (R)0.25 * (-p_p2 + (R)2.0 * p_p1 - p_00);
    const R dp2 = (R)0.25 * (-p_00 + (R)2.0 * p_m1 - p_m2);
    R ri = (R)0.5 * ((dp0 - dp1) * (dp0 - dp1) + (dp0 - dp2) * (dp0 - dp2)) / (p_00 * p_00) + (R)1e-16;
    ri = (R)1.0 - rth / ri;
    return (R)0.5 * (ri + fabs(ri));
}

// one pass along DIR over the box [lo, hi) (interior indices); R is the
// pressure's type, the update of U is FP64 either way
template <int DIR, typename R>
__global__ void k_filter(Params p, const R *__restrict__ P, int i0, int i1, int j0, int j1, int k0, int k1,
                         double s0, double rth) {
    const long long ni = i1 - i0, nj = j1 - j0, nk = k1 - k0;
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= ni * nj * nk) return;
    const int i = i0 + (int)(tid % ni);
    const long long r = tid / ni;
    const int j = j0 + (int)(r % nj), k = k0 + (int)(r / nj);
    const long long sd = DIR == 0 ? 1LL : (DIR == 1 ? p.ys : p.zs);
    const long long q = lap_index(p, i + OCFD_LAP, j + OCFD_LAP, k + OCFD_LAP);
    const double hm = (double)filter_sigma<R>(P, q - sd, sd, (R)rth);
    const double h0 = (double)filter_sigma<R>(P, q, sd, (R)rth);
    const double hp = (double)filter_sigma<R>(P, q + sd, sd, (R)rth);
    const double Sc1 = 0.5 * (h0 + hp) * s0;
    const double Sc2 = 0.5 * (h0 + hm) * s0;
    const long long ci = in_index(p, i, j, k);
#pragma unroll
    for (int m = 0; m < 5; m++) {
        const double *fl = p.flap + (long long)m * p.lapN;
        p.f[m * p.N + ci] = fl[q] - (Sc1 * (FC1 * (fl[q + sd] - fl[q]) + FC2 * (fl[q + 2 * sd] - fl[q - sd]))
                                   - Sc2 * (FC1 * (fl[q] - fl[q - sd]) + FC2 * (fl[q + sd] - fl[q - 2 * sd])));
    }
}

template <typename R>
void filter_pass(const Params &p, const R *P, int dir, const int lo[3], const int hi[3], double s0, double rth,
                 cudaStream_t st) {
    const long long n = (long long)(hi[0] - lo[0]) * (hi[1] - lo[1]) * (hi[2] - lo[2]);
    const unsigned nb = (unsigned)((n + 255) / 256);
    if (dir == 0)      k_filter<0, R><<<nb, 256, 0, st>>>(p, P, lo[0], hi[0], lo[1], hi[1], lo[2], hi[2], s0, rth);
    else if (dir == 1) k_filter<1, R><<<nb, 256, 0, st>>>(p, P, lo[0], hi[0], lo[1], hi[1], lo[2], hi[2], s0, rth);
    else               k_filter<2, R><<<nb, 256, 0, st>>>(p, P, lo[0], hi[0], lo[1], hi[1], lo[2], hi[2], s0, rth);
}

}  // namespace


// box = {ib, ie, jb, je, kb, ke} after the range clamps; the cells along
// DIR stop one short of the upper bound (the reference kernels' coverage)
cudaError_t launch_filter_pass(const Params &p, int dir, const int box[6], double s0, double rth, cudaStream_t st) {
    int lo[3] = { box[0], box[2], box[4] }, hi[3] = { box[1], box[3], box[5] };
    hi[dir] -= 1;
    for (int d = 0; d < 3; d++)
        if (hi[d] <= lo[d]) return cudaSuccess;
    if (p.mixed) filter_pass<float>(p, p.pfil32, dir, lo, hi, s0, rth, st);
    else         filter_pass<double>(p, p.pfil, dir, lo, hi, s0, rth, st);
    return cudaGetLastError();
}

}  // namespace ocfd
