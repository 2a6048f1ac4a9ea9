// ocfd_bc.cu -- compression-corner boundary conditions, IBC 108 (sm_100a, FP64).
//
// bc_user_Compression_conner (src/OCFD_boundary_compression_conner.cu:122-180) on
// the primitives, before OCFD_bc's face re-projection:
//   inlet  (x = 0): the ghost columns and the first column take the inflow
//          profile (d, u, v, T from flow1d-inlet.dat, w = 0);
//   top    (y = ny-1, x >= x_begin): the profile's last row;
//   wall   (y = 0): no slip with wall-normal blowing v = EPSL fx(x) gz(z) h(t),
//          then T = TW with the pressure extrapolated to the wall (and the
//          ghost rows mirrored: d, T even, u, v, w odd), or, for TW <= 0, T and
//          p extrapolated.  The wall kernels act on their own (x, z) column.
// In the precision form the values are formed in FP64 as above and also
// stored in the FP32 primitives the stencils read.
#include "ocfd_device.cuh"

#include <cuda_runtime.h>

namespace ocfd {

namespace {

// the five primitives of LAP-box point q into the FP32 copies (precision form)
__device__ __forceinline__ void to_fp32(const Params &p, long long q) {
    if (!p.mixed) return;
#pragma unroll
    for (int m = 0; m < 5; m++) p.prim32[m][q] = (float)p.prim[m][q];
}

__global__ void k_bc108_inlet(Params p) {
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= (long long)p.ny * p.nz) return;
    const int j = (int)(tid % p.ny), k = (int)(tid / p.ny);
    const double d = p.bc_ub1[j], u = p.bc_ub1[p.ny + j], v = p.bc_ub1[2 * p.ny + j], T = p.bc_ub1[3 * p.ny + j];
    for (int i = 0; i <= OCFD_LAP; i++) {
        const long long q = lap_index(p, i, j + OCFD_LAP, k + OCFD_LAP);
        p.prim[0][q] = d; p.prim[1][q] = u; p.prim[2][q] = v; p.prim[3][q] = 0.; p.prim[4][q] = T;
        to_fp32(p, q);
    }
}

__global__ void k_bc108_top(Params p) {
    const int nxs = p.nx - p.bc_xbegin;
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (nxs <= 0 || tid >= (long long)nxs * p.nz) return;
    const int i = p.bc_xbegin + (int)(tid % nxs), k = (int)(tid / nxs);
    const int j = p.ny - 1;
    const long long q = lap_index(p, i + OCFD_LAP, j + OCFD_LAP, k + OCFD_LAP);
    p.prim[0][q] = p.bc_ub1[j];
    p.prim[1][q] = p.bc_ub1[p.ny + j];
    p.prim[2][q] = p.bc_ub1[2 * p.ny + j];
    p.prim[3][q] = 0.;
    p.prim[4][q] = p.bc_ub1[3 * p.ny + j];
    to_fp32(p, q);
}

// do_wall_dist_kernel, then do_wall_Tp1_kernel / do_wall_Tp2_kernel
__global__ void k_bc108_wall(Params p, double ht) {
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= (long long)p.nx * p.nz) return;
    const int i = (int)(tid % p.nx), k = (int)(tid / p.nx);
    double *d = p.prim[0], *u = p.prim[1], *v = p.prim[2], *w = p.prim[3], *T = p.prim[4];
    const long long q = lap_index(p, i + OCFD_LAP, OCFD_LAP, k + OCFD_LAP);
    const long long sy = p.ys;
    u[q] = 0.;
    v[q] = p.bc_epsl * p.bc_fx[i] * p.bc_gz[k] * ht;
    w[q] = 0.;
    if (p.bc_wall_mode == 0) {                         // non-normal wall: not supported there either
        to_fp32(p, q);
        return;
    }
    if (p.bc_wall_mode == 1) {
        const double pw = (18. * d[q + sy] * T[q + sy] - 9. * d[q + 2 * sy] * T[q + 2 * sy]
                           + 2. * d[q + 3 * sy] * T[q + 3 * sy]) / 11.;
        T[q] = p.bc_tw;
        d[q] = pw / T[q];
        for (int g = 0; g < OCFD_LAP; g++) {
            const long long qg = lap_index(p, i + OCFD_LAP, g, k + OCFD_LAP);
            const long long qm = lap_index(p, i + OCFD_LAP, 2 * OCFD_LAP - g, k + OCFD_LAP);
            d[qg] = d[qm]; u[qg] = -u[qm]; v[qg] = -v[qm]; w[qg] = -w[qm]; T[qg] = T[qm];
            to_fp32(p, qg);
        }
    } else {
        T[q] = (18. * T[q + sy] - 9. * T[q + 2 * sy] + 2. * T[q + 3 * sy]) / 11.;
        const double pw = (18. * d[q + sy] * T[q + sy] - 9. * d[q + 2 * sy] * T[q + 2 * sy]
                           + 2. * d[q + 3 * sy] * T[q + 3 * sy]) / 11.;
        d[q] = pw / T[q];
    }
    to_fp32(p, q);
}

inline unsigned blocks(long long n) { return (unsigned)((n + 255) / 256); }

}  // namespace

// the boundary values of one application at wall-blowing amplitude ht
cudaError_t launch_bc108(const Params &p, double ht, cudaStream_t st) {
    k_bc108_inlet<<<blocks((long long)p.ny * p.nz), 256, 0, st>>>(p);
    if (p.nx > p.bc_xbegin) k_bc108_top<<<blocks((long long)(p.nx - p.bc_xbegin) * p.nz), 256, 0, st>>>(p);
    k_bc108_wall<<<blocks((long long)p.nx * p.nz), 256, 0, st>>>(p, ht);
    return cudaGetLastError();
}

}  // namespace ocfd
