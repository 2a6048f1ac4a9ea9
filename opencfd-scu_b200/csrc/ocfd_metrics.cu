// ocfd_metrics.cu -- grid metrics from mesh coordinates on the GPU (sm_100a, FP64).
//
// Replaces Comput_Jacobian3d (src/OCFD_Comput_Jacobian3d.cu:221-246):
// comput_Jac3d (:393-424) forms the nine derivatives d(x,y,z)/d(i,j,k) with
// OCFD_d{x,y,z}0_CD6_kernel (src/OCFD_Schemes.cu:1236-1304) and, where
// JAC_BOUND of a direction is non-zero, OCFD_D{x,y,z}0_bound_kernel_{m,p}
// (src/OCFD_bound_Scheme.cu:189-349) on the four points at each end;
// comput_Jac3d_kernal (:250-391) forms the nine conservative metrics and the
// inverse Jacobian and extrapolates them as constants into the ghost slabs.
// This is set-up work (once per grid), so every quotient is a plain IEEE
// division, as in the reference.
#include "ocfd_device.cuh"

#include <cuda_runtime.h>

namespace ocfd {

namespace {

// d f / d(index of DIR) at every interior cell of a LAP field
template <int DIR>
__global__ void k_jac_d0(Params p, const double *__restrict__ f, double *__restrict__ out, int bound) {
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= p.N) return;
    const int i = (int)(tid % p.nx);
    const long long r = tid / p.nx;
    const int j = (int)(r % p.ny), k = (int)(r / p.ny);
    const long long s = DIR == 0 ? 1LL : (DIR == 1 ? p.ys : p.zs);
    const double h = DIR == 0 ? p.hx : (DIR == 1 ? p.hy : p.hz);
    const int n = DIR == 0 ? p.nx : (DIR == 1 ? p.ny : p.nz);
    const int X = DIR == 0 ? i : (DIR == 1 ? j : k);
    const double *c = f + lap_index(p, i + OCFD_LAP, j + OCFD_LAP, k + OCFD_LAP);
    auto F = [&](int t) { return c[(long long)t * s]; };
    double v = (45.0 * (F(1) - F(-1)) - 9.0 * (F(2) - F(-2)) + (F(3) - F(-3))) / (60.0 * h);
    // CHECK_Z (src/OCFD_bound_Scheme.cu:64-72): with the grid split in z,
    // the z closures belong to the first and last slab only
    const bool lo_side = DIR != 2 || p.zface_lo, hi_side = DIR != 2 || p.zface_hi;
    if (bound && lo_side) {
        if (X == 0)      v = (F(1) - F(0)) / h;
        else if (X == 1) v = (F(1) - F(-1)) * 0.5 / h;
        else if (X == 2) v = (F(-2) - 8.0 * F(-1) + 8.0 * F(1) - F(2)) / (12.0 * h);
        else if (X == 3) v = (F(3) - F(-3) - 9.0 * (F(2) - F(-2)) + 45.0 * (F(1) - F(-1))) / (60.0 * h);
    }
    if (bound && hi_side) {
        const int u = X - (n - 1);
        if (DIR != 1) {
            if (u == 0)       v = (F(0) - F(-1)) / h;
            else if (u == -1) v = (F(1) - F(-1)) * 0.5 / h;
            else if (u == -2) v = (F(-2) - 8.0 * F(-1) + 8.0 * F(1) - F(2)) / (12.0 * h);
            else if (u == -3) v = (F(3) - F(-3) - 9.0 * (F(2) - F(-2)) + 45.0 * (F(1) - F(-1))) / (60.0 * h);
        } else {            // the y kernel writes these as negated differences
            if (u == 0)       v = -(F(-1) - F(0)) / h;
            else if (u == -1) v = -(F(-1) - F(1)) * 0.5 / h;
            else if (u == -2) v = -(F(2) - 8.0 * F(1) + 8.0 * F(-1) - F(-2)) / (12.0 * h);
            else if (u == -3) v = -(F(-3) - F(3) - 9.0 * (F(-2) - F(2)) + 45.0 * (F(-1) - F(1))) / (60.0 * h);
        }
    }
    out[tid] = v;
}

// D[3*dir + c] = d(coordinate c)/d(index dir), interior fields
__global__ void k_jac_metrics(Params p, const double *__restrict__ D) {
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= p.N) return;
    const int i = (int)(tid % p.nx);
    const long long r = tid / p.nx;
    const int j = (int)(r % p.ny), k = (int)(r / p.ny);
    const long long N = p.N;
    const double xi1 = D[tid], yi1 = D[N + tid], zi1 = D[2 * N + tid];
    const double xj1 = D[3 * N + tid], yj1 = D[4 * N + tid], zj1 = D[5 * N + tid];
    const double xk1 = D[6 * N + tid], yk1 = D[7 * N + tid], zk1 = D[8 * N + tid];
    double v[10];
    v[9] = 1.0 / (xi1 * yj1 * zk1 + yi1 * zj1 * xk1 + zi1 * xj1 * yk1
                  - zi1 * yj1 * xk1 - yi1 * xj1 * zk1 - xi1 * zj1 * yk1);   // Ajac
    v[0] = (yj1 * zk1 - zj1 * yk1);      // Akx
    v[1] = (zj1 * xk1 - xj1 * zk1);      // Aky
    v[2] = (xj1 * yk1 - yj1 * xk1);      // Akz
    v[3] = (yk1 * zi1 - zk1 * yi1);      // Aix
    v[4] = (zk1 * xi1 - xk1 * zi1);      // Aiy
    v[5] = (xk1 * yi1 - yk1 * xi1);      // Aiz
    v[6] = (yi1 * zj1 - zi1 * yj1);      // Asx
    v[7] = (zi1 * xj1 - xi1 * zj1);      // Asy
    v[8] = (xi1 * yj1 - yi1 * xj1);      // Asz
    const int L = OCFD_LAP;
    for (int m = 0; m < 10; m++) {
        double *A = const_cast<double *>(p.met[M_AKX + m]);
        const double a = v[m];
        A[lap_index(p, i + L, j + L, k + L)] = a;
        // constant extrapolation into the ghost slabs
        if (i == 0)        for (int g = 0; g < L; g++) A[lap_index(p, g, j + L, k + L)] = a;
        if (i == p.nx - 1) for (int g = 1; g <= L; g++) A[lap_index(p, i + L + g, j + L, k + L)] = a;
        if (j == 0)        for (int g = 0; g < L; g++) A[lap_index(p, i + L, g, k + L)] = a;
        if (j == p.ny - 1) for (int g = 1; g <= L; g++) A[lap_index(p, i + L, j + L + g, k + L)] = a;
        if (k == 0)        for (int g = 0; g < L; g++) A[lap_index(p, i + L, j + L, g)] = a;
        if (k == p.nz - 1) for (int g = 1; g <= L; g++) A[lap_index(p, i + L, j + L, k + L + g)] = a;
    }
}

// ana_Jac (src/OCFD_ana.cu:24-48): any negative Jacobian on the LAP box
__global__ void k_neg_jac(const double *__restrict__ ajac, long long n, unsigned *flag) {
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        if (ajac[q] < 0.0) { atomicOr(flag, 1u); return; }
}

inline unsigned blocks(long long n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

// coordinates are in met[0..2] (ghosts filled); scratch: 9 interior fields
cudaError_t launch_mesh_metrics(const Params &p, const int jac_bound[3], double *scratch, cudaStream_t st) {
    const unsigned nb = blocks(p.N, 256);
    for (int c = 0; c < 3; c++) {
        k_jac_d0<0><<<nb, 256, 0, st>>>(p, p.met[c], scratch + (size_t)(0 + c) * p.N, jac_bound[0]);
        k_jac_d0<1><<<nb, 256, 0, st>>>(p, p.met[c], scratch + (size_t)(3 + c) * p.N, jac_bound[1]);
        k_jac_d0<2><<<nb, 256, 0, st>>>(p, p.met[c], scratch + (size_t)(6 + c) * p.N, jac_bound[2]);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_jac_metrics<<<nb, 256, 0, st>>>(p, scratch);
    return cudaGetLastError();
}

cudaError_t launch_negative_jacobian(const Params &p, unsigned *flag, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(flag, 0, sizeof(unsigned), st);
    if (e != cudaSuccess) return e;
    k_neg_jac<<<4 * 148, 256, 0, st>>>(p.met[M_AJAC], p.lapN, flag);
    return cudaGetLastError();
}

}  // namespace ocfd
