// ocfd_sweep.cu -- inviscid flux sweeps, one launch per direction (sm_100a, FP64).
//
// Replaces OCFD_d{x,y,z}1 / OCFD_d{x,y,z}2 and the kernels they launch
// (src/OCFD_Schemes_Choose.cu:88-764, src/OCFD_Schemes.cu,
// src/OCFD_flux_charteric.cu, src/OCFD_Schemes_hybrid_auto.cu:862-1023).
//
// A block owns TS cells along the sweep direction and R rows across it.
//   A  : Steger-Warming split of every tile point (TS+8 per row) into shared
//        memory (sound speed formed on the fly);
//   A2 : for characteristic schemes, the face-averaged eigen-system of every
//        face (TS+1 per row) into shared memory;
//   B  : one thread per (face, sign).  The thread keeps the 8-point stencil
//        of all 5 components in registers, projects it on each
//        characteristic field in turn (5-term dot products), reconstructs,
//        and accumulates the back-projection, so every stencil value is read
//        from shared memory once.  For the hybrid scheme the faces are first
//        sorted into a characteristic list and a component-wise (UP7) list,
//        so the two costs do not diverge inside a warp;
//   C  : du of each tile cell from its two face fluxes, x+ then x- for every
//        component, as a single writer.
#include "ocfd_face.cuh"

#include <cuda_runtime.h>

namespace ocfd {

template <int DIR> struct Tile;
template <> struct Tile<0> { static constexpr int TS = 64, R = 2, THREADS = 128; };
template <> struct Tile<1> { static constexpr int TS = 16, R = 8, THREADS = 128; };
template <> struct Tile<2> { static constexpr int TS = 16, R = 8, THREADS = 128; };

// shared-memory position of tile point (s along DIR, row r): unit stride
// along the direction the consecutive threads of phase B walk
template <int DIR> __device__ __forceinline__ int spos(int s, int r) {
    constexpr int TS = Tile<DIR>::TS, R = Tile<DIR>::R;
    return DIR == 0 ? s + (TS + 8) * r : r + R * s;
}

// MINB: resident blocks per SM the register budget is fitted to (4 caps a
// thread at 128 registers and spills part of the characteristic path;
// 3 allows 170 and does not spill)
template <int DIR, bool UNI, bool EPS0, int MINB>
__global__ void __launch_bounds__(Tile<DIR>::THREADS, MINB)
k_sweep2(Params p) {
    constexpr int TS = Tile<DIR>::TS, R = Tile<DIR>::R;
    constexpr int NP = (TS + 8) * R;      // split points
    constexpr int NF = (TS + 1) * R;      // faces
    constexpr int NC = TS * R;            // cells
    extern __shared__ double smem[];
    double *spl = smem;                   // [10][NP]
    double *hat = smem + 10 * NP;         // [10][NF] final face fluxes, sign*5 + comp
    double *rec = hat + 10 * NF;          // [FP_N][NF] face records (characteristic schemes)
    __shared__ short list[2 * NF];        // face order: characteristic faces first
    __shared__ int nchar;

    const int n = t_ndir<DIR>(p), nr = t_nrow<DIR>(p);
    const int s0 = blockIdx.x * TS, r0 = blockIdx.y * R, c3 = blockIdx.z;
    const long long sd = t_sdir<DIR>(p), sr = t_srow<DIR>(p);
    const long long base = (long long)(c3 + OCFD_LAP) * t_s3rd<DIR>(p)
                         + (long long)(r0 + OCFD_LAP) * sr + (long long)s0 * sd;
    const double *d = p.prim[0], *u = p.prim[1], *v = p.prim[2], *w = p.prim[3], *T = p.prim[4];
    const int mA = M_AKX + 3 * DIR;
    const int scheme = p.scheme_invis;
    const bool char_scheme = p.charteric && (scheme == 304 || scheme == 305 || scheme == 310);
    const bool comp_none = p.charteric && !char_scheme;   // the reference adds nothing
    const bool hybrid = scheme == 310;
    const int8_t *flags = p.flag[DIR];

    if (threadIdx.x == 0) nchar = 0;

    // ---- A: split fluxes at interior-relative points s0-4 .. s0+TS+3
    for (int q = threadIdx.x; q < NP; q += blockDim.x) {
        int s, r;
        if (DIR == 0) { s = q % (TS + 8); r = q / (TS + 8); }
        else          { r = q % R; s = q / R; }
        if (r0 + r >= nr || s0 + s - 4 > n + 3) continue;
        long long o = base + (long long)s * sd + (long long)r * sr;
        double cc = div_const(sqrt(T[o]), p.Ama, p.inv_Ama);
        double fp[5], fm[5];
        if (UNI) {
            const DirConst &dc = p.dc[DIR];
            sw_split_pre<EPS0>(d[o] * p.tmp0, u[o], v[o], w[o], cc, dc.A[0], dc.A[1], dc.A[2], dc.ss,
                         dc.An[0], dc.An[1], dc.An[2], p, fp, fm);
        } else {
            sw_split(d[o] * p.tmp0, u[o], v[o], w[o], cc, metric<false>(p, mA, o), metric<false>(p, mA + 1, o),
                     metric<false>(p, mA + 2, o), p.Gamma, p.epsl_sw, p.split_C1, p.split_C3, fp, fm);
        }
        int pi = spos<DIR>(s, r);
#pragma unroll
        for (int m = 0; m < 5; m++) { spl[m * NP + pi] = fp[m]; spl[(5 + m) * NP + pi] = fm[m]; }
    }
    __syncthreads();

    // ---- A2: face records and the face order
    for (int fi = threadIdx.x; fi < NF; fi += blockDim.x) {
        int fs, r;
        if (DIR == 0) { fs = fi % (TS + 1); r = fi / (TS + 1); }
        else          { r = fi % R; fs = fi / R; }
        int F = s0 - 1 + fs;
        bool valid = !(r0 + r >= nr || F > n - 1);
        int hflag = 2;
        if (valid && hybrid) {
            long long fq;
            if (DIR == 0)      fq = (long long)(F + 1) + (long long)(p.nx + 1) * ((long long)(r0 + r) + (long long)p.ny * c3);
            else if (DIR == 1) fq = (long long)(r0 + r) + (long long)p.nx * ((long long)(F + 1) + (long long)(p.ny + 1) * c3);
            else               fq = (long long)(r0 + r) + (long long)p.nx * ((long long)c3 + (long long)p.ny * (F + 1));
            hflag = flags[fq];
        }
        bool proj = valid && char_scheme && !(hybrid && hflag == 1);
        if (proj) {
            long long o0 = base + (long long)(fs + 3) * sd + (long long)r * sr;   // cell F
            long long o1 = o0 + sd;                                                // cell F+1
            double c0v = div_const(sqrt(T[o0]), p.Ama, p.inv_Ama);
            double c1v = div_const(sqrt(T[o1]), p.Ama, p.inv_Ama);
            double u1 = (u[o0] + u[o1]) * 0.5, v1 = (v[o0] + v[o1]) * 0.5, w1 = (w[o0] + w[o1]) * 0.5;
            double c1 = (c0v + c1v) * 0.5;
            if (UNI) {
                const DirConst &dc = p.dc[DIR];
                double KK = (p.Gamma - 1.0) / (c1 * c1);
                double *rr = rec + fi;
                rr[FU * NF] = u1; rr[FV * NF] = v1; rr[FW * NF] = w1; rr[FC * NF] = c1; rr[FKK * NF] = KK;
                rr[FX1 * NF] = 1.0 / (2.0 * c1);
                double v2 = (u1 * u1 + v1 * v1 + w1 * w1) * 0.5;
                rr[FV2 * NF] = v2;
                rr[FUN * NF] = u1 * dc.n[0] + v1 * dc.n[1] + w1 * dc.n[2];
                rr[FH * NF] = v2 + 1.0 / KK;
                rr[FN1 * NF] = dc.n[0]; rr[FN2 * NF] = dc.n[1]; rr[FN3 * NF] = dc.n[2];
                rr[FL1 * NF] = dc.l[0]; rr[FL2 * NF] = dc.l[1]; rr[FL3 * NF] = dc.l[2];
                rr[FM1 * NF] = dc.m[0]; rr[FM2 * NF] = dc.m[1]; rr[FM3 * NF] = dc.m[2];
            } else {
                make_record(u1, v1, w1, c1,
                            (metric<false>(p, mA, o0) + metric<false>(p, mA, o1)) * 0.5,
                            (metric<false>(p, mA + 1, o0) + metric<false>(p, mA + 1, o1)) * 0.5,
                            (metric<false>(p, mA + 2, o0) + metric<false>(p, mA + 2, o1)) * 0.5,
                            p, rec + fi, NF);
            }
        }
        // face code: bits 0-9 index, bits 10-13 flag, bit 14 projected; -1 = no face
        short code = (short)(fi | (hflag << 10) | (proj ? (1 << 14) : 0));
        if (!valid) code = -1;
        list[NF + fi] = code;
        if (proj) atomicAdd(&nchar, 1);
    }
    __syncthreads();
    // Faces with a projection go first so the two costs do not share warps.
    // Slots come from shared counters; the order inside each class does not
    // change any result (every face writes its own flux slot).
    const int nproj = nchar;
    __shared__ int cnt[2];
    if (threadIdx.x < 2) cnt[threadIdx.x] = 0;
    __syncthreads();
    for (int fi = threadIdx.x; fi < NF; fi += blockDim.x) {
        short code = list[NF + fi];
        int slot;
        if (code < 0) continue;
        if (nproj == 0) slot = atomicAdd(&cnt[1], 1);
        else if (code & (1 << 14)) slot = atomicAdd(&cnt[0], 1);
        else slot = nproj + atomicAdd(&cnt[1], 1);
        list[slot] = code;
    }
    __syncthreads();
    const int nvalid = cnt[0] + cnt[1];

    // ---- B: one thread per (face, sign)
    for (int t = threadIdx.x; t < 2 * nvalid; t += blockDim.x) {
        int sign = t >= nvalid;
        short code = list[t - sign * nvalid];
        int fi = code & 1023, hflag = (code >> 10) & 15;
        bool proj = (code >> 14) & 1;
        int fs, r;
        if (DIR == 0) { fs = fi % (TS + 1); r = fi / (TS + 1); }
        else          { r = fi % R; fs = fi / R; }
        const double *sp = spl + (sign * 5) * NP + spos<DIR>(fs, r);
        constexpr int KS = DIR == 0 ? 1 : R;     // stencil stride in shared memory
        double out[5];
        if (comp_none) {
#pragma unroll
            for (int m = 0; m < 5; m++) out[m] = 0.0;
        } else if (proj) {
            double fv[5][8];
#pragma unroll
            for (int m = 0; m < 5; m++)
#pragma unroll
                for (int k = 0; k < 8; k++) fv[m][k] = sp[m * NP + k * KS];
            const double *rr = rec + fi;
#pragma unroll
            for (int c = 0; c < 5; c++) {
                double Lr[5], vals[8], Rc[5];
                L_row(rr, NF, c, Lr);
#pragma unroll
                for (int k = 0; k < 8; k++) vals[k] = dot5(Lr, fv[0][k], fv[1][k], fv[2][k], fv[3][k], fv[4][k]);
                double res = recon_one(p, scheme, hflag, sign, vals);
                R_col(rr, NF, c, Rc);
                if (c == 0) {
#pragma unroll
                    for (int m = 0; m < 5; m++) out[m] = Rc[m] * res;
                } else {
#pragma unroll
                    for (int m = 0; m < 5; m++) out[m] = out[m] + Rc[m] * res;
                }
            }
        } else {
#pragma unroll
            for (int m = 0; m < 5; m++) {
                double vals[8];
#pragma unroll
                for (int k = 0; k < 8; k++) vals[k] = sp[m * NP + k * KS];
                int hf = hflag;
                if (hybrid && !char_scheme && m > 0 && p.nochar_comp_flag) hf = p.nochar_comp_flag;
                out[m] = recon_one(p, scheme, hf, sign, vals);
            }
        }
#pragma unroll
        for (int m = 0; m < 5; m++) hat[(sign * 5 + m) * NF + fi] = out[m];
    }
    __syncthreads();

    // ---- C: du of each tile cell (x+ then x- for every component)
    const double h = t_h<DIR>(p), ih = p.inv_h[DIR];
    for (int t = threadIdx.x; t < NC; t += blockDim.x) {
        int s, r;
        if (DIR == 0) { s = t % TS; r = t / TS; }
        else          { r = t % R; s = t / R; }
        int X = s0 + s;
        if (r0 + r >= nr || X > n - 1) continue;
        long long o = base + (long long)(s + 4) * sd + (long long)r * sr;
        double aj = metric<UNI>(p, M_AJAC, o);
        int i, j, k;
        if (DIR == 0)      { i = X; j = r0 + r; k = c3; }
        else if (DIR == 1) { i = r0 + r; j = X; k = c3; }
        else               { i = r0 + r; j = c3; k = X; }
        long long ci = in_index(p, i, j, k);
        int fr = (DIR == 0) ? (s + 1) + (TS + 1) * r : r + R * (s + 1);
        int fl = (DIR == 0) ? s + (TS + 1) * r : r + R * s;
#pragma unroll
        for (int m = 0; m < 5; m++) {
            double acc = (DIR == 0) ? 0.0 : p.du[m * p.N + ci];
            acc += div_const(-aj * (hat[m * NF + fr] - hat[m * NF + fl]), h, ih);
            acc += div_const(-aj * (hat[(5 + m) * NF + fr] - hat[(5 + m) * NF + fl]), h, ih);
            p.du[m * p.N + ci] = acc;
        }
    }
}

template <int DIR, bool UNI, bool EPS0, int MINB>
static cudaError_t launch_sweep2(const Params &p, cudaStream_t st) {
    using S = Tile<DIR>;
    constexpr int NP = (S::TS + 8) * S::R, NF = (S::TS + 1) * S::R;
    const bool chars = p.charteric && (p.scheme_invis == 304 || p.scheme_invis == 305 || p.scheme_invis == 310);
    size_t smem = sizeof(double) * (10 * NP + 10 * NF + (chars ? FP_N * NF : 0));
    int n = DIR == 0 ? p.nx : (DIR == 1 ? p.ny : p.nz);
    int nr = DIR == 0 ? p.ny : p.nx;
    int n3 = DIR == 2 ? p.ny : p.nz;
    static size_t attr_bytes = 0;
    if (smem > attr_bytes) {
        cudaError_t e = cudaFuncSetAttribute(k_sweep2<DIR, UNI, EPS0, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        attr_bytes = smem;
    }
    dim3 grid((n + S::TS - 1) / S::TS, (nr + S::R - 1) / S::R, n3);
    k_sweep2<DIR, UNI, EPS0, MINB><<<grid, S::THREADS, smem, st>>>(p);
    return cudaGetLastError();
}

template <bool UNI, bool EPS0, int MINB>
static cudaError_t launch_sweeps2_m(const Params &p, cudaStream_t st) {
    cudaError_t e;
    if ((e = launch_sweep2<0, UNI, EPS0, MINB>(p, st)) != cudaSuccess) return e;
    if ((e = launch_sweep2<1, UNI, EPS0, MINB>(p, st)) != cudaSuccess) return e;
    return launch_sweep2<2, UNI, EPS0, MINB>(p, st);
}
template <bool UNI, bool EPS0>
static cudaError_t launch_sweeps2_t(const Params &p, cudaStream_t st) {
    return p.sweep_impl == 3 ? launch_sweeps2_m<UNI, EPS0, 3>(p, st) : launch_sweeps2_m<UNI, EPS0, 4>(p, st);
}

cudaError_t launch_sweeps2(const Params &p, cudaStream_t st) {
    // the EPSL_SW = 0 shortcut only exists on the precomputed (uniform) path
    if (p.uniform_metrics)
        return p.epsl_sw == 0.0 ? launch_sweeps2_t<true, true>(p, st) : launch_sweeps2_t<true, false>(p, st);
    return launch_sweeps2_t<false, false>(p, st);
}

// per-direction constants of a uniform grid, formed on the device with the
// same code the field path uses (sw_split's |A| and A/|A|, the face basis)
__global__ void k_dirconst(Params p, DirConst *out) {
    for (int dd = 0; dd < 3; dd++) {
        int mA = M_AKX + 3 * dd;
        double A1 = p.mc[mA], A2 = p.mc[mA + 1], A3 = p.mc[mA + 2];
        DirConst c;
        c.A[0] = A1; c.A[1] = A2; c.A[2] = A3;
        double ss = sqrt(A1 * A1 + A2 * A2 + A3 * A3);
        c.ss = ss;
        double inv = 1.0 / ss;
        c.An[0] = A1 * inv; c.An[1] = A2 * inv; c.An[2] = A3 * inv;
        CharPara cp;
        // face average of a constant metric is the constant itself
        char_para(0.0, 0.0, 0.0, 1.0, (A1 + A1) * 0.5, (A2 + A2) * 0.5, (A3 + A3) * 0.5, p.Gamma, cp);
        c.n[0] = cp.n1; c.n[1] = cp.n2; c.n[2] = cp.n3;
        c.l[0] = cp.l1; c.l[1] = cp.l2; c.l[2] = cp.l3;
        c.m[0] = cp.m1; c.m[1] = cp.m2; c.m[2] = cp.m3;
        out[dd] = c;
    }
}

cudaError_t compute_dirconst(Params &p, DirConst *dev_scratch, cudaStream_t st) {
    k_dirconst<<<1, 1, 0, st>>>(p, dev_scratch);
    cudaError_t e = cudaMemcpyAsync(p.dc, dev_scratch, sizeof(DirConst) * 3, cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(st);
}


}  // namespace ocfd
