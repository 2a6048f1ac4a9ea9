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
#include "ocfd_device.cuh"

#include <cuda_runtime.h>

namespace ocfd {

template <int DIR> struct Tile;
template <> struct Tile<0> { static constexpr int TS = 64, R = 2, THREADS = 128; };
template <> struct Tile<1> { static constexpr int TS = 16, R = 8, THREADS = 128; };
template <> struct Tile<2> { static constexpr int TS = 16, R = 8, THREADS = 128; };

// face record kept in shared memory for characteristic schemes
constexpr int FP_N = 18;   // u1 v1 w1 c1 KK X1 v2 un H  n1 n2 n3 l1 l2 l3 m1 m2 m3
enum { FU = 0, FV, FW, FC, FKK, FX1, FV2, FUN, FH, FN1, FN2, FN3, FL1, FL2, FL3, FM1, FM2, FM3 };

template <int DIR> __device__ __forceinline__ int t_ndir(const Params &p) { return DIR == 0 ? p.nx : (DIR == 1 ? p.ny : p.nz); }
template <int DIR> __device__ __forceinline__ int t_nrow(const Params &p) { return DIR == 0 ? p.ny : p.nx; }
template <int DIR> __device__ __forceinline__ long long t_sdir(const Params &p) { return DIR == 0 ? 1LL : (DIR == 1 ? p.ys : p.zs); }
template <int DIR> __device__ __forceinline__ long long t_srow(const Params &p) { return DIR == 0 ? p.ys : 1LL; }
template <int DIR> __device__ __forceinline__ long long t_s3rd(const Params &p) { return DIR == 2 ? p.ys : p.zs; }
template <int DIR> __device__ __forceinline__ double t_h(const Params &p) { return DIR == 0 ? p.hx : (DIR == 1 ? p.hy : p.hz); }

// Steger-Warming split with the direction's |A| and A/|A| already formed
// (same operations as sw_split, src/OCFD_split.cu:92-142)
// EPS0: EPSL_SW = 0, where sqrt(E*E + 0) is exactly |E| (the square root of
// a correctly rounded square returns the operand's magnitude), so the three
// square roots reduce to fabs with the same result.
template <bool EPS0>
__device__ __forceinline__ void sw_split_pre(double tmp0, double u, double v, double w, double cc,
                                             double A1, double A2, double A3, double ss,
                                             double An1, double An2, double An3,
                                             const Params &p, double *fp, double *fm) {
    const double eps = p.epsl_sw, G = p.Gamma;
    double E1 = A1 * u + A2 * v + A3 * w;
    double E2 = E1 - cc * ss;
    double E3 = E1 + cc * ss;
    double E1P = (E1 + (EPS0 ? fabs(E1) : sqrt(E1 * E1 + eps * eps))) * 0.50;
    double E2P = (E2 + (EPS0 ? fabs(E2) : sqrt(E2 * E2 + eps * eps))) * 0.50;
    double E3P = (E3 + (EPS0 ? fabs(E3) : sqrt(E3 * E3 + eps * eps))) * 0.50;
    double E1M = E1 - E1P, E2M = E2 - E2P, E3M = E3 - E3P;
    double uc1 = u - cc * An1, uc2 = u + cc * An1;
    double vc1 = v - cc * An2, vc2 = v + cc * An2;
    double wc1 = w - cc * An3, wc2 = w + cc * An3;
    double vvc1 = (uc1 * uc1 + vc1 * vc1 + wc1 * wc1) * 0.50;
    double vvc2 = (uc2 * uc2 + vc2 * vc2 + wc2 * wc2) * 0.50;
    double vv = (G - 1.0) * (u * u + v * v + w * w);
    double W2 = p.split_C3 * cc * cc;
    const double C1 = p.split_C1;
    fp[0] = tmp0 * (C1 * E1P + E2P + E3P);
    fp[1] = tmp0 * (C1 * E1P * u + E2P * uc1 + E3P * uc2);
    fp[2] = tmp0 * (C1 * E1P * v + E2P * vc1 + E3P * vc2);
    fp[3] = tmp0 * (C1 * E1P * w + E2P * wc1 + E3P * wc2);
    fp[4] = tmp0 * (E1P * vv + E2P * vvc1 + E3P * vvc2 + W2 * (E2P + E3P));
    fm[0] = tmp0 * (C1 * E1M + E2M + E3M);
    fm[1] = tmp0 * (C1 * E1M * u + E2M * uc1 + E3M * uc2);
    fm[2] = tmp0 * (C1 * E1M * v + E2M * vc1 + E3M * vc2);
    fm[3] = tmp0 * (C1 * E1M * w + E2M * wc1 + E3M * wc2);
    fm[4] = tmp0 * (E1M * vv + E2M * vvc1 + E3M * vvc2 + W2 * (E2M + E3M));
}

// row c of the left eigenvector matrix from a face record (ptoc,
// src/OCFD_flux_charteric.cu:617-676); r[k] = record value k
__device__ __forceinline__ void L_row(const double *r, int nf, int c, double S[5]) {
    const double u1 = r[FU * nf], v1 = r[FV * nf], w1 = r[FW * nf], KK = r[FKK * nf];
    switch (c) {
    case 0: S[0] = 1.0 - KK * r[FV2 * nf]; S[1] = KK * u1; S[2] = KK * v1; S[3] = KK * w1; S[4] = -KK; break;
    case 1: {
        double l1 = r[FL1 * nf], l2 = r[FL2 * nf], l3 = r[FL3 * nf];
        S[0] = -(u1 * l1 + v1 * l2 + w1 * l3); S[1] = l1; S[2] = l2; S[3] = l3; S[4] = 0.0; break; }
    case 2: {
        double m1 = r[FM1 * nf], m2 = r[FM2 * nf], m3 = r[FM3 * nf];
        double n1 = r[FN1 * nf], n2 = r[FN2 * nf], n3 = r[FN3 * nf];
        double l1 = r[FL1 * nf], l2 = r[FL2 * nf], l3 = r[FL3 * nf];
        S[0] = -(u1 * m1 + v1 * m2 + w1 * m3);
        S[1] = n2 * l3 - n3 * l2; S[2] = n3 * l1 - n1 * l3; S[3] = n1 * l2 - n2 * l1; S[4] = 0.0; break; }
    default: {
        double X1 = r[FX1 * nf], un = r[FUN * nf], v2 = r[FV2 * nf];
        double n1 = r[FN1 * nf], n2 = r[FN2 * nf], n3 = r[FN3 * nf];
        double s41 = KK * v2 * 0.5 + X1 * un;
        double s42 = -X1 * n1 - KK * u1 * 0.5;
        double s43 = -X1 * n2 - KK * v1 * 0.5;
        double s44 = -X1 * n3 - KK * w1 * 0.5;
        if (c == 3) { S[0] = s41; S[1] = s42; S[2] = s43; S[3] = s44; S[4] = KK * 0.5; }
        else { S[0] = s41 - 2 * X1 * un; S[1] = 2 * X1 * n1 + s42; S[2] = 2 * X1 * n2 + s43;
               S[3] = 2 * X1 * n3 + s44; S[4] = KK * 0.5; }
        break; }
    }
}

// column c of the right eigenvector matrix (ctop, :678-752)
__device__ __forceinline__ void R_col(const double *r, int nf, int c, double S[5]) {
    const double u1 = r[FU * nf], v1 = r[FV * nf], w1 = r[FW * nf], c1 = r[FC * nf];
    switch (c) {
    case 0: S[0] = 1.0; S[1] = u1; S[2] = v1; S[3] = w1; S[4] = r[FV2 * nf]; break;
    case 1: { double l1 = r[FL1 * nf], l2 = r[FL2 * nf], l3 = r[FL3 * nf];
        S[0] = 0.0; S[1] = l1; S[2] = l2; S[3] = l3; S[4] = u1 * l1 + v1 * l2 + w1 * l3; break; }
    case 2: { double n1 = r[FN1 * nf], n2 = r[FN2 * nf], n3 = r[FN3 * nf];
        double l1 = r[FL1 * nf], l2 = r[FL2 * nf], l3 = r[FL3 * nf];
        S[0] = 0.0; S[1] = n2 * l3 - n3 * l2; S[2] = n3 * l1 - n1 * l3; S[3] = n1 * l2 - n2 * l1;
        S[4] = u1 * r[FM1 * nf] + v1 * r[FM2 * nf] + w1 * r[FM3 * nf]; break; }
    default: { double n1 = r[FN1 * nf], n2 = r[FN2 * nf], n3 = r[FN3 * nf];
        double s24 = u1 - c1 * n1, s34 = v1 - c1 * n2, s44 = w1 - c1 * n3;
        double s54 = r[FH * nf] - c1 * r[FUN * nf];
        if (c == 3) { S[0] = 1.0; S[1] = s24; S[2] = s34; S[3] = s44; S[4] = s54; }
        else { S[0] = 1.0; S[1] = 2 * u1 - s24; S[2] = 2 * v1 - s34; S[3] = 2 * w1 - s44;
               S[4] = 2 * r[FH * nf] - s54; }
        break; }
    }
}

// face record from face-averaged values (get_para_charteric_*, :330-418)
__device__ __forceinline__ void make_record(double u1, double v1, double w1, double c1,
                                            double a1, double a2, double a3, const Params &p,
                                            double *r, int nf) {
    CharPara cp;
    char_para(u1, v1, w1, c1, a1, a2, a3, p.Gamma, cp);
    r[FU * nf] = u1; r[FV * nf] = v1; r[FW * nf] = w1; r[FC * nf] = c1; r[FKK * nf] = cp.KK;
    r[FX1 * nf] = 1.0 / (2.0 * c1);
    double v2 = (u1 * u1 + v1 * v1 + w1 * w1) * 0.5;
    r[FV2 * nf] = v2;
    r[FUN * nf] = u1 * cp.n1 + v1 * cp.n2 + w1 * cp.n3;
    r[FH * nf] = v2 + 1.0 / cp.KK;
    r[FN1 * nf] = cp.n1; r[FN2 * nf] = cp.n2; r[FN3 * nf] = cp.n3;
    r[FL1 * nf] = cp.l1; r[FL2 * nf] = cp.l2; r[FL3 * nf] = cp.l3;
    r[FM1 * nf] = cp.m1; r[FM2 * nf] = cp.m2; r[FM3 * nf] = cp.m3;
}

// UP7 (src/OCFD_Schemes.cu:865-907) with the /420 done by div_const
__device__ __forceinline__ double up7_p_q(const double *s) {
    return div_const(-3.0*s[0] + 25.0*s[1] - 101.0*s[2] + 319.0*s[3] + 214.0*s[4]
                     - 38.0*s[5] + 4.0*s[6], 420.0, 1.0 / 420.0);
}
__device__ __forceinline__ double up7_m_q(const double *s) {
    return div_const(-3.0*s[7] + 25.0*s[6] - 101.0*s[5] + 319.0*s[4] + 214.0*s[3]
                     - 38.0*s[2] + 4.0*s[1], 420.0, 1.0 / 420.0);
}

// reconstruction of one (face, sign) of one field from v[0..7] = f(F-3..F+4)
__device__ __forceinline__ double recon_one(const Params &p, int scheme, int hflag, int sign, const double *v) {
    if (sign == 0) {
        switch (scheme) {
        case 301: return up7_p_q(v);
        case 302: return weno5_p(v);
        case 303: return weno7_p(v);
        case 304: return symbo_p(0, p.tv_lim, p.tv_max, v);
        case 305: return symbo_p(1, p.tv_lim, p.tv_max, v);
        case 306: return nnd2_p(v);
        case 307: return omp6_p(0, v);
        case 308: return omp6_p(1, v);
        case 309: return omp6_p(2, v);
        default:
            if (hflag == 1) return up7_p_q(v);
            if (hflag == 2) return weno7_p(v);
            return weno5_p(v);
        }
    }
    switch (scheme) {
    case 301: return up7_m_q(v);
    case 302: return weno5_m(v);
    case 303: return weno7_m(v);
    case 304: return symbo_m(0, p.tv_lim, p.tv_max, v);
    case 305: return symbo_m(1, p.tv_lim, p.tv_max, v);
    case 306: return nnd2_m(v);
    case 307: return omp6_m(0, v);
    case 308: return omp6_m(1, v);
    case 309: return omp6_m(2, v);
    default:
        if (hflag == 1) return up7_m_q(v);
        if (hflag == 2) return weno7_m(v);
        return weno5_m(v);
    }
}

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


// ===========================================================================
// Third-generation sweeps: no block barriers.
//   x: a warp owns 32 consecutive faces of one row; its lanes compute the
//      40 split points of the strip into warp-private shared memory
//      (__syncwarp only), then each lane forms its face flux (both signs,
//      all five fields) and the du of its cell.
//   y, z: each lane owns one x column and marches along the sweep direction,
//      keeping the split values of the last 8 points in a lane-private ring
//      in shared memory; every point is split once, every face is formed
//      once, and du(X) uses the face kept from the previous step.
// Boundary closures of non-periodic directions (src/OCFD_bound_Scheme.cu)
// are applied per face; non-reflecting faces and the characteristic
// kernels' first-order boundary fluxes per cell.
// ===========================================================================

// one-sided WENO5 candidates used by the closures, src/OCFD_bound_Scheme.cu:554-745;
// s[0..4] = f(i-2..i+2)
__device__ __forceinline__ double w5_p_left(const double *s) {
    double S0 = 0.0, tmp; const double ep = 1e-6;
    tmp = s[2] - 2.0*s[3] + s[4]; S0 += 13*tmp*tmp;
    tmp = 3.0*s[2] - 4.0*s[3] + s[4]; S0 += 3*tmp*tmp;
    double a0 = 1.0/((12.0*ep + S0)*(12.0*ep + S0));
    double q03 = (2.0*s[2] + 5.0*s[3] - s[4]);
    return a0*q03/(6.0*a0);
}
__device__ __forceinline__ double w5_m_left(const double *s) {
    double S2 = 0.0, tmp; const double ep = 1e-6;
    tmp = s[4] - 2.0*s[3] + s[2]; S2 += 13*tmp*tmp;
    tmp = s[4] - 4.0*s[3] + 3.0*s[2]; S2 += 3*tmp*tmp;
    double a2 = 1.0/((12.0*ep + S2)*(12.0*ep + S2));
    double q23 = (2.0*s[4] - 7.0*s[3] + 11.0*s[2]);
    return a2*q23/(6.0*a2);
}
__device__ __forceinline__ double w5_p_right_plus(const double *s) {
    double S1 = 0.0, S2 = 0.0, tmp; const double ep = 1e-6;
    tmp = s[1] - 2.0*s[2] + s[3]; S1 += 13*tmp*tmp;
    tmp = s[1] - s[3]; S1 += 3*tmp*tmp;
    double a1 = 6.0/((12.0*ep + S1)*(12.0*ep + S1));
    double q13 = (-s[1] + 5.0*s[2] + 2.0*s[3]);
    tmp = s[0] - 2.0*s[1] + s[2]; S2 += 13*tmp*tmp;
    tmp = s[0] - 4.0*s[1] + 3.0*s[2]; S2 += 3*tmp*tmp;
    double a2 = 1.0/((12.0*ep + S2)*(12.0*ep + S2));
    double q23 = (2.0*s[0] - 7.0*s[1] + 11.0*s[2]);
    return (a1*q13 + a2*q23)/(6.0*(a1 + a2));
}
__device__ __forceinline__ double w5_p_left_plus(const double *s) {
    double S0 = 0.0, S1 = 0.0, tmp; const double ep = 1e-6;
    tmp = s[2] - 2.0*s[3] + s[4]; S0 += 13*tmp*tmp;
    tmp = 3.0*s[2] - 4.0*s[3] + s[4]; S0 += 3*tmp*tmp;
    double a0 = 3.0/((12.0*ep + S0)*(12.0*ep + S0));
    double q03 = (2.0*s[2] + 5.0*s[3] - s[4]);
    tmp = s[1] - 2.0*s[2] + s[3]; S1 += 13*tmp*tmp;
    tmp = s[1] - s[3]; S1 += 3*tmp*tmp;
    double a1 = 6.0/((12.0*ep + S1)*(12.0*ep + S1));
    double q13 = (-s[1] + 5.0*s[2] + 2.0*s[3]);
    return (a0*q03 + a1*q13)/(6.0*(a0 + a1));
}
__device__ __forceinline__ double w5_m_right_plus(const double *s) {
    double S0 = 0.0, S1 = 0.0, tmp; const double ep = 1e-6;
    tmp = s[2] - 2.0*s[1] + s[0]; S0 += 13*tmp*tmp;
    tmp = 3.0*s[2] - 4.0*s[1] + s[0]; S0 += 3*tmp*tmp;
    double a0 = 3.0/((12.0*ep + S0)*(12.0*ep + S0));
    double q03 = (2.0*s[2] + 5.0*s[1] - s[0]);
    tmp = s[3] - 2.0*s[2] + s[1]; S1 += 13*tmp*tmp;
    tmp = s[3] - s[1]; S1 += 3*tmp*tmp;
    double a1 = 6.0/((12.0*ep + S1)*(12.0*ep + S1));
    double q13 = (-s[3] + 5.0*s[2] + 2.0*s[1]);
    return (a0*q03 + a1*q13)/(6.0*(a0 + a1));
}
__device__ __forceinline__ double w5_m_left_plus(const double *s) {
    double S1 = 0.0, S2 = 0.0, tmp; const double ep = 1e-6;
    tmp = s[3] - 2.0*s[2] + s[1]; S1 += 13*tmp*tmp;
    tmp = s[3] - s[1]; S1 += 3*tmp*tmp;
    double a1 = 6.0/((12.0*ep + S1)*(12.0*ep + S1));
    double q13 = (-s[3] + 5.0*s[2] + 2.0*s[1]);
    tmp = s[4] - 2.0*s[3] + s[2]; S2 += 13*tmp*tmp;
    tmp = s[4] - 4.0*s[3] + 3.0*s[2]; S2 += 3*tmp*tmp;
    double a2 = 1.0/((12.0*ep + S2)*(12.0*ep + S2));
    double q23 = (2.0*s[4] - 7.0*s[3] + 11.0*s[2]);
    return (a1*q13 + a2*q23)/(6.0*(a1 + a2));
}

// Closure of face F+1/2 of a line of n cells, v[t] = f(F-3+t); returns true
// when it replaces the interior scheme (OCFD_bound_scheme_kernel_p / _m with
// boundp1/boundp2/boundm1/boundm2, :748-944).  KA, KB: stencil extents
// (-ia1, ib1) of the reference kernel of this sign.
__device__ __forceinline__ bool closure(int sign, bool lo, bool hi, int KA, int KB, int F, int n,
                                        const double *v, double &out) {
    int c = F + 1;
    if (sign == 0) {
        if (lo && c <= KA) {
            if (c == 0) out = v[4];
            else if (c == 1) out = w5_p_left(v + 1);
            else if (c == 2) out = w5_p_left_plus(v + 1);
            else out = weno5_p(v);
            return true;
        }
        if (hi) {
            int t = c - (n + 1);
            if (t >= -KB) {
                if (t == -1) out = v[3] + 0.5 * minmod2(v[3] - v[2], v[3] - v[2]);
                else if (t == -2) out = w5_p_right_plus(v + 1);
                else out = weno5_p(v);
                return true;
            }
        }
        return false;
    }
    if (lo && c < KA) {
        if (c == 0) out = w5_m_left(v + 2);
        else if (c == 1) out = w5_m_left_plus(v + 2);
        else out = weno5_m(v);
        return true;
    }
    if (hi) {
        int t = c - (n + 1);
        if (t >= -KB - 1) {
            if (t == -1) out = v[3];
            else if (t == -2) out = v[4] - 0.5 * minmod2(v[4] - v[3], v[4] - v[3]);
            else if (t == -3) out = w5_m_right_plus(v + 2);
            else out = weno5_m(v);
            return true;
        }
    }
    return false;
}

// stencil extents of the reference kernels per scheme and sign (P: -ia1, ib1)
__device__ __forceinline__ void extents(int scheme, bool chart, int sign, int &KA, int &KB) {
    if (chart) { KA = sign ? 4 : 3; KB = sign ? 3 : 4; return; }
    switch (scheme) {
    case 302: case 306: KA = 2; KB = 2; break;
    case 303: KA = 3; KB = 3; break;
    default: KA = sign ? 4 : 3; KB = sign ? 3 : 4; break;
    }
}

}  // namespace ocfd
