// ocfd_device.cuh -- device-side arithmetic of the RHS path (sm_100a, FP64).
//
// Point formulas restate the reference scheme kernels; each keeps the
// reference's expression order so nvcc contracts them the same way it does
// the reference build (both use the default -fmad=true).  References are to
// the OpenCFD-SCU tree.
#pragma once
#include <cstdint>

#define OCFD_LAP 4

namespace ocfd {

// per-direction constants of a uniform grid (see k_dirconst)
struct DirConst {
    double A[3];       // metric row of the direction (Akx Aky Akz for x, ...)
    double ss;         // |A|
    double An[3];      // A / |A|
    double n[3], l[3], m[3];   // characteristic basis of a face
};

// ---------------------------------------------------------------------------
// kernel parameter block (passed by value to every kernel)
// ---------------------------------------------------------------------------
struct Params {
    int nx, ny, nz;
    int pitch;              // x stride of LAP-box fields, elements
    long long ys, zs;       // y / z strides of LAP-box fields
    long long lapN;         // elements per LAP-box field
    long long N;            // interior cells
    double hx, hy, hz;
    double Ama, Gamma, epsl_sw, Cv, Tsb, amu_C0, tmp0, split_C1, split_C3, vis_c, dt, p00;
    double tv_lim, tv_max;
    double dp1, dp2;
    int scheme_invis, scheme_vis, charteric;
    int nochar_comp_flag;   // flag of components 1-4, non-characteristic hybrid (0 = face flag)
    int periodic[3];
    // whether the local z faces k = 0 / k = nz-1 are faces of the whole grid
    // (1 on one GPU; with the grid split in z, only on the first / last slab)
    int zface_lo, zface_hi;
    // faces of each direction: boundary closures where DIF_BOUND is 1
    // (OCFD_bound, src/OCFD_bound_Scheme.cu:436-469) and the NON_REFLETION
    // value (OCFD_bound_non_ref, :352-433); has_bnd: any of them is set
    int bnd_lo[3], bnd_hi[3];
    int nonref_lo[3], nonref_hi[3];
    int has_bnd;
    // state
    double *prim[5];        // d u v w T on the LAP box
    // precision form (mixed = 1): the primitives the stencils read, the stage
    // RHS and the viscous fluxes in FP32; the conserved state, the RK
    // update and cons->prim stay FP64 (null when the form is off)
    int mixed;
    float *prim32[5];
    float *du32;
    float *ev32;
    const double *met[13];  // Axx Ayy Azz Akx Aky Akz Aix Aiy Aiz Asx Asy Asz Ajac (LAP box)
    double *f, *fn, *du;    // [5][nz][ny][nx]
    double *ev;             // [12] LAP-box fields: Ev1..4 of x, then y, then z
    int8_t *flag[3];        // hybrid scheme flags (nx+1)ny nz, nx(ny+1)nz, nx ny(nz+1)
    // uniform grids: every metric field is one value; kernels read mc[] instead
    int uniform_metrics;
    double mc[13];
    DirConst dc[3];
    double inv_h[3], inv_Ama;   // reciprocals for div_const
    int sweep_impl;         // 4: the walks chosen per direction (default); 5: every face through the in-loop dispatch; 6: the in-line walk
    // viscous divergence + RK of whole steps: 0 Ev tiles staged in shared
    // memory in the precision form, read through L1/L2 in FP64 (each the
    // faster there); 1 read through L1/L2; 2 staged
    int vis_impl;
    // cells whose du the call-free sweep leaves to the fix-up kernel, per
    // direction (interior cell indices; capacity N each), and their counts
    unsigned *defer[3];
    unsigned *defer_count;
    unsigned *flag_count;          // faces per direction whose hybrid flag is not 1 (sensor), or null
    // set to 1 by a kernel whose wait on a staged copy ran out (the host
    // reports it as an error at the next synchronisation)
    int *kerr;
    // shock filter (null when no filter is set): U after the stage-3 update
    // before the face re-projection (5 LAP-box fields) and the pressure
    // cons_to_pri leaves after the last stage (1 LAP-box field)
    double *flap;
    double *pfil;
    // precision form: the filter's pressure in FP32 (1 LAP-box field; the
    // filter's weights are formed from it, its U update stays FP64)
    float *pfil32;
    // boundary-condition family (IBC; 0 none, 108 compression corner): the
    // inflow profile [4][ny] (d,u,v,T), wall blowing shapes fx [nx], gz [nz],
    // first x of the upper inflow row, wall treatment (0 none, 1 TW > 0,
    // 2 TW <= 0), wall temperature and blowing amplitude
    int ibc;
    const double *bc_ub1, *bc_fx, *bc_gz;
    int bc_xbegin, bc_wall_mode;
    double bc_tw, bc_epsl;
};

// host transport of the z split (ocfd_b200_slab_transport in the C ABI):
// op 0 swaps the packed ghost planes with the neighbour ranks, op 1 sums a
// buffer over the ranks in place; type 0 FP64, 1 uint64, 2 uint32, 3 FP32
typedef int (*SlabTransport)(void *user, int op, void *send, void *recv, size_t count, int type);

enum { M_AXX = 0, M_AYY, M_AZZ, M_AKX, M_AKY, M_AKZ, M_AIX, M_AIY, M_AIZ,
       M_ASX, M_ASY, M_ASZ, M_AJAC };

// Bounds-checked build (make bounds: -DOCFD_BOUNDS, libocfd_b200_bounds.so).
// The index helpers and the walks' global accesses check their indexes; one
// outside its array sets error word 3 and is replaced by 0, so that the
// access stays inside the allocation and the call that ran the kernel
// reports the error.  The default build compiles the checks away.
#ifdef OCFD_BOUNDS
// the first failed check also leaves, after the error word, the source line
// of the check and the offending value (an index, or packed coordinates)
__device__ __forceinline__ bool bounds_ok(const Params &p, bool ok, int line, long long value) {
    if (!ok && p.kerr && atomicCAS(p.kerr, 0, 3) == 0) {
        p.kerr[1] = line;
        p.kerr[2] = (int)(value & 0xffffffffLL);
        p.kerr[3] = (int)(value >> 32);
    }
    return ok;
}
__device__ __forceinline__ long long bounds_idx(const Params &p, long long q, long long n, int line) {
    return bounds_ok(p, q >= 0 && q < n, line, q) ? q : 0;
}
#define OCFD_IDX(p, q, n) ::ocfd::bounds_idx((p), (q), (n), __LINE__)
#else
#define OCFD_IDX(p, q, n) (q)
#endif

__device__ __forceinline__ long long lap_index(const Params &p, int i, int j, int k) {
    // i,j,k are LAP-box coordinates (0 .. n+2*LAP-1)
#ifdef OCFD_BOUNDS
    if (!bounds_ok(p, i >= 0 && j >= 0 && k >= 0 && i < p.nx + 2 * OCFD_LAP && j < p.ny + 2 * OCFD_LAP &&
                          k < p.nz + 2 * OCFD_LAP, __LINE__,
                   (long long)(i & 0xfffff) | (long long)(j & 0xfffff) << 20 | (long long)(k & 0xfffff) << 40))
        return 0;
#endif
    return (long long)i + p.ys * j + p.zs * k;
}
// metric m at LAP offset o; UNI selects the constant of a uniform grid (the
// same value every cell would hold, so the arithmetic is unchanged)
template <bool UNI>
__device__ __forceinline__ double metric(const Params &p, int m, long long o) {
    if (UNI) return p.mc[m];
    return p.met[m][OCFD_IDX(p, o, p.lapN)];
}

__device__ __forceinline__ long long in_index(const Params &p, int i, int j, int k) {
#ifdef OCFD_BOUNDS
    if (!bounds_ok(p, i >= 0 && j >= 0 && k >= 0 && i < p.nx && j < p.ny && k < p.nz, __LINE__,
                   (long long)(i & 0xfffff) | (long long)(j & 0xfffff) << 20 | (long long)(k & 0xfffff) << 40))
        return 0;
#endif
    return (long long)i + (long long)p.nx * ((long long)j + (long long)p.ny * k);
}
// entries of direction d's hybrid flag array ((n_d + 1) along d)
__device__ __forceinline__ long long flag_entries(const Params &p, int d) {
    return (long long)(p.nx + (d == 0)) * (p.ny + (d == 1)) * (p.nz + (d == 2));
}
// entry q of direction d's flag array from a pointer fl into it (checked in
// the bounds build, where an entry outside the array reads as flag 2)
__device__ __forceinline__ int flag_at(const Params &p, int d, const int8_t *fl, long long q) {
#ifdef OCFD_BOUNDS
    const long long a = (long long)(fl - p.flag[d]) + q;
    if (!bounds_ok(p, a >= 0 && a < flag_entries(p, d), __LINE__, a)) return 2;
#endif
    return (int)fl[q];
}

// x / c for a run-time constant c with inv = RN(1/c): the product plus one
// FMA residual correction (Markstein) returns the correctly rounded quotient
// except in rare last-ulp cases, at 3 FP64 operations instead of a full
// IEEE division sequence.
__device__ __forceinline__ double div_const(double x, double c, double inv) {
    double q = x * inv;
    double r = fma(-q, c, x);
    return fma(r, inv, q);
}

// ---------------------------------------------------------------------------
// Steger-Warming splitting of one point, src/OCFD_split.cu:92-142
// ---------------------------------------------------------------------------
__device__ __forceinline__ void sw_split(double tmp0, double u, double v, double w, double cc,
                                         double A1, double A2, double A3, double G, double eps,
                                         double split_C1, double split_C3,
                                         double *fp, double *fm) {
    double ss = sqrt(A1 * A1 + A2 * A2 + A3 * A3);
    double E1 = A1 * u + A2 * v + A3 * w;
    double E2 = E1 - cc * ss;
    double E3 = E1 + cc * ss;
    ss = 1.0 / ss;
    A1 *= ss; A2 *= ss; A3 *= ss;
    double E1P = (E1 + sqrt(E1 * E1 + eps * eps)) * 0.50;
    double E2P = (E2 + sqrt(E2 * E2 + eps * eps)) * 0.50;
    double E3P = (E3 + sqrt(E3 * E3 + eps * eps)) * 0.50;
    double E1M = E1 - E1P, E2M = E2 - E2P, E3M = E3 - E3P;
    double uc1 = u - cc * A1, uc2 = u + cc * A1;
    double vc1 = v - cc * A2, vc2 = v + cc * A2;
    double wc1 = w - cc * A3, wc2 = w + cc * A3;
    double vvc1 = (uc1 * uc1 + vc1 * vc1 + wc1 * wc1) * 0.50;
    double vvc2 = (uc2 * uc2 + vc2 * vc2 + wc2 * wc2) * 0.50;
    double vv = (G - 1.0) * (u * u + v * v + w * w);
    double W2 = split_C3 * cc * cc;
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

// ---------------------------------------------------------------------------
// reconstruction point formulas.  Stencil convention for a face F+1/2:
// s[t] = f(F-3+t), t = 0..7, for both signs.
// ---------------------------------------------------------------------------

// WENO7 positive side, src/OCFD_Schemes.cu:616-663 (uses s[0..6])
__device__ __forceinline__ double weno7_p(const double *s) {
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
    const double e = 3.456e-4;
    double b0 = (e + S0) * (e + S0), b1 = (e + S1) * (e + S1);
    double b2 = (e + S2) * (e + S2), b3 = (e + S3) * (e + S3);
    double a0 =        b1 * b2 * b3;
    double a1 = (12.0) * b0 * b2 * b3;
    double a2 = (18.0) * b0 * b1 * b3;
    double a3 =  (4.0) * b0 * b1 * b2;
    double am = a0 + a1 + a2 + a3;
    double r = 0.0;
    tmp = -3.0*s[0] + 13.0*s[1] - 23.0*s[2] + 25.0*s[3]; r += a0*tmp;
    tmp =      s[1] -  5.0*s[2] + 13.0*s[3] +  3.0*s[4]; r += a1*tmp;
    tmp =     -s[2] +  7.0*s[3] +  7.0*s[4] -      s[5]; r += a2*tmp;
    tmp =  3.0*s[3] + 13.0*s[4] -  5.0*s[5] +      s[6]; r += a3*tmp;
    return r / (12.0*am);
}

// WENO7 negative side, src/OCFD_Schemes.cu:691-741; q[k] = s[k+1] (f(F-2..F+4))
__device__ __forceinline__ double weno7_m(const double *s8) {
    const double *s = s8 + 1;
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
    const double e = 3.456e-4;
    double b0 = (e + S0) * (e + S0), b1 = (e + S1) * (e + S1);
    double b2 = (e + S2) * (e + S2), b3 = (e + S3) * (e + S3);
    double a0 =        b1 * b2 * b3;
    double a1 = (12.0) * b0 * b2 * b3;
    double a2 = (18.0) * b0 * b1 * b3;
    double a3 =  (4.0) * b0 * b1 * b2;
    double am = a0 + a1 + a2 + a3;
    double r = 0.0;
    tmp = -3.0*s[6] + 13.0*s[5] - 23.0*s[4] + 25.0*s[3]; r += a0*tmp;
    tmp =      s[5] -  5.0*s[4] + 13.0*s[3] +  3.0*s[2]; r += a1*tmp;
    tmp =     -s[4] +  7.0*s[3] +  7.0*s[2] -      s[1]; r += a2*tmp;
    tmp =  3.0*s[3] + 13.0*s[2] -  5.0*s[1] +      s[0]; r += a3*tmp;
    return r / (12.0*am);
}

// WENO5 positive side, src/OCFD_Schemes.cu:1118-1151; q = s+1 (f(F-2..F+2))
__device__ __forceinline__ double weno5_p(const double *s8) {
    const double *s = s8 + 1;
    double S0 = 0.0, S1 = 0.0, S2 = 0.0, tmp;
    const double ep = 1e-6;
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
    return (a0*q03 + a1*q13 + a2*q23)/(6.0*(a0 + a1 + a2));
}

// WENO5 negative side, src/OCFD_Schemes.cu:1176-1208; q = s+2 (f(F-1..F+3))
__device__ __forceinline__ double weno5_m(const double *s8) {
    const double *s = s8 + 2;
    double S0 = 0.0, S1 = 0.0, S2 = 0.0, tmp;
    const double ep = 1e-6;
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
    return (a0*q03 + a1*q13 + a2*q23)/(6.0*(a0 + a1 + a2));
}

// UP7, src/OCFD_Schemes.cu:865-907
__device__ __forceinline__ double up7_p(const double *s) {
    return (-3.0*s[0] + 25.0*s[1] - 101.0*s[2] + 319.0*s[3] + 214.0*s[4]
            - 38.0*s[5] + 4.0*s[6])/420.0;
}
__device__ __forceinline__ double up7_m(const double *s) {
    return (-3.0*s[7] + 25.0*s[6] - 101.0*s[5] + 319.0*s[4] + 214.0*s[3]
            - 38.0*s[2] + 4.0*s[1])/420.0;
}

// sign / minmod, src/OCFD_Schemes.cu:766-797 (minmod4 keeps the fmin of the
// signed arguments as the reference writes it)
__device__ __forceinline__ double sgn1(double x2) { return x2 >= 0 ? 1.0 : -1.0; }
__device__ __forceinline__ double minmod2(double x1, double x2) {
    return 0.5*(sgn1(x1) + sgn1(x2))*fmin(fabs(x1), fabs(x2));
}
__device__ __forceinline__ double minmod4(double x1, double x2, double x3, double x4) {
    double m = 0.5*(sgn1(x1) + sgn1(x2));
    m = m*fabs(0.5*(sgn1(x1) + sgn1(x3)));
    m = m*fabs(0.5*(sgn1(x1) + sgn1(x4)));
    double t = fmin(fmin(x1, x2), fmin(x3, x4));
    return m*t;
}

// NND2, src/OCFD_Schemes.cu:800-837: P uses f(F-1..F+1), M uses f(F..F+2)
__device__ __forceinline__ double nnd2_p(const double *s8) {
    const double *s = s8 + 2;
    return s[1] + 0.5*minmod2(s[2] - s[1], s[1] - s[0]);
}
__device__ __forceinline__ double nnd2_m(const double *s8) {
    const double *s = s8 + 3;
    return s[1] + 0.5*minmod2(s[0] - s[1], s[1] - s[2]);
}

__device__ __forceinline__ void omp6_mn(int flag, double &m, double &n) {
    if (flag == 1) { m = 0.001; n = 0.0; }
    else if (flag == 2) { m = 0.0; n = -1.0/140.0; }
    else { m = 0.015; n = 0.0; }
}

// OMP6 positive side, src/OCFD_Schemes.cu:936-1008
__device__ __forceinline__ double omp6_p(int flag, const double *s) {
    double m, n; omp6_mn(flag, m, n);
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
        double lo, hi;
        {
            lo = fmin(fmin(s[3], s[4]), tmp);
            double q = s[3] + 4.0*(s[3] - s[2]);
            q = fmin(fmin(s[3], q), tmp1);
            lo = fmax(lo, q);
        }
        {
            double t2 = fmax(s[4], fmax(s[3], tmp));
            double q = s[3] + 4.0*(s[3] - s[2]);
            q = fmax(fmax(s[3], q), tmp1);
            hi = fmin(t2, q);
        }
        mid_nf = mid_nf + minmod2(hi - mid_nf, lo - mid_nf);
    }
    return mid_nf;
}

// OMP6 negative side, src/OCFD_Schemes.cu:1037-1095 (s = f(F-3..F+4))
__device__ __forceinline__ double omp6_m(int flag, const double *s) {
    double m, n; omp6_mn(flag, m, n);
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
        double lo, hi;
        {
            lo = fmin(fmin(s[5], s[3]), tmp);
            double q = s[4] + 4.0*(s[4] - s[5]);
            q = fmin(fmin(s[4], q), tmp1);
            lo = fmax(lo, q);
        }
        {
            double t2 = fmax(s[3], fmax(s[4], tmp));
            double q = s[4] + 4.0*(s[4] - s[5]);
            q = fmax(fmax(s[4], q), tmp1);
            hi = fmin(t2, q);
        }
        mid_nf = mid_nf + minmod2(hi - mid_nf, lo - mid_nf);
    }
    return mid_nf;
}

// WENO7-SYMBO weights and reconstruction, shared by both signs once the
// stencil is mirrored; src/OCFD_Schemes.cu:391-478 (P) and :506-590 (M).
// v[t] is the stencil in upwind order (P: f(F-3+t); M: f(F+4-t)).
__device__ __forceinline__ double symbo_core(bool linear, const double *v) {
    double S0, S1, S2, S3, S4, tmp;
    if (linear) {
        S0 = 0.0401954833730; S1 = 0.2493800006710; S2 = 0.4802686256260;
        S3 = 0.2009775476730; S4 = 0.0291783426580;
    } else {
        S0 = 0.0; S1 = 0.0; S2 = 0.0; S3 = 0.0; S4 = 0.0;
        tmp =  -2.0*v[0] +  9.0*v[1] - 18.0*v[2] + 11.0*v[3]; S0 += 720.0*tmp*tmp;
        tmp =       v[1] -  6.0*v[2] +  3.0*v[3] +  2.0*v[4]; S1 += 720.0*tmp*tmp;
        tmp =  -2.0*v[2] -  3.0*v[3] +  6.0*v[4] -      v[5]; S2 += 720.0*tmp*tmp;
        tmp = -11.0*v[3] + 18.0*v[4] -  9.0*v[5] +  2.0*v[6]; S3 += 720.0*tmp*tmp;
        tmp = -26.0*v[4] + 57.0*v[5] - 42.0*v[6] + 11.0*v[7]; S4 += 720.0*tmp*tmp;
        tmp = -6.0*v[0] + 24.0*v[1] - 30.0*v[2] + 12.0*v[3]; S0 += 780.0*tmp*tmp;
        tmp =                    6.0*v[2] - 12.0*v[3] +  6.0*v[4]; S1 += 780.0*tmp*tmp;
        tmp =                    6.0*v[3] - 12.0*v[4] +  6.0*v[5]; S2 += 780.0*tmp*tmp;
        tmp = 12.0*v[3] - 30.0*v[4] + 24.0*v[5] -  6.0*v[6]; S3 += 780.0*tmp*tmp;
        tmp = 18.0*v[4] - 48.0*v[5] + 42.0*v[6] - 12.0*v[7]; S4 += 780.0*tmp*tmp;
        tmp = -6.0*v[0] + 18.0*( v[1] - v[2] ) + 6.0*v[3]; S0 += 781.0*tmp*tmp;
        tmp = -6.0*v[1] + 18.0*( v[2] - v[3] ) + 6.0*v[4]; S1 += 781.0*tmp*tmp;
        tmp = -6.0*v[2] + 18.0*( v[3] - v[4] ) + 6.0*v[5]; S2 += 781.0*tmp*tmp;
        tmp = -6.0*v[3] + 18.0*( v[4] - v[5] ) + 6.0*v[6]; S3 += 781.0*tmp*tmp;
        tmp = -6.0*v[4] + 18.0*( v[5] - v[6] ) + 6.0*v[7]; S4 += 781.0*tmp*tmp;
        S4 = fmax(fmax(fmax(S0, S1), fmax(S2, S3)), S4);
        const double e = 2.592e-6;
        double t0 =  (0.0401954833730)*(e+S1)*(e+S2)*(e+S3)*(e+S4);
        double t1 =  (0.2493800006710)*(e+S0)*(e+S2)*(e+S3)*(e+S4);
        double t2 =  (0.4802686256260)*(e+S0)*(e+S1)*(e+S3)*(e+S4);
        double t3 =  (0.2009775476730)*(e+S0)*(e+S1)*(e+S2)*(e+S4);
        S4 =         (0.0291783426580)*(e+S0)*(e+S1)*(e+S2)*(e+S3);
        S3 = t3; S2 = t2; S1 = t1; S0 = t0;
    }
    double am = S0 + S1 + S2 + S3 + S4;
    double r = 0.0;
    tmp = -3.0*v[0] + 13.0*v[1] - 23.0*v[2] + 25.0*v[3]; r += S0*tmp;
    tmp =      v[1] -  5.0*v[2] + 13.0*v[3] +  3.0*v[4]; r += S1*tmp;
    tmp =     -v[2] +  7.0*v[3] +  7.0*v[4] -      v[5]; r += S2*tmp;
    tmp =  3.0*v[3] + 13.0*v[4] -  5.0*v[5] +      v[6]; r += S3*tmp;
    tmp = 25.0*v[4] - 23.0*v[5] + 13.0*v[6] -  3.0*v[7]; r += S4*tmp;
    return r / (12.0*am);
}

__device__ __forceinline__ double symbo_p(int lmt, double tv_lim, double tv_max, const double *s) {
    double TVmin = 0, TVmax = 1;
    if (lmt == 1) {
        double S0 = fabs(s[1] - s[0]) + fabs(s[2] - s[1]) + fabs(s[3] - s[2]);
        double S1 = fabs(s[2] - s[1]) + fabs(s[3] - s[2]) + fabs(s[4] - s[3]);
        double S2 = fabs(s[3] - s[2]) + fabs(s[4] - s[3]) + fabs(s[5] - s[4]);
        double S3 = fabs(s[4] - s[3]) + fabs(s[5] - s[4]) + fabs(s[6] - s[5]);
        double S4 = fabs(s[5] - s[4]) + fabs(s[6] - s[5]) + fabs(s[7] - s[6]);
        TVmin = fmin(fmin(fmin(S0, S1), fmin(S2, S3)), S4);
        TVmax = fmax(fmax(fmax(S0, S1), fmax(S2, S3)), S4);
    }
    return symbo_core(TVmax < tv_lim*TVmin && TVmax < tv_max, s);
}

__device__ __forceinline__ double symbo_m(int lmt, double tv_lim, double tv_max, const double *s) {
    // mirrored stencil; the reference never sets TVmin on this side, so the
    // linear branch cannot be taken (it only evaluates TVmax)
    double v[8];
#pragma unroll
    for (int t = 0; t < 8; t++) v[t] = s[7 - t];
    double TVmin = 0, TVmax = 1;
    if (lmt == 1) {
        double S0 = fabs(v[0] - v[1]) + fabs(v[1] - v[2]) + fabs(v[2] - v[3]);
        double S1 = fabs(v[1] - v[2]) + fabs(v[2] - v[3]) + fabs(v[3] - v[4]);
        double S2 = fabs(v[2] - v[3]) + fabs(v[3] - v[4]) + fabs(v[4] - v[5]);
        double S3 = fabs(v[3] - v[4]) + fabs(v[4] - v[5]) + fabs(v[5] - v[6]);
        double S4 = fabs(v[4] - v[5]) + fabs(v[5] - v[6]) + fabs(v[6] - v[7]);
        TVmax = fmax(fmax(fmin(S0, S1), fmin(S2, S3)), S4);
    }
    return symbo_core(TVmax < tv_lim*TVmin && TVmax < tv_max, v);
}

// CD6 / CD8 first derivative, src/OCFD_Schemes.cu:96-126
__device__ __forceinline__ double cd6(double sm3, double sm2, double sm1, double sp1, double sp2, double sp3) {
    return (45.0*(sp1 - sm1) - 9.0*(sp2 - sm2) + (sp3 - sm3))/60.0;
}
__device__ __forceinline__ double cd8(double sm4, double sm3, double sm2, double sm1,
                                      double sp1, double sp2, double sp3, double sp4) {
    return (672.0*(sp1 - sm1) - 168.0*(sp2 - sm2) + 32.0*(sp3 - sm3) - 3.0*(sp4 - sm4))/840.0;
}

// ---------------------------------------------------------------------------
// characteristic system at a face, src/OCFD_flux_charteric.cu:321-752
// ---------------------------------------------------------------------------
struct CharPara { double u1, v1, w1, c1, n1, n2, n3, l1, l2, l3, m1, m2, m3, KK; };

__device__ __forceinline__ void char_para(double u1, double v1, double w1, double c1,
                                          double a1, double a2, double a3, double G, CharPara &p) {
    double ss = sqrt(a1*a1 + a2*a2 + a3*a3);
    double n1 = a1/ss, n2 = a2/ss, n3 = a3/ss, l1, l2, l3;
    if (fabs(n3) <= fabs(n2)) {
        ss = sqrt(n1*n1 + n2*n2);
        l1 = -n2/ss; l2 = n1/ss; l3 = 0.0;
    } else {
        ss = sqrt(n1*n1 + n3*n3);
        l1 = -n3/ss; l2 = 0.0; l3 = n1/ss;
    }
    p.u1 = u1; p.v1 = v1; p.w1 = w1; p.c1 = c1;
    p.n1 = n1; p.n2 = n2; p.n3 = n3; p.l1 = l1; p.l2 = l2; p.l3 = l3;
    p.m1 = n2*l3 - n3*l2; p.m2 = n3*l1 - n1*l3; p.m3 = n1*l2 - n2*l1;
    p.KK = (G - 1.0)/(c1*c1);
}

// face eigen-system kept in shared memory as NCP planes of nf faces
constexpr int NCP = 14;
__device__ __forceinline__ void store_para(const CharPara &p, double *b, int i, int nf) {
    b[0 * nf + i] = p.u1; b[1 * nf + i] = p.v1; b[2 * nf + i] = p.w1; b[3 * nf + i] = p.c1;
    b[4 * nf + i] = p.n1; b[5 * nf + i] = p.n2; b[6 * nf + i] = p.n3;
    b[7 * nf + i] = p.l1; b[8 * nf + i] = p.l2; b[9 * nf + i] = p.l3;
    b[10 * nf + i] = p.m1; b[11 * nf + i] = p.m2; b[12 * nf + i] = p.m3; b[13 * nf + i] = p.KK;
}
__device__ __forceinline__ void load_para(CharPara &p, const double *b, int i, int nf) {
    p.u1 = b[0 * nf + i]; p.v1 = b[1 * nf + i]; p.w1 = b[2 * nf + i]; p.c1 = b[3 * nf + i];
    p.n1 = b[4 * nf + i]; p.n2 = b[5 * nf + i]; p.n3 = b[6 * nf + i];
    p.l1 = b[7 * nf + i]; p.l2 = b[8 * nf + i]; p.l3 = b[9 * nf + i];
    p.m1 = b[10 * nf + i]; p.m2 = b[11 * nf + i]; p.m3 = b[12 * nf + i]; p.KK = b[13 * nf + i];
}

// row r of the left eigenvector matrix (flux_charteric_ptoc_kernel :617-676)
__device__ __forceinline__ void char_L_row(const CharPara &p, int r, double S[5]) {
    double X1 = 1.0/(2.0*p.c1);
    double un = p.u1*p.n1 + p.v1*p.n2 + p.w1*p.n3;
    double v2 = (p.u1*p.u1 + p.v1*p.v1 + p.w1*p.w1)*0.5;
    double KK = p.KK;
    switch (r) {
    case 0: S[0] = 1.0 - KK*v2; S[1] = KK*p.u1; S[2] = KK*p.v1; S[3] = KK*p.w1; S[4] = -KK; break;
    case 1: S[0] = -(p.u1*p.l1 + p.v1*p.l2 + p.w1*p.l3); S[1] = p.l1; S[2] = p.l2; S[3] = p.l3; S[4] = 0.0; break;
    case 2: S[0] = -(p.u1*p.m1 + p.v1*p.m2 + p.w1*p.m3);
            S[1] = p.n2*p.l3 - p.n3*p.l2; S[2] = p.n3*p.l1 - p.n1*p.l3; S[3] = p.n1*p.l2 - p.n2*p.l1; S[4] = 0.0; break;
    case 3: S[0] = KK*v2*0.5 + X1*un; S[1] = -X1*p.n1 - KK*p.u1*0.5; S[2] = -X1*p.n2 - KK*p.v1*0.5;
            S[3] = -X1*p.n3 - KK*p.w1*0.5; S[4] = KK*0.5; break;
    default: {
            double s41 = KK*v2*0.5 + X1*un, s42 = -X1*p.n1 - KK*p.u1*0.5;
            double s43 = -X1*p.n2 - KK*p.v1*0.5, s44 = -X1*p.n3 - KK*p.w1*0.5;
            S[0] = s41 - 2*X1*un; S[1] = 2*X1*p.n1 + s42; S[2] = 2*X1*p.n2 + s43;
            S[3] = 2*X1*p.n3 + s44; S[4] = KK*0.5; break; }
    }
}

// row r of the right eigenvector matrix (flux_charteric_ctop_kernel :678-752)
__device__ __forceinline__ void char_R_row(const CharPara &p, int r, double S[5]) {
    switch (r) {
    case 0: S[0] = 1.0; S[1] = 0.0; S[2] = 0.0; S[3] = 1.0; S[4] = 1.0; break;
    case 1: S[0] = p.u1; S[1] = p.l1; S[2] = p.n2*p.l3 - p.n3*p.l2; S[3] = p.u1 - p.c1*p.n1; S[4] = 2*p.u1 - S[3]; break;
    case 2: S[0] = p.v1; S[1] = p.l2; S[2] = p.n3*p.l1 - p.n1*p.l3; S[3] = p.v1 - p.c1*p.n2; S[4] = 2*p.v1 - S[3]; break;
    case 3: S[0] = p.w1; S[1] = p.l3; S[2] = p.n1*p.l2 - p.n2*p.l1; S[3] = p.w1 - p.c1*p.n3; S[4] = 2*p.w1 - S[3]; break;
    default: {
            S[0] = (p.u1*p.u1 + p.v1*p.v1 + p.w1*p.w1)*0.5;
            double H = S[0] + 1.0/p.KK;
            S[1] = p.u1*p.l1 + p.v1*p.l2 + p.w1*p.l3;
            S[2] = p.u1*p.m1 + p.v1*p.m2 + p.w1*p.m3;
            S[3] = H - p.c1*(p.u1*p.n1 + p.v1*p.n2 + p.w1*p.n3);
            S[4] = 2*H - S[3]; break; }
    }
}

__device__ __forceinline__ double dot5(const double S[5], double x0, double x1, double x2, double x3, double x4) {
    return S[0]*x0 + S[1]*x1 + S[2]*x2 + S[3]*x3 + S[4]*x4;
}

}  // namespace ocfd
