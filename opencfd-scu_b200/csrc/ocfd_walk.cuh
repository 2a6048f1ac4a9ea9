// ocfd_walk.cuh -- pieces shared by the line-walking inviscid sweep kernels
// (ocfd_sweep3.cu, ocfd_sweep4.cu): the split into a per-warp ring of
// shared memory, the face record, the UP7 face, the boundary tests and the
// du update of one cell.
#pragma once
#include "ocfd_fp32.cuh"

namespace ocfd {
namespace walk {

constexpr unsigned FULL = 0xffffffffu;

// window over the split values of one face: at(sv, k) = value sv
// (sign * 5 + field) of stencil point k (face F+1/2: point F-3+k)
struct Win {
    const double *b;
    int ks, vs, mask, s0;
    __device__ __forceinline__ double at(int sv, int k) const { return b[((s0 + k) & mask) * ks + sv * vs]; }
};

// Steger-Warming split of LAP point o along direction DIR into fp/fm, in
// the precision R of the primitives given
template <int DIR, bool UNI, bool EPS0, typename R>
__device__ __forceinline__ void split_point(const Params &p, long long o, R d, R u, R v,
                                            R w, R T, R *fp, R *fm) {
    R cc = div_const(sqrt_r(T), (R)p.Ama, (R)p.inv_Ama);
    if constexpr (UNI) {
        const DirConst &dc = p.dc[DIR];
        sw_split_pre<EPS0>(d * (R)p.tmp0, u, v, w, cc, (R)dc.A[0], (R)dc.A[1], (R)dc.A[2], (R)dc.ss,
                           (R)dc.An[0], (R)dc.An[1], (R)dc.An[2], p, fp, fm);
    } else {
        const int mA = M_AKX + 3 * DIR;
        sw_split(d * (R)p.tmp0, u, v, w, cc, (R)p.met[mA][o], (R)p.met[mA + 1][o], (R)p.met[mA + 2][o],
                 (R)p.Gamma, (R)p.epsl_sw, (R)p.split_C1, (R)p.split_C3, fp, fm);
    }
}

// characteristic face record between LAP cells o0 and o1 (get_para_charteric_*,
// src/OCFD_flux_charteric.cu:330-418)
template <bool UNI, typename R>
__device__ __forceinline__ void face_record(const Params &p, int dir, long long o0, long long o1, R *rec) {
    const R *u = prim_r<R>(p, 1), *v = prim_r<R>(p, 2), *w = prim_r<R>(p, 3), *T = prim_r<R>(p, 4);
    R c0v = div_const(sqrt_r(T[o0]), (R)p.Ama, (R)p.inv_Ama);
    R c1v = div_const(sqrt_r(T[o1]), (R)p.Ama, (R)p.inv_Ama);
    R u1 = (u[o0] + u[o1]) * (R)0.5, v1 = (v[o0] + v[o1]) * (R)0.5, w1 = (w[o0] + w[o1]) * (R)0.5;
    R c1 = (c0v + c1v) * (R)0.5;
    if (UNI) {
        const DirConst &dc = p.dc[dir];
        R KK = ((R)p.Gamma - (R)1.0) / (c1 * c1);
        rec[FU] = u1; rec[FV] = v1; rec[FW] = w1; rec[FC] = c1; rec[FKK] = KK;
        rec[FX1] = (R)1.0 / ((R)2.0 * c1);
        R v2 = (u1 * u1 + v1 * v1 + w1 * w1) * (R)0.5;
        rec[FV2] = v2;
        rec[FUN] = u1 * (R)dc.n[0] + v1 * (R)dc.n[1] + w1 * (R)dc.n[2];
        rec[FH] = v2 + (R)1.0 / KK;
        rec[FN1] = (R)dc.n[0]; rec[FN2] = (R)dc.n[1]; rec[FN3] = (R)dc.n[2];
        rec[FL1] = (R)dc.l[0]; rec[FL2] = (R)dc.l[1]; rec[FL3] = (R)dc.l[2];
        rec[FM1] = (R)dc.m[0]; rec[FM2] = (R)dc.m[1]; rec[FM3] = (R)dc.m[2];
    } else {
        const int mA = M_AKX + 3 * dir;
        make_record(u1, v1, w1, c1, (R)((p.met[mA][o0] + p.met[mA][o1]) * 0.5),
                    (R)((p.met[mA + 1][o0] + p.met[mA + 1][o1]) * 0.5),
                    (R)((p.met[mA + 2][o0] + p.met[mA + 2][o1]) * 0.5), p, rec, 1);
    }
}

// Flux of face F+1/2 of a line of n cells (both signs, all fields) from its
// 8-point window, any scheme: component-wise reconstruction, or projection on
// the face's characteristic fields, reconstruction and back-projection.  Near
// a face whose DIF_BOUND is 1 the boundary closure replaces the
// reconstruction, after the projection when there is one, as the reference's
// kernels call OCFD_bound_scheme_kernel_{p,m} (src/OCFD_bound_Scheme.cu:739-944).
// o0 is the LAP offset of the cell left of the face, sd the LAP stride.
template <bool UNI>
__device__ __noinline__ void face_generic(const Params &p, int dir, Win w, int hflag, long long o0,
                                          long long sd, int F, int n, double *out) {
    const int scheme = p.scheme_invis;
    const bool char_scheme = p.charteric && (scheme == 304 || scheme == 305 || scheme == 310);
    const bool hybrid = scheme == 310;
    if (p.charteric && !char_scheme) {          // the reference adds nothing
        for (int m = 0; m < 10; m++) out[m] = 0.0;
        return;
    }
    const bool lo = p.bnd_lo[dir], hi = p.bnd_hi[dir];
    const bool bnd = lo || hi;
    int KA[2], KB[2];
    extents(scheme, char_scheme, 0, KA[0], KB[0]);
    extents(scheme, char_scheme, 1, KA[1], KB[1]);
    if (char_scheme && !(hybrid && hflag == 1)) {
        double rec[FP_N];
        face_record<UNI>(p, dir, o0, o0 + sd, rec);
        for (int sign = 0; sign < 2; sign++) {
            double fv[5][8];
#pragma unroll
            for (int m = 0; m < 5; m++)
#pragma unroll
                for (int k = 0; k < 8; k++) fv[m][k] = w.at(sign * 5 + m, k);
            double o5[5];
#pragma unroll
            for (int c = 0; c < 5; c++) {
                double Lr[5], vals[8], Rc[5];
                L_row(rec, 1, c, Lr);
#pragma unroll
                for (int k = 0; k < 8; k++) vals[k] = dot5(Lr, fv[0][k], fv[1][k], fv[2][k], fv[3][k], fv[4][k]);
                double res;
                if (!(bnd && closure(sign, lo, hi, KA[sign], KB[sign], F, n, vals, res)))
                    res = recon_one(p, scheme, hflag, sign, vals);
                R_col(rec, 1, c, Rc);
                if (c == 0) {
#pragma unroll
                    for (int m = 0; m < 5; m++) o5[m] = Rc[m] * res;
                } else {
#pragma unroll
                    for (int m = 0; m < 5; m++) o5[m] = o5[m] + Rc[m] * res;
                }
            }
#pragma unroll
            for (int m = 0; m < 5; m++) out[sign * 5 + m] = o5[m];
        }
        return;
    }
    for (int sv = 0; sv < 10; sv++) {
        const int sign = sv >= 5, m = sv - 5 * sign;
        double vals[8];
#pragma unroll
        for (int k = 0; k < 8; k++) vals[k] = w.at(sv, k);
        int hf = hflag;
        if (hybrid && !char_scheme && m > 0 && p.nochar_comp_flag) hf = p.nochar_comp_flag;
        if (!(bnd && closure(sign, lo, hi, KA[sign], KB[sign], F, n, vals, out[sv])))
            out[sv] = recon_one(p, scheme, hf, sign, vals);
    }
}

// the face is within reach of a boundary closure (closure_p reaches F <= 2
// and F >= n-4, closure_m F <= 2 and F >= n-4; one more on each side here)
__device__ __forceinline__ bool near_closure(const Params &p, int dir, int F, int n) {
    return (p.bnd_lo[dir] && F <= 3) || (p.bnd_hi[dir] && F >= n - 5);
}

// the first / last cell of a line, where non-reflecting faces and the
// characteristic kernels' first-order boundary fluxes change du
__device__ __forceinline__ bool rule_cell(const Params &p, int dir, int X, int n) {
    return (X == 0 && (p.bnd_lo[dir] || p.nonref_lo[dir] == 1)) ||
           (X == n - 1 && (p.bnd_hi[dir] || p.nonref_hi[dir] == 1));
}

// the face takes the inline UP7 path: UP7 everywhere, or a hybrid face with
// flag 1 whose fields all use UP7
__device__ __forceinline__ bool up7_face(const Params &p, int hflag) {
    if (p.scheme_invis == 301) return !p.charteric;
    return p.scheme_invis == 310 && hflag == 1 && (p.charteric || !p.nochar_comp_flag);
}

// du of one cell from the face fluxes on its right (cur) and left (prv):
// x+ then x- for every field, as the reference's single-writer order
// (R: precision of the fluxes and of du; D: the storage of du)
template <bool FIRST, typename R, typename D>
__device__ __forceinline__ void add_du(D *__restrict__ du, long long N, long long ci, R aj,
                                       R h, R ih, const R *cur, const R *prv, const D *old) {
#pragma unroll
    for (int m = 0; m < 5; m++) {
        R acc = FIRST ? (R)0.0 : (R)old[m];
        acc += div_const(-aj * (cur[m] - prv[m]), h, ih);
        acc += div_const(-aj * (cur[5 + m] - prv[5 + m]), h, ih);
        du[m * N + ci] = (D)acc;
    }
}

// ---------------------------------------------------------------------------
// The sweep kernel.  A warp covers LC lines (consecutive x for y and z; one
// row for x) and LY = 32 / LC consecutive cells of each line, and walks its
// lines LY cells at a time.  Per pass every lane splits one new point into
// the warp's ring (RING points per line, value-major, line-minor, so a warp
// access is 32 consecutive doubles), then forms the flux of the face on the
// right of its cell and the du of its cell; the face on the left comes from
// the lane below it (a shuffle) or, for the first row of lanes, from the
// face kept from the previous pass.
// ---------------------------------------------------------------------------
constexpr int SW = 4;          // warps per block

template <int DIR> struct Shape;
template <> struct Shape<0> { static constexpr int LC = 1, RING = 64; };
template <> struct Shape<1> { static constexpr int LC = 8, RING = 16; };
template <> struct Shape<2> { static constexpr int LC = 8, RING = 16; };

// UP7 flux of face F+1/2 (both signs, all fields) from the ring
template <int RING, int LC, typename R>
__device__ __forceinline__ void face_up7(const R *ring, int col, int F, R (&out)[10]) {
#pragma unroll
    for (int sv = 0; sv < 10; sv++) {
        R vals[8];
#pragma unroll
        for (int t = 0; t < 8; t++) vals[t] = ring[(sv * RING + ((F - 3 + t) & (RING - 1))) * LC + col];
        out[sv] = sv < 5 ? up7_p_q(vals) : up7_m_q(vals);
    }
}


// split of one point (primitives q5, LAP offset o) into ring slot P
template <int DIR, int RING, int LC, bool UNI, bool EPS0, typename R>
__device__ __forceinline__ void ring_put(const Params &p, R *ring, int col, int P, long long o,
                                         const R (&q5)[5]) {
    R fp[5], fm[5];
    split_point<DIR, UNI, EPS0>(p, o, q5[0], q5[1], q5[2], q5[3], q5[4], fp, fm);
    const int q = P & (RING - 1);
#pragma unroll
    for (int m = 0; m < 5; m++) {
        ring[(m * RING + q) * LC + col] = fp[m];
        ring[((5 + m) * RING + q) * LC + col] = fm[m];
    }
}

template <typename R>
__device__ __forceinline__ void load5(const Params &p, long long o, R (&q5)[5]) {
    o = OCFD_IDX(p, o, p.lapN);
#pragma unroll
    for (int m = 0; m < 5; m++) q5[m] = __ldg(prim_r<R>(p, m) + o);
}

}  // namespace walk
}  // namespace ocfd
