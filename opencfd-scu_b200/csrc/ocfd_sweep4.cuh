// ocfd_sweep4.cuh -- inviscid flux sweeps with every face formed in the walk
// (sm_100a, FP64).
//
// Same results as the walk of ocfd_sweep3.cu, and so as the reference's
// OCFD_d{x,y,z}1/2 chain, for the two schemes whose faces are mostly not UP7:
//   K_HYBC  the hybrid scheme with its auto sensor and characteristic
//           projection (src/OCFD_Schemes_hybrid_auto.cu:862-1023 with
//           src/OCFD_flux_charteric.cu:330-752): a flag-1 face takes UP7 on
//           each flux component, a flag-2 face WENO7 and any other face WENO5
//           on the characteristic fields;
//   K_W7    WENO7 on each flux component (src/OCFD_Schemes.cu:640-741).
// Nothing goes out of line and no cell is left for a second kernel: one
// sign's stencil of a characteristic face (7 points x 5 fields) and the
// face's eigen-record are held in registers, and the boundary closures and
// the first/last-cell rules of bounded lines are applied where they fall.
// The fluxes of one pass go to a per-warp face buffer in shared memory, from
// which each lane takes the flux of the face on its left.
// (Templates; ocfd_sweep4.cu instantiates them in FP64, ocfd_sweep4_f32.cu in
// FP32 for the precision form.)
#pragma once
#include "ocfd_walk.cuh"

#include <cuda_runtime.h>

namespace ocfd {
namespace walk4 {


using namespace walk;

enum { K_HYBC = 0, K_W7 = 1 };

// ring value sv of point Q of line col
template <int RING, int LC, typename R>
__device__ __forceinline__ R rv(const R *ring, int col, int sv, int Q) {
    return ring[(sv * RING + (Q & (RING - 1))) * LC + col];
}

// One sign of a characteristic face F+1/2: the sign's 7-point stencil of
// the five split fields, projected on each characteristic field, the
// reconstruction (or the boundary closure) and the back-projection, with
// the operations and order of face_generic.  Point F-3+k is stencil entry k;
// sign 0 uses entries 0..6, sign 1 entries 1..7.
// HOT: a WENO7 face with no closure in reach -- the common case on grids
// without closed faces, kept compact so the loop's instruction footprint
// stays small; otherwise the general form (WENO7 or WENO5, closures)
template <int S, int RING, int LC, bool HOT, typename R>
__device__ __forceinline__ void char_sign(const R *ring, int col, int F, int n, bool w7, bool near,
                                          bool lo, bool hi, const R (&rec)[FP_N], R (&out)[10]) {
    constexpr int K0 = S, K1 = S + 6;
    R fv[5][8];
#pragma unroll
    for (int m = 0; m < 5; m++)
#pragma unroll
        for (int k = 0; k < 8; k++)
            fv[m][k] = (k >= K0 && k <= K1) ? rv<RING, LC>(ring, col, S * 5 + m, F - 3 + k) : (R)0.0;
    R o5[5];
    auto one = [&](int c) {
        R Lr[5], vals[8], Rc[5];
        L_row(rec, 1, c, Lr);
#pragma unroll
        for (int k = 0; k < 8; k++)
            vals[k] = (k >= K0 && k <= K1) ? dot5(Lr, fv[0][k], fv[1][k], fv[2][k], fv[3][k], fv[4][k]) : (R)0.0;
        R res;
        if (HOT)
            res = S ? weno7_m(vals) : weno7_p(vals);
        else if (!(near && closure(S, lo, hi, S ? 4 : 3, S ? 3 : 4, F, n, vals, res)))
            res = w7 ? (S ? weno7_m(vals) : weno7_p(vals)) : (S ? weno5_m(vals) : weno5_p(vals));
        R_col(rec, 1, c, Rc);
        if (c == 0) {
#pragma unroll
            for (int m = 0; m < 5; m++) o5[m] = Rc[m] * res;
        } else {
#pragma unroll
            for (int m = 0; m < 5; m++) o5[m] = o5[m] + Rc[m] * res;
        }
    };
    // the general form in FP32 keeps one copy of the field loop's body: its
    // five unrolled copies (a reconstruction, a closure and a WENO5 each)
    // left the walk waiting on instruction fetch (10 % slower on the ramp);
    // in FP64 the unrolled copies keep the walk's values in registers and
    // measured faster
    if constexpr (HOT || sizeof(R) == 8) {
#pragma unroll
        for (int c = 0; c < 5; c++) one(c);
    } else {
#pragma unroll 1
        for (int c = 0; c < 5; c++) one(c);
    }
#pragma unroll
    for (int m = 0; m < 5; m++) out[S * 5 + m] = o5[m];
}

// A face on the flux components with a boundary closure in reach: W7 picks
// WENO7, else UP7; (KA, KB) are the closure extents of the reference kernel
// of each sign.
template <int RING, int LC, bool W7, typename R>
__device__ __forceinline__ void comp_face_closure(const R *ring, int col, int F, int n, bool lo, bool hi,
                                                  int KA0, int KB0, int KA1, int KB1, R *out) {
    for (int sv = 0; sv < 10; sv++) {
        const int sign = sv >= 5;
        R vals[8];
#pragma unroll
        for (int k = 0; k < 8; k++) vals[k] = rv<RING, LC>(ring, col, sv, F - 3 + k);
        R r;
        if (!closure(sign, lo, hi, sign ? KA1 : KA0, sign ? KB1 : KB0, F, n, vals, r)) {
            if (W7) r = sign ? weno7_m(vals) : weno7_p(vals);
            else    r = sign ? up7_m_q(vals) : up7_p_q(vals);
        }
        out[sv] = r;
    }
}

template <int RING, int LC, typename R>
__device__ __forceinline__ void face_w7(const R *ring, int col, int F, R (&out)[10]) {
#pragma unroll
    for (int sv = 0; sv < 10; sv++) {
        R vals[8];
#pragma unroll
        for (int k = 0; k < 8; k++)
            vals[k] = (sv < 5 ? k < 7 : k > 0) ? rv<RING, LC>(ring, col, sv, F - 3 + k) : (R)0.0;
        out[sv] = sv < 5 ? weno7_p(vals) : weno7_m(vals);
    }
}

// Flux of face F+1/2 (both signs, all fields) of one lane's line.  Every
// path is in line: a call here, even on the rare closure faces alone,
// makes the walk keep its loop state in local memory around it.
// SPLIT (grids without closed faces): WENO7 characteristic faces take the
// compact copy and the rare others the general one; on bounded grids, where
// near-closure and WENO5 faces sit in many warps, one general copy measured
// faster (the two copies would run one after the other in those warps).
template <int KIND, int RING, int LC, bool UNI, bool SPLIT, typename R>
__device__ __forceinline__ void face4(const Params &p, int dir, const R *ring, int col, int F, int n,
                                      int hflag, long long o0, long long sd, bool lo, bool hi,
                                      R (&out)[10]) {
    const bool near = (lo && F <= 3) || (hi && F >= n - 5);
    if (near && (KIND == K_W7 || hflag == 1)) {
        R tmp[10];
        if (KIND == K_W7) comp_face_closure<RING, LC, true>(ring, col, F, n, lo, hi, 3, 3, 3, 3, tmp);
        else              comp_face_closure<RING, LC, false>(ring, col, F, n, lo, hi, 3, 4, 4, 3, tmp);
#pragma unroll
        for (int sv = 0; sv < 10; sv++) out[sv] = tmp[sv];
        return;
    }
    if (KIND == K_W7) { face_w7<RING, LC>(ring, col, F, out); return; }
    if (hflag == 1) { face_up7<RING, LC>(ring, col, F, out); return; }
    R rec[FP_N];
    face_record<UNI>(p, dir, o0, o0 + sd, rec);
    if (SPLIT && hflag == 2 && !near) {
        char_sign<0, RING, LC, true>(ring, col, F, n, true, false, lo, hi, rec, out);
        char_sign<1, RING, LC, true>(ring, col, F, n, true, false, lo, hi, rec, out);
    } else {
        char_sign<0, RING, LC, false>(ring, col, F, n, hflag == 2, near, lo, hi, rec, out);
        char_sign<1, RING, LC, false>(ring, col, F, n, hflag == 2, near, lo, hi, rec, out);
    }
}

// du of the first or last cell X of a bounded line (put_du_p/m_kernel,
// src/OCFD_Schemes.cu:293-381; put_du_character_{p,m}_kernel and
// OCFD_bound_character_kernel_{p,m}, src/OCFD_flux_charteric.cu:16-319):
// a non-reflecting face adds nothing, the characteristic kernels take a
// first-order flux difference from the split values at X-1 .. X+2.
template <int DIR, int KIND, int RING, int LC, typename R, typename D>
__device__ __forceinline__ void du_rule_cell(const Params &p, const R *ring, int col, int X, int n,
                                             D *__restrict__ du, long long ci, R aj, R h,
                                             R ih, const R (&cur)[10], const R (&prv)[10]) {
    constexpr bool char_kernel = KIND == K_HYBC;
    const bool lo = p.bnd_lo[DIR], hi = p.bnd_hi[DIR];
    const bool only_lo = lo && !hi, only_hi = hi && !lo;     // flag 1..6, not 7..9
    const bool first = X == 0, last = X == n - 1;
    const long long N = p.N;
    for (int m = 0; m < 5; m++) {
        R acc = DIR == 0 ? (R)0.0 : (R)du[m * N + ci];
        if (!char_kernel ? (first && p.nonref_lo[DIR] == 1) : (only_lo && p.nonref_lo[DIR] == 1 && first)) {
            acc += (R)0.0;
        } else if (char_kernel && ((only_lo && first) || (only_hi && last))) {
            R tmp;
            if (first) {
                tmp = rv<RING, LC>(ring, col, m, X + 1) - rv<RING, LC>(ring, col, m, X);
            } else {
                const R f0 = rv<RING, LC>(ring, col, m, X), f1 = rv<RING, LC>(ring, col, m, X - 1);
                const R f2 = rv<RING, LC>(ring, col, m, X - 2);
                const R tr = f0 + (R)0.5 * minmod2(f0 - f1, f0 - f1);
                const R tl = f1 + (R)0.5 * minmod2(f0 - f1, f1 - f2);
                tmp = tr - tl;
            }
            acc += div_const(-aj * tmp, h, ih);
        } else {
            acc += div_const(-aj * (cur[m] - prv[m]), h, ih);
        }
        // the reference's y kernel tests flag 3 for its lower face, so that
        // first-order flux never applies on y
        if (!char_kernel ? (last && p.nonref_hi[DIR] == 1) : (only_hi && p.nonref_hi[DIR] == 1 && last)) {
            acc += (R)0.0;
        } else if (char_kernel && ((DIR != 1 && only_lo && first) || (only_hi && last))) {
            R tmp;
            if (first) {
                const R f0 = rv<RING, LC>(ring, col, 5 + m, X), f1 = rv<RING, LC>(ring, col, 5 + m, X + 1);
                const R f2 = rv<RING, LC>(ring, col, 5 + m, X + 2);
                const R tr = f1 - (R)0.5 * minmod2(f2 - f1, f1 - f0);
                const R tl = f0 - (R)0.5 * minmod2(f1 - f0, f1 - f0);
                tmp = tr - tl;
            } else {
                tmp = rv<RING, LC>(ring, col, 5 + m, X) - rv<RING, LC>(ring, col, 5 + m, X - 1);
            }
            acc += div_const(-aj * tmp, h, ih);
        } else {
            acc += div_const(-aj * (cur[5 + m] - prv[5 + m]), h, ih);
        }
        du[m * N + ci] = (D)acc;
    }
}

// MINB: resident blocks per SM the register budget is fitted to; 3 (168
// registers, a few spills) runs faster than 2 (no spills) on the
// characteristic faces.
// The walk: a warp covers LC lines and LY = 32 / LC consecutive cells of
// each, LY cells per pass.  Per pass every lane splits one new point into
// the ring, forms the flux of the face on the right of its cell into the
// face buffer (FR = 2 LY slots per line, so a pass never overwrites a face
// that the previous pass's lanes still read), then adds its cell's du with
// the face on its left from the buffer.
template <int DIR, bool UNI, bool EPS0, int KIND, int MINB, bool SPLIT, typename R>
__global__ void __launch_bounds__(32 * SW, MINB) k_sweep4(const __grid_constant__ Params p, int seg_len) {
    constexpr int LC = Shape<DIR>::LC, LY = 32 / LC, RING = Shape<DIR>::RING, FR = 2 * LY;
    // the next pass's points overwrite slots this pass reads unless the
    // ring spans both windows
    constexpr bool SYNC2 = 2 * LY + 6 >= RING;
    extern __shared__ __align__(16) unsigned char smem4[];   // per warp: ring, then face buffer
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int col = lane % LC, ly = lane / LC;
    const long long grp = (long long)blockIdx.x * SW + wid;     // line group of this warp
    const int ngx = (p.nx + LC - 1) / LC;
    const long long ngroups = DIR == 0 ? (long long)p.ny * p.nz : (long long)ngx * (DIR == 1 ? p.nz : p.ny);
    if (grp >= ngroups) return;                                 // the whole warp
    R *ring = reinterpret_cast<R *>(smem4) + (size_t)wid * 10 * (RING + FR) * LC;
    R *fbuf = ring + 10 * RING * LC;
    const int n = DIR == 0 ? p.nx : (DIR == 1 ? p.ny : p.nz);
    const int y0 = blockIdx.y * seg_len;
    const int y1 = min(n, y0 + seg_len);

    long long base, cb, cst, fst, sd;
    const int8_t *fl;
    bool colok = true;
    if (DIR == 0) {
        const int j = (int)(grp % p.ny), k = (int)(grp / p.ny);
        base = (long long)(k + OCFD_LAP) * p.zs + (long long)(j + OCFD_LAP) * p.ys + OCFD_LAP;
        sd = 1;
        cb = in_index(p, 0, j, k); cst = 1;
        fl = p.flag[0] + (long long)(p.nx + 1) * ((long long)j + (long long)p.ny * k); fst = 1;
    } else {
        const int x = (int)(grp % ngx) * LC + col, c3 = (int)(grp / ngx);
        colok = x < p.nx;
        const int xs = colok ? x : p.nx - 1;                    // keep addresses in range
        if (DIR == 1) {
            base = (long long)(xs + OCFD_LAP) + (long long)OCFD_LAP * p.ys + (long long)(c3 + OCFD_LAP) * p.zs;
            sd = p.ys;
            cb = (long long)xs + (long long)p.nx * p.ny * c3; cst = p.nx;
            fl = p.flag[1] + (long long)xs + (long long)p.nx * (p.ny + 1) * c3; fst = p.nx;
        } else {
            base = (long long)(xs + OCFD_LAP) + (long long)(c3 + OCFD_LAP) * p.ys + (long long)OCFD_LAP * p.zs;
            sd = p.zs;
            cb = (long long)xs + (long long)p.nx * c3; cst = (long long)p.nx * p.ny;
            fl = p.flag[2] + (long long)xs + (long long)p.nx * c3; fst = (long long)p.nx * p.ny;
        }
    }
    R *__restrict__ du = du_r<R>(p);
    const long long N = p.N;
    const bool lo = p.bnd_lo[DIR], hi = p.bnd_hi[DIR];
    const R h = (R)(DIR == 0 ? p.hx : (DIR == 1 ? p.hy : p.hz)), ih = (R)p.inv_h[DIR];

    // points y0-4 .. y0+3 and the face left of cell y0
    for (int r = ly; r < 8; r += LY) {
        if (colok) {
            R q5[5];
            const long long o = base + (long long)(y0 - 4 + r) * sd;
            load5(p, o, q5);
            ring_put<DIR, RING, LC, UNI, EPS0>(p, ring, col, y0 - 4 + r, o, q5);
        }
    }
    __syncwarp();
    if (ly == 0 && colok) {
        const int hf = KIND == K_HYBC ? flag_at(p, DIR, fl, (long long)y0 * fst) : 2;
        R cur[10];
        face4<KIND, RING, LC, UNI, SPLIT>(p, DIR, ring, col, y0 - 1, n, hf, base + (long long)(y0 - 1) * sd, sd, lo, hi, cur);
#pragma unroll
        for (int sv = 0; sv < 10; sv++) fbuf[(sv * FR + ((y0 - 1) & (FR - 1))) * LC + col] = cur[sv];
    }

    for (int Y0 = y0; Y0 < y1; Y0 += LY) {
        const int P = Y0 + 4 + ly;
        const int F = Y0 + ly;
        const bool valid = colok && F < y1;
        if (colok && P <= y1 + 3) {
            R q5[5];
            const long long o = base + (long long)P * sd;
            load5(p, o, q5);
            ring_put<DIR, RING, LC, UNI, EPS0>(p, ring, col, P, o, q5);
        }
        const int hflag = (KIND == K_HYBC && valid) ? flag_at(p, DIR, fl, (long long)(F + 1) * fst) : 2;
        __syncwarp();
        R cur[10];
        if (valid) {
            face4<KIND, RING, LC, UNI, SPLIT>(p, DIR, ring, col, F, n, hflag, base + (long long)F * sd, sd, lo, hi, cur);
#pragma unroll
            for (int sv = 0; sv < 10; sv++) fbuf[(sv * FR + (F & (FR - 1))) * LC + col] = cur[sv];
        }
        __syncwarp();
        if (valid) {
            R prv[10];
#pragma unroll
            for (int sv = 0; sv < 10; sv++) prv[sv] = fbuf[(sv * FR + ((F - 1) & (FR - 1))) * LC + col];
            const long long ci = OCFD_IDX(p, cb + (long long)F * cst, N);
            const R aj = (R)metric<UNI>(p, M_AJAC, base + (long long)F * sd);
            if (p.has_bnd && rule_cell(p, DIR, F, n)) {
                du_rule_cell<DIR, KIND, RING, LC>(p, ring, col, F, n, du, ci, aj, h, ih, cur, prv);
            } else {
                R old[5];
                if (DIR != 0) {
#pragma unroll
                    for (int m = 0; m < 5; m++) old[m] = du[m * N + ci];
                }
                if (DIR == 0) add_du<true>(du, N, ci, aj, h, ih, cur, prv, old);
                else          add_du<false>(du, N, ci, aj, h, ih, cur, prv, old);
            }
        }
        if (SYNC2) __syncwarp();
    }
}

// Cells the call-free UP7 walk left (precision form, the characteristic
// hybrid scheme), one warp per cell: lanes 0..8 split the points X-4 .. X+4
// into the warp's window; lane (face, value) forms a value of the fluxes of
// faces X-1/2 and X+1/2 where the face is UP7 (with its closure when one is
// in reach); for a characteristic face lane (face, sign, field c) projects,
// reconstructs (WENO7 on flag 2, else WENO5, or the closure) and takes
// column c of R, and lane (face, sign, m) sums the products over c in
// char_sign's order; lanes 0..4 add the cell's du as the walk does.  The
// arithmetic of every value is face4's.
constexpr int FIX4W = 4;       // warps (cells in flight) per block

template <int DIR, bool UNI, bool EPS0, typename R>
__global__ void __launch_bounds__(32 * FIX4W) k_sweep4_fix(const __grid_constant__ Params p) {
    __shared__ R win_s[FIX4W][90];              // [point X-4+t][sign * 5 + field]
    __shared__ R res_s[FIX4W][20];
    __shared__ R rc_s[FIX4W][20][5];
    __shared__ R out_s[FIX4W][2][10];           // fluxes of faces X-1/2 and X+1/2
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned cnt = p.defer_count[DIR];
    const long long sd = DIR == 0 ? 1LL : (DIR == 1 ? p.ys : p.zs);
    const R h = (R)(DIR == 0 ? p.hx : (DIR == 1 ? p.hy : p.hz)), ih = (R)p.inv_h[DIR];
    const bool lo = p.bnd_lo[DIR], hi = p.bnd_hi[DIR];
    const int n = DIR == 0 ? p.nx : (DIR == 1 ? p.ny : p.nz);
    R *__restrict__ du = du_r<R>(p);
    const long long N = p.N;
    R *win = win_s[w];
    // value sv of point Q of the cell's window (point X-4 is entry 0)
    for (unsigned e = blockIdx.x * FIX4W + w; e < cnt; e += gridDim.x * FIX4W) {
        const long long ci = OCFD_IDX(p, (long long)p.defer[DIR][e], p.N);
        const int i = (int)(ci % p.nx);
        const long long r = ci / p.nx;
        const int j = (int)(r % p.ny), k = (int)(r / p.ny);
        const int X = DIR == 0 ? i : (DIR == 1 ? j : k);
        const long long oX = lap_index(p, i + OCFD_LAP, j + OCFD_LAP, k + OCFD_LAP);
        auto wv = [&](int sv, int Q) -> R { return win[(Q - X + 4) * 10 + sv]; };
        if (lane < 9) {
            const long long o = oX + (long long)(lane - 4) * sd;
            R q5[5], fp[5], fm[5];
            load5(p, o, q5);
            split_point<DIR, UNI, EPS0>(p, o, q5[0], q5[1], q5[2], q5[3], q5[4], fp, fm);
#pragma unroll
            for (int m = 0; m < 5; m++) { win[lane * 10 + m] = fp[m]; win[lane * 10 + 5 + m] = fm[m]; }
        }
        __syncwarp();
        const int side = (lane / 10) & 1, q = lane - 10 * (lane / 10);
        const int e1 = X + side;
        const long long qq = DIR == 0 ? (long long)e1 + (long long)(p.nx + 1) * ((long long)j + (long long)p.ny * k)
                           : DIR == 1 ? (long long)i + (long long)p.nx * ((long long)e1 + (long long)(p.ny + 1) * k)
                                      : (long long)i + (long long)p.nx * ((long long)j + (long long)p.ny * e1);
        const int hflag = flag_at(p, DIR, p.flag[DIR], qq);
        const int F = X - 1 + side;
        const bool near = (lo && F <= 3) || (hi && F >= n - 5);
        const bool charf = hflag != 1;
        if (lane < 20) {
            const int sign = q >= 5, mc = q - 5 * sign;
            if (!charf) {                                     // UP7 on the flux components
                R vals[8];
#pragma unroll
                for (int t = 0; t < 8; t++) vals[t] = wv(q, F - 3 + t);
                R o;
                if (!(near && closure(sign, lo, hi, sign ? 4 : 3, sign ? 3 : 4, F, n, vals, o)))
                    o = sign ? up7_m_q(vals) : up7_p_q(vals);
                out_s[w][side][q] = o;
            } else {                                          // characteristic field c = mc of this sign
                R rec[FP_N], Lr[5], Rc[5], vals[8];
                const long long o0 = oX + (long long)(side - 1) * sd;
                face_record<UNI>(p, DIR, o0, o0 + sd, rec);
                L_row(rec, 1, mc, Lr);
                const int K0 = sign, K1 = sign + 6;
#pragma unroll
                for (int t = 0; t < 8; t++)
                    vals[t] = (t >= K0 && t <= K1) ? dot5(Lr, wv(sign * 5 + 0, F - 3 + t), wv(sign * 5 + 1, F - 3 + t),
                                                          wv(sign * 5 + 2, F - 3 + t), wv(sign * 5 + 3, F - 3 + t),
                                                          wv(sign * 5 + 4, F - 3 + t))
                                                   : (R)0.0;
                R res;
                if (!(near && closure(sign, lo, hi, sign ? 4 : 3, sign ? 3 : 4, F, n, vals, res)))
                    res = hflag == 2 ? (sign ? weno7_m(vals) : weno7_p(vals)) : (sign ? weno5_m(vals) : weno5_p(vals));
                R_col(rec, 1, mc, Rc);
                res_s[w][lane] = res;
#pragma unroll
                for (int m = 0; m < 5; m++) rc_s[w][lane][m] = Rc[m];
            }
        }
        __syncwarp();
        if (lane < 20 && charf) {            // lane (face, sign, field m): the sum over c in order
            const int sign = q >= 5, m = q - 5 * sign, b0 = side * 10 + sign * 5;
            R o = rc_s[w][b0][m] * res_s[w][b0];
#pragma unroll
            for (int c = 1; c < 5; c++) o = o + rc_s[w][b0 + c][m] * res_s[w][b0 + c];
            out_s[w][side][q] = o;
        }
        __syncwarp();
        if (lane < 5) {
            const int m = lane;
            const R *cur = out_s[w][1], *prv = out_s[w][0];
            const R aj = (R)metric<UNI>(p, M_AJAC, oX);
            R acc = DIR == 0 ? (R)0.0 : (R)du[m * N + ci];
            if (p.has_bnd && rule_cell(p, DIR, X, n)) {       // du_rule_cell, field m
                const bool only_lo = lo && !hi, only_hi = hi && !lo;
                const bool first = X == 0, last = X == n - 1;
                if (only_lo && p.nonref_lo[DIR] == 1 && first) {
                    acc += (R)0.0;
                } else if ((only_lo && first) || (only_hi && last)) {
                    R tmp;
                    if (first) {
                        tmp = wv(m, X + 1) - wv(m, X);
                    } else {
                        const R f0 = wv(m, X), f1 = wv(m, X - 1), f2 = wv(m, X - 2);
                        const R tr = f0 + (R)0.5 * minmod2(f0 - f1, f0 - f1);
                        const R tl = f1 + (R)0.5 * minmod2(f0 - f1, f1 - f2);
                        tmp = tr - tl;
                    }
                    acc += div_const(-aj * tmp, h, ih);
                } else {
                    acc += div_const(-aj * (cur[m] - prv[m]), h, ih);
                }
                if (only_hi && p.nonref_hi[DIR] == 1 && last) {
                    acc += (R)0.0;
                } else if ((DIR != 1 && only_lo && first) || (only_hi && last)) {
                    R tmp;
                    if (first) {
                        const R f0 = wv(5 + m, X), f1 = wv(5 + m, X + 1), f2 = wv(5 + m, X + 2);
                        const R tr = f1 - (R)0.5 * minmod2(f2 - f1, f1 - f0);
                        const R tl = f0 - (R)0.5 * minmod2(f1 - f0, f1 - f0);
                        tmp = tr - tl;
                    } else {
                        tmp = wv(5 + m, X) - wv(5 + m, X - 1);
                    }
                    acc += div_const(-aj * tmp, h, ih);
                } else {
                    acc += div_const(-aj * (cur[5 + m] - prv[5 + m]), h, ih);
                }
            } else {                                          // add_du, field m
                acc += div_const(-aj * (cur[m] - prv[m]), h, ih);
                acc += div_const(-aj * (cur[5 + m] - prv[5 + m]), h, ih);
            }
            du[m * N + ci] = acc;
        }
        __syncwarp();
    }
}

template <int DIR, bool UNI, bool EPS0, int KIND, int MINB, bool SPLIT, typename R>
cudaError_t launch_dir4(const Params &p, cudaStream_t st) {
    constexpr int LC = Shape<DIR>::LC, LY = 32 / LC;
    const int n = DIR == 0 ? p.nx : (DIR == 1 ? p.ny : p.nz);
    const long long ngx = (p.nx + LC - 1) / LC;
    const long long groups = DIR == 0 ? (long long)p.ny * p.nz : ngx * (DIR == 1 ? p.nz : p.ny);
    // split lines into segments when there are fewer than about four waves
    // of warps; a segment re-splits 8 points and re-forms one face
    const long long want = 4LL * 148 * MINB * SW;
    long long nseg = (want + groups - 1) / groups;
    long long maxseg = n / (4 * LY) > 0 ? n / (4 * LY) : 1;
    if (nseg > maxseg) nseg = maxseg;
    if (nseg < 1) nseg = 1;
    int seg_len = (int)((n + nseg - 1) / nseg);
    seg_len = (seg_len + LY - 1) / LY * LY;
    nseg = (n + seg_len - 1) / seg_len;
    dim3 grid((unsigned)((groups + SW - 1) / SW), (unsigned)nseg);
    constexpr int smem = SW * 10 * (Shape<DIR>::RING + 2 * LY) * LC * (int)sizeof(R);
    static bool attr_set = false;             // above the 48 KB default
    if (!attr_set) {
        cudaError_t e = cudaFuncSetAttribute(k_sweep4<DIR, UNI, EPS0, KIND, MINB, SPLIT, R>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
        attr_set = true;
    }
    k_sweep4<DIR, UNI, EPS0, KIND, MINB, SPLIT, R><<<grid, 32 * SW, smem, st>>>(p, seg_len);
    return cudaGetLastError();
}

// FP64: register budget for 3 blocks per SM; FP32 (the precision form): 4
template <bool UNI, bool EPS0, int KIND, bool SPLIT, typename R>
cudaError_t dir4s(const Params &p, int dir, cudaStream_t st) {
    constexpr int MINB = sizeof(R) == 8 ? 3 : 4;
    if (dir == 0) return launch_dir4<0, UNI, EPS0, KIND, MINB, SPLIT, R>(p, st);
    if (dir == 1) return launch_dir4<1, UNI, EPS0, KIND, MINB, SPLIT, R>(p, st);
    return launch_dir4<2, UNI, EPS0, KIND, MINB, SPLIT, R>(p, st);
}
template <bool UNI, bool EPS0, int KIND, typename R>
cudaError_t dir4k(const Params &p, int dir, cudaStream_t st) {
    if (KIND == K_HYBC && !p.has_bnd) return dir4s<UNI, EPS0, KIND, true, R>(p, dir, st);
    return dir4s<UNI, EPS0, KIND, false, R>(p, dir, st);
}

template <bool UNI, bool EPS0, typename R>
cudaError_t dir4(const Params &p, int dir, cudaStream_t st) {
    if (p.scheme_invis == 310 && p.charteric) return dir4k<UNI, EPS0, K_HYBC, R>(p, dir, st);
    return dir4k<UNI, EPS0, K_W7, R>(p, dir, st);
}

template <typename R>
cudaError_t dir4r(const Params &p, int dir, cudaStream_t st) {
    if (p.uniform_metrics)
        return p.epsl_sw == 0.0 ? dir4<true, true, R>(p, dir, st) : dir4<true, false, R>(p, dir, st);
    return dir4<false, false, R>(p, dir, st);
}


}  // namespace walk4
}  // namespace ocfd
