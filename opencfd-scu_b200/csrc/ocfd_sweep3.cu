// ocfd_sweep3.cu -- inviscid flux sweeps without block barriers (sm_100a, FP64).
//
// Same results as the reference's OCFD_d{x,y,z}1/2 chain (src/OCFD_Schemes_Choose.cu:88-764,
// src/OCFD_Schemes.cu, src/OCFD_flux_charteric.cu, src/OCFD_Schemes_hybrid_auto.cu:862-1023),
// organised so that every split point and every face flux is formed once and
// nothing waits on other warps: each warp walks its own lines through a ring
// of split values in shared memory, synchronising only itself.
//
// Faces that need more than the upwind UP7 formula (WENO/SYMBO/OMP/NND,
// characteristic projection, hybrid flags other than 1) go through one
// out-of-line routine that reads the face's 8-point window from the ring.
#include "ocfd_face.cuh"

#include <cuda_runtime.h>

namespace ocfd {

namespace {

constexpr unsigned FULL = 0xffffffffu;

// window over the split values of one face: at(sv, k) = value sv
// (sign * 5 + field) of stencil point k (face F+1/2: point F-3+k)
struct Win {
    const double *b;
    int ks, vs, mask, s0;
    __device__ __forceinline__ double at(int sv, int k) const { return b[((s0 + k) & mask) * ks + sv * vs]; }
};

// Steger-Warming split of LAP point o along direction DIR into fp/fm
template <int DIR, bool UNI, bool EPS0>
__device__ __forceinline__ void split_point(const Params &p, long long o, double d, double u, double v,
                                            double w, double T, double *fp, double *fm) {
    double cc = div_const(sqrt(T), p.Ama, p.inv_Ama);
    if constexpr (UNI) {
        const DirConst &dc = p.dc[DIR];
        sw_split_pre<EPS0>(d * p.tmp0, u, v, w, cc, dc.A[0], dc.A[1], dc.A[2], dc.ss,
                           dc.An[0], dc.An[1], dc.An[2], p, fp, fm);
    } else {
        const int mA = M_AKX + 3 * DIR;
        sw_split(d * p.tmp0, u, v, w, cc, p.met[mA][o], p.met[mA + 1][o], p.met[mA + 2][o], p.Gamma,
                 p.epsl_sw, p.split_C1, p.split_C3, fp, fm);
    }
}

// characteristic face record between LAP cells o0 and o1 (get_para_charteric_*,
// src/OCFD_flux_charteric.cu:330-418)
template <bool UNI>
__device__ __forceinline__ void face_record(const Params &p, int dir, long long o0, long long o1, double *rec) {
    const double *u = p.prim[1], *v = p.prim[2], *w = p.prim[3], *T = p.prim[4];
    double c0v = div_const(sqrt(T[o0]), p.Ama, p.inv_Ama);
    double c1v = div_const(sqrt(T[o1]), p.Ama, p.inv_Ama);
    double u1 = (u[o0] + u[o1]) * 0.5, v1 = (v[o0] + v[o1]) * 0.5, w1 = (w[o0] + w[o1]) * 0.5;
    double c1 = (c0v + c1v) * 0.5;
    if (UNI) {
        const DirConst &dc = p.dc[dir];
        double KK = (p.Gamma - 1.0) / (c1 * c1);
        rec[FU] = u1; rec[FV] = v1; rec[FW] = w1; rec[FC] = c1; rec[FKK] = KK;
        rec[FX1] = 1.0 / (2.0 * c1);
        double v2 = (u1 * u1 + v1 * v1 + w1 * w1) * 0.5;
        rec[FV2] = v2;
        rec[FUN] = u1 * dc.n[0] + v1 * dc.n[1] + w1 * dc.n[2];
        rec[FH] = v2 + 1.0 / KK;
        rec[FN1] = dc.n[0]; rec[FN2] = dc.n[1]; rec[FN3] = dc.n[2];
        rec[FL1] = dc.l[0]; rec[FL2] = dc.l[1]; rec[FL3] = dc.l[2];
        rec[FM1] = dc.m[0]; rec[FM2] = dc.m[1]; rec[FM3] = dc.m[2];
    } else {
        const int mA = M_AKX + 3 * dir;
        make_record(u1, v1, w1, c1, (p.met[mA][o0] + p.met[mA][o1]) * 0.5,
                    (p.met[mA + 1][o0] + p.met[mA + 1][o1]) * 0.5,
                    (p.met[mA + 2][o0] + p.met[mA + 2][o1]) * 0.5, p, rec, 1);
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
template <bool FIRST>
__device__ __forceinline__ void add_du(double *__restrict__ du, long long N, long long ci, double aj,
                                       double h, double ih, const double *cur, const double *prv,
                                       const double *old) {
#pragma unroll
    for (int m = 0; m < 5; m++) {
        double acc = FIRST ? 0.0 : old[m];
        acc += div_const(-aj * (cur[m] - prv[m]), h, ih);
        acc += div_const(-aj * (cur[5 + m] - prv[5 + m]), h, ih);
        du[m * N + ci] = acc;
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
template <int RING, int LC>
__device__ __forceinline__ void face_up7(const double *ring, int col, int F, double (&out)[10]) {
#pragma unroll
    for (int sv = 0; sv < 10; sv++) {
        double vals[8];
#pragma unroll
        for (int t = 0; t < 8; t++) vals[t] = ring[(sv * RING + ((F - 3 + t) & (RING - 1))) * LC + col];
        out[sv] = sv < 5 ? up7_p_q(vals) : up7_m_q(vals);
    }
}

// flux of face F+1/2 of one lane's line: UP7 inline, anything else out of line
template <int RING, int LC, bool UNI>
__device__ __forceinline__ void face_flux(const Params &p, int dir, const double *ring, int col, int F, int n,
                                          int hflag, long long o0, long long sd, double (&out)[10]) {
    if (up7_face(p, hflag) && !near_closure(p, dir, F, n)) {
        face_up7<RING, LC>(ring, col, F, out);
    } else {
        double tmp[10];      // a separate array, so that out stays in registers
        face_generic<UNI>(p, dir, Win{ring + col, LC, RING * LC, RING - 1, F - 3}, hflag, o0, sd, F, n, tmp);
#pragma unroll
        for (int sv = 0; sv < 10; sv++) out[sv] = tmp[sv];
    }
}

// split of one point (primitives q5, LAP offset o) into ring slot P
template <int DIR, int RING, int LC, bool UNI, bool EPS0>
__device__ __forceinline__ void ring_put(const Params &p, double *ring, int col, int P, long long o,
                                         const double (&q5)[5]) {
    double fp[5], fm[5];
    split_point<DIR, UNI, EPS0>(p, o, q5[0], q5[1], q5[2], q5[3], q5[4], fp, fm);
    const int q = P & (RING - 1);
#pragma unroll
    for (int m = 0; m < 5; m++) {
        ring[(m * RING + q) * LC + col] = fp[m];
        ring[((5 + m) * RING + q) * LC + col] = fm[m];
    }
}

__device__ __forceinline__ void load5(const Params &p, long long o, double (&q5)[5]) {
#pragma unroll
    for (int m = 0; m < 5; m++) q5[m] = __ldg(p.prim[m] + o);
}

// The parameter block is __grid_constant__ so that passing it by reference
// to the out-of-line face routine does not copy it to local memory.
// FAST: the kernel makes no calls.  A face that is not plain UP7 gets no
// flux here; the cells on both sides of it are left for k_sweep3_fix, which
// recomputes them with the same arithmetic (their indices go to the
// direction's deferred-cell list).  Keeping the call out of this loop keeps
// its live values in registers.
// MINB: resident blocks per SM the register budget is fitted to (5: 96
// registers; 4: 128).
template <int DIR, bool UNI, bool EPS0, int MINB, bool FAST>
__global__ void __launch_bounds__(32 * SW, MINB) k_sweep3(const __grid_constant__ Params p, int seg_len) {
    constexpr int LC = Shape<DIR>::LC, LY = 32 / LC, RING = Shape<DIR>::RING;
    // the next pass's points overwrite slots this pass reads unless the
    // ring spans both windows
    constexpr bool SYNC2 = 2 * LY + 6 >= RING;
    __shared__ double ring_all[SW][10 * RING * LC];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int col = lane % LC, ly = lane / LC;
    const long long grp = (long long)blockIdx.x * SW + wid;     // line group of this warp
    const int ngx = (p.nx + LC - 1) / LC;
    const long long ngroups = DIR == 0 ? (long long)p.ny * p.nz : (long long)ngx * (DIR == 1 ? p.nz : p.ny);
    if (grp >= ngroups) return;                                 // the whole warp
    double *ring = ring_all[wid];
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
    double *__restrict__ du = p.du;
    const long long N = p.N;
    const bool hybrid = p.scheme_invis == 310;
    const double h = DIR == 0 ? p.hx : (DIR == 1 ? p.hy : p.hz), ih = p.inv_h[DIR];

    // points y0-4 .. y0+3 and the face left of cell y0
    for (int r = ly; r < 8; r += LY) {
        if (colok) {
            double q5[5];
            const long long o = base + (long long)(y0 - 4 + r) * sd;
            load5(p, o, q5);
            ring_put<DIR, RING, LC, UNI, EPS0>(p, ring, col, y0 - 4 + r, o, q5);
        }
    }
    __syncwarp();
    double carry[10], cur[10];
#pragma unroll
    for (int m = 0; m < 10; m++) cur[m] = 0.0;
    int slow = 0, carry_slow = 0;
    if (ly == 0 && colok) {
        const int hf = hybrid ? (int)fl[(long long)y0 * fst] : 2;
        if constexpr (FAST) {
            slow = !up7_face(p, hf) || near_closure(p, DIR, y0 - 1, n);
            if (!slow) face_up7<RING, LC>(ring, col, y0 - 1, cur);
        } else {
            face_flux<RING, LC, UNI>(p, DIR, ring, col, y0 - 1, n, hf, base + (long long)(y0 - 1) * sd, sd, cur);
        }
    }
#pragma unroll
    for (int m = 0; m < 10; m++) carry[m] = __shfl_sync(FULL, cur[m], col);
    if constexpr (FAST) carry_slow = __shfl_sync(FULL, slow, col);

    // the primitives of this lane's next point and the flag of its next
    // face are loaded one pass ahead
    double nq[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    int nflag = 2;
    if (colok && y0 + 4 + ly <= y1 + 3) load5(p, base + (long long)(y0 + 4 + ly) * sd, nq);
    if (hybrid && colok && y0 + ly < y1) nflag = fl[(long long)(y0 + ly + 1) * fst];

    for (int Y0 = y0; Y0 < y1; Y0 += LY) {
        const int P = Y0 + 4 + ly;
        const int F = Y0 + ly;
        const bool valid = colok && F < y1;
        if (colok && P <= y1 + 3) ring_put<DIR, RING, LC, UNI, EPS0>(p, ring, col, P, base + (long long)P * sd, nq);
        const int hflag = nflag;
        if (colok && P + LY <= y1 + 3) load5(p, base + (long long)(P + LY) * sd, nq);
        if (hybrid && colok && F + LY < y1) nflag = fl[(long long)(F + LY + 1) * fst];
        __syncwarp();
        const long long ci = cb + (long long)F * cst;
        double old[5];
        if (DIR != 0 && valid) {
#pragma unroll
            for (int m = 0; m < 5; m++) old[m] = du[m * N + ci];
        }
        if constexpr (FAST) {
            slow = valid && (!up7_face(p, hflag) || near_closure(p, DIR, F, n));
            if (valid && !slow) face_up7<RING, LC>(ring, col, F, cur);
        } else {
            if (valid) face_flux<RING, LC, UNI>(p, DIR, ring, col, F, n, hflag, base + (long long)F * sd, sd, cur);
        }
        double prv[10];
#pragma unroll
        for (int m = 0; m < 10; m++) {
            double t = __shfl_up_sync(FULL, cur[m], LC);
            prv[m] = ly == 0 ? carry[m] : t;
            carry[m] = __shfl_sync(FULL, cur[m], (LY - 1) * LC + col);
        }
        bool defer = false;
        if constexpr (FAST) {
            const int up = __shfl_up_sync(FULL, slow, LC);
            const int prv_slow = ly == 0 ? carry_slow : up;
            carry_slow = __shfl_sync(FULL, slow, (LY - 1) * LC + col);
            defer = valid && (slow || prv_slow);
        }
        // the first and last cells of a bounded line go to the fix-up kernel
        if (p.has_bnd) defer = defer || (valid && rule_cell(p, DIR, F, n));
        if (FAST || p.has_bnd) {
            const unsigned mask = __ballot_sync(FULL, defer);
            if (mask) {                       // one atomic per warp
                const int leader = __ffs(mask) - 1;
                unsigned slot = 0;
                if (lane == leader) slot = atomicAdd(p.defer_count + DIR, (unsigned)__popc(mask));
                slot = __shfl_sync(FULL, slot, leader);
                if (defer) p.defer[DIR][slot + __popc(mask & ((1u << lane) - 1u))] = (unsigned)ci;
            }
        }
        if (valid && !defer) {
            double aj = metric<UNI>(p, M_AJAC, base + (long long)F * sd);
            if (DIR == 0) add_du<true>(du, N, ci, aj, h, ih, cur, prv, old);
            else          add_du<false>(du, N, ci, aj, h, ih, cur, prv, old);
        }
        if (SYNC2) __syncwarp();
    }
}

// Cells the FAST sweep deferred: each thread takes one cell, splits the 9
// points X-4 .. X+4 of its line, forms the fluxes of faces X-1/2 and X+1/2
// (UP7 or the out-of-line routine, as the inline path would) and adds the
// cell's du in the same order.
template <int DIR, bool UNI, bool EPS0>
__global__ void __launch_bounds__(128) k_sweep3_fix(const __grid_constant__ Params p) {
    const unsigned cnt = p.defer_count[DIR];
    const long long sd = DIR == 0 ? 1LL : (DIR == 1 ? p.ys : p.zs);
    const bool hybrid = p.scheme_invis == 310;
    const double h = DIR == 0 ? p.hx : (DIR == 1 ? p.hy : p.hz), ih = p.inv_h[DIR];
    for (unsigned e = blockIdx.x * blockDim.x + threadIdx.x; e < cnt; e += gridDim.x * blockDim.x) {
        const long long ci = p.defer[DIR][e];
        const int i = (int)(ci % p.nx);
        const long long r = ci / p.nx;
        const int j = (int)(r % p.ny), k = (int)(r / p.ny);
        const int X = DIR == 0 ? i : (DIR == 1 ? j : k);
        const long long oX = lap_index(p, i + OCFD_LAP, j + OCFD_LAP, k + OCFD_LAP);
        double win[90];                       // [point X-4+t][sign * 5 + field]
        for (int t = 0; t < 9; t++) {
            const long long o = oX + (long long)(t - 4) * sd;
            double q5[5], fp[5], fm[5];
            load5(p, o, q5);
            split_point<DIR, UNI, EPS0>(p, o, q5[0], q5[1], q5[2], q5[3], q5[4], fp, fm);
#pragma unroll
            for (int m = 0; m < 5; m++) { win[t * 10 + m] = fp[m]; win[t * 10 + 5 + m] = fm[m]; }
        }
        // flag of face F+1/2 is entry F+1 of the direction's flag array
        auto flag_at = [&](int e1) -> int {
            if (!hybrid) return 2;
            long long q = DIR == 0 ? (long long)e1 + (long long)(p.nx + 1) * ((long long)j + (long long)p.ny * k)
                        : DIR == 1 ? (long long)i + (long long)p.nx * ((long long)e1 + (long long)(p.ny + 1) * k)
                                   : (long long)i + (long long)p.nx * ((long long)j + (long long)p.ny * e1);
            return p.flag[DIR][q];
        };
        const int n = DIR == 0 ? p.nx : (DIR == 1 ? p.ny : p.nz);
        double cur[10], prv[10];
        for (int side = 0; side < 2; side++) {          // 0: face X-1/2, 1: face X+1/2
            const int hf = flag_at(X + side);
            const int F = X - 1 + side;
            double *out = side ? cur : prv;
            if (up7_face(p, hf) && !near_closure(p, DIR, F, n)) {
                for (int sv = 0; sv < 10; sv++) {
                    double vals[8];
#pragma unroll
                    for (int t = 0; t < 8; t++) vals[t] = win[(side + t) * 10 + sv];
                    out[sv] = sv < 5 ? up7_p_q(vals) : up7_m_q(vals);
                }
            } else {
                face_generic<UNI>(p, DIR, Win{win, 10, 1, 15, side}, hf, oX + (long long)(side - 1) * sd, sd,
                                  F, n, out);
            }
        }
        const double aj = metric<UNI>(p, M_AJAC, oX);
        // du of the cell: x+ then x- for every field (put_du_p_kernel /
        // put_du_m_kernel, src/OCFD_Schemes.cu:293-381; the characteristic
        // kernels' put_du_character_{p,m}_kernel, src/OCFD_flux_charteric.cu:16-118,
        // and OCFD_bound_character_kernel_{p,m}, :121-319)
        const int scheme = p.scheme_invis;
        const bool char_kernel = p.charteric && (scheme == 304 || scheme == 305 || scheme == 310);
        const bool lo = p.bnd_lo[DIR], hi = p.bnd_hi[DIR];
        const bool only_lo = lo && !hi, only_hi = hi && !lo;     // flag 1..6, not 7..9
        const bool first = X == 0, last = X == n - 1;
        for (int m = 0; m < 5; m++) {
            double acc = DIR == 0 ? 0.0 : p.du[m * p.N + ci];
            // P side
            if (!char_kernel ? (first && p.nonref_lo[DIR] == 1) : (only_lo && p.nonref_lo[DIR] == 1 && first)) {
                acc += 0.0;
            } else if (char_kernel && ((only_lo && first) || (only_hi && last))) {
                double tmp;
                if (first) {
                    tmp = (win[5 * 10 + m] - win[4 * 10 + m]);
                } else {
                    const double f0 = win[4 * 10 + m], f1 = win[3 * 10 + m], f2 = win[2 * 10 + m];
                    const double tr = f0 + 0.5 * minmod2(f0 - f1, f0 - f1);
                    const double tl = f1 + 0.5 * minmod2(f0 - f1, f1 - f2);
                    tmp = tr - tl;
                }
                acc += div_const(-aj * tmp, h, ih);
            } else {
                acc += div_const(-aj * (cur[m] - prv[m]), h, ih);
            }
            // M side; the reference's y kernel tests flag 3 for its lower
            // face, so that first-order flux never applies on y
            if (!char_kernel ? (last && p.nonref_hi[DIR] == 1) : (only_hi && p.nonref_hi[DIR] == 1 && last)) {
                acc += 0.0;
            } else if (char_kernel && ((DIR != 1 && only_lo && first) || (only_hi && last))) {
                double tmp;
                if (first) {
                    const double f0 = win[4 * 10 + 5 + m], f1 = win[5 * 10 + 5 + m], f2 = win[6 * 10 + 5 + m];
                    const double tr = f1 - 0.5 * minmod2(f2 - f1, f1 - f0);
                    const double tl = f0 - 0.5 * minmod2(f1 - f0, f1 - f0);
                    tmp = tr - tl;
                } else {
                    tmp = (win[4 * 10 + 5 + m] - win[3 * 10 + 5 + m]);
                }
                acc += div_const(-aj * tmp, h, ih);
            } else {
                acc += div_const(-aj * (cur[5 + m] - prv[5 + m]), h, ih);
            }
            p.du[m * p.N + ci] = acc;
        }
    }
}

template <int DIR, bool UNI, bool EPS0, int MINB, bool FAST>
cudaError_t launch_dir(const Params &p, cudaStream_t st) {
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
    k_sweep3<DIR, UNI, EPS0, MINB, FAST><<<grid, 32 * SW, 0, st>>>(p, seg_len);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || !(FAST || p.has_bnd)) return e;
    // the deferred-cell count is only known on the device: a fixed grid
    // that strides over it (usually a few thousand cells, often none)
    k_sweep3_fix<DIR, UNI, EPS0><<<2 * 148, 128, 0, st>>>(p);
    return cudaGetLastError();
}

template <bool UNI, bool EPS0, int MINB, bool FAST>
cudaError_t launch3m(const Params &p, cudaStream_t st) {
    cudaError_t e;
    if ((FAST || p.has_bnd) && (e = cudaMemsetAsync(p.defer_count, 0, 3 * sizeof(unsigned), st)) != cudaSuccess)
        return e;
    if ((e = launch_dir<0, UNI, EPS0, MINB, FAST>(p, st)) != cudaSuccess) return e;
    if ((e = launch_dir<1, UNI, EPS0, MINB, FAST>(p, st)) != cudaSuccess) return e;
    return launch_dir<2, UNI, EPS0, MINB, FAST>(p, st);
}
// impl 4: the call-free kernel with deferred cells where the scheme has a
// UP7 fast path; impl 5 (and every other scheme): every face through the
// in-kernel dispatch
bool use_fast(const Params &p) {
    const bool fast_scheme = (p.scheme_invis == 301 && !p.charteric) || p.scheme_invis == 310;
    return p.sweep_impl == 4 && fast_scheme && p.defer[0];
}
template <bool UNI, bool EPS0>
cudaError_t launch3(const Params &p, cudaStream_t st) {
    if (p.has_bnd && !p.defer[0]) return cudaErrorNotSupported;   // boundary cells need the lists
    if (use_fast(p)) return launch3m<UNI, EPS0, 4, true>(p, st);
    return launch3m<UNI, EPS0, 5, false>(p, st);
}

}  // namespace

// kernels one launch_sweeps3 issues
int sweeps3_kernels(const Params &p) { return (use_fast(p) || p.has_bnd) ? 6 : 3; }

cudaError_t launch_sweeps3(const Params &p, cudaStream_t st) {
    if (p.uniform_metrics)
        return p.epsl_sw == 0.0 ? launch3<true, true>(p, st) : launch3<true, false>(p, st);
    return launch3<false, false>(p, st);
}

}  // namespace ocfd
