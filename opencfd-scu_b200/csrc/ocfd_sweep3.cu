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
#include "ocfd_walk.cuh"

#include <cuda_runtime.h>

namespace ocfd {

cudaError_t launch_sweep4_fix(const Params &p, int dir, cudaStream_t st);

namespace {

using namespace walk;

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

// The parameter block is __grid_constant__ so that passing it by reference
// to the out-of-line face routine does not copy it to local memory.
// FAST: the kernel makes no calls.  A face that is not plain UP7 gets no
// flux here; the cells on both sides of it are left for k_sweep3_fix, which
// recomputes them with the same arithmetic (their indices go to the
// direction's deferred-cell list).  Keeping the call out of this loop keeps
// its live values in registers.
// MINB: resident blocks per SM the register budget is fitted to (5: 96
// registers; 4: 128).
template <int DIR, bool UNI, bool EPS0, int MINB, bool FAST, typename R = double>
__global__ void __launch_bounds__(32 * SW, MINB) k_sweep3(const __grid_constant__ Params p, int seg_len) {
    constexpr int LC = Shape<DIR>::LC, LY = 32 / LC, RING = Shape<DIR>::RING;
    // the next pass's points overwrite slots this pass reads unless the
    // ring spans both windows
    constexpr bool SYNC2 = 2 * LY + 6 >= RING;
    static_assert(FAST || sizeof(R) == 8, "the in-loop dispatch is FP64 only");
    __shared__ R ring_all[SW][10 * RING * LC];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int col = lane % LC, ly = lane / LC;
    const long long grp = (long long)blockIdx.x * SW + wid;     // line group of this warp
    const int ngx = (p.nx + LC - 1) / LC;
    const long long ngroups = DIR == 0 ? (long long)p.ny * p.nz : (long long)ngx * (DIR == 1 ? p.nz : p.ny);
    if (grp >= ngroups) return;                                 // the whole warp
    R *ring = ring_all[wid];
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
    const bool hybrid = p.scheme_invis == 310;
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
    R carry[10], cur[10];
#pragma unroll
    for (int m = 0; m < 10; m++) cur[m] = (R)0.0;
    int slow = 0, carry_slow = 0;
    if (ly == 0 && colok) {
        const int hf = hybrid ? flag_at(p, DIR, fl, (long long)y0 * fst) : 2;
        if constexpr (FAST) {
            slow = !up7_face(p, hf) || near_closure(p, DIR, y0 - 1, n);
            if (!slow) face_up7<RING, LC>(ring, col, y0 - 1, cur);
        } else {
            if constexpr (sizeof(R) == 8)
                face_flux<RING, LC, UNI>(p, DIR, ring, col, y0 - 1, n, hf, base + (long long)(y0 - 1) * sd, sd, cur);
        }
    }
#pragma unroll
    for (int m = 0; m < 10; m++) carry[m] = __shfl_sync(FULL, cur[m], col);
    if constexpr (FAST) carry_slow = __shfl_sync(FULL, slow, col);

    // the primitives of this lane's next point and the flag of its next
    // face are loaded one pass ahead
    R nq[5] = {(R)0.0, (R)0.0, (R)0.0, (R)0.0, (R)0.0};
    int nflag = 2;
    if (colok && y0 + 4 + ly <= y1 + 3) load5(p, base + (long long)(y0 + 4 + ly) * sd, nq);
    if (hybrid && colok && y0 + ly < y1) nflag = flag_at(p, DIR, fl, (long long)(y0 + ly + 1) * fst);

    for (int Y0 = y0; Y0 < y1; Y0 += LY) {
        const int P = Y0 + 4 + ly;
        const int F = Y0 + ly;
        const bool valid = colok && F < y1;
        if (colok && P <= y1 + 3) ring_put<DIR, RING, LC, UNI, EPS0>(p, ring, col, P, base + (long long)P * sd, nq);
        const int hflag = nflag;
        if (colok && P + LY <= y1 + 3) load5(p, base + (long long)(P + LY) * sd, nq);
        if (hybrid && colok && F + LY < y1) nflag = flag_at(p, DIR, fl, (long long)(F + LY + 1) * fst);
        __syncwarp();
        // (lanes past the segment's end form an index they never use)
        const long long ci = valid ? OCFD_IDX(p, cb + (long long)F * cst, N) : 0;
        R old[5];
        if (DIR != 0 && valid) {
#pragma unroll
            for (int m = 0; m < 5; m++) old[m] = du[m * N + ci];
        }
        if constexpr (FAST) {
            slow = valid && (!up7_face(p, hflag) || near_closure(p, DIR, F, n));
            if (valid && !slow) face_up7<RING, LC>(ring, col, F, cur);
        } else {
            if constexpr (sizeof(R) == 8)
                if (valid) face_flux<RING, LC, UNI>(p, DIR, ring, col, F, n, hflag, base + (long long)F * sd, sd, cur);
        }
        R prv[10];
#pragma unroll
        for (int m = 0; m < 10; m++) {
            R t = __shfl_up_sync(FULL, cur[m], LC);
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
                if (defer) p.defer[DIR][OCFD_IDX(p, (long long)slot + __popc(mask & ((1u << lane) - 1u)), p.N)] = (unsigned)ci;
            }
        }
        if (valid && !defer) {
            R aj = (R)metric<UNI>(p, M_AJAC, base + (long long)F * sd);
            if (DIR == 0) add_du<true>(du, N, ci, aj, h, ih, cur, prv, old);
            else          add_du<false>(du, N, ci, aj, h, ih, cur, prv, old);
        }
        if (SYNC2) __syncwarp();
    }
}

// Cells the FAST sweep deferred, one warp per cell (few cells, each with the
// longest arithmetic of the path, so the work of a cell is spread over
// lanes): lanes 0..8 split the points X-4 .. X+4 into the warp's window;
// lane (face, value) forms a value of the fluxes of faces X-1/2 and X+1/2 --
// UP7, or the out-of-line routine's component-wise reconstruction or
// closure; for a characteristic face lane (face, sign, field c) projects on
// field c, reconstructs and takes column c of R, and lane (face, sign, m)
// sums the products over c in the routine's order (face_generic); lanes 0..4
// then add the cell's du, field by field, in the same order as the walk.
constexpr int FIXW = 4;        // warps (cells in flight) per block

template <int DIR, bool UNI, bool EPS0>
__global__ void __launch_bounds__(32 * FIXW) k_sweep3_fix(const __grid_constant__ Params p) {
    __shared__ double win_s[FIXW][90];          // [point X-4+t][sign * 5 + field]
    __shared__ double res_s[FIXW][20];          // characteristic faces: reconstruction of (face, sign, c)
    __shared__ double rc_s[FIXW][20][5];        //   and column c of R
    __shared__ double out_s[FIXW][2][10];       // fluxes of faces X-1/2 and X+1/2
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned cnt = p.defer_count[DIR];
    const long long sd = DIR == 0 ? 1LL : (DIR == 1 ? p.ys : p.zs);
    const int scheme = p.scheme_invis;
    const bool hybrid = scheme == 310;
    const bool char_scheme = p.charteric && (scheme == 304 || scheme == 305 || scheme == 310);
    const bool lo = p.bnd_lo[DIR], hi = p.bnd_hi[DIR];
    const bool bnd = lo || hi;
    const double h = DIR == 0 ? p.hx : (DIR == 1 ? p.hy : p.hz), ih = p.inv_h[DIR];
    const int n = DIR == 0 ? p.nx : (DIR == 1 ? p.ny : p.nz);
    double *win = win_s[w];
    for (unsigned e = blockIdx.x * FIXW + w; e < cnt; e += gridDim.x * FIXW) {
        const long long ci = OCFD_IDX(p, (long long)p.defer[DIR][e], p.N);
        const int i = (int)(ci % p.nx);
        const long long r = ci / p.nx;
        const int j = (int)(r % p.ny), k = (int)(r / p.ny);
        const int X = DIR == 0 ? i : (DIR == 1 ? j : k);
        const long long oX = lap_index(p, i + OCFD_LAP, j + OCFD_LAP, k + OCFD_LAP);
        if (lane < 9) {
            const long long o = oX + (long long)(lane - 4) * sd;
            double q5[5], fp[5], fm[5];
            load5(p, o, q5);
            split_point<DIR, UNI, EPS0>(p, o, q5[0], q5[1], q5[2], q5[3], q5[4], fp, fm);
#pragma unroll
            for (int m = 0; m < 5; m++) { win[lane * 10 + m] = fp[m]; win[lane * 10 + 5 + m] = fm[m]; }
        }
        __syncwarp();
        // flag of face F+1/2 is entry F+1 of the direction's flag array
        const int side = lane / 10, q = lane - 10 * (lane / 10);
        const int e1 = X + (side & 1);
        int hf = 2;
        if (hybrid) {
            const long long qq = DIR == 0 ? (long long)e1 + (long long)(p.nx + 1) * ((long long)j + (long long)p.ny * k)
                               : DIR == 1 ? (long long)i + (long long)p.nx * ((long long)e1 + (long long)(p.ny + 1) * k)
                                          : (long long)i + (long long)p.nx * ((long long)j + (long long)p.ny * e1);
            hf = flag_at(p, DIR, p.flag[DIR], qq);
        }
        const int F = X - 1 + (side & 1);
        const bool up7 = up7_face(p, hf) && !near_closure(p, DIR, F, n);
        const bool gchar = !up7 && char_scheme && !(hybrid && hf == 1);
        const Win wv{win, 10, 1, 15, side & 1};
        if (lane < 20) {
            const int sign = q >= 5, mc = q - 5 * sign;
            int KA, KB;
            extents(scheme, char_scheme, sign, KA, KB);
            if (up7) {
                double vals[8];
#pragma unroll
                for (int t = 0; t < 8; t++) vals[t] = win[(side + t) * 10 + q];
                out_s[w][side][q] = q < 5 ? up7_p_q(vals) : up7_m_q(vals);
            } else if (p.charteric && !char_scheme) {       // the reference adds nothing
                out_s[w][side][q] = 0.0;
            } else if (!gchar) {                             // component-wise
                double vals[8];
#pragma unroll
                for (int t = 0; t < 8; t++) vals[t] = wv.at(q, t);
                int hq = hf;
                if (hybrid && !char_scheme && mc > 0 && p.nochar_comp_flag) hq = p.nochar_comp_flag;
                double o;
                if (!(bnd && closure(sign, lo, hi, KA, KB, F, n, vals, o))) o = recon_one(p, scheme, hq, sign, vals);
                out_s[w][side][q] = o;
            } else {                                         // characteristic field c = mc of this sign
                double rec[FP_N], Lr[5], Rc[5], vals[8];
                const long long o0 = oX + (long long)(side - 1) * sd;
                face_record<UNI>(p, DIR, o0, o0 + sd, rec);
                L_row(rec, 1, mc, Lr);
#pragma unroll
                for (int t = 0; t < 8; t++)
                    vals[t] = dot5(Lr, wv.at(sign * 5 + 0, t), wv.at(sign * 5 + 1, t), wv.at(sign * 5 + 2, t),
                                   wv.at(sign * 5 + 3, t), wv.at(sign * 5 + 4, t));
                double res;
                if (!(bnd && closure(sign, lo, hi, KA, KB, F, n, vals, res)))
                    res = recon_one(p, scheme, hf, sign, vals);
                R_col(rec, 1, mc, Rc);
                res_s[w][lane] = res;
#pragma unroll
                for (int m = 0; m < 5; m++) rc_s[w][lane][m] = Rc[m];
            }
        }
        __syncwarp();
        if (lane < 20 && gchar) {        // lane (face, sign, field m): the sum over c in order
            const int sign = q >= 5, m = q - 5 * sign, b0 = side * 10 + sign * 5;
            double o = rc_s[w][b0][m] * res_s[w][b0];
#pragma unroll
            for (int c = 1; c < 5; c++) o = o + rc_s[w][b0 + c][m] * res_s[w][b0 + c];
            out_s[w][side][q] = o;
        }
        __syncwarp();
        if (lane < 5) {
            // du of the cell: x+ then x- for field m (put_du_p_kernel /
            // put_du_m_kernel, src/OCFD_Schemes.cu:293-381; the characteristic
            // kernels' put_du_character_{p,m}_kernel, src/OCFD_flux_charteric.cu:16-118,
            // and OCFD_bound_character_kernel_{p,m}, :121-319)
            const int m = lane;
            const double *cur = out_s[w][1], *prv = out_s[w][0];
            const double aj = metric<UNI>(p, M_AJAC, oX);
            const bool char_kernel = char_scheme;
            const bool only_lo = lo && !hi, only_hi = hi && !lo;     // flag 1..6, not 7..9
            const bool first = X == 0, last = X == n - 1;
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
        __syncwarp();                    // the window and fluxes are reused by the next cell
    }
}

template <int DIR, bool UNI, bool EPS0, int MINB, bool FAST, typename R = double>
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
    k_sweep3<DIR, UNI, EPS0, MINB, FAST, R><<<grid, 32 * SW, 0, st>>>(p, seg_len);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || !(FAST || p.has_bnd)) return e;
    // FP32: the fix-up of the precision form (ocfd_sweep4.cu)
    if (sizeof(R) == 4) return launch_sweep4_fix(p, DIR, st);
    // the deferred-cell count is only known on the device: a fixed grid
    // that strides over it (usually a few thousand cells, often none)
    k_sweep3_fix<DIR, UNI, EPS0><<<2 * 148, 32 * FIXW, 0, st>>>(p);
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

// One direction of the walk alone (1 or 2 kernels); when sweeps3_defers(p)
// the caller clears p.defer_count once before the first direction.
bool sweeps3_defers(const Params &p) { return use_fast(p) || p.has_bnd; }

namespace {
template <bool UNI, bool EPS0>
cudaError_t dir3(const Params &p, int dir, cudaStream_t st) {
    if (p.has_bnd && !p.defer[0]) return cudaErrorNotSupported;
    if (p.mixed) {              // precision form: the call-free walk in FP32
        if (!use_fast(p) || p.scheme_invis != 310) return cudaErrorNotSupported;
        if (dir == 0) return launch_dir<0, UNI, EPS0, 6, true, float>(p, st);
        if (dir == 1) return launch_dir<1, UNI, EPS0, 6, true, float>(p, st);
        return launch_dir<2, UNI, EPS0, 6, true, float>(p, st);
    }
    if (use_fast(p)) {
        if (dir == 0) return launch_dir<0, UNI, EPS0, 4, true>(p, st);
        if (dir == 1) return launch_dir<1, UNI, EPS0, 4, true>(p, st);
        return launch_dir<2, UNI, EPS0, 4, true>(p, st);
    }
    if (dir == 0) return launch_dir<0, UNI, EPS0, 5, false>(p, st);
    if (dir == 1) return launch_dir<1, UNI, EPS0, 5, false>(p, st);
    return launch_dir<2, UNI, EPS0, 5, false>(p, st);
}
}  // namespace

// the fix-up of one direction's deferred cells (FP64)
cudaError_t launch_sweep3_fix(const Params &p, int dir, cudaStream_t st) {
    if (p.uniform_metrics) {
        if (p.epsl_sw == 0.0) {
            if (dir == 0) k_sweep3_fix<0, true, true><<<2 * 148, 32 * FIXW, 0, st>>>(p);
            else if (dir == 1) k_sweep3_fix<1, true, true><<<2 * 148, 32 * FIXW, 0, st>>>(p);
            else k_sweep3_fix<2, true, true><<<2 * 148, 32 * FIXW, 0, st>>>(p);
        } else {
            if (dir == 0) k_sweep3_fix<0, true, false><<<2 * 148, 32 * FIXW, 0, st>>>(p);
            else if (dir == 1) k_sweep3_fix<1, true, false><<<2 * 148, 32 * FIXW, 0, st>>>(p);
            else k_sweep3_fix<2, true, false><<<2 * 148, 32 * FIXW, 0, st>>>(p);
        }
    } else {
        if (dir == 0) k_sweep3_fix<0, false, false><<<2 * 148, 32 * FIXW, 0, st>>>(p);
        else if (dir == 1) k_sweep3_fix<1, false, false><<<2 * 148, 32 * FIXW, 0, st>>>(p);
        else k_sweep3_fix<2, false, false><<<2 * 148, 32 * FIXW, 0, st>>>(p);
    }
    return cudaGetLastError();
}

cudaError_t launch_sweep3_dir(const Params &p, int dir, cudaStream_t st) {
    if (p.uniform_metrics)
        return p.epsl_sw == 0.0 ? dir3<true, true>(p, dir, st) : dir3<true, false>(p, dir, st);
    return dir3<false, false>(p, dir, st);
}

cudaError_t launch_sweeps3(const Params &p, cudaStream_t st) {
    if (p.uniform_metrics)
        return p.epsl_sw == 0.0 ? launch3<true, true>(p, st) : launch3<true, false>(p, st);
    return launch3<false, false>(p, st);
}

}  // namespace ocfd
