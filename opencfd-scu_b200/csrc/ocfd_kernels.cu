// ocfd_kernels.cu -- CUDA kernels of the per-RK-stage RHS path (sm_100a, FP64).
//
// One stage (reference driver order, src/OCFD_NS_Solver.cu:76-89 and
// src/OCFD_Stream.cu:28-54):
//   [KRK=1, hybrid] sensor        -> int8 face flags            (k_sensor_march)
//   ghost fill of d,u,v,w,T        (periodic wrap on device)    (k_ghost_prim)
//   inviscid x, y, z sweeps        -> du (single writer, fixed order)  (ocfd_sweep3/4.cu, ocfd_march.cu)
//   viscous gradients, Ev, Ev ghosts, divergence -> du         (k_vis_*)
//   RK stage + cons->prim + face re-projection                 (fused into k_vis_div / k_vdiv)
// and the reductions of the analysis after the path.
#include "ocfd_fp32.cuh"
#include "ocfd_tma.cuh"

#include <cuda_runtime.h>

namespace ocfd {

// ---------------------------------------------------------------------------
// hybrid sensor, style 2: Comput_P + Comput_Scheme_point_{x,y,z}_Jameson
// (src/OCFD_Schemes_hybrid_auto.cu:48-68, :611-703).  Flag q along DIR
// belongs to cell q-1; P = p00*d*T is formed on the fly from the LAP-box d,T
// as they stand before this stage's ghost fill.  The three arrays' entries
// of one cell share its value, so each cell of the extended box (-1 .. n-1
// in each direction) forms it once and writes the entries it owns: entry
// i+1 of the x array (j, k interior), j+1 of the y array, k+1 of the z
// array.
// ---------------------------------------------------------------------------
// Each thread marches along z through a segment of its (i, j) column of the
// extended box: a block covers a 32 x 8 tile of (i, j), P of the column's
// planes k-1, k, k+1 stays in registers, and the x and y neighbours of
// plane k are read through L1 from the rows the block's own warps load (10
// loads a cell instead of the 26 of one thread per cell).  The sum of the
// three terms is formed in the reference's order.
constexpr int SEN_X = 32, SEN_Y = 8;
template <typename R>
__global__ void __launch_bounds__(SEN_X * SEN_Y) k_sensor_march(Params p, int seg) {
    const int ex = p.nx + 1, ey = p.ny + 1, ez = p.nz + 1;
    const int ntx = (ex + SEN_X - 1) / SEN_X;
    const int i = (int)(blockIdx.x % ntx) * SEN_X + (int)(threadIdx.x % SEN_X) - 1;
    const int j = (int)(blockIdx.x / ntx) * SEN_Y + (int)(threadIdx.x / SEN_X) - 1;
    const int ka = (int)blockIdx.y * seg - 1, kb = min(ez - 1, ka + seg);   // planes ka .. kb-1
    const bool col = i < ex - 1 && j < ey - 1;              // i, j in -1 .. n-1
    const R *d = prim_r<R>(p, 0), *T = prim_r<R>(p, 4);
    const R p00 = (R)p.p00;
    auto P = [&](long long o) { return p00 * d[o] * T[o]; };
    const int lane = threadIdx.x & 31;
    // a column with i and j both ghost owns no entry; it still takes part in
    // the warp's ballots
    const bool any = col && (i >= 0 || j >= 0);
    long long c = any ? lap_index(p, i + OCFD_LAP, j + OCFD_LAP, ka + OCFD_LAP) : 0;
    R Pz0 = (R)0, Pz1 = (R)0;
    if (any) { Pz0 = P(c - p.zs); Pz1 = P(c); }
    unsigned nx1 = 0, ny1 = 0, nz1 = 0;
    for (int k = ka; k < kb; k++, c += p.zs) {
        int kp = 1;
        bool inx = false, iny = false, inz = false;
        if (any) {
            inx = j >= 0 && k >= 0; iny = i >= 0 && k >= 0; inz = i >= 0 && j >= 0;
            const R P0 = Pz1, Pzm = Pz0, Pzp = P(c + p.zs);
            R Pm = P(c - 1), Pp = P(c + 1);
            R dp0 = fabs(-Pm + 2*P0 - Pp)/(Pm + 2*P0 + Pp);
            Pm = P(c - p.ys); Pp = P(c + p.ys);
            dp0 += fabs(-Pm + 2*P0 - Pp)/(Pm + 2*P0 + Pp);
            dp0 += fabs(-Pzm + 2*P0 - Pzp)/(Pzm + 2*P0 + Pzp);
            if (dp0 > (R)p.dp1) kp += 1;
            if (dp0 > (R)p.dp2) kp += 1;
            if (inx) p.flag[0][(long long)(i + 1) + (long long)ex * ((long long)j + (long long)p.ny * k)] = (int8_t)kp;
            if (iny) p.flag[1][(long long)i + (long long)p.nx * ((long long)(j + 1) + (long long)ey * k)] = (int8_t)kp;
            if (inz) p.flag[2][(long long)i + (long long)p.nx * ((long long)j + (long long)p.ny * (k + 1))] = (int8_t)kp;
            Pz0 = P0; Pz1 = Pzp;
        }
        const bool non1 = kp != 1;
        nx1 += non1 && inx; ny1 += non1 && iny; nz1 += non1 && inz;
    }
    // faces per direction whose flag is not 1: one sum per warp for the
    // whole segment (an atomic per warp and plane queued on three words)
    if (p.flag_count) {
        nx1 = __reduce_add_sync(0xffffffffu, nx1);
        ny1 = __reduce_add_sync(0xffffffffu, ny1);
        nz1 = __reduce_add_sync(0xffffffffu, nz1);
        if (lane == 0) {
            if (nx1) atomicAdd(p.flag_count + 0, nx1);
            if (ny1) atomicAdd(p.flag_count + 1, ny1);
            if (nz1) atomicAdd(p.flag_count + 2, nz1);
        }
    }
}

// ---------------------------------------------------------------------------
// periodic ghost fill of LAP-box fields, exchange_boundary_{x,y,z}_packed_dev
// (src/OCFD_mpi_dev.cu:186-310) on one GPU: x ghosts for interior (y,z),
// y ghosts for interior (x,z), z ghosts for interior (x,y).  The three slabs
// read only interior cells, so one launch fills all of them.
// fields: list of base pointers; dirmask selects directions per field.
// ---------------------------------------------------------------------------
template <typename T> struct GhostList { T *f[12]; int dirmask[12]; int n; };

template <typename T>
__global__ void k_ghost(Params p, GhostList<T> g) {
    // one field per grid row; element q of its ghost slabs (x, then y, then
    // z), decomposed with 32-bit arithmetic (a field's slabs hold fewer than
    // 2^31 elements)
    constexpr unsigned L = OCFD_LAP, L2 = 2 * OCFD_LAP;
    const unsigned nx = (unsigned)p.nx, ny = (unsigned)p.ny, nz = (unsigned)p.nz;
    const unsigned sx = L2 * ny * nz, sy = L2 * nx * nz, sz = L2 * nx * ny;
    unsigned q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= sx + sy + sz) return;
    T *f = g.f[blockIdx.y];
    const int mask = g.dirmask[blockIdx.y];
    if (q < sx) {
        if (!(mask & 1) || !p.periodic[0]) return;
        const unsigned i = q % L2, r = q / L2;
        const unsigned j = r % ny + L, k = r / ny + L;
        const unsigned dst = i < L ? i : nx + i;             // 0..L-1  or  nx+L..nx+2L-1
        const unsigned src = i < L ? nx + i : i;             // wrap
        f[lap_index(p, dst, j, k)] = f[lap_index(p, src, j, k)];
    } else if (q < sx + sy) {
        if (!(mask & 2) || !p.periodic[1]) return;
        q -= sx;
        const unsigned i = q % nx + L, r = q / nx;
        const unsigned jj = r % L2, k = r / L2 + L;
        const unsigned dst = jj < L ? jj : ny + jj;
        const unsigned src = jj < L ? ny + jj : jj;
        f[lap_index(p, i, dst, k)] = f[lap_index(p, i, src, k)];
    } else {
        if (!(mask & 4) || !p.periodic[2]) return;
        q -= sx + sy;
        const unsigned i = q % nx + L, r = q / nx;
        const unsigned j = r % ny + L, kk = r / ny;
        const unsigned dst = kk < L ? kk : nz + kk;
        const unsigned src = kk < L ? nz + kk : kk;
        f[lap_index(p, i, j, dst)] = f[lap_index(p, i, j, src)];
    }
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

// ---------------------------------------------------------------------------
// viscous terms, src/OCFD_NS_Jacobian3d.cu:58-440
// ---------------------------------------------------------------------------

// first derivative of a LAP field along stride s at o (OCFD_d?0 with CD6 or
// CD8, src/OCFD_Schemes.cu:96-156; put_d0_kernel divides by h)
// (the division by h is the corrected product with RN(1/h), div_const)
template <typename R>
__device__ __forceinline__ R d0(const R *f, long long o, long long s, R h, R ih, bool c8) {
    R t;
    if (c8) t = cd8(f[o - 4 * s], f[o - 3 * s], f[o - 2 * s], f[o - s], f[o + s], f[o + 2 * s], f[o + 3 * s], f[o + 4 * s]);
    else    t = cd6(f[o - 3 * s], f[o - 2 * s], f[o - s], f[o + s], f[o + 2 * s], f[o + 3 * s]);
    return div_const(t, h, ih);
}

// The same derivative at point X of a line of n cells whose faces may be
// closed (DIF_BOUND = 1): the one-sided and lower-order formulas of
// OCFD_D0bound_scheme_kernel (src/OCFD_bound_Scheme.cu:79-186) on the four
// points next to a closed face, the lower face first as in its case 7/8/9.
template <typename R>
__device__ __forceinline__ R d0b(const R *f, long long o, long long s, R h, R ih, bool c8,
                                 int X, int n, bool lo, bool hi) {
    if (lo && X <= 3) {
        R t;
        if (X == 0)      t = (f[o + s] - f[o]);
        else if (X == 1) t = (f[o + s] - f[o - s]) * (R)0.5;
        else if (X == 2) t = (f[o - 2 * s] - (R)8.0 * f[o - s] + (R)8.0 * f[o + s] - f[o + 2 * s]) / (R)12.0;
        else             t = (f[o + 3 * s] - f[o - 3 * s] - (R)9.0 * (f[o + 2 * s] - f[o - 2 * s])
                             + (R)45.0 * (f[o + s] - f[o - s])) / (R)60.0;
        return div_const(t, h, ih);
    }
    if (hi && X >= n - 4) {
        R t;
        const int q = X - n;
        if (q == -1)      t = (f[o] - f[o - s]);
        else if (q == -2) t = (f[o + s] - f[o - s]) * (R)0.5;
        else if (q == -3) t = (f[o - 2 * s] - (R)8.0 * f[o - s] + (R)8.0 * f[o + s] - f[o + 2 * s]) / (R)12.0;
        else              t = (f[o + 3 * s] - f[o - 3 * s] - (R)9.0 * (f[o + 2 * s] - f[o - 2 * s])
                              + (R)45.0 * (f[o + s] - f[o - s])) / (R)60.0;
        return div_const(t, h, ih);
    }
    return d0(f, o, s, h, ih, c8);
}

// cons_to_pri of one cell (src/commen_kernel.cu:77-109): one reciprocal of
// rho and one of rho*Cv, each quotient formed as the corrected product
__device__ __forceinline__ void cons_to_prim(const Params &p, const double f[5], double &d1, double &u1,
                                             double &v1, double &w1, double &T2) {
    d1 = f[0];
    const double id = 1.0 / d1;
    u1 = div_const(f[1], d1, id);
    v1 = div_const(f[2], d1, id);
    w1 = div_const(f[3], d1, id);
    const double dcv = d1 * p.Cv;
    T2 = div_const(f[4] - 0.5 * d1 * (u1 * u1 + v1 * v1 + w1 * w1), dcv, 1.0 / dcv);
}

// Cell of a thread of the viscous kernels: a block of 256 threads covers a
// 32 x 8 tile of one z plane (grid: x tiles * y tiles, nz), so most y
// neighbours of its cells are loaded by the same block and meet in L1.
constexpr int VT_X = 32, VT_Y = 8;
__device__ __forceinline__ bool tile_cell(const Params &p, int &i, int &j, int &k, long long &tid, int k0 = 0) {
    const int ntx = (p.nx + VT_X - 1) / VT_X;
    i = (int)(blockIdx.x % ntx) * VT_X + (int)(threadIdx.x % VT_X);
    j = (int)(blockIdx.x / ntx) * VT_Y + (int)(threadIdx.x / VT_X);
    k = (int)blockIdx.y + k0;
    if (i >= p.nx || j >= p.ny) return false;
    tid = in_index(p, i, j, k);
    return true;
}

// Ev1..4 of all three directions (vis_flux_ker :178-236).  The 12 velocity
// and temperature derivatives (du_viscous_Jacobian3d_init :58-77) are formed
// here from the LAP-box primitives instead of being stored; the stress and
// heat flux do not depend on the direction, so they are formed once per cell.
template <bool UNI, typename R>
__global__ void __launch_bounds__(256, sizeof(R) == 8 ? 5 : 6) k_vis_ev(Params p) {
    int i, j, k;
    long long tid;
    if (!tile_cell(p, i, j, k, tid)) return;
    long long o = lap_index(p, i + OCFD_LAP, j + OCFD_LAP, k + OCFD_LAP);
    const bool c8 = p.scheme_vis == 204;
    R Akx = (R)metric<UNI>(p, M_AKX, o), Aix = (R)metric<UNI>(p, M_AIX, o), Asx = (R)metric<UNI>(p, M_ASX, o);
    R Aky = (R)metric<UNI>(p, M_AKY, o), Aiy = (R)metric<UNI>(p, M_AIY, o), Asy = (R)metric<UNI>(p, M_ASY, o);
    R Akz = (R)metric<UNI>(p, M_AKZ, o), Aiz = (R)metric<UNI>(p, M_AIZ, o), Asz = (R)metric<UNI>(p, M_ASZ, o);
    const R *U = prim_r<R>(p, 1), *V = prim_r<R>(p, 2), *W = prim_r<R>(p, 3), *TT = prim_r<R>(p, 4);
    R Tc = TT[o];
    R Amu = (R)p.amu_C0 * sqrt_r(Tc * Tc * Tc) / ((R)p.Tsb + Tc);      // get_Amu_kernal
    const R ihx = (R)p.inv_h[0], ihy = (R)p.inv_h[1], ihz = (R)p.inv_h[2];
    const R hx = (R)p.hx, hy = (R)p.hy, hz = (R)p.hz;
    R uk, ui, us, vk, vi, vs, wk, wi, ws, Tk, Ti, Ts;
    if (!p.has_bnd) {
        uk = d0(U, o, 1, hx, ihx, c8); ui = d0(U, o, p.ys, hy, ihy, c8); us = d0(U, o, p.zs, hz, ihz, c8);
        vk = d0(V, o, 1, hx, ihx, c8); vi = d0(V, o, p.ys, hy, ihy, c8); vs = d0(V, o, p.zs, hz, ihz, c8);
        wk = d0(W, o, 1, hx, ihx, c8); wi = d0(W, o, p.ys, hy, ihy, c8); ws = d0(W, o, p.zs, hz, ihz, c8);
        Tk = d0(TT, o, 1, hx, ihx, c8); Ti = d0(TT, o, p.ys, hy, ihy, c8); Ts = d0(TT, o, p.zs, hz, ihz, c8);
    } else {
        const bool bxl = p.bnd_lo[0], bxh = p.bnd_hi[0], byl = p.bnd_lo[1], byh = p.bnd_hi[1];
        const bool bzl = p.bnd_lo[2], bzh = p.bnd_hi[2];
        uk = d0b(U, o, 1, hx, ihx, c8, i, p.nx, bxl, bxh); ui = d0b(U, o, p.ys, hy, ihy, c8, j, p.ny, byl, byh);
        us = d0b(U, o, p.zs, hz, ihz, c8, k, p.nz, bzl, bzh);
        vk = d0b(V, o, 1, hx, ihx, c8, i, p.nx, bxl, bxh); vi = d0b(V, o, p.ys, hy, ihy, c8, j, p.ny, byl, byh);
        vs = d0b(V, o, p.zs, hz, ihz, c8, k, p.nz, bzl, bzh);
        wk = d0b(W, o, 1, hx, ihx, c8, i, p.nx, bxl, bxh); wi = d0b(W, o, p.ys, hy, ihy, c8, j, p.ny, byl, byh);
        ws = d0b(W, o, p.zs, hz, ihz, c8, k, p.nz, bzl, bzh);
        Tk = d0b(TT, o, 1, hx, ihx, c8, i, p.nx, bxl, bxh); Ti = d0b(TT, o, p.ys, hy, ihy, c8, j, p.ny, byl, byh);
        Ts = d0b(TT, o, p.zs, hz, ihz, c8, k, p.nz, bzl, bzh);
    }
    R ux = uk*Akx + ui*Aix + us*Asx;
    R vx = vk*Akx + vi*Aix + vs*Asx;
    R wx = wk*Akx + wi*Aix + ws*Asx;
    R uy = uk*Aky + ui*Aiy + us*Asy;
    R vy = vk*Aky + vi*Aiy + vs*Asy;
    R wy = wk*Aky + wi*Aiy + ws*Asy;
    R uz = uk*Akz + ui*Aiz + us*Asz;
    R vz = vk*Akz + vi*Aiz + vs*Asz;
    R wz = wk*Akz + wi*Aiz + ws*Asz;
    R div = ux + vy + wz;
    R s11 = ((R)2.0*ux - (R)(2.0/3.0)*div) * Amu;
    R s22 = ((R)2.0*vy - (R)(2.0/3.0)*div) * Amu;
    R s33 = ((R)2.0*wz - (R)(2.0/3.0)*div) * Amu;
    R s12 = (uy + vx) * Amu;
    R s13 = (uz + wx) * Amu;
    R s23 = (vz + wy) * Amu;
    R uu = U[o], vv = V[o], ww = W[o];
    R Amuk = Amu * (R)p.vis_c;
    R Tx = Tk*Akx + Ti*Aix + Ts*Asx;
    R Ty = Tk*Aky + Ti*Aiy + Ts*Asy;
    R Tz = Tk*Akz + Ti*Aiz + Ts*Asz;
    R E1 = uu*s11 + vv*s12 + ww*s13 + Amuk*Tx;
    R E2 = uu*s12 + vv*s22 + ww*s23 + Amuk*Ty;
    R E3 = uu*s13 + vv*s23 + ww*s33 + Amuk*Tz;
    R Aj1 = (R)metric<UNI>(p, M_AJAC, o);
    R *const evb = ev_r<R>(p);
#pragma unroll
    for (int dd = 0; dd < 3; dd++) {
        R akx = (R)metric<UNI>(p, M_AKX + 3 * dd, o) * Aj1;
        R aky = (R)metric<UNI>(p, M_AKX + 3 * dd + 1, o) * Aj1;
        R akz = (R)metric<UNI>(p, M_AKX + 3 * dd + 2, o) * Aj1;
        R *ev = evb + (long long)(4 * dd) * p.lapN;
        ev[o]              = (akx*s11 + aky*s12 + akz*s13);
        ev[p.lapN + o]     = (akx*s12 + aky*s22 + akz*s23);
        ev[2 * p.lapN + o] = (akx*s13 + aky*s23 + akz*s33);
        ev[3 * p.lapN + o] = (akx*E1  + aky*E2  + akz*E3);
    }
}

// RK stage (src/OCFD_time.cu:44-94) + cons_to_pri (src/commen_kernel.cu:77-109)
// + pri_to_cons re-projection on the six faces (src/OCFD_boundary.cu:40-91)
// for one cell, given its final du
// (fn0, fk0: U^n and U^k of the cell, read by the caller)
__device__ __forceinline__ void rk_cell_pre(const Params &p, int krk, long long tid, int i, int j, int k,
                                            const double du[5], const double fn0[5], const double fk0[5]) {
    const long long N = p.N;
    double f[5];
#pragma unroll
    for (int m = 0; m < 5; m++) {
        double fn = fn0[m];
        if (krk == 1) {
            f[m] = fn + p.dt * du[m];
        } else if (krk == 2) {
            double t1 = 3.0 / 4.0, t2 = 1.0 / 4.0;
            f[m] = t1 * fn + t2 * (fk0[m] + p.dt * du[m]);
        } else {
            double t1 = 1.0 / 3.0, t2 = 2.0 / 3.0;
            f[m] = t1 * fn + t2 * (fk0[m] + p.dt * du[m]);
        }
    }
    long long o = lap_index(p, i + OCFD_LAP, j + OCFD_LAP, k + OCFD_LAP);
    if (krk == 3 && p.flap) {       // pf_lap, OCFD_time_advance_ker3 (src/OCFD_time.cu:78-92)
#pragma unroll
        for (int m = 0; m < 5; m++) p.flap[m * p.lapN + o] = f[m];
    }
    double d1, u1, v1, w1, T2;
    cons_to_prim(p, f, d1, u1, v1, w1, T2);
    const bool face = (i == 0) || (i == p.nx - 1) || (j == 0) || (j == p.ny - 1) || (k == 0 && p.zface_lo) ||
                      (k == p.nz - 1 && p.zface_hi);
    if (p.mixed) {      // the stencils of the precision form read FP32 primitives
        p.prim32[0][o] = (float)d1; p.prim32[1][o] = (float)u1; p.prim32[2][o] = (float)v1;
        p.prim32[3][o] = (float)w1; p.prim32[4][o] = (float)T2;
        // the boundary-condition family works on FP64 primitives: its wall
        // law reads the four rows next to the wall and the face re-projection
        // reads the face cells.  With a filter the step's FP64 primitives are
        // the last stage's, before the filter changes U (cons_to_pri is not
        // run after filtering), so the last stage writes them all.
        if ((p.ibc && (face || j <= OCFD_LAP)) || (krk == 3 && p.flap)) {
            p.prim[0][o] = d1; p.prim[1][o] = u1; p.prim[2][o] = v1; p.prim[3][o] = w1; p.prim[4][o] = T2;
        }
    } else {
        p.prim[0][o] = d1; p.prim[1][o] = u1; p.prim[2][o] = v1; p.prim[3][o] = w1; p.prim[4][o] = T2;
    }
    // cons_to_pri_kernel also leaves the pressure (src/commen_kernel.cu:107),
    // which the filter after the step reads (FP32 in the precision form)
    if (krk == 3 && p.pfil) {
        const double pr = T2 * d1 / (p.Gamma * p.Ama * p.Ama);
        if (p.mixed) p.pfil32[o] = (float)pr;
        else         p.pfil[o] = pr;
    }
    // with a boundary-condition family the faces are re-projected after it
    // sets the boundary values (k_bc_faces)
    if (face && !p.ibc) {
        f[0] = d1;
        f[1] = u1 * d1;
        f[2] = v1 * d1;
        f[3] = w1 * d1;
        f[4] = d1 * ((u1 * u1 + v1 * v1 + w1 * w1) * 0.5 + p.Cv * T2);
    }
#pragma unroll
    for (int m = 0; m < 5; m++) p.f[m * N + tid] = f[m];
}
__device__ __forceinline__ void rk_cell(const Params &p, int krk, long long tid, int i, int j, int k,
                                        const double du[5]) {
    double fn0[5], fk0[5];
#pragma unroll
    for (int m = 0; m < 5; m++) {
        fn0[m] = p.fn[m * p.N + tid];
        fk0[m] = krk == 1 ? 0.0 : p.f[m * p.N + tid];
    }
    rk_cell_pre(p, krk, tid, i, j, k, du, fn0, fk0);
}

// du[1..4] += Ajac * d(Ev)/d(xi) for x, then y, then z
// (du_viscous_Jacobian3d_{x,y,z}_final + YF_Pe_XF, src/commen_kernel.cu:158-169).
// RK = true: the stage's du is complete here, so the RK update, cons->prim
// and the face re-projection follow in the same thread and du is not stored.
template <bool UNI, bool RK, typename R>
__global__ void __launch_bounds__(256, 6) k_vis_div(Params p, int krk, int k0) {
    int i, j, k;
    long long tid;
    if (!tile_cell(p, i, j, k, tid, k0)) return;
    long long o = lap_index(p, i + OCFD_LAP, j + OCFD_LAP, k + OCFD_LAP);
    const long long st[3] = { 1LL, p.ys, p.zs };
    const R hh[3] = { (R)p.hx, (R)p.hy, (R)p.hz };
    const R ihh[3] = { (R)p.inv_h[0], (R)p.inv_h[1], (R)p.inv_h[2] };
    const bool c8 = p.scheme_vis == 204;
    const R ajac = (R)metric<UNI>(p, M_AJAC, o);
    R *const du = du_r<R>(p);
    const R *const evb = ev_r<R>(p);
    R acc[5];
#pragma unroll
    for (int m = 0; m < 5; m++) acc[m] = (RK || m > 0) ? du[m * p.N + tid] : (R)0.0;
#pragma unroll
    for (int dd = 0; dd < 3; dd++) {
#pragma unroll
        for (int m = 0; m < 4; m++) {
            const R *f = evb + (long long)(4 * dd + m) * p.lapN;
            if (!p.has_bnd) {
                acc[m + 1] += ajac * d0(f, o, st[dd], hh[dd], ihh[dd], c8);
            } else {
                const int X = dd == 0 ? i : (dd == 1 ? j : k), n = dd == 0 ? p.nx : (dd == 1 ? p.ny : p.nz);
                acc[m + 1] += ajac * d0b(f, o, st[dd], hh[dd], ihh[dd], c8, X, n, p.bnd_lo[dd], p.bnd_hi[dd]);
            }
        }
    }
    if (RK) {
        double a64[5];
#pragma unroll
        for (int m = 0; m < 5; m++) a64[m] = (double)acc[m];
        rk_cell(p, krk, tid, i, j, k, a64);
    } else {
#pragma unroll
        for (int m = 0; m < 4; m++) du[(m + 1) * p.N + tid] = acc[m + 1];
    }
}

// ---------------------------------------------------------------------------
// The same divergence + RK stage with the Ev tiles staged in shared memory by
// bulk tensor copies (k_vis_div reads every Ev value through L1/L2).  A block
// owns a VX x VY tile of the x-y plane and marches along z over a segment of
// planes: per plane it takes Ev_x with an x halo, Ev_y with a y halo (one
// barrier for both, double-buffered) and Ev_z of plane k+H into a ring of
// 2H+2 planes, so that every Ev value crosses L2 once per block and every
// stencil read is a shared-memory read.  The Ev fields and their ghosts are
// those k_vis_ev and the ghost fill leave; the arithmetic per cell is
// k_vis_div's, in its order.  Blocks are persistent over (tile, segment)
// items.  H: half-width of the derivative stencil (3: CD6, 4: CD8).
// ---------------------------------------------------------------------------
constexpr int VX = 32, VY = 8, VXH = 4;      // tile; x halo of the Ev_x box (keeps its x start even)

template <typename R, int H>
struct VdivTiles {
    static constexpr int NZS = 2 * H + 2;                  // Ev_z ring slots
    static constexpr int ZE = 4 * VY * VX;                 // [field][y][x]
    static constexpr int XE = 4 * VY * (VX + 2 * VXH);
    static constexpr int YE = 4 * (VY + 2 * H) * VX;
    static constexpr size_t bytes = (size_t)(NZS * ZE + 2 * XE + 2 * YE) * sizeof(R);
};

// d0 / d0b of k_vis_div from a window v[0..2H] (v[H] the cell), same expressions
template <typename R, int H>
__device__ __forceinline__ R d0w(const R *v, R h, R ih, bool c8) {
    R t;
    if (c8) t = cd8(v[H - 4], v[H - 3], v[H - 2], v[H - 1], v[H + 1], v[H + 2], v[H + 3], v[H + 4]);
    else    t = cd6(v[H - 3], v[H - 2], v[H - 1], v[H + 1], v[H + 2], v[H + 3]);
    return div_const(t, h, ih);
}
template <typename R, int H>
__device__ __forceinline__ R d0bw(const R *v, R h, R ih, bool c8, int X, int n, bool lo, bool hi) {
    if (lo && X <= 3) {
        R t;
        if (X == 0)      t = (v[H + 1] - v[H]);
        else if (X == 1) t = (v[H + 1] - v[H - 1]) * (R)0.5;
        else if (X == 2) t = (v[H - 2] - (R)8.0 * v[H - 1] + (R)8.0 * v[H + 1] - v[H + 2]) / (R)12.0;
        else             t = (v[H + 3] - v[H - 3] - (R)9.0 * (v[H + 2] - v[H - 2])
                             + (R)45.0 * (v[H + 1] - v[H - 1])) / (R)60.0;
        return div_const(t, h, ih);
    }
    if (hi && X >= n - 4) {
        R t;
        const int q = X - n;
        if (q == -1)      t = (v[H] - v[H - 1]);
        else if (q == -2) t = (v[H + 1] - v[H - 1]) * (R)0.5;
        else if (q == -3) t = (v[H - 2] - (R)8.0 * v[H - 1] + (R)8.0 * v[H + 1] - v[H + 2]) / (R)12.0;
        else              t = (v[H + 3] - v[H - 3] - (R)9.0 * (v[H + 2] - v[H - 2])
                              + (R)45.0 * (v[H + 1] - v[H - 1])) / (R)60.0;
        return div_const(t, h, ih);
    }
    return d0w<R, H>(v, h, ih, c8);
}

template <bool UNI, typename R, int H>
// (two blocks per SM: a budget for three spills and measured 14 % slower in FP32)
__global__ void __launch_bounds__(VX * VY, 2)
k_vdiv(const __grid_constant__ Params p, const __grid_constant__ CUtensorMap tmx,
       const __grid_constant__ CUtensorMap tmy, const __grid_constant__ CUtensorMap tmz, int krk, int seg_len) {
    using T = VdivTiles<R, H>;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ unsigned long long zbar[T::NZS], xybar[2];
    R *zring = reinterpret_cast<R *>(smem_raw);
    R *xbuf = zring + T::NZS * T::ZE;                  // [2][XE]
    R *ybuf = xbuf + 2 * T::XE;                        // [2][YE]
    const int tid = threadIdx.x;
    const int ti = tid % VX, tj = tid / VX;
    const int ntx = (p.nx + VX - 1) / VX, nty = (p.ny + VY - 1) / VY;
    const int nseg = (p.nz + seg_len - 1) / seg_len;
    const long long nitems = (long long)ntx * nty * nseg;
    const bool c8 = p.scheme_vis == 204;
    const long long N = p.N;
    const R hh[3] = { (R)p.hx, (R)p.hy, (R)p.hz };
    const R ihh[3] = { (R)p.inv_h[0], (R)p.inv_h[1], (R)p.inv_h[2] };
    if (tid == 0) {
        for (int s = 0; s < T::NZS; s++) tma::mbar_init(&zbar[s], 1);
        tma::mbar_init(&xybar[0], 1);
        tma::mbar_init(&xybar[1], 1);
        tma::fence_mbar_init();
    }
    __syncthreads();
    unsigned zph = 0, xyph = 0;             // parity of each barrier's next phase
    unsigned zpend = 0, xypend = 0;         // barriers with a copy issued and not yet waited for
    bool failed = false;
    auto slot = [](int q) { return (q + T::NZS) % T::NZS; };      // q >= -H
    for (long long item = blockIdx.x; item < nitems && !failed; item += gridDim.x) {
        const int tile = (int)(item % ((long long)ntx * nty)), sg = (int)(item / ((long long)ntx * nty));
        const int x0 = (tile % ntx) * VX, y0 = (tile / ntx) * VY;
        const int k0 = sg * seg_len, k1 = min(p.nz, k0 + seg_len);
        const int i = x0 + ti, j = y0 + tj;
        const bool valid = i < p.nx && j < p.ny;
        // thread 0 issues: Ev_z of plane q into its ring slot; Ev_x and Ev_y of plane k into buffer b
        auto issue_z = [&](int q) {
            const int s = slot(q);
            tma::mbar_expect_tx(&zbar[s], (unsigned)(T::ZE * sizeof(R)));
            tma::load_4d(zring + s * T::ZE, &tmz, OCFD_LAP + x0, OCFD_LAP + y0, OCFD_LAP + q, 0, &zbar[s]);
        };
        auto issue_xy = [&](int k, int b) {
            tma::mbar_expect_tx(&xybar[b], (unsigned)((T::XE + T::YE) * sizeof(R)));
            tma::load_4d(xbuf + b * T::XE, &tmx, OCFD_LAP + x0 - VXH, OCFD_LAP + y0, OCFD_LAP + k, 0, &xybar[b]);
            tma::load_4d(ybuf + b * T::YE, &tmy, OCFD_LAP + x0, OCFD_LAP + y0 - H, OCFD_LAP + k, 0, &xybar[b]);
        };
        if (tid == 0) {
            for (int q = k0 - H; q <= k0 + H + 1 && q <= k1 - 1 + H; q++) { issue_z(q); zpend |= 1u << slot(q); }
            issue_xy(k0, 0); xypend |= 1u;
            if (k0 + 1 < k1) { issue_xy(k0 + 1, 1); xypend |= 2u; }
        }
        // the bookkeeping of thread 0 is replayed by every thread
        if (tid != 0) {
            for (int q = k0 - H; q <= k0 + H + 1 && q <= k1 - 1 + H; q++) zpend |= 1u << slot(q);
            xypend |= 1u;
            if (k0 + 1 < k1) xypend |= 2u;
        }
        for (int k = k0; k < k1; k++) {
            const int b = (k - k0) & 1;
            const long long ci = valid ? in_index(p, i, j, k) : 0;
            // this cell's state, read before the waits; the next plane's
            // cell into L1 meanwhile
            R acc[5];
            double fn0[5], fk0[5];
            if (valid) {
                const R *du = du_r<R>(p);
#pragma unroll
                for (int m = 0; m < 5; m++) {
                    acc[m] = du[m * N + ci];
                    fn0[m] = p.fn[m * N + ci];
                    fk0[m] = krk == 1 ? 0.0 : p.f[m * N + ci];
                }
                if (k + 1 < k1) {
                    const long long cn = ci + (long long)p.nx * p.ny;
#pragma unroll
                    for (int m = 0; m < 5; m++) {
                        tma::prefetch_l1(du + m * N + cn);
                        tma::prefetch_l1(p.fn + m * N + cn);
                        if (krk != 1) tma::prefetch_l1(p.f + m * N + cn);
                    }
                }
            }
            // planes k-H .. k+H of Ev_z, and Ev_x / Ev_y of plane k
            for (int q = k - H; q <= k + H; q++) {
                const int s = slot(q);
                if (zpend & (1u << s)) {
                    if (tma::mbar_wait(&zbar[s], (zph >> s) & 1u)) {
                        zph ^= 1u << s;
                        zpend &= ~(1u << s);
                    } else {
                        failed = true;          // still pending: waited for again on the way out
                    }
                }
            }
            if (xypend & (1u << b)) {
                if (tma::mbar_wait(&xybar[b], (xyph >> b) & 1u)) {
                    xyph ^= 1u << b;
                    xypend &= ~(1u << b);
                } else {
                    failed = true;
                }
            }
            if (valid && !failed) {
                const long long o = lap_index(p, i + OCFD_LAP, j + OCFD_LAP, k + OCFD_LAP);
                const R ajac = (R)metric<UNI>(p, M_AJAC, o);
                const R *xb = xbuf + b * T::XE, *yb = ybuf + b * T::YE;
                // the 12 derivatives first (shared memory only), then their
                // sums into du in k_vis_div's order, so that the first sum
                // does not wait on du's load
                R dv[3][4];
#pragma unroll
                for (int dd = 0; dd < 3; dd++) {
#pragma unroll
                    for (int m = 0; m < 4; m++) {
                        R v[2 * H + 1];
#pragma unroll
                        for (int t = 0; t <= 2 * H; t++) {
                            if (dd == 0)      v[t] = xb[(m * VY + tj) * (VX + 2 * VXH) + ti + VXH - H + t];
                            else if (dd == 1) v[t] = yb[(m * (VY + 2 * H) + tj + t) * VX + ti];
                            else              v[t] = zring[slot(k - H + t) * T::ZE + (m * VY + tj) * VX + ti];
                        }
                        if (!p.has_bnd) {
                            dv[dd][m] = d0w<R, H>(v, hh[dd], ihh[dd], c8);
                        } else {
                            const int X = dd == 0 ? i : (dd == 1 ? j : k), n = dd == 0 ? p.nx : (dd == 1 ? p.ny : p.nz);
                            dv[dd][m] = d0bw<R, H>(v, hh[dd], ihh[dd], c8, X, n, p.bnd_lo[dd], p.bnd_hi[dd]);
                        }
                    }
                }
#pragma unroll
                for (int dd = 0; dd < 3; dd++)
#pragma unroll
                    for (int m = 0; m < 4; m++) acc[m + 1] += ajac * dv[dd][m];
                double a64[5];
#pragma unroll
                for (int m = 0; m < 5; m++) a64[m] = (double)acc[m];
                rk_cell_pre(p, krk, ci, i, j, k, a64, fn0, fk0);
            }
            // plane k-H's slot and buffer b are free; a wait that ran out
            // anywhere in the block ends the block's work
            if (__syncthreads_or(failed)) { failed = true; break; }
            if (k + H + 2 <= k1 - 1 + H) {
                if (tid == 0) issue_z(k + H + 2);
                zpend |= 1u << slot(k + H + 2);
            }
            if (k + 2 < k1) {
                if (tid == 0) issue_xy(k + 2, b);
                xypend |= 1u << b;
            }
        }
    }
    if (failed) {
        if (tid == 0) atomicExch(p.kerr, 1);
        // copies still in flight land before the block's shared memory goes away
        for (int s = 0; s < T::NZS; s++)
            if (zpend & (1u << s)) tma::mbar_wait(&zbar[s], (zph >> s) & 1u);
        for (int b = 0; b < 2; b++)
            if (xypend & (1u << b)) tma::mbar_wait(&xybar[b], (xyph >> b) & 1u);
    }
}

// ---------------------------------------------------------------------------
// k_vis_ev with the primitives staged in shared memory: a block owns a
// VX x VY tile and marches along z; each plane of u, v, w, T arrives with
// its x and y halos (one bulk tensor copy per plane) into a ring of 2H+2
// planes, so the 12 derivative stencils read shared memory only and every
// primitive crosses L2 once per block.  Same arithmetic as k_vis_ev.
// ---------------------------------------------------------------------------
template <typename R, int H>
struct VevTiles {
    static constexpr int NZS = 2 * H + 2;
    static constexpr int PX = VX + 2 * VXH, PY = VY + 2 * H;     // plane box (x halo even)
    static constexpr int PE = 4 * PY * PX;                         // [field][y][x]
    static constexpr size_t bytes = (size_t)NZS * PE * sizeof(R);
};

template <bool UNI, typename R, int H>
__global__ void __launch_bounds__(VX * VY, sizeof(R) == 8 ? 1 : 3)
k_vev(const __grid_constant__ Params p, const __grid_constant__ CUtensorMap tmq, int seg_len) {
    using T = VevTiles<R, H>;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ unsigned long long zbar[T::NZS];
    R *ring = reinterpret_cast<R *>(smem_raw);
    const int tid = threadIdx.x;
    const int ti = tid % VX, tj = tid / VX;
    const int ntx = (p.nx + VX - 1) / VX, nty = (p.ny + VY - 1) / VY;
    const int nseg = (p.nz + seg_len - 1) / seg_len;
    const long long nitems = (long long)ntx * nty * nseg;
    const bool c8 = p.scheme_vis == 204;
    if (tid == 0) {
        for (int s = 0; s < T::NZS; s++) tma::mbar_init(&zbar[s], 1);
        tma::fence_mbar_init();
    }
    __syncthreads();
    unsigned zph = 0, zpend = 0;
    bool failed = false;
    auto slot = [](int q) { return (q + T::NZS) % T::NZS; };      // q >= -H
    // value of field f (0 u, 1 v, 2 w, 3 T) at tile offset (dx, dy) of plane q
    auto at = [&](int q, int f, int dy, int dx) -> R {
        return ring[slot(q) * T::PE + (f * T::PY + tj + H + dy) * T::PX + ti + VXH + dx];
    };
    for (long long item = blockIdx.x; item < nitems && !failed; item += gridDim.x) {
        const int tile = (int)(item % ((long long)ntx * nty)), sg = (int)(item / ((long long)ntx * nty));
        const int x0 = (tile % ntx) * VX, y0 = (tile / ntx) * VY;
        const int k0 = sg * seg_len, k1 = min(p.nz, k0 + seg_len);
        const int i = x0 + ti, j = y0 + tj;
        const bool valid = i < p.nx && j < p.ny;
        auto issue = [&](int q) {
            const int s = slot(q);
            tma::mbar_expect_tx(&zbar[s], (unsigned)(T::PE * sizeof(R)));
            tma::load_4d(ring + s * T::PE, &tmq, OCFD_LAP + x0 - VXH, OCFD_LAP + y0 - H, OCFD_LAP + q, 0, &zbar[s]);
        };
        for (int q = k0 - H; q <= k0 + H + 1 && q <= k1 - 1 + H; q++) {
            if (tid == 0) issue(q);
            zpend |= 1u << slot(q);
        }
        for (int k = k0; k < k1; k++) {
            for (int q = k - H; q <= k + H; q++) {
                const int s = slot(q);
                if (zpend & (1u << s)) {
                    if (tma::mbar_wait(&zbar[s], (zph >> s) & 1u)) {
                        zph ^= 1u << s;
                        zpend &= ~(1u << s);
                    } else {
                        failed = true;          // still pending: waited for again on the way out
                    }
                }
            }
            if (valid && !failed) {
                const long long o = lap_index(p, i + OCFD_LAP, j + OCFD_LAP, k + OCFD_LAP);
                R Akx = (R)metric<UNI>(p, M_AKX, o), Aix = (R)metric<UNI>(p, M_AIX, o), Asx = (R)metric<UNI>(p, M_ASX, o);
                R Aky = (R)metric<UNI>(p, M_AKY, o), Aiy = (R)metric<UNI>(p, M_AIY, o), Asy = (R)metric<UNI>(p, M_ASY, o);
                R Akz = (R)metric<UNI>(p, M_AKZ, o), Aiz = (R)metric<UNI>(p, M_AIZ, o), Asz = (R)metric<UNI>(p, M_ASZ, o);
                R Tc = at(k, 3, 0, 0);
                R Amu = (R)p.amu_C0 * sqrt_r(Tc * Tc * Tc) / ((R)p.Tsb + Tc);      // get_Amu_kernal
                const R ihx = (R)p.inv_h[0], ihy = (R)p.inv_h[1], ihz = (R)p.inv_h[2];
                const R hx = (R)p.hx, hy = (R)p.hy, hz = (R)p.hz;
                R dk[4], di[4], ds[4];         // d/dxi, d/deta, d/dzeta of u, v, w, T
#pragma unroll
                for (int f = 0; f < 4; f++) {
                    R vx[2 * H + 1], vy[2 * H + 1], vz[2 * H + 1];
#pragma unroll
                    for (int t = 0; t <= 2 * H; t++) {
                        vx[t] = at(k, f, 0, t - H);
                        vy[t] = at(k, f, t - H, 0);
                        vz[t] = at(k - H + t, f, 0, 0);
                    }
                    if (!p.has_bnd) {
                        dk[f] = d0w<R, H>(vx, hx, ihx, c8);
                        di[f] = d0w<R, H>(vy, hy, ihy, c8);
                        ds[f] = d0w<R, H>(vz, hz, ihz, c8);
                    } else {
                        dk[f] = d0bw<R, H>(vx, hx, ihx, c8, i, p.nx, p.bnd_lo[0], p.bnd_hi[0]);
                        di[f] = d0bw<R, H>(vy, hy, ihy, c8, j, p.ny, p.bnd_lo[1], p.bnd_hi[1]);
                        ds[f] = d0bw<R, H>(vz, hz, ihz, c8, k, p.nz, p.bnd_lo[2], p.bnd_hi[2]);
                    }
                }
                const R uk = dk[0], ui = di[0], us = ds[0], vk = dk[1], vi = di[1], vs = ds[1];
                const R wk = dk[2], wi = di[2], ws = ds[2], Tk = dk[3], Ti = di[3], Ts = ds[3];
                R ux = uk*Akx + ui*Aix + us*Asx;
                R vx = vk*Akx + vi*Aix + vs*Asx;
                R wx = wk*Akx + wi*Aix + ws*Asx;
                R uy = uk*Aky + ui*Aiy + us*Asy;
                R vy = vk*Aky + vi*Aiy + vs*Asy;
                R wy = wk*Aky + wi*Aiy + ws*Asy;
                R uz = uk*Akz + ui*Aiz + us*Asz;
                R vz = vk*Akz + vi*Aiz + vs*Asz;
                R wz = wk*Akz + wi*Aiz + ws*Asz;
                R div = ux + vy + wz;
                R s11 = ((R)2.0*ux - (R)(2.0/3.0)*div) * Amu;
                R s22 = ((R)2.0*vy - (R)(2.0/3.0)*div) * Amu;
                R s33 = ((R)2.0*wz - (R)(2.0/3.0)*div) * Amu;
                R s12 = (uy + vx) * Amu;
                R s13 = (uz + wx) * Amu;
                R s23 = (vz + wy) * Amu;
                R uu = at(k, 0, 0, 0), vv = at(k, 1, 0, 0), ww = at(k, 2, 0, 0);
                R Amuk = Amu * (R)p.vis_c;
                R Tx = Tk*Akx + Ti*Aix + Ts*Asx;
                R Ty = Tk*Aky + Ti*Aiy + Ts*Asy;
                R Tz = Tk*Akz + Ti*Aiz + Ts*Asz;
                R E1 = uu*s11 + vv*s12 + ww*s13 + Amuk*Tx;
                R E2 = uu*s12 + vv*s22 + ww*s23 + Amuk*Ty;
                R E3 = uu*s13 + vv*s23 + ww*s33 + Amuk*Tz;
                R Aj1 = (R)metric<UNI>(p, M_AJAC, o);
                R *const evb = ev_r<R>(p);
#pragma unroll
                for (int dd = 0; dd < 3; dd++) {
                    R akx = (R)metric<UNI>(p, M_AKX + 3 * dd, o) * Aj1;
                    R aky = (R)metric<UNI>(p, M_AKX + 3 * dd + 1, o) * Aj1;
                    R akz = (R)metric<UNI>(p, M_AKX + 3 * dd + 2, o) * Aj1;
                    R *ev = evb + (long long)(4 * dd) * p.lapN;
                    ev[o]              = (akx*s11 + aky*s12 + akz*s13);
                    ev[p.lapN + o]     = (akx*s12 + aky*s22 + akz*s23);
                    ev[2 * p.lapN + o] = (akx*s13 + aky*s23 + akz*s33);
                    ev[3 * p.lapN + o] = (akx*E1  + aky*E2  + akz*E3);
                }
            }
            if (__syncthreads_or(failed)) { failed = true; break; }
            if (k + H + 2 <= k1 - 1 + H) {          // into the slot of plane k-H, read for the last time
                if (tid == 0) issue(k + H + 2);
                zpend |= 1u << slot(k + H + 2);
            }
        }
    }
    if (failed) {
        if (tid == 0) atomicExch(p.kerr, 1);
        for (int s = 0; s < T::NZS; s++)
            if (zpend & (1u << s)) tma::mbar_wait(&zbar[s], (zph >> s) & 1u);
    }
}

// ---------------------------------------------------------------------------
// analysis after the path (src/OCFD_ana.cu)
// ---------------------------------------------------------------------------

// get_Q (src/OCFD_ana.cu:317-456): the derivatives of u, v, w along the three
// grid directions (OCFD_d{x,y,z}0 with the D0_bound closures, as in the Ev
// kernel), the velocity gradient through the metrics and
// Q = (ux vy + ux wz + vy wz - uy vx - uz wx - vz wy) Ajac^2, interior cells
// into q[nz][ny][nx].  The ghosts of u, v, w are the caller's to fill.
template <bool UNI>
__global__ void __launch_bounds__(256) k_qcrit(Params p, double *q) {
    int i, j, k;
    long long tid;
    if (!tile_cell(p, i, j, k, tid)) return;
    const long long o = lap_index(p, i + OCFD_LAP, j + OCFD_LAP, k + OCFD_LAP);
    const bool c8 = p.scheme_vis == 204;
    const double *U = p.prim[1], *V = p.prim[2], *W = p.prim[3];
    const double ih[3] = { p.inv_h[0], p.inv_h[1], p.inv_h[2] }, hh[3] = { p.hx, p.hy, p.hz };
    const long long st[3] = { 1LL, p.ys, p.zs };
    const int X[3] = { i, j, k }, n[3] = { p.nx, p.ny, p.nz };
    double g[3][3];                      // g[field][direction]: uk ui us, vk vi vs, wk wi ws
    const double *F[3] = { U, V, W };
#pragma unroll
    for (int m = 0; m < 3; m++)
#pragma unroll
        for (int d = 0; d < 3; d++)
            g[m][d] = p.has_bnd ? d0b(F[m], o, st[d], hh[d], ih[d], c8, X[d], n[d], p.bnd_lo[d], p.bnd_hi[d])
                                : d0(F[m], o, st[d], hh[d], ih[d], c8);
    const double Akx = metric<UNI>(p, M_AKX, o), Aix = metric<UNI>(p, M_AIX, o), Asx = metric<UNI>(p, M_ASX, o);
    const double Aky = metric<UNI>(p, M_AKY, o), Aiy = metric<UNI>(p, M_AIY, o), Asy = metric<UNI>(p, M_ASY, o);
    const double Akz = metric<UNI>(p, M_AKZ, o), Aiz = metric<UNI>(p, M_AIZ, o), Asz = metric<UNI>(p, M_ASZ, o);
    const double ux = g[0][0]*Akx + g[0][1]*Aix + g[0][2]*Asx;
    const double vx = g[1][0]*Akx + g[1][1]*Aix + g[1][2]*Asx;
    const double wx = g[2][0]*Akx + g[2][1]*Aix + g[2][2]*Asx;
    const double uy = g[0][0]*Aky + g[0][1]*Aiy + g[0][2]*Asy;
    const double vy = g[1][0]*Aky + g[1][1]*Aiy + g[1][2]*Asy;
    const double wy = g[2][0]*Aky + g[2][1]*Aiy + g[2][2]*Asy;
    const double uz = g[0][0]*Akz + g[0][1]*Aiz + g[0][2]*Asz;
    const double vz = g[1][0]*Akz + g[1][1]*Aiz + g[1][2]*Asz;
    const double wz = g[2][0]*Akz + g[2][1]*Aiz + g[2][2]*Asz;
    const double aj = metric<UNI>(p, M_AJAC, o);
    q[tid] = (ux*vy + ux*wz + vy*wz - uy*vx - uz*wx - vz*wy) * aj * aj;
}

// ana_time_average (src/OCFD_ana.cu:238-306): m = (n m + x) / (n + 1) for
// d, u, v, w, T of every interior cell, n the number of samples so far
__global__ void k_time_average(Params p, double *mean5, int n) {
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= p.N) return;
    const int i = (int)(tid % p.nx);
    const long long r = tid / p.nx;
    const int j = (int)(r % p.ny), k = (int)(r / p.ny);
    const long long o = lap_index(p, i + OCFD_LAP, j + OCFD_LAP, k + OCFD_LAP);
#pragma unroll
    for (int m = 0; m < 5; m++) {
        double *a = mean5 + m * p.N + tid;
        *a = (n * *a + p.prim[m][o]) / (n + 1.);
    }
}

// RK stage + cons->prim + face re-projection over the whole grid (du given)
__global__ void k_rk_update(Params p, int krk) {
    long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= p.N) return;
    int i = (int)(tid % p.nx); long long r = tid / p.nx;
    int j = (int)(r % p.ny); int k = (int)(r / p.ny);
    double du[5];
#pragma unroll
    for (int m = 0; m < 5; m++) du[m] = p.mixed ? (double)p.du32[m * p.N + tid] : p.du[m * p.N + tid];
    rk_cell(p, krk, tid, i, j, k, du);
}

// Unfused pieces of the same update for the reference-named per-stage API:
// RK stage only, cons->prim only, face re-projection only.
__global__ void k_rk_only(Params p, int krk) {
    long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= 5 * p.N) return;
    double fn = p.fn[tid], du = p.du[tid];
    if (krk == 1) p.f[tid] = fn + p.dt * du;
    else if (krk == 2) { double t1 = 3.0 / 4.0, t2 = 1.0 / 4.0; p.f[tid] = t1 * fn + t2 * (p.f[tid] + p.dt * du); }
    else {
        double t1 = 1.0 / 3.0, t2 = 2.0 / 3.0;
        const double v = t1 * fn + t2 * (p.f[tid] + p.dt * du);
        p.f[tid] = v;
        if (p.flap) {               // pf_lap
            const long long m = tid / p.N, c = tid - m * p.N;
            const int i = (int)(c % p.nx);
            const long long r = c / p.nx;
            const int j = (int)(r % p.ny), k = (int)(r / p.ny);
            p.flap[m * p.lapN + lap_index(p, i + OCFD_LAP, j + OCFD_LAP, k + OCFD_LAP)] = v;
        }
    }
}
__global__ void k_c2p(Params p) {
    long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= p.N) return;
    int i = (int)(tid % p.nx); long long r = tid / p.nx;
    int j = (int)(r % p.ny); int k = (int)(r / p.ny);
    const long long N = p.N;
    const double f[5] = {p.f[tid], p.f[N + tid], p.f[2 * N + tid], p.f[3 * N + tid], p.f[4 * N + tid]};
    long long o = lap_index(p, i + OCFD_LAP, j + OCFD_LAP, k + OCFD_LAP);
    double d1, u1, v1, w1, T2;
    cons_to_prim(p, f, d1, u1, v1, w1, T2);
    p.prim[0][o] = d1; p.prim[1][o] = u1; p.prim[2][o] = v1; p.prim[3][o] = w1; p.prim[4][o] = T2;
    if (p.pfil) p.pfil[o] = T2 * d1 / (p.Gamma * p.Ama * p.Ama);
}
__global__ void k_bc_faces(Params p) {
    long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= p.N) return;
    int i = (int)(tid % p.nx); long long r = tid / p.nx;
    int j = (int)(r % p.ny); int k = (int)(r / p.ny);
    bool face = (i == 0) || (i == p.nx - 1) || (j == 0) || (j == p.ny - 1) || (k == 0 && p.zface_lo) ||
                (k == p.nz - 1 && p.zface_hi);
    if (!face) return;
    long long o = lap_index(p, i + OCFD_LAP, j + OCFD_LAP, k + OCFD_LAP);
    double d = p.prim[0][o], u = p.prim[1][o], v = p.prim[2][o], w = p.prim[3][o], T = p.prim[4][o];
    const long long N = p.N;
    p.f[tid] = d;
    p.f[N + tid] = u * d;
    p.f[2 * N + tid] = v * d;
    p.f[3 * N + tid] = w * d;
    p.f[4 * N + tid] = d * ((u * u + v * v + w * w) * 0.5 + p.Cv * T);
}

// pri_to_cons over the interior (init, src/OCFD_init.cu:108-115)
__global__ void k_p2c(Params p, double *out) {
    long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= p.N) return;
    int i = (int)(tid % p.nx); long long r = tid / p.nx;
    int j = (int)(r % p.ny); int k = (int)(r / p.ny);
    long long o = lap_index(p, i + OCFD_LAP, j + OCFD_LAP, k + OCFD_LAP);
    double d = p.prim[0][o], u = p.prim[1][o], v = p.prim[2][o], w = p.prim[3][o], T = p.prim[4][o];
    const long long N = p.N;
    out[tid] = d;
    out[N + tid] = u * d;
    out[2 * N + tid] = v * d;
    out[3 * N + tid] = w * d;
    out[4 * N + tid] = d * ((u * u + v * v + w * w) * 0.5 + p.Cv * T);
}

// interior <-> LAP-box copy of one field (dense [nz][ny][nx] <-> LAP box)
__global__ void k_scatter_interior(Params p, const double *src, double *dst_lap) {
    long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= p.N) return;
    int i = (int)(tid % p.nx); long long r = tid / p.nx;
    int j = (int)(r % p.ny); int k = (int)(r / p.ny);
    dst_lap[lap_index(p, i + OCFD_LAP, j + OCFD_LAP, k + OCFD_LAP)] = src[tid];
}
__global__ void k_gather_interior(Params p, const double *src_lap, double *dst) {
    long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= p.N) return;
    int i = (int)(tid % p.nx); long long r = tid / p.nx;
    int j = (int)(r % p.ny); int k = (int)(r / p.ny);
    dst[tid] = src_lap[lap_index(p, i + OCFD_LAP, j + OCFD_LAP, k + OCFD_LAP)];
}
// the FP32 primitives of the precision form from the FP64 ones (whole LAP box)
__global__ void k_prims_to_fp32(Params p) {
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= 5 * p.lapN) return;
    const int m = (int)(tid / p.lapN);
    const long long q = tid - (long long)m * p.lapN;
    p.prim32[m][q] = (float)p.prim[m][q];
}

// HybridAuto_scheme_Proportion (src/OCFD_Schemes_hybrid_auto.cu:745-829):
// per direction, the entries of the flag array equal to 1, equal to 2, and
// any other value; counts[3 * dir + type]
__global__ void k_flag_hist(Params p, unsigned long long *counts) {
    const long long nfx = (long long)(p.nx + 1) * p.ny * p.nz, nfy = (long long)p.nx * (p.ny + 1) * p.nz,
                    nfz = (long long)p.nx * p.ny * (p.nz + 1);
    unsigned long long c[9] = {};
    const long long tot = nfx + nfy + nfz;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x) {
        const int d = t < nfx ? 0 : (t < nfx + nfy ? 1 : 2);
        const long long q = d == 0 ? t : (d == 1 ? t - nfx : t - nfx - nfy);
        const int f = p.flag[d][q];
        c[3 * d + (f == 1 ? 0 : (f == 2 ? 1 : 2))] += 1;
    }
#pragma unroll
    for (int i = 0; i < 9; i++) {
        unsigned long long v = c[i];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0 && v) atomicAdd(counts + i, v);
    }
}

__global__ void k_fill(double *f, long long n, double v) {
    long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid < n) f[tid] = v;
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static inline unsigned blocks_for(long long n, int t) { return (unsigned)((n + t - 1) / t); }

cudaError_t launch_sensor(const Params &p, cudaStream_t st) {
    const long long n = (long long)(p.nx + 1) * (p.ny + 1) * (p.nz + 1);
    if (p.flag_count) {
        cudaError_t e = cudaMemsetAsync(p.flag_count, 0, 3 * sizeof(unsigned), st);
        if (e != cudaSuccess) return e;
    }
    (void)n;
    // tiles of the extended box's (i, j), z split into segments so that
    // there are about eight blocks per SM
    const int ntiles = ((p.nx + 1 + SEN_X - 1) / SEN_X) * ((p.ny + 1 + SEN_Y - 1) / SEN_Y);
    const int ez = p.nz + 1;
    int nseg = (148 * 8 + ntiles - 1) / ntiles;
    if (nseg > ez) nseg = ez;
    if (nseg < 1) nseg = 1;
    const int seg = (ez + nseg - 1) / nseg;
    nseg = (ez + seg - 1) / seg;
    const dim3 grid((unsigned)ntiles, (unsigned)nseg);
    if (p.mixed) k_sensor_march<float><<<grid, SEN_X * SEN_Y, 0, st>>>(p, seg);
    else         k_sensor_march<double><<<grid, SEN_X * SEN_Y, 0, st>>>(p, seg);
    return cudaGetLastError();
}

template <typename T>
static cudaError_t launch_ghost_t(const Params &p, T *const *fields, const int *dirmask, int nf, cudaStream_t st) {
    const long long per = 2LL * OCFD_LAP * ((long long)p.ny * p.nz + (long long)p.nx * p.nz + (long long)p.nx * p.ny);
    if (nf <= 0) return cudaSuccess;
    if (per >= (1LL << 31) || nf > 12) return cudaErrorInvalidValue;
    GhostList<T> g;
    g.n = nf;
    for (int i = 0; i < nf; i++) { g.f[i] = fields[i]; g.dirmask[i] = dirmask[i]; }
    const dim3 grid((unsigned)((per + 255) / 256), (unsigned)nf);
    k_ghost<T><<<grid, 256, 0, st>>>(p, g);
    return cudaGetLastError();
}
cudaError_t launch_ghost(const Params &p, double *const *fields, const int *dirmask, int nf, cudaStream_t st) {
    return launch_ghost_t<double>(p, fields, dirmask, nf, st);
}
cudaError_t launch_ghost32(const Params &p, float *const *fields, const int *dirmask, int nf, cudaStream_t st) {
    return launch_ghost_t<float>(p, fields, dirmask, nf, st);
}



template <typename R>
static cudaError_t launch_vis_ev_t(const Params &p, cudaStream_t st) {
    const dim3 nb((unsigned)(((p.nx + VT_X - 1) / VT_X) * ((p.ny + VT_Y - 1) / VT_Y)), (unsigned)p.nz);
    if (p.uniform_metrics) k_vis_ev<true, R><<<nb, 256, 0, st>>>(p);
    else                   k_vis_ev<false, R><<<nb, 256, 0, st>>>(p);
    return cudaGetLastError();
}

template <typename R>
static cudaError_t launch_vis_div_t(const Params &p, int krk, int k0, int k1, cudaStream_t st) {
    if (k1 <= k0) return cudaSuccess;
    const dim3 nb((unsigned)(((p.nx + VT_X - 1) / VT_X) * ((p.ny + VT_Y - 1) / VT_Y)), (unsigned)(k1 - k0));
    if (krk == 0) {
        if (p.uniform_metrics) k_vis_div<true, false, R><<<nb, 256, 0, st>>>(p, 0, k0);
        else                   k_vis_div<false, false, R><<<nb, 256, 0, st>>>(p, 0, k0);
    } else {
        if (p.uniform_metrics) k_vis_div<true, true, R><<<nb, 256, 0, st>>>(p, krk, k0);
        else                   k_vis_div<false, true, R><<<nb, 256, 0, st>>>(p, krk, k0);
    }
    return cudaGetLastError();
}

// The viscous part in two launches with the Ev ghost exchange between them:
// k_vis_ev forms the 12 Ev fields (4 per direction) on the interior; the
// caller fills the ghosts of each direction's four (ev_ghost_fields); then
// k_vis_div.  krk = 0: viscous terms into du; krk = 1..3: viscous terms,
// then the RK stage update in the same kernel (du is not written).  FP32
// stencils in the precision form.
template <typename R, int H>
static bool launch_vev_h(const Params &p, cudaStream_t st, cudaError_t &err);
cudaError_t launch_vis_ev(const Params &p, cudaStream_t st) {
    const bool staged = p.vis_impl == 2 || (p.vis_impl == 0 && p.mixed);
    if (staged && p.kerr) {
        cudaError_t e = cudaSuccess;
        const bool c8 = p.scheme_vis == 204;
        const bool done = p.mixed ? (c8 ? launch_vev_h<float, 4>(p, st, e) : launch_vev_h<float, 3>(p, st, e))
                                  : (c8 ? launch_vev_h<double, 4>(p, st, e) : launch_vev_h<double, 3>(p, st, e));
        if (done) return e;
    }
    return p.mixed ? launch_vis_ev_t<float>(p, st) : launch_vis_ev_t<double>(p, st);
}

// persistent grid of the staged viscous kernels: blocks per SM from their
// shared memory, and the segment length along z with the fewest plane steps
// on the busiest block (two steps of ring fill counted per item)
template <typename K>
static void staged_grid(const Params &p, K kern, size_t smem_bytes, unsigned &nb, int &seg) {
    static int nsm = 0;
    if (!nsm) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
            cudaGetLastError();
            nsm = 148;
        }
    }
    // resident blocks per SM of this kernel (registers and shared memory)
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, VX * VY, smem_bytes) != cudaSuccess || occ < 1) {
        cudaGetLastError();
        occ = 1;
    }
    const long long bps = occ;
    const long long grid = (long long)nsm * bps;
    const long long tiles = (long long)((p.nx + VX - 1) / VX) * ((p.ny + VY - 1) / VY);
    int best = p.nz;
    long long best_cost = -1;
    for (int sl = 8; sl <= p.nz + 7; sl += 8) {
        const int len = sl < p.nz ? sl : p.nz;
        const long long items = tiles * ((p.nz + len - 1) / len);
        const long long cost = (items + grid - 1) / grid * (len + 2);
        if (best_cost < 0 || cost < best_cost) { best_cost = cost; best = len; }
        if (len == p.nz) break;
    }
    const long long items = tiles * ((p.nz + best - 1) / best);
    nb = (unsigned)(items < grid ? items : grid);
    seg = best;
}

// the staged Ev kernel; false when the tensor map cannot be formed
template <typename R, int H>
static bool launch_vev_h(const Params &p, cudaStream_t st, cudaError_t &err) {
    using T = VevTiles<R, H>;
    const unsigned long long eb = sizeof(R);
    const unsigned long long dims[4] = { (unsigned long long)p.ys, (unsigned long long)(p.ny + 2 * OCFD_LAP),
                                         (unsigned long long)(p.nz + 2 * OCFD_LAP), 4 };
    const unsigned long long strides[3] = { p.ys * eb, p.zs * eb, p.lapN * eb };
    const unsigned bq[4] = { (unsigned)T::PX, (unsigned)T::PY, 1, 4 };
    // (host code: the primitives of the form, u first)
    const R *prim1 = sizeof(R) == 4 ? reinterpret_cast<const R *>(p.prim32[1]) : reinterpret_cast<const R *>(p.prim[1]);
    if (p.prim[2] - p.prim[1] != p.lapN && sizeof(R) == 8) return false;
    if (sizeof(R) == 4 && p.prim32[2] - p.prim32[1] != p.lapN) return false;
    CUtensorMap tmq;
    if (!encode_map_4d(prim1, (int)eb, dims, strides, bq, &tmq)) return false;
    unsigned nb;
    int seg;
    auto kern = p.uniform_metrics ? k_vev<true, R, H> : k_vev<false, R, H>;
    staged_grid(p, kern, T::bytes, nb, seg);
    kern<<<nb, VX * VY, T::bytes, st>>>(p, tmq, seg);
    err = cudaGetLastError();
    return true;
}

// the staged divergence + RK stage over the whole slab; false when the tensor
// maps cannot be formed (the caller then uses k_vis_div)
template <typename R, int H>
static bool launch_vdiv_h(const Params &p, int krk, cudaStream_t st, cudaError_t &err) {
    using T = VdivTiles<R, H>;
    const unsigned long long eb = sizeof(R);
    const unsigned long long dims[4] = { (unsigned long long)p.ys, (unsigned long long)(p.ny + 2 * OCFD_LAP),
                                         (unsigned long long)(p.nz + 2 * OCFD_LAP), 4 };
    const unsigned long long strides[3] = { p.ys * eb, p.zs * eb, p.lapN * eb };
    const unsigned bx[4] = { VX + 2 * VXH, VY, 1, 4 }, by[4] = { VX, VY + 2 * H, 1, 4 }, bz[4] = { VX, VY, 1, 4 };
    // (host code: the Ev base of the form, not the device accessor ev_r)
    const R *ev = sizeof(R) == 4 ? reinterpret_cast<const R *>(p.ev32) : reinterpret_cast<const R *>(p.ev);
    CUtensorMap tmx, tmy, tmz;
    if (!encode_map_4d(ev, (int)eb, dims, strides, bx, &tmx) ||
        !encode_map_4d(ev + 4 * p.lapN, (int)eb, dims, strides, by, &tmy) ||
        !encode_map_4d(ev + 8 * p.lapN, (int)eb, dims, strides, bz, &tmz))
        return false;
    unsigned nb;
    int best;
    auto kern = p.uniform_metrics ? k_vdiv<true, R, H> : k_vdiv<false, R, H>;
    staged_grid(p, kern, T::bytes, nb, best);
    kern<<<nb, VX * VY, T::bytes, st>>>(p, tmx, tmy, tmz, krk, best);
    err = cudaGetLastError();
    return true;
}

// the dynamic shared-memory size of every staged-divergence instance, set on
// the current device before the first launch (and before any stream capture)
cudaError_t vdiv_prepare() {
    cudaError_t e = cudaSuccess;
    auto one = [&](auto kern, size_t bytes) {
        if (e == cudaSuccess) e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    };
    one(k_vdiv<true, double, 3>, VdivTiles<double, 3>::bytes);  one(k_vdiv<false, double, 3>, VdivTiles<double, 3>::bytes);
    one(k_vdiv<true, double, 4>, VdivTiles<double, 4>::bytes);  one(k_vdiv<false, double, 4>, VdivTiles<double, 4>::bytes);
    one(k_vdiv<true, float, 3>, VdivTiles<float, 3>::bytes);    one(k_vdiv<false, float, 3>, VdivTiles<float, 3>::bytes);
    one(k_vdiv<true, float, 4>, VdivTiles<float, 4>::bytes);    one(k_vdiv<false, float, 4>, VdivTiles<float, 4>::bytes);
    one(k_vev<true, double, 3>, VevTiles<double, 3>::bytes);    one(k_vev<false, double, 3>, VevTiles<double, 3>::bytes);
    one(k_vev<true, double, 4>, VevTiles<double, 4>::bytes);    one(k_vev<false, double, 4>, VevTiles<double, 4>::bytes);
    one(k_vev<true, float, 3>, VevTiles<float, 3>::bytes);      one(k_vev<false, float, 3>, VevTiles<float, 3>::bytes);
    one(k_vev<true, float, 4>, VevTiles<float, 4>::bytes);      one(k_vev<false, float, 4>, VevTiles<float, 4>::bytes);
    return e;
}

// planes k0 .. k1-1 (the whole slab: 0, nz)
cudaError_t launch_vis_div(const Params &p, int krk, int k0, int k1, cudaStream_t st) {
    const bool staged = p.vis_impl == 2 || (p.vis_impl == 0 && p.mixed);
    if (krk > 0 && k0 == 0 && k1 == p.nz && staged && p.kerr) {
        cudaError_t e = cudaSuccess;
        const bool c8 = p.scheme_vis == 204;
        const bool done = p.mixed ? (c8 ? launch_vdiv_h<float, 4>(p, krk, st, e) : launch_vdiv_h<float, 3>(p, krk, st, e))
                                  : (c8 ? launch_vdiv_h<double, 4>(p, krk, st, e) : launch_vdiv_h<double, 3>(p, krk, st, e));
        if (done) return e;
    }
    return p.mixed ? launch_vis_div_t<float>(p, krk, k0, k1, st) : launch_vis_div_t<double>(p, krk, k0, k1, st);
}

// base pointers of the 12 Ev fields (FP64, or FP32 in the precision form)
// and the direction each needs ghosts in (bit d for direction d)
void ev_ghost_fields(const Params &p, void *fields[12], int dirmask[12]) {
    char *evb = p.mixed ? (char *)p.ev32 : (char *)p.ev;
    const size_t es = p.mixed ? sizeof(float) : sizeof(double);
    for (int dd = 0; dd < 3; dd++)
        for (int m = 0; m < 4; m++) {
            fields[4 * dd + m] = evb + (size_t)(4 * dd + m) * (size_t)p.lapN * es;
            dirmask[4 * dd + m] = 1 << dd;
        }
}

cudaError_t launch_q_criterion(const Params &p, double *q, cudaStream_t st) {
    const dim3 nb((unsigned)(((p.nx + VT_X - 1) / VT_X) * ((p.ny + VT_Y - 1) / VT_Y)), (unsigned)p.nz);
    if (p.uniform_metrics) k_qcrit<true><<<nb, 256, 0, st>>>(p, q);
    else                   k_qcrit<false><<<nb, 256, 0, st>>>(p, q);
    return cudaGetLastError();
}

cudaError_t launch_time_average(const Params &p, double *mean5, int n, cudaStream_t st) {
    k_time_average<<<blocks_for(p.N, 256), 256, 0, st>>>(p, mean5, n);
    return cudaGetLastError();
}

cudaError_t launch_rk(const Params &p, int krk, cudaStream_t st) {
    k_rk_update<<<blocks_for(p.N, 256), 256, 0, st>>>(p, krk);
    return cudaGetLastError();
}

cudaError_t launch_p2c(const Params &p, double *out, cudaStream_t st) {
    k_p2c<<<blocks_for(p.N, 256), 256, 0, st>>>(p, out);
    return cudaGetLastError();
}

cudaError_t launch_scatter(const Params &p, const double *src, double *dst_lap, cudaStream_t st) {
    k_scatter_interior<<<blocks_for(p.N, 256), 256, 0, st>>>(p, src, dst_lap);
    return cudaGetLastError();
}

cudaError_t launch_gather(const Params &p, const double *src_lap, double *dst, cudaStream_t st) {
    k_gather_interior<<<blocks_for(p.N, 256), 256, 0, st>>>(p, src_lap, dst);
    return cudaGetLastError();
}

cudaError_t launch_fill(double *f, long long n, double v, cudaStream_t st) {
    k_fill<<<blocks_for(n, 256), 256, 0, st>>>(f, n, v);
    return cudaGetLastError();
}

cudaError_t launch_rk_only(const Params &p, int krk, cudaStream_t st) {
    k_rk_only<<<blocks_for(5 * p.N, 256), 256, 0, st>>>(p, krk);
    return cudaGetLastError();
}
cudaError_t launch_flag_hist(const Params &p, unsigned long long *counts, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(counts, 0, 9 * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    k_flag_hist<<<4 * 148, 256, 0, st>>>(p, counts);
    return cudaGetLastError();
}

cudaError_t launch_prims_to_fp32(const Params &p, cudaStream_t st) {
    k_prims_to_fp32<<<blocks_for(5 * p.lapN, 256), 256, 0, st>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_c2p(const Params &p, cudaStream_t st) {
    k_c2p<<<blocks_for(p.N, 256), 256, 0, st>>>(p);
    return cudaGetLastError();
}
cudaError_t launch_bc_faces(const Params &p, cudaStream_t st) {
    k_bc_faces<<<blocks_for(p.N, 256), 256, 0, st>>>(p);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// FP64 mean of an interior field (ana_residual, src/OCFD_ana.cu:50-105) and
// the NaN / negative-T scan (ana_NAN_and_NT, src/OCFD_ana.cu:107-222).
// Deterministic: a fixed grid of RED_BLOCKS blocks, each summing a fixed
// strided subset in a fixed order and reducing in a fixed tree; one block
// then sums the partials in order.  (The reference's reduction assumes
// 64-wide warps and is wrong on 32-wide ones; this one is not.)
// ---------------------------------------------------------------------------
constexpr int RED_BLOCKS = 592;     // 4 x 148 SMs
constexpr int RED_THREADS = 256;

// src: which = 0 conserved energy f[4] (dense), 1 temperature (LAP box)
__global__ void __launch_bounds__(RED_THREADS) k_reduce_partial(Params p, int which, double *partial,
                                                               unsigned long long *counts) {
    __shared__ double sh[RED_THREADS];
    __shared__ unsigned int nn[2];
    if (threadIdx.x < 2) nn[threadIdx.x] = 0;
    __syncthreads();
    double acc = 0.0;
    unsigned int nnan = 0, nneg = 0;
    long long stride = (long long)gridDim.x * blockDim.x;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < p.N; q += stride) {
        int i = (int)(q % p.nx); long long r = q / p.nx;
        int j = (int)(r % p.ny); int k = (int)(r / p.ny);
        double v;
        if (which == 0) {
            v = p.f[4 * p.N + q];
        } else {
            v = p.prim[4][lap_index(p, i + OCFD_LAP, j + OCFD_LAP, k + OCFD_LAP)];
        }
        acc += v;
        if (counts) {
            long long o = lap_index(p, i + OCFD_LAP, j + OCFD_LAP, k + OCFD_LAP);
            bool bad = false;
            for (int m = 0; m < 5; m++) bad |= isnan(p.prim[m][o]);
            nnan += bad;
            nneg += p.prim[4][o] < 0.0;
        }
    }
    sh[threadIdx.x] = acc;
    if (counts && (nnan | nneg)) { atomicAdd(&nn[0], nnan); atomicAdd(&nn[1], nneg); }
    __syncthreads();
    for (int h = RED_THREADS / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) sh[threadIdx.x] += sh[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partial[blockIdx.x] = sh[0];
        if (counts && (nn[0] | nn[1])) { atomicAdd(&counts[0], nn[0]); atomicAdd(&counts[1], nn[1]); }
    }
}

__global__ void __launch_bounds__(RED_THREADS) k_reduce_final(const double *partial, int n, double ncell,
                                                             double *out) {
    __shared__ double sh[RED_THREADS];
    double acc = 0.0;
    for (int q = threadIdx.x; q < n; q += blockDim.x) acc += partial[q];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int h = RED_THREADS / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) sh[threadIdx.x] += sh[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = sh[0] / ncell;       // E0 /= NX*NY*NZ (src/OCFD_ana.cu:103)
}

// scratch: RED_BLOCKS + 1 doubles and two counters
// ncell: the divisor (the cells of the whole grid; with the grid split in z
// each slab divides its sum by the whole grid's count and the slabs' results
// are summed)
cudaError_t launch_mean(const Params &p, int which, double *scratch, unsigned long long *counts, double ncell,
                        cudaStream_t st) {
    if (counts) {
        cudaError_t e = cudaMemsetAsync(counts, 0, 2 * sizeof(unsigned long long), st);
        if (e != cudaSuccess) return e;
    }
    k_reduce_partial<<<RED_BLOCKS, RED_THREADS, 0, st>>>(p, which, scratch, counts);
    k_reduce_final<<<1, RED_THREADS, 0, st>>>(scratch, RED_BLOCKS, ncell, scratch + RED_BLOCKS);
    return cudaGetLastError();
}
int reduce_scratch_doubles() { return RED_BLOCKS + 1; }

}  // namespace ocfd
