// ocfd_learned.cu -- learned scheme switch (sm_100a).
//
// Replaces the choice Comput_Scheme_point_Jameson makes
// (src/OCFD_Schemes_hybrid_auto.cu:611-703) with a small network and keeps
// that sensor as the fallback: the same int8 flag arrays are written (flag
// 1 UP7, 2 WENO7, 3 WENO5; the entry of face q along a direction belongs to
// cell q-1, so the cells of the extended box -1 .. n-1 are visited once
// and each writes the entries it owns in the three arrays).
//
// Features (14, FP32) of a cell, over the sensor's 7-point stencil, with
// P = p00 d T the sensor's pressure and D = d:
//   per direction x, y, z: |P- - 2P0 + P+| / (P- + 2P0 + P+),
//                          (P+ - P-) / (P- + 2P0 + P+), and the same for D;
//   the sums of the three second-difference terms of P and of D.
// The sum for P is the plain sensor's value, formed in the same order and
// precision as k_sensor, so the fallback flag is the plain flag exactly.
//
// Network: 14 -> 32 -> 32 -> 1 with ReLU, inputs standardised by (mu,
// sigma); parameter vector mu[14] sigma[14] W1[32][14] b1[32] W2[32][32]
// b2[32] W3[32] b3.  Inference runs the two hidden layers on the tensor
// cores (mma.sync m16n8k16, BF16 operands, FP32 accumulation), one warp per
// 32 cells; the output layer is an FP32 dot product.  A cell whose
// confidence max(s, 1-s), s = sigmoid(logit), is below the threshold keeps
// the plain flag; otherwise flag 1 for s < 1/2 and max(2, plain flag) for
// s >= 1/2.  Training runs in FP32: per-block forward and backward passes
// with the activations in shared memory, a fixed-order reduction of the
// block gradients, and Adam.
#include "ocfd_fp32.cuh"

#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace ocfd {

constexpr int MLP_IN = 14, MLP_H = 32;
constexpr int OFF_MU = 0, OFF_SG = 14, OFF_W1 = 28, OFF_B1 = OFF_W1 + MLP_H * MLP_IN, OFF_W2 = OFF_B1 + MLP_H,
              OFF_B2 = OFF_W2 + MLP_H * MLP_H, OFF_W3 = OFF_B2 + MLP_H, OFF_B3 = OFF_W3 + MLP_H,
              MLP_NPARAM = OFF_B3 + 1, MLP_NNET = MLP_NPARAM - OFF_W1;

// ---------------------------------------------------------------------------
// features
// ---------------------------------------------------------------------------
// om[a], op[a]: offsets of the minus / plus neighbour along direction a
template <typename R>
__device__ __forceinline__ void switch_features(const Params &p, long long c, const long long (&om)[3],
                                                const long long (&op)[3], float f[MLP_IN], R &dp) {
    const R *d = prim_r<R>(p, 0), *T = prim_r<R>(p, 4);
    const R p00 = (R)p.p00;
    auto P = [&](long long o) { return p00 * d[o] * T[o]; };
    const R P0 = P(c), D0 = d[c];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const R Pm = P(c + om[a]), Pp = P(c + op[a]);
        const R den = Pm + 2*P0 + Pp;
        const R t = fabs(-Pm + 2*P0 - Pp)/den;          // k_sensor's term
        dp = a == 0 ? t : dp + t;
        f[a] = (float)t;
        f[3 + a] = (float)((Pp - Pm) / den);
        const R Dm = d[c + om[a]], Dp = d[c + op[a]];
        const R rdd = (R)1 / (Dm + 2*D0 + Dp);
        f[6 + a] = (float)(fabs(-Dm + 2*D0 - Dp) * rdd);
        f[9 + a] = (float)((Dp - Dm) * rdd);
    }
    f[12] = f[0] + f[1] + f[2];
    f[13] = f[6] + f[7] + f[8];
}

template <typename R>
__device__ __forceinline__ int plain_flag(const Params &p, R dp) {
    int kp = 1;
    if (dp > (R)p.dp1) kp += 1;
    if (dp > (R)p.dp2) kp += 1;
    return kp;
}

// Features and labels (plain flag >= 2) of interior cells first ..
// first+count-1 of the current state.  A periodic direction takes its
// neighbours across the seam from the interior, not from the ghost layer
// (which after a step still holds the values of the last stage's start).
__global__ void k_switch_features(Params p, long long first, long long count, float *feat, float *label) {
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= count) return;
    const long long q = first + tid;
    const int i = (int)(q % p.nx);
    const long long r = q / p.nx;
    const int j = (int)(r % p.ny), k = (int)(r / p.ny);
    const long long c = lap_index(p, i + OCFD_LAP, j + OCFD_LAP, k + OCFD_LAP);
    const long long st[3] = {1LL, p.ys, p.zs};
    const int X[3] = {i, j, k}, n[3] = {p.nx, p.ny, p.nz};
    long long om[3], op[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        om[a] = (p.periodic[a] && X[a] == 0) ? (long long)(n[a] - 1) * st[a] : -st[a];
        op[a] = (p.periodic[a] && X[a] == n[a] - 1) ? -(long long)(n[a] - 1) * st[a] : st[a];
    }
    float f[MLP_IN];
    double dp;
    switch_features<double>(p, c, om, op, f, dp);
#pragma unroll
    for (int m = 0; m < MLP_IN; m++) feat[tid * MLP_IN + m] = f[m];
    label[tid] = plain_flag(p, dp) >= 2 ? 1.0f : 0.0f;
}

// ---------------------------------------------------------------------------
// tensor-core MLP of one warp: 32 rows of standardised features in, 32
// logits out (lane L gets row L)
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned pack_bf16(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<unsigned *>(&v);
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], const unsigned (&a)[4], unsigned b0, unsigned b1) {
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
                 "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// one lane's share of the network for the tensor-core products: B operands
// of layer 1 (n-tiles 0..3) and layer 2 (n-tiles 0..3, k-steps 0..1) as
// BF16 pairs, and the biases / output weights of its accumulator columns
struct MlpFrag {
    unsigned w1[4][2], w2[4][2][2];
    float b1[4][2], b2[4][2], w3[4][2], b3;
};

__device__ __forceinline__ void load_frags(const float *__restrict__ w, MlpFrag &fr) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int nt = 0; nt < 4; nt++) {
        const int n = nt * 8 + g;
        const float *W1 = w + OFF_W1 + n * MLP_IN;
        fr.w1[nt][0] = pack_bf16(W1[2 * t], W1[2 * t + 1]);
        fr.w1[nt][1] = 2 * t + 8 < MLP_IN ? pack_bf16(W1[2 * t + 8], W1[2 * t + 9]) : 0u;
        const float *W2 = w + OFF_W2 + n * MLP_H;
#pragma unroll
        for (int kk = 0; kk < 2; kk++) {
            fr.w2[nt][kk][0] = pack_bf16(W2[kk * 16 + 2 * t], W2[kk * 16 + 2 * t + 1]);
            fr.w2[nt][kk][1] = pack_bf16(W2[kk * 16 + 2 * t + 8], W2[kk * 16 + 2 * t + 9]);
        }
#pragma unroll
        for (int h = 0; h < 2; h++) {
            fr.b1[nt][h] = w[OFF_B1 + nt * 8 + 2 * t + h];
            fr.b2[nt][h] = w[OFF_B2 + nt * 8 + 2 * t + h];
            fr.w3[nt][h] = w[OFF_W3 + nt * 8 + 2 * t + h];
        }
    }
    fr.b3 = w[OFF_B3];
}

// x: this lane's 14 standardised features; sA: 32 x 16 bf16 (one warp's
// staging), sL: 32 floats; returns this lane's logit
__device__ __forceinline__ float warp_mlp(const MlpFrag &fr, const float (&x)[MLP_IN],
                                          __nv_bfloat16 *sA, float *sL) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    __syncwarp();                       // the previous tile's reads of sA / sL are done
#pragma unroll
    for (int m = 0; m < 16; m += 2) {
        const unsigned v = pack_bf16(m < MLP_IN ? x[m] : 0.0f, m + 1 < MLP_IN ? x[m + 1] : 0.0f);
        *reinterpret_cast<unsigned *>(sA + lane * 16 + m) = v;
    }
    __syncwarp();
    // layer 1: Z1 (32 x 32) = X (32 x 16) W1^T + b1; B[k][n] = W1[n][k]
    float z1[2][4][4];
#pragma unroll
    for (int mt = 0; mt < 2; mt++) {
        const __nv_bfloat16 *row0 = sA + (mt * 16 + g) * 16, *row1 = sA + (mt * 16 + g + 8) * 16;
        unsigned a[4];
        a[0] = *reinterpret_cast<const unsigned *>(row0 + 2 * t);
        a[1] = *reinterpret_cast<const unsigned *>(row1 + 2 * t);
        a[2] = *reinterpret_cast<const unsigned *>(row0 + 2 * t + 8);
        a[3] = *reinterpret_cast<const unsigned *>(row1 + 2 * t + 8);
#pragma unroll
        for (int nt = 0; nt < 4; nt++) {
            z1[mt][nt][0] = fr.b1[nt][0]; z1[mt][nt][1] = fr.b1[nt][1];
            z1[mt][nt][2] = fr.b1[nt][0]; z1[mt][nt][3] = fr.b1[nt][1];
            mma_bf16(z1[mt][nt], a, fr.w1[nt][0], fr.w1[nt][1]);
        }
    }
    // ReLU; the accumulator tiles of n-tiles 2kk and 2kk+1 are the A operand
    // of k-step kk of layer 2
    unsigned a2[2][2][4];
#pragma unroll
    for (int mt = 0; mt < 2; mt++)
#pragma unroll
        for (int kk = 0; kk < 2; kk++) {
            const float *lo = z1[mt][2 * kk], *hi = z1[mt][2 * kk + 1];
            a2[mt][kk][0] = pack_bf16(fmaxf(lo[0], 0.0f), fmaxf(lo[1], 0.0f));
            a2[mt][kk][1] = pack_bf16(fmaxf(lo[2], 0.0f), fmaxf(lo[3], 0.0f));
            a2[mt][kk][2] = pack_bf16(fmaxf(hi[0], 0.0f), fmaxf(hi[1], 0.0f));
            a2[mt][kk][3] = pack_bf16(fmaxf(hi[2], 0.0f), fmaxf(hi[3], 0.0f));
        }
    // layer 2 and the output layer's partial dot products
    float part[2][2] = {{0.0f, 0.0f}, {0.0f, 0.0f}};     // [m-tile][row g / g+8]
#pragma unroll
    for (int nt = 0; nt < 4; nt++) {
#pragma unroll
        for (int mt = 0; mt < 2; mt++) {
            float z[4] = {fr.b2[nt][0], fr.b2[nt][1], fr.b2[nt][0], fr.b2[nt][1]};
            mma_bf16(z, a2[mt][0], fr.w2[nt][0][0], fr.w2[nt][0][1]);
            mma_bf16(z, a2[mt][1], fr.w2[nt][1][0], fr.w2[nt][1][1]);
            part[mt][0] += fmaxf(z[0], 0.0f) * fr.w3[nt][0] + fmaxf(z[1], 0.0f) * fr.w3[nt][1];
            part[mt][1] += fmaxf(z[2], 0.0f) * fr.w3[nt][0] + fmaxf(z[3], 0.0f) * fr.w3[nt][1];
        }
    }
#pragma unroll
    for (int mt = 0; mt < 2; mt++)
#pragma unroll
        for (int h = 0; h < 2; h++) {
            float v = part[mt][h];
            v += __shfl_xor_sync(0xffffffffu, v, 1);
            v += __shfl_xor_sync(0xffffffffu, v, 2);
            if (t == 0) sL[mt * 16 + h * 8 + g] = v;
        }
    __syncwarp();
    return sL[lane] + fr.b3;
}

// (f - mu) / sigma, as a product with the block's reciprocals of sigma
__device__ __forceinline__ void standardise(const float *mu, const float *isg, const float (&f)[MLP_IN],
                                            float (&x)[MLP_IN]) {
#pragma unroll
    for (int m = 0; m < MLP_IN; m++) x[m] = (f[m] - mu[m]) * isg[m];
}

// the block's copy of the standardisation constants (mu, 1 / sigma)
__device__ __forceinline__ void load_standard(const float *__restrict__ w, float *sMu, float *sIsg) {
    if (threadIdx.x < MLP_IN) { sMu[threadIdx.x] = w[OFF_MU + threadIdx.x]; sIsg[threadIdx.x] = 1.0f / w[OFF_SG + threadIdx.x]; }
    __syncthreads();
}

// logits of n raw feature rows (the network alone, for checks); each warp
// loads its weight fragments once and walks 32-row tiles
__global__ void __launch_bounds__(128) k_mlp_infer(const float *__restrict__ w, const float *__restrict__ feat,
                                                   long long n, float *logit) {
    __shared__ __align__(16) __nv_bfloat16 sA[4][32 * 16];
    __shared__ float sL[4][32], sMu[MLP_IN], sIsg[MLP_IN];
    load_standard(w, sMu, sIsg);
    MlpFrag fr;
    load_frags(w, fr);
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long ntile = (n + 31) / 32, nw = (long long)gridDim.x * 4;
    for (long long tile = (long long)blockIdx.x * 4 + wid; tile < ntile; tile += nw) {
        const long long row = tile * 32 + lane;
        float f[MLP_IN], x[MLP_IN];
#pragma unroll
        for (int m = 0; m < MLP_IN; m++) f[m] = row < n ? feat[row * MLP_IN + m] : 0.0f;
        standardise(sMu, sIsg, f, x);
        const float z = warp_mlp(fr, x, sA[wid], sL[wid]);
        if (row < n) logit[row] = z;
    }
}

// The learned switch over the extended box: cell (i, j, k), each of -1 ..
// n-1, owns entry i+1 of the x array (when j, k are interior), entry j+1 of
// the y array and entry k+1 of the z array.  conf_logit = ln(c / (1 - c))
// for confidence threshold c.  stats (optional): cells decided by the
// network, cells left to the plain flag, network flags that differ from the
// plain flag.
template <typename R>
__global__ void __launch_bounds__(128) k_switch_infer(Params p, const float *__restrict__ w, float conf_logit,
                                                      unsigned long long *stats) {
    __shared__ __align__(16) __nv_bfloat16 sA[4][32 * 16];
    __shared__ float sL[4][32], sMu[MLP_IN], sIsg[MLP_IN];
    load_standard(w, sMu, sIsg);
    MlpFrag fr;
    load_frags(w, fr);
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long ex = p.nx + 1, ey = p.ny + 1, ez = p.nz + 1, total = ex * ey * ez;
    const long long ntile = (total + 31) / 32, nw = (long long)gridDim.x * 4;
    const long long om[3] = {-1LL, -p.ys, -p.zs}, op[3] = {1LL, p.ys, p.zs};
    unsigned long long n_sure = 0, n_unsure = 0, n_differ = 0;
    for (long long tile = (long long)blockIdx.x * 4 + wid; tile < ntile; tile += nw) {
        const long long tid = tile * 32 + lane;
        const bool live = tid < total;
        int i = 0, j = 0, k = 0;
        float f[MLP_IN] = {};
        R dp = (R)0;
        if (live) {
            i = (int)(tid % ex) - 1;
            const long long r = tid / ex;
            j = (int)(r % ey) - 1; k = (int)(r / ey) - 1;
            switch_features<R>(p, lap_index(p, i + OCFD_LAP, j + OCFD_LAP, k + OCFD_LAP), om, op, f, dp);
        }
        float x[MLP_IN];
        standardise(sMu, sIsg, f, x);
        const float z = warp_mlp(fr, x, sA[wid], sL[wid]);
        const int plain = plain_flag(p, dp);
        const bool sure = fabsf(z) >= conf_logit;
        const int kp = sure ? (z >= 0.0f ? max(2, plain) : 1) : plain;
        const bool inx = live && j >= 0 && k >= 0, iny = live && i >= 0 && k >= 0, inz = live && i >= 0 && j >= 0;
        if (inx) p.flag[0][(long long)(i + 1) + ex * ((long long)j + (long long)p.ny * k)] = (int8_t)kp;
        if (iny) p.flag[1][(long long)i + (long long)p.nx * ((long long)(j + 1) + ey * k)] = (int8_t)kp;
        if (inz) p.flag[2][(long long)i + (long long)p.nx * ((long long)j + (long long)p.ny * (k + 1))] = (int8_t)kp;
        if (p.flag_count) {          // faces per direction whose flag is not 1
            const bool non1 = kp != 1;
            const unsigned mx = __ballot_sync(0xffffffffu, non1 && inx), my = __ballot_sync(0xffffffffu, non1 && iny),
                           mz = __ballot_sync(0xffffffffu, non1 && inz);
            if (lane == 0) {
                if (mx) atomicAdd(p.flag_count + 0, (unsigned)__popc(mx));
                if (my) atomicAdd(p.flag_count + 1, (unsigned)__popc(my));
                if (mz) atomicAdd(p.flag_count + 2, (unsigned)__popc(mz));
            }
        }
        if (stats) {
            const unsigned ms = __ballot_sync(0xffffffffu, live && sure), mu = __ballot_sync(0xffffffffu, live && !sure),
                           md = __ballot_sync(0xffffffffu, live && sure && kp != plain);
            n_sure += __popc(ms); n_unsure += __popc(mu); n_differ += __popc(md);
        }
    }
    if (stats && lane == 0 && (n_sure | n_unsure | n_differ)) {
        atomicAdd(stats + 0, n_sure);
        atomicAdd(stats + 1, n_unsure);
        atomicAdd(stats + 2, n_differ);
    }
}

// ---------------------------------------------------------------------------
// training (FP32)
// ---------------------------------------------------------------------------
constexpr int TB = 64;     // samples (and threads) per block

// Forward and backward pass of TB samples (rows idx[0..], or 0.. when idx is
// null); writes this block's gradient sums (MLP_NNET values, in the order of
// the parameter vector from W1) to part[blockIdx.x] and its loss sum to
// lpart[blockIdx.x].  Loss: BCE with logits, positive samples weighted pos_w.
__global__ void __launch_bounds__(TB) k_mlp_grad(const float *__restrict__ w, const float *__restrict__ feat,
                                                 const float *__restrict__ label, const int *__restrict__ idx,
                                                 long long n, float pos_w, float *__restrict__ part,
                                                 float *__restrict__ lpart) {
    __shared__ float sX[TB][MLP_IN + 1], sH1[TB][MLP_H + 1], sD1[TB][MLP_H + 1], sH2[TB][MLP_H + 1],
        sD2[TB][MLP_H + 1], sD3[TB], sLoss[TB];
    const int s = threadIdx.x;
    const long long row = (long long)blockIdx.x * TB + s;
    const bool live = row < n;
    // this sample's vectors live in its own rows of the shared arrays; the
    // ReLU masks are bit masks
    const long long src = live ? (idx ? (long long)idx[row] : row) : 0;
    for (int m = 0; m < MLP_IN; m++)
        sX[s][m] = live ? (feat[src * MLP_IN + m] - w[OFF_MU + m]) / w[OFF_SG + m] : 0.0f;
    unsigned mask1 = 0u, mask2 = 0u;
#pragma unroll 4
    for (int a = 0; a < MLP_H; a++) {
        float acc = w[OFF_B1 + a];
        for (int m = 0; m < MLP_IN; m++) acc += w[OFF_W1 + a * MLP_IN + m] * sX[s][m];
        if (acc > 0.0f) mask1 |= 1u << a;
        sH1[s][a] = fmaxf(acc, 0.0f);
    }
    float z3 = w[OFF_B3];
#pragma unroll 4
    for (int a = 0; a < MLP_H; a++) {
        float acc = w[OFF_B2 + a];
        for (int m = 0; m < MLP_H; m++) acc += w[OFF_W2 + a * MLP_H + m] * sH1[s][m];
        if (acc > 0.0f) mask2 |= 1u << a;
        const float h = fmaxf(acc, 0.0f);
        sH2[s][a] = h;
        z3 += w[OFF_W3 + a] * h;
    }
    float d3 = 0.0f, loss = 0.0f;
    if (live) {
        const float y = label[src], wt = y > 0.5f ? pos_w : 1.0f;
        loss = wt * (fmaxf(z3, 0.0f) - z3 * y + log1pf(expf(-fabsf(z3))));
        d3 = wt * (1.0f / (1.0f + expf(-z3)) - y);
    }
    for (int a = 0; a < MLP_H; a++) sD2[s][a] = ((mask2 >> a) & 1u) ? d3 * w[OFF_W3 + a] : 0.0f;
#pragma unroll 4
    for (int m = 0; m < MLP_H; m++) {
        float acc = 0.0f;
        for (int a = 0; a < MLP_H; a++) acc += w[OFF_W2 + a * MLP_H + m] * sD2[s][a];
        sD1[s][m] = ((mask1 >> m) & 1u) ? acc : 0.0f;
    }
    sD3[s] = d3; sLoss[s] = loss;
    __syncthreads();
    float *out = part + (long long)blockIdx.x * MLP_NNET;
    for (int o = s; o < MLP_NNET; o += TB) {
        float acc = 0.0f;
        if (o < MLP_H * MLP_IN) {                       // W1[a][m]
            const int a = o / MLP_IN, m = o % MLP_IN;
            for (int q = 0; q < TB; q++) acc += sD1[q][a] * sX[q][m];
        } else if (o < MLP_H * MLP_IN + MLP_H) {        // b1
            const int a = o - MLP_H * MLP_IN;
            for (int q = 0; q < TB; q++) acc += sD1[q][a];
        } else if (o < MLP_H * MLP_IN + MLP_H + MLP_H * MLP_H) {   // W2[a][m]
            const int e = o - MLP_H * MLP_IN - MLP_H, a = e / MLP_H, m = e % MLP_H;
            for (int q = 0; q < TB; q++) acc += sD2[q][a] * sH1[q][m];
        } else if (o < MLP_H * MLP_IN + 2 * MLP_H + MLP_H * MLP_H) {   // b2
            const int a = o - MLP_H * MLP_IN - MLP_H - MLP_H * MLP_H;
            for (int q = 0; q < TB; q++) acc += sD2[q][a];
        } else if (o < MLP_NNET - 1) {                  // W3
            const int a = o - MLP_H * MLP_IN - 2 * MLP_H - MLP_H * MLP_H;
            for (int q = 0; q < TB; q++) acc += sD3[q] * sH2[q][a];
        } else {                                        // b3
            for (int q = 0; q < TB; q++) acc += sD3[q];
        }
        out[o] = acc;
    }
    if (s == 0) {
        float l = 0.0f;
        for (int q = 0; q < TB; q++) l += sLoss[q];
        lpart[blockIdx.x] = l;
    }
}

// fixed-order sum over blocks: grad[o] = sum_b part[b][o]; loss likewise
__global__ void k_mlp_reduce(const float *__restrict__ part, const float *__restrict__ lpart, int nb,
                             float *__restrict__ grad, double *__restrict__ loss) {
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o < MLP_NNET) {
        float acc = 0.0f;
        for (int b = 0; b < nb; b++) acc += part[(long long)b * MLP_NNET + o];
        grad[o] = acc;
    }
    if (o == 0) {
        double l = 0.0;
        for (int b = 0; b < nb; b++) l += lpart[b];
        *loss += l;
    }
}

// Adam on the network part of the parameter vector (grad = batch sum)
__global__ void k_mlp_adam(float *__restrict__ w, const float *__restrict__ grad, float *__restrict__ m1,
                           float *__restrict__ m2, float scale, float lr, float b1, float b2, float eps,
                           float c1, float c2) {
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= MLP_NNET) return;
    const float g = grad[o] * scale;
    const float a = b1 * m1[o] + (1.0f - b1) * g, v = b2 * m2[o] + (1.0f - b2) * g * g;
    m1[o] = a; m2[o] = v;
    w[OFF_W1 + o] -= lr * (a / c1) / (sqrtf(v / c2) + eps);
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
int mlp_nparam() { return MLP_NPARAM; }
int mlp_nnet() { return MLP_NNET; }
int mlp_grad_blocks(long long n) { return (int)((n + TB - 1) / TB); }

cudaError_t launch_switch_features(const Params &p, long long first, long long count, float *feat, float *label,
                                   cudaStream_t st) {
    k_switch_features<<<(unsigned)((count + 255) / 256), 256, 0, st>>>(p, first, count, feat, label);
    return cudaGetLastError();
}

cudaError_t launch_switch_infer(const Params &p, const float *w, float conf_logit, unsigned long long *stats,
                                cudaStream_t st) {
    if (p.flag_count) {
        cudaError_t e = cudaMemsetAsync(p.flag_count, 0, 3 * sizeof(unsigned), st);
        if (e != cudaSuccess) return e;
    }
    // persistent warps: a few resident blocks per SM, each warp over many tiles
    const long long n = (long long)(p.nx + 1) * (p.ny + 1) * (p.nz + 1);
    const long long need = (n + 127) / 128;
    const unsigned nb = (unsigned)(need < 148 * 4 ? need : 148 * 4);
    if (p.mixed) k_switch_infer<float><<<nb, 128, 0, st>>>(p, w, conf_logit, stats);
    else         k_switch_infer<double><<<nb, 128, 0, st>>>(p, w, conf_logit, stats);
    return cudaGetLastError();
}

cudaError_t launch_mlp_infer(const float *w, const float *feat, long long n, float *logit, cudaStream_t st) {
    const long long need = (n + 127) / 128;
    k_mlp_infer<<<(unsigned)(need < 148 * 8 ? need : 148 * 8), 128, 0, st>>>(w, feat, n, logit);
    return cudaGetLastError();
}

// gradient (batch sum) and loss sum of rows idx[0..n) (or 0..n)
cudaError_t launch_mlp_grad(const float *w, const float *feat, const float *label, const int *idx, long long n,
                            float pos_w, float *part, float *lpart, float *grad, double *loss, cudaStream_t st) {
    const int nb = mlp_grad_blocks(n);
    k_mlp_grad<<<nb, TB, 0, st>>>(w, feat, label, idx, n, pos_w, part, lpart);
    k_mlp_reduce<<<(MLP_NNET + 255) / 256, 256, 0, st>>>(part, lpart, nb, grad, loss);
    return cudaGetLastError();
}

cudaError_t launch_mlp_adam(float *w, const float *grad, float *m1, float *m2, float scale, float lr, int t,
                            cudaStream_t st) {
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - powf(b1, (float)t), c2 = 1.0f - powf(b2, (float)t);
    k_mlp_adam<<<(MLP_NNET + 255) / 256, 256, 0, st>>>(w, grad, m1, m2, scale, lr, b1, b2, 1e-8f, c1, c2);
    return cudaGetLastError();
}

}  // namespace ocfd
