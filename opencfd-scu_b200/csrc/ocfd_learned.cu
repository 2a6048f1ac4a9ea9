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
// precision as k_sensor_march, so the fallback flag is the plain flag exactly.
//
// Network: 14 -> 32 -> 32 -> 1 with ReLU, inputs standardised by (mu,
// sigma); parameter vector mu[14] sigma[14] W1[32][14] b1[32] W2[32][32]
// b2[32] W3[32] b3.  Inference runs the two hidden layers as tcgen05
// products of 128 cells (one block) at a time: BF16 operands in shared
// memory, FP32 accumulators in tensor memory, issued by one thread; the
// output layer is an FP32 dot product.  A cell whose
// confidence max(s, 1-s), s = sigmoid(logit), is below the threshold keeps
// the plain flag; otherwise flag 1 for s < 1/2 and max(2, plain flag) for
// s >= 1/2.  Training runs in FP32: per-block forward and backward passes
// with the activations in shared memory, a fixed-order reduction of the
// block gradients, and Adam.
#include "ocfd_fp32.cuh"
#include "ocfd_tma.cuh"

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
// quotient of a feature that only the network reads: exact in FP64 (the
// training features), the two-instruction approximate quotient in FP32 (its
// error, a few units in the last place, is far below the BF16 rounding the
// network's input takes)
template <typename R> __device__ __forceinline__ R feat_div(R a, R b) { return a / b; }
template <> __device__ __forceinline__ float feat_div<float>(float a, float b) { return __fdividef(a, b); }

// The 14 features and the sensor's sum dp of a cell from P = p00 d T and d
// at the cell (P0, D0) and at its minus / plus neighbours along x, y, z
template <typename R>
__device__ __forceinline__ void features_of(R P0, R D0, const R (&Pm)[3], const R (&Pp)[3], const R (&Dm)[3],
                                            const R (&Dp)[3], float f[MLP_IN], R &dp) {
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const R den = Pm[a] + 2*P0 + Pp[a];
        const R t = fabs(-Pm[a] + 2*P0 - Pp[a])/den;    // the sensor's term
        dp = a == 0 ? t : dp + t;
        f[a] = (float)t;
        f[3 + a] = (float)feat_div(Pp[a] - Pm[a], den);
        const R rdd = feat_div((R)1, Dm[a] + 2*D0 + Dp[a]);
        f[6 + a] = (float)(fabs(-Dm[a] + 2*D0 - Dp[a]) * rdd);
        f[9 + a] = (float)((Dp[a] - Dm[a]) * rdd);
    }
    f[12] = f[0] + f[1] + f[2];
    f[13] = f[6] + f[7] + f[8];
}

// om[a], op[a]: offsets of the minus / plus neighbour along direction a
template <typename R>
__device__ __forceinline__ void switch_features(const Params &p, long long c, const long long (&om)[3],
                                                const long long (&op)[3], float f[MLP_IN], R &dp) {
    const R *d = prim_r<R>(p, 0), *T = prim_r<R>(p, 4);
    const R p00 = (R)p.p00;
    auto P = [&](long long o) { return p00 * d[o] * T[o]; };
    R Pm[3], Pp[3], Dm[3], Dp[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        Pm[a] = P(c + om[a]); Pp[a] = P(c + op[a]);
        Dm[a] = d[c + om[a]]; Dp[a] = d[c + op[a]];
    }
    features_of<R>(P(c), d[c], Pm, Pp, Dm, Dp, f, dp);
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
// tensor-core MLP of one block (tcgen05): 128 rows of standardised features
// in, 128 logits out, thread t holding row t.  The block's features are
// written as the A operand of the first product in shared memory, one
// thread issues tcgen05.mma into a 128 x 32 FP32 accumulator in tensor
// memory (TMEM lane t = row t), each warp reads its 32 lanes back with
// tcgen05.ld, and the ReLU'd hidden layer goes back to shared memory as the
// A operand of the second product (two K = 16 steps).  The weights sit in
// shared memory as the B operands for the whole launch.
// ---------------------------------------------------------------------------
namespace umma {

constexpr int ROWS = 128;             // rows per product: the MMA's M, one TMEM lane each
constexpr unsigned TMEM_COLS = 32;    // the accumulator's columns (N = 32, FP32)
// kind::f16 instruction descriptor: D FP32 (bits 4-5 = 1), A and B BF16
// (bits 7-9 = 1, 10-12 = 1), both K-major (bits 15, 16 = 0), N >> 3 at
// bits 17-22, M >> 4 at bits 24-28
constexpr unsigned IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(MLP_H >> 3) << 17) |
                           ((unsigned)(ROWS >> 4) << 24);

// Element offset of (row, k) in a K-major BF16 operand of K = 16 without
// swizzling: core matrices of 8 rows x 8 elements (128 contiguous bytes,
// 16 per row), the two K halves of an 8-row group 128 B apart (the
// descriptor's leading byte offset), 8-row groups 256 B apart (its stride
// byte offset).
__host__ __device__ constexpr int cm(int row, int k) {
    return (row >> 3) * 128 + (k >> 3) * 64 + (row & 7) * 8 + (k & 7);
}
constexpr unsigned LBO = 128, SBO = 256;

struct __align__(128) Smem {
    __nv_bfloat16 w1[MLP_H * 16];         // B of layer 1: row n = W1[n][0..13], 0, 0
    __nv_bfloat16 w2[2][MLP_H * 16];      // B of layer 2, K steps 0..15 and 16..31
    __nv_bfloat16 a1[ROWS * 16];          // A of layer 1: the standardised features
    __nv_bfloat16 a2[2][ROWS * 16];       // A of layer 2: the hidden layer, K steps
    float b1[MLP_H], b2[MLP_H], w3[MLP_H], mu[16], isg[16];
    unsigned long long bar;               // completion of the block's products
    float b3;
    unsigned tmem;                        // TMEM address of the accumulator
};
static_assert(sizeof(Smem) < 16384, "one block's shared memory");

// shared-memory matrix descriptor: start address, leading and stride byte
// offsets (all >> 4), version 1 (bits 46-47), no swizzle (bits 61-63 = 0)
__device__ __forceinline__ unsigned long long desc(const void *ptr) {
    const unsigned a = tma::smem_u32(ptr);
    return (unsigned long long)((a >> 4) & 0x3FFFu) | ((unsigned long long)(LBO >> 4) << 16) |
           ((unsigned long long)(SBO >> 4) << 32) | (1ull << 46);
}
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// D (+)= A B over K = 16, issued by one thread
__device__ __forceinline__ void mma(unsigned tmem_d, unsigned long long a, unsigned long long b, bool accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(tmem_d), "l"(a), "l"(b), "r"(IDESC), "r"((unsigned)accumulate)
        : "memory");
}
// one arrival on bar once the products this thread issued are complete
__device__ __forceinline__ void commit(unsigned long long *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     tma::smem_u32(bar))
                 : "memory");
}
// this warp's 32 lanes x 32 columns of the accumulator (thread = lane = row)
__device__ __forceinline__ void load_row(unsigned taddr, float (&v)[32]) {
    unsigned r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int c = 0; c < 32; c++) v[c] = __uint_as_float(r[c]);
}

__device__ __forceinline__ unsigned pack_bf16(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<unsigned *>(&v);
}

// The block's set-up: weights into shared memory as B operands, the
// standardisation constants, the mbarrier, and 32 TMEM columns (warp 0).
// Every thread of the 128-thread block calls it.
__device__ void setup(Smem &s, const float *__restrict__ w) {
    const int t = threadIdx.x;
    for (int q = t; q < MLP_H * 16; q += ROWS) {          // B[k][n] = W1[n][k]
        const int n = q >> 4, k = q & 15;
        s.w1[cm(n, k)] = __float2bfloat16_rn(k < MLP_IN ? w[OFF_W1 + n * MLP_IN + k] : 0.0f);
    }
    for (int q = t; q < MLP_H * MLP_H; q += ROWS) {       // B[k][n] = W2[n][k]
        const int n = q >> 5, k = q & 31;
        s.w2[k >> 4][cm(n, k & 15)] = __float2bfloat16_rn(w[OFF_W2 + n * MLP_H + k]);
    }
    if (t < MLP_H) { s.b1[t] = w[OFF_B1 + t]; s.b2[t] = w[OFF_B2 + t]; s.w3[t] = w[OFF_W3 + t]; }
    if (t < 16) {
        s.mu[t] = t < MLP_IN ? w[OFF_MU + t] : 0.0f;
        s.isg[t] = t < MLP_IN ? 1.0f / w[OFF_SG + t] : 0.0f;
    }
    if (t == 0) {
        s.b3 = w[OFF_B3];
        tma::mbar_init(&s.bar, 1);
        tma::fence_mbar_init();
    }
    if (t < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         tma::smem_u32(&s.tmem)), "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_async_smem();
    before_sync();
    __syncthreads();
    after_sync();
}

// The block's teardown: a product still outstanding after a wait ran out is
// waited for once more (bounded; phase has moved past the parity that ran
// out), then warp 0 frees the TMEM columns.
__device__ void teardown(Smem &s, bool good, unsigned phase) {
    if (!__syncthreads_and(good) && threadIdx.x == 0) tma::mbar_wait(&s.bar, phase ^ 1u);
    before_sync();
    __syncthreads();
    after_sync();
    if (threadIdx.x < 32)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(s.tmem), "r"(TMEM_COLS)
                     : "memory");
}

// The network on the block's 128 rows.  x: this thread's standardised
// features.  good: this thread's last wait completed; phase: the mbarrier
// parity to wait for next.  Returns false for every thread of the block
// once a wait has run out (the block then stops), else this row's logit in z.
__device__ bool mlp(Smem &s, const float (&x)[MLP_IN], bool &good, unsigned &phase, float &z) {
    const int t = threadIdx.x;
    const unsigned trow = s.tmem + ((unsigned)(t & ~31) << 16);    // this warp's TMEM lanes
    uint4 c0, c1;
    c0.x = pack_bf16(x[0], x[1]);   c0.y = pack_bf16(x[2], x[3]);
    c0.z = pack_bf16(x[4], x[5]);   c0.w = pack_bf16(x[6], x[7]);
    c1.x = pack_bf16(x[8], x[9]);   c1.y = pack_bf16(x[10], x[11]);
    c1.z = pack_bf16(x[12], x[13]); c1.w = 0u;
    *reinterpret_cast<uint4 *>(s.a1 + cm(t, 0)) = c0;
    *reinterpret_cast<uint4 *>(s.a1 + cm(t, 8)) = c1;
    fence_async_smem();
    before_sync();
    if (!__syncthreads_and(good)) return false;
    after_sync();
    // layer 1: Z1 = X W1^T
    if (t == 0) {
        mma(s.tmem, desc(s.a1), desc(s.w1), false);
        commit(&s.bar);
    }
    good = tma::mbar_wait(&s.bar, phase);
    phase ^= 1u;
    after_sync();
    float v[32];
    load_row(trow, v);
    // ReLU(Z1 + b1) as BF16, hidden units 0..15 into K step 0, 16..31 into step 1
#pragma unroll
    for (int ks = 0; ks < 2; ks++)
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int u = ks * 16 + h * 8;
            uint4 c;
            c.x = pack_bf16(fmaxf(v[u + 0] + s.b1[u + 0], 0.0f), fmaxf(v[u + 1] + s.b1[u + 1], 0.0f));
            c.y = pack_bf16(fmaxf(v[u + 2] + s.b1[u + 2], 0.0f), fmaxf(v[u + 3] + s.b1[u + 3], 0.0f));
            c.z = pack_bf16(fmaxf(v[u + 4] + s.b1[u + 4], 0.0f), fmaxf(v[u + 5] + s.b1[u + 5], 0.0f));
            c.w = pack_bf16(fmaxf(v[u + 6] + s.b1[u + 6], 0.0f), fmaxf(v[u + 7] + s.b1[u + 7], 0.0f));
            *reinterpret_cast<uint4 *>(s.a2[ks] + cm(t, h * 8)) = c;
        }
    fence_async_smem();
    before_sync();
    if (!__syncthreads_and(good)) return false;
    after_sync();
    // layer 2: Z2 = H W2^T over two K steps
    if (t == 0) {
        mma(s.tmem, desc(s.a2[0]), desc(s.w2[0]), false);
        mma(s.tmem, desc(s.a2[1]), desc(s.w2[1]), true);
        commit(&s.bar);
    }
    good = tma::mbar_wait(&s.bar, phase);
    phase ^= 1u;
    after_sync();
    load_row(trow, v);
    // output layer in FP32
    float acc = s.b3;
#pragma unroll
    for (int c = 0; c < 32; c++) acc += fmaxf(v[c] + s.b2[c], 0.0f) * s.w3[c];
    z = acc;
    return true;
}

}  // namespace umma

// (f - mu) / sigma, as a product with the block's reciprocals of sigma
__device__ __forceinline__ void standardise(const umma::Smem &s, const float (&f)[MLP_IN], float (&x)[MLP_IN]) {
#pragma unroll
    for (int m = 0; m < MLP_IN; m++) x[m] = (f[m] - s.mu[m]) * s.isg[m];
}

// Logits of n raw feature rows (the network alone, for checks): persistent
// blocks of 128 threads over 128-row tiles.  err: set when a wait ran out.
__global__ void __launch_bounds__(umma::ROWS) k_mlp_infer(const float *__restrict__ w, const float *__restrict__ feat,
                                                          long long n, float *logit, int *err) {
    __shared__ umma::Smem s;
    umma::setup(s, w);
    bool good = true;
    unsigned phase = 0;
    const long long ntile = (n + umma::ROWS - 1) / umma::ROWS;
    for (long long tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
        const long long row = tile * umma::ROWS + threadIdx.x;
        float f[MLP_IN], x[MLP_IN];
#pragma unroll
        for (int m = 0; m < MLP_IN; m++) f[m] = row < n ? feat[row * MLP_IN + m] : 0.0f;
        standardise(s, f, x);
        float z;
        if (!umma::mlp(s, x, good, phase, z)) break;
        if (row < n) logit[row] = z;
    }
    if (!good) atomicExch(err, 2);
    umma::teardown(s, good, phase);
}

// The learned switch over the extended box: cell (i, j, k), each of -1 ..
// n-1, owns entry i+1 of the x array (when j, k are interior), entry j+1 of
// the y array and entry k+1 of the z array.  conf_logit = ln(c / (1 - c))
// for confidence threshold c.  stats (optional): cells decided by the
// network, cells left to the plain flag, network flags that differ from the
// plain flag.  A block covers a 32 x 4 tile of (i, j) -- the 128 rows of one
// product -- and marches along z through a segment of planes: P and d of
// the column's planes k-1, k, k+1 stay in registers, the x and y neighbours
// come through L1 from the rows the block's own warps load.
constexpr int SWX = 32, SWY = umma::ROWS / SWX;
template <typename R>
__global__ void __launch_bounds__(umma::ROWS) k_switch_infer(Params p, const float *__restrict__ w, float conf_logit,
                                                             unsigned long long *stats, int seg) {
    __shared__ umma::Smem s;
    umma::setup(s, w);
    const int lane = threadIdx.x & 31;
    const int ex = p.nx + 1, ey = p.ny + 1, ez = p.nz + 1;
    const int ntx = (ex + SWX - 1) / SWX;
    const int i = (int)(blockIdx.x % ntx) * SWX + (int)(threadIdx.x % SWX) - 1;
    const int j = (int)(blockIdx.x / ntx) * SWY + (int)(threadIdx.x / SWX) - 1;
    const int ka = (int)blockIdx.y * seg - 1, kb = min(ez - 1, ka + seg);   // planes ka .. kb-1
    const bool any = i < ex - 1 && j < ey - 1;          // a cell of the extended box
    const R *d = prim_r<R>(p, 0), *T = prim_r<R>(p, 4);
    const R p00 = (R)p.p00;
    auto P = [&](long long o) { return p00 * d[o] * T[o]; };
    long long c = any ? lap_index(p, i + OCFD_LAP, j + OCFD_LAP, ka + OCFD_LAP) : 0;
    R Pz0 = (R)0, Pz1 = (R)0, Dz0 = (R)0, Dz1 = (R)0;
    if (any) { Pz0 = P(c - p.zs); Pz1 = P(c); Dz0 = d[c - p.zs]; Dz1 = d[c]; }
    unsigned long long n_sure = 0, n_unsure = 0, n_differ = 0;
    unsigned nx1 = 0, ny1 = 0, nz1 = 0;
    bool good = true;
    unsigned phase = 0;
    for (int k = ka; k < kb; k++, c += p.zs) {
        float f[MLP_IN] = {};
        R dp = (R)0;
        if (any) {
            R Pm[3], Pp[3], Dm[3], Dp[3];
            Pm[0] = P(c - 1);      Pp[0] = P(c + 1);      Dm[0] = d[c - 1];      Dp[0] = d[c + 1];
            Pm[1] = P(c - p.ys);   Pp[1] = P(c + p.ys);   Dm[1] = d[c - p.ys];   Dp[1] = d[c + p.ys];
            Pm[2] = Pz0;           Pp[2] = P(c + p.zs);   Dm[2] = Dz0;           Dp[2] = d[c + p.zs];
            features_of<R>(Pz1, Dz1, Pm, Pp, Dm, Dp, f, dp);
            Pz0 = Pz1; Pz1 = Pp[2]; Dz0 = Dz1; Dz1 = Dp[2];
        }
        float x[MLP_IN];
        standardise(s, f, x);
        float z;
        if (!umma::mlp(s, x, good, phase, z)) break;
        const int plain = plain_flag(p, dp);
        const bool sure = fabsf(z) >= conf_logit;
        const int kp = sure ? (z >= 0.0f ? max(2, plain) : 1) : plain;
        const bool inx = any && j >= 0 && k >= 0, iny = any && i >= 0 && k >= 0, inz = any && i >= 0 && j >= 0;
        if (inx) p.flag[0][(long long)(i + 1) + (long long)ex * ((long long)j + (long long)p.ny * k)] = (int8_t)kp;
        if (iny) p.flag[1][(long long)i + (long long)p.nx * ((long long)(j + 1) + (long long)ey * k)] = (int8_t)kp;
        if (inz) p.flag[2][(long long)i + (long long)p.nx * ((long long)j + (long long)p.ny * (k + 1))] = (int8_t)kp;
        const bool non1 = kp != 1;
        nx1 += non1 && inx; ny1 += non1 && iny; nz1 += non1 && inz;
        if (stats) {
            const unsigned ms = __ballot_sync(0xffffffffu, any && sure), mu = __ballot_sync(0xffffffffu, any && !sure),
                           md = __ballot_sync(0xffffffffu, any && sure && kp != plain);
            n_sure += __popc(ms); n_unsure += __popc(mu); n_differ += __popc(md);
        }
    }
    if (stats && lane == 0 && (n_sure | n_unsure | n_differ)) {
        atomicAdd(stats + 0, n_sure);
        atomicAdd(stats + 1, n_unsure);
        atomicAdd(stats + 2, n_differ);
    }
    // faces per direction whose flag is not 1: one sum per warp for the
    // whole segment
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
    if (!good && p.kerr) atomicExch(p.kerr, 2);
    umma::teardown(s, good, phase);
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

// Persistent blocks: as many as fit on the SMs at once (registers, shared
// memory, threads; 32 TMEM columns each, so at most 16 by tensor memory), at
// most one per tile.  Counted from the kernel's attributes: the runtime's
// occupancy query gave one block per SM for these kernels, which left 4
// warps per SM to hide the feature loads.
template <typename K>
static unsigned resident_blocks(K kern, long long tiles) {
    int dev = 0, sms = 148, regs_sm = 65536, smem_sm = 233472, smem_rsv = 1024, thr_sm = 2048;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&smem_rsv, cudaDevAttrReservedSharedMemoryPerBlock, dev);
    cudaDeviceGetAttribute(&thr_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev);
    int per = 1;
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, reinterpret_cast<const void *>(kern)) == cudaSuccess) {
        const int regs = (fa.numRegs + 7) / 8 * 8;
        const int by_regs = regs_sm / (umma::ROWS * (regs > 0 ? regs : 1));
        const int by_smem = smem_sm / ((int)fa.sharedSizeBytes + smem_rsv);
        const int by_thr = thr_sm / umma::ROWS;
        per = by_regs < by_smem ? by_regs : by_smem;
        if (per > by_thr) per = by_thr;
        if (per > (int)(512 / umma::TMEM_COLS)) per = (int)(512 / umma::TMEM_COLS);
        if (per < 1) per = 1;
    } else {
        cudaGetLastError();
    }
    const long long nb = (long long)sms * per;
    return (unsigned)(tiles < nb ? tiles : nb);
}

cudaError_t launch_switch_infer(const Params &p, const float *w, float conf_logit, unsigned long long *stats,
                                cudaStream_t st) {
    if (p.flag_count) {
        cudaError_t e = cudaMemsetAsync(p.flag_count, 0, 3 * sizeof(unsigned), st);
        if (e != cudaSuccess) return e;
    }
    // tiles of the extended box's (i, j), z split into as many segments as
    // keep the grid within one wave of resident blocks
    const int ntiles = ((p.nx + 1 + SWX - 1) / SWX) * ((p.ny + 1 + SWY - 1) / SWY);
    const int ez = p.nz + 1;
    const long long want = p.mixed ? resident_blocks(k_switch_infer<float>, 1LL << 40)
                                   : resident_blocks(k_switch_infer<double>, 1LL << 40);
    int nseg = (int)(want / ntiles);
    if (nseg > ez) nseg = ez;
    if (nseg < 1) nseg = 1;
    const int seg = (ez + nseg - 1) / nseg;
    nseg = (ez + seg - 1) / seg;
    const dim3 grid((unsigned)ntiles, (unsigned)nseg);
    if (p.mixed) k_switch_infer<float><<<grid, umma::ROWS, 0, st>>>(p, w, conf_logit, stats, seg);
    else         k_switch_infer<double><<<grid, umma::ROWS, 0, st>>>(p, w, conf_logit, stats, seg);
    return cudaGetLastError();
}

cudaError_t launch_mlp_infer(const float *w, const float *feat, long long n, float *logit, int *err, cudaStream_t st) {
    const long long tiles = (n + umma::ROWS - 1) / umma::ROWS;
    k_mlp_infer<<<resident_blocks(k_mlp_infer, tiles), umma::ROWS, 0, st>>>(w, feat, n, logit, err);
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
