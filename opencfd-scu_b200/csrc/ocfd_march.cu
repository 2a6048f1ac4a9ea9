// ocfd_march.cu -- the UP7 walk of the y and z sweeps as per-lane marches
// over TMA-staged pencil tiles (sm_100a; FP64, and FP32 for the precision form).
//
// Same results as the UP7 walk of ocfd_sweep3.cu (the reference's
// OCFD_d{y,z}1/2 chain with the hybrid scheme's UP7 faces, src/OCFD_Schemes.cu:159-381,
// 865-907): every split point and face flux formed once, du in the
// reference's y+, y- (z+, z-) order, one writer per element.
//
// Organisation.  A warp owns 32 consecutive x columns of one z (y sweep) or
// y (z sweep) and a segment of the line; each lane walks its own column.
// The primitives of the pencil (32 columns x 8 points x 5 fields) arrive in
// shared memory by one 4-D bulk tensor copy per chunk, double-buffered per
// warp behind an mbarrier, so the loads of the next chunk run while the
// lane computes.  The lane keeps the split values of the last 8 points in
// registers (the window of the face it forms next); the 8-point chunk is
// unrolled, so a point's window slot is a compile-time index and nothing is
// shifted.  No shared-memory window reads remain (the ring walk reads 70
// per face), and no block barrier is taken.
//
// Faces that are not plain UP7 (hybrid flags other than 1, faces within
// reach of a boundary closure) defer the cells on both sides, and the first
// and last cells of a bounded line, to the same per-direction lists the
// ring walk uses; the fix-up kernel recomputes them.
#include "ocfd_tma.cuh"
#include "ocfd_walk.cuh"

#include <cudaTypedefs.h>

#include <mutex>

namespace ocfd {

cudaError_t launch_sweep3_fix(const Params &p, int dir, cudaStream_t st);
cudaError_t launch_sweep4_fix(const Params &p, int dir, cudaStream_t st);

namespace {

using namespace walk;

constexpr int MW = 4;          // warps per block
constexpr int CH = 8;          // points per staged chunk (the window length)
using namespace tma;

template <typename R>
constexpr int chunk_elems() { return 5 * CH * 32; }     // [field][point][column]

// DIR: 1 (y) or 2 (z).  tm: the primitives the stencils read as a 4-D
// tensor [x: row pitch][y: LAP rows][z: LAP planes][field: 5], box
// 32 x CH x 1 x 5 (y) or 32 x 1 x CH x 5 (z).
template <int DIR, bool UNI, bool EPS0, typename R>
__global__ void __launch_bounds__(32 * MW, sizeof(R) == 8 ? 2 : 3)
k_march(const __grid_constant__ Params p, const __grid_constant__ CUtensorMap tm, int seg_len) {
    static_assert(DIR == 1 || DIR == 2, "the march covers the y and z sweeps");
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ unsigned long long bars[MW][2];
    constexpr int CE = chunk_elems<R>();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int ngx = (p.nx + 31) / 32;
    const int n3 = DIR == 1 ? p.nz : p.ny;
    const long long grp = (long long)blockIdx.x * MW + wid;
    if (grp >= (long long)ngx * n3) return;                   // the whole warp
    R *buf = reinterpret_cast<R *>(smem_raw) + (size_t)wid * 2 * CE;
    unsigned long long *bar = bars[wid];

    const int g = (int)(grp % ngx), c3 = (int)(grp / ngx);
    const int x = g * 32 + lane;
    const bool colok = x < p.nx;
    const int xs = colok ? x : p.nx - 1;                      // keep addresses in range
    const int n = DIR == 1 ? p.ny : p.nz;
    const int y0 = blockIdx.y * seg_len;
    const int y1 = min(n, y0 + seg_len);
    long long base, sd, cb, cst, fst;
    const int8_t *fl;
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
    R *__restrict__ du = du_r<R>(p);
    const long long N = p.N;
    const bool hybrid = p.scheme_invis == 310;
    const R h = (R)(DIR == 1 ? p.hy : p.hz), ih = (R)p.inv_h[DIR];

    // points P0 .. y1+3 in chunks of CH; point P sits in window slot (P - P0) % CH
    const int P0 = y0 - 4;
    const int nch = (y1 - y0 + 8 + CH - 1) / CH;
    if (lane == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_mbar_init();
    }
    __syncwarp();
    auto issue = [&](int c) {           // lane 0: chunk c into buffer c % 2
        const int b = c & 1;
        mbar_expect_tx(&bar[b], (unsigned)(CE * sizeof(R)));
        const int cx = OCFD_LAP + g * 32, cp = OCFD_LAP + P0 + c * CH, cq = OCFD_LAP + c3;
        if (DIR == 1) load_4d(buf + b * CE, &tm, cx, cp, cq, 0, &bar[b]);
        else          load_4d(buf + b * CE, &tm, cx, cq, cp, 0, &bar[b]);
    };
    if (lane == 0) {
        issue(0);
        if (nch > 1) issue(1);
    }

    // flag of face F+1/2 is entry F+1: chunk c, slot t holds face F = P - 4,
    // entry P0 + c*CH + t - 3, used when y0 <= entry <= y1
    auto load_flags = [&](int c, int (&hf)[CH]) {
#pragma unroll
        for (int t = 0; t < CH; t++) {
            const int e = P0 + c * CH + t - 3;
            hf[t] = (hybrid && colok && e >= y0 && e <= y1) ? flag_at(p, DIR, fl, (long long)e * fst) : 2;
        }
    };
    // the chunk's flags, one byte each (flags are small integers)
    auto pack = [](const int (&hf)[CH]) {
        unsigned long long v = 0;
#pragma unroll
        for (int t = 0; t < CH; t++) v |= (unsigned long long)(hf[t] & 0xff) << (8 * t);
        return v;
    };
    int hn[CH];
    load_flags(0, hn);
    unsigned long long hpk = pack(hn);

    R wp[CH][5], wm[CH][5];             // split values of the window's points
    R prv[10];
#pragma unroll
    for (int m = 0; m < 10; m++) prv[m] = (R)0.0;
#pragma unroll
    for (int t = 0; t < CH; t++)
#pragma unroll
        for (int m = 0; m < 5; m++) { wp[t][m] = (R)0.0; wm[t][m] = (R)0.0; }
    int prv_slow = 0;
    unsigned phase = 0;                 // bit b: parity of buffer b's next phase

    for (int c = 0; c < nch; c++) {
        const int b = c & 1;
        if (c + 1 < nch) load_flags(c + 1, hn);
        {
            long long it = 0;
            while (!mbar_try_wait(&bar[b], (phase >> b) & 1u)) {
                if (++it > WAIT_LIMIT) {
                    if (lane == 0) atomicExch(p.kerr, 1);
                    // the other buffer's copy, if one is in flight, lands
                    // before the block's shared memory goes away
                    if (c + 1 < nch) {
                        long long it2 = 0;
                        while (!mbar_try_wait(&bar[b ^ 1], (phase >> (b ^ 1)) & 1u) && ++it2 <= WAIT_LIMIT) {}
                    }
                    return;
                }
            }
            phase ^= 1u << b;
        }
        const R *cbuf = buf + b * CE;
#pragma unroll
        for (int t = 0; t < CH; t++) {
            const int P = P0 + c * CH + t;
            if (P <= y1 + 3) {
                const int F = P - 4;
                // du of the next step's cell into L1 now, so that its read
                // after this step's faces does not wait on DRAM
                if (colok && F + 1 >= y0 && F + 1 < y1) {
                    const R *q = du + cb + (long long)(F + 1) * cst;
#pragma unroll
                    for (int m = 0; m < 5; m++) prefetch_l1(q + m * N);
                }
                // this step's cell: its du is read before the faces are formed
                R old[5];
                if (colok && F >= y0) {
#pragma unroll
                    for (int m = 0; m < 5; m++) old[m] = du[m * N + cb + (long long)F * cst];
                }
                // + sign of face F+1/2: points F-3 .. F+3 (slots t+1 .. t+7)
                R cur[10];
#pragma unroll
                for (int m = 0; m < 5; m++) {
                    R v[8];
#pragma unroll
                    for (int k = 0; k < 7; k++) v[k] = wp[(t + 1 + k) & (CH - 1)][m];
                    v[7] = (R)0.0;
                    cur[m] = up7_p_q(v);
                }
                // the split of point P into slot t (whose point P-8 is done)
                {
                    R q[5];
#pragma unroll
                    for (int m = 0; m < 5; m++) q[m] = cbuf[(m * CH + t) * 32 + lane];
                    split_point<DIR, UNI, EPS0>(p, base + (long long)P * sd, q[0], q[1], q[2], q[3], q[4],
                                                wp[t], wm[t]);
                }
                if (F >= y0 - 1) {
                    // - sign of face F+1/2: points F-2 .. F+4 (slots t+2 .. t+8)
#pragma unroll
                    for (int m = 0; m < 5; m++) {
                        R v[8];
                        v[0] = (R)0.0;
#pragma unroll
                        for (int k = 1; k < 8; k++) v[k] = wm[(t + 1 + k) & (CH - 1)][m];
                        cur[5 + m] = up7_m_q(v);
                    }
                    const int hflag = (int)(signed char)((hpk >> (8 * t)) & 0xff);
                    const int slow = !up7_face(p, hflag) || near_closure(p, DIR, F, n);
                    if (F >= y0) {               // cell F: faces F-1/2 (prv) and F+1/2 (cur)
                        bool defer = colok && (slow || prv_slow);
                        if (p.has_bnd) defer = defer || (colok && rule_cell(p, DIR, F, n));
                        const long long ci = OCFD_IDX(p, cb + (long long)F * cst, N);
                        const unsigned mask = __ballot_sync(FULL, defer);
                        if (mask) {              // one atomic per warp
                            const int leader = __ffs(mask) - 1;
                            unsigned slot = 0;
                            if (lane == leader) slot = atomicAdd(p.defer_count + DIR, (unsigned)__popc(mask));
                            slot = __shfl_sync(FULL, slot, leader);
                            if (defer) p.defer[DIR][OCFD_IDX(p, (long long)slot + __popc(mask & ((1u << lane) - 1u)), p.N)] = (unsigned)ci;
                        }
                        if (colok && !defer) {
                            const R aj = (R)metric<UNI>(p, M_AJAC, base + (long long)F * sd);
                            add_du<false>(du, N, ci, aj, h, ih, cur, prv, old);
                        }
                    }
#pragma unroll
                    for (int m = 0; m < 10; m++) prv[m] = cur[m];
                    prv_slow = slow;
                }
            }
        }
        __syncwarp();                    // every lane is done with buffer b
        if (lane == 0 && c + 2 < nch) issue(c + 2);
        if (c + 1 < nch) hpk = pack(hn);
    }
}

// ---------------------------------------------------------------------------
// host side: tensor maps and launches
// ---------------------------------------------------------------------------

template <typename R>
constexpr size_t smem_bytes() { return (size_t)MW * 2 * chunk_elems<R>() * sizeof(R); }

template <int DIR, bool UNI, bool EPS0, typename R>
cudaError_t set_smem() {
    return cudaFuncSetAttribute(k_march<DIR, UNI, EPS0, R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)smem_bytes<R>());
}

template <int DIR, bool UNI, bool EPS0, typename R>
cudaError_t launch_one(const Params &p, const CUtensorMap &tm, cudaStream_t st) {
    const int ngx = (p.nx + 31) / 32;
    const int n3 = DIR == 1 ? p.nz : p.ny;
    const int n = DIR == 1 ? p.ny : p.nz;
    const long long groups = (long long)ngx * n3;
    // segments of a line, so that there are about three waves of warps; a
    // segment re-splits 7 points
    constexpr int BLOCKS_PER_SM = sizeof(R) == 8 ? 2 : 3;
    const long long want = 3LL * 148 * BLOCKS_PER_SM * MW;
    long long nseg = (want + groups - 1) / groups;
    const long long maxseg = n / 32 > 0 ? n / 32 : 1;
    if (nseg > maxseg) nseg = maxseg;
    if (nseg < 1) nseg = 1;
    int seg_len = (int)((n + nseg - 1) / nseg);
    nseg = (n + seg_len - 1) / seg_len;
    const size_t smem = smem_bytes<R>();
    dim3 grid((unsigned)((groups + MW - 1) / MW), (unsigned)nseg);
    k_march<DIR, UNI, EPS0, R><<<grid, 32 * MW, smem, st>>>(p, tm, seg_len);
    return cudaGetLastError();
}

template <bool UNI, bool EPS0, typename R>
cudaError_t launch_dir_t(const Params &p, const CUtensorMap &tm, int dir, cudaStream_t st) {
    return dir == 1 ? launch_one<1, UNI, EPS0, R>(p, tm, st) : launch_one<2, UNI, EPS0, R>(p, tm, st);
}

}  // namespace

// The dynamic shared-memory size of every instance, set on the current
// device before the first launch (and before any stream capture).
cudaError_t march_prepare() {
    cudaError_t e = cudaSuccess;
    auto one = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
    one(set_smem<1, true, true, double>());  one(set_smem<2, true, true, double>());
    one(set_smem<1, true, false, double>()); one(set_smem<2, true, false, double>());
    one(set_smem<1, false, false, double>()); one(set_smem<2, false, false, double>());
    one(set_smem<1, true, true, float>());   one(set_smem<2, true, true, float>());
    one(set_smem<1, true, false, float>());  one(set_smem<2, true, false, float>());
    one(set_smem<1, false, false, float>()); one(set_smem<2, false, false, float>());
    return e;
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *ptr = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &ptr, 12000, cudaEnableDefault, &q) ==
                cudaSuccess && q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(ptr);
        else
            cudaGetLastError();
    });
    return fn;
}

bool encode_map_4d(const void *base, int elem_bytes, const unsigned long long dims[4],
                   const unsigned long long strides[3], const unsigned box[4], CUtensorMap *out) {
    PFN_cuTensorMapEncodeTiled_v12000 fn = encode_fn();
    if (!fn || !base || ((unsigned long long)base & 15)) return false;
    for (int i = 0; i < 3; i++)
        if (strides[i] % 16) return false;
    if (((unsigned long long)box[0] * elem_bytes) % 16) return false;
    cuuint64_t d[4] = { dims[0], dims[1], dims[2], dims[3] };
    cuuint64_t st[3] = { strides[0], strides[1], strides[2] };
    cuuint32_t bx[4] = { box[0], box[1], box[2], box[3] };
    cuuint32_t estr[4] = { 1, 1, 1, 1 };
    CUresult r = fn(out, elem_bytes == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4,
                    const_cast<void *>(base), d, st, bx, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// A 4-D tensor map over five LAP-box fields that start at base, field
// stride lapN elements: dims [pitch, ny + 2 LAP, nz + 2 LAP, 5], box
// 32 x CH x 1 x 5 along y (dir 1) or 32 x 1 x CH x 5 along z (dir 2).
bool march_tensor_map(const Params &p, const void *base, int elem_bytes, int dir, CUtensorMap *out) {
    if (dir != 1 && dir != 2) return false;
    const unsigned long long eb = (unsigned long long)elem_bytes;
    const unsigned long long dims[4] = { (unsigned long long)p.ys, (unsigned long long)(p.ny + 2 * OCFD_LAP),
                                         (unsigned long long)(p.nz + 2 * OCFD_LAP), 5 };
    const unsigned long long strides[3] = { p.ys * eb, p.zs * eb, p.lapN * eb };
    const unsigned box[4] = { 32, dir == 1 ? (unsigned)CH : 1u, dir == 2 ? (unsigned)CH : 1u, 5 };
    return encode_map_4d(base, elem_bytes, dims, strides, box, out);
}

// The march covers the UP7 walk's schemes (the hybrid scheme, UP7 without
// projection) on the y and z sweeps.
bool march_supported(const Params &p, int dir) {
    const bool fast_scheme = (p.scheme_invis == 301 && !p.charteric) || p.scheme_invis == 310;
    return (dir == 1 || dir == 2) && fast_scheme && p.defer[0] != nullptr && p.kerr != nullptr;
}

// one direction: the march, then the fix-up of its deferred cells (the
// caller clears the deferred counters once per stage, as for the ring walk)
cudaError_t launch_march_dir(const Params &p, const CUtensorMap &tm, int dir, cudaStream_t st) {
    cudaError_t e;
    if (p.mixed) {
        e = p.uniform_metrics ? (p.epsl_sw == 0.0 ? launch_dir_t<true, true, float>(p, tm, dir, st)
                                                  : launch_dir_t<true, false, float>(p, tm, dir, st))
                              : launch_dir_t<false, false, float>(p, tm, dir, st);
        if (e != cudaSuccess) return e;
        return launch_sweep4_fix(p, dir, st);
    }
    e = p.uniform_metrics ? (p.epsl_sw == 0.0 ? launch_dir_t<true, true, double>(p, tm, dir, st)
                                              : launch_dir_t<true, false, double>(p, tm, dir, st))
                          : launch_dir_t<false, false, double>(p, tm, dir, st);
    if (e != cudaSuccess) return e;
    return launch_sweep3_fix(p, dir, st);
}

}  // namespace ocfd
