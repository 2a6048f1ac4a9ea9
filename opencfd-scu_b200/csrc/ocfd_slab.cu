// ocfd_slab.cu -- the grid split in z across GPUs (one z slab per rank), with
// the ghost exchange between slabs over NCCL (sm_100a).
//
// Replaces the z part of the reference's halo exchange,
// exchange_boundary_z_packed_dev (src/OCFD_mpi_dev.cu:271-310): there the
// LAP planes next to each slab face are packed on the device, copied to the
// host, swapped with MPI_Sendrecv between ID_ZM1 and ID_ZP1
// (src/OCFD_mpi.c:183-189) and copied back.  Here the packed planes stay in
// HBM and go straight from GPU to GPU: one pack kernel for all fields and
// both faces, one NCCL group of two sends and two receives (NVLink /
// NVSwitch between the GPUs of a node), one unpack kernel.  As in the
// reference, only the interior (x, y) part of each ghost plane is carried;
// the x and y ghosts of a slab are its own periodic wraps.
//
// NCCL is opened at run time (dlopen of libnccl.so.2; in a process that has
// imported torch this is torch's own copy), so the library loads and runs
// single-GPU without it.  A host transport can stand in for NCCL
// (ocfd_b200_set_slab_host): the packed planes then go through pinned host
// memory and a caller's function, as the reference's MPI_Sendrecv does --
// for ranks without NCCL between their GPUs, and for tests that run several
// slabs on one GPU (each process's kernels then never wait on another's).  The reductions of the analysis step
// (ana_residual, src/OCFD_ana.cu:76-105, an MPI_Allreduce there) go through
// the same communicator.
#include "ocfd_device.cuh"

#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nccl.h>

#include <cstring>
#include <string>

namespace ocfd {

namespace {

struct NcclApi {
    bool ok = false;
    std::string err;
    ncclResult_t (*GetUniqueId)(ncclUniqueId *) = nullptr;
    ncclResult_t (*CommInitRank)(ncclComm_t *, int, ncclUniqueId, int) = nullptr;
    ncclResult_t (*CommDestroy)(ncclComm_t) = nullptr;
    ncclResult_t (*GroupStart)() = nullptr;
    ncclResult_t (*GroupEnd)() = nullptr;
    ncclResult_t (*Send)(const void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*Recv)(void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*AllReduce)(const void *, void *, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                              cudaStream_t) = nullptr;
    const char *(*GetErrorString)(ncclResult_t) = nullptr;
};

const NcclApi &nccl() {
    static NcclApi api = [] {
        NcclApi a;
        void *h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
        if (!h) h = dlopen("libnccl.so", RTLD_NOW | RTLD_GLOBAL);
        if (!h) { a.err = std::string("NCCL not found: ") + dlerror(); return a; }
        auto sym = [&](const char *name) { return dlsym(h, name); };
        a.GetUniqueId = (decltype(a.GetUniqueId))sym("ncclGetUniqueId");
        a.CommInitRank = (decltype(a.CommInitRank))sym("ncclCommInitRank");
        a.CommDestroy = (decltype(a.CommDestroy))sym("ncclCommDestroy");
        a.GroupStart = (decltype(a.GroupStart))sym("ncclGroupStart");
        a.GroupEnd = (decltype(a.GroupEnd))sym("ncclGroupEnd");
        a.Send = (decltype(a.Send))sym("ncclSend");
        a.Recv = (decltype(a.Recv))sym("ncclRecv");
        a.AllReduce = (decltype(a.AllReduce))sym("ncclAllReduce");
        a.GetErrorString = (decltype(a.GetErrorString))sym("ncclGetErrorString");
        a.ok = a.GetUniqueId && a.CommInitRank && a.CommDestroy && a.GroupStart && a.GroupEnd && a.Send &&
               a.Recv && a.AllReduce && a.GetErrorString;
        if (!a.ok) a.err = "NCCL library lacks the point-to-point or all-reduce entry points";
        return a;
    }();
    return api;
}

std::string nccl_msg(const char *what, ncclResult_t r) {
    const NcclApi &a = nccl();
    return std::string(what) + ": " + (a.GetErrorString ? a.GetErrorString(r) : "NCCL error");
}

constexpr int MAXF = 13;

template <typename T> struct PlaneList { T *f[MAXF]; int n; };

// send buffer [side][field][plane][y][x]: side 0 = the L lowest interior
// planes (for the neighbour below), side 1 = the L highest (for the one above)
template <typename T>
__global__ void k_halo_pack(Params p, PlaneList<T> g, T *__restrict__ send) {
    const int L = OCFD_LAP;
    const long long plane = (long long)p.nx * p.ny;
    const long long per_side = (long long)g.n * L * plane;
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= 2 * per_side) return;
    const int side = (int)(tid / per_side);
    long long q = tid - side * per_side;
    const int fi = (int)(q / (L * plane));
    q -= (long long)fi * L * plane;
    const int l = (int)(q / plane);
    q -= (long long)l * plane;
    const int j = (int)(q / p.nx), i = (int)(q - (long long)j * p.nx);
    const int k = side == 0 ? L + l : p.nz + l;            // LAP index of the source plane
    send[tid] = g.f[fi][lap_index(p, i + L, j + L, k)];
}

// receive buffer [side][field][plane][y][x]: side 0 from the neighbour below
// (its highest planes) into ghost planes 0..L-1, side 1 from the neighbour
// above (its lowest planes) into nz+L..nz+2L-1
template <typename T>
__global__ void k_halo_unpack(Params p, PlaneList<T> g, const T *__restrict__ recv) {
    const int L = OCFD_LAP;
    const long long plane = (long long)p.nx * p.ny;
    const long long per_side = (long long)g.n * L * plane;
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= 2 * per_side) return;
    const int side = (int)(tid / per_side);
    long long q = tid - side * per_side;
    const int fi = (int)(q / (L * plane));
    q -= (long long)fi * L * plane;
    const int l = (int)(q / plane);
    q -= (long long)l * plane;
    const int j = (int)(q / p.nx), i = (int)(q - (long long)j * p.nx);
    const int k = side == 0 ? l : p.nz + L + l;
    g.f[fi][lap_index(p, i + L, j + L, k)] = recv[tid];
}

template <typename T> ncclDataType_t nccl_type();
template <> ncclDataType_t nccl_type<double>() { return ncclFloat64; }
template <> ncclDataType_t nccl_type<float>() { return ncclFloat32; }

}  // namespace

struct Slab {
    ncclComm_t comm = nullptr;
    int nranks = 1, rank = 0, lo = 0, hi = 0;
    unsigned char *buf = nullptr;   // send (2 sides) then receive (2 sides)
    size_t side_bytes = 0;          // MAXF FP64 fields x L planes
    // host transport (instead of NCCL): the caller's function and its
    // pinned staging copy of buf
    SlabTransport fn = nullptr;
    void *user = nullptr;
    unsigned char *hbuf = nullptr;
};

int slab_unique_id(unsigned char id[128], std::string &err) {
    const NcclApi &a = nccl();
    if (!a.ok) { err = a.err; return -1; }
    static_assert(sizeof(ncclUniqueId) == 128, "NCCL unique id is 128 bytes");
    ncclUniqueId u;
    ncclResult_t r = a.GetUniqueId(&u);
    if (r != ncclSuccess) { err = nccl_msg("ncclGetUniqueId", r); return -1; }
    memcpy(id, &u, sizeof(u));
    return 0;
}

Slab *slab_create(const Params &p, int nranks, int rank, int lo, int hi, const unsigned char id[128],
                  std::string &err) {
    const NcclApi &a = nccl();
    if (!a.ok) { err = a.err; return nullptr; }
    Slab *s = new Slab();
    s->nranks = nranks; s->rank = rank; s->lo = lo; s->hi = hi;
    s->side_bytes = sizeof(double) * (size_t)MAXF * OCFD_LAP * (size_t)p.nx * p.ny;
    cudaError_t e = cudaMalloc(&s->buf, 4 * s->side_bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        err = std::string("cudaMalloc(slab exchange buffers): ") + cudaGetErrorString(e);
        delete s;
        return nullptr;
    }
    ncclUniqueId u;
    memcpy(&u, id, sizeof(u));
    ncclResult_t r = a.CommInitRank(&s->comm, nranks, u, rank);
    if (r != ncclSuccess) {
        err = nccl_msg("ncclCommInitRank", r);
        cudaFree(s->buf);
        delete s;
        return nullptr;
    }
    return s;
}

Slab *slab_create_host(const Params &p, int nranks, int rank, int lo, int hi, SlabTransport fn, void *user,
                       std::string &err) {
    Slab *s = new Slab();
    s->nranks = nranks; s->rank = rank; s->lo = lo; s->hi = hi;
    s->fn = fn; s->user = user;
    s->side_bytes = sizeof(double) * (size_t)MAXF * OCFD_LAP * (size_t)p.nx * p.ny;
    cudaError_t e = cudaMalloc(&s->buf, 4 * s->side_bytes);
    if (e == cudaSuccess) e = cudaHostAlloc((void **)&s->hbuf, 4 * s->side_bytes, cudaHostAllocDefault);
    if (e != cudaSuccess) {
        cudaGetLastError();
        err = std::string("slab exchange buffers: ") + cudaGetErrorString(e);
        cudaFree(s->buf);
        delete s;
        return nullptr;
    }
    return s;
}

void slab_destroy(Slab *s) {
    if (!s) return;
    if (s->comm) nccl().CommDestroy(s->comm);
    cudaFree(s->buf);
    if (s->hbuf) cudaFreeHost(s->hbuf);
    delete s;
}

// the packed planes (or a reduction buffer) through the host transport:
// device -> pinned host, the caller's function, pinned host -> device
static int host_round_trip(Slab *s, int op, const void *dsend, void *drecv, size_t count, size_t elem, int type,
                           cudaStream_t st, std::string &err) {
    const size_t nsend = (op == 0 ? 2 : 1) * count * elem;
    unsigned char *hs = s->hbuf, *hr = op == 0 ? s->hbuf + 2 * s->side_bytes : s->hbuf;
    cudaError_t e = cudaMemcpyAsync(hs, dsend, nsend, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) { err = std::string("host transport staging: ") + cudaGetErrorString(e); return -1; }
    if (s->fn(s->user, op, hs, hr, count, type) != 0) { err = "host transport: the caller's function failed"; return -1; }
    e = cudaMemcpyAsync(drecv, hr, nsend, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) { err = std::string("host transport staging: ") + cudaGetErrorString(e); return -1; }
    return 0;
}

template <typename T>
static int exchange_t(Slab *s, const Params &p, T *const *f, int nf, cudaStream_t st, std::string &err) {
    if (nf <= 0) return 0;
    if (nf > MAXF) { err = "slab exchange: too many fields"; return -1; }
    const NcclApi &a = nccl();
    PlaneList<T> g;
    for (int m = 0; m < nf; m++) g.f[m] = f[m];
    g.n = nf;
    const size_t count = (size_t)nf * OCFD_LAP * (size_t)p.nx * p.ny;       // elements per side
    T *send = reinterpret_cast<T *>(s->buf);
    T *recv = reinterpret_cast<T *>(s->buf + 2 * s->side_bytes);
    const long long total = 2LL * (long long)count;
    const unsigned nb = (unsigned)((total + 255) / 256);
    k_halo_pack<T><<<nb, 256, 0, st>>>(p, g, send);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) { err = std::string("halo pack: ") + cudaGetErrorString(e); return -1; }
    // per peer, sends and receives pair up in the order they are posted:
    // a rank's first send to its upper neighbour (its highest planes) meets
    // that neighbour's first receive from below, and the same for the
    // second pair, also when both neighbours are one rank (2 slabs) or this
    // rank itself (1 slab: the periodic wrap)
    if (s->fn) {
        if (host_round_trip(s, 0, send, recv, count, sizeof(T), sizeof(T) == 8 ? 0 : 3, st, err)) return -1;
        k_halo_unpack<T><<<nb, 256, 0, st>>>(p, g, recv);
        e = cudaGetLastError();
        if (e != cudaSuccess) { err = std::string("halo unpack: ") + cudaGetErrorString(e); return -1; }
        return 0;
    }
    ncclResult_t r = a.GroupStart();
    if (r == ncclSuccess) r = a.Send(send + count, count, nccl_type<T>(), s->hi, s->comm, st);
    if (r == ncclSuccess) r = a.Send(send, count, nccl_type<T>(), s->lo, s->comm, st);
    if (r == ncclSuccess) r = a.Recv(recv, count, nccl_type<T>(), s->lo, s->comm, st);
    if (r == ncclSuccess) r = a.Recv(recv + count, count, nccl_type<T>(), s->hi, s->comm, st);
    ncclResult_t r2 = a.GroupEnd();
    if (r == ncclSuccess) r = r2;
    if (r != ncclSuccess) { err = nccl_msg("slab exchange", r); return -1; }
    k_halo_unpack<T><<<nb, 256, 0, st>>>(p, g, recv);
    e = cudaGetLastError();
    if (e != cudaSuccess) { err = std::string("halo unpack: ") + cudaGetErrorString(e); return -1; }
    return 0;
}

int slab_exchange(Slab *s, const Params &p, double *const *f, int nf, cudaStream_t st, std::string &err) {
    return exchange_t<double>(s, p, f, nf, st, err);
}

int slab_exchange32(Slab *s, const Params &p, float *const *f, int nf, cudaStream_t st, std::string &err) {
    return exchange_t<float>(s, p, f, nf, st, err);
}

// in-place sum over the ranks; type 0 FP64, 1 uint64, 2 uint32
int slab_allreduce(Slab *s, void *buf, size_t count, int type, cudaStream_t st, std::string &err) {
    if (s->fn) {
        const size_t elem = type == 2 ? 4 : 8;
        if (count * elem > 2 * s->side_bytes) { err = "host transport: reduction larger than its buffer"; return -1; }
        return host_round_trip(s, 1, buf, buf, count, elem, type, st, err);
    }
    const ncclDataType_t t = type == 0 ? ncclFloat64 : (type == 1 ? ncclUint64 : ncclUint32);
    ncclResult_t r = nccl().AllReduce(buf, buf, count, t, ncclSum, s->comm, st);
    if (r != ncclSuccess) { err = nccl_msg("ncclAllReduce", r); return -1; }
    return 0;
}

int slab_launches_per_exchange() { return 2; }

}  // namespace ocfd
