"""The grid split in z across GPUs: one z slab per process.

The reference decomposes its grid over MPI ranks (part3d,
src/OCFD_mpi.c:120-190) and swaps ghost planes through host memory
(exchange_boundary_z_packed_dev, src/OCFD_mpi_dev.cu:271-310).  Here each
process holds one z slab on its own GPU; the library swaps the ghost planes
device to device over NCCL inside every ghost fill, and sums the analysis
reductions over the slabs (ocfd_b200_set_slab).  This module is the host
side: the decomposition (the reference's z rule with NPX0 = NPY0 = 1), the
neighbour ranks, cutting a whole-grid case into slabs, handing the
communicator id from rank 0 to the others and gathering slab results.
torch.distributed carries only that host traffic (any backend).

    import torch.distributed as dist
    dist.init_process_group("gloo")           # host plumbing; the slabs talk over NCCL
    run = SlabRun(case, dist.get_rank(), dist.get_world_size(), share_id(), device=local_rank)
    run.solver.step(100)
    u = gather_z(run.solver.conserved(), dist.get_rank(), dist.get_world_size())   # rank 0: whole grid
"""
import ctypes
import dataclasses
from typing import Callable, List, Optional, Tuple

import numpy as np

from . import lib
from .cases import Case


@dataclasses.dataclass(frozen=True)
class SlabSpec:
    """This rank's place in the z split, as ocfd_b200_set_slab takes it."""
    nranks: int
    rank: int
    rank_lo: int          # holds the planes below (ID_ZM1)
    rank_hi: int          # holds the planes above (ID_ZP1)
    z_offset: int         # first global plane of this slab (k_offset)
    nz_global: int
    comm_id: bytes


def part_z(nz_global: int, nranks: int) -> List[Tuple[int, int]]:
    """(first plane, plane count) of every slab: NZ_GLOBAL / NPZ0 planes each,
    one more on the first NZ_GLOBAL % NPZ0 slabs (src/OCFD_mpi.c:126-165)."""
    if nranks < 1 or nz_global < nranks:
        raise ValueError(f"cannot split {nz_global} planes over {nranks} slabs")
    base, rem = divmod(nz_global, nranks)
    return [(base * k + min(k, rem), base + (1 if k < rem else 0)) for k in range(nranks)]


def neighbours(rank: int, nranks: int) -> Tuple[int, int]:
    """Ranks below and above in the periodic z direction
    (ID_ZM1 / ID_ZP1 with my_mod1, src/OCFD_mpi.c:183-189)."""
    return (rank - 1) % nranks, (rank + 1) % nranks


def slab_spec(rank: int, nranks: int, nz_global: int, comm_id: bytes) -> SlabSpec:
    z0, _ = part_z(nz_global, nranks)[rank]
    lo, hi = neighbours(rank, nranks)
    return SlabSpec(nranks, rank, lo, hi, z0, nz_global, bytes(comm_id))


def slab_case(case: Case, z_offset: int, nz: int) -> Case:
    """The part of a whole-grid case on planes z_offset .. z_offset+nz-1."""
    sl = slice(z_offset, z_offset + nz)
    cfg = dataclasses.replace(case.cfg, nz=nz)
    prims = [np.ascontiguousarray(f[sl]) for f in case.prims]
    metrics = [np.ascontiguousarray(m[sl]) for m in case.metrics] if case.metrics is not None else None
    return Case(cfg, prims, metrics, case.description + f" [z {z_offset}..{z_offset + nz - 1}]", case.inlet)


def share_id(make: Callable[[], bytes] = lib.slab_unique_id, group=None) -> bytes:
    """Rank 0 makes the communicator id; every rank returns it."""
    import torch.distributed as dist
    box = [make() if dist.get_rank(group) == 0 else None]
    dist.broadcast_object_list(box, src=0, group=group)
    cid = box[0]
    if not isinstance(cid, (bytes, bytearray)) or len(cid) != lib.SLAB_ID_BYTES:
        raise RuntimeError("communicator id of the wrong size")
    return bytes(cid)


def gather_z(local: np.ndarray, rank: int, nranks: int, group=None, axis: int = -3) -> Optional[np.ndarray]:
    """Whole-grid array on rank 0 from every rank's slab (z is `axis`, the
    third from last in [..., nz, ny, nx]); None elsewhere."""
    import torch.distributed as dist
    parts = [None] * nranks if rank == 0 else None
    dist.gather_object(np.asarray(local), parts, dst=0, group=group)
    if rank != 0:
        return None
    return np.concatenate(parts, axis=axis)


class HostTransport:
    """The z split's exchange carried through host memory by
    torch.distributed point-to-point messages and all-reduce (a backend that
    moves CPU tensors, e.g. gloo), in place of NCCL: what the reference does
    with MPI_Sendrecv (src/OCFD_mpi_dev.cu:271-310).  Each slab process may
    then use any GPU, the same one as its neighbours included; no kernel of
    one process waits on another's.  Messages going up carry tag 1, going
    down tag 0, so that two slabs (the same rank above and below) pair their
    messages correctly."""

    _DT = {0: np.float64, 1: np.uint64, 2: np.uint32, 3: np.float32}
    _CT = {0: ctypes.c_double, 1: ctypes.c_uint64, 2: ctypes.c_uint32, 3: ctypes.c_float}

    def __init__(self, rank: int, rank_lo: int, rank_hi: int, group=None):
        self.rank, self.lo, self.hi, self.group = rank, rank_lo, rank_hi, group
        self.fn = lib.SLAB_TRANSPORT(self._call)
        self.error: Optional[BaseException] = None

    def _array(self, ptr, n, type_):
        return np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(self._CT[type_])), shape=(n,))

    def _call(self, user, op, send, recv, count, type_):
        import torch
        import torch.distributed as dist
        try:
            if op == 0:
                s = self._array(send, 2 * count, type_)
                r = self._array(recv, 2 * count, type_)
                if self.lo == self.rank and self.hi == self.rank:      # one slab: the periodic wrap
                    r[:count] = s[count:]
                    r[count:] = s[:count]
                    return 0
                down, up = torch.from_numpy(s[:count]), torch.from_numpy(s[count:])
                from_lo, from_hi = torch.from_numpy(r[:count]), torch.from_numpy(r[count:])
                reqs = [dist.isend(up, self.hi, group=self.group, tag=1),
                        dist.isend(down, self.lo, group=self.group, tag=0),
                        dist.irecv(from_lo, self.lo, group=self.group, tag=1),
                        dist.irecv(from_hi, self.hi, group=self.group, tag=0)]
                for q in reqs:
                    q.wait()
                return 0
            # op 1: sum over the ranks in place (counts as signed integers of
            # the same width: every sum here is far below 2^31)
            a = self._array(send, count, type_)
            view = {0: np.float64, 1: np.int64, 2: np.int32, 3: np.float32}[type_]
            t = torch.from_numpy(a.view(view))
            dist.all_reduce(t, group=self.group)
            return 0
        except BaseException as e:       # reported by the library as a failed exchange
            self.error = e
            return 1


class SlabRun:
    """One rank's solver on its slab of a whole-grid case.  comm_id: the NCCL
    id (share_id); None: the exchange goes through HostTransport."""

    def __init__(self, case: Case, rank: int, nranks: int, comm_id: Optional[bytes], device: int = 0,
                 group=None, **solver_kw):
        self.spec = slab_spec(rank, nranks, case.cfg.nz, comm_id if comm_id is not None else b"")
        nz = part_z(case.cfg.nz, nranks)[rank][1]
        self.case = slab_case(case, self.spec.z_offset, nz)
        transport = HostTransport(rank, self.spec.rank_lo, self.spec.rank_hi, group) if comm_id is None else None
        self.solver = lib.Solver(self.case.cfg, self.case.prims, self.case.metrics, device=device,
                                 inlet=self.case.inlet, slab=self.spec, transport=transport, **solver_kw)

    def close(self):
        self.solver.close()
