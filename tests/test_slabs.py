"""Host side of the grid split in z (ocfd_b200/slabs.py), on CPU: the
reference's z decomposition and neighbour ranks, cutting a case into slabs,
and the two host exchanges of a z-split run over gloo ranks (world size 2 and
3): the communicator id from rank 0, and slab results gathered into the whole
grid on rank 0."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from ocfd_b200 import cases, lib, slabs


def _reference_offsets(NZ, NPZ0):
    """k_offset / k_nn as part3d forms them (src/OCFD_mpi.c:157-165)."""
    off, nn = [], []
    for k in range(NPZ0):
        ka = min(k, NZ % NPZ0)
        off.append(NZ // NPZ0 * k + ka)
        nn.append(NZ // NPZ0 + (1 if k < NZ % NPZ0 else 0))
    return off, nn


@pytest.mark.parametrize("nz,nr", [(64, 1), (64, 2), (64, 8), (65, 8), (513, 7), (24, 5), (4, 4)])
def test_part_z_is_the_reference_rule(nz, nr):
    parts = slabs.part_z(nz, nr)
    off, nn = _reference_offsets(nz, nr)
    assert [p[0] for p in parts] == off and [p[1] for p in parts] == nn
    assert parts[0][0] == 0 and sum(p[1] for p in parts) == nz
    for a, b in zip(parts, parts[1:]):
        assert a[0] + a[1] == b[0]


def test_part_z_rejects_too_many_slabs():
    with pytest.raises(ValueError):
        slabs.part_z(3, 4)


def test_neighbours_wrap():
    assert slabs.neighbours(0, 1) == (0, 0)
    assert slabs.neighbours(0, 2) == (1, 1)
    assert slabs.neighbours(0, 4) == (3, 1)
    assert slabs.neighbours(3, 4) == (2, 0)


def test_slab_spec_fields():
    s = slabs.slab_spec(2, 3, 65, bytes(128))
    assert (s.rank_lo, s.rank_hi, s.z_offset, s.nz_global) == (1, 0, 44, 65)


def test_slab_cases_reassemble_the_grid():
    c = cases.random_smooth_case(12, 10, 22, seed=3, curvilinear=True)
    parts = slabs.part_z(c.cfg.nz, 3)
    subs = [slabs.slab_case(c, z0, nz) for z0, nz in parts]
    for s, (z0, nz) in zip(subs, parts):
        assert s.cfg.nz == nz and (s.cfg.nx, s.cfg.ny) == (c.cfg.nx, c.cfg.ny)
        assert s.prims[0].shape == (nz, c.cfg.ny, c.cfg.nx)
        assert s.cfg.dt == c.cfg.dt and s.cfg.scheme_invis == c.cfg.scheme_invis
    for m in range(5):
        assert np.array_equal(np.concatenate([s.prims[m] for s in subs]), c.prims[m])
    for m in range(len(c.metrics)):
        assert np.array_equal(np.concatenate([s.metrics[m] for s in subs]), c.metrics[m])


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    from datetime import timedelta
    import numpy as np
    import torch.distributed as dist
    from ocfd_b200 import cases, slabs
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        made = []

        def make():
            made.append(rank)
            return bytes((7 * i + 3) % 256 for i in range(128))

        cid = slabs.share_id(make)
        c = cases.random_smooth_case(8, 6, 4 * world + 1, seed=11)
        spec = slabs.slab_spec(rank, world, c.cfg.nz, cid)
        nz = slabs.part_z(c.cfg.nz, world)[rank][1]
        sub = slabs.slab_case(c, spec.z_offset, nz)
        # a slab result: the 5 fields of this slab (stand-in for conserved())
        whole = slabs.gather_z(np.stack(sub.prims), rank, world)
        ok_gather = whole is None if rank else np.array_equal(whole, np.stack(c.prims))
        q.put((rank, cid, made, spec.rank_lo, spec.rank_hi, ok_gather))
    finally:
        dist.barrier()
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_id_from_rank0_and_gather_over_gloo(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want = bytes((7 * i + 3) % 256 for i in range(128))
    for rank, cid, made, lo, hi, ok in res:
        assert cid == want
        assert made == ([0] if rank == 0 else [])      # only rank 0 makes the id
        assert (lo, hi) == slabs.neighbours(rank, world)
        assert ok


def _transport_worker(rank, world, port, q):
    """The host transport's two operations as the library calls them, on
    host buffers: the ghost-plane swap (each rank's lowest planes to the
    rank below, highest to the rank above) and the in-place sums."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    from datetime import timedelta
    import ctypes
    import numpy as np
    import torch.distributed as dist
    from ocfd_b200 import slabs
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        lo, hi = slabs.neighbours(rank, world)
        t = slabs.HostTransport(rank, lo, hi)
        count = 5
        send = np.concatenate([np.full(count, 100.0 * rank + 1.0), np.full(count, 100.0 * rank + 2.0)])
        recv = np.zeros(2 * count)
        rc = t.fn(None, 0, send.ctypes.data, recv.ctypes.data, count, 0)
        ok_swap = (rc == 0 and np.all(recv[:count] == 100.0 * lo + 2.0)      # the lower rank's highest planes
                   and np.all(recv[count:] == 100.0 * hi + 1.0))             # the upper rank's lowest planes
        f32 = np.full(2 * count, rank, dtype=np.float32)
        r32 = np.zeros(2 * count, dtype=np.float32)
        ok_f32 = t.fn(None, 0, f32.ctypes.data, r32.ctypes.data, count, 3) == 0 and \
            np.all(r32[:count] == lo) and np.all(r32[count:] == hi)
        acc = np.array([rank + 0.5, 2.0 * rank])
        c64 = np.array([rank + 1, 10], dtype=np.uint64)
        c32 = np.array([rank, 3, 7], dtype=np.uint32)
        ok_sum = (t.fn(None, 1, acc.ctypes.data, acc.ctypes.data, 2, 0) == 0 and
                  t.fn(None, 1, c64.ctypes.data, c64.ctypes.data, 2, 1) == 0 and
                  t.fn(None, 1, c32.ctypes.data, c32.ctypes.data, 3, 2) == 0)
        n = world
        ok_sum = ok_sum and np.allclose(acc, [n * (n - 1) / 2 + 0.5 * n, n * (n - 1)]) and \
            list(c64) == [n * (n + 1) // 2, 10 * n] and list(c32) == [n * (n - 1) // 2, 3 * n, 7 * n]
        q.put((rank, bool(ok_swap), bool(ok_f32), bool(ok_sum)))
    finally:
        dist.barrier()
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [1, 2, 3])
def test_host_transport_over_gloo(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_transport_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ok_swap, ok_f32, ok_sum in res:
        assert ok_swap and ok_f32 and ok_sum, (rank, ok_swap, ok_f32, ok_sum)
