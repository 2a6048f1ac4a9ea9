"""The grid split in z on one GPU: a single slab whose neighbour below and
above is itself.  Its z ghost planes then come through the whole exchange
path -- the pack kernel, an NCCL group of two sends and two receives, the
unpack kernel -- instead of the periodic wrap, and every result must equal
the single-GPU run bit for bit: the ghost values are the same copies, so
any plane sent to the wrong side, any field missed, or any fill that the
split path skips shows as a difference.  Runs with more than one GPU use the
same kernels with other neighbour ranks (one GPU per process)."""
import numpy as np
import pytest

from ocfd_b200 import cases, lib, slabs

pytestmark = pytest.mark.gpu


def _pair(case, prep=None, **kw):
    a = lib.Solver(case.cfg, case.prims, case.metrics, inlet=case.inlet, **kw)
    run = slabs.SlabRun(case, 0, 1, lib.slab_unique_id(), **kw)
    b = run.solver
    if prep:
        prep(a)
        prep(b)
    return a, b


def _same(a, b):
    assert np.array_equal(a.conserved(), b.conserved())
    assert np.array_equal(a.primitives(), b.primitives())


@pytest.mark.parametrize("name", ["tgv_weno7", "iso_hybrid", "iso_hybrid_fp32", "iso_hybrid_impl5", "curvilinear",
                                  "ramp_bc_filter"])
def test_one_slab_equals_single_gpu(name, gpu_lib):
    prep = None
    steps = 4
    if name == "tgv_weno7":
        c = cases.taylor_green(16, seed=3)
    elif name.startswith("iso_hybrid"):
        c = cases.isotropic_turbulence(24, seed=9, charteric=1, hy_dp_intv=(0.002, 0.02))
        if name.endswith("fp32"):
            prep = lambda s: s.set_precision(1)
        elif name.endswith("impl5"):         # all three sweeps launched together
            prep = lambda s: s.set_sweep_impl(5)
    elif name == "curvilinear":
        c = cases.random_smooth_case(20, 16, 12, seed=5, curvilinear=True, shock=True)
    else:
        c = cases.ramp_case(48, 24, 12, seed=4)
        steps = 3
    a, b = _pair(c, prep)
    a.step(steps)
    b.step(steps)
    _same(a, b)
    if c.cfg.scheme_invis == "SCHEME_HYBRIDAUTO":
        for fa, fb in zip(a.flags(), b.flags()):
            assert np.array_equal(fa, fb)
        assert np.array_equal(a.scheme_proportion(), b.scheme_proportion())
    for which in (0, 1):
        assert a.ana_residual(which) == b.ana_residual(which)
    assert a.check_state() == b.check_state()


def test_one_slab_mesh_metrics_equal(gpu_lib):
    """Metrics from mesh coordinates with JAC_BOUND closures in every
    direction: the coordinate and metric ghost planes come through the
    exchange, and the single slab is both the first and the last."""
    c = cases.ramp_case(40, 20, 12, seed=6)
    a, b = _pair(c)
    assert np.array_equal(a.metrics(), b.metrics())


def test_set_slab_order_and_arguments(gpu_lib):
    c = cases.taylor_green(16, seed=3)
    s = lib.Solver(c.cfg, c.prims, c.metrics)
    spec = slabs.slab_spec(0, 1, c.cfg.nz, lib.slab_unique_id())
    with pytest.raises(lib.OcfdError):           # after the metrics and state
        s._check(s.L.ocfd_b200_set_slab(s.h, 1, 0, 0, 0, 0, c.cfg.nz, spec.comm_id), "set_slab")
    bad = slabs.SlabSpec(1, 0, 0, 0, 0, c.cfg.nz - 1, spec.comm_id)       # slab beyond the grid
    with pytest.raises(lib.OcfdError):
        lib.Solver(c.cfg, None, None, slab=bad)
    cp = cases.random_smooth_case(12, 10, 12, seed=2, iperiodic=(1, 1, 0))
    with pytest.raises(lib.OcfdError):           # z must be periodic
        lib.Solver(cp.cfg, None, None, slab=slabs.slab_spec(0, 1, 12, spec.comm_id))


def _distinct_worker(rank, world, port, name, steps, outdir):
    """One slab process; all share GPU 0 and exchange through host memory."""
    import os
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    from datetime import timedelta
    import numpy as np
    import torch.distributed as dist
    from ocfd_b200 import slabs
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        case, prep = _distinct_case(name, world)
        run = slabs.SlabRun(case, rank, world, None, device=0)
        if prep:
            prep(run.solver)
        run.solver.step(steps)
        np.save(os.path.join(outdir, f"u{rank}.npy"), run.solver.conserved())
        res = [run.solver.ana_residual(0), run.solver.ana_residual(1), run.solver.check_state()]
        np.save(os.path.join(outdir, f"r{rank}.npy"), np.array([res[0], res[1], *res[2]], dtype=np.float64))
        if case.cfg.scheme_invis == "SCHEME_HYBRIDAUTO":
            for d, f in zip("xyz", run.solver.flags()):
                np.save(os.path.join(outdir, f"f{d}{rank}.npy"), f)
        run.close()
    finally:
        dist.barrier()
        dist.destroy_process_group()


def _distinct_case(name, world):
    n = 12
    if name == "tgv_weno7":
        return cases.random_smooth_case(n, n, n * world, seed=3, scheme_invis="WENO7"), None
    if name.startswith("iso_hybrid"):
        c = cases.random_smooth_case(n, n, n * world, seed=9, scheme_invis="SCHEME_HYBRIDAUTO", charteric=1,
                                     shock=True)
        c.cfg.hy_dp_intv = (0.01, 0.2)
        if "edge" not in name:
            # the plane below each slab boundary three times as hot: there
            # the sensor takes flag 3 on both sides of the split (below)
            for z0, _ in slabs.part_z(n * world, world)[1:]:
                c.prims[4][z0 - 1] *= 3.0
        return c, ((lambda s: s.set_precision(1)) if "fp32" in name else None)
    c = cases.random_smooth_case(n, n + 2, n * world, seed=5, curvilinear=True, shock=True)
    return c, None


def _run_distinct(name, world, steps, tmp_path):
    import socket
    import torch.multiprocessing as mp
    s = socket.socket(); s.bind(("127.0.0.1", 0)); port = s.getsockname()[1]; s.close()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_distinct_worker, args=(r, world, port, name, steps, str(tmp_path)))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0


def _slab_flags(tmp_path, d, world):
    return [np.load(tmp_path / f"f{d}{r}.npy") for r in range(world)]


@pytest.mark.parametrize("name,world", [("tgv_weno7", 2), ("iso_hybrid", 3), ("iso_hybrid_fp32", 2),
                                        ("curvilinear", 3)])
def test_distinct_slabs_equal_single_gpu(name, world, gpu_lib, tmp_path):
    """2 or 3 slab processes on one GPU, each with its own z slab of an
    n x n x (n world) grid and its neighbours' ghost planes through host
    memory (slabs.HostTransport over gloo): the gathered state equals the
    single-GPU run of the whole grid bit for bit, and the reductions summed
    over the slabs equal the whole grid's to 1e-15.  An error in which planes
    a slab packs, sends to which side, or unpacks where, would show.

    With the hybrid scheme the split changes the sensor on the plane below
    each slab (its corner cells are zero, test_slab_sensor_edge_lines); the
    hybrid case heats that plane so that its flags are 3 either way, and the
    flags of the last step's sensor pass must then match the whole grid's."""
    steps = 3
    case, prep = _distinct_case(name, world)
    a = lib.Solver(case.cfg, case.prims, case.metrics)
    if prep:
        prep(a)
    a.step(steps)
    want = a.conserved()
    want_r = [a.ana_residual(0), a.ana_residual(1), *a.check_state()]
    _run_distinct(name, world, steps, tmp_path)
    if case.cfg.scheme_invis == "SCHEME_HYBRIDAUTO":
        fx, fy, fz = a.flags()
        assert np.array_equal(np.concatenate(_slab_flags(tmp_path, "x", world)), fx)
        assert np.array_equal(np.concatenate(_slab_flags(tmp_path, "y", world)), fy)
        for (z0, nzl), f in zip(slabs.part_z(case.cfg.nz, world), _slab_flags(tmp_path, "z", world)):
            assert np.array_equal(f, fz[z0:z0 + nzl + 1]), z0
    got = np.concatenate([np.load(tmp_path / f"u{r}.npy") for r in range(world)], axis=1)
    assert np.array_equal(got, want), np.abs(got - want).max()
    for r in range(world):
        rr = np.load(tmp_path / f"r{r}.npy")
        assert abs(rr[0] - want_r[0]) <= 1e-15 * abs(want_r[0]) and abs(rr[1] - want_r[1]) <= 1e-15 * abs(want_r[1])
        assert rr[2] == want_r[2] and rr[3] == want_r[3]
        assert abs(rr[4] - want_r[4]) <= 1e-15 * abs(want_r[4])


def _jameson_ghost_plane(cfg, prims, g):
    """Flags of the Jameson sensor (src/OCFD_Schemes_hybrid_auto.cu:611-703)
    for the cells of global plane g as a slab whose first plane is g + 1
    sees them: in its z ghost plane, whose x and y neighbours outside the
    interior are corner cells that no exchange fills, zero since init()
    (src/OCFD_init.cu:37-41; the x, y and z exchanges of
    src/OCFD_mpi_dev.cu:186-310 carry the interior of a plane only)."""
    d, T = prims[0], prims[4]
    nz = d.shape[0]
    P = (1.0 / (cfg.gamma * cfg.ama * cfg.ama)) * d * T
    P0 = P[g]
    zero = np.zeros_like(P0)

    def term(m, q):
        return np.abs(-m + 2 * P0 - q) / (m + 2 * P0 + q)
    xm = np.concatenate([zero[:, :1], P0[:, :-1]], axis=1)
    xp = np.concatenate([P0[:, 1:], zero[:, :1]], axis=1)
    ym = np.concatenate([zero[:1], P0[:-1]], axis=0)
    yp = np.concatenate([P0[1:], zero[:1]], axis=0)
    dp0 = term(xm, xp) + term(ym, yp) + term(P[(g - 1) % nz], P[(g + 1) % nz])
    lo, hi = cfg.hy_dp_intv
    return (1 + (dp0 > lo) + (dp0 > hi)).astype(np.int8)


def test_slab_sensor_edge_lines(gpu_lib, tmp_path):
    """The sensor pass of a split grid, as the reference's own decomposition
    has it: a slab's z flags of its own cells equal the whole grid's, and
    its lowest entry -- the cell just below the slab, in its ghost plane --
    equals the whole grid's away from the edge lines of the plane and, on
    them, the sensor with the plane's corner cells at zero."""
    world = 3
    case, _ = _distinct_case("iso_hybrid_edge", world)
    a = lib.Solver(case.cfg, case.prims, case.metrics)
    a.step(1)
    fz = a.flags()[2]
    _run_distinct("iso_hybrid_edge", world, 1, tmp_path)
    edge = np.zeros(fz.shape[1:], dtype=bool)
    edge[0] = edge[-1] = True
    edge[:, 0] = edge[:, -1] = True
    changed = 0
    for (z0, nzl), f in zip(slabs.part_z(case.cfg.nz, world), _slab_flags(tmp_path, "z", world)):
        assert np.array_equal(f[1:], fz[z0 + 1:z0 + nzl + 1]), z0
        if z0 == 0:             # the whole grid's own lower ghost plane: the same cells
            assert np.array_equal(f[0], fz[0])
            continue
        assert np.array_equal(f[0][~edge], fz[z0][~edge]), z0
        want = _jameson_ghost_plane(case.cfg, case.prims, z0 - 1)
        assert np.array_equal(f[0][edge], want[edge]), z0
        changed += int(np.count_nonzero(f[0][edge] != fz[z0][edge]))
    assert changed > 0          # the case does reach the difference
