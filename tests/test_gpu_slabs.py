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
