"""The precision form (FP32 split / projection / reconstruction / sensor /
viscous stencils, FP64 conserved state and RK3 update) against the FP64
path, which is itself pinned to the oracle.  The bounds below come from the
first measurements on these cases (relative L2 per conserved variable after
ten steps, about 1e-6), with a margin of 20x."""
import numpy as np
import pytest

from ocfd_b200 import cases, lib

pytestmark = pytest.mark.gpu

TOL_FP32_10STEPS = 2e-5


def rel_l2(a, b):
    """Per variable; the three momentum (or velocity) components against the
    norm of the whole vector, since one of them may start at zero."""
    vec = np.sqrt(sum(np.linalg.norm(b[m]) ** 2 for m in (1, 2, 3)))
    return np.array([np.linalg.norm(a[m] - b[m]) / (vec if m in (1, 2, 3) else np.linalg.norm(b[m]))
                     for m in range(len(b))])


@pytest.mark.parametrize("maker", [
    lambda: cases.isotropic_turbulence(24, seed=9, charteric=1),
    lambda: cases.isotropic_turbulence(24, seed=9, charteric=1, hy_dp_intv=(1e-4, 0.05)),
    lambda: cases.taylor_green(24, seed=3),
    lambda: cases.random_smooth_case(17, 18, 13, seed=65, scheme_invis="SCHEME_HYBRIDAUTO", charteric=1,
                                     shock=True, curvilinear=True),
], ids=["iso_hybrid_char", "iso_hybrid_char_weno", "tgv_weno7", "curv_hybrid_char_shock"])
def test_fp32_form_tracks_fp64(maker, gpu_lib):
    case = maker()
    a = lib.Solver(case.cfg, case.prims, case.metrics)
    b = lib.Solver(case.cfg, case.prims, case.metrics)
    b.set_precision(1)
    a.step(10)
    b.step(10)
    err = rel_l2(b.conserved(), a.conserved())
    assert np.all(np.isfinite(err)) and np.all(err > 0), err       # it does compute in FP32
    assert np.all(err <= TOL_FP32_10STEPS), err
    ep = rel_l2(b.primitives(), a.primitives())
    assert np.all(ep <= TOL_FP32_10STEPS), ep


def test_precision_switch_round_trip(gpu_lib):
    """FP64 -> FP32 -> FP64 within one run: the FP64 steps after the switch
    back start from the FP64 primitives of the conserved state."""
    case = cases.isotropic_turbulence(16, seed=12, charteric=1)
    a = lib.Solver(case.cfg, case.prims, case.metrics)
    a.step(2)
    a.set_precision(1)
    a.step(2)
    u_mid = a.conserved()
    a.set_precision(0)
    a.step(2)
    b = lib.Solver(case.cfg, case.prims, case.metrics)
    b.step(2)
    b.set_precision(1)
    b.step(2)
    assert np.array_equal(b.conserved(), u_mid)
    b.set_precision(0)
    b.step(2)
    assert np.array_equal(a.conserved(), b.conserved())
    # the per-stage API needs the FP64 form
    b.set_precision(1)
    with pytest.raises(lib.OcfdError) as ei:
        b.du_comput(1)
    assert ei.value.status == -2


def test_precision_form_refuses_uncovered(gpu_lib):
    """Schemes outside the FP32 walks (here UP7 alone) are refused."""
    case = cases.random_smooth_case(12, 11, 10, seed=21, scheme_invis="UP7", shock=True)
    s = lib.Solver(case.cfg, case.prims, case.metrics, inlet=case.inlet)
    with pytest.raises(lib.OcfdError) as ei:
        s.set_precision(1)
    assert ei.value.status == -2


@pytest.mark.parametrize("maker", [
    lambda: cases.ramp_case(30, 18, 8, seed=66),
    lambda: cases.ramp_case(30, 18, 8, seed=67, tw=-1.0, epsl=0.01, beta=0.5, mtmax=4),
], ids=["ramp_bc108_tw_filter", "ramp_bc108_adiabatic_blowing_filter"])
def test_fp32_form_tracks_fp64_on_the_ramp(maker, gpu_lib):
    """The compression ramp (metrics from the mesh, closures in x and y,
    IBC 108 inflow, top and wall, the shock filter every step) in the
    precision form against the FP64 path after ten steps: the boundary
    values are formed in FP64, the filter weights from the FP32 pressure."""
    case = maker()
    a = lib.Solver(case.cfg, case.prims, case.metrics, inlet=case.inlet)
    b = lib.Solver(case.cfg, case.prims, case.metrics, inlet=case.inlet)
    b.set_precision(1)
    a.step(10)
    b.step(10)
    err = rel_l2(b.conserved(), a.conserved())
    print("ramp FP32 vs FP64 rel L2 after 10 steps:", err)
    assert np.all(np.isfinite(err)) and np.all(err > 0), err
    assert np.all(err <= TOL_FP32_10STEPS), err
    ep = rel_l2(b.primitives(), a.primitives())
    assert np.all(ep <= TOL_FP32_10STEPS), ep
    # the wall rows carry the boundary law exactly: no slip, T = Tw
    pb = b.primitives()
    assert np.all(pb[1][:, 0, :] == 0.0) and np.all(pb[3][:, 0, :] == 0.0)
    if case.cfg.bc_rpara[0] > 0:
        assert np.allclose(pb[4][:, 0, :], case.cfg.bc_rpara[0], rtol=1e-14)
