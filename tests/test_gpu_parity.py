"""Parity of the sm_100a library against the CPU oracle and against the
reference build's golden outputs.  All calls go through the C ABI.

Tolerances (relative L2 per variable, FP64):
  * one RHS evaluation (du)            <= 1e-10
    du is a difference of O(1/h) face fluxes; in the low-Mach Taylor-Green
    case the energy RHS cancels by ~1e3 (p0 = 1/(gamma Ma^2) = 71), so FMA
    contraction on the GPU against none in the oracle shows up as ~1e-12
    relative in du while the state itself agrees to ~1e-15
  * trajectories of a few steps        <= 1e-12
  * vs the reference's own outputs     <= 1e-12  (the north-star bound)
"""
import glob
import json
import os

import numpy as np
import pytest

from ocfd_b200 import cases, lib
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "*.npz")))

TOL_RHS = 1e-10
TOL_TRAJ = 1e-12


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    out = []
    for m in range(a.shape[0]):
        den = np.linalg.norm(b[m])
        num = np.linalg.norm(a[m] - b[m])
        out.append(num / den if den > 0 else num)
    return np.array(out)


def small_cases():
    out = [
        ("tgv16_weno7", cases.taylor_green(16, seed=3)),
        ("iso16_hybrid_char", cases.isotropic_turbulence(16, seed=9, charteric=1)),
        ("iso16_hybrid_nochar", cases.isotropic_turbulence(16, seed=9, charteric=0)),
        ("rnd_weno7_curv", cases.random_smooth_case(19, 13, 11, seed=3, curvilinear=True)),
        ("rnd_hybrid_char_shock", cases.random_smooth_case(13, 17, 11, seed=4, scheme_invis="SCHEME_HYBRIDAUTO",
                                                            charteric=1, shock=True, curvilinear=True)),
        ("rnd_weno7_cd8", cases.random_smooth_case(12, 11, 10, seed=22, scheme_vis="CD8")),
    ]
    for sch in ("UP7", "WENO5", "WENO7_SYMBO", "WENO7_SYMBO_LIM", "NND2", "OMP6_HR", "OMP6_LD", "OMP6_CD8"):
        out.append((f"rnd_{sch.lower()}", cases.random_smooth_case(12, 11, 10, seed=21, scheme_invis=sch,
                                                                   shock=True)))
    for sch in ("WENO7_SYMBO", "WENO7_SYMBO_LIM"):
        out.append((f"rnd_{sch.lower()}_char", cases.random_smooth_case(12, 11, 10, seed=23, scheme_invis=sch,
                                                                        charteric=1, shock=True)))
    out.extend(bounded_cases())
    out.append(("mesh_weno7", cases.mesh_case(14, 13, 12, seed=61, scheme_invis="WENO7")))
    c = cases.mesh_case(13, 14, 12, seed=62, scheme_invis="SCHEME_HYBRIDAUTO", charteric=1, shock=True,
                        non_ref=(1, 0, 0, 1, 0, 0))
    c.cfg.hy_dp_intv = (0.01, 0.2)
    out.append(("mesh_hybrid_char", c))
    c = cases.random_smooth_case(17, 18, 13, seed=65, scheme_invis="SCHEME_HYBRIDAUTO", charteric=1, shock=True,
                                 iperiodic=(1, 0, 1), dif_bound=(0, 0, 1, 1, 0, 0))
    c.cfg.hy_dp_intv = (0.01, 0.2)
    c.cfg.filters = (((1, 1, 1, 1, 2, 15, 0, 18, 0, 13, 2), (0.9, 1e-5, 10.0)),
                     ((2, 0, 0, 1, 0, 17, 0, 18, 3, 11, 2), (0.5, 2e-5, 10.0)))
    out.append(("filter_hybrid_char", c))
    out.append(("ramp_bc108", cases.ramp_case(30, 18, 8, seed=66)))
    c = cases.ramp_case(28, 18, 8, seed=67, tw=-1.0, epsl=0.05, beta=40.0, mtmax=3, filters=())
    c.cfg.bc_rpara = (-1.0, 0.05, 4.0, 30.0, 40.0, 0.0, 30.0, 8.0)
    out.append(("ramp_bc108_adiabatic_blowing", c))
    return out


def bounded_cases():
    """Non-periodic directions with boundary closures (DIF_BOUND = 1) and
    non-reflecting faces: both faces closed, or one face of each direction."""
    both = dict(iperiodic=(0, 0, 0), dif_bound=(1, 1, 1, 1, 1, 1))
    one = dict(iperiodic=(0, 0, 0), dif_bound=(1, 0, 0, 1, 1, 0), non_ref=(1, 0, 0, 1, 0, 0))
    out = [
        ("bnd_up7_both", cases.random_smooth_case(14, 13, 12, seed=41, scheme_invis="UP7", **both)),
        ("bnd_up7_one", cases.random_smooth_case(14, 13, 12, seed=42, scheme_invis="UP7", **one)),
        ("bnd_weno7_cd8_one", cases.random_smooth_case(13, 12, 11, seed=43, scheme_vis="CD8", **one)),
        ("bnd_hybrid_char_both", cases.random_smooth_case(13, 14, 12, seed=44, scheme_invis="SCHEME_HYBRIDAUTO",
                                                          charteric=1, shock=True, **both)),
        ("bnd_hybrid_char_one", cases.random_smooth_case(13, 14, 12, seed=45, scheme_invis="SCHEME_HYBRIDAUTO",
                                                         charteric=1, shock=True, **one)),
        ("bnd_symbo_char_one", cases.random_smooth_case(12, 13, 11, seed=46, scheme_invis="WENO7_SYMBO",
                                                        charteric=1, shock=True, **one)),
    ]
    for _, c in out:
        if c.cfg.scheme_invis == "SCHEME_HYBRIDAUTO":
            c.cfg.hy_dp_intv = (0.01, 0.2)
    return out


CASES = small_cases()


@pytest.mark.parametrize("name,case", CASES, ids=[n for n, _ in CASES])
def test_rhs_matches_oracle(name, case, gpu_lib):
    o = Oracle(case.cfg, case.prims, case.metrics, inlet=case.inlet)
    s = lib.Solver(case.cfg, case.prims, case.metrics, inlet=case.inlet)
    o.swap(); s.swap()
    o.du_comput(1)
    s.du_comput(1)
    err = rel_l2(s.du(), o.du())
    assert np.all(err <= TOL_RHS), (name, err)
    if case.cfg.scheme_invis_id == 310:
        for a, b in zip(s.flags(), o.flags()):
            assert np.array_equal(a.astype(np.int32), b), name


@pytest.mark.parametrize("name,case", CASES, ids=[n for n, _ in CASES])
def test_steps_match_oracle(name, case, gpu_lib):
    nsteps = 3
    o = Oracle(case.cfg, case.prims, case.metrics, inlet=case.inlet)
    s = lib.Solver(case.cfg, case.prims, case.metrics, inlet=case.inlet)
    o.step(nsteps)
    s.step(nsteps)
    ep = rel_l2(s.primitives(), o.primitives())
    ec = rel_l2(s.conserved(), o.conserved())
    assert np.all(ep <= TOL_TRAJ), (name, ep)
    assert np.all(ec <= TOL_TRAJ), (name, ec)
    assert s.time()[0] == o.istep == nsteps


def test_per_stage_api_equals_step(gpu_lib):
    case = cases.isotropic_turbulence(16, seed=12, charteric=1)
    a = lib.Solver(case.cfg, case.prims, case.metrics)
    b = lib.Solver(case.cfg, case.prims, case.metrics)
    a.step(2)
    for _ in range(2):
        b.swap()
        for krk in (1, 2, 3):
            b.du_comput(krk)
            b.time_advance(krk)
            b.get_duvwT()
            b.bc()
    assert np.array_equal(a.primitives(), b.primitives())
    assert np.array_equal(a.conserved(), b.conserved())


def test_repeat_runs_bitwise_identical(gpu_lib):
    case = cases.random_smooth_case(13, 17, 11, seed=4, scheme_invis="SCHEME_HYBRIDAUTO",
                                    charteric=1, shock=True, curvilinear=True)
    r = []
    for _ in range(2):
        s = lib.Solver(case.cfg, case.prims, case.metrics)
        s.step(3)
        r.append(s.primitives())
    assert np.array_equal(r[0], r[1])


def _golden_case(path):
    z = np.load(path)
    cfgd = json.loads(str(z["config"]))
    from ocfd_b200.formats import CaseConfig
    cfg = CaseConfig(**{k: (tuple(v) if isinstance(v, list) else v) for k, v in cfgd.items()})
    return z, cfg


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_matches_reference_golden(path, gpu_lib):
    z, cfg = _golden_case(path)
    nsteps = int(z["nsteps"])
    inlet = z["inlet"] if "inlet" in z.files else None
    s = lib.Solver(cfg, list(z["prims_in"]), list(z["metrics"]), inlet=inlet)
    s.step(nsteps)
    got = s.primitives()
    ref = z["out_run0"]
    err = rel_l2(got, ref)
    name = os.path.basename(path)
    assert np.all(err <= TOL_TRAJ), (name, err)


@pytest.mark.parametrize("name,case", bounded_cases(), ids=[n for n, _ in bounded_cases()])
def test_bounded_sweep_variants(name, case, gpu_lib):
    """Cells next to closed faces go through the fix-up kernel (variant 4) or
    the in-loop dispatch (variant 5): same results; a variant number that
    does not exist is refused."""
    a = lib.Solver(case.cfg, case.prims, case.metrics)
    b = lib.Solver(case.cfg, case.prims, case.metrics)
    b.set_sweep_impl(5)
    a.step(2)
    b.step(2)
    assert np.all(rel_l2(a.primitives(), b.primitives()) <= 1e-13), name
    for bad in (0, 2, 9):
        with pytest.raises(lib.OcfdError) as ei:
            a.set_sweep_impl(bad)
        assert ei.value.status == -1


def _walk4_supported(cfg):
    return (cfg.scheme_invis == "SCHEME_HYBRIDAUTO" and cfg.charteric) or \
           (cfg.scheme_invis == "WENO7" and not cfg.charteric)


@pytest.mark.parametrize("name,case", CASES, ids=[n for n, _ in CASES])
def test_inline_walk_matches_dispatch(name, case, gpu_lib):
    """Variant 6 forms every face of the characteristic hybrid scheme and of
    WENO7 inside the walk (closures and first/last-cell rules included);
    variant 5 sends them through the out-of-line face routine.  Same
    arithmetic, so the same state after two steps to the last bits; any other
    scheme is refused."""
    a = lib.Solver(case.cfg, case.prims, case.metrics, inlet=case.inlet)
    a.set_sweep_impl(6)
    if not _walk4_supported(case.cfg):
        with pytest.raises(lib.OcfdError) as ei:
            a.step(1)
        assert ei.value.status == -2
        return
    b = lib.Solver(case.cfg, case.prims, case.metrics, inlet=case.inlet)
    b.set_sweep_impl(5)
    a.step(2)
    b.step(2)
    assert np.all(rel_l2(a.primitives(), b.primitives()) <= 1e-14), name


def _march_cases():
    """Hybrid-scheme cases for the UP7 walk: periodic boxes (x narrower than
    a warp, odd sizes, x wider than a warp), a curvilinear grid with a shock,
    and closed faces in every direction or in one.  With the walk threshold
    at 3 every direction stays on the UP7 walk, so shocked cases defer many
    cells to the fix-up kernel."""
    out = [
        ("iso24_hybrid_char", cases.isotropic_turbulence(24, seed=5, charteric=1)),
        ("iso40_hybrid_char", cases.isotropic_turbulence(40, seed=6, charteric=1)),
        ("rnd17x18x13_hybrid_char_curv_shock",
         cases.random_smooth_case(17, 18, 13, seed=65, scheme_invis="SCHEME_HYBRIDAUTO", charteric=1,
                                  shock=True, curvilinear=True)),
        ("rnd37x20x19_hybrid_char_shock",
         cases.random_smooth_case(37, 20, 19, seed=8, scheme_invis="SCHEME_HYBRIDAUTO", charteric=1, shock=True)),
    ]
    out += [(n, c) for n, c in bounded_cases() if n.startswith("bnd_hybrid")]
    return out


@pytest.mark.parametrize("name,case", _march_cases(), ids=[n for n, _ in _march_cases()])
def test_march_matches_ring_walk(name, case, gpu_lib):
    """The y and z UP7 walks run as per-lane marches over staged pencil tiles
    (variant 8; variant 4 in the precision form) or through the shared-memory
    ring (variant 7).  Same face and cell arithmetic and the same deferred
    cells, so the same state to the last bit, in FP64 and in the precision
    form; and the FP64 state matches the in-loop dispatch (variant 5) to the
    walk-equivalence bound."""
    for form in (0, 1):
        a = lib.Solver(case.cfg, case.prims, case.metrics, inlet=case.inlet)
        b = lib.Solver(case.cfg, case.prims, case.metrics, inlet=case.inlet)
        a.set_sweep_impl(8)
        b.set_sweep_impl(7)
        for s in (a, b):
            s.set_walk_threshold(3.0)
            if form:
                s.set_precision(1)
        a.step(3)
        b.step(3)
        assert a.sweep_walks() == 0 and b.sweep_walks() == 0
        assert np.array_equal(a.conserved(), b.conserved()), (name, form, rel_l2(a.conserved(), b.conserved()))
        if form == 0:
            c = lib.Solver(case.cfg, case.prims, case.metrics, inlet=case.inlet)
            c.set_sweep_impl(5)
            c.step(3)
            assert np.all(rel_l2(a.primitives(), c.primitives()) <= 1e-14), name


def _viscous_cases():
    """Viscous-kernel cases: CD6 and CD8, uniform and curvilinear metrics,
    closed faces, a width that is not a multiple of the 32-cell tile, the
    ramp with its boundary conditions and filter."""
    out = [
        ("tgv24_cd6", cases.taylor_green(24, seed=3)),
        ("iso40_hybrid_char", cases.isotropic_turbulence(40, seed=6, charteric=1)),
        ("rnd_weno7_cd8", cases.random_smooth_case(37, 11, 10, seed=22, scheme_vis="CD8")),
        ("rnd_weno7_curv", cases.random_smooth_case(19, 13, 11, seed=3, curvilinear=True)),
        ("ramp_bc108", cases.ramp_case(30, 18, 8, seed=66)),
    ]
    out += [(n, c) for n, c in bounded_cases() if n in ("bnd_weno7_cd8_one", "bnd_hybrid_char_both")]
    return out


@pytest.mark.parametrize("name,case", _viscous_cases(), ids=[n for n, _ in _viscous_cases()])
def test_staged_viscous_matches_cached(name, case, gpu_lib):
    """The viscous kernels with their stencil inputs staged in shared memory
    (variant 2: the primitives of the Ev kernel, the Ev tiles of the
    divergence + RK kernel) against the kernels that read them through the
    caches:
    the same arithmetic in the same order, so the same state to the last bit,
    in FP64 and (where the form covers the scheme) in the precision form."""
    forms = [0, 1] if case.cfg.scheme_invis in ("SCHEME_HYBRIDAUTO", "WENO7") and \
        (case.cfg.charteric or case.cfg.scheme_invis == "WENO7") else [0]
    for form in forms:
        a = lib.Solver(case.cfg, case.prims, case.metrics, inlet=case.inlet)
        b = lib.Solver(case.cfg, case.prims, case.metrics, inlet=case.inlet)
        a.set_viscous_impl(2)
        b.set_viscous_impl(1)
        if form:
            try:
                a.set_precision(1)
            except lib.OcfdError:
                continue
            b.set_precision(1)
        a.step(3)
        b.step(3)
        assert np.array_equal(a.conserved(), b.conserved()), (name, form, rel_l2(a.conserved(), b.conserved()))
        assert np.array_equal(a.primitives(), b.primitives()), (name, form)


def test_walk_choice_follows_sensor(gpu_lib):
    """Variant 4 picks a walk per direction after each sensor pass: the UP7
    walk where (almost) every face is UP7, the in-line walk where many are
    not; WENO7 always takes the in-line walk.  Either way the state matches
    the in-loop dispatch."""
    smooth = cases.isotropic_turbulence(16, seed=9, charteric=1)
    s = lib.Solver(smooth.cfg, smooth.prims, smooth.metrics)
    s.step(1)
    nonup7 = [int(np.count_nonzero(f != 1)) for f in s.flags()]
    walks = s.sweep_walks()
    for d in range(3):
        assert ((walks >> d) & 1) == (2 * nonup7[d] / s.flags()[d].size > 0.002), (d, nonup7, walks)
    shock = cases.random_smooth_case(13, 17, 11, seed=4, scheme_invis="SCHEME_HYBRIDAUTO", charteric=1,
                                     shock=True, curvilinear=True)
    s = lib.Solver(shock.cfg, shock.prims, shock.metrics)
    s.step(2)
    assert s.sweep_walks() == 7
    b = lib.Solver(shock.cfg, shock.prims, shock.metrics)
    b.set_sweep_impl(5)
    b.step(2)
    assert np.all(rel_l2(s.primitives(), b.primitives()) <= 1e-14)
    tgv = cases.taylor_green(16, seed=3)
    s = lib.Solver(tgv.cfg, tgv.prims, tgv.metrics)
    s.step(1)
    assert s.sweep_walks() == 7


def test_scheme_proportion(gpu_lib):
    """HybridAuto_scheme_Proportion: the shares of flags 1, 2 and other per
    direction, against counts of the flag arrays read back."""
    c = cases.random_smooth_case(13, 17, 11, seed=4, scheme_invis="SCHEME_HYBRIDAUTO", charteric=1,
                                 shock=True, curvilinear=True)
    s = lib.Solver(c.cfg, c.prims, c.metrics)
    s.step(1)
    got = s.scheme_proportion()
    for d, f in enumerate(s.flags()):
        want = [np.mean(f == 1), np.mean(f == 2), np.mean((f != 1) & (f != 2))]
        assert np.allclose(got[d], want, rtol=0, atol=1e-15), (d, got[d], want)
    assert np.allclose(got.sum(1), 1.0)


@pytest.mark.parametrize("iperiodic", [(0, 0, 1), (1, 0, 0), (0, 0, 0)], ids=["z_per", "x_per", "closed"])
def test_metrics_from_mesh_match_oracle(iperiodic, gpu_lib):
    """Comput_Jacobian3d on the GPU against the oracle's restatement: the 13
    metric fields (FP64, tolerance 1e-14 relative per field).  JAC_BOUND is
    set in every direction: without it a periodic copy of an increasing
    coordinate makes the Jacobian negative at the seam, where the reference
    stops."""
    case = cases.mesh_case(15, 13, 12, seed=63, jac_bound=(1, 1, 1), iperiodic=iperiodic)
    o = Oracle(case.cfg, case.prims, case.metrics)
    s = lib.Solver(case.cfg, case.prims, case.metrics)
    assert not s.uniform_metrics
    err = rel_l2(s.metrics(), o.metrics())
    assert np.all(err <= 1e-14), err


def test_negative_jacobian_is_rejected(gpu_lib):
    case = cases.mesh_case(12, 12, 11, seed=64)
    case.metrics[0] = case.metrics[0][:, :, ::-1].copy()      # mirror x: det < 0
    with pytest.raises(lib.OcfdError) as ei:
        lib.Solver(case.cfg, case.prims, case.metrics)
    assert ei.value.status == -1


def test_per_stage_api_equals_step_with_bc_and_filter(gpu_lib):
    """The compat sequence (du_comput, time_advance, get_duvwT, OCFD_bc,
    filtering) against step(), with IBC 108 and the shock filter."""
    case = cases.ramp_case(26, 16, 8, seed=68)
    a = lib.Solver(case.cfg, case.prims, case.metrics, inlet=case.inlet)
    b = lib.Solver(case.cfg, case.prims, case.metrics, inlet=case.inlet)
    a.step(2)
    for n in range(2):
        b.swap()
        for krk in (1, 2, 3):
            b.du_comput(krk)
            b.time_advance(krk)
            b.get_duvwT()
            b.bc()
        b.L.ocfd_b200_set_time(b.h, n + 1, (n + 1) * case.cfg.dt)
        assert b.L.ocfd_b200_filtering(b.h) == 0
    assert np.array_equal(a.primitives(), b.primitives())
    assert np.array_equal(a.conserved(), b.conserved())
