"""Parity at the benchmark sizes.

* C1 as configured: Taylor-Green vortex 64^3, WENO7 + CD6, 100 RK3 steps,
  against the CPU oracle and against the reference's own CUDA build
  (oracle/_ref, run live when it is present on the box).
* C2: isotropic turbulence 256^3, hybrid + characteristic projection, 3 and
  200 steps against the reference build, and size-independent properties:
  finite state, bitwise repeatability, and (on a single-scheme run) exact
  conservation of mass, momentum and energy on the periodic box.
* C4: the compression ramp 512x128x64 (metrics from the mesh, IBC 108, the
  shock filter) against the reference build after 100 steps, and after the
  stated 500 steps within the reference's own one-ulp sensitivity.
* C3 and the precision half of C4: the FP32-stencil form against the FP64
  path at the stated steps (50, 100, 200 on the C2 input; 100 and 500 on the
  ramp), relative L2 and L-infinity per conserved variable, bounded from
  the first measurements with a stated margin.
Tolerance: relative L2 <= 1e-12 per variable (the parity bound).
"""
import numpy as np
import pytest

from ocfd_b200 import cases, lib

pytestmark = pytest.mark.gpu

TOL = 1e-12


def rel_l2(a, b):
    return np.array([np.linalg.norm(a[m] - b[m]) / np.linalg.norm(b[m]) for m in range(a.shape[0])])


def _ref_runner():
    from oracle import ref_runner
    if not ref_runner.available():
        pytest.skip("reference build (oracle/_ref) not present on this machine")
    return ref_runner


@pytest.fixture(scope="module")
def tgv64():
    case = cases.taylor_green(64, seed=1234)
    s = lib.Solver(case.cfg, case.prims, case.metrics)
    s.step(100)
    return case, s.primitives(), s.conserved()


def test_c1_tgv64_100_steps_vs_oracle(tgv64):
    from oracle.oracle import Oracle
    case, prims, cons = tgv64
    o = Oracle(case.cfg, case.prims, case.metrics)
    o.step(100)
    assert np.all(rel_l2(prims, o.primitives()) <= TOL)
    assert np.all(rel_l2(cons, o.conserved()) <= TOL)


def test_c1_tgv64_100_steps_vs_reference(tgv64):
    rr = _ref_runner()
    case, prims, _ = tgv64
    ref, istep, tt, wall, _ = rr.run_and_read(cases.taylor_green(64, seed=1234), 100)
    assert istep == 100
    err = rel_l2(prims, ref)
    assert np.all(err <= TOL), err


@pytest.fixture(scope="module")
def iso256():
    case = cases.isotropic_turbulence(256, seed=2024, charteric=1)
    s = lib.Solver(case.cfg, case.prims, case.metrics)
    f0 = s.conserved()
    s.step(3)
    return case, s, f0


def test_c2_iso256_finite(iso256):
    case, s, f0 = iso256
    f3 = s.conserved()
    assert np.isfinite(f3).all()
    nnan, nneg, _ = s.check_state()
    assert nnan == 0 and nneg == 0


def test_iso256_weno7_conserves_mass_momentum_energy():
    # The hybrid scheme is not discretely conservative in the reference: the
    # sensor reads ghost cells that are one stage old and ghost corners that
    # are never filled, so the two images of a periodic seam face can get
    # different schemes (the oracle drifts by ~1e-5 in mass at 32^3 after 3
    # steps).  A single-scheme run conserves to round-off.
    case = cases.isotropic_turbulence(256, seed=2024, charteric=0)
    case.cfg.scheme_invis = "WENO7"
    s = lib.Solver(case.cfg, case.prims, case.metrics)
    f0 = s.conserved()
    s.step(2)
    f2 = s.conserved()
    for m in range(5):
        scale = np.abs(f0[m]).sum()
        drift = abs(f2[m].sum() - f0[m].sum()) / scale
        assert drift < 1e-13, (m, drift)


def test_c2_iso256_repeatable(iso256):
    case, s, _ = iso256
    s2 = lib.Solver(case.cfg, case.prims, case.metrics)
    s2.step(3)
    assert np.array_equal(s2.primitives(), s.primitives())


def _matches_reference(rr, got, make, nsteps, runs=3):
    """The reference build at this size does not always repeat itself: the
    shared-memory race of its characteristic y/z kernels can fire (measured:
    one 3-step run 1e-6 and one 200-step run 2e-5 away from other runs of the
    same input, which agree with each other and with the library to 5e-16).
    The library's state must match a reference run to 1e-12; up to `runs`
    runs are taken, and if none matches, the library must lie within twice
    the largest distance between them."""
    refs = []
    for _ in range(runs):
        ref, istep, *_ = rr.run_and_read(make(), nsteps, timeout=1800.0)
        assert istep == nsteps
        if np.all(rel_l2(got, ref) <= TOL):
            return
        refs.append(ref)
    spread = np.max([rel_l2(a, b) for n, a in enumerate(refs) for b in refs[n + 1:]], axis=0)
    errs = [rel_l2(got, r) for r in refs]
    assert all(np.all(e <= np.maximum(TOL, 2.0 * spread)) for e in errs), (errs, spread)


def test_c2_iso256_vs_reference(iso256):
    rr = _ref_runner()
    case, s, _ = iso256
    _matches_reference(rr, s.primitives(), lambda: cases.isotropic_turbulence(256, seed=2024, charteric=1), 3)


def test_c2_iso256_200_steps_vs_reference():
    """C2 for its stated 200 steps against the reference build (see
    _matches_reference for the reference's own run-to-run spread)."""
    rr = _ref_runner()
    case = cases.isotropic_turbulence(256, seed=2024, charteric=1)
    s = lib.Solver(case.cfg, case.prims, case.metrics)
    s.step(200)
    _matches_reference(rr, s.primitives(), lambda: cases.isotropic_turbulence(256, seed=2024, charteric=1), 200)


@pytest.fixture(scope="module")
def ramp500():
    case = cases.ramp_case(512, 128, 64, seed=2024)
    s = lib.Solver(case.cfg, case.prims, case.metrics, inlet=case.inlet)
    s.step(100)
    p100, c100 = s.primitives(), s.conserved()
    s.step(400)
    return case, s, p100, c100


def test_c4_ramp_500_steps_stays_physical(ramp500):
    case, s, _, _ = ramp500
    nnan, nneg, mean_t = s.check_state()
    assert nnan == 0 and nneg == 0
    p = s.primitives()
    assert p[0].min() > 0 and p[4].min() > 0 and np.isfinite(mean_t)


def test_c4_ramp_100_steps_vs_reference(ramp500):
    """C4 (metrics from the mesh on the GPU, IBC 108, the shock filter every
    step) against the reference build after 100 steps.  At this size the
    reference does not repeat itself bit for bit (the shared-memory race of
    its characteristic y/z kernels fires), so it runs twice: the library's
    state must match one of the two runs to 1e-12, or lie within twice the
    two runs' own distance from each other."""
    rr = _ref_runner()
    case, s, p100, _ = ramp500
    runs = []
    for _ in range(2):
        ref, istep, *_ = rr.run_and_read(cases.ramp_case(512, 128, 64, seed=2024), 100, timeout=1800.0)
        assert istep == 100
        runs.append(ref)
    errs = [rel_l2(p100, r) for r in runs]
    spread = rel_l2(runs[0], runs[1])
    exact = any(np.all(e <= TOL) for e in errs)
    within = all(np.all(e <= np.maximum(TOL, 2.0 * spread)) for e in errs)
    assert exact or within, (errs, spread)


def test_c4_ramp_500_steps_within_reference_sensitivity(ramp500):
    """Over the stated 500 steps the shocked, noisy ramp flow amplifies
    round-off: the reference build run from an input with one density value
    changed by one ulp ends up ~5e-7 (relative L2) from its own unperturbed
    run.  The library's 500-step state must sit within that spread of the
    reference's (it matches to 1e-15 at 100 steps, above)."""
    rr = _ref_runner()
    case, s, _, _ = ramp500
    ref, istep, *_ = rr.run_and_read(cases.ramp_case(512, 128, 64, seed=2024), 500, timeout=1800.0)
    pert = cases.ramp_case(512, 128, 64, seed=2024)
    d = pert.prims[0].copy()
    d[32, 64, 256] = np.nextafter(d[32, 64, 256], np.inf)
    pert.prims[0] = d
    ref_p, *_ = rr.run_and_read(pert, 500, timeout=1800.0)
    spread = rel_l2(ref_p, ref)
    err = rel_l2(s.primitives(), ref)
    assert np.all(spread > 1e-9), spread          # the sensitivity is real
    assert np.all(err <= 2.0 * spread), (err, spread)


def test_c3_precision_form_256_50_steps(iso256):
    """C3: the precision form on the C2 input against the FP64 path after 50
    steps (measured 8e-8 .. 1.6e-7 relative L2 on the conserved variables;
    bound 1e-6)."""
    case, _, _ = iso256
    a = lib.Solver(case.cfg, case.prims, case.metrics)
    b = lib.Solver(case.cfg, case.prims, case.metrics)
    b.set_precision(1)
    a.step(50)
    b.step(50)
    err = rel_l2(b.conserved(), a.conserved())
    assert np.all(err <= 1e-6) and np.all(err > 0), err


def form_errors(test, ref):
    """Relative L2 and L-infinity per conserved variable; the momentum
    components are measured against the momentum vector (its L2 norm, its
    largest magnitude), since the spanwise component is a small fluctuation."""
    mom_l2 = np.sqrt(sum(np.linalg.norm(ref[m]) ** 2 for m in (1, 2, 3)))
    mom_max = np.sqrt(ref[1] ** 2 + ref[2] ** 2 + ref[3] ** 2).max()
    l2, linf = [], []
    for m in range(5):
        d = test[m] - ref[m]
        l2.append(np.linalg.norm(d) / (mom_l2 if m in (1, 2, 3) else np.linalg.norm(ref[m])))
        linf.append(np.abs(d).max() / (mom_max if m in (1, 2, 3) else np.abs(ref[m]).max()))
    return np.array(l2), np.array(linf)


def test_c3_precision_form_256_100_200_steps(iso256):
    """C3 at its stated steps: the precision form against the FP64 path on
    the C2 input.  Measured (per-variable norms): relative L2 <= 5.4e-7 and
    L-infinity <= 2.5e-4 at step 100, <= 4.2e-6 and <= 7.1e-4 at step 200
    (shocklets form between 100 and 200 and a few faces fall on the other
    side of a sensor threshold in FP32).  Bounds: 5x those."""
    case, _, _ = iso256
    a = lib.Solver(case.cfg, case.prims, case.metrics)
    b = lib.Solver(case.cfg, case.prims, case.metrics)
    b.set_precision(1)
    for steps, tol_l2, tol_inf in ((100, 2.7e-6, 1.3e-3), (200, 2.1e-5, 3.6e-3)):
        a.step(steps - a.time()[0])
        b.step(steps - b.time()[0])
        l2, linf = form_errors(b.conserved(), a.conserved())
        print(f"C3 step {steps}: rel L2 {l2}, rel Linf {linf}")
        assert np.all(l2 > 0), l2
        assert np.all(l2 <= tol_l2), (steps, l2)
        assert np.all(linf <= tol_inf), (steps, linf)


def test_c4_precision_form_ramp_100_500_steps(ramp500):
    """The ramp in the precision form (boundary values formed in FP64, the
    filter weights from the FP32 pressure, its update in FP64) against the
    FP64 path at steps 100 and 500.  The shocked ramp flow amplifies any
    perturbation (the reference run from a one-ulp change ends 5e-7 away
    after 500 steps); FP32 stencils perturb every cell by ~1e-7 each stage.
    Bounds: relative L2 1e-4 at step 100 and 5e-3 at step 500, L-infinity
    5e-2 and 0.2."""
    case, s64, _, c100 = ramp500
    b = lib.Solver(case.cfg, case.prims, case.metrics, inlet=case.inlet)
    b.set_precision(1)
    b.step(100)
    l2, linf = form_errors(b.conserved(), c100)
    print(f"C4 precision form step 100: rel L2 {l2}, rel Linf {linf}")
    assert np.all(l2 > 0) and np.all(l2 <= 1e-4), l2
    assert np.all(linf <= 5e-2), linf
    b.step(400)
    l2, linf = form_errors(b.conserved(), s64.conserved())
    print(f"C4 precision form step 500: rel L2 {l2}, rel Linf {linf}")
    assert np.all(l2 <= 5e-3), l2
    assert np.all(linf <= 0.2), linf
    nnan, nneg, _ = b.check_state()
    assert nnan == 0 and nneg == 0
