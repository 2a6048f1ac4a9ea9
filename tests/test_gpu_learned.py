"""The learned scheme switch on the GPU against its CPU oracle
(oracle/mlp_oracle.py): features, FP32 gradients, the BF16 tensor-core
forward pass, training, and the switch inside the solver -- the plain
sensor as fallback (a network that is never confident reproduces the plain
run bit for bit) and as judge (a trained network stays within 1e-3 of the
plain FP64 run)."""
import numpy as np
import pytest

import os

from ocfd_b200 import cases, learned, lib
from oracle import mlp_oracle as mo

pytestmark = pytest.mark.gpu

# the network the package ships (trained on the plain solver's labels of
# Taylor-Green 64^3 and isotropic turbulence 256^3)
MODEL = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "opencfd-scu_b200", "ocfd_b200",
                     "data", "switch_c1c3.npz")


def random_params(rng, scale=0.4):
    w = (rng.standard_normal(mo.NPARAM) * scale).astype(np.float32)
    w[mo.OFF_MU:mo.OFF_MU + 14] = rng.standard_normal(14) * 0.1
    w[mo.OFF_SG:mo.OFF_SG + 14] = 0.5 + rng.random(14)
    return w


def test_parameter_count(gpu_lib):
    assert lib.mlp_nparam() == mo.NPARAM == 1597


def test_features_match_oracle(gpu_lib):
    """14 features (FP64 arithmetic, FP32 result) and labels of every
    interior cell of a periodic shocked state."""
    case = cases.isotropic_turbulence(24, seed=5, charteric=1, hy_dp_intv=(0.002, 0.02))
    s = lib.Solver(case.cfg, case.prims, case.metrics)
    s.step(2)
    f, y = s.switch_features()
    pr = s.primitives()
    p00 = 1.0 / (case.cfg.gamma * case.cfg.ama ** 2)
    fo, dp = mo.features(pr[0], pr[4], p00)
    np.testing.assert_allclose(f, fo, rtol=2e-6, atol=1e-9)
    yo = (dp > case.cfg.hy_dp_intv[0]).astype(np.float32)
    near = np.abs(dp - case.cfg.hy_dp_intv[0]) < 1e-12 * case.cfg.hy_dp_intv[0]
    assert np.array_equal(y[~near], yo[~near])
    assert 0 < y.sum() < y.size                       # both classes present


def test_gradient_matches_oracle(gpu_lib):
    """FP32 forward/backward kernels against FP64 back-propagation."""
    rng = np.random.default_rng(3)
    w = random_params(rng)
    f = rng.standard_normal((3000, 14)).astype(np.float32)
    y = (rng.random(3000) < 0.3).astype(np.float32)
    g, loss = lib.mlp_grad(w, f, y, pos_w=2.5)
    lo, go = mo.forward_backward(w, f, y, pos_w=2.5)
    assert abs(loss - lo) <= 1e-5 * abs(lo)
    assert np.linalg.norm(g - go) <= 1e-5 * np.linalg.norm(go), np.abs(g - go).max()


def test_tensor_core_forward_matches_bf16_oracle(gpu_lib):
    rng = np.random.default_rng(4)
    w = random_params(rng)
    f = rng.standard_normal((5000, 14)).astype(np.float32)        # not a multiple of 32
    z = lib.mlp_infer(w, f)
    zo = mo.logits_bf16(w, f)
    assert np.max(np.abs(z - zo)) <= 1e-3 * max(1.0, np.max(np.abs(zo))), np.max(np.abs(z - zo))


def test_training_learns_threshold_rule(gpu_lib):
    """Labels given by a threshold on one feature (as the plain sensor's are
    on the summed pressure term): Adam on the GPU reaches > 99 % accuracy."""
    rng = np.random.default_rng(5)
    f = np.abs(rng.standard_normal((40000, 14))).astype(np.float32) * 0.01
    y = (f[:, 12] > 0.012).astype(np.float32)
    w0 = learned.init_params(f.mean(0), f.std(0), seed=1)
    w, hist = lib.mlp_train(w0, f, y, epochs=20, batch=2048, lr=3e-3, seed=2)
    assert hist[-1] < 0.25 * hist[0]
    acc = np.mean((lib.mlp_infer(w, f) >= 0) == (y > 0.5))
    assert acc > 0.99, acc
    # same seed, same result: the gradient reduction has a fixed order
    w2, _ = lib.mlp_train(w0, f, y, epochs=20, batch=2048, lr=3e-3, seed=2)
    assert np.array_equal(w, w2)


def _shock_case():
    c = cases.isotropic_turbulence(24, seed=9, charteric=1, hy_dp_intv=(0.002, 0.02))
    return c


def test_unconfident_network_is_the_plain_sensor(gpu_lib):
    """Output always 0 (confidence 1/2): every cell keeps the plain flag, so
    the run equals the plain run bit for bit; the counters say so."""
    c = _shock_case()
    w = np.zeros(mo.NPARAM, np.float32)
    w[mo.OFF_SG:mo.OFF_SG + 14] = 1.0
    a = lib.Solver(c.cfg, c.prims, c.metrics)
    b = lib.Solver(c.cfg, c.prims, c.metrics)
    b.set_switch(w, 0.9)
    a.step(3)
    b.step(3)
    assert np.array_equal(a.conserved(), b.conserved())
    for fa, fb in zip(a.flags(), b.flags()):
        assert np.array_equal(fa, fb)
    sure, unsure, differ = b.switch_stats()
    assert sure == 0 and differ == 0 and unsure == 3 * 25 ** 3      # three sensor passes
    # FP32 form: the same with its FP32 sensor arithmetic
    a32 = lib.Solver(c.cfg, c.prims, c.metrics); a32.set_precision(1)
    b32 = lib.Solver(c.cfg, c.prims, c.metrics); b32.set_precision(1); b32.set_switch(w, 0.9)
    a32.step(2); b32.step(2)
    assert np.array_equal(a32.conserved(), b32.conserved())


@pytest.mark.parametrize("bias,expect", [(-10.0, "all_up7"), (10.0, "weno_everywhere")])
def test_confident_network_overrides(bias, expect, gpu_lib):
    c = _shock_case()
    w = np.zeros(mo.NPARAM, np.float32)
    w[mo.OFF_SG:mo.OFF_SG + 14] = 1.0
    w[mo.OFF_B3] = bias
    p = lib.Solver(c.cfg, c.prims, c.metrics)
    p.step(1)
    s = lib.Solver(c.cfg, c.prims, c.metrics)
    s.set_switch(w, 0.9)
    s.step(1)
    for fp, fs in zip(p.flags(), s.flags()):
        if expect == "all_up7":
            assert np.all(fs == 1)
        else:
            assert np.array_equal(fs, np.maximum(2, fp))
    s.set_switch(None)                 # back to the plain sensor
    s.step(1)
    assert any((f != 1).any() for f in s.flags())


def test_trained_switch_tracks_plain_run(gpu_lib):
    """Train on the plain solver's labels of a small shocked turbulence run,
    then run the switch inline: the network decides most cells, agrees with
    the plain sensor on nearly all of them, and the solution stays within
    1e-3 (relative L2) of the plain FP64 run with shock positions within a
    cell."""
    c = _shock_case()
    s = lib.Solver(c.cfg, c.prims, c.metrics)
    rng = np.random.default_rng(0)
    f, y = learned.collect(s, [1, 3, 6, 10], rng, neg_ratio=4.0, min_neg=2000)
    assert 100 < y.sum() < len(y)
    w0 = learned.init_params(f.mean(0), f.std(0) + 1e-12, seed=3)
    w, hist = lib.mlp_train(w0, f, y, epochs=60, batch=1024, lr=3e-3, seed=4)
    assert np.mean((lib.mlp_infer(w, f) >= 0) == (y > 0.5)) > 0.97
    a = lib.Solver(c.cfg, c.prims, c.metrics)
    b = lib.Solver(c.cfg, c.prims, c.metrics)
    b.set_switch(w, 0.9)
    a.step(10)
    b.step(10)
    sure, unsure, differ = b.switch_stats()
    assert sure > 0.9 * (sure + unsure)
    assert differ < 0.02 * sure
    ua, ub = a.conserved(), b.conserved()
    err = [np.linalg.norm(ub[m] - ua[m]) / np.linalg.norm(ua[m]) for m in range(5)]
    assert max(err) <= 1e-3, err
    pa, pb = a.primitives(), b.primitives()
    sh = learned.shock_error(pa[0] * pa[4], pb[0] * pb[4], q=0.9)
    assert sh["max_cells"] <= 1, sh


def _vec_rel_l2(test, ref):
    """Relative L2 per conserved variable; the momentum components against
    the momentum vector's norm (the spanwise one is a small fluctuation)."""
    mom = np.sqrt(sum(np.linalg.norm(ref[m]) ** 2 for m in (1, 2, 3)))
    return np.array([np.linalg.norm(test[m] - ref[m]) / (mom if m in (1, 2, 3) else np.linalg.norm(ref[m]))
                     for m in range(5)])


@pytest.mark.parametrize("which", ["iso128", "ramp256x64x32"])
def test_shipped_switch_cost_and_accuracy(which, gpu_lib):
    """What the shipped network changes, against the same precision form with
    the plain sensor: the time per step of each (recorded; the network pass
    costs more than the sensor formula it replaces, so the ratio is at or
    below 1 -- on these flows both mark the same faces, so the walks do the
    same work), and the state against the plain FP64 run: within 1e-3
    relative L2 and shock positions within one cell.  Isotropic turbulence
    is the flow the network was trained on; the ramp (IBC 108, the filter,
    half the faces non-UP7) is not."""
    import time

    if which == "iso128":
        c = cases.isotropic_turbulence(128, seed=2024, charteric=1)
        steps = 30
    else:
        c = cases.ramp_case(256, 64, 32, seed=2024)
        steps = 50
    w = learned.load_model(MODEL)
    ref = lib.Solver(c.cfg, c.prims, c.metrics, inlet=c.inlet)
    ref.step(steps)
    u_ref, p_ref = ref.conserved(), ref.primitives()
    ms = {}
    out = {}
    for name, use in (("plain", False), ("switch", True)):
        s = lib.Solver(c.cfg, c.prims, c.metrics, inlet=c.inlet)
        s.set_precision(1)
        if use:
            s.set_switch(w, 0.9)
        s.step(2)
        s.synchronize()
        t0 = time.perf_counter()
        s.step(steps - 2)
        s.synchronize()
        ms[name] = (time.perf_counter() - t0) * 1e3 / (steps - 2)
        out[name] = (s.conserved(), s.primitives())
        if use:
            sure, unsure, differ = s.switch_stats()
    err = _vec_rel_l2(out["switch"][0], u_ref)
    pr = out["switch"][1]
    sh = learned.shock_error(p_ref[0] * p_ref[4], pr[0] * pr[4], q=0.99)
    print(f"{which}: ms/step plain sensor {ms['plain']:.3f}, switch {ms['switch']:.3f} "
          f"(ratio {ms['plain'] / ms['switch']:.3f}); rel L2 vs FP64 {err}; shock {sh}; "
          f"network cells {sure}, plain fallbacks {unsure}, differing {differ}")
    assert sure > 0.9 * (sure + unsure)
    assert np.all(err <= 1e-3), err
    assert sh["max_cells"] <= 1, sh
    assert ms["plain"] / ms["switch"] > 0.5
