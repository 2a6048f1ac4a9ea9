"""The bounds-checked build (libocfd_b200_bounds.so, -DOCFD_BOUNDS) on every
reference golden case and on the paths the golden cases do not reach (the
precision form's marches and staged viscous kernels, the learned switch, the
FP64 marches and staged viscous kernels, the in-line walk in FP32 on the
ramp).  In that build the index helpers and the walks' global accesses check
each index against its array; one outside it is recorded in the error word
and redirected into the array, and the call reports the error.  The run
here stands in for a memory checker: every case must finish without an
index error and give the state of the default build: relative L2 <= 1e-13
per variable in FP64, <= 1e-6 in the precision form (the same sources,
compiled with the checks; the compiler contracts a few FP32 multiply-adds
differently around them, a difference at FP32 rounding level).

The bounds build runs in a child process (one library per process)."""
import glob
import os

import numpy as np
import pytest

from ocfd_b200 import cases, learned, lib

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BOUNDS_LIB = os.path.join(ROOT, "opencfd-scu_b200", "libocfd_b200_bounds.so")
GOLDEN = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "*.npz")))
MODEL = os.path.join(ROOT, "opencfd-scu_b200", "ocfd_b200", "data", "switch_c1c3.npz")
TOL = 1e-13
TOL_FP32 = 1e-6


def _golden(path):
    import json
    from ocfd_b200.formats import CaseConfig
    z = np.load(path)
    cfgd = json.loads(str(z["config"]))
    cfg = CaseConfig(**{k: (tuple(v) if isinstance(v, list) else v) for k, v in cfgd.items()})
    case = cases.Case(cfg, list(z["prims_in"]), list(z["metrics"]), os.path.basename(path),
                      z["inlet"] if "inlet" in z.files else None)
    return case, int(z["nsteps"])


def _extra():
    """(name, case, settings, steps) beyond the golden cases."""
    out = []
    iso = cases.isotropic_turbulence(24, seed=41, charteric=1, hy_dp_intv=(0.002, 0.02))
    out.append(("iso24_fp32_march_staged", iso, {"precision": 1}, 3))
    out.append(("iso24_fp32_switch", iso, {"precision": 1, "switch": True}, 3))
    out.append(("iso24_fp64_march_staged", iso, {"sweep": 8, "viscous": 2}, 3))
    out.append(("iso24_fp64_inline", iso, {"sweep": 6}, 2))
    ramp = cases.ramp_case(64, 32, 16, seed=7)
    out.append(("ramp64_fp32", ramp, {"precision": 1}, 2))
    return out


def _all_cases():
    out = []
    for p in GOLDEN:
        c, n = _golden(p)
        out.append((os.path.basename(p)[:-4], c, {}, n))
    return out + _extra()


def _run(case, settings, steps):
    s = lib.Solver(case.cfg, case.prims, case.metrics, inlet=case.inlet)
    if "precision" in settings:
        s.set_precision(settings["precision"])
    if settings.get("switch"):
        s.set_switch(learned.load_model(MODEL), 0.9)
    if "sweep" in settings:
        s.set_sweep_impl(settings["sweep"])
    if "viscous" in settings:
        s.set_viscous_impl(settings["viscous"])
    s.step(steps)
    s.synchronize()
    u = s.conserved()
    s.close()
    return u


def _child(outdir):
    """Every case through the bounds-checked library; a case whose call
    reports an error stores the message instead of the state."""
    lib.load(BOUNDS_LIB)
    for name, case, settings, steps in _all_cases():
        try:
            np.save(os.path.join(outdir, name + ".npy"), _run(case, settings, steps))
        except lib.OcfdError as e:
            with open(os.path.join(outdir, name + ".err"), "w") as fh:
                fh.write(str(e))


def test_bounds_build_runs_clean(gpu_lib, tmp_path):
    if not os.path.exists(BOUNDS_LIB):
        pytest.fail(f"{BOUNDS_LIB} missing: build it with `make -C opencfd-scu_b200 bounds`")
    import multiprocessing as mp
    p = mp.get_context("spawn").Process(target=_child, args=(str(tmp_path),))
    p.start()
    p.join(timeout=900)
    assert p.exitcode == 0
    errors = {f[:-4]: open(tmp_path / f).read() for f in os.listdir(tmp_path) if f.endswith(".err")}
    assert not errors, "\n".join(f"{k}: {v}" for k, v in sorted(errors.items()))
    bad = {}
    for name, case, settings, steps in _all_cases():
        want = _run(case, settings, steps)
        got = np.load(tmp_path / (name + ".npy"))
        err = max(np.linalg.norm(got[m] - want[m]) / np.linalg.norm(want[m]) for m in range(5))
        if not err <= (TOL_FP32 if settings.get("precision") else TOL):
            bad[name] = err
    assert not bad, bad
