"""Precision-form evaluation: the FP32-stencil / FP64-accumulation form run
beside the FP64 form from the same initial state, with per-variable errors
at chosen steps and the device time of each form.

The FP64 form is the reference here: it agrees with the CPU oracle to the
1e-12 parity bound on every case the tests run, and at 256^3 over 200 steps
the oracle itself would take hours, so the FP64 GPU run stands in for it.

    python -m ocfd_b200.precision --n 256 --steps 50,100,200 --out prec.json
    python -m ocfd_b200.precision --workload ramp --n 128 --steps 100,500

(--workload ramp: the compression ramp 4n x n x n/2, IBC 108 and the shock
filter every step.)
"""
import argparse
import json
import time
from typing import Dict, List, Sequence

import numpy as np

from . import cases, lib

NAMES = ("rho", "rho_u", "rho_v", "rho_w", "rho_E")


def field_errors(test: np.ndarray, ref: np.ndarray) -> Dict[str, Dict[str, float]]:
    """Relative L2 and L-infinity (max |diff| / max |ref|) per variable."""
    out = {}
    for m, name in enumerate(NAMES):
        d = test[m] - ref[m]
        out[name] = {
            "rel_l2": float(np.linalg.norm(d) / np.linalg.norm(ref[m])),
            "rel_linf": float(np.max(np.abs(d)) / np.max(np.abs(ref[m]))),
        }
    return out


def _timed_steps(s: "lib.Solver", n: int) -> float:
    """Device-synchronised wall time of n steps, in ms per step."""
    s.synchronize()
    t0 = time.perf_counter()
    s.step(n)
    s.synchronize()
    return (time.perf_counter() - t0) * 1e3 / max(n, 1)


def compare_forms(case, checkpoints: Sequence[int]) -> dict:
    ref = lib.Solver(case.cfg, case.prims, case.metrics, inlet=case.inlet)
    low = lib.Solver(case.cfg, case.prims, case.metrics, inlet=case.inlet)
    low.set_precision(1)
    # one warm-up step each outside the comparison would change the state;
    # the first segment's timing includes the first launches instead
    rows: List[dict] = []
    done = 0
    t64 = t32 = 0.0
    for c in sorted(checkpoints):
        n = c - done
        t64 += _timed_steps(ref, n) * n
        t32 += _timed_steps(low, n) * n
        done = c
        ec = field_errors(low.conserved(), ref.conserved())
        pr, pl = ref.primitives(), low.primitives()
        prim_err = {k: float(np.linalg.norm(pl[m] - pr[m]) / np.linalg.norm(pr[m]))
                    for m, k in enumerate(("d", "u", "v", "w", "T"))}
        rows.append({"step": c, "conserved": ec, "primitives_rel_l2": prim_err})
    ncell = case.cfg.nx * case.cfg.ny * case.cfg.nz
    return {
        "case": case.description,
        "cells": ncell,
        "checkpoints": rows,
        "ms_per_step_fp64": t64 / done,
        "ms_per_step_fp32_form": t32 / done,
        "gcell_stage_per_s_fp64": ncell * 3 / (t64 / done) / 1e6,
        "gcell_stage_per_s_fp32_form": ncell * 3 / (t32 / done) / 1e6,
    }


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--steps", default="50,100,200")
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--out", default="")
    ap.add_argument("--workload", choices=("iso", "ramp"), default="iso")
    a = ap.parse_args(argv)
    if a.workload == "ramp":
        case = cases.ramp_case(4 * a.n, a.n, a.n // 2, seed=a.seed)
    else:
        case = cases.isotropic_turbulence(a.n, seed=a.seed, charteric=1)
    res = compare_forms(case, [int(x) for x in a.steps.split(",")])
    txt = json.dumps(res, indent=1)
    if a.out:
        with open(a.out, "w") as f:
            f.write(txt + "\n")
    print(txt)


if __name__ == "__main__":
    main()
