"""Learned scheme switch: data from the plain solver, training on the GPU,
evaluation against the plain FP64 run.

Data: states of the plain FP64 solver on the Taylor-Green case (64^3) and
on decaying isotropic turbulence (256^3) at chosen steps; per interior cell
the 14 switch features and the plain sensor's label (flag 2 or 3).  Every
positive cell is kept and negatives are subsampled to at most `neg_ratio`
per positive (at least `min_neg` per state), with a seeded generator.

Training: the library's FP32 forward/backward and Adam kernels
(ocfd_b200_mlp_train); features standardised by the training set's mean
and standard deviation, stored in the parameter vector.

Evaluation (the 512^3 run): the precision form with the learned switch
against the plain FP64 run from the same initial state -- relative L2 of
the conserved variables and the shock-position error (per x-line, the cell
of the strongest pressure jump, over lines where that jump is in the top
0.1 % of the plain run's), plus the device time per step of both runs.

    python -m ocfd_b200.learned train --out switch.npz
    python -m ocfd_b200.learned eval --model switch.npz --n 512 --steps 100
"""
import argparse
import json
import time
from typing import Dict, List, Sequence, Tuple

import numpy as np

from . import cases, lib

NIN, NH = 14, 32


def init_params(mu: np.ndarray, sigma: np.ndarray, seed: int = 7) -> np.ndarray:
    """He-initialised weights, zero biases, the given standardisation."""
    rng = np.random.default_rng(seed)
    w = np.zeros(lib.mlp_nparam(), np.float32)
    w[0:NIN] = mu
    w[NIN:2 * NIN] = sigma
    o = 2 * NIN
    w[o:o + NH * NIN] = rng.standard_normal(NH * NIN) * np.sqrt(2.0 / NIN); o += NH * NIN
    o += NH
    w[o:o + NH * NH] = rng.standard_normal(NH * NH) * np.sqrt(2.0 / NH); o += NH * NH
    o += NH
    w[o:o + NH] = rng.standard_normal(NH) * np.sqrt(1.0 / NH)
    return w


def collect(solver: "lib.Solver", checkpoints: Sequence[int], rng: np.random.Generator,
            neg_ratio: float = 8.0, min_neg: int = 20000, chunk: int = 1 << 22) -> Tuple[np.ndarray, np.ndarray]:
    """Features and labels of the solver's states at the given steps."""
    feats, labels = [], []
    done = solver.time()[0]
    n = solver.cfg.nx * solver.cfg.ny * solver.cfg.nz
    for c in sorted(checkpoints):
        if c > done:
            solver.step(c - done)
            done = c
        pos_f, neg_f = [], []
        for first in range(0, n, chunk):
            f, y = solver.switch_features(first, min(chunk, n - first))
            pos_f.append(f[y > 0.5])
            neg_f.append(f[y <= 0.5])
        pos = np.concatenate(pos_f)
        neg = np.concatenate(neg_f)
        keep = min(len(neg), max(min_neg, int(neg_ratio * len(pos))))
        neg = neg[rng.choice(len(neg), keep, replace=False)]
        feats += [pos, neg]
        labels += [np.ones(len(pos), np.float32), np.zeros(len(neg), np.float32)]
    return np.concatenate(feats), np.concatenate(labels)


def dataset(seed: int = 11, tgv_n: int = 64, iso_n: int = 256,
            tgv_steps=(0, 25, 50, 75, 100), iso_steps=(50, 100, 150, 200)) -> Dict[str, np.ndarray]:
    """Training data from the Taylor-Green and isotropic-turbulence runs."""
    rng = np.random.default_rng(seed)
    out = {}
    c1 = cases.taylor_green(tgv_n, seed=1234)
    s = lib.Solver(c1.cfg, c1.prims, c1.metrics)
    f1, y1 = collect(s, tgv_steps, rng)
    s.close()
    c3 = cases.isotropic_turbulence(iso_n, seed=2024, charteric=1)
    s = lib.Solver(c3.cfg, c3.prims, c3.metrics)
    f3, y3 = collect(s, iso_steps, rng)
    s.close()
    out["feat"] = np.concatenate([f1, f3])
    out["label"] = np.concatenate([y1, y3])
    out["source"] = np.concatenate([np.zeros(len(y1), np.int8), np.ones(len(y3), np.int8)])
    return out


def train(data: Dict[str, np.ndarray], epochs: int = 12, batch: int = 16384, lr: float = 2e-3,
          seed: int = 7, holdout: float = 0.1) -> Dict[str, object]:
    """Train on a seeded split of the data; report held-out accuracy."""
    feat, label = data["feat"], data["label"]
    rng = np.random.default_rng(seed)
    perm = rng.permutation(len(label))
    nh = int(holdout * len(label))
    te, tr = perm[:nh], perm[nh:]
    mu = feat[tr].mean(0).astype(np.float32)
    sigma = (feat[tr].std(0) + 1e-12).astype(np.float32)
    npos, nneg = float(label[tr].sum()), float(len(tr) - label[tr].sum())
    w0 = init_params(mu, sigma, seed)
    w, hist = lib.mlp_train(w0, feat[tr], label[tr], epochs, batch, lr, pos_w=1.0, seed=seed)
    z = lib.mlp_infer(w, feat[te])
    yhat = z >= 0
    yt = label[te] > 0.5
    sure = np.abs(z) >= np.log(9.0)
    return {
        "params": w,
        "loss": hist,
        "train_rows": int(len(tr)), "train_pos": int(npos), "train_neg": int(nneg),
        "holdout_accuracy": float(np.mean(yhat == yt)),
        "holdout_recall_pos": float(np.mean(yhat[yt])) if yt.any() else float("nan"),
        "holdout_sure_fraction": float(np.mean(sure)),
        "holdout_sure_accuracy": float(np.mean((yhat == yt)[sure])) if sure.any() else float("nan"),
    }


def save(path: str, params: np.ndarray, meta: dict):
    np.savez(path, params=np.asarray(params, np.float32), meta=json.dumps(meta))


def load_model(path: str) -> np.ndarray:
    return np.load(path)["params"].astype(np.float32)


def shock_positions(p: np.ndarray, q: float = 0.999):
    """Per x-line, the cell of the strongest pressure jump |p[i+1] - p[i]|
    (periodic) and its size; the lines kept are those whose jump exceeds
    the q-quantile over all lines."""
    jump = np.abs(np.roll(p, -1, axis=2) - p)
    pos = np.argmax(jump, axis=2)
    mag = np.max(jump, axis=2)
    return pos, mag, mag >= np.quantile(mag, q)


def shock_error(p_ref: np.ndarray, p_test: np.ndarray, q: float = 0.999) -> Dict[str, float]:
    pr, mr, keep = shock_positions(p_ref, q)
    pt, _, _ = shock_positions(p_test, q)
    nx = p_ref.shape[2]
    d = np.abs(pr - pt)
    d = np.minimum(d, nx - d)[keep]
    return {"lines": int(keep.sum()), "max_cells": int(d.max()) if d.size else 0,
            "mean_cells": float(d.mean()) if d.size else 0.0, "frac_within_1": float(np.mean(d <= 1))}


def _timed(s: "lib.Solver", n: int) -> float:
    s.synchronize()
    t0 = time.perf_counter()
    s.step(n)
    s.synchronize()
    return (time.perf_counter() - t0) * 1e3 / max(n, 1)


def evaluate(params: np.ndarray, n: int = 512, steps: int = 100, confidence: float = 0.9,
             seed: int = 2024, workload: str = "iso") -> dict:
    """Plain FP64 against the precision form with the learned switch, and the
    precision form with the plain sensor: isotropic turbulence n^3, or the
    compression ramp 4n x n x n/2 (IBC 108, the shock filter), where the
    plain sensor marks most faces for the characteristic WENO schemes."""
    if workload == "ramp":
        c = cases.ramp_case(4 * n, n, n // 2, seed=seed)
    else:
        c = cases.isotropic_turbulence(n, seed=seed, charteric=1)
    ncell = c.cfg.nx * c.cfg.ny * c.cfg.nz
    out = {"case": c.description, "steps": steps, "confidence": confidence}
    ref = lib.Solver(c.cfg, c.prims, c.metrics, inlet=c.inlet)
    ref.step(1)                                   # first launches outside the timing
    t_ref = _timed(ref, steps - 1)
    u_ref, p_ref = ref.conserved(), ref.primitives()
    ref.close()
    runs = {}
    for name, use in (("fp32_plain_sensor", False), ("fp32_learned", True)):
        s = lib.Solver(c.cfg, c.prims, c.metrics, inlet=c.inlet)
        s.set_precision(1)
        if use:
            s.set_switch(params, confidence)
        s.step(1)
        t = _timed(s, steps - 1)
        u, pr = s.conserved(), s.primitives()
        r = {"ms_per_step": t, "gcell_stage_per_s": ncell * 3 / t / 1e6,
             "rel_l2": [float(np.linalg.norm(u[m] - u_ref[m]) / np.linalg.norm(u_ref[m])) for m in range(5)]}
        pres = pr[0] * pr[4]
        r["shock"] = shock_error(p_ref[0] * p_ref[4], pres)
        r["non_up7_faces"] = [float(np.mean(f != 1)) for f in s.flags()]
        if use:
            sure, unsure, differ = s.switch_stats()
            r["switch"] = {"network_cells": sure, "plain_fallback_cells": unsure, "network_differs_from_plain": differ}
        runs[name] = r
        s.close()
    out["fp64_plain"] = {"ms_per_step": t_ref, "gcell_stage_per_s": ncell * 3 / t_ref / 1e6}
    out.update(runs)
    out["speedup_learned_fp32_vs_fp64"] = t_ref / runs["fp32_learned"]["ms_per_step"]
    out["switch_vs_plain_sensor"] = runs["fp32_plain_sensor"]["ms_per_step"] / runs["fp32_learned"]["ms_per_step"]
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description="learned scheme switch: train or evaluate")
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train")
    t.add_argument("--out", required=True)
    t.add_argument("--epochs", type=int, default=12)
    t.add_argument("--iso-n", type=int, default=256)
    e = sub.add_parser("eval")
    e.add_argument("--model", required=True)
    e.add_argument("--n", type=int, default=512)
    e.add_argument("--steps", type=int, default=100)
    e.add_argument("--out", default="")
    e.add_argument("--workload", choices=("iso", "ramp"), default="iso")
    a = ap.parse_args(argv)
    if a.cmd == "train":
        data = dataset(iso_n=a.iso_n)
        res = train(data, epochs=a.epochs)
        meta = {k: v for k, v in res.items() if k != "params"}
        meta["loss"] = [float(x) for x in res["loss"]]
        save(a.out, res["params"], meta)
        print(json.dumps(meta, indent=1))
    else:
        res = evaluate(load_model(a.model), a.n, a.steps, workload=a.workload)
        txt = json.dumps(res, indent=1)
        if a.out:
            with open(a.out, "w") as f:
                f.write(txt + "\n")
        print(txt)


if __name__ == "__main__":
    main()
