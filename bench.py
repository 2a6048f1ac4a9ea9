#!/usr/bin/env python
"""Throughput benchmark of the per-RK-stage RHS path on B200.

Workload (default): decaying compressible isotropic turbulence on a 256^3
periodic grid, SCHEME_HYBRIDAUTO (style 2 Jameson sensor: UP7 / WENO7 /
WENO5) with characteristic projection, CD6 viscous terms, SSP-RK3, plain
FP64.  Synthetic, seeded input (no dataset).  One "step" is one RK3 time
step (3 stages) over the whole grid.

Metric: Gcell-RK-stage/s = cells x 3 x steps / seconds / 1e9.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun) every rank runs an independent replica of the same
grid on its own GPU (the path has no exchange step on one grid per GPU);
value = all ranks' cell-stages / max-over-ranks time ("scaling": "weak").
With --decomp z the N ranks instead hold the z slabs of one grid of
n x n x (n N) cells (each slab the n^3 case, so the whole grid is that case
repeated N times in z and stays periodic); the slabs swap ghost planes over
NCCL inside every ghost fill ("scaling": "weak", per-GPU work fixed).  On one
GPU, --decomp z runs a single slab whose neighbour is itself, which times the
exchange path against the periodic wrap.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "opencfd-scu_b200"))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "Gcell-RK-stage/s"
B_ALG = 120.0          # algorithmic bytes per cell-stage (read U^k, U^n, write U^k+1; FP64)


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# clocks sampling during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = os.path.join("/tmp", f"ocfd_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as fh:
            for line in fh:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax = float(parts[2])
                except ValueError:
                    continue
                for nm, val in zip(names, parts[5:9]):
                    if val.lower().startswith("active"):
                        reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------
# The three plain-FP64 workloads (the benchmark configurations):
#   iso  decaying isotropic turbulence n^3 (default 256^3), hybrid UP7/WENO7/WENO5
#        with the Jameson sensor and characteristic projection, CD6, periodic;
#   tgv  Taylor-Green vortex n^3 (64^3), WENO7 + CD6, Mach 0.1, Re 1600;
#   ramp 24-degree compression ramp 512x128x64 (scaled by n/128 in y), metrics
#        computed from the mesh, IBC 108 walls and inflow, hybrid + shock filter.
WORKLOADS = {
    "iso": "isotropic turbulence {nx}^3, hybrid UP7/WENO7/WENO5 (Jameson sensor) + characteristic "
           "projection, CD6 viscous, SSP-RK3, plain FP64",
    "tgv": "Taylor-Green vortex {nx}^3, WENO7 + CD6 viscous, SSP-RK3, plain FP64",
    "ramp": "24-degree compression ramp {nx}x{ny}x{nz}, Mach 2.9, Re 5000, Tw 2.5, metrics from the mesh "
            "(FP64), IBC 108, hybrid + characteristic + shock filter, CD6, SSP-RK3, plain FP64",
}


def make_case(workload: str, n: int):
    from ocfd_b200 import cases
    if workload == "tgv":
        return cases.taylor_green(n, seed=1234)
    if workload == "ramp":
        return cases.ramp_case(4 * n, n, n // 2, seed=2024)
    return cases.isotropic_turbulence(n, seed=2024, charteric=1)


def default_n(workload: str) -> int:
    return {"iso": 256, "tgv": 64, "ramp": 128}[workload]


def cells_of(case) -> int:
    return case.cfg.nx * case.cfg.ny * case.cfg.nz


def config_of(args, case, world: int) -> dict:
    """The workload description both arms print (the reference arm runs the
    same case, so the two dicts are equal)."""
    nx, ny, nz = case.cfg.nx, case.cfg.ny, case.cfg.nz
    cells = nx * ny * nz
    state_gb = 8 * cells * (15 + 35 * (nx + 8) * (ny + 8) * (nz + 8) / cells) / 1e9
    return {"workload": WORKLOADS[args.workload].format(nx=nx, ny=ny, nz=nz),
            "grid": [nx, ny, nz], "stages_per_step": 3, "form": args.form,
            "scheme": f"SCHEME_INVIS {case.cfg.scheme_invis}, CHARTERIC={case.cfg.charteric}",
            "seed": 2024 if args.workload != "tgv" else 1234,
            "l2": f"inputs larger than L2 (state ~{state_gb:.1f} GB/GPU)" if state_gb > 0.5
                  else f"state ~{state_gb:.2f} GB/GPU, partly L2-resident",
            "parallelism": (f"z slabs x{world} (grid {nx}x{ny}x{nz * world}, ghost planes over NCCL)"
                            if args.decomp == "z" else f"replicas x{world}")}


def cpu_baseline(workload: str, n_sample: int, steps: int = 0, budget_s: float = 12.0):
    """The OpenMP FP64 oracle timed on this host on a bounded sample: whole
    RK3 steps of the case at a reduced size until about budget_s seconds of
    CPU work have run (or exactly `steps` steps when given)."""
    from oracle.oracle import Oracle
    c = make_case(workload, n_sample)
    cores = os.cpu_count() or 1
    o = Oracle(c.cfg, c.prims, c.metrics, nthreads=cores, inlet=c.inlet)
    o.step(1)                                   # warm-up
    t0 = time.perf_counter()
    done = 0
    while True:
        o.step(1)
        done += 1
        dt = time.perf_counter() - t0
        if (steps and done >= steps) or (not steps and dt >= budget_s) or done >= 10000:
            break
    steps = done
    v = cells_of(c) * 3 * steps / dt / 1e9
    return {"value": v, "unit": METRIC, "cores": cores, "kind": "port",
            "sample": f"{steps} RK3 step(s) of the same case at {c.cfg.nx}x{c.cfg.ny}x{c.cfg.nz} "
                      f"(OpenMP FP64 oracle, {cores} threads, {dt:.2f} s)"}


def max_over_ranks(x: float, dist, device=None) -> float:
    """Max of a per-rank float over all ranks (the slowest replica sets the
    time); works for the nccl (device tensor) and gloo (CPU tensor) groups."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(cells: int, stages: int, seconds_max: float, world: int) -> float:
    """Whole-job Gcell-RK-stage/s: every replica processes `cells` x `stages`."""
    return world * cells * stages / seconds_max / 1e9


def make_solver(args, case, dev, form, slab=None):
    from ocfd_b200 import lib
    solver = lib.Solver(case.cfg, case.prims, case.metrics, device=dev, inlet=case.inlet, slab=slab)
    if args.no_graphs:                  # every kernel launched one by one
        solver.set_graphs(False)
    if form != "fp64":                  # precision form (and the learned switch)
        solver.set_precision(1)
    if form == "fp32-learned":
        from ocfd_b200 import learned
        solver.set_switch(learned.load_model(SWITCH_MODEL), 0.9)
    return solver


def timed_steps(solver, stream, steps, warmup, dist, dev, sample_clocks=True):
    """W untimed steps, one timing pass (per-family device times, untimed),
    then exactly `steps` steps between CUDA events on the solver's stream,
    barrier + synchronize on both sides.  Returns (ms, launches, families,
    clocks)."""
    import torch
    solver.step(warmup)
    solver.synchronize()
    solver.set_timing(True)
    solver.step(1)
    solver.synchronize()
    fam = solver.timing()
    solver.set_timing(False)
    sampler = ClockSampler(dev) if sample_clocks else None
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    if sampler:
        sampler.start()
        time.sleep(0.3)
    l0 = solver.launch_count()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    solver.step(steps)
    ev1.record(stream)
    ev1.synchronize()
    launches = solver.launch_count() - l0
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = sampler.stop() if sampler else None
    return ev0.elapsed_time(ev1), launches, fam, clocks


def rel_l2_per_variable(a, b):
    """Relative L2 of each conserved variable; the momentum components
    against the norm of the whole momentum vector (one may start near 0)."""
    vec = float(np.sqrt(sum(np.linalg.norm(b[m]) ** 2 for m in (1, 2, 3))))
    return [float(np.linalg.norm(a[m] - b[m]) / (vec if m in (1, 2, 3) else np.linalg.norm(b[m])))
            for m in range(5)]


def learned_leg(args, case, dev, ref_cons, ref_ms, steps_done):
    """The precision form with the plain sensor and with the learned switch
    on the same case, each timed like the main run (W warm-up steps, one
    timing pass, `steps` timed steps), with the relative L2 of its conserved
    state against the FP64 state after the same number of steps."""
    import torch
    out = {}
    cells = cells_of(case)
    for form in ("fp32", "fp32-learned"):
        s = make_solver(args, case, dev, form)
        stream = torch.cuda.Stream(device=dev)
        s.set_stream(stream.cuda_stream)
        ms, launches, fam, _ = timed_steps(s, stream, args.steps, args.warmup, None, dev, sample_clocks=False)
        assert args.warmup + 1 + args.steps == steps_done
        err = rel_l2_per_variable(s.conserved(), ref_cons)
        leg = {"value": cells * 3 * args.steps / (ms / 1e3) / 1e9, "unit": METRIC,
               "ms_per_step": ms / args.steps, "speedup_vs_fp64": ref_ms / ms,
               "rel_l2_vs_fp64": err, "after_steps": steps_done,
               "kernel_ms_per_stage": {k: v[0] / 3.0 for k, v in fam.items()}}
        if form == "fp32-learned":
            dec, plain, differ = s.switch_stats()
            leg["switch_decisions"] = {"network": dec, "plain_sensor": plain, "network_differs": differ}
        out[form] = leg
        s.close()
        del stream
    out["switch_vs_plain_sensor"] = out["fp32"]["ms_per_step"] / out["fp32-learned"]["ms_per_step"]
    return out


def run_ours(args, rank, world, dist):
    import torch

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    n = args.n
    case = make_case(args.workload, n)
    slab = None
    if args.decomp == "z":
        from ocfd_b200 import lib, slabs
        if args.workload == "ramp" and world > 1:
            raise SystemExit("--decomp z repeats the case in z; the ramp's mesh coordinates would not follow")
        cid = slabs.share_id(group=None) if dist else lib.slab_unique_id()
        slab = slabs.slab_spec(rank, world, case.cfg.nz * world, cid)
    solver = make_solver(args, case, dev, args.form, slab)
    stream = torch.cuda.Stream(device=dev)
    solver.set_stream(stream.cuda_stream)
    cells = cells_of(case)
    nx, ny, nz = case.cfg.nx, case.cfg.ny, case.cfg.nz

    ms, launches, fam, clocks = timed_steps(solver, stream, args.steps, args.warmup, dist, dev)
    ms_max = max_over_ranks(ms, dist, f"cuda:{dev}")
    value = aggregate_rate(cells, 3 * args.steps, ms_max / 1e3, world)
    steps_done = args.warmup + 1 + args.steps
    want_learned = (rank == 0 and world == 1 and args.learned and args.form == "fp64" and args.workload == "iso"
                    and args.decomp == "replicas")
    ref_cons = solver.conserved() if want_learned else None

    # end to end through the C ABI with host buffers (pinned), one RK3 step
    # per call: H2D of the primitives, the step, D2H of the primitives
    shape = (5, nz, ny, nx)
    hin = torch.empty(shape, dtype=torch.float64).pin_memory()
    hout = torch.empty(shape, dtype=torch.float64).pin_memory()
    a_in = hin.numpy()
    a_in[:] = np.stack(case.prims)
    a_out = hout.numpy()
    e2e_steps = max(1, min(args.steps, args.e2e_steps))
    solver.advance_host(a_in, a_out, 1)        # warm-up of the path
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        solver.advance_host(a_in, a_out, 1)
    e2e_s = max_over_ranks(time.perf_counter() - t0, dist, f"cuda:{dev}")
    e2e_val = aggregate_rate(cells, 3 * e2e_steps, e2e_s, world)
    nbytes = 5 * cells * 8
    uniform = solver.uniform_metrics
    if want_learned:
        solver.close()

    if rank != 0:
        return None
    hbm, peak_kind = peaks()
    # dominant kernel family; its roofline uses the algorithmic bytes of a
    # stage (read U^k and U^n, write U^k+1: 120 B per cell-stage; 200 B with
    # the 10 metric fields of a curvilinear grid) over the family's time
    dom = max(fam, key=lambda k: fam[k][0])
    dom_ms_per_stage = fam[dom][0] / 3.0                  # one step = 3 stages
    impl_table = DOM_BYTES if uniform else DOM_BYTES_FIELDS
    if args.form != "fp64":
        impl_table = DOM_BYTES_FP32
    b_alg = B_ALG if uniform else B_ALG_FIELDS
    achieved = b_alg * cells / (dom_ms_per_stage / 1e3) / 1e9
    stage_ms = ms_max / args.steps / 3.0
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.form == "fp64" else "f32 stencils / f64 RK3 accumulation",
        "data": "synthetic",
        "config": config_of(args, case, world),
        "execution": "launched kernels" if args.no_graphs else "whole steps as CUDA graphs where eligible",
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / hbm,
                     "algorithmic_bytes_per_cell_stage": b_alg,
                     "traffic": (TRAFFIC_PER_CELL[dom] * cells
                                 if (uniform and args.form == "fp64" and dom in TRAFFIC_PER_CELL) else None),
                     "traffic_source": TRAFFIC_SOURCE,
                     "launch_ms": dom_ms_per_stage},
        "implementation_bytes": {"bytes_per_cell": impl_table.get(dom, b_alg),
                                 "gbs": impl_table.get(dom, b_alg) * cells / (dom_ms_per_stage / 1e3) / 1e9,
                                 "note": "fields this implementation's kernels of the family read and write "
                                         "once each per stage"},
        "stage_roofline": {"bytes_per_cell_stage": b_alg, "achieved_gbs": b_alg * cells / (stage_ms / 1e3) / 1e9,
                           "frac": b_alg * cells / (stage_ms / 1e3) / 1e9 / hbm},
        "kernel_ms_per_stage": {k: fam[k][0] / 3.0 for k in fam},
        "fp64_flops": ({"flop_per_cell_stage": FP64_FLOP_PER_CELL_STAGE[args.workload],
                        "achieved_tflops": FP64_FLOP_PER_CELL_STAGE[args.workload] * value / 1e3,
                        "source": FLOP_SOURCE} if args.form == "fp64" else None),
        "e2e": {"value": e2e_val, "unit": METRIC, "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
                "steps": e2e_steps, "api": "ocfd_b200_advance_host"},
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    if want_learned:
        line["learned"] = learned_leg(args, case, dev, ref_cons, ms, steps_done)
    return line


# Bytes per cell that this implementation's kernels of each family move in
# one stage, every field they touch counted once (reported beside the
# roofline, which uses the stage's algorithmic bytes, B_ALG); uniform grid,
# metrics constants:
#   inviscid_sweeps: each of the x, y, z sweeps reads d,u,v,w,T; x writes du
#                    (5), y and z read and write du (10 each)      -> 40 words
#   viscous_rk_update: Ev kernel reads u,v,w,T, writes 12 Ev; divergence +
#                    RK kernel reads 12 Ev, du, fn, f and writes f and
#                    d,u,v,w,T                                     -> 53 words
#   sensor: d,T in, three int8 flags out                           -> 19 bytes
DOM_BYTES = {
    "inviscid_sweeps": 40 * 8.0,
    "viscous_rk_update": 53 * 8.0,
    "ghost_fill": 0.0,
    "sensor": 19.0,
}

# Grids whose metrics are fields (the ramp): the sweeps also read the
# direction's 3 metrics at every split point and Ajac per cell (+4 words per
# direction), k_vis_ev reads 9 metrics and Ajac, k_vis_div Ajac (+11 words);
# the stage-level bound adds the 10 metric fields (200 B per cell-stage).
DOM_BYTES_FIELDS = {
    "inviscid_sweeps": (40 + 12) * 8.0,
    "viscous_rk_update": (53 + 11) * 8.0,
    "ghost_fill": 0.0,
    "sensor": 19.0,
}
B_ALG_FIELDS = 200.0

# The precision form (uniform grids): FP32 primitives, du and Ev, FP64 f, fn:
#   inviscid_sweeps: 40 FP32 words                                 -> 160 B
#   viscous_rk_update: u,v,w,T in, 12 Ev out and in, du in (FP32, 33 words),
#                    fn, f in and f out (FP64, 15 words), d,u,v,w,T out (FP32)
#                                                                  -> 272 B
#   sensor / learned switch: d,T in (FP32), three int8 flags out   -> 11 B
DOM_BYTES_FP32 = {
    "inviscid_sweeps": 160.0,
    "viscous_rk_update": 272.0,
    "ghost_fill": 0.0,
    "sensor": 11.0,
}

SWITCH_MODEL = os.path.join(os.path.dirname(os.path.abspath(__file__)), "opencfd-scu_b200", "ocfd_b200", "data",
                            "switch_c1c3.npz")

# Measured DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per cell
# for one stage's launches of each family, from one ncu capture of the same
# kernels at 160^3 (profiles/stage_traffic_iso160.txt); the traffic scales with
# the cells processed, so the bench line reports it times the cells of a launch.
TRAFFIC_PER_CELL = {
    "inviscid_sweeps": 304.6,       # 3 sweeps + 3 fix-ups
    "viscous_rk_update": 385.6,     # k_vis_ev + k_vis_div (Ev ghost fill not captured)
}
TRAFFIC_SOURCE = "ncu capture at 160^3 scaled by cells (profiles/stage_traffic_iso160.txt)"

# FP64 operations executed per cell and stage (2 x DFMA + DADD + DMUL, counted
# by ncu over one stage's kernels: profiles/fp64_flops_iso160_tgv128_ramp256.txt);
# times the measured rate, the FP64 rate the whole stage sustains.  The hybrid
# count depends on how many faces the sensor flags (isotropic turbulence: UP7
# almost everywhere).
FP64_FLOP_PER_CELL_STAGE = {"iso": 2353.0, "tgv": 7353.0, "ramp": 10712.0}
FLOP_SOURCE = "ncu executed FP64 instructions per stage (profiles/fp64_flops_iso160_tgv128_ramp256.txt)"


def run_reference(args, rank, world):
    """The reference's own CUDA build on the same workload (rank 0 only):
    the same case, W warm-up steps and exactly K timed steps."""
    if rank != 0:
        return None
    from oracle import ref_runner
    n = args.n
    case = make_case(args.workload, n)
    if not ref_runner.available():
        c = cpu_baseline(args.workload, max(8, n // 4))
        return {"impl": "reference", "metric": METRIC, "value": c["value"], "unit": METRIC,
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
                "config": config_of(args, case, world),
                "note": "reference build missing; CPU oracle port timed instead",
                "cpu_baseline": c, "e2e": {"value": c["value"], "unit": METRIC,
                                            "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    ref_steps = args.ref_steps if args.ref_steps > 0 else args.steps
    secs, interval, _ = ref_runner.time_steps(case, args.warmup, ref_steps)
    v = cells_of(case) * 3 * ref_steps / secs / 1e9
    return {"impl": "reference", "metric": METRIC, "value": v, "unit": METRIC, "n_gpus": world,
            "steps": ref_steps, "warmup": args.warmup, "ms_per_step": secs * 1e3 / ref_steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": config_of(args, case, world),
            "execution": "reference sources, nvcc -O3 sm_100a, single-rank MPI shim",
            "timing": (f"the reference's own MPI_Wtime interval prints every {interval} steps; "
                       f"the {ref_steps // interval} intervals after the {args.warmup} warm-up steps summed"),
            "cpu_baseline": {"value": v, "unit": METRIC, "cores": 1, "kind": "reference",
                             "sample": f"{ref_steps} steps of the reference CUDA build on 1 B200, "
                                       f"driven by 1 host thread"},
            "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", choices=tuple(WORKLOADS), default="iso")
    ap.add_argument("--form", choices=("fp64", "fp32", "fp32-learned"), default="fp64",
                    help="fp64: the plain path; fp32: FP32 stencils with FP64 RK3 accumulation; "
                         "fp32-learned: that with the learned scheme switch")
    ap.add_argument("--n", type=int, default=0,
                    help="grid size (iso, tgv: n^3; ramp: 4n x n x n/2); 0 = the configuration's own")
    ap.add_argument("--decomp", choices=("replicas", "z"), default="replicas",
                    help="N > 1: independent replicas, or the z slabs of one grid (ghost planes over NCCL)")
    ap.add_argument("--no-graphs", action="store_true",
                    help="launch every kernel one by one instead of replaying whole steps as CUDA graphs")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--ref-steps", type=int, default=0,
                    help="timed steps of the reference arm (0: the same as --steps)")
    ap.add_argument("--no-learned", dest="learned", action="store_false",
                    help="skip the precision-form and learned-switch legs of the default run")
    ap.add_argument("--cpu-sample", type=int, default=96)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.n <= 0:
        args.n = default_n(args.workload)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if world > 1:
        import torch
        import torch.distributed as tdist
        from datetime import timedelta
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        tdist.init_process_group("nccl", timeout=timedelta(seconds=600))
        dist = tdist

    if args.impl == "reference":
        line = run_reference(args, rank, world)
    else:
        line = run_ours(args, rank, world, dist)
        if line is not None and not args.no_cpu_baseline:
            sample = {"iso": args.cpu_sample, "tgv": args.cpu_sample, "ramp": args.cpu_sample // 2}[args.workload]
            line["cpu_baseline"] = cpu_baseline(args.workload, sample)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
