"""Generate the golden fixtures that pin the oracle to the reference.

Runs the reference's own CUDA build (oracle/_ref/opencfd-scu.out, made by
``make -f oracle/ref.mk``) on small synthetic cases, on a B200, through the
reference's own file interface (opencfd-scu.in, opencfd.dat,
OCFD3d-Jacobi.dat -> OCFD%08d.dat), and stores inputs and outputs as .npz.

    python tests/golden/make_golden.py --out <directory>

(default: a new temporary directory, printed at the end; copy the .npz files
that should become fixtures into tests/golden/).

Each case is run twice so that a non-deterministic reference result (the
shared-memory race of the characteristic kernels) shows up as a difference
between the runs; both outputs are stored.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "opencfd-scu_b200"))

from ocfd_b200 import cases  # noqa: E402

sys.path.insert(0, ROOT)
from oracle import ref_runner  # noqa: E402


def golden_cases():
    """(name, Case, nsteps) -- small enough that the oracle finishes in seconds."""
    out = []
    tg = cases.taylor_green(16, seed=11)
    out.append(("tgv16_weno7_cd6", tg, 10))
    iso = cases.isotropic_turbulence(16, seed=5, charteric=1)
    out.append(("iso16_hybrid_char", iso, 10))
    iso0 = cases.isotropic_turbulence(16, seed=6, charteric=0)
    out.append(("iso16_hybrid_nochar", iso0, 4))
    rs = cases.random_smooth_case(19, 13, 11, seed=3, scheme_invis="WENO7", curvilinear=True)
    out.append(("rnd19x13x11_weno7_curv", rs, 4))
    sh = cases.random_smooth_case(13, 17, 11, seed=4, scheme_invis="SCHEME_HYBRIDAUTO",
                                  charteric=1, shock=True, curvilinear=True)
    sh.cfg.hy_dp_intv = (0.01, 0.2)
    out.append(("rnd13x17x11_hybrid_char_shock", sh, 4))
    for sch in ("UP7", "WENO5", "WENO7_SYMBO", "WENO7_SYMBO_LIM", "NND2",
                "OMP6_HR", "OMP6_LD", "OMP6_CD8"):
        c = cases.random_smooth_case(12, 11, 10, seed=21, scheme_invis=sch, shock=True)
        out.append((f"rnd12x11x10_{sch.lower()}", c, 3))
    c = cases.random_smooth_case(12, 11, 10, seed=22, scheme_invis="WENO7", scheme_vis="CD8")
    out.append(("rnd12x11x10_weno7_cd8", c, 3))
    for sch in ("WENO7_SYMBO", "WENO7_SYMBO_LIM"):
        c = cases.random_smooth_case(12, 11, 10, seed=23, scheme_invis=sch, charteric=1, shock=True)
        out.append((f"rnd12x11x10_{sch.lower()}_char", c, 3))
    out.extend(bounded_cases())
    out.extend(mesh_cases())
    out.extend(filter_cases())
    out.extend(ramp_cases())
    return out


def ramp_cases():
    """The compression-corner boundary family (IBC 108) on a small ramp mesh:
    isothermal wall with the inflow profile file, hybrid scheme and filter;
    adiabatic wall with time-dependent wall blowing; the default profile;
    blowing with random-phase spanwise modes."""
    out = []
    c = cases.ramp_case(32, 20, 8, seed=91)
    out.append(("ramp32x20x8_bc108_tw_filter", c, 3))
    c = cases.ramp_case(30, 18, 8, seed=92, tw=-1.0, epsl=0.05, beta=40.0, mtmax=3,
                        scheme_invis="WENO7", charteric=0, filters=())
    c.cfg.bc_rpara = (-1.0, 0.05, 4.0, 30.0, 40.0, 0.0, 30.0, 8.0)
    out.append(("ramp30x18x8_bc108_adiabatic_blowing", c, 3))
    c = cases.ramp_case(28, 18, 8, seed=93, filters=())
    c.cfg.bc_npara = (0, 0, 0, 0)            # INLET_BOUNDARY 0: d = u = T = 1, v = 0
    c.inlet = None
    out.append(("ramp28x18x8_bc108_default_inlet", c, 3))
    # three spanwise modes with phases from rand() (MZMAX = 3), a span of 8
    # cells over SLZ = 2 so that the modes vary across it
    c = cases.ramp_case(30, 18, 8, seed=94, tw=-1.0, epsl=0.05, beta=40.0, mtmax=3,
                        scheme_invis="WENO7", charteric=0, filters=())
    c.cfg.bc_npara = (3, 3, 1, 0)
    c.cfg.bc_rpara = (-1.0, 0.05, 4.0, 30.0, 40.0, 0.0, 30.0, 2.0)
    out.append(("ramp30x18x8_bc108_mz3_blowing", c, 3))
    return out


def filter_cases():
    """The shock-capturing filter after each step (FILTER_NPARA / FILTER_RPARA,
    scheme 2) on the hybrid scheme, whose sensor provides the pressure it
    reads: partial ranges, the z pass that filters along y (A-3), a closed
    direction (ranges kept 6/5 cells from the faces), two filters with
    different intervals and a time limit."""
    out = []

    def hyb(nx, ny, nz, seed, **kw):
        c = cases.random_smooth_case(nx, ny, nz, seed=seed, scheme_invis="SCHEME_HYBRIDAUTO", charteric=1,
                                     shock=True, **kw)
        c.cfg.hy_dp_intv = (0.01, 0.2)
        return c
    # z pass without the y pass: the y ghosts are not exchanged then, so the
    # y range keeps every read inside the box (rows 3..18 of 22); the z pass
    # reaches rows 3..14 only
    c = hyb(18, 22, 13, 71)
    c.cfg.filters = (((1, 1, 0, 1, 0, 18, 3, 19, 0, 13, 2), (1.0, 1e-5, 10.0)),)
    out.append(("fil18x22x13_hybrid_x_zquirk", c, 3))
    c = hyb(19, 14, 13, 72, iperiodic=(0, 1, 1), dif_bound=(1, 1, 0, 0, 0, 0))
    c.cfg.filters = (((1, 1, 1, 1, 0, 19, 0, 14, 0, 13, 2), (0.8, 1e-5, 10.0)),)
    out.append(("fil19x14x13_hybrid_xyz_bounded", c, 3))
    c = hyb(17, 18, 13, 73)
    c.cfg.filters = (((2, 1, 0, 0, 0, 17, 0, 18, 0, 13, 2), (1.0, 1e-5, 10.0)),
                     ((1, 0, 1, 0, 3, 12, 2, 16, 1, 12, 2), (0.7, 2e-5, 0.003)))
    out.append(("fil17x18x13_hybrid_two_filters", c, 3))
    return out


def mesh_cases():
    """Metrics computed by the solver from mesh coordinates (OCFD3d-Mesh.dat,
    JAC_BOUND = 1 1 1) on a skewed, stretched grid, x and y closed, z
    periodic."""
    out = []
    c = cases.mesh_case(14, 13, 12, seed=51, scheme_invis="WENO7")
    out.append(("mesh14x13x12_weno7", c, 3))
    c = cases.mesh_case(13, 14, 12, seed=52, scheme_invis="SCHEME_HYBRIDAUTO", charteric=1, shock=True,
                        non_ref=(1, 0, 0, 1, 0, 0))
    c.cfg.hy_dp_intv = (0.01, 0.2)
    out.append(("mesh13x14x12_hybrid_char_nonref", c, 3))
    c = cases.mesh_case(12, 12, 11, seed=53, scheme_invis="UP7", jac_bound=(1, 1, 1),
                        dif_bound=(1, 1, 1, 1, 0, 0))
    c.cfg.scheme_vis = "CD8"
    out.append(("mesh12x12x11_up7_cd8", c, 3))
    return out


def bounded_cases():
    """Non-periodic directions with the boundary closures (DIF_BOUND = 1) and
    non-reflecting faces, no boundary-condition family (IBC = 0): both faces
    closed (flag 7/8/9), one face closed (1..6), and closures on a periodic
    direction, for component-wise and characteristic kernels."""
    out = []
    both = dict(iperiodic=(0, 0, 0), dif_bound=(1, 1, 1, 1, 1, 1))
    one = dict(iperiodic=(0, 0, 0), dif_bound=(1, 0, 0, 1, 1, 0), non_ref=(1, 0, 0, 1, 0, 0))
    for sch in ("UP7", "WENO7", "WENO5", "NND2", "WENO7_SYMBO", "OMP6_HR"):
        c = cases.random_smooth_case(14, 13, 12, seed=31, scheme_invis=sch, **both)
        out.append((f"bnd14x13x12_{sch.lower()}_both", c, 3))
    c = cases.random_smooth_case(14, 13, 12, seed=32, scheme_invis="UP7", **one)
    out.append(("bnd14x13x12_up7_one_nonref", c, 3))
    c = cases.random_smooth_case(14, 13, 12, seed=33, scheme_invis="WENO7", scheme_vis="CD8", **one)
    out.append(("bnd14x13x12_weno7_cd8_one_nonref", c, 3))
    for tag, kw in (("both", both), ("one_nonref", one)):
        c = cases.random_smooth_case(13, 14, 12, seed=34, scheme_invis="SCHEME_HYBRIDAUTO",
                                     charteric=1, shock=True, **kw)
        c.cfg.hy_dp_intv = (0.01, 0.2)
        out.append((f"bnd13x14x12_hybrid_char_{tag}", c, 3))
        c = cases.random_smooth_case(12, 13, 11, seed=35, scheme_invis="WENO7_SYMBO_LIM",
                                     charteric=1, shock=True, **kw)
        out.append((f"bnd12x13x11_symbo_lim_char_{tag}", c, 3))
    c = cases.random_smooth_case(13, 12, 11, seed=36, scheme_invis="SCHEME_HYBRIDAUTO", charteric=1,
                                 shock=True, curvilinear=True, iperiodic=(1, 0, 1),
                                 dif_bound=(1, 1, 1, 1, 0, 0), non_ref=(0, 1, 1, 0, 0, 0))
    c.cfg.hy_dp_intv = (0.01, 0.2)
    out.append(("bnd13x12x11_hybrid_char_curv_mixed", c, 3))
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default="", help="output directory (default: a new temporary directory)")
    ap.add_argument("--only", default="")
    args = ap.parse_args(argv)
    if not ref_runner.available():
        raise SystemExit(f"{ref_runner.REF_BIN} missing: build it with make -f oracle/ref.mk")
    if not args.out:
        import tempfile
        args.out = tempfile.mkdtemp(prefix="ocfd_golden_")
    os.makedirs(args.out, exist_ok=True)
    summary = {}
    for name, case, nsteps in golden_cases():
        if args.only and args.only not in name:
            continue
        runs = []
        for rep in range(2):
            out, istep, tt, wall, log = ref_runner.run_and_read(case, nsteps)
            runs.append(out)
        same = bool(np.array_equal(runs[0], runs[1]))
        c = case.cfg
        extra = {} if case.inlet is None else {"inlet": np.asarray(case.inlet)}
        np.savez_compressed(
            os.path.join(args.out, name + ".npz"), **extra,
            prims_in=np.stack(case.prims), metrics=np.stack(case.metrics),
            out_run0=runs[0], out_run1=runs[1], nsteps=nsteps, istep=istep, tt=tt,
            config=json.dumps({k: (list(v) if isinstance(v, tuple) else v)
                               for k, v in c.__dict__.items()}))
        summary[name] = {"nsteps": nsteps, "repeat_bitwise_equal": same,
                         "max_abs_diff_between_runs": float(np.max(np.abs(runs[0] - runs[1]))),
                         "wall_s": wall}
        print(name, summary[name], flush=True)
    with open(os.path.join(args.out, "summary.json"), "w") as fh:
        json.dump(summary, fh, indent=1)
    print("fixtures written to", args.out, flush=True)


if __name__ == "__main__":
    main()
