"""Run the reference's own CUDA build (oracle/_ref/opencfd-scu.out) on a case.

TEST / BENCH INFRASTRUCTURE ONLY.  The binary is compiled from the reference
sources by oracle/ref.mk; this module only writes the reference's input files
(opencfd-scu.in, opencfd.dat, OCFD3d-Jacobi.dat), runs it in a scratch
directory and parses what it prints or saves.
"""
from __future__ import annotations

import math
import os
import re
import resource
import shutil
import subprocess
import sys
import tempfile
import time
from typing import Optional, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
REF_BIN = os.path.join(HERE, "_ref", "opencfd-scu.out")
# the reference's program with its RHS-path calls served by libocfd_b200 (oracle/dropin.mk)
DROPIN_BIN = os.path.join(HERE, "_ref", "dropin", "opencfd-scu-dropin.out")

sys.path.insert(0, os.path.join(ROOT, "opencfd-scu_b200"))
from ocfd_b200 import formats  # noqa: E402


def _big_stack():
    # The reference's host halo exchange keeps four LAP*n*n double arrays on
    # the stack (src/OCFD_mpi.c:304-306): 8 MB at 256^3, past the default
    # limit.  Raise the child's soft limit to its hard limit.
    soft, hard = resource.getrlimit(resource.RLIMIT_STACK)
    try:
        resource.setrlimit(resource.RLIMIT_STACK, (hard, hard))
    except (ValueError, OSError):
        pass


def available(binary: str = REF_BIN) -> bool:
    return os.path.exists(binary) and os.access(binary, os.X_OK)


def _write_inputs(case, workdir: str) -> None:
    formats.write_config(os.path.join(workdir, "opencfd-scu.in"), case.cfg)
    formats.write_field_file(os.path.join(workdir, "opencfd.dat"), case.prims, 0, 0.0)
    # 13 fields: the metrics themselves; 3 fields: mesh coordinates, which
    # the reference turns into metrics when OCFD3d-Jacobi.dat is absent
    name = "OCFD3d-Mesh.dat" if len(case.metrics) == 3 else "OCFD3d-Jacobi.dat"
    formats.write_metric_file(os.path.join(workdir, name), case.metrics)
    inlet = getattr(case, "inlet", None)
    if inlet is not None:
        formats.write_inlet_file(os.path.join(workdir, "flow1d-inlet.dat"), inlet)


def run_and_read(case, nsteps: int, timeout: float = 900.0, binary: str = REF_BIN):
    """Run nsteps steps and return (prims[5,nz,ny,nx], Istep, tt, wall_s, stdout)."""
    cfg = case.cfg
    cfg.set_steps(nsteps)
    cfg.kstep_save = nsteps
    cfg.kstep_show = 10 ** 8
    wd = tempfile.mkdtemp(prefix="ocfd_ref_")
    try:
        _write_inputs(case, wd)
        t0 = time.time()
        p = subprocess.run([binary], cwd=wd, capture_output=True, text=True, timeout=timeout,
                           preexec_fn=_big_stack)
        wall = time.time() - t0
        if p.returncode != 0:
            raise RuntimeError(f"reference exited {p.returncode}:\n{p.stdout[-3000:]}\n{p.stderr[-3000:]}")
        fields, istep, tt = formats.read_field_file(os.path.join(wd, "OCFD%08d.dat" % nsteps),
                                                    case.shape)
        return np.stack(fields), istep, tt, wall, p.stdout
    finally:
        shutil.rmtree(wd, ignore_errors=True)


_INTERVAL = re.compile(r"^(\d+) steps GPU time ([0-9.eE+-]+)", re.M)


def time_steps(case, warmup: int, steps: int, timeout: float = 1800.0) -> Tuple[float, int, str]:
    """Seconds for exactly `steps` RK3 steps after exactly `warmup` steps, from
    the reference's own MPI_Wtime interval print (src/OCFD_NS_Solver.cu:104-153).
    The print interval is gcd(warmup, steps); the intervals after the warm-up
    are summed (each interval excludes the analysis the print itself runs).
    Returns (seconds, interval, stdout)."""
    cfg = case.cfg
    interval = math.gcd(max(1, warmup), steps)
    cfg.set_steps(warmup + steps)
    cfg.kstep_show = interval
    cfg.kstep_save = 10 ** 8
    wd = tempfile.mkdtemp(prefix="ocfd_ref_")
    try:
        _write_inputs(case, wd)
        p = subprocess.run([REF_BIN], cwd=wd, capture_output=True, text=True, timeout=timeout,
                           preexec_fn=_big_stack)
        if p.returncode != 0:
            raise RuntimeError(f"reference exited {p.returncode}:\n{p.stdout[-3000:]}\n{p.stderr[-3000:]}")
        m = _INTERVAL.findall(p.stdout)
        need = steps // interval
        if len(m) < need:
            raise RuntimeError(f"{len(m)} interval prints in the reference output, {need} needed:\n"
                               + p.stdout[-3000:])
        return sum(float(t) for _, t in m[-need:]), interval, p.stdout
    finally:
        shutil.rmtree(wd, ignore_errors=True)
