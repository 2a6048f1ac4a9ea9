"""ctypes wrapper of the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py as the checker.  The product never
imports this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import List, Optional, Sequence, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")


class OroConfig(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("iperiodic", ctypes.c_int * 3),
        ("jac_bound", ctypes.c_int * 3),
        ("d0_bound", ctypes.c_int * 6),
        ("non_ref", ctypes.c_int * 6),
        ("scheme_invis", ctypes.c_int),
        ("scheme_vis", ctypes.c_int),
        ("charteric", ctypes.c_int),
        ("hy_style", ctypes.c_int),
        ("hy_dp_intv", ctypes.c_double * 2),
        ("re", ctypes.c_double), ("ama", ctypes.c_double), ("gamma", ctypes.c_double),
        ("pr", ctypes.c_double), ("t_ref", ctypes.c_double), ("epsl_sw", ctypes.c_double),
        ("dt", ctypes.c_double),
        ("weno_tv_limiter", ctypes.c_double), ("weno_tv_max", ctypes.c_double),
        ("nthreads", ctypes.c_int),
        ("hy_nochar_fixed", ctypes.c_int),
        ("ibc", ctypes.c_int),
        ("bc_npara", ctypes.c_int * 4),
        ("bc_rpara", ctypes.c_double * 8),
        ("nfilter", ctypes.c_int),
        ("filter_ipara", (ctypes.c_int * 11) * 8),
        ("filter_rpara", (ctypes.c_double * 3) * 8),
    ]


_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        D = ctypes.POINTER(ctypes.c_double)
        L.oro_create.restype = P
        L.oro_create.argtypes = [ctypes.POINTER(OroConfig)]
        L.oro_destroy.argtypes = [P]
        L.oro_set_metrics.argtypes = [P, D]
        L.oro_set_mesh.argtypes = [P, D]
        L.oro_set_inlet.argtypes = [P, D]
        L.oro_get_metrics.argtypes = [P, D]
        L.oro_negative_jacobian.argtypes = [P]
        L.oro_negative_jacobian.restype = ctypes.c_int
        L.oro_set_primitives.argtypes = [P, D, ctypes.c_int, ctypes.c_double]
        for name in ("oro_prepare", "oro_get_duvwT", "oro_bc", "oro_get_amu",
                     "oro_swap_time_levels"):
            getattr(L, name).argtypes = [P]
        for name in ("oro_du_comput", "oro_time_advance", "oro_step"):
            getattr(L, name).argtypes = [P, ctypes.c_int]
        for name in ("oro_get_primitives", "oro_get_pressure", "oro_get_conserved",
                     "oro_get_conserved_n", "oro_get_du", "oro_q_criterion"):
            getattr(L, name).argtypes = [P, D]
        IP = ctypes.POINTER(ctypes.c_int)
        L.oro_get_flags.argtypes = [P, IP, IP, IP]
        L.oro_libc_rand.argtypes = [ctypes.c_int, IP]
        L.oro_istep.argtypes = [P]
        L.oro_istep.restype = ctypes.c_int
        L.oro_tt.argtypes = [P]
        L.oro_tt.restype = ctypes.c_double
        for name in ("oro_weno7_p", "oro_weno7_m", "oro_weno5_p", "oro_weno5_m",
                     "oro_up7_p", "oro_up7_m", "oro_nnd2_p", "oro_nnd2_m",
                     "oro_cd6", "oro_cd8"):
            getattr(L, name).argtypes = [D]
            getattr(L, name).restype = ctypes.c_double
        for name in ("oro_omp6_p", "oro_omp6_m"):
            getattr(L, name).argtypes = [ctypes.c_int, D]
            getattr(L, name).restype = ctypes.c_double
        for name in ("oro_weno7_symbo_p", "oro_weno7_symbo_m"):
            getattr(L, name).argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, D]
            getattr(L, name).restype = ctypes.c_double
        L.oro_sw_split.argtypes = [ctypes.c_double] * 10 + [D]
        L.oro_char_matrices.argtypes = [ctypes.c_double] * 8 + [D, D]
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def make_config(cfg, nthreads: int = 0, hy_nochar_fixed: int = 3) -> OroConfig:
    """OroConfig from an ocfd_b200.formats.CaseConfig."""
    c = OroConfig()
    c.nx, c.ny, c.nz = cfg.nx, cfg.ny, cfg.nz
    c.iperiodic[:] = list(cfg.iperiodic)
    c.jac_bound[:] = list(cfg.jac_bound)
    c.d0_bound[:] = list(cfg.dif_bound)
    c.non_ref[:] = list(cfg.non_ref)
    c.scheme_invis = cfg.scheme_invis_id
    c.scheme_vis = cfg.scheme_vis_id
    c.charteric = cfg.charteric
    c.hy_style = cfg.hy_style
    c.hy_dp_intv[:] = list(cfg.hy_dp_intv)
    c.re, c.ama, c.gamma, c.pr = cfg.re, cfg.ama, cfg.gamma, cfg.pr
    c.t_ref, c.epsl_sw, c.dt = cfg.t_ref, cfg.epsl_sw, cfg.dt
    c.weno_tv_limiter, c.weno_tv_max = 5.0, 0.2
    c.nthreads = nthreads
    c.hy_nochar_fixed = hy_nochar_fixed
    c.ibc = int(getattr(cfg, "ibc", 0))
    for t, v in enumerate(list(getattr(cfg, "bc_npara", ()) or ())[:4]):
        c.bc_npara[t] = int(v)
    for t, v in enumerate(list(getattr(cfg, "bc_rpara", ()) or ())[:8]):
        c.bc_rpara[t] = float(v)
    filters = list(getattr(cfg, "filters", ()) or ())[:8]
    c.nfilter = len(filters)
    for n, (ip, rp) in enumerate(filters):
        for t in range(11):
            c.filter_ipara[n][t] = int(ip[t])
        for t in range(3):
            c.filter_rpara[n][t] = float(rp[t])
    return c


class Oracle:
    """One solver instance; mirrors the reference driver's call sequence.

    hy_nochar_fixed: scheme flag that components 1-4 of the non-characteristic
    hybrid kernels use.  The reference reads an uninitialised variable there
    (src/OCFD_Schemes_hybrid_auto.cu:907,1005); its sm_100a build behaves as
    flag 3 (WENO5), measured against the golden fixtures, hence the default.
    0 gives the face flag to every component."""

    def __init__(self, cfg, prims: Sequence[np.ndarray], metrics: Sequence[np.ndarray],
                 nthreads: int = 0, istep: int = 0, tt: float = 0.0, hy_nochar_fixed: int = 3,
                 inlet=None):
        if cfg.hy_style != 2 and cfg.scheme_invis_id == 310:
            raise NotImplementedError("oracle covers HY_STYLE=2 only")
        self.cfg = cfg
        self._c = make_config(cfg, nthreads, hy_nochar_fixed)
        self.L = lib()
        self.h = self.L.oro_create(ctypes.byref(self._c))
        self.shape = (cfg.nz, cfg.ny, cfg.nx)
        # 13 fields: OCFD3d-Jacobi.dat content; 3 fields: OCFD3d-Mesh.dat
        # coordinates, from which the metrics are computed
        met = np.ascontiguousarray(np.stack([np.asarray(m, np.float64) for m in metrics]))
        if met.shape[0] == 3:
            self.L.oro_set_mesh(self.h, _dp(met))
            if self.L.oro_negative_jacobian(self.h):
                raise ValueError("negative Jacobian (the reference stops here)")
        else:
            self.L.oro_set_metrics(self.h, _dp(met))
        if inlet is not None:           # IBC 108 profile [4][ny]
            ub = np.ascontiguousarray(np.asarray(inlet, np.float64))
            self.L.oro_set_inlet(self.h, _dp(ub))
        pr = np.ascontiguousarray(np.stack([np.asarray(p, np.float64) for p in prims]))
        self.L.oro_set_primitives(self.h, _dp(pr), istep, tt)
        self.L.oro_prepare(self.h)

    def close(self):
        if self.h:
            self.L.oro_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n: int = 1):
        self.L.oro_step(self.h, n)

    def swap(self):
        self.L.oro_swap_time_levels(self.h)

    def du_comput(self, krk: int):
        self.L.oro_du_comput(self.h, krk)

    def time_advance(self, krk: int):
        self.L.oro_time_advance(self.h, krk)

    def get_duvwT(self):
        self.L.oro_get_duvwT(self.h)

    def bc(self):
        self.L.oro_bc(self.h)

    def get_amu(self):
        self.L.oro_get_amu(self.h)

    def _get5(self, fn) -> np.ndarray:
        out = np.empty((5,) + self.shape, dtype=np.float64)
        fn(self.h, _dp(out))
        return out

    def primitives(self) -> np.ndarray:
        return self._get5(self.L.oro_get_primitives)

    def conserved(self) -> np.ndarray:
        return self._get5(self.L.oro_get_conserved)

    def conserved_n(self) -> np.ndarray:
        return self._get5(self.L.oro_get_conserved_n)

    def du(self) -> np.ndarray:
        return self._get5(self.L.oro_get_du)

    def metrics(self) -> np.ndarray:
        out = np.empty((13,) + self.shape, dtype=np.float64)
        self.L.oro_get_metrics(self.h, _dp(out))
        return out

    def pressure(self) -> np.ndarray:
        out = np.empty(self.shape, dtype=np.float64)
        self.L.oro_get_pressure(self.h, _dp(out))
        return out

    def q_criterion(self) -> np.ndarray:
        """Q of the current primitives (get_Q, src/OCFD_ana.cu:317-456)."""
        out = np.empty(self.shape, dtype=np.float64)
        self.L.oro_q_criterion(self.h, _dp(out))
        return out

    def flags(self) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
        nz, ny, nx = self.shape
        sx = np.empty((nz, ny, nx + 1), dtype=np.int32)
        sy = np.empty((nz, ny + 1, nx), dtype=np.int32)
        sz = np.empty((nz + 1, ny, nx), dtype=np.int32)
        IP = ctypes.POINTER(ctypes.c_int)
        self.L.oro_get_flags(self.h, sx.ctypes.data_as(IP), sy.ctypes.data_as(IP),
                             sz.ctypes.data_as(IP))
        return sx, sy, sz

    @property
    def istep(self) -> int:
        return self.L.oro_istep(self.h)

    @property
    def tt(self) -> float:
        return self.L.oro_tt(self.h)


def libc_rand(n: int) -> np.ndarray:
    """The first n draws of the C library's rand() from its initial state,
    as the oracle restates it (the spanwise phases of IBC 108, MZMAX > 0)."""
    out = np.zeros(n, dtype=np.int32)
    lib().oro_libc_rand(int(n), out.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
    return out


def point(name: str, stencil: Sequence[float], *args) -> float:
    a = np.ascontiguousarray(np.asarray(stencil, dtype=np.float64))
    return getattr(lib(), "oro_" + name)(*args, _dp(a))


def sw_split(d, u, v, w, cc, a1, a2, a3, gamma=1.4, eps=0.0) -> np.ndarray:
    out = np.empty(10)
    lib().oro_sw_split(d, u, v, w, cc, a1, a2, a3, gamma, eps, _dp(out))
    return out


def char_matrices(u1, v1, w1, c1, a1, a2, a3, gamma=1.4):
    Lm = np.empty(25)
    Rm = np.empty(25)
    lib().oro_char_matrices(u1, v1, w1, c1, a1, a2, a3, gamma, _dp(Lm), _dp(Rm))
    return Lm.reshape(5, 5), Rm.reshape(5, 5)
