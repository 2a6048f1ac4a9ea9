"""ctypes binding of libocfd_b200.so (include/ocfd_b200.h).

The library is the product; this module only marshals numpy arrays (host)
or raw device pointers across the C ABI.  Loading fails loudly when the
shared object is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional, Sequence, Tuple

import numpy as np

from .formats import CaseConfig

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))   # opencfd-scu_b200/
LIB_PATH = os.path.join(PKG_DIR, "libocfd_b200.so")

OCFD_OK = 0
STATUS = {0: "ok", -1: "invalid argument", -2: "unsupported configuration", -3: "CUDA error",
          -4: "device out of memory", -5: "call out of order", -6: "no CUDA device"}
TIMER_COUNT = 8

# every function the header declares (the non-GPU tests check the exports)
EXPORTED = (
    "ocfd_b200_abi_version", "ocfd_b200_status_string", "ocfd_b200_last_error",
    "ocfd_b200_create", "ocfd_b200_destroy", "ocfd_b200_set_stream", "ocfd_b200_get_stream",
    "ocfd_b200_synchronize", "ocfd_b200_set_metrics", "ocfd_b200_set_metrics_device",
    "ocfd_b200_set_metric_mode", "ocfd_b200_uniform_metrics", "ocfd_b200_set_sweep_impl",
    "ocfd_b200_sweep_walks", "ocfd_b200_set_walk_threshold", "ocfd_b200_q_criterion", "ocfd_b200_time_average", "ocfd_b200_get_time_average", "ocfd_b200_set_viscous_impl", "ocfd_b200_set_precision", "ocfd_b200_slab_unique_id", "ocfd_b200_set_slab", "ocfd_b200_set_slab_host",
    "ocfd_b200_set_graphs", "ocfd_b200_graph_captures",
    "ocfd_b200_scheme_proportion", "ocfd_b200_mlp_nparam", "ocfd_b200_set_switch", "ocfd_b200_switch_stats", "ocfd_b200_switch_features",
    "ocfd_b200_mlp_last_error", "ocfd_b200_mlp_infer", "ocfd_b200_mlp_grad", "ocfd_b200_mlp_train",
    "ocfd_b200_set_mesh", "ocfd_b200_set_mesh_device", "ocfd_b200_get_metrics",
    "ocfd_b200_set_filter", "ocfd_b200_filtering", "ocfd_b200_set_time", "filtering", "ocfd_b200_set_bc",
    "ocfd_b200_set_primitives", "ocfd_b200_set_primitives_device", "ocfd_b200_step",
    "ocfd_b200_advance_host", "ocfd_b200_swap_time_levels", "ocfd_b200_du_comput",
    "ocfd_b200_time_advance", "ocfd_b200_get_duvwT", "ocfd_b200_bc",
    "ocfd_b200_get_primitives", "ocfd_b200_get_primitives_device", "ocfd_b200_get_conserved",
    "ocfd_b200_get_du", "ocfd_b200_get_flags", "ocfd_b200_get_time", "ocfd_b200_set_timing",
    "ocfd_b200_ana_residual", "ocfd_b200_check_state",
    "ocfd_b200_get_timing", "ocfd_b200_timer_name", "ocfd_b200_launch_count",
    "ocfd_b200_compat_bind", "ocfd_b200_field_means_noalloc", "du_comput", "OCFD_time_advance", "get_duvwT", "get_Amu",
    "OCFD_bc", "Set_Scheme_HybridAuto",
)


class Config(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("iperiodic", ctypes.c_int * 3),
        ("jac_bound", ctypes.c_int * 3),
        ("dif_bound", ctypes.c_int * 6),
        ("non_reflection", ctypes.c_int * 6),
        ("scheme_invis", ctypes.c_int),
        ("scheme_vis", ctypes.c_int),
        ("charteric", ctypes.c_int),
        ("hy_style", ctypes.c_int),
        ("hy_dp_intv", ctypes.c_double * 2),
        ("re", ctypes.c_double), ("ama", ctypes.c_double), ("gamma", ctypes.c_double),
        ("pr", ctypes.c_double), ("t_ref", ctypes.c_double), ("epsl_sw", ctypes.c_double),
        ("dt", ctypes.c_double),
        ("device", ctypes.c_int),
        ("hybrid_nochar_same_flag", ctypes.c_int),
    ]


class OcfdError(RuntimeError):
    def __init__(self, status: int, what: str, detail: str = ""):
        super().__init__(f"{what}: {STATUS.get(status, status)} {detail}".strip())
        self.status = status


_lib = None


def build(force: bool = False) -> str:
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-s", "-C", PKG_DIR], check=True)
    return LIB_PATH


def load(path: Optional[str] = None):
    """Load the shared library (never builds implicitly on a GPU box)."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise OSError(f"{path} not found: build it with `make -C opencfd-scu_b200` "
                      "(the CUDA library is required; there is no CPU fallback)")
    L = ctypes.CDLL(path)
    P = ctypes.c_void_p
    D = ctypes.POINTER(ctypes.c_double)
    I8 = ctypes.POINTER(ctypes.c_int8)
    F = ctypes.POINTER(ctypes.c_float)
    sig = {
        "ocfd_b200_abi_version": (ctypes.c_int, []),
        "ocfd_b200_status_string": (ctypes.c_char_p, [ctypes.c_int]),
        "ocfd_b200_last_error": (ctypes.c_char_p, [P]),
        "ocfd_b200_create": (ctypes.c_int, [ctypes.POINTER(Config), ctypes.POINTER(P)]),
        "ocfd_b200_destroy": (ctypes.c_int, [P]),
        "ocfd_b200_set_stream": (ctypes.c_int, [P, P]),
        "ocfd_b200_get_stream": (P, [P]),
        "ocfd_b200_synchronize": (ctypes.c_int, [P]),
        "ocfd_b200_set_metrics": (ctypes.c_int, [P, D]),
        "ocfd_b200_set_metrics_device": (ctypes.c_int, [P, P]),
        "ocfd_b200_set_mesh": (ctypes.c_int, [P, D]),
        "ocfd_b200_set_mesh_device": (ctypes.c_int, [P, P]),
        "ocfd_b200_get_metrics": (ctypes.c_int, [P, D]),
        "ocfd_b200_set_filter": (ctypes.c_int, [P, ctypes.c_int, ctypes.POINTER(ctypes.c_int), D]),
        "ocfd_b200_filtering": (ctypes.c_int, [P]),
        "ocfd_b200_set_time": (ctypes.c_int, [P, ctypes.c_int, ctypes.c_double]),
        "ocfd_b200_set_bc": (ctypes.c_int, [P, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.c_int, D,
                                            ctypes.c_int, D]),
        "filtering": (None, [D, D, D]),
        "ocfd_b200_set_metric_mode": (ctypes.c_int, [P, ctypes.c_int]),
        "ocfd_b200_uniform_metrics": (ctypes.c_int, [P]),
        "ocfd_b200_set_sweep_impl": (ctypes.c_int, [P, ctypes.c_int]),
        "ocfd_b200_sweep_walks": (ctypes.c_int, [P]),
        "ocfd_b200_set_walk_threshold": (ctypes.c_int, [P, ctypes.c_double]),
        "ocfd_b200_set_viscous_impl": (ctypes.c_int, [P, ctypes.c_int]),
        "ocfd_b200_q_criterion": (ctypes.c_int, [P, D]),
        "ocfd_b200_time_average": (ctypes.c_int, [P, ctypes.c_int]),
        "ocfd_b200_get_time_average": (ctypes.c_int, [P, D, ctypes.POINTER(ctypes.c_int)]),
        "ocfd_b200_set_precision": (ctypes.c_int, [P, ctypes.c_int]),
        "ocfd_b200_slab_unique_id": (ctypes.c_int, [ctypes.c_char_p]),
        "ocfd_b200_set_slab_host": (ctypes.c_int, [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                   ctypes.c_int, ctypes.c_int, SLAB_TRANSPORT, ctypes.c_void_p]),
        "ocfd_b200_set_graphs": (ctypes.c_int, [P, ctypes.c_int]),
        "ocfd_b200_graph_captures": (ctypes.c_longlong, [P]),
        "ocfd_b200_set_slab": (ctypes.c_int, [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_int, ctypes.c_int, ctypes.c_char_p]),
        "ocfd_b200_scheme_proportion": (ctypes.c_int, [P, D]),
        "ocfd_b200_mlp_nparam": (ctypes.c_int, []),
        "ocfd_b200_set_switch": (ctypes.c_int, [P, F, ctypes.c_int, ctypes.c_double]),
        "ocfd_b200_switch_stats": (ctypes.c_int, [P, ctypes.POINTER(ctypes.c_longlong)]),
        "ocfd_b200_switch_features": (ctypes.c_int, [P, ctypes.c_longlong, ctypes.c_longlong, F, F]),
        "ocfd_b200_mlp_last_error": (ctypes.c_char_p, []),
        "ocfd_b200_mlp_infer": (ctypes.c_int, [F, F, ctypes.c_longlong, F]),
        "ocfd_b200_mlp_grad": (ctypes.c_int, [F, F, F, ctypes.c_longlong, ctypes.c_float, F, D]),
        "ocfd_b200_mlp_train": (ctypes.c_int, [F, F, F, ctypes.c_longlong, ctypes.c_int, ctypes.c_int,
                                               ctypes.c_float, ctypes.c_float, ctypes.c_ulonglong, D]),
        "ocfd_b200_set_primitives": (ctypes.c_int, [P, D, ctypes.c_int, ctypes.c_double]),
        "ocfd_b200_set_primitives_device": (ctypes.c_int, [P, P, ctypes.c_int, ctypes.c_double]),
        "ocfd_b200_step": (ctypes.c_int, [P, ctypes.c_int]),
        "ocfd_b200_advance_host": (ctypes.c_int, [P, D, D, ctypes.c_int]),
        "ocfd_b200_swap_time_levels": (ctypes.c_int, [P]),
        "ocfd_b200_du_comput": (ctypes.c_int, [P, ctypes.c_int]),
        "ocfd_b200_time_advance": (ctypes.c_int, [P, ctypes.c_int]),
        "ocfd_b200_get_duvwT": (ctypes.c_int, [P]),
        "ocfd_b200_bc": (ctypes.c_int, [P]),
        "ocfd_b200_get_primitives": (ctypes.c_int, [P, D]),
        "ocfd_b200_get_primitives_device": (ctypes.c_int, [P, P]),
        "ocfd_b200_get_conserved": (ctypes.c_int, [P, D]),
        "ocfd_b200_get_du": (ctypes.c_int, [P, D]),
        "ocfd_b200_get_flags": (ctypes.c_int, [P, I8, I8, I8]),
        "ocfd_b200_get_time": (ctypes.c_int, [P, ctypes.POINTER(ctypes.c_int), D]),
        "ocfd_b200_set_timing": (ctypes.c_int, [P, ctypes.c_int]),
        "ocfd_b200_ana_residual": (ctypes.c_int, [P, ctypes.c_int, D]),
        "ocfd_b200_check_state": (ctypes.c_int, [P, ctypes.POINTER(ctypes.c_longlong),
                                                 ctypes.POINTER(ctypes.c_longlong), D]),
        "ocfd_b200_get_timing": (ctypes.c_int, [P, D, ctypes.POINTER(ctypes.c_longlong), ctypes.c_int]),
        "ocfd_b200_timer_name": (ctypes.c_char_p, [ctypes.c_int]),
        "ocfd_b200_launch_count": (ctypes.c_longlong, [P]),
        "ocfd_b200_compat_bind": (ctypes.c_int, [P]),
        "ocfd_b200_field_means_noalloc": (ctypes.c_int, [P, ctypes.c_int, ctypes.c_longlong, P, P]),
        "du_comput": (None, [ctypes.c_int]),
        "OCFD_time_advance": (None, [ctypes.c_int]),
        "get_duvwT": (None, []),
        "get_Amu": (None, []),
        "OCFD_bc": (None, []),
        "Set_Scheme_HybridAuto": (None, [P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _fp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _mlp_check(rc: int, what: str):
    if rc != 0:
        L = load()
        raise OcfdError(rc, f"{what}: {L.ocfd_b200_status_string(rc).decode()} "
                            f"({L.ocfd_b200_mlp_last_error().decode()})")


def mlp_nparam() -> int:
    return int(load().ocfd_b200_mlp_nparam())


def mlp_infer(params: np.ndarray, feat: np.ndarray) -> np.ndarray:
    """Logits of feature rows (n x 14) through the tensor-core network."""
    w = np.ascontiguousarray(params, np.float32)
    f = np.ascontiguousarray(feat, np.float32)
    out = np.empty(f.shape[0], np.float32)
    _mlp_check(load().ocfd_b200_mlp_infer(_fp(w), _fp(f), f.shape[0], _fp(out)), "mlp_infer")
    return out


def mlp_grad(params: np.ndarray, feat: np.ndarray, label: np.ndarray, pos_w: float = 1.0):
    """(gradient of the summed loss w.r.t. the network parameters, summed loss)."""
    w = np.ascontiguousarray(params, np.float32)
    f = np.ascontiguousarray(feat, np.float32)
    y = np.ascontiguousarray(label, np.float32)
    g = np.empty(w.size - 28, np.float32)
    loss = ctypes.c_double()
    _mlp_check(load().ocfd_b200_mlp_grad(_fp(w), _fp(f), _fp(y), f.shape[0], pos_w, _fp(g), ctypes.byref(loss)),
               "mlp_grad")
    return g, loss.value


def mlp_train(params: np.ndarray, feat: np.ndarray, label: np.ndarray, epochs: int, batch: int = 16384,
              lr: float = 1e-3, pos_w: float = 1.0, seed: int = 1):
    """Adam on the GPU; returns (trained parameter vector, mean loss per epoch)."""
    w = np.array(params, np.float32)
    f = np.ascontiguousarray(feat, np.float32)
    y = np.ascontiguousarray(label, np.float32)
    hist = np.zeros(max(epochs, 1), np.float64)
    _mlp_check(load().ocfd_b200_mlp_train(_fp(w), _fp(f), _fp(y), f.shape[0], epochs, batch, lr, pos_w, seed,
                                          _dp(hist)), "mlp_train")
    return w, hist[:epochs]


SLAB_ID_BYTES = 128


def _torch_nccl_first():
    """The library opens NCCL by its soname (libnccl.so.2) into the process's
    global symbols.  torch links against its own, newer copy; loaded first,
    an older system copy would shadow it and break torch's later import.  So
    torch (where installed) is imported before the library touches NCCL,
    and the library then shares torch's copy."""
    try:
        import torch  # noqa: F401
    except ImportError:
        pass


def slab_unique_id() -> bytes:
    """The communicator id one rank makes for a z-split run (NCCL's unique
    id, 128 bytes) and hands to the others."""
    _torch_nccl_first()
    L = load()
    buf = ctypes.create_string_buffer(SLAB_ID_BYTES)
    rc = L.ocfd_b200_slab_unique_id(buf)
    if rc != OCFD_OK:
        raise OcfdError(rc, "ocfd_b200_slab_unique_id", (L.ocfd_b200_last_error(None) or b"").decode())
    return buf.raw


def make_config(cfg: CaseConfig, device: int = 0) -> Config:
    c = Config()
    c.nx, c.ny, c.nz = cfg.nx, cfg.ny, cfg.nz
    c.iperiodic[:] = list(cfg.iperiodic)
    c.jac_bound[:] = list(cfg.jac_bound)
    c.dif_bound[:] = list(cfg.dif_bound)
    c.non_reflection[:] = list(cfg.non_ref)
    c.scheme_invis = cfg.scheme_invis_id
    c.scheme_vis = cfg.scheme_vis_id
    c.charteric = cfg.charteric
    c.hy_style = cfg.hy_style
    c.hy_dp_intv[:] = list(cfg.hy_dp_intv)
    c.re, c.ama, c.gamma, c.pr = cfg.re, cfg.ama, cfg.gamma, cfg.pr
    c.t_ref, c.epsl_sw, c.dt = cfg.t_ref, cfg.epsl_sw, cfg.dt
    c.device = device
    return c


# ocfd_b200_slab_transport: (user, op, send, recv, count, type) -> status
SLAB_TRANSPORT = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                  ctypes.c_size_t, ctypes.c_int)


class Solver:
    """One B200 solver context.  Same call surface as the reference driver."""

    def __init__(self, cfg: CaseConfig, prims: Optional[Sequence[np.ndarray]] = None,
                 metrics: Optional[Sequence[np.ndarray]] = None, device: int = 0,
                 istep: int = 0, tt: float = 0.0, metric_mode: int = 0, inlet=None, slab=None, transport=None):
        self.L = load()
        self.cfg = cfg
        self.shape = (cfg.nz, cfg.ny, cfg.nx)
        self._c = make_config(cfg, device)
        h = ctypes.c_void_p()
        rc = self.L.ocfd_b200_create(ctypes.byref(self._c), ctypes.byref(h))
        if rc != OCFD_OK:
            raise OcfdError(rc, "ocfd_b200_create", (self.L.ocfd_b200_last_error(None) or b"").decode())
        self.h = h
        self.slab = slab
        self.transport = transport              # kept alive with the context
        if slab is not None and transport is not None:     # exchange through the caller (slabs.HostTransport)
            self._check(self.L.ocfd_b200_set_slab_host(self.h, slab.nranks, slab.rank, slab.rank_lo, slab.rank_hi,
                                                       slab.z_offset, slab.nz_global, transport.fn, None),
                        "set_slab_host")
        elif slab is not None:      # slabs.SlabSpec: before the filters, metrics and state
            _torch_nccl_first()
            self._check(self.L.ocfd_b200_set_slab(self.h, slab.nranks, slab.rank, slab.rank_lo, slab.rank_hi,
                                                  slab.z_offset, slab.nz_global, slab.comm_id), "set_slab")
        if metric_mode:
            self._check(self.L.ocfd_b200_set_metric_mode(self.h, metric_mode), "set_metric_mode")
        for n, (ip, rp) in enumerate(getattr(cfg, "filters", ()) or ()):
            self.set_filter(n, ip, rp)
        if metrics is not None:
            self.set_metrics(metrics)
            if getattr(cfg, "ibc", 0):
                self.set_bc(cfg.ibc, cfg.bc_npara, cfg.bc_rpara, inlet)
        if prims is not None:
            self.set_primitives(prims, istep, tt)

    def _check(self, rc: int, what: str):
        if rc != OCFD_OK:
            raise OcfdError(rc, what, (self.L.ocfd_b200_last_error(self.h) or b"").decode())

    def close(self):
        if getattr(self, "h", None):
            self.L.ocfd_b200_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # set-up -----------------------------------------------------------
    def set_metrics(self, metrics: Sequence[np.ndarray]):
        """13 fields: the metrics (OCFD3d-Jacobi.dat); 3 fields: mesh
        coordinates (OCFD3d-Mesh.dat), from which the GPU computes them."""
        a = np.ascontiguousarray(np.stack([np.asarray(m, np.float64) for m in metrics]))
        if a.shape == (3,) + self.shape:
            self._check(self.L.ocfd_b200_set_mesh(self.h, _dp(a)), "set_mesh")
            return
        if a.shape != (13,) + self.shape:
            raise ValueError(f"metrics shape {a.shape} != {(13,) + self.shape} (or 3 mesh fields)")
        self._check(self.L.ocfd_b200_set_metrics(self.h, _dp(a)), "set_metrics")

    def set_bc(self, ibc: int, npara, rpara, inlet=None):
        ia = (ctypes.c_int * max(1, len(npara)))(*[int(v) for v in npara])
        da = (ctypes.c_double * max(1, len(rpara)))(*[float(v) for v in rpara])
        ip = None
        if inlet is not None:
            self._inlet = np.ascontiguousarray(np.asarray(inlet, np.float64))
            ip = _dp(self._inlet)
        self._check(self.L.ocfd_b200_set_bc(self.h, int(ibc), ia, len(npara), da, len(rpara), ip), "set_bc")

    def set_filter(self, n: int, npara, rpara):
        ia = (ctypes.c_int * 11)(*[int(v) for v in npara])
        da = (ctypes.c_double * 3)(*[float(v) for v in rpara])
        self._check(self.L.ocfd_b200_set_filter(self.h, n, ia, da), "set_filter")

    def metrics(self) -> np.ndarray:
        out = np.empty((13,) + self.shape, dtype=np.float64)
        self._check(self.L.ocfd_b200_get_metrics(self.h, _dp(out)), "get_metrics")
        return out

    def set_sweep_impl(self, impl: int):
        self._check(self.L.ocfd_b200_set_sweep_impl(self.h, impl), "set_sweep_impl")

    def set_graphs(self, enabled: bool):
        """Replay whole steps from CUDA graphs where nothing in a step goes to the host (default on)."""
        self._check(self.L.ocfd_b200_set_graphs(self.h, int(bool(enabled))), "set_graphs")

    def set_precision(self, form: int):
        """0: FP64 throughout; 1: FP32 stencils with FP64 RK3 accumulation."""
        self._check(self.L.ocfd_b200_set_precision(self.h, form), "set_precision")

    def set_switch(self, params: Optional[np.ndarray], confidence: float = 0.9):
        """Learned scheme switch with the plain sensor below `confidence`; None: plain."""
        if params is None:
            self._check(self.L.ocfd_b200_set_switch(self.h, None, 0, 0.0), "set_switch")
            return
        self._switch_w = np.ascontiguousarray(params, np.float32)
        self._check(self.L.ocfd_b200_set_switch(self.h, _fp(self._switch_w), self._switch_w.size, confidence),
                    "set_switch")

    def switch_stats(self) -> Tuple[int, int, int]:
        c = (ctypes.c_longlong * 3)()
        self._check(self.L.ocfd_b200_switch_stats(self.h, c), "switch_stats")
        return int(c[0]), int(c[1]), int(c[2])

    def switch_features(self, first: int = 0, count: Optional[int] = None):
        """(features count x 14, labels count) of interior cells first.. (x fastest)."""
        n = self.cfg.nx * self.cfg.ny * self.cfg.nz
        count = n - first if count is None else count
        f = np.empty((count, 14), np.float32)
        y = np.empty(count, np.float32)
        self._check(self.L.ocfd_b200_switch_features(self.h, first, count, _fp(f), _fp(y)), "switch_features")
        return f, y

    def scheme_proportion(self) -> np.ndarray:
        """[direction][type]: share of each flag array's entries that are 1, 2, other."""
        out = np.zeros(9)
        self._check(self.L.ocfd_b200_scheme_proportion(self.h, _dp(out)), "scheme_proportion")
        return out.reshape(3, 3)

    def sweep_walks(self) -> int:
        """Bit d set: direction d takes the walk that forms every face in line."""
        return int(self.L.ocfd_b200_sweep_walks(self.h))

    def q_criterion(self) -> np.ndarray:
        """Q of the current primitives (get_Q, src/OCFD_ana.cu:317-456), [nz][ny][nx]."""
        out = np.empty(self.shape, dtype=np.float64)
        self._check(self.L.ocfd_b200_q_criterion(self.h, _dp(out)), "q_criterion")
        return out

    def time_average(self, reset: bool = False):
        """Add the current primitives to the running means (or reset them)."""
        self._check(self.L.ocfd_b200_time_average(self.h, int(bool(reset))), "time_average")

    def get_time_average(self) -> Tuple[np.ndarray, int]:
        out = np.empty((5,) + self.shape, dtype=np.float64)
        n = ctypes.c_int()
        self._check(self.L.ocfd_b200_get_time_average(self.h, _dp(out), ctypes.byref(n)), "get_time_average")
        return out, n.value

    def set_viscous_impl(self, impl: int):
        """0: the faster kernel of the form (default); 1: Ev read through the caches; 2: Ev tiles staged in shared memory."""
        self._check(self.L.ocfd_b200_set_viscous_impl(self.h, impl), "set_viscous_impl")

    def set_walk_threshold(self, frac: float):
        """Deferred-cell fraction above which a hybrid direction takes the
        in-line walk (default 0.002; 3 or more keeps every direction on the
        UP7 walk with its other cells deferred)."""
        self._check(self.L.ocfd_b200_set_walk_threshold(self.h, float(frac)), "set_walk_threshold")

    @property
    def uniform_metrics(self) -> bool:
        return bool(self.L.ocfd_b200_uniform_metrics(self.h))

    def set_primitives(self, prims: Sequence[np.ndarray], istep: int = 0, tt: float = 0.0):
        a = np.ascontiguousarray(np.stack([np.asarray(p, np.float64) for p in prims]))
        if a.shape != (5,) + self.shape:
            raise ValueError(f"primitives shape {a.shape} != {(5,) + self.shape}")
        self._check(self.L.ocfd_b200_set_primitives(self.h, _dp(a), istep, tt), "set_primitives")

    def set_primitives_device(self, ptr: int, istep: int = 0, tt: float = 0.0):
        self._check(self.L.ocfd_b200_set_primitives_device(self.h, ctypes.c_void_p(ptr), istep, tt),
                    "set_primitives_device")

    def set_stream(self, stream_ptr: Optional[int]):
        self._check(self.L.ocfd_b200_set_stream(self.h, ctypes.c_void_p(stream_ptr or 0)), "set_stream")

    # stepping ---------------------------------------------------------
    def step(self, n: int = 1):
        self._check(self.L.ocfd_b200_step(self.h, n), "step")

    def synchronize(self):
        self._check(self.L.ocfd_b200_synchronize(self.h), "synchronize")

    def advance_host(self, prims_in: np.ndarray, prims_out: np.ndarray, n: int):
        self._check(self.L.ocfd_b200_advance_host(self.h, _dp(prims_in), _dp(prims_out), n),
                    "advance_host")

    def swap(self):
        self._check(self.L.ocfd_b200_swap_time_levels(self.h), "swap")

    def du_comput(self, krk: int):
        self._check(self.L.ocfd_b200_du_comput(self.h, krk), "du_comput")

    def time_advance(self, krk: int):
        self._check(self.L.ocfd_b200_time_advance(self.h, krk), "time_advance")

    def get_duvwT(self):
        self._check(self.L.ocfd_b200_get_duvwT(self.h), "get_duvwT")

    def bc(self):
        self._check(self.L.ocfd_b200_bc(self.h), "bc")

    # read-back --------------------------------------------------------
    def _get5(self, fn, what) -> np.ndarray:
        out = np.empty((5,) + self.shape, dtype=np.float64)
        self._check(fn(self.h, _dp(out)), what)
        return out

    def primitives(self) -> np.ndarray:
        return self._get5(self.L.ocfd_b200_get_primitives, "get_primitives")

    def conserved(self) -> np.ndarray:
        return self._get5(self.L.ocfd_b200_get_conserved, "get_conserved")

    def du(self) -> np.ndarray:
        return self._get5(self.L.ocfd_b200_get_du, "get_du")

    def flags(self) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
        nz, ny, nx = self.shape
        fx = np.empty((nz, ny, nx + 1), dtype=np.int8)
        fy = np.empty((nz, ny + 1, nx), dtype=np.int8)
        fz = np.empty((nz + 1, ny, nx), dtype=np.int8)
        I8 = ctypes.POINTER(ctypes.c_int8)
        self._check(self.L.ocfd_b200_get_flags(self.h, fx.ctypes.data_as(I8), fy.ctypes.data_as(I8),
                                               fz.ctypes.data_as(I8)), "get_flags")
        return fx, fy, fz

    def time(self) -> Tuple[int, float]:
        i = ctypes.c_int()
        t = ctypes.c_double()
        self._check(self.L.ocfd_b200_get_time(self.h, ctypes.byref(i), ctypes.byref(t)), "get_time")
        return i.value, t.value

    # analysis ---------------------------------------------------------
    def ana_residual(self, which: int) -> float:
        """Mean of E (which=0) or T (which=1) over the interior, FP64."""
        out = ctypes.c_double()
        self._check(self.L.ocfd_b200_ana_residual(self.h, which, ctypes.byref(out)), "ana_residual")
        return out.value

    def check_state(self) -> Tuple[int, int, float]:
        """(cells with NaN, cells with T < 0, mean T)."""
        a = ctypes.c_longlong()
        b = ctypes.c_longlong()
        t = ctypes.c_double()
        self._check(self.L.ocfd_b200_check_state(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(t)),
                    "check_state")
        return a.value, b.value, t.value

    # timing -----------------------------------------------------------
    def set_timing(self, on: bool):
        self._check(self.L.ocfd_b200_set_timing(self.h, int(on)), "set_timing")

    def timing(self):
        ms = (ctypes.c_double * TIMER_COUNT)()
        n = (ctypes.c_longlong * TIMER_COUNT)()
        self._check(self.L.ocfd_b200_get_timing(self.h, ms, n, TIMER_COUNT), "get_timing")
        out = {}
        for i in range(TIMER_COUNT):
            name = self.L.ocfd_b200_timer_name(i).decode()
            if name != "-":
                out[name] = (ms[i], n[i])
        return out

    def launch_count(self) -> int:
        return int(self.L.ocfd_b200_launch_count(self.h))

    def graph_captures(self) -> int:
        """Step graphs captured so far; replayed steps add none."""
        return int(self.L.ocfd_b200_graph_captures(self.h))
