"""On-disk formats shared with OpenCFD-SCU.

Both the reference build and this library read the same case files, so the
parity tests can drive both from one set of inputs:

* ``opencfd-scu.in`` -- ``KEY = value`` lines, spaces inside the key ignored,
  order free (reference: src/parameters.c:666-792, SearchItem/ExtarctItem).
* ``opencfd.dat`` / ``OCFD%08d.dat`` -- Fortran-record primitives: a 20-byte
  header ``[int 12][int Istep][double tt][int 12]`` and then, for each of
  d,u,v,w,T and each k-plane, ``[int NX*NY*8][NX*NY doubles][int NX*NY*8]``
  (src/OCFD_IO.c:157-228, src/OCFD_IO_mpi.c:562-700).
* ``OCFD3d-Jacobi.dat`` -- 13 such 3-D blocks without a header, in the order
  Axx Ayy Azz Akx Aky Akz Aix Aiy Aiz Asx Asy Asz Ajac
  (src/OCFD_Comput_Jacobian3d.cu:142-181); ``OCFD3d-Mesh.dat`` holds the first 3.

Arrays are numpy float64 of shape (nz, ny, nx) (x fastest), the reference's
memory order.
"""
from __future__ import annotations

import dataclasses
import os
import struct
from typing import Dict, Iterable, List, Optional, Sequence, Tuple

import numpy as np

METRIC_NAMES = ("Axx", "Ayy", "Azz", "Akx", "Aky", "Akz", "Aix", "Aiy", "Aiz",
                "Asx", "Asy", "Asz", "Ajac")
PRIMITIVE_NAMES = ("d", "u", "v", "w", "T")

# scheme names -> IDs (src/parameters.c:567-665)
SCHEME_INVIS_IDS = {
    "UP7": 301, "WENO5": 302, "WENO7": 303, "WENO7_SYMBO": 304,
    "WENO7_SYMBO_LIM": 305, "NND2": 306, "OMP6_HR": 307, "OMP6_LD": 308,
    "OMP6_CD8": 309, "SCHEME_HYBRIDAUTO": 310,
}
SCHEME_VIS_IDS = {"CD6": 203, "CD8": 204}


class FormatError(ValueError):
    """Raised for a malformed or truncated case file."""


@dataclasses.dataclass
class CaseConfig:
    """The subset of ``opencfd-scu.in`` the RHS path consumes."""
    nx: int
    ny: int
    nz: int
    iperiodic: Tuple[int, int, int] = (1, 1, 1)
    jac_bound: Tuple[int, int, int] = (0, 0, 0)
    dif_bound: Tuple[int, ...] = (0, 0, 0, 0, 0, 0)
    non_ref: Tuple[int, ...] = (0, 0, 0, 0, 0, 0)
    scheme_invis: str = "WENO7"
    scheme_vis: str = "CD6"
    charteric: int = 0
    hy_style: int = 2
    hy_dp_intv: Tuple[float, float] = (0.01, 0.2)
    re: float = 1600.0
    ama: float = 0.1
    gamma: float = 1.4
    pr: float = 0.72
    t_ref: float = 288.15
    epsl_sw: float = 0.0
    dt: float = 1e-3
    end_time: float = 1.0
    kstep_show: int = 1000000
    kstep_save: int = 1000000
    init_stat: int = 1
    ibc: int = 0
    stream: int = 0
    # FILTER_NPARA<n> / FILTER_RPARA<n> (src/parameters.c:305-325): per filter
    # ((ntime, filter_x, filter_y, filter_z, ib, ie, jb, je, kb, ke, scheme),
    #  (s0, rth, time limit)); scheme 2 is the shock-capturing filter
    filters: Tuple = ()
    # BC_NPARA / BC_RPARA of the boundary family IBC (src/parameters.c:290-298);
    # IBC 108: (MZMAX, MTMAX, INLET_BOUNDARY, IFLAG_WALL_NOT_NORMAL) and
    # (TW, EPSL, X_DIST_BEGIN, X_DIST_END, BETA, X_WALL_BEGIN, X_UP_BOUNDARY_BEGIN, SLZ)
    bc_npara: Tuple = ()
    bc_rpara: Tuple = ()

    @property
    def scheme_invis_id(self) -> int:
        return SCHEME_INVIS_IDS[self.scheme_invis]

    @property
    def scheme_vis_id(self) -> int:
        return SCHEME_VIS_IDS[self.scheme_vis]

    def steps_for_end_time(self) -> int:
        """Number of steps the reference loop runs (do-while tt < end_time)."""
        n, tt = 0, 0.0
        while True:
            n += 1
            tt += self.dt
            if not tt < self.end_time:
                return n

    def set_steps(self, nsteps: int) -> None:
        """Choose END_TIME so the reference loop runs exactly ``nsteps`` steps."""
        self.end_time = (nsteps - 0.5) * self.dt
        assert self.steps_for_end_time() == nsteps


def _fmt(v) -> str:
    if isinstance(v, (tuple, list)):
        return "   ".join(_fmt(x) for x in v)
    if isinstance(v, float):
        return repr(float(v))
    return str(v)


def write_config(path: str, cfg: CaseConfig) -> None:
    """Write ``opencfd-scu.in`` for a single-rank, Stream_MODE 0 run."""
    lines = [
        "# written by ocfd_b200.formats",
        f"GRID_3D = {cfg.nx}   {cfg.ny}   {cfg.nz}",
        "PARALLEL_3D = 1   1   1",
        f"STREAM = {cfg.stream}",
        f"CHARTERIC = {cfg.charteric}",
        "TEST = 0",
        "LAP = 4",
        "MSG_BLOCK_SIZE = 0",
        f"IPERIODIC = {_fmt(cfg.iperiodic)}",
        f"JAC_BOUND = {_fmt(cfg.jac_bound)}",
        f"DIF_BOUND = {_fmt(cfg.dif_bound)}",
        f"NON_REFLETION = {_fmt(cfg.non_ref)}",
        f"SCHEME_INVIS = {cfg.scheme_invis}",
        f"SCHEME_VIS = {cfg.scheme_vis}",
        f"HY_DP_INTV = {_fmt(cfg.hy_dp_intv)}",
        "HY_SMOOTH_DP = 0",
        f"HY_STYLE = {cfg.hy_style}",
        "HY_PATCH_ZONE = 0",
        f"RE = {_fmt(float(cfg.re))}",
        f"AMA = {_fmt(float(cfg.ama))}",
        f"GAMMA = {_fmt(float(cfg.gamma))}",
        f"PR = {_fmt(float(cfg.pr))}",
        f"T_REF = {_fmt(float(cfg.t_ref))}",
        f"EPSL_SW = {_fmt(float(cfg.epsl_sw))}",
        f"DT = {_fmt(float(cfg.dt))}",
        f"END_TIME = {_fmt(float(cfg.end_time))}",
        f"KSTEP_SHOW = {cfg.kstep_show}",
        f"KSTEP_SAVE = {cfg.kstep_save}",
        f"INIT_STAT = {cfg.init_stat}",
        f"IBC = {cfg.ibc}",
        f"BC_NPARA = {_fmt(tuple(int(v) for v in cfg.bc_npara)) if cfg.bc_npara else 0}",
        f"BC_RPARA = {_fmt(tuple(float(v) for v in cfg.bc_rpara)) if cfg.bc_rpara else 0}",
    ]
    for n, (ip, rp) in enumerate(cfg.filters, start=1):
        lines.append(f"FILTER_NPARA{n} = {_fmt(tuple(int(v) for v in ip))}")
        lines.append(f"FILTER_RPARA{n} = {_fmt(tuple(float(v) for v in rp))}")
    lines.append("")
    with open(path, "w") as fh:
        fh.write("\n".join(lines))


def parse_config_text(text: str) -> Dict[str, str]:
    """KEY=value pairs as the reference reads them (spaces stripped from keys;
    a line needs both '=' and a newline, src/parameters.c:666-680)."""
    out: Dict[str, str] = {}
    for raw in text.splitlines(keepends=True):
        if "=" not in raw or "\n" not in raw:
            continue
        name, value = raw.split("=", 1)
        out[name.replace(" ", "")] = value.rstrip("\n")
    return out


def read_config(path: str) -> CaseConfig:
    with open(path) as fh:
        kv = parse_config_text(fh.read())

    def ints(key, n, default):
        if key not in kv:
            return default
        vals = [int(x) for x in kv[key].split()[:n]]
        if len(vals) < n:
            raise FormatError(f"{key}: expected {n} integers")
        return tuple(vals)

    def flt(key, default):
        return float(kv[key].split()[0]) if key in kv else default

    try:
        nx, ny, nz = ints("GRID_3D", 3, None)
    except TypeError:
        raise FormatError("GRID_3D missing") from None
    inv = kv.get("SCHEME_INVIS", "WENO7").split()[0]
    vis = kv.get("SCHEME_VIS", "CD6").split()[0]
    if inv not in SCHEME_INVIS_IDS or vis not in SCHEME_VIS_IDS:
        # the reference prints "SCHEMES CHOOSE IS WRONG" and exits
        raise FormatError(f"unknown scheme {inv!r}/{vis!r}")
    cfg = CaseConfig(nx=nx, ny=ny, nz=nz)
    cfg.iperiodic = ints("IPERIODIC", 3, cfg.iperiodic)
    cfg.jac_bound = ints("JAC_BOUND", 3, cfg.jac_bound)
    cfg.dif_bound = ints("DIF_BOUND", 6, cfg.dif_bound)
    cfg.non_ref = ints("NON_REFLETION", 6, cfg.non_ref)
    cfg.scheme_invis, cfg.scheme_vis = inv, vis
    cfg.charteric = int(kv.get("CHARTERIC", "0").split()[0])
    cfg.hy_style = int(kv.get("HY_STYLE", "2").split()[0])
    if "HY_DP_INTV" in kv:
        a = [float(x) for x in kv["HY_DP_INTV"].split()[:2]]
        cfg.hy_dp_intv = (a[0], a[1])
    cfg.re = flt("RE", cfg.re)
    cfg.ama = flt("AMA", cfg.ama)
    cfg.gamma = flt("GAMMA", cfg.gamma)
    cfg.pr = flt("PR", cfg.pr)
    cfg.t_ref = flt("T_REF", cfg.t_ref)
    if cfg.t_ref <= 0:
        cfg.t_ref = 288.15      # src/parameters.c:497
    cfg.epsl_sw = flt("EPSL_SW", cfg.epsl_sw)
    cfg.dt = flt("DT", cfg.dt)
    cfg.end_time = flt("END_TIME", cfg.end_time)
    cfg.kstep_show = int(kv.get("KSTEP_SHOW", str(cfg.kstep_show)).split()[0])
    cfg.kstep_save = int(kv.get("KSTEP_SAVE", str(cfg.kstep_save)).split()[0])
    cfg.init_stat = int(kv.get("INIT_STAT", "1").split()[0])
    cfg.ibc = int(kv.get("IBC", "0").split()[0])
    cfg.stream = int(kv.get("STREAM", "0").split()[0])
    if "BC_NPARA" in kv and cfg.ibc:
        cfg.bc_npara = tuple(int(x) for x in kv["BC_NPARA"].split())
        cfg.bc_rpara = tuple(float(x) for x in kv.get("BC_RPARA", "").split())
    filters = []
    for key in sorted((k for k in kv if k.startswith("FILTER_NPARA")), key=lambda k: int(k[12:] or 0)):
        rkey = "FILTER_RPARA" + key[12:]
        ip = tuple(int(x) for x in kv[key].split()[:11])
        rp = tuple(float(x) for x in kv.get(rkey, "0 0 0").split()[:3])
        filters.append((ip, rp))
    cfg.filters = tuple(filters)
    return cfg


# --------------------------------------------------------------------------
# Fortran-record 3-D blocks
# --------------------------------------------------------------------------

def _block_bytes(arr: np.ndarray) -> bytes:
    nz, ny, nx = arr.shape
    rec = nx * ny * 8
    marker = struct.pack("<i", rec)
    a = np.ascontiguousarray(arr, dtype="<f8")
    out = bytearray()
    for k in range(nz):
        out += marker
        out += a[k].tobytes()
        out += marker
    return bytes(out)


def _read_blocks(buf: memoryview, offset: int, shape: Tuple[int, int, int], count: int,
                 what: str) -> Tuple[List[np.ndarray], int]:
    nz, ny, nx = shape
    rec = nx * ny * 8
    out = []
    for b in range(count):
        arr = np.empty(shape, dtype=np.float64)
        for k in range(nz):
            if offset + 8 + rec > len(buf):
                raise FormatError(f"{what}: truncated at block {b}, plane {k}")
            m0 = struct.unpack_from("<i", buf, offset)[0]
            m1 = struct.unpack_from("<i", buf, offset + 4 + rec)[0]
            if m0 != rec or m1 != rec:
                raise FormatError(f"{what}: bad record marker ({m0},{m1}) != {rec} "
                                  f"at block {b}, plane {k}")
            arr[k] = np.frombuffer(buf, dtype="<f8", count=nx * ny,
                                   offset=offset + 4).reshape(ny, nx)
            offset += rec + 8
        out.append(arr)
    return out, offset


def write_field_file(path: str, fields: Sequence[np.ndarray], istep: int = 0,
                     tt: float = 0.0) -> None:
    """Write opencfd.dat / OCFD%08d.dat (d,u,v,w,T)."""
    if len(fields) != 5:
        raise ValueError("need 5 primitive fields")
    with open(path, "wb") as fh:
        fh.write(struct.pack("<iidi", 12, istep, tt, 12))
        for f in fields:
            fh.write(_block_bytes(np.asarray(f, dtype=np.float64)))


def read_field_file(path: str, shape: Tuple[int, int, int]) -> Tuple[List[np.ndarray], int, float]:
    """Read d,u,v,w,T; returns (fields, Istep, tt)."""
    with open(path, "rb") as fh:
        data = fh.read()
    if len(data) < 20:
        raise FormatError(f"{path}: header truncated")
    m0, istep, tt, m1 = struct.unpack_from("<iidi", data, 0)
    if m0 != 12 or m1 != 12:
        raise FormatError(f"{path}: bad header markers ({m0},{m1})")
    fields, _ = _read_blocks(memoryview(data), 20, shape, 5, path)
    return fields, istep, tt


# --------------------------------------------------------------------------
# restart: Opencfd.msg names the field file a run starts from
# --------------------------------------------------------------------------

def read_restart_step(path: str = "Opencfd.msg") -> int:
    """The restart step Opencfd.msg holds (read_file, src/OCFD_IO.c:38-58: one
    native int read with fread); -1 when the file is absent."""
    try:
        with open(path, "rb") as fh:
            raw = fh.read(4)
    except FileNotFoundError:
        return -1
    if len(raw) < 4:
        raise FormatError(f"{path}: shorter than one int")
    return struct.unpack("<i", raw)[0]


def write_restart_step(path: str, istep: int) -> None:
    """Opencfd.msg for a restart from OCFD%08d.dat of step istep."""
    with open(path, "wb") as fh:
        fh.write(struct.pack("<i", int(istep)))


def initial_field_file(directory: str = ".") -> str:
    """The field file a run reads first: opencfd.dat, or OCFD%08d.dat of the
    step in Opencfd.msg when that file exists and holds a step >= 0
    (src/OCFD_IO.c:53-60)."""
    step = read_restart_step(os.path.join(directory, "Opencfd.msg"))
    name = "opencfd.dat" if step < 0 else f"OCFD{step:08d}.dat"
    return os.path.join(directory, name)


def write_metric_file(path: str, fields: Sequence[np.ndarray]) -> None:
    """Write OCFD3d-Jacobi.dat (13 blocks) or OCFD3d-Mesh.dat (3 blocks)."""
    if len(fields) not in (3, 13):
        raise ValueError("need 3 (mesh) or 13 (Jacobi) fields")
    with open(path, "wb") as fh:
        for f in fields:
            fh.write(_block_bytes(np.asarray(f, dtype=np.float64)))


def read_metric_file(path: str, shape: Tuple[int, int, int], count: int = 13) -> List[np.ndarray]:
    with open(path, "rb") as fh:
        data = fh.read()
    fields, _ = _read_blocks(memoryview(data), 0, shape, count, path)
    return fields


# --------------------------------------------------------------------------
# flow1d-inlet.dat (IBC 108 inlet profile, src/OCFD_boundary_init.c:386-394)
# --------------------------------------------------------------------------

def write_inlet_file(path: str, profile: np.ndarray, y: Optional[np.ndarray] = None) -> None:
    """One header line, then NY rows ``y d u v T``; profile is [4][ny] (d,u,v,T)."""
    profile = np.asarray(profile, dtype=np.float64)
    ny = profile.shape[1]
    yy = np.arange(ny, dtype=np.float64) if y is None else np.asarray(y, dtype=np.float64)
    with open(path, "w") as fh:
        fh.write("variables = y d u v T\n")
        for j in range(ny):
            fh.write("%.17e %.17e %.17e %.17e %.17e\n" % (yy[j], profile[0, j], profile[1, j],
                                                         profile[2, j], profile[3, j]))


def read_inlet_file(path: str, ny: int) -> np.ndarray:
    with open(path) as fh:
        fh.readline()
        rows = [[float(x) for x in fh.readline().split()[:5]] for _ in range(ny)]
    a = np.array(rows, dtype=np.float64)
    return np.ascontiguousarray(a[:, 1:5].T)
