"""Synthetic case generators (no dataset is involved; every input is analytic
or drawn from a seeded numpy PRNG).

Non-dimensionalisation follows the reference: p = rho*T/(gamma*Ma^2), sound
speed c = sqrt(T)/Ma (src/commen_kernel.cu:102,151), Sutherland viscosity with
mu(T=1) = 1/Re (src/OCFD_init.cu:384-386).

Grid metrics for a uniform periodic Cartesian grid with spacing ``delta``:
the computational coordinate steps are h = 1/(N-1) (src/OCFD_init.cu:29-31),
so x_xi = delta/h and the conservative metrics of comput_Jac3d_kernal
(src/OCFD_Comput_Jacobian3d.cu:283-296) reduce to Akx = y_eta*z_zeta,
Aiy = z_zeta*x_xi, Asz = x_xi*y_eta, Ajac = 1/(x_xi*y_eta*z_zeta), all other
entries zero.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Tuple

import numpy as np

from .formats import CaseConfig


@dataclasses.dataclass
class Case:
    cfg: CaseConfig
    prims: List[np.ndarray]       # d,u,v,w,T each (nz,ny,nx)
    metrics: List[np.ndarray]     # 13 fields each (nz,ny,nx)
    description: str = ""

    @property
    def shape(self) -> Tuple[int, int, int]:
        return (self.cfg.nz, self.cfg.ny, self.cfg.nx)


def cartesian_metrics(nx: int, ny: int, nz: int, dx: float, dy: float, dz: float) -> List[np.ndarray]:
    hx, hy, hz = 1.0 / (nx - 1.0), 1.0 / (ny - 1.0), 1.0 / (nz - 1.0)
    xi, yj, zk = dx / hx, dy / hy, dz / hz
    shape = (nz, ny, nx)
    z = np.zeros(shape)
    x1 = np.arange(nx) * dx
    y1 = np.arange(ny) * dy
    z1 = np.arange(nz) * dz
    Z, Y, X = np.meshgrid(z1, y1, x1, indexing="ij")
    # same evaluation order as comput_Jac3d_kernal: products left to right,
    # det = xi*yj*zk + 0 + 0 - 0 - 0 - 0
    jac = 1.0 / (xi * yj * zk)
    full = lambda v: np.full(shape, v, dtype=np.float64)
    return [X.copy(), Y.copy(), Z.copy(),
            full(yj * zk), z.copy(), z.copy(),
            z.copy(), full(zk * xi), z.copy(),
            z.copy(), z.copy(), full(xi * yj),
            full(jac)]


def acoustic_dt(prims: List[np.ndarray], ama: float, delta: float, cfl: float) -> float:
    """dt = cfl*delta / max(max(|u|,|v|,|w|) + c), c = sqrt(T)/Ma, computed once in FP64."""
    d, u, v, w, T = prims
    vmax = np.maximum(np.maximum(np.abs(u), np.abs(v)), np.abs(w))
    lam = float(np.max(vmax + np.sqrt(T) / ama))
    return cfl * delta / lam


def taylor_green(n: int = 64, ama: float = 0.1, re: float = 1600.0, gamma: float = 1.4,
                 pr: float = 0.72, seed: int = 1234, cfl: float = 0.5,
                 scheme_invis: str = "WENO7", scheme_vis: str = "CD6",
                 charteric: int = 0, t_ref: float = 288.15) -> Case:
    """3-D Taylor-Green vortex on an n^3 periodic grid over [0, 2*pi)^3.

    u = sin x cos y cos z, v = -cos x sin y cos z, w = 0,
    p = p0 + (cos 2x + cos 2y)(cos 2z + 2)/16 with p0 = 1/(gamma Ma^2),
    rho = 1 + U(-1e-4, 1e-4) (numpy default_rng(seed)), T = gamma Ma^2 p / rho.
    """
    delta = 2.0 * math.pi / n
    x = np.arange(n) * delta
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
    u = np.sin(X) * np.cos(Y) * np.cos(Z)
    v = -np.cos(X) * np.sin(Y) * np.cos(Z)
    w = np.zeros_like(u)
    p0 = 1.0 / (gamma * ama * ama)
    p = p0 + (np.cos(2 * X) + np.cos(2 * Y)) * (np.cos(2 * Z) + 2.0) / 16.0
    rng = np.random.default_rng(seed)
    d = 1.0 + rng.uniform(-1e-4, 1e-4, size=u.shape)
    T = gamma * ama * ama * p / d
    prims = [d, u, v, w, T]
    cfg = CaseConfig(nx=n, ny=n, nz=n, iperiodic=(1, 1, 1), scheme_invis=scheme_invis,
                     scheme_vis=scheme_vis, charteric=charteric, re=re, ama=ama,
                     gamma=gamma, pr=pr, t_ref=t_ref, epsl_sw=0.0)
    cfg.dt = acoustic_dt(prims, ama, delta, cfl)
    met = cartesian_metrics(n, n, n, delta, delta, delta)
    return Case(cfg, prims, met, f"TGV {n}^3 Ma={ama} Re={re} seed={seed}")


def isotropic_turbulence(n: int = 256, mach_t: float = 0.6, re_lambda: float = 100.0,
                         k0: float = 4.0, gamma: float = 1.4, pr: float = 0.72,
                         seed: int = 2024, cfl: float = 0.5,
                         hy_dp_intv: Tuple[float, float] = (0.01, 0.2),
                         charteric: int = 1, t_ref: float = 288.15) -> Case:
    """Decaying compressible isotropic turbulence on an n^3 periodic box.

    Random solenoidal velocity with E(k) ~ k^4 exp(-2 (k/k0)^2), uniform rho = 1
    and T = 1 (so p = 1/(gamma Ma^2)).  The field is scaled so each component
    has rms 1; Mach_t = sqrt(<u.u>)/c = sqrt(3)*Ma fixes Ma.  Re is chosen so
    that Re_lambda = u_rms*lambda/nu, lambda = sqrt(<u^2>/<(du/dx)^2>), with
    nu = 1/Re at the reference state.
    """
    rng = np.random.default_rng(seed)
    k1 = np.fft.fftfreq(n, d=1.0 / n)
    KZ, KY, KX = np.meshgrid(k1, k1, k1, indexing="ij")
    kk = np.sqrt(KX**2 + KY**2 + KZ**2)
    kk_safe = np.where(kk == 0, 1.0, kk)
    spec = kk_safe**4 * np.exp(-2.0 * (kk_safe / k0) ** 2)
    amp = np.sqrt(spec / (4.0 * math.pi * kk_safe**2))
    amp[kk == 0] = 0.0
    comps = []
    for _ in range(3):
        ph = rng.uniform(0.0, 2.0 * math.pi, size=kk.shape)
        a = rng.standard_normal(size=kk.shape)
        comps.append(amp * a * np.exp(1j * ph))
    ax, ay, az = comps
    # project onto divergence-free modes
    kdot = (KX * ax + KY * ay + KZ * az) / (kk_safe**2)
    ax = ax - KX * kdot
    ay = ay - KY * kdot
    az = az - KZ * kdot
    u = np.real(np.fft.ifftn(ax))
    v = np.real(np.fft.ifftn(ay))
    w = np.real(np.fft.ifftn(az))
    urms = math.sqrt(float(np.mean(u * u + v * v + w * w)) / 3.0)
    u, v, w = u / urms, v / urms, w / urms
    ama = mach_t / math.sqrt(3.0)
    delta = 2.0 * math.pi / n
    # Taylor microscale from spectral derivatives
    dudx = np.real(np.fft.ifftn(1j * KX * np.fft.fftn(u)))
    lam = math.sqrt(float(np.mean(u * u)) / float(np.mean(dudx * dudx)))
    re = re_lambda / (1.0 * lam)
    d = np.ones_like(u)
    T = np.ones_like(u)
    prims = [d, u, v, w, T]
    cfg = CaseConfig(nx=n, ny=n, nz=n, iperiodic=(1, 1, 1), scheme_invis="SCHEME_HYBRIDAUTO",
                     scheme_vis="CD6", charteric=charteric, hy_style=2,
                     hy_dp_intv=tuple(hy_dp_intv), re=re, ama=ama, gamma=gamma, pr=pr,
                     t_ref=t_ref, epsl_sw=0.0)
    cfg.dt = acoustic_dt(prims, ama, delta, cfl)
    met = cartesian_metrics(n, n, n, delta, delta, delta)
    return Case(cfg, prims, met,
                f"isotropic {n}^3 Mt={mach_t} Re_lambda={re_lambda} k0={k0} seed={seed}")


def random_smooth_case(nx: int, ny: int, nz: int, seed: int = 7, scheme_invis: str = "WENO7",
                       scheme_vis: str = "CD6", charteric: int = 0, ama: float = 0.5,
                       amp: float = 0.2, shock: bool = False, curvilinear: bool = False,
                       dt: float = 2e-3, iperiodic=(1, 1, 1), dif_bound=(0, 0, 0, 0, 0, 0),
                       non_ref=(0, 0, 0, 0, 0, 0)) -> Case:
    """Odd-sized box with a few random Fourier modes (optionally a steep tanh
    front so the hybrid sensor switches) for kernel parity tests.
    ``curvilinear`` gives a smoothly sheared metric field so that every metric
    entry is non-zero.  ``iperiodic`` / ``dif_bound`` / ``non_ref`` are the
    IPERIODIC / DIF_BOUND / NON_REFLETION keys: a non-periodic direction with
    DIF_BOUND = 1 uses the boundary closures (no boundary-condition family,
    IBC = 0, so the faces only get the re-projection)."""
    rng = np.random.default_rng(seed)
    Lx, Ly, Lz = 2 * math.pi, 2 * math.pi, 2 * math.pi
    dx, dy, dz = Lx / nx, Ly / ny, Lz / nz
    x = np.arange(nx) * dx
    y = np.arange(ny) * dy
    z = np.arange(nz) * dz
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")

    def field(base, a):
        f = np.full(X.shape, base, dtype=np.float64)
        for _ in range(3):
            kx, ky, kz = rng.integers(1, 3, size=3)
            ph = rng.uniform(0, 2 * math.pi, size=3)
            f += a * rng.uniform(0.3, 1.0) * np.sin(kx * X + ph[0]) * np.cos(ky * Y + ph[1]) \
                * np.cos(kz * Z + ph[2])
        return f

    d = field(1.0, 0.1 * amp)
    u = field(0.0, amp)
    v = field(0.0, amp)
    w = field(0.0, amp)
    T = field(1.0, 0.1 * amp)
    if shock:
        front = 0.5 * (1 + np.tanh(8.0 * np.sin(X) * np.cos(0.5 * Y)))
        d = d * (1.0 + 0.8 * front)
        T = T * (1.0 + 0.5 * front)
    prims = [d, u, v, w, T]
    cfg = CaseConfig(nx=nx, ny=ny, nz=nz, iperiodic=tuple(iperiodic), scheme_invis=scheme_invis,
                     scheme_vis=scheme_vis, charteric=charteric, re=500.0, ama=ama,
                     gamma=1.4, pr=0.72, epsl_sw=0.0, dt=dt, dif_bound=tuple(dif_bound),
                     non_ref=tuple(non_ref))
    met = cartesian_metrics(nx, ny, nz, dx, dy, dz)
    if curvilinear:
        # smooth periodic perturbation of all nine conservative metrics and of Ajac
        for m in range(3, 13):
            base = met[m]
            pert = 0.05 * np.sin(X + 0.3 * m) * np.cos(Y - 0.2 * m) * np.cos(Z + 0.1 * m)
            scale = float(np.max(np.abs(met[3])))
            met[m] = base + (scale if m != 12 else float(met[12].max())) * pert
    return Case(cfg, prims, met, f"random {nx}x{ny}x{nz} seed={seed} shock={shock}")


def mesh_case(nx: int, ny: int, nz: int, seed: int = 7, scheme_invis: str = "WENO7",
              charteric: int = 0, shock: bool = False, jac_bound=(1, 1, 1),
              iperiodic=(0, 0, 1), dif_bound=(1, 1, 1, 1, 0, 0), non_ref=(0, 0, 0, 0, 0, 0),
              skew: float = 0.08) -> Case:
    """A case whose metrics the solver computes from mesh coordinates
    (OCFD3d-Mesh.dat: x, y, z; JAC_BOUND selects the derivative closures at
    both ends of each direction).  The grid is a smoothly skewed and
    stretched box, the flow the random fields of random_smooth_case.
    ``Case.metrics`` holds the three coordinate fields."""
    base = random_smooth_case(nx, ny, nz, seed=seed, scheme_invis=scheme_invis, charteric=charteric,
                              shock=shock, iperiodic=iperiodic, dif_bound=dif_bound, non_ref=non_ref)
    rng = np.random.default_rng(seed + 1000)
    xi = np.arange(nx) / (nx - 1.0)
    eta = np.arange(ny) / (ny - 1.0)
    zeta = np.arange(nz) / float(nz)
    Z, Y, X = np.meshgrid(zeta, eta, xi, indexing="ij")
    Lx, Ly, Lz = 2 * math.pi, 2 * math.pi, 2 * math.pi
    a = skew * rng.uniform(0.5, 1.0, size=3)
    x = Lx * X + a[0] * Lx * np.sin(math.pi * Y) * np.sin(2 * math.pi * Z)
    y = Ly * Y * (1.0 + 0.3 * X * (1.0 - X)) + a[1] * Ly * np.sin(math.pi * X)
    z = Lz * Z + a[2] * Lz * np.sin(math.pi * X) * np.sin(math.pi * Y)
    cfg = base.cfg
    cfg.jac_bound = tuple(jac_bound)
    return Case(cfg, base.prims, [x, y, z],
                f"mesh {nx}x{ny}x{nz} seed={seed} skew={skew} scheme={scheme_invis}")
