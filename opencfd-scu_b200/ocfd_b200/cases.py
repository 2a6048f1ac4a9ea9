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
from typing import Optional, List, Tuple

import numpy as np

from .formats import CaseConfig


@dataclasses.dataclass
class Case:
    cfg: CaseConfig
    prims: List[np.ndarray]       # d,u,v,w,T each (nz,ny,nx)
    metrics: List[np.ndarray]     # 13 metric fields, or 3 mesh coordinate fields, each (nz,ny,nx)
    description: str = ""
    inlet: Optional[np.ndarray] = None   # IBC 108 inflow profile [4][ny] (d,u,v,T), flow1d-inlet.dat

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



def ramp_case(nx: int = 512, ny: int = 128, nz: int = 64, angle_deg: float = 24.0, ama: float = 2.9,
              re: float = 5000.0, tw: float = 2.5, seed: int = 2024, fluct: float = 0.02,
              scheme_invis: str = "SCHEME_HYBRIDAUTO", charteric: int = 1, cfl: float = 0.3,
              filters=(((1, 1, 1, 0, 0, 100000, 0, 100000, 0, 100000, 2), (1.0, 1e-5, 1e9)),),
              epsl: float = 0.0, beta: float = 0.0, mtmax: int = 0) -> Case:
    """24-degree compression ramp (the compression-corner family, IBC 108).

    Mesh (OCFD3d-Mesh.dat, metrics computed by the solver): x in [0, Lx]
    with the corner at 0.5 Lx, the wall following the ramp, wall-normal
    tanh stretching with a first cell of 0.01 delta up to Ly, periodic span
    Lz.  Inflow: a 1/7-power boundary layer of thickness delta = 1 at an
    isothermal wall (T_w = tw, linear T(u), uniform pressure), written as the
    flow1d-inlet.dat profile; the initial field is that profile everywhere
    plus seeded relative fluctuations of size ``fluct``.  x and y are closed
    (DIF_BOUND = 1, JAC_BOUND = 1), z periodic; hybrid scheme with the shock
    filter every step; dt from the CFL number at t = 0."""
    rng = np.random.default_rng(seed)
    Lx, Ly, Lz = 40.0, 15.0, 8.0
    xc = 0.5 * Lx
    t = math.tan(math.radians(angle_deg))
    xs = np.linspace(0.0, Lx, nx)
    yw = np.where(xs > xc, (xs - xc) * t, 0.0)
    eta = np.linspace(0.0, 1.0, ny)
    # tanh stretching: y(eta) = H (1 - tanh(b (1-eta)) / tanh(b)), first cell 0.01
    b = 1.0
    for _ in range(60):
        h1 = Ly * (1.0 - math.tanh(b * (1.0 - eta[1])) / math.tanh(b))
        b *= (h1 / 0.01) ** 0.25
    st = 1.0 - np.tanh(b * (1.0 - eta)) / math.tanh(b)
    zs = np.arange(nz) * (Lz / nz)
    Z, Y, X = np.meshgrid(zs, st, xs, indexing="ij")
    ywall = np.broadcast_to(yw[None, None, :], X.shape)
    x = X.copy()
    y = ywall + (Ly - ywall) * Y
    z = Z.copy()
    # inflow profile from the wall distance at x = 0
    dist = y[0, :, 0]
    # profile wall temperature: tw, or the recovery temperature for an
    # adiabatic wall (tw <= 0 selects the adiabatic boundary condition)
    tpw = tw if tw > 0 else 1.0 + 0.89 * 0.2 * ama * ama
    u_in = np.clip(dist / 1.0, 0.0, 1.0) ** (1.0 / 7.0)
    T_in = tpw - (tpw - 1.0) * u_in
    d_in = 1.0 / T_in
    inlet = np.stack([d_in, u_in, np.zeros(ny), T_in])
    # initial field: the profile by wall distance, plus fluctuations
    dwall = y - ywall
    uu = np.clip(dwall, 0.0, 1.0) ** (1.0 / 7.0)
    TT = tpw - (tpw - 1.0) * uu
    dd = 1.0 / TT
    noise = lambda: fluct * rng.standard_normal(X.shape)
    d = dd * (1.0 + noise())
    u = uu * (1.0 + noise())
    v = 0.01 * noise()
    w = 0.01 * noise()
    T = TT * (1.0 + noise())
    c0 = math.sqrt(tpw) / ama
    dx = Lx / (nx - 1)
    dt = cfl * min(dx, 0.01) / (1.0 + c0)
    cfg = CaseConfig(nx=nx, ny=ny, nz=nz, iperiodic=(0, 0, 1), jac_bound=(1, 1, 1),
                     dif_bound=(1, 1, 1, 1, 0, 0), non_ref=(0, 0, 0, 0, 0, 0),
                     scheme_invis=scheme_invis, scheme_vis="CD6", charteric=charteric,
                     hy_dp_intv=(0.01, 0.2), re=re, ama=ama, gamma=1.4, pr=0.72, epsl_sw=0.0, dt=dt,
                     ibc=108, bc_npara=(0, mtmax, 1, 0),
                     bc_rpara=(tw, epsl, 0.25 * Lx, 0.4 * Lx, beta, 0.0, 0.8 * Lx, Lz))
    # the filter ranges are clamped to the box by the solver
    cfg.filters = tuple(((ip[0], ip[1], ip[2], ip[3], 0, nx, 0, ny, 0, nz, ip[10]), rp) for ip, rp in filters)
    return Case(cfg, [d, u, v, w, T], [x, y, z],
                f"compression ramp {nx}x{ny}x{nz} angle={angle_deg} Ma={ama} Re={re} Tw={tw} seed={seed}",
                inlet=inlet)
