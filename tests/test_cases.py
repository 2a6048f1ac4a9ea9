"""The synthetic inputs the benchmarks and parity tests run on, on CPU: the
Taylor-Green vortex and the isotropic-turbulence field have the stated
formulas, spectrum normalisation, Mach numbers and time steps, and are fixed
by their seeds."""
import math

import numpy as np
import pytest

from ocfd_b200 import cases


def test_taylor_green_fields():
    n, ama, g = 16, 0.1, 1.4
    c = cases.taylor_green(n, ama=ama, gamma=g, seed=7)
    d, u, v, w, T = c.prims
    h = 2 * math.pi / n
    k, j, i = 3, 5, 11
    x, y, z = i * h, j * h, k * h
    assert u[k, j, i] == pytest.approx(math.sin(x) * math.cos(y) * math.cos(z), abs=1e-15)
    assert v[k, j, i] == pytest.approx(-math.cos(x) * math.sin(y) * math.cos(z), abs=1e-15)
    assert not w.any()
    assert np.all(np.abs(d - 1.0) <= 1e-4) and d.std() > 1e-5
    p0 = 1.0 / (g * ama * ama)
    p = p0 + (math.cos(2 * x) + math.cos(2 * y)) * (math.cos(2 * z) + 2.0) / 16.0
    assert T[k, j, i] == pytest.approx(g * ama * ama * p / d[k, j, i], rel=1e-14)
    # dt = 0.5 * delta / max(max|u_i| + c), c = sqrt(T)/Ma
    lam = np.max(np.maximum(np.maximum(np.abs(u), np.abs(v)), np.abs(w)) + np.sqrt(T) / ama)
    assert c.cfg.dt == pytest.approx(0.5 * h / lam, rel=1e-14)
    assert (c.cfg.scheme_invis, c.cfg.scheme_vis, c.cfg.iperiodic) == ("WENO7", "CD6", (1, 1, 1))
    assert np.array_equal(d, cases.taylor_green(n, ama=ama, gamma=g, seed=7).prims[0])


def _spectral_div(u, v, w):
    """Spectral divergence without the Nyquist planes (there the derivative of
    a real field has no sign: the generator's +k and -k coefficients share one
    DFT entry)."""
    n = u.shape[0]
    k1 = np.fft.fftfreq(n, d=1.0 / n)
    KZ, KY, KX = np.meshgrid(k1, k1, k1, indexing="ij")
    keep = (np.abs(KX) < n // 2) & (np.abs(KY) < n // 2) & (np.abs(KZ) < n // 2)
    s = KX * np.fft.fftn(u) + KY * np.fft.fftn(v) + KZ * np.fft.fftn(w)
    return np.real(np.fft.ifftn(1j * s * keep))


def test_isotropic_turbulence_field():
    n, mt = 32, 0.6
    c = cases.isotropic_turbulence(n, mach_t=mt, seed=5)
    d, u, v, w, T = c.prims
    assert np.all(d == 1.0) and np.all(T == 1.0)
    # solenoidal: the spectral divergence vanishes to round-off
    dudx = np.real(np.fft.ifftn(1j * np.meshgrid(np.fft.fftfreq(n, 1.0 / n), np.fft.fftfreq(n, 1.0 / n),
                                                np.fft.fftfreq(n, 1.0 / n), indexing="ij")[2] * np.fft.fftn(u)))
    assert np.abs(_spectral_div(u, v, w)).max() <= 1e-12 * np.abs(dudx).max()
    # rms 1 per component on average, so Mach_t = sqrt(<u.u>) / c with c = 1/Ma
    assert np.mean(u * u + v * v + w * w) / 3.0 == pytest.approx(1.0, rel=1e-12)
    assert math.sqrt(np.mean(u * u + v * v + w * w)) * c.cfg.ama == pytest.approx(mt, rel=1e-12)
    # energy where the spectrum k^4 exp(-2 (k/4)^2) puts it: the peak shell is near k = 4
    k1 = np.fft.fftfreq(n, d=1.0 / n)
    KZ, KY, KX = np.meshgrid(k1, k1, k1, indexing="ij")
    shell = np.rint(np.sqrt(KX**2 + KY**2 + KZ**2)).astype(int)
    e = sum(np.abs(np.fft.fftn(f)) ** 2 for f in (u, v, w))
    Ek = np.bincount(shell.ravel(), weights=e.ravel())
    assert 3 <= int(np.argmax(Ek)) <= 5
    assert c.cfg.scheme_invis == "SCHEME_HYBRIDAUTO" and c.cfg.hy_style == 2 and c.cfg.charteric == 1
    assert np.array_equal(u, cases.isotropic_turbulence(n, mach_t=mt, seed=5).prims[1])
    assert not np.array_equal(u, cases.isotropic_turbulence(n, mach_t=mt, seed=6).prims[1])


def test_isotropic_turbulence_reynolds_number():
    """Re is chosen so that u_rms * lambda * Re = Re_lambda, lambda from the
    spectral x derivative of u."""
    n = 32
    c = cases.isotropic_turbulence(n, re_lambda=100.0, seed=3)
    u = c.prims[1]
    k1 = np.fft.fftfreq(n, d=1.0 / n)
    KX = np.meshgrid(k1, k1, k1, indexing="ij")[2]
    dudx = np.real(np.fft.ifftn(1j * KX * np.fft.fftn(u)))
    lam = math.sqrt(np.mean(u * u) / np.mean(dudx * dudx))
    assert c.cfg.re * lam == pytest.approx(100.0, rel=1e-12)


def test_ramp_mesh_and_inflow():
    """The 24-degree ramp: flat wall up to the corner at mid-length, then the
    wall rises at the ramp angle; tanh wall-normal stretching with a first
    cell of 0.01 boundary-layer thicknesses; periodic span; the inflow is the
    1/7-power layer at the isothermal wall temperature."""
    nx, ny, nz = 64, 32, 8
    c = cases.ramp_case(nx, ny, nz, seed=1)
    x, y, z = c.metrics
    assert x.shape == (nz, ny, nx)
    wall = y[0, 0, :]
    xs = x[0, 0, :]
    flat = xs <= 20.0
    assert np.all(np.abs(wall[flat]) < 1e-12)
    slope = np.diff(wall[~flat]) / np.diff(xs[~flat])
    assert np.allclose(slope, math.tan(math.radians(24.0)), rtol=1e-12)
    assert y[0, 1, 0] - y[0, 0, 0] == pytest.approx(0.01, rel=1e-6)      # first cell at x = 0
    assert np.all(np.diff(y[0, :, 0]) > 0) and y[0, -1, 0] == pytest.approx(15.0)
    assert np.all(np.diff(y[0, :, 0])[1:] > np.diff(y[0, :, 0])[:-1])    # stretched away from the wall
    assert np.allclose(np.diff(z[:, 0, 0]), 1.0)                          # span 8, 8 planes
    d_in, u_in, v_in, T_in = c.inlet
    dist = y[0, :, 0]
    assert np.allclose(u_in, np.clip(dist, 0, 1) ** (1 / 7))
    # T linear in u from the wall temperature 2.5 to 1 at the edge, uniform pressure
    assert np.allclose(T_in, 2.5 - 1.5 * u_in) and np.allclose(d_in * T_in, 1.0) and not v_in.any()
    assert u_in[0] < 0.01 and u_in[-1] == 1.0
    assert c.cfg.iperiodic == (0, 0, 1) and c.cfg.ibc == 108 and c.cfg.dif_bound[:4] == (1, 1, 1, 1)
    # seeded fluctuations of about 2 %
    d = c.prims[0]
    dwall = y - y[:, :1, :]
    base = 1.0 / (2.5 - 1.5 * np.clip(dwall, 0, 1) ** (1 / 7))
    assert np.std(d / base - 1.0) == pytest.approx(0.02, rel=0.05)
