"""Unit checks of the CPU oracle's point formulas (the checker itself).

Exactness properties of the reference schemes (src/OCFD_Schemes.cu) on
polynomial data, the Steger-Warming split identity (src/OCFD_split.cu), and
L*R = I for the characteristic matrices (src/OCFD_flux_charteric.cu).
"""
import math

import numpy as np
import pytest

from oracle import oracle as oro


def _poly_cells(coef, x):
    return sum(c * x**k for k, c in enumerate(coef))


def _flux_diff(name, coef, sign, args=()):
    """(F(i+1/2) - F(i-1/2)) at i = 0 on a unit grid from point values f(x_j)."""
    h = 1.0
    xs = np.arange(-8, 9) * h
    f = _poly_cells(coef, xs)
    off = 8

    def face(F):
        s8 = f[off + F - 3: off + F + 5]
        if name in ("weno7_p", "up7_p", "omp6_p", "weno7_symbo_p"):
            return oro.point(name, s8, *args)
        if name == "weno5_p":
            return oro.point(name, s8[1:6], *args)
        if name == "weno7_m":
            return oro.point(name, s8[1:8], *args)
        if name == "weno5_m":
            return oro.point(name, s8[2:7], *args)
        if name in ("up7_m", "omp6_m", "weno7_symbo_m"):
            return oro.point(name, s8, *args)
        raise KeyError(name)
    return face(0) - face(-1)


def _exact_derivative(coef):
    return coef[1] if len(coef) > 1 else 0.0


@pytest.mark.parametrize("name,deg", [("up7_p", 7), ("up7_m", 7), ("weno7_p", 3), ("weno7_m", 3),
                                      ("weno5_p", 2), ("weno5_m", 2)])
def test_scheme_polynomial_exactness(name, deg):
    rng = np.random.default_rng(deg)
    for trial in range(5):
        coef = list(rng.uniform(-1, 1, size=deg + 1) * 1e-2)
        got = _flux_diff(name, coef, 0)
        assert abs(got - _exact_derivative(coef)) < 1e-12, (name, coef, got)


def test_weno7_smooth_order():
    # on a smooth sine the WENO7 face difference converges at high order
    errs = []
    for n in (16, 32, 64):
        h = 2 * math.pi / n
        xs = np.arange(-8, 9) * h + 0.3
        f = np.sin(xs)
        s = lambda F: oro.point("weno7_p", f[8 + F - 3: 8 + F + 4])
        d = (s(0) - s(-1)) / h
        errs.append(abs(d - math.cos(0.3)))
    assert errs[2] < errs[1] < errs[0]
    assert errs[1] / errs[2] > 30   # better than 5th order on this range


@pytest.mark.parametrize("name,n,deg", [("cd6", 7, 6), ("cd8", 9, 8)])
def test_central_derivative_exactness(name, n, deg):
    rng = np.random.default_rng(n)
    half = n // 2
    xs = np.arange(-half, half + 1, dtype=float)
    for _ in range(5):
        coef = rng.uniform(-1, 1, size=deg + 1)
        f = _poly_cells(coef, xs)
        assert abs(oro.point(name, f) - coef[1]) < 1e-10


def test_steger_warming_split_identity():
    rng = np.random.default_rng(3)
    gamma, ama = 1.4, 0.5
    for _ in range(20):
        d = rng.uniform(0.5, 2.0)
        u, v, w = rng.uniform(-1, 1, size=3)
        T = rng.uniform(0.5, 2.0)
        c = math.sqrt(T) / ama
        A = rng.uniform(-2, 2, size=3)
        out = oro.sw_split(d, u, v, w, c, *A, gamma=gamma, eps=0.0)
        fsum = out[:5] + out[5:]
        U = A @ np.array([u, v, w])
        p = d * c * c / gamma
        E = p / (gamma - 1) + 0.5 * d * (u * u + v * v + w * w)
        exact = np.array([d * U, d * u * U + p * A[0], d * v * U + p * A[1],
                          d * w * U + p * A[2], (E + p) * U])
        assert np.allclose(fsum, exact, rtol=1e-12, atol=1e-12)


def test_split_upwinding_signs():
    # supersonic to the right: all flux in f+, none in f-
    gamma, ama = 1.4, 1.0
    out = oro.sw_split(1.0, 3.0, 0.0, 0.0, 1.0, 1.0, 0.0, 0.0, gamma=gamma, eps=0.0)
    assert np.all(np.abs(out[5:]) < 1e-15)


def test_characteristic_matrices_are_inverse():
    rng = np.random.default_rng(5)
    for _ in range(20):
        u, v, w = rng.uniform(-1, 1, size=3)
        c = rng.uniform(0.5, 3.0)
        A = rng.uniform(-2, 2, size=3)
        L, R = oro.char_matrices(u, v, w, c, *A, gamma=1.4)
        assert np.allclose(L @ R, np.eye(5), atol=1e-12)


def test_symbo_limiter_linear_branch_p_only():
    # a linear ramp has equal total variation in every substencil: the
    # limited positive side takes the linear weights, the negative side
    # never does (its TVmin is never computed in the reference)
    s = np.linspace(0, 0.07, 8)
    lp = oro.point("weno7_symbo_p", s, 1, 5.0, 0.2)
    np_ = oro.point("weno7_symbo_p", s, 0, 5.0, 0.2)
    assert np.isfinite(lp) and np.isfinite(np_)
    # linear data: every candidate stencil is exact, so both give the face value
    assert abs(lp - np_) < 1e-12


def test_oracle_q_criterion_matches_its_formula():
    """The oracle's Q (get_Q, src/OCFD_ana.cu:317-456) on a periodic grid
    against the same formula in numpy: sixth-order central derivatives with
    the periodic wrap, the metrics, Q = (ux vy + ux wz + vy wz - uy vx -
    uz wx - vz wy) Ajac^2."""
    from ocfd_b200 import cases
    case = cases.random_smooth_case(12, 11, 10, seed=5, curvilinear=True)
    o = oro.Oracle(case.cfg, case.prims, case.metrics)
    q = o.q_criterion()
    prims = np.asarray(case.prims)
    met = np.asarray(case.metrics)
    nz, ny, nx = prims.shape[1:]
    h = [1.0 / (n - 1.0) for n in (nx, ny, nz)]
    axis = [2, 1, 0]

    def d(f, dir_):
        a = axis[dir_]
        r = lambda k: np.roll(f, -k, axis=a)
        return (45.0 * (r(1) - r(-1)) - 9.0 * (r(2) - r(-2)) + (r(3) - r(-3))) / 60.0 / h[dir_]

    g = [[d(prims[m], dd) for dd in range(3)] for m in (1, 2, 3)]
    Akx, Aky, Akz, Aix, Aiy, Aiz, Asx, Asy, Asz, Aj = (met[k] for k in (3, 4, 5, 6, 7, 8, 9, 10, 11, 12))
    grad = [[g[m][0] * A0 + g[m][1] * A1 + g[m][2] * A2 for (A0, A1, A2) in ((Akx, Aix, Asx), (Aky, Aiy, Asy), (Akz, Aiz, Asz))]
            for m in range(3)]
    (ux, uy, uz), (vx, vy, vz), (wx, wy, wz) = grad
    want = (ux * vy + ux * wz + vy * wz - uy * vx - uz * wx - vz * wy) * Aj * Aj
    assert np.linalg.norm(q - want) / np.linalg.norm(want) < 1e-12


def test_libc_rand_restatement():
    """The oracle's restatement of rand() from the C library's initial state
    (the phases of IBC 108's spanwise modes, MZMAX > 0) equals this host's
    own rand() after srand(1), draw for draw."""
    import ctypes
    libc = ctypes.CDLL(None)
    libc.srand(1)
    want = np.array([libc.rand() for _ in range(1000)], dtype=np.int64)
    got = oro.libc_rand(1000).astype(np.int64)
    assert np.array_equal(got, want)
    assert got[0] == 1804289383 and got[1] == 846930886
