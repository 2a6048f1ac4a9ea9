"""Host-side evaluation helpers on CPU: the shock-position measure of the
learned-switch evaluation, the per-variable error table of the precision
form, and the parameter-vector layout the switch kernels and the oracle
share.  No GPU calls."""
import numpy as np
import pytest

from ocfd_b200 import learned, lib, precision
from oracle import mlp_oracle as mo


def _shock_field(shift=0, n=32, seed=0):
    """Pressure with one strong jump per x line at a line-dependent cell,
    plus small noise."""
    rng = np.random.default_rng(seed)
    # a slow decrease along x keeps the periodic wrap's jump (0.1) below the shock's (0.5)
    p = 1.0 - 0.2 * np.arange(n) / n + 1e-3 * rng.standard_normal((4, 6, n))
    pos = (np.arange(24).reshape(4, 6) * 5 + 3) % (n - 6)
    for k in range(4):
        for j in range(6):
            p[k, j, pos[k, j] + 1 + shift:] += 0.5
    return p, pos


def test_shock_positions_find_the_jumps():
    p, pos = _shock_field()
    found, mag, keep = learned.shock_positions(p, q=0.0)
    assert np.array_equal(found, pos)
    assert keep.all() and np.all(mag > 0.4)


def test_shock_error_counts_cell_shifts():
    p0, _ = _shock_field()
    p1, _ = _shock_field(shift=1)
    assert learned.shock_error(p0, p0, q=0.0)["max_cells"] == 0
    e = learned.shock_error(p0, p1, q=0.0)
    assert e["max_cells"] == 1 and e["frac_within_1"] == 1.0 and e["lines"] == 24
    p2, _ = _shock_field(shift=3)
    assert learned.shock_error(p0, p2, q=0.0)["max_cells"] == 3


def test_shock_error_wraps_periodically():
    """Positions are compared around the periodic x direction: a jump found at
    cell n-2 and one found at cell 0 are 2 cells apart, not n-2."""
    n = 16
    a = np.ones((1, 1, n)); a[..., n - 1] += 1.0     # strongest |p[i+1]-p[i]| first at i = n-2
    b = np.ones((1, 1, n)); b[..., 0] += 1.0         # first at i = 0
    assert learned.shock_positions(a, q=0.0)[0][0, 0] == n - 2
    assert learned.shock_positions(b, q=0.0)[0][0, 0] == 0
    assert learned.shock_error(a, b, q=0.0)["max_cells"] == 2


def test_field_errors_relative_norms():
    rng = np.random.default_rng(1)
    ref = rng.standard_normal((5, 4, 4, 4)) + 3.0
    test = ref.copy()
    test[2] += 1e-6 * ref[2]
    e = precision.field_errors(test, ref)
    assert set(e) == set(precision.NAMES)
    assert e["rho"]["rel_l2"] == 0.0 and e["rho"]["rel_linf"] == 0.0
    assert e["rho_v"]["rel_l2"] == pytest.approx(1e-6, rel=1e-6)
    assert e["rho_v"]["rel_linf"] == pytest.approx(1e-6, rel=1e-6)


def test_parameter_vector_layout_matches_oracle():
    """init_params writes mu, sigma, W1, b1, W2, b2, W3, b3 at the offsets the
    oracle (and the kernels) read them from; biases start at zero."""
    mu = np.arange(14, dtype=np.float32)
    sg = np.arange(14, dtype=np.float32) + 1.0
    w = learned.init_params(mu, sg, seed=3)
    assert w.size == lib.mlp_nparam() == mo.NPARAM
    m, s, W1, b1, W2, b2, W3, b3 = mo.unpack(w)
    assert np.array_equal(m, mu) and np.array_equal(s, sg)
    assert W1.shape == (32, 14) and W2.shape == (32, 32) and W3.shape == (32,)
    assert not b1.any() and not b2.any() and b3 == 0.0
    assert W1.std() > 0.1 and W2.std() > 0.05
    # deterministic in the seed
    assert np.array_equal(w, learned.init_params(mu, sg, seed=3))
    assert not np.array_equal(w, learned.init_params(mu, sg, seed=4))
