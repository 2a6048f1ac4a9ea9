"""The allocation-free field-mean entry point (ocfd_b200_field_means_noalloc)
against the context reduction (ocfd_b200_ana_residual), called through the
C ABI.  Collected last so that it also runs after everything else in the
process has used the library; it passes alone in a fresh process too.

Tolerance: the mean of E must match ana_residual to 1e-14 relative (the two
use the same summation order, so it is expected to be bitwise); the other
fields are checked against numpy to 1e-13 relative.
"""
import ctypes

import numpy as np
import pytest

from ocfd_b200 import cases, lib

pytestmark = pytest.mark.gpu

TOL_SAME = 1e-14
TOL_NUMPY = 1e-13


def _means_noalloc(L, dev_fields, nfield, n, torch):
    out = torch.full((nfield,), float("nan"), dtype=torch.float64, device=dev_fields.device)
    stream = torch.cuda.current_stream().cuda_stream
    rc = L.ocfd_b200_field_means_noalloc(ctypes.c_void_p(dev_fields.data_ptr()), nfield, n,
                                         ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream))
    assert rc == lib.OCFD_OK, (L.ocfd_b200_last_error(None) or b"").decode()
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _check_state(L, s, torch):
    cons = s.conserved()                                # [5, nz, ny, nx]
    n = cons[0].size
    dev = torch.from_numpy(np.ascontiguousarray(cons)).to("cuda:0")
    got = _means_noalloc(L, dev, 5, n, torch)
    ref_e = s.ana_residual(0)
    assert abs(got[4] - ref_e) <= TOL_SAME * abs(ref_e), (got[4], ref_e)
    for m in range(5):
        want = cons[m].mean(dtype=np.float64)
        scale = max(abs(want), np.abs(cons[m]).mean())
        assert abs(got[m] - want) <= TOL_NUMPY * scale, (m, got[m], want)
    return got


def test_field_means_noalloc_matches_ana_residual_on_two_calls_in_a_row():
    torch = pytest.importorskip("torch")
    L = lib.load()
    case = cases.isotropic_turbulence(32, seed=11, charteric=1)
    s = lib.Solver(case.cfg, case.prims, case.metrics)
    try:
        s.step(1)
        first = _check_state(L, s, torch)
        s.step(1)
        second = _check_state(L, s, torch)
        assert not np.array_equal(first, second)      # the state moved; each call saw its own
    finally:
        s.close()


def test_field_means_noalloc_rejects_sizes_beyond_the_scratch():
    torch = pytest.importorskip("torch")
    L = lib.load()
    dev = torch.zeros(9 * 16, dtype=torch.float64, device="cuda:0")
    out = torch.zeros(9, dtype=torch.float64, device="cuda:0")
    rc = L.ocfd_b200_field_means_noalloc(ctypes.c_void_p(dev.data_ptr()), 9, 16,
                                         ctypes.c_void_p(out.data_ptr()), None)
    assert rc == -1
    assert b"outside 1..8" in L.ocfd_b200_last_error(None)
    rc = L.ocfd_b200_field_means_noalloc(ctypes.c_void_p(dev.data_ptr()), 1, 0,
                                         ctypes.c_void_p(out.data_ptr()), None)
    assert rc == -1
