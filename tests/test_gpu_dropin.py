"""The drop-in boundary, end to end: the reference's own program (its
main, parameter reader, initialisation, time loop, filter call, analysis and
output files, compiled from its sources) with its RHS-path calls --
du_comput, OCFD_time_advance, get_duvwT, get_Amu, OCFD_bc, filtering --
served by libocfd_b200 through opencfd-scu_b200/glue/ocfd_b200_glue.cu
(oracle/dropin.mk links it; the reference's sources are not edited).  Given
the same opencfd-scu.in / opencfd.dat / OCFD3d-Jacobi.dat, its OCFD%08d.dat
must match the stock reference build's to the parity bound."""
import numpy as np
import pytest

from ocfd_b200 import cases

pytestmark = pytest.mark.gpu

TOL = 1e-12


def rel_l2(a, b):
    return np.array([np.linalg.norm(a[m] - b[m]) / np.linalg.norm(b[m]) for m in range(a.shape[0])])


def _cases():
    filt = cases.random_smooth_case(17, 18, 13, seed=65, scheme_invis="SCHEME_HYBRIDAUTO", charteric=1, shock=True,
                                    iperiodic=(1, 0, 1), dif_bound=(0, 0, 1, 1, 0, 0))
    filt.cfg.hy_dp_intv = (0.01, 0.2)
    filt.cfg.filters = (((1, 1, 1, 1, 2, 15, 0, 18, 0, 13, 2), (0.9, 1e-5, 10.0)),)
    return [
        ("tgv16_weno7", lambda: cases.taylor_green(16, seed=3), 5),
        ("iso16_hybrid_char", lambda: cases.isotropic_turbulence(16, seed=9, charteric=1), 5),
        ("rnd_hybrid_char_closed_y_filter", lambda: filt, 4),
    ]


@pytest.mark.parametrize("name,make,nsteps", _cases(), ids=[c[0] for c in _cases()])
def test_reference_program_with_library_rhs(name, make, nsteps, gpu_lib):
    from oracle import ref_runner
    if not (ref_runner.available() and ref_runner.available(ref_runner.DROPIN_BIN)):
        pytest.skip("reference build or drop-in build (oracle/_ref) not present on this machine")
    stock, istep, tt, _, _ = ref_runner.run_and_read(make(), nsteps)
    mixed, istep2, tt2, _, out = ref_runner.run_and_read(make(), nsteps, binary=ref_runner.DROPIN_BIN)
    assert istep2 == istep == nsteps and tt2 == tt
    assert "ocfd_b200 glue" not in out
    err = rel_l2(mixed, stock)
    assert np.all(err <= TOL), (name, err)
    assert np.all(err > 0) or np.array_equal(mixed, stock)
