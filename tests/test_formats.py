"""Case-file formats shared with the reference: round trips and the error
behaviour on corrupted or truncated input (the reference aborts; this side
raises FormatError)."""
import os
import struct

import numpy as np
import pytest

from ocfd_b200 import cases, formats


def test_field_file_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    fields = [rng.standard_normal((3, 4, 5)) for _ in range(5)]
    p = tmp_path / "opencfd.dat"
    formats.write_field_file(str(p), fields, istep=17, tt=0.25)
    out, istep, tt = formats.read_field_file(str(p), (3, 4, 5))
    assert istep == 17 and tt == 0.25
    for a, b in zip(fields, out):
        assert np.array_equal(a, b)
    # layout: 20-byte header then per plane [int][nx*ny doubles][int]
    raw = p.read_bytes()
    assert len(raw) == 20 + 5 * 3 * (8 + 4 * 5 * 8)
    assert struct.unpack_from("<iidi", raw, 0) == (12, 17, 0.25, 12)
    assert struct.unpack_from("<i", raw, 20)[0] == 4 * 5 * 8


def test_metric_file_round_trip(tmp_path):
    met = cases.cartesian_metrics(6, 5, 4, 0.1, 0.2, 0.3)
    p = tmp_path / "OCFD3d-Jacobi.dat"
    formats.write_metric_file(str(p), met)
    out = formats.read_metric_file(str(p), (4, 5, 6))
    for a, b in zip(met, out):
        assert np.array_equal(a, b)


def test_truncated_field_file_raises(tmp_path):
    fields = [np.zeros((3, 4, 5)) for _ in range(5)]
    p = tmp_path / "f.dat"
    formats.write_field_file(str(p), fields)
    data = p.read_bytes()
    p.write_bytes(data[:-9])
    with pytest.raises(formats.FormatError):
        formats.read_field_file(str(p), (3, 4, 5))
    p.write_bytes(data[:10])
    with pytest.raises(formats.FormatError):
        formats.read_field_file(str(p), (3, 4, 5))


def test_corrupted_record_marker_raises(tmp_path):
    fields = [np.zeros((3, 4, 5)) for _ in range(5)]
    p = tmp_path / "f.dat"
    formats.write_field_file(str(p), fields)
    data = bytearray(p.read_bytes())
    struct.pack_into("<i", data, 20, 12345)
    p.write_bytes(bytes(data))
    with pytest.raises(formats.FormatError):
        formats.read_field_file(str(p), (3, 4, 5))


def test_config_round_trip(tmp_path):
    c = cases.taylor_green(16).cfg
    c.set_steps(7)
    p = tmp_path / "opencfd-scu.in"
    formats.write_config(str(p), c)
    r = formats.read_config(str(p))
    assert (r.nx, r.ny, r.nz) == (16, 16, 16)
    assert r.scheme_invis_id == 303 and r.scheme_vis_id == 203
    assert r.dt == c.dt and r.end_time == c.end_time
    assert r.steps_for_end_time() == 7


def test_config_parser_rules(tmp_path):
    # spaces inside keys are ignored; a last line without newline is skipped,
    # as in src/parameters.c:666-680
    text = "GRID _3D = 8 9 10\nSCHEME_INVIS = WENO5\nSCHEME_VIS = CD8\nRE = 10\nDT = 0.5"
    p = tmp_path / "opencfd-scu.in"
    p.write_text(text)
    c = formats.read_config(str(p))
    assert (c.nx, c.ny, c.nz) == (8, 9, 10)
    assert c.scheme_invis_id == 302 and c.scheme_vis_id == 204
    assert c.re == 10.0
    assert c.dt != 0.5        # no trailing newline: not read


def test_config_unknown_scheme_raises(tmp_path):
    p = tmp_path / "opencfd-scu.in"
    p.write_text("GRID_3D = 8 8 8\nSCHEME_INVIS = WENO9\nSCHEME_VIS = CD6\n")
    with pytest.raises(formats.FormatError):
        formats.read_config(str(p))


def test_restart_message_selects_the_field_file(tmp_path):
    """Opencfd.msg absent or negative: opencfd.dat; otherwise OCFD%08d.dat of
    its step, and that file reads back with its step and time."""
    d = str(tmp_path)
    assert formats.initial_field_file(d).endswith("opencfd.dat")
    formats.write_restart_step(os.path.join(d, "Opencfd.msg"), -1)
    assert formats.initial_field_file(d).endswith("opencfd.dat")
    formats.write_restart_step(os.path.join(d, "Opencfd.msg"), 1200)
    assert formats.read_restart_step(os.path.join(d, "Opencfd.msg")) == 1200
    path = formats.initial_field_file(d)
    assert os.path.basename(path) == "OCFD00001200.dat"
    rng = np.random.default_rng(0)
    f = [rng.standard_normal((3, 4, 5)) for _ in range(5)]
    formats.write_field_file(path, f, istep=1200, tt=0.25)
    g, istep, tt = formats.read_field_file(path, (3, 4, 5))
    assert istep == 1200 and tt == 0.25 and all(np.array_equal(a, b) for a, b in zip(f, g))
    with open(os.path.join(d, "Opencfd.msg"), "wb") as fh:
        fh.write(b"\x01\x02")
    with pytest.raises(formats.FormatError):
        formats.read_restart_step(os.path.join(d, "Opencfd.msg"))
