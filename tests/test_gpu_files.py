"""Restart and physical-field files (cdns_write_restart / cdns_read_restart /
cdns_write_physical) against the files the reference's own FieldIO writes for
the same state (tests/golden/golden_files.npz, made by
tests/golden/make_golden.py): restart files byte for byte in both forms, the
physical files' headers byte for byte and their values (transform outputs) to
round-off; reading back, and the checks a reader makes."""
import numpy as np
import pytest

from golden_io import load
from test_gpu_parity import ctx_for

pytestmark = pytest.mark.gpu


def state():
    m, p, d = load("golden_files.npz")
    c = ctx_for(m, p)
    c.set_velocity(np.stack(list(d["u"]), axis=-1))
    c.set_pressure(d["p"])
    return m, p, d, c


def test_restart_files_match_reference_bytes(tmp_path):
    m, p, d, c = state()
    step, time = int(d["ntpit"]), float(d["time"])
    for text, key in ((False, "field_S__0_bin"), (True, "field_S__0_dat")):
        path = tmp_path / ("field_S_ 0." + ("dat" if text else "bin"))
        c.write_restart(str(path), step, time, text=text)
        assert path.read_bytes() == bytes(d[key])
        assert not (tmp_path / (path.name + ".tmp")).exists()


def test_physical_files_match_reference(tmp_path):
    m, p, d, c = state()
    step, time = int(d["ntpit"]), float(d["time"])
    path = tmp_path / "field_P_ 0.bin"
    c.write_physical(str(path), step, time)
    got, ref = path.read_bytes(), bytes(d["field_P__0_bin"])
    assert len(got) == len(ref) and got[:128] == ref[:128]
    a, b = np.frombuffer(got[128:], "<f8"), np.frombuffer(ref[128:], "<f8")
    assert np.abs(a - b).max() <= 1e-13 * np.abs(b).max()
    path = tmp_path / "field_P_ 0.dat"
    c.write_physical(str(path), step, time, text=True)
    gl, rl = path.read_text().split("\n"), bytes(d["field_P__0_dat"]).decode().split("\n")
    assert gl[0] == rl[0] and len(gl) == len(rl)
    a = np.array([float(x) for x in gl[1:] if x])
    b = np.array([float(x) for x in rl[1:] if x])
    assert np.abs(a - b).max() <= 1e-13 * np.abs(b).max()


def test_read_reference_restart_files(tmp_path):
    m, p, d, _ = state()
    u = np.stack(list(d["u"]), axis=-1)
    for key, name in (("field_S__0_bin", "r.bin"), ("field_S__0_dat", "r.dat")):
        path = tmp_path / name
        path.write_bytes(bytes(d[key]))
        c = ctx_for(m, p)
        step, time = c.read_restart(str(path))
        assert step == int(d["ntpit"]) and time == float(d["time"])
        assert np.array_equal(c.get_velocity(), u)


def test_restart_reader_checks(tmp_path):
    import cdns
    from oracle_cases import channel_case
    m, p, d, c = state()
    good = bytes(d["field_S__0_bin"])
    bad_mesh = ctx_for(*channel_case(32))
    path = tmp_path / "r.bin"
    path.write_bytes(good)
    with pytest.raises(cdns.CdnsError, match="does not match"):
        bad_mesh.read_restart(str(path))
    path.write_bytes(good[:-8])
    with pytest.raises(cdns.CdnsError, match="length"):
        c.read_restart(str(path))
    raw = bytearray(good)
    raw[128:136] = np.array([np.nan]).tobytes()
    path.write_bytes(bytes(raw))
    with pytest.raises(cdns.CdnsError, match="non-finite"):
        c.read_restart(str(path))
    text = tmp_path / "r.dat"
    text.write_text(bytes(d["field_S__0_dat"]).decode() + "(1,2)\n")
    with pytest.raises(cdns.CdnsError, match="extra"):
        c.read_restart(str(text))
    # tests/test_field_io.cpp:99-120: a restart cut to 64 bytes, in either
    # form, is rejected and leaves the state as it was
    u = np.stack(list(d["u"]), axis=-1)
    for key in ("field_S__0_bin", "field_S__0_dat"):
        path.write_bytes(bytes(d[key])[:64])
        with pytest.raises(cdns.CdnsError):
            c.read_restart(str(path))
        assert np.array_equal(c.get_velocity(), u)
