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


@pytest.mark.parametrize("text", [False, True])
def test_saved_restart_matches_continuous_run(tmp_path, text):
    """tests/test_simulation.cpp:169-231: an 8^3 channel (NXS = NZS = 4,
    NYS = 6, no dealiasing, constant flow rate, DT = 1e-4) run 6 steps, against
    3 steps, a restart file (text or binary), a fresh context that reads it
    (the checkpoint bit for bit, step 3, time 3 DT) and 3 more steps.  A restart
    holds no multistep history, so the continuation repeats the first-order
    startup (src/sim/simulation.cpp:36-45): relative L2 below 1e-7."""
    import dataclasses
    from oracle_cases import divergence_free_field, example_case
    m, p = example_case(NXS=4, NYS=6, NZS=4, N2=8, N=8)
    p = dataclasses.replace(p, DT=1e-4)
    u0 = np.stack(divergence_free_field(m, p, seed=12, amp=0.01), axis=-1)
    cont = ctx_for(m, p)
    cont.set_velocity(u0)
    cont.run(1, 6)
    cont.synchronize()
    ucont = cont.get_velocity()
    first = ctx_for(m, p)
    first.set_velocity(u0)
    first.run(1, 3)
    first.synchronize()
    ck = first.get_velocity()
    path = tmp_path / ("field_S_ 0.dat" if text else "field_S_ 0.bin")
    first.write_restart(str(path), 3, 3 * p.DT, text=text)
    first.close()
    res = ctx_for(m, p)
    step, time = res.read_restart(str(path))
    assert step == 3 and abs(time - 3 * p.DT) <= 1e-18
    assert np.array_equal(res.get_velocity(), ck)
    res.run(1, 3)
    res.synchronize()
    u = res.get_velocity()
    assert np.isfinite(u).all()
    assert np.sum(np.abs(ucont - u0) ** 2) > 1e-16          # an evolving field
    err = np.sqrt(np.sum(np.abs(u - ucont) ** 2) / np.sum(np.abs(ucont) ** 2))
    assert err < 1e-7
