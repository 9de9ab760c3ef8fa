"""The reference's own driver with the GPU time step, against the reference's
own CPU build, on the same run directory.

tests/dropin builds the reference's src/main.cpp and the rest of its sources
unchanged, with Simulation::enqueue_serial_step (src/sim/simulation.cpp:142-171)
taken by channel-dns_b200/driver/cdns_serial_step.cpp (the cdns C ABI).  Both
binaries run the same config.toml from the same seeded restart (INDEX_CONT = 1,
binary v1 field_S_): 20 steps of the 32 x 33 x 32 channel (48^3 product
grid) at Re_tau 180 with diagnostics every 5 steps, restart and physical files
every 10 (format "both"), statistics sampled after step 10 and written every 5,
and two zero-amplitude disturbance injections (steps 7 and 14: the state goes
to the host and back with the multistep history kept); then 10 more steps
continued from the restart file each run wrote (Simulation::initialize,
src/sim/simulation.cpp:72-90), as the reference's restart test does
(tests/test_simulation.cpp:169-231).

Compared: the printed diagnostics and diagnostics.csv (EKT, TKE to 1e-10
relative, the divergence norm to 1e-10 of the velocity scale), the restart
files (same header bytes; payload relative L2 <= 1e-10 per component), the
physical files (relative max <= 1e-10 per field), and the statistics files
(Result/, which the reference prints with 8 decimals: equal to 2e-8)."""
import os
import re
import struct
import subprocess

import numpy as np
import pytest

import ref_io
from oracle_cases import channel_case, divergence_free_field, orc

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROPIN = os.path.join(ROOT, "tests", "dropin", "_build", "channel_dns_cdns")
REFCLI = os.path.join(ROOT, "oracle", "_ref", "channel_dns")


def run_dir(path, m, p, u0, nsteps):
    os.makedirs(path, exist_ok=True)
    ref_io.write_config(path, m, p, nsteps, ndumfrq=10, nprnfrq=5, fmt="both", nstat=10, physical_interval=10,
                        statistics_interval=5, ncount_disturb=2, ndisturbfrq=7, eps_disturb=0.0)
    if u0 is not None:
        ref_io.write_restart(path, m, u0)


def run(binary, path):
    r = subprocess.run([binary, "--threads", "4", path], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, f"{binary} failed:\n{r.stdout}\n{r.stderr}"
    return r.stdout


def diagnostics(stdout):
    out = {}
    for line in stdout.splitlines():
        mt = re.match(r"step = (\d+) TIME = (\S+) EKT = (\S+) TKE = (\S+) div_L2 = (\S+) finite = (\w+)", line)
        if mt:
            out[int(mt.group(1))] = (float(mt.group(2)), float(mt.group(3)), float(mt.group(4)),
                                     float(mt.group(5)), mt.group(6))
    return out


def restart_payload(path, m):
    raw = open(path, "rb").read()
    data = np.frombuffer(raw[128:], dtype="<c16").reshape(m.nkz, m.ncy, m.nkx, 3)
    return raw[:128], data


def numbers(path):
    """Every number of a text file; complex values "(re,im)" give two."""
    text = open(path).read().replace("(", " ").replace(")", " ").replace(",", " ")
    return np.array([float(t) for t in text.split()])


def compare_runs(gpu, ref, m, nsteps_printed):
    dg, dr = diagnostics(gpu[1]), diagnostics(ref[1])
    assert sorted(dg) == sorted(dr) and len(dg) == nsteps_printed
    for step in dr:
        tg, eg, kg, vg, fg = dg[step]
        tr, er, kr, vr, fr = dr[step]
        assert tg == tr and fg == fr == "true"
        assert abs(eg - er) <= 1e-10 * abs(er) and abs(kg - kr) <= 1e-10 * abs(kr)
        assert abs(vg - vr) <= 1e-10 * max(1.0, er) ** 0.5
    for name in ("diagnostics.csv",):
        lg = open(os.path.join(gpu[0], name)).read().splitlines()
        lr = open(os.path.join(ref[0], name)).read().splitlines()
        assert len(lg) == len(lr) and lg[0] == lr[0]
        for x, y in zip(lg[1:], lr[1:]):
            xs, ys = [float(t) for t in x.split(",")], [float(t) for t in y.split(",")]
            assert xs[:2] == ys[:2]
            assert np.all(np.abs(np.array(xs) - np.array(ys)) <= 1e-10 * np.maximum(1.0, np.abs(ys)))
    hg, ug = restart_payload(os.path.join(gpu[0], "field_S_ 0.bin"), m)
    hr, ur = restart_payload(os.path.join(ref[0], "field_S_ 0.bin"), m)
    assert hg == hr
    for k in range(3):
        assert orc.rel_l2(ug[..., k], ur[..., k]) <= 1e-10
    tg, tr = numbers(os.path.join(gpu[0], "field_S_ 0.dat")), numbers(os.path.join(ref[0], "field_S_ 0.dat"))
    assert tg.shape == tr.shape and np.abs(tg - tr).max() <= 1e-10 * np.abs(tr).max()
    pg = open(os.path.join(gpu[0], "field_P_ 0.bin"), "rb").read()
    pr = open(os.path.join(ref[0], "field_P_ 0.bin"), "rb").read()
    assert pg[:128] == pr[:128] and len(pg) == len(pr)
    fg = np.frombuffer(pg[128:], dtype="<f8").reshape(4, -1)
    fr = np.frombuffer(pr[128:], dtype="<f8").reshape(4, -1)
    for k in range(4):
        assert np.abs(fg[k] - fr[k]).max() <= 1e-10 * np.abs(fr[k]).max()
    for sub in ("0/DPDX_DPDZ.dat", "1/V_Pre_mean_Field_ 0.dat", "2/V_Pre_moment2_Field_ 0.dat",
                "3/V_Pre_moment3_Field_ 0.dat", "4/V_Pre_moment4_Field_ 0.dat"):
        sg = numbers(os.path.join(gpu[0], "Result", sub))
        sr = numbers(os.path.join(ref[0], "Result", sub))
        assert sg.shape == sr.shape and np.abs(sg - sr).max() <= 2e-8 * max(1.0, np.abs(sr).max())


def test_reference_driver_with_gpu_step(tmp_path):
    if not (os.access(DROPIN, os.X_OK) and os.access(REFCLI, os.X_OK)):
        pytest.fail("build tests/dropin and oracle/_ref first (python __graft_entry__.py)")
    m, p = channel_case(32)
    u0 = divergence_free_field(m, p, seed=0, amp=0.05, kmax=4)
    gpu, ref = str(tmp_path / "gpu"), str(tmp_path / "ref")
    for d in (gpu, ref):
        run_dir(d, m, p, u0, 20)
    out_g, out_r = run(DROPIN, gpu), run(REFCLI, ref)
    assert out_g.count("disturbance at step") == out_r.count("disturbance at step") == 2
    compare_runs((gpu, out_g), (ref, out_r), m, 4)
    # continuation from the restart each run wrote at step 20
    for d in (gpu, ref):
        run_dir(d, m, p, None, 10)
        assert struct.unpack("<q", open(os.path.join(d, "field_S_ 0.bin"), "rb").read()[16:24])[0] == 20
    out_g, out_r = run(DROPIN, gpu), run(REFCLI, ref)
    compare_runs((gpu, out_g), (ref, out_r), m, 2)
    assert "step = 30 " in out_g


def test_update_velocity_keeps_the_multistep_history():
    """cdns_update_velocity between steps 3 and 4 against the oracle's step
    loop with the same change made to its velocity (second order continues,
    as after Simulation::apply_disturbance)."""
    from test_gpu_parity import ctx_for
    m, p = channel_case(16)
    u0 = divergence_free_field(m, p, seed=5, amp=0.05, kmax=4)
    delta = divergence_free_field(m, p, seed=6, amp=0.01, kmax=3)
    delta[0][m.NZS, :, 0] = 0.0   # a mean-free change
    sim = orc.Simulation(m, p, u0)
    with np.errstate(all="ignore"):
        sim.run(3)
        sim.u = [sim.u[k] + delta[k] for k in range(3)]
        sim.run(3)
    c = ctx_for(m, p)
    c.set_velocity(np.stack(u0, axis=-1))
    c.run(1, 3)
    c.synchronize()
    c.update_velocity(c.get_velocity() + np.stack(delta, axis=-1))
    c.run(4, 3)
    c.synchronize()
    v = c.get_velocity()
    for k in range(3):
        assert orc.rel_l2(v[..., k], sim.u[k]) <= 1e-10
