"""Drive the reference's own sources built in oracle/_ref (test infrastructure).

Writes run directories in the reference's formats -- ``config.toml``
(src/core/params.cpp:130-228 keys) and the binary v1 restart
``field_S_ 0.bin`` (src/io/field_io.cpp:121-140, 128-byte header) -- runs
``_ref/ref_runner`` and reads its outputs back as numpy arrays in the
spectral layout [kz][y][kx] per component.
"""
from __future__ import annotations

import os
import struct
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
RUNNER = os.path.join(REF_DIR, "ref_runner")
CLI = os.path.join(REF_DIR, "channel_dns")


def available() -> bool:
    return os.access(RUNNER, os.X_OK)


def build(ref_root: str) -> bool:
    """Compile the reference sources with the shims (needs the reference tree)."""
    if not os.path.isdir(os.path.join(ref_root, "src")):
        return available()
    subprocess.run(["make", "-s", "-C", HERE, f"REF={ref_root}", "-j8"], check=True)
    return available()


def write_config(run_dir: str, m, p, nsteps: int, index_cont: int = 1, ndumfrq: int | None = None,
                 nprnfrq: int | None = None, fmt: str = "binary", nstat: int | None = None,
                 physical_interval: int = 0, statistics_interval: int | None = None,
                 ncount_disturb: int = 0, ndisturbfrq: int = 1, eps_disturb: float = 0.0) -> None:
    def f(x):
        return repr(float(x))

    big = 10 ** 9
    text = f"""[mesh]
NX = {m.NX}
NY = {m.NY}
NZ = {m.NZ}
INDEX_disturb_Z = 3
NXS = {m.NXS}
NYS = {m.NYS}
NZS = {m.NZS}
NX2 = {m.NX2}
NY2 = {m.NY2}
NZ2 = {m.NZ2}
INDEX_Serial = 1

[parm]
XL = {f(m.XL)}
ZL = {f(m.ZL)}
THETA = {f(p.THETA)}
INDEX_GRAD_PRE = {p.INDEX_GRAD_PRE}
Re = {f(p.Re)}
INDEX_UNSTEADY_BC = 0
G_pre = {f(p.G_pre)}
a_pre0 = {f(p.a_pre0)}
b_pre0 = {f(p.b_pre0)}
a_V = [{f(p.a_V[0])}, {f(p.a_V[1])}, {f(p.a_V[2])}]
b_V = [{f(p.b_V[0])}, {f(p.b_V[1])}, {f(p.b_V[2])}]

[control]
INDEX_CONT = {index_cont}
EPS_init = 0.0
NSTEPS = {nsteps}
NDUMFRQ = {ndumfrq or big}
NPRNFRQ = {nprnfrq or big}
DT = {f(p.DT)}
NCOUNT_disturb = {ncount_disturb}
NDISTURBFRQ = {ndisturbfrq}
EPS_disturb = {f(eps_disturb)}
V_Microblow0 = {f(p.V_Microblow0)}
Nstat = {big if nstat is None else nstat}

[output]
format = "{fmt}"
physical_interval = {physical_interval}
statistics_interval = {big if statistics_interval is None else statistics_interval}
"""
    with open(os.path.join(run_dir, "config.toml"), "w") as fh:
        fh.write(text)


def write_restart(run_dir: str, m, velocity, ntpit: int = 0, time: float = 0.0) -> None:
    """Binary v1 restart (src/io/field_io.cpp:121-140, :286-299)."""
    hdr = b"CHDNS\x00\x00\x00" + struct.pack("<IIqd", 1, 1, ntpit, time)
    dims = [m.NX, m.NY + 1, m.NZ, 3, m.nkz, m.nkx, 0, 1, 0, m.nkx, 0, m.NYS + 1]
    hdr += struct.pack("<12q", *dims)
    assert len(hdr) == 128
    a = np.stack([np.asarray(v, dtype=np.complex128) for v in velocity], axis=-1)
    with open(os.path.join(run_dir, "field_S_ 0.bin"), "wb") as fh:
        fh.write(hdr)
        fh.write(np.ascontiguousarray(a).astype("<c16").tobytes())


def run_steps(m, p, velocity, nsteps: int, threads: int = 1, workdir: str | None = None,
              nstat: int | None = None):
    """Run the reference step loop from a restart; returns (u list, pressure,
    wall_s), and with ``nstat`` (Simulation::run samples statistics at every
    step ntpit > nstat, src/sim/simulation.cpp:225-250) a fourth item: the
    Statistics running means at full precision, a dict with "count",
    "dp_means" (dpdx, dpdz) and "means" [20][NY+1] in Statistics::write's
    order (u v w, p, uu vv ww uv vw wu, pp, pu pv pw, u^3 v^3 w^3, u^4 v^4 w^4)."""
    own = workdir is None
    d = workdir or tempfile.mkdtemp(prefix="cdns_ref_")
    write_config(d, m, p, nsteps, nstat=nstat)
    write_restart(d, m, velocity)
    out = os.path.join(d, "out.bin")
    cmd = [RUNNER, "run", d, out, str(threads)]
    if nstat is not None:
        cmd.append(os.path.join(d, "stats.bin"))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"ref_runner run failed: {r.stderr}\n{r.stdout}")
    wall = None
    for line in r.stdout.splitlines():
        if line.startswith("ref_runner: steps"):
            wall = float(line.split()[4])
    raw = open(out, "rb").read()
    nt, t = struct.unpack("<qd", raw[:16])
    n = m.nkz * m.ncy * m.nkx
    data = np.frombuffer(raw[16:], dtype="<c16")
    vel = data[: 3 * n].reshape(m.nkz, m.ncy, m.nkx, 3)
    pres = data[3 * n: 4 * n].reshape(m.nkz, m.ncy, m.nkx).copy()
    stats = None
    if nstat is not None:
        sraw = open(os.path.join(d, "stats.bin"), "rb").read()
        count, = struct.unpack("<q", sraw[:8])
        vals = np.frombuffer(sraw[8:], dtype="<f8")
        stats = {"count": int(count), "dp_means": (float(vals[0]), float(vals[1])),
                 "means": vals[2:].reshape(20, m.NY + 1).copy()}
    if own:
        _rmtree(d)
    u = [vel[..., k].copy() for k in range(3)]
    return (u, pres, wall) if nstat is None else (u, pres, wall, stats)


def nonlinear(m, p, velocity):
    d = tempfile.mkdtemp(prefix="cdns_ref_")
    write_config(d, m, p, 1)
    inp = os.path.join(d, "u.bin")
    np.stack(velocity, axis=-1).astype("<c16").tofile(inp)
    out = os.path.join(d, "nl.bin")
    subprocess.run([RUNNER, "nonlinear", d, inp, out], check=True, capture_output=True)
    raw = np.fromfile(out, dtype="<c16")
    n = m.nkz * m.ncy * m.nkx
    N = raw[: 3 * n].reshape(m.nkz, m.ncy, m.nkx, 3)
    bc = raw[3 * n:].reshape(m.nkz, 2, m.nkx)
    _rmtree(d)
    return [N[..., k].copy() for k in range(3)], (bc[:, 0].copy(), bc[:, 1].copy())


def fine(m, p, spectral):
    d = tempfile.mkdtemp(prefix="cdns_ref_")
    write_config(d, m, p, 1)
    inp = os.path.join(d, "s.bin")
    np.asarray(spectral, dtype="<c16").tofile(inp)
    out = os.path.join(d, "f.bin")
    subprocess.run([RUNNER, "fine", d, inp, out], check=True, capture_output=True)
    raw = open(out, "rb").read()
    nphys = m.NZ2 * m.ny2 * m.NX2
    phys = np.frombuffer(raw[: 8 * nphys], dtype="<f8").reshape(m.fine_shape()).copy()
    back = np.frombuffer(raw[8 * nphys:], dtype="<c16").reshape(m.spectral_shape()).copy()
    _rmtree(d)
    return phys, back


def coarse(m, p, spectral):
    """Reference coarse transform 'B' then 'F' (physical [NZ][NY+1][NX], spectral)."""
    d = tempfile.mkdtemp(prefix="cdns_ref_")
    write_config(d, m, p, 1)
    inp = os.path.join(d, "s.bin")
    np.asarray(spectral, dtype="<c16").tofile(inp)
    out = os.path.join(d, "c.bin")
    subprocess.run([RUNNER, "coarse", d, inp, out], check=True, capture_output=True)
    raw = open(out, "rb").read()
    nphys = m.NZ * (m.NY + 1) * m.NX
    phys = np.frombuffer(raw[: 8 * nphys], dtype="<f8").reshape(m.NZ, m.NY + 1, m.NX).copy()
    back = np.frombuffer(raw[8 * nphys:], dtype="<c16").reshape(m.spectral_shape()).copy()
    _rmtree(d)
    return phys, back


def blocks(m, p, ranks: int):
    """The reference Mesh's block tables for a `ranks`-way split: int array
    [ranks][5] (x_begin, x_count, y2_begin, y2_count, owns_zero_x_mode), or
    None if Mesh rejects the split."""
    d = tempfile.mkdtemp(prefix="cdns_ref_")
    write_config(d, m, p, 1)
    out = os.path.join(d, "b.bin")
    subprocess.run([RUNNER, "blocks", d, str(ranks), out], check=True, capture_output=True)
    raw = np.frombuffer(open(out, "rb").read(), dtype="<i4").copy()
    _rmtree(d)
    if raw.size == 1 and raw[0] == -1:
        return None
    return raw.reshape(ranks, 5)


def reduce(m, p, velocity, pressure):
    """Reference output branch on a state: physical (u, v, w, p), plane sums
    [NY+1][20], plane finite flags, (EKT, TKE, div_L2, finite)."""
    d = tempfile.mkdtemp(prefix="cdns_ref_")
    write_config(d, m, p, 1)
    inp = os.path.join(d, "st.bin")
    with open(inp, "wb") as fh:
        fh.write(np.stack(velocity, axis=-1).astype("<c16").tobytes())
        fh.write(np.asarray(pressure).astype("<c16").tobytes())
    out = os.path.join(d, "r.bin")
    subprocess.run([RUNNER, "reduce", d, inp, out], check=True, capture_output=True)
    raw = np.frombuffer(open(out, "rb").read(), dtype="<f8")
    nphys = m.NZ * (m.NY + 1) * m.NX
    ny1 = m.NY + 1
    phys = raw[: 4 * nphys].reshape(4, m.NZ, ny1, m.NX).copy()
    planes = raw[4 * nphys: 4 * nphys + 20 * ny1].reshape(ny1, 20).copy()
    flags = raw[4 * nphys + 20 * ny1: 4 * nphys + 21 * ny1].copy()
    values = raw[4 * nphys + 21 * ny1:].copy()
    _rmtree(d)
    return phys, planes, flags, values


def dump(m, p, velocity, pressure, ntpit: int, time: float) -> dict:
    """The reference's FieldIO files (format "both") of a state: returns
    {file name: bytes} for field_S_ 0.bin/.dat and field_P_ 0.bin/.dat."""
    d = tempfile.mkdtemp(prefix="cdns_ref_")
    write_config(d, m, p, 1)
    inp = os.path.join(d, "st.bin")
    with open(inp, "wb") as fh:
        fh.write(np.stack(velocity, axis=-1).astype("<c16").tobytes())
        fh.write(np.asarray(pressure).astype("<c16").tobytes())
    subprocess.run([RUNNER, "dump", d, inp, str(int(ntpit)), repr(float(time))], check=True, capture_output=True)
    out = {}
    for name in ("field_S_ 0.bin", "field_S_ 0.dat", "field_P_ 0.bin", "field_P_ 0.dat"):
        with open(os.path.join(d, name), "rb") as fh:
            out[name] = fh.read()
    _rmtree(d)
    return out


def solve(m, p, g, rhs_v, bc_p, bc_v):
    d = tempfile.mkdtemp(prefix="cdns_ref_")
    write_config(d, m, p, 1)
    inp = os.path.join(d, "r.bin")
    with open(inp, "wb") as fh:
        fh.write(np.stack(rhs_v, axis=-1).astype("<c16").tobytes())
        fh.write(np.stack(bc_p, axis=1).astype("<c16").tobytes())
        fh.write(np.stack([np.stack(b, axis=1) for b in bc_v], axis=-1).astype("<c16").tobytes())
    out = os.path.join(d, "o.bin")
    subprocess.run([RUNNER, "solve", d, repr(float(g)), inp, out], check=True, capture_output=True)
    raw = open(out, "rb").read()
    n = m.nkz * m.ncy * m.nkx
    c = np.frombuffer(raw[: 16 * 4 * n], dtype="<c16")
    pres = c[:n].reshape(m.spectral_shape()).copy()
    vel = c[n:4 * n].reshape(m.nkz, m.ncy, m.nkx, 3)
    units = np.frombuffer(raw[16 * 4 * n:], dtype="<f8")
    _rmtree(d)
    return pres, [vel[..., k].copy() for k in range(3)], units[: m.ncy].copy(), units[m.ncy:].copy()


def _rmtree(d: str) -> None:
    import shutil
    shutil.rmtree(d, ignore_errors=True)
