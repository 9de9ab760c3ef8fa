"""The oracle against golden vectors produced by the reference's own sources
(tests/golden/make_golden.py).  CPU only."""
import os

import numpy as np
import pytest

from golden_io import GOLDEN, load
from oracle_cases import orc


def _rel_max(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("name", ["golden_step.npz", "golden_example.npz"])
def test_oracle_steps_match_reference(name):
    m, p, d = load(name)
    sim = orc.Simulation(m, p, list(d["u0"]))
    with np.errstate(all="ignore"):
        sim.run(int(d["nsteps"]))
    for k in range(3):
        assert orc.rel_l2(sim.u[k], d["u"][k]) <= 1e-12
    assert orc.rel_l2(sim.pressure, d["p"]) <= 1e-10


def test_oracle_nonlinear_matches_reference():
    m, p, d = load("golden_nonlinear.npz")
    c = orc.make_constants(m, p.Re)
    N, _, B = orc.nonlinear_term(m, c, list(d["u"]))
    for k in range(3):
        assert _rel_max(N[k], d["N"][k]) <= 1e-12
    assert _rel_max(B[0], d["B"][0]) <= 1e-12 and _rel_max(B[1], d["B"][1]) <= 1e-12


def test_oracle_solve_matches_reference():
    m, p, d = load("golden_solve.npz")
    c = orc.make_constants(m, p.Re)
    s = orc.Solver(m, p, c)
    with np.errstate(all="ignore"):
        s.setup(float(d["g"]))
    bcv = [(d["bc_v"][k][0], d["bc_v"][k][1]) for k in range(3)]
    pres, vel = s.solve_modes(None, (d["bc_p"][0], d["bc_p"][1]), list(d["rhs"]), bcv, True)
    assert np.all(np.abs(pres - d["p"]) <= 1e-10 * np.maximum(1.0, np.abs(d["p"])))
    for k in range(3):
        assert np.all(np.abs(vel[k] - d["v"][k]) <= 1e-10 * np.maximum(1.0, np.abs(d["v"][k])))
    assert np.abs(s.state.u_unit - d["u_unit"]).max() <= 1e-12 * np.abs(d["u_unit"]).max()
    assert np.abs(s.state.w_unit - d["w_unit"]).max() <= 1e-12 * np.abs(d["w_unit"]).max()


def test_oracle_fine_transforms_match_reference():
    m, p, d = load("golden_fine.npz")
    phys = orc.fine_backward(m, d["U"])
    assert np.abs(phys - d["phys"]).max() <= 1e-13 * np.abs(d["phys"]).max()
    assert np.abs(orc.fine_forward(m, d["phys"]) - d["back"]).max() <= 1e-13


def plane_sum_scale(vp, pp):
    """Per-plane sums of the absolute values of the 20 moment terms (the
    round-off scale of sums that cancel, e.g. the plane mean of v)."""
    a = [np.abs(x) for x in vp]
    ap = np.abs(pp) + 0.5 * (a[0] ** 2 + a[1] ** 2 + a[2] ** 2)
    return orc.plane_moments(a, ap + 0.5 * (a[0] ** 2 + a[1] ** 2 + a[2] ** 2)) + 1e-300


def _coarse_case(d, tag):
    mm = [int(v) for v in d[f"{tag}_mesh"]]
    m = orc.Mesh(*mm, float(d[f"{tag}_dom"][0]), float(d[f"{tag}_dom"][1]))
    return m


@pytest.mark.parametrize("tag", ["full", "ragged"])
@pytest.mark.parametrize("kind", ["real", "arb"])
def test_oracle_coarse_transforms_match_reference(tag, kind):
    """Transforms::channel_xyzfft 'B'/'F' (src/fft/transforms.cpp:452-582),
    full spectrum (Nyquist halve/mirror) and ragged, realisable and arbitrary."""
    d = dict(np.load(os.path.join(GOLDEN, "golden_coarse.npz")))
    m = _coarse_case(d, tag)
    U, phys, back = d[f"{tag}_{kind}_U"], d[f"{tag}_{kind}_phys"], d[f"{tag}_{kind}_back"]
    assert _rel_max(orc.coarse_backward(m, U), phys) <= 1e-14
    assert _rel_max(orc.coarse_forward(m, phys), back) <= 1e-14


def test_oracle_output_reduction_matches_reference():
    """FieldIO::to_physical + Statistics::reduce + Diagnostics::evaluate
    (src/io/field_io.cpp:199-220, src/sim/statistics.cpp:55-110,
    src/sim/diagnostics.cpp:14-80) on a 16x17x16 state."""
    m, p, d = load("golden_reduce.npz")
    u = list(d["u"])
    vp, pp = orc.to_physical(m, u, d["p"])
    for k in range(3):
        assert _rel_max(vp[k], d["phys"][k]) <= 1e-14
    assert _rel_max(pp, d["phys"][3]) <= 1e-14
    planes = orc.plane_moments(vp, pp)
    ref = d["planes"]
    scale = plane_sum_scale(vp, pp).max(axis=0)   # per moment: its largest plane
    assert np.all(np.abs(planes - ref) <= 1e-13 * scale[None, :])
    assert np.all(d["flags"] == 1.0)
    ekt, tke, div = orc.diagnostics(m, orc.make_constants(m, p.Re), ref, u)
    v = d["values"]
    assert abs(ekt - v[0]) <= 1e-14 * v[0] and abs(tke - v[1]) <= 1e-13 * v[1]
    assert v[2] > 0.1 and abs(div - v[2]) <= 1e-12 * v[2] and v[3] == 1.0


def statistics_scale(m, u_list, p):
    """Per moment, the largest plane magnitude of the sums of absolute values
    of its terms over the sampled states: the round-off scale of a mean that
    cancels (the plane mean of v, the means at the no-slip walls)."""
    vp, pp = orc.to_physical(m, u_list, p)
    return plane_sum_scale(vp, pp).max(axis=0) / float(m.NX * m.NZ)


def test_oracle_statistics_run_matches_reference():
    """Simulation::run sampling Statistics after Nstat (src/sim/simulation.cpp:225-250,
    src/sim/statistics.cpp:117-139): the running means of the reference's own
    run, read at full precision, against the oracle's step loop and
    Statistics restatement (4 samples after 6 steps of a 16x17x16 channel)."""
    m, p, d = load("golden_stats.npz")
    sim = orc.Simulation(m, p, list(d["u0"]))
    st = orc.Statistics(m)
    scale = np.zeros(20)
    with np.errstate(all="ignore"):
        for it in range(1, int(d["nsteps"]) + 1):
            sim.step()
            if it > int(d["nstat"]):
                vp, pp = orc.to_physical(m, sim.u, sim.pressure)
                st.accumulate(orc.plane_moments(vp, pp), sim.dpdx, sim.dpdz)
                scale = np.maximum(scale, statistics_scale(m, sim.u, sim.pressure))
    for k in range(3):
        assert orc.rel_l2(sim.u[k], d["u"][k]) <= 1e-12
    assert st.count == int(d["count"]) == 4
    assert np.allclose(st.dp, d["dp_means"], rtol=0, atol=1e-14)
    # The states themselves agree to ~1e-12 (numpy's FFTs against the shim's),
    # so the means agree to that level of their round-off scale (measured
    # 2.1e-12 at most, in the pressure-velocity moments).
    slots = np.array(orc.STAT_SOURCE)   # plane moment behind each mean slot
    assert np.all(np.abs(st.means - d["means"]) <= 1e-11 * scale[slots][:, None])
