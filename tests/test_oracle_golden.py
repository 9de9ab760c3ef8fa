"""The oracle against golden vectors produced by the reference's own sources
(tests/golden/make_golden.py).  CPU only."""
import numpy as np
import pytest

from golden_io import load
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
