"""Stage-by-stage parity at the full Re_tau = 180 size (128 x 129 x 128 base
grid, 196 x 193 x 196 product grid): fine transforms, nonlinear term, solver
and two time steps against the oracle.  Needs a B200; the oracle takes a few
seconds per stage at this size.  Tolerances as in test_gpu_parity.py."""
import numpy as np
import pytest

from oracle_cases import band_spectrum, divergence_free_field, orc, retau180_case
from test_gpu_parity import ctx_for, rel_max

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case():
    m, p = retau180_case()
    u0 = divergence_free_field(m, p, seed=1, amp=0.1, spectrum="k53", mean="loglaw")
    return m, p, u0


def test_retau180_fine_transforms(case):
    m, p, _ = case
    U = band_spectrum(m, 9)
    c = ctx_for(m, p)
    phys_ref = orc.fine_backward(m, U)
    phys = c.transform_fine("B", U)
    assert rel_max(phys, phys_ref) <= 1e-12
    back = c.transform_fine("F", phys_ref)
    assert rel_max(back, orc.fine_forward(m, phys_ref)) <= 1e-12
    assert np.abs(back - U).max() <= 1e-12 * np.abs(U).max()


def test_retau180_nonlinear(case):
    m, p, u0 = case
    cst = orc.make_constants(m, p.Re)
    N_ref, _, B_ref = orc.nonlinear_term(m, cst, u0)
    c = ctx_for(m, p)
    N, B = c.nonlinear(np.stack(u0, axis=-1))
    for k in range(3):
        assert rel_max(N[..., k], N_ref[k]) <= 1e-12
    scale = max(np.abs(B_ref[0]).max(), np.abs(N_ref[1]).max() * (m.NYS + 1))
    assert np.abs(B[:, 0] - B_ref[0]).max() <= 1e-12 * scale
    assert np.abs(B[:, 1] - B_ref[1]).max() <= 1e-12 * scale


def test_retau180_solver(case):
    m, p, _ = case
    a0, a1, b0, b1, g = orc.step_coefficients(2, p.DT, p.Re)
    cst = orc.make_constants(m, p.Re)
    s = orc.Solver(m, p, cst)
    with np.errstate(all="ignore"):
        s.setup(g)
    rng = np.random.default_rng(5)
    sh = m.spectral_shape()
    rv = [(rng.standard_normal(sh) + 1j * rng.standard_normal(sh)) for _ in range(3)]
    zb = np.zeros((m.nkz, m.nkx), dtype=np.complex128)
    bp = (rng.standard_normal((m.nkz, m.nkx)) + 0j, rng.standard_normal((m.nkz, m.nkx)) + 0j)
    ep, ev = s.solve_modes(None, bp, rv, [(zb, zb)] * 3, True)
    c = ctx_for(m, p)
    pres, vel, uu, wu = c.solve(g, np.stack(rv, axis=-1), np.stack(bp, axis=1),
                                np.zeros((m.nkz, 2, m.nkx, 3), dtype=np.complex128))
    assert np.abs(pres - ep).max() <= 1e-10 * max(1.0, np.abs(ep).max())
    for k in range(3):
        assert np.abs(vel[..., k] - ev[k]).max() <= 1e-10 * max(1.0, np.abs(ev[k]).max())
    assert np.abs(uu - s.state.u_unit).max() <= 1e-12 * np.abs(s.state.u_unit).max()


def test_retau180_two_steps(case):
    m, p, u0 = case
    sim = orc.Simulation(m, p, u0)
    with np.errstate(all="ignore"):
        sim.run(2)
    c = ctx_for(m, p)
    c.set_velocity(np.stack(u0, axis=-1))
    c.run(1, 2)
    c.synchronize()
    v = c.get_velocity()
    for k in range(3):
        assert orc.rel_l2(v[..., k], sim.u[k]) <= 1e-10
    cst = orc.make_constants(m, p.Re)
    div = orc.divergence(cst, [v[..., k] for k in range(3)])
    assert np.abs(div).max() <= 1e-12 * max(1.0, np.abs(v).max())
