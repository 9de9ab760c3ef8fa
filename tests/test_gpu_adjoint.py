"""Discrete adjoint of the FP64 step (cdns_adjoint_run and the stage
transposes).  The reference has no adjoint, so nothing pins it to the
reference itself; it is pinned to the library's own forward step, which is
pinned to the reference at 1e-10:

- the solve transpose by the dot-product identity <lx, S x> = <S^T lx, x>
  (S linear) under the real inner product Re sum conj(a) b;
- the nonlinear-term transpose by <lN, N(u+d) - N(u-d)> = 2 <N'(u)^T lN, d>
  (exact for the quadratic u x omega);
- the full gradient (initial velocity and wall blowing/suction) by central
  finite differences along seeded random directions: of a projection
  objective Re <w, u^n> (every stage of the step, well conditioned), and of
  the wall-shear objective with the adjoint workload's sizes: 64 x 65 x 64
  at Re_tau 180, 50 steps, checkpoints every 10 steps, 8 directions,
  agreement to 1e-6."""
import numpy as np
import pytest

import cdns
from oracle_cases import band_spectrum, channel_case, divergence_free_field
from test_gpu_parity import ctx_for

pytestmark = pytest.mark.gpu


def rdot(a, b):
    """Real inner product Re sum conj(a) b."""
    return float(np.sum(np.real(np.conj(a) * b)))


def crandom(rng, shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def wall_control(m, seed, kmax=8, amp=1.0):
    """Wall-normal blowing/suction of the |k| <= kmax modes at both walls."""
    from cdns.fields import blowing_suction
    return blowing_suction(m, seed, kmax=kmax, amp=amp)


@pytest.mark.parametrize("n", [32, 64])
def test_solve_adjoint_dot_product(n):
    m, p = channel_case(n)
    ctx = ctx_for(m, p)
    nkz, ncy, nkx = m.spectral_shape()
    rng = np.random.default_rng(3 + n)
    for it in (1, 2):
        a0, a1, b0, b1, g = cdns.step_coefficients(it, p.DT, p.Re)
        rhs = crandom(rng, (nkz, ncy, nkx, 3))
        pbc = crandom(rng, (nkz, 2, nkx))
        vbc = crandom(rng, (nkz, 2, nkx, 3))
        P, V, _, _ = ctx.solve(g, rhs, pbc, vbc)
        lp = crandom(rng, (nkz, ncy, nkx))
        lv = crandom(rng, (nkz, ncy, nkx, 3))
        lr, lpb, lvb = ctx.solve_adjoint(g, lp, lv)
        lhs = rdot(lp, P) + rdot(lv, V)
        rhs_ = rdot(lr, rhs) + rdot(lpb, pbc) + rdot(lvb, vbc)
        scale = sum(np.abs(np.conj(x) * y).sum() for x, y in ((lp, P), (lv, V)))
        assert abs(lhs - rhs_) <= 1e-12 * scale, (it, lhs, rhs_, scale)


@pytest.mark.parametrize("form", ["matrix", "fft"])
@pytest.mark.parametrize("n", [32, 48])
def test_nonlinear_adjoint_dot_product(n, form, monkeypatch):
    """<lN, N(u+d) - N(u-d)> = 2 <N'(u)^T lN, d> (u x omega is quadratic), with
    the Chebyshev stages and their transposes in the matrix or the FFT form."""
    monkeypatch.setenv("CDNS_Y_TRANSFORM", form)
    m, p = channel_case(n)
    ctx = ctx_for(m, p)
    assert ctx.tuning()["y_synthesis"] == form
    nkz, ncy, nkx = m.spectral_shape()
    u = np.stack(divergence_free_field(m, p, seed=5, amp=0.1, kmax=6), axis=-1)
    d = np.stack([band_spectrum(m, seed=20 + c, amp=0.05) for c in range(3)], axis=-1)
    rng = np.random.default_rng(n)
    lN = crandom(rng, (nkz, ncy, nkx, 3))
    lB = crandom(rng, (nkz, 2, nkx))
    Np, Bp = ctx.nonlinear(u + d)
    Nm, Bm = ctx.nonlinear(u - d)
    lhs = rdot(lN, Np - Nm) + rdot(lB, Bp - Bm)
    lu = ctx.nonlinear_adjoint(u, lN, lB)
    rhs_ = 2.0 * rdot(lu, d)
    scale = np.abs(np.conj(lN) * (Np - Nm)).sum() + np.abs(np.conj(lB) * (Bp - Bm)).sum()
    assert abs(lhs - rhs_) <= 1e-11 * scale, (lhs, rhs_, scale)


def perturbation(m, p, seed):
    """Divergence-free, no-slip direction of the initial field (no mean flow)."""
    du = np.stack(divergence_free_field(m, p, seed=seed, amp=0.05, kmax=8), axis=-1)
    du[m.NZS, :, 0, :] = 0.0
    return du


def _fd_check(m, p, u0, bc0, nsteps, kck, directions, eps_u, eps_c, tol, weights=None, order=2):
    """Gradient of the objective against central differences (order 2 or 4)
    along each (kind, du, dc) direction of (initial velocity, wall data)."""
    ctx = ctx_for(m, p)
    ctx.set_velocity(u0)
    J0, gu, gb = ctx.adjoint_run(nsteps, kck, control=bc0, weights=weights)
    # the context now holds the state after nsteps steps, as after run(1, nsteps)
    ref = ctx_for(m, p)
    ref.set_velocity(u0)
    ref.set_velocity_bc(bc0)
    ref.run(1, nsteps)
    ref.synchronize()
    assert np.array_equal(ctx.get_velocity(), ref.get_velocity())

    def J(t, du, dc):
        ctx.set_velocity(u0 + t * du)
        return ctx.adjoint_run(nsteps, kck, control=bc0 + t * dc, gradient=False, weights=weights)[0]

    assert J(0.0, u0, bc0) == J0
    for kind, du, dc in directions:
        h = eps_u if kind == "u" else eps_c
        if order == 2:
            fd = (J(h, du, dc) - J(-h, du, dc)) / (2.0 * h)
        else:
            fd = (J(-2 * h, du, dc) - 8 * J(-h, du, dc) + 8 * J(h, du, dc) - J(2 * h, du, dc)) / (12.0 * h)
        ad = rdot(gu, du) + rdot(gb, dc)
        assert abs(fd - ad) <= tol * abs(ad), (kind, fd, ad, abs(fd - ad) / abs(ad))


def mean_profile(m, rng, scale=0.3):
    """Random streamwise mean-profile direction (the (0, 0) mode of u)."""
    d = np.zeros((2 * m.NZS + 1, m.NYS + 1, m.NXS + 1, 3), dtype=np.complex128)
    d[m.NZS, :, 0, 0] = rng.standard_normal(m.NYS + 1) * scale
    return d


@pytest.mark.parametrize("form", ["matrix", "fft"])
def test_adjoint_vjp_small_channel(form, monkeypatch):
    """Vector-Jacobian product of 6 steps of a 32^3 channel (projection
    objective Re <w, u^6>, checkpoints every 4 steps: a partial last
    interval): initial-field fluctuations, mean profile, blowing/suction
    modes and uniform blowing; Chebyshev stages in either form."""
    monkeypatch.setenv("CDNS_Y_TRANSFORM", form)
    m, p = channel_case(32)
    u0 = np.stack(divergence_free_field(m, p, seed=1, amp=0.1, spectrum="k53", mean="loglaw"), axis=-1)
    bc0 = wall_control(m, seed=2, amp=1e-3)
    rng = np.random.default_rng(5)
    w = crandom(rng, u0.shape)
    uniform = np.zeros_like(bc0)
    uniform[m.NZS, :, 0, 1] = [1.0, 0.7]
    zu, zb = np.zeros_like(u0), np.zeros_like(bc0)
    dirs = [("u", perturbation(m, p, 40), zb), ("u", perturbation(m, p, 41), zb), ("u", mean_profile(m, rng), zb),
            ("bc", zu, wall_control(m, seed=60)), ("bc", zu, wall_control(m, seed=61)), ("bc", zu, uniform)]
    _fd_check(m, p, u0, bc0, nsteps=6, kck=4, directions=dirs, eps_u=1e-3, eps_c=1e-5, tol=1e-7, weights=w)


def _config4():
    m, p = channel_case(64)
    u0 = np.stack(divergence_free_field(m, p, seed=1, amp=0.1, spectrum="k53", mean="loglaw"), axis=-1)
    bc0 = wall_control(m, seed=2, amp=1e-2)
    return m, p, u0, bc0


@pytest.mark.slow
def test_adjoint_wall_shear_gradient_64_channel_50_steps():
    """The adjoint workload: 64 x 65 x 64 at Re_tau 180, log-law mean plus a
    k^-5/3 perturbation, wall shear averaged over 50 steps, checkpoints every
    10 steps, a blowing/suction control of the |k| <= 8 modes (amplitude
    0.01 u_tau per mode); 4th-order central differences along 8 seeded
    directions: 4 of the initial field (2 mean-free, 2 with a mean-profile
    part) and 4 of the control (2 with the uniform mode)."""
    m, p, u0, bc0 = _config4()
    rng = np.random.default_rng(5)
    zu, zb = np.zeros_like(u0), np.zeros_like(bc0)
    dirs = []
    for i in range(2):
        du = perturbation(m, p, 80 + i)
        dirs.append(("u", du, zb))
        dirs.append(("u", du + mean_profile(m, rng), zb))
        dc = wall_control(m, seed=90 + i)
        dirs.append(("bc", zu, dc))
        dk = dc.copy()
        dk[m.NZS, :, 0, 1] = rng.standard_normal(2)
        dirs.append(("bc", zu, dk))
    _fd_check(m, p, u0, bc0, nsteps=50, kck=10, directions=dirs, eps_u=1e-2, eps_c=1e-4, tol=1e-6, order=4)


@pytest.mark.slow
def test_adjoint_vjp_64_channel_50_steps():
    """Vector-Jacobian product of the 50-step map at the adjoint workload's sizes."""
    m, p, u0, bc0 = _config4()
    rng = np.random.default_rng(9)
    w = crandom(rng, u0.shape)
    zu, zb = np.zeros_like(u0), np.zeros_like(bc0)
    dirs = [("u", perturbation(m, p, 70), zb), ("u", mean_profile(m, rng), zb),
            ("bc", zu, wall_control(m, seed=71)), ("bc", zu, wall_control(m, seed=72))]
    _fd_check(m, p, u0, bc0, nsteps=50, kck=10, directions=dirs, eps_u=1e-3, eps_c=1e-5, tol=1e-6, weights=w)


def test_adjoint_rejects_unsupported_modes():
    m, p = channel_case(32)
    mesh = cdns.Mesh(m.NX, m.NY, m.NZ, m.NXS, m.NYS, m.NZS, m.NX2, m.NY2, m.NZ2, m.XL, m.ZL)
    params = cdns.Params(Re=p.Re, DT=p.DT, G_pre=p.G_pre, a_pre0=p.a_pre0, b_pre0=p.b_pre0,
                         a_V=p.a_V, b_V=p.b_V, INDEX_GRAD_PRE=p.INDEX_GRAD_PRE, THETA=p.THETA,
                         V_Microblow0=p.V_Microblow0)
    mixed = cdns.Context(mesh, params, precision=cdns.PRECISION_MIXED)
    mixed.set_velocity(np.stack(divergence_free_field(m, p, seed=1, amp=0.1), axis=-1))
    with pytest.raises(cdns.CdnsError, match="FP64"):
        mixed.adjoint_run(2, 1)
    ctx = ctx_for(m, p)
    with pytest.raises(cdns.CdnsError, match="set_velocity"):
        ctx.adjoint_run(2, 1)


def test_autograd_function_matches_finite_differences():
    """torch.autograd through the C-ABI adjoint (tests/adjoint_autograd.py):
    a nonlinear loss of u^4 differentiated by loss.backward() against central
    differences of the same loss along the initial field and the wall data."""
    import torch
    from adjoint_autograd import channel_steps

    m, p = channel_case(32)
    u0n = np.stack(divergence_free_field(m, p, seed=1, amp=0.1, spectrum="k53", mean="loglaw"), axis=-1)
    bc0n = wall_control(m, seed=2, amp=1e-2)
    ctx = ctx_for(m, p)
    rng = np.random.default_rng(11)
    wt = torch.from_numpy(rng.uniform(0.5, 1.5, u0n.shape))

    def loss_of(u0, bc):
        uk = channel_steps(u0, bc, ctx, 4, 2)
        return (wt * uk.abs() ** 2).sum() + uk[m.NZS, :, 0, 0].real.sum()

    u0 = torch.from_numpy(u0n).requires_grad_(True)
    bc = torch.from_numpy(bc0n).requires_grad_(True)
    loss = loss_of(u0, bc)
    loss.backward()
    du = perturbation(m, p, 12)
    dc = wall_control(m, seed=13)
    ad = rdot(u0.grad.numpy(), du) + rdot(bc.grad.numpy(), dc)
    with torch.no_grad():
        h = 1e-4
        f = lambda t: float(loss_of(torch.from_numpy(u0n + t * du), torch.from_numpy(bc0n + t * dc)))
        fd = (f(-2 * h) - 8 * f(-h) + 8 * f(h) - f(2 * h)) / (12 * h)
    assert abs(fd - ad) <= 1e-7 * abs(ad), (fd, ad)
