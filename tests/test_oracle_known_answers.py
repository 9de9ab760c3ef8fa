"""Pin the numpy oracle against the reference's own known-answer tests.

Each test restates, by value, a check the reference makes in its GoogleTest
suite (file:line cited) and applies it to the oracle.  These run on CPU only.
"""
import math

import numpy as np
import pytest

from oracle_cases import PI, band_spectrum, example_case, orc


def dct1_definition(x):
    """REDFT00 definition as written in tests/test_xyzfft.cpp:79-91."""
    n = len(x)
    ny = n - 1
    y = np.zeros(n)
    for k in range(n):
        s = x[0] + (x[ny] if k % 2 == 0 else -x[ny])
        for j in range(1, ny):
            s += 2.0 * x[j] * math.cos(PI * j * k / ny)
        y[k] = s
    return y


def y_spectrum_expected(my, NY, NYS):
    """tests/test_xyzfft.cpp:93-100."""
    f = np.array([math.cos(my * PI * j / NY) for j in range(NY + 1)])
    Y = dct1_definition(f)
    return np.array([Y[k] / (2.0 * NY) if k == 0 else Y[k] / NY for k in range(NYS + 1)])


def x2_peak(kxx, kx, NXH, NXS):
    """tests/test_xyzfft.cpp:114-119 (fine grid: no Nyquist halving)."""
    if kx == 0:
        return 1.0 if kxx == 0 else 0.0
    if kx > NXS:
        return 0.0
    return (1.0 if kx == NXH else 0.5) if kxx == kx else 0.0


def z2_peak(izz, kz, NZH, NZS):
    """tests/test_xyzfft.cpp:120-125."""
    if kz == 0:
        return 1.0 if izz == 0 else 0.0
    if abs(kz) > NZS:
        return 0.0
    if izz != kz and izz != -kz:
        return 0.0
    return 1.0 if abs(kz) == NZH else 0.5


def _full_mesh():
    # 32^3 coarse = fine, NXS=NZS=16 (full spectrum, Nyquist branch), NYS=30
    return orc.Mesh(32, 32, 32, 16, 30, 16, 32, 32, 32, 2 * PI, 2 * PI)


@pytest.mark.parametrize("kx,kz", [(5, 3), (5, -9), (5, 16), (16, 3), (16, -9), (16, 16)])
def test_fine_forward_analytic(kx, kz):
    """tests/test_xyzfft.cpp:323-353 (F5a): cos x T_3 x cos modes to 1e-12,
    including the fine-grid Nyquist peak of 1.0."""
    m = _full_mesh()
    my = 3
    Uy = y_spectrum_expected(my, m.NY2, m.NYS)
    iz = np.arange(m.NZ2)[:, None, None]
    iy = np.arange(m.NY2 + 1)[None, :, None]
    ix = np.arange(m.NX2)[None, None, :]
    P = np.cos(2 * PI * kx * ix / m.NX2) * np.cos(my * PI * iy / m.NY2) * np.cos(2 * PI * kz * iz / m.NZ2)
    U = orc.fine_forward(m, P)
    exp = np.zeros_like(U)
    for izz in range(-m.NZS, m.NZS + 1):
        for kxx in range(m.NXS + 1):
            exp[izz + m.NZS, :, kxx] = x2_peak(kxx, kx, m.NX2 // 2, m.NXS) * Uy * \
                z2_peak(izz, kz, m.NZ2 // 2, m.NZS)
    assert np.abs(U - exp).max() < 1e-12


@pytest.mark.parametrize("cfg", [(16, 30, 16), (10, 20, 10)])
def test_fine_round_trips(cfg):
    """tests/test_xyzfft.cpp:355-372 (F5b/F5c): band spectrum -> B -> F and
    physical -> F -> B round trips to 1e-12."""
    NXS, NYS, NZS = cfg
    m = orc.Mesh(32, 32, 32, NXS, NYS, NZS, 32, 32, 32, 2 * PI, 2 * PI)
    U0 = band_spectrum(m, 0xF5)
    P = orc.fine_backward(m, U0)
    U1 = orc.fine_forward(m, P)
    assert np.abs(U1 - U0).max() < 1e-12
    U2 = orc.fine_forward(m, P)
    P2 = orc.fine_backward(m, U2)
    assert np.abs(P2 - P).max() < 1e-12


def test_dealiased_round_trip():
    """3/2 product grid (18x13x18 fine on 12x9x12 coarse shapes, as the MPI
    transform tests use): spectral -> physical -> spectral is the identity."""
    m = orc.Mesh(12, 8, 12, 6, 7, 6, 18, 12, 18, 2 * PI, 2 * PI)
    U0 = band_spectrum(m, 7)
    # a proper 3/2 grid has no Nyquist coupling: every slot is independent
    assert np.abs(orc.fine_forward(m, orc.fine_backward(m, U0)) - U0).max() < 1e-12


def test_chebyshev_derivative_and_flow_rate():
    """tests/test_vector_ops.cpp:34-47: d/dy T_4 -> 8 T_3 + 8 T_1; Q(2 T_0 + 3 T_2) = 1."""
    m, p = example_case()
    f = np.zeros(m.spectral_shape(), dtype=np.complex128)
    f[m.NZS, 4, 0] = 1.0
    d = orc.derivative_y(f)
    assert d[m.NZS, 3, 0].real == 8.0
    assert d[m.NZS, 1, 0].real == 8.0
    g = np.zeros(m.ncy, dtype=np.complex128)
    g[0] = 2.0
    g[2] = 3.0
    assert orc.flow_rate(g) == 1.0


def test_fourier_derivative_matches_complex_multiplication():
    """tests/test_vector_ops.cpp:12-17."""
    for k in (-3.0, -0.1, 0.0, 0.1, 3.0):
        for i in range(31):
            v = complex(math.sin(i * 0.3), math.cos(i * 0.7))
            assert orc.fourier_derivative(k, np.array(v)) == complex(0.0, k) * v


def test_div_curl_vanishes():
    """tests/test_vector_ops.cpp:49-64."""
    m, p = example_case()
    c = orc.make_constants(m, p.Re)
    v = [np.zeros(m.spectral_shape(), dtype=np.complex128) for _ in range(3)]
    for iz in range(-2, 3):
        for iy in range(5):
            for ix in range(m.nkx):
                for k in range(3):
                    v[k][iz + m.NZS, iy, ix] = complex(0.01 * (1 + ix + iy + k), 0.02 * iz)
    div = orc.divergence(c, orc.curl(c, v))
    assert np.abs(div).max() < 1e-12


@pytest.mark.parametrize("nys", [4, 7, 30])
@pytest.mark.parametrize("nxs", [7, 8, 16])
def test_curl_matches_independent_derivatives(nys, nxs):
    """tests/test_vector_ops.cpp:66-103."""
    m, p = example_case(NXS=nxs, NYS=nys)
    c = orc.make_constants(m, p.Re)
    zz, yy, xx = np.meshgrid(np.arange(-m.NZS, m.NZS + 1), np.arange(m.ncy), np.arange(m.nkx),
                             indexing="ij")
    comps = [np.sin(0.3 * xx + 0.7 * yy + k) + 1j * np.cos(0.2 * zz + 0.9 * yy + k) for k in range(3)]

    def deriv(axis, f):
        if axis == 0:
            return orc.fourier_derivative(c.WAVX[None, None, :], f)
        if axis == 2:
            return orc.fourier_derivative(c.WAVZ[:, None, None], f)
        return orc.derivative_y(f)

    res = orc.curl(c, comps)
    for k in range(3):
        j, l = (k + 1) % 3, (k + 2) % 3
        exp = deriv(j, comps[l]) - deriv(l, comps[j])
        assert np.abs(res[k] - exp).max() < 1e-12


def test_cross_product_constant_vectors():
    """tests/test_nonlinear_ops.cpp:9-33: (1,2,3) x (4,3,2) = (-5,10,-5),
    a x a = 0 and antisymmetry, through the fine transforms."""
    m, p = example_case()

    def const_field(vals):
        out = []
        for k in range(3):
            f = np.zeros(m.spectral_shape(), dtype=np.complex128)
            f[m.NZS, 0, 0] = vals[k]
            out.append(f)
        return out

    a = const_field([1.0, 2.0, 3.0])
    b = const_field([4.0, 3.0, 2.0])

    def cross(x, y):
        xp = [orc.fine_backward(m, f) for f in x]
        yp = [orc.fine_backward(m, f) for f in y]
        return [orc.fine_forward(m, f) for f in orc.cross_product_physical(xp, yp)]

    ab, ba, aa = cross(a, b), cross(b, a), cross(a, a)
    for k, e in enumerate([-5.0, 10.0, -5.0]):
        assert abs(ab[k][m.NZS, 0, 0] - e) < 1e-12
    assert max(np.abs(f).max() for f in aa) < 1e-13
    assert max(np.abs(ab[k] + ba[k]).max() for k in range(3)) < 1e-13


def _setup(m, p, g=150.0):
    c = orc.make_constants(m, p.Re)
    s = orc.Solver(m, p, c)
    with np.errstate(all="ignore"):
        s.setup(g)
    return c, s


def test_setup_finite_and_wn():
    """tests/test_eqsolve.cpp:57-75."""
    m, p = example_case()
    c, s = _setup(m, p)
    exp = -((c.WAVX[None, :] ** 2 + c.WAVZ[:, None] ** 2) + 150.0)
    assert np.array_equal(s.state.wn_v, exp)
    assert np.all(np.isfinite(s.state.ad_v[:, 2:]))
    assert math.isfinite(s.state.qx_unit) and s.state.qx_unit != 0.0
    assert math.isfinite(s.state.qz_unit) and s.state.qz_unit != 0.0


def test_zero_input_has_zero_wall_divergence():
    """tests/test_eqsolve.cpp:77-94."""
    m, p = example_case()
    c, s = _setup(m, p)
    z = np.zeros(m.spectral_shape(), dtype=np.complex128)
    zb = np.zeros((m.nkz, m.nkx), dtype=np.complex128)
    pres, vel = s.solve_modes(z, (zb, zb), [z, z, z], [(zb, zb)] * 3, correct_sigma=False)
    assert np.all(np.isfinite(pres))
    lo, up = orc.divergence_boundary(c, vel)
    assert np.abs(lo).max() < 1e-10 and np.abs(up).max() < 1e-10


def test_unit_responses_satisfy_no_slip_and_setup_reuse():
    """tests/test_eqsolve.cpp:112-136."""
    m, p = example_case()
    c, s = _setup(m, p, 150.0)
    first = s.state.u_unit.copy()
    with np.errstate(all="ignore"):
        s.setup(300.0)
    assert s.state.g_v == 300.0
    assert not np.array_equal(s.state.u_unit, first)
    for resp in (s.state.u_unit, s.state.w_unit):
        upper = float(np.sum(resp))
        lower = float(np.sum(resp * (-1.0) ** np.arange(m.ncy)))
        assert abs(upper) < 1e-12 and abs(lower) < 1e-12
    with np.errstate(all="ignore"):
        s.setup(150.0)
    assert np.abs(s.state.u_unit - first).max() <= 1e-15


def _staged(m, c, s, rhs_p, bc_p, rhs_v, bc_v, correct):
    """Staged solver of tests/test_eqsolve.cpp:17-47: coupled base solve,
    explicit influence correction, then EqSolvePV::apply_sigma_correction
    (src/solver/eqsolve_pv.cpp:511-533)."""
    pres, vel = s.solve_coupled_base(rhs_p, bc_p, rhs_v, bc_v)
    lo, up = orc.divergence_boundary(c, vel)
    ID0, ID1 = s.state.inf_div
    c0 = (up * ID1[0] - lo * ID1[1])[:, None, :]
    c1 = (lo * ID0[1] - up * ID0[0])[:, None, :]
    pres = pres + (c0 * s.state.p_inf[0] + c1 * s.state.p_inf[1])
    vel = [vel[k] + (c0 * s.state.v_inf[0][k] + c1 * s.state.v_inf[1][k]) for k in range(3)]
    if correct:
        st = s.state
        ny = m.NYS
        w = st.wn_v
        sig0 = ((-w) * vel[1][:, ny] - s.p.Re * rhs_v[1][:, ny]) / st.sigma0[0]
        sig1 = ((-w) * vel[1][:, ny - 1] + s.p.Re * (2.0 * ny * pres[:, ny] - rhs_v[1][:, ny - 1])) \
            / st.sigma0[1]
        sig = [sig0, sig1]
        pres = pres.copy()
        vel = [v.copy() for v in vel]
        for iy in range(ny + 1):
            q = (iy + 1) % 2
            pres[:, iy] += sig[q] * st.p_b[:, iy]
            vel[0][:, iy] += sig[q] * st.v_b[0][:, iy]
            vel[1][:, iy] += sig[1 - q] * st.v_b[1][:, iy]
            vel[2][:, iy] += sig[q] * st.v_b[2][:, iy]
    return pres, vel


@pytest.mark.parametrize("nxs", [7, 8, 10, 16])
@pytest.mark.parametrize("neumann", [False, True])
def test_fused_solver_matches_staged(nxs, neumann):
    """tests/test_eqsolve.cpp:138-185: fused solve_modes vs staged solver to
    1e-10 max(1,|x|), Dirichlet and Neumann v, sigma on/off, fused RHS on/off."""
    m, p = example_case(NXS=nxs, a_v1=0.0 if neumann else 1.0, b_v1=1.0 if neumann else 0.0)
    c, s = _setup(m, p)
    sh = m.spectral_shape()
    n = int(np.prod(sh))
    i = np.arange(n).reshape(sh)
    rhs_p = np.sin(i * 0.13) * 0.001 + 1j * np.cos(i * 0.19) * 0.002
    iv = np.arange(3 * n).reshape(sh + (3,))
    rv = np.sin(iv * 0.17) * 0.001 + 1j * np.cos(iv * 0.23) * 0.002
    rhs_v = [np.ascontiguousarray(rv[..., k]) for k in range(3)]
    ib = np.arange(m.nkz * 2 * m.nkx).reshape(m.nkz, 2, m.nkx)
    bp = np.sin(ib * 0.11) * 0.001 + 1j * np.cos(ib * 0.29) * 0.002
    bc_p = (bp[:, 0], bp[:, 1])
    ibv = np.arange(m.nkz * 2 * m.nkx * 3).reshape(m.nkz, 2, m.nkx, 3)
    bv = np.sin(ibv * 0.31) * 0.001 + 1j * np.cos(ibv * 0.37) * 0.002
    bc_v = [(bv[:, 0, :, k], bv[:, 1, :, k]) for k in range(3)]
    for correct in (False, True):
        for fuse in (False, True):
            ref_rhs = orc.divergence(c, rhs_v) if fuse else rhs_p
            ep, ev = _staged(m, c, s, ref_rhs, bc_p, rhs_v, bc_v, correct)
            ap, av = s.solve_modes(None if fuse else rhs_p, bc_p, rhs_v, bc_v, correct)
            assert np.all(np.abs(ap - ep) <= 1e-10 * np.maximum(1.0, np.abs(ep)))
            for k in range(3):
                assert np.all(np.abs(av[k] - ev[k]) <= 1e-10 * np.maximum(1.0, np.abs(ev[k])))


def test_step_coefficients():
    """tests/test_simulation.cpp:5-21 and :29-34."""
    assert orc.step_coefficients(1, 0.25, 10.0) == (4.0, 0.0, 1.0, 0.0, 40.0)
    a0, a1, b0, b1, g = orc.step_coefficients(2, 0.25, 10.0)
    assert (a0, a1, b0, b1) == (8.0, -2.0, 2.0, -1.0)
    assert orc.step_coefficients(3, 0.25, 10.0) == orc.step_coefficients(2, 0.25, 10.0)
    for bad in ((0, 0.1), (-1, 0.1), (1, 0.0), (1, -0.1)):
        with pytest.raises(ValueError):
            orc.step_coefficients(bad[0], bad[1], 10.0)


def test_uniform_velocity_has_zero_nonlinear_term():
    """tests/test_timestepper.cpp:7-19 and :57-74."""
    m, p = example_case()
    c = orc.make_constants(m, p.Re)
    u = [np.zeros(m.spectral_shape(), dtype=np.complex128) for _ in range(3)]
    N, _, B = orc.nonlinear_term(m, c, u)
    assert all(np.all(f == 0) for f in N) and np.all(B[0] == 0) and np.all(B[1] == 0)
    for k in range(3):
        u[k][m.NZS, 0, 0] = k + 1.0
    N, _, B = orc.nonlinear_term(m, c, u)
    assert max(np.abs(f).max() for f in N) < 1e-12
    assert np.abs(B[0]).max() < 1e-12 and np.abs(B[1]).max() < 1e-12


def test_zero_mode_projection():
    """tests/test_timestepper.cpp:36-55: v(0,0,:) = (1e-3, 0, ...)."""
    m, p = example_case()
    c, s = _setup(m, p)
    z = np.zeros(m.spectral_shape(), dtype=np.complex128)
    zb = np.zeros((m.nkz, m.nkx), dtype=np.complex128)
    bc_v = orc.velocity_boundary(m, p)
    pres, vel = s.solve_modes(None, (zb, zb), [z, z, z], bc_v, correct_sigma=True)
    vel[1][m.NZS, 0, 0] = 0.5 * (bc_v[1][0][m.NZS, 0] + bc_v[1][1][m.NZS, 0])
    vel[1][m.NZS, 1:, 0] = 0.0
    assert vel[1][m.NZS, 0, 0] == complex(1e-3, 0.0)
    assert np.all(np.isfinite(pres))
