"""Pin the oracle's coarse-grid transform and output reduction against the
reference's own known-answer tests (tests/test_xyzfft.cpp,
tests/test_diagnostics.cpp, tests/test_statistics.cpp), restated by value.
CPU only."""
import math

import numpy as np
import pytest

from oracle_cases import PI, band_spectrum, example_case, orc
from test_oracle_known_answers import y_spectrum_expected


def x_peak(kxx, kx, NXS):
    """tests/test_xyzfft.cpp:101-105: DC 1, interior and Nyquist 0.5 (the
    coarse transform halves the full-spectrum Nyquist bin), 0 past NXS."""
    if kx == 0:
        return 1.0 if kxx == 0 else 0.0
    if kx > NXS:
        return 0.0
    return 0.5 if kxx == kx else 0.0


def z_peak(izz, kz, NZS):
    """tests/test_xyzfft.cpp:107-111: 0.5 at +-kz, the Nyquist slots included
    (halved and mirrored)."""
    if kz == 0:
        return 1.0 if izz == 0 else 0.0
    if abs(kz) > NZS:
        return 0.0
    return 0.5 if izz in (kz, -kz) else 0.0


def _mesh(NXS, NYS, NZS):
    # tests/test_xyzfft.cpp:20-30: 32^3 coarse = fine grid, 2 pi x 2 pi
    return orc.Mesh(32, 32, 32, NXS, NYS, NZS, 32, 32, 32, 2 * PI, 2 * PI)


FULL_MODES = [(16, 3, 16), (0, 0, 0), (5, 7, -9), (16, 30, 16)]
TRUNC_MODES = [(3, 3, -4), (10, 20, 10), (0, 2, 0)]


@pytest.mark.parametrize("cfg,mode", [((16, 30, 16), md) for md in FULL_MODES] +
                         [((10, 20, 10), md) for md in TRUNC_MODES])
def test_coarse_forward_analytic(cfg, mode):
    """tests/test_xyzfft.cpp:201-246 (F1): cos(kx x) T_my(y) cos(kz z) through
    the coarse forward transform equals x_peak * y spectrum * z_peak to 1e-12,
    at a full spectrum (Nyquist branches) and a truncated one."""
    m = _mesh(*cfg)
    kx, my, kz = mode
    iz = np.arange(m.NZ)[:, None, None]
    iy = np.arange(m.NY + 1)[None, :, None]
    ix = np.arange(m.NX)[None, None, :]
    P = np.cos(2 * PI * kx * ix / m.NX) * np.cos(my * PI * iy / m.NY) * np.cos(2 * PI * kz * iz / m.NZ)
    U = orc.coarse_forward(m, P)
    Uy = y_spectrum_expected(my, m.NY, m.NYS)
    exp = np.zeros_like(U)
    for izz in range(-m.NZS, m.NZS + 1):
        for kxx in range(m.NXS + 1):
            exp[izz + m.NZS, :, kxx] = x_peak(kxx, kx, m.NXS) * Uy * z_peak(izz, kz, m.NZS)
    assert np.abs(U - exp).max() < 1e-12


@pytest.mark.parametrize("cfg", [(16, 30, 16), (10, 20, 10)])
def test_coarse_round_trips(cfg):
    """tests/test_xyzfft.cpp:251-276 (F3, F2): realisable band spectrum -> B ->
    F is the identity, and the band-limited physical field -> F -> B too."""
    m = _mesh(*cfg)
    U0 = band_spectrum(m, 0xC0DE + (0 if cfg[0] == 16 else 1))
    P = orc.coarse_backward(m, U0)
    assert np.abs(orc.coarse_forward(m, P) - U0).max() < 1e-12
    P2 = orc.coarse_backward(m, orc.coarse_forward(m, P))
    assert np.abs(P2 - P).max() < 1e-12


def _xz_plane(m, UP):
    """The coarse forward transform of a y-independent field, read at the
    Chebyshev mode 0 (where a constant line maps to 1): the 2-D x-z transform
    Transforms::xzfft makes of one plane (src/fft/transforms.cpp:407-450)."""
    P = np.broadcast_to(UP[:, None, :], (m.NZ, m.NY + 1, m.NX)).copy()
    return orc.coarse_forward(m, P)[:, 0, :]


@pytest.mark.parametrize("kz", [3, -5, 0, 16])
@pytest.mark.parametrize("kx", [5, 0, 16])
def test_xz_plane_analytic(kx, kz):
    """tests/test_xyzfft.cpp:279-303 (F4, analytic part)."""
    m = _mesh(16, 30, 16)
    iz = np.arange(m.NZ)[:, None]
    ix = np.arange(m.NX)[None, :]
    UP = np.cos(2 * PI * kx * ix / m.NX) * np.cos(2 * PI * kz * iz / m.NZ)
    U = _xz_plane(m, UP)
    exp = np.zeros_like(U)
    for izz in range(-m.NZS, m.NZS + 1):
        for kxx in range(m.NXS + 1):
            exp[izz + m.NZS, kxx] = x_peak(kxx, kx, m.NXS) * z_peak(izz, kz, m.NZS)
    assert np.abs(U - exp).max() < 1e-12


def test_xz_plane_naive_dft():
    """tests/test_xyzfft.cpp:165-195, 305-316 (F4, naive part): a random
    plane against the direct 2-D DFT with the coarse conventions -- 1/(NX NZ),
    x0.5 on a full-spectrum Nyquist in x and in z, U(-NZ/2) = U(+NZ/2)."""
    m = _mesh(16, 30, 16)
    rng = np.random.default_rng(0xDA7A)
    UP = rng.uniform(-1.0, 1.0, (m.NZ, m.NX))
    NXH, NZH = m.NX // 2, m.NZ // 2
    ref = np.zeros((2 * m.NZS + 1, m.NXS + 1), dtype=np.complex128)
    ix = np.arange(m.NX)[None, :]
    iz = np.arange(m.NZ)[:, None]
    for kxx in range(m.NXS + 1):
        for kzz in range(-m.NZS, m.NZS + 1):
            if kzz == -NZH:
                continue
            ph = -2.0 * PI * (kxx * ix / m.NX + kzz * iz / m.NZ)
            s = np.sum(UP * (np.cos(ph) + 1j * np.sin(ph)))
            norm = 1.0 / (m.NX * m.NZ)
            if kxx == NXH:
                norm *= 0.5
            if kzz == NZH:
                norm *= 0.5
            ref[kzz + m.NZS, kxx] = s * norm
        ref[-NZH + m.NZS, kxx] = ref[NZH + m.NZS, kxx]
    assert np.abs(_xz_plane(m, UP) - ref).max() < 1e-12


def _coordinates(m):
    """src/core/mesh.cpp:94-116: XC = (i+1) XL/NX, ZC = (k+1) ZL/NZ, YC the
    Gauss-Lobatto points cos(pi j/NY) filled antisymmetrically, 0 mid-channel."""
    xc = (np.arange(m.NX) + 1.0) * (m.XL / m.NX)
    zc = (np.arange(m.NZ) + 1.0) * (m.ZL / m.NZ)
    yc = np.empty(m.NY + 1)
    for j in range(m.NY + 1):
        yc[j] = math.cos(PI * j / m.NY)
        yc[m.NY - j] = -yc[j]
    yc[m.NY // 2] = 0.0
    return xc, yc, zc


def diagnostics_fields(m):
    """The fields of tests/test_diagnostics.cpp:20-32 on the coarse grid --
    u = y cos(kx x), v = sin(kx x), w = 2 cos(kz z), raw pressure
    5 + |v|^2/2 -- and the values Diagnostics::evaluate gives for them:
    EKT = NX NZ (NY+1) / 2, TKE = 4/3, divergence L2 = sqrt(kx^2/6 + 2 kz^2),
    corrected-pressure plane mean 5 (:45-50)."""
    xc, yc, zc = _coordinates(m)
    kx, kz = 2 * PI / m.XL, 2 * PI / m.ZL
    X, Y, Z = xc[None, None, :], yc[None, :, None], zc[:, None, None]
    shape = (m.NZ, m.NY + 1, m.NX)
    u = np.broadcast_to(Y * np.cos(kx * X), shape).copy()
    v = np.broadcast_to(np.sin(kx * X), shape).copy()
    w = np.broadcast_to(2 * np.cos(kz * Z), shape).copy()
    pr = 5 + 0.5 * (u * u + v * v + w * w)
    want = {"ekt": 0.5 * m.NX * m.NZ * (m.NY + 1), "tke": 4.0 / 3.0,
            "divergence_l2": math.sqrt(kx * kx / 6 + 2 * kz * kz), "pressure": 5.0}
    return (u, v, w), pr, want


def test_diagnostics_analytic_fields():
    """tests/test_diagnostics.cpp:11-55 on the example mesh: u = y cos(kx x),
    v = sin(kx x), w = 2 cos(kz z), p = 5 + |v|^2/2.  EKT = NX NZ (NY+1) / 2,
    TKE = 4/3, divergence L2 = sqrt(kx^2/6 + 2 kz^2), and the corrected
    pressure has plane mean 5."""
    m, p = example_case()
    c = orc.make_constants(m, p.Re)
    (u, v, w), pr, want = diagnostics_fields(m)
    spectral = [orc.coarse_forward(m, f) for f in (u, v, w)]
    planes = orc.plane_moments([u, v, w], pr, True)
    ekt, tke, div = orc.diagnostics(m, c, planes, spectral)
    assert abs(ekt - want["ekt"]) <= 1e-8 * want["ekt"]
    assert abs(tke - want["tke"]) <= 1e-12
    assert abs(div - want["divergence_l2"]) <= 1e-11
    assert np.all(np.abs(planes[:, 3] / (m.NX * m.NZ) - want["pressure"]) <= 1e-13)


def uniform_sample(m, sample):
    """tests/test_statistics.cpp:69-75: v = (1, 2, 3) + 2 sample and raw
    pressure 4 + 2 sample + |v|^2/2, so the corrected pressure is 4 + 2 sample."""
    shape = (m.NZ, m.NY + 1, m.NX)
    vel = [np.full(shape, 1.0 + comp + 2 * sample) for comp in range(3)]
    kinetic = 0.5 * sum(x[0, 0, 0] ** 2 for x in vel)
    return vel, np.full(shape, 4.0 + 2 * sample + kinetic)


# The 20 means after the two samples (tests/test_statistics.cpp:77-78), in
# Statistics::write's order: mean u v w p; uu vv ww uv vw wu pp pu pv pw;
# uuu vvv www; uuuu vvvv wwww.
UNIFORM_MEANS = [2, 3, 4, 5, 5, 10, 17, 7, 13, 9, 26, 11, 16, 21, 14, 36, 76, 41, 136, 353]


def test_statistics_analytic_means_and_cross_moments():
    """tests/test_statistics.cpp:62-111: two uniform samples give the exact
    means, cross moments and corrected-pressure moments, and the dp/dx, dp/dz
    means 0 and 3."""
    m, _ = example_case()
    st = orc.Statistics(m)
    for sample in range(2):
        vel, pr = uniform_sample(m, sample)
        st.sample(vel, pr, -1 + 2 * sample, 2 + 2 * sample)
    assert st.count == 2
    assert st.dp[0] == 0.0 and st.dp[1] == 3.0
    for slot, want in enumerate(UNIFORM_MEANS):
        assert np.all(st.means[slot] == want), slot


def test_statistics_update_rule_and_pressure_untouched():
    """tests/test_statistics.cpp:10-26: dp/dx samples -1, 3 and dp/dz 2, 4
    average to 1 and 3; the pressure field is not modified."""
    m, _ = example_case()
    st = orc.Statistics(m)
    shape = (m.NZ, m.NY + 1, m.NX)
    vel = [np.full(shape, 1.0), np.full(shape, 2.0), np.full(shape, 3.0)]
    pr = np.full(shape, 10.0)
    orig = pr.copy()
    st.sample(vel, pr, -1.0, 2.0)
    st.sample(vel, pr, 3.0, 4.0)
    assert st.count == 2 and st.dp[0] == 1.0 and st.dp[1] == 3.0
    assert np.array_equal(pr, orig)


def test_statistics_rejects_wrong_sizes_without_changes():
    """tests/test_statistics.cpp:42-60: a short component or pressure raises
    and leaves the count and the means as they were."""
    m, _ = example_case()
    st = orc.Statistics(m)
    shape = (m.NZ, m.NY + 1, m.NX)
    vel = [np.full(shape, 1.0) for _ in range(3)]
    pr = np.full(shape, 2.0)
    st.sample(vel, pr, 3.0, 4.0)
    before = st.means.copy()
    for comp in range(4):
        bad_v = [x.copy() for x in vel]
        bad_p = pr.copy()
        if comp == 3:
            bad_p = bad_p[:, :, :-1]
        else:
            bad_v[comp] = bad_v[comp][:, :, :-1]
        with pytest.raises(ValueError):
            st.sample(bad_v, bad_p, 99.0, 99.0)
        assert st.count == 1 and st.dp[0] == 3.0 and st.dp[1] == 4.0
        assert np.array_equal(st.means, before)
