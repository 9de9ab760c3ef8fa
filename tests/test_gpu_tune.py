"""Launch-shape tuning: the choices are valid and cached per mesh, and both
forms of the Chebyshev transforms (FP64 MMA products and the FFT / DCT-I form)
meet the reference's golden vectors, whichever the tuner picks."""
import numpy as np
import pytest

import cdns
from golden_io import load
from oracle_cases import band_spectrum, channel_case, divergence_free_field, orc
from test_gpu_parity import ctx_for

pytestmark = pytest.mark.gpu


def rel_max(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def test_tuning_is_valid_and_cached(tmp_path):
    m, p, _ = load("golden_step.npz")
    a = ctx_for(m, p)
    t = a.tuning()
    assert 8 <= t["z_lines"] <= 17
    assert t["y_synthesis"] in ("fft", "matrix") and t["y_analysis"] in ("fft", "matrix")
    assert t["x_rows"] in (1, 2, 3, 4, 5)
    assert ctx_for(m, p).tuning() == t        # the process cache
    path = tmp_path / "wisdom.json"
    cdns.wisdom_export(str(path))
    assert f"|{m.NX2},{m.NY2},{m.NZ2}|{m.NXS},{m.NYS},{m.NZS}\"" in path.read_text()
    a.tune()                                    # times again; the step still runs
    a.set_velocity(np.zeros((m.nkz, m.ncy, m.nkx, 3), dtype=np.complex128))
    a.run(1, 3)
    a.synchronize()


@pytest.mark.parametrize("form", ["matrix", "fft"])
def test_chebyshev_forms_match_oracle(form, monkeypatch):
    """A 32^3 channel (NY2 = 48 = 6 x 8 has a register split): fine transforms
    and the nonlinear term in either form against the oracle (pinned to the
    reference's own transforms and nonlinear term)."""
    monkeypatch.setenv("CDNS_Y_TRANSFORM", form)
    m, p = channel_case(32)
    c = ctx_for(m, p)
    t = c.tuning()
    assert t["y_synthesis"] == form and t["y_analysis"] == form
    U = band_spectrum(m, 5)
    phys = c.transform_fine("B", U)
    assert rel_max(phys, orc.fine_backward(m, U)) <= 1e-12
    assert rel_max(c.transform_fine("F", phys), orc.fine_forward(m, phys)) <= 1e-12
    u = divergence_free_field(m, p, seed=4, amp=0.1, spectrum="k53", mean="loglaw")
    N, B = c.nonlinear(np.stack(u, axis=-1))
    Nr, _, Br = orc.nonlinear_term(m, orc.make_constants(m, p.Re), u)
    for k in range(3):
        assert rel_max(N[..., k], Nr[k]) <= 1e-12


@pytest.mark.parametrize("n", [32, 64])
def test_fft_form_matches_matrix_form(n, monkeypatch):
    """Sizes with a register split of NY2 (48 = 6 x 8, 96 = 8 x 12): 20 steps of
    the FFT form against the matrix form."""
    m, p = channel_case(n)
    u0 = np.stack(divergence_free_field(m, p, seed=2, amp=0.1, spectrum="k53", mean="loglaw"), axis=-1)
    out = {}
    for form in ("matrix", "fft"):
        monkeypatch.setenv("CDNS_Y_TRANSFORM", form)
        c = ctx_for(m, p)
        assert c.tuning()["y_synthesis"] == form
        c.set_velocity(u0)
        c.run(1, 20)
        c.synchronize()
        out[form] = c.get_velocity()
    assert orc.rel_l2(out["fft"], out["matrix"]) <= 1e-12


@pytest.mark.parametrize("lines", [8, 11, 13, 16])
@pytest.mark.parametrize("ny2", [48, 192])
def test_fft_form_line_widths(lines, ny2, monkeypatch):
    """The DCT-I kernels at every compiled kx-line width (CDNS_YDCT_LINES), with
    NY2 = 48 (6 x 8) and the Re_tau180 y grid NY2 = 192 (12 x 16): fine
    transforms and the nonlinear term against the oracle."""
    monkeypatch.setenv("CDNS_Y_TRANSFORM", "fft")
    monkeypatch.setenv("CDNS_YDCT_LINES", str(lines))
    nys = 30 if ny2 == 48 else 126
    m = orc.Mesh(32, nys + 2, 16, 16, nys, 8, 48, ny2, 24, 4 * np.pi, 2 * np.pi)
    _, p = channel_case(16)
    c = ctx_for(m, p)
    assert c.tuning()["y_synthesis"] == "fft"
    U = band_spectrum(m, 6)
    phys = c.transform_fine("B", U)
    assert rel_max(phys, orc.fine_backward(m, U)) <= 1e-12
    assert rel_max(c.transform_fine("F", phys), orc.fine_forward(m, phys)) <= 1e-12
    u = divergence_free_field(m, p, seed=8, amp=0.1, spectrum="k53", mean="loglaw")
    N, _ = c.nonlinear(np.stack(u, axis=-1))
    Nr, _, _ = orc.nonlinear_term(m, orc.make_constants(m, p.Re), u)
    for k in range(3):
        assert rel_max(N[..., k], Nr[k]) <= 1e-12
