"""Every form of the register-form x stage (k_x_cross_r with 4 or 2 rows per
block, with 4 or 2 rows and the forward phases split over lane pairs, k_x_cross_h
with a half-warp per row pair) against the oracle's
nonlinear term (src/solver/vector_ops.cpp:250-272 with the fine transforms
of src/fft/transforms.cpp:641-741), on every x length split the register
forms cover and at a full x spectrum (Nyquist branches); the FP32 stages of
the mixed form against the FP64 path.  The form is fixed with CDNS_X_STAGE,
read when a context is created.  Tolerances as in test_gpu_parity.py."""
import numpy as np
import pytest

import cdns
from oracle_cases import channel_case, divergence_free_field, example_case, orc
from test_gpu_parity import ctx_for, rel_max

pytestmark = pytest.mark.gpu

FORMS = ["rows4", "rows2", "halfwarp", "split", "split2"]


def mesh_x(nxs, nx2, nzs=8, nz2=32, nys=14, ny2=24):
    m = orc.Mesh(2 * nxs, nys + 2, 2 * nzs, nxs, nys, nzs, nx2, ny2, nz2, 4 * np.pi, 2 * np.pi)
    _, p = channel_case(16)
    return m, p


CASES = {
    "x32_full": lambda: example_case(),        # NX2 = 2 NXS = 32 (4 x 8): Nyquist branches
    "x48": lambda: channel_case(32),           # 6 x 8
    "x72": lambda: mesh_x(24, 72),             # 8 x 9
    "x192": lambda: mesh_x(64, 192),           # 12 x 16
    "x196": lambda: mesh_x(64, 196),           # 14 x 14 (the Re_tau180 product grid)
}


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("case", sorted(CASES))
def test_x_stage_forms_nonlinear_term(monkeypatch, form, case):
    monkeypatch.setenv("CDNS_X_STAGE", form)
    m, p = CASES[case]()
    u = divergence_free_field(m, p, seed=17, amp=0.1, spectrum="k53", mean="loglaw")
    cst = orc.make_constants(m, p.Re)
    N_ref, _, B_ref = orc.nonlinear_term(m, cst, u)
    c = ctx_for(m, p)
    # (72 = 8 x 9 has an odd factor: "split" runs the 4-rows form there)
    assert c.tuning()["x_rows"] == {"rows4": 4, "rows2": 2, "halfwarp": 1, "split": 3, "split2": 5}[form]
    N, B = c.nonlinear(np.stack(u, axis=-1))
    for k in range(3):
        assert rel_max(N[..., k], N_ref[k]) <= 1e-12
    scale = max(np.abs(B_ref[0]).max(), np.abs(N_ref[1]).max() * (m.NYS + 1))
    assert np.abs(B[:, 0] - B_ref[0]).max() <= 1e-12 * scale


@pytest.mark.parametrize("form", ["halfwarp", "split", "split2"])
@pytest.mark.parametrize("case", ["x48", "x196"])
def test_x_stage_halfwarp_mixed(monkeypatch, case, form):
    """FP32 stages (mean profiles kept in FP64) through the half-warp and the
    split forms against the FP64 nonlinear term: the bound of test_gpu_mixed.py."""
    m, p = CASES[case]()
    u = np.stack(divergence_free_field(m, p, seed=19, amp=0.05, kmax=4), axis=-1)
    N64, _ = ctx_for(m, p).nonlinear(u)
    monkeypatch.setenv("CDNS_X_STAGE", form)
    mesh = cdns.Mesh(m.NX, m.NY, m.NZ, m.NXS, m.NYS, m.NZS, m.NX2, m.NY2, m.NZ2, m.XL, m.ZL)
    cm = cdns.Context(mesh, cdns.Params(Re=p.Re, DT=p.DT), precision=cdns.PRECISION_MIXED)
    assert cm.tuning()["x_rows"] == {"halfwarp": 1, "split": 3, "split2": 5}[form]
    N32, _ = cm.nonlinear(u)
    for k in range(3):
        assert orc.rel_l2(N32[..., k], N64[..., k]) <= 1e-5
