"""The Re_tau = 180 workload at its stated run lengths against the reference
solver itself: 100 and 1000 FP64 steps of the 128 x 129 x 128 channel
(196 x 193 x 196 product grid, dt = 5e-5, fixed pressure gradient) from the
seeded log-law + k^-5/3 field, on the GPU through the C ABI and in the
reference's own sources (oracle/_ref, Simulation::run,
src/sim/simulation.cpp:173-258) on all host cores.

Checked after the run: the relative L2 difference of every velocity
component (<= 1e-10), the spectral divergence of the GPU velocity
(<= 1e-12 of its largest coefficient), the pressure, and the mean-profile
statistics -- the running means Statistics::accumulate keeps
(src/sim/statistics.cpp:117-139), sampled at every step after Nstat on both
sides (the GPU through cdns_statistics_sample) and read from the reference
at full precision.  Each mean must agree to 1e-10 of its round-off scale
(the largest plane average of the absolute values of its terms), the
tolerance of the velocity itself."""
import os

import numpy as np
import pytest

import ref_io
from oracle_cases import divergence_free_field, orc, retau180_case
from test_gpu_parity import ctx_for

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case():
    if not ref_io.available():
        pytest.fail("oracle/_ref/ref_runner is not built (make -C oracle)")
    m, p = retau180_case()
    u0 = divergence_free_field(m, p, seed=1, amp=0.1, spectrum="k53", mean="loglaw")
    return m, p, u0


def mean_scale(m, u, pres):
    """Per mean slot: the largest plane average of |terms| of its moment."""
    vp, pp = orc.to_physical(m, u, pres)
    a = [np.abs(x) for x in vp]
    ap = np.abs(pp) + (a[0] ** 2 + a[1] ** 2 + a[2] ** 2)
    s = orc.plane_moments(a, ap).max(axis=0) / float(m.NX * m.NZ)
    return s[np.array(orc.STAT_SOURCE)]


def run_both(m, p, u0, nsteps, nstat):
    c = ctx_for(m, p)
    c.set_velocity(np.stack(u0, axis=-1))
    c.statistics_reset()
    for it in range(1, nsteps + 1):
        c.step(it)
        if it > nstat:
            c.statistics_sample()
    c.synchronize()
    v = c.get_velocity()
    pres = c.get_pressure()
    count, dp, means = c.statistics_read()
    dpdx = c.dpdx()
    c.close()
    ru, rp, _, rs = ref_io.run_steps(m, p, u0, nsteps, threads=os.cpu_count() or 1, nstat=nstat)
    return v, pres, (count, dp, means), dpdx, ru, rp, rs


@pytest.mark.parametrize("nsteps,nstat", [(100, 0), pytest.param(1000, 900, marks=pytest.mark.slow)])
def test_retau180_against_reference(case, nsteps, nstat):
    m, p, u0 = case
    v, pres, (count, dp, means), dpdx, ru, rp, rs = run_both(m, p, u0, nsteps, nstat)
    errs = [orc.rel_l2(v[..., k], ru[k]) for k in range(3)]
    print(f"{nsteps} steps: rel L2 per component {errs}, pressure {orc.rel_l2(pres, rp):.3e}")
    assert max(errs) <= 1e-10
    assert orc.rel_l2(pres, rp) <= 1e-9
    cst = orc.make_constants(m, p.Re)
    div = orc.divergence(cst, [v[..., k] for k in range(3)])
    assert np.abs(div).max() <= 1e-12 * np.abs(v).max()
    # statistics of the same run
    assert count == rs["count"] == nsteps - nstat
    assert dp == pytest.approx(rs["dp_means"], abs=1e-14) and dp == pytest.approx(dpdx, abs=1e-14)
    scale = mean_scale(m, [v[..., k] for k in range(3)], pres)
    rel = np.abs(means - rs["means"]) / scale[:, None]
    print(f"statistics: largest difference per mean over its scale {rel.max():.3e}")
    assert np.all(rel <= 1e-10)
