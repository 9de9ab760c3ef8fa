"""Coarse-grid transform and the device-side output reduction (cdns_transform_coarse,
cdns_output_reduce) against the reference's own channel_xyzfft, to_physical,
Statistics::reduce and Diagnostics::evaluate (golden fixtures made by
tests/golden/make_golden.py from the reference sources), and against the
oracle at the Re_tau180 size."""
import os

import numpy as np
import pytest

import cdns
from golden_io import GOLDEN, load
from oracle_cases import channel_case, divergence_free_field, example_case, orc, retau180_case
from test_gpu_parity import ctx_for
from test_oracle_output_known_answers import UNIFORM_MEANS, diagnostics_fields, uniform_sample

pytestmark = pytest.mark.gpu


def rel_max(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def plane_scale(vp, pp):
    """Per moment, the largest plane sum of |term|: the round-off scale of
    plane sums that cancel (mean-free components) or that sample the
    round-off of the no-slip walls (high powers of values ~1e-14)."""
    a = [np.abs(x) for x in vp]
    s = orc.plane_moments(a, np.abs(pp) + (a[0] ** 2 + a[1] ** 2 + a[2] ** 2))
    return s.max(axis=0)[None, :]


@pytest.mark.parametrize("tag", ["full", "ragged"])
@pytest.mark.parametrize("kind", ["real", "arb"])
def test_coarse_transform_matches_reference(tag, kind):
    """Full spectrum (Nyquist halve/mirror branches) and ragged (NXS < NX/2),
    realisable and arbitrary spectra."""
    d = dict(np.load(os.path.join(GOLDEN, "golden_coarse.npz")))
    mm = [int(v) for v in d[f"{tag}_mesh"]]
    m = orc.Mesh(*mm, float(d[f"{tag}_dom"][0]), float(d[f"{tag}_dom"][1]))
    _, p = channel_case(16)
    c = ctx_for(m, p)
    U, phys, back = d[f"{tag}_{kind}_U"], d[f"{tag}_{kind}_phys"], d[f"{tag}_{kind}_back"]
    assert rel_max(c.transform_coarse("B", U), phys) <= 1e-13
    assert rel_max(c.transform_coarse("F", phys), back) <= 1e-13


@pytest.mark.parametrize("n", [32, 48])
def test_coarse_transform_matches_oracle(n):
    """Register-form sizes (NX = NZ = 32 = 4 x 8; 48 = 6 x 8)."""
    m, p = channel_case(n)
    rng = np.random.default_rng(n)
    U = orc.coarse_forward(m, rng.standard_normal((m.NZ, m.NY + 1, m.NX)))
    c = ctx_for(m, p)
    P = c.transform_coarse("B", U)
    assert rel_max(P, orc.coarse_backward(m, U)) <= 1e-13
    assert rel_max(c.transform_coarse("F", P), orc.coarse_forward(m, P)) <= 1e-13


def test_output_reduction_matches_reference():
    m, p, d = load("golden_reduce.npz")
    c = ctx_for(m, p)
    c.set_velocity(np.stack(list(d["u"]), axis=-1))
    c.set_pressure(d["p"])
    planes, values, phys = c.output_reduce(higher_moments=True, snapshot=True)
    for k in range(4):
        assert rel_max(phys[k], d["phys"][k]) <= 1e-13
    vp = [phys[0], phys[1], phys[2]]
    assert np.all(np.abs(planes - d["planes"]) <= 1e-12 * plane_scale(vp, phys[3]))
    ref = d["values"]
    assert abs(values["ekt"] - ref[0]) <= 1e-13 * ref[0]
    assert abs(values["tke"] - ref[1]) <= 1e-12 * ref[1]
    assert ref[2] > 0.1 and abs(values["divergence_l2"] - ref[2]) <= 1e-12 * ref[2]
    assert values["finite"] and ref[3] == 1.0
    # without higher moments, Statistics::reduce leaves sums 7..19 at zero
    low, _, _ = c.output_reduce(higher_moments=False)
    assert np.array_equal(low[:, :7], planes[:, :7]) and not low[:, 7:].any()


def test_output_reduction_reports_nonfinite():
    m, p, d = load("golden_reduce.npz")
    c = ctx_for(m, p)
    u = np.stack(list(d["u"]), axis=-1)
    u[2, 3, 1, 0] = np.inf
    c.set_velocity(u)
    c.set_pressure(d["p"])
    _, values, _ = c.output_reduce()
    assert not values["finite"]


@pytest.mark.slow
def test_output_reduction_retau180():
    """128 x 129 x 128 coarse grid after 5 steps of the Re_tau180 case: plane
    sums, diagnostics and snapshot against the oracle on the same state; the
    plane mean of u equals the Chebyshev mean profile at each point."""
    m, p = retau180_case()
    c = ctx_for(m, p)
    u0 = divergence_free_field(m, p, seed=1, amp=0.1, spectrum="k53", mean="loglaw")
    c.set_velocity(np.stack(u0, axis=-1))
    c.run(1, 5)
    c.synchronize()
    u = c.get_velocity()
    pr = c.get_pressure()
    planes, values, phys = c.output_reduce(snapshot=True)
    vel = [u[..., k] for k in range(3)]
    vp, pp = orc.to_physical(m, vel, pr)
    for k in range(3):
        assert rel_max(phys[k], vp[k]) <= 1e-12
    assert rel_max(phys[3], pp) <= 1e-12
    ref = orc.plane_moments(vp, pp)
    assert np.all(np.abs(planes - ref) <= 1e-12 * plane_scale(vp, pp))
    ekt, tke, div = orc.diagnostics(m, orc.make_constants(m, p.Re), ref, vel)
    assert abs(values["ekt"] - ekt) <= 1e-12 * ekt and abs(values["tke"] - tke) <= 1e-12 * tke
    # a solenoidal field: both divergence norms are round-off
    assert values["divergence_l2"] <= 1e-9 and div <= 1e-9
    yj = np.cos(np.pi * np.arange(m.NY + 1) / m.NY)
    mean_u = np.polynomial.chebyshev.chebval(yj, u[m.NZS, :, 0, 0].real)
    assert np.abs(planes[:, 0] / (m.NX * m.NZ) - mean_u).max() <= 1e-11 * np.abs(mean_u).max()


def test_statistics_sampling_matches_host_accumulate():
    """cdns_statistics_sample (device-side Statistics::accumulate) against the
    reference's update rule applied on the host to the plane sums of the same
    states, over 5 steps of a 32^3 channel."""
    m, p = channel_case(32)
    c = ctx_for(m, p)
    c.set_velocity(np.stack(divergence_free_field(m, p, seed=3, amp=0.1, spectrum="k53", mean="loglaw"), axis=-1))
    host = orc.Statistics(m)
    for it in range(1, 6):
        c.step(it)
        c.synchronize()
        planes, _, _ = c.output_reduce()
        host.accumulate(planes, *c.dpdx())
        c.statistics_sample()
    n, dp, means = c.statistics_read()
    assert n == 5
    assert np.allclose(np.array(dp), host.dp, rtol=1e-15, atol=0.0)
    assert np.allclose(means, host.means, rtol=1e-14, atol=0.0)
    c.statistics_reset()
    assert c.statistics_read()[0] == 0


def test_output_reduction_analytic_fields():
    """tests/test_diagnostics.cpp:11-55 through cdns_output_reduce on the
    example mesh (32^3, full spectrum): u = y cos(kx x), v = sin(kx x),
    w = 2 cos(kz z), raw p = 5 + |v|^2/2 give EKT = NX NZ (NY+1) / 2,
    TKE = 4/3, divergence L2 = sqrt(kx^2/6 + 2 kz^2) and a corrected-pressure
    plane mean of 5."""
    m, p = example_case()
    vel, pr, want = diagnostics_fields(m)
    c = ctx_for(m, p)
    c.set_velocity(np.stack([orc.coarse_forward(m, f) for f in vel], axis=-1))
    c.set_pressure(orc.coarse_forward(m, pr))
    planes, values, _ = c.output_reduce(higher_moments=True)
    assert values["finite"]
    assert abs(values["ekt"] - want["ekt"]) <= 1e-8 * want["ekt"]
    assert abs(values["tke"] - want["tke"]) <= 1e-12
    assert abs(values["divergence_l2"] - want["divergence_l2"]) <= 1e-11
    assert np.all(np.abs(planes[:, 3] / (m.NX * m.NZ) - want["pressure"]) <= 1e-13)


def test_output_reduction_flags_discarded_infinite_imaginary_part():
    """tests/test_diagnostics.cpp:57-69: an infinite imaginary part in the
    pressure's kz = 0, T_0, kx = 0 coefficient -- a value the real transform
    drops -- still marks the state non-finite."""
    m, p = example_case()
    c = ctx_for(m, p)
    shape = m.spectral_shape()
    c.set_velocity(np.zeros(shape + (3,), dtype=np.complex128))
    pr = np.zeros(shape, dtype=np.complex128)
    pr[m.NZS, 0, 0] = complex(0.0, np.inf)
    c.set_pressure(pr)
    _, values, _ = c.output_reduce()
    assert not values["finite"]


def test_statistics_uniform_samples():
    """tests/test_statistics.cpp:62-111 through cdns_statistics_sample: the
    uniform states v = (1, 2, 3), (3, 4, 5) with corrected pressure 4, 6 give
    the exact means, cross moments and pressure moments."""
    m, p = example_case()
    c = ctx_for(m, p)
    for sample in range(2):
        vel, pr = uniform_sample(m, sample)
        c.set_velocity(np.stack([orc.coarse_forward(m, f) for f in vel], axis=-1))
        c.set_pressure(orc.coarse_forward(m, pr))
        c.statistics_sample()
    n, _, means = c.statistics_read()
    assert n == 2
    want = np.array(UNIFORM_MEANS, dtype=np.float64)[:, None]
    assert np.allclose(means, np.broadcast_to(want, means.shape), rtol=1e-14, atol=0.0)
