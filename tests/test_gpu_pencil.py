"""The pencil decomposition on one B200: every rank of a decomposition runs in
this process (cdns.pencil.LocalPencil, exchanges by device copies), and the
decomposed step must equal the single-context step on the same state --
kx-block rank contexts (zero mode on rank 0 only), the y-slab stages and the
pack/unpack kernels together.  The NCCL path (cdns.pencil.step, the call each
GPU of a multi-GPU run makes) is run with a one-rank process group."""
import datetime
import os
import socket

import numpy as np
import pytest

import cdns
from cdns import pencil
from oracle_cases import channel_case, divergence_free_field, example_case, orc
from test_gpu_parity import ctx_for

pytestmark = pytest.mark.gpu


def _desc(m, p):
    mesh = cdns.Mesh(m.NX, m.NY, m.NZ, m.NXS, m.NYS, m.NZS, m.NX2, m.NY2, m.NZ2, m.XL, m.ZL)
    params = cdns.Params(Re=p.Re, DT=p.DT, G_pre=p.G_pre, a_pre0=p.a_pre0, b_pre0=p.b_pre0, a_V=p.a_V,
                         b_V=p.b_V, INDEX_GRAD_PRE=p.INDEX_GRAD_PRE, THETA=p.THETA,
                         V_Microblow0=p.V_Microblow0)
    return mesh, params


def rel_max(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


_ORACLE = {}


def _oracle(case, m, p, u0, nsteps):
    """The oracle's step loop from the same state (cached per case)."""
    if case not in _ORACLE:
        sim = orc.Simulation(m, p, [u0[..., k] for k in range(3)])
        with np.errstate(all="ignore"):
            sim.run(nsteps)
        _ORACLE[case] = sim.u
    return _ORACLE[case]


def _reference(m, p, u0, nsteps):
    c = ctx_for(m, p)
    c.set_velocity(u0)
    c.run(1, nsteps)
    c.synchronize()
    out = (c.get_velocity(), c.get_pressure(), c.dpdx())
    c.close()
    return out


@pytest.mark.parametrize("case,ranks,exchange", [("channel32", 1, "copy"), ("channel32", 2, "copy"),
                                                 ("channel32", 3, "copy"), ("example", 3, "copy"),
                                                 ("example", 5, "copy"), ("channel32", 1, "peer"),
                                                 ("channel32", 3, "peer"), ("example", 5, "peer")])
def test_local_pencil_matches_single_context(case, ranks, exchange, monkeypatch):
    """4 steps (the two setup steps and two steady ones): velocity, pressure
    and dp/dx of the decomposed step equal the single-context step to 1e-13,
    and the velocity the oracle's step loop to 1e-10
    (32 x 33 x 32 channel at fixed dp/dx, 48^3 product grid; the 32^3 example
    case at constant flow rate, full Nyquist spectrum, ragged blocks), with the
    exchange by packed buffers and with the fused exchange (z transforms on
    the other ranks' column buffers)."""
    monkeypatch.setenv("CDNS_Y_TRANSFORM", "matrix")   # the forms the rank contexts use
    monkeypatch.setenv("CDNS_X_STAGE", "rows4")
    if case == "channel32":
        m, p = channel_case(32)
        u0 = np.stack(divergence_free_field(m, p, seed=2, amp=0.1, spectrum="k53", mean="loglaw"), axis=-1)
    else:
        m, p = example_case()
        u0 = np.stack(divergence_free_field(m, p, seed=3, amp=0.05), axis=-1)
    uref, pref, dref = _reference(m, p, u0, 4)
    mesh, params = _desc(m, p)
    lp = pencil.LocalPencil(mesh, params, ranks, exchange=exchange)
    try:
        lp.set_velocity(u0)
        lp.run(1, 4)
        u, pr, dp = lp.get_velocity(), lp.get_pressure(), lp.dpdx()
    finally:
        lp.close()
    assert rel_max(u, uref) <= 1e-13
    assert rel_max(pr, pref) <= 1e-13
    assert np.allclose(dp, dref, rtol=1e-13, atol=1e-300)
    # and against the oracle directly (the time-step tolerance)
    uo = _oracle(case, m, p, u0, 4)
    for k in range(3):
        assert orc.rel_l2(u[..., k], uo[k]) <= 1e-10


def test_pencil_rank_refuses_whole_channel_calls_and_misordered_stages():
    m, p = channel_case(16)
    mesh, params = _desc(m, p)
    r = pencil.PencilRank(mesh, params, 2, 1)
    try:
        assert r.spectral_shape == (2 * m.NZS + 1, m.NYS + 1, pencil.layout(mesh, 2)[1][1])
        r.set_velocity(np.zeros(r.spectral_shape + (3,), dtype=np.complex128))
        with pytest.raises(cdns.CdnsError) as e:
            r.step(1)
        assert e.value.code == 3
        with pytest.raises(cdns.CdnsError) as e:
            r.stage(1, 1)          # stage 1 before stage 0
        assert e.value.code == 3
        with pytest.raises(ValueError):
            r.set_velocity(np.zeros(m.spectral_shape() + (3,), dtype=np.complex128))   # whole channel
        with pytest.raises(cdns.CdnsError, match="register split"):
            r.set_peers([r.columns(), r.columns()])   # NX2 = NZ2 = 24: no fused exchange
    finally:
        r.close()
    m, p = channel_case(32)
    mesh, params = _desc(m, p)
    r = pencil.PencilRank(mesh, params, 2, 1)
    try:
        own = r.columns()
        own_bytes = 16 * 6 * (m.NY2 + 1) * (2 * m.NZS + 1) * pencil.layout(mesh, 2)[1][1]
        host = np.zeros(16)
        # near the end of the own buffer: a rank-0 block from there overruns the allocation
        tail = own + own_bytes - 16
        for bad, what in (([own, 0], "null"), ([0, own], "null"), ([own, own + 16], "own column"),
                          ([host.ctypes.data, own], "not device memory"), ([tail, own], "smaller")):
            with pytest.raises(cdns.CdnsError, match=what) as e:
                r.set_peers(bad)
            assert e.value.code == 1
    finally:
        r.close()


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_nccl_step_one_rank(monkeypatch):
    """cdns.pencil.step through a one-rank NCCL group: the stages on the
    context stream, the all-to-alls ordered on it, 3 steps as the single
    context."""
    import torch
    import torch.distributed as dist
    monkeypatch.setenv("CDNS_Y_TRANSFORM", "matrix")   # the forms the rank contexts use
    monkeypatch.setenv("CDNS_X_STAGE", "rows4")
    m, p = channel_case(32)
    u0 = np.stack(divergence_free_field(m, p, seed=4, amp=0.1), axis=-1)
    uref, pref, _ = _reference(m, p, u0, 3)
    mesh, params = _desc(m, p)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(_free_port())
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    r = pencil.PencilRank(mesh, params, 1, 0)
    try:
        r.set_velocity(u0)
        pencil.run(r, 1, 3)
        r.synchronize()
        u, pr = r.get_velocity(), r.get_pressure()
    finally:
        r.close()
        dist.destroy_process_group()
    assert rel_max(u, uref) <= 1e-13 and rel_max(pr, pref) <= 1e-13
