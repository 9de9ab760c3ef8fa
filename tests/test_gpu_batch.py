"""Ensemble batch (cdns_batch_*): channels of different sizes and Reynolds
numbers advanced together (steady steps as one graph of parallel branches)
give, member by member, exactly the fields of the same channel run alone;
member errors are reported with their index."""
import numpy as np
import pytest

import cdns
from oracle_cases import channel_case, divergence_free_field

pytestmark = pytest.mark.gpu


def mesh_params(n, re):
    m, p = channel_case(n, Re=re)
    mesh = cdns.Mesh(m.NX, m.NY, m.NZ, m.NXS, m.NYS, m.NZS, m.NX2, m.NY2, m.NZ2, m.XL, m.ZL)
    params = cdns.Params(Re=p.Re, DT=p.DT, G_pre=p.G_pre, a_pre0=p.a_pre0, b_pre0=p.b_pre0,
                         a_V=p.a_V, b_V=p.b_V, INDEX_GRAD_PRE=p.INDEX_GRAD_PRE, THETA=p.THETA,
                         V_Microblow0=p.V_Microblow0)
    return m, p, mesh, params


MEMBERS = [(32, 180.0), (48, 120.0), (64, 150.0), (32, 100.0)]


def fields(members):
    out = []
    for i, (n, re) in enumerate(members):
        m, p, _, _ = mesh_params(n, re)
        out.append(np.stack(divergence_free_field(m, p, seed=10 + i, amp=0.05, kmax=4), axis=-1))
    return out


@pytest.mark.parametrize("precision", [cdns.PRECISION_FP64, cdns.PRECISION_MIXED])
def test_batch_members_match_single_runs(precision):
    mp = [mesh_params(n, re) for n, re in MEMBERS]
    u0 = fields(MEMBERS)
    batch = cdns.Batch([x[2] for x in mp], [x[3] for x in mp], precision=precision)
    for ctx, u in zip(batch.members, u0):
        ctx.set_velocity(u)
    batch.run(1, 12)
    batch.synchronize()
    got = [ctx.get_velocity() for ctx in batch.members]
    for (m, p, mesh, params), u, g in zip(mp, u0, got):
        single = cdns.Context(mesh, params, precision=precision)
        single.set_velocity(u)
        single.run(1, 12)
        single.synchronize()
        assert np.array_equal(g, single.get_velocity())
        assert np.all(np.isfinite(g))
    batch.close()


def test_batch_continues_after_more_steps():
    """Two batch runs (graph replay across calls, both rotation parities) equal one run."""
    mp = [mesh_params(n, re) for n, re in MEMBERS[:2]]
    u0 = fields(MEMBERS[:2])
    a = cdns.Batch([x[2] for x in mp], [x[3] for x in mp])
    b = cdns.Batch([x[2] for x in mp], [x[3] for x in mp])
    for x, y, u in zip(a.members, b.members, u0):
        x.set_velocity(u)
        y.set_velocity(u)
    a.run(1, 9)
    b.run(1, 4)
    b.run(5, 5)
    a.synchronize()
    b.synchronize()
    for x, y in zip(a.members, b.members):
        assert np.array_equal(x.get_velocity(), y.get_velocity())


def test_batch_reports_member_error():
    mp = [mesh_params(n, re) for n, re in MEMBERS[:3]]
    u0 = fields(MEMBERS[:3])
    u0[1][0, 0, 0, 0] = np.nan
    batch = cdns.Batch([x[2] for x in mp], [x[3] for x in mp])
    for ctx, u in zip(batch.members, u0):
        ctx.set_velocity(u)
    batch.run(1, 4)
    with pytest.raises(cdns.CdnsError, match="member 1"):
        batch.synchronize()


@pytest.mark.parametrize("n", [32, 48, 64, 96])
def test_batch_member_against_oracle(n):
    """One member of each ensemble grid size against the oracle's step loop
    directly (src/sim/simulation.cpp:142-218): a batch of that member beside a
    member of another size, 4 steps (the two setup steps and two graph-replayed
    steady ones), relative L2 <= 1e-10 per velocity component."""
    from oracle_cases import orc
    other = 32 if n != 32 else 48
    members = [(n, 100.0 + n), (other, 160.0)]
    mp = [mesh_params(a, b) for a, b in members]
    u0 = fields(members)
    batch = cdns.Batch([x[2] for x in mp], [x[3] for x in mp])
    for ctx, u in zip(batch.members, u0):
        ctx.set_velocity(u)
    batch.run(1, 4)
    batch.synchronize()
    got = batch.members[0].get_velocity()
    batch.close()
    m, p = mp[0][0], mp[0][1]
    sim = orc.Simulation(m, p, [u0[0][..., k] for k in range(3)])
    with np.errstate(all="ignore"):
        sim.run(4)
    for k in range(3):
        assert orc.rel_l2(got[..., k], sim.u[k]) <= 1e-10
