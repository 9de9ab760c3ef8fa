"""The fused exchange of the pencil decomposition across processes, on one
B200: two or three rank processes (a gloo group) each hold one rank context
on GPU 0, exchange CUDA IPC handles of their column buffers
(cdns.pencil.map_peers: cdns_pencil_ipc_handle / cdns_pencil_open_peer) and
run the step with the stage sequence of cdns.pencil.step_fused -- each stage
on the rank's stream, the stream drained and a barrier over the group between
stages, so no kernel ever waits on another process -- then unmap the peers
(cdns.pencil.unmap_peers) before closing.  This replaces the reference's
distributed step (the MPI_Alltoallv transposes, src/fft/transforms.cpp:304-403,
and the dp/dx broadcast, src/sim/simulation.cpp:135-139).

After 4 steps each rank's block of the velocity and pressure must equal the
single-context step to 1e-13 (the LocalPencil tolerance) and the oracle's
step loop to 1e-10 relative L2 per component, and dp/dx must reach every
rank."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

NSTEPS = 4


def _case():
    from oracle_cases import channel_case, divergence_free_field
    m, p = channel_case(32)
    u0 = np.stack(divergence_free_field(m, p, seed=2, amp=0.1, spectrum="k53", mean="loglaw"), axis=-1)
    return m, p, u0


def _desc(m, p):
    import cdns
    mesh = cdns.Mesh(m.NX, m.NY, m.NZ, m.NXS, m.NYS, m.NZS, m.NX2, m.NY2, m.NZ2, m.XL, m.ZL)
    params = cdns.Params(Re=p.Re, DT=p.DT, G_pre=p.G_pre, a_pre0=p.a_pre0, b_pre0=p.b_pre0, a_V=p.a_V,
                         b_V=p.b_V, INDEX_GRAD_PRE=p.INDEX_GRAD_PRE, THETA=p.THETA,
                         V_Microblow0=p.V_Microblow0)
    return mesh, params


def _worker(rank, world, port, q):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(here)
    sys.path[:0] = [here, os.path.join(root, "oracle"), os.path.join(root, "channel-dns_b200")]
    os.environ["CDNS_Y_TRANSFORM"] = "matrix"   # the forms the rank contexts use
    os.environ["CDNS_X_STAGE"] = "rows4"
    import torch.distributed as dist
    from cdns import pencil
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    r = None
    try:
        m, p, u0 = _case()
        mesh, params = _desc(m, p)
        r = pencil.PencilRank(mesh, params, world, rank, device=0)
        r.set_velocity(r.block(u0))
        cols = pencil.map_peers(r)
        opened = sum(1 for q_, c in enumerate(cols) if q_ != rank and c != r.columns())
        for it in range(1, NSTEPS + 1):
            pencil.step_fused(r, it)
        r.synchronize()
        u, pr = r.get_velocity(), r.get_pressure()
        dp = pencil.share_dpdx(r)
        pencil.unmap_peers(r)
        out = [None] * world
        dist.all_gather_object(out, (rank, u, pr, dp, opened))
        if rank == 0:
            q.put(out)
    finally:
        if r is not None:
            r.close()
        dist.destroy_process_group()


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3])
def test_fused_exchange_across_processes(world, monkeypatch):
    from cdns import pencil
    from oracle_cases import orc
    from test_gpu_parity import ctx_for
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    try:
        res = q.get(timeout=240)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    m, p, u0 = _case()
    monkeypatch.setenv("CDNS_Y_TRANSFORM", "matrix")   # the forms the rank contexts use
    monkeypatch.setenv("CDNS_X_STAGE", "rows4")
    c = ctx_for(m, p)
    c.set_velocity(u0)
    c.run(1, NSTEPS)
    c.synchronize()
    uref, pref, dref = c.get_velocity(), c.get_pressure(), c.dpdx()
    c.close()
    sim = orc.Simulation(m, p, [u0[..., k] for k in range(3)])
    with np.errstate(all="ignore"):
        sim.run(NSTEPS)
    mesh, _ = _desc(m, p)
    lay = pencil.layout(mesh, world)
    u = np.concatenate([res[q][1] for q in range(world)], axis=2)
    pr = np.concatenate([res[q][2] for q in range(world)], axis=2)
    for q in range(world):
        assert res[q][0] == q and res[q][4] == world - 1        # every peer mapped through IPC
        assert res[q][1].shape[2] == lay[q][1]
        assert np.allclose(res[q][3], dref, rtol=1e-13, atol=1e-300)
    scale = np.abs(uref).max()
    assert np.abs(u - uref).max() <= 1e-13 * scale
    assert np.abs(pr - pref).max() <= 1e-13 * np.abs(pref).max()
    for k in range(3):
        assert orc.rel_l2(u[..., k], sim.u[k]) <= 1e-10
