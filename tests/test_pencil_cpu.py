"""The pencil decomposition's host side on CPU: the block tables (the
reference's tests/test_mesh.cpp:26-51 restated, and the reference Mesh's own
tables as golden vectors), the per-peer exchange counts,
and both exchanges of a step between two gloo ranks through cdns.pencil's
exchange() -- the call the GPU ranks make over NCCL -- with the packed chunk
order the device pack and unpack kernels use ([field][y][kz][kx], chunks in
rank order)."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import cdns
from cdns import pencil


def _distributed_mesh(NXS=16):
    # tests/test_mesh.cpp:10-22: 32^3 base grid, NXS = NZS = 16, NYS = 30, 48^3 product grid
    return cdns.Mesh(32, 32, 32, NXS, 30, 16, 48, 48, 48, 2.0, 3.0)


@pytest.mark.parametrize("ranks", [1, 2, 3, 4, 7])
def test_blocks_cover_every_index_once(ranks):
    """tests/test_mesh.cpp:26-43: every kx mode and every fine y point is on
    exactly one rank, in rank order, and rank 0 holds the zero mode; the last
    n % ranks ranks take the extra entries (src/core/mesh.cpp:28-40)."""
    m = _distributed_mesh()
    lay = pencil.layout(m, ranks)
    x, y2 = np.zeros(17, int), np.zeros(49, int)
    for kx0, nkx, j0, nj in lay:
        x[kx0:kx0 + nkx] += 1
        y2[j0:j0 + nj] += 1
    assert np.all(x == 1) and np.all(y2 == 1)
    assert [r for r, (kx0, _, _, _) in enumerate(lay) if kx0 == 0] == [0]
    for n, col in ((17, 1), (49, 3)):
        sizes = [t[col] for t in lay]
        extra = n % ranks
        assert sizes == [n // ranks + (1 if r >= ranks - extra else 0) for r in range(ranks)]


def test_layout_matches_the_reference_mesh_tables():
    """tests/golden/golden_blocks.npz: the reference Mesh's own block tables
    (its sources compiled in oracle/_ref) for 1..12 ranks on four meshes --
    the kx block, the fine-grid y slab and the zero-mode owner of every rank,
    and the splits it rejects."""
    from golden_io import GOLDEN
    d = np.load(os.path.join(GOLDEN, "golden_blocks.npz"))
    for tag in ("distributed", "channel32", "retau180", "narrow"):
        mesh = cdns.Mesh(*[int(v) for v in d[f"{tag}_mesh"]], 1.0, 1.0)
        for ranks in range(1, 13):
            ref = d[f"{tag}_{ranks}"]
            if ref.size == 1 and ref[0] == -1:
                with pytest.raises(cdns.CdnsError):
                    pencil.layout(mesh, ranks)
                continue
            lay = pencil.layout(mesh, ranks)
            assert [list(t) for t in lay] == ref[:, :4].tolist(), (tag, ranks)
            assert [1 if t[0] == 0 else 0 for t in lay] == ref[:, 4].tolist()


def test_rejects_empty_blocks():
    """tests/test_mesh.cpp:45-51: NXS = 1 over 3 ranks leaves a rank no kx."""
    with pytest.raises(cdns.CdnsError):
        pencil.layout(_distributed_mesh(NXS=1), 3)
    with pytest.raises(cdns.CdnsError):
        pencil.layout(_distributed_mesh(), 0)


def test_host_calls_reject_bad_arguments():
    """The host-only entry points check their arguments before any work:
    exchange index, rank index, rank count (1..64) and empty blocks."""
    m = _distributed_mesh()
    for bad in [(2, 0, 2), (2, 2, 0), (2, -1, 0), (65, 0, 0), (18, 0, 0)]:
        ranks, rank, exchange = bad
        with pytest.raises(cdns.CdnsError) as e:
            pencil.counts(m, ranks, rank, exchange)
        assert e.value.code == 1, bad
    with pytest.raises(cdns.CdnsError):
        pencil.layout(m, 65)


@pytest.mark.parametrize("ranks", [2, 3, 5])
def test_exchange_counts_pair_up(ranks):
    """What rank r sends to q is what q expects from r, and each exchange moves
    whole fields: six y-physical fields out, three back."""
    m = _distributed_mesh()
    lay = pencil.layout(m, ranks)
    nkz, ny2 = 2 * m.NZS + 1, m.NY2 + 1
    for e, nf in ((0, 6), (1, 3)):
        c = [pencil.counts(m, ranks, r, e) for r in range(ranks)]
        for r in range(ranks):
            for q in range(ranks):
                assert c[r][0][q] == c[q][1][r]
        total = sum(sum(s) for s, _ in c)
        assert total == 2 * nf * ny2 * nkz * (m.NXS + 1)
        for r, (kx0, nkx, j0, nj) in enumerate(lay):
            block = 2 * nf * ny2 * nkz * nkx
            assert sum(c[r][0 if e == 0 else 1]) == block


def _pack_block(a, lay, me):
    """Block side [f][y][kz][kx_me] -> chunks for each peer q: q's y slab."""
    return np.concatenate([a[:, j0:j0 + nj].ravel() for (_, _, j0, nj) in lay])


def _unpack_slab(flat, lay, me, nf, nkz, nkxg):
    """Chunks from each peer q ([f][my y slab][kz][q's kx block]) -> slab side
    [f][y][kz][all kx]."""
    nj = lay[me][3]
    out = np.zeros((nf, nj, nkz, nkxg), dtype=np.complex128)
    o = 0
    for kx0, nkx, _, _ in lay:
        n = nf * nj * nkz * nkx
        out[..., kx0:kx0 + nkx] = flat[o:o + n].reshape(nf, nj, nkz, nkx)
        o += n
    return out


def _pack_slab(s, lay):
    return np.concatenate([s[..., kx0:kx0 + nkx].ravel() for (kx0, nkx, _, _) in lay])


def _unpack_block(flat, lay, me, nf, ny2, nkz):
    nkx = lay[me][1]
    out = np.zeros((nf, ny2, nkz, nkx), dtype=np.complex128)
    o = 0
    for _, _, j0, nj in lay:
        n = nf * nj * nkz * nkx
        out[:, j0:j0 + nj] = flat[o:o + n].reshape(nf, nj, nkz, nkx)
        o += n
    return out


def _as_doubles(z):
    import torch
    return torch.from_numpy(np.ascontiguousarray(z).view(np.float64).copy())


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        m = cdns.Mesh(16, 16, 16, 8, 14, 8, 24, 24, 24, 1.0, 1.0)
        lay = pencil.layout(m, world)
        nkz, ny2, nkxg = 2 * m.NZS + 1, m.NY2 + 1, m.NXS + 1
        rng = np.random.default_rng(5)   # the same whole-channel fields on every rank
        full = rng.standard_normal((6, ny2, nkz, nkxg)) + 1j * rng.standard_normal((6, ny2, nkz, nkxg))
        kx0, nkx, j0, nj = lay[rank]
        # exchange 0: kx blocks -> y slabs
        send_c, recv_c = pencil.counts(m, world, rank, 0)
        send = _as_doubles(_pack_block(full[..., kx0:kx0 + nkx], lay, rank))
        recv = torch.zeros(sum(recv_c), dtype=torch.float64)
        pencil.exchange(send, recv, send_c, recv_c)
        slab = _unpack_slab(recv.numpy().view(np.complex128), lay, rank, 6, nkz, nkxg)
        ok0 = np.array_equal(slab, full[:, j0:j0 + nj])
        # exchange 1: the first three fields of the slabs back to kx blocks
        send_c, recv_c = pencil.counts(m, world, rank, 1)
        send = _as_doubles(_pack_slab(slab[:3], lay))
        recv = torch.zeros(sum(recv_c), dtype=torch.float64)
        pencil.exchange(send, recv, send_c, recv_c)
        back = _unpack_block(recv.numpy().view(np.complex128), lay, rank, 3, ny2, nkz)
        ok1 = np.array_equal(back, full[:3, ..., kx0:kx0 + nkx])
        flags = [None] * world
        dist.all_gather_object(flags, (ok0, ok1))
        if rank == 0:
            q.put(flags)
    finally:
        dist.destroy_process_group()


class _RankStub:
    """The attributes share_dpdx reads from a PencilRank."""

    def __init__(self, rank):
        self.rank, self.device = rank, 0

    def dpdx(self):
        assert self.rank == 0, "only the zero-mode owner computes dp/dx"
        return (1.5, -0.25)


def _dpdx_worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        got = pencil.share_dpdx(_RankStub(rank))
        out = [None] * world
        dist.all_gather_object(out, got)
        if rank == 0:
            q.put(out)
    finally:
        dist.destroy_process_group()


def _spawn(target, world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=target, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    try:
        res = q.get(timeout=120)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    return res


def test_pressure_gradient_reaches_every_rank():
    """src/sim/simulation.cpp:135-139: the zero-mode owner's dp/dx, dp/dz
    broadcast to the other ranks (3 gloo ranks)."""
    assert _spawn(_dpdx_worker, 3) == [(1.5, -0.25)] * 3


class _FusedStub:
    """A rank as map_peers and step_fused see it: fake device pointers and
    handles, and stages that log their start and end (the first stage of
    rank 0 is slow, so an ordering mistake shows)."""

    def __init__(self, rank):
        self.rank, self.peers, self.log = rank, None, []

    def columns(self):
        return 1000 + self.rank

    def ipc_handle(self):
        return bytes([self.rank]) * 64

    def open_peer(self, handle):
        assert len(handle) == 64 and handle[0] != self.rank
        return 5000 + handle[0]

    def set_peers(self, cols):
        self.peers = list(cols)

    def stage(self, it, st):
        import time
        t0 = time.monotonic()
        if self.rank == 0 and st == 0:
            time.sleep(0.3)
        self.log.append((it, st, t0, time.monotonic()))

    def synchronize(self):
        pass


def _fused_worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        r = _FusedStub(rank)
        pencil.map_peers(r)
        pencil.step_fused(r, 5)
        out = [None] * world
        dist.all_gather_object(out, (r.peers, r.log))
        if rank == 0:
            q.put(out)
    finally:
        dist.destroy_process_group()


def test_fused_exchange_host_sequence():
    """Across processes: every rank maps its peers' column buffers from the
    gathered IPC handles (its own buffer at its own index), and a step's stage
    1 starts on no rank before stage 0 ended on all, nor stage 2 before stage 1
    (3 gloo ranks, stub device calls)."""
    out = _spawn(_fused_worker, 3)
    for r, (peers, log) in enumerate(out):
        assert peers == [1000 + q if q == r else 5000 + q for q in range(3)]
        assert [(it, st) for it, st, _, _ in log] == [(5, 0), (5, 1), (5, 2)]
    for st in (0, 1):
        end = max(log[st][3] for _, log in out)
        start = min(log[st + 1][2] for _, log in out)
        assert end <= start, st


@pytest.mark.parametrize("world", [2, 3])
def test_two_exchanges_of_a_step_over_gloo(world):
    assert _spawn(_worker, world) == [(True, True)] * world


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]
