"""Pencil decomposition of one channel over several ranks, one GPU each: the
host side of the reference's distributed step (Simulation::run's multi-rank
branch, src/sim/simulation.cpp:191-218, with the transposes of
src/fft/transforms.cpp:304-404 and MpiContext::alltoallv_doubles).

Rank r holds the spectral state of one kx block and, inside a step, one slab
of the fine-grid y points (``layout``).  A step is three device stages on the
rank's context stream with two all-to-all exchanges between them
(``step``): the six y-physical fields (u, omega) go from kx blocks to y slabs
after the Chebyshev synthesis, the three nonlinear-term fields come back
before the Chebyshev analysis.  The exchange is ``torch.distributed``'s
all-to-all (NCCL between GPUs, gloo between CPU processes) ordered on the
context stream; ``LocalPencil`` runs every rank of a decomposition in one
process and exchanges by device copies.
"""
from __future__ import annotations

import ctypes
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import Context, Mesh, Params, PRECISION_FP64, _check, lib


def layout(mesh: Mesh, ranks: int) -> List[Tuple[int, int, int, int]]:
    """(kx0, nkx, j0, nj) of every rank: the kx block and the fine-grid y slab
    (the reference's block rule, src/core/mesh.cpp:28-85: n // ranks each,
    one more on each of the last n % ranks ranks).  Raises CdnsError if a
    rank would get an empty block."""
    table = np.zeros(4 * max(ranks, 1), dtype=np.int32)
    md = mesh.desc()
    _check(lib().cdns_pencil_layout(ctypes.byref(md), ranks, table.ctypes.data_as(ctypes.c_void_p)))
    return [tuple(int(v) for v in table[4 * r:4 * r + 4]) for r in range(ranks)]


def counts(mesh: Mesh, ranks: int, rank: int, exchange: int) -> Tuple[List[int], List[int]]:
    """Doubles rank `rank` sends to and receives from each peer in exchange 0
    (kx blocks -> y slabs, six fields) or 1 (y slabs -> kx blocks, three)."""
    send = np.zeros(ranks, dtype=np.int64)
    recv = np.zeros(ranks, dtype=np.int64)
    md = mesh.desc()
    _check(lib().cdns_pencil_counts(ctypes.byref(md), ranks, rank, exchange,
                                    send.ctypes.data_as(ctypes.c_void_p), recv.ctypes.data_as(ctypes.c_void_p)))
    return [int(v) for v in send], [int(v) for v in recv]


class _DeviceArray:
    """A float64 vector in device memory owned by the C context, for
    torch.as_tensor (CUDA array interface, no copy)."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False),
                                         "version": 3, "strides": None, "stream": None}


class PencilRank(Context):
    """Rank `rank` of a `ranks`-way pencil decomposition: a context holding
    the kx block [kx0, kx0 + nkx) of the spectral state.  set_velocity,
    get_velocity, get_pressure and set_velocity_bc take that block in the
    reference layout."""

    def __init__(self, mesh: Mesh, params: Params, ranks: int, rank: int, device: int = 0):
        self.mesh = mesh
        self.params = params
        self.precision = PRECISION_FP64
        self.ranks, self.rank, self.device = ranks, rank, device
        self.kx0, self.nkx, self.j0, self.nj = layout(mesh, ranks)[rank]
        self._h = ctypes.c_void_p()
        md, pd = mesh.desc(), params.desc()
        _check(lib().cdns_pencil_create(ctypes.byref(md), ctypes.byref(pd), ranks, rank, device,
                                        ctypes.byref(self._h)))
        self._counts = [counts(mesh, ranks, rank, e) for e in (0, 1)]

    @property
    def spectral_shape(self) -> Tuple[int, int, int]:
        nkz, ncy, _ = self.mesh.spectral_shape
        return (nkz, ncy, self.nkx)

    def block(self, full: np.ndarray) -> np.ndarray:
        """This rank's kx block of a whole-channel spectral array [..][..][kx](..)."""
        return np.ascontiguousarray(full[:, :, self.kx0:self.kx0 + self.nkx])

    def stage(self, iteration: int, stage: int) -> None:
        _check(lib().cdns_pencil_stage(self._h, iteration, stage))

    def exchange_counts(self, exchange: int) -> Tuple[List[int], List[int]]:
        """(send, recv) doubles per peer of one exchange."""
        return self._counts[exchange]

    def buffer(self, exchange: int, recv: bool):
        """The send (recv=False) or receive buffer of one exchange as a flat
        float64 torch tensor on the rank's device (no copy; valid while the
        context is open)."""
        import torch
        p = ctypes.c_void_p()
        n = ctypes.c_longlong(0)
        _check(lib().cdns_pencil_buffer(self._h, exchange, int(recv), ctypes.byref(p), ctypes.byref(n)))
        return torch.as_tensor(_DeviceArray(int(p.value), int(n.value)), device=f"cuda:{self.device}")

    def columns(self) -> int:
        """Device pointer of this rank's y-physical column buffer (the
        fused exchange's peer view)."""
        p = ctypes.c_void_p()
        n = ctypes.c_longlong(0)
        _check(lib().cdns_pencil_columns(self._h, ctypes.byref(p), ctypes.byref(n)))
        return int(p.value)

    def set_peers(self, columns: Optional[Sequence[int]]) -> None:
        """Every rank's column buffer (device pointers in this process, rank
        order) for the fused exchange; None returns to the exchange buffers."""
        if columns is None:
            _check(lib().cdns_pencil_set_peers(self._h, None))
            return
        arr = (ctypes.c_void_p * len(columns))(*[ctypes.c_void_p(int(c)) for c in columns])
        _check(lib().cdns_pencil_set_peers(self._h, ctypes.cast(arr, ctypes.c_void_p)))

    def ipc_handle(self) -> bytes:
        """CUDA IPC handle of this rank's column buffer (to send to the other
        ranks of a multi-process decomposition)."""
        buf = ctypes.create_string_buffer(64)
        _check(lib().cdns_pencil_ipc_handle(self._h, ctypes.cast(buf, ctypes.c_void_p)))
        return buf.raw

    def open_peer(self, handle: bytes) -> int:
        """Map a peer rank's column buffer into this process; its device pointer."""
        if len(handle) != 64:
            raise ValueError("a CUDA IPC handle has 64 bytes")
        buf = ctypes.create_string_buffer(bytes(handle), 64)
        p = ctypes.c_void_p()
        _check(lib().cdns_pencil_open_peer(self._h, ctypes.cast(buf, ctypes.c_void_p), ctypes.byref(p)))
        return int(p.value)

    def close_peers(self) -> None:
        """Unmap the peers' column buffers this process opened (every rank,
        then a barrier, before any rank closes its context)."""
        _check(lib().cdns_pencil_close_peers(self._h))

    def torch_stream(self):
        import torch
        return torch.cuda.ExternalStream(self.stream_ptr(), device=f"cuda:{self.device}")


def exchange(send, recv, send_counts: Sequence[int], recv_counts: Sequence[int], group=None) -> None:
    """One all-to-all: chunk q of `send` (send_counts[q] values, in rank
    order) goes to rank q, which stores it as chunk `rank` of its `recv`
    (MpiContext::alltoallv_doubles, src/core/mpi_context.cpp)."""
    import torch.distributed as dist
    dist.all_to_all_single(recv, send, output_split_sizes=list(recv_counts),
                           input_split_sizes=list(send_counts), group=group)


def step(rank: PencilRank, iteration: int, group=None) -> None:
    """One time step of this rank (every rank of the group calls it for the
    same iteration).  The exchanges are queued on the context stream, so the
    call returns without waiting for the device."""
    import torch
    s = rank.torch_stream()
    rank.stage(iteration, 0)
    for e in (0, 1):
        send_c, recv_c = rank.exchange_counts(e)
        with torch.cuda.stream(s):
            exchange(rank.buffer(e, False), rank.buffer(e, True), send_c, recv_c, group)
        rank.stage(iteration, e + 1)


def share_dpdx(rank, group=None) -> Tuple[float, float]:
    """dp/dx and dp/dz of the last step on every rank of the group: rank 0
    holds the zero mode and computes them, the others receive them (the
    reference's broadcast from the zero-mode owner after correct_flow,
    src/sim/simulation.cpp:135-139).
    Uses `rank.rank`, `rank.device` and `rank.dpdx()` (rank 0 only); a CUDA
    tensor over NCCL, a CPU tensor over gloo."""
    import torch
    import torch.distributed as dist
    dev = torch.device(f"cuda:{rank.device}") if dist.get_backend(group) == "nccl" else torch.device("cpu")
    t = torch.tensor(rank.dpdx() if rank.rank == 0 else (0.0, 0.0), dtype=torch.float64, device=dev)
    dist.broadcast(t, src=dist.get_global_rank(group, 0) if group is not None else 0, group=group)
    return float(t[0].item()), float(t[1].item())


def map_peers(rank, group=None) -> List[int]:
    """Set up the fused exchange of a multi-process decomposition (one rank
    per process and GPU): gather every rank's IPC handle over the group, map
    the peers' column buffers into this process and hand the pointers, in rank
    order, to the rank context.  Uses `rank.rank`, `rank.columns()`,
    `rank.ipc_handle()`, `rank.open_peer()` and `rank.set_peers()`."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    handles = [None] * world
    dist.all_gather_object(handles, rank.ipc_handle(), group=group)
    cols = [rank.columns() if q == rank.rank else rank.open_peer(handles[q]) for q in range(world)]
    rank.set_peers(cols)
    return cols


def unmap_peers(rank, group=None) -> None:
    """End the fused exchange of a multi-process decomposition: every rank
    unmaps the peers' buffers, then all meet at a barrier, so that no rank
    frees its column buffer while another still maps it.  Call it on every
    rank before closing the rank contexts.  Uses `rank.close_peers()`."""
    import torch.distributed as dist
    rank.close_peers()
    dist.barrier(group=group)


def step_fused(rank, iteration: int, group=None) -> None:
    """One time step with the fused exchange across processes: each stage on
    the rank's stream, then the stream drained and a barrier over the group,
    so that no rank reads a peer's column buffer before the peer wrote it
    (stage 0 -> 1), nor its own before every peer wrote its rows there
    (stage 1 -> 2).
    Uses `rank.stage()` and `rank.synchronize()`."""
    import torch.distributed as dist
    for st in range(3):
        rank.stage(iteration, st)
        if st < 2:
            rank.synchronize()
            dist.barrier(group=group)


def run(rank: PencilRank, first_iteration: int, nsteps: int, group=None) -> None:
    for it in range(first_iteration, first_iteration + nsteps):
        step(rank, it, group)


class LocalPencil:
    """Every rank of a pencil decomposition in one process on one device.
    Each stage runs on all ranks, then (exchange="copy") the exchange copies
    each peer's chunk between the ranks' buffers on the device, or
    (exchange="peer") the fused exchange's z transforms read and write the
    other ranks' column buffers directly; either way no kernel of one rank
    waits on another's, the stages are ordered by host synchronisation.  The
    whole-channel state goes in and out in the reference layout."""

    def __init__(self, mesh: Mesh, params: Params, ranks: int, device: int = 0, exchange: str = "copy"):
        if exchange not in ("copy", "peer"):
            raise ValueError("exchange must be 'copy' or 'peer'")
        self.mesh = mesh
        self.exchange = exchange
        self.members = [PencilRank(mesh, params, ranks, r, device) for r in range(ranks)]
        if exchange == "peer":
            cols = [m.columns() for m in self.members]
            for m in self.members:
                m.set_peers(cols)

    def close(self) -> None:
        for m in self.members:
            m.close()

    def set_velocity(self, u: np.ndarray) -> None:
        for m in self.members:
            m.set_velocity(m.block(u))

    def set_velocity_bc(self, bc: np.ndarray) -> None:
        for m in self.members:
            m.set_velocity_bc(m.block(bc))

    def get_velocity(self) -> np.ndarray:
        return np.concatenate([m.get_velocity() for m in self.members], axis=2)

    def get_pressure(self) -> np.ndarray:
        return np.concatenate([m.get_pressure() for m in self.members], axis=2)

    def dpdx(self) -> Tuple[float, float]:
        """The pressure gradient of the last step (computed by rank 0, which
        holds the zero mode)."""
        return self.members[0].dpdx()

    def synchronize(self) -> None:
        for m in self.members:
            m.synchronize()

    def _exchange(self, e: int) -> None:
        import torch
        self.synchronize()
        P = len(self.members)
        sends = [m.buffer(e, False) for m in self.members]
        recvs = [m.buffer(e, True) for m in self.members]
        soff = [np.concatenate([[0], np.cumsum(m.exchange_counts(e)[0])]) for m in self.members]
        roff = [np.concatenate([[0], np.cumsum(m.exchange_counts(e)[1])]) for m in self.members]
        for r in range(P):
            for q in range(P):
                n = int(soff[r][q + 1] - soff[r][q])
                if n != int(roff[q][r + 1] - roff[q][r]):
                    raise RuntimeError("pencil exchange counts disagree between ranks")
                recvs[q][int(roff[q][r]):int(roff[q][r]) + n].copy_(sends[r][int(soff[r][q]):int(soff[r][q]) + n])
        torch.cuda.synchronize(self.members[0].device)

    def step(self, iteration: int) -> None:
        for st in range(3):
            for m in self.members:
                m.stage(iteration, st)
            if st < 2:
                if self.exchange == "peer":
                    self.synchronize()     # every rank's stage done before any reads it
                else:
                    self._exchange(st)

    def run(self, first_iteration: int, nsteps: int) -> None:
        for it in range(first_iteration, first_iteration + nsteps):
            self.step(it)
        self.synchronize()
