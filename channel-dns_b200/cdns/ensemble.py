"""Ensemble of independent channels: the seeded member draw and, on several
GPUs, the static partition of members over ranks ("replicas only": members
never exchange data, so each rank steps its own batch and only the timing is
reduced).

The partition balances an estimate of each member's bytes moved per step (the
stage-pass traffic of one step on its product grid), greedily: members in
decreasing cost, each to the least-loaded rank (ties to the lowest rank), so
every rank computes the same assignment without communication.
"""
from __future__ import annotations

import math
from typing import List, Sequence, Tuple

import numpy as np

SIZES = (32, 48, 64, 96)


def members(count: int, seed: int = 3) -> List[Tuple[int, float]]:
    """(N, Re_tau) of each member: N drawn from {32, 48, 64, 96}, Re_tau from
    U[100, 180], from one seeded generator."""
    rng = np.random.default_rng(seed)
    sizes = rng.choice(list(SIZES), size=count)
    res = rng.uniform(100.0, 180.0, size=count)
    return [(int(n), float(r)) for n, r in zip(sizes, res)]


def step_bytes(n: int) -> float:
    """Bytes one step of an N x (N+1) x N channel (NXS = NZS = N/2, NYS = N-2,
    3/2 product grid) moves through HBM in the stage-pass model: 16 bytes per
    complex value, curl 6 Ns, synthesis 6 Ns + 6 Ny, z synthesis 6 (Ny + Nz),
    x stage 9 Nz, z analysis 3 (Nz + Ny), analysis 3 (Ny + Ns), solve 29 Ns."""
    nkx, nkz, ncy = n // 2 + 1, n + 1, n - 1
    n2 = 3 * n // 2
    ns = nkz * ncy * nkx
    ny = nkz * (n2 + 1) * nkx
    nz = n2 * (n2 + 1) * nkx
    values = 6 * ns + (6 * ns + 6 * ny) + 6 * (ny + nz) + 9 * nz + 3 * (nz + ny) + 3 * (ny + ns) + 29 * ns
    return 16.0 * values


def partition(costs: Sequence[float], world: int) -> List[List[int]]:
    """Member indices per rank, balancing the summed costs (greedy, longest
    first; deterministic)."""
    if world < 1:
        raise ValueError("world size must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(i)
        load[r] += costs[i]
    return [sorted(x) for x in out]


def rank_members(count: int, world: int, rank: int, seed: int = 3) -> List[Tuple[int, int, float]]:
    """(member index, N, Re_tau) of the members rank `rank` of `world` steps."""
    ms = members(count, seed)
    part = partition([step_bytes(n) for n, _ in ms], world)
    return [(i, ms[i][0], ms[i][1]) for i in part[rank]]


def imbalance(count: int, world: int, seed: int = 3) -> float:
    """Largest rank load over the mean load (1.0 = perfect balance)."""
    ms = members(count, seed)
    costs = [step_bytes(n) for n, _ in ms]
    loads = [sum(costs[i] for i in p) for p in partition(costs, world)]
    return max(loads) / (sum(loads) / world) if sum(loads) > 0 else math.nan
