"""Shared test inputs: mesh/parameter cases and seeded spectra.

The cases restate the reference's test fixtures by value (the example case
used by its unit tests: 32^3 grid, NXS=NZS=16, NYS=30, XL=ZL=10, Re=2800,
constant flow rate, V_Microblow0=1e-3) and the benchmark workloads (the
4pi x 2 x 2pi channel at Re_tau=180 with a 3/2-dealiased product grid).
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np

_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for _p in (os.path.join(_ROOT, "oracle"), os.path.join(_ROOT, "channel-dns_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import channel_oracle as orc  # noqa: E402

PI = math.acos(-1.0)


def example_case(NXS=16, NYS=30, NZS=16, N2=32, a_v1=1.0, b_v1=0.0, N=32):
    """The reference unit-test fixture (examples/config.toml values); ``N``
    shrinks the base grid for small fixtures."""
    m = orc.Mesh(N, N, N, NXS, NYS, NZS, N2, N2, N2, 10.0, 10.0)
    a_V = (1.0, a_v1, 1.0)
    b_V = (0.0, b_v1, 0.0)
    p = orc.Parm(Re=2800.0, G_pre=0.0, a_pre0=0.0, b_pre0=1.0, a_V=a_V, b_V=b_V,
                 INDEX_GRAD_PRE=0, THETA=0.0, DT=3e-3, V_Microblow0=1e-3)
    return m, p


def channel_case(n: int, Re: float = 180.0, dt: float = 5e-5):
    """Benchmark channel: N x (N+1) x N base grid, NXS=NZS=N/2, NYS=N-2,
    3/2 product grid, 4pi x 2 x 2pi, fixed pressure gradient."""
    n2 = 3 * n // 2
    m = orc.Mesh(n, n, n, n // 2, n - 2, n // 2, n2, n2, n2, 4.0 * PI, 2.0 * PI)
    p = orc.Parm(Re=Re, G_pre=0.0, a_pre0=0.0, b_pre0=1.0, a_V=(1.0, 1.0, 1.0),
                 b_V=(0.0, 0.0, 0.0), INDEX_GRAD_PRE=1, THETA=0.0, DT=dt, V_Microblow0=0.0)
    return m, p


def retau180_case():
    """examples/Re_tau180 values: 128 x 129 x 128, NYS=126, product 196 x 193 x 196."""
    m = orc.Mesh(128, 128, 128, 64, 126, 64, 196, 192, 196, 12.56637061435917, 6.283185307179586)
    p = orc.Parm(Re=180.0, G_pre=0.0, a_pre0=0.0, b_pre0=1.0, a_V=(1.0, 1.0, 1.0),
                 b_V=(0.0, 0.0, 0.0), INDEX_GRAD_PRE=1, THETA=0.0, DT=5e-5, V_Microblow0=0.0)
    return m, p


def band_spectrum(m: orc.Mesh, seed: int, amp: float = 1.0) -> np.ndarray:
    """Band-limited spectrum that a real physical field can produce.

    kx=0 (and kx=NX/2 at a full x spectrum) columns are Hermitian in kz
    (U(-kz) = conj U(kz), U(0) real, U(+-NZ/2) real and equal at a full z
    spectrum); other kx are free complex values, with U(-NZ/2) = U(+NZ/2) at a
    full z spectrum.  Same realisability rules as the reference's
    tests/test_xyzfft.cpp:126-162, drawn from numpy's generator.
    """
    rng = np.random.default_rng(seed)
    nkz, ncy, nkx = m.spectral_shape()
    U = np.zeros((nkz, ncy, nkx), dtype=np.complex128)
    fullz = (2 * m.NZS == m.NZ2)
    fullx = (2 * m.NXS == m.NX2)
    zk = m.NZS
    for kx in range(nkx):
        dc_type = kx == 0 or (fullx and kx == m.NXS)
        if dc_type:
            U[zk, :, kx] = rng.uniform(-1, 1, ncy)
            for kz in range(1, m.NZS + 1):
                if fullz and kz == m.NZS:
                    r = rng.uniform(-1, 1, ncy)
                    U[zk + kz, :, kx] = r
                    U[zk - kz, :, kx] = r
                else:
                    v = rng.uniform(-1, 1, ncy) + 1j * rng.uniform(-1, 1, ncy)
                    U[zk + kz, :, kx] = v
                    U[zk - kz, :, kx] = np.conj(v)
        else:
            U[:, :, kx] = rng.uniform(-1, 1, (nkz, ncy)) + 1j * rng.uniform(-1, 1, (nkz, ncy))
            if fullz:
                U[0, :, kx] = U[2 * m.NZS, :, kx]
    return U * amp


def divergence_free_field(m: orc.Mesh, p: orc.Parm, seed: int, amp: float,
                          kmax: int | None = None, spectrum: str = "flat",
                          mean: str = "laminar"):
    """Seeded, exactly divergence-free spectral velocity satisfying no-slip
    (the generator the benchmark uses, channel-dns_b200/cdns/fields.py)."""
    from cdns.fields import divergence_free_field as gen
    return gen(m, p, seed, amp, kmax=kmax, spectrum=spectrum, mean=mean)
