"""Shared test inputs: mesh/parameter cases and seeded spectra.

The cases restate the reference's test fixtures by value (the example case
used by its unit tests: 32^3 grid, NXS=NZS=16, NYS=30, XL=ZL=10, Re=2800,
constant flow rate, V_Microblow0=1e-3) and the north-star workloads (the
4pi x 2 x 2pi channel at Re_tau=180 with a 3/2-dealiased product grid).
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np

_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if os.path.join(_ROOT, "oracle") not in sys.path:
    sys.path.insert(0, os.path.join(_ROOT, "oracle"))

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
    """North-star channel: N x (N+1) x N base grid, NXS=NZS=N/2, NYS=N-2,
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
    """Seeded, exactly divergence-free spectral velocity satisfying no-slip.

    The perturbation is u = curl(psi) with psi = (0, phi(y) g, 0) + (0,0,...)
    built from wall-vanishing Chebyshev combinations, so div u = 0 holds to
    rounding and u vanishes at both walls.  ``spectrum`` "flat" keeps Fourier
    modes with |kx|,|kz| <= kmax; "k53" applies a k^-5/3 envelope.  ``mean``
    "laminar" adds u = (Re/2)(1-y^2) (fixed pressure gradient); "loglaw" adds a
    turbulent-like mean profile projected on Chebyshev modes.
    """
    rng = np.random.default_rng(seed)
    c = orc.make_constants(m, p.Re)
    nkz, ncy, nkx = m.spectral_shape()
    zk = m.NZS
    ny = m.NYS
    # Chebyshev coefficients of (1-y^2)^2 * q(y): use a random low-order q and
    # multiply in physical space on Gauss-Lobatto points, then transform.
    npts = 2 * ncy
    yj = np.cos(PI * np.arange(npts) / (npts - 1))

    def cheb_coeffs(vals):
        # DCT-I based interpolation on npts Gauss-Lobatto points
        import scipy.fft as sfft
        a = sfft.dct(vals, type=1, axis=-1) / (npts - 1)
        a[..., 0] *= 0.5
        a[..., -1] *= 0.5
        return a[..., :ncy]

    nq = min(8, max(ncy - 5, 1))
    ux = np.zeros((nkz, ncy, nkx), dtype=np.complex128)
    uy = np.zeros_like(ux)
    uz = np.zeros_like(ux)
    env = (1.0 - yj * yj) ** 2
    T = np.cos(np.outer(np.arange(nq), np.arccos(np.clip(yj, -1, 1))))
    for ikz in range(nkz):
        kz = ikz - zk
        for kx in range(nkx):
            if kx == 0 and kz == 0:
                continue
            if spectrum == "flat":
                if kmax is not None and (kx > kmax or abs(kz) > kmax):
                    continue
                scale = 1.0
            else:
                k = math.sqrt(kx * kx + kz * kz)
                scale = k ** (-5.0 / 6.0)  # energy ~ k^-5/3
            if kx == 0 and kz < 0:
                continue  # filled by Hermitian symmetry below
            # two potentials A, B (complex Chebyshev combos, wall-vanishing with
            # vanishing derivative): u = curl((0, A, 0)) + curl(curl((0, B, 0)))
            qa = (rng.standard_normal(nq) + 1j * rng.standard_normal(nq)) * scale
            qb = (rng.standard_normal(nq) + 1j * rng.standard_normal(nq)) * scale
            A = cheb_coeffs(env * (qa @ T))
            B = cheb_coeffs(env * (qb @ T))
            ax = c.WAVX[kx]
            az = c.WAVZ[ikz]
            dB = orc.derivative_y(B[None, :, None])[0, :, 0]
            # curl((0,A,0)) = (-dA/dz, 0, dA/dx) = (-i az A, 0, i ax A)
            # curl curl((0,B,0)) = (i ax dB/dy, ax^2 B + az^2 B, i az dB/dy)
            vx = -1j * az * A + 1j * ax * dB
            vy = (ax * ax + az * az) * B
            vz = 1j * ax * A + 1j * az * dB
            ux[ikz, :, kx] = vx
            uy[ikz, :, kx] = vy
            uz[ikz, :, kx] = vz
            if kx == 0:
                ux[2 * zk - ikz, :, 0] = np.conj(vx)
                uy[2 * zk - ikz, :, 0] = np.conj(vy)
                uz[2 * zk - ikz, :, 0] = np.conj(vz)
    # full-spectrum Nyquist slots are left empty (never used by the configs)
    # normalise perturbation rms in physical space
    up = [orc.fine_backward(m, f) for f in (ux, uy, uz)]
    rms = math.sqrt(sum(float(np.mean(f * f)) for f in up) / 3.0)
    uc = p.Re / 2.0 if p.INDEX_GRAD_PRE == 1 else 1.5
    if mean == "laminar":
        mean_vals = uc * (1.0 - yj * yj)
        ref = uc
    else:
        # Reichardt's smooth law of the wall in wall units (u_tau = 1,
        # Re_tau = Re): a turbulent-mean-like profile.
        yp = (1.0 - np.abs(yj)) * p.Re
        kappa = 0.41
        mean_vals = (np.log1p(kappa * yp) / kappa
                     + 7.8 * (1.0 - np.exp(-yp / 11.0) - (yp / 11.0) * np.exp(-yp / 3.0)))
        ref = float(mean_vals.max())
    s = (amp * ref / rms) if rms > 0 else 0.0
    ux *= s
    uy *= s
    uz *= s
    a = cheb_coeffs(mean_vals)
    # enforce u = 0 at both walls exactly after truncation (T0, T1 correction)
    top = float(np.sum(a))
    bot = float(np.sum(a * (-1.0) ** np.arange(ncy)))
    a[0] -= 0.5 * (top + bot)
    a[1] -= 0.5 * (top - bot)
    ux[zk, :, 0] = a
    return [ux, uy, uz]
