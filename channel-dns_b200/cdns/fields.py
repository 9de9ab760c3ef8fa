"""Seeded, divergence-free initial velocity fields in the reference spectral layout.

The reference's own initial condition (src/sim/initial_bc.cpp:20-93) is clock
seeded and not divergence free, so benchmark and test workloads start from a
restart-style field built here instead:

  u = U(y) e_x + curl((0, A, 0)) + curl(curl((0, B, 0)))

with A, B = (1 - y^2)^2 q(y) e^{i(kx x + kz z)} for a random low-order
Chebyshev polynomial q per Fourier mode.  Every perturbation mode is then
exactly solenoidal and vanishes with its wall-normal derivative at y = +-1.
The mean profile U(y) is laminar (uc (1 - y^2), uc = Re/2 at a fixed pressure
gradient, 1.5 at a fixed flow rate) or Reichardt's smooth law of the wall in
wall units.  The perturbation is scaled to an rms of ``amp`` times the
centreline mean velocity over the product-grid points.
"""
from __future__ import annotations

import math
from typing import List

import numpy as np

PI = math.acos(-1.0)


def _cheb_coeffs(vals: np.ndarray, npts: int, ncy: int) -> np.ndarray:
    """Chebyshev coefficients (first ncy) of samples on npts Gauss-Lobatto points."""
    j = np.arange(npts)
    k = np.arange(npts)
    C = np.cos(PI * np.outer(k, j) / (npts - 1))
    w = np.full(npts, 2.0)
    w[0] = w[-1] = 1.0
    a = (C @ (vals * w)) / (npts - 1)
    a[0] *= 0.5
    a[-1] *= 0.5
    return a[:ncy]


def _dy(f: np.ndarray) -> np.ndarray:
    """Chebyshev derivative coefficients of one column (descending recurrence)."""
    ny = f.shape[0] - 1
    d = np.zeros_like(f)
    if ny == 0:
        return d
    d[ny - 1] = (2.0 * ny) * f[ny]
    for y in range(ny - 2, -1, -1):
        d[y] = d[y + 2] + (2.0 * (y + 1)) * f[y + 1]
    d[0] *= 0.5
    return d


def divergence_free_field(mesh, params, seed: int, amp: float, kmax: int | None = None,
                          spectrum: str = "flat", mean: str = "laminar") -> List[np.ndarray]:
    """Three spectral components [2 NZS+1][NYS+1][NXS+1] (complex128).

    ``mesh`` needs NXS, NYS, NZS, NY2, XL, ZL; ``params`` needs Re and
    INDEX_GRAD_PRE.  ``spectrum`` "flat" keeps modes with kx, |kz| <= kmax at
    unit amplitude; "k53" weights every mode by k^(-5/6) (energy ~ k^-5/3).
    """
    rng = np.random.default_rng(seed)
    nkz, ncy, nkx = 2 * mesh.NZS + 1, mesh.NYS + 1, mesh.NXS + 1
    zk = mesh.NZS
    alx, alz = 2.0 * PI / mesh.XL, 2.0 * PI / mesh.ZL
    npts = 2 * ncy
    yj = np.cos(PI * np.arange(npts) / (npts - 1))
    nq = min(8, max(ncy - 5, 1))
    env = (1.0 - yj * yj) ** 2
    T = np.cos(np.outer(np.arange(nq), np.arccos(np.clip(yj, -1, 1))))
    ux = np.zeros((nkz, ncy, nkx), dtype=np.complex128)
    uy = np.zeros_like(ux)
    uz = np.zeros_like(ux)
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
                scale = math.sqrt(kx * kx + kz * kz) ** (-5.0 / 6.0)
            if kx == 0 and kz < 0:
                continue  # Hermitian partner of kz > 0
            qa = (rng.standard_normal(nq) + 1j * rng.standard_normal(nq)) * scale
            qb = (rng.standard_normal(nq) + 1j * rng.standard_normal(nq)) * scale
            A = _cheb_coeffs(env * (qa @ T), npts, ncy)
            B = _cheb_coeffs(env * (qb @ T), npts, ncy)
            ax, az = kx * alx, kz * alz
            dB = _dy(B)
            vx = -1j * az * A + 1j * ax * dB
            vy = (ax * ax + az * az) * B
            vz = 1j * ax * A + 1j * az * dB
            ux[ikz, :, kx], uy[ikz, :, kx], uz[ikz, :, kx] = vx, vy, vz
            if kx == 0:
                ux[2 * zk - ikz, :, 0] = np.conj(vx)
                uy[2 * zk - ikz, :, 0] = np.conj(vy)
                uz[2 * zk - ikz, :, 0] = np.conj(vz)
    # rms over the product-grid points: Parseval in x and z (kx > 0 counts
    # twice for its conjugate), Chebyshev sums on the NY2+1 Gauss-Lobatto points
    ny2 = mesh.NY2 + 1
    M = np.cos(PI * np.outer(np.arange(ny2), np.arange(ncy)) / mesh.NY2)
    wx = np.full(nkx, 2.0)
    wx[0] = 1.0
    ms = 0.0
    for f in (ux, uy, uz):
        phys = np.einsum("jk,zkx->zjx", M, f)
        ms += float(np.sum(wx[None, None, :] * np.abs(phys) ** 2)) / ny2
    rms = math.sqrt(ms / 3.0)
    uc = params.Re / 2.0 if params.INDEX_GRAD_PRE == 1 else 1.5
    if mean == "laminar":
        mean_vals = uc * (1.0 - yj * yj)
        ref = uc
    else:
        yp = (1.0 - np.abs(yj)) * params.Re
        kappa = 0.41
        mean_vals = (np.log1p(kappa * yp) / kappa
                     + 7.8 * (1.0 - np.exp(-yp / 11.0) - (yp / 11.0) * np.exp(-yp / 3.0)))
        ref = float(mean_vals.max())
    s = (amp * ref / rms) if rms > 0 else 0.0
    ux *= s
    uy *= s
    uz *= s
    a = _cheb_coeffs(mean_vals, npts, ncy)
    top = float(np.sum(a))
    bot = float(np.sum(a * (-1.0) ** np.arange(ncy)))
    a[0] -= 0.5 * (top + bot)
    a[1] -= 0.5 * (top - bot)
    ux[zk, :, 0] = a
    return [ux, uy, uz]


def blowing_suction(mesh, seed: int, kmax: int = 8, amp: float = 1.0) -> np.ndarray:
    """Seeded wall blowing/suction in the velocity wall-data layout
    [2 NZS+1][2][NXS+1][3]: wall-normal velocity of the Fourier modes
    kx <= kmax, |kz| <= kmax (mean mode excluded) at both walls, standard
    normal real and imaginary parts times ``amp``, Hermitian in kz at kx = 0
    (a real wall velocity)."""
    rng = np.random.default_rng(seed)
    nkz, nkx = 2 * mesh.NZS + 1, mesh.NXS + 1
    bc = np.zeros((nkz, 2, nkx, 3), dtype=np.complex128)
    zk = mesh.NZS
    for w in range(2):
        for kx in range(0, min(kmax, mesh.NXS) + 1):
            for kz in range(-min(kmax, mesh.NZS), min(kmax, mesh.NZS) + 1):
                if kx == 0 and kz <= 0:
                    continue
                bc[zk + kz, w, kx, 1] = complex(rng.standard_normal(), rng.standard_normal())
                if kx == 0:
                    bc[zk - kz, w, kx, 1] = np.conj(bc[zk + kz, w, kx, 1])
    return bc * amp
