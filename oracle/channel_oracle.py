"""CPU oracle for the channel-dns time step -- TEST INFRASTRUCTURE ONLY.

This module is a numpy restatement of the reference CPU solver's per-step hot
path (hesse-x/channel-dns, C++17 + FFTW3).  It exists to check the CUDA
implementation; only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` leg of ``bench.py`` may import it.  The product path never
calls it and never falls back to it.

Parity pinning: the restatement is checked against (1) the reference's own
known-answer tests restated in ``tests/test_oracle_known_answers.py``
(analytic Fourier/Chebyshev modes, round trips, exact Chebyshev derivative
values, the constant cross product, no-slip unit responses, the staged
versus fused solver equivalence) and (2) golden vectors produced by the
reference's own C++ sources compiled here against project-written FFTW/MPI
shims (``oracle/Makefile`` -> ``oracle/_ref``), committed under
``tests/golden/``.

Every function cites the reference file:line it restates.  Arrays use the
reference's spectral layout ``[kz+NZS][y][kx]`` per component (complex128) and
the fine physical layout ``[z][y][x]`` (float64).  Vectorisation runs over the
independent (kz, kx) columns; recurrences along y stay sequential and in the
reference's order.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Tuple

import numpy as np
import scipy.fft as sfft

PI = math.acos(-1.0)


# --------------------------------------------------------------------------
# Mesh / parameters  (src/core/mesh.cpp:7-116, src/core/params.cpp:296-307)
# --------------------------------------------------------------------------
@dataclass
class Mesh:
    NX: int
    NY: int
    NZ: int
    NXS: int
    NYS: int
    NZS: int
    NX2: int
    NY2: int
    NZ2: int
    XL: float
    ZL: float

    @property
    def nkx(self) -> int:  # NXSP+1 on a single rank (src/core/mesh.cpp:350-361)
        return self.NXS + 1

    @property
    def nkz(self) -> int:  # NZS2P1
        return 2 * self.NZS + 1

    @property
    def ncy(self) -> int:  # NYS+1
        return self.NYS + 1

    @property
    def ny2(self) -> int:  # NY2P+1 on a single rank
        return self.NY2 + 1

    def spectral_shape(self) -> Tuple[int, int, int]:
        return (self.nkz, self.ncy, self.nkx)

    def fine_shape(self) -> Tuple[int, int, int]:
        return (self.NZ2, self.ny2, self.NX2)


@dataclass
class Parm:
    Re: float
    G_pre: float = 0.0
    a_pre0: float = 0.0
    b_pre0: float = 1.0
    a_V: Tuple[float, float, float] = (1.0, 1.0, 1.0)
    b_V: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    INDEX_GRAD_PRE: int = 1
    THETA: float = 0.0
    DT: float = 5e-5
    V_Microblow0: float = 0.0

    # derived (src/core/params.cpp:296-307)
    @property
    def theta_rad(self) -> float:
        return self.THETA * PI / 180.0

    @property
    def grad_pre(self) -> Tuple[float, float]:
        if self.INDEX_GRAD_PRE == 1:
            return (-math.cos(self.theta_rad), -math.sin(self.theta_rad))
        return (0.0, 0.0)

    @property
    def qmean(self) -> Tuple[float, float]:
        if self.INDEX_GRAD_PRE == 1:
            return (0.0, 0.0)
        return (math.cos(self.theta_rad), math.sin(self.theta_rad))


# --------------------------------------------------------------------------
# Wavenumbers and Chebyshev integration weights (src/fft/transforms.cpp:71-108)
# --------------------------------------------------------------------------
@dataclass
class Constants:
    WAVX: np.ndarray  # [nkx]
    WAVZ: np.ndarray  # [nkz], index kz+NZS
    WL: np.ndarray    # [ncy]
    WD: np.ndarray
    WR: np.ndarray
    Re: float

    @property
    def CWAVXRe_imag(self) -> np.ndarray:
        return self.WAVX / self.Re

    @property
    def CWAVZRe_imag(self) -> np.ndarray:
        return self.WAVZ / self.Re


def make_constants(m: Mesh, Re: float) -> Constants:
    """src/fft/transforms.cpp:71-108 (single rank: LSUBX[0] = 0)."""
    alphax = 2.0 * PI / m.XL
    alphaz = 2.0 * PI / m.ZL
    wavx = np.array([k * alphax for k in range(m.nkx)], dtype=np.float64)
    wavz = np.array([k * alphaz for k in range(-m.NZS, m.NZS + 1)], dtype=np.float64)
    n = m.NYS
    WL = np.zeros(n + 1)
    WD = np.zeros(n + 1)
    WR = np.zeros(n + 1)
    for iy in range(n, 1, -1):
        WL[iy] = 1.0 / (4.0 * iy * (iy - 1))
        WD[iy] = -1.0 / (2.0 * (iy * iy - 1))
        WR[iy] = 1.0 / (4.0 * iy * (iy + 1))
    WL[2] = 2.0 * WL[2]
    for iy in range(n - 1, n + 1):
        WD[iy] = 0.0
    for iy in range(n - 3, n + 1):
        WR[iy] = 0.0
    return Constants(wavx, wavz, WL, WD, WR, Re)


def fourier_derivative(wave, value):
    """(i*k)*(a+i*b) written as in src/core/complex_ops.hpp:6-8."""
    return (-wave * value.imag) + 1j * (wave * value.real)


# --------------------------------------------------------------------------
# Fine-grid transforms (src/fft/transforms.cpp:615-741)
# FFTW semantics: r2c/c2c forward sign -1, backward +1, all unnormalised;
# REDFT00 Y_k = x_0 + (-1)^k x_{n-1} + 2 sum_{j=1}^{n-2} x_j cos(pi j k/(n-1))
# (scipy.fft.dct type 1, unnormalised).
# --------------------------------------------------------------------------
def fine_backward(m: Mesh, U: np.ndarray) -> np.ndarray:
    """Spectral [nkz][ncy][nkx] -> fine physical [NZ2][NY2+1][NX2].

    y: copy NYS+1 coefficients, zero-pad, double c_0, DCT-I (:692-707);
    z: expand into NZ2 slots scaled by 0.5, negative Nyquist slot wins at a
    full z spectrum, backward c2c (:715-732); x: c2r over NX2 (:734-740).
    """
    nkz, ncy, nkx = m.spectral_shape()
    assert U.shape == (nkz, ncy, nkx)
    Y = np.zeros((nkz, m.ny2, nkx), dtype=np.complex128)
    Y[:, :ncy, :] = U
    Y[:, 0, :] = Y[:, 0, :] + Y[:, 0, :]
    Y = sfft.dct(Y.real, type=1, axis=1) + 1j * sfft.dct(Y.imag, type=1, axis=1)
    ldx2 = m.NX2 // 2 + 1
    X = np.zeros((m.NZ2, m.ny2, ldx2), dtype=np.complex128)
    nxs1 = m.NXS + 1
    for iz in range(m.NZ2):
        retained = iz <= m.NZS or iz >= m.NZ2 - m.NZS
        if retained:
            kz = iz if iz <= m.NZS else iz - m.NZ2
            X[iz, :, :nxs1] = Y[kz + m.NZS] * 0.5
            if iz == m.NZ2 - m.NZS and iz <= m.NZS:
                X[iz, :, :nxs1] = Y[-m.NZS + m.NZS] * 0.5
    X = np.fft.ifft(X, axis=0) * m.NZ2
    # FFTW c2r ignores the imaginary part of the DC and (even N) Nyquist bins;
    # numpy's irfft does the same.
    return np.fft.irfft(X, n=m.NX2, axis=2) * m.NX2


def fine_forward(m: Mesh, P: np.ndarray) -> np.ndarray:
    """Fine physical [NZ2][NY2+1][NX2] -> spectral [nkz][ncy][nkx].

    x r2c, x1/NX2 on kx<=NXS (:643-655); z forward c2c, x1/NZ2, keep
    |kz|<=NZS with no Nyquist halving (:658-665); DCT-I, x1/(2 NY2) at j=0 and
    1/NY2 for j>=1, keep j<=NYS (:673-682).
    """
    assert P.shape == m.fine_shape()
    nxs1 = m.NXS + 1
    X = np.fft.rfft(P, axis=2)[:, :, :nxs1] * (1.0 / m.NX2)
    Z = np.fft.fft(X, axis=0)
    invnz = 1.0 / m.NZ2
    K = np.zeros((m.nkz, m.ny2, nxs1), dtype=np.complex128)
    for kz in range(0, m.NZS + 1):
        K[kz + m.NZS] = Z[kz] * invnz
    for kz in range(-m.NZS, 0):
        K[kz + m.NZS] = Z[m.NZ2 + kz] * invnz
    Y = sfft.dct(K.real, type=1, axis=1) + 1j * sfft.dct(K.imag, type=1, axis=1)
    out = np.empty((m.nkz, m.ncy, nxs1), dtype=np.complex128)
    out[:, 0, :] = Y[:, 0, :] * (1.0 / (2.0 * m.NY2))
    out[:, 1:, :] = Y[:, 1:m.ncy, :] * (1.0 / m.NY2)
    return out


# --------------------------------------------------------------------------
# Coarse-grid transform (src/fft/transforms.cpp:452-582): physical
# [NZ][NY+1][NX], full spectra allowed (NXS = NX/2, NZS = NZ/2) with the
# Nyquist halve/mirror convention.
# --------------------------------------------------------------------------
def coarse_backward(m: Mesh, U: np.ndarray) -> np.ndarray:
    """Spectral [nkz][ncy][nkx] -> coarse physical [NZ][NY+1][NX].

    y: copy NYS+1 coefficients, zero-pad to NY+1, double c_0, DCT-I
    (:536-552); z: expand into NZ slots scaled by 0.5, at a full z spectrum the
    Nyquist slot is 0.5 (K(NZH) + K(-NZH)) (:560-572), backward c2c; a full
    x spectrum doubles the Nyquist bin (:574-576); x: c2r over NX (:580).
    """
    nkz, ncy, nkx = m.spectral_shape()
    assert U.shape == (nkz, ncy, nkx)
    NX, NY, NZ = m.NX, m.NY, m.NZ
    NZH, NXH = NZ // 2, NX // 2
    fullz, fullx = m.NZS == NZH, m.NXS == NXH
    Y = np.zeros((nkz, NY + 1, nkx), dtype=np.complex128)
    Y[:, :ncy, :] = U
    Y[:, 0, :] = Y[:, 0, :] + Y[:, 0, :]
    Y = sfft.dct(Y.real, type=1, axis=1) + 1j * sfft.dct(Y.imag, type=1, axis=1)
    X = np.zeros((NZ, NY + 1, NX // 2 + 1), dtype=np.complex128)
    for iz in range(NZ):
        if iz <= m.NZS or iz >= NZ - m.NZS:
            kz = iz if iz <= m.NZS else iz - NZ
            X[iz, :, :nkx] = Y[kz + m.NZS] * 0.5
            if fullz and iz == NZH:
                X[iz, :, :nkx] = Y[NZH + m.NZS] * 0.5 + Y[-NZH + m.NZS] * 0.5
    X = np.fft.ifft(X, axis=0) * NZ
    if fullx:
        X[:, :, NXH] *= 2.0
    return np.fft.irfft(X, n=NX, axis=2) * NX


def coarse_forward(m: Mesh, P: np.ndarray) -> np.ndarray:
    """Coarse physical [NZ][NY+1][NX] -> spectral [nkz][ncy][nkx].

    x r2c, x1/NX on kx <= NXS and x0.5 on a full-spectrum Nyquist bin
    (:480-496); z forward c2c, x1/NZ, a full-spectrum Nyquist halved and
    mirrored to -NZH (:498-512); DCT-I, x1/(2 NY) at j = 0 and 1/NY for
    j >= 1, keep j <= NYS (:518-529).
    """
    NX, NY, NZ = m.NX, m.NY, m.NZ
    assert P.shape == (NZ, NY + 1, NX)
    NZH, NXH = NZ // 2, NX // 2
    fullz, fullx = m.NZS == NZH, m.NXS == NXH
    nxs1 = m.NXS + 1
    X = np.fft.rfft(P, axis=2)[:, :, :nxs1] * (1.0 / NX)
    if fullx:
        X[:, :, NXH] *= 0.5
    Z = np.fft.fft(X, axis=0)
    invnz = 1.0 / NZ
    K = np.zeros((m.nkz, NY + 1, nxs1), dtype=np.complex128)
    for kz in range(0, m.NZS + 1):
        K[kz + m.NZS] = Z[kz] * invnz
    for kz in range(-m.NZS, 0):
        K[kz + m.NZS] = Z[NZ + kz] * invnz
    if fullz:
        K[NZH + m.NZS] = Z[NZH] * invnz * 0.5
        K[-NZH + m.NZS] = K[NZH + m.NZS]
    Y = sfft.dct(K.real, type=1, axis=1) + 1j * sfft.dct(K.imag, type=1, axis=1)
    out = np.empty((m.nkz, m.ncy, nxs1), dtype=np.complex128)
    out[:, 0, :] = Y[:, 0, :] * (1.0 / (2.0 * NY))
    out[:, 1:, :] = Y[:, 1:m.ncy, :] * (1.0 / NY)
    return out


# --------------------------------------------------------------------------
# Output reduction: FieldIO::to_physical (src/io/field_io.cpp:199-220),
# Statistics::reduce (src/sim/statistics.cpp:55-110) and
# Diagnostics::evaluate (src/sim/diagnostics.cpp:14-80).
# --------------------------------------------------------------------------
def to_physical(m: Mesh, velocity, pressure):
    """Four coarse backward transforms: (u, v, w) and p on [NZ][NY+1][NX]."""
    return [coarse_backward(m, np.asarray(v)) for v in velocity], coarse_backward(m, np.asarray(pressure))


def plane_moments(velocity_phys, pressure_phys, higher: bool = True) -> np.ndarray:
    """Per-plane sums [NY+1][20] in PlaneMoments order (statistics.cpp:58-86):
    u, v, w, p, uu, vv, ww, uv, vw, wu, pu, pv, pw, pp, uuu, vvv, www, uuuu,
    vvvv, wwww, with p = raw p - 0.5 (uu + vv + ww).  Sums over (z, x)."""
    u, v, w = velocity_phys
    p = pressure_phys - 0.5 * (u * u + v * v + w * w)
    terms = [u, v, w, p, u * u, v * v, w * w]
    if higher:
        terms += [u * v, v * w, w * u, p * u, p * v, p * w, p * p,
                  u * u * u, v * v * v, w * w * w, u * u * u * u, v * v * v * v, w * w * w * w]
    out = np.zeros((u.shape[1], 20))
    for k, t in enumerate(terms):
        out[:, k] = t.sum(axis=(0, 2))
    return out


def clenshaw_curtis_weights(NY: int) -> np.ndarray:
    """Clenshaw-Curtis weights on the NY+1 Gauss-Lobatto points, divided by
    the channel height 2 (diagnostics.cpp:18-36)."""
    n = NY
    w = np.zeros(n + 1)
    for j in range(n + 1):
        th = PI * j / n
        if j == 0 or j == n:
            wt = 1.0 / (n * n - (1.0 if n % 2 == 0 else 0.0))
        else:
            val = 1.0
            for k in range(1, (n - 1) // 2 + 1):
                val -= 2.0 * math.cos(2 * k * th) / (4.0 * k * k - 1.0)
            if n % 2 == 0:
                val -= math.cos(n * th) / (n * n - 1.0)
            wt = 2.0 * val / n
        w[j] = wt / 2.0
    return w


def diagnostics(m: Mesh, c: Constants, planes: np.ndarray, velocity) -> Tuple[float, float, float]:
    """(EKT, TKE, divergence L2) of Diagnostics::evaluate (diagnostics.cpp:38-80):
    EKT = sum v^2 over the grid nodes, TKE = sum_y 0.5 w_y sum_c var_c, div L2
    = sqrt(sum_y w_y mean_xz(div^2)) with div from the coarse transform of the
    spectral divergence."""
    wts = clenshaw_curtis_weights(m.NY)
    inv_plane = 1.0 / (m.NX * m.NZ)
    div = coarse_backward(m, divergence(c, velocity))
    ekt = float(planes[:, 5].sum())
    tke = 0.0
    for iy in range(m.NY + 1):
        var = 0.0
        for k in range(3):
            mean = planes[iy, k] * inv_plane
            var += max(0.0, planes[iy, 4 + k] * inv_plane - mean * mean)
        tke += 0.5 * wts[iy] * var
    div_sq = float(np.sum(wts[None, :, None] * inv_plane * div * div))
    return ekt, tke, math.sqrt(div_sq)


# Plane-sum index of each running mean, in the order Statistics::write prints
# them: u v w, p, uu vv ww uv vw wu, pp, pu pv pw, uuu vvv www, uuuu vvvv wwww
# (src/sim/statistics.cpp:121-136).
STAT_SOURCE = (0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 13, 10, 11, 12, 14, 15, 16, 17, 18, 19)


class Statistics:
    """Running means of Statistics::accumulate (src/sim/statistics.cpp:3-5,
    117-139): every mean becomes (old * count + sample) / (count + 1), the
    samples being plane sums / (NX NZ) and the step's dp/dx, dp/dz."""

    def __init__(self, m: Mesh):
        self.ny1 = m.NY + 1
        self.plane = float(m.NX * m.NZ)
        self.count = 0
        self.dp = np.zeros(2)
        self.means = np.zeros((20, self.ny1))

    @staticmethod
    def _update(old, sample, count):
        return (old * float(count) + sample) / float(count + 1)

    def accumulate(self, planes: np.ndarray, dpdx: float, dpdz: float) -> None:
        planes = np.asarray(planes, dtype=np.float64)
        if planes.shape != (self.ny1, 20):   # statistics.cpp:118-119 leaves the state as it was
            raise ValueError("plane moments size mismatch")
        scale = 1.0 / self.plane
        self.dp = self._update(self.dp, np.array([dpdx, dpdz], dtype=np.float64), self.count)
        for slot, k in enumerate(STAT_SOURCE):
            self.means[slot] = self._update(self.means[slot], planes[:, k] * scale, self.count)
        self.count += 1

    def sample(self, velocity_phys, pressure_phys, dpdx: float, dpdz: float) -> None:
        """Statistics::accumulate from physical fields (statistics.cpp:112-115);
        a field of the wrong size raises before any mean changes (:95-99)."""
        n = None
        for f in list(velocity_phys) + [pressure_phys]:
            if n is None:
                n = np.shape(f)
            if np.shape(f) != n or len(n) != 3 or n[1] != self.ny1 or n[0] * n[2] != self.plane:
                raise ValueError("physical field size mismatch in statistics")
        self.accumulate(plane_moments(velocity_phys, pressure_phys, True), dpdx, dpdz)


# --------------------------------------------------------------------------
# Spectral operators (src/solver/vector_ops.cpp)
# Vector fields are tuples/lists of 3 arrays [nkz][ncy][nkx].
# --------------------------------------------------------------------------
def derivative_y(f: np.ndarray) -> np.ndarray:
    """Backward Chebyshev derivative recurrence, src/solver/vector_ops.cpp:17-25."""
    ny = f.shape[1] - 1
    d = np.zeros_like(f)
    if ny == 0:
        return d
    d[:, ny - 1] = (2.0 * ny) * f[:, ny]
    for y in range(ny - 2, -1, -1):
        d[:, y] = d[:, y + 2] + (2.0 * (y + 1)) * f[:, y + 1]
    d[:, 0] *= 0.5
    return d


def curl(c: Constants, u):
    """src/solver/vector_ops.cpp:112-151 (enqueue_curl)."""
    u0, u1, u2 = u
    kx = c.WAVX[None, None, :]
    kz = c.WAVZ[:, None, None]
    o0 = derivative_y(u2)
    o2 = derivative_y(u0)
    o0 = o0 - fourier_derivative(kz, u1)
    o1 = fourier_derivative(kz, u0) - fourier_derivative(kx, u2)
    o2 = fourier_derivative(kx, u1) - o2
    return [o0, o1, o2]


def divergence(c: Constants, v):
    """src/solver/vector_ops.cpp:90-105."""
    kx = c.WAVX[None, None, :]
    kz = c.WAVZ[:, None, None]
    return (fourier_derivative(kx, v[0]) + derivative_y(v[1])) + fourier_derivative(kz, v[2])


def gradient(c: Constants, p):
    """src/solver/vector_ops.cpp:73-88."""
    kx = c.WAVX[None, None, :]
    kz = c.WAVZ[:, None, None]
    return [fourier_derivative(kx, p), derivative_y(p), fourier_derivative(kz, p)]


def divergence_boundary(c: Constants, v):
    """Wall divergence by endpoint sums, src/solver/vector_ops.cpp:159-176.

    Returns (lower, upper) arrays [nkz][nkx]: lower is the y=+1 wall (index
    0), upper the y=-1 wall (index 1)."""
    kx = c.WAVX[None, :]
    kz = c.WAVZ[:, None]
    ny = v[0].shape[1] - 1
    lower = np.zeros((v[0].shape[0], v[0].shape[2]), dtype=np.complex128)
    upper = np.zeros_like(lower)
    for y in range(ny + 1):
        tangential = fourier_derivative(kx, v[0][:, y]) + fourier_derivative(kz, v[2][:, y])
        normal = float(y * y) * v[1][:, y]
        lower = lower + (tangential + normal)
        if y % 2 == 0:
            upper = upper + (tangential - normal)
        else:
            upper = upper + (-tangential + normal)
    return lower, upper


def cross_product_physical(a, b):
    """Pointwise N = a x b, src/solver/vector_ops.cpp:263-269."""
    a0, a1, a2 = a
    b0, b1, b2 = b
    return [a1 * b2 - a2 * b1, a2 * b0 - a0 * b2, a0 * b1 - a1 * b0]


def flow_rate(f: np.ndarray) -> float:
    """Q(f) = -sum_{j even} Re f_j / (j^2-1) on the (0,0) column,
    src/solver/vector_ops.cpp:186-191 and src/sim/simulation.cpp:104-109.
    ``f`` is the (kz=0, kx=0) column [ncy]."""
    q = 0.0
    for iy in range(0, f.shape[0], 2):
        q -= f[iy].real / float(iy * iy - 1)
    return q


# --------------------------------------------------------------------------
# Nonlinear term + pressure wall BC (src/solver/timestepper.cpp:19-43)
# --------------------------------------------------------------------------
def nonlinear_term(m: Mesh, c: Constants, u):
    """Returns (N, omega, bc) with bc = (bc_top, bc_bottom) [nkz][nkx]."""
    omega = curl(c, u)
    up = [fine_backward(m, u[k]) for k in range(3)]
    wp = [fine_backward(m, omega[k]) for k in range(3)]
    prod = cross_product_physical(up, wp)
    N = [fine_forward(m, prod[k]) for k in range(3)]
    bc = pressure_boundary(c, N, omega)
    return N, omega, bc


def pressure_boundary(c: Constants, N, omega):
    """src/solver/timestepper.cpp:26-43: w_j = (i kx/Re) wz - (i kz/Re) wx + N_y;
    B_top = sum_j w_j, B_bottom = sum_j (-1)^{j+1} w_j."""
    kxr = c.CWAVXRe_imag[None, :]
    kzr = c.CWAVZRe_imag[:, None]
    ny = N[1].shape[1] - 1
    b0 = np.zeros((N[1].shape[0], N[1].shape[2]), dtype=np.complex128)
    b1 = np.zeros_like(b0)
    for iy in range(ny + 1):
        wall = (fourier_derivative(kxr, omega[2][:, iy]) - fourier_derivative(kzr, omega[0][:, iy])) \
            + N[1][:, iy]
        b0 = b0 + wall
        b1 = b1 + (-wall if iy % 2 == 0 else wall)
    return (b0, b1)


# --------------------------------------------------------------------------
# Chebyshev-tau solver (src/solver/eqsolve_pv.cpp)
# --------------------------------------------------------------------------
def _tau_func(a: float, b: float, y: int) -> float:
    q = y % 2
    if a == 0.0 and b == 0.0:
        return float((1 - q) * y * y + q)
    return a + b * y * y


def solve_tau(c: Constants, ny: int, g: float, a: float, b: float, zero_mode: bool,
              lower: np.ndarray, upper: np.ndarray, wn: np.ndarray, ad: np.ndarray,
              rhs: np.ndarray) -> np.ndarray:
    """Column tau solve of (D^2 - k^2 - g) f = rhs with a f + b f' = bc at both
    walls, vectorised over columns.  src/solver/eqsolve_pv.cpp:17-60 (column) and
    :64-128 (tile: same arithmetic).

    Shapes: rhs/ad [nkz][ncy][nkx]; lower/upper/wn [nkz][nkx].  ``zero_mode`` marks
    that the (kz=0, kx=0) column is the global zero mode of this rank.
    """
    WL, WD, WR = c.WL, c.WD, c.WR
    nkz, _, nkx = rhs.shape
    zk = (nkz - 1) // 2
    normalize = g == 0.0 and a == 0.0 and zero_mode
    rhs_eff = rhs
    if normalize:
        corr = 0j
        for y in range(2, ny + 1, 2):
            corr = corr + rhs[zk, y, 0] / float(y * y - 1)
        if b != 0.0:
            corr = corr + (lower[zk, 0] + upper[zk, 0]) / (2.0 * b)
        rhs_eff = rhs.copy()
        rhs_eff[zk, 0, 0] = corr
    w = wn
    out = np.zeros_like(rhs)
    out[:, 0] = (lower + upper) / 2.0
    out[:, 1] = (lower - upper) / 2.0
    for y in range(2, ny - 1):
        out[:, y] = (WL[y] * rhs_eff[:, y - 2] + WD[y] * rhs_eff[:, y]) + WR[y] * rhs_eff[:, y + 2]
    out[:, ny - 1] = WL[ny - 1] * rhs_eff[:, ny - 3] + WD[ny - 1] * rhs_eff[:, ny - 1]
    out[:, ny] = WL[ny] * rhs_eff[:, ny - 2] + WD[ny] * rhs_eff[:, ny]
    for y in range(ny - 2, 1, -1):
        out[:, y] = out[:, y] - ((WR[y] * w) * ad[:, y + 2]) * out[:, y + 2]
    ad01 = [np.zeros((nkz, nkx)), np.zeros((nkz, nkx))]
    for y in (ny, ny - 1):
        ad01[y % 2] = np.full((nkz, nkx), _tau_func(a, b, y))
    for y in range(ny - 2, -1, -1):
        q = y % 2
        v = _tau_func(a, b, y)
        out[:, q] = out[:, q] - (ad01[q] * ad[:, y + 2]) * out[:, y + 2]
        ad01[q] = v - ((WL[y + 2] * w) * ad01[q]) * ad[:, y + 2]
    if normalize:
        out[zk, 0, 0] = 0.0
        ad01[0] = ad01[0].copy()
        ad01[0][zk, 0] = 1.0
    out[:, 0] = out[:, 0] / ad01[0]
    out[:, 1] = out[:, 1] / ad01[1]
    for y in range(2, ny + 1):
        out[:, y] = (out[:, y] - (WL[y] * w) * out[:, y - 2]) * ad[:, y]
    return out


def build_wn_ad(c: Constants, m: Mesh, g: float):
    """src/solver/eqsolve_pv.cpp:148-168.  Returns wn [nkz][nkx] and
    ad [nkz][ncy][nkx] (ad[0], ad[1] stay zero as in the reference)."""
    kx = c.WAVX[None, :]
    kz = c.WAVZ[:, None]
    wn = -((kx * kx + kz * kz) + g)
    n = m.NYS
    ad = np.zeros((m.nkz, m.ncy, m.nkx))
    ad[:, n] = 1.0 / (1.0 + c.WD[n] * wn)
    ad[:, n - 1] = 1.0 / (1.0 + c.WD[n - 1] * wn)
    for iy in range(n - 2, 1, -1):
        fc = c.WR[iy] * c.WL[iy + 2]
        den = 1.0 + (c.WD[iy] - (fc * wn) * ad[:, iy + 2]) * wn
        ad[:, iy] = 1.0 / den
    return wn, ad


@dataclass
class SolverState:
    """Precomputes of EqSolvePV::setup (src/solver/eqsolve_pv.hpp:60-76)."""
    g_v: float
    wn_p: np.ndarray
    ad_p: np.ndarray
    wn_v: np.ndarray
    ad_v: np.ndarray
    p_inf: list = field(default_factory=list)        # 2 x [nkz][ncy][nkx]
    v_inf: list = field(default_factory=list)        # 2 x 3 x [nkz][ncy][nkx]
    inf_div: list = field(default_factory=list)      # 2 x (wall0, wall1) [nkz][nkx]
    p_b: np.ndarray = None
    v_b: list = None
    sigma0: tuple = None                             # (wall0, wall1) [nkz][nkx]
    u_unit: np.ndarray = None
    w_unit: np.ndarray = None
    qx_unit: float = 0.0
    qz_unit: float = 0.0
    pressure_a: float = 0.0
    pressure_b: float = 0.0


class Solver:
    """Restatement of EqSolvePV (src/solver/eqsolve_pv.cpp:132-533)."""

    def __init__(self, m: Mesh, p: Parm, c: Constants):
        self.m, self.p, self.c = m, p, c
        self.state: SolverState | None = None

    # src/solver/eqsolve_pv.cpp:241-264
    def solve_coupled_base(self, rhs_p, bc_p, rhs_v, bc_v):
        s, m, p, c = self.state, self.m, self.p, self.c
        pres = solve_tau(c, m.NYS, p.G_pre, s.pressure_a, s.pressure_b, True,
                         bc_p[0], bc_p[1], s.wn_p, s.ad_p, rhs_p)
        grad = gradient(c, pres)
        vel = []
        for k in range(3):
            forcing = p.Re * (grad[k] - rhs_v[k])
            vel.append(solve_tau(c, m.NYS, s.g_v, p.a_V[k], p.b_V[k], True,
                                 bc_v[k][0], bc_v[k][1], s.wn_v, s.ad_v, forcing))
        return pres, vel

    # src/solver/eqsolve_pv.cpp:311-450 (fused per-column solve)
    def solve_modes(self, rhs_p, bc_p, rhs_v, bc_v, correct_sigma: bool):
        """rhs_p None -> divergence of rhs_v computed in place (fuse_rhs)."""
        s, m, p, c = self.state, self.m, self.p, self.c
        ny = m.NYS
        kx = c.WAVX[None, :]
        kz = c.WAVZ[:, None]
        if rhs_p is None:
            rp = derivative_y(rhs_v[1])
            rp = (fourier_derivative(c.WAVX[None, None, :], rhs_v[0]) + rp) + \
                fourier_derivative(c.WAVZ[:, None, None], rhs_v[2])
        else:
            rp = rhs_p
        pc = solve_tau(c, ny, p.G_pre, s.pressure_a, s.pressure_b, True,
                       bc_p[0], bc_p[1], s.wn_p, s.ad_p, rp)
        dy = derivative_y(pc)
        tail0 = rhs_v[1][:, ny].copy()
        tail1 = rhs_v[1][:, ny - 1].copy()
        vc = []
        for k in range(3):
            if k == 0:
                grad = fourier_derivative(c.WAVX[None, None, :], pc)
            elif k == 1:
                grad = dy
            else:
                grad = fourier_derivative(c.WAVZ[:, None, None], pc)
            forcing = p.Re * (grad - rhs_v[k])
            vc.append(solve_tau(c, ny, s.g_v, p.a_V[k], p.b_V[k], True,
                                bc_v[k][0], bc_v[k][1], s.wn_v, s.ad_v, forcing))
        div0 = np.zeros((m.nkz, m.nkx), dtype=np.complex128)
        div1 = np.zeros_like(div0)
        for y in range(ny + 1):
            tangential = fourier_derivative(kx, vc[0][:, y]) + fourier_derivative(kz, vc[2][:, y])
            normal = float(y * y) * vc[1][:, y]
            div0 = div0 + (tangential + normal)
            if y % 2 == 0:
                div1 = div1 + (tangential - normal)
            else:
                div1 = div1 + (-tangential + normal)
        ID0, ID1 = s.inf_div
        c0 = div1 * ID1[0] - div0 * ID1[1]
        c1 = div0 * ID0[1] - div1 * ID0[0]
        if correct_sigma:
            ptop = pc[:, ny] + (c0 * s.p_inf[0][:, ny] + c1 * s.p_inf[1][:, ny])

            def vtail(y):
                return vc[1][:, y] + (c0 * s.v_inf[0][1][:, y] + c1 * s.v_inf[1][1][:, y])

            w = s.wn_v
            sig0 = ((-w) * vtail(ny) - p.Re * tail0) / s.sigma0[0]
            sig1 = ((-w) * vtail(ny - 1) + p.Re * ((2.0 * ny) * ptop - tail1)) / s.sigma0[1]
        pressure = np.empty_like(pc)
        velocity = [np.empty_like(pc) for _ in range(3)]
        c0e = c0[:, None, :]
        c1e = c1[:, None, :]
        pres = pc + (c0e * s.p_inf[0] + c1e * s.p_inf[1])
        if correct_sigma:
            qsel = np.array([(y + 1) % 2 for y in range(ny + 1)])
            sig = np.stack([sig0, sig1])  # [2][nkz][nkx]
            sq = np.transpose(sig[qsel], (1, 0, 2))          # sigma[q]
            snq = np.transpose(sig[1 - qsel], (1, 0, 2))     # sigma[1-q]
            pres = pres + sq * s.p_b
        pressure[...] = pres
        for k in range(3):
            v = vc[k] + (c0e * s.v_inf[0][k] + c1e * s.v_inf[1][k])
            if correct_sigma:
                v = v + (snq if k == 1 else sq) * s.v_b[k]
            velocity[k][...] = v
        return pressure, velocity

    # src/solver/eqsolve_pv.cpp:266-303
    def build_influence_coefficients(self):
        s, m, p, c = self.state, self.m, self.p, self.c
        zero_s = np.zeros(m.spectral_shape(), dtype=np.complex128)
        zero_b = np.zeros((m.nkz, m.nkx), dtype=np.complex128)
        s.p_inf, s.v_inf, raw = [], [], []
        for i in range(2):
            bc_p = (np.full((m.nkz, m.nkx), float(1 - i), dtype=np.complex128),
                    np.full((m.nkz, m.nkx), float(i), dtype=np.complex128))
            pres, vel = self.solve_coupled_base(zero_s, bc_p, [zero_s] * 3, [(zero_b, zero_b)] * 3)
            s.p_inf.append(pres)
            s.v_inf.append(vel)
            raw.append(divergence_boundary(c, vel))
        den = raw[0][0] * raw[1][1] - raw[0][1] * raw[1][0]
        zk = m.NZS
        if p.a_V[1] == 0.0:
            root_den = complex(1.0, 0.0)
        else:
            root_den = complex(0.25, 0.0) / raw[0][0][zk, 0]
        s.inf_div = []
        for i in range(2):
            w0 = raw[i][0] / den
            w1 = raw[i][1] / den
            # The global zero mode keeps only its independent wall constraint.
            w0[zk, 0] = root_den
            w1[zk, 0] = 0.0
            s.inf_div.append((w0, w1))

    # src/solver/eqsolve_pv.cpp:452-477
    def build_b_problem(self):
        s, m, p, c = self.state, self.m, self.p, self.c
        rhs_p = np.zeros(m.spectral_shape(), dtype=np.complex128)
        rhs_p[:, 0, :] = float(m.NYS - 1)
        for iy in range(1, m.NYS):
            rhs_p[:, iy, :] = float(2 * (m.NYS - ((iy + 1) % 2)))
        zero_s = np.zeros(m.spectral_shape(), dtype=np.complex128)
        zero_b = np.zeros((m.nkz, m.nkx), dtype=np.complex128)
        pb, vb = self.solve_modes(rhs_p, (zero_b, zero_b), [zero_s] * 3,
                                  [(zero_b, zero_b)] * 3, correct_sigma=False)
        s.p_b, s.v_b = pb, vb
        w = s.wn_v
        s0 = p.Re + w * vb[1][:, m.NYS]
        s1 = (p.Re + w * vb[1][:, m.NYS - 1]) - (p.Re * (2.0 * m.NYS)) * pb[:, m.NYS]
        s1 = s1.copy()
        s1[m.NZS, 0] = 1.0
        s.sigma0 = (s0, s1)

    # src/solver/eqsolve_pv.cpp:479-493
    def build_pressure_gradient_responses(self):
        s, m, p, c = self.state, self.m, self.p, self.c
        rhs = np.zeros(m.spectral_shape(), dtype=np.complex128)
        rhs[m.NZS, 0, 0] = p.Re
        zero_b = np.zeros((m.nkz, m.nkx), dtype=np.complex128)
        su = solve_tau(c, m.NYS, s.g_v, p.a_V[0], p.b_V[0], True, zero_b, zero_b,
                       s.wn_v, s.ad_v, rhs)
        s.qx_unit = flow_rate(su[m.NZS, :, 0])
        s.u_unit = su[m.NZS, :, 0].real.copy()
        sw = solve_tau(c, m.NYS, s.g_v, p.a_V[2], p.b_V[2], True, zero_b, zero_b,
                       s.wn_v, s.ad_v, rhs)
        s.qz_unit = flow_rate(sw[m.NZS, :, 0])
        s.w_unit = sw[m.NZS, :, 0].real.copy()

    # src/solver/eqsolve_pv.cpp:495-509
    def setup(self, g_v: float):
        m, p, c = self.m, self.p, self.c
        wn_p, ad_p = build_wn_ad(c, m, p.G_pre)
        wn_v, ad_v = build_wn_ad(c, m, g_v)
        self.state = SolverState(g_v=g_v, wn_p=wn_p, ad_p=ad_p, wn_v=wn_v, ad_v=ad_v)
        self.state.pressure_a, self.state.pressure_b = 1.0, 0.0
        self.build_influence_coefficients()
        self.build_b_problem()
        self.state.pressure_a, self.state.pressure_b = p.a_pre0, p.b_pre0
        self.build_pressure_gradient_responses()


# --------------------------------------------------------------------------
# Time stepping (src/sim/simulation.cpp:36-45, :111-171; timestepper.cpp:60-68)
# --------------------------------------------------------------------------
def step_coefficients(iteration: int, dt: float, reynolds: float):
    """src/sim/simulation.cpp:36-45."""
    if iteration < 1 or dt <= 0.0:
        raise ValueError("invalid time-step coefficients")
    eff = iteration if iteration < 3 else 2
    a0 = float(eff) / dt
    a1 = float(1 - eff) / (2.0 * dt)
    b0 = float(eff)
    b1 = float(1 - eff)
    return a0, a1, b0, b1, (a0 + a1) * reynolds


def velocity_boundary(m: Mesh, p: Parm):
    """src/sim/initial_bc.cpp:95-101: list of 3 (wall0, wall1) arrays."""
    bc = []
    for k in range(3):
        w0 = np.zeros((m.nkz, m.nkx), dtype=np.complex128)
        w1 = np.zeros_like(w0)
        if k == 1:
            w0[m.NZS, 0] = p.V_Microblow0
            w1[m.NZS, 0] = p.V_Microblow0
        bc.append((w0, w1))
    return bc


class Simulation:
    """Single-rank step loop, src/sim/simulation.cpp:142-218 (INDEX_Serial=1),
    starting from a restart (INDEX_CONT=1: first step is first order)."""

    def __init__(self, m: Mesh, p: Parm, velocity):
        self.m, self.p = m, p
        self.c = make_constants(m, p.Re)
        self.solver = Solver(m, p, self.c)
        z = lambda: np.zeros(m.spectral_shape(), dtype=np.complex128)
        zb = lambda: np.zeros((m.nkz, m.nkx), dtype=np.complex128)
        self.u = [np.array(v, dtype=np.complex128) for v in velocity]
        self.u_prev = [z() for _ in range(3)]
        self.N_prev = [z() for _ in range(3)]
        self.B_prev = (zb(), zb())
        self.pressure = z()
        self.vbc = velocity_boundary(m, p)
        self.dpdx = 0.0
        self.dpdz = 0.0
        self.it = 0

    def step(self):
        m, p, c = self.m, self.p, self.c
        self.it += 1
        a0, a1, b0, b1, g_v = step_coefficients(self.it, p.DT, p.Re)
        if self.it < 3:
            self.solver.setup(g_v)
        N, _, B = nonlinear_term(m, c, self.u)
        bcomb = (b0 * B[0] + b1 * self.B_prev[0], b0 * B[1] + b1 * self.B_prev[1])
        R = [((a0 * self.u[k] + a1 * self.u_prev[k]) + b0 * N[k]) + b1 * self.N_prev[k]
             for k in range(3)]
        pres, vel = self.solver.solve_modes(None, bcomb, R, self.vbc, correct_sigma=True)
        # correct_zero_mode (src/solver/timestepper.cpp:60-68)
        zk = m.NZS
        vel[1][zk, 0, 0] = 0.5 * (self.vbc[1][0][zk, 0] + self.vbc[1][1][zk, 0])
        vel[1][zk, 1:, 0] = 0.0
        self.u_prev = self.u
        self.u = vel
        self.pressure = pres
        self.N_prev = N
        self.B_prev = B
        self.correct_flow()

    def correct_flow(self):
        """src/sim/simulation.cpp:111-140."""
        m, p = self.m, self.p
        s = self.solver.state
        zk = m.NZS
        qx = flow_rate(self.u[0][zk, :, 0])
        qz = flow_rate(self.u[2][zk, :, 0])
        if p.INDEX_GRAD_PRE == 1:
            self.dpdx, self.dpdz = p.grad_pre
        else:
            qxm, qzm = p.qmean
            self.dpdx = (qxm - qx) / s.qx_unit
            self.dpdz = (qzm - qz) / s.qz_unit
        self.u[0][zk, :, 0] = self.u[0][zk, :, 0] + self.dpdx * s.u_unit
        self.u[2][zk, :, 0] = self.u[2][zk, :, 0] + self.dpdz * s.w_unit

    def run(self, nsteps: int):
        for _ in range(nsteps):
            self.step()


# --------------------------------------------------------------------------
# Diagnostics used by the parity tests
# --------------------------------------------------------------------------
def interleave(v) -> np.ndarray:
    """3 component arrays -> reference layout [nkz][ncy][nkx][3] complex."""
    return np.stack(v, axis=-1)


def deinterleave(a: np.ndarray):
    return [np.ascontiguousarray(a[..., k]) for k in range(3)]


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    den = np.sqrt(np.sum(np.abs(b) ** 2))
    return float(np.sqrt(np.sum(np.abs(a - b) ** 2)) / max(den, 1e-300))
