"""Python host side of the B200 channel-dns time step (ctypes over the C ABI).

The product is ``libcdns_cuda.so`` (``include/cdns.h``); this module mirrors
the reference driver's view of the hot path -- the Mesh and Params values the
driver hands over (src/core/params.hpp:6-35; reading config.toml stays the
driver's), a context that owns the device state, ``step``/``run`` of
Simulation::run (src/sim/simulation.cpp:173-185) and the state hand-over in
the reference's spectral layout.  There is no CPU fallback: every call goes to the CUDA
library, and importing without the built library raises.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass
from typing import Optional, Sequence, Tuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcdns_cuda.so")

CDNS_OK = 0
STATUS = {1: "CDNS_ERR_ARG", 2: "CDNS_ERR_CUDA", 3: "CDNS_ERR_STATE", 4: "CDNS_ERR_NONFINITE",
          5: "CDNS_ERR_PIVOT", 6: "CDNS_ERR_NOMEM"}


class CdnsError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{STATUS.get(code, code)}: {message}")
        self.code = code


class MeshDesc(ctypes.Structure):
    _fields_ = [("NX", ctypes.c_int), ("NY", ctypes.c_int), ("NZ", ctypes.c_int),
                ("NXS", ctypes.c_int), ("NYS", ctypes.c_int), ("NZS", ctypes.c_int),
                ("NX2", ctypes.c_int), ("NY2", ctypes.c_int), ("NZ2", ctypes.c_int),
                ("XL", ctypes.c_double), ("ZL", ctypes.c_double)]


class ParamsDesc(ctypes.Structure):
    _fields_ = [("Re", ctypes.c_double), ("G_pre", ctypes.c_double), ("a_pre0", ctypes.c_double),
                ("b_pre0", ctypes.c_double), ("a_V", ctypes.c_double * 3), ("b_V", ctypes.c_double * 3),
                ("INDEX_GRAD_PRE", ctypes.c_int), ("THETA", ctypes.c_double), ("DT", ctypes.c_double),
                ("V_Microblow0", ctypes.c_double)]


_lib = None

_SIGNATURES = {
    "cdns_create": [ctypes.POINTER(MeshDesc), ctypes.POINTER(ParamsDesc), ctypes.c_int, ctypes.c_int,
                    ctypes.POINTER(ctypes.c_void_p)],
    "cdns_destroy": [ctypes.c_void_p],
    "cdns_set_velocity": [ctypes.c_void_p, ctypes.c_void_p],
    "cdns_get_velocity": [ctypes.c_void_p, ctypes.c_void_p],
    "cdns_get_pressure": [ctypes.c_void_p, ctypes.c_void_p],
    "cdns_set_velocity_bc": [ctypes.c_void_p, ctypes.c_void_p],
    "cdns_set_pressure": [ctypes.c_void_p, ctypes.c_void_p],
    "cdns_transform_coarse": [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p],
    "cdns_output_reduce": [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
    "cdns_statistics_sample": [ctypes.c_void_p],
    "cdns_tune": [ctypes.c_void_p],
    "cdns_write_restart": [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_longlong, ctypes.c_double, ctypes.c_int],
    "cdns_read_restart": [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_longlong),
                          ctypes.POINTER(ctypes.c_double)],
    "cdns_write_physical": [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_longlong, ctypes.c_double, ctypes.c_int],
    "cdns_get_tuning": [ctypes.c_void_p, ctypes.c_void_p],
    "cdns_wisdom_export": [ctypes.c_char_p],
    "cdns_wisdom_import": [ctypes.c_char_p],
    "cdns_wisdom_forget": [],
    "cdns_statistics_read": [ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong), ctypes.c_void_p, ctypes.c_void_p],
    "cdns_statistics_reset": [ctypes.c_void_p],
    "cdns_set_velocity_device": [ctypes.c_void_p, ctypes.c_void_p],
    "cdns_update_velocity": [ctypes.c_void_p, ctypes.c_void_p],
    "cdns_get_velocity_device": [ctypes.c_void_p, ctypes.c_void_p],
    "cdns_step": [ctypes.c_void_p, ctypes.c_int],
    "cdns_run": [ctypes.c_void_p, ctypes.c_int, ctypes.c_int],
    "cdns_synchronize": [ctypes.c_void_p],
    "cdns_get_dpdx": [ctypes.c_void_p, ctypes.c_void_p],
    "cdns_nonlinear": [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
    "cdns_transform_fine": [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p],
    "cdns_solve": [ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
    "cdns_profile_begin": [ctypes.c_void_p],
    "cdns_profile_end": [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)],
    "cdns_stage_count": [],
    "cdns_stage_name": [ctypes.c_int],
    "cdns_device_bytes": [ctypes.c_void_p, ctypes.POINTER(ctypes.c_size_t)],
    "cdns_get_stream": [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)],
    "cdns_debug_copy": [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t],
    "cdns_transform_fine_backward_noalloc": [ctypes.POINTER(MeshDesc), ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.c_void_p],
    "cdns_last_error": [ctypes.c_char_p, ctypes.c_size_t],
    "cdns_version": [],
    "cdns_adjoint_run": [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
    "cdns_solve_adjoint": [ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                           ctypes.c_void_p, ctypes.c_void_p],
    "cdns_nonlinear_adjoint": [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                               ctypes.c_void_p],
    "cdns_batch_create": [ctypes.c_int, ctypes.POINTER(MeshDesc), ctypes.POINTER(ParamsDesc), ctypes.c_int,
                          ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)],
    "cdns_batch_destroy": [ctypes.c_void_p],
    "cdns_batch_size": [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)],
    "cdns_batch_member": [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)],
    "cdns_batch_run": [ctypes.c_void_p, ctypes.c_int, ctypes.c_int],
    "cdns_batch_synchronize": [ctypes.c_void_p],
    "cdns_batch_stream": [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)],
    "cdns_pencil_layout": [ctypes.POINTER(MeshDesc), ctypes.c_int, ctypes.c_void_p],
    "cdns_pencil_counts": [ctypes.POINTER(MeshDesc), ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                           ctypes.c_void_p],
    "cdns_pencil_create": [ctypes.POINTER(MeshDesc), ctypes.POINTER(ParamsDesc), ctypes.c_int, ctypes.c_int,
                           ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)],
    "cdns_pencil_buffer": [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p),
                           ctypes.POINTER(ctypes.c_longlong)],
    "cdns_pencil_stage": [ctypes.c_void_p, ctypes.c_int, ctypes.c_int],
    "cdns_pencil_columns": [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_longlong)],
    "cdns_pencil_set_peers": [ctypes.c_void_p, ctypes.c_void_p],
    "cdns_pencil_ipc_handle": [ctypes.c_void_p, ctypes.c_void_p],
    "cdns_pencil_open_peer": [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)],
    "cdns_pencil_close_peers": [ctypes.c_void_p],
}


def lib() -> ctypes.CDLL:
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with channel-dns_b200/build.py")
        L = ctypes.CDLL(LIB_PATH)
        for name, args in _SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = ctypes.c_int
        L.cdns_stage_name.restype = ctypes.c_char_p
        L.cdns_version.restype = ctypes.c_char_p
        _lib = L
    return _lib


def _check(code: int) -> None:
    if code != CDNS_OK:
        buf = ctypes.create_string_buffer(1024)
        lib().cdns_last_error(buf, 1024)
        raise CdnsError(code, buf.value.decode(errors="replace"))


# ---------------------------------------------------------------------------
# Mesh / parameters (src/core/params.hpp, src/core/params.cpp)
# ---------------------------------------------------------------------------
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
    def spectral_shape(self) -> Tuple[int, int, int]:
        return (2 * self.NZS + 1, self.NYS + 1, self.NXS + 1)

    @property
    def fine_shape(self) -> Tuple[int, int, int]:
        return (self.NZ2, self.NY2 + 1, self.NX2)

    def desc(self) -> MeshDesc:
        return MeshDesc(self.NX, self.NY, self.NZ, self.NXS, self.NYS, self.NZS, self.NX2, self.NY2,
                        self.NZ2, self.XL, self.ZL)


@dataclass
class Params:
    Re: float
    DT: float
    G_pre: float = 0.0
    a_pre0: float = 0.0
    b_pre0: float = 1.0
    a_V: Sequence[float] = (1.0, 1.0, 1.0)
    b_V: Sequence[float] = (0.0, 0.0, 0.0)
    INDEX_GRAD_PRE: int = 1
    THETA: float = 0.0
    V_Microblow0: float = 0.0

    def desc(self) -> ParamsDesc:
        return ParamsDesc(self.Re, self.G_pre, self.a_pre0, self.b_pre0, (ctypes.c_double * 3)(*self.a_V),
                          (ctypes.c_double * 3)(*self.b_V), self.INDEX_GRAD_PRE, self.THETA, self.DT,
                          self.V_Microblow0)


def step_coefficients(iteration: int, dt: float, reynolds: float):
    """src/sim/simulation.cpp:36-45 (host mirror of the coefficients the
    library computes)."""
    if iteration < 1 or dt <= 0.0:
        raise ValueError("invalid time-step coefficients")
    eff = iteration if iteration < 3 else 2
    a0 = float(eff) / dt
    a1 = float(1 - eff) / (2.0 * dt)
    return a0, a1, float(eff), float(1 - eff), (a0 + a1) * reynolds


def _ptr(a: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data)


def _input(a, shape, dtype, name: str) -> np.ndarray:
    """`a` as a C-contiguous array of `dtype`; ValueError unless its shape is
    `shape`, the number of values the C call reads."""
    a = np.ascontiguousarray(a, dtype=dtype)
    if a.shape != tuple(shape):
        raise ValueError(f"{name} must have shape {tuple(shape)}, got {a.shape}")
    return a


def _output(out, shape, name: str) -> np.ndarray:
    """A fresh complex128 array of `shape`, or `out` after checking that the C
    call may write `shape` values into it."""
    if out is None:
        return np.empty(shape, dtype=np.complex128)
    if out.dtype != np.complex128 or out.shape != tuple(shape) or not out.flags.c_contiguous \
            or not out.flags.writeable:
        raise ValueError(f"{name} output must be a writeable C-contiguous complex128 array of shape {tuple(shape)}")
    return out


# cdns_precision (include/cdns.h)
PRECISION_FP64 = 0
PRECISION_MIXED = 1
OBJECTIVE_WALL_SHEAR = 0
OBJECTIVE_PROJECTION = 1


class Context:
    """One device context: the state of Simulation's hot path on a B200."""

    def __init__(self, mesh: Mesh, params: Params, device: int = 0, precision: int = PRECISION_FP64):
        self.mesh = mesh
        self.precision = precision
        self.params = params
        self._h = ctypes.c_void_p()
        md, pd = mesh.desc(), params.desc()
        _check(lib().cdns_create(ctypes.byref(md), ctypes.byref(pd), precision, device,
                                 ctypes.byref(self._h)))

    _owned = True

    @classmethod
    def _member(cls, handle: ctypes.c_void_p, mesh: Mesh, params: Params, precision: int) -> "Context":
        """A view of a batch member (owned and destroyed by its batch)."""
        c = cls.__new__(cls)
        c.mesh, c.params, c.precision, c._h, c._owned = mesh, params, precision, handle, False
        return c

    def close(self) -> None:
        if self._h and self._owned:
            lib().cdns_destroy(self._h)
        self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    @property
    def spectral_shape(self) -> Tuple[int, int, int]:
        """[2 NZS + 1][NYS + 1][kx] of the spectral arrays this context holds."""
        return self.mesh.spectral_shape

    # ---- state hand-over (reference layout) ----
    def set_velocity(self, u: np.ndarray) -> None:
        u = _input(u, self.spectral_shape + (3,), np.complex128, "velocity")
        _check(lib().cdns_set_velocity(self._h, _ptr(u)))

    def update_velocity(self, u: np.ndarray) -> None:
        """Replace the current velocity, keeping the multistep history (the
        next step stays second order), as a disturbance injection does."""
        u = _input(u, self.spectral_shape + (3,), np.complex128, "velocity")
        _check(lib().cdns_update_velocity(self._h, _ptr(u)))

    def get_velocity(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        """The velocity [nkz][ncy][nkx][3]; into ``out`` (e.g. a pinned
        buffer) when given, which must be C-contiguous complex128 of that shape."""
        out = _output(out, self.spectral_shape + (3,), "velocity")
        _check(lib().cdns_get_velocity(self._h, _ptr(out)))
        return out

    def get_pressure(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        out = _output(out, self.spectral_shape, "pressure")
        _check(lib().cdns_get_pressure(self._h, _ptr(out)))
        return out

    def set_velocity_bc(self, bc: np.ndarray) -> None:
        nkz, _, nkx = self.spectral_shape
        bc = np.ascontiguousarray(bc, dtype=np.complex128)
        if bc.shape != (nkz, 2, nkx, 3):
            raise ValueError("velocity BC must have shape [2*NZS+1][2][NXS+1][3]")
        _check(lib().cdns_set_velocity_bc(self._h, _ptr(bc)))

    def set_velocity_device(self, ptr: int) -> None:
        _check(lib().cdns_set_velocity_device(self._h, ctypes.c_void_p(ptr)))

    def get_velocity_device(self, ptr: int) -> None:
        _check(lib().cdns_get_velocity_device(self._h, ctypes.c_void_p(ptr)))

    # ---- stepping ----
    def step(self, iteration: int) -> None:
        _check(lib().cdns_step(self._h, iteration))

    def run(self, first_iteration: int, nsteps: int) -> None:
        _check(lib().cdns_run(self._h, first_iteration, nsteps))

    def synchronize(self) -> None:
        _check(lib().cdns_synchronize(self._h))

    def dpdx(self) -> Tuple[float, float]:
        out = np.zeros(2)
        _check(lib().cdns_get_dpdx(self._h, _ptr(out)))
        return float(out[0]), float(out[1])

    # ---- pieces of the hot path ----
    def nonlinear(self, u: np.ndarray):
        nkz, ncy, nkx = self.spectral_shape
        u = _input(u, (nkz, ncy, nkx, 3), np.complex128, "velocity")
        N = np.empty((nkz, ncy, nkx, 3), dtype=np.complex128)
        B = np.empty((nkz, 2, nkx), dtype=np.complex128)
        _check(lib().cdns_nonlinear(self._h, _ptr(u), _ptr(N), _ptr(B)))
        return N, B

    def transform_fine(self, direction: str, data: np.ndarray) -> np.ndarray:
        if direction == "B":
            src = _input(data, self.spectral_shape, np.complex128, "spectral field")
            out = np.empty(self.mesh.fine_shape, dtype=np.float64)
        elif direction == "F":
            src = _input(data, self.mesh.fine_shape, np.float64, "physical field")
            out = np.empty(self.spectral_shape, dtype=np.complex128)
        else:
            raise ValueError("direction must be 'B' or 'F'")
        _check(lib().cdns_transform_fine(self._h, ord(direction), _ptr(src), _ptr(out)))
        return out

    def solve(self, g: float, rhs: np.ndarray, pressure_bc: np.ndarray, velocity_bc: np.ndarray):
        nkz, ncy, nkx = self.spectral_shape
        rhs = _input(rhs, (nkz, ncy, nkx, 3), np.complex128, "rhs")
        pbc = _input(pressure_bc, (nkz, 2, nkx), np.complex128, "pressure_bc")
        vbc = _input(velocity_bc, (nkz, 2, nkx, 3), np.complex128, "velocity_bc")
        p = np.empty((nkz, ncy, nkx), dtype=np.complex128)
        v = np.empty((nkz, ncy, nkx, 3), dtype=np.complex128)
        units = np.empty(2 * ncy)
        _check(lib().cdns_solve(self._h, g, _ptr(rhs), _ptr(pbc), _ptr(vbc), _ptr(p), _ptr(v),
                                _ptr(units)))
        return p, v, units[:ncy].copy(), units[ncy:].copy()

    def set_pressure(self, p: np.ndarray) -> None:
        p = _input(p, self.spectral_shape, np.complex128, "pressure")
        _check(lib().cdns_set_pressure(self._h, _ptr(p)))

    # ---- coarse grid and output reduction ----
    def transform_coarse(self, direction: str, data: np.ndarray) -> np.ndarray:
        """Transforms::channel_xyzfft of one scalar field: 'B' spectral ->
        physical [NZ][NY+1][NX], 'F' the inverse."""
        m = self.mesh
        if direction == "B":
            src = _input(data, m.spectral_shape, np.complex128, "spectral field")
            out = np.empty((m.NZ, m.NY + 1, m.NX))
        elif direction == "F":
            src = _input(data, (m.NZ, m.NY + 1, m.NX), np.float64, "physical field")
            out = np.empty(m.spectral_shape, dtype=np.complex128)
        else:
            raise ValueError("direction must be 'B' or 'F'")
        _check(lib().cdns_transform_coarse(self._h, ord(direction), _ptr(src), _ptr(out)))
        return out

    def output_reduce(self, higher_moments: bool = True, snapshot: bool = False):
        """The output branch on the device: plane sums [NY+1][20], diagnostics
        (EKT, TKE, divergence L2, finite) and, with snapshot=True, the physical
        u, v, w, p [4][NZ][NY+1][NX]."""
        m = self.mesh
        planes = np.empty((m.NY + 1, 20))
        diag = np.empty(4)
        phys = np.empty((4, m.NZ, m.NY + 1, m.NX)) if snapshot else None
        _check(lib().cdns_output_reduce(self._h, int(higher_moments), _ptr(planes), _ptr(diag),
                                        None if phys is None else _ptr(phys)))
        values = {"ekt": float(diag[0]), "tke": float(diag[1]), "divergence_l2": float(diag[2]),
                  "finite": bool(diag[3] == 1.0)}
        return planes, values, phys

    def statistics_sample(self) -> None:
        """Queue a statistics sample of the current state (no host sync)."""
        _check(lib().cdns_statistics_sample(self._h))

    def statistics_read(self):
        """(count, (dpdx_mean, dpdz_mean), means [20][NY+1]) of the samples so far."""
        n = ctypes.c_longlong(0)
        dp = np.zeros(2)
        means = np.zeros((20, self.mesh.NY + 1))
        _check(lib().cdns_statistics_read(self._h, ctypes.byref(n), _ptr(dp), _ptr(means)))
        return int(n.value), (float(dp[0]), float(dp[1])), means

    def statistics_reset(self) -> None:
        _check(lib().cdns_statistics_reset(self._h))

    # ---- restart and physical files (the reference's formats) ----
    def write_restart(self, path: str, step: int, time: float, text: bool = False) -> None:
        _check(lib().cdns_write_restart(self._h, path.encode(), step, time, int(text)))

    def read_restart(self, path: str):
        """Sets the velocity from a restart file; returns (step, time)."""
        s = ctypes.c_longlong(0)
        t = ctypes.c_double(0.0)
        _check(lib().cdns_read_restart(self._h, path.encode(), ctypes.byref(s), ctypes.byref(t)))
        return int(s.value), float(t.value)

    def write_physical(self, path: str, step: int, time: float, text: bool = False) -> None:
        _check(lib().cdns_write_physical(self._h, path.encode(), step, time, int(text)))

    # ---- launch-shape tuning ----
    def tune(self) -> None:
        _check(lib().cdns_tune(self._h))

    def tuning(self) -> dict:
        """{"z_lines": kx lines per z-transform block (0: rule), "y_synthesis":
        "fft" or "matrix", "y_analysis": "fft" or "matrix", "x_rows": the
        x-stage form (4 or 2 rows per block, 0: 4; 1: half-warp form; 3 or 5:
        lane-pair split form with 4 or 2 rows)}."""
        out = np.zeros(4, dtype=np.int32)
        _check(lib().cdns_get_tuning(self._h, out.ctypes.data_as(ctypes.c_void_p)))
        return {"z_lines": int(out[0]), "y_synthesis": "fft" if out[1] else "matrix",
                "y_analysis": "fft" if out[2] else "matrix", "x_rows": int(out[3])}

    # ---- discrete adjoint ----
    def adjoint_run(self, nsteps: int, checkpoint_interval: int, control: Optional[np.ndarray] = None,
                    gradient: bool = True, weights: Optional[np.ndarray] = None):
        """Objective over iterations 1..nsteps from the current velocity and,
        with gradient=True, its gradients with respect to the initial velocity
        [nkz][ncy][nkx][3] and the velocity wall data [nkz][2][nkx][3]
        (d/dRe + i d/dIm of every stored coefficient).  The objective is the
        time-averaged wall shear stress, or Re <weights, u^nsteps> when
        weights (velocity layout) are given.  Returns (J, gu, gbc)."""
        nkz, ncy, nkx = self.mesh.spectral_shape
        ctl = None if control is None else _input(control, (nkz, 2, nkx, 3), np.complex128, "control")
        wts = None if weights is None else _input(weights, (nkz, ncy, nkx, 3), np.complex128, "weights")
        objective = OBJECTIVE_WALL_SHEAR if wts is None else OBJECTIVE_PROJECTION
        J = np.zeros(1)
        gu = np.empty((nkz, ncy, nkx, 3), dtype=np.complex128) if gradient else None
        gb = np.empty((nkz, 2, nkx, 3), dtype=np.complex128) if gradient else None
        _check(lib().cdns_adjoint_run(self._h, nsteps, checkpoint_interval, objective,
                                      None if wts is None else _ptr(wts), None if ctl is None else _ptr(ctl),
                                      _ptr(J), None if gu is None else _ptr(gu),
                                      None if gb is None else _ptr(gb)))
        return float(J[0]), gu, gb

    def solve_adjoint(self, g: float, pressure_adj: Optional[np.ndarray], velocity_adj: np.ndarray):
        """Transpose of solve(): adjoints of (pressure, velocity) -> adjoints
        of (rhs, pressure_bc, velocity_bc)."""
        nkz, ncy, nkx = self.mesh.spectral_shape
        lp = None if pressure_adj is None else _input(pressure_adj, (nkz, ncy, nkx), np.complex128, "pressure_adj")
        lv = _input(velocity_adj, (nkz, ncy, nkx, 3), np.complex128, "velocity_adj")
        lr = np.empty((nkz, ncy, nkx, 3), dtype=np.complex128)
        lpb = np.empty((nkz, 2, nkx), dtype=np.complex128)
        lvb = np.empty((nkz, 2, nkx, 3), dtype=np.complex128)
        _check(lib().cdns_solve_adjoint(self._h, g, None if lp is None else _ptr(lp), _ptr(lv), _ptr(lr),
                                        _ptr(lpb), _ptr(lvb)))
        return lr, lpb, lvb

    def nonlinear_adjoint(self, u: np.ndarray, nonlinear_adj: np.ndarray,
                          pressure_bc_adj: Optional[np.ndarray] = None) -> np.ndarray:
        """Transpose of the linearisation of nonlinear() about u."""
        nkz, ncy, nkx = self.mesh.spectral_shape
        u = _input(u, (nkz, ncy, nkx, 3), np.complex128, "velocity")
        ln = _input(nonlinear_adj, (nkz, ncy, nkx, 3), np.complex128, "nonlinear_adj")
        lb = None if pressure_bc_adj is None else _input(pressure_bc_adj, (nkz, 2, nkx), np.complex128,
                                                         "pressure_bc_adj")
        lu = np.empty((nkz, ncy, nkx, 3), dtype=np.complex128)
        _check(lib().cdns_nonlinear_adjoint(self._h, _ptr(u), _ptr(ln), None if lb is None else _ptr(lb),
                                            _ptr(lu)))
        return lu

    # ---- per-stage timing ----
    def profile_begin(self) -> None:
        _check(lib().cdns_profile_begin(self._h))

    def profile_end(self):
        n = lib().cdns_stage_count()
        ms = np.zeros(n)
        steps = ctypes.c_int(0)
        _check(lib().cdns_profile_end(self._h, _ptr(ms), ctypes.byref(steps)))
        names = [lib().cdns_stage_name(i).decode() for i in range(n)]
        return dict(zip(names, ms.tolist())), steps.value

    def debug_buffer(self, which: int) -> np.ndarray:
        """Stage buffer of the last nonlinear evaluation (see cdns_debug_copy)."""
        m = self.mesh
        nkz, ncy, nkx = m.spectral_shape
        ny2 = m.NY2 + 1
        if which == 4:
            out = np.zeros(7)
            _check(lib().cdns_debug_copy(self._h, 4, _ptr(out), 7))
            return out
        if which == 9:
            out = np.zeros((2, nkz, nkx))
            _check(lib().cdns_debug_copy(self._h, 9, _ptr(out), out.size * 2))
            return out
        shapes = {0: (6, ny2, nkz, nkx), 1: (6, ny2, m.NZ2, nkx), 2: (3, ny2, m.NZ2, nkx),
                  3: (2, nkz, nkx), 5: (2, 2, nkz, nkx), 6: (2, 3, nkz, ncy, nkx),
                  7: (2, nkz, ncy, nkx), 8: (2, nkz, nkx)}
        out = np.empty(shapes[which], dtype=np.complex128)
        _check(lib().cdns_debug_copy(self._h, which, _ptr(out), out.size * 2))
        return out

    def stream_ptr(self) -> int:
        s = ctypes.c_void_p()
        _check(lib().cdns_get_stream(self._h, ctypes.byref(s)))
        return int(s.value or 0)

    def device_bytes(self) -> int:
        b = ctypes.c_size_t(0)
        _check(lib().cdns_device_bytes(self._h, ctypes.byref(b)))
        return int(b.value)


def fine_backward_noalloc(mesh: Mesh, spectral_ptr: int, physical_ptr: int, stream: int = 0) -> None:
    """Allocation-free fine backward transform on caller-owned device buffers
    (cdns_transform_fine_backward_noalloc); queued on ``stream``, not waited for."""
    md = mesh.desc()
    _check(lib().cdns_transform_fine_backward_noalloc(ctypes.byref(md), ctypes.c_void_p(spectral_ptr),
                                                      ctypes.c_void_p(physical_ptr),
                                                      ctypes.c_void_p(stream)))


class Batch:
    """An ensemble of independent channels advanced together (cdns_batch_*):
    members are full contexts; steady steps replay one graph with every
    member's step as a parallel branch."""

    def __init__(self, meshes, params, device: int = 0, precision: int = PRECISION_FP64):
        if len(meshes) != len(params) or not meshes:
            raise ValueError("one Params per Mesh, at least one member")
        n = len(meshes)
        md = (MeshDesc * n)(*[m.desc() for m in meshes])
        pd = (ParamsDesc * n)(*[p.desc() for p in params])
        self._h = ctypes.c_void_p()
        _check(lib().cdns_batch_create(n, md, pd, precision, device, ctypes.byref(self._h)))
        self.members = []
        for i in range(n):
            h = ctypes.c_void_p()
            _check(lib().cdns_batch_member(self._h, i, ctypes.byref(h)))
            self.members.append(Context._member(h, meshes[i], params[i], precision))

    def __len__(self) -> int:
        return len(self.members)

    def run(self, first_iteration: int, nsteps: int) -> None:
        _check(lib().cdns_batch_run(self._h, first_iteration, nsteps))

    def synchronize(self) -> None:
        _check(lib().cdns_batch_synchronize(self._h))

    def stream_ptr(self) -> int:
        s = ctypes.c_void_p()
        _check(lib().cdns_batch_stream(self._h, ctypes.byref(s)))
        return s.value

    def close(self) -> None:
        if self._h:
            for m in self.members:
                m._h = ctypes.c_void_p()
            lib().cdns_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def wisdom_export(path: str) -> None:
    _check(lib().cdns_wisdom_export(path.encode()))


def wisdom_import(path: str) -> None:
    _check(lib().cdns_wisdom_import(path.encode()))


def wisdom_forget() -> None:
    _check(lib().cdns_wisdom_forget())


def version() -> str:
    return lib().cdns_version().decode()
