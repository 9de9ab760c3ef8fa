"""CPU checks of the C ABI: the library builds for sm_100a, loads, and
exports every function include/cdns.h declares (no compute without a GPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "cdns.h")


def declared_functions(path):
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|const char \*)\s*(cdns_\w+)\s*\(", text, flags=re.M)))


@pytest.fixture(scope="module")
def library():
    import sys
    sys.path.insert(0, os.path.join(ROOT, "channel-dns_b200"))
    import build
    path = build.build()
    return ctypes.CDLL(path)


def test_header_declares_entry_points():
    names = declared_functions(HEADER)
    assert "cdns_create" in names and "cdns_step" in names and len(names) >= 20


def test_library_exports_every_declared_symbol(library):
    missing = [n for n in declared_functions(HEADER) if not hasattr(library, n)]
    assert not missing, missing


def test_no_gpu_create_fails_loudly(library):
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present: covered by the -m gpu tests")
    import cdns
    with pytest.raises(cdns.CdnsError):
        cdns.Context(cdns.Mesh(8, 8, 8, 4, 6, 4, 12, 8, 12, 1.0, 1.0), cdns.Params(Re=100.0, DT=1e-3))


def test_python_mirror_step_coefficients_match_reference_values():
    """tests/test_simulation.cpp:5-21 values through the host mirror."""
    import sys
    sys.path.insert(0, os.path.join(ROOT, "channel-dns_b200"))
    import cdns
    assert cdns.step_coefficients(1, 0.25, 10.0) == (4.0, 0.0, 1.0, 0.0, 40.0)
    assert cdns.step_coefficients(2, 0.25, 10.0)[:4] == (8.0, -2.0, 2.0, -1.0)
    with pytest.raises(ValueError):
        cdns.step_coefficients(0, 0.1, 10.0)


def test_bindings_reject_wrong_shapes_before_the_c_call():
    """Every array the Python host side hands to the C ABI has the shape the
    call reads: a wrong shape raises ValueError in the binding, before any
    library call (a short array would otherwise be read past its end)."""
    import sys
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "channel-dns_b200"))
    import cdns
    mesh = cdns.Mesh(16, 16, 16, 8, 14, 8, 24, 24, 24, 1.0, 1.0)
    c = cdns.Context._member(ctypes.c_void_p(), mesh, cdns.Params(Re=100.0, DT=1e-3), cdns.PRECISION_FP64)
    nkz, ncy, nkx = mesh.spectral_shape
    short = np.zeros((nkz, ncy, nkx - 1), dtype=np.complex128)
    short4 = np.zeros((nkz, ncy, nkx - 1, 3), dtype=np.complex128)
    good4 = np.zeros((nkz, ncy, nkx, 3), dtype=np.complex128)
    pbc = np.zeros((nkz, 2, nkx), dtype=np.complex128)
    vbc = np.zeros((nkz, 2, nkx, 3), dtype=np.complex128)
    calls = [
        lambda: c.set_velocity(short4),
        lambda: c.set_velocity_bc(vbc[:, :1]),
        lambda: c.set_pressure(short),
        lambda: c.nonlinear(short4),
        lambda: c.transform_fine("B", short),
        lambda: c.transform_fine("F", np.zeros((24, 24, 24))),
        lambda: c.transform_coarse("B", short),
        lambda: c.transform_coarse("F", np.zeros((16, 16, 16))),
        lambda: c.transform_coarse("X", short),
        lambda: c.solve(1.0, short4, pbc, vbc),
        lambda: c.solve(1.0, good4, pbc[:, :1], vbc),
        lambda: c.solve(1.0, good4, pbc, vbc[..., :2]),
        lambda: c.solve_adjoint(1.0, short, good4),
        lambda: c.solve_adjoint(1.0, None, short4),
        lambda: c.nonlinear_adjoint(short4, good4),
        lambda: c.nonlinear_adjoint(good4, short4),
        lambda: c.nonlinear_adjoint(good4, good4, pbc[:, :1]),
        lambda: c.adjoint_run(2, 1, weights=short4),
        lambda: c.adjoint_run(2, 1, control=vbc[:, :1]),
    ]
    for k, call in enumerate(calls):
        with pytest.raises(ValueError):
            call()
