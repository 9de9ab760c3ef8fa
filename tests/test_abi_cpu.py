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
