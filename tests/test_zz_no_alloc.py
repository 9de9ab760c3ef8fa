"""The allocation-free fine backward transform (cdns_transform_fine_backward_noalloc).

Some callers cannot let a library call cudaMalloc: they run under a memory
pool or an embedding framework that owns every device allocation, or in code
where an allocation would synchronise the device.  This entry point serves
them from a fixed array in device memory; here it is called through the C ABI
on caller-owned buffers and must reproduce the oracle's fine backward
transform (Transforms::channel_xyzfft2 'B', src/fft/transforms.cpp:687-741)
and the context-based transform (cdns_transform_fine 'B') within the
transform tolerance of the other GPU tests, on two calls in a row with
different inputs (the shared array keeps the previous call's contents), and
a call after the first must leave the device's free memory unchanged.  The
file sorts last so that a run stopping at the first failure has already run
every other test.
"""
import ctypes

import numpy as np
import pytest

import cdns
from oracle_cases import band_spectrum, channel_case, example_case, orc, retau180_case
from test_gpu_parity import ctx_for, rel_max

pytestmark = pytest.mark.gpu


def _mesh(m):
    return cdns.Mesh(m.NX, m.NY, m.NZ, m.NXS, m.NYS, m.NZS, m.NX2, m.NY2, m.NZ2, m.XL, m.ZL)


@pytest.mark.parametrize("case", ["channel48", "full_nyquist"])
def test_noalloc_matches_context_transform(case):
    import torch
    m, p = channel_case(32) if case == "channel48" else example_case()
    ctx = ctx_for(m, p)
    mesh = _mesh(m)
    stream = torch.cuda.current_stream()
    out = torch.empty(m.fine_shape(), dtype=torch.float64, device="cuda")
    for seed in (17, 18):
        U = band_spectrum(m, seed)
        ref = ctx.transform_fine("B", U)
        dev_in = torch.from_numpy(np.ascontiguousarray(U).view(np.float64).copy()).cuda()
        out.fill_(float("nan"))
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        cdns.fine_backward_noalloc(mesh, dev_in.data_ptr(), out.data_ptr(), stream.cuda_stream)
        torch.cuda.synchronize()
        if seed == 18:   # the first call may commit the array's memory (lazy module loading)
            assert torch.cuda.mem_get_info()[0] == free0
        got = out.cpu().numpy()
        assert np.isfinite(got).all()
        assert rel_max(got, ref) <= 1e-12
        assert rel_max(got, orc.fine_backward(m, U)) <= 1e-12


def test_noalloc_rejects_meshes_beyond_its_scratch():
    import torch
    m, _ = retau180_case()
    dev_in = torch.zeros(16, dtype=torch.float64, device="cuda")
    lib = cdns.lib()
    md = _mesh(m).desc()
    code = lib.cdns_transform_fine_backward_noalloc(ctypes.byref(md), ctypes.c_void_p(dev_in.data_ptr()),
                                                    ctypes.c_void_p(dev_in.data_ptr()), None)
    assert code == 1
    buf = ctypes.create_string_buffer(512)
    lib.cdns_last_error(buf, 512)
    assert b"at most" in buf.value


def test_noalloc_alternating_meshes():
    """Calls alternating between two meshes: each call with a mesh other than
    the previous call's rebuilds the tables in the shared array."""
    import torch
    stream = torch.cuda.current_stream()
    cases = [channel_case(32), example_case(), channel_case(32)]
    for i, (m, p) in enumerate(cases):
        U = band_spectrum(m, 40 + i)
        dev_in = torch.from_numpy(np.ascontiguousarray(U).view(np.float64).copy()).cuda()
        out = torch.full(m.fine_shape(), float("nan"), dtype=torch.float64, device="cuda")
        cdns.fine_backward_noalloc(_mesh(m), dev_in.data_ptr(), out.data_ptr(), stream.cuda_stream)
        torch.cuda.synchronize()
        assert rel_max(out.cpu().numpy(), orc.fine_backward(m, U)) <= 1e-12
