"""bench.py's algorithmic-bytes model at Re_tau180 (the numerator of the
roofline key): 16 B per complex value, each stage reading and writing its
operands once, with Ns = 1,064,895, Ny = 1,618,305 and Nz = 2,458,820."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_stage_bytes_at_retau180():
    mesh, _ = bench.workload_mesh()
    nkx, nkz, ncy, ny2 = mesh.NXS + 1, 2 * mesh.NZS + 1, mesh.NYS + 1, mesh.NY2 + 1
    Ns, Ny, Nz = nkz * ncy * nkx, nkz * ny2 * nkx, mesh.NZ2 * ny2 * nkx
    assert (Ns, Ny, Nz) == (1_064_895, 1_618_305, 2_458_820)
    sb = bench.stage_bytes(mesh)
    mb = {k: round(v / 1e6, 1) for k, v in sb.items()}
    assert mb == {"curl": 102.2, "y_synthesis": 257.6, "z_backward": 391.4, "x_cross": 354.1,
                  "z_forward": 195.7, "y_analysis": 128.8, "solve": 494.1}
    assert round(bench.step_bytes_model(mesh) / 1e6, 1) == 1923.9


def test_measured_peak_is_positive():
    peak, source = bench.measured_peak()
    assert peak > 1000.0 and isinstance(source, str)
