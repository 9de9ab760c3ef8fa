"""cdns.load_config against the reference's config tests (tests/test_params.cpp:
ExampleTomlParameters, TomlRejectsMissingAndUnknownKeys, IntWithDecimalPointThrows,
MissingFileThrows), on a config.toml written here with the values of the
reference's examples/config.toml."""
import pytest

import cdns

EXAMPLE = """[mesh]
NX = 32
NY = 32
NZ = 32
INDEX_disturb_Z = 3
NXS = 16
NYS = 30
NZS = 16
NX2 = 32
NY2 = 32
NZ2 = 32
INDEX_Serial = 1

[parm]
XL = 1.0e1
ZL = 1.0e1
THETA = 0.0e0
INDEX_GRAD_PRE = 0
Re = 2.8e3
INDEX_UNSTEADY_BC = 0
G_pre = 0.0e0
a_pre0 = 0.0e0
b_pre0 = 1.0e0
a_V = [1.0e0, 1.0e0, 1.0e0]
b_V = [0.0e0, 0.0e0, 0.0e0]

[control]
INDEX_CONT = 0
EPS_init = 0.0e0
NSTEPS = 5
NDUMFRQ = 1
NPRNFRQ = 1
DT = 3.0e-3
NCOUNT_disturb = 0
NDISTURBFRQ = 300
EPS_disturb = 0.1e0
V_Microblow0 = 1.0e-3
Nstat = 50000

[output]
format = "ascii"
"""


def _write(tmp_path, text):
    (tmp_path / "config.toml").write_text(text)
    return str(tmp_path)


def test_example_parameters(tmp_path):
    """tests/test_params.cpp:153-168."""
    mesh, params, ctrl = cdns.load_config(_write(tmp_path, EXAMPLE))
    assert (mesh.NX, mesh.NY, mesh.NZ, mesh.NXS, mesh.NYS, mesh.NZS) == (32, 32, 32, 16, 30, 16)
    assert (mesh.NX2, mesh.NY2, mesh.NZ2) == (32, 32, 32)
    assert mesh.XL == 10.0 and mesh.ZL == 10.0
    assert params.Re == 2800.0 and params.DT == 0.003 and params.INDEX_GRAD_PRE == 0
    assert params.V_Microblow0 == 1e-3 and params.a_V == (1.0, 1.0, 1.0)
    assert ctrl["nsteps"] == 5 and ctrl["nstat"] == 50000
    assert ctrl["index_serial"] == 1 and ctrl["output_format"] == "ascii"


def test_keys_are_case_insensitive(tmp_path):
    mesh, params, _ = cdns.load_config(_write(tmp_path, EXAMPLE.replace("NXS = 16", "nxs = 16")
                                              .replace("Re = 2.8e3", "RE = 2.8e3")))
    assert mesh.NXS == 16 and params.Re == 2800.0


@pytest.mark.parametrize("mutate,message", [
    (lambda t: t + "typo = 1\n", "unknown TOML key"),                      # tests/test_params.cpp:170-176
    (lambda t: t.replace("NX = 32\n", ""), "integer required: mesh.NX"),    # :177-181
    (lambda t: t.replace("NX = 32", "NX = 32.0"), "integer required"),      # :122-133
    (lambda t: t.replace("a_V = [1.0e0, 1.0e0, 1.0e0]", "a_V = [1.0e0, 1.0e0]"), "three numbers"),
    (lambda t: t.replace("DT = 3.0e-3", "DT = nan"), "finite number required"),
    (lambda t: t.replace('format = "ascii"', 'format = "hdf5"'), "ascii, binary, or both"),
    (lambda t: t + "[extra]\nx = 1\n", "unknown TOML table"),
    (lambda t: t.replace("[control]", "[controls]"), "unknown TOML table"),
])
def test_rejects_bad_configs(tmp_path, mutate, message):
    with pytest.raises(ValueError, match=message):
        cdns.load_config(_write(tmp_path, mutate(EXAMPLE)))


def test_missing_file(tmp_path):
    """tests/test_params.cpp:135-137."""
    with pytest.raises(FileNotFoundError):
        cdns.load_config(str(tmp_path / "nowhere"))


def test_distributed_config_is_returned_for_pencil_ranks(tmp_path):
    mesh, _, ctrl = cdns.load_config(_write(tmp_path, EXAMPLE.replace("INDEX_Serial = 1", "INDEX_Serial = 0")))
    assert ctrl["index_serial"] == 0 and mesh.NXS == 16
