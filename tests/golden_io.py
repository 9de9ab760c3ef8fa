"""Load the golden fixtures (tests/golden/*.npz) into oracle mesh/parameter objects."""
import os

import numpy as np

from oracle_cases import orc

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    d = dict(np.load(os.path.join(GOLDEN, name)))
    mm = [int(v) for v in d["mesh"]]
    m = orc.Mesh(*mm, float(d["dom"][0]), float(d["dom"][1]))
    pa = d["parm"]
    p = orc.Parm(Re=float(pa[0]), G_pre=float(pa[1]), a_pre0=float(pa[2]), b_pre0=float(pa[3]),
                 a_V=tuple(float(v) for v in pa[4:7]), b_V=tuple(float(v) for v in pa[7:10]),
                 INDEX_GRAD_PRE=int(pa[10]), THETA=float(pa[11]), DT=float(pa[12]),
                 V_Microblow0=float(pa[13]))
    return m, p, d
