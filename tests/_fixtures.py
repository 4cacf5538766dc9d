"""Loaders for the golden fixtures (tests/golden/*.npz, written by tests/golden/make_golden.py from the reference)."""
import glob
import os

import numpy as np

from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def eval_names():
    return sorted(os.path.basename(p)[5:-4] for p in glob.glob(os.path.join(GOLDEN, "eval_*.npz")))


def sep_names():
    return sorted(os.path.basename(p)[4:-4] for p in glob.glob(os.path.join(GOLDEN, "sep_*.npz")))


def reduce_names():
    return sorted(os.path.basename(p)[7:-4] for p in glob.glob(os.path.join(GOLDEN, "reduce_*.npz")))


def graph_names():
    return sorted(os.path.basename(p)[6:-4] for p in glob.glob(os.path.join(GOLDEN, "graph_*.npz")))


class EvalCase:
    """An eval_<name>.npz fixture as oracle objects: instance, V, levels, triangles and the reference outputs."""

    def __init__(self, name):
        z = np.load(os.path.join(GOLDEN, f"eval_{name}.npz"))
        self.z = z
        self.name = name
        self.inst = O.Instance(int(z["n"]), z["indptr"], z["indices"], z["data"], z["d"], float(z["L"]), float(z["C0"]))
        self.V = z["V"]
        self.TI = z["TI"]; self.lam = z["lam"]
        self.rho = float(z["rho"]); self.tri_weight = float(z["tri_weight"])
        self.w_pair = float(z["w_pair"]); self.wv = float(z["vc_weight"]) * self.w_pair
        self.plev = []
        for li in range(int(z["npl"])):
            Lv = O.PairLevelData(z[f"plab{li}"], self.inst.d, z[f"psig{li}"], self.w_pair)
            assert np.allclose(Lv.rq, z[f"prq{li}"], rtol=0, atol=0)
            self.plev.append(Lv)
        self.vlev = []
        for m in range(int(z["nvl"])):
            Lv = O.VCSLevelData(z[f"vlab{m}"], self.inst.d, z[f"vptr{m}"], z[f"vcol{m}"], z[f"vsig{m}"])
            assert np.array_equal(Lv.own, z[f"vown{m}"])
            self.vlev.append(Lv)

    def __getitem__(self, key):
        return self.z[key]


def rel(a, b):
    a = np.asarray(a, np.float64); b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def vsep_names():
    return sorted(os.path.basename(p)[5:-4] for p in glob.glob(os.path.join(GOLDEN, "vsep_*.npz")))
