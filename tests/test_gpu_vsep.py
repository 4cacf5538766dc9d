"""GPU VCS working-set separation against the reference's own separate() outputs (golden) and the oracle.

The GPU forms v_i . Y_R in FP64 in a fixed order, the reference with BLAS: scores agree to rounding (1e-12
relative) and the selected sets are identical unless a score lies within rounding of the cut-off, which the seeded
cases here do not have."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from _fixtures import GOLDEN, vsep_names

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from lagbound_b200 import Context
    c = Context(0)
    yield c
    c.close()


def ring_problem(ctx, d, r, dtype, order=None):
    """A problem whose graph is a ring (separation reads only d, V and the level)."""
    from lagbound_b200 import Problem
    n = len(d)
    idx = np.stack([(np.arange(n) - 1) % n, (np.arange(n) + 1) % n], 1)
    idx.sort(1)
    indptr = np.arange(0, 2 * n + 1, 2, dtype=np.int64)
    return Problem(ctx, n, indptr, idx.reshape(-1), None, d, float(d.sum()), 0.0, r, dtype=dtype, order=order)


def _check_same(rows, cols, sc, rows_ref, cols_ref, sc_ref):
    o = np.lexsort((cols, rows))
    assert np.array_equal(rows[o], rows_ref) and np.array_equal(cols[o], cols_ref)
    assert np.allclose(sc[o], sc_ref, rtol=1e-12, atol=0)


@pytest.mark.parametrize("name", vsep_names())
def test_vcs_separation_matches_reference(ctx, name):
    from lagbound_b200.vcs import merge_working_set
    z = np.load(os.path.join(GOLDEN, f"vsep_{name}.npz"))
    V = z["V"]; d = z["d"]
    p = ring_problem(ctx, d, V.shape[1], "f64")
    p.set_V(V)
    lv = p.add_vcs_level(z["lab"], wv=float(z["wv"]))
    p.set_vcs_ws(lv, z["ptr"], z["col"], z["sig"], z["age"])
    P = int(z["lab"].max()) + 1
    for c in range(int(z["ncase"])):
        rows, cols, sc, st = p.vcs_separate(lv, int(z[f"nadd{c}"]), float(z[f"tol{c}"]), str(z[f"mode{c}"]))
        _check_same(rows, cols, sc, z[f"rows{c}"], z[f"cols{c}"], z[f"scores{c}"])
        assert np.all(np.diff(sc) <= 0)                            # best first
        ref = z[f"stats{c}"]
        assert st["nviol"] == ref[0] and st["nviol_ws"] == ref[2]
        assert st["mass"] == pytest.approx(ref[1], rel=1e-11) and st["mass_ws"] == pytest.approx(ref[3], rel=1e-11)
        if c == 0:
            keep = z["age"] < int(z["vcs_drop"])
            m = merge_working_set(len(d), P, z["ptr"], z["col"], z["sig"], z["age"], keep, rows, cols)
            for k_, got in zip(("m_ptr", "m_col", "m_sig", "m_age"), m):
                assert np.array_equal(got, z[k_]), k_
            # the merged working set round-trips through the device
            p.set_vcs_ws(lv, *m)
            sig2, age2 = p.get_vcs_ws(lv)
            assert np.array_equal(sig2, m[2]) and np.array_equal(age2, m[3])
            p.set_vcs_ws(lv, z["ptr"], z["col"], z["sig"], z["age"])     # the next cases start from the fixture's
    p.close()


def random_case(n, P, k, seed, ws_per_row=3):
    rng = np.random.default_rng(seed)
    d = rng.integers(1, 40, n).astype(np.float64)
    V = rng.standard_normal((n, k)); V /= np.linalg.norm(V, axis=1, keepdims=True)
    lab = rng.integers(0, P, n); lab[:P] = np.arange(P)
    cols = [np.unique(np.r_[lab[i], rng.integers(0, P, ws_per_row)]) for i in range(n)]
    ptr = np.r_[0, np.cumsum([len(c) for c in cols])].astype(np.int64)
    col = np.concatenate(cols).astype(np.int32)
    return d, V, lab, ptr, col


@pytest.mark.parametrize("dtype", ["f64", "f32", "bf16"])
@pytest.mark.parametrize("mode,nadd", [("pen", 5000), ("mean", 10 ** 7), ("mass", 777)])
def test_vcs_separation_matches_oracle(ctx, dtype, mode, nadd):
    """Stored V in each dtype (the oracle runs on the stored values); locality order on for the reduced forms."""
    n, P, k = 6000, 150, 24
    d, V, lab, ptr, col = random_case(n, P, k, seed=10 * ["f64", "f32", "bf16"].index(dtype) + len(mode) + nadd % 7)
    order = None if dtype == "f64" else np.argsort(lab, kind="stable")
    p = ring_problem(ctx, d, k, dtype, order=order)
    p.set_V(V)
    Vs = p.get_V()                                     # the stored values, in FP64
    lv = p.add_vcs_level(lab, wv=0.3)
    p.set_vcs_ws(lv, ptr, col, np.zeros(len(col)))
    rows, cols, sc, st = p.vcs_separate(lv, nadd, 1e-4, mode)
    r_o, c_o, s_o, st_o = O.vcs_separate(Vs, d, lab, ptr, col, 0.3, nadd, 1e-4, mode)
    o = np.lexsort((c_o, r_o))
    _check_same(rows, cols, sc, r_o[o], c_o[o], s_o[o])
    assert st["nviol"] == st_o[0] and st["nviol_ws"] == st_o[2]
    assert st["mass"] == pytest.approx(st_o[1], rel=1e-10)
    p.close()


def test_vcs_separation_selects_across_many_candidates(ctx):
    """More candidates than fit one radix bin (the refinement passes run): the cut equals the oracle's."""
    n, P, k = 20000, 400, 8
    d, V, lab, ptr, col = random_case(n, P, k, seed=5, ws_per_row=1)
    p = ring_problem(ctx, d, k, "f64")
    p.set_V(V)
    lv = p.add_vcs_level(lab, wv=1.0)
    p.set_vcs_ws(lv, ptr, col, np.zeros(len(col)))
    for nadd in (1, 1000, 123457):
        rows, cols, sc, st = p.vcs_separate(lv, nadd, 1e-4, "pen")
        r_o, c_o, s_o, st_o = O.vcs_separate(V, d, lab, ptr, col, 1.0, nadd, 1e-4, "pen")
        assert len(rows) == min(nadd, int(st_o[0] - st_o[2]))
        o = np.lexsort((c_o, r_o))
        _check_same(rows, cols, sc, r_o[o], c_o[o], s_o[o])
    rows, cols, sc, st = p.vcs_separate(lv, 0, 1e-4, "pen")
    assert len(rows) == 0 and st["nviol"] > 0
    p.close()
