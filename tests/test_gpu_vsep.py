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


@pytest.mark.parametrize("name", vsep_names())
def test_vcs_grow_matches_reference_update(ctx, name):
    """Drop + separate + update_ws on the device gives the reference's merged working set (golden, case 0)."""
    z = np.load(os.path.join(GOLDEN, f"vsep_{name}.npz"))
    p = ring_problem(ctx, z["d"], z["V"].shape[1], "f64")
    p.set_V(z["V"])
    lv = p.add_vcs_level(z["lab"], wv=float(z["wv"]))
    p.set_vcs_ws(lv, z["ptr"], z["col"], z["sig"], z["age"])
    drop = int(z["vcs_drop"])
    dropped, added, st = p.vcs_grow(lv, int(z["nadd0"]), float(z["tol0"]), str(z["mode0"]), drop_age=drop)
    assert dropped == int((z["age"] >= drop).sum()) and added == len(z["rows0"])
    ptr, col = p.get_vcs_structure(lv)
    sig, age = p.get_vcs_ws(lv)
    assert np.array_equal(ptr, z["m_ptr"]) and np.array_equal(col, z["m_col"])
    assert np.array_equal(sig, z["m_sig"]) and np.array_equal(age, z["m_age"])
    assert st["nviol"] == z["stats0"][0] and st["nviol_ws"] == z["stats0"][2]
    p.close()


def _grid_problem(ctx, n, k, dtype, order, seed):
    """A problem with a real graph (ring plus random chords) so the evaluation exercises the VCS terms."""
    from lagbound_b200 import Problem
    rng = np.random.default_rng(seed)
    u = np.r_[np.arange(n), rng.integers(0, n, 3 * n)]
    v = np.r_[(np.arange(n) + 1) % n, rng.integers(0, n, 3 * n)]
    keep = u != v
    keys = np.unique(np.minimum(u, v)[keep] * n + np.maximum(u, v)[keep])
    a, b = keys // n, keys % n
    rows = np.r_[a, b]; cols = np.r_[b, a]
    o = np.lexsort((cols, rows))
    indptr = np.zeros(n + 1, np.int64); np.cumsum(np.bincount(rows, minlength=n), out=indptr[1:])
    d = np.diff(indptr).astype(np.float64)
    return Problem(ctx, n, indptr, cols[o], None, d, float(d.sum()), 0.0, k, dtype=dtype, order=order), d


@pytest.mark.parametrize("dtype,permute", [("f64", False), ("f32", True), ("bf16", True)])
def test_vcs_grow_matches_host_update(ctx, dtype, permute):
    """Rounds of the device update against separate + host merge + set_vcs_ws on a twin problem: the same working
    set, the same ages after multiplier updates and bit-identical evaluations (the column views agree)."""
    from lagbound_b200.vcs import merge_working_set
    n, P, k = 5000, 120, 16
    rng = np.random.default_rng(7)
    lab = rng.integers(0, P, n); lab[:P] = np.arange(P)
    order = np.argsort(lab, kind="stable") if permute else None
    V = rng.standard_normal((n, k)); V /= np.linalg.norm(V, axis=1, keepdims=True)
    cols = [np.unique(np.r_[lab[i], rng.integers(0, P, 2)]) for i in range(n)]
    ptr = np.r_[0, np.cumsum([len(c) for c in cols])].astype(np.int64)
    col = np.concatenate(cols).astype(np.int32)
    sig = np.where(rng.random(len(col)) < 0.5, 0.0, rng.random(len(col)))
    age = rng.integers(0, 4, len(col)).astype(np.uint8)
    probs = []
    for _ in range(2):
        p, d = _grid_problem(ctx, n, k, dtype, order, seed=3)
        p.set_V(V)
        p.set_light_threshold(256)          # the same row schedule on both (the autotune times the candidates)
        lv = p.add_vcs_level(lab, wv=0.5)
        p.set_vcs_ws(lv, ptr, col, sig, age)
        probs.append(p)
    dev, host = probs
    hptr, hcol = ptr, col
    for rnd, (nadd, drop, vmax) in enumerate([(3000, 3, 10 ** 9), (2000, 2, 10 ** 9), (500, 0, 16000),
                                              (800, 3, 1)]):
        for p in probs:
            p.eval(0.05, 1.0, grad=False)
            p.multiplier_update()
        s_, a_ = host.get_vcs_ws(0)
        keep = (a_ < drop) if drop > 0 else np.ones(len(a_), bool)
        room = max(0, vmax - int(keep.sum()))
        ni, nR, _, st_h = host.vcs_separate(0, max(1, min(nadd, room)), 1e-4, "pen")
        if room == 0:
            ni, nR = ni[:0], nR[:0]
        m = merge_working_set(n, P, hptr, hcol, s_, a_, keep, ni, nR)
        host.set_vcs_ws(0, *m)
        hptr, hcol = m[0], m[1]
        dropped, added, st_d = dev.vcs_grow(0, nadd, 1e-4, "pen", drop_age=drop, max_nnz=vmax)
        assert (dropped, added) == (len(keep) - int(keep.sum()), len(ni)), rnd
        assert st_d["nviol"] == st_h["nviol"] and st_d["nviol_ws"] == st_h["nviol_ws"]
        # the masses are FP64 sums whose block order varies from run to run
        assert st_d["mass"] == pytest.approx(st_h["mass"], rel=1e-12)
        assert st_d["mass_ws"] == pytest.approx(st_h["mass_ws"], rel=1e-12)
        dptr, dcol = dev.get_vcs_structure(0)
        assert np.array_equal(dptr, hptr) and np.array_equal(dcol, hcol), rnd
        for x, y in zip(dev.get_vcs_ws(0), host.get_vcs_ws(0)):
            assert np.array_equal(x, y), rnd
        e_d = dev.eval(0.05, 1.0, grad=True); e_h = host.eval(0.05, 1.0, grad=True)
        for key in e_h:   # sums over rows: the dynamic row schedule orders the block partials run by run
            assert np.allclose(np.asarray(e_d[key]), np.asarray(e_h[key]), rtol=1e-13, atol=0), (rnd, key)
        assert np.array_equal(dev.G(), host.G()), rnd
        assert np.array_equal(dev.vcs_ppv(0)[0], host.vcs_ppv(0)[0]), rnd
    for p in probs:
        p.close()
