"""The benchmark configurations as parity cases (the bench line itself runs the n = 2.4M configuration):

  C1  planted SBM n = 2000, r = 16, 20,000 triples, pair and VCS level = planted blocks, FP64 V
  C2  Chung-Lu + communities n = 300,000, r = 32, 1M triples, one pair level (communities) and one VCS level
      (working set = the neighbour pattern), FP64, FP32 and BF16 V
  C4  a batch of graphs (n log-uniform in [500, 50,000], mean degree 5-40, SBM / Chung-Lu alternating,
      r in {8, 16, 32}, 10 n triples), FP32 V
  C5  request-sized Chung-Lu graphs (n 1,000 to 100,000, mean degree 8-50, r 16-32), BF16 V

Every evaluation (value, dual residuals, G) is compared with the FP64 oracle at the stored V: FP64 form 1e-10
(value) and 1e-11 (G) relative, reduced forms 1e-6 (value) and 2e-5 (G)."""
import numpy as np
import pytest

from oracle import oracle as O
from _fixtures import rel

pytestmark = pytest.mark.gpu
RHO, TRI_W, W_PAIR, VC_W = 0.02, 1.0, 0.3, 1.0


@pytest.fixture(scope="module")
def ctx():
    from lagbound_b200 import Context
    c = Context(0)
    yield c
    c.close()


def neighbour_pattern(g, lab):
    """VCS working set: for every row its own cluster and the clusters of its neighbours (aggops.neighbour_pattern)."""
    rows = np.repeat(np.arange(g.n), np.diff(g.indptr))
    keys = np.unique(np.concatenate([np.arange(g.n) * (lab.max() + 1) + lab, rows * (lab.max() + 1) + lab[g.indices]]))
    P = lab.max() + 1
    r, c = keys // P, keys % P
    ptr = np.zeros(g.n + 1, np.int64)
    np.cumsum(np.bincount(r, minlength=g.n), out=ptr[1:])
    return ptr, c.astype(np.int32)


def build_case(g, r, T, seed, pair=True, vcs=True):
    """Instance, V, levels with multipliers on the PHR scale of V (as the solver's would be), triangles."""
    from lagbound_b200 import synth
    rng = np.random.default_rng(seed)
    inst = O.Instance(g.n, g.indptr, g.indices, g.data, g.d, g.L, g.C0)
    V = synth.random_V(g.n, r, seed=seed)
    lab = np.unique(g.labels, return_inverse=True)[1]
    plev, vlev = [], []
    if pair:
        Lv = O.PairLevelData(lab, g.d, None, W_PAIR)
        Y = np.zeros((Lv.P, r)); np.add.at(Y, Lv.lab, g.d[:, None] * V)
        H = Y @ Y.T; H[np.diag_indices(Lv.P)] -= Lv.dsq
        rqq = np.outer(Lv.rq, Lv.rq) * W_PAIR
        S = RHO * rqq * np.abs(H) * rng.uniform(0, 3, H.shape) * (rng.random(H.shape) < 0.6)
        Lv.sig = 0.5 * (S + S.T)
        plev.append(Lv)
    if vcs:
        ptr, col = neighbour_pattern(g, lab)
        rows = np.repeat(np.arange(g.n), np.diff(ptr))
        L0 = O.VCSLevelData(lab, g.d, ptr, col, np.zeros(len(col)))
        Y = np.zeros((L0.P, r)); np.add.at(Y, L0.lab, g.d[:, None] * V)
        s_ = np.einsum("ij,ij->i", V[rows], Y[col])
        dd = g.d[rows]
        gg = dd * (s_ - np.where(col == L0.lab[rows], dd, 0.0))
        rr = W_PAIR * VC_W * L0.rq[col] / dd ** 2
        sig = RHO * rr * np.abs(gg) * rng.uniform(0, 3, len(col)) * (rng.random(len(col)) < 0.5)
        vlev.append(O.VCSLevelData(lab, g.d, ptr, col, sig))
    TI = synth.wedge_triples(g, T, seed=seed + 1) if T else np.zeros((0, 3), np.int64)
    lam = synth.tri_multipliers(len(TI), seed=seed + 1)
    return inst, V, plev, vlev, TI, lam


def run_case(ctx, inst, V, plev, vlev, TI, lam, dtype, order=None):
    from lagbound_b200 import Problem
    w = None if np.all(inst.data == 1.0) else inst.data
    p = Problem(ctx, inst.n, inst.indptr, inst.indices, w, inst.d, inst.L, inst.C0, V.shape[1], dtype, order=order)
    p.set_V(V)
    for Lv in plev:
        lid = p.add_pair_level(Lv.lab, Lv.P, Lv.w)
        p.set_pair_sigma(lid, Lv.sig)
    for Lv in vlev:
        m = p.add_vcs_level(Lv.lab, Lv.P, W_PAIR * VC_W)
        p.set_vcs_ws(m, Lv.ptr, Lv.col, Lv.sig)
    if len(TI):
        p.set_triangles(TI, lam)
    out = p.eval(RHO, TRI_W, grad=True)
    Vs = p.get_V()
    G = p.G()
    p.close()
    ref = O.evaluate(inst, Vs, plev, TI, lam, vlev, RHO, TRI_W, W_PAIR * VC_W)
    return out, G, ref


def check(out, G, ref, dtype):
    scale = max(abs(ref["value"]), abs(ref["primal"]), 1.0)
    tv, tg = (1e-10, 1e-11) if dtype == "f64" else (1e-6, 2e-5)
    assert abs(out["value"] - ref["value"]) / scale < tv
    assert abs(out["primal"] - ref["primal"]) / scale < tv
    assert rel(G, ref["G"]) < tg
    assert out["nviol"] == int(np.sum(ref["nviol"]))
    assert out["vcs_nviol"] == int(np.sum(ref["vcs_nviol"]))


def test_c1_sbm_2000(ctx):
    from lagbound_b200 import synth
    g = synth.config_graph("c1", seed=0)
    case = build_case(g, 16, 20_000, seed=1)
    out, G, ref = run_case(ctx, *case, "f64")
    check(out, G, ref, "f64")


@pytest.fixture(scope="module")
def c2_case():
    from lagbound_b200 import synth
    g = synth.config_graph("c2", seed=0)
    return g, build_case(g, 32, 1_000_000, seed=2)


@pytest.mark.parametrize("dtype", ["f64", "f32", "bf16"])
def test_c2_chung_lu_300k(ctx, c2_case, dtype):
    from lagbound_b200.problem import locality_order
    g, case = c2_case
    order = None if dtype == "f64" else locality_order(g.labels)
    out, G, ref = run_case(ctx, *case, dtype, order=order)
    check(out, G, ref, dtype)


def test_c4_batch_of_graphs(ctx):
    from lagbound_b200 import synth
    rng = np.random.default_rng(4)
    for k in range(6):
        n = int(np.exp(rng.uniform(np.log(500), np.log(50_000))))
        mean = float(rng.uniform(5, 40))
        r = int(rng.choice([8, 16, 32]))
        if k % 2 == 0 and n <= 6000:                    # the dense-pair SBM generator is for small n
            blocks = max(2, n // 250)
            p_in = min(0.5, mean * 0.8 / (n / blocks))
            p_out = mean * 0.2 / n
            g = synth.sbm(n, blocks, p_in, p_out, seed=k)
        else:
            g = synth.chung_lu_communities(n, mean, 2.3, max(50, n // 10), max(2, n // 120), 0.25, seed=k)
        case = build_case(g, r, 10 * g.n, seed=10 + k, pair=True, vcs=(k % 3 == 0))
        out, G, ref = run_case(ctx, *case, "f32")
        check(out, G, ref, "f32")


def test_c5_request_sized_graphs(ctx):
    from lagbound_b200 import synth
    from lagbound_b200.problem import locality_order
    for k, (n, mean, r) in enumerate([(1000, 8.0, 16), (20_000, 30.0, 24), (100_000, 50.0, 32)]):
        g = synth.chung_lu_communities(n, mean, 2.2, n // 10, max(2, n // 100), 0.3, seed=20 + k)
        case = build_case(g, r, 5 * g.n, seed=30 + k)
        out, G, ref = run_case(ctx, *case, "bf16", order=locality_order(g.labels))
        check(out, G, ref, "bf16")
