"""Parity at the configuration the headline number is measured on: the Chung-Lu + planted-communities graph with
n = 2.4M, m = 62.4M (mean degree 52, exponent 2.3, max degree 1e5), 20,000 communities, r = 32, 5M wedge triples,
rows in the community order, evaluated in the FP64, FP32 and BF16 storage forms.

* FP64 form against the FP64 oracle (the C restatement of the reference's kernels) at the same V: value and G within
  1e-10 relative.
* FP32 and BF16 forms against the FP64 GPU form evaluated at the V they store (their rounding of V): value within
  1e-6 and G within 2e-5 relative (Frobenius), the tolerances of the smaller parity cases.
* With the production levels (one pair level of the communities capped at 6000 clusters, one VCS level on the
  neighbour pattern, 53M working-set entries) the BF16 form against the oracle at its stored V, same tolerances.
"""
import numpy as np
import pytest

from oracle import oracle as O
from _fixtures import rel

pytestmark = pytest.mark.gpu
RHO, TRI_W = 0.02, 1.0


@pytest.fixture(scope="module")
def c3():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from lagbound_b200 import Context, synth
    from lagbound_b200.problem import locality_order
    g = synth.config_graph("c3", seed=0, device="cuda:0")
    TI = synth.wedge_triples_torch(g, synth.CONFIG_TRIANGLES["c3"], seed=1, device="cuda:0")
    lam = synth.tri_multipliers(len(TI), seed=1)
    V = synth.random_V(g.n, 32, seed=0)
    ctx = Context(0)
    yield dict(g=g, TI=TI, lam=lam, V=V, order=locality_order(g.labels), ctx=ctx,
               inst=O.Instance(g.n, g.indptr, g.indices, g.data, g.d, g.L, g.C0))
    ctx.close()


def _problem(c, dtype):
    from lagbound_b200 import Problem
    g = c["g"]
    p = Problem(c["ctx"], g.n, g.indptr, g.indices, None, g.d, g.L, g.C0, 32, dtype, order=c["order"])
    p.set_triangles(c["TI"], c["lam"])
    return p


def test_c3_storage_forms(c3):
    g = c3["g"]
    assert g.n == 2_400_000 and g.nnz == 124_800_000 and len(c3["TI"]) == 5_000_000
    p64 = _problem(c3, "f64")
    p64.set_V(c3["V"])
    o64 = p64.eval(RHO, TRI_W, grad=True)
    ref = O.evaluate(c3["inst"], c3["V"], (), c3["TI"], c3["lam"], (), RHO, TRI_W, want_G=True)
    assert o64["value"] == pytest.approx(ref["value"], rel=1e-10)
    assert rel(p64.G(), ref["G"]) < 1e-10
    del ref
    for dtype in ("f32", "bf16"):
        p = _problem(c3, dtype)
        p.set_V(c3["V"])
        o = p.eval(RHO, TRI_W, grad=True)
        G = p.G()
        p64.set_V(p.get_V())
        os_ = p64.eval(RHO, TRI_W, grad=True)
        assert o["value"] == pytest.approx(os_["value"], rel=1e-6), dtype
        assert rel(G, p64.G()) < 2e-5, dtype
        assert o["quadA"] == pytest.approx(os_["quadA"], rel=1e-6) and o["gmin"] == pytest.approx(os_["gmin"], rel=1e-5)
        p.close()
    p64.close()


def test_c3_with_levels_against_oracle(c3):
    from lagbound_b200.stages.alm_vcs import capped_labels
    import scipy.sparse as sp
    g, V = c3["g"], c3["V"]
    rng = np.random.default_rng(7)
    w_pair = 0.03
    lab_p = capped_labels(g.labels, g.d, 6000, lambda *a: None, "pair level")
    P = int(lab_p.max()) + 1
    Lp = O.PairLevelData(lab_p, g.d, None, w_pair)
    W = sp.csr_matrix((g.d, (Lp.lab, np.arange(g.n))), shape=(P, g.n))
    Y = W @ V
    H = Y @ Y.T
    H[np.diag_indices(P)] -= Lp.dsq
    S = RHO * np.outer(Lp.rq, Lp.rq) * w_pair * np.abs(H) * rng.uniform(0, 3, (P, P)) * (rng.random((P, P)) < 0.6)
    Lp.sig = 0.5 * (S + S.T)
    del S, H, W
    lab_v = np.unique(g.labels, return_inverse=True)[1].astype(np.int64)
    rows = np.repeat(np.arange(g.n), np.diff(g.indptr))
    Pv = int(lab_v.max()) + 1
    keys = np.unique(np.concatenate([np.arange(g.n) * Pv + lab_v, rows * Pv + lab_v[g.indices]]))
    del rows
    vptr = np.zeros(g.n + 1, np.int64)
    np.cumsum(np.bincount(keys // Pv, minlength=g.n), out=vptr[1:])
    vcol = (keys % Pv).astype(np.int32)
    del keys
    vsig = rng.exponential(0.05, len(vcol)) * (rng.random(len(vcol)) < 0.5)
    Lv = O.VCSLevelData(lab_v, g.d, vptr, vcol, vsig)
    p = _problem(c3, "bf16")
    p.set_V(V)
    lid = p.add_pair_level(Lp.lab, P, w_pair)
    p.set_pair_sigma(lid, Lp.sig)
    m = p.add_vcs_level(lab_v, Pv, w_pair)
    p.set_vcs_ws(m, vptr, vcol, vsig)
    o = p.eval(RHO, TRI_W, grad=True)
    G = p.G()
    ref = O.evaluate(c3["inst"], p.get_V(), [Lp], c3["TI"], c3["lam"], [Lv], RHO, TRI_W, wv=w_pair, want_G=True)
    assert o["value"] == pytest.approx(ref["value"], rel=1e-6)
    assert rel(G, ref["G"]) < 2e-5
    assert o["nviol"] == int(ref["nviol"].sum()) and o["vcs_nviol"] == int(ref["vcs_nviol"].sum())
    p.close()
