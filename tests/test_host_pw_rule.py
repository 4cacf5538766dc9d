"""The pair weight of --pw_rule and the phase-2 switch against the reference's own code.

tests/golden/pw_sbm900.npz holds, at a fixed V and two pair levels, the reference's mobility ratio
(src/lagbound/_core/alm_vcs.py:1625-1641), the weight its --pw_rule block sets (alm_vcs.py:1643-1653) for five rule
strings, and the outer iteration and weight of its phase-2 switch (alm_vcs.py:1663-1667), all executed from the
reference file by tests/golden/make_golden.py.  The stage restates them in lagbound_b200/stages/alm_vcs.py
(mobility_ratio_from, pair_weight_rule, phase2_due, phase2_weight).
"""
import os
import types

import numpy as np
import pytest

from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden", "pw_sbm900.npz")


def _fixture():
    from lagbound_b200.stages.alm_vcs import Level
    f = np.load(GOLD, allow_pickle=False)
    inst = O.Instance(int(f["n"]), f["indptr"], f["indices"], f["data"], f["d"], float(f["L"]))
    levels = [Level(np.unique(f[f"lab{li}"], return_inverse=True)[1], inst.d) for li in range(int(f["nlev"]))]
    return f, inst, levels


def _args(f, rule):
    return types.SimpleNamespace(pw_rule=rule, rho=float(f["rho"]), phase2_at=0.0,
                                 phase2_at_it=int(f["phase2_at_it"]), phase2_w=float(f["phase2_w"]))


def test_pw_rule_weight_and_phase2_switch_match_reference():
    from lagbound_b200.stages.alm_vcs import mobility_ratio_from, pair_weight_rule, phase2_due, phase2_weight
    f, inst, levels = _fixture()
    V = f["V"]
    gB = np.linalg.norm(O.apply_C(inst, V), axis=1)           # |(B V)_i| in FP64 (the oracle's A V - d d^T V / L)
    R0 = mobility_ratio_from(gB, inst.d, V, levels, float(f["rho"]), float(f["w0"]))
    rules = [str(r) for r in f["rules"]]
    assert len(rules) == 5
    kinds = set()
    for c, rule in enumerate(rules):
        assert R0 == pytest.approx(float(f[f"R0_{c}"]), rel=1e-12)
        a = _args(f, rule)
        w, msg = pair_weight_rule(rule, R0, float(f["w0"]), a.rho, inst.n, inst.L)
        kinds.add(msg.rsplit("(", 1)[1].rstrip(")"))
        assert w == pytest.approx(float(f[f"w_auto_{c}"]), rel=1e-12), rule
        switched = None
        for it in range(1, int(f["outer"]) + 1):
            if switched is None and phase2_due(a, it, 0.0):
                switched = it
        assert switched == int(f[f"switch_it_{c}"]), rule
        assert phase2_weight(a, w) == pytest.approx(float(f[f"w_phase2_{c}"]), rel=1e-12), rule
    assert kinds == {"mob", "step"}          # both arms of the rule's minimum are exercised


def test_phase2_without_rule_and_by_time():
    from lagbound_b200.stages.alm_vcs import phase2_due, phase2_weight
    a = types.SimpleNamespace(phase2_at=30.0, phase2_at_it=0, phase2_w=0.2)
    assert phase2_weight(a, None) == 0.2
    assert not phase2_due(a, 100, 29.0) and phase2_due(a, 1, 31.0)
    a = types.SimpleNamespace(phase2_at=0.0, phase2_at_it=0, phase2_w=0.2)
    assert not any(phase2_due(a, it, 1e9) for it in range(1, 50))


@pytest.mark.gpu
def test_mobility_ratio_on_gpu_matches_reference():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from lagbound_b200 import Context
    from lagbound_b200.stages.alm_vcs import mobility_ratio
    f, inst, levels = _fixture()
    ctx = Context(0)
    try:
        d = dict(n=inst.n, indptr=inst.indptr, indices=inst.indices, weights=None, d=inst.d, L=inst.L, C0=0.0)
        R0 = mobility_ratio(ctx, d, f["V"], levels, float(f["rho"]), float(f["w0"]))
    finally:
        ctx.close()
    assert R0 == pytest.approx(float(f["R0_0"]), rel=1e-10)
