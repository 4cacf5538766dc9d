"""The GPU stages as a drop-in for the reference's solve and estimate stages, accepted by the reference's own
certificate chain and verifier, on the reference tests' graphs (tests/test_bounds.py of the reference: karate
optimum <= U < 0.44; Les Miserables 72259/129032 <= U < 0.58) and on the planted SBM of n = 2000 (8 blocks, p_in
0.08, p_out 0.002; its planted partition's modularity is a lower bound, U must stay above it).

The fixtures under tests/golden/dropin/<graph>/ were made in two steps:

1. on a B200, the GPU stages (reduction, main phase, proximal phase, estimates of both checkpoints; the pipeline's
   flags, api.py:224-270):
       python -m lagbound_b200.stages.workflow --workdir W --graph karate --time 30 --polish_time 60 --eig_time 60
       python -m lagbound_b200.stages.workflow --workdir W --graph lesmis --time 60 --polish_time 60 --eig_time 60
       python -m lagbound_b200.stages.workflow --workdir W --n 2000 --time 90 --polish_time 120 --eig_time 120
   (summary.json, runs/est_*.json, runs/proximal_last.npz, data/keys.npy and data/partition.npy: the input);
2. on CPU, where the reference is importable, its repair, estimate, repair, sparse lifted certificate and
   independent verification (api.py:272-298) on that workspace:
       LAGBOUND_REF=<reference root> python oracle/reference_chain.py W --polish_time 120 --eig_time 120
   (--polish_time 300 --eig_time 300 for the SBM; its checkpoint is not kept here, it holds 718k triangles)
   (reference_chain.json, runs/cert_est.json, runs/certificate.json, runs/verify.json; the certificate and verifier
   order their factorizations with the RCM stand-in for the absent pymetis), and again with this library's nested
   dissection as their pymetis (--ordering nd: reference_chain_nd.json).

tests/golden/dropin/c1_precision/<form>/ holds the same two steps for the SBM at two storage precisions of V
(step 1 with --vdtype f64, and with --vdtype bf16 --proximal_vdtype f32; step 2 with --ckpt runs/proximal_last.npz
--polish_time 300 --eig_time 300 --ordering nd); the instance files are the c1 fixture's.

The verifier alone decides validity; these tests check its decision and the bounds' brackets.
"""
import json
import os
from fractions import Fraction

import numpy as np
import pytest

HERE = os.path.join(os.path.dirname(__file__), "golden", "dropin")
KARATE_OPT = 0.4197896120973044
LESMIS_OPT = 72259 / 129032


def _load(graph, name):
    with open(os.path.join(HERE, graph, name)) as fh:
        return json.load(fh)


def _modularity(graph):
    g = _load(graph, "data/graph.json")
    n = int(g["n"])
    keys = np.load(os.path.join(HERE, graph, "data", "keys.npy"))
    lab = np.load(os.path.join(HERE, graph, "data", "partition.npy"))
    u, v = keys // n, keys % n
    m = len(keys)
    vol = np.bincount(lab, weights=np.bincount(np.r_[u, v], minlength=n)).astype(np.int64)
    return Fraction(int((lab[u] == lab[v]).sum()), m) - Fraction(sum(int(x) ** 2 for x in vol), 4 * m * m)


CASES = [("karate", KARATE_OPT, 0.44), ("lesmis", LESMIS_OPT, 0.58), ("c1", 0.7266864064952987, 0.7275)]


@pytest.mark.parametrize("graph,lo,hi", CASES)
def test_gpu_stages_certified_and_verified_by_the_reference(graph, lo, hi):
    s = _load(graph, "summary.json")
    chain = _load(graph, "reference_chain.json")
    ver = _load(graph, "runs/verify.json")
    assert s["graph"] == {"c1": "sbm"}.get(graph, graph) and s["best"] in s["estimates"]
    # the starting partition's exact modularity (a lower bound) as the workflow recorded it
    assert abs(float(_modularity(graph)) - s["planted_modularity"]) < 1e-15
    # the GPU estimate of the certified checkpoint brackets the optimum
    assert lo <= s["estimate"] < hi
    # the reference chain certified the GPU stages' checkpoint and its verifier accepted it
    assert chain["ckpt"] == os.path.join("runs", os.path.basename(s["best_ckpt"]))
    assert chain["verified"] is True and ver["passed"] is True
    # runs/verify.json is the last chain's result (the RCM run's, or the nested-dissection run's where it came last)
    runs = [chain] + ([_load(graph, "reference_chain_nd.json")]
                      if os.path.exists(os.path.join(HERE, graph, "reference_chain_nd.json")) else [])
    assert any(abs(ver["UB"] - c["verified_UB"]) <= 1e-12 * abs(c["verified_UB"]) for c in runs)
    assert lo <= chain["verified_UB"] < hi
    assert chain["verified_UB"] >= chain["gpu_estimate"] - 1e-9   # certification only loosens the estimate
    assert abs(chain["cpu_cert_estimate"] - chain["gpu_estimate"]) < 1e-6
    ck_path = os.path.join(HERE, graph, chain["ckpt"])
    if os.path.exists(ck_path):
        ck = np.load(ck_path)
        for key in ("TI", "lam", "V", "nlev"):                   # the checkpoint schema alm_vcs.py:1576-1589 writes
            assert key in ck.files


@pytest.mark.parametrize("graph,lo,hi", CASES)
def test_nested_dissection_in_the_reference_certificate(graph, lo, hi):
    rcm = _load(graph, "reference_chain.json")
    nd = _load(graph, "reference_chain_nd.json")
    cert = _load(graph, "runs/certificate.json")
    assert nd["ordering"] == "nd" and nd["verified"] is True and lo <= nd["verified_UB"] < hi
    assert abs(nd["verified_UB"] - rcm["verified_UB"]) < 1e-8           # the ordering only changes the fill
    rcm_fill = rcm.get("cert_fill") or cert["fill"]                     # runs/certificate.json: the RCM run's
    assert nd["cert_fill"] < rcm_fill                                    # less fill than the RCM stand-in


PRECISION = os.path.join(HERE, "c1_precision")


def _load_form(form, name):
    with open(os.path.join(PRECISION, form, name)) as fh:
        return json.load(fh)


def test_bf16_solver_certified_within_1e_4_of_fp64():
    """Storage precision of V against the FP64 run, compared where it matters: the certified and verified U.  Both
    runs are the SBM workflow above (same instance: the planted modularity equals the c1 fixture's); one keeps V in
    FP64 throughout, the other runs the main phase with BF16 V and the proximal phase with FP32 V
    (--vdtype bf16 --proximal_vdtype f32), then the reference's chain with the nested-dissection ordering
    (reference_chain_nd.json, runs/verify.json).  Both are accepted by the reference verifier and their verified U
    differ by less than 1e-4 (absolute).  The BF16 main phase's own estimate is recorded too: its rounding of V
    (about 1e-3 on every inner product) separates spurious triangles whose multipliers the FP32 proximal phase
    releases, so the main checkpoint's bound is the looser of the two."""
    c1 = _load("c1", "summary.json")
    out = {}
    for form, (vd, pvd) in {"f64": ("f64", "f64"), "bf16_f32": ("bf16", "f32")}.items():
        s = _load_form(form, "summary.json")
        chain = _load_form(form, "reference_chain_nd.json")
        ver = _load_form(form, "runs/verify.json")
        assert (s["graph"], s["n"], s["m"]) == (c1["graph"], c1["n"], c1["m"])
        assert s["planted_modularity"] == c1["planted_modularity"]
        assert (s["vdtype"], s["proximal_vdtype"]) == (vd, pvd)
        assert chain["ckpt"] == s["best_ckpt"] and chain["ordering"] == "nd"
        assert chain["verified"] is True and ver["passed"] is True
        assert abs(ver["UB"] - chain["verified_UB"]) <= 1e-12 * chain["verified_UB"]
        assert s["planted_modularity"] <= chain["gpu_estimate"] <= chain["verified_UB"] < 0.7275
        out[form] = (s, chain)
    assert abs(out["bf16_f32"][1]["verified_UB"] - out["f64"][1]["verified_UB"]) < 1e-4
    assert abs(out["bf16_f32"][0]["estimate"] - out["f64"][0]["estimate"]) < 1e-6
    # the BF16 main phase alone: looser by more than the target
    assert out["bf16_f32"][0]["estimates"]["main"]["ub"] - out["f64"][0]["estimates"]["main"]["ub"] > 1e-4
