"""Host-side logic of the drop-in stages (no GPU): the VCS working-set merge, the triangle pool merge, checkpoint
triangle normalisation, the instance CSR, the --init_partition colouring and the command lines the reference
pipeline passes, against the reference's own outputs (golden fixtures) and the oracle."""
import glob
import json
import os
import tempfile

import numpy as np
import pytest

from oracle import oracle as O
from _fixtures import GOLDEN, sep_names, vsep_names


@pytest.mark.parametrize("name", vsep_names())
def test_working_set_merge_matches_reference(name):
    from lagbound_b200.vcs import merge_working_set
    z = np.load(os.path.join(GOLDEN, f"vsep_{name}.npz"))
    keep = z["age"] < int(z["vcs_drop"])
    P = int(z["lab"].max()) + 1
    rng = np.random.default_rng(0)
    perm = rng.permutation(len(z["rows0"]))                  # any order of the new entries
    m = merge_working_set(len(z["d"]), P, z["ptr"], z["col"], z["sig"], z["age"], keep, z["rows0"][perm],
                          z["cols0"][perm])
    for k_, got in zip(("m_ptr", "m_col", "m_sig", "m_age"), m):
        assert np.array_equal(got, z[k_]) and got.dtype == z[k_].dtype, k_
    with pytest.raises(ValueError):
        merge_working_set(len(z["d"]), P, z["ptr"], z["col"], z["sig"], z["age"], np.ones(len(keep), bool),
                          z["rows0"][:1].repeat(2), z["cols0"][:1].repeat(2))


def test_working_set_merge_matches_oracle_random():
    from lagbound_b200.vcs import merge_working_set
    rng = np.random.default_rng(3)
    n, P = 500, 37
    dense = rng.random((n, P)) < 0.1
    ptr = np.r_[0, np.cumsum(dense.sum(1))].astype(np.int64)
    col = np.nonzero(dense)[1].astype(np.int32)
    sig = rng.random(len(col)); age = rng.integers(0, 9, len(col)).astype(np.uint8)
    keep = age < 5
    free = np.argwhere(~dense)
    pick = free[rng.choice(len(free), 300, replace=False)]
    got = merge_working_set(n, P, ptr, col, sig, age, keep, pick[:, 0], pick[:, 1])
    ref = O.vcs_update_ws(n, ptr, col, sig, age, keep, pick[:, 0], pick[:, 1])
    for g_, r_ in zip(got, ref):
        assert np.array_equal(g_, r_)


@pytest.mark.parametrize("name", sep_names())
def test_pool_merge_matches_reference(name):
    from lagbound_b200 import pool
    z = np.load(os.path.join(GOLDEN, f"sep_{name}.npz"))
    TI, lam = pool.purge(z["TI0"], z["lam0"])
    room = max(0, int(z["tri_max"]) - len(TI))
    TIp, lamp, nadd = pool.merge(int(z["n"]), TI, lam, z["both_new0"], z["both_val0"], z["both_new1"], z["both_val1"],
                                 int(z["tri_add"]), int(z["tri1_add"]), room)
    assert np.array_equal(TIp, z["pool_TI"]) and np.array_equal(lamp, z["pool_lam"])
    assert nadd == len(TIp) - len(TI)


def test_pool_normalise_merges_duplicates():
    from lagbound_b200 import pool
    TI = np.array([[5, 1, 2], [2, 1, 5], [0, 3, 4], [4, 3, 0], [4, 3, 0]])
    lam = np.array([1.0, 2.0, 0.5, 0.25, 0.25])
    TIn, lamn, merged = pool.normalise(TI, lam, 6)
    assert merged and TIn.tolist() == [[0, 3, 4], [2, 1, 5]] and lamn.tolist() == [1.0, 3.0]
    _, _, merged = pool.normalise(TIn, lamn, 6)
    assert not merged


def _write_instance(tmp, n, keys, weights=None, vol=None, meta=None):
    D = os.path.join(tmp, "data", "g"); os.makedirs(D, exist_ok=True)
    np.save(os.path.join(D, "keys.npy"), keys)
    json.dump({"n": n, "m": len(keys)}, open(os.path.join(D, "graph.json"), "w"))
    if weights is not None:
        np.save(os.path.join(D, "weights.npy"), weights)
    if vol is not None:
        np.save(os.path.join(D, "vol.npy"), vol); json.dump(meta, open(os.path.join(D, "meta.json"), "w"))
    return os.path.join(tmp, "data") + "/"


def test_load_instance_matches_the_reference_csr():
    import scipy.sparse as sp
    from lagbound_b200.stages.common import load_instance
    z = np.load(os.path.join(GOLDEN, "reduce_sbm_leaves_twins.npz"))
    n, keys, w, vol = int(z["rn"]), z["rkeys"], z["rweights"], z["rvol"]
    tmp = tempfile.mkdtemp()
    D = _write_instance(tmp, n, keys, w, vol, {"L_orig": int(z["L_orig"]), "leaf_edges": int(z["leaf_edges"])})
    inst = load_instance("g", D)
    u, v = keys // n, keys % n
    A = sp.csr_matrix((np.r_[w, w], (np.r_[u, v], np.r_[v, u])), shape=(n, n)); A.sort_indices()
    assert np.array_equal(inst["indptr"], A.indptr) and np.array_equal(inst["indices"], A.indices)
    assert np.array_equal(inst["weights"], A.data)
    assert np.array_equal(inst["d"], vol.astype(float)) and inst["L"] == int(z["L_orig"])
    assert inst["C0"] == 2.0 * int(z["leaf_edges"])
    D2 = _write_instance(tempfile.mkdtemp(), n, keys)
    inst2 = load_instance("g", D2)
    assert inst2["weights"] is None and inst2["L"] == 2 * len(keys)
    assert np.array_equal(inst2["d"], np.bincount(np.r_[u, v], minlength=n).astype(float))


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "init_*.npz"))))
def test_init_partition_colouring_matches_reference(path):
    from lagbound_b200.stages.alm_vcs import colouring_start
    z = np.load(path)
    inst = dict(n=int(z["n"]), indptr=z["indptr"], indices=z["indices"], d=z["d"])
    V = colouring_start(z["lab"], inst, int(z["k"]), np.random.default_rng(int(z["seed"])), lambda *s: None)
    assert np.array_equal(V, z["V"])


def test_stage_command_lines_of_the_pipeline_parse():
    """Every flag the reference pipeline passes (pipeline.py:116-128, 160-165) is accepted as given."""
    from lagbound_b200.stages import alm_vcs, est_dual_vcs
    base = ["--tag", "g__rx", "--pair_labels", "a.npy", "b.npy", "--max_clusters", "6000", "--k", "32", "--nbatch", "31",
            "--inner", "1", "--est_every", "0", "--tri_max", "16000000", "--mom", "0", "--lb", "nan", "--shift_p", "0",
            "--time_limit", "100", "--seed", "0", "--vcs_labels", "c.npy", "--vcs_max", "150000000", "--vcs_add",
            "10000000", "--outer", "3000", "--save", "runs/main.npz"]
    main = base + ["--tri_add", "600000", "--tri1_add", "300000", "--tri_every", "9", "--init_partition", "p.npy",
                   "--pw_rule", "default", "--ckpt_every", "50"]
    prox = base + ["--resume", "runs/main_last.npz", "--tri_add", "0", "--tri1_add", "0", "--tri_every", "1000000",
                   "--pairlvl_weight", "0.01", "--phase2_at_it", "1", "--phase2_w", "0.01", "--phase2_inner", "4",
                   "--phase2_tri_every", "1000000", "--phase2_est_every", "0", "--ckpt_every", "20"]
    a = alm_vcs.parse(main)
    assert a.pair_labels == ["a.npy", "b.npy"] and a.tri1_add == 300000 and a.pw_rule == "default"
    b = alm_vcs.parse(prox)
    assert b.phase2_inner == 4 and b.pairlvl_weight == 0.01
    e = est_dual_vcs.parse(["--tag", "g__rx", "--ckpt", "x.npz", "--lb", "nan", "--polish", "rgd", "--polish_time",
                            "900", "--scale", "vol", "--eig_time", "900", "--out", "o.json", "--initV", "w.npz",
                            "--saveW", "s.npz"])
    assert e.polish == "rgd" and e.scale == "vol"
    with pytest.raises(SystemExit):
        alm_vcs.parse(base + ["--nbr_cut", "1"])


def test_install_redirects_only_the_gpu_stages():
    from lagbound_b200 import stages

    class FakeWorkspace:
        calls = []

        def run(self, script, args, log, threads=None, blas_threads=None, extra_env=None):
            import lagbound.pipeline as P
            FakeWorkspace.calls.append((os.path.join(P.CORE, script), list(args)))
            return log

    import sys
    import types
    fake_pkg = types.ModuleType("lagbound"); fake_pipe = types.ModuleType("lagbound.pipeline")
    fake_pipe.CORE = "/ref/core"; fake_pipe.Workspace = FakeWorkspace; fake_pkg.pipeline = fake_pipe
    saved = {k: sys.modules.get(k) for k in ("lagbound", "lagbound.pipeline")}
    sys.modules["lagbound"] = fake_pkg; sys.modules["lagbound.pipeline"] = fake_pipe
    try:
        stages.install(FakeWorkspace, vdtype="bf16")
        w = FakeWorkspace()
        w.run("alm_vcs.py", ["--tag", "g"], "x.log")
        w.run("certify_lifted_vc.py", ["g"], "c.log")
        w.run("est_dual_vcs.py", ["--tag", "g"], "e.log")
        assert FakeWorkspace.calls[0] == (stages.STAGES["alm_vcs.py"], ["--tag", "g", "--vdtype", "bf16"])
        assert FakeWorkspace.calls[1] == ("/ref/core/certify_lifted_vc.py", ["g"])
        assert FakeWorkspace.calls[2] == (stages.STAGES["est_dual_vcs.py"], ["--tag", "g"])
        assert fake_pipe.CORE == "/ref/core"
        stages.uninstall(FakeWorkspace)
        assert not hasattr(FakeWorkspace, "_lagbound_b200_original_run")
        # BF16 main phase, FP32 proximal phase (the solver run that resumes the main checkpoint)
        stages.install(FakeWorkspace, vdtype="bf16", proximal_vdtype="f32")
        w = FakeWorkspace()
        w.run("alm_vcs.py", ["--tag", "g"], "m.log")
        w.run("alm_vcs.py", ["--tag", "g", "--resume", "runs/main_last.npz"], "p.log")
        assert FakeWorkspace.calls[-2][1] == ["--tag", "g", "--vdtype", "bf16"]
        assert FakeWorkspace.calls[-1][1] == ["--tag", "g", "--resume", "runs/main_last.npz", "--vdtype", "f32"]
        stages.uninstall(FakeWorkspace)
    finally:
        for k, v in saved.items():
            if v is None:
                sys.modules.pop(k, None)
            else:
                sys.modules[k] = v
