"""The drop-in stage scripts end to end on the GPU: reduction, solver main and proximal phases, bound estimates, on
a small planted-partition graph, with the pipeline's own flags.  Checks the files the reference's later stages read
(checkpoint schema, estimate JSON keys, the pair-weight log line) and that the estimates bound the planted
partition's modularity from above."""
import json
import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def run():
    wd = tempfile.mkdtemp(prefix="lb_stages_")
    cmd = [sys.executable, "-m", "lagbound_b200.stages.workflow", "--workdir", wd, "--n", "600", "--blocks", "6",
           "--p_in", "0.1", "--p_out", "0.01", "--time", "24", "--polish_time", "20", "--eig_time", "20"]
    proc = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=900)
    assert proc.returncode == 0, proc.stdout[-3000:] + proc.stderr[-3000:]
    return wd, json.load(open(os.path.join(wd, "summary.json")))


def test_workflow_bounds_the_planted_partition(run):
    wd, s = run
    assert set(s["estimates"]) == {"main", "proximal"}
    for name, e in s["estimates"].items():
        assert np.isfinite(e["ub"]) and e["ub"] >= e["dv"] - 1e-12
        assert e["ub"] >= s["planted_modularity"] - 1e-6, (name, e, s["planted_modularity"])
        assert e["ub"] < 1.0
    assert s["pair_weight"] is not None and s["pair_weight"] > 0


def test_checkpoint_schema(run):
    wd, s = run
    for ck in ("main_last.npz", "proximal_last.npz"):
        z = np.load(os.path.join(wd, "runs", ck))
        for key in ("TI", "lam", "V", "nlev", "mu", "CI", "om", "PI", "psi", "nvc", "nvcs"):
            assert key in z.files, key
        assert z["V"].dtype == np.float32 and int(z["nlev"]) == 1 and int(z["nvcs"]) == 1
        sig = z["sig0"]
        assert np.array_equal(sig, sig.T) and (sig >= 0).all() and int(z["pair0"]) == 1 and int(z["dense0"]) == 1
        ptr, col = z["vcsptr0"], z["vcscol0"]
        assert ptr[0] == 0 and ptr[-1] == len(col) == len(z["vcssig0"]) and z["vcssig0"].dtype == np.float32
        assert (z["lam"] >= 0).all() and len(z["lam"]) == len(z["TI"])
        rows = np.repeat(np.arange(len(ptr) - 1), np.diff(ptr))
        assert np.all((np.diff(col) > 0) | (np.diff(rows) > 0))          # rows sorted by cluster
    z = np.load(os.path.join(wd, "runs", "main_last.npz"))
    assert len(z["TI"]) > 0 and int((z["lam"] > 0).sum()) > 0 and z["vcsptr0"][-1] > 0


def test_logs_and_estimate_json(run):
    wd, s = run
    main_log = open(os.path.join(wd, "runs", "main.log")).read()
    assert "-> pairlvl_weight" in main_log and "it 1 L " in main_log and "PHASE2" not in main_log
    prox_log = open(os.path.join(wd, "runs", "proximal.log")).read()
    assert "PHASE2 at outer 2" in prox_log
    assert os.path.exists(os.path.join(wd, "runs", "main.history.json"))
    e = json.load(open(os.path.join(wd, "runs", "est_main.json")))
    for key in ("ub", "dv", "dv0", "s_vol", "escape_rounds", "polish_hist"):
        assert key in e, key
    assert "lmin_est" in e["s_vol"] and e["s_vol"]["ub"] >= e["ub"] - 1e-12
