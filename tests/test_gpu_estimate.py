"""The GPU-resident estimate (lagbound_b200/estimator_gpu.py) against the host path (NumPy vectors, SciPy LOBPCG,
the reference's algorithm) on the same instance and multipliers: the device operator reproduces C(y) X, the polish
reaches the same dual value, and both eigensolvers bracket the same pencil eigenvalue."""
import numpy as np
import pytest

from oracle import oracle as O
from _fixtures import EvalCase, rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    import torch
    from lagbound_b200 import Context
    from lagbound_b200 import estimator as E
    from lagbound_b200 import estimator_gpu as EG
    case = EvalCase("sbm400_k16")
    ctx = Context(0)
    inst = case.inst
    pair = [(Lv.lab, Lv.P, Lv.sig) for Lv in case.plev]
    vcs = [(Lv.lab, Lv.P, Lv.ptr, Lv.col, Lv.sig) for Lv in case.vlev]
    w = None if np.all(inst.data == 1.0) else inst.data
    args = (ctx, inst.n, inst.indptr, inst.indices, w, inst.d, inst.L, inst.C0, pair, vcs, case.TI, case.lam)
    host, dev = E.FixedOperator(*args), EG.DeviceOperator(*args)
    yield case, host, dev, torch
    host.close(); dev.close(); ctx.close()


def test_device_operator_matches_reference(setup):
    case, host, dev, torch = setup
    W = case.V
    CW = dev(torch.as_tensor(W, device=dev.dev)).cpu().numpy()
    assert rel(CW, case["est_CW"]) < 1e-10
    X = np.random.default_rng(0).standard_normal((case.inst.n, 70))      # two column blocks, odd width
    assert rel(dev(torch.as_tensor(X, device=dev.dev)).cpu().numpy(), host(X)) < 1e-12


def test_polish_and_eigenvalue_agree_with_host(setup):
    case, host, dev, torch = setup
    from lagbound_b200 import estimator as E
    from lagbound_b200 import estimator_gpu as EG
    const = case.inst.C0 + case.lam.sum()
    L = case.inst.L
    quiet = lambda *s: None
    Vh = E.polish_rgd(host, case.V.copy(), const, L, iters=60, time_limit=60, log=quiet)
    Vd = EG.polish_rgd(dev, torch.as_tensor(case.V, device=dev.dev), const, L, iters=60, time_limit=60, log=quiet)
    dvh, gh, _ = E.value(host, Vh, const, L)
    dvd, gd, _ = EG.value(dev, Vd, const, L)
    assert abs(dvh - dvd) < 1e-6 * max(1.0, abs(dvh))          # same steps; reductions round differently
    rh, _ = E.eig_round(host, Vh, dvh, gh, case.inst.d, L, np.random.default_rng(0), ("vol",), maxiter=200,
                        chunk=20, atol=1e-7, log=quiet)
    rd, _ = EG.eig_round(dev, Vd, dvd, gd, case.inst.d, L, 0, ("vol",), maxiter=200, chunk=20, atol=1e-7, log=quiet)
    th_h, th_d = rh["vol"]["theta"][0], rd["vol"]["theta"][0]
    # both Ritz values bound the pencil's smallest eigenvalue from above; at convergence they agree to the residuals
    tol = 10 * (rh["vol"]["resid"][0] + rd["vol"]["resid"][0]) + 1e-8
    assert abs(th_h - th_d) < tol, (th_h, th_d, tol)
    assert abs(rh["vol"]["ub"] - rd["vol"]["ub"]) < 1e-4
