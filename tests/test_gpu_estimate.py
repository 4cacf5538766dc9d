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


def test_native_lobpcg_matches_tensor_lobpcg(setup):
    """lb_lobpcg (the iteration in the library) against estimator_gpu.lobpcg (the same iteration as tensor
    operations) from the same start block: Ritz values within 1e-7 after 20 iterations, the returned vectors
    B-orthonormal with those Rayleigh quotients, and eig_round's bound the same either way."""
    case, host, dev, torch = setup
    from lagbound_b200 import estimator_gpu as EG
    n, L = case.inst.n, case.inst.L
    const = case.inst.C0 + case.lam.sum()
    W = torch.as_tensor(case.V, device=dev.dev)
    dv, g, _ = EG.value(dev, W, const, L)
    dT = torch.as_tensor(case.inst.d, dtype=torch.float64, device=dev.dev)
    s = dT.clamp_min(1.0)
    prec = 1.0 / ((g + dT ** 2 / L).abs() + 1e-2 * s)
    gen = torch.Generator(device=dev.dev)
    gen.manual_seed(3)
    X0 = torch.randn(n, 32, dtype=torch.float64, device=dev.dev, generator=gen)
    Mop = lambda X: g[:, None] * X - dev(X)
    th_t, X_t = EG.lobpcg(Mop, s, prec, X0.clone(), 20)
    th_n, X_n = dev.lobpcg(X0.clone(), g, s, prec, 20)
    th_t = th_t.cpu().numpy()
    assert np.allclose(th_n, th_t, rtol=1e-7, atol=1e-9), np.abs(th_n - th_t).max()
    B = X_n.T @ (s[:, None] * X_n)
    assert torch.allclose(B, torch.eye(32, dtype=torch.float64, device=dev.dev), atol=1e-8)
    q = ((X_n * Mop(X_n)).sum(0) / (X_n * (s[:, None] * X_n)).sum(0)).cpu().numpy()
    assert np.allclose(np.sort(q), th_n, rtol=1e-8, atol=1e-10)
    quiet = lambda *a: None
    rn, _ = EG.eig_round(dev, W, dv, g, case.inst.d, L, 0, ("vol",), maxiter=100, chunk=20, atol=1e-7, log=quiet)
    rt, _ = EG.eig_round(dev, W, dv, g, case.inst.d, L, 0, ("vol",), maxiter=100, chunk=20, atol=1e-7, log=quiet,
                         native=False)
    assert abs(rn["vol"]["ub"] - rt["vol"]["ub"]) < 1e-8
    assert rn["vol"]["eig_trace"][-1][0] == rt["vol"]["eig_trace"][-1][0]     # same number of iterations
