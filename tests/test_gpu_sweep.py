"""GPU batched Gauss-Seidel sweeps (lb_sweeps) against the oracle's sweeps (the reference's batch_step6 row step in
the Jacobi-within-batch form, with its pair rows, VCS pre/post terms and aggregate updates).

Tolerances: FP64 V within 1e-10 (relative Frobenius) after two sweeps; FP32 V within 1e-5 and BF16 V within 5e-3
after one sweep (the stored rows are rounded to the storage type after every step; the oracle steps in FP64 from
the same rounded start).
"""
import numpy as np
import pytest

from oracle import oracle as O
from _fixtures import EvalCase, eval_names, rel
from test_gpu_eval import make_problem

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from lagbound_b200 import Context
    c = Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module", params=eval_names())
def case(request):
    return EvalCase(request.param)


@pytest.mark.parametrize("dtype,nsw,tol", [("f64", 2, 1e-10), ("f32", 1, 1e-5), ("bf16", 1, 5e-3)])
def test_sweeps_match_oracle(ctx, case, dtype, nsw, tol):
    p = make_problem(ctx, case, dtype)
    V0 = p.get_V()
    rng = np.random.default_rng(3)
    perms = np.stack([rng.permutation(case.inst.n) for _ in range(nsw)])
    nbatch = 5
    damp = 0.1
    p.sweeps(perms, case.rho, case.rho * case.tri_weight, damp, nbatch)
    Vg = p.get_V()
    Vo = O.sweeps(case.inst, V0, perms, nbatch, case.plev, case.TI, case.lam, case.vlev, case.rho, case.tri_weight,
                  case.wv, damp)
    assert np.allclose(np.linalg.norm(Vg, axis=1), 1.0, atol=1e-2 if dtype == "bf16" else 1e-6)
    assert rel(Vg, Vo) < tol, rel(Vg, Vo)
    p.close()


def test_plain_mixing_sweeps_match_oracle(ctx, case):
    """rho = 0: plain damped mixing at fixed multipliers (the estimator's polishing sweeps)."""
    p = make_problem(ctx, case, "f64")
    V0 = p.get_V()
    perms = np.random.default_rng(4).permutation(case.inst.n)[None]
    p.sweeps(perms, 0.0, 0.0, 0.5, 7)
    Vo = O.sweeps(case.inst, V0, perms, 7, case.plev, case.TI, case.lam, case.vlev, 0.0, case.tri_weight, case.wv, 0.5)
    assert rel(p.get_V(), Vo) < 1e-10
    p.close()


def test_sweeps_raise_the_augmented_lagrangian(ctx, case):
    """A few sweeps at fixed multipliers do not decrease the augmented Lagrangian (minorant steps)."""
    p = make_problem(ctx, case, "f64")
    before = p.eval(case.rho, case.tri_weight, grad=False)["value"]
    rng = np.random.default_rng(9)
    p.sweeps(np.stack([rng.permutation(case.inst.n) for _ in range(3)]), case.rho, case.rho * case.tri_weight, 0.0, 8)
    after = p.eval(case.rho, case.tri_weight, grad=False)["value"]
    assert after >= before - 1e-9 * abs(before)
    p.close()
