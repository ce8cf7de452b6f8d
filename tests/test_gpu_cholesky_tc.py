"""The mixed-precision MinSR solve (reference src/nqs/minsr.py:76-81) with the preconditioner
Cholesky's K = 256 trailing updates on the tensor cores (split-TF32 operands,
nqs_set_cholesky_tc, default on) against the same solve with float64 CUDA-core updates: the
conjugate gradients solve the exact system either way, so the directions agree when both are
solved tightly, and the preconditioner is as good (same iteration count at the default tolerance).
Sizes with one, several and many trailing updates (n = 2W = 1400, 2600, 8192)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _problem(W, P, seed):
    rng = np.random.default_rng(seed)
    O = rng.standard_normal((2 * W, P)) * np.exp(-np.linspace(0.0, 6.0, P))[None, :]
    eps = rng.standard_normal(W) + 1j * rng.standard_normal(W)
    return torch.as_tensor(O), torch.as_tensor(eps)


def _dir(O, eps, lam, tc, **kw):
    from nqs import _lib
    from nqs.minsr import minsr_step
    info = torch.zeros(5, dtype=torch.int32, device="cuda")
    _lib.lib().nqs_set_cholesky_tc(tc)
    try:
        rows = O.cuda().to(torch.float32).contiguous()
        d = minsr_step(rows, eps, lam, "bf16", info=info, **kw).cpu()
    finally:
        _lib.lib().nqs_set_cholesky_tc(1)
    return d, [int(v) for v in info.cpu()]


@pytest.mark.parametrize("W,P", [(700, 3000), (1300, 5000), (4096, 12000)])
def test_tensor_core_trailing_updates_same_solution_and_iterations(W, P):
    O, eps = _problem(W, P, W)
    lam = 1e-3
    a, ia = _dir(O, eps, lam, 1, n_refine=64, tol=1e-10)
    b, ib = _dir(O, eps, lam, 0, n_refine=64, tol=1e-10)
    assert ia[0] == 0 and ia[1] == 0 and ib[0] == 0
    assert ia[4] == 1 and ib[4] == 1  # both converged
    assert float((a - b).norm() / b.norm()) < 1e-8
    assert abs(ia[3] - ib[3]) <= 1, (ia, ib)
    # default tolerance: the preconditioner quality shows in the iteration count
    c, ic = _dir(O, eps, lam, 1, n_refine=64)
    d, id_ = _dir(O, eps, lam, 0, n_refine=64)
    assert ic[3] <= id_[3] + 1, (ic, id_)
    assert float((c - a).norm() / a.norm()) < 2e-2
    assert float((d - a).norm() / a.norm()) < 2e-2
