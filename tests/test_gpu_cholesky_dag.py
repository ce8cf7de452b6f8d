"""The task-graph float64 Cholesky (one persistent kernel over 128 x 128 tiles; off by default,
nqs_set_cholesky_dag) against the launch-per-panel factorization and a CPU float64 solve,
inside the MinSR sample-space solve (reference src/nqs/minsr.py:76-81) and the explicit Gram solve (:84-88):
sizes that are one tile, several tiles with a partial last tile, and the benchmark's 8192."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _problem(W, P, seed, decay=True):
    rng = np.random.default_rng(seed)
    O = rng.standard_normal((2 * W, P))
    if decay:  # a spread spectrum like the wavefunction Jacobians'
        O *= np.exp(-np.linspace(0.0, 6.0, P))[None, :]
    eps = rng.standard_normal(W) + 1j * rng.standard_normal(W)
    return torch.as_tensor(O), torch.as_tensor(eps)


def _dir(O, eps, lam, gram, dag, **kw):
    from nqs import _lib
    from nqs.minsr import minsr_step
    _lib.lib().nqs_set_cholesky_dag(dag)
    try:
        rows = O.cuda().to(torch.float64 if gram == "fp64" else torch.float32).contiguous()
        return minsr_step(rows.clone(), eps, lam, gram, **kw).cpu()
    finally:
        _lib.lib().nqs_set_cholesky_dag(0)


def _cpu_direction(O, eps, lam):
    """[Re; Im] rows of the walker-centred complex O, (T + lam I) y = [Re; Im](e - mean e),
    dtheta = rows^T y, in float64 on the CPU."""
    W = O.shape[0] // 2
    Oc = torch.complex(O[:W], O[W:])
    Oc = Oc - Oc.mean(0, keepdim=True)
    rows = torch.cat([Oc.real, Oc.imag], 0)
    e = eps - eps.mean()
    et = torch.cat([e.real, e.imag])
    T = rows @ rows.T + lam * torch.eye(2 * W, dtype=torch.float64)
    y = torch.linalg.solve(T, et)
    return rows.T @ y


@pytest.mark.parametrize("W,P", [(8, 40), (100, 600), (700, 3000)])
def test_dag_cholesky_minsr_matches_panel_cholesky_and_cpu(W, P):
    O, eps = _problem(W, P, W)
    lam = 1e-3
    a = _dir(O, eps, lam, "fp64", 1, n_refine=3)
    b = _dir(O, eps, lam, "fp64", 0, n_refine=3)
    ref = _cpu_direction(O, eps, lam)
    assert float((a - b).norm() / b.norm()) < 1e-10
    assert float((a - ref).norm() / ref.norm()) < 1e-9


def test_dag_cholesky_preconditioner_at_benchmark_size():
    """n = 8192 (W = 4096): the BF16-Gram PCG solved to 1e-10 with either factorization as the
    preconditioner gives the same direction, and so does the float64 solve with either factor;
    the two agree to the float32 rounding of the PCG's operand."""
    O, eps = _problem(4096, 12000, 5)
    lam = 1e-3
    info_a = torch.zeros(5, dtype=torch.int32, device="cuda")
    info_b = torch.zeros(5, dtype=torch.int32, device="cuda")
    a = _dir(O, eps, lam, "bf16", 1, n_refine=64, tol=1e-10, info=info_a)
    b = _dir(O, eps, lam, "bf16", 0, n_refine=64, tol=1e-10, info=info_b)
    assert int(info_a[0]) == 0 and int(info_b[0]) == 0
    assert float((a - b).norm() / b.norm()) < 1e-8
    c = _dir(O, eps, lam, "fp64", 1, n_refine=2)
    d = _dir(O, eps, lam, "fp64", 0, n_refine=2)
    assert float((c - d).norm() / d.norm()) < 1e-10
    # the PCG's operator reads the float32 rows: 1e-7-level operand rounding against float64
    assert float((a - c).norm() / c.norm()) < 1e-6


def test_dag_cholesky_gram_solve():
    """nqs_gram_solve (explicit parameter-space solve) with the task-graph factor: odd and even
    sizes against the CPU."""
    from nqs import _lib
    from nqs.minsr import gram_solve
    rng = np.random.default_rng(3)
    for M, K in ((130, 300), (256, 900)):
        A = torch.as_tensor(rng.standard_normal((M, K)))
        rhs = torch.as_tensor(rng.standard_normal(M))
        _lib.lib().nqs_set_cholesky_dag(1)
        try:
            x = gram_solve(A.cuda(), rhs, 1e-2).cpu()
        finally:
            _lib.lib().nqs_set_cholesky_dag(0)
        y = gram_solve(A.cuda(), rhs, 1e-2).cpu()
        ref = torch.linalg.solve(A @ A.T + 1e-2 * torch.eye(M, dtype=torch.float64), rhs)
        assert float((x - ref).norm() / ref.norm()) < 1e-10
        assert float((x - y).norm() / y.norm()) < 1e-10
