"""tcgen05 Gram (BF16 / TF32 operands, float32 accumulation in tensor memory) against a float64
product of the identically rounded operands; MinSR with the tensor-core Gram against float64."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _tf32(x):
    """TF32 operand as the tensor core reads it: the low 13 mantissa bits of float32 dropped."""
    i = x.to(torch.float32).contiguous().view(torch.int32)
    return (i & ~0x1FFF).view(torch.float32)


@pytest.mark.parametrize("M,K", [(128, 64), (300, 1000), (520, 3001), (1030, 777)])
@pytest.mark.parametrize("kind", ["bf16", "tf32"])
@pytest.mark.parametrize("wide", [1, 0])
def test_gram_tc_matches_fp64_of_rounded_operands(M, K, kind, wide):
    """wide: 256 x 256 tiles (two accumulators per CTA, the default above 256 rows); 0: 128 x 256."""
    from nqs import _lib
    from nqs.minsr import gram_lower
    g = torch.Generator().manual_seed(M * 7 + K)
    A = torch.randn(M, K, generator=g, dtype=torch.float32)
    _lib.lib().nqs_set_gram_wide(wide)
    try:
        T = gram_lower(A.cuda(), kind).cpu()
    finally:
        _lib.lib().nqs_set_gram_wide(1)
    Ar = A.to(torch.bfloat16).double() if kind == "bf16" else _tf32(A).double()
    ref = torch.tril(Ar @ Ar.T)
    scale = (Ar.abs() @ Ar.abs().T).max()
    err = (T - ref).abs().max() / scale
    # float32 accumulation over K terms: relative error ~ sqrt(K) 2^-24, bounded by K 2^-24
    assert err < 3e-5, float(err)
    assert torch.count_nonzero(torch.triu(T, 1)) == 0


def test_minsr_tensor_core_gram_solves_at_lam():
    """With a tensor-core Gram the factor of T + (lam + delta) I only preconditions conjugate
    gradients on the exact system: run to a tight tolerance, the direction equals the float64
    solve at lam itself."""
    from nqs.minsr import minsr_direction, minsr_step, _as_rows
    rng = np.random.default_rng(2)
    W, P = 256, 4000
    Oc = torch.as_tensor(rng.normal(size=(W, P)) + 1j * rng.normal(size=(W, P)))
    eps = torch.as_tensor(rng.normal(size=W) + 1j * rng.normal(size=W))
    d64 = minsr_direction(Oc.cuda(), eps, 1e-3, gram="fp64")
    for kind in ("bf16", "tf32"):
        delta = torch.zeros(1, dtype=torch.float64, device="cuda")
        info = torch.zeros(5, dtype=torch.int32, device="cuda")
        d = minsr_step(_as_rows(Oc).cuda(), eps, 1e-3, kind, n_refine=64, damping_out=delta,
                       info=info, tol=1e-12)
        assert float(delta.item()) > 0
        rel = float((d - d64).norm() / d64.norm())
        assert rel < 1e-9, (kind, rel, info.tolist())
        assert info[0] == 0 and info[1] == 0 and info[4] in (0, 1)


@pytest.mark.parametrize("lam", [1e-3, 1e-4])
def test_mixed_minsr_at_configured_damping_config2_jacobian(lam):
    """Configuration-2 model, W = 1024 thermalised walkers, the float32 Jacobian of the mixed
    network: the BF16-Gram-preconditioned CG direction at lam (default tolerance) is within 1e-2
    of the float64 solve at lam of the same Jacobian, and within 1e-2 of the all-float64 path's
    direction (float64 network, float64 Jacobian, float64 Gram)."""
    from nqs.configs import config
    from nqs.ewald import make_ewald
    from nqs.minsr import VMCIteration, minsr_step
    from nqs.sampler import init_walkers_uniform
    model, params, su = config(2, 1024)
    R0, S0 = init_walkers_uniform(5, 1024, su.N, su.L)
    _, _, coul = make_ewald(su.L, alpha=1.0, ewald_alpha=su.ewald_eta, n_real=su.n_real,
                            n_recip=su.n_recip)
    kw = dict(m_star=1.0, lambda_r=su.lambda_r, h_z=su.h_z, coulomb=coul, lam=lam,
              n_sweeps=10, step_size=su.step, seed=3)
    it = VMCIteration(model, model.theta(params), R0, S0, precision="mixed", **kw)
    it.sample(30)
    it.energies()
    it.jacobian()
    info = torch.zeros(5, dtype=torch.int32, device="cuda")
    d = minsr_step(it.O.clone(), it.e, lam, "bf16", info=info)
    d_same = minsr_step(it.O.double(), it.e, lam, "fp64")
    rel = float((d - d_same).norm() / d_same.norm())
    assert rel < 1e-2, (rel, info.tolist())
    it64 = VMCIteration(model, it.theta, it.R, it.S, precision="fp64", **kw)
    it64.energies()
    it64.jacobian()
    d64 = minsr_step(it64.O.clone(), it64.e, lam, "fp64")
    rel64 = float((d - d64).norm() / d64.norm())
    assert rel64 < 1e-2, (rel64, info.tolist())
