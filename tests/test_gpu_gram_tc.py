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
def test_gram_tc_matches_fp64_of_rounded_operands(M, K, kind):
    from nqs.minsr import gram_lower
    g = torch.Generator().manual_seed(M * 7 + K)
    A = torch.randn(M, K, generator=g, dtype=torch.float32)
    T = gram_lower(A.cuda(), kind).cpu()
    Ar = A.to(torch.bfloat16).double() if kind == "bf16" else _tf32(A).double()
    ref = torch.tril(Ar @ Ar.T)
    scale = (Ar.abs() @ Ar.abs().T).max()
    err = (T - ref).abs().max() / scale
    # float32 accumulation over K terms: relative error ~ sqrt(K) 2^-24, bounded by K 2^-24
    assert err < 3e-5, float(err)
    assert torch.count_nonzero(torch.triu(T, 1)) == 0


def test_minsr_tensor_core_gram_refined_to_fp64():
    """With a tensor-core Gram the solve uses lam + delta (delta = u mean diag T, u its rounding
    level); refinement against the exact operator reproduces the float64 solve at that damping."""
    from nqs.minsr import minsr_direction, minsr_step, _as_rows
    rng = np.random.default_rng(2)
    W, P = 256, 4000
    Oc = torch.as_tensor(rng.normal(size=(W, P)) + 1j * rng.normal(size=(W, P)))
    eps = torch.as_tensor(rng.normal(size=W) + 1j * rng.normal(size=W))
    for kind in ("bf16", "tf32"):
        delta = torch.zeros(1, dtype=torch.float64, device="cuda")
        d = minsr_step(_as_rows(Oc).cuda(), eps, 1e-3, kind, n_refine=3, damping_out=delta)
        dl = float(delta.item())
        assert dl > 0
        d64 = minsr_direction(Oc.cuda(), eps, 1e-3 + dl, gram="fp64")
        rel = float((d - d64).norm() / d64.norm())
        assert rel < 1e-8, (kind, rel)
