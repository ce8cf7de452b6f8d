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


def test_minsr_bf16_gram_close_to_fp64():
    """The BF16 Gram plus refinement against the exact operator gives a direction close to the
    float64 one on a well-conditioned problem."""
    from nqs.minsr import minsr_direction
    rng = np.random.default_rng(2)
    W, P = 256, 4000
    Oc = torch.as_tensor(rng.normal(size=(W, P)) + 1j * rng.normal(size=(W, P)))
    eps = torch.as_tensor(rng.normal(size=W) + 1j * rng.normal(size=W))
    d64 = minsr_direction(Oc.cuda(), eps, 1e-3, gram="fp64")
    for kind in ("bf16", "tf32"):
        d = minsr_direction(Oc.cuda(), eps, 1e-3, gram=kind, n_refine=4)
        rel = float((d - d64).norm() / d64.norm())
        assert rel < 1e-6, (kind, rel)
