"""Attention of the multi-channel batches on the tensor cores (nqs_set_attention_mma: mma.sync
TF32 products, accumulator fragments carried across the forward-Laplacian channels) against the
float32 CUDA-core kernels and the float64 path: local energies (forward-Laplacian batch and
spin-orbit flips) and log psi, for 16, 26 and 48 electrons (one to three 16-row query tiles).
The bar is the mixed path's own error against float64 (its TF32 Dense layers)."""
import numpy as np
import pytest
import torch

from helpers import build, configs, perturb

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N,embed,heads", [(16, 64, 4), (26, 64, 4), (48, 128, 8)])
def test_tensor_core_attention_local_energy(N, embed, heads):
    from nqs import _lib
    from nqs.local_energy import make_local_energy
    from nqs.psiformer import make_logpsi
    g, model = build(N=N, L=1.9 * np.sqrt(N), embed=embed, depth=2, heads=heads, n_dets=2,
                     use_jastrow=True, n_knots=6)
    p = perturb(model.init(0), 0.03, 70 + N)
    R, S = configs(model.n_elec, model.L, 24, 71 + N)

    def run(prec, mma):
        _lib.lib().nqs_set_attention_mma(mma)
        try:
            lp = make_logpsi(model, p, precision=prec)
            return lp(R, S).cpu(), make_local_energy(lp, 1.0, 0.7, 0.3)(R, S).cpu()
        finally:
            _lib.lib().nqs_set_attention_mma(1)

    l64, e64 = run("fp64", 0)
    l_mma, e_mma = run("mixed", 1)
    l_f32, e_f32 = run("mixed", 0)
    assert torch.isfinite(e_mma).all()
    # value passes keep the float32 kernels: log psi is unchanged by the switch
    assert torch.equal(l_mma, l_f32)
    err_mma = float((e_mma - e64).abs().median())
    err_f32 = float((e_f32 - e64).abs().median())
    # the mixed path's error against float64 comes mostly from its TF32 Dense layers: the TF32
    # attention may add to it, by less than that error again
    assert err_mma < 2.0 * err_f32, (err_mma, err_f32)
