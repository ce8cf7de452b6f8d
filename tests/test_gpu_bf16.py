"""BF16 operands on the tensor cores (precision "mixed_bf16": kind::f16 MMAs with float32
accumulation in the fused value-pass blocks and the row GEMMs, width 64) against the float64
oracle and against an emulation of the same operand rounding in the oracle (each Dense layer's
input and kernel rounded to BF16, products exact): the device follows the BF16 semantics an order
of magnitude more closely than it follows the unrounded float64 network (reference
src/nqs/psiformer.py:50-81, 139-143)."""
import numpy as np
import pytest
import torch

from helpers import build, configs, perturb
from oracle import nqs_oracle as O

pytestmark = pytest.mark.gpu


def _bf16(x):
    return x.to(torch.bfloat16).to(x.dtype)


def _model():
    g, model = build(N=6, L=7.5, embed=64, depth=2, heads=4, n_freq=8, n_dets=2,
                     use_jastrow=True, n_knots=6)
    p = perturb(model.init(0), 0.05, 91)
    return model, p


def _oracle(model, p, R, S, rounded):
    O.OPERAND_ROUND = _bf16 if rounded else None
    try:
        return torch.stack([O.logpsi(model, p, R[w], S[w]) for w in range(R.shape[0])])
    finally:
        O.OPERAND_ROUND = None


def _dist(a, b):
    d = a - b
    return (d.real.abs() + ((d.imag + np.pi) % (2 * np.pi) - np.pi).abs()).mean().item()


@pytest.mark.parametrize("fused", [True, False])
def test_bf16_logpsi_follows_bf16_rounding(fused):
    """Value passes (fused block, or unfused LayerNorm / row GEMMs / attention) with BF16
    operands against the oracle with BF16-rounded operands and against the exact oracle."""
    from nqs import _lib
    from nqs.psiformer import make_logpsi
    model, p = _model()
    R, S = configs(model.n_elec, model.L, 24, 92)
    _lib.lib().nqs_set_block_fusion(1 if fused else 0)
    try:
        lb = make_logpsi(model, p, precision="mixed_bf16")(R, S).cpu()
        lt = make_logpsi(model, p, precision="mixed")(R, S).cpu()
    finally:
        _lib.lib().nqs_set_block_fusion(1)
    exact = _oracle(model, p, R, S, False)
    emu = _oracle(model, p, R, S, True)
    d_emu, d_exact, d_tf32 = _dist(lb, emu), _dist(lb, exact), _dist(lt, exact)
    assert d_exact > 1e-5  # the rounding is visible
    assert d_emu < 0.1 * d_exact, (d_emu, d_exact)
    assert d_tf32 < d_exact, (d_tf32, d_exact)


def test_bf16_local_energy_close_to_fp64():
    """Forward-Laplacian and spin-orbit batches through the BF16 row GEMMs: per-walker local
    energy errors against the float64 path scale like the operand rounding. BF16 keeps 8
    significant bits and TF32 11, so the BF16 errors are expected ~8x the TF32 ones: the median
    BF16 error lies between the TF32 median and 32x it, and below 5% of the median |E_loc|."""
    from nqs.local_energy import make_local_energy
    from nqs.psiformer import make_logpsi
    model, p = _model()
    R, S = configs(model.n_elec, model.L, 64, 93)
    el = {prec: make_local_energy(make_logpsi(model, p, precision=prec), 1.0, 1.0, 0.5)(R, S).cpu()
          for prec in ("mixed_bf16", "mixed", "fp64")}
    assert torch.isfinite(el["mixed_bf16"]).all()
    d_bf = float((el["mixed_bf16"] - el["fp64"]).abs().median())
    d_tf = float((el["mixed"] - el["fp64"]).abs().median())
    scale = float(el["fp64"].abs().median())
    assert d_tf < d_bf < 32.0 * d_tf, (d_bf, d_tf, scale)
    assert d_bf < 0.05 * scale, (d_bf, d_tf, scale)
