"""The fused transformer block of single-channel (value) passes (block_tc.cu: LayerNorm, QKV,
attention, projection, MLP and both residual adds of src/nqs/psiformer.py:50-81 in one tcgen05
launch) against the unfused float32 launches of the same block and against the FP64 path, on
shapes with whole, partial (N = 5, 12: 125 / 120 rows per 128-row tile) and ragged last tiles.

Both float32 paths take the same TF32 products; they differ only in float32 summation order
(LayerNorm sums, attention sums, residual adds in registers instead of bulk reductions), so most
walkers come out bit-identical and the rest differ by a TF32 rounding flip of some activation.
The gates are therefore: fused and unfused sit at the same distance from FP64, and with the
benchmark's weight scale they agree closely."""
import pytest
import torch

from helpers import build, configs, perturb

pytestmark = pytest.mark.gpu


def _three_ways(model, p, R, S):
    from nqs import _lib
    from nqs.psiformer import make_logpsi
    L = _lib.lib()
    f = make_logpsi(model, p, precision="mixed")
    f(R, S)  # first call: weight copies and workspace
    torch.cuda.synchronize()
    try:
        _lib.check(L.nqs_set_block_fusion(0), "nqs_set_block_fusion")
        n0 = L.nqs_kernel_launches()
        unf = f(R, S).cpu()
        n1 = L.nqs_kernel_launches()
        _lib.check(L.nqs_set_block_fusion(1), "nqs_set_block_fusion")
        fus = f(R, S).cpu()
        n2 = L.nqs_kernel_launches()
        fus2 = f(R, S).cpu()
    finally:
        L.nqs_set_block_fusion(1)
    # the fused kernel ran: one launch per block instead of seven
    assert (n1 - n0) - (n2 - n1) == 6 * model.depth, (n1 - n0, n2 - n1)
    assert torch.equal(fus, fus2)  # deterministic
    return unf, fus, make_logpsi(model, p)(R, S).cpu()


@pytest.mark.parametrize("kw,W", [
    # N = 16 (8 walkers per tile), 4 blocks, 4 heads of 16, RBF Jastrow
    (dict(N=16, L=9.0, embed=64, depth=4, heads=4, n_freq=8, n_dets=2, use_jastrow=True,
          n_knots=8), 77),
    # 5 electrons: 125-row tiles, ragged last tile; 8 heads of 8
    (dict(N=5, L=7.0, embed=64, depth=2, heads=8, n_freq=4, n_dets=2), 53),
    # two electrons, width 32 (the small configuration's shape)
    (dict(N=2, L=5.0, embed=32, depth=2, heads=4, n_freq=8), 301),
    # 12 electrons: 120-row tiles
    (dict(N=12, L=8.0, embed=64, depth=3, heads=4, n_freq=8, n_dets=2, use_jastrow=True,
          n_knots=8), 41),
])
def test_fused_value_block_same_error_as_unfused(kw, W):
    """Strongly perturbed weights (0.05 on every leaf), where TF32 rounding is amplified."""
    g, model = build(**kw)
    p = perturb(model.init(0), 0.05, 61)
    R, S = configs(model.n_elec, model.L, W, 62)
    unf, fus, f64 = _three_ways(model, p, R, S)
    assert torch.isfinite(fus.real).all()
    eu, ef = (unf - f64).real.abs(), (fus - f64).real.abs()
    assert ef.mean() <= 1.25 * eu.mean() + 1e-7, (float(ef.mean()), float(eu.mean()))
    assert ef.max() <= 1.5 * eu.max() + 1e-7, (float(ef.max()), float(eu.max()))
    dph = torch.remainder((fus - unf).imag + torch.pi, 2 * torch.pi) - torch.pi
    assert dph.abs().max() < 5e-2


def test_fused_value_block_benchmark_weights():
    """The benchmark's weight scale (Dense ~N(0, 0.02^2), backflow 1e-3, Jastrow 0.02) at its
    shape (N = 16, width 64, 4 blocks, 4 heads): fused and unfused agree to a few 1e-5."""
    g, model = build(N=16, L=9.0, embed=64, depth=4, heads=4, n_freq=8, n_dets=2,
                     use_jastrow=True, n_knots=8)
    p = model.init_normal(0, std=0.02, backflow_std=1e-3, jastrow_std=0.02)
    R, S = configs(model.n_elec, model.L, 256, 62)
    unf, fus, f64 = _three_ways(model, p, R, S)
    d = (fus - unf).real.abs()
    assert d.max() < 1e-3 and d.mean() < 5e-5, (float(d.max()), float(d.mean()))
    ef = (fus - f64).real.abs()
    assert ef.max() < 2e-3 and ef.mean() < 2e-4, (float(ef.max()), float(ef.mean()))
