"""Per-sample Jacobian (hand-written reverse mode) and MinSR on the device against the oracle,
central finite differences and the explicit parameter-space solve (reference
src/nqs/minsr.py:30-88; tests/test_nqs_minsr.py:46-61)."""
import numpy as np
import pytest
import torch

from helpers import build, configs, perturb
from oracle import nqs_oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kw", [
    dict(embed=12, heads=3),
    dict(n_dets=3, use_jastrow=True, n_knots=5),
    dict(use_jastrow=True, jastrow_kind="cusp", learnable_env=True, n_dets=2),
])
def test_per_sample_O_matches_oracle_jacobian(kw):
    from nqs.minsr import per_sample_O, real_ravel
    g, model = build(**kw)
    p = perturb(model.init(0), 0.05, 31)
    theta, unravel = real_ravel(p)
    R, S = configs(model.n_elec, model.L, 5, 32)
    Og = per_sample_O(model, theta.cuda(), unravel, R, S).cpu()
    ot, ou = O.real_ravel(p["params"])
    Oo = O.per_sample_O(model, ot, ou, R, S)
    scale = Oo.abs().max()
    assert (Og - Oo).abs().max() < 1e-10 * max(1.0, float(scale))


def test_per_sample_O_central_fd_large_model():
    """Config-3 style check: N=16, width 64, 4 blocks, 4 heads, K=4, RBF Jastrow (16 knots):
    O v against (log psi(theta + h v) - log psi(theta - h v)) / 2h, h = 1e-5, 64 directions."""
    from nqs import rashba
    from nqs.minsr import per_sample_O_rows
    from nqs.psiformer import ContinuumSpinorPsiformer, make_logpsi
    L = float(np.sqrt(np.pi * 16) * 5.0)
    env = rashba.cell_rashba_envelope(L, 16, 1.0, 0.3, 0.05, 10, (0.1, 0.17))
    model = ContinuumSpinorPsiformer(16, env["Gs"], env["W"], L, embed_dim=64, depth=4, n_heads=4,
                                     n_freq=8, n_dets=4, use_jastrow=True, n_knots=16)
    p = model.init_normal(0, std=0.02, backflow_std=1e-3, jastrow_std=0.02, logw_std=0.1)
    theta = model.theta(p)
    R, S = configs(16, L, 4, 5)
    rows = per_sample_O_rows(model, theta, R, S).cpu()
    Oc = torch.complex(rows[:4], rows[4:])
    rng = np.random.default_rng(0)
    h = 1e-5
    worst = 0.0
    for _ in range(64):
        v = torch.as_tensor(rng.standard_normal(theta.shape[0]))
        v /= v.norm()
        vd = v.cuda()
        fp = make_logpsi(model, theta + h * vd)(R, S).cpu()
        fm = make_logpsi(model, theta - h * vd)(R, S).cpu()
        fd = (fp - fm) / (2 * h)
        an = Oc @ v.to(torch.complex128)
        # compare modulo 2 pi branch jumps of Im log psi (none expected for h = 1e-5)
        worst = max(worst, float((fd - an).abs().max()))
    assert worst < 1e-6, worst


def test_minsr_equals_paramsr_1e10():
    """minsr.py:76-88 push-through identity on the device, float64 (north-star bar 1e-10)."""
    from nqs.minsr import minsr_direction, paramsr_direction, per_sample_O, real_ravel
    g, model = build(embed=12, heads=3)
    p = model.init(0)
    theta, unravel = real_ravel(p)
    R, S = configs(5, 7.0, 24, 4)
    Og = per_sample_O(model, theta.cuda(), unravel, R, S)
    rng = np.random.default_rng(4)
    eps = torch.as_tensor(rng.normal(size=24) + 1j * rng.normal(size=24))
    for lam in (1e-2, 1e-4):
        d1 = minsr_direction(Og, eps, lam)
        d2 = paramsr_direction(Og, eps, lam)
        rel = float((d1 - d2).abs().max() / d2.abs().max())
        assert rel < 1e-10, (lam, rel)


def test_minsr_matches_oracle_on_same_O():
    from nqs.minsr import minsr_direction
    rng = np.random.default_rng(7)
    W, P = 96, 700
    Oc = torch.as_tensor(rng.normal(size=(W, P)) + 1j * rng.normal(size=(W, P)))
    eps = torch.as_tensor(rng.normal(size=W) + 1j * rng.normal(size=W))
    for lam in (1e-3, 1e-1):
        d_dev = minsr_direction(Oc.cuda(), eps, lam).cpu()
        d_ref = O.minsr_direction(Oc, eps, lam)
        assert float((d_dev - d_ref).abs().max() / d_ref.abs().max()) < 1e-10


def test_minsr_large_gram_split_paths():
    """2W = 640 (5 row tiles, split-K) and 2W = 1040 (ragged tiles) against the oracle."""
    from nqs.minsr import minsr_direction
    rng = np.random.default_rng(8)
    for W, P in ((320, 5000), (520, 3001)):
        Oc = torch.as_tensor(rng.normal(size=(W, P)) + 1j * rng.normal(size=(W, P)))
        eps = torch.as_tensor(rng.normal(size=W) + 1j * rng.normal(size=W))
        d_dev = minsr_direction(Oc.cuda(), eps, 1e-3).cpu()
        d_ref = O.minsr_direction(Oc, eps, 1e-3)
        assert float((d_dev - d_ref).abs().max() / d_ref.abs().max()) < 1e-9


def test_clip_energies_matches_oracle():
    from nqs.minsr import clip_energies
    rng = np.random.default_rng(3)
    for W in (7, 256, 1000):
        e = torch.as_tensor(rng.standard_cauchy(W) + 1j * rng.normal(size=W))
        c, stats = clip_energies(e.cuda(), 5.0)
        ref = O.clip_energies(e, 5.0)
        assert torch.equal(c.cpu(), ref)
        st = stats.cpu()
        assert abs(float(st[0]) - float(e.real.mean())) < 1e-12 * max(1, float(e.real.abs().max()))


def test_mixed_O_close_to_fp64():
    from nqs.minsr import per_sample_O_rows, real_ravel
    g, model = build(n_dets=2)
    p = perturb(model.init(0), 0.05, 3)
    theta, _ = real_ravel(p)
    R, S = configs(5, 7.0, 8, 1)
    a = per_sample_O_rows(model, theta.cuda(), R, S)
    b = per_sample_O_rows(model, theta.cuda(), R, S, dtype=torch.float32, precision="mixed")
    assert float((a - b.double()).abs().max() / a.abs().max()) < 1e-4
