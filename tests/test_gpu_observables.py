"""Spin estimators from flip ratios (reference src/nqs/observables.py:31-53) against the oracle's
log psi, and the spin-spiral state's texture (non-collinear, as tests/test_nqs_spiral.py:60-70)."""
import numpy as np
import pytest
import torch

from helpers import build, configs, perturb
from oracle import nqs_oracle as O

pytestmark = pytest.mark.gpu


def test_spin_estimators_match_oracle():
    from nqs.observables import make_spin_estimators
    from nqs.psiformer import make_logpsi
    g, model = build(n_dets=2, use_jastrow=True, n_knots=4)
    p = perturb(model.init(0), 0.05, 71)
    R, S = configs(model.n_elec, model.L, 4, 72)
    sx, sy, sz = make_spin_estimators(make_logpsi(model, p))(R, S)
    sx, sy, sz = sx.cpu(), sy.cpu(), sz.cpu()
    for w in range(4):
        L0 = O.logpsi(model, p, R[w], S[w])
        for i in range(model.n_elec):
            Sf = S[w].clone()
            Sf[i] = 1 - Sf[i]
            r = complex(torch.exp(O.logpsi(model, p, R[w], Sf) - L0))
            z = 1.0 - 2.0 * float(S[w, i])
            assert abs(complex(sx[w, i]) - r) < 1e-10 * max(1.0, abs(r))
            assert abs(complex(sy[w, i]) - (-1j * z * r)) < 1e-10 * max(1.0, abs(r))
            assert float(sz[w, i]) == z


def test_spiral_texture_is_noncollinear():
    """Sampled from the exact spin-spiral determinant (zero-backflow Psiformer on the spiral
    envelope): the in-plane magnetisation changes sign across the cell in both x and y."""
    from nqs.observables import spin_estimates
    from nqs.psiformer import ContinuumSpinorPsiformer, make_logpsi
    from nqs.sampler import run_chain
    from nqs.spiral import spiral_gs
    res = spiral_gs(N=7, L=8.0, Q_int=(1, 0), B=0.3, lambda_r=1.0, h_z=0.0, n_cut=10,
                    twist=(0.1, 0.17))
    model = ContinuumSpinorPsiformer(n_elec=7, Gs=res["Gs"], W=res["W"], L=8.0, embed_dim=16,
                                     depth=1, n_heads=4, n_freq=4)
    lp = make_logpsi(model, model.init(0))
    R, S, _, _ = run_chain(lp, 8.0, 7, 3, n_walkers=2048, n_sweeps=30, burn=60, step=0.6)
    ng, L = 8, 8.0
    # bin the per-electron estimators by position (bin sums / number of configurations)
    sx, sy, sz = spin_estimates(lp, R, S)
    gi = np.clip((np.mod(R.cpu().numpy(), L) / L * ng).astype(int), 0, ng - 1)
    m = np.zeros((ng, ng, 3))
    for c, v in enumerate((sx, sy, sz)):
        np.add.at(m[..., c], (gi[..., 0].ravel(), gi[..., 1].ravel()), v.ravel())
    m /= R.shape[0]
    mx, my = m[..., 0], m[..., 1]
    assert mx.max() > 0 > mx.min() and my.max() > 0 > my.min()
    # the determinant's exact spin density at the bin centres, times the bin area
    sig = [np.array([[0, 1], [1, 0]]), np.array([[0, -1j], [1j, 0]]), np.diag([1.0, -1.0])]
    xs = (np.arange(ng) + 0.5) * L / ng
    exact = np.zeros((ng, ng, 3))
    for ix, x in enumerate(xs):
        for iy, y in enumerate(xs):
            phi = np.einsum("g,ags->as", np.exp(1j * (res["Gs"] @ np.array([x, y]))), res["W"]) / L
            for c in range(3):
                exact[ix, iy, c] = np.real(np.einsum("as,st,at->", phi.conj(), sig[c], phi))
    exact *= (L / ng) ** 2
    assert np.mean(np.abs(m - exact)) < 0.02, np.mean(np.abs(m - exact))
