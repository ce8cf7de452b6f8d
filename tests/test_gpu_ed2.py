"""Whole-iteration physics against the two-electron exact diagonalisation (oracle/ed2.py,
tests/golden/ed2_config1.json): configuration-1 physics with Coulomb (N = 2, r_s = 2,
lambda_R = 0.5, h_z = 0.1, Ewald eta = 5/L).

Two checks of the trained wavefunction, besides the variational bound of its VMC energy:
  - its exact energy: psi sampled on a G^4 grid of (r_1, r_2) for the four spin pairs, Fourier
    transformed to plane-wave amplitudes and <H> evaluated with the ED Hamiltonian
    (ed2.expectation). For a smooth psi (no Jastrow) the VMC energy from the local energies
    agrees with it within the statistical error: the device's local energy, Ewald sum included,
    and the ED Hamiltonian are the same operator.
  - the reference's cusp pair Jastrow is a function of the minimum-image distance, so psi has a
    derivative jump on the Wigner-Seitz boundary; the local energy misses the resulting
    delta-function kinetic term. Trained with it, the VMC energy falls below E_ED while the
    exact energy of the same psi stays above it.
(The reference's README states 0.7 mHa at two electrons for its own, unstated, setting; here the
correlation energy E_HF - E_ED is 145 mHa and the Jastrow-free ansatz recovers ~60% of it in 400
MinSR steps.)"""
import json
import os

import numpy as np
import pytest
import torch

from oracle import ed2

pytestmark = pytest.mark.gpu

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "ed2_config1.json")))


def _train(**jastrow):
    from nqs import rashba
    from nqs.ewald import make_ewald
    from nqs.minsr import VMCIteration, real_ravel, train_minsr
    from nqs.psiformer import ContinuumSpinorPsiformer
    L, lr_r, hz = GOLDEN["L"], GOLDEN["lambda_r"], GOLDEN["h_z"]
    gs = rashba.noninteracting_gs(N=2, L=L, m_star=1.0, lambda_r=lr_r, h_z=hz, n_cut=10,
                                  twist=(0.0, 0.0))
    Gs, W = rashba.planewave_envelope(*rashba.occupied_orbital_matrix(gs))
    model = ContinuumSpinorPsiformer(n_elec=2, Gs=Gs, W=W, L=L, embed_dim=32, depth=2,
                                     n_heads=4, n_freq=8, n_dets=1, **jastrow)
    _, _, coul = make_ewald(L, alpha=1.0, ewald_alpha=5.0 / L, n_real=3, n_recip=8)
    params, hist, R, S = train_minsr(model, model.init(0), L, 2, 0, m_star=1.0, lambda_r=lr_r,
                                     h_z=hz, coulomb=coul, n_walkers=2048, n_steps=400, lr=0.03,
                                     lam=1e-3, n_sweeps=10, step_size=0.4, burn=200, log_every=0,
                                     return_walkers=True)
    theta, _ = real_ravel(params)
    it = VMCIteration(model, theta, R, S, lambda_r=lr_r, h_z=hz, coulomb=coul, lr=0.0,
                      n_sweeps=10, step_size=0.4)
    Es = []
    for _ in range(30):
        it.sample()
        it.energies()
        Es.append(float(it.e.real.mean()))
    return model, theta, float(np.mean(Es)), float(np.std(Es) / np.sqrt(len(Es)))


def _exact_energy(model, theta, G=48, n_cut=14):
    """<H> of psi truncated to |n| <= n_cut plane waves per particle (amplitudes from a G^4 grid
    by FFT), with the ED Hamiltonian."""
    from nqs.psiformer import make_logpsi
    L = GOLDEN["L"]
    lp = make_logpsi(model, theta)
    f = torch.arange(G, dtype=torch.float64, device="cuda") * (L / G)
    x1, y1, x2, y2 = torch.meshgrid(f, f, f, f, indexing="ij")
    R = torch.stack([torch.stack([x1, y1], -1), torch.stack([x2, y2], -1)], -2).reshape(-1, 2, 2)
    logs = torch.empty(4, R.shape[0], dtype=torch.complex128, device="cuda")
    chunk = 1 << 20
    for s in range(4):
        S = torch.tensor([s // 2, s % 2], dtype=torch.int32, device="cuda").expand(chunk, 2)
        for a in range(0, R.shape[0], chunk):
            b = min(R.shape[0], a + chunk)
            logs[s, a:b] = lp(R[a:b].contiguous(), S[: b - a].contiguous())
    del R
    ok = torch.isfinite(logs.real)
    assert bool(ok.any())
    assert bool((ok | (logs.real == -float("inf"))).all())  # only exact nodes are non-finite
    mx = logs.real[ok].max()
    psi = torch.where(ok, torch.exp(logs - mx), torch.zeros((), dtype=logs.dtype, device="cuda"))
    psi = psi.reshape(2, 2, G, G, G, G).permute(2, 3, 4, 5, 0, 1)
    c = torch.fft.fftn(psi, dim=(0, 1, 2, 3)) / G ** 4
    idx = torch.arange(-n_cut, n_cut + 1, device="cuda") % G
    cc = c[idx][:, idx][:, :, idx][:, :, :, idx].cpu().numpy()
    return ed2.expectation(np.diag([L, L]), cc, n_cut, 1.0, GOLDEN["lambda_r"], GOLDEN["h_z"],
                           alpha=1.0, ewald_alpha=5.0 / L)


def test_minsr_two_electrons_variational_against_ed():
    """Jastrow-free: E_VMC >= E_ED (within 4 sigma), > 40% of the correlation energy recovered,
    and E_VMC equal to the exact <H> of the same psi within 4 sigma + 1 mHa."""
    model, theta, E, err = _train()
    E_ed, E_hf = GOLDEN["E_ed_ncut24"], GOLDEN["zeta_M"]
    assert E > E_ed - 4 * err - 1e-4, (E, err, E_ed)           # variational bound
    assert (E_hf - E) / (E_hf - E_ed) > 0.4, (E, E_hf, E_ed)   # correlation recovered
    E_exact = _exact_energy(model, theta)
    assert E_exact > E_ed
    assert abs(E - E_exact) < 4 * err + 1e-3, (E, err, E_exact)


def test_minimum_image_cusp_jastrow_is_not_variational():
    """With the cusp Jastrow of the minimum-image distance the trained VMC energy lies more than
    10 mHa below E_ED while the exact <H> of the same psi lies above E_ED."""
    model, theta, E, err = _train(use_jastrow=True, jastrow_kind="cusp")
    E_ed = GOLDEN["E_ed_ncut24"]
    assert E < E_ed - 1e-2 - 4 * err, (E, err, E_ed)
    assert _exact_energy(model, theta) > E_ed
