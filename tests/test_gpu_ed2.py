"""Whole-iteration physics against the two-electron exact diagonalisation (oracle/ed2.py,
tests/golden/ed2_config1.json): configuration-1 physics with Coulomb (N = 2, r_s = 2,
lambda_R = 0.5, h_z = 0.1, Ewald eta = 5/L). A Jastrow-free Psiformer trained with MinSR on the
device must respect the variational bound (E_VMC >= E_ED within the statistical error) and
recover part of the correlation energy E_HF - E_ED, E_HF = zeta_M for the initial determinant.
(The reference's README states 0.7 mHa at two electrons for its own, unstated, setting; here the
correlation energy is 145 mHa and the Jastrow-free ansatz recovers ~60% of it in 400 steps.)"""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_minsr_two_electrons_variational_against_ed():
    from nqs import rashba
    from nqs.ewald import make_ewald
    from nqs.minsr import VMCIteration, real_ravel, train_minsr
    from nqs.psiformer import ContinuumSpinorPsiformer
    g = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "ed2_config1.json")))
    L, lr_r, hz = g["L"], g["lambda_r"], g["h_z"]
    gs = rashba.noninteracting_gs(N=2, L=L, m_star=1.0, lambda_r=lr_r, h_z=hz, n_cut=10,
                                  twist=(0.0, 0.0))
    Gs, W = rashba.planewave_envelope(*rashba.occupied_orbital_matrix(gs))
    model = ContinuumSpinorPsiformer(n_elec=2, Gs=Gs, W=W, L=L, embed_dim=32, depth=2,
                                     n_heads=4, n_freq=8, n_dets=1)
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
    E, err = float(np.mean(Es)), float(np.std(Es) / np.sqrt(len(Es)))
    E_ed, E_hf = g["E_ed_ncut24"], g["zeta_M"]
    assert E > E_ed - 4 * err - 1e-4, (E, err, E_ed)           # variational bound
    assert (E_hf - E) / (E_hf - E_ed) > 0.4, (E, E_hf, E_ed)   # correlation recovered
