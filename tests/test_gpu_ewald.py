"""Ewald kernels against the oracle and the reference's analytic checks
(src/nqs/ewald.py:26-73; tests/test_nqs_ewald.py:21-99, tests/test_nqs_cell.py:39-78)."""
import numpy as np
import pytest
import torch

from oracle import nqs_oracle as O

pytestmark = pytest.mark.gpu


def test_pair_and_energy_match_oracle():
    from nqs.ewald import make_ewald
    L = 8.0
    ep, zM, ce = make_ewald(L, alpha=1.0, n_real=6, n_recip=12)
    ref = O.Ewald(np.eye(2) * L, 1.0, None, 6, 12)
    assert abs(zM - ref.zeta_M) < 1e-12
    rng = np.random.default_rng(0)
    r = rng.uniform(-L, L, (50, 2))
    assert np.abs(ep(r).cpu().numpy() - ref.pair(r)).max() < 1e-11
    R = rng.uniform(0, L, (7, 6, 2))
    assert np.abs(ce(R).cpu().numpy() - ref.energy(R)).max() < 1e-10


def test_splitting_independence():
    from nqs.ewald import make_ewald
    L = 7.0
    r = torch.tensor([1.3, -2.1], dtype=torch.float64)
    vals, zs = [], []
    for c in (0.8, 1.0, 1.25):
        ep, zM, _ = make_ewald(L, 1.0, c * np.sqrt(np.pi) / L, 8, 14)
        vals.append(float(ep(r)))
        zs.append(zM)
    assert np.ptp(vals) < 1e-7 and np.ptp(zs) < 1e-7


def test_periodicity_evenness_alpha_short_range():
    from nqs.ewald import make_ewald
    L = 7.0
    ep, _, _ = make_ewald(L, alpha=1.0, n_real=8, n_recip=12)
    r = torch.tensor([1.1, 2.7], dtype=torch.float64)
    assert abs(float(ep(r)) - float(ep(r + torch.tensor([L, 0.0], dtype=torch.float64)))) < 1e-8
    assert abs(float(ep(r)) - float(ep(-r))) < 1e-10
    ep2, z2, _ = make_ewald(L, alpha=2.5, n_real=8, n_recip=12)
    _, z1, _ = make_ewald(L, alpha=1.0, n_real=8, n_recip=12)
    assert abs(2.5 * float(ep(r)) - float(ep2(r))) < 1e-9 and abs(2.5 * z1 - z2) < 1e-9
    for d in (1e-3, 1e-4):
        assert abs(float(ep(torch.tensor([d, 0.0], dtype=torch.float64))) * d - 1.0) < 1e-2 + 5e-3


def test_energy_translation_invariant_and_general_cells():
    from nqs.cell import hex_cell, rect_cell
    from nqs.ewald import make_ewald, make_ewald_lattice
    L = 8.0
    ep, zM, ce = make_ewald(L, alpha=1.0, n_real=6, n_recip=12)
    rng = np.random.default_rng(0)
    R = torch.as_tensor(rng.uniform(0, L, (6, 2)))
    E = float(ce(R))
    pairs = sum(float(ep(R[i] - R[j])) for i in range(6) for j in range(i + 1, 6))
    assert abs(E - (pairs + 6 * zM / 2.0)) < 1e-9
    assert abs(E - float(ce(R + torch.tensor([2.3, -1.1], dtype=torch.float64)))) < 1e-8
    for A in (rect_cell(7.0, 7.0 * np.sqrt(3)), hex_cell(8.0)):
        Es = []
        Rf = torch.as_tensor(rng.uniform(0, 1, (6, 2)) @ np.asarray(A).T)
        for c in (0.7, 1.0, 1.4):
            eta = c * np.sqrt(np.pi) / np.sqrt(abs(np.linalg.det(A)))
            _, _, ce2 = make_ewald_lattice(A, 1.0, eta, 9, 16)
            Es.append(float(ce2(Rf)))
        assert np.ptp(Es) < 1e-6
