"""Pinning fields in the device local energy (reference src/nqs/pinning.py feeding
local_energy.py:86-88,109-111) against the oracle, and the observables built on the device spin
estimators on the reference's analytic case (tests/test_nqs_observables.py:17-40): a spin-
independent wavefunction is the uniform +x state, so every sigma_x estimator is exactly 1 and
every sigma_y estimator exactly 0."""
import numpy as np
import pytest
import torch

from helpers import build, configs, perturb
from oracle import nqs_oracle as O

pytestmark = pytest.mark.gpu

QSTAR = 0.9548
Q1 = QSTAR * np.array([1.0, 0.0])
Q2 = QSTAR * np.array([-0.5, np.sqrt(3) / 2])


@pytest.mark.parametrize("kind", ["skx", "overhauser"])
def test_pinning_field_local_energy_matches_oracle(kind):
    from nqs.local_energy import make_local_energy
    from nqs.pinning import make_pin
    from nqs.psiformer import make_logpsi
    g, model = build(n_dets=2, use_jastrow=True, n_knots=4)
    p = perturb(model.init(0), 0.05, 81)
    f = make_pin(kind, Q1, Q2, 0.4)
    R, S = configs(model.n_elec, model.L, 3, 82)
    E = make_local_energy(make_logpsi(model, p), 1.0, 1.0, 0.2, ext_field=f)(R, S).cpu()
    for w in range(3):
        ref = O.local_energy(lambda r, s: O.logpsi(model, p, r, s), R[w], S[w], 1.0, 1.0, 0.2,
                             ext_field=f)
        assert abs(complex(E[w]) - complex(ref)) < 1e-10 * max(1.0, abs(complex(ref)))


def _spin_independent_model(N=8, L=5.0, seed=3):
    """Zero backflow, no Jastrow, the same envelope weights for both spins: psi(R, S) does not
    depend on S."""
    from nqs.psiformer import ContinuumSpinorPsiformer
    ns = np.array([[0, 0], [1, 0], [0, 1], [-1, 0], [0, -1], [1, 1], [-1, -1], [1, -1]])
    Gs = (2.0 * np.pi * ns[:N] + np.array([0.1, 0.17])) / L  # distinct plane waves
    rng = np.random.default_rng(seed)
    Wu = rng.normal(size=(N, Gs.shape[0])) + 1j * rng.normal(size=(N, Gs.shape[0]))
    W = np.stack([Wu, Wu], axis=-1)
    return ContinuumSpinorPsiformer(n_elec=N, Gs=Gs, W=W, L=L, embed_dim=16, depth=1, n_heads=4,
                                    n_freq=4)


def test_observables_on_spin_independent_state():
    from nqs.observables import (classify_state, skx_arms, spin_order_parameter, spin_texture,
                                 structure_factor)
    from nqs.psiformer import make_logpsi
    model = _spin_independent_model()
    lp = make_logpsi(model, model.init(0))
    N, L, B = model.n_elec, model.L, 600
    rng = np.random.default_rng(4)
    R = torch.as_tensor(rng.uniform(0, L, (B, N, 2)))
    S = torch.as_tensor(rng.integers(0, 2, (B, N)))
    A = np.array([[L, 0.0], [0.0, L]])
    tex = spin_texture(lp, R, S, A, ngrid=8)
    assert abs(tex["mbar"][0] - 1.0) < 1e-9 and abs(tex["mbar"][1]) < 1e-9
    assert abs(tex["mbar"][2]) < 0.12
    sf = structure_factor(lp, R, S, A, nshell=3)
    qn = np.linalg.norm(sf["q"], axis=1)
    assert abs(sf["Sperp"][qn < 1e-9][0] - N) < 1e-8  # |sum_i 1|^2 / N
    assert sf["Sperp"][qn < 1e-9][0] > 3.0 * sf["Sperp"][qn > 1e-9].max()
    mG = spin_order_parameter(lp, R, S, A, skx_arms(Q1, Q2))
    assert abs(mG[0, 0] - 1.0) < 1e-9 and abs(mG[1, 0]) < 1e-9
    cl = classify_state(lp, R, S, A, ngrid=8, nshell=3)
    assert cl["label"] == "in-plane / Rashba-FM", cl["label"]


def test_skyrmion_envelope_is_an_eigenstate_under_its_texture():
    """Zero-backflow Psiformer on the skyrmion-background envelope (nqs.rashba.cell_skx_envelope:
    the occupied orbitals of h0 - lambda_tex n(r).sigma on a hexagonal supercell, 421 plane
    waves) with ext_field = lambda_tex n(r): the local energy is the band energy E_band at every
    configuration (to the basis truncation, ~1e-6 here), and matches the oracle."""
    import importlib.util
    import os
    from nqs import rashba
    from nqs.local_energy import make_local_energy
    from nqs.psiformer import ContinuumSpinorPsiformer, make_logpsi
    spec = importlib.util.spec_from_file_location(
        "make_golden", os.path.join(os.path.dirname(__file__), "golden", "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    q1, q2, A, keys, vals = mg.skx_case()
    lam_tex, N = 0.5, 7
    skx = rashba.cell_skx_envelope(A, N, keys, vals, q1, q2, lam_tex, 1.0, 0.3, 0.05, 12,
                                   (0.1, 0.17), gtol=1e-16)
    G = np.array([a * q1 + b * q2 for a, b in keys])

    def field(R):  # lambda_tex Re sum_Q S_Q e^{i Q.r}
        R = torch.as_tensor(R)
        g = torch.as_tensor(G, dtype=R.dtype, device=R.device)
        ph = R @ g.T
        Sr = torch.as_tensor(vals.real, dtype=R.dtype, device=R.device)
        Si = torch.as_tensor(vals.imag, dtype=R.dtype, device=R.device)
        return lam_tex * (torch.cos(ph) @ Sr - torch.sin(ph) @ Si)

    model = ContinuumSpinorPsiformer(n_elec=N, Gs=skx["Gs"], W=skx["W"], L=A, embed_dim=16,
                                     depth=1, n_heads=4, n_freq=4)
    p = model.init(0)
    rng = np.random.default_rng(91)
    R = torch.as_tensor(rng.uniform(0, 1, (24, N, 2)) @ np.asarray(A).T)
    S = torch.as_tensor(rng.integers(0, 2, (24, N)))
    E = make_local_energy(make_logpsi(model, p), 1.0, 0.3, 0.05, ext_field=field)(R, S).cpu()
    assert (E.real - skx["E_band"]).abs().max() < 2e-5, float((E.real - skx["E_band"]).abs().max())
    assert E.imag.abs().max() < 2e-5
    for w in range(2):
        ref = O.local_energy(lambda r, s: O.logpsi(model, p, r, s), R[w], S[w], 1.0, 0.3, 0.05,
                             ext_field=field)
        assert abs(complex(E[w]) - complex(ref)) < 1e-9 * max(1.0, abs(complex(ref)))
