"""Pinning fields in the device local energy (reference src/nqs/pinning.py feeding
local_energy.py:86-88,109-111) against the oracle, and the device spin estimators on the
reference's analytic case (tests/test_nqs_observables.py:17-40): a spin-independent wavefunction
is the uniform +x state, so every sigma_x estimator is exactly 1 and every sigma_y estimator
exactly 0."""
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


def test_spin_estimators_on_spin_independent_state():
    """A spin-independent wavefunction is the uniform +x state: every sigma_x estimator is exactly
    1, every sigma_y estimator exactly 0, and sigma_z = 1 - 2 s (reference
    tests/test_nqs_observables.py:17-40)."""
    from nqs.observables import spin_estimates
    from nqs.psiformer import make_logpsi
    model = _spin_independent_model()
    lp = make_logpsi(model, model.init(0))
    N, L, B = model.n_elec, model.L, 600
    rng = np.random.default_rng(4)
    R = torch.as_tensor(rng.uniform(0, L, (B, N, 2)))
    S = torch.as_tensor(rng.integers(0, 2, (B, N)))
    sx, sy, sz = spin_estimates(lp, R, S)
    assert np.abs(sx - 1.0).max() < 1e-9 and np.abs(sy).max() < 1e-9
    assert np.array_equal(sz, 1.0 - 2.0 * S.numpy())
