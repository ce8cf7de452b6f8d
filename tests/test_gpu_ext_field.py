"""External spin field in the local energy (reference src/nqs/local_energy.py:41-42,86-88,109-111;
the spin-spiral gate tests/test_nqs_spiral.py:45-57 and tests/test_nqs_folx.py:59-70)."""
import numpy as np
import pytest
import torch

from helpers import build, configs, perturb
from oracle import nqs_oracle as O

pytestmark = pytest.mark.gpu

SPIRAL = dict(N=7, L=8.0, Q_int=(1, 0), B=0.3, lambda_r=1.0, h_z=0.0, n_cut=10, twist=(0.1, 0.17))


def _spiral_model():
    from nqs.psiformer import ContinuumSpinorPsiformer
    from nqs.spiral import spiral_gs
    res = spiral_gs(**SPIRAL)
    model = ContinuumSpinorPsiformer(n_elec=res["N"], Gs=res["Gs"], W=res["W"], L=res["L"],
                                     embed_dim=16, depth=2, n_heads=4, n_freq=4)
    return res, model


def test_spiral_zero_variance():
    """Zero-backflow Psiformer on the exact spiral envelope (441 plane waves): E_loc = E_gs."""
    from nqs.local_energy import make_local_energy
    from nqs.psiformer import make_logpsi
    from nqs.spiral import spiral_field
    res, model = _spiral_model()
    R, S = configs(res["N"], res["L"], 16, 61)
    E = make_local_energy(make_logpsi(model, model.init(0)), 1.0, res["lambda_r"], res["h_z"],
                          ext_field=spiral_field(res["B"], res["Q"]))(R, S).cpu()
    assert E.real.std() < 1e-10
    assert abs(float(E.real.mean()) - res["E_gs"]) < 1e-10
    assert E.imag.abs().max() < 1e-10


@pytest.mark.parametrize("lr", [1.0, 0.0])
def test_ext_field_matches_oracle(lr):
    """Perturbed network, a spiral field (and the field alone, lambda_R = 0: the flipped states
    are still needed for the sigma_x, sigma_y part)."""
    from nqs.local_energy import make_local_energy
    from nqs.psiformer import make_logpsi
    from nqs.spiral import spiral_field
    res, model = _spiral_model()
    p = perturb(model.init(0), 0.05, 62)
    f = spiral_field(res["B"], res["Q"])
    R, S = configs(res["N"], res["L"], 3, 63)
    E = make_local_energy(make_logpsi(model, p), 1.0, lr, 0.2, ext_field=f)(R, S).cpu()
    for w in range(3):
        ref = O.local_energy(lambda r, s: O.logpsi(model, p, r, s), R[w], S[w], 1.0, lr, 0.2,
                             ext_field=f)
        assert abs(complex(E[w]) - complex(ref)) < 1e-10 * max(1.0, abs(complex(ref)))


def test_ext_field_with_z_component_matches_oracle():
    """A pinning-like field with all three components on the usual Rashba model."""
    from nqs.local_energy import make_local_energy
    from nqs.psiformer import make_logpsi
    g, model = build(n_dets=2, use_jastrow=True, n_knots=4)
    p = perturb(model.init(0), 0.05, 64)

    def field(R):
        R = torch.as_tensor(R)
        a = 2 * np.pi * R[..., 0] / model.L
        b = 2 * np.pi * R[..., 1] / model.L
        return torch.stack([0.1 * torch.cos(a), 0.2 * torch.sin(b), 0.3 * torch.cos(a + b)], -1)

    R, S = configs(model.n_elec, model.L, 3, 65)
    E = make_local_energy(make_logpsi(model, p), 1.0, 1.0, 0.5, ext_field=field)(R, S).cpu()
    for w in range(3):
        ref = O.local_energy(lambda r, s: O.logpsi(model, p, r, s), R[w], S[w], 1.0, 1.0, 0.5,
                             ext_field=field)
        assert abs(complex(E[w]) - complex(ref)) < 1e-10 * max(1.0, abs(complex(ref)))


def test_vmc_iteration_energies_with_field():
    """The training loop's E_loc (VMCIteration, used by train_minsr) takes the same field."""
    from nqs.local_energy import make_local_energy
    from nqs.minsr import VMCIteration, real_ravel
    from nqs.psiformer import make_logpsi
    from nqs.spiral import spiral_field
    res, model = _spiral_model()
    p = perturb(model.init(0), 0.05, 66)
    f = spiral_field(res["B"], res["Q"])
    R, S = configs(res["N"], res["L"], 8, 67)
    theta, _ = real_ravel(p)
    it = VMCIteration(model, theta, R, S, lambda_r=1.0, h_z=0.2, ext_field=f)
    it.energies()
    ref = make_local_energy(make_logpsi(model, p), 1.0, 1.0, 0.2, ext_field=f)(R, S)
    assert (it.e - ref).abs().max() < 1e-12 * max(1.0, float(ref.abs().max()))
