"""Forward-Laplacian local energy against the oracle's dense Hessian and the analytic
certificates (reference src/nqs/local_energy.py:40-117; tests/test_nqs_local_energy.py:22-66,
tests/test_nqs_folx.py:22-82)."""
import numpy as np
import pytest
import torch

from helpers import TWIST, build, configs, perturb
from nqs import rashba
from oracle import nqs_oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kw", [
    dict(),
    dict(n_dets=3, use_jastrow=True, n_knots=5),
    dict(use_jastrow=True, jastrow_kind="cusp", N=4, L=6.0),
])
def test_grad_laplacian_vs_dense_hessian(kw):
    """forward Laplacian == dense Hessian trace (reference folx test asserts 1e-9)."""
    from nqs.local_energy import grad_and_laplacian
    from nqs.psiformer import make_logpsi
    g, model = build(**kw)
    p = perturb(model.init(0), 0.05, 11)
    R, S = configs(model.n_elec, model.L, 4, 12)
    L, gr, lap = grad_and_laplacian(make_logpsi(model, p), R, S)
    for w in range(4):
        L0, g0, lap0 = O.grad_and_lap(lambda r, s: O.logpsi(model, p, r, s), R[w], S[w])
        assert (gr[w].cpu() - g0).abs().max() < 1e-10
        assert abs(complex(lap[w]) - complex(lap0)) < 1e-10 * max(1.0, abs(complex(lap0)))


@pytest.mark.parametrize("case", [(5, 7.0, 1.0, 0.5), (7, 8.0, 1.0, 0.5), (9, 9.0, 1.0, 0.0)])
def test_zero_variance_equals_Egs(case):
    """tests/test_nqs_local_energy.py:38-46, tightened to 1e-10: the zero-backflow Psiformer is
    the exact non-interacting eigenstate, so E_loc == E_gs at every (R, S)."""
    from nqs.local_energy import make_local_energy
    from nqs.psiformer import make_logpsi
    N, L, lr, hz = case
    g, model = build(N=N, L=L, lr=lr, hz=hz)
    p = model.init(0)
    R, S = configs(N, L, 24, 0)
    e = make_local_energy(make_logpsi(model, p), 1.0, lr, hz)(R, S).cpu()
    assert e.real.std() < 1e-10
    assert abs(e.real.mean() - g["E_gs"]) < 1e-10
    assert e.imag.abs().max() < 1e-10


def test_zeeman_polarised_limit():
    """tests/test_nqs_local_energy.py:49-66."""
    from nqs.local_energy import make_local_energy
    from nqs.psiformer import make_logpsi
    N, L, hz = 5, 9.0, 4.0
    g, model = build(N=N, L=L, lr=0.0, hz=hz)
    assert all(d["band"] == 0 for d in g["occ"])
    Kvecs, _ = rashba.occupied_orbital_matrix(g)
    R, _ = configs(N, L, 1, 1)
    S = torch.zeros(1, N, dtype=torch.int64)
    E = complex(make_local_energy(make_logpsi(model, model.init(0)), 1.0, 0.0, hz)(R, S)[0])
    Ekin = float(np.sum(np.sum(Kvecs ** 2, axis=1) / 2.0))
    assert abs(E.real - (Ekin - 0.5 * hz * N)) < 1e-10
    assert abs(E.real - g["E_gs"]) < 1e-10


@pytest.mark.parametrize("kw", [dict(), dict(n_dets=2, use_jastrow=True, n_knots=4)])
def test_local_energy_matches_oracle(kw):
    from nqs.local_energy import make_local_energy
    from nqs.psiformer import make_logpsi
    g, model = build(**kw)
    p = perturb(model.init(0), 0.05, 21)
    R, S = configs(model.n_elec, model.L, 3, 22)
    e = make_local_energy(make_logpsi(model, p), 1.0, 1.0, 0.5)(R, S).cpu()
    for w in range(3):
        ref = O.local_energy(lambda r, s: O.logpsi(model, p, r, s), R[w], S[w], 1.0, 1.0, 0.5)
        assert abs(complex(e[w]) - complex(ref)) < 1e-10 * max(1.0, abs(complex(ref)))
