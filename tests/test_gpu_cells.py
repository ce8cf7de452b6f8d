"""Non-square cells (the reference accepts any 2x2 cell matrix A: src/nqs/cell.py:21-53,
psiformer.py:88,163-166, sampler.py:19-31): a triangular (hex) and a rectangular cell through the
features, minimum image, kinetic / spin-orbit terms and the periodic wrap of the sampler."""
import numpy as np
import pytest
import torch

from helpers import TWIST, perturb
from oracle import nqs_oracle as O

pytestmark = pytest.mark.gpu


def _model(A, N=5, lr=1.0, hz=0.5, **mkw):
    from nqs import rashba
    from nqs.psiformer import ContinuumSpinorPsiformer
    env = rashba.cell_rashba_envelope(A, N, 1.0, lr, hz, n_cut=8, twist=TWIST)
    model = ContinuumSpinorPsiformer(n_elec=N, Gs=env["Gs"], W=env["W"], L=A, embed_dim=16,
                                     depth=2, n_heads=4, n_freq=4, **mkw)
    return env, model


def _configs(A, N, n, seed):
    rng = np.random.default_rng(seed)
    f = rng.uniform(0.0, 1.0, (n, N, 2))
    R = torch.as_tensor(f @ np.asarray(A).T)  # uniform over the cell
    S = torch.as_tensor(rng.integers(0, 2, (n, N)))
    return R, S


def _cells():
    from nqs.cell import hex_cell, rect_cell
    return [hex_cell(8.0), rect_cell(6.0, 9.0)]


def _close_mod_2pi(a, b, tol):
    d = complex(a) - complex(b)
    return abs(d.real) < tol and abs((d.imag + np.pi) % (2 * np.pi) - np.pi) < tol


@pytest.mark.parametrize("ci", [0, 1])
def test_logpsi_general_cell_matches_oracle(ci):
    from nqs.psiformer import make_logpsi
    A = _cells()[ci]
    env, model = _model(A, n_dets=2, use_jastrow=True, n_knots=5)
    p = perturb(model.init(0), 0.05, 51)
    R, S = _configs(A, model.n_elec, 5, 52)
    lp = make_logpsi(model, p)(R, S).cpu()
    for w in range(5):
        assert _close_mod_2pi(lp[w], O.logpsi(model, p, R[w], S[w]), 1e-11)
    # shifting one electron by a lattice vector: |psi| unchanged (the twisted boundary condition
    # changes only the phase), and the shifted configuration still matches the oracle
    R2 = R.clone()
    R2[:, 2] += torch.as_tensor(np.asarray(A)[:, 1])
    l2 = make_logpsi(model, p)(R2, S).cpu()
    for w in range(5):
        assert abs(float(l2[w].real - lp[w].real)) < 1e-9
        assert _close_mod_2pi(l2[w], O.logpsi(model, p, R2[w], S[w]), 1e-10)


@pytest.mark.parametrize("ci", [0, 1])
def test_zero_variance_general_cell(ci):
    """Zero backflow and no Jastrow: the Psiformer is the non-interacting eigenstate of the cell,
    so E_loc == E_gs at every configuration (kinetic, Rashba and Zeeman terms on a general A)."""
    from nqs.local_energy import make_local_energy
    from nqs.psiformer import make_logpsi
    A = _cells()[ci]
    env, model = _model(A)
    R, S = _configs(A, model.n_elec, 16, 53)
    e = make_local_energy(make_logpsi(model, model.init(0)), 1.0, 1.0, 0.5)(R, S).cpu()
    assert e.real.std() < 1e-10
    assert abs(float(e.real.mean()) - env["E_gs"]) < 1e-10


def test_local_energy_hex_matches_oracle():
    from nqs.local_energy import make_local_energy
    from nqs.psiformer import make_logpsi
    A = _cells()[0]
    env, model = _model(A, n_dets=2, use_jastrow=True, n_knots=4)
    p = perturb(model.init(0), 0.05, 54)
    R, S = _configs(A, model.n_elec, 3, 55)
    e = make_local_energy(make_logpsi(model, p), 1.0, 1.0, 0.5)(R, S).cpu()
    for w in range(3):
        ref = O.local_energy(lambda r, s: O.logpsi(model, p, r, s), R[w], S[w], 1.0, 1.0, 0.5)
        assert abs(complex(e[w]) - complex(ref)) < 1e-10 * max(1.0, abs(complex(ref)))


def test_metropolis_hex_matches_oracle_injected():
    """Wrap into the triangular cell (fractional coordinates) and the accept rule, given the same
    injected proposals and uniforms."""
    from nqs.psiformer import make_logpsi
    from nqs.sampler import mcmc_sweeps
    A = _cells()[0]
    env, model = _model(A, n_dets=2, use_jastrow=True, n_knots=4)
    p = perturb(model.init(0), 0.05, 56)
    Wn, N, ns, nf = 4, model.n_elec, 3, 2
    R, S = _configs(A, N, Wn, 57)
    rng = np.random.default_rng(58)
    nrm = rng.standard_normal((ns, Wn, N, 2)) * 2.0  # large steps: many moves cross the boundary
    up = rng.uniform(size=(ns, Wn))
    fi = rng.integers(0, N, (ns, nf, Wn)).astype(np.int32)
    uf = rng.uniform(size=(ns, nf, Wn))
    Rg, Sg, ap, asp, Lg, d = mcmc_sweeps(make_logpsi(model, p), R, S, ns, 0.6, 0, 0, nf, nrm, up,
                                         fi, uf, return_d=True)
    Rg, Sg, d = Rg.cpu(), Sg.cpu(), d.cpu().numpy()
    f = lambda r, s: O.logpsi(model, p, r, s)  # noqa: E731
    for w in range(Wn):
        Rw, Sw, Lc = R[w].clone(), S[w].clone(), None
        for s in range(ns):
            Rw, Sw, acc, nacc, Lc, ds = O.mcmc_sweep(
                f, A, Rw, Sw, 0.6, torch.as_tensor(nrm[s, w]), up[s, w], fi[s, :, w],
                uf[s, :, w], Lc)
            assert np.abs(np.array(ds) - d[s, :, w]).max() < 1e-10
        assert torch.equal(Sg[w], Sw.to(Sg.dtype)), w
        assert (Rg[w] - Rw).abs().max() < 1e-12, w
