"""The benchmark configurations' exact models against the float64 oracle, and one whole VMC
iteration against the oracle's (reference src/nqs/minsr.py:139-156: sample, E_loc with the Ewald
term, O, median-MAD clip, MinSR direction, theta -= lr dtheta) with the same injected proposals
and uniforms."""
import numpy as np
import pytest
import torch

from oracle import nqs_oracle as O

pytestmark = pytest.mark.gpu


def _setup(n):
    from nqs.configs import config
    from nqs.ewald import make_ewald
    model, params, su = config(n, 8)
    _, _, coul = make_ewald(su.L, alpha=1.0, ewald_alpha=su.ewald_eta, n_real=su.n_real,
                            n_recip=su.n_recip)
    ew = O.Ewald(su.L, 1.0, su.ewald_eta, su.n_real, su.n_recip)
    return model, params, su, coul, ew


def _walkers(su, W, seed):
    """Uniform positions and spins; at configuration 1 the two occupied orbitals are the two
    k = 0 spinors, so psi vanishes when both spins agree: those walkers get opposite spins (the
    sampler never visits a node)."""
    rng = np.random.default_rng(seed)
    R = torch.as_tensor(rng.uniform(0, su.L, (W, su.N, 2)))
    S = torch.as_tensor(rng.integers(0, 2, (W, su.N)))
    if su.N == 2:
        S[:, 1] = 1 - S[:, 0]
    return R, S


@pytest.mark.parametrize("cfg,W", [(1, 8), (2, 4)])
def test_config_model_logpsi_eloc_O_match_oracle(cfg, W):
    """log psi (1e-11), E_loc including Ewald at eta = 5/L, n_real 3, n_recip 8 against the
    dense-Hessian oracle (1e-10), and O against the oracle's reverse mode (1e-10), at the exact
    configuration-1 (d 32, 2 blocks, 8 harmonics, K 1) and configuration-2 (N 16, d 64, 4 blocks,
    4 heads, K 4, 16-knot Jastrow) models."""
    from nqs.local_energy import make_local_energy
    from nqs.minsr import per_sample_O, real_ravel
    from nqs.psiformer import make_logpsi
    model, params, su, coul, ew = _setup(cfg)
    R, S = _walkers(su, W, 100 + cfg)
    lp = make_logpsi(model, params)
    L = lp(R, S).cpu()
    E = make_local_energy(lp, 1.0, su.lambda_r, su.h_z, coulomb=coul)(R, S).cpu()
    f = lambda r, s: O.logpsi(model, params, r, s)  # noqa: E731
    for w in range(W):
        lo = complex(f(R[w], S[w]))
        d = complex(L[w]) - lo
        assert abs(d.real) < 1e-11 * max(1.0, abs(lo.real))
        assert abs((d.imag + np.pi) % (2 * np.pi) - np.pi) < 1e-11
        eo = complex(O.local_energy(f, R[w], S[w], 1.0, su.lambda_r, su.h_z)) \
            + ew.energy(R[w].numpy())
        assert abs(complex(E[w]) - eo) < 1e-10 * max(1.0, abs(eo)), (w, complex(E[w]), eo)
    theta, unravel = real_ravel(params)
    Og = per_sample_O(model, theta.cuda(), unravel, R, S).cpu()
    ot, ou = O.real_ravel(params["params"])
    Oo = O.per_sample_O(model, ot, ou, R, S)
    assert float((Og - Oo).abs().max()) < 1e-10 * max(1.0, float(Oo.abs().max()))


def test_whole_iteration_matches_oracle_config1():
    """One VMCIteration.step() at configuration 1 (W = 8) with injected proposals and uniforms
    equals oracle.vmc_iteration on the same draws: walkers R to 1e-12 and S exactly after the
    sweeps, local energies to 1e-10, theta after the update to 1e-9 relative to the step."""
    from nqs.minsr import VMCIteration, real_ravel
    model, params, su, coul, ew = _setup(1)
    W, N, n_sw, nf = 8, su.N, su.n_sweeps, 2
    R, S = _walkers(su, W, 7)
    rng = np.random.default_rng(8)
    draws = (rng.standard_normal((n_sw, W, N, 2)), rng.uniform(size=(n_sw, W)),
             rng.integers(0, N, (n_sw, nf, W)).astype(np.int32), rng.uniform(size=(n_sw, nf, W)))
    theta, unravel = real_ravel(params)
    it = VMCIteration(model, theta, R, S, m_star=1.0, lambda_r=su.lambda_r, h_z=su.h_z,
                      coulomb=coul, lr=su.lr, lam=su.lam, n_sweeps=n_sw, step_size=su.step,
                      clip_k=5.0, n_spin_flips=nf, seed=3)
    it.step(inject=draws)
    th_dev = it.theta.cpu()
    ot, ou = O.real_ravel(params["params"])
    Ro, So = R.clone(), S.clone()
    th_o, Ro, So, eo = O.vmc_iteration(model, ot, ou, Ro, So, A=su.L, step=su.step,
                                       n_sweeps=n_sw, n_spin_flips=nf, rng=None, m_star=1.0,
                                       lambda_r=su.lambda_r, h_z=su.h_z, ewald=ew, lam=su.lam,
                                       lr=su.lr, clip_k=5.0, draws=draws)
    assert torch.equal(it.S.cpu().long(), So.long())
    assert float((it.R.cpu() - Ro).abs().max()) < 1e-12
    assert float((it.e.cpu() - eo).abs().max()) < 1e-10 * max(1.0, float(eo.abs().max()))
    step_o = (th_o - ot).norm()
    assert float((th_dev - th_o).norm() / step_o) < 1e-9, float((th_dev - th_o).norm() / step_o)
