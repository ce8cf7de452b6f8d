"""Metropolis kernels: accept decisions against the oracle given identical proposals and
uniforms, the Philox stream against a host restatement, and the reference's statistical checks
(src/nqs/sampler.py:25-98; tests/test_nqs_sampler.py:31-56)."""
import numpy as np
import pytest
import torch

from helpers import build, configs, perturb
from oracle import nqs_oracle as O

pytestmark = pytest.mark.gpu

M32 = 0xFFFFFFFF


def philox4x32_10(ctr, key):
    """Philox4x32-10 (Salmon et al. 2011), host restatement for the stream check."""
    x, y, z, w = ctr
    k0, k1 = key & M32, key >> 32
    for _ in range(10):
        p0 = 0xD2511F53 * x
        p1 = 0xCD9E8D57 * z
        x, y, z, w = ((p1 >> 32) ^ y ^ k0) & M32, p1 & M32, ((p0 >> 32) ^ w ^ k1) & M32, p0 & M32
        k0 = (k0 + 0x9E3779B9) & M32
        k1 = (k1 + 0xBB67AE85) & M32
    return x, y, z, w


def u53(a, b):
    return (((a << 32) | b) >> 11) * (1.0 / 9007199254740992.0)


def test_accept_decisions_match_oracle_injected():
    from nqs.psiformer import make_logpsi
    from nqs.sampler import mcmc_sweeps
    g, model = build(n_dets=2, use_jastrow=True, n_knots=4)
    p = perturb(model.init(0), 0.05, 3)
    Wn, N, ns, nf = 6, model.n_elec, 3, 2
    R, S = configs(N, model.L, Wn, 4)
    rng = np.random.default_rng(9)
    nrm = rng.standard_normal((ns, Wn, N, 2))
    up = rng.uniform(size=(ns, Wn))
    fi = rng.integers(0, N, (ns, nf, Wn)).astype(np.int32)
    uf = rng.uniform(size=(ns, nf, Wn))
    lp = make_logpsi(model, p)
    Rg, Sg, ap, asp, Lg, d = mcmc_sweeps(lp, R, S, ns, 0.6, 0, 0, nf, nrm, up, fi, uf,
                                         return_d=True)
    Rg, Sg, d = Rg.cpu(), Sg.cpu(), d.cpu().numpy()
    f = lambda r, s: O.logpsi(model, p, r, s)  # noqa: E731
    for w in range(Wn):
        Rw, Sw, Lc = R[w].clone(), S[w].clone(), None
        for s in range(ns):
            Rw, Sw, acc, nacc, Lc, ds = O.mcmc_sweep(
                f, model.L, Rw, Sw, 0.6, torch.as_tensor(nrm[s, w]), up[s, w], fi[s, :, w],
                uf[s, :, w], Lc)
            assert np.abs(np.array(ds) - d[s, :, w]).max() < 1e-10
            # device d reproduces the device decision with the host's exp (bit-exact rule)
        assert torch.equal(Sg[w], Sw.to(Sg.dtype)), w
        assert (Rg[w] - Rw).abs().max() < 1e-12, w


def test_philox_stream_matches_host():
    from nqs.psiformer import make_logpsi
    from nqs.sampler import mcmc_sweeps
    g, model = build()
    lp = make_logpsi(model, model.init(0))
    Wn, N = 5, 5
    R, S = configs(N, model.L, Wn, 1)
    seed, counter, step = 1234567, 77, 0.5
    Rg, Sg, ap, asp, Lg, d = mcmc_sweeps(lp, R, S, 1, step, seed, counter, 0, return_d=True)
    Rg = Rg.cpu().numpy()
    d = d.cpu().numpy()
    L = model.L
    for w in range(Wn):
        prop = np.zeros((N, 2))
        for i in range(N):
            x, y, z, ww = philox4x32_10((w, i, counter & M32, counter >> 32), seed)
            u1, u2 = u53(x, y), u53(z, ww)
            rad = np.sqrt(-2.0 * np.log(1.0 - u1))
            n0, n1 = rad * np.cos(2 * np.pi * u2), rad * np.sin(2 * np.pi * u2)
            prop[i] = np.mod((R[w, i].numpy() + step * np.array([n0, n1])) / L, 1.0) * L
        x, y, _, _ = philox4x32_10((w, N, counter & M32, counter >> 32), seed)
        acc = u53(x, y) < np.exp(min(0.0, d[0, 0, w]))
        expect = prop if acc else R[w].numpy()
        assert np.abs(Rg[w] - expect).max() < 1e-12


def test_sampled_energy_equals_Egs():
    """tests/test_nqs_sampler.py:31-37 on the zero-backflow Psiformer (== the Slater trial)."""
    from nqs.local_energy import make_local_energy
    from nqs.psiformer import make_logpsi
    from nqs.sampler import run_chain, vmc_energy
    g, model = build(N=7, L=8.0)
    lp = make_logpsi(model, model.init(0))
    R, S, ap, asp = run_chain(lp, model.L, 7, 0, n_walkers=256, n_sweeps=120, burn=120, step=0.5)
    Em, Ee, _ = vmc_energy(make_local_energy(lp, 1.0, 1.0, 0.5), R, S)
    assert 0.1 < ap < 0.95
    assert abs(Em - g["E_gs"]) < 1e-9


def test_density_is_uniform():
    """tests/test_nqs_sampler.py:40-56: binned density of a plane-wave determinant is uniform
    at the Poisson level."""
    from nqs.psiformer import make_logpsi
    from nqs.sampler import run_chain
    g, model = build(N=9, L=9.0)
    lp = make_logpsi(model, model.init(0))
    R, S, ap, asp = run_chain(lp, 9.0, 9, 1, n_walkers=2048, n_sweeps=300, burn=200, step=0.5)
    pos = R.cpu().numpy().reshape(-1, 2) % 9.0
    H, _, _ = np.histogram2d(pos[:, 0], pos[:, 1], bins=6, range=[[0, 9.0], [0, 9.0]])
    rel, pois = np.std(H) / H.mean(), 1.0 / np.sqrt(H.mean())
    assert rel < 1.8 * pois
