"""Metropolis MCMC over (positions, spins) on the torus (drop-in for src/nqs/sampler.py:25-98).

A sweep = one joint all-electron Gaussian position proposal (PBC wrapped) + ``n_spin_flips``
single-spin flips, each accepted iff u < exp(min(0, 2 Re dlog psi)). Each sweep runs as fused
libnqs kernels over all walkers (``nqs_mcmc_sweeps``): proposal, wavefunction ratio and accept,
with counter-based Philox4x32-10 randomness (or injected proposals / uniforms for parity tests).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .cell import cell_matrix
from .psiformer import LogPsi, as_batch
from .random import as_key, key_to_seed, split


def _check_cell(logpsi: LogPsi, cell):
    A = cell_matrix(cell)
    if not np.allclose(A, cell_matrix(logpsi.model.L), rtol=0, atol=1e-12):
        raise ValueError("the sampler cell must equal the wavefunction's cell")


def mcmc_sweeps(logpsi: LogPsi, R, S, n_sweeps, step, seed, counter, n_spin_flips=2,
                inj_normals=None, inj_u_pos=None, inj_flip_idx=None, inj_u_flip=None,
                return_d=False):
    """Run n_sweeps sweeps on a batch IN PLACE-style: returns new (R, S, acc_pos (W,),
    acc_spin (W,), logpsi (W,)[, d]). R (W,N,2), S (W,N) are device tensors (copied)."""
    R, S, _ = as_batch(R, S)
    R, S = R.clone(), S.clone()
    W, N = R.shape[0], R.shape[1]
    dev = R.device
    h = logpsi.model.native().handle
    acc_p = torch.empty(W, dtype=torch.float64, device=dev)
    acc_s = torch.empty(W, dtype=torch.float64, device=dev)
    lp = torch.empty(W, dtype=torch.complex128, device=dev)
    d = (torch.empty(n_sweeps, 1 + n_spin_flips, W, dtype=torch.float64, device=dev)
         if return_d else None)

    def dv(x, dt):
        return None if x is None else torch.as_tensor(x).to(dev, dt).contiguous()

    inj = [dv(inj_normals, torch.float64), dv(inj_u_pos, torch.float64),
           dv(inj_flip_idx, torch.int32), dv(inj_u_flip, torch.float64)]
    ws, _ = _lib.workspace_for(h, _lib.OP_MCMC, W, logpsi.precision)
    _lib.check(_lib.lib().nqs_mcmc_sweeps(
        h, _lib.ptr(logpsi.theta), _lib.ptr(R), _lib.ptr(S), _lib.ptr(lp), W, int(n_sweeps),
        int(n_spin_flips), float(step), int(seed) & ((1 << 64) - 1),
        int(counter) & ((1 << 64) - 1), *[_lib.ptr(x) for x in inj], _lib.ptr(acc_p),
        _lib.ptr(acc_s), _lib.ptr(d), logpsi.precision, _lib.ptr(ws), ws.numel(),
        _lib.stream_ptr()), "nqs_mcmc_sweeps")
    if return_d:
        return R, S, acc_p, acc_s, lp, d
    return R, S, acc_p, acc_s, lp


def make_mcmc(logpsi, cell, n_elec, n_spin_flips=2):
    """Return sweep(key, R, S, step) -> (R', S', acc_pos, acc_spin) (sampler.py:25-59).
    Works on one walker (R (N,2)) or a batch (R (W,N,2))."""
    if not isinstance(logpsi, LogPsi):
        raise NotImplementedError("make_mcmc needs a logpsi from nqs.psiformer.make_logpsi")
    _check_cell(logpsi, cell)

    def sweep(key, R, S, step):
        single = torch.as_tensor(R).dim() == 2
        s, c = as_key(key)
        Rn, Sn, ap, asp, _ = mcmc_sweeps(logpsi, R, S, 1, step, key_to_seed((s, 0)), c,
                                         n_spin_flips)
        if single:
            return Rn[0], Sn[0], ap[0], asp[0]
        return Rn, Sn, ap, asp

    return sweep


def init_walkers_uniform(key, n_walkers, n_elec, cell):
    """R ~ U(cell) (fractional uniform mapped by A), S ~ U{0,1}, on the device."""
    A = torch.as_tensor(cell_matrix(cell), dtype=torch.float64)
    g = torch.Generator().manual_seed(key_to_seed(key))
    R = torch.rand(n_walkers, n_elec, 2, generator=g, dtype=torch.float64) @ A.T
    S = torch.randint(0, 2, (n_walkers, n_elec), generator=g, dtype=torch.int32)
    dev = _lib.device()
    return R.to(dev), S.to(dev)


def run_chain(logpsi, cell, n_elec, key, n_walkers=256, n_sweeps=200, burn=100, step=0.4,
              n_spin_flips=2, R0=None, S0=None):
    """Batched MCMC; returns (R, S, accept_pos, accept_spin) after burn-in (sampler.py:62-91)."""
    _check_cell(logpsi, cell)
    k0, k1, k2 = split(as_key(key), 3)
    R, S = init_walkers_uniform(k0, n_walkers, n_elec, cell)
    dev = _lib.device()
    if R0 is not None:
        R = torch.as_tensor(R0, dtype=torch.float64).to(dev).expand(n_walkers, n_elec, 2).clone()
    if S0 is not None:
        S = torch.as_tensor(S0).to(dev, torch.int32).expand(n_walkers, n_elec).clone()
    seed = key_to_seed(k2)
    R, S, *_ = mcmc_sweeps(logpsi, R, S, burn, step, seed, 0, n_spin_flips)
    R, S, ap, asp, _ = mcmc_sweeps(logpsi, R, S, n_sweeps, step, seed, burn, n_spin_flips)
    return R, S, float(ap.mean()), float(asp.mean())


def vmc_energy(E_loc, R, S):
    """Mean local energy + standard error over the ensemble (sampler.py:94-98)."""
    e = E_loc(R, S)
    er = e.real
    return float(er.mean()), float(er.std(unbiased=False) / np.sqrt(er.shape[0])), e
