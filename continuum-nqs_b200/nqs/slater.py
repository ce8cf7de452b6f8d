"""Spinor Slater-determinant trial wavefunctions on the device (drop-in for the reference's
src/nqs/slater_reference.py: make_logpsi_general :21-37, make_logpsi_slater :40-45).

    phi_a(r, s) = sum_G W[a, G, s] exp(i G . r),     Psi(R, S) = det[phi_a(r_i, s_i)]

Realised as the network with this envelope and its backflow, determinant weights and Jastrow
absent or zero: the backflow-dressed orbital matrix env (1 + 0) is then exactly the Slater matrix,
so log psi, the local energy and the Metropolis sweeps of these callables are the Slater
determinant's, through the same kernels as every other wavefunction. Adaptation forced by the
device path: the callables carry a cell (`cell`, default the unit square), which the Slater
determinant itself does not depend on but the sampler checks its own cell against; pass the
simulation cell when the callable is sampled.
"""
from __future__ import annotations

import numpy as np

from .psiformer import ContinuumSpinorPsiformer, make_logpsi
from .rashba import planewave_envelope


def slater_model(Gs, W, cell=None):
    """(model, params) whose log psi is the Slater determinant of (Gs, W)."""
    Gs = np.asarray(Gs, dtype=float).reshape(-1, 2)
    W = np.asarray(W, dtype=complex)
    model = ContinuumSpinorPsiformer(n_elec=W.shape[0], Gs=Gs, W=W,
                                     L=1.0 if cell is None else cell, embed_dim=8, depth=1,
                                     n_heads=2, n_freq=1, n_dets=1, use_jastrow=False)
    return model, model.init(0)  # zero-initialised backflow and determinant weights


def make_logpsi_general(Gs, W, cell=None):
    """logpsi(R, S) of the multi-plane-wave spinor determinant, Gs (n_G, 2), W (N, n_G, 2)."""
    model, params = slater_model(Gs, W, cell)
    return make_logpsi(model, params)


def make_logpsi_slater(Kvecs, Chi, cell=None):
    """One plane wave per orbital, phi_a(r, s) = exp(i K_a . r) chi_a(s)."""
    Gs, W = planewave_envelope(Kvecs, Chi)
    return make_logpsi_general(Gs, W, cell)
