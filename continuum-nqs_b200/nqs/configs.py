"""The synthetic benchmark configurations of the VMC iteration.

config1: N=2 electrons, r_s=2 (L = sqrt(pi N) r_s), Rashba 0.5, Zeeman 0.1; width 32, 2 blocks,
         4 heads, 8 Fourier harmonics, K=1, no Jastrow; 256 walkers, Gaussian step 0.2 r_s,
         10 sweeps, MinSR damping 1e-3, lr 0.05; flax-default initialisation, zero backflow.
config2: N=16, r_s=5, Rashba 0.3, Zeeman 0.05; width 64, 4 blocks, 4 heads, 8 harmonics, K=4,
         RBF pair Jastrow with 16 centres; Bloch envelopes of the non-interacting Rashba orbitals
         (twist (0.1, 0.17), where the closed shell has a gap); Dense kernels ~N(0, 0.02^2),
         backflow ~N(0, 1e-3^2), Jastrow ~N(0, 0.02^2); 4096 walkers; step 0.2 r_s; 10 sweeps.
config3: the configuration-2 model and walkers with MinSR damping 1e-4 and the per-block
         checkpointed reverse pass for the per-sample Jacobian.
config5: N=48, r_s=5, Rashba 0.3, Zeeman 0.05; width 128, 6 blocks, 8 heads, 8 harmonics, K=8,
         RBF pair Jastrow with 16 centres; Bloch envelopes at zero twist (the closed shell's gap
         there is 3.8e-4 Ha, against 5.1e-6 at twist (0.1, 0.17)); initialisation as
         configuration 2; 8192 walkers, 20 sweeps; checkpointed reverse pass.
config4: 64 independent VMC instances (config4_instances): electron counts drawn uniformly from
         {6, 8, ..., 26}, walkers from {512, 640, ..., 4096}, r_s in [2, 10], Rashba in
         [0, 0.8], Zeeman in [0, 0.2]; width 64, 3 blocks, 4 heads, 8 harmonics, K = 2, no
         Jastrow; twist (0.1, 0.17) envelopes; initialisation as configuration 2.
All: Coulomb coupling 1 through the 2D Ewald sum with eta = 5/L, 7x7 real-space images
(n_real = 3) and the |m| <= 8 reciprocal index box; 2 spin-flip proposals per sweep.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

from . import rashba
from .psiformer import ContinuumSpinorPsiformer


@dataclass
class VMCSetup:
    name: str
    N: int
    L: float
    lambda_r: float
    h_z: float
    n_walkers: int
    n_sweeps: int
    step: float
    lam: float
    lr: float
    ewald_eta: float
    n_real: int = 3
    n_recip: int = 8
    E_gs: float = 0.0
    checkpoint_blocks: bool = False


def config(n: int, n_walkers: int | None = None):
    """(model, params, setup) of configuration n (1, 2, 3 or 5)."""
    if n == 1:
        N, rs, lr_soc, hz = 2, 2.0, 0.5, 0.1
        L = math.sqrt(math.pi * N) * rs
        env = rashba.cell_rashba_envelope(L, N, 1.0, lr_soc, hz, 10, (0.0, 0.0))
        model = ContinuumSpinorPsiformer(N, env["Gs"], env["W"], L, embed_dim=32, depth=2,
                                         n_heads=4, n_freq=8, n_dets=1)
        params = model.init(0)
        W = 256
    elif n in (2, 3):
        N, rs, lr_soc, hz = 16, 5.0, 0.3, 0.05
        L = math.sqrt(math.pi * N) * rs
        env = rashba.cell_rashba_envelope(L, N, 1.0, lr_soc, hz, 10, (0.1, 0.17))
        model = ContinuumSpinorPsiformer(N, env["Gs"], env["W"], L, embed_dim=64, depth=4,
                                         n_heads=4, n_freq=8, n_dets=4, use_jastrow=True,
                                         n_knots=16)
        params = model.init_normal(0, std=0.02, backflow_std=1e-3, jastrow_std=0.02)
        W = 4096
    elif n == 5:
        N, rs, lr_soc, hz = 48, 5.0, 0.3, 0.05
        L = math.sqrt(math.pi * N) * rs
        env = rashba.cell_rashba_envelope(L, N, 1.0, lr_soc, hz, 10, (0.0, 0.0))
        model = ContinuumSpinorPsiformer(N, env["Gs"], env["W"], L, embed_dim=128, depth=6,
                                         n_heads=8, n_freq=8, n_dets=8, use_jastrow=True,
                                         n_knots=16)
        params = model.init_normal(0, std=0.02, backflow_std=1e-3, jastrow_std=0.02)
        W = 8192
    else:
        raise ValueError(f"unknown configuration {n}")
    setup = VMCSetup(f"config{n}", N, L, lr_soc, hz, n_walkers or W, 20 if n == 5 else 10,
                     0.2 * rs, 1e-4 if n == 3 else 1e-3, 0.05, 5.0 / L, E_gs=env["E_gs"],
                     checkpoint_blocks=n in (3, 5))
    return model, params, setup


def config4_instances(n_instances: int = 64, seed: int = 0, scale_walkers: float = 1.0):
    """The configuration-4 batch: a list of nqs.batched.Instance (model, theta, uniform walkers,
    VMCIteration keyword arguments with the instance's own Hamiltonian and Ewald sum).
    scale_walkers < 1 shrinks every walker count (multiples of 128 kept) for tests."""
    import numpy as np
    from .batched import Instance
    from .ewald import make_ewald
    from .sampler import init_walkers_uniform
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_instances):
        N = int(rng.choice(np.arange(6, 27, 2)))
        W = int(rng.choice(np.arange(512, 4097, 128)))
        W = max(128, int(round(W * scale_walkers / 128.0)) * 128)
        rs = float(rng.uniform(2.0, 10.0))
        lam_r = float(rng.uniform(0.0, 0.8))
        hz = float(rng.uniform(0.0, 0.2))
        L = math.sqrt(math.pi * N) * rs
        env = rashba.cell_rashba_envelope(L, N, 1.0, lam_r, hz, 8, (0.1, 0.17))
        model = ContinuumSpinorPsiformer(N, env["Gs"], env["W"], L, embed_dim=64, depth=3,
                                         n_heads=4, n_freq=8, n_dets=2)
        params = model.init_normal(1000 + i, std=0.02, backflow_std=1e-3)
        R, S = init_walkers_uniform(7919 * (i + 1), W, N, L)
        _, _, coul = make_ewald(L, alpha=1.0, ewald_alpha=5.0 / L, n_real=3, n_recip=8)
        kw = dict(m_star=1.0, lambda_r=lam_r, h_z=hz, coulomb=coul, lr=0.05, lam=1e-3,
                  n_sweeps=10, step_size=0.2 * rs, clip_k=5.0, seed=101 + i)
        out.append(Instance(model, model.theta(params), R, S, kw))
    return out
