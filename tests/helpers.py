"""Shared builders for the tests (mirrors the module-level builders of the reference tests,
e.g. tests/test_nqs_psiformer.py:24-33, tests/test_nqs_minsr.py:22-29)."""
from __future__ import annotations

import numpy as np
import torch

from nqs import rashba
from nqs.psiformer import ContinuumSpinorPsiformer

TWIST = (0.1, 0.17)


def build(N=5, L=7.0, lr=1.0, hz=0.5, embed=16, depth=2, heads=4, n_freq=4, **mkw):
    g = rashba.noninteracting_gs(N=N, L=L, m_star=1.0, lambda_r=lr, h_z=hz, n_cut=10, twist=TWIST)
    Kvecs, Chi = rashba.occupied_orbital_matrix(g)
    Gs, W = rashba.planewave_envelope(Kvecs, Chi)
    model = ContinuumSpinorPsiformer(n_elec=N, Gs=Gs, W=W, L=L, embed_dim=embed, depth=depth,
                                     n_heads=heads, n_freq=n_freq, **mkw)
    return g, model


def perturb(params, scale, seed, only=None):
    """Add scale * N(0,1) noise (complex leaves get re and im noise) to every leaf whose path
    contains `only` (all leaves if None)."""
    rng = np.random.default_rng(seed)

    def walk(node, path):
        out = {}
        for k, v in node.items():
            if isinstance(v, dict):
                out[k] = walk(v, path + (k,))
            else:
                if only is None or only in path + (k,):
                    n = torch.as_tensor(rng.standard_normal(tuple(v.shape)))
                    if v.is_complex():
                        n = torch.complex(n, torch.as_tensor(rng.standard_normal(tuple(v.shape))))
                    v = v + scale * n.to(v.dtype)
                out[k] = v
        return out

    return {"params": walk(params["params"], ())}


def configs(N, L, n, seed):
    rng = np.random.default_rng(seed)
    R = torch.as_tensor(rng.uniform(0, L, (n, N, 2)))
    S = torch.as_tensor(rng.integers(0, 2, (n, N)))
    return R, S
