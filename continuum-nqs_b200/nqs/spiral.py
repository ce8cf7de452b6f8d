"""Exact non-interacting spin-spiral ground state and its field (host-side setup).

Restates the reference module src/nqs/spiral_reference.py (spiral_gs :24-65, spiral_field
:68-75), which imports JAX and cannot run here. Single-particle Hamiltonian:

    h = h0(k) - B (sigma_x cos Q.r + sigma_y sin Q.r),     Q = (2 pi / L) Q_int

with h0 the Rashba + Zeeman block of nqs.rashba.h0_k. In the plane-wave basis |k, s> with
k = (2 pi n + twist)/L, |n_x|, |n_y| <= n_cut, the field term couples |k, up> to |k + Q, down>
with amplitude -B (and the Hermitian conjugate). The N lowest eigenvectors form a Slater
determinant given as a multi-plane-wave envelope (Gs, W) for the Psiformer; its local energy with
ext_field = spiral_field(B, Q) equals E_gs at every configuration when the basis is converged
(boundary_weight, the occupied weight on the outermost plane waves, ~0).
"""
from __future__ import annotations

import numpy as np
import torch

from .rashba import h0_k


def spiral_gs(N, L, Q_int, B, m_star=1.0, lambda_r=1.0, h_z=0.0, n_cut=6, twist=(0.0, 0.0)):
    qx, qy = int(Q_int[0]), int(Q_int[1])
    Q = (2.0 * np.pi * qx / L, 2.0 * np.pi * qy / L)
    ns = np.arange(-n_cut, n_cut + 1)
    grid = [(int(a), int(b)) for a in ns for b in ns]
    where = {nm: p for p, nm in enumerate(grid)}
    npw = len(grid)
    if 2 * npw < N + 1:
        raise ValueError("basis too small for N")
    kx = np.array([(2.0 * np.pi * a + twist[0]) / L for a, _ in grid])
    ky = np.array([(2.0 * np.pi * b + twist[1]) / L for _, b in grid])
    H = np.zeros((2 * npw, 2 * npw), dtype=complex)
    for p in range(npw):
        H[2 * p:2 * p + 2, 2 * p:2 * p + 2] = h0_k(kx[p], ky[p], m_star, lambda_r, h_z)
    for p, (a, b) in enumerate(grid):
        q = where.get((a + qx, b + qy))
        if q is not None:  # <k+Q, down| h |k, up> = -B and its conjugate
            H[2 * q + 1, 2 * p] += -B
            H[2 * p, 2 * q + 1] += -B
    E, V = np.linalg.eigh(H)
    occ = V[:, :N]
    Gs = np.stack([kx, ky], axis=-1)
    W = occ.T.reshape(N, npw, 2).copy()  # W[a, g, s] = <g, s | orbital a>
    edge = np.array([abs(a) == n_cut or abs(b) == n_cut for a, b in grid])
    bweight = float(np.sum(np.abs(occ.reshape(npw, 2, N)[edge]) ** 2))
    return dict(E_gs=float(np.sum(E[:N])), gap=float(E[N] - E[N - 1]), Gs=Gs, W=W, N=N, L=L,
                Q=Q, Q_int=(qx, qy), B=float(B), m_star=m_star, lambda_r=lambda_r, h_z=h_z,
                twist=twist, boundary_weight=bweight, cutoff_ok=bool(bweight < 1e-13))


def spiral_field(B, Q):
    """ext_field for make_local_energy: positions (..., 2) -> (B cos Q.r, B sin Q.r, 0)."""
    Qx, Qy = float(Q[0]), float(Q[1])

    def f(R):
        R = torch.as_tensor(R)
        ph = Qx * R[..., 0] + Qy * R[..., 1]
        return torch.stack([B * torch.cos(ph), B * torch.sin(ph), torch.zeros_like(ph)], dim=-1)
    return f
