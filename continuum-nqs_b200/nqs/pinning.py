"""Pinning fields: external spin fields that seed a competing order (host-side setup).

Restates the reference module src/nqs/pinning.py (make_skx_pin :22-42, make_fm_pin :45-51,
make_spiral_pin :54-67, make_overhauser_pin :70-78, make_pin :112-129), which imports JAX. A pinning field
adds H_pin = -sum_i B(r_i) . sigma_i to the Hamiltonian; the constructors return the ext_field
B(r) that nqs.local_energy.make_local_energy(..., ext_field=...) takes (and evaluates on the
device at the walkers' positions): a callable vectorised over positions, torch (..., 2) ->
(..., 3), same device and dtype as its input.

Targets: "skx" (triple-Q Neel skyrmion, in-plane component along q_hat; "skx_bloch" the Bloch
control, along z_hat x q_hat), "spiral" (single-Q cycloid in the z_hat-q_hat plane;
"spiral_xy" the flat in-plane helix), "overhauser" (collinear z spin-density wave), "fm"
(uniform axis) and "fluid" (no field).
"""
from __future__ import annotations

import numpy as np
import torch

_EPS = 1e-12  # added to |m| before normalising a texture


def _vec(x):
    return np.asarray(x, dtype=float).reshape(-1)


def _unit(m, h_pin):
    """h_pin m / (|m| + 1e-12) along the last axis."""
    return h_pin * m / (torch.linalg.vector_norm(m, dim=-1, keepdim=True) + _EPS)


def make_skx_pin(q1, q2, h_pin, m0=0.3, chirality=1.0, neel=True):
    """h_pin times the unit triple-Q texture with arms q1, q2, q3 = -(q1 + q2):
        m_z = m0 + sum_j cos(q_j . r),  m_par = chirality sum_j sin(q_j . r) e_j,
    e_j = q_hat_j (Neel, the Rashba-favoured chirality) or z_hat x q_hat_j (Bloch)."""
    q1, q2 = _vec(q1), _vec(q2)
    qs = np.stack([q1, q2, -(q1 + q2)])                     # (3, 2)
    qh = qs / np.linalg.norm(qs, axis=1, keepdims=True)
    eh = qh if neel else np.stack([-qh[:, 1], qh[:, 0]], axis=1)

    def ext_field(R):
        R = torch.as_tensor(R)
        q = torch.as_tensor(qs, dtype=R.dtype, device=R.device)
        e = torch.as_tensor(eh, dtype=R.dtype, device=R.device)
        ph = R @ q.T                                         # (..., 3)
        s = torch.sin(ph)
        mx = chirality * (s * e[:, 0]).sum(-1)
        my = chirality * (s * e[:, 1]).sum(-1)
        mz = m0 + torch.cos(ph).sum(-1)
        return _unit(torch.stack([mx, my, mz], dim=-1), h_pin)
    return ext_field


def make_fm_pin(h_pin, axis=(0.0, 0.0, 1.0)):
    """Uniform field h_pin along the unit vector of `axis`."""
    ax = _vec(axis)
    ax = ax / np.linalg.norm(ax)

    def ext_field(R):
        R = torch.as_tensor(R)
        b = torch.as_tensor(h_pin * ax, dtype=R.dtype, device=R.device)
        return b.expand(*R.shape[:-1], 3).clone()
    return ext_field


def make_spiral_pin(Q, h_pin, cycloidal=True):
    """Single-Q spiral of wave vector Q: the cycloid h_pin (sin(Q.r) q_hat, cos(Q.r)) (spin turning
    in the z_hat-q_hat plane), or with cycloidal=False the flat helix h_pin (cos Q.r, sin Q.r, 0)."""
    Q = _vec(Q)
    qh = Q / (np.linalg.norm(Q) + _EPS)

    def ext_field(R):
        R = torch.as_tensor(R)
        ph = Q[0] * R[..., 0] + Q[1] * R[..., 1]
        if cycloidal:
            s = torch.sin(ph)
            return h_pin * torch.stack([s * qh[0], s * qh[1], torch.cos(ph)], dim=-1)
        return h_pin * torch.stack([torch.cos(ph), torch.sin(ph), torch.zeros_like(ph)], dim=-1)
    return ext_field


def make_overhauser_pin(Q, h_pin):
    """Collinear spin-density wave h_pin (0, 0, cos(Q.r))."""
    Q = _vec(Q)

    def ext_field(R):
        R = torch.as_tensor(R)
        c = torch.cos(Q[0] * R[..., 0] + Q[1] * R[..., 1])
        z = torch.zeros_like(c)
        return h_pin * torch.stack([z, z, c], dim=-1)
    return ext_field


def make_pin(kind, q1, q2, h_pin, **kw):
    """Field by competitor name ("fluid" gives None: no field)."""
    if kind == "fluid":
        return None
    if kind == "fm":
        return make_fm_pin(h_pin, **kw)
    if kind == "spiral":
        return make_spiral_pin(q1, h_pin)
    if kind == "spiral_xy":
        return make_spiral_pin(q1, h_pin, cycloidal=False)
    if kind == "overhauser":
        return make_overhauser_pin(q1, h_pin)
    if kind == "skx":
        return make_skx_pin(q1, q2, h_pin, **kw)
    if kind == "skx_bloch":
        return make_skx_pin(q1, q2, h_pin, neel=False, **kw)
    raise ValueError(kind)
