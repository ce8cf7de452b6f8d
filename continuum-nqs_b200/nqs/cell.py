"""General 2D simulation cell (host-side setup; reference src/nqs/cell.py:21-53).

A cell is a 2x2 matrix A whose columns are the lattice vectors: r = A s with fractional s.
"""
from __future__ import annotations

import numpy as np
import torch


def square_cell(L):
    return np.array([[float(L), 0.0], [0.0, float(L)]])


def rect_cell(Lx, Ly):
    return np.array([[float(Lx), 0.0], [0.0, float(Ly)]])


def hex_cell(a):
    """Triangular lattice: a1 = (a, 0), a2 = (a/2, a sqrt3/2)."""
    a = float(a)
    return np.array([[a, a / 2.0], [0.0, a * np.sqrt(3) / 2.0]])


def cell_matrix(cell) -> np.ndarray:
    """Scalar L -> L I; a 2x2 matrix passes through."""
    return square_cell(cell) if np.ndim(cell) == 0 else np.asarray(cell, dtype=float)


def reciprocal(A):
    """B = 2 pi (A^-1)^T; a_i . b_j = 2 pi delta_ij."""
    return 2.0 * np.pi * np.linalg.inv(np.asarray(A, float)).T


def cell_area(A):
    return float(abs(np.linalg.det(np.asarray(A, float))))


def frac(r, A):
    """Cartesian -> fractional coordinates mod 1 (r (...,2), numpy or torch)."""
    Ainv = np.linalg.inv(np.asarray(A, float))
    if isinstance(r, torch.Tensor):
        return torch.remainder(r @ torch.as_tensor(Ainv.T, dtype=r.dtype, device=r.device), 1.0)
    return np.mod(np.asarray(r) @ Ainv.T, 1.0)


def wrap(r, A):
    """Wrap a Cartesian point into the cell."""
    A = np.asarray(A, float)
    s = frac(r, A)
    if isinstance(s, torch.Tensor):
        return s @ torch.as_tensor(A.T, dtype=s.dtype, device=s.device)
    return s @ A.T
