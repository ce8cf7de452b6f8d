"""2D Ewald Coulomb on a general cell (drop-in for src/nqs/ewald.py:26-73).

``make_ewald_lattice(A, alpha, ewald_alpha, n_real, n_recip)`` and ``make_ewald(L, ...)`` return
``(ewald_pair, zeta_M, coulomb_energy)`` as in the reference. The two callables run in libnqs
(``nqs_ewald_pair`` / ``nqs_ewald_energy``) and accept a single input or a batch:
``ewald_pair`` takes r (2,) or (M,2); ``coulomb_energy`` takes R (N,2) or (W,N,2).
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib
from .cell import cell_matrix, square_cell


class _Ewald:
    def __init__(self, A, alpha, ewald_alpha, n_real, n_recip):
        A = cell_matrix(A)
        arr = (ctypes.c_double * 4)(*[float(x) for x in A.reshape(-1)])
        h = ctypes.c_void_p()
        _lib.check(_lib.lib().nqs_ewald_create(arr, float(alpha),
                                               -1.0 if ewald_alpha is None else float(ewald_alpha),
                                               int(n_real), int(n_recip), ctypes.byref(h)),
                   "nqs_ewald_create")
        self.handle = h
        z = ctypes.c_double()
        _lib.check(_lib.lib().nqs_ewald_zeta(h, ctypes.byref(z)), "nqs_ewald_zeta")
        self.zeta_M = float(z.value)

    def __del__(self):
        try:
            _lib.lib().nqs_ewald_destroy(self.handle)
        except Exception:
            pass

    def pair(self, r):
        dev = _lib.device()
        r = torch.as_tensor(r)
        single = r.dim() == 1
        r = r.reshape(-1, 2).to(dev, torch.float64).contiguous()
        out = torch.empty(r.shape[0], dtype=torch.float64, device=dev)
        _lib.check(_lib.lib().nqs_ewald_pair(self.handle, _lib.ptr(r), r.shape[0], _lib.ptr(out),
                                             _lib.stream_ptr()), "nqs_ewald_pair")
        return out[0] if single else out

    def energy(self, R):
        dev = _lib.device()
        R = torch.as_tensor(R)
        single = R.dim() == 2
        if single:
            R = R[None]
        R = R.to(dev, torch.float64).contiguous()
        W, N = R.shape[0], R.shape[1]
        out = torch.empty(W, dtype=torch.float64, device=dev)
        _lib.check(_lib.lib().nqs_ewald_energy(self.handle, _lib.ptr(R), W, N, _lib.ptr(out),
                                               _lib.stream_ptr()), "nqs_ewald_energy")
        return out[0] if single else out


class CoulombEnergy:
    """coulomb_energy(R): sum_{i<j} ewald_pair(r_i - r_j) + N zeta_M / 2 (ewald.py:60-65)."""

    def __init__(self, ew: _Ewald):
        self.ewald = ew

    def __call__(self, R):
        return self.ewald.energy(R)


def make_ewald_lattice(A, alpha=1.0, ewald_alpha=None, n_real=5, n_recip=10):
    _lib.require_cuda()
    ew = _Ewald(A, alpha, ewald_alpha, n_real, n_recip)
    return ew.pair, ew.zeta_M, CoulombEnergy(ew)


def make_ewald(L, alpha=1.0, ewald_alpha=None, n_real=4, n_recip=8):
    """Square-box special case A = L I (ewald.py:70-73)."""
    return make_ewald_lattice(square_cell(L), alpha=alpha, ewald_alpha=ewald_alpha,
                              n_real=n_real, n_recip=n_recip)
