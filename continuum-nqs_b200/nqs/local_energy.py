"""Local energy of the spinor wavefunction (drop-in for src/nqs/local_energy.py:40-117).

E_loc(R,S) = -1/(2 m*) (Lap L + grad L . grad L) - (h_z/2) sum_i (1 - 2 s_i)
             + lambda_R sum_i [(sigma_x)_{s_i s'} (-i) d_y_i + (sigma_y)_{s_i s'} (-i) d_x_i] Psi(s')/Psi
             - sum_i f_z(r_i) (sigma_z)_{s_i s_i} - sum_i [f_x sigma_x + f_y sigma_y]_{s_i s'} Psi(s')/Psi
with L = log Psi and f = ext_field (optional). The kinetic Laplacian always comes from the forward
Laplacian kernel
(``use_folx`` is accepted for signature compatibility; the dense Hessian and the forward Laplacian
are the same quantity and are checked against each other in the tests). The SOC term evaluates
the N spin-flipped states with a 2-tangent forward JVP each. Non-finite flip terms are set to 0
as in the reference (local_energy.py:99-105).
"""
from __future__ import annotations

import torch

from . import _lib
from .psiformer import LogPsi, as_batch


class LocalEnergy:
    def __init__(self, logpsi: LogPsi, m_star, lambda_r, h_z, coulomb=None, ext_field=None):
        self.logpsi = logpsi
        self.m_star, self.lambda_r, self.h_z = float(m_star), float(lambda_r), float(h_z)
        self.coulomb = coulomb
        self.ext_field = ext_field

    def __call__(self, R, S, return_logpsi=False):
        R, S, single = as_batch(R, S)
        W = R.shape[0]
        lp = self.logpsi
        h = lp.model.native().handle
        out = torch.empty(W, dtype=torch.complex128, device=R.device)
        lpo = torch.empty(W, dtype=torch.complex128, device=R.device) if return_logpsi else None
        ws, _ = _lib.workspace_for(h, _lib.OP_LOCAL_E, W, lp.precision)
        ew = self.coulomb.ewald.handle if self.coulomb is not None else None
        if self.ext_field is None:
            _lib.check(_lib.lib().nqs_local_energy(
                h, _lib.ptr(lp.theta), _lib.ptr(R), _lib.ptr(S), W, self.m_star, self.lambda_r,
                self.h_z, ew, _lib.ptr(out), _lib.ptr(lpo), lp.precision, _lib.ptr(ws),
                ws.numel(), _lib.stream_ptr()), "nqs_local_energy")
        else:
            f = torch.as_tensor(self.ext_field(R), dtype=torch.float64, device=R.device)
            if f.shape != (W, R.shape[1], 3):
                raise ValueError(f"ext_field(R) must have shape {(W, R.shape[1], 3)}, got "
                                 f"{tuple(f.shape)}")
            f = f.contiguous()
            _lib.check(_lib.lib().nqs_local_energy_field(
                h, _lib.ptr(lp.theta), _lib.ptr(R), _lib.ptr(S), W, self.m_star, self.lambda_r,
                self.h_z, ew, _lib.ptr(f), _lib.ptr(out), _lib.ptr(lpo), lp.precision,
                _lib.ptr(ws), ws.numel(), _lib.stream_ptr()), "nqs_local_energy_field")
        if return_logpsi:
            return (out[0], lpo[0]) if single else (out, lpo)
        return out[0] if single else out


def make_local_energy(logpsi, m_star=1.0, lambda_r=1.0, h_z=0.0, ext_field=None, use_folx=False,
                      coulomb=None):
    """Return E_loc(R, S) -> complex for a logpsi made by nqs.psiformer.make_logpsi.
    `coulomb` (an nqs.ewald coulomb_energy) optionally fuses the Ewald term into the same call.
    `ext_field`: the reference's ext_field(r) -> (f_x, f_y, f_z), here vectorised over positions
    (a torch tensor (..., 2) -> (..., 3), e.g. nqs.spiral.spiral_field), since it is evaluated on
    the device for all walkers at once; it is called once per E_loc evaluation."""
    if not isinstance(logpsi, LogPsi):
        raise NotImplementedError("make_local_energy needs a logpsi from nqs.psiformer.make_logpsi "
                                  "(arbitrary Python callables have no CUDA path)")
    return LocalEnergy(logpsi, m_star, lambda_r, h_z, coulomb, ext_field)


def grad_and_laplacian(logpsi: LogPsi, R, S):
    """(log psi (W,), grad log psi (W, 2N), Laplacian (W,)) from the forward-Laplacian kernel."""
    R, S, single = as_batch(R, S)
    W, N = R.shape[0], R.shape[1]
    h = logpsi.model.native().handle
    L = torch.empty(W, dtype=torch.complex128, device=R.device)
    g = torch.empty(W, 2 * N, dtype=torch.complex128, device=R.device)
    lap = torch.empty(W, dtype=torch.complex128, device=R.device)
    ws, _ = _lib.workspace_for(h, _lib.OP_LOCAL_E, W, logpsi.precision)
    _lib.check(_lib.lib().nqs_grad_laplacian(
        h, _lib.ptr(logpsi.theta), _lib.ptr(R), _lib.ptr(S), W, _lib.ptr(L), _lib.ptr(g),
        _lib.ptr(lap), logpsi.precision, _lib.ptr(ws), ws.numel(), _lib.stream_ptr()),
        "nqs_grad_laplacian")
    if single:
        return L[0], g[0], lap[0]
    return L, g, lap
