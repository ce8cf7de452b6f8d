"""Spin observables from the flip ratios (drop-in for src/nqs/observables.py:31-53).

Per configuration (R, S), with ratio_i = Psi(s_i -> 1 - s_i) / Psi:
    sigma_z^i = 1 - 2 s_i,   sigma_x^i = ratio_i,   sigma_y^i = -i (1 - 2 s_i) ratio_i
(the same flip ratios as the spin-orbit local energy; a non-finite ratio, from an exactly singular
flipped determinant, gives 0). The ratios come from nqs_spin_estimators on the device.
"""
from __future__ import annotations

import torch

from . import _lib
from .psiformer import LogPsi, as_batch


def make_spin_estimators(logpsi: LogPsi):
    """per_config(R, S) -> (sx, sy, sz), each (N,) or batched (W, N); sx, sy complex."""
    if not isinstance(logpsi, LogPsi):
        raise NotImplementedError("spin estimators need a logpsi from nqs.psiformer.make_logpsi")

    def per_config(R, S):
        R, S, single = as_batch(R, S)
        W, N = S.shape
        h = logpsi.model.native().handle
        sx = torch.empty(W, N, dtype=torch.complex128, device=R.device)
        sy = torch.empty_like(sx)
        sz = torch.empty(W, N, dtype=torch.float64, device=R.device)
        ws, _ = _lib.workspace_for(h, _lib.OP_LOCAL_E, W, logpsi.precision)
        _lib.check(_lib.lib().nqs_spin_estimators(
            h, _lib.ptr(logpsi.theta), _lib.ptr(R), _lib.ptr(S), W, _lib.ptr(sx), _lib.ptr(sy),
            _lib.ptr(sz), logpsi.precision, _lib.ptr(ws), ws.numel(), _lib.stream_ptr()),
            "nqs_spin_estimators")
        return (sx[0], sy[0], sz[0]) if single else (sx, sy, sz)
    return per_config


def spin_estimates(logpsi: LogPsi, R_batch, S_batch):
    """Batched estimators -> real parts (sx, sy, sz), each numpy (B, N)."""
    sx, sy, sz = make_spin_estimators(logpsi)(R_batch, S_batch)
    return sx.real.cpu().numpy(), sy.real.cpu().numpy(), sz.cpu().numpy()
