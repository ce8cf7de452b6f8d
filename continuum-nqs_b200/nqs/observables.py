"""Spin observables from the flip ratios (drop-in for src/nqs/observables.py:31-74).

Per configuration (R, S), with ratio_i = Psi(s_i -> 1 - s_i) / Psi:
    sigma_z^i = 1 - 2 s_i,   sigma_x^i = ratio_i,   sigma_y^i = -i (1 - 2 s_i) ratio_i
(the same flip ratios as the spin-orbit local energy; a non-finite ratio, from an exactly singular
flipped determinant, gives 0). The ratios come from nqs_spin_estimators on the device. The
texture binning, lattice skyrmion number, structure factor, coherent order parameter, the
Fourier-reconstructed skyrmion number, the exact Slater spin density and the state classifier
below are host post-processing (numpy, vectorised), restated from the reference
(observables.py:55-200).
"""
from __future__ import annotations

import numpy as np
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


def spin_texture(logpsi: LogPsi, R_batch, S_batch, A, ngrid=12):
    """Magnetisation density on an ngrid x ngrid grid over cell A (columns = lattice vectors):
    dict(m (ngrid, ngrid, 3), rho (ngrid, ngrid), mbar (3,) net moment per electron, mabs mean
    |m|), binned by fractional coordinates as the reference (observables.py:55-74)."""
    sx, sy, sz = spin_estimates(logpsi, R_batch, S_batch)
    B, N = sz.shape
    Ainv = np.linalg.inv(np.asarray(A, float))
    fr = np.mod(torch.as_tensor(R_batch).cpu().numpy() @ Ainv.T, 1.0)
    gi = np.clip((fr * ngrid).astype(int), 0, ngrid - 1)
    ix, iy = gi[..., 0].ravel(), gi[..., 1].ravel()
    m = np.zeros((ngrid, ngrid, 3))
    rho = np.zeros((ngrid, ngrid))
    for c, v in enumerate((sx, sy, sz)):
        np.add.at(m[..., c], (ix, iy), v.ravel())
    np.add.at(rho, (ix, iy), 1.0)
    m /= B
    rho /= B
    return dict(m=m, rho=rho, mbar=m.reshape(-1, 3).sum(0) / N,
                mabs=float(np.mean(np.linalg.norm(m, axis=-1))))


def _solid_angle(p, q, w):
    """Signed solid angle of the spherical triangle (p, q, w) of unit vectors (..., 3):
    2 atan2(p . (q x w), 1 + p.q + q.w + w.p)."""
    num = np.einsum("...k,...k->...", p, np.cross(q, w))
    den = 1.0 + np.einsum("...k,...k->...", p, q) + np.einsum("...k,...k->...", q, w) \
        + np.einsum("...k,...k->...", w, p)
    return 2.0 * np.arctan2(num, den)


def berg_luscher(m):
    """Lattice skyrmion number of a periodic texture m (n1, n2, 3): m is normalised per site; each
    plaquette (a = m[i, j], b = m[i+1, j], c = m[i, j+1], d = m[i+1, j+1]) is split into the
    triangles (a, b, d) and (a, d, c), whose solid angles sum to 4 pi Q (reference
    observables.py:77-90)."""
    m = np.asarray(m, dtype=float)
    n = m / (np.linalg.norm(m, axis=-1, keepdims=True) + 1e-12)
    b = np.roll(n, -1, axis=0)
    c = np.roll(n, -1, axis=1)
    d = np.roll(b, -1, axis=1)
    return float((_solid_angle(n, b, d) + _solid_angle(n, d, c)).sum() / (4.0 * np.pi))


def _recip_grid(A, nshell):
    Bm = 2.0 * np.pi * np.linalg.inv(np.asarray(A, float)).T  # columns b1, b2
    mn = [(p, q) for p in range(-nshell, nshell + 1) for q in range(-nshell, nshell + 1)]
    qs = np.array([p * Bm[:, 0] + q * Bm[:, 1] for p, q in mn])
    return mn, qs


def structure_factor(logpsi: LogPsi, R_batch, S_batch, A, nshell=4):
    """S_zz(q) = <|sum_i sigma_z^i e^{-i q.r_i}|^2> / N and S_perp(q) (the same with sigma_x and
    sigma_y summed) on the reciprocal grid q = m b1 + n b2, |m|, |n| <= nshell:
    dict(q (Q, 2), qfrac [(m, n)], Szz (Q,), Sperp (Q,)) (reference observables.py:93-108)."""
    sx, sy, sz = spin_estimates(logpsi, R_batch, S_batch)
    N = sz.shape[1]
    mn, qs = _recip_grid(A, nshell)
    R = torch.as_tensor(R_batch).cpu().numpy()
    ph = np.exp(-1j * np.einsum("bnd,qd->bnq", R, qs))
    rz, rx, ry = (np.einsum("bn,bnq->bq", a, ph) for a in (sz, sx, sy))
    return dict(q=qs, qfrac=mn, Szz=np.mean(np.abs(rz) ** 2, axis=0) / N,
                Sperp=np.mean(np.abs(rx) ** 2 + np.abs(ry) ** 2, axis=0) / N)


def spin_order_parameter(logpsi: LogPsi, R_batch, S_batch, A, Gset):
    """Coherent order parameter m_a(G) = < sum_i sigma_a^i e^{-i G.r_i} > / N for each G of Gset
    (nG, 2): complex (3, nG), rows x, y, z (reference observables.py:111-120)."""
    sx, sy, sz = spin_estimates(logpsi, R_batch, S_batch)
    R = torch.as_tensor(R_batch).cpu().numpy()
    N = R.shape[1]
    G = np.asarray(Gset, float).reshape(-1, 2)
    ph = np.exp(-1j * np.einsum("bnd,gd->bng", R, G))
    return np.stack([np.einsum("bn,bng->bg", a, ph).mean(0) / N for a in (sx, sy, sz)])


def skx_arms(q1, q2, nharm=1):
    """G = 0 and +-h q_j for the arms q1, q2, q3 = -(q1 + q2), harmonics h = 1..nharm, in that
    order (reference observables.py:123-130)."""
    q1, q2 = np.asarray(q1, float), np.asarray(q2, float)
    out = [np.zeros(2)]
    for h in range(1, nharm + 1):
        for q in (q1, q2, -(q1 + q2)):
            out += [h * q, -h * q]
    return np.array(out)


def _cell_grid(A, ngrid):
    f = (np.arange(ngrid) + 0.5) / ngrid
    fu, fv = np.meshgrid(f, f, indexing="ij")
    return np.stack([fu, fv], axis=-1) @ np.asarray(A, float).T  # (ngrid, ngrid, 2)


def skyrmion_number_fourier(logpsi: LogPsi, R_batch, S_batch, A, q1, q2, nharm=1, ngrid=24):
    """Skyrmion number of the smooth texture m(r) = Re sum_G m(G) e^{i G.r} rebuilt from the
    coherent order parameter at the skyrmion arms, and the order amplitude (mean |m(G)| over the
    arms): dict(Q, order_amp, m_recon, mG, m0) (reference observables.py:133-147)."""
    G = skx_arms(q1, q2, nharm)
    mG = spin_order_parameter(logpsi, R_batch, S_batch, A, G)
    r = _cell_grid(A, ngrid)
    m = np.real(np.einsum("ag,xyg->xya", mG, np.exp(1j * (r @ G.T))))
    amp = float(np.mean(np.linalg.norm(mG[:, 1:], axis=0)))
    return dict(Q=berg_luscher(m), order_amp=amp, m_recon=m, mG=mG, m0=np.real(mG[:, 0]))


def slater_spin_density(Gs, W, A, ngrid=24):
    """Spin density m(r) = sum_a phi_a(r)^dagger sigma phi_a(r) of the Slater determinant with
    orbitals phi_a(r, s) = sum_G W[a, G, s] e^{i G.r}, exactly on the cell-centred ngrid x ngrid
    grid: (ngrid, ngrid, 3) (reference observables.py:150-165)."""
    Gs = np.asarray(Gs, float)
    W = np.asarray(W, complex)
    r = _cell_grid(A, ngrid)
    e = np.exp(1j * (r @ Gs.T))                                  # (x, y, G)
    phi = np.einsum("ags,xyg->xyas", W, e)                       # (x, y, a, s)
    up, dn = phi[..., 0], phi[..., 1]
    cud = np.sum(np.conj(up) * dn, axis=-1)
    mz = np.sum(np.abs(up) ** 2 - np.abs(dn) ** 2, axis=-1)
    return np.stack([2.0 * cud.real, 2.0 * cud.imag, mz], axis=-1)


def classify_state(logpsi: LogPsi, R_batch, S_batch, A, ngrid=12, nshell=4, q1=None, q2=None,
                   nharm=1):
    """Texture, skyrmion number, structure-factor peak and a heuristic label, with the reference's
    thresholds and labels (observables.py:168-200): ordered when the Fourier order amplitude
    exceeds 0.05 (arms given) or the largest finite-q peak exceeds 1.5 x the q = 0 weight;
    ordered states are "SKYRMION (Q!=0, ordered)" (|Q| > 0.4), "z-SDW / collinear (Overhauser)"
    (the peak more than 60% S_zz) or "spiral / in-plane (1Q)"; others "ferromagnet (m_z)"
    (|m_z| > 0.3), "in-plane / Rashba-FM" (|m_xy| > 0.3) or "fluid / disordered"."""
    tex = spin_texture(logpsi, R_batch, S_batch, A, ngrid=ngrid)
    if q1 is not None:
        fou = skyrmion_number_fourier(logpsi, R_batch, S_batch, A, q1, q2, nharm=nharm,
                                      ngrid=max(20, ngrid))
        Q, order_amp = fou["Q"], fou["order_amp"]
    else:
        fou = None
        Q, order_amp = berg_luscher(tex["m"]), float("nan")
    sf = structure_factor(logpsi, R_batch, S_batch, A, nshell=nshell)
    qn = np.linalg.norm(sf["q"], axis=1)
    fin = qn > 1e-9
    tot = sf["Szz"] + sf["Sperp"]
    gamma = float(tot[~fin].sum())
    if fin.any():
        k = int(np.argmax(tot * fin))
        peak_frac, peak_val = sf["qfrac"][k], float(tot[k])
        zfrac = float(sf["Szz"][k] / (tot[k] + 1e-12))
    else:
        peak_frac, peak_val, zfrac = (0, 0), 0.0, 0.0
    mz, mxy = abs(tex["mbar"][2]), float(np.hypot(*tex["mbar"][:2]))
    finite_q = peak_val > 1.5 * (gamma / max(1, int((~fin).sum())))
    ordered = (order_amp > 0.05) if order_amp == order_amp else finite_q
    if not ordered:
        label = ("ferromagnet (m_z)" if mz > 0.3 else
                 "in-plane / Rashba-FM" if mxy > 0.3 else "fluid / disordered")
    else:
        label = ("SKYRMION (Q!=0, ordered)" if abs(Q) > 0.4 else
                 "z-SDW / collinear (Overhauser)" if zfrac > 0.6 else "spiral / in-plane (1Q)")
    return dict(skyrmion_Q=float(Q), order_amp=order_amp, mbar=tex["mbar"].tolist(),
                mabs=tex["mabs"], peak_qfrac=peak_frac, peak_val=peak_val, gamma_weight=gamma,
                peak_is_z=zfrac, label=label, _tex=tex, _sf=sf, _fou=fou)
