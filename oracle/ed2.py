"""Exact diagonalisation of two interacting electrons on the periodic cell — TEST INFRASTRUCTURE.

Only tests/ may import this module; it is the checker of the whole-iteration physics (the
reference claims its trained ansatz reaches this ground state within 0.7 mHa at two electrons,
README.md:47-49, but ships no ED code, number or test; this is a plane-wave ED written here).

Hamiltonian (the conventions of the reference's local energy and Ewald sum):

    H = sum_{i=1,2} h0(p_i) + phi(r_1 - r_2) + 2 zeta_M / 2
    h0(k) = k^2/(2 m*) + lambda_R (sigma_x k_y + sigma_y k_x) - (h_z/2) sigma_z
            (src/nqs/rashba_reference.py:36-39, src/nqs/local_energy.py:78-111)
    phi(r) = (alpha/A) sum_{q != 0} (2 pi/|q|) e^{i q.r}: the Ewald pair potential
            (src/nqs/ewald.py:1-10,47-51) written as its Fourier series; zeta_M the Madelung term
            (ewald.py:53-65), taken from the oracle's Ewald class.

Basis: plane waves k(n) = B n + A^-T twist (B = 2 pi A^-T), |n_x|, |n_y| <= n_cut, for each
particle. H conserves the total momentum K = k_1 + k_2 = B m + 2 A^-T twist (integer m), so each
sector m is diagonalised separately. The two-electron amplitude is c(n_1, s_1, s_2) with
k_2 = K - k(n_1) (both particles inside the box). The Coulomb term acts on the relative momentum
only: (V c)(n') = sum_{n != n'} (2 pi alpha / (A |B (n' - n)|)) c(n), a 2D convolution applied by
FFT. The fermionic ground state is the lowest eigenvalue on the subspace antisymmetric under
exchange c(n, s_1, s_2) -> c(m - n, s_2, s_1) (Lanczos, scipy eigsh); the symmetric part and the
amplitudes outside the box are shifted out of the way.
"""
from __future__ import annotations

import numpy as np
from scipy.sparse.linalg import LinearOperator, eigsh

from . import nqs_oracle as O

_SX = np.array([[0, 1], [1, 0]], dtype=complex)
_SY = np.array([[0, -1j], [1j, 0]], dtype=complex)
_SZ = np.array([[1, 0], [0, -1]], dtype=complex)


def h0(k, m_star, lambda_r, h_z):
    """Bloch Hamiltonian (2x2) at momenta k (..., 2) -> (..., 2, 2)."""
    kx, ky = k[..., 0], k[..., 1]
    e = (kx * kx + ky * ky) / (2.0 * m_star)
    out = e[..., None, None] * np.eye(2) + lambda_r * (ky[..., None, None] * _SX
                                                       + kx[..., None, None] * _SY)
    return out - 0.5 * h_z * _SZ


class Sector:
    """The two-electron Hamiltonian restricted to total momentum K = B m + 2 A^-T twist: the
    amplitudes c(n_1, s_1, s_2) (shape (S, S, 4), S = 2 n_cut + 1, spin index s_1 * 2 + s_2) with
    k_2 = K - k(n_1), both particles inside the box."""

    def __init__(self, A, m_vec, n_cut, m_star=1.0, lambda_r=1.0, h_z=0.0, alpha=1.0,
                 twist=(0.0, 0.0), zeta_M=0.0):
        A = np.asarray(A, float)
        Ainv = np.linalg.inv(A)
        B = 2.0 * np.pi * Ainv.T
        kt = Ainv.T @ np.asarray(twist, float)
        area = float(abs(np.linalg.det(A)))
        n1 = np.arange(-n_cut, n_cut + 1)
        nx, ny = np.meshgrid(n1, n1, indexing="ij")
        self.n = np.stack([nx, ny], -1).astype(float)               # (S, S, 2)
        self.S = S = 2 * n_cut + 1
        self.n_cut = n_cut
        self.m_vec = m_vec = np.asarray(m_vec, float)
        k1 = self.n @ B.T + kt
        K = B @ m_vec + 2.0 * kt
        k2 = K - k1
        n2 = m_vec - self.n
        self.valid = (np.abs(n2) <= n_cut).all(-1)                  # particle 2 inside the box
        # one-body part: h0(k1) x I + I x h0(k2), a 4x4 block per n (index s1 * 2 + s2)
        H1 = np.einsum("xyab,cd->xyacbd", h0(k1, m_star, lambda_r, h_z), np.eye(2))
        H1 = H1 + np.einsum("ab,xycd->xyacbd", np.eye(2), h0(k2, m_star, lambda_r, h_z))
        self.H1 = H1.reshape(S, S, 4, 4)
        # Coulomb kernel over differences d in [-2 n_cut, 2 n_cut]^2, zero-padded FFT convolution
        self.P = P = 4 * n_cut + 2
        d1 = np.arange(-2 * n_cut, 2 * n_cut + 1)
        dx, dy = np.meshgrid(d1, d1, indexing="ij")
        q = np.stack([dx, dy], -1).astype(float) @ B.T
        qn = np.linalg.norm(q, axis=-1)
        ker = np.where(qn > 0, 2.0 * np.pi * alpha / (area * np.where(qn > 0, qn, 1.0)), 0.0)
        kpad = np.zeros((P, P))
        kpad[:4 * n_cut + 1, :4 * n_cut + 1] = ker
        self.kf = np.fft.fft2(kpad)
        self.const = zeta_M  # N zeta_M / 2 with N = 2
        self.mask = self.valid[..., None].astype(float)             # (S, S, 1)
        self.perm = np.array([0, 2, 1, 3])                          # (s1, s2) -> (s2, s1)

    def exch(self, c):  # c(n, s1, s2) -> c(m - n, s2, s1): n -> m - n reverses the box about m/2
        out = np.zeros_like(c)
        n_cut, n, m_vec, ok = self.n_cut, self.n, self.m_vec, self.valid
        ix = (m_vec[0] - n[..., 0] + n_cut).astype(int)
        iy = (m_vec[1] - n[..., 1] + n_cut).astype(int)
        out[ok] = c[ix[ok], iy[ok]][:, self.perm]
        return out

    def proj(self, c):  # antisymmetric part, inside the box
        c = c * self.mask
        return 0.5 * (c - self.exch(c))

    def apply_H(self, c):
        S, P, n_cut = self.S, self.P, self.n_cut
        out = np.einsum("xyab,xyb->xya", self.H1, c) + self.const * c
        cp = np.zeros((P, P, 4), dtype=complex)
        cp[:S, :S] = c
        conv = np.fft.ifft2(np.fft.fft2(cp, axes=(0, 1)) * self.kf[..., None], axes=(0, 1))
        return out + conv[2 * n_cut:2 * n_cut + S, 2 * n_cut:2 * n_cut + S]


def sector_ground_energy(A, m_vec, n_cut, m_star=1.0, lambda_r=1.0, h_z=0.0, alpha=1.0,
                         twist=(0.0, 0.0), zeta_M=0.0, tol=1e-12, shift=1.0e4, offset=10.0):
    sec = Sector(A, m_vec, n_cut, m_star, lambda_r, h_z, alpha, twist, zeta_M)
    S = sec.S
    dim = S * S * 4

    # `offset` keeps the sought eigenvalue away from 0, where ARPACK's relative residual test
    # cannot converge; it is removed from the result
    def mv(x):
        c = x.reshape(S, S, 4)
        pc = sec.proj(c)
        y = sec.proj(sec.apply_H(pc)) + offset * pc + shift * (c - pc)
        return y.reshape(-1)

    op = LinearOperator((dim, dim), matvec=mv, dtype=complex)
    rng = np.random.default_rng(0)
    v0 = sec.proj((rng.standard_normal((S, S, 4)) + 1j * rng.standard_normal((S, S, 4)))).reshape(-1)
    w = eigsh(op, k=1, which="SA", v0=v0, tol=tol, maxiter=20000, return_eigenvectors=False)
    return float(w[0]) - offset


def expectation(A, coeff, n_cut, m_star=1.0, lambda_r=1.0, h_z=0.0, alpha=1.0,
                twist=(0.0, 0.0), ewald_alpha=None):
    """<psi|H|psi> / <psi|psi> of a two-electron state given by its plane-wave amplitudes
    coeff[n1x, n1y, n2x, n2y, s1, s2] (indices n + n_cut, |n| <= n_cut per component), with
    every total-momentum sector's Hamiltonian (the same H as ground_energy). The exact
    variational energy of the state truncated to the basis; no sampling, no local energy."""
    ew = O.Ewald(A, alpha=alpha, ewald_alpha=ewald_alpha, n_real=6, n_recip=12)
    S = 2 * n_cut + 1
    num, den = 0.0, 0.0
    for mx in range(-2 * n_cut, 2 * n_cut + 1):
        for my in range(-2 * n_cut, 2 * n_cut + 1):
            sec = Sector(A, (mx, my), n_cut, m_star, lambda_r, h_z, alpha, twist, ew.zeta_M)
            n = sec.n.astype(int)
            ix2, iy2 = mx - n[..., 0] + n_cut, my - n[..., 1] + n_cut
            ok = sec.valid
            c = np.zeros((S, S, 4), dtype=complex)
            c[ok] = coeff[n[ok][:, 0] + n_cut, n[ok][:, 1] + n_cut, ix2[ok], iy2[ok]].reshape(-1, 4)
            den += float(np.vdot(c, c).real)
            num += float(np.vdot(c, sec.apply_H(c)).real)
    return num / den
def ground_energy(A, n_cut, m_star=1.0, lambda_r=1.0, h_z=0.0, alpha=1.0, twist=(0.0, 0.0),
                  ewald_alpha=None, m_range=1):
    """Two-electron ground-state energy: the lowest over total-momentum sectors
    m in [-m_range, m_range]^2; zeta_M from the oracle's Ewald sum of the same cell."""
    ew = O.Ewald(A, alpha=alpha, ewald_alpha=ewald_alpha, n_real=6, n_recip=12)
    best = None
    for mx in range(-m_range, m_range + 1):
        for my in range(-m_range, m_range + 1):
            e = sector_ground_energy(A, (mx, my), n_cut, m_star, lambda_r, h_z, alpha, twist,
                                     ew.zeta_M)
            best = e if best is None else min(best, e)
    return best
