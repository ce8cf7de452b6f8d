"""Exact non-interacting Rashba + Zeeman ground state on a periodic 2D cell (host-side setup).

The warm-start envelope of the wavefunction (plane-wave momenta Gs and spinor coefficients W) and
the analytic energy E_gs used by the zero-variance certificates come from here. It restates the
reference module src/nqs/rashba_reference.py (h0_k :36-39, bands_k :42-46, bands_analytic :49-54,
allowed_k :57-65, single_particle_levels :68-80, noninteracting_gs :83-108,
occupied_orbital_matrix :111-119, planewave_envelope :122-133, cell_rashba_envelope :136-160)
with the same conventions:

    h0(k) = k^2/(2 m*) I + lambda_R (sigma_x k_y + sigma_y k_x) - (h_z/2) sigma_z

momenta k = (2 pi n + twist)/L on the square torus (k = B n + A^-T twist on a general cell),
levels sorted by energy with a stable sort over (n_x outer, n_y inner, lower band first).
Spinors come from numpy's Hermitian eigensolver on the 2x2 block, the same solver the
reference calls, so eigenvector phases agree.
"""
from __future__ import annotations

import numpy as np

_SX = np.array([[0, 1], [1, 0]], dtype=complex)
_SY = np.array([[0, -1j], [1j, 0]], dtype=complex)
_SZ = np.array([[1, 0], [0, -1]], dtype=complex)


def h0_k(kx, ky, m_star=1.0, lambda_r=1.0, h_z=0.0):
    """2x2 Bloch Hamiltonian at momentum (kx, ky)."""
    return ((kx * kx + ky * ky) / (2.0 * m_star)) * np.eye(2) + lambda_r * (_SX * ky + _SY * kx) \
        - 0.5 * h_z * _SZ


def _bands(kx, ky, m_star, lambda_r, h_z):
    w, v = np.linalg.eigh(h0_k(kx, ky, m_star, lambda_r, h_z))
    return float(w[0]), float(w[1]), v[:, 0].copy(), v[:, 1].copy()


def bands_k(kx, ky, m_star=1.0, lambda_r=1.0, h_z=0.0):
    """(E_lower, E_upper, chi_lower, chi_upper) of h0(k) (Hermitian eigensolver)."""
    return _bands(kx, ky, m_star, lambda_r, h_z)


def bands_analytic(kx, ky, m_star=1.0, lambda_r=1.0, h_z=0.0):
    """Closed-form band energies k^2/(2 m*) -+ sqrt(lambda_R^2 k^2 + h_z^2 / 4)."""
    k2 = kx * kx + ky * ky
    d = np.sqrt(lambda_r * lambda_r * k2 + 0.25 * h_z * h_z)
    return k2 / (2.0 * m_star) - d, k2 / (2.0 * m_star) + d


def allowed_k(L, n_cut, twist=(0.0, 0.0)):
    """Flattened (kx, ky) of k = (2 pi n + twist) / L, |n_x|, |n_y| <= n_cut, n_x the slow index."""
    n = np.arange(-n_cut, n_cut + 1)
    nx, ny = np.meshgrid(n, n, indexing="ij")
    return ((2.0 * np.pi * nx + twist[0]) / L).ravel(), ((2.0 * np.pi * ny + twist[1]) / L).ravel()


def single_particle_levels(L, m_star=1.0, lambda_r=1.0, h_z=0.0, n_cut=8, twist=(0.0, 0.0)):
    """All 2 (2 n_cut + 1)^2 spin-orbital levels of the L x L torus, stably sorted by energy:
    dicts E, kx, ky, band (0 lower, 1 upper), n (integer momentum index), chi (2-spinor)."""
    n = np.arange(-n_cut, n_cut + 1)
    out = []
    for nx in n:
        for ny in n:
            kx = (2.0 * np.pi * nx + twist[0]) / L
            ky = (2.0 * np.pi * ny + twist[1]) / L
            El, Eu, cl, cu = _bands(kx, ky, m_star, lambda_r, h_z)
            out.append(dict(E=El, kx=kx, ky=ky, band=0, n=(int(nx), int(ny)), chi=cl))
            out.append(dict(E=Eu, kx=kx, ky=ky, band=1, n=(int(nx), int(ny)), chi=cu))
    out.sort(key=lambda d: d["E"])
    return out


def _levels(kpts, m_star, lambda_r, h_z):
    """All spin-orbital levels (E, k, spinor, band) in enumeration order, then stably sorted."""
    levels = []
    for k in kpts:
        El, Eu, cl, cu = _bands(k[0], k[1], m_star, lambda_r, h_z)
        levels.append((El, k, cl, 0))
        levels.append((Eu, k, cu, 1))
    levels.sort(key=lambda t: t[0])
    return levels


def _square_kpts(L, n_cut, twist):
    js = np.arange(-n_cut, n_cut + 1)
    return [np.array([(2.0 * np.pi * nx + twist[0]) / L, (2.0 * np.pi * ny + twist[1]) / L])
            for nx in js for ny in js]


def noninteracting_gs(N, L, m_star=1.0, lambda_r=1.0, h_z=0.0, n_cut=8, twist=(0.0, 0.0)):
    """Lowest-N-level Slater determinant on the L x L torus: dict with E_gs, gap, occ, ..."""
    levels = _levels(_square_kpts(L, n_cut, twist), m_star, lambda_r, h_z)
    if len(levels) < N + 1:
        raise ValueError("n_cut too small for N levels")
    occ = [dict(E=e, kx=float(k[0]), ky=float(k[1]), band=b, chi=c) for e, k, c, b in levels[:N]]
    E_gs = float(sum(d["E"] for d in occ))
    k2_occ = max(d["kx"] ** 2 + d["ky"] ** 2 for d in occ)
    k2_edge = (2.0 * np.pi * n_cut / L) ** 2
    return dict(E_gs=E_gs, E_per=E_gs / N, gap=float(levels[N][0] - levels[N - 1][0]), occ=occ,
                E_homo=float(levels[N - 1][0]), E_lumo=float(levels[N][0]), density=N / (L * L),
                N=N, L=L, m_star=m_star, lambda_r=lambda_r, h_z=h_z, twist=twist,
                k2_occ_max=k2_occ, k2_cut=k2_edge, cutoff_ok=bool(k2_occ < 0.5 * k2_edge))


def occupied_orbital_matrix(gs):
    """(Kvecs (N,2), Chi (N,2) complex) of the occupied levels."""
    Kvecs = np.array([[d["kx"], d["ky"]] for d in gs["occ"]], dtype=float)
    Chi = np.array([d["chi"] for d in gs["occ"]], dtype=complex)
    return Kvecs, Chi


def planewave_envelope(Kvecs, Chi):
    """One plane wave per orbital: Gs = Kvecs, W[a, g, :] = Chi[a] delta(g, a)."""
    Kvecs = np.asarray(Kvecs, dtype=float)
    Chi = np.asarray(Chi, dtype=complex)
    n = Kvecs.shape[0]
    W = np.zeros((n, n, 2), dtype=complex)
    W[np.arange(n), np.arange(n), :] = Chi
    return Kvecs.copy(), W


def cell_rashba_envelope(A, N, m_star=1.0, lambda_r=1.0, h_z=0.0, n_cut=8, twist=(0.0, 0.0)):
    """Occupied Rashba orbitals on a general cell A (columns = lattice vectors) -> envelope."""
    A = np.array([[float(A), 0.0], [0.0, float(A)]]) if np.ndim(A) == 0 else np.asarray(A, float)
    Ainv = np.linalg.inv(A)
    B = 2.0 * np.pi * Ainv.T
    kt = Ainv.T @ np.asarray(twist, float)
    js = np.arange(-n_cut, n_cut + 1)
    kpts = [B @ np.array([float(nx), float(ny)]) + kt for nx in js for ny in js]
    levels = _levels(kpts, m_star, lambda_r, h_z)
    occ = levels[:N]
    Kvecs = np.array([t[1] for t in occ])
    Chi = np.array([t[2] for t in occ])
    Gs, W = planewave_envelope(Kvecs, Chi)
    area = float(abs(np.linalg.det(A)))
    return dict(Gs=Gs, W=W, E_gs=float(sum(t[0] for t in occ)),
                gap=float(levels[N][0] - levels[N - 1][0]), Kvecs=Kvecs, Chi=Chi, area=area, N=N,
                density=N / area)
