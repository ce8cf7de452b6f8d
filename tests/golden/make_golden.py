"""Generate tests/golden/rashba_gs.npz from the REFERENCE's own pure-numpy module
src/nqs/rashba_reference.py (it imports without JAX). Run in a container where the reference is
mounted:  python tests/golden/make_golden.py /path/to/continuum-nqs
The fixture pins the host-side restatement nqs.rashba (and through it every E_gs certificate)."""
import os
import sys

import numpy as np

CASES = [  # (N, L, lambda_r, h_z, twist)
    (5, 7.0, 1.0, 0.5, (0.1, 0.17)),
    (7, 8.0, 1.0, 0.5, (0.1, 0.17)),
    (9, 9.0, 1.0, 0.0, (0.1, 0.17)),
    (5, 9.0, 0.0, 4.0, (0.1, 0.17)),
    (2, float(np.sqrt(np.pi * 2) * 2.0), 0.5, 0.1, (0.0, 0.0)),       # config 1 cell
    (16, float(np.sqrt(np.pi * 16) * 5.0), 0.3, 0.05, (0.1, 0.17)),   # config 2 cell
]


def main(ref_root):
    sys.path.insert(0, ref_root)
    from src.nqs.rashba_reference import (cell_rashba_envelope, noninteracting_gs,
                                          occupied_orbital_matrix)
    out = {}
    for c, (N, L, lr, hz, tw) in enumerate(CASES):
        g = noninteracting_gs(N=N, L=L, m_star=1.0, lambda_r=lr, h_z=hz, n_cut=10, twist=tw)
        K, Chi = occupied_orbital_matrix(g)
        env = cell_rashba_envelope(L, N, 1.0, lr, hz, 10, tw)
        out[f"c{c}_params"] = np.array([N, L, lr, hz, tw[0], tw[1]])
        out[f"c{c}_E_gs"] = np.array(g["E_gs"])
        out[f"c{c}_gap"] = np.array(g["gap"])
        out[f"c{c}_K"] = K
        out[f"c{c}_Chi"] = Chi
        out[f"c{c}_env_Gs"] = env["Gs"]
        out[f"c{c}_env_W"] = env["W"]
    # skyrmion-background envelope on a commensurate supercell (texture harmonics from a fixed
    # seed), band energies at a few momenta, and the ring minimum at h_z = 0
    from src.nqs.rashba_reference import (bands_analytic, bands_k, cell_skx_envelope,
                                          ring_minimum)
    q1, q2, A, keys, vals = skx_case()
    skx = cell_skx_envelope(A, 7, keys, vals, q1, q2, 0.5, 1.0, 0.3, 0.05, 4, (0.1, 0.17))
    out["skx_E_band"] = np.array(skx["E_band"])
    out["skx_gap"] = np.array(skx["gap"])
    out["skx_w"] = skx["w"]
    out["skx_Gs"] = skx["Gs"]
    out["skx_W"] = skx["W"]
    ks = np.array([[0.0, 0.0], [0.3, -0.7], [1.1, 0.4]])
    out["bands_k"] = np.array([bands_k(kx, ky, 1.0, 0.7, 0.3)[:2] for kx, ky in ks])
    out["bands_analytic"] = np.array([bands_analytic(kx, ky, 1.0, 0.7, 0.3) for kx, ky in ks])
    out["ring_hz0"] = np.array(ring_minimum(1.0, 0.3, 0.0))
    np.savez(os.path.join(os.path.dirname(os.path.abspath(__file__)), "rashba_gs.npz"), **out)


def skx_case():
    """Triple-Q texture on the doubled magnetic cell (q* = 0.9548), six harmonics, seed 0."""
    qs = 0.9548
    q1 = qs * np.array([1.0, 0.0])
    q2 = qs * np.array([-0.5, np.sqrt(3) / 2])
    A = 2.0 * np.pi * np.linalg.inv(np.array([q1, q2])) * 2
    keys = np.array([[1, 0], [0, 1], [-1, -1], [-1, 0], [0, -1], [1, 1]])
    rng = np.random.default_rng(0)
    vals = 0.2 * (rng.normal(size=(6, 3)) + 1j * rng.normal(size=(6, 3)))
    return q1, q2, A, keys, vals


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
