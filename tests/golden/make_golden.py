"""Generate tests/golden/rashba_gs.npz from the REFERENCE's own pure-numpy module
src/nqs/rashba_reference.py (it imports without JAX). Run in a container where the reference is
mounted:  python tests/golden/make_golden.py /path/to/continuum-nqs
(or with the environment variable NQS_REFERENCE_ROOT naming that checkout). The fixture pins the
host-side restatement nqs.rashba (and through it every E_gs certificate)."""
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
    # band energies at a few momenta
    from src.nqs.rashba_reference import bands_analytic, bands_k
    ks = np.array([[0.0, 0.0], [0.3, -0.7], [1.1, 0.4]])
    out["bands_k"] = np.array([bands_k(kx, ky, 1.0, 0.7, 0.3)[:2] for kx, ky in ks])
    out["bands_analytic"] = np.array([bands_analytic(kx, ky, 1.0, 0.7, 0.3) for kx, ky in ks])
    np.savez(os.path.join(os.path.dirname(os.path.abspath(__file__)), "rashba_gs.npz"), **out)


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("NQS_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: make_golden.py <reference checkout> (or set NQS_REFERENCE_ROOT)")
    main(root)
