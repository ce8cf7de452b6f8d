"""Writes tests/golden/ed2_config1.json: the two-electron exact ground-state energy (plane-wave ED,
oracle/ed2.py) of the configuration-1 physics with Coulomb: N = 2, r_s = 2 (L = sqrt(2 pi) 2),
m* = 1, lambda_R = 0.5, h_z = 0.1, twist 0, alpha_C = 1, at plane-wave cutoffs 16 and 24.

Run from the repository root:  python tests/golden/make_ed2.py
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), os.pardir, os.pardir))
sys.path.insert(0, ROOT)
from oracle import ed2  # noqa: E402
from oracle import nqs_oracle as O  # noqa: E402

L = float(np.sqrt(np.pi * 2) * 2.0)
A = np.diag([L, L])
out = dict(N=2, r_s=2.0, L=L, m_star=1.0, lambda_r=0.5, h_z=0.1, twist=[0.0, 0.0], alpha=1.0,
           zeta_M=O.Ewald(A, 1.0, 5.0 / L, 6, 12).zeta_M)
for nc in (16, 24):
    out[f"E_ed_ncut{nc}"] = ed2.ground_energy(A, nc, 1.0, 0.5, 0.1, alpha=1.0, ewald_alpha=5.0 / L)
with open(os.path.join(os.path.dirname(__file__), "ed2_config1.json"), "w") as f:
    json.dump(out, f, indent=1)
print(out)
