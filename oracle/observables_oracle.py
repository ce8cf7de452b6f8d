"""Pinning fields and texture observables, one point / one plaquette at a time — TEST
INFRASTRUCTURE.

Only tests/ may import this module. It restates, in plain per-point numpy, the reference's
pinning-field definitions (src/nqs/pinning.py:22-109) and texture diagnostics
(src/nqs/observables.py:77-90 lattice skyrmion number, :123-130 skyrmion arms, :150-165 Slater spin
density), so that the vectorised package versions (nqs.pinning, nqs.observables) can be checked
against an independent evaluation. The reference module imports JAX and cannot run here; its
own test of the skyrmion number (tests/test_nqs_observables.py:47-66: a nonzero integer on the
triple-Q field, zero on a uniform texture) is the known answer these pin to.
"""
from __future__ import annotations

import math

import numpy as np


def _norm(v):
    return math.sqrt(sum(float(x) * float(x) for x in v))


def skx_field(r, q1, q2, h_pin, m0=0.3, chirality=1.0, neel=True):
    arms = [np.asarray(q1, float), np.asarray(q2, float)]
    arms.append(-(arms[0] + arms[1]))
    m = [0.0, 0.0, m0]
    for q in arms:
        qn = _norm(q)
        e = (q[0] / qn, q[1] / qn) if neel else (-q[1] / qn, q[0] / qn)
        ph = q[0] * r[0] + q[1] * r[1]
        m[0] += chirality * math.sin(ph) * e[0]
        m[1] += chirality * math.sin(ph) * e[1]
        m[2] += math.cos(ph)
    n = _norm(m) + 1e-12
    return [h_pin * x / n for x in m]


def fm_field(r, h_pin, axis=(0.0, 0.0, 1.0)):
    n = _norm(axis)
    return [h_pin * a / n for a in axis]


def spiral_field(r, Q, h_pin, cycloidal=True):
    ph = Q[0] * r[0] + Q[1] * r[1]
    if cycloidal:
        qn = _norm(Q) + 1e-12
        return [h_pin * math.sin(ph) * Q[0] / qn, h_pin * math.sin(ph) * Q[1] / qn,
                h_pin * math.cos(ph)]
    return [h_pin * math.cos(ph), h_pin * math.sin(ph), 0.0]


def overhauser_field(r, Q, h_pin):
    return [0.0, 0.0, h_pin * math.cos(Q[0] * r[0] + Q[1] * r[1])]


def hf_field(r, s_keys, s_vals, q1, q2, h_pin):
    m = [0.0, 0.0, 0.0]
    for (a, b), S in zip(np.asarray(s_keys), np.asarray(s_vals, complex)):
        g = a * np.asarray(q1, float) + b * np.asarray(q2, float)
        e = complex(math.cos(g[0] * r[0] + g[1] * r[1]), math.sin(g[0] * r[0] + g[1] * r[1]))
        for k in range(3):
            m[k] += (e * S[k]).real
    n = _norm(m) + 1e-12
    return [h_pin * x / n for x in m]


def berg_luscher(m):
    """Sum over plaquettes of the solid angles of triangles (a, b, d) and (a, d, c), / 4 pi."""
    m = np.asarray(m, float)
    n1, n2 = m.shape[0], m.shape[1]

    def unit(v):
        return v / (np.linalg.norm(v) + 1e-12)

    def omega(p, q, w):
        num = float(np.dot(p, np.cross(q, w)))
        den = 1.0 + float(np.dot(p, q)) + float(np.dot(q, w)) + float(np.dot(w, p))
        return 2.0 * math.atan2(num, den)

    tot = 0.0
    for i in range(n1):
        for j in range(n2):
            a, b = unit(m[i, j]), unit(m[(i + 1) % n1, j])
            c, d = unit(m[i, (j + 1) % n2]), unit(m[(i + 1) % n1, (j + 1) % n2])
            tot += omega(a, b, d) + omega(a, d, c)
    return tot / (4.0 * math.pi)


def slater_spin_density_at(r, Gs, W):
    """m(r) of the determinant with orbitals phi_a(r, s) = sum_G W[a, G, s] e^{i G.r}."""
    Gs = np.asarray(Gs, float)
    W = np.asarray(W, complex)
    mx = my = mz = 0.0
    for a in range(W.shape[0]):
        up = dn = 0j
        for g in range(Gs.shape[0]):
            e = complex(math.cos(Gs[g] @ r), math.sin(Gs[g] @ r))
            up += W[a, g, 0] * e
            dn += W[a, g, 1] * e
        c = up.conjugate() * dn
        mx += 2.0 * c.real
        my += 2.0 * c.imag
        mz += abs(up) ** 2 - abs(dn) ** 2
    return [mx, my, mz]
