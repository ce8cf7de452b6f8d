"""Pinning fields, one point at a time — TEST INFRASTRUCTURE.

Only tests/ may import this module. It restates, in plain per-point Python, the reference's
pinning-field definitions (src/nqs/pinning.py:20-72: triple-Q skyrmion, uniform FM, single-Q
spiral, Overhauser wave), so that the vectorised ext_field callables of nqs.pinning can be
checked against an independent evaluation. The reference module imports JAX and cannot run
here; parity is therefore pinned to these formulas and to the field magnitude h_pin.
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
