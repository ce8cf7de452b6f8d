"""Counter-based keys standing in for jax.random keys on the host side.

A key is a (seed, counter) pair of 64-bit integers. ``PRNGKey(seed)``, ``split`` and ``fold_in``
mirror the jax.random calls the reference drivers make (minsr.py:130-140, sampler.py:79-91);
the device streams are Philox4x32-10 keyed by the seed with the counter as the sweep index, so
they are NOT the reference's threefry streams (no test of the reference pins those).
"""
from __future__ import annotations

_M64 = (1 << 64) - 1


def _mix(x: int) -> int:
    """splitmix64 finaliser (Steele, Lea, Flood 2014)."""
    x = (x + 0x9E3779B97F4A7C15) & _M64
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & _M64
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & _M64
    return x ^ (x >> 31)


def PRNGKey(seed: int):
    return (int(seed) & _M64, 0)


def key_to_seed(key) -> int:
    if isinstance(key, tuple):
        return _mix(key[0] ^ _mix(key[1])) & 0x7FFFFFFF
    return int(key) & 0x7FFFFFFF


def as_key(key):
    return key if isinstance(key, tuple) else PRNGKey(key)


def fold_in(key, data: int):
    s, c = as_key(key)
    return (_mix(s ^ _mix(int(data) + 0x632BE59BD9B4E019)), c)


def split(key, num: int = 2):
    s, c = as_key(key)
    return [(_mix(s + 0x9E3779B97F4A7C15 * (i + 1)), c) for i in range(num)]
