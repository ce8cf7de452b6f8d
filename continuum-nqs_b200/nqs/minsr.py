"""MinSR natural-gradient optimizer and driver (drop-in for src/nqs/minsr.py:30-159).

real_ravel flattens the parameter tree exactly as the reference (sorted keys; complex leaf ->
[re, im]), so theta / O columns line up with the reference's. per_sample_O, minsr_direction and
paramsr_direction run in libnqs kernels.
"""
from __future__ import annotations

import torch

F64 = torch.float64


def _flatten_sorted(tree, prefix=()):
    out = []
    for k in sorted(tree.keys()):
        v = tree[k]
        if isinstance(v, dict):
            out.extend(_flatten_sorted(v, prefix + (k,)))
        else:
            out.append((prefix + (k,), v))
    return out


def real_ravel(pytree):
    """Flatten a param tree to a REAL float64 vector (complex leaves -> [re, im]); returns
    (vec, unravel) (minsr.py:30-53). The vector lives on the leaves' device."""
    if "params" in pytree and isinstance(pytree["params"], dict) and len(pytree) == 1:
        wrapped = True
        tree = pytree["params"]
    else:
        wrapped = False
        tree = pytree
    leaves = _flatten_sorted(tree)
    specs, flats = [], []
    for path, leaf in leaves:
        leaf = torch.as_tensor(leaf)
        if leaf.is_complex():
            specs.append((path, True, tuple(leaf.shape), leaf.numel()))
            flats += [leaf.real.reshape(-1).to(F64), leaf.imag.reshape(-1).to(F64)]
        else:
            specs.append((path, False, tuple(leaf.shape), leaf.numel()))
            flats.append(leaf.reshape(-1).to(F64))
    dev = flats[0].device
    vec = torch.cat([f.to(dev) for f in flats])

    def unravel(v):
        out: dict = {}
        i = 0
        for path, is_c, shape, size in specs:
            if is_c:
                leaf = torch.complex(v[i:i + size], v[i + size:i + 2 * size]).reshape(shape)
                i += 2 * size
            else:
                leaf = v[i:i + size].reshape(shape)
                i += size
            node = out
            for k in path[:-1]:
                node = node.setdefault(k, {})
            node[path[-1]] = leaf
        return {"params": out} if wrapped else out

    return vec, unravel
