"""Drop-in check of the Python surface: every public function of the reference modules on the
path (src/nqs/{psiformer, local_energy, ewald, sampler, minsr, train, cell, rashba_reference,
slater_reference, spiral_reference, pinning, observables}.py) exists in the matching nqs module,
and the reference's parameters are a prefix of ours with the same names, order and defaults
(extra trailing keyword arguments - precision, gram, cell - are the stated adaptations). Reads the
reference sources with `ast` (no JAX needed); skipped where the reference is not mounted."""
import ast
import importlib
import inspect
import os

import pytest
import torch

REF = "/root/reference/src/nqs"
MODULES = {"psiformer": "psiformer", "local_energy": "local_energy", "ewald": "ewald",
           "sampler": "sampler", "minsr": "minsr", "train": "train", "cell": "cell",
           "rashba_reference": "rashba", "slater_reference": "slater",
           "spiral_reference": "spiral", "pinning": "pinning", "observables": "observables"}


def _reference_functions(mod):
    tree = ast.parse(open(os.path.join(REF, mod + ".py")).read())
    for node in tree.body:
        if isinstance(node, ast.FunctionDef) and not node.name.startswith("_"):
            a = node.args
            pos = a.posonlyargs + a.args
            defaults = [None] * (len(pos) - len(a.defaults)) + list(a.defaults)
            params = [(p.arg, d) for p, d in zip(pos, defaults)]
            params += [(p.arg, d) for p, d in zip(a.kwonlyargs, a.kw_defaults)]
            yield node.name, params


@pytest.mark.skipif(not os.path.isdir(REF), reason="reference not mounted")
@pytest.mark.parametrize("ref_mod", sorted(MODULES))
def test_signatures_match_reference(ref_mod):
    ours = importlib.import_module("nqs." + MODULES[ref_mod])
    for name, params in _reference_functions(ref_mod):
        f = getattr(ours, name, None)
        assert f is not None, f"{ref_mod}.{name} missing"
        sig = inspect.signature(f)
        names = list(sig.parameters)
        assert names[:len(params)] == [n for n, _ in params], (name, names)
        for n, d in params:
            ours_d = sig.parameters[n].default
            if d is None:
                continue
            try:
                ref_d = ast.literal_eval(d)
            except ValueError:
                continue  # a non-literal default (an expression of other names)
            assert ours_d == ref_d, (name, n, ours_d, ref_d)


def test_split_merge_heads_roundtrip():
    from nqs.psiformer import merge_heads, split_heads
    x = torch.arange(2 * 5 * 12, dtype=torch.float64).reshape(2, 5, 12)
    h = split_heads(x, 4)
    assert h.shape == (2, 4, 5, 3)
    assert torch.equal(h[1, 2, 3], x[1, 3, 6:9])  # head 2 = features [6, 9)
    assert torch.equal(merge_heads(h), x)


@pytest.mark.skipif(not os.path.isdir(REF), reason="reference not mounted")
def test_wavefunction_fields_match_reference():
    """ContinuumSpinorPsiformer's constructor fields and defaults equal the flax module's
    (psiformer.py:100-116)."""
    from nqs.psiformer import ContinuumSpinorPsiformer
    tree = ast.parse(open(os.path.join(REF, "psiformer.py")).read())
    cls = next(n for n in tree.body
               if isinstance(n, ast.ClassDef) and n.name == "ContinuumSpinorPsiformer")
    fields = [(s.target.id, s.value) for s in cls.body if isinstance(s, ast.AnnAssign)]
    sig = inspect.signature(ContinuumSpinorPsiformer)
    assert list(sig.parameters)[:len(fields)] == [n for n, _ in fields]
    for n, v in fields:
        if v is not None:
            assert sig.parameters[n].default == ast.literal_eval(v), n
