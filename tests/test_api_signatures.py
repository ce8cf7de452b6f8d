"""Drop-in check of the Python surface: every public function of the reference modules on the
path (src/nqs/{psiformer, local_energy, ewald, sampler, minsr, train, cell, rashba_reference,
slater_reference, spiral_reference, pinning, observables}.py) exists in the matching nqs module,
and the reference's parameters are a prefix of ours with the same names, order and defaults
(extra trailing keyword arguments - precision, gram, cell - are the stated adaptations). The
reference signatures come from tests/golden/reference_signatures.json, which
tests/golden/make_signatures.py reads from the reference sources with `ast` (no JAX needed); when
a checkout is named by NQS_REFERENCE_ROOT the fixture is also checked against it. Functions off
the VMC iteration's path (texture post-processing, Hartree-Fock texture files, the
skyrmion-background envelope) are not part of this library."""
import importlib
import inspect
import json
import os
import sys

import pytest
import torch

MODULES = {"psiformer": "psiformer", "local_energy": "local_energy", "ewald": "ewald",
           "sampler": "sampler", "minsr": "minsr", "train": "train", "cell": "cell",
           "rashba_reference": "rashba", "slater_reference": "slater",
           "spiral_reference": "spiral", "pinning": "pinning", "observables": "observables"}
GOLD = os.path.join(os.path.dirname(__file__), "golden", "reference_signatures.json")
REF = os.path.join(os.environ.get("NQS_REFERENCE_ROOT", ""), "src", "nqs")
HAVE_REF = bool(os.environ.get("NQS_REFERENCE_ROOT")) and os.path.isdir(REF)
OFF_PATH = {"observables": {"spin_texture", "berg_luscher", "structure_factor",
                            "spin_order_parameter", "skx_arms", "skyrmion_number_fourier",
                            "slater_spin_density", "classify_state"},
            "pinning": {"load_hf_texture", "make_hf_skx_pin", "berg_luscher_realspace"},
            "rashba_reference": {"cell_skx_envelope", "ring_minimum"},
            "spiral_reference": {"spin_texture"}}


def _golden():
    with open(GOLD) as f:
        return json.load(f)


def _check_module(ref_mod, funcs):
    ours = importlib.import_module("nqs." + MODULES[ref_mod])
    for name, params in funcs.items():
        if name in OFF_PATH.get(ref_mod, ()):
            continue
        f = getattr(ours, name, None)
        assert f is not None, f"{ref_mod}.{name} missing"
        sig = inspect.signature(f)
        names = list(sig.parameters)
        assert names[:len(params)] == [n for n, _ in params], (name, names)
        for n, d in params:
            if d["kind"] != "literal":
                continue  # no default, or a non-literal one (an expression of other names)
            ours_d = sig.parameters[n].default
            assert type(ours_d).__name__ == d["type"], (name, n)
            assert json.loads(json.dumps(ours_d)) == d["value"], (name, n)


@pytest.mark.parametrize("ref_mod", sorted(MODULES))
def test_signatures_match_reference(ref_mod):
    _check_module(ref_mod, _golden()["modules"][ref_mod])


@pytest.mark.skipif(not HAVE_REF, reason="reference checkout not given (NQS_REFERENCE_ROOT)")
def test_signature_fixture_is_current():
    """The committed fixture equals what the reference sources give today."""
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import make_signatures
    live = {m: make_signatures.functions(os.path.join(REF, m + ".py")) for m in MODULES}
    assert json.loads(json.dumps(live)) == _golden()["modules"]


def test_split_merge_heads_roundtrip():
    from nqs.psiformer import merge_heads, split_heads
    x = torch.arange(2 * 5 * 12, dtype=torch.float64).reshape(2, 5, 12)
    h = split_heads(x, 4)
    assert h.shape == (2, 4, 5, 3)
    assert torch.equal(h[1, 2, 3], x[1, 3, 6:9])  # head 2 = features [6, 9)
    assert torch.equal(merge_heads(h), x)


def test_wavefunction_fields_match_reference():
    """ContinuumSpinorPsiformer's constructor fields and defaults equal the flax module's
    (psiformer.py:100-116)."""
    from nqs.psiformer import ContinuumSpinorPsiformer
    fields = _golden()["psiformer_fields"]
    sig = inspect.signature(ContinuumSpinorPsiformer)
    assert list(sig.parameters)[:len(fields)] == [n for n, _ in fields]
    for n, v in fields:
        if v["kind"] == "literal":
            ours_d = sig.parameters[n].default
            assert type(ours_d).__name__ == v["type"], n
            assert json.loads(json.dumps(ours_d)) == v["value"], n
