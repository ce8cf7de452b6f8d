"""Writes tests/golden/reference_signatures.json: the public function signatures (parameter names,
order and literal defaults) of the reference modules on the VMC path, and the constructor fields
of ContinuumSpinorPsiformer, read from the reference sources with `ast` (no JAX needed).

Run from the repository root with the reference checkout as argument (or NQS_REFERENCE_ROOT):
    python tests/golden/make_signatures.py /path/to/continuum-nqs
"""
import ast
import json
import os
import sys

MODULES = ["cell", "ewald", "local_energy", "minsr", "observables", "pinning", "psiformer",
           "rashba_reference", "sampler", "slater_reference", "spiral_reference", "train"]


def _literal(node):
    if node is None:
        return {"kind": "none"}
    try:
        v = ast.literal_eval(node)
        return {"kind": "literal", "value": v, "type": type(v).__name__}
    except ValueError:
        return {"kind": "expr"}  # a default computed from other names


def functions(path):
    tree = ast.parse(open(path).read())
    out = {}
    for node in tree.body:
        if isinstance(node, ast.FunctionDef) and not node.name.startswith("_"):
            a = node.args
            pos = a.posonlyargs + a.args
            defaults = [None] * (len(pos) - len(a.defaults)) + list(a.defaults)
            params = [[p.arg, _literal(d)] for p, d in zip(pos, defaults)]
            params += [[p.arg, _literal(d)] for p, d in zip(a.kwonlyargs, a.kw_defaults)]
            out[node.name] = params
    return out


def main(root):
    src = os.path.join(root, "src", "nqs")
    out = {"modules": {m: functions(os.path.join(src, m + ".py")) for m in MODULES}}
    tree = ast.parse(open(os.path.join(src, "psiformer.py")).read())
    cls = next(n for n in tree.body
               if isinstance(n, ast.ClassDef) and n.name == "ContinuumSpinorPsiformer")
    out["psiformer_fields"] = [[s.target.id, _literal(s.value)] for s in cls.body
                               if isinstance(s, ast.AnnAssign)]
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_signatures.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("NQS_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: make_signatures.py <reference checkout> (or set NQS_REFERENCE_ROOT)")
    main(root)
