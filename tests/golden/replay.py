"""Helpers to read golden vectors recorded by ``make_golden.py`` (test
infrastructure): rebuild the argument tuples of each recorded reference call
and compare results with a tolerance."""
import re

import numpy as np

_KEY = re.compile(r"^(?P<fn>[A-Za-z0-9_]+)\.(?P<call>\d+)\.(?P<kind>in|out)(?P<idx>\d+(?:\.\d+)*)$")


def load(path):
    """{key: ndarray} of a golden file (blobs de-duplicated on disk)."""
    import json
    with np.load(path, allow_pickle=False) as z:
        blobs = {k: z[k] for k in z.files}
    index = json.loads(str(blobs.pop("index")))
    return {k: blobs[b] for k, b in index.items()}


def _insert(tree, idx, value):
    node = tree
    for i in idx[:-1]:
        node = node.setdefault(i, {})
    node[idx[-1]] = value


def _freeze(node):
    if not isinstance(node, dict):
        return node
    n = max(node) + 1
    return tuple(_freeze(node.get(i)) for i in range(n))


def calls(g):
    """{(fn, call): {"in": tuple, "out": tuple, "iteration": int}}"""
    trees = {}
    for k, v in g.items():
        m = _KEY.match(k)
        if not m:
            continue
        key = (m["fn"], int(m["call"]))
        t = trees.setdefault(key, {"in": {}, "out": {}})
        _insert(t[m["kind"]], [int(i) for i in m["idx"].split(".")], v)
    out = {}
    for key, t in trees.items():
        out[key] = {"in": _freeze(t["in"]) if t["in"] else (),
                    "out": _freeze(t["out"]) if t["out"] else (),
                    "iteration": int(g.get(f"{key[0]}.{key[1]}.iteration", -1))}
    return out


def flat(x, prefix="", out=None):
    """[(path, ndarray)] of every array leaf of a nested tuple."""
    if out is None:
        out = []
    if isinstance(x, (tuple, list)):
        for j, e in enumerate(x):
            flat(e, f"{prefix}.{j}" if prefix else str(j), out)
    elif x is not None:
        out.append((prefix, np.asarray(x)))
    return out


def rel_err(a, b):
    """max |a-b| / max(max|b|, tiny): the relative infinity-norm error."""
    a = np.asarray(a)
    b = np.asarray(b)
    scale = max(float(np.max(np.abs(b))) if b.size else 0.0, 1e-300)
    if a.shape != b.shape:
        return np.inf
    return float(np.max(np.abs(a - b))) / scale if b.size else 0.0
