"""Helpers to read the committed golden fixtures (tests/golden/<case>/)."""
import gzip
import hashlib
import json
import os

import numpy as np

from prism_b200 import fields

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = {c["name"]: c for c in json.load(open(os.path.join(GOLDEN, "cases.json")))}


def meta(name):
    m = {}
    for line in open(os.path.join(GOLDEN, name, "meta.txt")):
        k, *v = line.split()
        m.setdefault(k, []).append(v)
    return m


def digests(name):
    d = {}
    for line in open(os.path.join(GOLDEN, name, "digests.txt")):
        f, s, h = line.split()
        d[f] = (int(s), h)
    return d


def raw(name, fn):
    p = os.path.join(GOLDEN, name, fn + ".gz")
    return gzip.open(p).read() if os.path.exists(p) else None


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def dtype_of(case):
    return np.float32 if case["dtype"] == "f" else np.float64


def field(name):
    c = CASES[name]
    nx, ny, nz = c["dims"]
    return fields.make(c["gen"], (nz, ny, nx), dtype_of(c), c["seed"])


def flags(name):
    m = meta(name)
    return [int(v) for v in m["use_md"][0]], [int(v) for v in m["reverse"][0]]


def steps(name):
    out = []
    for v in meta(name).get("step", []):
        # step i target t begin b0 b1 b2 b3 end e0 e1 e2 e3 maxlevel m
        b = [int(x) for x in v[4:8]]
        e = [int(x) for x in v[9:13]]
        out.append((float(v[2]), b, e, int(v[14])))
    return out
