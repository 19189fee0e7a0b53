"""Access to the committed golden fixtures (tests/golden/*.npz)."""
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def names():
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz"))


def load(name):
    d = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    d["name"] = name
    return d


def params(d):
    """FF_set_* parameters recorded for the case (what the reference chose)."""
    return dict(cutoff=float(d["cutoff"]), nu=int(d["nu"]),
                levels=int(d["levels"]), top_grid=tuple(int(v) for v in d["top_grid"]))


def index():
    with open(os.path.join(GOLDEN, "index.json")) as f:
        return json.load(f)


def rel_rms(a, b):
    """sqrt(sum |a-b|^2 / sum |b|^2)"""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.sqrt((b ** 2).sum())
    return float(np.sqrt(((a - b) ** 2).sum()) / max(den, 1e-300))
