"""Generate the golden fixtures under tests/golden/ (run in a container that
has the reference; the GPU box does not).

Sources:
* the reference's own fixtures (data/*.ini positions and charges, *.pot
  high-accuracy energies, *.acc high-accuracy -F/q; CC0, data/LICENSE);
* the reference library itself, built by oracle/build_ref.py (the shipped
  sources plus the two documented index patches), run through its C API on
  those inputs: energy, forces and (for small systems) potentials by central
  differences in q (exact, U is quadratic in q);
* published values from results/TableII.json, results/Figure1.txt.

Usage: python tests/golden/make_golden.py [--reference DIR]   (default: $MSMPB_REFERENCE)
"""
import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import build_ref  # noqa: E402
from oracle.oracle import RefFF, read_acc, read_ini  # noqa: E402

# name, data file, FF_set_* parameters (None = automatic), potentials?
CASES = [
    ("spceN300_M24_a9_nu4", "spceN300", dict(levels=1, top_grid=24, cutoff=9.0, nu=4), True),
    ("spceN300_M30_a11_nu10", "spceN300", dict(levels=1, top_grid=30, cutoff=11.0, nu=10), True),
    ("spceN600_M20_a8_nu6", "spceN600", dict(levels=1, top_grid=20, cutoff=8.0, nu=6), True),
    ("spceN2250_L2_M16_a9_nu6", "spceN2250", dict(levels=2, top_grid=16, cutoff=9.0, nu=6), False),
    ("spceN900_L3_M6_a8_nu8", "spceN900", dict(levels=3, top_grid=6, cutoff=8.0, nu=8), False),
    ("NaClN512_auto", "NaClN512", dict(levels=1), True),
    ("CsClN16_auto", "CsClN16", dict(), True),
    ("changaN512_L2_M8_a0.25_nu6", "changaN512", dict(levels=2, top_grid=8, cutoff=0.25, nu=6), True),
    ("changaN64_auto", "changaN64", dict(levels=1), True),
    ("Box44_L2_M18_a12_nu6", "Box44", dict(levels=2, top_grid=18, cutoff=12.0, nu=6), False),
]


def make(reference):
    build_ref.build(reference, quiet=True)
    data = os.path.join(reference, "data")
    index = {}
    for name, src, kw, pots in CASES:
        edges, q, pos, mass = read_ini(os.path.join(data, src + ".ini"))
        r = RefFF(q, pos, edges, **kw)
        e, f = r.energy()
        out = dict(q=q, pos=pos, edges=edges, energy=np.array(e), force=f,
                   cutoff=np.array(r.cutoff), nu=np.array(r.nu),
                   levels=np.array(r.levels), top_grid=np.array(r.top_grid),
                   nlim=np.array(r.nlim))
        if pots:
            out["phi"] = r.potentials()
        potf = os.path.join(data, src + ".pot")
        if os.path.exists(potf):
            out["pot_exact"] = np.array(float(open(potf).read().split()[0]))
        accf = os.path.join(data, src + ".acc")
        if os.path.exists(accf):
            out["acc_exact"] = read_acc(accf, len(q))
        if src == "Box44":  # keep the fixture small: no per-atom forces
            del out["force"]
            out["force_checksum"] = np.array([np.abs(f).sum(), (f ** 2).sum()])
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        index[name] = dict(source=src, params={k: v for k, v in kw.items()},
                           energy=e, N=len(q))
        r.close()
    # published numbers the oracle reproduces
    t2 = json.load(open(os.path.join(reference, "results", "TableII.json")))
    index["published"] = dict(
        TableII_Box44_L2_M18_utotal=t2["trial"][0]["msmout"]["utotal"],
        TableII_Box44_L2_M18_poterror=t2["trial"][0]["msmout"]["poterror"],
        Figure1=[l.split() for l in open(os.path.join(
            reference, "results", "Figure1.txt")).read().split("\n")[1:] if l.strip()],
    )
    with open(os.path.join(HERE, "index.json"), "w") as fh:
        json.dump(index, fh, indent=1)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=build_ref.REFERENCE)
    make(ap.parse_args().reference)
