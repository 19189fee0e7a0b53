"""Generate the PME golden fixtures under tests/golden/pme/ (run in a
container that has the reference; the GPU box does not).

Source: the reference smooth-PME comparator itself (code/pme0.c,
code/pme1.c, unmodified), built by oracle/build_ref.py into
oracle/_ref/libpme_ref.so, run through its own C API (code/pme.h) on the
reference's data files (data/*.ini, CC0): energy, forces, the chosen
parameters (grid, beta), the constant-term coefficients, the error estimate
and, for small systems, per-atom potentials by central differences in q
(exact: U is quadratic in q).

Usage: python tests/golden/make_golden_pme.py [--reference DIR]   (default: $MSMPB_REFERENCE)
"""
import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "pme")
sys.path.insert(0, ROOT)

from oracle import build_ref  # noqa: E402
from oracle.oracle import RefPme, read_ini  # noqa: E402

# name, data file, FF_set_* parameters (omitted = the reference default), potentials?
CASES = [
    ("spceN300_auto", "spceN300", dict(), True),
    ("spceN600_a9_nu4", "spceN600", dict(cutoff=9.0, nu=4), True),
    ("spceN900_a7_tol1e-6", "spceN900", dict(cutoff=7.0, tol_dir=1e-6), False),
    ("spceN2250_a10_M32", "spceN2250", dict(cutoff=10.0, nu=6, grid=32), False),
    ("NaClN512_a6_M16", "NaClN512", dict(cutoff=6.0, nu=6, grid=16), True),
    # a box edge (2 A) shorter than the cutoff: an ion's own images count
    ("CsClN16_a3_M8_nu4", "CsClN16", dict(cutoff=3.0, nu=4, grid=8), True),
]


def potentials(r):
    out = []
    for i in range(r.N):
        q0 = r.q[i]
        r.q[i] = q0 + 1.0
        ep, _ = r.energy()
        r.q[i] = q0 - 1.0
        em, _ = r.energy()
        r.q[i] = q0
        out.append((ep - em) / 2.0)
    return np.array(out)


def make(reference):
    build_ref.build(reference, quiet=True)
    data = os.path.join(reference, "data")
    os.makedirs(OUT, exist_ok=True)
    index = {}
    for name, src, kw, pots in CASES:
        edges, q, pos, _ = read_ini(os.path.join(data, src + ".ini"))
        r = RefPme(q, pos, edges, **kw)
        e, f = r.energy()
        s = r.struct()
        out = dict(q=q, pos=pos, edges=edges, energy=np.array(e), force=f,
                   cutoff=np.array(r.cutoff), nu=np.array(r.nu), grid=np.array(r.grid),
                   tol_dir=np.array(r.tol_dir), beta=np.array(r.beta),
                   coeff1=np.array(s.coeff1), coeff2=np.array(s.coeff2),
                   err_est=np.array(r.err_est()))
        if pots:
            out["phi"] = potentials(r)
        r.close()
        np.savez_compressed(os.path.join(OUT, name + ".npz"), **out)
        index[name] = dict(source="data/%s.ini" % src, set=kw, energy=e, grid=list(r.grid),
                           beta=r.beta)
        print(name, e, r.grid)
    with open(os.path.join(OUT, "index.json"), "w") as fh:
        json.dump(index, fh, indent=1)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=build_ref.REFERENCE)
    make(ap.parse_args().reference)
