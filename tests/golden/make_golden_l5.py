"""Generate tests/golden/water215_L5.npz: the headline grid depth (5 levels,
top grid 9^3, finest 144^3, a 25^3 stencil at levels 1-3 and a full-period
18^3 stencil at level 4) on the 215.30 A box of the 1M-atom workload, with
fewer atoms so that the CPU codes finish in minutes. The grid sizes, stencil
widths and level count depend on the box, the cutoff and the top grid, not on
the atom count.

Inputs: 2,000 seeded rigid 3-site waters (6,000 atoms, seed 21) in the cubic
215.30 A box; order 6, cutoff 9 A, 5 levels, top grid 9.

Outputs: energy and forces of the reference library itself (the patched
build of oracle/build_ref.py, run through its own C API: code/forcefield1.c
FF_energy), and per-atom potentials of the project's FP64 restatement
(oracle/msm_oracle.c; the reference has no potential output). The script
checks that the two CPU codes agree on energy and forces before it writes
anything. Run in a container that has the reference (the GPU box does not):

    python tests/golden/make_golden_l5.py [--reference DIR]   (default: $MSMPB_REFERENCE)
"""
import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from msmpb_b200 import systems  # noqa: E402
from oracle import build_ref  # noqa: E402
from oracle.oracle import Oracle, RefFF  # noqa: E402

NAME = "water215_L5"
N_WATERS, EDGE, SEED = 2000, 215.30, 21
PARAMS = dict(cutoff=9.0, nu=6, levels=5, top_grid=9)


def make(reference):
    build_ref.build(reference, quiet=True)
    q, pos, edges = systems.water(N_WATERS, EDGE, SEED)
    t0 = time.time()
    r = RefFF(q, pos, edges, **PARAMS)
    e, f = r.energy()
    geom = (r.cutoff, r.nu, r.levels, r.top_grid, r.nlim)
    r.close()
    t1 = time.time()
    o = Oracle(q, edges, **PARAMS)
    eo, fo, po = o.energy(pos)
    t2 = time.time()
    de = abs(eo - e) / abs(e)
    df = float(np.sqrt(((fo - f) ** 2).sum() / (f ** 2).sum()))
    print("reference %.1f s, oracle %.1f s; energy %.17g, oracle rel diff %.2e, "
          "force rel rms %.2e" % (t1 - t0, t2 - t1, e, de, df))
    if not (de < 1e-12 and df < 1e-11):
        raise SystemExit("oracle and reference disagree; nothing written")
    np.savez_compressed(os.path.join(HERE, NAME + ".npz"), q=q, pos=pos, edges=edges,
                        energy=np.array(e), force=f, phi=po,
                        cutoff=np.array(geom[0]), nu=np.array(geom[1]),
                        levels=np.array(geom[2]), top_grid=np.array(geom[3]),
                        nlim=np.array(geom[4]))


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=build_ref.REFERENCE)
    make(ap.parse_args().reference)
