"""The reference's CLI driver (code/msmpb.c), compiled unmodified against this
library (oracle/_ref/msmpb_dropin, built by oracle/build_ref.py), against the
same driver over the patched reference library (oracle/_ref/msmpb_ref), on
the same input files: .ini written from the golden fixtures, .acc and .pot
from the reference outputs recorded in them (code/msmpb.c:93-127, :254-360).

The JSON has the same keys in the same order. Values agree: the run set-up
(levels, order, grids, cutoff, edges) exactly, energies and error metrics to
FP64 rounding with MSMPB_PRECISION=fp64, the energy to the mixed form's
tolerance by default. Timings differ by construction; the pair-list counts
are 0 here (the pair set is rebuilt on the GPU at every evaluation, there is
no host list).
"""
import json
import os
import re
import subprocess

import numpy as np
import pytest

from golden_cases import load, params

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "msmpb_ref")
DROPIN = os.path.join(ROOT, "oracle", "_ref", "msmpb_dropin")

# (case, pass the recorded parameters on the command line)
CASES = [("spceN300_M24_a9_nu4", True), ("spceN900_L3_M6_a8_nu8", True),
         ("spceN2250_L2_M16_a9_nu6", True), ("changaN512_L2_M8_a0.25_nu6", True),
         ("CsClN16_auto", False), ("NaClN512_auto", False)]
SKIP = ("time_", "nlist_len", "nlist_interaction_count")
EXACT = ("data", "NumberOfLevels", "Nrep", "N", "repl", "Perturbationx", "Perturbationy",
         "Perturbationz", "nu", "ntc", "tmax", "cutoff", "margin", "Edge row1",
         "Edge row2", "Edge row3", "TopLevelMx", "TopLevelMy", "TopLevelMz")


def write_inputs(d, base):
    q, pos, edges = d["q"], d["pos"], d["edges"]
    with open(base + ".ini", "w") as f:
        f.write(" ".join("%.17g" % v for v in np.asarray(edges).ravel()) + "\n")
        f.write("%d\n" % len(q))
        for qi, p in zip(q, pos):
            f.write("%.17g %.17g %.17g %.17g 1.0\n" % (qi, p[0], p[1], p[2]))
    with open(base + ".pot", "w") as f:
        f.write("%.17g\n" % float(d["energy"]))
    if np.all(q != 0):  # the driver turns accelerations into forces, F = -q acc
        acc = -d["force"] / q[:, None]
        with open(base + ".acc", "w") as f:
            f.write("accelerations\n")
            for k in range(3):
                f.write("".join("%.17g\n" % v for v in acc[:, k]))


def run(exe, base, args, env):
    p = subprocess.run([exe, base, *args], cwd=os.path.dirname(base), env=env,
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    text = re.sub(r",\s*}\s*$", "}", p.stdout.strip())  # no .pot: trailing comma
    return json.loads(text, object_pairs_hook=lambda kv: kv)


@pytest.mark.skipif(not (os.path.exists(REF) and os.path.exists(DROPIN)),
                    reason="reference drivers not built (oracle/build_ref.py)")
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("case,explicit", CASES)
def test_cli_driver_parity(tmp_path, case, explicit, precision):
    d = load(case)
    base = str(tmp_path / case)
    write_inputs(d, base)
    args = []
    if explicit:
        p = params(d)
        args = ["--a0", repr(p["cutoff"]), "--nu", str(p["nu"]), "-M", str(p["top_grid"][0]),
                "-L", str(p["levels"])]
    env = dict(os.environ)
    env["MSMPB_PRECISION"] = precision
    ref = run(REF, base, args, env)
    ours = run(DROPIN, base, args, env)
    assert [k for k, _ in ours] == [k for k, _ in ref]
    rv, ov = dict(ref), dict(ours)
    u = abs(rv["utotal"])
    tol = 1e-10 if precision == "fp64" else 1e-5
    # differences from the recorded reference outputs, on their own scales:
    # forces on the larger of Fref and the RMS force (the non-neutral ChaNGa
    # boxes have forces far above Fref), as in test_gpu_parity.force_err
    fref = rv.get("fref", 1.0)
    fscale = max(fref, float(np.sqrt((d["force"] ** 2).sum() / len(d["q"]))))
    errors = {"deltaF": fscale, "deltaF/Fref": fscale / fref, "poterror": 1.0,
              "potabserror": u}
    # the energy and what is derived from it
    energies = {"utotal": u, "utotal_kcal_mol": 332.0636 * u}
    for k, v in rv.items():
        if k.startswith(SKIP):
            continue
        if k in EXACT:
            assert ov[k] == v, k
        elif k in errors:
            assert abs(ov[k] - v) <= 10 * tol * errors[k], (k, ov[k], v)
        elif k in energies:
            assert abs(ov[k] - v) <= tol * energies[k], (k, ov[k], v)
        else:  # set-up figures that do not depend on the arithmetic
            assert abs(ov[k] - v) <= 1e-12 * max(abs(v), 1e-300), (k, ov[k], v)


# ---- the PME comparator's driver (code/pme.c) ----
PME_REF = os.path.join(ROOT, "oracle", "_ref", "pme_ref")
PME_DROPIN = os.path.join(ROOT, "oracle", "_ref", "pme_dropin")
PME_GOLDEN = os.path.join(ROOT, "tests", "golden", "pme")
# keys that depend only on the inputs and the parameter choice
PME_EXACT = ("data", "nu", "beta", "TopLevelMx", "TopLevelMy", "TopLevelMz", "NumberOfLevels",
             "Edge row1", "Edge row2", "Edge row3", "cutoff", "nbar", "tol_dir", "detA",
             "fref", "uref", "Q2", "uintra")
# driver arguments per fixture (code/pme.c:40-58; --nu is parsed into a
# shadowing local there, so the order stays at its default in both builds)
PME_ARGS = {"spceN300_auto": [], "spceN900_a7_tol1e-6": ["--a0", "7.0", "--tol-dir", "1e-6"],
            "spceN2250_a10_M32": ["--a0", "10.0", "-M", "32"],
            "spceN600_a9_nu4": ["--a0", "9.0"]}
# (the driver sums an intramolecular energy over consecutive atom triples,
# code/pme.c:235-260, reading past the arrays unless N is a multiple of 3:
# only the water boxes are driven through it)


@pytest.mark.skipif(not (os.path.exists(PME_REF) and os.path.exists(PME_DROPIN)),
                    reason="reference PME drivers not built (oracle/build_ref.py)")
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("case", sorted(PME_ARGS))
def test_pme_cli_driver_parity(tmp_path, case, precision):
    d = dict(np.load(os.path.join(PME_GOLDEN, case + ".npz")))
    base = str(tmp_path / case)
    write_inputs(d, base)
    env = dict(os.environ)
    env["MSMPB_PRECISION"] = precision
    ref = run(PME_REF, base, PME_ARGS[case], env)
    ours = run(PME_DROPIN, base, PME_ARGS[case], env)
    assert [k for k, _ in ours] == [k for k, _ in ref]
    rv, ov = dict(ref), dict(ours)
    tol = 1e-10 if precision == "fp64" else 1e-5
    u = abs(rv["utotal"])
    fscale = max(rv["fref"], float(np.sqrt((d["force"] ** 2).sum() / len(d["q"]))))
    for k, v in rv.items():
        if k.startswith(("time_", "nlist_")):
            continue
        if k in PME_EXACT:
            assert ov[k] == v, k
        elif k in ("utotal", "utotal_kcal_mol", "potabserror"):
            scale = 332.0636 * u if k == "utotal_kcal_mol" else u
            assert abs(ov[k] - v) <= tol * scale, (k, ov[k], v)
        elif k in ("deltaF", "deltaF/Fref"):
            s = fscale if k == "deltaF" else fscale / rv["fref"]
            assert abs(ov[k] - v) <= 10 * tol * s, (k, ov[k], v)
        elif k == "poterror":
            assert abs(ov[k] - v) <= tol, (k, ov[k], v)
        else:
            raise AssertionError("unchecked key %s" % k)
