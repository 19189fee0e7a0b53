"""The smooth-PME comparator (libpme.so behind include/pme.h).

Without a GPU: the oracle (oracle/pme_oracle.c) is pinned to the reference
PME built from its own sources (tests/golden/pme/, made by
tests/golden/make_golden_pme.py; and live through oracle/_ref/libpme_ref.so
when present); the library's host-side parameter choice and tables match
the oracle; the C ABI exports every symbol of include/pme.h and
include/pme_b200.h with the reference's struct layout; the reference's
exit paths become error codes.

On the GPU: energies, forces and potentials against the fixtures and the
oracle, FP64 to 1e-10 and the mixed form to the FP32 level, plus weights,
rebuild and the device-pointer entry point.
"""
import ctypes as C
import json
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

from msmpb_b200 import _lib
from msmpb_b200.pme import PME, PMEError
from oracle import build_ref
from oracle.oracle import PmeOracle, RefPme

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden", "pme")
INCLUDE = os.path.join(ROOT, "include")
REF_CODE = os.path.join(build_ref.REFERENCE, "code")


def cases():
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz"))


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def set_params(d):
    """The FF_set_* values recorded for a fixture (index.json)."""
    with open(os.path.join(GOLDEN, "index.json")) as f:
        kw = dict(json.load(f)[d])["set"]
    return kw


def force_scale(d):
    """The larger of the driver's Fref (code/pme.c:206-208) and the RMS
    force: crystal forces vanish by symmetry and are rounding noise."""
    q, edges = d["q"], d["edges"]
    n = len(q)
    fref = (q @ q / n) / (abs(np.linalg.det(edges)) / n) ** (2.0 / 3.0)
    return max(fref, float(np.sqrt((d["force"] ** 2).sum() / n)))


def rms(a):
    return float(np.sqrt((np.asarray(a) ** 2).sum() / len(a)))


def oracle_for(name, d):
    kw = set_params(name)
    return PmeOracle(d["q"], d["edges"], cutoff=kw.get("cutoff", -1), nu=kw.get("nu", -1),
                     grid=kw.get("grid"), tol_dir=kw.get("tol_dir", -1))


def pme_for(name, d, precision="mixed"):
    kw = set_params(name)
    return PME(d["q"], d["pos"], d["edges"], cutoff=kw.get("cutoff"), order=kw.get("nu"),
               grid=kw.get("grid"), tol_dir=kw.get("tol_dir"), precision=precision)


# --------------------------------------------------------------- no GPU ----

@pytest.mark.parametrize("name", cases())
def test_oracle_matches_reference_fixtures(name):
    d = load(name)
    o = oracle_for(name, d)
    assert o.grid == tuple(d["grid"])
    assert o.beta == pytest.approx(float(d["beta"]), rel=1e-15)
    c1, c2 = o.coeffs()
    assert c1 == pytest.approx(float(d["coeff1"]), rel=1e-13, abs=1e-15)
    assert c2 == pytest.approx(float(d["coeff2"]), rel=1e-13)
    assert o.err_est() == pytest.approx(float(d["err_est"]), rel=1e-13)
    e, f, phi = o.energy(d["pos"])
    assert abs(e - float(d["energy"])) <= 1e-12 * abs(float(d["energy"]))
    assert rms(f - d["force"]) <= 1e-10 * force_scale(d)
    if "phi" in d:
        assert rms(phi - d["phi"]) <= 1e-10 * rms(d["phi"])
    # U = 1/2 sum q phi (the potentials are dU/dq: U is quadratic in q)
    assert abs(0.5 * d["q"] @ phi - e) <= 1e-12 * abs(e)


@pytest.mark.skipif(not RefPme.available(), reason="reference PME not built")
def test_oracle_matches_reference_live():
    """Random ion boxes, orthorhombic and triclinic, explicit and default
    parameters, against the reference library run here."""
    rng = np.random.default_rng(5)
    for edges, kw in ((np.diag([21.0, 23.0, 22.0]), dict()),
                      (np.array([[20.0, 2.0, 1.0], [0.0, 21.0, 3.0], [0.0, 0.0, 22.0]]),
                       dict(cutoff=7.5, nu=4, grid=(20, 24, 18))),
                      (np.diag([9.0, 9.0, 9.0]), dict(cutoff=10.0, nu=6, grid=12,
                                                      tol_dir=1e-7))):
        n = 200
        q = rng.choice([-1.0, 1.0], n)
        pos = rng.uniform(0, 1, (n, 3)) @ edges.T
        r = RefPme(q, pos, edges, **kw)
        o = PmeOracle(q, edges, cutoff=kw.get("cutoff", -1), nu=kw.get("nu", -1),
                      grid=kw.get("grid"), tol_dir=kw.get("tol_dir", -1))
        assert o.grid == r.grid and o.beta == r.beta
        er, fr = r.energy()
        eo, fo, _ = o.energy(pos)
        assert abs(eo - er) <= 1e-12 * abs(er)
        assert rms(fo - fr) <= 1e-11 * rms(fr)
        assert np.allclose(o.khat(), r.khat(), rtol=1e-13, atol=1e-13 * np.abs(r.khat()).max())
        r.close()


def test_oracle_rebuild_matches_fresh_build():
    d = load("spceN300_auto")
    o = PmeOracle(d["q"], d["edges"], grid=16)
    o.rebuild(d["edges"] * 1.02)
    fresh = PmeOracle(d["q"], d["edges"] * 1.02, grid=16)
    assert o.beta == fresh.beta and o.coeffs() == fresh.coeffs()
    assert np.array_equal(o.khat(), fresh.khat())


@pytest.mark.parametrize("name", cases())
def test_host_tables_match_oracle(name):
    """FF_build on the host (no device needed): grid, beta, constants,
    multiplier and error estimate as the oracle computes them."""
    d = load(name)
    p = pme_for(name, d)
    o = oracle_for(name, d)
    assert p.grid == o.grid and p.order == o.nu and p.cutoff == o.cutoff
    assert p.tol_dir == o.tol_dir and p.beta == o.beta
    c1, c2 = p.coeffs()
    o1, o2 = o.coeffs()
    assert c1 == pytest.approx(o1, rel=1e-14, abs=1e-16) and c2 == pytest.approx(o2, rel=1e-14)
    kh, ko = p.khat(), o.khat()
    assert np.abs(kh - ko).max() <= 1e-14 * np.abs(ko).max()
    assert p.err_est() == pytest.approx(o.err_est(), rel=1e-14)
    p.close()


def test_no_default_grid_is_an_error_not_an_exit():
    """The reference prints and exits when its spacing table has no entry
    (order 8, or a cutoff outside 6..10 A; code/pme0.c:230-242)."""
    d = load("spceN300_auto")
    for kw in (dict(order=8), dict(cutoff=12.0), dict(cutoff=5.0)):
        with pytest.raises(PMEError) as ex:
            PME(d["q"], d["pos"], d["edges"], **kw)
        assert ex.value.code == _lib.ERR_UNSUPPORTED
    PME(d["q"], d["pos"], d["edges"], order=8, grid=16).close()  # explicit grid: fine


def header_functions(headers):
    out = []
    for h in headers:
        text = open(os.path.join(INCLUDE, h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"#define.*?(\n(?!\s)|$)", "\n", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \*\(\)]*?\b(\w+)\s*\([^;{]*\)\s*;", text, re.M):
            if m.group(1) not in ("if", "while", "sizeof"):
                out.append(m.group(1))
    return sorted(set(out))


def test_pme_exports_every_declared_symbol():
    lib = _lib.load_pme()
    declared = header_functions(("pme.h", "pme_b200.h"))
    assert len(declared) >= 28
    assert not [n for n in declared if not hasattr(lib, n)]
    assert set(declared) <= set(_lib.PME_EXPORTED)


PME_FIELDS = ["N", "q", "A", "Ai", "detA", "cutoff", "orderAcc", "topGridDim", "nlist",
              "nlist_len", "nlist_interaction_count", "tolDir", "fftw_in", "forward",
              "backward", "beta", "Q", "cL", "khat", "coeff1", "coeff2", "time_partcl2partcl",
              "time_nlist", "time_grid2grid", "time_stencil", "time_anterpolation",
              "time_interpolation"]


@pytest.mark.skipif(not os.path.isdir(REF_CODE) or not shutil.which("gcc"),
                    reason="reference headers not present")
def test_struct_layout_matches_reference_pme(tmp_path):
    """Every member of the reference's PME struct FF sits at the same offset
    (code/pme.h:16-44), so code/pme.c reads our struct unchanged."""
    src = ['#include <stdio.h>', '#include <stddef.h>', '#include "pme.h"', 'struct O o;',
           'int main(void){']
    src += ['printf("%s %%zu\\n", offsetof(FF, %s));' % (f, f) for f in PME_FIELDS]
    src.append('return 0;}')
    res = {}
    for tag, incs in (("ours", ["-I", INCLUDE]),
                      ("ref", ["-I", os.path.join(ROOT, "oracle", "fftw_shim"), "-I", REF_CODE])):
        c = tmp_path / ("off_%s.c" % tag)
        c.write_text("\n".join(src))
        exe = tmp_path / ("off_%s" % tag)
        subprocess.run(["gcc", "-std=gnu11", *incs, str(c), "-o", str(exe)], check=True)
        res[tag] = subprocess.run([str(exe)], capture_output=True, text=True).stdout
    assert res["ours"] == res["ref"]


# ----------------------------------------------------------------- GPU ----

TOL = {"fp64": (1e-11, 1e-10, 1e-10), "mixed": (1e-6, 1e-5, 1e-5)}


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", cases())
def test_gpu_matches_reference_fixtures(name, precision):
    d = load(name)
    p = pme_for(name, d, precision)
    e, f, phi = p.energy(d["pos"], potentials=True)
    te, tf, tp = TOL[precision]
    ref = float(d["energy"])
    assert abs(e - ref) <= te * abs(ref), (e, ref)
    assert rms(f - d["force"]) <= tf * force_scale(d)
    if "phi" in d:
        assert rms(phi - d["phi"]) <= tp * rms(d["phi"])
    p.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_gpu_matches_oracle_triclinic_and_weights(precision):
    rng = np.random.default_rng(9)
    edges = np.array([[24.0, 3.0, 1.5], [0.0, 23.0, 2.0], [0.0, 0.0, 25.0]])
    n = 1200
    q = rng.choice([-1.0, 1.0], n)
    pos = rng.uniform(0, 1, (n, 3)) @ edges.T
    w = np.array([0.75, 1.5])
    o = PmeOracle(q, edges, cutoff=8.5, nu=6, grid=(24, 24, 25))
    p = PME(q, pos, edges, cutoff=8.5, order=6, grid=(24, 24, 25), precision=precision)
    te, tf, tp = TOL[precision]
    for weight in (None, w):
        eo, fo, po = o.energy(pos, weight=weight)
        e, f, phi = p.energy(pos, weights=weight, potentials=True)
        assert abs(e - eo) <= te * abs(eo) * 10
        assert rms(f - fo) <= tf * rms(fo)
        assert rms(phi - po) <= tp * rms(po)
    p.close()


@pytest.mark.gpu
def test_gpu_rebuild_and_device_entry():
    import torch
    d = load("spceN600_a9_nu4")
    p = pme_for("spceN600_a9_nu4", d, "fp64")
    edges2 = d["edges"] * 1.015
    pos2 = d["pos"] * 1.015
    p.rebuild(edges2, pos2)
    o = PmeOracle(d["q"], edges2, cutoff=9.0, nu=4, grid=p.grid)
    eo, fo, po = o.energy(pos2)
    e, f = p.energy(pos2)
    assert abs(e - eo) <= 1e-11 * abs(eo)
    assert rms(f - fo) <= 1e-10 * rms(fo)
    dev = torch.device("cuda", 0)
    pd = torch.tensor(pos2, device=dev)
    qd = torch.tensor(d["q"], device=dev)
    fd = torch.empty((len(d["q"]), 3), dtype=torch.float64, device=dev)
    phid = torch.empty(len(d["q"]), dtype=torch.float64, device=dev)
    ed = torch.empty(1, dtype=torch.float64, device=dev)
    p.set_timing(False)  # graph replay
    p.energy_device(pd.data_ptr(), qd.data_ptr(), fd.data_ptr(), phid.data_ptr(), ed.data_ptr(),
                    torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert abs(ed.item() - eo) <= 1e-11 * abs(eo)
    assert rms(fd.cpu().numpy() - fo) <= 1e-10 * rms(fo)
    assert rms(phid.cpu().numpy() - po) <= 1e-10 * rms(po)
    p.close()
