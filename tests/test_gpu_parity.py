"""GPU parity: the CUDA library through its C ABI against the reference's own
outputs (golden fixtures made by the patched reference build) and against
the CPU oracle run live on the same inputs.

Tolerances (per-case, stated below): the FP64 GPU form must agree with the
FP64 reference to ~1e-10; the mixed form (FP32 bulk, FP64 FFT and sums) to
the FP32 rounding level, which sits orders of magnitude below the method's
own error (checked separately against the high-accuracy .acc/.pot data).
"""
import numpy as np
import pytest

from golden_cases import load, names, params, rel_rms
from msmpb_b200 import systems
from msmpb_b200.forcefield import ForceField
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

# (energy rel, force metric, potential rel-rms). The mixed bound is the FP32
# arithmetic level: sums of many cancelling terms (the rock-salt crystals'
# grid charges, the non-neutral ChaNGa boxes) lose a few FP32 digits; the
# method's own error is 1e-3..1e-8 for these parameters.
TOL = {"fp64": (1e-11, 1e-10, 1e-10), "mixed": (1e-5, 1e-4, 5e-5)}


def fref(q, edges):
    """Force scale of the reference's error metric (code/msmpb.c:271-273)."""
    n = len(q)
    return (q @ q / n) / (abs(np.linalg.det(edges)) / n) ** (2.0 / 3.0)


def force_err(f, g, q, edges):
    """RMS force difference over the larger of the reference driver's force
    scale Fref (code/msmpb.c:271-306; the right scale for the symmetric
    crystals, whose forces vanish) and the RMS reference force (the right
    scale for the non-neutral ChaNGa boxes, whose forces exceed Fref)."""
    rms = np.sqrt(((f - g) ** 2).sum() / len(q))
    scale = max(fref(q, edges), np.sqrt((g ** 2).sum() / len(q)))
    return rms / scale


def make_ff(d, precision):
    p = params(d)
    return ForceField(d["q"], d["pos"], d["edges"], cutoff=p["cutoff"],
                      order=p["nu"], levels=p["levels"], top_grid=p["top_grid"],
                      precision=precision)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("case", [n for n in names() if not n.startswith("Box44")])
def test_golden(case, precision):
    d = load(case)
    ff = make_ff(d, precision)
    e, f, phi = ff.energy(d["pos"], potentials=True)
    te, tf, tp = TOL[precision]
    scale = max(abs(float(d["energy"])), 1e-300)
    assert abs(e - float(d["energy"])) / scale < te
    assert force_err(f, d["force"], d["q"], d["edges"]) < tf
    if "phi" in d:
        assert rel_rms(phi, d["phi"]) < tp
    # U = 1/2 sum q_i phi_i holds for the quadratic form
    assert abs(0.5 * d["q"] @ phi - e) / scale < te * 10


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_box44_table2(precision):
    """Box44 (65,850 atoms), L=2, M=18, a0=12, nu=6: the published Table II
    energy (results/TableII.json) and the reference's force checksum."""
    d = load("Box44_L2_M18_a12_nu6")
    ff = make_ff(d, precision)
    e, f = ff.energy(d["pos"])
    te, _, _ = TOL[precision]
    assert abs(e - (-13831.986893278543)) / 13831.98 < te
    cs = d["force_checksum"]
    assert abs((f ** 2).sum() - cs[1]) / cs[1] < (1e-10 if precision == "fp64" else 1e-5)


def _oracle_case(name):
    q, pos, edges, kw = systems.config(name)
    return q, pos, edges, kw


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", ["water300", "rocksalt4096"])
def test_synthetic_vs_oracle(name, precision):
    q, pos, edges, kw = _oracle_case(name)
    o = Oracle(q, edges, cutoff=kw.get("cutoff", -1), nu=kw.get("order", -1),
               levels=kw.get("levels", -1), top_grid=kw.get("top_grid"))
    eo, fo, po = o.energy(pos)
    ff = ForceField(q, pos, edges, **kw, precision=precision)
    assert (ff.cutoff, ff.order, ff.levels, ff.top_grid) == (o.cutoff, o.nu, o.levels, o.top_grid)
    e, f, phi = ff.energy(pos, potentials=True)
    te, tf, tp = TOL[precision]
    assert abs(e - eo) / abs(eo) < te
    assert force_err(f, fo, q, edges) < tf
    assert rel_rms(phi, po) < tp


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_three_levels_truncated_stencil(precision):
    """L=3 with a truncated level-1 stencil (sd < M) and a full-period
    level-2 stencil (sd = M)."""
    q, pos, edges = systems.water(8000, 62.0, 11)
    kw = dict(cutoff=9.0, order=6, levels=3, top_grid=6)
    o = Oracle(q, edges, cutoff=9.0, nu=6, levels=3, top_grid=6)
    ff = ForceField(q, pos, edges, **kw, precision=precision)
    s1 = ff.khat(1).shape
    assert s1[0] < 24 and ff.khat(2).shape[0] == 12
    eo, fo, po = o.energy(pos)
    e, f, phi = ff.energy(pos, potentials=True)
    te, tf, tp = TOL[precision]
    assert abs(e - eo) / abs(eo) < te
    assert force_err(f, fo, q, edges) < tf
    assert rel_rms(phi, po) < tp


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_four_levels_shared_stencil_width(precision):
    """L=4: levels 1 and 2 use the same 13-wide stencil on 48^3 and 24^3
    grids (one kernel instantiation, two launch shapes), level 3 a
    full-period 12^3 stencil."""
    q, pos, edges = systems.water(64000, 124.0, 12)
    o = Oracle(q, edges, cutoff=9.0, nu=6, levels=4, top_grid=6)
    ff = ForceField(q, pos, edges, cutoff=9.0, order=6, levels=4, top_grid=6,
                    precision=precision)
    assert ff.khat(1).shape == ff.khat(2).shape == (13, 13, 13)
    eo, fo, po = o.energy(pos)
    e, f, phi = ff.energy(pos, potentials=True)
    te, tf, tp = TOL[precision]
    assert abs(e - eo) / abs(eo) < te
    assert force_err(f, fo, q, edges) < tf
    assert rel_rms(phi, po) < tp


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_five_levels_headline_depth(precision):
    """The grid hierarchy of the 1M-atom workload (215.30 A box, order 6,
    cutoff 9 A, 5 levels, top grid 9^3): finest grid 144^3, the truncated
    25^3 stencil at levels 1-3 (144^3, 72^3, 36^3), the full-period 18^3
    stencil at level 4 and the 9^3 FFT at level 5 (code/forcefield1.c:158-191,
    stencils code/forcefield0.c:661-675), here with 6,000 atoms: the reference
    library's own energy and forces and the oracle's potentials
    (tests/golden/make_golden_l5.py)."""
    d = load("water215_L5")
    ff = make_ff(d, precision)
    assert (ff.levels, ff.top_grid) == (5, (9, 9, 9))
    for level in (1, 2, 3):
        assert ff.khat(level).shape == (25, 25, 25)
    assert ff.khat(4).shape == (18, 18, 18)
    e, f, phi = ff.energy(d["pos"], potentials=True)
    te, tf, tp = TOL[precision]
    scale = abs(float(d["energy"]))
    assert abs(e - float(d["energy"])) / scale < te
    assert force_err(f, d["force"], d["q"], d["edges"]) < tf
    assert rel_rms(phi, d["phi"]) < tp
    assert abs(0.5 * d["q"] @ phi - e) / scale < te * 10


def test_mixed_close_to_fp64_on_dense_water():
    """The mixed form against the FP64 form on a water box at liquid density
    (24,000 atoms, order 6, cutoff 9 A, three levels): pairs closer than
    2.5 A (bonded and overlapping atoms) are summed in FP64 and the rest
    compensated, so the two forms agree to the FP32 rounding level of the far
    pairs, far below the method's error (~2e-6 of the force at these
    parameters): RMS force difference < 3e-7 of the RMS force, energy < 1e-8."""
    q, pos, edges = systems.water(8000, systems.water_edge(8000), 41)
    kw = dict(cutoff=9.0, order=6, levels=3, top_grid=10)
    f64 = ForceField(q, pos, edges, **kw, precision="fp64")
    mix = ForceField(q, pos, edges, **kw, precision="mixed")
    e1, f1 = f64.energy(pos)
    e2, f2 = mix.energy(pos)
    assert abs(e2 - e1) / abs(e1) < 1e-8
    assert rel_rms(f2, f1) < 3e-7


def test_high_accuracy_parameters_match_oracle():
    """The parameters of the bench's high-accuracy reference (the FP64 GPU
    MSM with order 10, cutoff 12 A, one level, h ~ 1.0 A, against which the
    method errors of the headline forms are measured) on a small box: the
    FP64 form against the oracle to 1e-11 (energy) and 1e-10 (forces,
    potentials), so that the reference of those errors is itself pinned."""
    q, pos, edges = systems.water(600, 26.0, 31)
    kw = dict(cutoff=12.0, order=10, levels=1, top_grid=27)
    o = Oracle(q, edges, cutoff=12.0, nu=10, levels=1, top_grid=27)
    ff = ForceField(q, pos, edges, **kw, precision="fp64")
    assert (ff.cutoff, ff.order, ff.levels, ff.top_grid) == (12.0, 10, 1, (27, 27, 27))
    eo, fo, po = o.energy(pos)
    e, f, phi = ff.energy(pos, potentials=True)
    assert abs(e - eo) / abs(eo) < 1e-11
    assert force_err(f, fo, q, edges) < 1e-10
    assert rel_rms(phi, po) < 1e-10


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_level_weights(precision):
    """Weighted evaluation is linear in each level weight (the oracle's
    definition; the reference only defines unit weights)."""
    d = load("spceN900_L3_M6_a8_nu8")
    p = params(d)
    o = Oracle(d["q"], d["edges"], cutoff=p["cutoff"], nu=p["nu"],
               levels=p["levels"], top_grid=p["top_grid"])
    w = np.array([0.5, 1.5, -0.25, 2.0])
    eo, fo, po = o.energy(d["pos"], weight=w)
    ff = make_ff(d, precision)
    e, f, phi = ff.energy(d["pos"], weights=w, potentials=True)
    te, tf, tp = TOL[precision]
    assert abs(e - eo) / abs(eo) < te * 10
    assert force_err(f, fo, d["q"], d["edges"]) < tf
    assert rel_rms(phi, po) < tp


@pytest.mark.parametrize("variant", [("MSMPB_PAIR", "thread"), ("MSMPB_ANTERP", "gather"),
                                     ("MSMPB_STENCIL", "full")])
@pytest.mark.parametrize("case", ["spceN900_L3_M6_a8_nu8", "changaN512_L2_M8_a0.25_nu6",
                                  "CsClN16_auto"])
def test_alternative_kernels(case, variant, monkeypatch):
    """The fallback kernels, forced everywhere (one thread per atom for the
    pair sum, the form for geometries the cluster form does not take; the
    slab-staged gather for anterpolation, the form for grids smaller than the
    order; the unfolded level stencil, the form for stencils without mirror
    symmetry) give the same results as the default ones."""
    monkeypatch.setenv(*variant)
    d = load(case)
    for precision in ("fp64", "mixed"):
        ff = make_ff(d, precision)
        e, f = ff.energy(d["pos"])
        te, tf, _ = TOL[precision]
        assert abs(e - float(d["energy"])) / abs(float(d["energy"])) < te
        assert force_err(f, d["force"], d["q"], d["edges"]) < tf
        ff.close()


@pytest.mark.parametrize("variant", ["clusters", "thread"])
def test_box_smaller_than_cutoff(variant, monkeypatch):
    """Boxes with a lattice vector shorter than the cutoff: an atom's own
    periodic images lie within a0. The reference sums them once, in the
    constant coeff1 (code/forcefield0.c:612-636), and its pair list never
    pairs an atom with itself (code/forcefield1.c:240-321), so every pair
    kernel must skip the atom at all its images."""
    if variant != "clusters":
        monkeypatch.setenv("MSMPB_PAIR", variant)
    rng = np.random.default_rng(21)
    n = 24
    q = rng.choice([-1.0, 1.0], n)
    q -= q.mean()
    for edges in (np.diag([6.0, 7.0, 6.5]), np.array([[6.0, 1.0, 0.5], [0.0, 6.5, 1.2],
                                                      [0.0, 0.0, 7.0]])):
        pos = rng.uniform(0, 1, (n, 3)) @ edges.T
        o = Oracle(q, edges, cutoff=8.0, nu=4, levels=1, top_grid=[8, 8, 8])
        eo, fo, po = o.energy(pos)
        for precision in ("fp64", "mixed"):
            ff = ForceField(q, pos, edges, cutoff=8.0, order=4, levels=1, top_grid=8,
                            precision=precision)
            e, f, phi = ff.energy(pos, potentials=True)
            te, tf, tp = TOL[precision]
            assert abs(e - eo) / abs(eo) < te, (precision, e, eo)
            assert force_err(f, fo, q, edges) < tf
            assert rel_rms(phi, po) < tp
            ff.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_large_top_grid(precision):
    """A one-level plan whose top grid (96 x 90 x 98) is too large for the
    plane-staged FFT: the five line passes of the large-grid path, against
    the oracle's FFT."""
    q, pos, edges = systems.water(400, 24.0, 11)
    o = Oracle(q, edges, cutoff=8.0, nu=6, levels=1, top_grid=[96, 90, 98])
    eo, fo, po = o.energy(pos)
    ff = ForceField(q, pos, edges, cutoff=8.0, order=6, levels=1, top_grid=(96, 90, 98),
                    precision=precision)
    e, f, phi = ff.energy(pos, potentials=True)
    te, tf, tp = TOL[precision]
    assert abs(e - eo) / abs(eo) < te
    assert force_err(f, fo, q, edges) < tf
    assert rel_rms(phi, po) < tp
    ff.close()


TINY = [  # (N, order, top grid, levels, cutoff)
    (1, 6, 6, 1, 4.5), (2, 4, 4, 1, 4.0), (3, 6, 6, 1, 4.5), (8, 8, 8, 1, 5.0), (33, 10, 8, 1, 5.0),
    (8, 10, 4, 1, 4.0), (33, 6, 4, 2, 4.0), (33, 4, 4, 3, 3.0), (16, 8, 6, 2, 4.5),
]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("n,nu,m,levels,a0", TINY)
def test_tiny_systems(n, nu, m, levels, a0, precision):
    """Few atoms (one ion, ragged clusters of 2..33), every order, grids smaller than
    the B-spline order (charges wrap several times), up to three levels,
    atoms given outside the primary box (the reference wraps fractional
    coordinates, code/forcefield1.c:349-352)."""
    rng = np.random.default_rng(100 * n + nu)
    edges = np.diag([10.0, 11.0, 9.5])
    q = rng.uniform(-1, 1, n)
    if n > 1:
        q -= q.mean()
    pos = rng.uniform(0, 1, (n, 3)) @ edges.T
    pos[::2] += edges @ rng.integers(-2, 3, (3,))  # some atoms a few boxes away
    o = Oracle(q, edges, cutoff=a0, nu=nu, levels=levels, top_grid=[m, m, m])
    eo, fo, po = o.energy(pos)
    ff = ForceField(q, pos, edges, cutoff=a0, order=nu, levels=levels, top_grid=m,
                    precision=precision)
    e, f, phi = ff.energy(pos, potentials=True)
    te, tf, tp = TOL[precision]
    assert abs(e - eo) <= te * max(abs(eo), 1e-3)
    assert force_err(f, fo, q, edges) < tf
    assert rel_rms(phi, po) < tp
    ff.close()


def test_non_finite_input_is_reported():
    """A NaN position or an infinite charge is caught on the device (the
    atom is binned at a safe cell and a check flag set): the call reports
    MSMPB_ERR_DEVICE_CHECK instead of reading out of bounds, and the next
    valid call is clean."""
    from msmpb_b200 import _lib as L
    from msmpb_b200.forcefield import MSMError
    d = load("spceN300_M24_a9_nu4")
    ff = make_ff(d, "mixed")
    pos = d["pos"].copy()
    pos[5, 1] = np.nan
    with pytest.raises(MSMError) as ex:
        ff.energy(pos)
    assert ex.value.code == L.ERR_DEVICE_CHECK
    q = d["q"].copy()
    q[7] = np.inf
    with pytest.raises(MSMError) as ex:
        ff.energy(d["pos"], charges=q)
    assert ex.value.code == L.ERR_DEVICE_CHECK
    e, f = ff.energy(d["pos"], charges=d["q"])
    assert abs(e - float(d["energy"])) / abs(float(d["energy"])) < TOL["mixed"][0]
    ff.close()


def test_repeat_and_charge_update():
    """Repeated calls give identical results; charge edits between calls
    are seen (FF_new keeps the caller's pointer, code/forcefield0.c:172)."""
    d = load("spceN600_M20_a8_nu6")
    ff = make_ff(d, "mixed")
    e1, f1 = ff.energy(d["pos"])
    e2, f2 = ff.energy(d["pos"])
    assert e1 == e2 and np.array_equal(f1, f2)
    q2 = d["q"] * 0.5
    e3, _ = ff.energy(d["pos"], charges=q2)
    assert abs(e3 - 0.25 * e1) / abs(e1) < 1e-5


def test_rebuild_box_change():
    """FF_rebuild with a new box keeps the parameters and matches a fresh
    build with those parameters."""
    d = load("spceN600_M20_a8_nu6")
    p = params(d)
    ff = make_ff(d, "fp64")
    edges2 = d["edges"] * 1.03
    pos2 = d["pos"] * 1.03
    ff.rebuild(edges2, pos2)
    e, f = ff.energy(pos2)
    o = Oracle(d["q"], edges2, cutoff=p["cutoff"], nu=p["nu"], levels=1,
               top_grid=p["top_grid"])
    eo, fo, _ = o.energy(pos2)
    assert abs(e - eo) / abs(eo) < 1e-10
    assert force_err(f, fo, d["q"], edges2) < 1e-10


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_triclinic_box_vs_oracle(precision):
    """A skewed box: every neighbour column is swept (no gap pruning) and
    the column images carry the off-diagonal edge components."""
    q, pos, _ = systems.water(300, 24.0, 5)
    edges = np.array([[24.0, 0.0, 0.0], [4.0, 24.0, 0.0], [3.0, -2.5, 24.0]])
    o = Oracle(q, edges, cutoff=9.0, nu=6, levels=2, top_grid=6)
    eo, fo, po = o.energy(pos)
    ff = ForceField(q, pos, edges, cutoff=9.0, order=6, levels=2, top_grid=6,
                    precision=precision)
    e, f, phi = ff.energy(pos, potentials=True)
    te, tf, tp = TOL[precision]
    assert abs(e - eo) / abs(eo) < te
    assert force_err(f, fo, q, edges) < tf
    assert rel_rms(phi, po) < tp


def test_error_estimate_after_evaluation():
    """FF_energy refreshes errEst (code/forcefield1.c:233); the library takes
    sum q^2 from its device reduction, so it agrees with the host formula to
    rounding."""
    q, pos, edges, kw = _oracle_case("water300")
    o = Oracle(q, edges, cutoff=kw.get("cutoff", -1), nu=kw.get("order", -1))
    ff = ForceField(q, pos, edges, **kw, precision="mixed")
    ff.energy(pos)
    assert ff.err_est() == pytest.approx(o.err_est(), rel=1e-12)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_rebuild_device_box_change(precision):
    """FF_rebuild_device (level stencils computed on the GPU) against the FP64
    FF_rebuild of the same box on the host, for a larger, a smaller and a
    triclinic box (where the stencils lose their mirror symmetry), and against
    the oracle where the new box keeps the build-time nLim (a rebuild keeps
    every build-time choice, code/forcefield0.c:598-680)."""
    q, pos, edges = systems.water(8000, 62.0, 11)
    kw = dict(cutoff=9.0, order=6, levels=3, top_grid=6)
    te, tf, tp = TOL[precision]
    ff = ForceField(q, pos, edges, **kw, precision=precision)
    ff.set_timing(False)
    ff.energy(pos)  # a captured graph exists before the box changes
    tri = np.array([[62.0, 0.0, 0.0], [5.0, 62.0, 0.0], [-3.0, 2.0, 62.0]])
    for e2, p2 in ((edges * 1.03, pos * 1.03), (edges * 0.98, pos * 0.98), (tri, pos)):
        ff.rebuild_device(e2)
        e, f, phi = ff.energy(p2, potentials=True)
        host = ForceField(q, pos, edges, **kw, precision="fp64")
        host.rebuild(e2, p2)
        eh, fh, ph = host.energy(p2, potentials=True)
        host.close()
        scale = 1e-1 if precision == "fp64" else 1.0  # FP64: 1e-12 / 1e-11
        assert abs(e - eh) / abs(eh) < te * scale
        assert force_err(f, fh, q, e2) < tf * scale
        assert rel_rms(phi, ph) < tp * scale
    # the larger box keeps nLim: the oracle built there is the same operator
    e2, p2 = edges * 1.03, pos * 1.03
    ff.rebuild_device(e2)
    e, f, phi = ff.energy(p2, potentials=True)
    o = Oracle(q, e2, cutoff=9.0, nu=6, levels=3, top_grid=6)
    assert o.nlim == ff.nlim
    eo, fo, po = o.energy(p2)
    assert abs(e - eo) / abs(eo) < te
    assert force_err(f, fo, q, e2) < tf
    assert rel_rms(phi, po) < tp
    ff.close()
