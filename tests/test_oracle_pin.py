"""Pins the CPU oracle (oracle/msm_oracle.c) before it is trusted as the
checker:

* against the reference's own outputs on its fixtures (tests/golden/*.npz,
  made by the patched reference build, oracle/build_ref.py);
* against published numbers: the Box44 energy of results/TableII.json and
  the force errors of results/Figure1.txt (computed with the reference
  driver's metric, code/msmpb.c:254-306, against the high-accuracy data/*.acc);
* against the reference library run live, when oracle/_ref has been built
  in this container (skipped elsewhere).
"""
import numpy as np
import pytest

from golden_cases import index, load, names, params, rel_rms
from msmpb_b200 import systems
from oracle.oracle import Oracle, RefFF


def fref(q, edges):
    n = len(q)
    return (q @ q / n) / (abs(np.linalg.det(edges)) / n) ** (2.0 / 3.0)


def oracle_for(d):
    p = params(d)
    return Oracle(d["q"], d["edges"], cutoff=p["cutoff"], nu=p["nu"],
                  levels=p["levels"], top_grid=p["top_grid"])


# water215_L5 (the 5-level hierarchy of the 1M-atom workload) takes the
# oracle about two minutes (the 144^3 grid with a 25^3 stencil); its
# generator (tests/golden/make_golden_l5.py) ran the same comparison, to
# 1e-12 in energy and 1e-11 in force, before writing the fixture, and
# test_oracle_l5_parameters below checks the parameters it derives.
SLOW_ORACLE = ("water215_L5",)


@pytest.mark.parametrize("case", [n for n in names()
                                  if not n.startswith("Box44") and n not in SLOW_ORACLE])
def test_oracle_matches_reference_outputs(case):
    d = load(case)
    o = oracle_for(d)
    assert (o.levels, o.nu, o.top_grid, o.nlim) == (
        int(d["levels"]), int(d["nu"]), tuple(d["top_grid"]), int(d["nlim"]))
    e, f, phi = o.energy(d["pos"])
    ref = float(d["energy"])
    assert abs(e - ref) / abs(ref) < 1e-12
    err = np.sqrt(((f - d["force"]) ** 2).sum() / len(d["q"])) / fref(d["q"], d["edges"])
    assert err < 1e-11
    if "phi" in d:
        assert rel_rms(phi, d["phi"]) < 1e-10
    # the quadratic form: U = 1/2 sum_i q_i phi_i
    assert abs(0.5 * d["q"] @ phi - e) / abs(e) < 1e-12


def test_oracle_l5_parameters():
    """The oracle derives the reference's own level count, top grid and
    stencil half-width for the 5-level fixture, and its stencil widths."""
    d = load("water215_L5")
    o = oracle_for(d)
    assert (o.levels, o.nu, o.top_grid, o.nlim) == (
        int(d["levels"]), int(d["nu"]), tuple(d["top_grid"]), int(d["nlim"]))
    for level, width in ((1, 25), (2, 25), (3, 25), (4, 18)):
        assert o.khat(level).shape == (width,) * 3


def test_oracle_box44_published_energy():
    """results/TableII.json: Box44, L=2, nu=6, M=18 (finest 36), a0=12."""
    d = load("Box44_L2_M18_a12_nu6")
    o = oracle_for(d)
    e, f, _ = o.energy(d["pos"])
    pub = index()["published"]
    assert abs(e - pub["TableII_Box44_L2_M18_utotal"]) / 13831.98 < 1e-12
    pot = float(d["pot_exact"])
    assert abs(abs(e - pot) / abs(pot) - pub["TableII_Box44_L2_M18_poterror"]) < 1e-12
    cs = d["force_checksum"]
    assert abs((f ** 2).sum() - cs[1]) / cs[1] < 1e-11


def _figure1_rows(n):
    rows = index()["published"]["Figure1"]
    return [r for r in rows if int(r[0]) == n]


@pytest.mark.parametrize("row", _figure1_rows(300) + _figure1_rows(600))
def test_oracle_reproduces_figure1(row):
    """results/Figure1.txt: deltaF/Fref of the SPC/E boxes (printed to 4
    significant digits) from the oracle's forces and data/spceN*.acc."""
    n, M, a0, nu, pub = int(row[0]), int(row[1]), float(row[2]), int(row[3]), float(row[4])
    d = load("spceN300_M24_a9_nu4" if n == 300 else "spceN600_M20_a8_nu6")
    o = Oracle(d["q"], d["edges"], cutoff=a0, nu=nu, levels=1, top_grid=M)
    _, f, _ = o.energy(d["pos"])
    exact = -d["acc_exact"] * d["q"][:, None]
    err = np.sqrt(((exact - f) ** 2).sum() / n) / fref(d["q"], d["edges"])
    assert abs(err - pub) / pub < 6e-4, (err, pub)


def test_oracle_potentials_are_energy_gradient():
    """phi_i = dU/dq_i by central differences (exact for quadratic U)."""
    q, pos, edges = systems.water(40, 11.0, 5)
    o = Oracle(q, edges, cutoff=5.0, nu=6, levels=2, top_grid=6)
    _, _, phi = o.energy(pos)
    for i in (0, 7, 61, 119):
        qp = q.copy()
        qp[i] += 1.0
        ep, _, _ = o.energy(pos, q=qp)
        qp[i] -= 2.0
        em, _, _ = o.energy(pos, q=qp)
        assert abs((ep - em) / 2.0 - phi[i]) < 1e-10 * max(1.0, abs(phi[i]))


def test_oracle_forces_are_energy_gradient():
    """F = -dU/dr by central differences on a small system."""
    q, pos, edges = systems.water(30, 10.0, 6)
    o = Oracle(q, edges, cutoff=4.5, nu=6, levels=1, top_grid=12)
    _, f, _ = o.energy(pos)
    h = 1e-5
    for i, k in ((0, 0), (13, 1), (44, 2)):
        p = pos.copy()
        p[i, k] += h
        ep, _, _ = o.energy(p)
        p[i, k] -= 2 * h
        em, _, _ = o.energy(p)
        fd = -(ep - em) / (2 * h)
        assert abs(fd - f[i, k]) < 2e-6 * max(1.0, abs(f[i, k]))


def test_oracle_translation_by_grid_cell_is_exact():
    """Shifting every atom by whole top-level grid spacings leaves the MSM
    energy unchanged up to rounding (every level's grid maps onto itself,
    the pair sum is periodic). A shift by one finest spacing is not a
    symmetry once L > 1: the restriction to the coarser grid changes."""
    q, pos, edges = systems.water(60, 12.0, 8)
    o = Oracle(q, edges, cutoff=5.0, nu=4, levels=2, top_grid=5)
    e0, f0, _ = o.energy(pos)
    e1, f1, _ = o.energy(pos + np.array([12.0 / 5, 0.0, 2 * 12.0 / 5]))
    assert abs(e1 - e0) < 1e-11 * abs(e0)
    assert rel_rms(f1, f0) < 1e-10


needs_ref = pytest.mark.skipif(not RefFF.available(),
                               reason="oracle/_ref not built (no reference here)")


@needs_ref
@pytest.mark.parametrize("seed,levels,nu,M,a0", [
    (1, 1, 4, 10, 5.0), (2, 1, 8, 12, 6.0), (3, 2, 6, 6, 5.0), (4, 3, 6, 4, 4.0),
])
def test_oracle_vs_live_reference(seed, levels, nu, M, a0):
    """Level grids stay at least nu wide: below that the reference's halo
    allocation (code/forcefield1.c:147, nu-1) is smaller than what padding()
    writes (code/forcefield1.c:63, nu) and the reference corrupts its heap."""
    q, pos, edges = systems.water(120, 15.0, seed)
    pos = pos + np.random.default_rng(seed).normal(0, 3.0, pos.shape)  # also outside the box
    r = RefFF(q, pos, edges, cutoff=a0, nu=nu, levels=levels, top_grid=M)
    er, fr = r.energy()
    o = Oracle(q, edges, cutoff=a0, nu=nu, levels=levels, top_grid=M)
    e, f, _ = o.energy(pos)
    assert abs(e - er) / abs(er) < 1e-12
    assert rel_rms(f, fr) < 1e-11


@needs_ref
def test_reference_bugs_are_real():
    """The unpatched reference differs from the patched one at L=1 (energy)
    and at L>=2 (energy and forces): the two index fixes matter."""
    d = load("spceN2250_L2_M16_a9_nu6")
    p = params(d)
    r = RefFF(d["q"], d["pos"], d["edges"], cutoff=p["cutoff"], nu=p["nu"],
              levels=2, top_grid=p["top_grid"], unpatched=True)
    e, f = r.energy()
    assert rel_rms(f, d["force"]) > 1e-3
    d1 = load("spceN300_M30_a11_nu10")
    p1 = params(d1)
    r1 = RefFF(d1["q"], d1["pos"], d1["edges"], cutoff=p1["cutoff"], nu=p1["nu"],
               levels=1, top_grid=p1["top_grid"], unpatched=True)
    e1, f1 = r1.energy()
    assert abs(e1 - float(d1["energy"])) / abs(float(d1["energy"])) > 1e-5
    assert rel_rms(f1, d1["force"]) < 1e-12
