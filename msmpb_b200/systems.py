"""Seeded synthetic periodic systems with the shapes of the benchmark
workloads (all lengths in Angstrom, charges in elementary charges).

* ``water``: rigid 3-site molecules (O q=-0.8476, two H q=+0.4238, O-H 1.0,
  H-O-H 109.47 deg), molecule centres uniform in a cubic box, uniformly random
  orientations (QR of a Gaussian matrix). Atom order O, H, H per molecule,
  as in the reference's SPC/E fixtures.
* ``rock_salt``: NaCl conventional cells (Na on fcc sites, Cl shifted by
  a/2 along x) with Gaussian displacements.
* ``ions``: charge-neutral +-1 ions at number density rho with a minimum
  separation, from a randomly occupied jittered lattice relaxed by
  overlap-rejecting random moves.

Each returns ``(charges[N], positions[N,3], edges[3,3])`` with the box
vectors as the columns of ``edges``.
"""
import numpy as np

Q_O, Q_H = -0.8476, 0.4238
OH_BOND = 1.0
HOH_ANGLE_DEG = 109.47
WATER_DENSITY_PER_NM3 = 33.4


def water_edge(n_molecules, density_per_nm3=WATER_DENSITY_PER_NM3):
    return (n_molecules / density_per_nm3) ** (1.0 / 3.0) * 10.0


def water(n_molecules, edge, seed):
    rng = np.random.default_rng(seed)
    th = np.deg2rad(HOH_ANGLE_DEG)
    local = np.array([[0.0, 0.0, 0.0],
                      [OH_BOND, 0.0, 0.0],
                      [OH_BOND * np.cos(th), OH_BOND * np.sin(th), 0.0]])
    centres = rng.uniform(0.0, edge, (n_molecules, 3))
    g = rng.normal(size=(n_molecules, 3, 3))
    qm, r = np.linalg.qr(g)
    qm = qm * np.sign(np.einsum("nii->ni", r))[:, None, :]
    pos = centres[:, None, :] + np.einsum("nij,kj->nki", qm, local)
    q = np.tile([Q_O, Q_H, Q_H], n_molecules)
    return q, pos.reshape(-1, 3), np.eye(3) * edge


def rock_salt(cells, a, sigma, seed):
    rng = np.random.default_rng(seed)
    base = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    idx = np.array([[i, j, k] for i in range(cells) for j in range(cells)
                    for k in range(cells)], dtype=float)
    na = (idx[:, None, :] + base[None]).reshape(-1, 3) * a
    cl = na + np.array([0.5, 0.0, 0.0]) * a
    pos = np.vstack([na, cl])
    pos = pos + rng.normal(0.0, sigma, pos.shape)
    q = np.concatenate([np.ones(len(na)), -np.ones(len(cl))])
    return q, pos, np.eye(3) * (cells * a)


def ions(n, density, min_sep, seed, sweeps=6):
    """Charge-neutral +-1 ions at uniform random positions with a minimum
    separation, cubic periodic box at `density` atoms per cubic Angstrom.

    Random sequential addition jams near a packing fraction of 0.38, and
    0.1 / A^3 at 2 A is 0.42, so the ions start on randomly chosen sites of an
    fcc lattice whose nearest-neighbour distance is at least min_sep and are
    then randomised by hard-sphere Monte Carlo sweeps: every ion proposes a
    uniform displacement at once; proposals closer than min_sep to another
    ion are undone (both ions of a pair, repeated until no pair is left,
    which always ends because the undone positions are pairwise valid).
    """
    from scipy.spatial import cKDTree

    if n % 2:
        raise ValueError("charge-neutral +-1 ions need an even count")
    rng = np.random.default_rng(seed)
    edge = (n / density) ** (1.0 / 3.0)
    m = int(np.floor(edge / (min_sep * np.sqrt(2.0))))
    if m < 1 or 4 * m ** 3 < n:
        raise ValueError("density too high for the minimum separation")
    a = edge / m
    g = np.stack(np.meshgrid(*[np.arange(m)] * 3, indexing="ij"), -1).reshape(-1, 1, 3)
    basis = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    sites = ((g + basis).reshape(-1, 3) + 0.25) * a
    pos = sites[rng.choice(len(sites), n, replace=False)]
    step = 0.5 * density ** (-1.0 / 3.0)

    def wrap(x):
        x = np.mod(x, edge)
        return np.where(x >= edge, x - edge, x)

    for _ in range(sweeps):
        new = wrap(pos + rng.uniform(-step, step, pos.shape))
        tree = cKDTree(new, boxsize=edge)
        pairs = tree.query_pairs(min_sep, output_type="ndarray")
        moved = np.ones(n, bool)
        undo = np.unique(pairs.ravel())
        while len(undo):
            moved[undo] = False
            new[undo] = pos[undo]
            # undone ions against the proposals still kept (the tree holds the
            # proposals; undone positions are pairwise valid)
            hits = tree.query_ball_point(pos[undo], min_sep, return_sorted=False)
            cand = np.unique(np.fromiter((j for h in hits for j in h), dtype=np.int64))
            cand = cand[moved[cand]] if len(cand) else cand
            if len(cand) == 0:
                break
            near = cKDTree(pos[undo], boxsize=edge).query(new[cand], distance_upper_bound=min_sep)[0]
            undo = cand[near < min_sep]
        pos = new
    q = np.where(rng.permutation(n) < n // 2, 1.0, -1.0)
    return q, pos, np.eye(3) * edge


def _ion_system(args):
    i, n, seed, density, min_sep = args
    q, p, e = ions(n, density, min_sep, seed * 100003 + i)
    return q, p, e, dict(order=(4, 6, 8)[i % 3], cutoff=8.0)


def ion_batch(count=256, seed=5, n_min=500, n_max=20000, density=0.1, min_sep=2.0,
              workers=1):
    """Independent ion boxes of uneven size: N uniform in [n_min, n_max]
    (even), B-spline order cycled over 4, 6, 8, cutoff 8 A, grid and levels
    automatic. Returns a list of (charges, positions, edges, params).
    workers > 1 generates in a process pool started with spawn (safe after
    CUDA is initialised)."""
    rng = np.random.default_rng(seed)
    ns = 2 * rng.integers(n_min // 2, n_max // 2 + 1, count)
    jobs = [(i, int(n), seed, density, min_sep) for i, n in enumerate(ns)]
    if workers > 1:
        import concurrent.futures as cf
        import multiprocessing as mp
        with cf.ProcessPoolExecutor(workers, mp_context=mp.get_context("spawn")) as ex:
            return list(ex.map(_ion_system, jobs, chunksize=4))
    return [_ion_system(j) for j in jobs]


# The benchmark workloads (sizes and parameters of the published configs)
def config(name):
    """Return (charges, positions, edges, params) for a named workload."""
    if name == "water300":
        q, p, e = water(100, 14.4, 0)
        return q, p, e, dict(order=6, cutoff=8.0)
    if name == "rocksalt4096":
        q, p, e = rock_salt(8, 5.64, 0.1, 1)
        return q, p, e, dict(order=8, cutoff=10.0, top_grid=32)
    if name == "water1M":
        n = 333333
        q, p, e = water(n, water_edge(n), 2)
        return q, p, e, dict(order=6, cutoff=9.0, levels=5, top_grid=9)
    if name == "water3000":
        q, p, e = water(1000, water_edge(1000), 3)
        return q, p, e, dict(order=6, cutoff=9.0)
    raise KeyError(name)
