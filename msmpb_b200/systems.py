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


def ions(n, density, min_sep, seed, sweeps=8):
    if n % 2:
        raise ValueError("charge-neutral +-1 ions need an even count")
    rng = np.random.default_rng(seed)
    edge = (n / density) ** (1.0 / 3.0)
    m = int(np.ceil(n ** (1.0 / 3.0)))
    while m ** 3 < n:
        m += 1
    d = edge / m
    sites = np.array([[i, j, k] for i in range(m) for j in range(m)
                      for k in range(m)], dtype=float)
    pick = rng.choice(len(sites), n, replace=False)
    pos = (sites[pick] + 0.5) * d
    # overlap-rejecting random displacements on a cell list
    step = 0.5 * max(d - min_sep, 0.05 * d) + 0.25 * d
    nc = max(1, int(edge // min_sep))
    for _ in range(sweeps):
        cell = np.floor(pos / edge * nc).astype(int) % nc
        buckets = {}
        for i, c in enumerate(map(tuple, cell)):
            buckets.setdefault(c, []).append(i)
        for i in rng.permutation(n):
            trial = (pos[i] + rng.uniform(-step, step, 3)) % edge
            c = tuple(np.floor(trial / edge * nc).astype(int) % nc)
            ok = True
            for dx in (-1, 0, 1):
                for dy in (-1, 0, 1):
                    for dz in (-1, 0, 1):
                        key = ((c[0] + dx) % nc, (c[1] + dy) % nc, (c[2] + dz) % nc)
                        for j in buckets.get(key, ()):
                            if j == i:
                                continue
                            r = trial - pos[j]
                            r -= edge * np.round(r / edge)
                            if r @ r < min_sep * min_sep:
                                ok = False
                                break
                        if not ok:
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if ok:
                old = tuple(cell[i])
                buckets[old].remove(i)
                buckets.setdefault(c, []).append(i)
                cell[i] = c
                pos[i] = trial
    q = np.where(rng.permutation(n) < n // 2, 1.0, -1.0)
    return q, pos, np.eye(3) * edge


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
