"""msmpb_level_stencil_noalloc (the level stencil with its scratch in a fixed
array compiled into the library, for callers that cannot let a library
allocate device memory) against the same level stencil inside the existing
evaluation entry point.

With level weights (0, w, 0, 0) FF_energy_potentials returns only the
level-1 stencil term: U = 1/2 q1 . e1 with e1 = w * (k1 conv q1), and
phi_i = interpolation of e1 at atom i. The test feeds the oracle's level-1
charge grid q1 and the library's own level-1 stencil k1 to the new entry
point, then rebuilds U and phi from its e1 with the oracle's transfers.
Tolerances are the FP64 parity ones: 1e-11 (energy), 1e-10 (potentials).
This file is collected last so that it also runs after every other test.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from golden_cases import rel_rms
from msmpb_b200 import _lib, systems
from msmpb_b200.forcefield import ForceField
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

TOL_ENERGY, TOL_PHI = 1e-11, 1e-10


def _entry():
    f = _lib.load().msmpb_level_stencil_noalloc
    f.restype = C.c_int
    f.argtypes = [C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_void_p,
                  C.c_void_p, C.c_double, C.c_void_p, C.c_void_p]
    return f


def _call(f, M, S, q_d, k_d, w, e_d):
    stream = torch.cuda.current_stream().cuda_stream
    return f((C.c_int * 3)(*M), (C.c_int * 3)(*S), C.c_void_p(q_d.data_ptr()),
             C.c_void_p(k_d.data_ptr()), w, C.c_void_p(e_d.data_ptr()),
             C.c_void_p(stream) if stream else None)


def test_noalloc_stencil_matches_energy_entry_point():
    q, pos, edges = systems.water(8000, 62.0, 11)
    ff = ForceField(q, pos, edges, cutoff=9.0, order=6, levels=3, top_grid=6,
                    precision="fp64")
    o = Oracle(q, edges, cutoff=9.0, nu=6, levels=3, top_grid=6)
    k1 = ff.khat(1)
    M = o.grid_dims(1)
    # a truncated stencil on a small grid: the tap-plane split (partial sums
    # in the scratch array) is in use
    assert k1.shape == (13, 13, 13) and M == (24, 24, 24)
    dev = torch.device("cuda:0")
    k_d = torch.from_numpy(k1).to(dev)
    f = _entry()

    cases = [(1.0, 1.0), (2.0, -0.75)]  # (charge scale, level-1 weight)
    grids, outs = [], []
    for scale, w in cases:
        q1 = o.anterpolate(pos, q=q * scale)
        grids.append(q1)
        outs.append((torch.from_numpy(q1).to(dev),
                     torch.full(M, 0.0, dtype=torch.float64, device=dev)))
    # two calls in a row, the second on the scratch the first left behind
    for (scale, w), (q_d, e_d) in zip(cases, outs):
        assert _call(f, M, k1.shape, q_d, k_d, w, e_d) == _lib.OK
    torch.cuda.synchronize()

    for (scale, w), q1, (_, e_d) in zip(cases, grids, outs):
        e1 = e_d.cpu().numpy()
        u_ref, f_ref, phi_ref = ff.energy(pos, weights=[0.0, w, 0.0, 0.0],
                                          potentials=True, charges=q * scale)
        u = 0.5 * float((q1 * e1).sum())
        efield, phi = o.interpolate(pos, e1)
        assert abs(u - u_ref) / abs(u_ref) < TOL_ENERGY
        assert rel_rms(phi, phi_ref) < TOL_PHI
        assert rel_rms((q * scale)[:, None] * efield, f_ref) < TOL_PHI
        # and the oracle's own level stencil
        assert rel_rms(e1, w * o.stencil_add(1, q1, np.zeros_like(q1))) < TOL_PHI
    ff.close()


def _periodic_stencil(q, k):
    """sum_d k[d] q[(x + d - S//2) mod M] by FFT (circular cross-correlation)."""
    M, S = q.shape, k.shape
    K = np.zeros(M)
    for d0 in range(S[0]):
        for d1 in range(S[1]):
            for d2 in range(S[2]):
                K[(d0 - S[0] // 2) % M[0], (d1 - S[1] // 2) % M[1],
                  (d2 - S[2] // 2) % M[2]] = k[d0, d1, d2]
    return np.real(np.fft.ifftn(np.fft.fftn(q) * np.conj(np.fft.fftn(K))))


# (grid, stencil): tap planes split over fewer CTAs than the default because
# the partial sums would not fit beside the padded grid (64^3: 9 chunks cut to
# 5), no room for partial sums at all (80^3: one chunk), and a stencil wider
# than the templated sweeps (z width 35: the one-output-per-thread kernel)
@pytest.mark.parametrize("M,S", [((64, 64, 64), (25, 25, 25)), ((80, 80, 80), (25, 25, 25)),
                                 ((10, 12, 40), (3, 5, 35))])
def test_noalloc_stencil_scratch_limits_and_wide_stencil(M, S):
    rng = np.random.default_rng(sum(M) + sum(S))
    q = rng.standard_normal(M)
    k = rng.standard_normal(S)
    e0 = rng.standard_normal(M)
    dev = torch.device("cuda:0")
    q_d, k_d = torch.from_numpy(q).to(dev), torch.from_numpy(k).to(dev)
    e_d = torch.from_numpy(e0.copy()).to(dev)
    f = _entry()
    w = 0.625
    assert _call(f, M, S, q_d, k_d, w, e_d) == _lib.OK
    torch.cuda.synchronize()
    ref = w * _periodic_stencil(q, k)
    assert rel_rms(e_d.cpu().numpy() - e0, ref) < 1e-12


def test_noalloc_stencil_rejects_what_does_not_fit():
    f = _entry()
    dev = torch.device("cuda:0")
    M, S = (100, 100, 100), (25, 25, 25)  # padded grid > 16 MiB
    q_d = torch.zeros(M, dtype=torch.float64, device=dev)
    e_d = torch.full(M, 3.0, dtype=torch.float64, device=dev)
    k_d = torch.zeros(S, dtype=torch.float64, device=dev)
    assert _call(f, M, S, q_d, k_d, 1.0, e_d) == _lib.ERR_UNSUPPORTED
    assert _call(f, (24, 24, 24), (25, 25, 25), q_d, k_d, 1.0, e_d) == _lib.ERR_ARGUMENT
    torch.cuda.synchronize()
    assert bool((e_d == 3.0).all())  # nothing was launched
