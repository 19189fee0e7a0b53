"""In-process Python binding of the smooth-PME comparator (libpme.so).

Mirrors the reference's PME C API (code/pme.h: ``FF_new(N, q, edges)`` ->
``FF_set_*`` -> ``FF_build(ff, pos)`` -> ``FF_energy``) on the GPU, for
MSM-versus-PME cost and error comparisons on identical inputs.
"""
import ctypes as C

import numpy as np

from . import _lib as L
from .forcefield import MSMError, _f64, _ptr


class PMEError(MSMError):
    pass


class PME:
    """One periodic system evaluated with smooth PME on the GPU.

    charges: (N,) ; positions: (N, 3) ; edges: 3x3 with the box vectors as
    columns. ``cutoff`` (8 A), ``order`` (6), ``tol_dir`` (1e-5) and ``grid``
    default to the reference's choices (FF_build, code/pme0.c:192-260).
    precision: "mixed" (FP32 direct sum and grid transfers, FP64 FFT and
    sums) or "fp64".
    """

    def __init__(self, charges, positions, edges, cutoff=None, order=None, grid=None,
                 tol_dir=None, precision="mixed", device=0):
        self._lib = L.load_pme()
        lib = self._lib
        self.q = _f64(charges).copy()
        self.N = int(self.q.shape[0])
        self.edges = _f64(np.asarray(edges, dtype=np.float64).reshape(3, 3)).copy()
        pos = _f64(positions).reshape(self.N, 3)
        self.ff = lib.FF_new(self.N, _ptr(self.q), _ptr(self.edges))
        lib.FF_set_precision(self.ff, L.PRECISION_FP64 if precision == "fp64"
                             else L.PRECISION_MIXED)
        lib.FF_set_device(self.ff, int(device))
        if cutoff is not None:
            lib.FF_set_cutoff(self.ff, float(cutoff))
        if order is not None:
            lib.FF_set_orderAcc(self.ff, int(order))
        if grid is not None:
            self._g = np.ascontiguousarray(np.broadcast_to(np.asarray(grid), (3,)),
                                           dtype=np.int32)
            lib.FF_set_topGridDim(self.ff, self._g.ctypes.data_as(C.POINTER(C.c_int)))
        if tol_dir is not None:
            lib.FF_set_tolDir(self.ff, float(tol_dir))
        lib.FF_build(self.ff, _ptr(pos))
        err = lib.FF_last_error(self.ff)
        if err not in (L.OK, L.ERR_NODEVICE):
            raise PMEError(err, "FF_build")

    def _s(self):
        return self.ff.contents

    @property
    def cutoff(self):
        return self._s().cutoff

    @property
    def order(self):
        return self._s().orderAcc

    @property
    def grid(self):
        return tuple(self._s().topGridDim)

    @property
    def tol_dir(self):
        return self._s().tolDir

    @property
    def beta(self):
        return self._s().beta

    def coeffs(self):
        s = self._s()
        return s.coeff1, s.coeff2

    def khat(self):
        g = self.grid
        return np.ctypeslib.as_array(self._s().khat, (g[0] * g[1] * g[2],)).copy().reshape(g)

    def err_est(self):
        return self._lib.FF_get_errEst(self.ff, self.N, _ptr(self.q))

    def energy(self, positions, weights=None, potentials=False, charges=None):
        """Energy and forces (and per-atom potentials) through the host C ABI."""
        if charges is not None:
            self.q[:] = _f64(charges)
        pos = _f64(positions).reshape(self.N, 3)
        f = np.zeros((self.N, 3))
        phi = np.zeros(self.N) if potentials else None
        w = None if weights is None else _f64(weights)
        e = self._lib.FF_energy_potentials(self.ff, _ptr(f), _ptr(pos),
                                           _ptr(w) if w is not None else None,
                                           _ptr(phi) if phi is not None else None)
        err = self._lib.FF_last_error(self.ff)
        if err != L.OK:
            raise PMEError(err, "FF_energy")
        return (e, f, phi) if potentials else (e, f)

    def energy_device(self, pos_ptr, q_ptr, force_ptr=0, phi_ptr=0, energy_ptr=0, stream=0,
                      weights=None):
        """Asynchronous evaluation on device pointers (ints) on a CUDA stream."""
        w = None if weights is None else _f64(weights)
        st = self._lib.FF_energy_device(
            self.ff, C.c_void_p(pos_ptr), C.c_void_p(q_ptr), _ptr(w) if w is not None else None,
            C.c_void_p(force_ptr or None), C.c_void_p(phi_ptr or None),
            C.c_void_p(energy_ptr or None), C.c_void_p(stream or None))
        if st != L.OK:
            raise PMEError(st, "FF_energy_device")

    def rebuild(self, edges, positions=None):
        self.edges = _f64(np.asarray(edges).reshape(3, 3)).copy()
        pos = np.zeros((self.N, 3)) if positions is None else _f64(positions)
        self._lib.FF_rebuild(self.ff, _ptr(self.edges), _ptr(pos))
        err = self._lib.FF_last_error(self.ff)
        if err not in (L.OK, L.ERR_NODEVICE):
            raise PMEError(err, "FF_rebuild")

    def set_timing(self, enabled):
        self._lib.FF_set_timing(self.ff, 1 if enabled else 0)

    def phase_times(self):
        ms = (C.c_double * 16)()
        n = self._lib.FF_phase_times(self.ff, ms, 16)
        names = ["bin", "pair", "anterpolation", "restriction", "stencil", "top",
                 "prolongation", "interpolation", "combine", "total"]
        return {names[k]: ms[k] for k in range(min(n, len(names)))}

    def kernel_launches(self):
        return self._lib.FF_kernel_launches(self.ff)

    def sync(self):
        st = self._lib.FF_sync(self.ff)
        if st != L.OK:
            raise PMEError(st, "FF_sync")

    def close(self):
        if getattr(self, "ff", None):
            self._lib.FF_delete(self.ff)
            self.ff = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
