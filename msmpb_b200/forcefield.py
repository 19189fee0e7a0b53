"""In-process Python binding of the MSM force field.

Mirrors the reference's C API call order (``FF_new`` -> ``FF_set_*`` ->
``FF_build`` -> ``FF_energy``; code/forcefield0.c:4-8) and the parameters
that ``runMSM`` in code/msmpb_wrapper.py:48-66 passes to the ``msmpb``
driver (``-L``, ``--a0``, ``--nu``, ``-M``). The reference wrapper runs the
C driver as a subprocess; this class calls the CUDA library directly through
its C ABI.
"""
import ctypes as C

import numpy as np

from . import _lib as L

_dp = C.POINTER(C.c_double)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _ptr(a):
    return a.ctypes.data_as(_dp)


class MSMError(RuntimeError):
    def __init__(self, code, where):
        lib = L.load()
        msg = lib.FF_error_string(code).decode()
        super().__init__("%s: %s (code %d)" % (where, msg, code))
        self.code = code


class ForceField:
    """One periodic system evaluated with B-spline MSM on the GPU.

    charges: (N,) ; positions: (N, 3) ; edges: 3x3 with the box vectors as
    columns (code/forcefield0.c:275). ``cutoff``, ``order``, ``levels``,
    ``top_grid`` and ``est_err`` default to the reference's automatic
    choices (FF_build, code/forcefield0.c:286-348).
    precision: "mixed" (FP32 bulk, FP64 FFT and sums) or "fp64".
    """

    def __init__(self, charges, positions, edges, cutoff=None, order=None,
                 levels=None, top_grid=None, est_err=None, fft=True,
                 margin=0.0, precision="mixed", device=0, charges_buffer=None):
        self._lib = L.load()
        # FF_new keeps this pointer: the library re-reads the charges every
        # evaluation. charges_buffer (a contiguous float64 array, e.g. a
        # pinned one) is used in place instead of a private copy.
        if charges_buffer is not None:
            if charges_buffer.dtype != np.float64 or not charges_buffer.flags.c_contiguous:
                raise ValueError("charges_buffer must be contiguous float64")
            self.q = charges_buffer
        else:
            self.q = _f64(charges).copy()
        self.N = int(self.q.shape[0])
        pos = _f64(positions).reshape(self.N, 3)
        self.edges = _f64(np.asarray(edges, dtype=np.float64).reshape(3, 3)).copy()
        lib = self._lib
        self.ff = lib.FF_new(self.N, _ptr(self.q))
        if not self.ff:
            raise MemoryError("FF_new failed")
        lib.FF_set_precision(self.ff, L.PRECISION_FP64 if precision == "fp64"
                             else L.PRECISION_MIXED)
        lib.FF_set_device(self.ff, int(device))
        if levels is not None:
            lib.FF_set_maxLevel(self.ff, int(levels))
        if top_grid is not None:
            tg = np.ascontiguousarray(np.broadcast_to(np.asarray(top_grid), (3,)),
                                      dtype=np.int32)
            lib.FF_set_topGridDim(self.ff, tg.ctypes.data_as(C.POINTER(C.c_int)))
        if order is not None:
            lib.FF_set_orderAcc(self.ff, int(order))
        if cutoff is not None:
            lib.FF_set_cutoff(self.ff, float(cutoff))
        if est_err is not None:
            lib.FF_set_estErr(self.ff, float(est_err))
        if not fft:
            lib.FF_set_FFT(self.ff, False)
        lib.FF_build(self.ff, self.N, _ptr(pos), _ptr(self.edges), float(margin))
        err = lib.FF_last_error(self.ff)
        if err not in (L.OK, L.ERR_NODEVICE):
            raise MSMError(err, "FF_build")
        self.build_error = err

    # ---- parameters (FF_get_*) ----
    @property
    def struct(self):
        return self.ff.contents

    @property
    def cutoff(self):
        return self._lib.FF_get_cutoff(self.ff)

    @property
    def order(self):
        return self._lib.FF_get_orderAcc(self.ff)

    @property
    def levels(self):
        return self._lib.FF_get_maxLevel(self.ff)

    @property
    def top_grid(self):
        d = (C.c_int * 3)()
        self._lib.FF_get_topGridDim(self.ff, d)
        return tuple(d)

    @property
    def nlim(self):
        return self.struct.nLim

    def err_est(self):
        return self._lib.FF_get_errEst(self.ff)

    def delta_f(self):
        return self._lib.FF_get_deltaF(self.ff)

    def khat(self, level):
        """Level stencil (l < levels) or top-level multiplier (l == levels)."""
        s = self.struct
        if level == self.levels:
            dims = self.top_grid
        else:
            m = np.array(self.top_grid) * 2 ** (self.levels - level)
            dims = tuple(int(min(2 * self.nlim + 1, v)) for v in m)
        n = int(np.prod(dims))
        return np.ctypeslib.as_array(s.khat[level], shape=(n,)).reshape(dims).copy()

    def coeffs(self):
        s = self.struct
        return s.coeff1, s.coeff2

    # ---- evaluation ----
    def energy(self, positions, weights=None, potentials=False, charges=None):
        """Energy, forces (N,3) and optionally potentials (N,) through the
        host-array C ABI (FF_energy / FF_energy_potentials)."""
        if charges is not None:
            self.q[:] = _f64(charges)
        pos = _f64(positions).reshape(self.N, 3)
        f = np.zeros((self.N, 3))
        phi = np.zeros(self.N) if potentials else None
        w = None if weights is None else _f64(weights)
        e = self._lib.FF_energy_potentials(
            self.ff, _ptr(f), _ptr(pos), _ptr(w) if w is not None else None,
            _ptr(phi) if phi is not None else None)
        err = self._lib.FF_last_error(self.ff)
        if err != L.OK:
            raise MSMError(err, "FF_energy")
        return (e, f, phi) if potentials else (e, f)

    def energy_device(self, pos_ptr, q_ptr, force_ptr=0, phi_ptr=0,
                      energy_ptr=0, stream=0, weights=None):
        """Asynchronous evaluation on device pointers (ints, e.g. from
        ``tensor.data_ptr()``) on a CUDA stream handle."""
        w = None if weights is None else _f64(weights)
        st = self._lib.FF_energy_device(
            self.ff, C.c_void_p(pos_ptr), C.c_void_p(q_ptr),
            _ptr(w) if w is not None else None, C.c_void_p(force_ptr or None),
            C.c_void_p(phi_ptr or None), C.c_void_p(energy_ptr or None),
            C.c_void_p(stream or None))
        if st != L.OK:
            raise MSMError(st, "FF_energy_device")

    def adjoint_device(self, pos_ptr, q_ptr, fbar_ptr, ubar=0.0, dq_ptr=0, dr_ptr=0,
                       reuse=False, stream=0, weights=None):
        """FF_adjoint_device: charge and position gradients of
        ubar U + sum Fbar . F (device pointers as ints; outputs in input
        order). reuse: the last evaluation had these inputs and weights."""
        w = None if weights is None else _f64(weights)
        st = self._lib.FF_adjoint_device(
            self.ff, C.c_void_p(pos_ptr), C.c_void_p(q_ptr), _ptr(w) if w is not None else None,
            C.c_void_p(fbar_ptr), float(ubar), C.c_void_p(dq_ptr) if dq_ptr else None,
            C.c_void_p(dr_ptr) if dr_ptr else None, 1 if reuse else 0,
            C.c_void_p(stream) if stream else None)
        if st != L.OK:
            raise MSMError(st, "FF_adjoint_device")

    def evaluation_count(self):
        return int(self._lib.FF_evaluation_count(self.ff))

    def sync(self):
        st = self._lib.FF_sync(self.ff)
        if st != L.OK:
            raise MSMError(st, "FF_sync")

    def phase_times(self):
        ms = (C.c_double * 16)()
        n = self._lib.FF_phase_times(self.ff, ms, 16)
        names = ["bin", "pair", "anterpolation", "restriction", "stencil",
                 "top", "prolongation", "interpolation", "combine", "total"]
        return {names[k]: ms[k] for k in range(min(n, len(names)))}

    def kernel_launches(self):
        return self._lib.FF_kernel_launches(self.ff)

    def stencil_times(self):
        """Per-level stencil kernel ms of the last timed evaluation."""
        ms = (C.c_double * 16)()
        n = self._lib.FF_stencil_times(self.ff, ms, 16)
        return [ms[k] for k in range(n)]

    def set_timing(self, enabled):
        """True: eager launches with per-phase events (fills time_*);
        False: replay of the captured CUDA graph."""
        self._lib.FF_set_timing(self.ff, 1 if enabled else 0)

    def set_precision(self, precision):
        self._lib.FF_set_precision(self.ff, L.PRECISION_FP64 if precision == "fp64"
                                   else L.PRECISION_MIXED)

    def rebuild(self, edges, positions=None, margin=0.0):
        self.edges = _f64(np.asarray(edges).reshape(3, 3)).copy()
        pos = np.zeros((self.N, 3)) if positions is None else _f64(positions)
        self._lib.FF_rebuild(self.ff, _ptr(self.edges), _ptr(pos), float(margin))
        err = self._lib.FF_last_error(self.ff)
        if err not in (L.OK, L.ERR_NODEVICE):
            raise MSMError(err, "FF_rebuild")

    def rebuild_device(self, edges, stream=0):
        """FF_rebuild_device: new box, level stencils computed on the GPU in
        the order of `stream` (a CUDA stream handle; 0 = legacy default)."""
        self.edges = _f64(np.asarray(edges).reshape(3, 3)).copy()
        st = self._lib.FF_rebuild_device(self.ff, _ptr(self.edges),
                                         C.c_void_p(stream) if stream else None)
        if st != L.OK:
            raise MSMError(st, "FF_rebuild_device")

    def close(self):
        if getattr(self, "ff", None):
            self._lib.FF_delete(self.ff)
            self.ff = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many built ForceField handles evaluated by one CUDA graph launch
    (FF_batch_new / FF_batch_energy_device). ``branches``: parallel branches
    of the graph, -K = the members' launches merged into one launch per
    kernel on each of K branches (``Batch.MERGED`` = -1: one branch), 0 = the
    form tuned on the first evaluation."""

    MERGED = -1  # FF_BATCH_MERGED

    def __init__(self, members, branches=0):
        self._lib = L.load()
        self.members = list(members)
        n = len(self.members)
        arr = (C.POINTER(L.FFStruct) * n)(*[m.ff for m in self.members])
        st = C.c_int(0)
        self.b = self._lib.FF_batch_new(arr, n, int(branches), C.byref(st))
        if not self.b:
            raise MSMError(st.value, "FF_batch_new")

    def energy_device(self, pos_ptrs, q_ptrs, force_ptrs=None, phi_ptrs=None,
                      energy_ptr=0, stream=0, weights=None):
        """Device pointers (ints) per member, in member order; energy_ptr:
        one device buffer of len(members) doubles."""
        n = len(self.members)
        vp = lambda ps: (C.c_void_p * n)(*[p or None for p in ps]) if ps is not None else None
        keep = []
        w = None
        if weights is not None:
            w = (_dp * n)()
            for i, wi in enumerate(weights):
                if wi is not None:
                    a = _f64(wi)
                    keep.append(a)
                    w[i] = _ptr(a)
        st = self._lib.FF_batch_energy_device(
            self.b, vp(pos_ptrs), vp(q_ptrs), w, vp(force_ptrs), vp(phi_ptrs),
            C.c_void_p(energy_ptr or None), C.c_void_p(stream or None))
        if st != L.OK:
            raise MSMError(st, "FF_batch_energy_device")

    def branches(self):
        return self._lib.FF_batch_branches(self.b)

    def kernel_launches(self):
        return self._lib.FF_batch_kernel_launches(self.b)

    def last_error(self):
        return self._lib.FF_batch_last_error(self.b)

    def close(self):
        if getattr(self, "b", None):
            self._lib.FF_batch_delete(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
