"""ctypes access to the CPU oracle and to the reference build (test
infrastructure only).

* ``Oracle``: the project's FP64 C restatement (oracle/msm_oracle.c), built
  into oracle/libmsm_oracle.so by ``build_oracle()``.
* ``RefFF``: the reference library itself (oracle/_ref/libmsmpb_ref.so, built
  by oracle/build_ref.py from the reference sources plus two index patches)
  driven through its own forcefield.h API (code/forcefield.h:70-97).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module. The product library never does.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libmsm_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libmsmpb_ref.so")
REF_UNPATCHED_SO = os.path.join(HERE, "_ref", "libmsmpb_ref_unpatched.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def build_oracle(force=False):
    """Compile the C restatement (gcc, no GPU needed)."""
    srcs = [os.path.join(HERE, "msm_oracle.c"), os.path.join(HERE, "pme_oracle.c"),
            os.path.join(HERE, "fftw_shim", "fft_shim.c")]
    if (not force and os.path.exists(ORACLE_SO) and
            all(os.path.getmtime(s) <= os.path.getmtime(ORACLE_SO) for s in srcs)):
        return ORACLE_SO
    cmd = [os.environ.get("CC", "gcc"), "-O3", "-std=gnu11", "-fPIC", "-shared",
           "-I", HERE, *srcs, "-lm", "-o", ORACLE_SO]
    subprocess.run(cmd, check=True)
    return ORACLE_SO


def _ptr(a, ctype=C.c_double):
    return a.ctypes.data_as(C.POINTER(ctype))


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Oracle:
    """FP64 CPU restatement of the reference MSM path."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            build_oracle()
            lib = C.CDLL(ORACLE_SO)
            lib.msmo_create.restype = C.c_void_p
            lib.msmo_create.argtypes = [C.c_int, _dp, _dp, C.c_double, C.c_int,
                                        C.c_int, _ip, C.c_double, C.c_int]
            lib.msmo_destroy.argtypes = [C.c_void_p]
            lib.msmo_params.argtypes = [C.c_void_p, _dp, _ip, _ip, _ip, _ip, _dp]
            lib.msmo_errEst.restype = C.c_double
            lib.msmo_errEst.argtypes = [C.c_void_p, _dp]
            lib.msmo_deltaF.restype = C.c_double
            lib.msmo_deltaF.argtypes = [C.c_void_p, _dp]
            lib.msmo_coeffs.argtypes = [C.c_void_p, _dp, _dp]
            lib.msmo_khat.restype = _dp
            lib.msmo_khat.argtypes = [C.c_void_p, C.c_int, _ip]
            lib.msmo_omegap.restype = _dp
            lib.msmo_omegap.argtypes = [C.c_void_p, C.c_int, C.c_int, _ip]
            lib.msmo_cL.restype = _dp
            lib.msmo_cL.argtypes = [C.c_void_p, C.c_int]
            lib.msmo_energy.restype = C.c_double
            lib.msmo_energy.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp, _dp]
            lib.msmo_short_range.restype = C.c_double
            lib.msmo_short_range.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp]
            lib.msmo_anterpolate.argtypes = [C.c_void_p, _dp, _dp, _dp]
            lib.msmo_grid_chain.argtypes = [C.c_void_p, _dp, _dp, _dp]
            lib.msmo_restrict.argtypes = [C.c_void_p, C.c_int, _dp, _dp]
            lib.msmo_prolong_add.argtypes = [C.c_void_p, C.c_int, _dp, _dp]
            lib.msmo_stencil_add.argtypes = [C.c_void_p, C.c_int, _dp, _dp]
            lib.msmo_top_solve.argtypes = [C.c_void_p, _dp, _dp]
            lib.msmo_interpolate.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp]
            lib.msmo_grid_dims.restype = C.c_int
            lib.msmo_grid_dims.argtypes = [C.c_void_p, C.c_int, _ip]
            lib.msmo_pair_count.restype = C.c_long
            lib.msmo_pair_count.argtypes = [C.c_void_p, _dp]
            cls._lib = lib
        return cls._lib

    def __init__(self, q, edges, cutoff=-1, nu=-1, levels=-1, top_grid=None,
                 est_err=-1, fft=True):
        self.q = _f64(q)
        self.N = len(self.q)
        self.edges = _f64(np.asarray(edges).reshape(3, 3))
        lib = self.lib()
        tg = None
        if top_grid is not None:
            tg = np.ascontiguousarray(np.broadcast_to(np.asarray(top_grid), (3,)),
                                      dtype=np.int32)
        self._tg = tg
        self.h = lib.msmo_create(self.N, _ptr(self.q), _ptr(self.edges),
                                 float(cutoff), int(nu), int(levels),
                                 _ptr(tg, C.c_int) if tg is not None else None,
                                 float(est_err), 1 if fft else 0)
        if not self.h:
            raise ValueError("oracle rejected the parameters")
        c, n, L, nl, d = C.c_double(), C.c_int(), C.c_int(), C.c_int(), C.c_double()
        M = (C.c_int * 3)()
        lib.msmo_params(self.h, C.byref(c), C.byref(n), C.byref(L), M,
                        C.byref(nl), C.byref(d))
        self.cutoff, self.nu, self.levels = c.value, n.value, L.value
        self.top_grid = tuple(M)
        self.nlim, self.detA = nl.value, d.value

    def __del__(self):
        if getattr(self, "h", None) and self._lib is not None:
            self._lib.msmo_destroy(self.h)
            self.h = None

    def grid_dims(self, l):
        d = (C.c_int * 3)()
        self.lib().msmo_grid_dims(self.h, l, d)
        return tuple(d)

    def energy(self, pos, weight=None, q=None):
        """(energy, forces[N,3], potentials[N])"""
        pos = _f64(pos)
        q = self.q if q is None else _f64(q)
        f = np.zeros((self.N, 3))
        phi = np.zeros(self.N)
        w = None if weight is None else _f64(weight)
        e = self.lib().msmo_energy(self.h, _ptr(q), _ptr(pos),
                                   _ptr(w) if w is not None else None,
                                   _ptr(f), _ptr(phi))
        return e, f, phi

    def short_range(self, pos, q=None):
        pos = _f64(pos)
        q = self.q if q is None else _f64(q)
        f = np.zeros((self.N, 3))
        phi = np.zeros(self.N)
        e = self.lib().msmo_short_range(self.h, _ptr(q), _ptr(pos), _ptr(f),
                                        _ptr(phi))
        return e, f, phi

    def anterpolate(self, pos, q=None):
        q = self.q if q is None else _f64(q)
        g = np.zeros(self.grid_dims(1))
        self.lib().msmo_anterpolate(self.h, _ptr(q), _ptr(_f64(pos)), _ptr(g))
        return g

    def grid_chain(self, q1, weight=None):
        e1 = np.zeros(self.grid_dims(1))
        w = None if weight is None else _f64(weight)
        self.lib().msmo_grid_chain(self.h, _ptr(_f64(q1)),
                                   _ptr(w) if w is not None else None, _ptr(e1))
        return e1

    def restrict(self, l, ql):
        out = np.zeros(self.grid_dims(l + 1))
        self.lib().msmo_restrict(self.h, l, _ptr(_f64(ql)), _ptr(out))
        return out

    def prolong_add(self, l, elp1, el):
        el = _f64(el).copy()
        self.lib().msmo_prolong_add(self.h, l, _ptr(_f64(elp1)), _ptr(el))
        return el

    def stencil_add(self, l, ql, el):
        el = _f64(el).copy()
        self.lib().msmo_stencil_add(self.h, l, _ptr(_f64(ql)), _ptr(el))
        return el

    def top_solve(self, qL):
        out = np.zeros(self.grid_dims(self.levels))
        self.lib().msmo_top_solve(self.h, _ptr(_f64(qL)), _ptr(out))
        return out

    def interpolate(self, pos, e1):
        ef = np.zeros((self.N, 3))
        ph = np.zeros(self.N)
        self.lib().msmo_interpolate(self.h, _ptr(_f64(pos)), _ptr(_f64(e1)),
                                    _ptr(ef), _ptr(ph))
        return ef, ph

    def khat(self, l):
        d = (C.c_int * 3)()
        p = self.lib().msmo_khat(self.h, l, d)
        n = d[0] * d[1] * d[2]
        return np.ctypeslib.as_array(p, shape=(n,)).reshape(tuple(d)).copy()

    def omegap(self, l, axis):
        n = C.c_int()
        p = self.lib().msmo_omegap(self.h, l, axis, C.byref(n))
        return np.ctypeslib.as_array(p, shape=(n.value,)).copy()

    def cL(self, axis):
        p = self.lib().msmo_cL(self.h, axis)
        return np.ctypeslib.as_array(p, shape=(self.top_grid[axis],)).copy()

    def coeffs(self):
        a, b = C.c_double(), C.c_double()
        self.lib().msmo_coeffs(self.h, C.byref(a), C.byref(b))
        return a.value, b.value

    def err_est(self):
        return self.lib().msmo_errEst(self.h, _ptr(self.q))

    def delta_f(self):
        return self.lib().msmo_deltaF(self.h, _ptr(self.q))

    def pair_count(self, pos):
        return self.lib().msmo_pair_count(self.h, _ptr(_f64(pos)))


# ---------------------------------------------------------------------------
# The reference library through its own API

class FFStruct(C.Structure):
    """Layout of ``FF`` (code/forcefield.h:22-69) on x86-64."""
    _fields_ = [
        ("N", C.c_int), ("q", _dp),
        ("A", C.c_double * 9), ("Ai", C.c_double * 9),
        ("detA", C.c_double), ("relCutoff", C.c_double),
        ("errEst", C.c_double), ("errEstMoore", C.c_double),
        ("ntc", C.c_int), ("tmax", C.c_int), ("estErr", C.c_double),
        ("orderAcc", C.c_int), ("maxLevel", C.c_int),
        ("topGridDim", C.c_int * 3), ("nlist", _ip),
        ("nlist_len", C.c_int), ("nlist_interaction_count", C.c_int),
        ("FFT", C.c_bool), ("fftw_in", C.c_void_p),
        ("forward", C.c_void_p), ("backward", C.c_void_p),
        ("tau", _dp), ("dsigma", _dp), ("sigmad", C.c_void_p), ("Q", _dp),
        ("J", _dp), ("omegap", C.c_void_p), ("nLim", C.c_int),
        ("aCut", _dp), ("cutoff", C.c_double), ("cL", _dp * 3),
        ("khat", C.POINTER(_dp)), ("coeff1", C.c_double), ("coeff2", C.c_double),
        ("time_partcl2partcl", C.c_double), ("time_nlist", C.c_double),
        ("time_grid2grid", C.c_double * 10), ("time_stencil", C.c_double * 10),
        ("time_anterpolation", C.c_double), ("time_interpolation", C.c_double),
        ("time_restriction", C.c_double * 10),
        ("time_prolongation", C.c_double * 10),
        ("time_padding", C.c_double * 10),
    ]


def bind_ff_api(lib):
    """Declare the forcefield.h signatures (code/forcefield.h:70-97) on a
    loaded library (the reference build or the product library)."""
    P = C.POINTER(FFStruct)
    lib.FF_new.restype = P
    lib.FF_new.argtypes = [C.c_int, _dp]
    lib.FF_set_cutoff.argtypes = [P, C.c_double]
    lib.FF_set_orderAcc.argtypes = [P, C.c_int]
    lib.FF_set_maxLevel.argtypes = [P, C.c_int]
    lib.FF_set_topGridDim.argtypes = [P, _ip]
    lib.FF_set_FFT.argtypes = [P, C.c_bool]
    lib.FF_set_estErr.argtypes = [P, C.c_double]
    lib.FF_build.argtypes = [P, C.c_int, _dp, _dp, C.c_double]
    lib.FF_rebuild.argtypes = [P, _dp, _dp, C.c_double]
    lib.FF_energy.restype = C.c_double
    lib.FF_energy.argtypes = [P, _dp, _dp, _dp]
    lib.FF_delete.argtypes = [P]
    lib.FF_get_cutoff.restype = C.c_double
    lib.FF_get_cutoff.argtypes = [P]
    lib.FF_get_orderAcc.restype = C.c_int
    lib.FF_get_orderAcc.argtypes = [P]
    lib.FF_get_maxLevel.restype = C.c_int
    lib.FF_get_maxLevel.argtypes = [P]
    lib.FF_get_topGridDim.argtypes = [P, _ip]
    lib.FF_get_FFT.restype = C.c_bool
    lib.FF_get_FFT.argtypes = [P]
    lib.FF_get_errEst.restype = C.c_double
    lib.FF_get_errEst.argtypes = [P]
    lib.FF_get_estErr.restype = C.c_double
    lib.FF_get_estErr.argtypes = [P]
    lib.FF_get_deltaF.restype = C.c_double
    lib.FF_get_deltaF.argtypes = [P]
    return lib


class RefFF:
    """The reference MSM library (patched build) through its C API."""

    _libs = {}

    @classmethod
    def available(cls, unpatched=False):
        return os.path.exists(REF_UNPATCHED_SO if unpatched else REF_SO)

    @classmethod
    def lib(cls, unpatched=False, path=None):
        """The patched (default) or unpatched build; ``path`` names another
        build of the patched sources (build_ref.build_native)."""
        path = path or (REF_UNPATCHED_SO if unpatched else REF_SO)
        if path not in cls._libs:
            if not os.path.exists(path):
                raise FileNotFoundError(path + " (run oracle/build_ref.py)")
            cls._libs[path] = bind_ff_api(C.CDLL(path))
        return cls._libs[path]

    def __init__(self, q, pos, edges, cutoff=None, nu=None, levels=None,
                 top_grid=None, margin=0.0, unpatched=False, lib_path=None):
        lib = self.lib(unpatched, lib_path)
        self._lib = lib
        self.q = _f64(q).copy()  # FF_new keeps the caller's pointer
        self.N = len(self.q)
        self.edges = _f64(np.asarray(edges).reshape(3, 3)).copy()
        self.pos = _f64(pos).copy()
        self.ff = lib.FF_new(self.N, _ptr(self.q))
        if levels is not None:
            lib.FF_set_maxLevel(self.ff, int(levels))
        if top_grid is not None:
            tg = np.ascontiguousarray(np.broadcast_to(np.asarray(top_grid), (3,)),
                                      dtype=np.int32)
            lib.FF_set_topGridDim(self.ff, _ptr(tg, C.c_int))
        if nu is not None:
            lib.FF_set_orderAcc(self.ff, int(nu))
        if cutoff is not None:
            lib.FF_set_cutoff(self.ff, float(cutoff))
        lib.FF_build(self.ff, self.N, _ptr(self.pos), _ptr(self.edges),
                     float(margin))
        s = self.ff.contents
        self.cutoff = s.cutoff
        self.nu = s.orderAcc
        self.levels = s.maxLevel
        self.top_grid = tuple(s.topGridDim)
        self.nlim = s.nLim

    def energy(self, pos=None):
        pos = self.pos if pos is None else _f64(pos)
        f = np.zeros((self.N, 3))
        e = self._lib.FF_energy(self.ff, _ptr(f), _ptr(pos), None)
        return e, f

    def potentials(self, pos=None, idx=None, h=1.0):
        """dU/dq_i by central differences in q (exact for the quadratic U)."""
        idx = range(self.N) if idx is None else idx
        out = []
        for i in idx:
            q0 = self.q[i]
            self.q[i] = q0 + h
            ep, _ = self.energy(pos)
            self.q[i] = q0 - h
            em, _ = self.energy(pos)
            self.q[i] = q0
            out.append((ep - em) / (2 * h))
        return np.array(out)

    def struct(self):
        return self.ff.contents

    def close(self):
        if self.ff:
            self._lib.FF_delete(self.ff)
            self.ff = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PmeOracle:
    """FP64 CPU restatement of the reference smooth-PME path
    (oracle/pme_oracle.c)."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            lib = Oracle.lib()
            lib.pmeo_create.restype = C.c_void_p
            lib.pmeo_create.argtypes = [C.c_int, _dp, C.c_double, C.c_int, _ip, C.c_double]
            lib.pmeo_destroy.argtypes = [C.c_void_p]
            lib.pmeo_rebuild.argtypes = [C.c_void_p, _dp]
            lib.pmeo_params.argtypes = [C.c_void_p, _dp, _ip, _ip, _dp, _dp, _dp]
            lib.pmeo_coeffs.argtypes = [C.c_void_p, _dp, _dp]
            lib.pmeo_khat.restype = _dp
            lib.pmeo_khat.argtypes = [C.c_void_p]
            lib.pmeo_cL.restype = _dp
            lib.pmeo_cL.argtypes = [C.c_void_p, C.c_int]
            lib.pmeo_errEst.restype = C.c_double
            lib.pmeo_errEst.argtypes = [C.c_void_p, _dp]
            lib.pmeo_energy.restype = C.c_double
            lib.pmeo_energy.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp, _dp]
            lib.pmeo_short_range.restype = C.c_double
            lib.pmeo_short_range.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp]
            cls._lib = lib
        return cls._lib

    def __init__(self, q, edges, cutoff=-1, nu=-1, grid=None, tol_dir=-1):
        lib = self.lib()
        self.q = _f64(q)
        self.N = len(self.q)
        self.edges = _f64(np.asarray(edges).reshape(3, 3)).copy()
        g = None
        if grid is not None:
            g = np.ascontiguousarray(np.broadcast_to(np.asarray(grid), (3,)), dtype=np.int32)
        self.h = lib.pmeo_create(self.N, _ptr(self.edges), float(cutoff), int(nu),
                                 _ptr(g, C.c_int) if g is not None else None, float(tol_dir))
        if not self.h:
            raise ValueError("no default PME grid for this order and cutoff")
        self._read()

    def _read(self):
        c, n, t, b, d = C.c_double(), C.c_int(), C.c_double(), C.c_double(), C.c_double()
        M = (C.c_int * 3)()
        self.lib().pmeo_params(self.h, C.byref(c), C.byref(n), M, C.byref(t), C.byref(b),
                               C.byref(d))
        self.cutoff, self.nu, self.grid = c.value, n.value, tuple(M)
        self.tol_dir, self.beta, self.detA = t.value, b.value, d.value

    def rebuild(self, edges):
        self.edges = _f64(np.asarray(edges).reshape(3, 3)).copy()
        self.lib().pmeo_rebuild(self.h, _ptr(self.edges))
        self._read()

    def energy(self, pos, weight=None, q=None):
        q = self.q if q is None else _f64(q)
        pos = _f64(pos)
        f = np.zeros((self.N, 3))
        phi = np.zeros(self.N)
        w = None if weight is None else _f64(weight)
        e = self.lib().pmeo_energy(self.h, _ptr(q), _ptr(pos), _ptr(w) if w is not None else None,
                                   _ptr(f), _ptr(phi))
        return e, f, phi

    def short_range(self, pos, q=None):
        q = self.q if q is None else _f64(q)
        f = np.zeros((self.N, 3))
        phi = np.zeros(self.N)
        e = self.lib().pmeo_short_range(self.h, _ptr(q), _ptr(_f64(pos)), _ptr(f), _ptr(phi))
        return e, f, phi

    def coeffs(self):
        c1, c2 = C.c_double(), C.c_double()
        self.lib().pmeo_coeffs(self.h, C.byref(c1), C.byref(c2))
        return c1.value, c2.value

    def khat(self):
        n = self.grid[0] * self.grid[1] * self.grid[2]
        return np.ctypeslib.as_array(self.lib().pmeo_khat(self.h), (n,)).copy().reshape(self.grid)

    def err_est(self):
        return self.lib().pmeo_errEst(self.h, _ptr(self.q))

    def __del__(self):
        if getattr(self, "h", None) and self._lib is not None:
            self._lib.pmeo_destroy(self.h)
            self.h = None


REF_PME_SO = os.path.join(HERE, "_ref", "libpme_ref.so")


class PmeStruct(C.Structure):
    """struct FF of the reference's code/pme.h:16-44."""
    _fields_ = [
        ("N", C.c_int), ("q", _dp), ("A", C.c_double * 9), ("Ai", C.c_double * 9),
        ("detA", C.c_double), ("cutoff", C.c_double), ("orderAcc", C.c_int),
        ("topGridDim", C.c_int * 3), ("nlist", _ip), ("nlist_len", C.c_int),
        ("nlist_interaction_count", C.c_int), ("tolDir", C.c_double),
        ("fftw_in", C.c_void_p), ("forward", C.c_void_p), ("backward", C.c_void_p),
        ("beta", C.c_double), ("Q", _dp), ("cL", _dp * 3), ("khat", _dp),
        ("coeff1", C.c_double), ("coeff2", C.c_double),
        ("time_partcl2partcl", C.c_double), ("time_nlist", C.c_double),
        ("time_grid2grid", C.c_double), ("time_stencil", C.c_double),
        ("time_anterpolation", C.c_double), ("time_interpolation", C.c_double),
    ]


def bind_pme_api(lib, struct=PmeStruct):
    """Signatures of the PME C API (code/pme.h:45-68)."""
    P = C.POINTER(struct)
    sig = {
        "FF_new": (P, [C.c_int, _dp, _dp]),
        "FF_set_cutoff": (None, [P, C.c_double]),
        "FF_set_orderAcc": (None, [P, C.c_int]),
        "FF_set_topGridDim": (None, [P, _ip]),
        "FF_set_tolDir": (None, [P, C.c_double]),
        "FF_build": (None, [P, _dp]),
        "FF_get_cutoff": (C.c_double, [P]),
        "FF_get_orderAcc": (C.c_int, [P]),
        "FF_get_topGridDim": (None, [P, _ip]),
        "FF_get_tolDir": (C.c_double, [P]),
        "FF_get_errEst": (C.c_double, [P, C.c_int, _dp]),
        "FF_rebuild": (None, [P, _dp, _dp]),
        "FF_energy": (C.c_double, [P, _dp, _dp, _dp]),
        "FF_delete": (None, [P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


class RefPme:
    """The reference PME library (oracle/_ref/libpme_ref.so, built from
    code/pme0.c and code/pme1.c) through its own C API."""

    _lib = None

    @classmethod
    def available(cls):
        return os.path.exists(REF_PME_SO)

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not os.path.exists(REF_PME_SO):
                raise FileNotFoundError(REF_PME_SO + " (run oracle/build_ref.py)")
            cls._lib = bind_pme_api(C.CDLL(REF_PME_SO))
        return cls._lib

    def __init__(self, q, pos, edges, cutoff=None, nu=None, grid=None, tol_dir=None):
        lib = self.lib()
        self.q = _f64(q).copy()
        self.N = len(self.q)
        self.edges = _f64(np.asarray(edges).reshape(3, 3)).copy()
        self.pos = _f64(pos).copy()
        self.ff = lib.FF_new(self.N, _ptr(self.q), _ptr(self.edges))
        if cutoff is not None:
            lib.FF_set_cutoff(self.ff, float(cutoff))
        if grid is not None:
            self._g = np.ascontiguousarray(np.broadcast_to(np.asarray(grid), (3,)),
                                           dtype=np.int32)
            lib.FF_set_topGridDim(self.ff, _ptr(self._g, C.c_int))
        if nu is not None:
            lib.FF_set_orderAcc(self.ff, int(nu))
        if tol_dir is not None:
            lib.FF_set_tolDir(self.ff, float(tol_dir))
        lib.FF_build(self.ff, _ptr(self.pos))
        s = self.ff.contents
        self.cutoff, self.nu, self.grid = s.cutoff, s.orderAcc, tuple(s.topGridDim)
        self.tol_dir, self.beta = s.tolDir, s.beta

    def energy(self, pos=None):
        pos = self.pos if pos is None else _f64(pos)
        f = np.zeros((self.N, 3))
        e = self._lib.FF_energy(self.ff, _ptr(f), _ptr(pos), None)
        return e, f

    def err_est(self):
        return self._lib.FF_get_errEst(self.ff, self.N, _ptr(self.q))

    def struct(self):
        return self.ff.contents

    def khat(self):
        g = self.grid
        return np.ctypeslib.as_array(self.ff.contents.khat, (g[0] * g[1] * g[2],)).copy().reshape(g)

    def close(self):
        if getattr(self, "ff", None):
            self._lib.FF_delete(self.ff)
            self.ff = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def read_ini(path):
    """Reference .ini fixture (code/msmpb.c:93-118): edges row, N, then
    ``q x y z mass ...`` per atom."""
    with open(path) as f:
        lines = f.read().split("\n")
    edges = np.array([float(v) for v in lines[0].split()[:9]]).reshape(3, 3)
    n = int(lines[1].split()[0])
    rows = np.array([[float(v) for v in lines[2 + i].split()[:5]] for i in range(n)])
    return edges, rows[:, 0].copy(), rows[:, 1:4].copy(), rows[:, 4].copy()


def read_acc(path, n):
    """.acc fixture: N then x-, y-, z-blocks of -F/q (code/msmpb.c:254-270)."""
    v = np.loadtxt(path, skiprows=1)
    return np.stack([v[:n], v[n:2 * n], v[2 * n:3 * n]], axis=1)
