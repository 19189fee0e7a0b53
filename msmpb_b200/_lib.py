"""Loader for the in-tree CUDA library ``msmpb_b200/libmsmpb.so``.

The library is the product: there is no Python or CPU fallback. If it is
missing, ``load()`` raises.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmsmpb.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)

# status codes (include/msmpb_b200.h)
OK = 0
ERR_ARGUMENT = 1
ERR_STATE = 2
ERR_CUDA = 3
ERR_NOMEM = 4
ERR_NODEVICE = 5
ERR_DEVICE_CHECK = 6
ERR_UNSUPPORTED = 7

PRECISION_MIXED = 0
PRECISION_FP64 = 1

# Every symbol the public headers declare (include/forcefield.h,
# include/msmpb_b200.h)
EXPORTED = [
    "FF_new", "FF_get_cutoff", "FF_set_cutoff", "FF_set_orderAcc",
    "FF_set_maxLevel", "FF_set_topGridDim", "FF_set_FFT", "FF_build",
    "FF_get_orderAcc", "FF_get_maxLevel", "FF_get_topGridDim", "FF_get_FFT",
    "FF_get_errEst", "FF_get_estErr", "FF_set_estErr", "FF_rebuild",
    "FF_energy", "FF_delete", "FF_get_deltaF", "msm4g_tictocmanager",
    "msm4g_tic", "msm4g_toc", "invert", "omegap", "prod", "prodT",
    "_FF_get_errEst",
    "FF_last_error", "FF_error_string", "FF_set_precision",
    "FF_get_precision", "FF_set_device", "FF_energy_potentials",
    "FF_energy_device", "FF_sync", "FF_phase_times", "FF_kernel_launches",
    "FF_stencil_times", "FF_set_timing", "msmpb_measure_fp32_tflops",
    "msmpb_level_stencil_noalloc", "FF_rebuild_device", "FF_adjoint_device",
    "FF_evaluation_count", "FF_batch_new", "FF_batch_energy_device",
    "FF_batch_branches", "FF_batch_kernel_launches", "FF_batch_last_error",
    "FF_batch_delete",
]

_lib = None


class FFStruct(C.Structure):
    """struct FF of include/forcefield.h (reference layout + appended
    members)."""
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
        ("khat", C.POINTER(_dp)), ("coeff1", C.c_double),
        ("coeff2", C.c_double),
        ("time_partcl2partcl", C.c_double), ("time_nlist", C.c_double),
        ("time_grid2grid", C.c_double * 10), ("time_stencil", C.c_double * 10),
        ("time_anterpolation", C.c_double), ("time_interpolation", C.c_double),
        ("time_restriction", C.c_double * 10),
        ("time_prolongation", C.c_double * 10),
        ("time_padding", C.c_double * 10),
        ("dev", C.c_void_p), ("host_state", C.c_void_p),
        ("last_error", C.c_int), ("precision", C.c_int), ("device", C.c_int),
        ("timing", C.c_int), ("margin", C.c_double),
    ]


def load():
    """Load and bind the library (raises OSError if it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError("msmpb_b200: %s is missing; run `python -m "
                      "msmpb_b200.build`" % LIB_PATH)
    lib = C.CDLL(LIB_PATH)
    P = C.POINTER(FFStruct)
    sig = {
        "FF_new": (P, [C.c_int, _dp]),
        "FF_set_cutoff": (None, [P, C.c_double]),
        "FF_set_orderAcc": (None, [P, C.c_int]),
        "FF_set_maxLevel": (None, [P, C.c_int]),
        "FF_set_topGridDim": (None, [P, _ip]),
        "FF_set_FFT": (None, [P, C.c_bool]),
        "FF_set_estErr": (None, [P, C.c_double]),
        "FF_build": (None, [P, C.c_int, _dp, _dp, C.c_double]),
        "FF_rebuild": (None, [P, _dp, _dp, C.c_double]),
        "FF_rebuild_device": (C.c_int, [P, _dp, C.c_void_p]),
        "FF_adjoint_device": (C.c_int, [P, C.c_void_p, C.c_void_p, _dp, C.c_void_p,
                                        C.c_double, C.c_void_p, C.c_void_p, C.c_int,
                                        C.c_void_p]),
        "FF_evaluation_count": (C.c_long, [P]),
        "FF_energy": (C.c_double, [P, _dp, _dp, _dp]),
        "FF_energy_potentials": (C.c_double, [P, _dp, _dp, _dp, _dp]),
        "FF_energy_device": (C.c_int, [P, C.c_void_p, C.c_void_p, _dp,
                                       C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_void_p]),
        "FF_delete": (None, [P]),
        "FF_get_cutoff": (C.c_double, [P]),
        "FF_get_orderAcc": (C.c_int, [P]),
        "FF_get_maxLevel": (C.c_int, [P]),
        "FF_get_topGridDim": (None, [P, _ip]),
        "FF_get_FFT": (C.c_bool, [P]),
        "FF_get_errEst": (C.c_double, [P]),
        "FF_get_estErr": (C.c_double, [P]),
        "FF_get_deltaF": (C.c_double, [P]),
        "_FF_get_errEst": (C.c_double, [P, C.c_int]),
        "FF_last_error": (C.c_int, [P]),
        "FF_error_string": (C.c_char_p, [C.c_int]),
        "FF_set_precision": (None, [P, C.c_int]),
        "FF_get_precision": (C.c_int, [P]),
        "FF_set_device": (None, [P, C.c_int]),
        "FF_sync": (C.c_int, [P]),
        "FF_phase_times": (C.c_int, [P, _dp, C.c_int]),
        "FF_kernel_launches": (C.c_int, [P]),
        "FF_stencil_times": (C.c_int, [P, _dp, C.c_int]),
        "FF_set_timing": (None, [P, C.c_int]),
        "msmpb_measure_fp32_tflops": (C.c_double, [C.c_int, C.c_int]),
        "FF_batch_new": (C.c_void_p, [C.POINTER(P), C.c_int, C.c_int, _ip]),
        "FF_batch_energy_device": (C.c_int, [C.c_void_p] + [C.POINTER(C.c_void_p)] * 2 +
                                   [C.POINTER(_dp)] + [C.POINTER(C.c_void_p)] * 2 +
                                   [C.c_void_p, C.c_void_p]),
        "FF_batch_branches": (C.c_int, [C.c_void_p]),
        "FF_batch_kernel_launches": (C.c_int, [C.c_void_p]),
        "FF_batch_last_error": (C.c_int, [C.c_void_p]),
        "FF_batch_delete": (None, [C.c_void_p]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


# ---------------------------------------------------------------------------
# The smooth-PME comparator library (include/pme.h, include/pme_b200.h)

PME_LIB_PATH = os.path.join(HERE, "libpme.so")

PME_EXPORTED = [
    "FF_new", "FF_set_cutoff", "FF_get_cutoff", "FF_set_orderAcc", "FF_set_topGridDim",
    "FF_set_tolDir", "FF_build", "FF_get_orderAcc", "FF_get_topGridDim", "FF_get_tolDir",
    "FF_get_errEst", "FF_rebuild", "FF_energy", "FF_delete", "msm4g_tictocmanager",
    "msm4g_tic", "msm4g_toc", "prod", "prodT",
    "FF_last_error", "FF_error_string", "FF_set_precision", "FF_get_precision",
    "FF_set_device", "FF_set_timing", "FF_energy_potentials", "FF_energy_device",
    "FF_sync", "FF_phase_times", "FF_kernel_launches",
]

_pme = None


class PmeStruct(C.Structure):
    """struct FF of include/pme.h (reference layout + appended members)."""
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
        ("dev", C.c_void_p), ("host_state", C.c_void_p), ("last_error", C.c_int),
        ("precision", C.c_int), ("device", C.c_int), ("timing", C.c_int),
    ]


def load_pme():
    """Load and bind libpme.so (raises OSError if it is not built)."""
    global _pme
    if _pme is not None:
        return _pme
    if not os.path.exists(PME_LIB_PATH):
        raise OSError("msmpb_b200: %s is missing; run `python -m msmpb_b200.build`"
                      % PME_LIB_PATH)
    lib = C.CDLL(PME_LIB_PATH)
    P = C.POINTER(PmeStruct)
    sig = {
        "FF_new": (P, [C.c_int, _dp, _dp]),
        "FF_set_cutoff": (None, [P, C.c_double]),
        "FF_get_cutoff": (C.c_double, [P]),
        "FF_set_orderAcc": (None, [P, C.c_int]),
        "FF_set_topGridDim": (None, [P, _ip]),
        "FF_set_tolDir": (None, [P, C.c_double]),
        "FF_build": (None, [P, _dp]),
        "FF_get_orderAcc": (C.c_int, [P]),
        "FF_get_topGridDim": (None, [P, _ip]),
        "FF_get_tolDir": (C.c_double, [P]),
        "FF_get_errEst": (C.c_double, [P, C.c_int, _dp]),
        "FF_rebuild": (None, [P, _dp, _dp]),
        "FF_energy": (C.c_double, [P, _dp, _dp, _dp]),
        "FF_energy_potentials": (C.c_double, [P, _dp, _dp, _dp, _dp]),
        "FF_energy_device": (C.c_int, [P, C.c_void_p, C.c_void_p, _dp, C.c_void_p,
                                       C.c_void_p, C.c_void_p, C.c_void_p]),
        "FF_delete": (None, [P]),
        "FF_last_error": (C.c_int, [P]),
        "FF_error_string": (C.c_char_p, [C.c_int]),
        "FF_set_precision": (None, [P, C.c_int]),
        "FF_get_precision": (C.c_int, [P]),
        "FF_set_device": (None, [P, C.c_int]),
        "FF_set_timing": (None, [P, C.c_int]),
        "FF_sync": (C.c_int, [P]),
        "FF_phase_times": (C.c_int, [P, _dp, C.c_int]),
        "FF_kernel_launches": (C.c_int, [P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _pme = lib
    return lib
