"""ctypes binding of libexcfv (the C ABI declared in include/excfv.h).

The shared library is built in-tree (``exciting_b200/libexcfv.so``) by
``exciting_b200.build.build_library``.  There is no fallback: if the library
is missing, :func:`load` raises.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libexcfv.so")

EXCFV_OK = 0
EXCFV_ERR_ARG = -1
EXCFV_ERR_UNSUPPORTED = -2
EXCFV_ERR_CUDA = -3
EXCFV_ERR_ALLOC = -4
EXCFV_ERR_STATE = -5
EXCFV_ERR_TIMEOUT = -6
EXCFV_ERR_NOCONV = -7

EXCFV_PREC_FP64 = 0
EXCFV_PREC_MIXED = 1

EXCFV_BATCH_LANES = 0
EXCFV_BATCH_GROUPED = 1
EXCFV_BATCH_AUTO = 2
EXCFV_BATCH_GROUPED_LANES = 3

_i32p = C.POINTER(C.c_int32)
_f64p = C.POINTER(C.c_double)


class ExcfvStatic(C.Structure):
    """Mirror of ``struct excfv_static`` (field order and types must match)."""
    _fields_ = [
        ("natmtot", C.c_int32), ("nspecies", C.c_int32), ("idxis", _i32p),
        ("omega", C.c_double), ("rmt", _f64p),
        ("lmaxapw", C.c_int32), ("lmaxmat", C.c_int32), ("apwordmax", C.c_int32),
        ("apword", _i32p), ("nlomax", C.c_int32), ("nlorb", _i32p), ("lorbl", _i32p),
        ("lolmax", C.c_int32), ("idxlo", _i32p), ("nlotot", C.c_int32),
        ("maxaa", C.c_int32), ("maxnlo", C.c_int32), ("losize", _i32p),
        ("aa", _f64p), ("loa", _f64p), ("lolo", _f64p), ("oalo", _f64p), ("ololo", _f64p),
        ("h1aa", _f64p), ("h1loa", _f64p), ("h1lolo", _f64p), ("h1on", C.c_int32),
        ("valence_relativity", C.c_int32),
        ("ngvec", C.c_int32), ("ngrtot", C.c_int32), ("ivg", _i32p), ("ivgig", _i32p),
        ("intgv", C.c_int32 * 6),
        ("veffig", _f64p), ("meffig", _f64p), ("cfunig", _f64p), ("m2effig", _f64p),
        ("npmatch", C.c_int32), ("sprwin", _f64p), ("apwfrwin", _f64p),
        ("nstfv", C.c_int32), ("evaltol", C.c_double),
    ]


class ExcfvMtrad(C.Structure):
    """Mirror of ``struct excfv_mtrad`` (field order and types must match)."""
    _fields_ = [
        ("lmaxvr", C.c_int32), ("nrmtmax", C.c_int32), ("nrmt", _i32p), ("spr", _f64p),
        ("apwfr", _f64p), ("lofr", _f64p), ("veffmt", _f64p),
    ]


class ExcfvRhoset(C.Structure):
    """Mirror of ``struct excfv_rhoset`` (field order and types must match)."""
    _fields_ = [
        ("lmaxvr", C.c_int32), ("lradstep", C.c_int32), ("nrmtmax", C.c_int32), ("nrmt", _i32p),
        ("apwfr", _f64p), ("lofr", _f64p), ("zbshtvr", _f64p), ("rfshtvr", _f64p),
    ]


class ExcfvBfield(C.Structure):
    """Mirror of ``struct excfv_bfield`` (field order and types must match)."""
    _fields_ = [
        ("rad", C.POINTER(ExcfvMtrad)), ("bxcmt", _f64p), ("bmtconst", _f64p), ("ngrid", _i32p),
        ("bxcir", _f64p), ("cfunir", _f64p), ("birconst", C.c_double),
    ]


class ExcfvBfieldNc(C.Structure):
    """Mirror of ``struct excfv_bfield_nc`` (field order and types must match)."""
    _fields_ = [
        ("rad", C.POINTER(ExcfvMtrad)), ("bxcmt", _f64p), ("bmtconst", _f64p), ("ngrid", _i32p),
        ("bxcir", _f64p), ("cfunir", _f64p), ("birconst", C.c_double * 3), ("spinorb", C.c_int32),
    ]


#: name -> (restype, argtypes); every symbol declared in include/excfv.h
SIGNATURES = {
    "excfv_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "excfv_destroy": (C.c_int, [C.c_void_p]),
    "excfv_last_error": (C.c_char_p, []),
    "excfv_set_precision": (C.c_int, [C.c_void_p, C.c_int]),
    "excfv_set_batch_graph": (C.c_int, [C.c_void_p, C.c_int]),
    "excfv_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "excfv_reserve": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32]),
    "excfv_set_static": (C.c_int, [C.c_void_p, C.POINTER(ExcfvStatic)]),
    "excfv_genveffig": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "excfv_genmeffig": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.c_void_p]),
    "excfv_set_rho": (C.c_int, [C.c_void_p, C.POINTER(ExcfvRhoset)]),
    "excfv_rhovalk": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                C.c_int32, C.c_void_p, C.c_void_p, C.c_double]),
    "excfv_rhovalk_dev": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_int32, C.c_void_p, C.c_void_p, C.c_double]),
    "excfv_get_rhomt": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32]),
    "excfv_get_magmt": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32]),
    "excfv_rhovalk_sv": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double]),
    "excfv_rhovalk_sv_nc": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double]),
    "excfv_get_magmt3": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32]),
    "excfv_set_bfield": (C.c_int, [C.c_void_p, C.POINTER(ExcfvBfield)]),
    "excfv_set_bfield_nc": (C.c_int, [C.c_void_p, C.POINTER(ExcfvBfieldNc)]),
    "excfv_seceqnsv": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                 C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "excfv_seceqnsv_dev": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "excfv_hmlint": (C.c_int, [C.c_void_p, C.POINTER(ExcfvMtrad), C.c_void_p, C.c_void_p, C.c_void_p,
                               C.c_void_p, C.c_void_p]),
    "excfv_match": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p,
                              C.c_void_p, C.c_void_p]),
    "excfv_hamiltonandoverlapsetup": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32,
                                                C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                C.c_void_p]),
    "excfv_solvewithlapack": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32,
                                        C.c_double, C.c_void_p, C.c_void_p, C.c_int32]),
    "excfv_seceqnfv": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                 C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p,
                                 C.c_void_p]),
    "excfv_seceqn": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_void_p,
                               C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32,
                               C.c_void_p, C.c_void_p]),
    "excfv_seceqn_dev": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_void_p,
                                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32,
                                   C.c_void_p, C.c_void_p]),
    "excfv_sync": (C.c_int, [C.c_void_p]),
    "excfv_get_timings": (C.c_int, [C.c_void_p, C.c_void_p]),
    "excfv_profile": (C.c_int, [C.c_void_p, C.c_int]),
    "excfv_profile_read": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    "excfv_launch_count": (C.c_longlong, []),
    "excfv_tridiag_tail_start": (C.c_int, [C.c_int, C.c_int]),
    "excfv_test_set_wait_limit": (C.c_int, [C.c_int64, C.c_int32]),
    "excfv_set_reduction": (C.c_int, [C.c_void_p, C.c_int]),
    "excfv_set_lattice": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "excfv_putevecfv": (C.c_int, [C.c_char_p, C.c_int32, C.c_void_p, C.c_int32, C.c_int32, C.c_int32,
                                  C.c_void_p]),
    "excfv_putevecfv_dev": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int32, C.c_void_p, C.c_int32, C.c_int32,
                                      C.c_int32, C.c_void_p]),
    "excfv_getevecfv": (C.c_int, [C.c_char_p, C.c_int32, C.c_void_p, C.c_int32, C.c_int32, C.c_int32,
                                  C.c_void_p]),
    "excfv_gengpvec": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_int32, C.c_void_p,
                                 C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "excfv_gengpvec_dev": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_int32, C.c_void_p,
                                     C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "excfv_gensfacgp": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_void_p]),
    "excfv_gensfacgp_dev": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_void_p]),
    "excfv_test_reduce_band": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_void_p,
                                         C.c_void_p, C.c_void_p, C.c_void_p]),
    "excfv_seceqn_batched_dev": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32,
                                           C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]),
    "excfv_seceqn_batched": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32,
                                       C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "excfv_batch_info": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p]),
    "excfv_set_lanes": (C.c_int, [C.c_void_p, C.c_int32]),
    "excfv_set_batch_mode": (C.c_int, [C.c_void_p, C.c_int32]),
    "excfv_get_batch_mode": (C.c_int, [C.c_void_p]),
    "excfv_group_launches": (C.c_longlong, [C.c_void_p]),
    "excfv_set_group_tile": (C.c_int, [C.c_void_p, C.c_int32]),
    "excfv_get_group_tile": (C.c_int, [C.c_void_p]),
    "excfv_get_lanes": (C.c_int, [C.c_void_p]),
    "excfv_autotune_lanes": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32,
                                       C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "excfv_match_noalloc": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p]),
}

#: bytes of the fixed scratch array of excfv_match_noalloc (EXCFV_NOALLOC_SCRATCH_BYTES)
NOALLOC_SCRATCH_BYTES = 32 << 20

PROF_CLASSES = ["match", "setup_gemm", "setup_other", "potrf", "hegst", "trd_panel",
                "trd_update", "steig", "backtr", "trd_chase", "trd_tail"]

EXCFV_REDUCTION_AUTO = 0
EXCFV_REDUCTION_ONE_STAGE = 1
EXCFV_REDUCTION_TWO_STAGE = 2

_lib: Optional[C.CDLL] = None


def load(path: str = LIB_PATH) -> C.CDLL:
    """Load libexcfv and declare every C-ABI signature.  Raises if missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(
            f"libexcfv not found at {path}: build it with exciting_b200.build.build_library() "
            "(there is no CPU fallback)")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def last_error() -> str:
    return load().excfv_last_error().decode(errors="replace")


class ExcfvError(RuntimeError):
    def __init__(self, code: int, where: str):
        self.code = code
        super().__init__(f"{where} failed with status {code}: {last_error()}")


def putevecfv(path: str, ik: int, vkl, evecfv) -> None:
    """Write record ik (1-based) of an EVECFV file; evecfv is (nmatmax, nstfv[, nspnfv]) complex."""
    import numpy as np
    L = load()
    e = np.asfortranarray(evecfv, dtype=np.complex128)
    if e.ndim == 2:
        e = e[:, :, None]
    v = np.ascontiguousarray(vkl, dtype=np.float64)
    rc = L.excfv_putevecfv(path.encode(), ik, v.ctypes.data, e.shape[0], e.shape[1], e.shape[2], e.ctypes.data)
    if rc:
        raise ExcfvError(rc, "excfv_putevecfv")


def getevecfv(path: str, ik: int, vkl, nmatmax: int, nstfv: int, nspnfv: int = 1):
    """Read record ik of an EVECFV file with the reference's consistency checks."""
    import numpy as np
    L = load()
    e = np.zeros((nmatmax, nstfv, nspnfv), dtype=np.complex128, order="F")
    v = None if vkl is None else np.ascontiguousarray(vkl, dtype=np.float64)
    rc = L.excfv_getevecfv(path.encode(), ik, None if v is None else v.ctypes.data, nmatmax, nstfv, nspnfv,
                           e.ctypes.data)
    if rc:
        raise ExcfvError(rc, "excfv_getevecfv")
    return e
