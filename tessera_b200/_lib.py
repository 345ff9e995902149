"""ctypes binding of libtessera_qa.so (declarations mirror include/tessera_qa.h).

The library is loaded from this package directory.  There is no fallback: when the
library is missing or cannot be loaded, ``load()`` raises, so no code path silently runs
anything but the CUDA engine.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtessera_qa.so")

c_size_p = C.POINTER(C.c_size_t)
c_double_p = C.POINTER(C.c_double)
c_int8_p = C.POINTER(C.c_int8)

TESSERA_QA_C128 = 0
TESSERA_QA_C64 = 1

EINVAL, ECUDA, ESTATUS, ESMALL = -1, -2, -3, -4
ST_JACOBI_NOT_CONVERGED, ST_BARRIER_TIMEOUT, ST_BAD_DIMS, ST_NONFINITE = 1, 2, 4, 8


class Problem(C.Structure):
    _fields_ = [("n", C.c_size_t), ("h", c_double_p), ("m", C.c_size_t), ("ei", c_size_p), ("ej", c_size_p),
                ("ew", c_double_p), ("steps", C.c_size_t), ("schedule_a", c_double_p),
                ("schedule_b", c_double_p), ("bias", c_double_p), ("schedule_c", c_double_p)]


class Config(C.Structure):
    _fields_ = [("dt", C.c_double), ("zz_substeps", C.c_int), ("precision", C.c_int), ("chi", C.c_size_t),
                ("jacobi_tol", C.c_double), ("jacobi_max_sweeps", C.c_int), ("jacobi_block", C.c_int),
                ("device", C.c_int), ("step_begin", C.c_size_t), ("step_end", C.c_size_t),
                ("initial_mps", C.c_void_p), ("skip_observables", C.c_int), ("kernel_timing", C.c_int),
                ("theta_tensor_cores", C.c_int), ("jacobi_precondition", C.c_int),
                ("reserved", C.c_int * 4)]


class Result(C.Structure):
    _fields_ = [("spins", c_int8_p), ("entropy", c_double_p), ("final_mps", C.c_void_p),
                ("final_mps_bytes", C.c_size_t), ("z_expect", c_double_p), ("energy", C.c_double), ("expected_energy", C.c_double),
                ("prob", C.c_double), ("max_trunc", C.c_double), ("norm2", C.c_double),
                ("two_site_updates", C.c_longlong), ("status", C.c_int), ("max_sweeps", C.c_int),
                ("max_bond", C.c_int), ("reserved_i", C.c_int), ("device_ms", C.c_double),
                ("min_cut_gap", C.c_double), ("svd_ms", C.c_double), ("svd_bytes", C.c_double),
                ("svd_launches", C.c_longlong), ("svd_sweeps", C.c_longlong), ("kernel_launches", C.c_longlong),
                ("svd_flops", C.c_double), ("precond_ms", C.c_double)]


_lib = None
_lock = threading.Lock()


class SvResult(C.Structure):
    _fields_ = [("spins", c_int8_p), ("sign_spins", c_int8_p), ("entropy", c_double_p), ("state", c_double_p),
                ("energy", C.c_double), ("expected_energy", C.c_double), ("prob", C.c_double),
                ("sign_energy", C.c_double), ("sign_prob", C.c_double), ("norm2", C.c_double),
                ("device_ms", C.c_double), ("reserved", C.c_double * 4)]


def load(path: str = LIB_PATH) -> C.CDLL:
    """Load libtessera_qa.so (building it first if the sources are newer)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(path):
            from . import build as _b
            _b.build()
        if not os.path.exists(path):
            raise RuntimeError(f"libtessera_qa.so not found at {path}; run python -m tessera_b200.build")
        L = C.CDLL(path)
        L.tessera_qa_anneal.argtypes = [c_double_p, C.c_size_t, c_size_p, c_size_p, c_double_p, C.c_size_t,
                                        c_double_p, c_double_p, C.c_size_t, C.c_size_t, c_int8_p, c_double_p]
        L.tessera_qa_anneal.restype = C.c_double
        L.tessera_qa_config_init.argtypes = [C.POINTER(Config)]
        L.tessera_qa_config_init.restype = None
        L.tessera_qa_anneal_ex.argtypes = [C.POINTER(Problem), C.POINTER(Config), C.POINTER(Result)]
        L.tessera_qa_anneal_ex.restype = C.c_int
        L.tessera_qa_anneal_batch.argtypes = [C.POINTER(Problem), C.POINTER(Config), C.POINTER(Result), C.c_size_t]
        L.tessera_qa_anneal_batch.restype = C.c_int
        L.tessera_qa_checkpoint_bytes.argtypes = [C.c_size_t, C.c_size_t]
        L.tessera_qa_checkpoint_bytes.restype = C.c_size_t
        L.tessera_qa_svd.argtypes = [c_double_p, C.c_size_t, C.c_size_t, c_double_p, c_double_p, c_double_p]
        L.tessera_qa_svd.restype = C.c_int
        L.tessera_qa_svd_noalloc.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, C.c_void_p, C.c_void_p,
                                             C.c_void_p]
        L.tessera_qa_svd_noalloc.restype = C.c_int
        L.tessera_qa_last_error.argtypes = [C.c_char_p, C.c_size_t]
        L.tessera_qa_last_error.restype = C.c_int
        L.tessera_qa_sa_solve.argtypes = [C.POINTER(Problem), C.c_size_t, C.c_size_t, C.c_size_t, C.c_double,
                                          C.c_double, C.c_uint64, c_int8_p, c_double_p]
        L.tessera_qa_sa_solve.restype = C.c_int
        L.tessera_qa_debug_fail_allocations.argtypes = [C.c_int, C.c_int]
        L.tessera_qa_debug_fail_allocations.restype = C.c_int
        L.tessera_qa_session_create.argtypes = [C.POINTER(Problem), C.POINTER(Config)]
        L.tessera_qa_session_create.restype = C.c_void_p
        L.tessera_qa_session_create_batch.argtypes = [C.POINTER(Problem), C.POINTER(Config), C.c_size_t]
        L.tessera_qa_session_create_batch.restype = C.c_void_p
        L.tessera_qa_session_run_gates.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, C.c_size_t]
        L.tessera_qa_session_run_gates.restype = C.c_int
        L.tessera_qa_session_run_host.argtypes = [C.c_void_p, C.POINTER(Problem), C.c_size_t, C.c_size_t, C.c_size_t,
                                                  C.c_size_t, C.POINTER(Result)]
        L.tessera_qa_session_run_host.restype = C.c_int
        L.tessera_qa_session_randomize.argtypes = [C.c_void_p, C.c_uint64]
        L.tessera_qa_session_randomize.restype = C.c_int
        L.tessera_qa_session_randomize_graded.argtypes = [C.c_void_p, C.c_uint64, C.c_double]
        L.tessera_qa_session_randomize_graded.restype = C.c_int
        L.tessera_qa_session_run.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t]
        L.tessera_qa_session_run.restype = C.c_int
        L.tessera_qa_session_stream.argtypes = [C.c_void_p]
        L.tessera_qa_session_stream.restype = C.c_void_p
        L.tessera_qa_session_sync.argtypes = [C.c_void_p, C.POINTER(Result)]
        L.tessera_qa_session_sync.restype = C.c_int
        L.tessera_qa_session_observe.argtypes = [C.c_void_p, C.POINTER(Result)]
        L.tessera_qa_session_observe.restype = C.c_int
        L.tessera_qa_session_save.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
        L.tessera_qa_session_save.restype = C.c_int
        L.tessera_qa_session_load.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
        L.tessera_qa_session_load.restype = C.c_int
        L.tessera_qa_session_save_instance.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t]
        L.tessera_qa_session_save_instance.restype = C.c_int
        L.tessera_qa_session_sample.argtypes = [C.c_void_p, C.c_size_t, C.c_uint64, c_int8_p, c_double_p]
        L.tessera_qa_session_sample.restype = C.c_int
        L.tessera_qa_sv_anneal.argtypes = [C.POINTER(Problem), C.c_double, C.c_int, C.POINTER(SvResult)]
        L.tessera_qa_sv_anneal.restype = C.c_int
        L.tessera_qa_session_destroy.argtypes = [C.c_void_p]
        L.tessera_qa_session_destroy.restype = None
        _lib = L
        return L


def last_error() -> str:
    L = load()
    buf = C.create_string_buffer(1024)
    L.tessera_qa_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


class EngineError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"tessera_qa error {code}: {msg}")
        self.code = code
