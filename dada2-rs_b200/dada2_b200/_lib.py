"""ctypes binding of libdada2_b200.so (the C ABI in include/dada2_b200.h).

The library is loaded from this package directory. There is no CPU fallback:
every entry point runs on the GPU and raises if the library or a device is
missing.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libdada2_b200.so")
_lib = None

DGPU_OK, DGPU_E_INVALID, DGPU_E_CUDA, DGPU_E_DEVICE, DGPU_E_UNSUPPORTED, DGPU_E_NOMEM = 0, -1, -2, -3, -4, -5
_CODE_NAMES = {-1: "invalid input", -2: "CUDA error", -3: "device error", -4: "unsupported", -5: "out of memory"}


class DgpuError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{_CODE_NAMES.get(code, code)}: {msg}")
        self.code = code


class InvalidInput(DgpuError, ValueError):
    pass


class AlignParamsC(C.Structure):
    _fields_ = [
        ("match_score", C.c_int32), ("mismatch", C.c_int32), ("gap_p", C.c_int32),
        ("homo_gap_p", C.c_int32), ("use_kmers", C.c_int32), ("kdist_cutoff", C.c_double),
        ("kmer_size", C.c_int32), ("band", C.c_int32), ("vectorized", C.c_int32),
        ("gapless", C.c_int32),
    ]


class DadaParamsC(C.Structure):
    _fields_ = [
        ("align", AlignParamsC), ("omega_a", C.c_double), ("omega_p", C.c_double),
        ("omega_c", C.c_double), ("detect_singletons", C.c_int32), ("max_clust", C.c_int32),
        ("min_fold", C.c_double), ("min_hamming", C.c_uint32), ("min_abund", C.c_uint32),
        ("use_quals", C.c_int32), ("greedy", C.c_int32), ("host_threads", C.c_int32),
        ("transitions", C.c_int32), ("lambda_fp32", C.c_int32),
    ]


class KernelStatsC(C.Structure):
    _fields_ = [("launches", C.c_uint64 * 4), ("ms", C.c_double * 4), ("rounds", C.c_uint64),
                ("compares", C.c_uint64), ("screened", C.c_uint64), ("screen_bytes", C.c_uint64),
                ("timed_rounds", C.c_uint64), ("timed_screen_bytes", C.c_uint64), ("timed_compares", C.c_uint64),
                ("h2d_bytes", C.c_uint64), ("batch_ms", C.c_double * 3), ("prepare_ms", C.c_double * 4)]


class TuningC(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("launch_slots", "samples_per_launch", "dedicated_slots",
                                         "align_ctas_per_sm", "screen_chunk_max", "screen_blocks_per_sm",
                                         "pivot_min_items", "programmatic_launch")]


class ErrFunC(C.Structure):
    _fields_ = [("kind", C.c_int32), ("surface", C.c_int32), ("cell", C.c_double),
                ("max_error_rate", C.c_double), ("min_error_rate", C.c_double), ("pseudocount", C.c_double),
                ("bins", C.c_void_p), ("nbins", C.c_int32), ("cmd", C.c_char_p)]


class CountersC(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("screened", "aligned", "shrouded", "stored", "gapless",
                                          "vectorized", "homo", "endsfree")]


_P = C.c_void_p


class DadaOutC(C.Structure):
    _fields_ = [(n, _P) for n in (
        "cl_reads", "cl_birth_type", "cl_birth_from", "cl_birth_pval", "cl_birth_fold",
        "cl_birth_e", "cl_birth_hamming", "cl_seq_off", "cl_seq", "cl_mem_off", "mem_raw",
        "mem_hamming", "mem_lambda", "mem_pval", "map", "pvals", "counters", "times")]


# dgpu_allgather_fn: (user, send, bytes, recv) -> 0 or nonzero
ALLGATHER_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python dada2-rs_b200/build.py`")
        L = C.CDLL(LIB_PATH)
        L.dgpu_last_error.restype = C.c_char_p
        L.dgpu_device_count.argtypes = [C.POINTER(C.c_int)]
        L.dgpu_ctx_create.argtypes = [C.c_int, C.POINTER(AlignParamsC), _P, C.c_int, C.c_int, C.POINTER(_P)]
        L.dgpu_ctx_destroy.argtypes = [_P]
        L.dgpu_ctx_destroy.restype = None
        L.dgpu_upload_raws.argtypes = [_P, C.c_int, _P, _P, _P, _P, _P]
        L.dgpu_set_locks.argtypes = [_P, _P]
        L.dgpu_reset_e_minmax.argtypes = [_P]
        L.dgpu_get_e_minmax.argtypes = [_P, _P]
        L.dgpu_compare.argtypes = [_P, C.c_int, C.c_double, C.c_int, _P, _P, _P, C.POINTER(CountersC)]
        L.dgpu_compare_store.argtypes = [_P, C.c_int, C.c_int, C.c_double, C.c_int, _P, _P, _P,
                                         C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(CountersC)]
        L.dgpu_dada.argtypes = [C.c_int, C.POINTER(DadaParamsC), C.c_int, _P, _P, _P, _P, _P, _P, _P,
                                C.c_int, C.POINTER(_P)]
        L.dgpu_dada_batch.argtypes = [C.c_int, C.POINTER(DadaParamsC), C.c_int, _P, _P, _P, _P, _P, _P,
                                      _P, _P, C.c_int, _P]
        L.dgpu_dada_sharded.argtypes = [C.c_int, C.POINTER(DadaParamsC), C.c_int, _P, _P, _P, _P, _P, _P, _P,
                                        C.c_int, C.c_int, C.c_int, ALLGATHER_FN, _P, C.POINTER(_P)]
        L.dgpu_result_sizes.argtypes = [_P, _P]
        L.dgpu_result_fill.argtypes = [_P, C.POINTER(DadaOutC)]
        L.dgpu_result_transitions.argtypes = [_P, _P]
        L.dgpu_result_fp32_stats.argtypes = [_P, _P]
        L.dgpu_result_margins.argtypes = [_P, _P]
        L.dgpu_errfun_apply.argtypes = [C.POINTER(ErrFunC), _P, C.c_int, _P]
        L.dgpu_learn_errors.argtypes = [C.c_int, C.POINTER(DadaParamsC), C.POINTER(ErrFunC), C.c_int, C.c_int, _P, _P,
                                        _P, _P, _P, _P, C.POINTER(_P)]
        L.dgpu_learn_read.argtypes = [_P, _P, _P, _P, _P]
        L.dgpu_learn_free.argtypes = [_P]
        L.dgpu_learn_free.restype = None
        L.dgpu_tuning_get.argtypes = [C.c_int, C.POINTER(TuningC)]
        L.dgpu_tuning_set.argtypes = [C.c_int, C.POINTER(TuningC)]
        L.dgpu_tuning_load.argtypes = [C.c_char_p]
        L.dgpu_tuning_save.argtypes = [C.c_char_p]
        L.dgpu_tuning_reset.argtypes = []
        L.dgpu_get_methods.argtypes = [_P, _P]
        L.dgpu_service_create.argtypes = [C.c_int, C.POINTER(DadaParamsC), _P, C.c_int, C.c_uint64, _P]
        L.dgpu_service_submit.argtypes = [_P, C.c_int, _P, _P, _P, _P, _P, _P, _P]
        L.dgpu_service_wait.argtypes = [_P, C.c_uint64, _P, _P]
        L.dgpu_service_stats.argtypes = [_P, _P, _P]
        L.dgpu_derep_fastq.argtypes = [C.c_char_p, C.c_int, C.c_int, _P]
        L.dgpu_derep_sizes.argtypes = [_P, _P]
        L.dgpu_derep_fill.argtypes = [_P, _P, _P, _P, _P, _P, _P]
        L.dgpu_derep_free.argtypes = [_P]
        L.dgpu_derep_free.restype = None
        L.dgpu_service_hold.argtypes = [_P, C.c_int]
        L.dgpu_service_destroy.argtypes = [_P]
        L.dgpu_service_destroy.restype = None
        L.dgpu_ctx_set_lambda32.argtypes = [_P, C.c_int]
        L.dgpu_get_loglambda32.argtypes = [_P, _P]
        L.dgpu_calc_pA.argtypes = [C.c_uint32, C.c_double, C.c_int]
        L.dgpu_calc_pA.restype = C.c_double
        L.dgpu_result_transitions.restype = C.c_int
        L.dgpu_result_free.argtypes = [_P]
        L.dgpu_result_free.restype = None
        L.dgpu_batch_prepare.argtypes = [C.c_int, C.POINTER(DadaParamsC), C.c_int, _P, _P, _P, _P, _P, _P,
                                         _P, _P, C.c_int, C.POINTER(_P)]
        L.dgpu_batch_run.argtypes = [_P, _P]
        L.dgpu_batch_free.argtypes = [_P]
        L.dgpu_batch_free.restype = None
        L.dgpu_stats_reset.argtypes = []
        L.dgpu_stats_timing.argtypes = [C.c_int]
        L.dgpu_cache_release.argtypes = [C.c_int, C.POINTER(C.c_uint64)]
        L.dgpu_stats_read.argtypes = [C.POINTER(KernelStatsC)]
        L.dgpu_stats_latencies.argtypes = [_P, C.c_int]
        L.dgpu_align_debug.argtypes = [C.c_int, C.c_int, C.c_int, _P, _P, _P, _P, _P, _P,
                                       C.POINTER(AlignParamsC), C.c_int, _P, _P, _P, _P]
        _lib = L
    return _lib


def check(rc: int):
    if rc != 0:
        msg = lib().dgpu_last_error().decode(errors="replace")
        if rc == DGPU_E_INVALID:
            raise InvalidInput(rc, msg)
        raise DgpuError(rc, msg)


def ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def device_count() -> int:
    n = C.c_int(0)
    rc = lib().dgpu_device_count(C.byref(n))
    return n.value if rc == 0 else 0
