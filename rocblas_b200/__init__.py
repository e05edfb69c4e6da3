"""rocblas_b200 -- B200-native level-3 triangular solve behind the rocBLAS C ABI.

The product is ``librocblas_b200.so`` (C++ host layer + sm_100a CUDA kernels, sources in
``csrc/``, interface in ``include/rocblas.h``).  This module is the Python side of that
boundary: it builds the library, loads it with ctypes, and mirrors the reference's C entry
points under the same names and argument meaning (``rocblas_dtrsm(handle, side, uplo,
transA, diag, m, n, alpha, A, lda, B, ldb)`` with device addresses as integers), so that
tests read like the reference's own client code.

There is no fallback: if the shared library is missing or no CUDA device is present, calls
fail with an exception or a non-success rocblas_status.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB_PATH = os.path.join(HERE, "librocblas_b200.so")
HEADER = os.path.join(REPO, "include", "rocblas.h")
EXT_HEADER = os.path.join(REPO, "include", "rocblas_b200_ext.h")
HEADERS = [HEADER, EXT_HEADER]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "-shared",
]
SOURCES = ["rocblas_api.cu"]

# ---- enums (include/rocblas.h; library/include/internal/rocblas-types.h:123-234) ---------
operation_none, operation_transpose, operation_conjugate_transpose = 111, 112, 113
fill_upper, fill_lower, fill_full = 121, 122, 123
diagonal_non_unit, diagonal_unit = 131, 132
side_left, side_right, side_both = 141, 142, 143
datatype_f32_r, datatype_f64_r, datatype_f32_c, datatype_f64_c = 151, 152, 154, 155
pointer_mode_host, pointer_mode_device = 0, 1

STATUS = {
    0: "success", 1: "invalid_handle", 2: "not_implemented", 3: "invalid_pointer",
    4: "invalid_size", 5: "memory_error", 6: "internal_error", 7: "perf_degraded",
    8: "size_query_mismatch", 9: "size_increased", 10: "size_unchanged", 11: "invalid_value",
    12: "continue", 13: "check_numerics_fail", 14: "excluded_from_build", 15: "arch_mismatch",
}
status_success = 0
status_invalid_handle = 1
status_not_implemented = 2
status_invalid_pointer = 3
status_invalid_size = 4
status_memory_error = 5
status_internal_error = 6
status_perf_degraded = 7
status_size_query_mismatch = 8
status_size_increased = 9
status_size_unchanged = 10
status_invalid_value = 11
status_check_numerics_fail = 13
atomics_not_allowed, atomics_allowed = 0, 1

SIDE = {"L": side_left, "R": side_right}
UPLO = {"U": fill_upper, "L": fill_lower}
TRANS = {"N": operation_none, "T": operation_transpose, "C": operation_conjugate_transpose}
DIAG = {"N": diagonal_non_unit, "U": diagonal_unit}


class RocblasError(RuntimeError):
    def __init__(self, fn, status):
        super().__init__(f"{fn} returned rocblas_status_{STATUS.get(status, status)} ({status})")
        self.status = status


def _sources():
    out = []
    for f in os.listdir(CSRC):
        if f.endswith((".cu", ".cuh", ".hpp", ".h", ".cpp")):
            out.append(os.path.join(CSRC, f))
    out.extend(HEADERS)
    return out


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile librocblas_b200.so in-tree with nvcc for sm_100a."""
    newest = max(os.path.getmtime(f) for f in _sources())
    if not force and os.path.exists(LIB_PATH) and os.path.getmtime(LIB_PATH) >= newest:
        return LIB_PATH
    cmd = ["nvcc", *NVCC_FLAGS, "-o", LIB_PATH, *[os.path.join(CSRC, s) for s in SOURCES]]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd, cwd=CSRC)
    return LIB_PATH


# ---- ctypes binding -----------------------------------------------------------------------
_i, _i64, _p, _sz = ctypes.c_int, ctypes.c_int64, ctypes.c_void_p, ctypes.c_size_t
_H = ctypes.c_void_p

# name -> (restype, argtypes); mirrors include/rocblas.h
_TRSM = [_H, _i, _i, _i, _i, _i, _i, _p, _p, _i, _p, _i]
_TRSM_B = _TRSM + [_i]
_TRSM_SB = [_H, _i, _i, _i, _i, _i, _i, _p, _p, _i, _i64, _p, _i, _i64, _i]
# trmm: handle, side, uplo, trans, diag, m, n, alpha, A, lda, B, ldb, C, ldc (+ batch / strides)
_TRMM = [_H, _i, _i, _i, _i, _i, _i, _p, _p, _i, _p, _i, _p, _i]
_TRMM_B = _TRMM + [_i]
_TRMM_SB = [_H, _i, _i, _i, _i, _i, _i, _p, _p, _i, _i64, _p, _i, _i64, _p, _i, _i64, _i]
# the ILP64 (_64) forms: every size, leading dimension, increment and batch count 64-bit
_L = _i64
_TRSM_64 = [_H, _i, _i, _i, _i, _L, _L, _p, _p, _L, _p, _L]
_TRSM_B_64 = _TRSM_64 + [_L]
_TRSM_SB_64 = [_H, _i, _i, _i, _i, _L, _L, _p, _p, _L, _i64, _p, _L, _i64, _L]
_TRMM_64 = [_H, _i, _i, _i, _i, _L, _L, _p, _p, _L, _p, _L, _p, _L]
_TRMM_B_64 = _TRMM_64 + [_L]
_TRMM_SB_64 = [_H, _i, _i, _i, _i, _L, _L, _p, _p, _L, _i64, _p, _L, _i64, _p, _L, _i64, _L]
_TRSV_64 = [_H, _i, _i, _i, _L, _p, _L, _p, _L]
_TRSV_B_64 = _TRSV_64 + [_L]
_TRSV_SB_64 = [_H, _i, _i, _i, _L, _p, _L, _i64, _p, _L, _i64, _L]
_TRTRI = [_H, _i, _i, _i, _p, _i, _p, _i]
_TRTRI_B = _TRTRI + [_i]
_TRTRI_SB = [_H, _i, _i, _i, _p, _i, _i64, _p, _i, _i64, _i]
SIGNATURES = {
    "rocblas_create_handle": (_i, [ctypes.POINTER(_H)]),
    "rocblas_destroy_handle": (_i, [_H]),
    "rocblas_set_stream": (_i, [_H, _p]),
    "rocblas_get_stream": (_i, [_H, ctypes.POINTER(_p)]),
    "rocblas_set_pointer_mode": (_i, [_H, _i]),
    "rocblas_get_pointer_mode": (_i, [_H, ctypes.POINTER(_i)]),
    "rocblas_set_atomics_mode": (_i, [_H, _i]),
    "rocblas_set_math_mode": (_i, [_H, _i]),
    "rocblas_get_math_mode": (_i, [_H, ctypes.POINTER(_i)]),
    "rocblas_set_performance_metric": (_i, [_H, _i]),
    "rocblas_get_performance_metric": (_i, [_H, ctypes.POINTER(_i)]),
    "rocblas_set_solution_fitness_query": (_i, [_H, ctypes.POINTER(ctypes.c_double)]),
    "rocblas_get_atomics_mode": (_i, [_H, ctypes.POINTER(_i)]),
    "rocblas_pointer_to_mode": (_i, [_p]),
    "rocblas_set_vector": (_i, [_i, _i, _p, _i, _p, _i]),
    "rocblas_set_vector_async": (_i, [_i, _i, _p, _i, _p, _i, _p]),
    "rocblas_set_matrix": (_i, [_i, _i, _i, _p, _i, _p, _i]),
    "rocblas_set_matrix_async": (_i, [_i, _i, _i, _p, _i, _p, _i, _p]),
    "rocblas_get_vector": (_i, [_i, _i, _p, _i, _p, _i]),
    "rocblas_get_vector_async": (_i, [_i, _i, _p, _i, _p, _i, _p]),
    "rocblas_get_matrix": (_i, [_i, _i, _i, _p, _i, _p, _i]),
    "rocblas_get_matrix_async": (_i, [_i, _i, _i, _p, _i, _p, _i, _p]),
    "rocblas_set_vector_64": (_i, [_i64, _i64, _p, _i64, _p, _i64]),
    "rocblas_set_vector_async_64": (_i, [_i64, _i64, _p, _i64, _p, _i64, _p]),
    "rocblas_set_matrix_64": (_i, [_i64, _i64, _i64, _p, _i64, _p, _i64]),
    "rocblas_set_matrix_async_64": (_i, [_i64, _i64, _i64, _p, _i64, _p, _i64, _p]),
    "rocblas_get_vector_64": (_i, [_i64, _i64, _p, _i64, _p, _i64]),
    "rocblas_get_vector_async_64": (_i, [_i64, _i64, _p, _i64, _p, _i64, _p]),
    "rocblas_get_matrix_64": (_i, [_i64, _i64, _i64, _p, _i64, _p, _i64]),
    "rocblas_get_matrix_async_64": (_i, [_i64, _i64, _i64, _p, _i64, _p, _i64, _p]),
    "rocblas_start_device_memory_size_query": (_i, [_H]),
    "rocblas_stop_device_memory_size_query": (_i, [_H, ctypes.POINTER(_sz)]),
    "rocblas_is_device_memory_size_query": (ctypes.c_bool, [_H]),
    "rocblas_get_device_memory_size": (_i, [_H, ctypes.POINTER(_sz)]),
    "rocblas_set_device_memory_size": (_i, [_H, _sz]),
    "rocblas_set_workspace": (_i, [_H, _p, _sz]),
    "rocblas_is_managing_device_memory": (ctypes.c_bool, [_H]),
    "rocblas_is_user_managing_device_memory": (ctypes.c_bool, [_H]),
    "rocblas_strsv": (_i, [_H, _i, _i, _i, _i, _p, _i, _p, _i]),
    "rocblas_dtrsv": (_i, [_H, _i, _i, _i, _i, _p, _i, _p, _i]),
    "rocblas_strsv_batched": (_i, [_H, _i, _i, _i, _i, _p, _i, _p, _i, _i]),
    "rocblas_dtrsv_batched": (_i, [_H, _i, _i, _i, _i, _p, _i, _p, _i, _i]),
    "rocblas_strsv_strided_batched": (_i, [_H, _i, _i, _i, _i, _p, _i, _i64, _p, _i, _i64, _i]),
    "rocblas_dtrsv_strided_batched": (_i, [_H, _i, _i, _i, _i, _p, _i, _i64, _p, _i, _i64, _i]),
    "rocblas_strmm": (_i, _TRMM),
    "rocblas_dtrmm": (_i, _TRMM),
    "rocblas_strmm_batched": (_i, _TRMM_B),
    "rocblas_dtrmm_batched": (_i, _TRMM_B),
    "rocblas_strmm_strided_batched": (_i, _TRMM_SB),
    "rocblas_dtrmm_strided_batched": (_i, _TRMM_SB),
    "rocblas_strsm": (_i, _TRSM),
    "rocblas_dtrsm": (_i, _TRSM),
    "rocblas_strsm_batched": (_i, _TRSM_B),
    "rocblas_dtrsm_batched": (_i, _TRSM_B),
    "rocblas_strsm_strided_batched": (_i, _TRSM_SB),
    "rocblas_dtrsm_strided_batched": (_i, _TRSM_SB),
    "rocblas_trsm_ex": (_i, [_H, _i, _i, _i, _i, _i, _i, _p, _p, _i, _p, _i, _p, _i, _i]),
    "rocblas_trsm_batched_ex": (_i, [_H, _i, _i, _i, _i, _i, _i, _p, _p, _i, _p, _i, _i, _p, _i, _i]),
    "rocblas_trsm_strided_batched_ex": (
        _i, [_H, _i, _i, _i, _i, _i, _i, _p, _p, _i, _i64, _p, _i, _i64, _i, _p, _i, _i64, _i]),
    **{f"rocblas_{t}{name}": (_i, sig) for t in "cz" for name, sig in (
        ("trsm", _TRSM), ("trsm_batched", _TRSM_B), ("trsm_strided_batched", _TRSM_SB),
        ("trmm", _TRMM), ("trmm_batched", _TRMM_B), ("trmm_strided_batched", _TRMM_SB),
        ("trsv", [_H, _i, _i, _i, _i, _p, _i, _p, _i]),
        ("trsv_batched", [_H, _i, _i, _i, _i, _p, _i, _p, _i, _i]),
        ("trsv_strided_batched", [_H, _i, _i, _i, _i, _p, _i, _i64, _p, _i, _i64, _i]))},
    **{f"rocblas_{t}{name}_64": (_i, sig) for t in "sdcz" for name, sig in (
        ("trsm", _TRSM_64), ("trsm_batched", _TRSM_B_64), ("trsm_strided_batched", _TRSM_SB_64),
        ("trmm", _TRMM_64), ("trmm_batched", _TRMM_B_64), ("trmm_strided_batched", _TRMM_SB_64),
        ("trsv", _TRSV_64), ("trsv_batched", _TRSV_B_64), ("trsv_strided_batched", _TRSV_SB_64))},
    **{f"rocblas_{t}{name}": (_i, sig) for t in "cz" for name, sig in (
        ("trtri", _TRTRI), ("trtri_batched", _TRTRI_B), ("trtri_strided_batched", _TRTRI_SB))},
    "rocblas_strtri": (_i, _TRTRI),
    "rocblas_dtrtri": (_i, _TRTRI),
    "rocblas_strtri_batched": (_i, _TRTRI_B),
    "rocblas_dtrtri_batched": (_i, _TRTRI_B),
    "rocblas_strtri_strided_batched": (_i, _TRTRI_SB),
    "rocblas_dtrtri_strided_batched": (_i, _TRTRI_SB),
    # include/rocblas_b200_ext.h
    "rocblas_b200_kernel_launch_count": (ctypes.c_uint64, []),
    "rocblas_b200_dtrsm_vbatched": (_i, [_H, _p, _p, _i, _i, _p]),
    "rocblas_b200_strsm_vbatched": (_i, [_H, _p, _p, _i, _i, _p]),
    "rocblas_b200_dtrsm_vbatched_noalloc": (_i, [_H, _p, _p, _i, _i, _p]),
    "rocblas_b200_dtrsm_vbatched_ex": (_i, [_H, _p, _p, _p, _i, _i, _i, _p]),
    "rocblas_b200_strsm_vbatched_ex": (_i, [_H, _p, _p, _p, _i, _i, _i, _p]),
    "rocblas_b200_dgemm_sliced": (_i, [_H, _i, _i, _i, _i, _i, _p, _p, _i, _p, _i, _p, _p, _i, _i]),
    "rocblas_b200_dgemm_crt": (_i, [_H, _i, _i, _i, _i, _i, _p, _p, _i, _p, _i, _p, _p, _i, _i]),
    "rocblas_b200_dtrsm_mixed": (_i, [_H, _i, _i, _i, _i, _i, _i, _p, _p, _i, _p, _i, _i]),
    "rocblas_b200_dtrsm_mixed_host": (_i, [_H, _i, _i, _i, _i, _i, _i, _p, _p, _i, _p, _i, _i]),
    "rocblas_b200_dtrsm_refined": (_i, [_H, _i, _i, _i, _i, _i, _i, _p, _p, _i, _p, _i, _p, _p]),
    "rocblas_b200_dgemm": (_i, [_H, _i, _i, _i, _i, _i, _p, _p, _i, _p, _i, _p, _p, _i]),
    "rocblas_b200_zgemm": (_i, [_H, _i, _i, _i, _i, _i, _p, _p, _i, _p, _i, _p, _p, _i]),
    "rocblas_b200_cgemm": (_i, [_H, _i, _i, _i, _i, _i, _p, _p, _i, _p, _i, _p, _p, _i]),
    "rocblas_b200_get_device_error": (_i, [_H, ctypes.POINTER(_i)]),
    "rocblas_b200_server_create": (_i, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_size_t, _i,
                                        ctypes.c_double, _i]),
    "rocblas_b200_server_destroy": (_i, [_p]),
    "rocblas_b200_server_add_resident": (_i, [_p, _i, _i, _p, _i, ctypes.POINTER(_i)]),
    "rocblas_b200_server_set_budget": (_i, [_p, ctypes.c_size_t]),
    "rocblas_b200_server_used_bytes": (_i, [_p, ctypes.POINTER(ctypes.c_size_t)]),
    "rocblas_b200_server_run": (_i, [_p, _p, _i, _p, _p]),
    "rocblas_b200_kernel_timing_enable": (_i, [_i]),
    "rocblas_b200_kernel_timing_query": (_i, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_double),
                                              ctypes.POINTER(ctypes.c_double), ctypes.POINTER(_i)]),
    "rocblas_b200_set_tuning": (_i, [ctypes.c_char_p, _i]),
    "rocblas_b200_get_tuning": (_i, [ctypes.c_char_p, ctypes.POINTER(_i)]),
}

class RefineOptions(ctypes.Structure):
    """rocblas_b200_refine_options (include/rocblas_b200_ext.h)."""
    _fields_ = [("slices", _i), ("max_iterations", _i), ("check_columns", _i), ("fallback", _i),
                ("tolerance", ctypes.c_double)]


class RefineInfo(ctypes.Structure):
    """rocblas_b200_refine_info (include/rocblas_b200_ext.h)."""
    _fields_ = [("iterations", _i), ("converged", _i), ("fell_back", _i), ("checked_columns", _i),
                ("error_estimate_first", ctypes.c_double), ("error_estimate", ctypes.c_double),
                ("tolerance", ctypes.c_double)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


_lib = None


def lib() -> ctypes.CDLL:
    """Load librocblas_b200.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run rocblas_b200.build() (needs nvcc)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def __getattr__(name):
    # rocblas_* names resolve to the bound C functions
    if name.startswith("rocblas_") and name in SIGNATURES:
        return getattr(lib(), name)
    raise AttributeError(name)


def check(fn_name, status, allow=(status_success,)):
    if status not in allow:
        raise RocblasError(fn_name, status)
    return status


class Handle:
    """RAII wrapper of rocblas_handle."""

    def __init__(self, stream=None):
        self.h = _H()
        check("rocblas_create_handle", lib().rocblas_create_handle(ctypes.byref(self.h)))
        if stream is not None:
            check("rocblas_set_stream", lib().rocblas_set_stream(self.h, stream))

    @property
    def value(self):
        return self.h

    def set_pointer_mode(self, mode):
        check("rocblas_set_pointer_mode", lib().rocblas_set_pointer_mode(self.h, mode))

    def set_stream(self, stream):
        check("rocblas_set_stream", lib().rocblas_set_stream(self.h, stream))

    def close(self):
        if self.h:
            lib().rocblas_destroy_handle(self.h)
            self.h = _H()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
