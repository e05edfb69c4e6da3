"""The C ABI boundary on CPU: the library builds, loads, exports every symbol that
include/rocblas.h declares, and applies the reference's argument checks and
device-memory protocol without touching a GPU (clients/include/blas3/testing_trsm.hpp:
33-186 is the bad-argument spec)."""
import ctypes
import re
import subprocess
import sys

import pytest

import rocblas_b200 as rb


def _declared_symbols():
    src = "".join(open(h).read() for h in rb.HEADERS)
    return sorted(set(re.findall(r"ROCBLAS_EXPORT\s+[\w ]+?\s+(rocblas_\w+)\s*\(", src)))


def test_header_symbols_exported(rocblas_lib):
    declared = _declared_symbols()
    assert len(declared) >= 30
    out = subprocess.check_output(["nm", "-D", "--defined-only", rb.LIB_PATH], text=True)
    exported = set(re.findall(r"\bT (rocblas_\w+)", out))
    missing = [s for s in declared if s not in exported]
    assert not missing, missing
    # and nothing else leaks out of the C ABI
    assert exported == set(declared), sorted(exported - set(declared))
    for s in declared:
        assert s in rb.SIGNATURES, s


@pytest.mark.parametrize("header", rb.HEADERS)
def test_header_compiles_as_c(header):
    cmd = ["gcc", "-fsyntax-only", "-x", "c", "-std=c99", "-I/usr/local/cuda/include", header]
    subprocess.check_call(cmd)


@pytest.fixture()
def handle(rocblas_lib):
    h = rb.Handle()
    yield h
    h.close()


def _trsm(h, side=rb.side_left, uplo=rb.fill_lower, trans=rb.operation_none,
          diag=rb.diagonal_non_unit, m=10, n=10, alpha=1.0, A=1, lda=10, B=1, ldb=10, fn="d"):
    L = rb.lib()
    ap = None
    if alpha is not None:
        a = ctypes.c_double(alpha) if fn == "d" else ctypes.c_float(alpha)
        ap = ctypes.cast(ctypes.byref(a), ctypes.c_void_p)
    f = L.rocblas_dtrsm if fn == "d" else L.rocblas_strsm
    hv = h.value if h is not None else None
    return f(hv, side, uplo, trans, diag, m, n, ap, A, lda, B, ldb)


def test_trsm_bad_args(handle):
    """testing_trsm_bad_arg (clients/include/blas3/testing_trsm.hpp:33-186)."""
    assert _trsm(None) == rb.status_invalid_handle
    assert _trsm(handle, side=rb.side_both) == rb.status_invalid_value
    assert _trsm(handle, uplo=rb.fill_full) == rb.status_invalid_value
    assert _trsm(handle, trans=99) == rb.status_invalid_value
    assert _trsm(handle, diag=99) == rb.status_invalid_value
    assert _trsm(handle, m=-1) == rb.status_invalid_size
    assert _trsm(handle, n=-1) == rb.status_invalid_size
    assert _trsm(handle, lda=9) == rb.status_invalid_size  # lda < k = m (side left)
    assert _trsm(handle, side=rb.side_right, m=10, n=12, lda=11, ldb=10) == rb.status_invalid_size
    assert _trsm(handle, ldb=9) == rb.status_invalid_size
    # quick returns before any pointer is looked at
    assert _trsm(handle, m=0, A=None, B=None, alpha=None) == rb.status_success
    assert _trsm(handle, n=0, A=None, B=None, alpha=None) == rb.status_success
    # null pointers
    assert _trsm(handle, alpha=None) == rb.status_invalid_pointer
    assert _trsm(handle, B=None) == rb.status_invalid_pointer
    assert _trsm(handle, A=None) == rb.status_invalid_pointer
    # device pointer mode: A is not checked (alpha is not readable on the host)
    handle.set_pointer_mode(rb.pointer_mode_device)
    assert _trsm(handle, A=None, B=None) == rb.status_invalid_pointer
    handle.set_pointer_mode(rb.pointer_mode_host)
    for fn in "sd":
        assert _trsm(handle, m=-1, fn=fn) == rb.status_invalid_size


def test_trsm_ex_type_switch(handle):
    L = rb.lib()
    a = ctypes.c_double(1.0)
    ap = ctypes.cast(ctypes.byref(a), ctypes.c_void_p)
    args = [rb.side_left, rb.fill_lower, rb.operation_none, rb.diagonal_non_unit, 4, 4, ap, 1, 4, 1, 4,
            None, 0]
    assert L.rocblas_trsm_ex(handle.value, *args, 168) == rb.status_not_implemented  # bf16
    assert L.rocblas_trsm_ex(None, *args, rb.datatype_f64_c) == rb.status_invalid_handle
    bad = list(args)
    bad[4] = -1
    # real and complex compute types run the same argument rules
    for dt in (rb.datatype_f64_r, rb.datatype_f32_r, rb.datatype_f64_c, rb.datatype_f32_c):
        assert L.rocblas_trsm_ex(handle.value, *bad, dt) == rb.status_invalid_size


def test_batched_bad_args(handle):
    L = rb.lib()
    a = ctypes.c_float(1.0)
    ap = ctypes.cast(ctypes.byref(a), ctypes.c_void_p)
    st = L.rocblas_strsm_strided_batched(handle.value, rb.side_left, rb.fill_lower, rb.operation_none,
                                         rb.diagonal_non_unit, 4, 4, ap, 1, 4, 16, 1, 4, 16, -1)
    assert st == rb.status_invalid_size
    st = L.rocblas_strsm_strided_batched(handle.value, rb.side_left, rb.fill_lower, rb.operation_none,
                                         rb.diagonal_non_unit, 4, 4, ap, None, 4, 16, None, 4, 16, 0)
    assert st == rb.status_success
    st = L.rocblas_dtrsm_batched(handle.value, rb.side_right, rb.fill_lower, rb.operation_none,
                                 rb.diagonal_non_unit, 4, 4, ap, 1, 4, None, 4, 3)
    assert st == rb.status_invalid_pointer


def test_trtri_bad_args(handle):
    L = rb.lib()
    assert L.rocblas_dtrtri(None, rb.fill_lower, rb.diagonal_unit, 4, 1, 4, 1, 4) == rb.status_invalid_handle
    assert L.rocblas_dtrtri(handle.value, rb.fill_full, rb.diagonal_unit, 4, 1, 4, 1, 4) == rb.status_invalid_value
    assert L.rocblas_dtrtri(handle.value, rb.fill_lower, 7, 4, 1, 4, 1, 4) == rb.status_invalid_value
    assert L.rocblas_dtrtri(handle.value, rb.fill_lower, rb.diagonal_unit, 4, 1, 3, 1, 4) == rb.status_invalid_size
    assert L.rocblas_dtrtri(handle.value, rb.fill_lower, rb.diagonal_unit, 4, 1, 4, 1, 3) == rb.status_invalid_size
    assert L.rocblas_dtrtri(handle.value, rb.fill_lower, rb.diagonal_unit, 0, None, 4, None, 4) == rb.status_success
    assert L.rocblas_dtrtri(handle.value, rb.fill_lower, rb.diagonal_unit, 4, None, 4, 1, 4) == rb.status_invalid_pointer


def test_math_mode_metric_and_fitness(handle):
    """rocblas_auxiliary.cpp:126-178 and handle.cpp: the math mode (xf32 not supported here:
    ignored, success), the performance metric, and the fitness query set to the lowest double."""
    L = rb.lib()
    v = ctypes.c_int(-1)
    assert L.rocblas_get_math_mode(handle.value, ctypes.byref(v)) == 0 and v.value == 0
    assert L.rocblas_set_math_mode(handle.value, 1) == 0
    assert L.rocblas_get_math_mode(handle.value, ctypes.byref(v)) == 0 and v.value == 0
    assert L.rocblas_set_math_mode(None, 0) == rb.status_invalid_handle
    assert L.rocblas_get_math_mode(handle.value, None) == rb.status_invalid_pointer
    assert L.rocblas_get_performance_metric(handle.value, ctypes.byref(v)) == 0 and v.value == 0
    assert L.rocblas_set_performance_metric(handle.value, 2) == 0
    assert L.rocblas_get_performance_metric(handle.value, ctypes.byref(v)) == 0 and v.value == 2
    assert L.rocblas_get_performance_metric(handle.value, None) == rb.status_invalid_pointer
    f = ctypes.c_double(1.0)
    assert L.rocblas_set_solution_fitness_query(handle.value, ctypes.byref(f)) == 0
    assert f.value == -sys.float_info.max
    assert L.rocblas_set_solution_fitness_query(handle.value, None) == 0


def test_copy_helpers_argument_rules(rocblas_lib):
    """rocblas_{set,get}_{vector,matrix}[_async][_64] argument rules (rocblas_auxiliary.cpp:
    305-790): quick return first, then sizes, then pointers; nothing here touches a device."""
    L = rb.lib()
    p = ctypes.c_void_p(0x1000)
    for suf in ("", "_64"):
        for d in ("set", "get"):
            vec = getattr(L, f"rocblas_{d}_vector{suf}")
            veca = getattr(L, f"rocblas_{d}_vector_async{suf}")
            mat = getattr(L, f"rocblas_{d}_matrix{suf}")
            mata = getattr(L, f"rocblas_{d}_matrix_async{suf}")
            assert vec(0, 8, None, 1, None, 1) == rb.status_success
            assert veca(0, 8, None, 1, None, 1, None) == rb.status_success
            assert vec(-1, 8, p, 1, p, 1) == rb.status_invalid_size
            assert vec(4, 0, p, 1, p, 1) == rb.status_invalid_size
            assert vec(4, 8, p, 0, p, 1) == rb.status_invalid_size
            assert veca(4, 8, p, 1, p, -1, None) == rb.status_invalid_size
            assert vec(4, 8, None, 1, p, 1) == rb.status_invalid_pointer
            assert veca(4, 8, p, 1, None, 1, None) == rb.status_invalid_pointer
            assert mat(0, 5, 8, None, 1, None, 1) == rb.status_success
            assert mat(5, 0, 8, None, 1, None, 1) == rb.status_success
            assert mat(-1, 5, 8, p, 5, p, 5) == rb.status_invalid_size
            assert mat(6, 5, 8, p, 5, p, 6) == rb.status_invalid_size  # rows > lda
            assert mat(6, 5, 8, p, 6, p, 5) == rb.status_invalid_size  # rows > ldb
            assert mata(6, 5, 0, p, 6, p, 6, None) == rb.status_invalid_size
            assert mata(6, 5, 8, p, 6, None, 6, None) == rb.status_invalid_pointer


def test_atomics_mode(handle):
    """rocblas_set/get_atomics_mode (rocblas_auxiliary.cpp:87-117): allowed by default."""
    L = rb.lib()
    mode = ctypes.c_int(-1)
    assert L.rocblas_get_atomics_mode(handle.value, ctypes.byref(mode)) == 0
    assert mode.value == rb.atomics_allowed
    assert L.rocblas_set_atomics_mode(handle.value, rb.atomics_not_allowed) == 0
    assert L.rocblas_get_atomics_mode(handle.value, ctypes.byref(mode)) == 0
    assert mode.value == rb.atomics_not_allowed
    assert L.rocblas_set_atomics_mode(None, rb.atomics_allowed) == rb.status_invalid_handle
    assert L.rocblas_get_atomics_mode(handle.value, None) == rb.status_invalid_pointer


def test_handle_state(handle):
    L = rb.lib()
    mode = ctypes.c_int(-1)
    assert L.rocblas_get_pointer_mode(handle.value, ctypes.byref(mode)) == 0 and mode.value == 0
    assert L.rocblas_set_pointer_mode(handle.value, 1) == 0
    assert L.rocblas_get_pointer_mode(handle.value, ctypes.byref(mode)) == 0 and mode.value == 1
    assert L.rocblas_set_pointer_mode(handle.value, 5) == rb.status_invalid_value
    s = ctypes.c_void_p(1)
    assert L.rocblas_get_stream(handle.value, ctypes.byref(s)) == 0 and not s.value
    assert L.rocblas_set_stream(handle.value, 12345) == 0
    assert L.rocblas_get_stream(handle.value, ctypes.byref(s)) == 0 and s.value == 12345
    assert L.rocblas_set_stream(handle.value, None) == 0
    assert L.rocblas_get_stream(None, ctypes.byref(s)) == rb.status_invalid_handle


def test_device_memory_size_query(handle):
    """The query protocol of rocblas-test (testing_trsm.hpp:327-340; handle.cpp:449-484)."""
    L = rb.lib()
    size = ctypes.c_size_t(123)
    assert L.rocblas_stop_device_memory_size_query(handle.value, ctypes.byref(size)) == rb.status_size_query_mismatch
    assert L.rocblas_start_device_memory_size_query(handle.value) == 0
    assert L.rocblas_is_device_memory_size_query(handle.value)
    assert L.rocblas_start_device_memory_size_query(handle.value) == rb.status_size_query_mismatch
    # small problem: no workspace
    assert _trsm(handle, m=64, n=64, lda=64, ldb=64, A=None, B=None, alpha=None) == rb.status_size_unchanged
    # large problem: invA for 128 * k elements, then the chain solve's flags (one int per
    # 128-row block and 64-column strip) and its counter
    st = _trsm(handle, m=4096, n=4096, lda=4096, ldb=4096, A=None, B=None, alpha=None)
    assert st == rb.status_size_increased
    st = _trsm(handle, m=2048, n=4096, lda=4096, ldb=4096, A=None, B=None, alpha=None)
    assert st == rb.status_size_unchanged
    assert L.rocblas_stop_device_memory_size_query(handle.value, ctypes.byref(size)) == 0
    want = 128 * 4096 * 8 + (4096 // 128) * (4096 // 64) * 4 + 16
    assert size.value == (want + 63) // 64 * 64  # the handle rounds sizes up to 64 bytes
    assert not L.rocblas_is_device_memory_size_query(handle.value)


def test_workspace_ownership(handle):
    L = rb.lib()
    assert L.rocblas_is_managing_device_memory(handle.value)
    assert L.rocblas_set_workspace(handle.value, 0x1000, 4096) == 0
    assert not L.rocblas_is_managing_device_memory(handle.value)
    size = ctypes.c_size_t(0)
    assert L.rocblas_get_device_memory_size(handle.value, ctypes.byref(size)) == 0 and size.value == 4096
    assert L.rocblas_set_workspace(handle.value, None, 0) == 0
    assert L.rocblas_is_managing_device_memory(handle.value)
    assert not L.rocblas_is_user_managing_device_memory(handle.value)
    assert L.rocblas_set_workspace(None, None, 0) == rb.status_invalid_handle


def test_ilp64_arguments_and_size_query(handle):
    """The _64 forms: the 32-bit argument rules on 64-bit values, invalid_size for an order of A
    beyond 32 bits (src64/blas3/rocblas_trsm_kernels_64.cpp:57-62,
    src64/blas2/rocblas_trsv_kernels_64.cpp:50-51), and a size query over a B whose rows are
    cut into chunks (2^28 rows for side right) equal to the query of one full chunk.  No call
    here reaches the device."""
    L = rb.lib()
    one = ctypes.c_double(1.0)
    p = ctypes.cast(ctypes.byref(one), ctypes.c_void_p)
    big = (1 << 31) + 5
    X, Y = 0x1000, 0x2000  # never dereferenced: every call returns before any device work
    h = handle.value
    lo, nn, nu = rb.fill_lower, rb.operation_none, rb.diagonal_non_unit
    f = L.rocblas_dtrsm_64
    assert f(h, rb.side_left, lo, nn, nu, big, 4, p, X, big, Y, big) == rb.status_invalid_size
    assert f(h, rb.side_right, lo, nn, nu, 4, big, p, X, big, Y, 4) == rb.status_invalid_size
    assert f(h, rb.side_both, lo, nn, nu, big, 4, p, X, big, Y, big) == rb.status_invalid_value
    assert f(h, rb.side_left, lo, nn, nu, 8, big, p, X, 7, Y, 8) == rb.status_invalid_size
    assert f(h, rb.side_left, lo, nn, nu, 8, 0, None, None, 8, None, 8) == rb.status_success
    assert L.rocblas_dtrsm_strided_batched_64(h, rb.side_left, lo, nn, nu, 8, 8, p, X, 8, 64, Y, 8, 64,
                                              -1) == rb.status_invalid_size
    assert L.rocblas_dtrsv_64(h, lo, nn, nu, big, X, big, Y, 1) == rb.status_invalid_size
    assert L.rocblas_dtrsv_64(h, lo, nn, nu, 8, X, 8, Y, 0) == rb.status_invalid_size
    assert L.rocblas_dtrmm_64(h, rb.side_left, lo, nn, nu, big, 4, p, X, big, Y, big, Y + 64,
                              big) == rb.status_invalid_size
    assert L.rocblas_dtrmm_64(h, rb.side_left, lo, nn, nu, 8, 8, p, X, 8, Y, 8, Y, 9) == rb.status_invalid_value

    size64, size32 = ctypes.c_size_t(0), ctypes.c_size_t(0)
    m64 = (1 << 31) + 77  # nine chunks of rows
    assert L.rocblas_start_device_memory_size_query(h) == 0
    assert f(h, rb.side_right, lo, nn, nu, m64, 1024, p, None, 1024, None, m64) == rb.status_size_increased
    assert L.rocblas_stop_device_memory_size_query(h, ctypes.byref(size64)) == 0
    assert L.rocblas_start_device_memory_size_query(h) == 0
    assert L.rocblas_dtrsm(h, rb.side_right, lo, nn, nu, 1 << 28, 1024, p, None, 1024, None,
                           1 << 28) == rb.status_size_increased
    assert L.rocblas_stop_device_memory_size_query(h, ctypes.byref(size32)) == 0
    assert size64.value == size32.value > 0


def test_complex_argument_rules(handle):
    """rocblas_{c,z}trsm / trsv / trmm follow the real argument rules (checked without a device:
    every call below returns before any device work)."""
    L = rb.lib()
    h = handle.value
    z = (ctypes.c_double * 2)(1.0, 0.0)
    zp = ctypes.cast(z, ctypes.c_void_p)
    X, Y = 0x1000, 0x2000
    lo, nn, nu = rb.fill_lower, rb.operation_none, rb.diagonal_non_unit
    for S in "cz":
        trsm = getattr(L, f"rocblas_{S}trsm")
        assert trsm(None, rb.side_left, lo, nn, nu, 8, 8, zp, X, 8, Y, 8) == rb.status_invalid_handle
        assert trsm(h, rb.side_both, lo, nn, nu, 8, 8, zp, X, 8, Y, 8) == rb.status_invalid_value
        assert trsm(h, rb.side_left, lo, rb.operation_conjugate_transpose + 1, nu, 8, 8, zp, X, 8, Y, 8) \
            == rb.status_invalid_value
        assert trsm(h, rb.side_left, lo, nn, nu, 8, 8, zp, X, 7, Y, 8) == rb.status_invalid_size
        assert trsm(h, rb.side_left, lo, nn, nu, 0, 8, None, None, 8, None, 8) == rb.status_success
        assert trsm(h, rb.side_left, lo, nn, nu, 8, 8, None, X, 8, Y, 8) == rb.status_invalid_pointer
        assert getattr(L, f"rocblas_{S}trsm_64")(h, rb.side_left, lo, nn, nu, (1 << 31) + 1, 1, zp, X,
                                                 (1 << 31) + 1, Y, (1 << 31) + 1) == rb.status_invalid_size
        assert getattr(L, f"rocblas_{S}trsv")(h, lo, rb.operation_conjugate_transpose, nu, 8, X, 8, Y, 0) \
            == rb.status_invalid_size
        assert getattr(L, f"rocblas_{S}trmm")(h, rb.side_right, lo, nn, nu, 8, 8, zp, X, 8, Y, 8, Y, 9) \
            == rb.status_invalid_value
