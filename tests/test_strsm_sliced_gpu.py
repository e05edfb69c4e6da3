"""FP32 trsm with its trailing updates on the int8 slice engine (tuning key strsm_slices,
default 4): every update with an inner dimension of at least strsm_sliced_min_k is an exact
product of 7-bit slices of the FP32 operands (4 slices keep 28 bits of every entry relative to
its row's or column's largest, more than FP32's 24), combined in FP64 and rounded once to FP32.

* all 16 combinations against the oracle at the rocblas-test gate (40 eps max(m, n)), and
  against the same solve on the FFMA tiles (strsm_slices 0);
* host and device pointer mode alpha, alpha == 0 in device mode;
* the slice panels are part of the size query.
"""
import contextlib
import ctypes
import itertools

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle  # noqa: E402
import rocblas_b200 as rb  # noqa: E402
from rocblas_b200 import devmem as dm  # noqa: E402

pytestmark = pytest.mark.gpu
COMBOS = list(itertools.product("LR", "UL", "NT", "NU"))


@contextlib.contextmanager
def tuning(**keys):
    L = rb.lib()
    old = {}
    for k, v in keys.items():
        o = ctypes.c_int(-1)
        assert L.rocblas_b200_get_tuning(k.encode(), ctypes.byref(o)) == 0
        old[k] = o.value
        assert L.rocblas_b200_set_tuning(k.encode(), v) == 0
    try:
        yield
    finally:
        for k, v in old.items():
            L.rocblas_b200_set_tuning(k.encode(), v)


SLICED = dict(strsm_slices=4, strsm_sliced_min_k=256)


@pytest.fixture(scope="module")
def handle():
    rb.build()
    h = rb.Handle()
    yield h
    h.close()


def _solve(h, side, uplo, trans, diag, m, n, alpha, A, B, alpha_on_device=False):
    dA, dB = dm.to_device(A), dm.to_device(B)
    dm.trsm(h, side, uplo, trans, diag, m, n, alpha, dA, A.shape[0], dB, B.shape[0],
            alpha_on_device=alpha_on_device)
    torch.cuda.synchronize()
    code = ctypes.c_int(-1)
    assert rb.lib().rocblas_b200_get_device_error(h.value, ctypes.byref(code)) == 0
    assert code.value == 0
    return dm.to_host(dB)


@pytest.mark.parametrize("side,uplo,trans,diag", COMBOS)
def test_strsm_sliced_all_combos(handle, side, uplo, trans, diag):
    m, n = (1500, 700) if side == "L" else (700, 1500)
    k = m if side == "L" else n
    A, B = oracle.nan_triangle_problem(53, side, uplo, trans, diag, m, n, k + 1, m + 2, np.float32)
    with tuning(**SLICED):
        out = _solve(handle, side, uplo, trans, diag, m, n, -0.5, A, B)
    X = oracle.trsm(side, uplo, trans, diag, -0.5, A, np.asfortranarray(B[:m]))
    err = oracle.matrix_norm_1(X, out[:m])
    assert err <= oracle.trsm_tolerance(np.float32, max(m, n)), err
    assert np.isnan(out[m:]).all()
    with tuning(strsm_slices=0):
        ffma = _solve(handle, side, uplo, trans, diag, m, n, -0.5, A, B)
    assert oracle.matrix_norm_1(ffma[:m], out[:m]) <= oracle.trsm_tolerance(np.float32, max(m, n))


@pytest.mark.parametrize("alpha", [2.0, 0.0])
def test_strsm_sliced_device_alpha(handle, alpha):
    m, n = 1100, 640
    A, B = oracle.nan_triangle_problem(8, "L", "L", "N", "N", m, n, m, m, np.float32)
    with tuning(**SLICED):
        out = _solve(handle, "L", "L", "N", "N", m, n, alpha, A, B, alpha_on_device=True)
    if alpha == 0.0:
        assert np.array_equal(out, np.zeros_like(out))
        return
    X = oracle.trsm("L", "L", "N", "N", alpha, A, B)
    assert oracle.matrix_norm_1(X, out) <= oracle.trsm_tolerance(np.float32, max(m, n))


def _query_size(m, n):
    with rb.Handle() as h:
        L = rb.lib()
        assert L.rocblas_start_device_memory_size_query(h.value) == 0
        one = ctypes.c_float(1.0)
        st = L.rocblas_strsm(h.value, rb.side_left, rb.fill_lower, rb.operation_none, rb.diagonal_non_unit,
                             m, n, ctypes.cast(ctypes.byref(one), ctypes.c_void_p), None, m, None, m)
        assert st == rb.status_size_increased, st
        size = ctypes.c_size_t(0)
        assert L.rocblas_stop_device_memory_size_query(h.value, ctypes.byref(size)) == 0
        return size.value


def test_strsm_sliced_workspace_query(handle):
    """The slice panels are part of the size query (invA alone without them); with a fixed
    workspace of the queried size the sliced solve runs and passes."""
    m, n = 2048, 1024
    with tuning(**SLICED):
        size_on = _query_size(m, n)
    with tuning(strsm_slices=0):
        size_off = _query_size(m, n)
    assert size_off == 128 * m * 4, size_off
    # slices of the top update: 4 x (1024 + 1024) x 1024 int8 plus exponents
    assert size_on >= size_off + 4 * 2048 * 1024, (size_on, size_off)
    A, B = oracle.nan_triangle_problem(9, "L", "L", "N", "N", m, n, m, m, np.float32)
    with tuning(**SLICED), rb.Handle() as h:
        assert rb.lib().rocblas_set_device_memory_size(h.value, size_on) == 0
        out = _solve(h, "L", "L", "N", "N", m, n, 1.0, A, B)
    X = oracle.trsm("L", "L", "N", "N", 1.0, A, B)
    assert oracle.matrix_norm_1(X, out) <= oracle.trsm_tolerance(np.float32, max(m, n))
