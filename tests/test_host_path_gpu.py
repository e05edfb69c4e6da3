"""rocblas_b200_dtrsm_mixed_host: the precision form with A and B in host memory.

The pipelined path (side left, recursive sizes) runs left-looking over steps of rows as their
block rows of op(A) and rows of B arrive, so it groups the sliced updates differently from the
device entry point rocblas_b200_dtrsm_mixed; it must meet the same error bound against the
oracle and stay within the precision form's accuracy of the device result, for every side-left
uplo/trans/diag combination (forward and backward solve orders, block rows copied as rows or
columns of A) and for step sizes below, at and above the chain solve's limit.  Side right
and small orders take the copy-then-solve path and match the device entry point bitwise.  The
unused triangle of A is NaN in host memory and must not reach X.
"""
import ctypes
import itertools

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle  # noqa: E402
import rocblas_b200 as rb  # noqa: E402
from rocblas_b200 import devmem as dm  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def handle():
    rb.build()
    h = rb.Handle()
    yield h
    h.close()


def _pinned(arr):
    """A pinned host copy of a Fortran-ordered array, as (tensor, column-major numpy view)."""
    t = torch.from_numpy(np.ascontiguousarray(arr.T)).pin_memory()
    return t, t.numpy().T


def _run_host(h, side, uplo, trans, diag, m, n, alpha, A, B, slices=7):
    tA, _ = _pinned(A)
    tB, vB = _pinned(B)
    a = ctypes.c_double(alpha)
    st = rb.lib().rocblas_b200_dtrsm_mixed_host(h.value, rb.SIDE[side], rb.UPLO[uplo], rb.TRANS[trans],
                                                rb.DIAG[diag], m, n, ctypes.byref(a),
                                                ctypes.c_void_p(tA.data_ptr()), A.shape[0],
                                                ctypes.c_void_p(tB.data_ptr()), B.shape[0], slices)
    assert st == 0, st
    return np.array(vB)


def _run_device(h, side, uplo, trans, diag, m, n, alpha, A, B, slices=7):
    dA, dB = dm.to_device(A), dm.to_device(B)
    a = ctypes.c_double(alpha)
    st = rb.lib().rocblas_b200_dtrsm_mixed(h.value, rb.SIDE[side], rb.UPLO[uplo], rb.TRANS[trans],
                                           rb.DIAG[diag], m, n, ctypes.byref(a),
                                           ctypes.c_void_p(dA.data_ptr()), A.shape[0],
                                           ctypes.c_void_p(dB.data_ptr()), B.shape[0], slices)
    assert st == 0, st
    torch.cuda.synchronize()
    return dm.to_host(dB)


@pytest.mark.parametrize("uplo,trans,diag", list(itertools.product("UL", "NT", "NU")))
def test_host_path_matches_device_side_left(handle, uplo, trans, diag):
    m, n = 4700, 96  # 37 blocks of 128: diagonal solves of 16 blocks and a ragged last one
    A, B = oracle.nan_triangle_problem(71, "L", uplo, trans, diag, m, n, m + 3, m + 1, np.float64)
    got = _run_host(handle, "L", uplo, trans, diag, m, n, -0.75, A, B)
    ref = _run_device(handle, "L", uplo, trans, diag, m, n, -0.75, A, B)
    assert np.isnan(got[m:]).all()  # the padding rows of B are not written
    X = oracle.trsm("L", uplo, trans, diag, -0.75, A, np.asfortranarray(B[:m]))
    err = oracle.matrix_norm_1(X, np.asfortranarray(got[:m]))
    assert err <= oracle.trsm_tolerance(np.float64, m)
    assert err <= 1e-12
    assert oracle.normwise_forward_error(got[:m], ref[:m]) <= 1e-12


@pytest.mark.parametrize("step", [1, 3, "above_chain"])
def test_host_path_step_sizes(handle, step):
    """One step per 128-row block, a ragged step size, and steps of more blocks than the chain
    solve takes (each step's diagonal solve then recurses with a sliced update of its own)."""
    if step == "above_chain":
        mcb = ctypes.c_int()
        assert rb.lib().rocblas_b200_get_tuning(b"mixed_chain_blocks", ctypes.byref(mcb)) == 0
        step = max(mcb.value, 1) + 4
    L = rb.lib()
    old = ctypes.c_int()
    assert L.rocblas_b200_get_tuning(b"host_step_blocks", ctypes.byref(old)) == 0
    assert L.rocblas_b200_set_tuning(b"host_step_blocks", step) == 0
    try:
        m, n = 4700, 70
        for uplo, trans in (("L", "N"), ("L", "T")):
            A, B = oracle.nan_triangle_problem(73, "L", uplo, trans, "N", m, n, m, m + 5, np.float64)
            got = _run_host(handle, "L", uplo, trans, "N", m, n, 2.0, A, B)
            assert np.isnan(got[m:]).all()
            X = oracle.trsm("L", uplo, trans, "N", 2.0, A, np.asfortranarray(B[:m]))
            assert oracle.matrix_norm_1(X, np.asfortranarray(got[:m])) <= 1e-12
    finally:
        L.rocblas_b200_set_tuning(b"host_step_blocks", old.value)
    assert L.rocblas_b200_set_tuning(b"host_step_blocks", 0) == rb.status_invalid_value


@pytest.mark.parametrize("side,m,n", [("R", 90, 1300), ("L", 300, 40)])
def test_host_path_copy_then_solve(handle, side, m, n):
    A, B = oracle.nan_triangle_problem(72, side, "U", "T", "N", m, n, (m if side == "L" else n) + 2, m, np.float64)
    got = _run_host(handle, side, "U", "T", "N", m, n, 1.5, A, B)
    ref = _run_device(handle, side, "U", "T", "N", m, n, 1.5, A, B)
    assert np.array_equal(got, ref)


def test_host_path_alpha_zero_and_arguments(handle):
    A = np.full((50, 50), np.nan, order="F")
    B = np.full((50, 4), 3.0, order="F")
    assert np.all(_run_host(handle, "L", "L", "N", "N", 50, 4, 0.0, A, B) == 0.0)
    L = rb.lib()
    a = ctypes.c_double(1.0)
    x = ctypes.c_void_p(0x1000)
    f = L.rocblas_b200_dtrsm_mixed_host
    assert f(None, 141, 122, 111, 131, 8, 8, ctypes.byref(a), x, 8, x, 8, 7) == rb.status_invalid_handle
    assert f(handle.value, 141, 122, 111, 131, 8, 8, ctypes.byref(a), x, 7, x, 8, 7) == rb.status_invalid_size
    assert f(handle.value, 141, 122, 111, 131, 8, 8, ctypes.byref(a), x, 8, x, 8, 9) == rb.status_invalid_value
