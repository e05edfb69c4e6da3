"""rocblas_?trmm (C := alpha op(A) B or alpha B op(A), A triangular) against the oracle's
restatement of the reference BLAS xTRMM (the forward operator of rocblas-test's trsm check):
all 16 side/uplo/trans/diag combinations, out of place and in place, alpha 0 on the host and
on the device, the strided batch, and the argument rules of rocblas_trmm_arg_check
(library/src/blas3/rocblas_trmm.hpp:51-105)."""
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
DT = {"d": np.float64, "s": np.float32}


def _tol(npdt, k):
    eps = np.finfo(npdt).eps
    return 4 * eps * max(k, 1)


def _check(side, uplo, trans, diag, alpha, A, B, out, npdt, m, n):
    ref = oracle.trmm(side, uplo, trans, diag, alpha, A, np.asfortranarray(B[:m, :n]))
    scale = np.abs(oracle.trmm(side, uplo, trans, diag, abs(alpha), np.abs(np.nan_to_num(A)),
                               np.abs(np.asfortranarray(B[:m, :n])))) + 1e-300
    err = np.max(np.abs(out[:m, :n] - ref) / scale)
    assert not np.isnan(out[:m, :n]).any()
    assert err <= _tol(npdt, m if side == "L" else n), (side, uplo, trans, diag, m, n, err)


@pytest.fixture(scope="module")
def handle():
    rb.build()
    h = rb.Handle()
    yield h
    h.close()


@pytest.mark.parametrize("dt", ["d", "s"])
@pytest.mark.parametrize("side,uplo,trans,diag", COMBOS)
def test_trmm_all_combos(handle, dt, side, uplo, trans, diag):
    npdt = DT[dt]
    for i, (m, n) in enumerate([(37, 29), (300, 140), (140, 300), (1, 5)]):
        k = m if side == "L" else n
        A, B = oracle.nan_triangle_problem(600 + i, side, uplo, trans, diag, m, n, k + 1, m + 2, npdt)
        alpha = [1.0, -0.75, 2.5, 0.5][i]
        dA, dB = dm.to_device(A), dm.to_device(B)
        C = np.full((m + 3, n), np.nan, dtype=npdt, order="F")
        dC = dm.to_device(C)
        dm.trmm(handle, side, uplo, trans, diag, m, n, alpha, dA, A.shape[0], dB, B.shape[0], dC, C.shape[0])
        torch.cuda.synchronize()
        out = dm.to_host(dC)
        _check(side, uplo, trans, diag, alpha, A, B, out, npdt, m, n)
        assert np.isnan(out[m:]).all()  # rows past m are not written
        # B is not modified out of place
        assert np.array_equal(dm.to_host(dB), B, equal_nan=True)
        # in place: C == B, ldc == ldb
        dm.trmm(handle, side, uplo, trans, diag, m, n, alpha, dA, A.shape[0], dB, B.shape[0], dB, B.shape[0])
        torch.cuda.synchronize()
        _check(side, uplo, trans, diag, alpha, A, B, dm.to_host(dB), npdt, m, n)


@pytest.mark.parametrize("on_device", [False, True])
def test_trmm_alpha_zero(handle, on_device):
    """alpha == 0: C := 0 without reading A or B (both all NaN here)."""
    m, n = 70, 40
    A = np.full((m, m), np.nan, order="F")
    B = np.full((m, n), np.nan, order="F")
    dA, dB = dm.to_device(A), dm.to_device(B)
    dC = dm.to_device(np.full((m, n), 5.0, order="F"))
    dm.trmm(handle, "L", "U", "T", "N", m, n, 0.0, dA, m, dB, m, dC, m, alpha_on_device=on_device)
    torch.cuda.synchronize()
    assert np.all(dm.to_host(dC) == 0.0)


def test_trmm_strided_batched(handle):
    batch, m, n = 5, 96, 33
    for side, uplo, trans, diag in [("L", "L", "N", "U"), ("R", "U", "T", "N")]:
        k = m if side == "L" else n
        lda, ldb, ldc = k, m + 1, m + 2
        sa, sb, sc = lda * k + 3, ldb * n + 1, ldc * n + 5
        probs = [oracle.nan_triangle_problem(700 + b, side, uplo, trans, diag, m, n, lda, ldb, np.float64)
                 for b in range(batch)]
        dA = torch.full((batch * sa,), float("nan"), dtype=torch.float64, device="cuda")
        dB = torch.full((batch * sb,), float("nan"), dtype=torch.float64, device="cuda")
        dC = torch.full((batch * sc,), float("nan"), dtype=torch.float64, device="cuda")
        for b, (A, B) in enumerate(probs):
            dA[b * sa: b * sa + lda * k] = torch.from_numpy(A.ravel(order="F")).cuda()
            dB[b * sb: b * sb + ldb * n] = torch.from_numpy(B.ravel(order="F")).cuda()
        dm.trmm_strided_batched(handle, side, uplo, trans, diag, m, n, 1.5, dA, lda, sa, dB, ldb, sb,
                                dC, ldc, sc, batch)
        torch.cuda.synchronize()
        hC = dC.cpu().numpy()
        for b, (A, B) in enumerate(probs):
            out = hC[b * sc: b * sc + ldc * n].reshape((ldc, n), order="F")
            _check(side, uplo, trans, diag, 1.5, A, B, out, np.float64, m, n)


def test_trmm_arguments(handle):
    L = rb.lib()
    one = ctypes.c_double(1.0)
    p = ctypes.cast(ctypes.byref(one), ctypes.c_void_p)
    x = torch.zeros(64 * 64, dtype=torch.float64, device="cuda")
    y = torch.zeros(64 * 64, dtype=torch.float64, device="cuda")
    X, Y = ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr())
    f = L.rocblas_dtrmm
    assert f(None, 141, 122, 111, 131, 8, 8, p, X, 8, X, 8, Y, 8) == rb.status_invalid_handle
    assert f(handle.value, 140, 122, 111, 131, 8, 8, p, X, 8, X, 8, Y, 8) == rb.status_invalid_value
    assert f(handle.value, 141, 122, 111, 131, 8, 8, p, X, 7, X, 8, Y, 8) == rb.status_invalid_size
    assert f(handle.value, 141, 122, 111, 131, 8, 8, p, X, 8, X, 8, Y, 7) == rb.status_invalid_size
    assert f(handle.value, 141, 122, 111, 131, 0, 8, None, None, 8, None, 8, None, 8) == rb.status_success
    assert f(handle.value, 141, 122, 111, 131, 8, 8, p, None, 8, X, 8, Y, 8) == rb.status_invalid_pointer
    # in place needs ldb == ldc
    assert f(handle.value, 141, 122, 111, 131, 8, 8, p, X, 8, Y, 8, Y, 9) == rb.status_invalid_value
