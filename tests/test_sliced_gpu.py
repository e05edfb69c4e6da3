"""Integer-slice tensor-core FP64 GEMM (tcgen05 kind::i8) and the precision form of dtrsm.

* exactness: integer inputs that fit one 7-bit slice give bit-exact integer products;
* accuracy: S slices carry 7S bits relative to each row's (column's) largest entry: 7 slices
  give ~1e-13 of |A||B| on Gaussian data, 8 slices ~1e-16; the error falls by ~2^-7 per slice;
* the precision form of the trsm meets the rocblas-test gate (40 eps max(M,N)) for all 16
  combinations and matches the float128 oracle on condition-band problems.
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
COMBOS = list(itertools.product("LR", "UL", "NT", "NU"))


def _dptr(x):
    c = ctypes.c_double(x)
    return c, ctypes.cast(ctypes.byref(c), ctypes.c_void_p)


def sliced_gemm(h, ta, tb, A, B, C, alpha, beta, slices):
    """A, B, C Fortran-ordered numpy; returns the new C."""
    m, n = C.shape
    k = A.shape[1] if ta == "N" else A.shape[0]
    dA, dB, dC = dm.to_device(A), dm.to_device(B), dm.to_device(C)
    ka, pa = _dptr(alpha)
    kb, pb = _dptr(beta)
    st = rb.lib().rocblas_b200_dgemm_sliced(h.value, rb.TRANS[ta], rb.TRANS[tb], m, n, k, pa,
                                            ctypes.c_void_p(dA.data_ptr()), A.shape[0],
                                            ctypes.c_void_p(dB.data_ptr()), B.shape[0], pb,
                                            ctypes.c_void_p(dC.data_ptr()), C.shape[0], slices)
    assert st == 0, st
    torch.cuda.synchronize()
    code = ctypes.c_int(-1)
    assert rb.lib().rocblas_b200_get_device_error(h.value, ctypes.byref(code)) == 0
    assert code.value == 0
    return dm.to_host(dC)


@pytest.fixture(scope="module")
def handle():
    rb.build()
    h = rb.Handle()
    yield h
    h.close()


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "N"), ("N", "T"), ("T", "T")])
def test_sliced_gemm_integer_exact(handle, ta, tb):
    rng = np.random.default_rng(1)
    m, n, k = 200, 130, 1000
    Ai = rng.integers(-127, 128, size=(m, k))
    Bi = rng.integers(-127, 128, size=(k, n))
    Ai[:, 0] = 127  # every row / column reaches the 7-bit range: one slice is exact
    Bi[0, :] = -127
    A = np.asfortranarray((Ai if ta == "N" else Ai.T).astype(np.float64))
    B = np.asfortranarray((Bi if tb == "N" else Bi.T).astype(np.float64))
    C = np.zeros((m, n), order="F")
    got = sliced_gemm(handle, ta, tb, A, B, C, 1.0, 0.0, 1)
    exact = (Ai @ Bi).astype(np.float64)
    assert np.array_equal(got, exact)


@pytest.mark.parametrize("m,n,k", [(128, 64, 64), (300, 200, 777), (1, 1, 1), (129, 65, 5000),
                                   (64, 300, 20000)])
def test_sliced_gemm_fp64_accuracy(handle, m, n, k):
    rng = np.random.default_rng(m + n + k)
    A = np.asfortranarray(rng.standard_normal((m, k)) * np.exp(rng.uniform(-5, 5, size=(m, 1))))
    B = np.asfortranarray(rng.standard_normal((k, n)))
    C = np.asfortranarray(rng.standard_normal((m, n)))
    ref = 0.5 * C.astype(np.longdouble) - A.astype(np.longdouble) @ B.astype(np.longdouble)
    scale = np.abs(A) @ np.abs(B) + 0.5 * np.abs(C)
    for S, tol in ((7, 64 * 2.0 ** -49), (8, 2e-15)):
        got = sliced_gemm(handle, "N", "N", A, B, C, -1.0, 0.5, S)
        err = np.max(np.abs(got - ref.astype(np.float64)) / scale)
        assert err < tol, (S, err)


def test_sliced_gemm_error_per_slice(handle):
    rng = np.random.default_rng(7)
    m, n, k = 256, 128, 512
    A = np.asfortranarray(rng.uniform(-1, 1, (m, k)))
    B = np.asfortranarray(rng.uniform(-1, 1, (k, n)))
    ref = (A.astype(np.longdouble) @ B.astype(np.longdouble)).astype(np.float64)
    scale = np.abs(A) @ np.abs(B)
    errs = []
    for S in range(1, 9):
        got = sliced_gemm(handle, "N", "N", A, B, np.zeros((m, n), order="F"), 1.0, 0.0, S)
        errs.append(np.max(np.abs(got - ref) / scale))
    for S in range(1, 7):
        assert errs[S] < errs[S - 1] * 2.0 ** -4, errs  # about 2^-7 per slice
    assert errs[7] < 1e-15, errs


def _mixed(h, side, uplo, trans, diag, m, n, alpha, A, B, slices=7):
    dA, dB = dm.to_device(A), dm.to_device(B)
    ka, pa = _dptr(alpha)
    st = rb.lib().rocblas_b200_dtrsm_mixed(h.value, rb.SIDE[side], rb.UPLO[uplo], rb.TRANS[trans],
                                           rb.DIAG[diag], m, n, pa, ctypes.c_void_p(dA.data_ptr()),
                                           A.shape[0], ctypes.c_void_p(dB.data_ptr()), B.shape[0], slices)
    assert st == 0, st
    torch.cuda.synchronize()
    return dm.to_host(dB)


@pytest.mark.parametrize("side,uplo,trans,diag", COMBOS)
def test_mixed_trsm_all_combos(handle, side, uplo, trans, diag):
    m, n = (700, 300) if side == "L" else (300, 700)
    k = m if side == "L" else n
    A, B = oracle.nan_triangle_problem(31, side, uplo, trans, diag, m, n, k + 3, m + 1, np.float64)
    out = _mixed(handle, side, uplo, trans, diag, m, n, -0.75, A, B)
    X = oracle.trsm(side, uplo, trans, diag, -0.75, A, np.asfortranarray(B[:m]))
    err = oracle.matrix_norm_1(X, out[:m])
    assert err <= oracle.trsm_tolerance(np.float64, max(m, n)), err
    assert np.isnan(out[m:]).all()


@pytest.mark.parametrize("kband", [0, 2, 4, 6])
def test_mixed_trsm_condition_bands(handle, kband):
    """Normwise forward error against the float128 oracle, the precision form next to the
    plain FP64 form (both must be at the FP64 oracle's own level)."""
    m, n = 1536, 24
    A, B = oracle.condition_band_problem(kband, m, n, kband)
    Xq = oracle.trsm("L", "L", "N", "N", 1.0, A, B, precision="q")
    Xd = oracle.trsm("L", "L", "N", "N", 1.0, A, B, precision="d")
    e_ref = oracle.normwise_forward_error(Xd, Xq)
    mixed = _mixed(handle, "L", "L", "N", "N", m, n, 1.0, A, B)
    e_mixed = oracle.normwise_forward_error(mixed, Xq)
    dA, dB = dm.to_device(A), dm.to_device(B)
    dm.trsm(handle, "L", "L", "N", "N", m, n, 1.0, dA, m, dB, m)
    torch.cuda.synchronize()
    e_plain = oracle.normwise_forward_error(dm.to_host(dB), Xq)
    assert e_mixed <= max(1e-12, 10 * e_ref), (e_mixed, e_ref, e_plain)
    assert e_plain <= max(1e-12, 10 * e_ref), (e_plain, e_ref)


@pytest.mark.parametrize("chain_blocks", [0, 4])
def test_mixed_trsm_chain_bottom(handle, chain_blocks):
    """The precision form with its bottom levels on the chain solve (mixed_chain_blocks > 0)
    and with recursion down to the leaves (0): both at the FP64 oracle's level."""
    L = rb.lib()
    old = ctypes.c_int(-1)
    assert L.rocblas_b200_get_tuning(b"mixed_chain_blocks", ctypes.byref(old)) == 0
    assert L.rocblas_b200_set_tuning(b"mixed_chain_blocks", chain_blocks) == 0
    try:
        for side, uplo, trans, diag in [("L", "L", "N", "N"), ("R", "U", "T", "U"), ("L", "U", "N", "N")]:
            m, n = (2100, 40) if side == "L" else (40, 2100)
            k = m if side == "L" else n
            A, B = oracle.nan_triangle_problem(91, side, uplo, trans, diag, m, n, k, m, np.float64)
            out = _mixed(handle, side, uplo, trans, diag, m, n, -1.25, A, B)
            X = oracle.trsm(side, uplo, trans, diag, -1.25, A, np.asfortranarray(B[:m]))
            err = oracle.matrix_norm_1(X, out[:m])
            assert err <= oracle.trsm_tolerance(np.float64, max(m, n)), (side, uplo, trans, diag, err)
        code = ctypes.c_int(-1)
        assert L.rocblas_b200_get_device_error(handle.value, ctypes.byref(code)) == 0
        assert code.value == 0
    finally:
        L.rocblas_b200_set_tuning(b"mixed_chain_blocks", old.value)
