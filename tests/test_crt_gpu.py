"""Residue (Chinese-remainder) tensor-core FP64 GEMM (tcgen05 kind::i8) and the precision form
of dtrsm on it.

* exactness: integer inputs whose products fit FP64 come back bit-exact;
* accuracy: with 16 moduli every entry keeps 55 bits relative to its row's (column's) largest
  entry (K <= 4096 per exponent range), so the product is within ~2^-50 of |A||B|, at the level
  of the 8-slice engine; 15 and 14 moduli keep about 4 and 8 bits less;
* the precision form with its updates on this engine meets the rocblas-test gate for all 16
  combinations and the float128 oracle on the condition bands.
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
from rocblas_b200 import workloads  # noqa: E402

pytestmark = pytest.mark.gpu
COMBOS = list(itertools.product("LR", "UL", "NT", "NU"))


def _dptr(x):
    c = ctypes.c_double(x)
    return c, ctypes.cast(ctypes.byref(c), ctypes.c_void_p)


def crt_gemm(h, ta, tb, A, B, C, alpha, beta, moduli):
    """A, B, C Fortran-ordered numpy; returns the new C."""
    m, n = C.shape
    k = A.shape[1] if ta == "N" else A.shape[0]
    dA, dB, dC = dm.to_device(A), dm.to_device(B), dm.to_device(C)
    ka, pa = _dptr(alpha)
    kb, pb = _dptr(beta)
    st = rb.lib().rocblas_b200_dgemm_crt(h.value, rb.TRANS[ta], rb.TRANS[tb], m, n, k, pa,
                                         ctypes.c_void_p(dA.data_ptr()), A.shape[0],
                                         ctypes.c_void_p(dB.data_ptr()), B.shape[0], pb,
                                         ctypes.c_void_p(dC.data_ptr()), C.shape[0], moduli)
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


@pytest.fixture(params=[0, 1], ids=["cta", "pair"])
def form(request):
    """The one-CTA kernel (128 x 256 tiles) and the CTA-pair kernel (cta_group::2, 256 x 256)."""
    L = rb.lib()
    old = ctypes.c_int(-1)
    assert L.rocblas_b200_get_tuning(b"crt_pair", ctypes.byref(old)) == 0
    assert L.rocblas_b200_set_tuning(b"crt_pair", request.param) == 0
    yield request.param
    L.rocblas_b200_set_tuning(b"crt_pair", old.value)


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "N"), ("N", "T"), ("T", "T")])
def test_crt_gemm_integer_exact(handle, form, ta, tb):
    rng = np.random.default_rng(11)
    m, n, k = 300, 270, 1000
    Ai = rng.integers(-(1 << 15), 1 << 15, size=(m, k))
    Bi = rng.integers(-(1 << 15), 1 << 15, size=(k, n))
    A = np.asfortranarray((Ai if ta == "N" else Ai.T).astype(np.float64))
    B = np.asfortranarray((Bi if tb == "N" else Bi.T).astype(np.float64))
    C = np.full((m, n), np.nan, order="F")  # beta == 0: C is not read
    got = crt_gemm(handle, ta, tb, A, B, C, 1.0, 0.0, 16)
    assert np.array_equal(got, (Ai @ Bi).astype(np.float64))


@pytest.mark.parametrize("m,n,k", [(128, 256, 64), (300, 200, 777), (1, 1, 1), (129, 65, 5000),
                                   (64, 300, 20000), (1000, 513, 4096)])
def test_crt_gemm_fp64_accuracy(handle, form, m, n, k):
    rng = np.random.default_rng(m + n + k)
    A = np.asfortranarray(rng.standard_normal((m, k)) * np.exp(rng.uniform(-5, 5, size=(m, 1))))
    B = np.asfortranarray(rng.standard_normal((k, n)))
    C = np.asfortranarray(rng.standard_normal((m, n)))
    ref = 0.5 * C.astype(np.longdouble) - A.astype(np.longdouble) @ B.astype(np.longdouble)
    scale = np.abs(A) @ np.abs(B) + 0.5 * np.abs(C)
    got = crt_gemm(handle, "N", "N", A, B, C, -1.0, 0.5, 16)
    err = np.max(np.abs(got - ref.astype(np.float64)) / scale)
    assert err < 2e-15, err


def test_crt_gemm_bits_per_modulus(handle, form):
    """Fewer moduli keep fewer bits: 14 < 15 < 16 in accuracy; 16 at the 8-slice level."""
    rng = np.random.default_rng(3)
    m, n, k = 256, 512, 2048
    A = np.asfortranarray(rng.uniform(-1, 1, (m, k)))
    B = np.asfortranarray(rng.uniform(-1, 1, (k, n)))
    ref = (A.astype(np.longdouble) @ B.astype(np.longdouble)).astype(np.float64)
    scale = np.abs(A) @ np.abs(B)
    errs = {}
    for nm in (14, 15, 16):
        got = crt_gemm(handle, "N", "N", A, B, np.zeros((m, n), order="F"), 1.0, 0.0, nm)
        errs[nm] = np.max(np.abs(got - ref) / scale)
    assert errs[16] < 1e-15 and errs[15] < errs[14], errs
    assert errs[14] < 2.0 ** -40, errs


def test_crt_gemm_zero_rows_and_columns(handle, form):
    rng = np.random.default_rng(4)
    m, n, k = 257, 300, 700
    A = np.asfortranarray(rng.standard_normal((m, k)))
    B = np.asfortranarray(rng.standard_normal((k, n)))
    A[5, :] = 0.0
    B[:, 7] = 0.0
    A[9, :] = 1e-300 * rng.standard_normal(k)  # tiny rows take the ldexp path
    C = np.asfortranarray(rng.standard_normal((m, n)))
    got = crt_gemm(handle, "N", "N", A, B, C, 2.0, -1.0, 16)
    ref = (2.0 * (A.astype(np.longdouble) @ B.astype(np.longdouble)) - C).astype(np.float64)
    scale = 2.0 * (np.abs(A) @ np.abs(B)) + np.abs(C)
    assert np.max(np.abs(got - ref) / scale) < 2e-15
    assert np.array_equal(got[5, :], -C[5, :]) and np.array_equal(got[:, 7], -C[:, 7])


def test_crt_gemm_rejects_unsupported_moduli(handle):
    A = np.zeros((4, 4), order="F")
    dA = dm.to_device(A)
    ka, pa = _dptr(1.0)
    p = ctypes.c_void_p(dA.data_ptr())
    for nm in (1, 13, 17, -1):
        st = rb.lib().rocblas_b200_dgemm_crt(handle.value, rb.TRANS["N"], rb.TRANS["N"], 4, 4, 4, pa,
                                             p, 4, p, 4, pa, p, 4, nm)
        assert st == rb.status_invalid_value, (nm, st)


@contextlib.contextmanager
def _moduli(nm):
    """Route the precision form's updates through the residue engine, down to short updates
    (sliced_min_k 128) and chain solves of at most two 128-row blocks, for one test."""
    L = rb.lib()
    keys = dict(mixed_moduli=nm, sliced_min_k=128, mixed_chain_blocks=2)
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


def _mixed(h, side, uplo, trans, diag, m, n, alpha, A, B):
    dA, dB = dm.to_device(A), dm.to_device(B)
    ka, pa = _dptr(alpha)
    st = rb.lib().rocblas_b200_dtrsm_mixed(h.value, rb.SIDE[side], rb.UPLO[uplo], rb.TRANS[trans],
                                           rb.DIAG[diag], m, n, pa, ctypes.c_void_p(dA.data_ptr()),
                                           A.shape[0], ctypes.c_void_p(dB.data_ptr()), B.shape[0], 0)
    assert st == 0, st
    torch.cuda.synchronize()
    code = ctypes.c_int(-1)
    assert rb.lib().rocblas_b200_get_device_error(h.value, ctypes.byref(code)) == 0
    assert code.value == 0
    return dm.to_host(dB)


@pytest.mark.parametrize("side,uplo,trans,diag", COMBOS)
def test_mixed_trsm_crt_all_combos(handle, form, side, uplo, trans, diag):
    m, n = (2100, 300) if side == "L" else (300, 2100)
    k = m if side == "L" else n
    A, B = oracle.nan_triangle_problem(37, side, uplo, trans, diag, m, n, k + 3, m + 1, np.float64)
    with _moduli(16):
        out = _mixed(handle, side, uplo, trans, diag, m, n, -0.75, A, B)
    X = oracle.trsm(side, uplo, trans, diag, -0.75, A, np.asfortranarray(B[:m]))
    err = oracle.matrix_norm_1(X, out[:m])
    assert err <= oracle.trsm_tolerance(np.float64, max(m, n)), err
    assert np.isnan(out[m:]).all()


@pytest.mark.parametrize("kband", [0, 2, 4, 6])
def test_mixed_trsm_crt_condition_bands(handle, form, kband):
    """Normwise forward error against the float128 oracle on the graded-singular-value bands
    (kappa_2 = 10^kband): the residue engine at the FP64 oracle's own level."""
    m, n = 1536, 24
    A, B = workloads.graded_condition_problem(11 + kband, m, n, kband)
    Xh, Xl = oracle.refined_solution("L", "L", "N", "N", 1.0, A, B)
    e_cblas = oracle.forward_error_dd(oracle.cblas_trsm("L", "L", "N", "N", 1.0, A, B), Xh, Xl)
    with _moduli(16):
        out = _mixed(handle, "L", "L", "N", "N", m, n, 1.0, A, B)
    e = oracle.forward_error_dd(out, Xh, Xl)
    assert e <= max(1e-12, 10 * e_cblas), (e, e_cblas)
