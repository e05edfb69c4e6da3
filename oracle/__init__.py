"""CPU oracle for the TRSM hot path -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline / reference leg of
``bench.py`` import this package, and only as the checker.  The shipped library never
links or calls anything here.

Contents
--------
* ``trsm`` / ``trmm`` / ``trtri``: ctypes bindings of ``trsm_oracle.c``, a C restatement of
  the netlib reference-BLAS xTRSM / xTRMM that rocblas-test calls through
  ``ref_trsm`` / ``ref_trmm`` (clients/common/cblas_interface.cpp:2352-2575), in float,
  double and __float128 arithmetic ("s", "d", "q").
* ``cblas_trsm`` / ``cblas_trmm``: the host CBLAS itself -- OpenBLAS as bundled with scipy
  (``scipy_cblas_?trsm``), one of the CBLAS builds the reference links
  (clients/CMakeLists.txt:103-165).  It pins the C restatement (tests/test_oracle.py) and is
  the timed CPU baseline.
* generators that restate the reference test data (diagonally dominant triangular A,
  clients/include/rocblas_init.hpp:257-300; unit-diagonal randomisation,
  clients/include/client_utility.hpp:419-447); the benchmark workloads (NaN-filled unused
  triangle, condition bands) are re-exported from rocblas_b200.workloads.
* error metrics: the reference's ``matrix_norm_1`` (clients/include/norm.hpp:449-492) with
  its 40*eps*M gate (clients/include/blas3/testing_trsm.hpp:30-31, unit.hpp:578-583), and
  normwise forward / backward errors.
"""
from __future__ import annotations

import ctypes
import glob
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_trsm.so")

# rocblas / CBLAS enum values (library/include/internal/rocblas-types.h:123-172)
SIDE = {"L": 141, "R": 142}
UPLO = {"U": 121, "L": 122}
TRANS = {"N": 111, "T": 112, "C": 113}
DIAG = {"N": 131, "U": 132}
CBLAS_COL_MAJOR = 102


def build(force: bool = False) -> str:
    """Compile the C oracle with the committed Makefile."""
    newest = max(os.path.getmtime(os.path.join(HERE, f))
                 for f in ("trsm_oracle.c", "trsm_oracle_complex.c", "trsm_oracle_dd.c", "Makefile"))
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < newest:
        subprocess.check_call(["make", "-s", "-C", HERE])
    return LIB_PATH


_lib = None


def _load():
    global _lib
    if _lib is None:
        build()
        lib = ctypes.CDLL(LIB_PATH)
        i, i64, d, p = ctypes.c_int, ctypes.c_int64, ctypes.c_double, ctypes.c_void_p
        for pre in "sdq":
            f = getattr(lib, f"oracle_{pre}trsm")
            f.argtypes = [i, i, i, i, i64, i64, d, p, i64, p, i64]
            f.restype = None
            f = getattr(lib, f"oracle_{pre}trmm")
            f.argtypes = [i, i, i, i, i64, i64, d, p, i64, p, i64, p, i64]
            f.restype = None
            f = getattr(lib, f"oracle_{pre}trtri")
            f.argtypes = [i, i, i64, p, i64, p, i64]
            f.restype = None
        lib.oracle_matrix_norm_1_d.argtypes = [i64, i64, p, i64, p, i64]
        lib.oracle_matrix_norm_1_d.restype = d
        for pre in "cz":  # trsm_oracle_complex.c: alpha as (re, im)
            f = getattr(lib, f"oracle_{pre}trsm")
            f.argtypes = [i, i, i, i, i64, i64, d, d, p, i64, p, i64]
            f.restype = None
            f = getattr(lib, f"oracle_{pre}trmm")
            f.argtypes = [i, i, i, i, i64, i64, d, d, p, i64, p, i64, p, i64]
            f.restype = None
        lib.oracle_matrix_norm_1_z.argtypes = [i64, i64, p, i64, p, i64]
        lib.oracle_matrix_norm_1_z.restype = d
        lib.oracle_dd_residual.argtypes = [i64, i64, i, i, p, i64, p, p, i64, d, p, i64, p, i64]
        lib.oracle_dd_residual.restype = None
        _lib = lib
    return _lib


def _code(table, v):
    return v if isinstance(v, int) else table[v]


def _f(x, dtype):
    """Fortran-ordered array of dtype (a view when already so)."""
    return np.asfortranarray(x, dtype=dtype)


def _prec(dtype, precision):
    if precision is not None:
        return precision
    dt = np.dtype(dtype)
    if dt == np.complex64:
        return "c"
    if dt == np.complex128:
        return "z"
    return "s" if dt == np.float32 else "d"


_PREC_DTYPE = {"s": np.float32, "d": np.float64, "q": np.float64, "c": np.complex64, "z": np.complex128}


def _alpha_args(pre, alpha):
    """alpha as the C functions take it: (re, im) for the complex ones."""
    if pre in "cz":
        a = complex(alpha)
        return (a.real, a.imag)
    return (float(alpha),)


def trsm(side, uplo, trans, diag, alpha, A, B, precision=None):
    """Return X with op(A) X = alpha B (side L) or X op(A) = alpha B (side R).

    ``A`` and ``B`` are 2-D numpy arrays in column-major (Fortran) order; their leading
    dimensions are the allocated row counts, so padded layouts are expressed by passing
    the padded array and slicing nothing.  ``precision``: "s", "d" (default by dtype) or
    "q" (__float128 arithmetic, float64 storage).
    """
    pre = _prec(B.dtype, precision)
    dt = _PREC_DTYPE[pre]
    A = _f(A, dt)
    X = np.array(B, dtype=dt, order="F", copy=True)
    m, n = X.shape
    getattr(_load(), f"oracle_{pre}trsm")(
        _code(SIDE, side), _code(UPLO, uplo), _code(TRANS, trans), _code(DIAG, diag),
        m, n, *_alpha_args(pre, alpha), A.ctypes.data, A.shape[0], X.ctypes.data, X.shape[0])
    return X


def trmm(side, uplo, trans, diag, alpha, A, X, precision=None):
    """Return alpha op(A) X (side L) or alpha X op(A) (side R); only the triangle of A is
    read, and with diag U its diagonal is taken as 1."""
    pre = _prec(X.dtype, precision)
    dt = _PREC_DTYPE[pre]
    A = _f(A, dt)
    X = _f(X, dt)
    m, n = X.shape
    C = np.empty((m, n), dtype=dt, order="F")
    getattr(_load(), f"oracle_{pre}trmm")(
        _code(SIDE, side), _code(UPLO, uplo), _code(TRANS, trans), _code(DIAG, diag),
        m, n, *_alpha_args(pre, alpha), A.ctypes.data, A.shape[0], X.ctypes.data, X.shape[0],
        C.ctypes.data, m)
    return C


def trtri(uplo, diag, A, n=None, precision=None):
    """Inverse of the leading n x n triangle of A (opposite triangle returned as 0)."""
    pre = _prec(A.dtype, precision)
    dt = np.float32 if pre == "s" else np.float64
    A = _f(A, dt)
    n = A.shape[1] if n is None else n
    inv = np.zeros((n, n), dtype=dt, order="F")
    getattr(_load(), f"oracle_{pre}trtri")(
        _code(UPLO, uplo), _code(DIAG, diag), n, A.ctypes.data, A.shape[0], inv.ctypes.data, n)
    return inv


def invA_blocks(uplo, diag, A, k, nb=128, precision=None):
    """The packed diagonal-block inverses that rocblas_trsm_ex accepts as invA
    (library/include/internal/rocblas-functions.h:23112-23135): the k//nb full nb x nb
    blocks with ld = nb and stride nb*nb, followed by the k % nb remainder block (ld nb)."""
    pre = _prec(A.dtype, precision)
    dt = np.float32 if pre == "s" else np.float64
    out = np.zeros(nb * k, dtype=dt)
    nfull, rem = divmod(k, nb)
    for b in range(nfull + (1 if rem else 0)):
        s = nb if b < nfull else rem
        blk = np.asfortranarray(A[b * nb: b * nb + s, b * nb: b * nb + s])
        inv = trtri(uplo, diag, blk, precision=pre)
        view = np.zeros((nb, s), dtype=dt, order="F")
        view[:s, :s] = inv
        out[b * nb * nb: b * nb * nb + nb * s] = view.ravel(order="F")
    return out


def matrix_norm_1(gold, x):
    """The reference's forward-error norm (clients/include/norm.hpp:449-492), restated in
    C; the running sums are never reset per column, exactly as in the reference."""
    if np.iscomplexobj(gold) or np.iscomplexobj(x):
        g = np.asfortranarray(gold, dtype=np.complex128)
        v = np.asfortranarray(x, dtype=np.complex128)
        m, n = g.shape
        return _load().oracle_matrix_norm_1_z(m, n, g.ctypes.data, g.shape[0], v.ctypes.data, v.shape[0])
    g = np.asfortranarray(gold, dtype=np.float64)
    v = np.asfortranarray(x, dtype=np.float64)
    m, n = g.shape
    return _load().oracle_matrix_norm_1_d(m, n, g.ctypes.data, g.shape[0], v.ctypes.data, v.shape[0])


def trsm_tolerance(dtype, m):
    """rocblas-test's gate for both forward error and residual: 40 * eps * M
    (testing_trsm.hpp:30-31 and trsm_err_res_check in clients/include/unit.hpp:578-583)."""
    return 40.0 * float(np.finfo(dtype).eps) * m


def normwise_forward_error(X, Xstar):
    """||X - X*||_F / ||X*||_F."""
    Xs = np.asarray(Xstar, dtype=np.float64)
    d = np.asarray(X, dtype=np.float64) - Xs
    return float(np.linalg.norm(d) / np.linalg.norm(Xs))


def normwise_backward_error(side, uplo, trans, diag, alpha, A, X, B, precision="q"):
    """||alpha B - op(A) X||_F / (||op(A)||_F ||X||_F + |alpha| ||B||_F), residual in
    extended precision by default."""
    k = X.shape[0] if _code(SIDE, side) == SIDE["L"] else X.shape[1]
    R = trmm(side, uplo, trans, diag, 1.0, A, X, precision=precision).astype(np.float64)
    R = alpha * np.asarray(B, dtype=np.float64) - R
    tri = np.tril(A[:k, :k]) if _code(UPLO, uplo) == UPLO["L"] else np.triu(A[:k, :k])
    tri = np.array(tri, dtype=np.float64)
    if _code(DIAG, diag) == DIAG["U"]:
        np.fill_diagonal(tri, 1.0)
    den = np.linalg.norm(tri) * np.linalg.norm(X) + abs(alpha) * np.linalg.norm(B)
    return float(np.linalg.norm(R) / den)


def dd_residual(lower, unit, T, Xh, Xl, alpha, B):
    """r = alpha B - T (Xh + Xl) for a k x k triangle T (only its triangle is read), every
    entry accumulated in double-double and rounded once (trsm_oracle_dd.c)."""
    T = _f(T, np.float64)
    Xh = _f(Xh, np.float64)
    Xl = _f(Xl, np.float64) if Xl is not None else None
    B = _f(B, np.float64)
    k, nrhs = Xh.shape
    R = np.empty((k, nrhs), dtype=np.float64, order="F")
    _load().oracle_dd_residual(k, nrhs, int(bool(lower)), int(bool(unit)), T.ctypes.data, T.shape[0],
                               Xh.ctypes.data, Xl.ctypes.data if Xl is not None else None, Xh.shape[0],
                               float(alpha), B.ctypes.data, B.shape[0], R.ctypes.data, k)
    return R


def refined_solution(side, uplo, trans, diag, alpha, A, B, steps=2):
    """The extended-precision solution X* of op(A) X = alpha B (side L) or X op(A) = alpha B
    (side R) as an unevaluated sum Xh + Xl: the host CBLAS solve, then `steps` rounds of
    Wilkinson's iterative refinement with double-double residuals (dd_residual) and CBLAS
    corrections.  Each round multiplies the error by about cond(A, x) eps, so two rounds reach
    far below the FP64 rounding level for the condition numbers of the benchmark bands
    (<= 1e7); agreement with the __float128 substitution is checked in tests/test_oracle.py.
    FP64 only; A's other triangle is never read.  B holds exactly the m rows of the problem."""
    A = _f(A, np.float64)
    B = _f(B, np.float64)
    m, n = B.shape
    left = _code(SIDE, side) == SIDE["L"]
    notrans = _code(TRANS, trans) == TRANS["N"]
    lower = _code(UPLO, uplo) == UPLO["L"]
    unit = _code(DIAG, diag) == DIAG["U"]
    k = m if left else n
    # as a side-left, non-transposed system S Y = alpha C
    if left == notrans:
        S = A
    else:
        S = np.asfortranarray(A[:k, :k].T)
        lower = not lower
    C = B if left else np.asfortranarray(B.T)
    up = "L" if lower else "U"
    dg = "U" if unit else "N"
    Xh = cblas_trsm("L", up, "N", dg, alpha, S, C)
    Xl = np.zeros_like(Xh)
    for _ in range(steps):
        r = dd_residual(lower, unit, S, Xh, Xl, alpha, C)
        d = cblas_trsm("L", up, "N", dg, 1.0, S, r)
        t = Xl + d
        s = Xh + t
        Xl = t - (s - Xh)  # Fast2Sum: |t| << |Xh| wherever Xh is not 0
        Xh = s
    if not left:
        Xh, Xl = np.asfortranarray(Xh.T), np.asfortranarray(Xl.T)
    return Xh, Xl


def forward_error_dd(X, Xh, Xl):
    """||X - (Xh + Xl)||_F / ||Xh + Xl||_F, with the difference formed as (X - Xh) - Xl."""
    X = np.asarray(X, dtype=np.float64)
    d = (X - Xh) - Xl
    return float(np.linalg.norm(d) / np.linalg.norm(Xh))


# ---------------------------------------------------------------------------------------
# Host CBLAS (OpenBLAS bundled with scipy): the library rocblas-test's ref_trsm wraps
# ---------------------------------------------------------------------------------------
_blas = None


def openblas_path():
    import scipy

    libs = glob.glob(os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs",
                                  "libscipy_openblas-*.so"))
    if not libs:
        raise RuntimeError("scipy's bundled OpenBLAS was not found")
    return libs[0]


def _load_blas():
    global _blas
    if _blas is None:
        lib = ctypes.CDLL(openblas_path())
        i, d, f, p = ctypes.c_int, ctypes.c_double, ctypes.c_float, ctypes.c_void_p
        lib.scipy_cblas_dtrsm.argtypes = [i, i, i, i, i, i, i, d, p, i, p, i]
        lib.scipy_cblas_strsm.argtypes = [i, i, i, i, i, i, i, f, p, i, p, i]
        lib.scipy_cblas_dtrmm.argtypes = [i, i, i, i, i, i, i, d, p, i, p, i]
        lib.scipy_cblas_strmm.argtypes = [i, i, i, i, i, i, i, f, p, i, p, i]
        for fn in ("scipy_cblas_ztrsm", "scipy_cblas_ctrsm", "scipy_cblas_ztrmm", "scipy_cblas_ctrmm"):
            getattr(lib, fn).argtypes = [i, i, i, i, i, i, i, p, p, i, p, i]  # alpha by pointer
        for fn in ("scipy_cblas_dtrsm", "scipy_cblas_strsm", "scipy_cblas_dtrmm", "scipy_cblas_strmm",
                   "scipy_cblas_ztrsm", "scipy_cblas_ctrsm", "scipy_cblas_ztrmm", "scipy_cblas_ctrmm"):
            getattr(lib, fn).restype = None
        lib.scipy_openblas_set_num_threads.argtypes = [i]
        lib.scipy_openblas_get_num_threads.restype = i
        lib.scipy_openblas_get_config.restype = ctypes.c_char_p
        _blas = lib
    return _blas


def cblas_set_threads(n):
    _load_blas().scipy_openblas_set_num_threads(int(n))


def cblas_get_threads():
    return int(_load_blas().scipy_openblas_get_num_threads())


def cblas_config():
    return _load_blas().scipy_openblas_get_config().decode()


_CBLAS_PRE = {np.dtype(np.float32): "s", np.dtype(np.float64): "d", np.dtype(np.complex64): "c",
              np.dtype(np.complex128): "z"}


def _cblas_alpha(dtype, alpha):
    """A complex alpha goes to cblas by pointer (the array keeps it alive)."""
    if np.iscomplexobj(np.empty(0, dtype=dtype)):
        a = np.array([alpha], dtype=dtype)
        return a, ctypes.c_void_p(a.ctypes.data)
    return None, float(alpha)


def cblas_trsm_inplace(side, uplo, trans, diag, alpha, A, B):
    """cblas_?trsm(CblasColMajor, ...) on Fortran-ordered arrays, B overwritten."""
    lib = _load_blas()
    fn = getattr(lib, f"scipy_cblas_{_CBLAS_PRE[B.dtype]}trsm")
    assert A.flags.f_contiguous and B.flags.f_contiguous and A.dtype == B.dtype
    m, n = B.shape
    keep, a = _cblas_alpha(B.dtype, alpha)
    fn(CBLAS_COL_MAJOR, _code(SIDE, side), _code(UPLO, uplo), _code(TRANS, trans),
       _code(DIAG, diag), m, n, a, A.ctypes.data, A.shape[0], B.ctypes.data, B.shape[0])
    return B


def cblas_trsm(side, uplo, trans, diag, alpha, A, B):
    X = np.array(B, order="F", copy=True)
    return cblas_trsm_inplace(side, uplo, trans, diag, alpha, _f(A, B.dtype), X)


def cblas_trmm(side, uplo, trans, diag, alpha, A, X):
    lib = _load_blas()
    C = np.array(X, order="F", copy=True)
    A = _f(A, C.dtype)
    fn = getattr(lib, f"scipy_cblas_{_CBLAS_PRE[C.dtype]}trmm")
    m, n = C.shape
    keep, a = _cblas_alpha(C.dtype, alpha)
    fn(CBLAS_COL_MAJOR, _code(SIDE, side), _code(UPLO, uplo), _code(TRANS, trans),
       _code(DIAG, diag), m, n, a, A.ctypes.data, A.shape[0], C.ctypes.data, C.shape[0])
    return C


# ---------------------------------------------------------------------------------------
# Generators
# ---------------------------------------------------------------------------------------
def diag_dominant_triangular(rng, k, lda, uplo, dtype, low=1, high=10):
    """rocblas_client_diagonally_dominant_triangular_matrix (rocblas_init.hpp:257-300):
    random integer entries in [low, high] in the triangle (rocblas_random.hpp:306-308),
    then every diagonal entry set to 1.01 x (|row| + |column| off-diagonal sums); the
    opposite triangle is 0."""
    A = np.zeros((lda, k), dtype=np.float64, order="F")
    vals = rng.integers(low, high + 1, size=(k, k)).astype(np.float64)
    tri = np.triu(vals) if _code(UPLO, uplo) == UPLO["U"] else np.tril(vals)
    off = tri - np.diag(np.diag(tri))
    rows = np.abs(off).sum(axis=1)
    cols = np.abs(off).sum(axis=0)
    d = (rows + cols) * 1.01
    d[d == 0] = 1.0
    tri = off + np.diag(d)
    A[:k, :k] = tri
    return A.astype(dtype, order="F")


def make_unit_diagonal(rng, A, k, uplo):
    """client_utility.hpp:419-447: scale each row (lower) / column (upper) of the triangle
    by its diagonal, then overwrite the stored diagonal with random values so that any
    read of it shows up as a wrong answer."""
    A = np.array(A, order="F", copy=True)
    if _code(UPLO, uplo) == UPLO["L"]:
        for i in range(k):
            A[i, : i + 1] /= A[i, i]
    else:
        for j in range(k):
            A[: j + 1, j] /= A[j, j]
    for i in range(k):
        A[i, i] = rng.integers(1, 11)
    return A


def rocblas_test_problem(seed, side, uplo, trans, diag, m, n, lda, ldb, alpha, dtype):
    """The rocblas-test recipe (testing_trsm.hpp:283-315): A diagonally dominant, X random
    integers in [1, 10], B = op(A) X / alpha (side L) or X op(A) / alpha (side R) computed
    by trmm.  Returns (A, B, X) with A lda x k and B ldb x n (padding filled with NaN so
    that reads or writes outside the m x n window are visible)."""
    rng = np.random.default_rng(seed)
    k = m if _code(SIDE, side) == SIDE["L"] else n
    A = diag_dominant_triangular(rng, k, lda, uplo, np.float64)
    if _code(DIAG, diag) == DIAG["U"]:
        A = make_unit_diagonal(rng, A, k, uplo)
    X = rng.integers(1, 11, size=(m, n)).astype(np.float64)
    X = np.asfortranarray(X.astype(dtype))
    Ad = A.astype(dtype, order="F")
    Bcore = trmm(side, uplo, trans, diag, 1.0 / alpha, Ad[:k, :k], X)
    B = np.full((ldb, n), np.nan, dtype=dtype, order="F")
    B[:m, :] = Bcore
    return Ad, B, X


# the workload generators live with the benchmarks; the oracle re-exports them so that tests
# build exactly the inputs the benchmark uses
from rocblas_b200.workloads import condition_band_problem, nan_triangle_problem  # noqa: E402,F401


def clean_triangle(A, k, uplo, diag):
    """A copy of A's k x k triangle with the unused half 0 and, for diag U, a unit diagonal
    (for checkers that use dense algebra)."""
    T = np.array(A[:k, :k], dtype=np.float64)
    T = np.tril(np.nan_to_num(T)) if _code(UPLO, uplo) == UPLO["L"] else np.triu(np.nan_to_num(T))
    if _code(DIAG, diag) == DIAG["U"]:
        np.fill_diagonal(T, 1.0)
    else:
        np.fill_diagonal(T, np.diag(np.array(A[:k, :k], dtype=np.float64)))
    return T
