"""The precision form with FP64 iterative refinement (rocblas_b200_dtrsm_refined).

* every side/uplo/trans/diag combination converges and meets the rocblas-test gate;
* with few slices (14-28 bits per entry) the first solve fails the test (agreement with the
  plain FP64 form on the tested right-hand sides) and the FP64-residual corrections bring the
  result to the plain FP64 form's accuracy, measured against the double-double-refined X* of
  the oracle, on matrices whose conditioning no diagonal scaling removes (singular values
  graded to 10^-k);
* on those graded bands the refined form ends within 1e-12 of X*;
* the test's counters (iterations, error estimates, checked right-hand sides) are consistent;
* without convergence the plain FP64 form takes over (or, with fallback off, the refined
  iterate is returned as it is);
* argument rules: host alpha only, slices 1..8, quick returns, alpha == 0, size query.

The sliced updates start at K >= sliced_min_k and the bottom rows run on the FP64 chain in
blocks of mixed_chain_blocks x 128, so these sizes lower both tuning keys to put the sliced
engine on the path being refined."""
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


@pytest.fixture(scope="module")
def handle():
    rb.build()
    h = rb.Handle()
    yield h
    h.close()


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


SLICED_SMALL = dict(sliced_min_k=128, mixed_chain_blocks=2)


def _refined(h, side, uplo, trans, diag, m, n, alpha, A, B, **opts):
    dA, dB = dm.to_device(A), dm.to_device(B)
    info = dm.trsm_refined(h, side, uplo, trans, diag, m, n, alpha, dA, A.shape[0], dB, B.shape[0], **opts)
    torch.cuda.synchronize()
    code = ctypes.c_int(-1)
    assert rb.lib().rocblas_b200_get_device_error(h.value, ctypes.byref(code)) == 0
    assert code.value == 0
    return dm.to_host(dB), info


def _plain(h, side, uplo, trans, diag, m, n, alpha, A, B):
    dA, dB = dm.to_device(A), dm.to_device(B)
    dm.trsm(h, side, uplo, trans, diag, m, n, alpha, dA, A.shape[0], dB, B.shape[0])
    torch.cuda.synchronize()
    return dm.to_host(dB)


CHECK_FORMS = {"flag-check": dict(refine_check_flag=1),
               "chain32-check": dict(refine_check_flag=0, refine_check_w=32, refine_check_pairs=0),
               "chain16-check": dict(refine_check_flag=0, refine_check_w=16, refine_check_pairs=0),
               "paired-check": dict(refine_check_flag=0, refine_check_pairs=1)}


@pytest.mark.parametrize("check", list(CHECK_FORMS))
@pytest.mark.parametrize("side,uplo,trans,diag", COMBOS)
def test_refined_all_combos(handle, side, uplo, trans, diag, check):
    """Every form of the test's FP64 solve of the sampled right-hand sides (the memory-bound
    flag solve, the chain with 32- or 16-column strips) agrees with the precision form's first
    solve to the tolerance."""
    m, n = (900, 120) if side == "L" else (120, 900)
    k = m if side == "L" else n
    A, B = oracle.nan_triangle_problem(41, side, uplo, trans, diag, m, n, k + 3, m + 2, np.float64)
    with tuning(**CHECK_FORMS[check], **SLICED_SMALL):
        out, info = _refined(handle, side, uplo, trans, diag, m, n, -0.75, A, B)
    assert info["error_estimate_first"] <= info["tolerance"], info
    X = oracle.trsm(side, uplo, trans, diag, -0.75, A, np.asfortranarray(B[:m]))
    assert oracle.matrix_norm_1(X, out[:m]) <= oracle.trsm_tolerance(np.float64, max(m, n))
    assert np.isnan(out[m:]).all()
    assert info["converged"] == 1 and info["fell_back"] == 0, info
    assert info["checked_columns"] == min(8, n if side == "L" else m)
    assert info["tolerance"] == 1e-12
    assert info["error_estimate"] <= info["tolerance"]


@pytest.mark.parametrize("side,uplo,trans,diag,slices,kband",
                         [("L", "L", "N", "N", 2, 2), ("L", "U", "T", "N", 3, 4), ("R", "L", "N", "U", 3, 2),
                          ("R", "U", "T", "N", 4, 4), ("L", "L", "T", "U", 2, 1)])
def test_refinement_restores_fp64_accuracy(handle, side, uplo, trans, diag, slices, kband):
    """14, 21 or 28 bits per entry in the first solve; with a tolerance of 1e-14 the
    corrections restore the plain FP64 form's accuracy on a graded matrix (kappa_2 = 10^kband;
    a unit diagonal scales the rows of that triangle to 1 first)."""
    k = 1024
    m, n = (k, 48) if side == "L" else (48, k)
    T, _ = workloads.graded_condition_problem(7, k, 1, kband)  # lower, NaN upper triangle
    Tl = np.tril(np.nan_to_num(T))
    if diag == "U":
        Tl = Tl / np.diag(Tl)[:, None]
    A = np.array(Tl if uplo == "L" else Tl.T, order="F")
    A[np.triu_indices(k, 1) if uplo == "L" else np.tril_indices(k, -1)] = np.nan
    if diag == "U":
        A[np.arange(k), np.arange(k)] = np.nan  # must never be read
    rng = np.random.default_rng(slices)
    B = np.asfortranarray(rng.uniform(-1, 1, size=(m, n)))
    with tuning(**SLICED_SMALL):
        out, info = _refined(handle, side, uplo, trans, diag, m, n, 1.5, A, B, slices=slices,
                             check_columns=1 << 20, tolerance=1e-14)
    Xh, Xl = oracle.refined_solution(side, uplo, trans, diag, 1.5, A, B)
    plain = _plain(handle, side, uplo, trans, diag, m, n, 1.5, A, B)
    e_ref = oracle.forward_error_dd(plain, Xh, Xl)
    e = oracle.forward_error_dd(out, Xh, Xl)
    assert info["checked_columns"] == (n if side == "L" else m)  # all right-hand sides tested
    assert info["error_estimate_first"] > info["tolerance"], info  # too few bits at first
    assert info["iterations"] >= 1 and info["converged"] == 1 and info["fell_back"] == 0, info
    assert info["error_estimate"] <= info["tolerance"], info
    assert e <= max(10 * e_ref, 1e-14), (e, e_ref, info)


@pytest.mark.parametrize("kband", [0, 2, 4, 6])
def test_refined_graded_bands(handle, kband):
    """Singular values graded from 1 to 10^-k (kappa_2 = 10^k, not removable by diagonal
    scaling): with every right-hand side tested, the refined precision form ends within the
    default 1e-12 of the plain FP64 form, and so within about 1e-12 of X*, in every band."""
    m, n = 1536, 40
    A, B = workloads.graded_condition_problem(11 + kband, m, n, kband)
    Xh, Xl = oracle.refined_solution("L", "L", "N", "N", 1.0, A, B)
    e_cblas = oracle.forward_error_dd(oracle.cblas_trsm("L", "L", "N", "N", 1.0, A, B), Xh, Xl)
    with tuning(**SLICED_SMALL):
        out, info = _refined(handle, "L", "L", "N", "N", m, n, 1.0, A, B, check_columns=n)
    e = oracle.forward_error_dd(out, Xh, Xl)
    assert info["converged"] == 1, info
    assert e <= 1e-12 + 10 * e_cblas, (e, e_cblas, info)


def test_refined_fallback_and_no_fallback(handle):
    """One slice and no corrections allowed: the test fails; with fallback the result is the
    plain FP64 form's, bit for bit; without it, the precision-form iterate as it is."""
    m, n = 1024, 64
    A, B = oracle.nan_triangle_problem(5, "L", "L", "N", "N", m, n, m, m, np.float64)
    plain = _plain(handle, "L", "L", "N", "N", m, n, 0.5, A, B)
    with tuning(**SLICED_SMALL):
        out, info = _refined(handle, "L", "L", "N", "N", m, n, 0.5, A, B, slices=1, max_iterations=0,
                             fallback=1)
        assert info["converged"] == 0 and info["fell_back"] == 1 and info["iterations"] == 0, info
        np.testing.assert_array_equal(out, plain)
        out2, info2 = _refined(handle, "L", "L", "N", "N", m, n, 0.5, A, B, slices=1, max_iterations=0,
                               fallback=0)
        assert info2["converged"] == 0 and info2["fell_back"] == 0, info2
        dA, dB = dm.to_device(A), dm.to_device(B)
        a = ctypes.c_double(0.5)
        assert rb.lib().rocblas_b200_dtrsm_mixed(handle.value, rb.SIDE["L"], rb.UPLO["L"], rb.TRANS["N"],
                                                 rb.DIAG["N"], m, n, ctypes.cast(ctypes.byref(a), ctypes.c_void_p),
                                                 ctypes.c_void_p(dA.data_ptr()), m,
                                                 ctypes.c_void_p(dB.data_ptr()), m, 1) == 0
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out2, dm.to_host(dB))
        assert info2["error_estimate"] == info2["error_estimate_first"] > info2["tolerance"]


def test_refined_arguments(handle):
    L = rb.lib()
    m, n = 200, 10
    A, B = oracle.nan_triangle_problem(2, "L", "L", "N", "N", m, n, m, m, np.float64)
    dA, dB = dm.to_device(A), dm.to_device(B)
    args = (rb.SIDE["L"], rb.UPLO["L"], rb.TRANS["N"], rb.DIAG["N"])
    one = ctypes.c_double(1.0)
    p1 = ctypes.cast(ctypes.byref(one), ctypes.c_void_p)
    pa, pb = ctypes.c_void_p(dA.data_ptr()), ctypes.c_void_p(dB.data_ptr())
    info = rb.RefineInfo()
    pinfo = ctypes.cast(ctypes.byref(info), ctypes.c_void_p)
    fn = L.rocblas_b200_dtrsm_refined
    bad = rb.RefineOptions(9, -1, 0, 1, 0.0)
    assert fn(handle.value, *args, m, n, p1, pa, m, pb, m, ctypes.cast(ctypes.byref(bad), ctypes.c_void_p),
              None) == rb.status_invalid_value
    # quick return, with null pointers allowed
    assert fn(handle.value, *args, 0, n, p1, None, m, None, m, None, pinfo) == rb.status_success
    assert info.converged == 1 and info.iterations == 0
    # device pointer mode is not supported
    handle.set_pointer_mode(rb.pointer_mode_device)
    try:
        dalpha = torch.ones(1, dtype=torch.float64, device="cuda")
        assert fn(handle.value, *args, m, n, ctypes.c_void_p(dalpha.data_ptr()), pa, m, pb, m, None,
                  None) == rb.status_not_implemented
    finally:
        handle.set_pointer_mode(rb.pointer_mode_host)
    # alpha == 0: B := 0, A not read
    zero = ctypes.c_double(0.0)
    assert fn(handle.value, *args, m, n, ctypes.cast(ctypes.byref(zero), ctypes.c_void_p), None, m, pb, m,
              None, pinfo) == rb.status_success
    torch.cuda.synchronize()
    assert (dm.to_host(dB)[:m] == 0).all() and info.converged == 1
    # the size query reports the refined solve's workspace: two m x n copies beyond the
    # precision form's
    size = ctypes.c_size_t(0)
    assert L.rocblas_start_device_memory_size_query(handle.value) == 0
    st = fn(handle.value, *args, 4096, 512, p1, pa, 4096, pb, 4096, None, None)
    assert st in (rb.status_success, rb.status_size_increased, rb.status_size_unchanged), st
    assert L.rocblas_stop_device_memory_size_query(handle.value, ctypes.byref(size)) == 0
    assert size.value >= 2 * 4096 * 512 * 8
