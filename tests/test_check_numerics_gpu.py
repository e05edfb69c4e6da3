"""Check-numerics (ROCBLAS_CHECK_NUMERICS) of the TRSM entry points.

The reference scans A's referenced triangle (diagonal included) and B before the solve and B
after it (library/src/blas3/rocblas_trmm_kernels.cpp:2306-2362 from rocblas_trsm_imp.hpp:159-181
and :248-270), one flag each for NaN, zero, Inf and denormal values; fail mode returns
rocblas_status_check_numerics_fail for NaN, Inf or (unless bit 8 is set) denormal values,
info and warn print the flags (library/src/check_numerics_vector.cpp:95-136). The mode is read
when the handle is created.
"""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import rocblas_b200 as rb  # noqa: E402
from rocblas_b200 import devmem as dm  # noqa: E402
from rocblas_b200 import workloads  # noqa: E402

pytestmark = pytest.mark.gpu

FAIL = rb.status_check_numerics_fail


def _handle(mode):
    rb.build()
    os.environ["ROCBLAS_CHECK_NUMERICS"] = str(mode)
    try:
        return rb.Handle()
    finally:
        del os.environ["ROCBLAS_CHECK_NUMERICS"]


def _solve(h, A, B, m, n, alpha=1.0, uplo="L", diag="N"):
    dA, dB = dm.to_device(A), dm.to_device(B)
    st = dm.trsm(h, "L", uplo, "N", diag, m, n, alpha, dA, A.shape[0], dB, B.shape[0],
                 allow=(rb.status_success, FAIL))
    torch.cuda.synchronize()
    return st, dm.to_host(dB)


def _problem(m=300, n=40, uplo="L", diag="N", dtype=np.float64):
    return workloads.nan_triangle_problem(81, "L", uplo, "N", diag, m, n, m + 3, m + 2, dtype)


def test_clean_inputs_pass_and_match_the_unchecked_solve():
    """NaN in the unused triangle and in B's padding rows is not looked at."""
    A, B = _problem()
    h, plain = _handle(4), rb.Handle()
    try:
        st, got = _solve(h, A, B, 300, 40)
        st0, ref = _solve(plain, A, B, 300, 40)
        assert st == 0 and st0 == 0
        assert np.array_equal(got[:300], ref[:300])
    finally:
        h.close()
        plain.close()


@pytest.mark.parametrize("where", ["A", "B_inf", "B_denorm"])
def test_fail_mode_rejects_inputs_before_the_solve(where):
    A, B = _problem()
    if where == "A":
        A[200, 17] = np.nan  # inside the lower triangle
    elif where == "B_inf":
        B[123, 39] = np.inf
    else:
        B[5, 0] = 1e-310
    h = _handle(4)
    try:
        st, got = _solve(h, A, B, 300, 40)
        assert st == FAIL
        assert np.array_equal(got[:300], B[:300], equal_nan=True)  # B untouched
    finally:
        h.close()


def test_only_nan_inf_ignores_denormals():
    A, B = _problem()
    B[5, 0] = 1e-310
    h = _handle(4 | 8)
    try:
        assert _solve(h, A, B, 300, 40)[0] == 0
    finally:
        h.close()


def test_fail_mode_checks_the_result():
    """Finite inputs whose solution overflows: the output check of B fails after the solve."""
    m, n = 64, 8
    A = np.zeros((m, m), order="F")
    A[np.arange(m), np.arange(m)] = 1e-10
    B = np.full((m, n), 1e300, order="F")
    h = _handle(4)
    try:
        st, got = _solve(h, A, B, m, n)
        assert st == FAIL
        assert not np.isfinite(got).any()  # 1e310 overflows; 0 * inf below the first row is NaN
    finally:
        h.close()


def test_unit_diagonal_stored_values_are_checked():
    """The triangle is scanned with its diagonal whatever diag says, as the reference does: the
    recipe's NaN on a unit diagonal fails."""
    A, B = _problem(diag="U")
    h = _handle(4)
    try:
        assert _solve(h, A, B, 300, 40, diag="U")[0] == FAIL
    finally:
        h.close()


def test_host_alpha_zero_checks_nothing():
    A, B = _problem()
    A[200, 17] = np.nan
    h = _handle(4)
    try:
        st, got = _solve(h, A, B, 300, 40, alpha=0.0)
        assert st == 0 and np.all(got[:300] == 0.0)
    finally:
        h.close()


def test_info_and_warn_print(capfd):
    A, B = _problem()
    h = _handle(1)
    try:
        assert _solve(h, A, B, 300, 40)[0] == 0
    finally:
        h.close()
    err = capfd.readouterr().err.splitlines()
    lines = [l for l in err if l.startswith("Function name:")]
    assert lines == ["Function name:\trocblas_dtrsm :- Input :\t has_NaN 0 has_zero 0 has_Inf 0 has_denorm 0"] * 2 \
        + ["Function name:\trocblas_dtrsm :- Output :\t has_NaN 0 has_zero 0 has_Inf 0 has_denorm 0"]
    A[200, 17] = np.nan
    h = _handle(2)
    try:
        assert _solve(h, A, B, 300, 40)[0] == 0  # warn only
    finally:
        h.close()
    err = capfd.readouterr().err.splitlines()
    lines = [l for l in err if l.startswith("Function name:")]
    assert lines[0] == "Function name:\trocblas_dtrsm :- Input :\t has_NaN 1 has_zero 0 has_Inf 0 has_denorm 0"
    # warn prints only abnormal checks: not B's clean input, but the result the NaN reached
    assert all("Input :\t has_NaN 0" not in l for l in lines)
    assert lines[-1].startswith("Function name:\trocblas_dtrsm :- Output :\t has_NaN 1")


def test_strided_batched_and_complex():
    m, n, batch = 96, 12, 5
    A1, B1 = _problem(m, n)
    As = np.stack([A1] * batch)
    Bs = np.stack([B1] * batch)
    Bs[3, 10, 4] = -np.inf
    h = _handle(4)
    try:
        dA = torch.from_numpy(np.ascontiguousarray(As.transpose(0, 2, 1))).cuda()
        dB = torch.from_numpy(np.ascontiguousarray(Bs.transpose(0, 2, 1))).cuda()
        lda, ldb = A1.shape[0], B1.shape[0]
        st = dm.trsm_strided_batched(h, "L", "L", "N", "N", m, n, 1.0, dA, lda, lda * m, dB, ldb,
                                     ldb * n, batch, allow=(0, FAIL))
        assert st == FAIL
        Az, Bz = _problem(m, n, dtype=np.complex128)
        Bz[7, 3] = complex(1.0, np.nan)
        st, _ = _solve(h, Az, Bz, m, n, alpha=1.0)
        assert st == FAIL
    finally:
        h.close()
