"""Pin the CPU oracle before trusting it (CPU only).

The reference has no golden trsm vectors; its tests compare against the host CBLAS
(ref_trsm -> cblas_?trsm) and against the X the right-hand side was built from.  These
tests check the C restatement in oracle/ against both, through the committed fixtures
made by tests/golden/make_golden.py and live against the host CBLAS.
"""
import itertools
import os

import numpy as np
import pytest

import oracle

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
COMBOS = list(itertools.product("LR", "UL", "NT", "NU"))


def _cases(npz):
    keys = sorted({k.rsplit("_", 1)[0] for k in npz.files})
    return keys


@pytest.mark.parametrize("dt", ["d", "s"])
def test_oracle_matches_cblas_golden(dt):
    z = np.load(os.path.join(GOLDEN, f"cblas_{dt}.npz"))
    keys = _cases(z)
    assert len(keys) == 16 * 4
    eps = np.finfo(np.float64 if dt == "d" else np.float32).eps
    for key in keys:
        combo, shape = key.split("_")
        side, uplo, trans, diag = combo
        m, n = map(int, shape.split("x"))
        A, B, X, alpha = z[key + "_A"], z[key + "_B"], z[key + "_X"], float(z[key + "_alpha"])
        got = oracle.trsm(side, uplo, trans, diag, alpha, A, np.asfortranarray(B[:m]))
        assert not np.isnan(got).any(), key
        err = oracle.matrix_norm_1(X, got)
        assert err <= oracle.trsm_tolerance(got.dtype, max(m, n)), (key, err)
        # much tighter in practice: the two differ only in operation order
        assert err <= 64 * eps, (key, err)


@pytest.mark.parametrize("dt", ["d", "s"])
def test_oracle_recovers_protocol_x(dt):
    """rocblas-test's own check: forward error and residual within 40 eps M."""
    z = np.load(os.path.join(GOLDEN, f"protocol_{dt}.npz"))
    for key in _cases(z):
        side, uplo, trans, diag = key
        A, B, X, alpha = z[key + "_A"], z[key + "_B"], z[key + "_X"], float(z[key + "_alpha"])
        m, n = B.shape
        got = oracle.trsm(side, uplo, trans, diag, alpha, A, B)
        tol = oracle.trsm_tolerance(got.dtype, m)
        assert oracle.matrix_norm_1(X, got) <= tol, key
        res = oracle.trmm(side, uplo, trans, diag, 1.0 / alpha, A, got)
        assert oracle.matrix_norm_1(B, res) <= tol, key


def test_quad_oracle_tighter_than_double():
    A, B = oracle.condition_band_problem(3, 300, 7, 4)
    Xq = oracle.trsm("L", "L", "N", "N", 1.0, A, B, precision="q")
    Xd = oracle.trsm("L", "L", "N", "N", 1.0, A, B, precision="d")
    Xc = oracle.cblas_trsm("L", "L", "N", "N", 1.0, A, B)
    e_d = oracle.normwise_forward_error(Xd, Xq)
    e_c = oracle.normwise_forward_error(Xc, Xq)
    assert e_d < 1e-9 and e_c < 1e-9
    # the quad residual is at the double rounding level of X
    assert oracle.normwise_backward_error("L", "L", "N", "N", 1.0, A, Xq, B) < 1e-16


@pytest.mark.parametrize("side,uplo,trans,diag", COMBOS)
def test_oracle_vs_live_cblas(side, uplo, trans, diag):
    m, n = 70, 45
    k = m if side == "L" else n
    A, B = oracle.nan_triangle_problem(11, side, uplo, trans, diag, m, n, k, m, np.float64)
    X = oracle.trsm(side, uplo, trans, diag, -1.5, A, B)
    Xc = oracle.cblas_trsm(side, uplo, trans, diag, -1.5, A, B)
    assert oracle.matrix_norm_1(Xc, X) < 1e-14


def test_alpha_zero_and_trtri():
    A, B = oracle.nan_triangle_problem(5, "L", "U", "N", "N", 9, 4, 9, 9, np.float64)
    assert np.all(oracle.trsm("L", "U", "N", "N", 0.0, A, B) == 0)
    inv = oracle.trtri("U", "N", A)
    T = oracle.clean_triangle(A, 9, "U", "N")
    assert np.allclose(inv @ T, np.eye(9), atol=1e-13)
    assert np.all(np.tril(inv, -1) == 0)
    # zero diagonal entries are treated as 1 (rocblas_trtri.hpp:138-141)
    Z = np.eye(3)
    Z[1, 1] = 0.0
    assert oracle.trtri("L", "N", Z)[1, 1] == 1.0


def test_matrix_norm_1_is_cumulative():
    """The reference never resets its per-column sums: the metric is sum|e| / sum|x|."""
    gold = np.array([[1.0, 100.0], [1.0, 100.0]], order="F")
    x = gold.copy(order="F")
    x[0, 0] = 2.0
    assert abs(oracle.matrix_norm_1(gold, x) - 1.0 / 202.0) < 1e-15


def test_workload_generators_shapes_and_nan_triangle():
    import torch

    from rocblas_b200 import workloads

    At, Bt = workloads.condition_band_lower_torch(64, 5, 4, seed=3, device="cpu")
    A = At.numpy().T
    assert A.shape == (64, 64) and Bt.shape == (5, 64)
    assert np.isnan(A[np.triu_indices(64, 1)]).all()
    assert not np.isnan(np.tril(A)).any()
    d = np.diag(A)
    assert d[0] > 1.0 and d[-1] < 1.1e-4 * 1.0001 * 1.1 and np.all(d > 0)
    # off-diagonals of row i are scaled by d_i
    assert np.all(np.abs(A[40, :40]) <= d[40] * 6.0 / np.sqrt(64))
    assert float(Bt.abs().max()) <= 1.0
    del torch


COMBOS_C = list(itertools.product("LR", "UL", "NTC", "NU"))


@pytest.mark.parametrize("dt", ["z", "c"])
def test_complex_oracle_matches_cblas_golden(dt):
    """The complex restatement (trsm_oracle_complex.c) against cblas_{c,z}trsm answers
    recorded in tests/golden (all 24 side/uplo/trans/diag combinations, trans C included)."""
    z = np.load(os.path.join(GOLDEN, f"cblas_{dt}.npz"))
    keys = _cases(z)
    assert len(keys) == 24 * 2
    eps = np.finfo(np.complex128 if dt == "z" else np.complex64).eps
    for key in keys:
        combo, shape = key.split("_")
        side, uplo, trans, diag = combo
        m, n = map(int, shape.split("x"))
        A, B, X, alpha = z[key + "_A"], z[key + "_B"], z[key + "_X"], complex(z[key + "_alpha"])
        got = oracle.trsm(side, uplo, trans, diag, alpha, A, np.asfortranarray(B[:m]))
        assert got.dtype == A.dtype and not np.isnan(got).any(), key
        err = oracle.matrix_norm_1(X, got)
        assert err <= 64 * eps, (key, err)


@pytest.mark.parametrize("side,uplo,trans,diag", COMBOS_C)
def test_complex_oracle_vs_live_cblas_and_trmm(side, uplo, trans, diag):
    m, n = 40, 27
    k = m if side == "L" else n
    alpha = -1.5 + 0.25j
    A, B = oracle.nan_triangle_problem(12, side, uplo, trans, diag, m, n, k + 1, m, np.complex128)
    X = oracle.trsm(side, uplo, trans, diag, alpha, A, B)
    Xc = oracle.cblas_trsm(side, uplo, trans, diag, alpha, A, B)
    assert oracle.matrix_norm_1(Xc, X) < 1e-14
    # the forward operator: trmm against the host CBLAS, and op(A) X / alpha gives back B
    R = oracle.trmm(side, uplo, trans, diag, 1 / alpha, A, X)
    assert oracle.matrix_norm_1(oracle.cblas_trmm(side, uplo, trans, diag, 1 / alpha, A, X), R) < 1e-14
    assert oracle.matrix_norm_1(B, R) <= oracle.trsm_tolerance(np.complex128, k)
    # trans C differs from trans T exactly by conj(A)
    if trans == "C":
        Xt = oracle.trsm(side, uplo, "T", diag, alpha, np.conj(A), B)
        assert oracle.matrix_norm_1(Xt, X) == 0.0


def test_complex_matrix_norm_uses_modulus():
    gold = np.array([[3 + 4j]], dtype=np.complex128, order="F")
    x = np.array([[0j]], dtype=np.complex128, order="F")
    assert oracle.matrix_norm_1(gold, x) == 1.0
    x[0, 0] = 3 + 0j
    assert abs(oracle.matrix_norm_1(gold, x) - 4.0 / 5.0) < 1e-15


@pytest.mark.parametrize("side,uplo,trans,diag", COMBOS)
def test_dd_refined_solution_matches_float128(side, uplo, trans, diag):
    """The extended-precision X* of the benchmarks (host CBLAS + two double-double refinement
    steps) agrees with the __float128 substitution to the rounding of the latter's double
    output, on square, tall, wide and degenerate shapes, padded leading dimensions included."""
    for m, n in [(301, 21), (7, 3), (1, 1), (4, 9), (600, 5)]:
        k = m if side == "L" else n
        A, B = oracle.nan_triangle_problem(3, side, uplo, trans, diag, m, n, k + 7, m + 5, np.float64)
        B = np.asfortranarray(B[:m])
        Xq = oracle.trsm(side, uplo, trans, diag, 0.7, A, B, precision="q")
        Xh, Xl = oracle.refined_solution(side, uplo, trans, diag, 0.7, A, B)
        assert oracle.forward_error_dd(Xq, Xh, Xl) < 1e-16, (m, n)


@pytest.mark.parametrize("kband", [0, 2, 4])
def test_graded_generator_condition_and_dd_oracle(kband):
    """Singular values graded to 10^-k give kappa_2 = 10^k exactly; scaling the rows to a unit
    diagonal does not remove it; the dd X* matches the __float128 one on that matrix too."""
    from rocblas_b200 import workloads

    m = 256
    A, B = workloads.graded_condition_problem(1, m, 6, kband)
    assert np.isnan(A[np.triu_indices(m, 1)]).all()
    T = np.tril(np.nan_to_num(A))
    s = np.linalg.svd(T, compute_uv=False)
    assert s[0] / s[-1] == pytest.approx(10.0 ** kband, rel=1e-6)
    s2 = np.linalg.svd(T / np.diag(T)[:, None], compute_uv=False)
    assert s2[0] / s2[-1] >= 0.5 * 10.0 ** kband
    Xq = oracle.trsm("L", "L", "N", "N", 1.0, A, B, precision="q")
    Xh, Xl = oracle.refined_solution("L", "L", "N", "N", 1.0, A, B)
    assert oracle.forward_error_dd(Xq, Xh, Xl) < 1e-16
