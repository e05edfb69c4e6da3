"""GPU parity tests: librocblas_b200.so through its C ABI against the CPU oracle.

Gates (floating point):
* rocblas-test's own: forward error ||X - X_true||_1-cumulative and residual, each
  <= 40 * eps * M (clients/include/blas3/testing_trsm.hpp:30-31, 437-448);
* against the oracle restatement of the host CBLAS (and the committed cblas fixtures) on the
  NaN-triangle workload generator: the same norm <= 40 * eps * max(M, N).
Sizes follow clients/gtest/trsm_gtest.yaml (small :6-19, medium :21-46, substitution
:48-113, large :57-61).
"""
import itertools
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle  # noqa: E402
import rocblas_b200 as rb  # noqa: E402
from rocblas_b200 import devmem as dm  # noqa: E402

pytestmark = pytest.mark.gpu
COMBOS = list(itertools.product("LR", "UL", "NT", "NU"))
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
DT = {"d": (np.float64, torch.float64), "s": (np.float32, torch.float32)}


@pytest.fixture(scope="module")
def handle():
    rb.build()
    h = rb.Handle()
    yield h
    h.close()


def _gpu_solve(handle, side, uplo, trans, diag, m, n, alpha, A, B, alpha_on_device=False,
               allow=(rb.status_success,)):
    dA = dm.to_device(A)
    dB = dm.to_device(B)
    st = dm.trsm(handle, side, uplo, trans, diag, m, n, alpha, dA, A.shape[0], dB, B.shape[0],
                 alpha_on_device=alpha_on_device, allow=allow)
    torch.cuda.synchronize()
    return dm.to_host(dB), st


def _check_vs_oracle(side, uplo, trans, diag, m, n, alpha, A, B, Bout, dt):
    X = oracle.trsm(side, uplo, trans, diag, alpha, A, np.asfortranarray(B[:m]))
    got = Bout[:m]
    assert not np.isnan(got).any(), "NaN in the solution (stray read of the unused triangle?)"
    err = oracle.matrix_norm_1(X, got)
    tol = oracle.trsm_tolerance(dt, max(m, n))
    assert err <= tol, (side, uplo, trans, diag, m, n, err, tol)
    # rows between m and ldb are not written
    if B.shape[0] > m:
        assert np.isnan(Bout[m:]).all()
    return err


SMALL = [(10, 10, 20, 100), (24, 33, 33, 33), (32, 33, 33, 33), (33, 32, 33, 33), (64, 65, 65, 65),
         (65, 64, 65, 65), (1, 2, 30, 30), (2, 1, 30, 30), (32, 3, 32, 32), (35, 7, 48, 52),
         (3, 61, 62, 63), (7, 58, 59, 130)]
MEDIUM = [(129, 129, 129, 129), (192, 192, 192, 192), (600, 500, 600, 600), (800, 700, 801, 701),
          (500, 32, 500, 500), (8, 128, 200, 200), (128, 8, 200, 200), (340, 128, 340, 340),
          (450, 19, 500, 500)]


def _sizes_for(side, sizes):
    out = []
    for (m, n, lda, ldb) in sizes:
        k = m if side == "L" else n
        out.append((m, n, max(lda, k), max(ldb, m)))
    return out


@pytest.mark.parametrize("dt", ["d", "s"])
@pytest.mark.parametrize("side,uplo,trans,diag", COMBOS)
def test_trsm_small_medium_all_combos(handle, dt, side, uplo, trans, diag):
    npdt, _ = DT[dt]
    for i, (m, n, lda, ldb) in enumerate(_sizes_for(side, SMALL + MEDIUM)):
        A, B = oracle.nan_triangle_problem(100 + i, side, uplo, trans, diag, m, n, lda, ldb, npdt)
        alpha = [1.0, -0.5, 2.0][i % 3]
        out, _ = _gpu_solve(handle, side, uplo, trans, diag, m, n, alpha, A, B)
        _check_vs_oracle(side, uplo, trans, diag, m, n, alpha, A, B, out, npdt)


@pytest.mark.parametrize("dt", ["d", "s"])
@pytest.mark.parametrize("side,uplo,trans,diag", COMBOS)
def test_trsm_rocblas_test_protocol(handle, dt, side, uplo, trans, diag):
    """testing_trsm's numerical check: X known, B = op(A) X / alpha, both gates."""
    npdt, _ = DT[dt]
    for i, (m, n, lda, ldb) in enumerate(_sizes_for(side, [(65, 64, 65, 65), (640, 640, 960, 960),
                                                          (1000, 1000, 1000, 1000), (192, 192, 192, 192)])):
        alpha = 1.0 if i % 2 else 2.5
        A, B, X = oracle.rocblas_test_problem(7 + i, side, uplo, trans, diag, m, n, lda, ldb, alpha, npdt)
        out, _ = _gpu_solve(handle, side, uplo, trans, diag, m, n, alpha, A, B)
        got = out[:m]
        tol = oracle.trsm_tolerance(npdt, m)
        err = oracle.matrix_norm_1(X, got)
        assert err <= tol, ("forward", m, n, err, tol)
        res = oracle.trmm(side, uplo, trans, diag, 1.0 / alpha, A, got)
        err_res = oracle.matrix_norm_1(np.asfortranarray(B[:m]), res)
        assert err_res <= tol, ("residual", m, n, err_res, tol)


@pytest.mark.parametrize("dt", ["d", "s"])
def test_trsm_against_cblas_golden(handle, dt):
    npdt, _ = DT[dt]
    z = np.load(os.path.join(GOLDEN, f"cblas_{dt}.npz"))
    keys = sorted({k.rsplit("_", 1)[0] for k in z.files})
    for key in keys:
        combo, shape = key.split("_")
        side, uplo, trans, diag = combo
        m, n = map(int, shape.split("x"))
        A, B, X, alpha = z[key + "_A"], z[key + "_B"], z[key + "_X"], float(z[key + "_alpha"])
        out, _ = _gpu_solve(handle, side, uplo, trans, diag, m, n, alpha, A, B)
        err = oracle.matrix_norm_1(X, out[:m])
        assert err <= oracle.trsm_tolerance(npdt, max(m, n)), (key, err)


@pytest.mark.parametrize("side,uplo,trans,diag", [("L", "L", "N", "N"), ("R", "U", "T", "U"),
                                                  ("L", "U", "T", "N"), ("R", "L", "N", "N")])
def test_trsm_device_pointer_mode(handle, side, uplo, trans, diag):
    m, n = 300, 200
    k = m if side == "L" else n
    A, B = oracle.nan_triangle_problem(3, side, uplo, trans, diag, m, n, k, m, np.float64)
    out, _ = _gpu_solve(handle, side, uplo, trans, diag, m, n, -1.25, A, B, alpha_on_device=True)
    _check_vs_oracle(side, uplo, trans, diag, m, n, -1.25, A, B, out, np.float64)


@pytest.mark.parametrize("on_device", [False, True])
@pytest.mark.parametrize("m,n", [(64, 50), (700, 300)])
def test_trsm_alpha_zero(handle, on_device, m, n):
    """alpha == 0: B := 0 and neither A nor B is read (rocblas-functions.h trsm docs;
    testing_trsm.hpp:423-432).  A and B are all NaN here."""
    A = np.full((m, m), np.nan, order="F")
    B = np.full((m + 3, n), np.nan, order="F")
    out, _ = _gpu_solve(handle, "L", "L", "N", "N", m, n, 0.0, A, B, alpha_on_device=on_device)
    assert np.all(out[:m] == 0.0)
    assert np.isnan(out[m:]).all()


def test_trsm_large_left_property(handle):
    """A size the oracle cannot check quickly: residual of op(A) X = alpha B in fp64 on the
    GPU (torch matmul as the checker) for the recursive path, all orientations of side L."""
    m, n = 3000, 257
    for (uplo, trans) in [("L", "N"), ("U", "N"), ("L", "T"), ("U", "T")]:
        A, B = oracle.nan_triangle_problem(9, "L", uplo, trans, "N", m, n, m, m, np.float64)
        out, _ = _gpu_solve(handle, "L", uplo, trans, "N", m, n, 1.0, A, B)
        T = torch.from_numpy(oracle.clean_triangle(A, m, uplo, "N")).cuda()
        opT = T if trans == "N" else T.T
        X = torch.from_numpy(np.ascontiguousarray(out)).cuda()
        R = opT @ X - torch.from_numpy(np.ascontiguousarray(B)).cuda()
        rel = (R.abs().sum() / (opT.abs() @ X.abs()).sum()).item()
        assert rel < 1e-13, (uplo, trans, rel)


@pytest.mark.parametrize("dt", ["d", "s"])
def test_trsm_strided_batched(handle, dt):
    npdt, tdt = DT[dt]
    batch, m, n = 37, 128, 32
    for side, uplo, trans, diag in [("L", "L", "N", "N"), ("R", "U", "T", "U"), ("L", "U", "N", "U"),
                                    ("R", "L", "T", "N")]:
        k = m if side == "L" else n
        lda, ldb = k + 1, m + 2
        sa, sb = lda * k + 5, ldb * n + 3
        As, Bs = [], []
        for b in range(batch):
            A, B = oracle.nan_triangle_problem(50 + b, side, uplo, trans, diag, m, n, lda, ldb, npdt)
            As.append(A)
            Bs.append(B)
        dA = torch.full((batch * sa,), float("nan"), dtype=tdt, device="cuda")
        dB = torch.full((batch * sb,), float("nan"), dtype=tdt, device="cuda")
        for b in range(batch):
            dA[b * sa: b * sa + lda * k] = torch.from_numpy(As[b].ravel(order="F")).cuda()
            dB[b * sb: b * sb + ldb * n] = torch.from_numpy(Bs[b].ravel(order="F")).cuda()
        dm.trsm_strided_batched(handle, side, uplo, trans, diag, m, n, 0.5, dA, lda, sa, dB, ldb, sb, batch)
        torch.cuda.synchronize()
        hB = dB.cpu().numpy()
        for b in range(batch):
            out = hB[b * sb: b * sb + ldb * n].reshape((ldb, n), order="F")
            _check_vs_oracle(side, uplo, trans, diag, m, n, 0.5, As[b], Bs[b], out, npdt)
            if b + 1 < batch:
                assert np.isnan(hB[b * sb + ldb * n: (b + 1) * sb]).all()


@pytest.mark.parametrize("dt", ["d", "s"])
def test_trsm_batched_pointer_arrays(handle, dt):
    npdt, _ = DT[dt]
    batch = 9
    for (side, uplo, trans, diag, m, n) in [("L", "L", "T", "N", 300, 40), ("R", "U", "N", "N", 50, 600),
                                            ("L", "U", "N", "U", 40, 40)]:
        k = m if side == "L" else n
        probs = [oracle.nan_triangle_problem(200 + b, side, uplo, trans, diag, m, n, k, m, npdt)
                 for b in range(batch)]
        dAs = [dm.to_device(A) for A, _ in probs]
        dBs = [dm.to_device(B) for _, B in probs]
        dm.trsm_batched(handle, side, uplo, trans, diag, m, n, 1.5, dAs, k, dBs, m)
        for b in range(batch):
            _check_vs_oracle(side, uplo, trans, diag, m, n, 1.5, probs[b][0], probs[b][1],
                             dm.to_host(dBs[b]), npdt)


@pytest.mark.parametrize("dt", ["d", "s"])
@pytest.mark.parametrize("uplo,diag", [("L", "N"), ("U", "N"), ("L", "U"), ("U", "U")])
def test_trtri_blocks_match_oracle(handle, dt, uplo, diag):
    npdt, tdt = DT[dt]
    for n in [1, 5, 31, 32, 33, 100, 128, 129, 300, 513]:
        A, _ = oracle.nan_triangle_problem(n, "L", uplo, "N", diag, n, 1, n + 2, n, npdt)
        dA = dm.to_device(A)
        dInv = dm.empty(n, n, tdt)
        dm.trtri(handle, uplo, diag, n, dA, n + 2, dInv, n)
        torch.cuda.synchronize()
        inv = dm.to_host(dInv)
        ref = oracle.trtri(uplo, diag, A, n)
        tri = np.tril if uplo == "L" else np.triu
        got = tri(inv)
        err = np.abs(got - ref).max() / np.abs(ref).max()
        assert err < (1e-13 if dt == "d" else 2e-5), (n, err)
        # the diagonal blocks' opposite triangles are cleared
        for b0 in range(0, n, 128):
            blk = inv[b0:b0 + 128, b0:b0 + 128]
            opp = np.triu(blk, 1) if uplo == "L" else np.tril(blk, -1)
            assert np.all(opp == 0)


@pytest.mark.parametrize("dt", ["d", "s"])
@pytest.mark.parametrize("side,uplo,trans,diag", [("L", "L", "N", "N"), ("L", "U", "T", "U"),
                                                  ("R", "U", "N", "N"), ("R", "L", "T", "U")])
def test_trsm_ex_with_supplied_invA(handle, dt, side, uplo, trans, diag):
    """_ex with invA built by trtri_strided_batched the way testing_trsm_ex does."""
    npdt, _ = DT[dt]
    m, n = (700, 300) if side == "L" else (300, 700)
    k = m if side == "L" else n
    A, B = oracle.nan_triangle_problem(77, side, uplo, trans, diag, m, n, k, m, npdt)
    dA, dB = dm.to_device(A), dm.to_device(B)
    invA = dm.build_invA(handle, uplo, diag, dA, k, k)
    # invA against the oracle's packed blocks
    ref = oracle.invA_blocks(uplo, diag, A, k)
    got = invA.cpu().numpy()
    assert np.allclose(got, ref, rtol=0, atol=(1e-12 if dt == "d" else 1e-4) * np.abs(ref).max())
    st = dm.trsm_ex(handle, side, uplo, trans, diag, m, n, 0.75, dA, k, dB, m, invA, 128 * k)
    torch.cuda.synchronize()
    assert st == rb.status_success
    _check_vs_oracle(side, uplo, trans, diag, m, n, 0.75, A, B, dm.to_host(dB), npdt)
    # too small an invA is ignored with perf_degraded (rocblas_trsm_kernels.hpp:3832-3836)
    dB2 = dm.to_device(B)
    st = dm.trsm_ex(handle, side, uplo, trans, diag, m, n, 0.75, dA, k, dB2, m, invA, 128 * k - 1,
                    allow=(rb.status_perf_degraded,))
    torch.cuda.synchronize()
    _check_vs_oracle(side, uplo, trans, diag, m, n, 0.75, A, B, dm.to_host(dB2), npdt)


def test_trsm_without_workspace_is_degraded_but_correct(handle):
    """A user workspace too small for invA: the backup path (block-solver leaves) runs and the
    call reports perf_degraded, as rocblas_trsm_kernels.hpp:1926-1944 does."""
    import ctypes

    m, n = 900, 100
    A, B = oracle.nan_triangle_problem(5, "L", "L", "N", "N", m, n, m, m, np.float64)
    small = torch.empty(64, dtype=torch.uint8, device="cuda")
    with rb.Handle() as h:
        assert rb.lib().rocblas_set_workspace(h.value, ctypes.c_void_p(small.data_ptr()), 64) == 0
        out, st = _gpu_solve(h, "L", "L", "N", "N", m, n, 1.0, A, B, allow=(rb.status_perf_degraded,))
        assert st == rb.status_perf_degraded
        _check_vs_oracle("L", "L", "N", "N", m, n, 1.0, A, B, out, np.float64)


def test_size_query_then_fixed_memory(handle):
    """rocblas-test's flow: query, set_device_memory_size, run (testing_trsm.hpp:327-340)."""
    import ctypes

    m, n = 1024, 64
    A, B = oracle.nan_triangle_problem(6, "R", "U", "N", "N", n, m, m, n, np.float64)
    with rb.Handle() as h:
        L = rb.lib()
        assert L.rocblas_start_device_memory_size_query(h.value) == 0
        one = ctypes.c_double(1.0)
        st = L.rocblas_dtrsm(h.value, rb.side_right, rb.fill_upper, rb.operation_none,
                             rb.diagonal_non_unit, n, m, ctypes.cast(ctypes.byref(one), ctypes.c_void_p),
                             None, m, None, n)
        assert st == rb.status_size_increased
        size = ctypes.c_size_t(0)
        assert L.rocblas_stop_device_memory_size_query(h.value, ctypes.byref(size)) == 0
        # invA for the 1024-order triangle, plus the flags of the chain solve (64 columns)
        assert 128 * m * 8 <= size.value <= 128 * m * 8 + 4096
        assert L.rocblas_set_device_memory_size(h.value, size.value) == 0
        assert L.rocblas_is_user_managing_device_memory(h.value)
        out, st = _gpu_solve(h, "R", "U", "N", "N", n, m, 1.0, A, B)
        assert st == rb.status_success
        _check_vs_oracle("R", "U", "N", "N", n, m, 1.0, A, B, out, np.float64)


def test_repeatability_bitwise(handle):
    """trsm_gtest.yaml:1311-1334: repeated runs are bitwise identical (no atomics)."""
    m, n = 1500, 300
    A, B = oracle.nan_triangle_problem(8, "L", "U", "T", "N", m, n, m, m, np.float64)
    first, _ = _gpu_solve(handle, "L", "U", "T", "N", m, n, 1.0, A, B)
    for _ in range(3):
        again, _ = _gpu_solve(handle, "L", "U", "T", "N", m, n, 1.0, A, B)
        assert np.array_equal(first, again, equal_nan=True)


def test_graph_capture_host_and_device_mode(handle):
    """trsm_gtest.yaml:1288-1309: the call can be captured into a CUDA graph; with alpha on
    the device there is no host synchronisation to break the capture."""
    m, n = 600, 200
    A, B = oracle.nan_triangle_problem(12, "L", "L", "N", "N", m, n, m, m, np.float64)
    dA, dB = dm.to_device(A), dm.to_device(B)
    alpha = torch.tensor([1.0], dtype=torch.float64, device="cuda")
    s = torch.cuda.Stream()
    with rb.Handle() as h:
        import ctypes
        L = rb.lib()
        # reserve workspace before capture (allocation is not capturable): invA plus the
        # chain solve's flags
        assert L.rocblas_set_device_memory_size(h.value, 128 * m * 8 + 4096) == 0
        h.set_stream(ctypes.c_void_p(s.cuda_stream))
        h.set_pointer_mode(rb.pointer_mode_device)
        g = torch.cuda.CUDAGraph()
        torch.cuda.synchronize()
        with torch.cuda.graph(g, stream=s):
            st = L.rocblas_dtrsm(h.value, rb.side_left, rb.fill_lower, rb.operation_none,
                                 rb.diagonal_non_unit, m, n, ctypes.c_void_p(alpha.data_ptr()),
                                 ctypes.c_void_p(dA.data_ptr()), m, ctypes.c_void_p(dB.data_ptr()), m)
        assert st == 0
        g.replay()
        torch.cuda.synchronize()
        _check_vs_oracle("L", "L", "N", "N", m, n, 1.0, A, B, dm.to_host(dB), np.float64)
        del g


@pytest.mark.parametrize("dt", ["d", "s"])
@pytest.mark.parametrize("side,uplo,trans,diag", COMBOS)
def test_trsm_large_all_combos_residual(handle, dt, side, uplo, trans, diag):
    """Sizes the oracle cannot check quickly (the drop-in sweep's shapes scaled down to
    m = 2500, n = 300 and the transpose): the normwise residual of the solve in FP64 on the GPU
    (torch as the checker), for every combination through the chain solve (FP64) and the
    recursive solve (FP32 with more than 512 columns)."""
    npdt, tdt = DT[dt]
    for (m, n) in [(2500, 300), (300, 2500)]:
        k = m if side == "L" else n
        A, B = oracle.nan_triangle_problem(4242, side, uplo, trans, diag, m, n, k, m, npdt)
        out, _ = _gpu_solve(handle, side, uplo, trans, diag, m, n, -0.5, A, B)
        T = torch.from_numpy(oracle.clean_triangle(A, k, uplo, diag).astype(np.float64)).cuda()
        opT = T if trans == "N" else T.T
        X = torch.from_numpy(np.ascontiguousarray(out[:m]).astype(np.float64)).cuda()
        Bd = torch.from_numpy(np.ascontiguousarray(B[:m]).astype(np.float64)).cuda()
        R = (opT @ X if side == "L" else X @ opT) + 0.5 * Bd
        scale = (opT.abs() @ X.abs() if side == "L" else X.abs() @ opT.abs()).sum()
        rel = (R.abs().sum() / scale).item()
        assert rel < (1e-13 if dt == "d" else 1e-4), (side, uplo, trans, diag, m, n, rel)
