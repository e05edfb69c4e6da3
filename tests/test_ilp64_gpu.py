"""The ILP64 (_64) entry points on the GPU.

* At ordinary sizes every _64 form gives bitwise the result of its 32-bit twin (they share one
  body; rocblas-test runs its trsm cases through both APIs the same way).
* Past 32 bits (src64/blas3/rocblas_trsm_kernels_64.cpp:31-225): a B with more than 2^31 rows
  (side right) or columns (side left), leading dimensions of A and B beyond 2^31, a trsv
  increment beyond 2^31 and a trmm with more than 2^31 rows.  These use FP32 buffers of 9 to
  35 GB; the solution is checked against the oracle on sampled rows or columns (each row of B
  is an independent system for side right, each column for side left), taken where the chunks
  of the 64-bit body meet and at the ends.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle  # noqa: E402
import rocblas_b200 as rb  # noqa: E402
from rocblas_b200 import devmem as dm  # noqa: E402

pytestmark = pytest.mark.gpu
T32 = 1 << 31


@pytest.fixture(scope="module")
def handle():
    rb.build()
    h = rb.Handle()
    yield h
    h.close()


@pytest.fixture(autouse=True)
def _release_memory():
    yield
    torch.cuda.synchronize()
    torch.cuda.empty_cache()


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _alpha(value, dt):
    c = ctypes.c_double(value) if dt == "d" else ctypes.c_float(value)
    return c, ctypes.cast(ctypes.byref(c), ctypes.c_void_p)


def _fn(name):
    return getattr(rb.lib(), name)


# ---- ordinary sizes: _64 == 32-bit, bitwise ------------------------------------------------
@pytest.mark.parametrize("dt", ["d", "s"])
@pytest.mark.parametrize("side,uplo,trans,diag", [("L", "L", "N", "N"), ("R", "U", "T", "U"),
                                                  ("L", "U", "T", "N"), ("R", "L", "N", "N")])
def test_trsm_64_matches_32(handle, dt, side, uplo, trans, diag):
    npdt = np.float64 if dt == "d" else np.float32
    m, n = 700, 300
    k = m if side == "L" else n
    A, B = oracle.nan_triangle_problem(41, side, uplo, trans, diag, m, n, k + 1, m + 2, npdt)
    keep, ap = _alpha(-1.25, dt)
    args = (rb.SIDE[side], rb.UPLO[uplo], rb.TRANS[trans], rb.DIAG[diag], m, n, ap)
    dA = dm.to_device(A)
    outs = []
    for name in (f"rocblas_{dt}trsm", f"rocblas_{dt}trsm_64"):
        dB = dm.to_device(B)
        assert _fn(name)(handle.value, *args, _ptr(dA), A.shape[0], _ptr(dB), B.shape[0]) == 0
        outs.append(dB)
    # strided batch of two through both forms: bitwise equal to each other; against the single
    # solve within rounding, since the batch count enters the engine choice (the block solver
    # takes over once the batch's strips fill the machine)
    sb = B.shape[0] * n
    batched = []
    for name in (f"rocblas_{dt}trsm_strided_batched", f"rocblas_{dt}trsm_strided_batched_64"):
        dB2 = torch.cat([dm.to_device(B).reshape(-1)] * 2)
        assert _fn(name)(handle.value, *args, _ptr(dA), A.shape[0], 0, _ptr(dB2), B.shape[0], sb, 2) == 0
        batched.append(dB2)
    torch.cuda.synchronize()
    ref = outs[0].cpu()
    assert torch.equal(outs[1].cpu().nan_to_num(7.0), ref.nan_to_num(7.0))
    assert torch.equal(batched[1].cpu().nan_to_num(7.0), batched[0].cpu().nan_to_num(7.0))
    rtol = 1e-12 if dt == "d" else 1e-4
    for b in range(2):
        got = batched[1][b * sb:(b + 1) * sb].view(n, B.shape[0]).cpu()
        assert torch.equal(got.isnan(), ref.isnan())
        g, r = got.nan_to_num(0.0), ref.nan_to_num(0.0)
        assert float((g - r).abs().max()) <= rtol * float(r.abs().max())


@pytest.mark.parametrize("dt", ["d", "s"])
def test_trsv_trmm_64_match_32(handle, dt):
    npdt = np.float64 if dt == "d" else np.float32
    n = 500
    A, B = oracle.nan_triangle_problem(43, "L", "U", "N", "N", n, 4, n, n, npdt)
    dA = dm.to_device(A)
    res = []
    for name in (f"rocblas_{dt}trsv", f"rocblas_{dt}trsv_64"):
        x = torch.from_numpy(np.ascontiguousarray(B[:, 0])).cuda()
        assert _fn(name)(handle.value, rb.UPLO["U"], rb.TRANS["N"], rb.DIAG["N"], n, _ptr(dA), n,
                         _ptr(x), 1) == 0
        res.append(x)
    for name in (f"rocblas_{dt}trmm", f"rocblas_{dt}trmm_64"):
        keep, ap = _alpha(0.5, dt)
        dB = dm.to_device(B)
        dC = torch.empty_like(dB)
        assert _fn(name)(handle.value, rb.SIDE["L"], rb.UPLO["U"], rb.TRANS["T"], rb.DIAG["N"], n, 4, ap,
                         _ptr(dA), n, _ptr(dB), n, _ptr(dC), n) == 0
        res.append(dC)
    torch.cuda.synchronize()
    assert torch.equal(res[0], res[1]) and torch.equal(res[2], res[3])


# ---- sizes past 32 bits (FP32) -------------------------------------------------------------
def _lower2(seed, k):
    """A k x k lower triangle (column-major, NaN above) of the drop-in recipe, as numpy."""
    A, _ = oracle.nan_triangle_problem(seed, "L", "L", "N", "N", k, 1, k, k, np.float32)
    return A


def _sample(total, chunk):
    rng = np.random.default_rng(5)
    picks = {0, 1, total - 1, total - 2}
    for c in range(chunk, total, chunk):
        picks.update({c - 1, c, c + 1})
    picks.update(int(v) for v in rng.integers(0, total, size=200))
    return np.array(sorted(p for p in picks if 0 <= p < total), dtype=np.int64)


def test_trsm_64_side_right_rows_past_int32(handle):
    m, n = T32 + 64, 2
    A = _lower2(51, n)
    dA = dm.to_device(A)
    g = torch.Generator(device="cuda")
    g.manual_seed(3)
    Bt = torch.rand((n, m), generator=g, device="cuda", dtype=torch.float32) * 2 - 1  # (col, row)
    rows = _sample(m, 1 << 28)
    idx = torch.from_numpy(rows).cuda()
    before = Bt[:, idx].cpu().numpy().T  # (s, n)
    keep, ap = _alpha(1.0, "s")
    st = rb.lib().rocblas_strsm_64(handle.value, rb.SIDE["R"], rb.UPLO["L"], rb.TRANS["N"], rb.DIAG["N"],
                                   m, n, ap, _ptr(dA), n, _ptr(Bt), m)
    assert st == 0
    torch.cuda.synchronize()
    got = Bt[:, idx].cpu().numpy().T
    X = oracle.trsm("R", "L", "N", "N", 1.0, A, np.asfortranarray(before))
    assert oracle.matrix_norm_1(X, np.asfortranarray(got)) <= oracle.trsm_tolerance(np.float32, n)


def test_trsm_64_side_left_columns_past_int32(handle):
    m, n = 2, T32 + 64
    A = _lower2(52, m)
    dA = dm.to_device(A)
    g = torch.Generator(device="cuda")
    g.manual_seed(4)
    Bt = torch.rand((n, m), generator=g, device="cuda", dtype=torch.float32) * 2 - 1  # (col, row)
    cols = _sample(n, 1 << 20)
    idx = torch.from_numpy(cols).cuda()
    before = Bt[idx, :].cpu().numpy().T  # (m, s)
    keep, ap = _alpha(-0.5, "s")
    st = rb.lib().rocblas_strsm_64(handle.value, rb.SIDE["L"], rb.UPLO["L"], rb.TRANS["T"], rb.DIAG["N"],
                                   m, n, ap, _ptr(dA), m, _ptr(Bt), m)
    assert st == 0
    torch.cuda.synchronize()
    got = Bt[idx, :].cpu().numpy().T
    X = oracle.trsm("L", "L", "T", "N", -0.5, A, np.asfortranarray(before))
    assert oracle.matrix_norm_1(X, np.asfortranarray(got)) <= oracle.trsm_tolerance(np.float32, m)


def test_trsm_64_leading_dimensions_past_int32(handle):
    keep, ap = _alpha(1.0, "s")
    # ldb > 2^31: side left, m = 100, n = 2
    m, n, ldb = 100, 2, T32 + 3
    A, B = oracle.nan_triangle_problem(53, "L", "U", "N", "N", m, n, m, m, np.float32)
    dA = dm.to_device(A)
    buf = torch.full((ldb * (n - 1) + m + 1,), float("nan"), device="cuda", dtype=torch.float32)
    for j in range(n):
        buf[j * ldb: j * ldb + m] = torch.from_numpy(np.ascontiguousarray(B[:, j])).cuda()
    assert rb.lib().rocblas_strsm_64(handle.value, rb.SIDE["L"], rb.UPLO["U"], rb.TRANS["N"], rb.DIAG["N"],
                                     m, n, ap, _ptr(dA), m, _ptr(buf), ldb) == 0
    torch.cuda.synchronize()
    got = np.stack([buf[j * ldb: j * ldb + m].cpu().numpy() for j in range(n)], axis=1)
    X = oracle.trsm("L", "U", "N", "N", 1.0, A, B[:m])
    assert oracle.matrix_norm_1(X, np.asfortranarray(got)) <= oracle.trsm_tolerance(np.float32, m)
    assert torch.isnan(buf[m]).item() and torch.isnan(buf[ldb - 1]).item()
    assert torch.isnan(buf[ldb + m]).item()
    del buf
    torch.cuda.empty_cache()
    # lda > 2^31: side right, n = k = 3, m = 50
    m, n, lda = 50, 3, T32 + 1
    A, B = oracle.nan_triangle_problem(54, "R", "L", "T", "N", m, n, n, m, np.float32)
    abuf = torch.full((lda * (n - 1) + n,), float("nan"), device="cuda", dtype=torch.float32)
    for j in range(n):
        abuf[j * lda: j * lda + n] = torch.from_numpy(np.ascontiguousarray(A[:n, j])).cuda()
    dB = dm.to_device(B)
    assert rb.lib().rocblas_strsm_64(handle.value, rb.SIDE["R"], rb.UPLO["L"], rb.TRANS["T"], rb.DIAG["N"],
                                     m, n, ap, _ptr(abuf), lda, _ptr(dB), m) == 0
    torch.cuda.synchronize()
    X = oracle.trsm("R", "L", "T", "N", 1.0, A, B)
    assert oracle.matrix_norm_1(X, dm.to_host(dB)) <= oracle.trsm_tolerance(np.float32, n)


def test_trsv_64_increment_past_int32(handle):
    n, incx = 3, T32 + 1
    A, B = oracle.nan_triangle_problem(55, "L", "L", "T", "N", n, 1, n, n, np.float32)
    dA = dm.to_device(A)
    buf = torch.full((incx * (n - 1) + 1,), float("nan"), device="cuda", dtype=torch.float32)
    for i in range(n):
        buf[i * incx] = float(B[i, 0])
    assert rb.lib().rocblas_strsv_64(handle.value, rb.UPLO["L"], rb.TRANS["T"], rb.DIAG["N"], n,
                                     _ptr(dA), n, _ptr(buf), incx) == 0
    torch.cuda.synchronize()
    got = np.array([buf[i * incx].item() for i in range(n)], dtype=np.float32).reshape(n, 1)
    X = oracle.trsm("L", "L", "T", "N", 1.0, A, np.asfortranarray(B[:, :1]))
    assert oracle.matrix_norm_1(X, np.asfortranarray(got)) <= oracle.trsm_tolerance(np.float32, n)
    assert torch.isnan(buf[1]).item() and torch.isnan(buf[incx - 1]).item()


def test_trmm_64_rows_past_int32(handle):
    m, n = T32 + 64, 2
    A = _lower2(56, n)
    dA = dm.to_device(A)
    g = torch.Generator(device="cuda")
    g.manual_seed(6)
    Bt = torch.rand((n, m), generator=g, device="cuda", dtype=torch.float32) * 2 - 1
    Ct = torch.empty_like(Bt)
    keep, ap = _alpha(1.5, "s")
    assert rb.lib().rocblas_strmm_64(handle.value, rb.SIDE["R"], rb.UPLO["L"], rb.TRANS["N"], rb.DIAG["N"],
                                     m, n, ap, _ptr(dA), n, _ptr(Bt), m, _ptr(Ct), m) == 0
    torch.cuda.synchronize()
    rows = _sample(m, 1 << 28)
    idx = torch.from_numpy(rows).cuda()
    Bs = Bt[:, idx].cpu().numpy().T
    got = Ct[:, idx].cpu().numpy().T
    ref = oracle.trmm("R", "L", "N", "N", 1.5, A, np.asfortranarray(Bs))
    assert np.max(np.abs(got - ref)) <= 1e-5
