"""The drop-in sweep at its stated size: rocblas_{s,d}trsm for all 16 side/uplo/trans/diag
combinations at m = n = 8192 and the rectangular 8192 x 512 and 512 x 8192 (the reference's
large gtest sizes, clients/gtest/trsm_gtest.yaml:57-61), and rocblas_trsm_ex with an invA of
NB = 128 built by rocblas_?trtri_strided_batched the way testing_trsm_ex.hpp:329-336 builds it.

A follows the drop-in recipe on the device (strict triangle U(-1,1)/k, diagonal 1 + U(0,1), the
other triangle NaN, a NaN diagonal for diag U).  Two checks per solve:
* the normwise residual ||op(A) X - alpha B|| / (|op(A)| |X|) in FP64 on the GPU (torch as the
  checker) over the whole solution;
* four right-hand sides (columns for side left, rows for side right) against the CPU oracle,
  with rocblas-test's gate 40 eps max(m, n) (testing_trsm.hpp:30-31)."""
import ctypes
import itertools

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle  # noqa: E402
import rocblas_b200 as rb  # noqa: E402

pytestmark = pytest.mark.gpu
COMBOS = list(itertools.product("LR", "UL", "NT", "NU"))
SHAPES = [(8192, 8192), (8192, 512), (512, 8192)]
DT = {"d": (torch.float64, np.float64, 1e-13), "s": (torch.float32, np.float32, 1e-4)}


@pytest.fixture(scope="module")
def handle():
    rb.build()
    h = rb.Handle()
    yield h
    h.close()


_cache = {}


def _matrix(k, uplo, diag, dt):
    """(At device (ncols, ld) view, A host Fortran) for the recipe, cached per (k, uplo, diag, dt)."""
    key = (k, uplo, diag, dt)
    if key not in _cache:
        if len(_cache) > 6:
            _cache.clear()
        tdt = DT[dt][0]
        g = torch.Generator(device="cuda")
        g.manual_seed(k * 8 + 4 * (uplo == "L") + 2 * (diag == "U") + (dt == "s"))
        At = (torch.rand(k, k, generator=g, device="cuda", dtype=torch.float64) * 2 - 1) / k
        At.diagonal().copy_(1.0 + torch.rand(k, generator=g, device="cuda", dtype=torch.float64))
        mask = torch.ones(k, k, dtype=torch.bool, device="cuda")
        mask = mask.tril_(-1) if uplo == "L" else mask.triu_(1)  # A's other triangle (At transposed)
        At.masked_fill_(mask, float("nan"))
        if diag == "U":
            At.diagonal().fill_(float("nan"))
        At = At.to(tdt).contiguous()
        _cache[key] = (At, np.asfortranarray(At.cpu().numpy().T))
    return _cache[key]


def _op_dense(At, uplo, diag, trans):
    """op(A) as a dense FP64 device matrix (row-major (i, j) = op(A)(i, j))."""
    A = At.double().T.clone()  # A(i, j)
    A = torch.nan_to_num(A, nan=0.0)
    A = A.tril() if uplo == "L" else A.triu()
    if diag == "U":
        A.fill_diagonal_(1.0)
    return A if trans == "N" else A.T


def _check(At, Ahost, Bt0, Bt, side, uplo, trans, diag, m, n, alpha, dt):
    opA = _op_dense(At, uplo, diag, trans)
    X = Bt.double().T  # (m, n)
    B = Bt0.double().T
    R = (opA @ X if side == "L" else X @ opA) - alpha * B
    scale = (opA.abs() @ X.abs() if side == "L" else X.abs() @ opA.abs()).sum()
    rel = (R.abs().sum() / scale).item()
    assert rel < DT[dt][2], (side, uplo, trans, diag, m, n, rel)
    # four right-hand sides against the oracle
    npdt = DT[dt][1]
    if side == "L":
        idx = np.linspace(0, n - 1, 4).round().astype(int)
        Bs = np.asfortranarray(Bt0[idx].cpu().numpy().T)  # the 4 sampled columns, m x 4
        got = Bt[idx].cpu().numpy().T
    else:
        idx = np.linspace(0, m - 1, 4).round().astype(int)
        Bs = np.asfortranarray(Bt0[:, idx].cpu().numpy().T)  # the 4 sampled rows, 4 x n
        got = Bt[:, idx].cpu().numpy().T
    Xo = oracle.trsm(side, uplo, trans, diag, alpha, Ahost, Bs)
    err = oracle.matrix_norm_1(Xo.astype(np.float64), got.astype(np.float64))
    assert err <= oracle.trsm_tolerance(npdt, max(m, n)), (side, uplo, trans, diag, m, n, err)
    assert not np.isnan(got).any()


@pytest.mark.parametrize("dt", ["d", "s"])
@pytest.mark.parametrize("side,uplo,trans,diag", COMBOS)
def test_sweep_all_combos_full_size(handle, dt, side, uplo, trans, diag):
    fn = getattr(rb.lib(), f"rocblas_{dt}trsm")
    alpha = -0.5
    a = ctypes.c_double(alpha) if dt == "d" else ctypes.c_float(alpha)
    for m, n in SHAPES:
        k = m if side == "L" else n
        At, Ahost = _matrix(k, uplo, diag, dt)
        g = torch.Generator(device="cuda")
        g.manual_seed(m * 7 + n)
        Bt0 = (torch.rand(n, m, generator=g, device="cuda", dtype=torch.float64) * 2 - 1).to(DT[dt][0])
        Bt = Bt0.clone()
        st = fn(handle.value, rb.SIDE[side], rb.UPLO[uplo], rb.TRANS[trans], rb.DIAG[diag], m, n,
                ctypes.cast(ctypes.byref(a), ctypes.c_void_p), ctypes.c_void_p(At.data_ptr()), k,
                ctypes.c_void_p(Bt.data_ptr()), m)
        assert st == 0, st
        torch.cuda.synchronize()
        _check(At, Ahost, Bt0, Bt, side, uplo, trans, diag, m, n, alpha, dt)


@pytest.mark.parametrize("dt", ["d", "s"])
@pytest.mark.parametrize("side,uplo,trans,diag", COMBOS)
def test_sweep_ex_with_trtri_invA(handle, dt, side, uplo, trans, diag):
    """rocblas_trsm_ex at m = n = 8192 with the caller's invA: 64 blocks of 128 x 128 from
    rocblas_?trtri_strided_batched over A's diagonal blocks (stride 128 lda + 128)."""
    L = rb.lib()
    m = n = 8192
    alpha = 1.25
    a = ctypes.c_double(alpha) if dt == "d" else ctypes.c_float(alpha)
    At, Ahost = _matrix(m, uplo, diag, dt)
    inv = torch.zeros(128 * m, dtype=DT[dt][0], device="cuda")
    tri = getattr(L, f"rocblas_{dt}trtri_strided_batched")
    assert tri(handle.value, rb.UPLO[uplo], rb.DIAG[diag], 128, ctypes.c_void_p(At.data_ptr()), m, 128 * m + 128,
               ctypes.c_void_p(inv.data_ptr()), 128, 128 * 128, m // 128) == 0
    g = torch.Generator(device="cuda")
    g.manual_seed(31)
    Bt0 = (torch.rand(n, m, generator=g, device="cuda", dtype=torch.float64) * 2 - 1).to(DT[dt][0])
    Bt = Bt0.clone()
    st = L.rocblas_trsm_ex(handle.value, rb.SIDE[side], rb.UPLO[uplo], rb.TRANS[trans], rb.DIAG[diag], m, n,
                           ctypes.cast(ctypes.byref(a), ctypes.c_void_p), ctypes.c_void_p(At.data_ptr()), m,
                           ctypes.c_void_p(Bt.data_ptr()), m, ctypes.c_void_p(inv.data_ptr()), 128 * m,
                           rb.datatype_f64_r if dt == "d" else rb.datatype_f32_r)
    assert st == 0, st
    torch.cuda.synchronize()
    _check(At, Ahost, Bt0, Bt, side, uplo, trans, diag, m, n, alpha, dt)
