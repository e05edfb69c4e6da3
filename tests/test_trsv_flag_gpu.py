"""The memory-bound single-vector solve (rocblas_?trsv with one vector and a positive increment,
order >= trsv_flag_min_n): flag-synchronised row blocks of 64 over a persistent grid.

* every uplo / transA / diag combination, FP64 and FP32, blocks of 64 and 128 rows, orders that
  are and are not multiples of the block, increments 1 and 3, against the oracle at the
  rocblas-test gate;
* the same solve through the blocked trsm path (trsv_flag_min_n above the order) agrees;
* a large order against a GPU residual, and bitwise repeatability.
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

pytestmark = pytest.mark.gpu
COMBOS = list(itertools.product("UL", "NTC", "NU"))
DT = {"d": (np.float64, torch.float64), "s": (np.float32, torch.float32)}


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


def _trsv(h, dt, uplo, trans, diag, n, A, b, incx):
    buf = np.full(1 + (n - 1) * incx + 2, np.nan, dtype=b.dtype)
    buf[0:(n - 1) * incx + 1:incx] = b
    dA = dm.to_device(A)
    dx = torch.from_numpy(buf).cuda()
    fn = getattr(rb.lib(), f"rocblas_{dt}trsv")
    st = fn(h.value, rb.UPLO[uplo], rb.TRANS[trans], rb.DIAG[diag], n, ctypes.c_void_p(dA.data_ptr()),
            A.shape[0], ctypes.c_void_p(dx.data_ptr()), incx)
    assert st == 0, st
    torch.cuda.synchronize()
    code = ctypes.c_int(-1)
    assert rb.lib().rocblas_b200_get_device_error(h.value, ctypes.byref(code)) == 0
    assert code.value == 0
    out = dx.cpu().numpy()
    gaps = np.ones(out.shape[0], dtype=bool)
    gaps[0:(n - 1) * incx + 1:incx] = False
    assert np.isnan(out[gaps]).all()  # nothing between the vector's elements is written
    return out[0:(n - 1) * incx + 1:incx].copy()


@pytest.mark.parametrize("nb", [64, 128])
@pytest.mark.parametrize("dt", ["d", "s"])
@pytest.mark.parametrize("uplo,trans,diag", COMBOS)
def test_trsv_flag_combos(dt, uplo, trans, diag, nb):
    npdt, _ = DT[dt]
    with rb.Handle() as h, tuning(trsv_flag_nb=nb):
        for i, (n, incx) in enumerate([(256, 1), (1000, 3), (4097, 1)]):
            A, B = oracle.nan_triangle_problem(900 + i, "L", uplo, trans, diag, n, 1, n + 2, n, npdt)
            b = B[:, 0].copy()
            got = _trsv(h, dt, uplo, trans, diag, n, A, b, incx)
            X = oracle.trsm("L", uplo, trans, diag, 1.0, A, np.asfortranarray(b.reshape(n, 1)))
            err = oracle.matrix_norm_1(X, np.asfortranarray(got.reshape(n, 1)))
            assert err <= oracle.trsm_tolerance(npdt, n), (n, incx, err)
            with tuning(trsv_flag_min_n=1 << 30):
                blocked = _trsv(h, dt, uplo, trans, diag, n, A, b, incx)
            err2 = oracle.matrix_norm_1(blocked.reshape(n, 1), np.asfortranarray(got.reshape(n, 1)))
            assert err2 <= oracle.trsm_tolerance(npdt, n), (n, incx, err2)


@pytest.mark.parametrize("uplo,trans", [("L", "N"), ("U", "T")])
def test_trsv_flag_large_residual_and_repeatable(uplo, trans):
    n = 16384
    g = torch.Generator(device="cuda").manual_seed(3)
    T = torch.rand(n, n, generator=g, device="cuda", dtype=torch.float64) * 2 - 1
    T = torch.tril(T) / n if uplo == "L" else torch.triu(T) / n
    T.diagonal().add_(1.5)
    Acm = T.t().contiguous()  # column-major storage of T
    b = torch.rand(n, generator=g, device="cuda", dtype=torch.float64) * 2 - 1
    L = rb.lib()
    outs = []
    with rb.Handle() as h:
        for _ in range(2):
            x = b.clone()
            st = L.rocblas_dtrsv(h.value, rb.UPLO[uplo], rb.TRANS[trans], rb.DIAG["N"], n,
                                 ctypes.c_void_p(Acm.data_ptr()), n, ctypes.c_void_p(x.data_ptr()), 1)
            assert st == 0, st
            torch.cuda.synchronize()
            outs.append(x)
    assert torch.equal(outs[0], outs[1])
    opT = T if trans == "N" else T.t()
    r = opT @ outs[0] - b
    rel = (r.abs().max() / (opT.abs() @ outs[0].abs()).max()).item()
    assert rel < 1e-14, rel
