"""rocblas_?trsv (x := op(A)^-1 x) against the oracle's trsm with one right-hand side:
uplo / transA / diag combinations, positive and negative increments (a negative increment
traverses x backwards, as in the reference BLAS), the batched forms, and the argument rules
of rocblas_trsv_arg_check (library/src/blas2/rocblas_trsv.hpp:31-80)."""
import ctypes
import itertools

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle  # noqa: E402
import rocblas_b200 as rb  # noqa: E402
from rocblas_b200 import devmem as dm  # noqa: E402

pytestmark = pytest.mark.gpu
COMBOS = list(itertools.product("UL", "NT", "NU"))
DT = {"d": (np.float64, torch.float64), "s": (np.float32, torch.float32)}


def _fn(name, dt):
    return getattr(rb.lib(), f"rocblas_{dt}{name}")


def _vec_layout(b, incx):
    """A strided buffer holding vector b with increment incx (backwards for incx < 0)."""
    n = b.shape[0]
    buf = np.full(1 + (n - 1) * abs(incx) + 2, np.nan, dtype=b.dtype)
    for i in range(n):
        buf[(n - 1 - i) * abs(incx) if incx < 0 else i * incx] = b[i]
    return buf


def _vec_read(buf, n, incx):
    return np.array([buf[(n - 1 - i) * abs(incx) if incx < 0 else i * incx] for i in range(n)])


@pytest.mark.parametrize("dt", ["d", "s"])
@pytest.mark.parametrize("uplo,trans,diag", COMBOS)
def test_trsv_combos_and_increments(dt, uplo, trans, diag):
    npdt, tdt = DT[dt]
    with rb.Handle() as h:
        for i, (n, incx) in enumerate([(50, 1), (700, 3), (130, -2), (1, 1), (600, -1)]):
            A, B = oracle.nan_triangle_problem(800 + i, "L", uplo, trans, diag, n, 1, n + 1, n, npdt)
            b = B[:, 0].copy()
            buf = _vec_layout(b, incx)
            dA = dm.to_device(A)
            dx = torch.from_numpy(buf).cuda()
            st = _fn("trsv", dt)(h.value, rb.UPLO[uplo], rb.TRANS[trans], rb.DIAG[diag], n,
                                 ctypes.c_void_p(dA.data_ptr()), A.shape[0], ctypes.c_void_p(dx.data_ptr()), incx)
            assert st == 0, st
            torch.cuda.synchronize()
            out = dx.cpu().numpy()
            got = _vec_read(out, n, incx)
            X = oracle.trsm("L", uplo, trans, diag, 1.0, A, np.asfortranarray(b.reshape(n, 1)))
            err = oracle.matrix_norm_1(X, np.asfortranarray(got.reshape(n, 1)))
            assert err <= oracle.trsm_tolerance(npdt, n), (n, incx, err)
            # entries between the vector's elements are untouched
            mask = np.ones(out.shape[0], dtype=bool)
            for j in range(n):
                mask[(n - 1 - j) * abs(incx) if incx < 0 else j * incx] = False
            assert np.isnan(out[mask]).all()


@pytest.mark.parametrize("dt", ["d", "s"])
def test_trsv_strided_and_pointer_batches(dt):
    npdt, tdt = DT[dt]
    batch, n, incx = 4, 300, 2
    probs = [oracle.nan_triangle_problem(900 + b, "L", "U", "T", "N", n, 1, n, n, npdt) for b in range(batch)]
    with rb.Handle() as h:
        # strided
        sa, sx = n * n + 7, 2 * n + 5
        dA = torch.full((batch * sa,), float("nan"), dtype=tdt, device="cuda")
        dx = torch.full((batch * sx,), float("nan"), dtype=tdt, device="cuda")
        for b, (A, B) in enumerate(probs):
            dA[b * sa: b * sa + n * n] = torch.from_numpy(A.ravel(order="F")).cuda()
            v = _vec_layout(B[:, 0], incx)
            dx[b * sx: b * sx + v.shape[0]] = torch.from_numpy(v).cuda()
        st = _fn("trsv_strided_batched", dt)(h.value, rb.UPLO["U"], rb.TRANS["T"], rb.DIAG["N"], n,
                                             ctypes.c_void_p(dA.data_ptr()), n, sa,
                                             ctypes.c_void_p(dx.data_ptr()), incx, sx, batch)
        assert st == 0, st
        torch.cuda.synchronize()
        hx = dx.cpu().numpy()
        for b, (A, B) in enumerate(probs):
            got = _vec_read(hx[b * sx:], n, incx)
            X = oracle.trsm("L", "U", "T", "N", 1.0, A, np.asfortranarray(B[:, :1]))
            assert oracle.matrix_norm_1(X, np.asfortranarray(got.reshape(n, 1))) <= oracle.trsm_tolerance(npdt, n)
        # pointer arrays, negative increment
        As = [dm.to_device(A) for A, _ in probs]
        xs = [torch.from_numpy(_vec_layout(B[:, 0], -3)).cuda() for _, B in probs]
        Ap = torch.tensor([a.data_ptr() for a in As], dtype=torch.int64, device="cuda")
        xp = torch.tensor([x.data_ptr() for x in xs], dtype=torch.int64, device="cuda")
        st = _fn("trsv_batched", dt)(h.value, rb.UPLO["U"], rb.TRANS["T"], rb.DIAG["N"], n,
                                     ctypes.c_void_p(Ap.data_ptr()), n, ctypes.c_void_p(xp.data_ptr()), -3, batch)
        assert st == 0, st
        torch.cuda.synchronize()
        for (A, B), x in zip(probs, xs):
            got = _vec_read(x.cpu().numpy(), n, -3)
            X = oracle.trsm("L", "U", "T", "N", 1.0, A, np.asfortranarray(B[:, :1]))
            assert oracle.matrix_norm_1(X, np.asfortranarray(got.reshape(n, 1))) <= oracle.trsm_tolerance(npdt, n)


def test_trsv_arguments():
    L = rb.lib()
    x = torch.zeros(64, dtype=torch.float64, device="cuda")
    X = ctypes.c_void_p(x.data_ptr())
    with rb.Handle() as h:
        assert L.rocblas_dtrsv(None, 122, 111, 131, 4, X, 4, X, 1) == rb.status_invalid_handle
        assert L.rocblas_dtrsv(h.value, 120, 111, 131, 4, X, 4, X, 1) == rb.status_invalid_value
        assert L.rocblas_dtrsv(h.value, 122, 111, 131, 4, X, 3, X, 1) == rb.status_invalid_size
        assert L.rocblas_dtrsv(h.value, 122, 111, 131, 4, X, 4, X, 0) == rb.status_invalid_size
        assert L.rocblas_dtrsv(h.value, 122, 111, 131, 0, None, 1, None, 1) == rb.status_success
        assert L.rocblas_dtrsv(h.value, 122, 111, 131, 4, None, 4, X, 1) == rb.status_invalid_pointer
