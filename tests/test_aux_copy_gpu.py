"""rocblas_{set,get}_{vector,matrix}[_async][_64]: host <-> device copies with increments and
leading dimensions (rocblas_auxiliary.cpp:305-790), round trips through device memory."""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import rocblas_b200 as rb  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    rb.build()
    return rb.lib()


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


@pytest.mark.parametrize("suf", ["", "_64"])
def test_matrix_round_trip(lib, suf):
    rows, cols, lda, ldd, ldb = 37, 11, 40, 45, 39
    rng = np.random.default_rng(3)
    A = rng.standard_normal(lda * cols)
    dev = torch.zeros(ldd * cols, dtype=torch.float64, device="cuda")
    assert getattr(lib, f"rocblas_set_matrix{suf}")(rows, cols, 8, _p(A), lda,
                                                   ctypes.c_void_p(dev.data_ptr()), ldd) == 0
    d = dev.cpu().numpy().reshape(cols, ldd)
    assert np.array_equal(d[:, :rows], A.reshape(cols, lda)[:, :rows])
    assert np.all(d[:, rows:] == 0)  # outside the rows nothing is written
    out = np.full(ldb * cols, -7.0)
    assert getattr(lib, f"rocblas_get_matrix{suf}")(rows, cols, 8, ctypes.c_void_p(dev.data_ptr()), ldd,
                                                   _p(out), ldb) == 0
    o = out.reshape(cols, ldb)
    assert np.array_equal(o[:, :rows], A.reshape(cols, lda)[:, :rows])
    assert np.all(o[:, rows:] == -7.0)
    # dense on both sides: one contiguous copy
    dev2 = torch.zeros(rows * cols, dtype=torch.float64, device="cuda")
    Ad = np.ascontiguousarray(A.reshape(cols, lda)[:, :rows]).ravel()
    assert getattr(lib, f"rocblas_set_matrix{suf}")(rows, cols, 8, _p(Ad), rows,
                                                   ctypes.c_void_p(dev2.data_ptr()), rows) == 0
    assert np.array_equal(dev2.cpu().numpy(), Ad)


@pytest.mark.parametrize("suf", ["", "_64"])
def test_vector_round_trip_and_async(lib, suf):
    n, incx, incy = 50, 3, 2
    x = np.arange(n * incx, dtype=np.float32)
    dev = torch.zeros(n * incy, dtype=torch.float32, device="cuda")
    assert getattr(lib, f"rocblas_set_vector{suf}")(n, 4, _p(x), incx, ctypes.c_void_p(dev.data_ptr()), incy) == 0
    d = dev.cpu().numpy()
    assert np.array_equal(d[::incy], x[::incx]) and np.all(d[1::incy] == 0)
    y = np.zeros(n, dtype=np.float32)
    s = torch.cuda.Stream()
    pinned = torch.zeros(n, dtype=torch.float32).pin_memory()
    assert getattr(lib, f"rocblas_get_vector_async{suf}")(n, 4, ctypes.c_void_p(dev.data_ptr()), incy,
                                                         ctypes.c_void_p(pinned.data_ptr()), 1,
                                                         ctypes.c_void_p(s.cuda_stream)) == 0
    s.synchronize()
    y[:] = pinned.numpy()
    assert np.array_equal(y, x[::incx])
    # async matrix upload on the stream, then a synchronous read back
    rows, cols = 8, 3
    M = torch.arange(rows * cols, dtype=torch.float64).pin_memory()
    dm_ = torch.zeros(10 * cols, dtype=torch.float64, device="cuda")
    assert getattr(lib, f"rocblas_set_matrix_async{suf}")(rows, cols, 8, ctypes.c_void_p(M.data_ptr()), rows,
                                                         ctypes.c_void_p(dm_.data_ptr()), 10,
                                                         ctypes.c_void_p(s.cuda_stream)) == 0
    s.synchronize()
    got = dm_.cpu().numpy().reshape(cols, 10)[:, :rows]
    assert np.array_equal(got, M.numpy().reshape(cols, rows))
