"""Failure detection of the bounded device waits, without faulting or hanging the GPU.

The chain solve's CTAs wait on flags that earlier items release (an ld.acquire spin bounded by
wait_cycles_log2).  The failure is injected on the host: chain_first_item makes the launch start
claiming items past the first ones, so nothing ever sets their flags.  With a short limit every
wait runs out within microseconds; the kernel records error 4 in the handle's device error word,
drains its copies and returns.  The test checks that the call returns, that
rocblas_b200_get_device_error reports the code (and clears it), and that the same handle solves
correctly right afterwards.  The reference's counterpart is the unbounded flag spin of its trsv
(library/src/blas2/rocblas_trsv_kernels.cpp:655-663)."""
import contextlib
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle  # noqa: E402
import rocblas_b200 as rb  # noqa: E402
from rocblas_b200 import devmem as dm  # noqa: E402

pytestmark = pytest.mark.gpu


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


def _error_code(h):
    code = ctypes.c_int(-1)
    assert rb.lib().rocblas_b200_get_device_error(h.value, ctypes.byref(code)) == 0
    return code.value


@pytest.mark.parametrize("first_item", [1, 5])
def test_chain_wait_runs_out_and_is_reported(first_item):
    rb.build()
    m, n = 2048, 64  # 16 row blocks, one strip of 64 columns: item j is block j
    A, B = oracle.nan_triangle_problem(3, "L", "L", "N", "N", m, n, m, m, np.float64)
    with rb.Handle() as h:
        assert _error_code(h) == 0
        dA, dB = dm.to_device(A), dm.to_device(B)
        with tuning(wait_cycles_log2=16, chain_first_item=first_item):
            dm.trsm(h, "L", "L", "N", "N", m, n, 1.0, dA, m, dB, m)
            torch.cuda.synchronize()  # returns: every wait ran out
        assert _error_code(h) == 4
        assert _error_code(h) == 0  # read and cleared
        # the context and the handle still work
        dB = dm.to_device(B)
        dm.trsm(h, "L", "L", "N", "N", m, n, 1.0, dA, m, dB, m)
        torch.cuda.synchronize()
        X = oracle.trsm("L", "L", "N", "N", 1.0, A, B)
        assert oracle.matrix_norm_1(X, dm.to_host(dB)) <= oracle.trsm_tolerance(np.float64, m)
        assert _error_code(h) == 0


def test_wait_limit_keys_are_range_checked():
    L = rb.lib()
    assert L.rocblas_b200_set_tuning(b"wait_cycles_log2", 9) != 0
    assert L.rocblas_b200_set_tuning(b"wait_cycles_log2", 41) != 0
    assert L.rocblas_b200_set_tuning(b"chain_first_item", -1) != 0
    v = ctypes.c_int(0)
    assert L.rocblas_b200_get_tuning(b"wait_cycles_log2", ctypes.byref(v)) == 0 and v.value == 31
    assert L.rocblas_b200_get_tuning(b"chain_first_item", ctypes.byref(v)) == 0 and v.value == 0
