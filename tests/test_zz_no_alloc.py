"""rocblas_b200_dtrsm_vbatched_noalloc: the variable-size batch for callers that cannot let a
library allocate device memory (an application pool that has already reserved the GPU's
memory, loops that cannot take the synchronisation of a cudaFree).  Its scratch is one fixed
array inside the library that every call reuses, so it must give the same results as
rocblas_b200_dtrsm_vbatched call after call, on both of its kernel paths (the one-warp strips
for k <= 32 and the CTA strips above), and count rejected descriptors the same way.

This file is collected last so that a failure here comes after every other test has run; it
also passes on its own in a fresh process."""
import ctypes
import itertools

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle  # noqa: E402
import rocblas_b200 as rb  # noqa: E402
from rocblas_b200 import devmem as dm  # noqa: E402

pytestmark = pytest.mark.gpu
COMBOS = list(itertools.product("LR", "UL", "NT", "NU"))
MAX_COUNT = 65536  # the fixed scratch limit of the entry point


def _batch(seed, count, kmax=299):
    rng = np.random.default_rng(seed)
    probs, dev = [], []
    for i in range(count):
        side, uplo, trans, diag = COMBOS[i % 16]
        m = int(rng.integers(1, 300))
        n = int(rng.integers(1, 70))
        if side == "L":
            m = min(m, kmax)
        else:
            n = min(n, kmax)
        k = m if side == "L" else n
        A, B = oracle.nan_triangle_problem(seed * 1000 + i, side, uplo, trans, diag, m, n, k + 1, m + 2,
                                           np.float64)
        probs.append((A, B, m, n, side, uplo, trans, diag))
        dev.append(dm.to_device(A))
    return probs, dev


def _descriptors(probs, dA, dB, spoil=()):
    rec = np.zeros(len(probs), dtype=np.dtype([
        ("A", np.uint64), ("B", np.uint64), ("m", np.int32), ("n", np.int32), ("lda", np.int32),
        ("ldb", np.int32), ("side", np.int32), ("uplo", np.int32), ("trans", np.int32),
        ("diag", np.int32)]))
    for i, (A, B, m, n, side, uplo, trans, diag) in enumerate(probs):
        rec[i] = (dA[i].data_ptr(), dB[i].data_ptr(), m, n, A.shape[0], B.shape[0], rb.SIDE[side],
                  rb.UPLO[uplo], rb.TRANS[trans], rb.DIAG[diag])
    for i, field, value in spoil:  # descriptors the prepass must reject
        rec[i][field] = value
    return torch.from_numpy(rec.view(np.uint8).copy()).cuda()


def _run(fn, h, probs, dA, alpha, max_k=512, spoil=()):
    dB = [dm.to_device(p[1]) for p in probs]
    desc = _descriptors(probs, dA, dB, spoil)
    invalid = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    a = ctypes.c_double(alpha)
    st = fn(h.value, ctypes.cast(ctypes.byref(a), ctypes.c_void_p), ctypes.c_void_p(desc.data_ptr()),
            len(probs), max_k, ctypes.c_void_p(invalid.data_ptr()))
    assert st == rb.status_success, st
    torch.cuda.synchronize()
    return [dm.to_host(b) for b in dB], int(invalid.item())


def test_noalloc_matches_allocating_entry_point_twice():
    L = rb.lib()
    probs, dA = _batch(5, 200)
    with rb.Handle() as h:
        ref, inv_ref = _run(L.rocblas_b200_dtrsm_vbatched, h, probs, dA, -1.5)
        assert inv_ref == 0
        for call in range(2):  # two calls in a row: the shared scratch keeps the last contents
            got, inv = _run(L.rocblas_b200_dtrsm_vbatched_noalloc, h, probs, dA, -1.5)
            assert inv == 0
            for (A, B, m, n, *_), r, g in zip(probs, ref, got):
                tol = oracle.trsm_tolerance(np.float64, max(m, n))
                assert oracle.matrix_norm_1(r[:m], g[:m]) <= tol, (call, m, n)
                assert np.isnan(g[m:]).all()


def test_noalloc_warp_class_and_rejected_descriptors():
    """max_k = 32 runs the one-warp strip kernel; three spoiled descriptors (a bad side, ldb
    below m, an order above max_k) are skipped and counted, and their B stays as it was."""
    L = rb.lib()
    probs, dA = _batch(7, 300, kmax=32)
    spoil = [(3, "side", 7), (40, "ldb", 0), (77, "m" if probs[77][4] == "L" else "n", 33)]
    bad = {i for i, _, _ in spoil}
    with rb.Handle() as h:
        ref, inv_ref = _run(L.rocblas_b200_dtrsm_vbatched, h, probs, dA, 0.75, 32, spoil)
        assert inv_ref == 3
        for call in range(2):
            got, inv = _run(L.rocblas_b200_dtrsm_vbatched_noalloc, h, probs, dA, 0.75, 32, spoil)
            assert inv == 3, (call, inv)
            for i, ((A, B, m, n, *_), r, g) in enumerate(zip(probs, ref, got)):
                if i in bad:
                    np.testing.assert_array_equal(g, B)  # rejected: B untouched (NaN rows too)
                    continue
                tol = oracle.trsm_tolerance(np.float64, max(m, n))
                assert oracle.matrix_norm_1(r[:m], g[:m]) <= tol, (call, i, m, n)
                assert np.isnan(g[m:]).all()


def test_noalloc_limits_and_workspace():
    L = rb.lib()
    one = ctypes.c_double(1.0)
    p = ctypes.cast(ctypes.byref(one), ctypes.c_void_p)
    with rb.Handle() as h:
        assert L.rocblas_b200_dtrsm_vbatched_noalloc(h.value, p, None, MAX_COUNT + 1, 64, None) == \
            rb.status_invalid_size
        assert L.rocblas_b200_dtrsm_vbatched_noalloc(h.value, p, None, 0, 64, None) == rb.status_success
        # it takes nothing from the handle: a size query reports no workspace
        assert L.rocblas_start_device_memory_size_query(h.value) == 0
        assert L.rocblas_b200_dtrsm_vbatched_noalloc(h.value, p, None, 10, 64, None) == \
            rb.status_size_unchanged
        size = ctypes.c_size_t(1)
        assert L.rocblas_stop_device_memory_size_query(h.value, ctypes.byref(size)) == 0
        assert size.value == 0
        # and it leaves the handle's workspace alone while it solves
        probs, dA = _batch(6, 40)
        before = ctypes.c_size_t(0)
        assert L.rocblas_get_device_memory_size(h.value, ctypes.byref(before)) == 0
        _run(L.rocblas_b200_dtrsm_vbatched_noalloc, h, probs, dA, 1.0)
        after = ctypes.c_size_t(0)
        assert L.rocblas_get_device_memory_size(h.value, ctypes.byref(after)) == 0
        assert after.value == before.value == 0
