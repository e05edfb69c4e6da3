"""Variable-size batched trsm (rocblas_b200_?trsm_vbatched) against the oracle.

The batch mixes every side/uplo/trans/diag combination and uneven (m, n), including empty
systems and one malformed descriptor that must be skipped and counted."""
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


def _descriptors(entries):
    """entries: list of (A_tensor, B_tensor, m, n, lda, ldb, side, uplo, trans, diag)."""
    buf = np.zeros(len(entries), dtype=np.dtype([
        ("A", np.uint64), ("B", np.uint64), ("m", np.int32), ("n", np.int32), ("lda", np.int32),
        ("ldb", np.int32), ("side", np.int32), ("uplo", np.int32), ("trans", np.int32),
        ("diag", np.int32)]))
    for i, (A, B, m, n, lda, ldb, side, uplo, trans, diag) in enumerate(entries):
        buf[i] = (A.data_ptr() if A is not None else 0, B.data_ptr() if B is not None else 0, m, n,
                  lda, ldb, rb.SIDE[side], rb.UPLO[uplo], rb.TRANS[trans], rb.DIAG[diag])
    assert buf.dtype.itemsize == 48
    return torch.from_numpy(buf.view(np.uint8).copy()).cuda()


@pytest.mark.parametrize("dt", ["d", "s"])
def test_vbatched_mixed(dt):
    npdt = np.float64 if dt == "d" else np.float32
    rng = np.random.default_rng(4)
    host, entries = [], []
    for i in range(300):
        side, uplo, trans, diag = COMBOS[i % 16]
        m = int(np.exp(rng.uniform(np.log(1), np.log(512))))
        n = int(rng.integers(1, 65))
        if i % 97 == 5:
            n = 0  # empty system
        k = m if side == "L" else n
        lda, ldb = max(k, 1) + int(rng.integers(0, 3)), max(m, 1) + int(rng.integers(0, 3))
        if k > 512:
            m, k = (512, 512) if side == "L" else (m, k)
        A, B = oracle.nan_triangle_problem(i, side, uplo, trans, diag, m, n, max(lda, k), ldb, npdt)
        dA, dB = dm.to_device(A), dm.to_device(B)
        host.append((A, B, m, n, side, uplo, trans, diag))
        entries.append((dA, dB, m, n, A.shape[0], B.shape[0], side, uplo, trans, diag))
    # one malformed descriptor (ldb < m): skipped and counted
    bad_B = dm.to_device(np.full((4, 8), 7.0, dtype=npdt, order="F"))
    entries.append((entries[0][0], bad_B, 8, 8, 600, 4, "L", "L", "N", "N"))
    desc = _descriptors(entries)
    invalid = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    alpha = ctypes.c_double(1.25) if dt == "d" else ctypes.c_float(1.25)
    fn = rb.lib().rocblas_b200_dtrsm_vbatched if dt == "d" else rb.lib().rocblas_b200_strsm_vbatched
    with rb.Handle() as h:
        st = fn(h.value, ctypes.cast(ctypes.byref(alpha), ctypes.c_void_p), ctypes.c_void_p(desc.data_ptr()),
                len(entries), 512, ctypes.c_void_p(invalid.data_ptr()))
        assert st == 0
        torch.cuda.synchronize()
    assert int(invalid.item()) == 1
    assert np.all(bad_B.cpu().numpy() == 7.0)
    for (A, B, m, n, side, uplo, trans, diag), e in zip(host, entries):
        out = dm.to_host(e[1])
        if m == 0 or n == 0:
            continue
        X = oracle.trsm(side, uplo, trans, diag, 1.25, A, np.asfortranarray(B[:m]))
        err = oracle.matrix_norm_1(X, out[:m])
        assert err <= oracle.trsm_tolerance(npdt, max(m, n)), (side, uplo, trans, diag, m, n, err)
        if B.shape[0] > m:
            assert np.isnan(out[m:]).all()


def test_vbatched_arguments():
    L = rb.lib()
    one = ctypes.c_double(1.0)
    p = ctypes.cast(ctypes.byref(one), ctypes.c_void_p)
    with rb.Handle() as h:
        assert L.rocblas_b200_dtrsm_vbatched(None, p, None, 1, 64, None) == rb.status_invalid_handle
        assert L.rocblas_b200_dtrsm_vbatched(h.value, p, None, 1, 513, None) == rb.status_invalid_size
        assert L.rocblas_b200_dtrsm_vbatched(h.value, p, None, -1, 64, None) == rb.status_invalid_size
        assert L.rocblas_b200_dtrsm_vbatched(h.value, p, None, 0, 64, None) == rb.status_success
        assert L.rocblas_b200_dtrsm_vbatched(h.value, p, None, 3, 64, None) == rb.status_invalid_pointer


@pytest.mark.parametrize("dt", ["d", "s"])
def test_vbatched_ex_any_order(dt):
    """rocblas_b200_?trsm_vbatched_ex: systems up to k = 1500 in one call, k > 512 through the
    chain with the caller's invA (built by trtri_strided_batched), k <= 512 through the strip
    solver; malformed descriptors (no invA, too many right-hand sides) skipped and counted."""
    npdt = np.float64 if dt == "d" else np.float32
    rng = np.random.default_rng(9)
    host, entries, invs = [], [], []
    with rb.Handle() as h:
        for i in range(48):
            side, uplo, trans, diag = COMBOS[i % 16]
            k = int(rng.choice([40, 300, 513, 700, 1100, 1500]))
            ncols = int(rng.integers(1, 90))
            m, n = (k, ncols) if side == "L" else (ncols, k)
            lda, ldb = k + int(rng.integers(0, 3)), m + int(rng.integers(0, 3))
            A, B = oracle.nan_triangle_problem(500 + i, side, uplo, trans, diag, m, n, lda, ldb, npdt)
            dA, dB = dm.to_device(A), dm.to_device(B)
            inv = dm.build_invA(h, uplo, diag, dA, lda, k) if k > 512 else None
            host.append((A, B, m, n, side, uplo, trans, diag))
            entries.append((dA, dB, m, n, lda, ldb, side, uplo, trans, diag))
            invs.append(inv)
        # malformed: a k > 512 system without invA, and one with more right-hand sides than max_n
        big_A, big_B = oracle.nan_triangle_problem(77, "L", "L", "N", "N", 600, 200, 600, 600, npdt)
        dbA, dbB = dm.to_device(big_A), dm.to_device(big_B)
        bad1 = dm.to_device(np.full((600, 4), 7.0, dtype=npdt, order="F"))
        entries.append((dbA, bad1, 600, 4, 600, 600, "L", "L", "N", "N"))
        invs.append(None)
        entries.append((dbA, dbB, 600, 200, 600, 600, "L", "L", "N", "N"))
        invs.append(dm.build_invA(h, "L", "N", dbA, 600, 600))
        desc = _descriptors(entries)
        ptrs = torch.tensor([(t.data_ptr() if t is not None else 0) for t in invs], dtype=torch.int64,
                            device="cuda")
        invalid = torch.full((1,), -1, dtype=torch.int32, device="cuda")
        alpha = ctypes.c_double(-0.5) if dt == "d" else ctypes.c_float(-0.5)
        fn = rb.lib().rocblas_b200_dtrsm_vbatched_ex if dt == "d" else rb.lib().rocblas_b200_strsm_vbatched_ex
        st = fn(h.value, ctypes.cast(ctypes.byref(alpha), ctypes.c_void_p), ctypes.c_void_p(desc.data_ptr()),
                ctypes.c_void_p(ptrs.data_ptr()), len(entries), 1500, 100, ctypes.c_void_p(invalid.data_ptr()))
        assert st == 0
        torch.cuda.synchronize()
        code = ctypes.c_int(-1)
        assert rb.lib().rocblas_b200_get_device_error(h.value, ctypes.byref(code)) == 0 and code.value == 0
    assert int(invalid.item()) == 2
    assert np.all(bad1.cpu().numpy() == 7.0)
    assert np.array_equal(dm.to_host(dbB), big_B, equal_nan=True)
    for (A, B, m, n, side, uplo, trans, diag), e in zip(host, entries):
        out = dm.to_host(e[1])
        X = oracle.trsm(side, uplo, trans, diag, -0.5, A, np.asfortranarray(B[:m]))
        err = oracle.matrix_norm_1(X, out[:m])
        assert err <= oracle.trsm_tolerance(npdt, max(m, n)), (side, uplo, trans, diag, m, n, err)
        if B.shape[0] > m:
            assert np.isnan(out[m:]).all()
