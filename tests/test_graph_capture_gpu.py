"""CUDA-graph capture of the variable-size batch (rocblas_b200_?trsm_vbatched and _vbatched_ex),
the form the reference's capture tests take for trsm, its batched forms and _ex
(clients/gtest/trsm_gtest.yaml:1288-1309): with the workspace reserved by the size-query
protocol and one eager call made first, the call records into a graph on the handle's stream,
and two replays give the eager result bit for bit."""
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
    buf = np.zeros(len(entries), dtype=np.dtype([
        ("A", np.uint64), ("B", np.uint64), ("m", np.int32), ("n", np.int32), ("lda", np.int32),
        ("ldb", np.int32), ("side", np.int32), ("uplo", np.int32), ("trans", np.int32),
        ("diag", np.int32)]))
    for i, (A, B, m, n, lda, ldb, side, uplo, trans, diag) in enumerate(entries):
        buf[i] = (A.data_ptr(), B.data_ptr(), m, n, lda, ldb, rb.SIDE[side], rb.UPLO[uplo], rb.TRANS[trans],
                  rb.DIAG[diag])
    return torch.from_numpy(buf.view(np.uint8).copy()).cuda()


def _batch(h, dt, count, ks, ex):
    npdt = np.float64 if dt == "d" else np.float32
    rng = np.random.default_rng(count + (7 if ex else 0))
    entries, B0s, invs = [], [], []
    for i in range(count):
        side, uplo, trans, diag = COMBOS[i % 16]
        k = int(rng.choice(ks))
        ncols = int(rng.integers(1, 70))
        m, n = (k, ncols) if side == "L" else (ncols, k)
        A, B = oracle.nan_triangle_problem(900 + i, side, uplo, trans, diag, m, n, k + 1, m + 1, npdt)
        dA, dB = dm.to_device(A), dm.to_device(B)
        entries.append((dA, dB, m, n, k + 1, m + 1, side, uplo, trans, diag))
        B0s.append(dB.clone())
        invs.append(dm.build_invA(h, uplo, diag, dA, k + 1, k) if ex and k > 512 else None)
    return entries, B0s, invs


@pytest.mark.parametrize("dt", ["d", "s"])
@pytest.mark.parametrize("ex", [False, True])
def test_vbatched_graph_replay_equals_eager(dt, ex):
    L = rb.lib()
    s = torch.cuda.Stream()
    with rb.Handle() as h:
        h.set_stream(ctypes.c_void_p(s.cuda_stream))
        ks = [20, 64, 200, 512, 700, 1100] if ex else [16, 40, 100, 300, 512]
        entries, B0s, invs = _batch(h, dt, 40 if ex else 120, ks, ex)
        desc = _descriptors(entries)
        ptrs = torch.tensor([(t.data_ptr() if t is not None else 0) for t in invs], dtype=torch.int64,
                            device="cuda")
        invalid = torch.full((1,), -1, dtype=torch.int32, device="cuda")
        alpha = ctypes.c_double(0.75) if dt == "d" else ctypes.c_float(0.75)
        ap = ctypes.cast(ctypes.byref(alpha), ctypes.c_void_p)
        n = len(entries)
        if ex:
            fn = getattr(L, f"rocblas_b200_{dt}trsm_vbatched_ex")
            call = lambda: fn(h.value, ap, ctypes.c_void_p(desc.data_ptr()), ctypes.c_void_p(ptrs.data_ptr()),  # noqa: E731
                              n, 1100, 80, ctypes.c_void_p(invalid.data_ptr()))
        else:
            fn = getattr(L, f"rocblas_b200_{dt}trsm_vbatched")
            call = lambda: fn(h.value, ap, ctypes.c_void_p(desc.data_ptr()), n, 512,  # noqa: E731
                              ctypes.c_void_p(invalid.data_ptr()))
        # workspace by the size query, reserved before capture (allocation is not captured)
        assert L.rocblas_start_device_memory_size_query(h.value) == 0
        assert call() in (rb.status_size_increased, rb.status_size_unchanged)
        size = ctypes.c_size_t(0)
        assert L.rocblas_stop_device_memory_size_query(h.value, ctypes.byref(size)) == 0
        assert L.rocblas_set_device_memory_size(h.value, size.value) == 0

        def reset():
            for e, b0 in zip(entries, B0s):
                e[1].copy_(b0)
            torch.cuda.synchronize()

        reset()
        with torch.cuda.stream(s):
            assert call() == 0
        torch.cuda.synchronize()
        eager = [e[1].clone() for e in entries]
        assert int(invalid.item()) == 0
        reset()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            st = call()
        assert st == 0
        for _ in range(2):
            reset()
            g.replay()
            torch.cuda.synchronize()
            for e, x in zip(entries, eager):
                assert torch.equal(torch.nan_to_num(e[1], nan=7.0), torch.nan_to_num(x, nan=7.0))
        del g
        code = ctypes.c_int(-1)
        assert L.rocblas_b200_get_device_error(h.value, ctypes.byref(code)) == 0 and code.value == 0
