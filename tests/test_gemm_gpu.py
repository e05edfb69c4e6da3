"""rocblas_b200_dgemm: the FP64 DMMA tiles of the trsm updates, as a GEMM, for every tile
shape (forced through the tuning table) and transpose combination, against torch FP64."""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import rocblas_b200 as rb  # noqa: E402

pytestmark = pytest.mark.gpu
TILES = {1: "128x128", 2: "128x64", 3: "64x128", 4: "64x64", 5: "128x32", 6: "32x128", 7: "128x128/bk32",
         8: "128x64/warp64x32", 9: "64x128/warp32x64", 10: "64x64/warp64x32", 11: "64x64/k16"}


def _gemm(h, ta, tb, m, n, k, alpha, A, B, beta, C):
    a, b = ctypes.c_double(alpha), ctypes.c_double(beta)
    st = rb.lib().rocblas_b200_dgemm(h.value, rb.TRANS[ta], rb.TRANS[tb], m, n, k,
                                     ctypes.cast(ctypes.byref(a), ctypes.c_void_p),
                                     ctypes.c_void_p(A.data_ptr()), A.shape[1],
                                     ctypes.c_void_p(B.data_ptr()), B.shape[1],
                                     ctypes.cast(ctypes.byref(b), ctypes.c_void_p),
                                     ctypes.c_void_p(C.data_ptr()), C.shape[1])
    assert st == 0, st


@pytest.mark.parametrize("tile", sorted(TILES))
@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "N"), ("N", "T"), ("T", "T")])
def test_dgemm_tiles(tile, ta, tb):
    L = rb.lib()
    assert L.rocblas_b200_set_tuning(b"dmma_force_tile", tile) == 0
    try:
        g = torch.Generator(device="cuda").manual_seed(tile)
        for (m, n, k) in [(1, 1, 1), (131, 67, 45), (300, 257, 129), (64, 128, 16)]:
            # column-major storage as (ncols, ld) tensors
            A = torch.randn((k if ta == "N" else m), (m if ta == "N" else k) + 3, generator=g,
                            device="cuda", dtype=torch.float64)
            B = torch.randn((n if tb == "N" else k), (k if tb == "N" else n) + 1, generator=g,
                            device="cuda", dtype=torch.float64)
            C = torch.randn(n, m + 2, generator=g, device="cuda", dtype=torch.float64)
            opA = A[:, :m].T if ta == "N" else A[:, :k]        # m x k
            opB = B[:, :k].T if tb == "N" else B[:, :n]        # k x n
            ref = -0.5 * (opA @ opB) + 2.0 * C[:, :m].T
            with rb.Handle() as h:
                _gemm(h, ta, tb, m, n, k, -0.5, A, B, 2.0, C)
                torch.cuda.synchronize()
            err = (C[:, :m].T - ref).abs().max().item() / max(1.0, ref.abs().max().item())
            assert err < 1e-14 * max(1, k), (TILES[tile], ta, tb, m, n, k, err)
    finally:
        L.rocblas_b200_set_tuning(b"dmma_force_tile", 0)


def test_tuning_table_api():
    L = rb.lib()
    v = ctypes.c_int(-1)
    assert L.rocblas_b200_get_tuning(b"sliced_min_k", ctypes.byref(v)) == 0 and v.value > 0
    assert L.rocblas_b200_set_tuning(b"no_such_key", 1) == rb.status_invalid_value
    assert L.rocblas_b200_set_tuning(b"mixed_slices", 9) == rb.status_invalid_value
    assert L.rocblas_b200_get_tuning(b"mixed_slices", None) == rb.status_invalid_pointer
