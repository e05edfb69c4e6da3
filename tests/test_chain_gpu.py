"""The one-launch chain solve (trsm_chain.cuh) against the oracle and against the recursive
path it replaces for few right-hand sides: all 16 side/uplo/trans/diag combinations, triangle
orders that are not multiples of 128, both strip widths, strided batches, the _ex path with a
supplied invA and alpha on the device."""
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


def _tune(key, value):
    assert rb.lib().rocblas_b200_set_tuning(key.encode(), value) == 0


@pytest.fixture()
def chain_setting():
    L = rb.lib()
    old = {}
    for key in ("chain_max_cols", "chain_max_cols_f32", "chain_w"):
        v = ctypes.c_int(-1)
        assert L.rocblas_b200_get_tuning(key.encode(), ctypes.byref(v)) == 0
        old[key] = v.value
    yield _tune
    for key, v in old.items():
        _tune(key, v)


def _solve(h, side, uplo, trans, diag, m, n, alpha, A, B, on_device=False):
    dA, dB = dm.to_device(A), dm.to_device(B)
    dm.trsm(h, side, uplo, trans, diag, m, n, alpha, dA, A.shape[0], dB, B.shape[0],
            alpha_on_device=on_device)
    torch.cuda.synchronize()
    return dm.to_host(dB)


def _check(side, uplo, trans, diag, m, n, alpha, A, B, out):
    X = oracle.trsm(side, uplo, trans, diag, alpha, A, np.asfortranarray(B[:m]))
    assert not np.isnan(out[:m]).any()
    err = oracle.matrix_norm_1(X, out[:m])
    assert err <= oracle.trsm_tolerance(np.float64, max(m, n)), (side, uplo, trans, diag, m, n, err)
    if B.shape[0] > m:
        assert np.isnan(out[m:]).all()


def _err_word(h):
    code = ctypes.c_int(-1)
    assert rb.lib().rocblas_b200_get_device_error(h.value, ctypes.byref(code)) == 0
    return code.value


@pytest.mark.parametrize("side,uplo,trans,diag", COMBOS)
def test_chain_all_combos(chain_setting, side, uplo, trans, diag):
    with rb.Handle() as h:
        for i, (m, n, w) in enumerate([(700, 45, 0), (45, 700, 64), (333, 130, 32), (130, 333, 0)]):
            if side == "R":
                m, n = n, m
            k = m if side == "L" else n
            A, B = oracle.nan_triangle_problem(300 + i, side, uplo, trans, diag, m, n, k + 2, m + 1,
                                               np.float64)
            alpha = [1.0, -0.75, 2.0, 0.5][i]
            chain_setting("chain_max_cols", 1 << 20)
            chain_setting("chain_w", w)
            out_chain = _solve(h, side, uplo, trans, diag, m, n, alpha, A, B)
            chain_setting("chain_max_cols", 0)
            out_rec = _solve(h, side, uplo, trans, diag, m, n, alpha, A, B)
            _check(side, uplo, trans, diag, m, n, alpha, A, B, out_chain)
            _check(side, uplo, trans, diag, m, n, alpha, A, B, out_rec)
        assert _err_word(h) == 0


def test_chain_large_order_device_alpha(chain_setting):
    """k = 3000 (24 blocks, a partial last one), 40 right-hand sides, alpha on the device;
    residual checked on the GPU in FP64."""
    chain_setting("chain_max_cols", 1 << 20)
    m, n = 3000, 40
    with rb.Handle() as h:
        for (uplo, trans) in [("L", "N"), ("U", "N"), ("L", "T"), ("U", "T")]:
            A, B = oracle.nan_triangle_problem(19, "L", uplo, trans, "N", m, n, m, m, np.float64)
            out = _solve(h, "L", uplo, trans, "N", m, n, -1.5, A, B, on_device=True)
            T = torch.from_numpy(oracle.clean_triangle(A, m, uplo, "N")).cuda()
            opT = T if trans == "N" else T.T
            X = torch.from_numpy(np.ascontiguousarray(out)).cuda()
            R = opT @ X + 1.5 * torch.from_numpy(np.ascontiguousarray(B)).cuda()
            rel = (R.abs().sum() / (opT.abs() @ X.abs()).sum()).item()
            assert rel < 1e-13, (uplo, trans, rel)
        assert _err_word(h) == 0


def test_chain_strided_batched(chain_setting):
    chain_setting("chain_max_cols", 1 << 20)
    batch, m, n = 6, 300, 20
    for side, uplo, trans, diag in [("L", "L", "N", "N"), ("R", "U", "T", "U")]:
        if side == "R":
            m, n = n, m
        k = m if side == "L" else n
        lda, ldb = k + 1, m + 2
        sa, sb = lda * k + 5, ldb * n + 3
        probs = [oracle.nan_triangle_problem(60 + b, side, uplo, trans, diag, m, n, lda, ldb, np.float64)
                 for b in range(batch)]
        dA = torch.full((batch * sa,), float("nan"), dtype=torch.float64, device="cuda")
        dB = torch.full((batch * sb,), float("nan"), dtype=torch.float64, device="cuda")
        for b, (A, B) in enumerate(probs):
            dA[b * sa: b * sa + lda * k] = torch.from_numpy(A.ravel(order="F")).cuda()
            dB[b * sb: b * sb + ldb * n] = torch.from_numpy(B.ravel(order="F")).cuda()
        with rb.Handle() as h:
            dm.trsm_strided_batched(h, side, uplo, trans, diag, m, n, 0.5, dA, lda, sa, dB, ldb, sb, batch)
            torch.cuda.synchronize()
            assert _err_word(h) == 0
        hB = dB.cpu().numpy()
        for b, (A, B) in enumerate(probs):
            out = hB[b * sb: b * sb + ldb * n].reshape((ldb, n), order="F")
            _check(side, uplo, trans, diag, m, n, 0.5, A, B, out)


def test_chain_ex_supplied_invA_and_repeatability(chain_setting):
    chain_setting("chain_max_cols", 1 << 20)
    m, n = 900, 100
    A, B = oracle.nan_triangle_problem(81, "L", "U", "T", "U", m, n, m, m, np.float64)
    with rb.Handle() as h:
        dA = dm.to_device(A)
        invA = dm.build_invA(h, "U", "U", dA, m, m)
        outs = []
        for _ in range(3):
            dB = dm.to_device(B)
            st = dm.trsm_ex(h, "L", "U", "T", "U", m, n, 1.25, dA, m, dB, m, invA, 128 * m)
            torch.cuda.synchronize()
            assert st == rb.status_success
            outs.append(dm.to_host(dB))
        _check("L", "U", "T", "U", m, n, 1.25, A, B, outs[0])
        assert all(np.array_equal(outs[0], o, equal_nan=True) for o in outs[1:])
        assert _err_word(h) == 0


@pytest.mark.parametrize("side,uplo,trans,diag", [("L", "L", "N", "N"), ("L", "U", "T", "U"),
                                                  ("R", "U", "N", "N"), ("R", "L", "T", "U")])
def test_chain_fp32(chain_setting, side, uplo, trans, diag):
    """FP32 systems through the chain: staged in FP32, computed in FP64, rounded once."""
    chain_setting("chain_max_cols_f32", 1 << 20)
    m, n = (600, 70) if side == "L" else (70, 600)
    k = m if side == "L" else n
    A, B = oracle.nan_triangle_problem(400, side, uplo, trans, diag, m, n, k + 1, m + 2, np.float32)
    with rb.Handle() as h:
        out = _solve(h, side, uplo, trans, diag, m, n, 1.5, A, B)
        assert _err_word(h) == 0
    X = oracle.trsm(side, uplo, trans, diag, 1.5, A, np.asfortranarray(B[:m]))
    err = oracle.matrix_norm_1(X, out[:m])
    assert err <= oracle.trsm_tolerance(np.float32, max(m, n)), err
    assert np.isnan(out[m:]).all()
