"""Complex trsm / trsv / trmm (rocblas_{c,z}*) on the GPU against the complex oracle
(oracle/trsm_oracle_complex.c, the netlib CTRSM/ZTRSM restatement pinned against
cblas_{c,z}trsm).

All 24 side/uplo/trans/diag combinations (trans C reads conj(A)) at orders that take the
one-CTA block solve and orders that take the recursive solve with the complex DMMA GEMM
updates; the gate is rocblas-test's 40 * eps * k on the reference's forward-error norm with the
complex modulus (testing_trsm.hpp:30-31, norm.hpp:449-492).  Also: complex alpha on the host and
on the device, alpha 0, the batched and strided-batched forms, rocblas_trsm_ex with complex
compute types, the ILP64 forms, trsv with positive and negative increments, and trmm in and
out of place.
"""
import ctypes
import itertools

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle  # noqa: E402
import rocblas_b200 as rb  # noqa: E402
from rocblas_b200 import devmem as dm  # noqa: E402

pytestmark = pytest.mark.gpu
COMBOS = list(itertools.product("LR", "UL", "NTC", "NU"))
DT = {"z": (np.complex128, torch.complex128), "c": (np.complex64, torch.complex64)}


@pytest.fixture(scope="module")
def handle():
    rb.build()
    h = rb.Handle()
    yield h
    h.close()


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _check(side, uplo, trans, diag, alpha, A, B, out, npdt, m, n):
    k = m if side == "L" else n
    X = oracle.trsm(side, uplo, trans, diag, alpha, A, np.asfortranarray(B[:m, :n]))
    got = np.asfortranarray(out[:m, :n])
    assert not np.isnan(got).any()
    err = oracle.matrix_norm_1(X, got)
    assert err <= oracle.trsm_tolerance(npdt, k), (side, uplo, trans, diag, m, n, err)


@pytest.mark.parametrize("dt", ["z", "c"])
@pytest.mark.parametrize("side,uplo,trans,diag", COMBOS)
def test_complex_trsm_all_combos(handle, dt, side, uplo, trans, diag):
    npdt, _ = DT[dt]
    for i, (m, n) in enumerate([(37, 29), (300, 140), (140, 300), (600, 70), (70, 600)]):
        k = m if side == "L" else n
        A, B = oracle.nan_triangle_problem(900 + i, side, uplo, trans, diag, m, n, k + 1, m + 2, npdt)
        alpha = [1.0, -0.75 + 0.5j, 2.0 - 1.0j, 0.5j, 1.0][i]
        dA, dB = dm.to_device(A), dm.to_device(B)
        dm.trsm(handle, side, uplo, trans, diag, m, n, alpha, dA, A.shape[0], dB, B.shape[0])
        torch.cuda.synchronize()
        out = dm.to_host(dB)
        _check(side, uplo, trans, diag, alpha, A, B, out, npdt, m, n)
        assert np.isnan(out[m:]).all()  # rows past m are not written


@pytest.mark.parametrize("dt", ["z", "c"])
def test_complex_trsm_large_recursive(handle, dt):
    """An order of 2000 (16 leaves of 128, GEMM updates up to 1000 deep) for every trans."""
    npdt, _ = DT[dt]
    for side, trans in (("L", "N"), ("R", "C"), ("L", "T")):
        m, n = (2000, 96) if side == "L" else (96, 2000)
        A, B = oracle.nan_triangle_problem(77, side, "L", trans, "N", m, n, 2000, m, npdt)
        dA, dB = dm.to_device(A), dm.to_device(B)
        dm.trsm(handle, side, "L", trans, "N", m, n, 1.0 - 0.25j, dA, 2000, dB, m)
        torch.cuda.synchronize()
        _check(side, "L", trans, "N", 1.0 - 0.25j, A, B, dm.to_host(dB), npdt, m, n)


@pytest.mark.parametrize("dt", ["z", "c"])
def test_complex_alpha_device_and_zero(handle, dt):
    npdt, tdt = DT[dt]
    m, n = 400, 50
    A, B = oracle.nan_triangle_problem(5, "L", "U", "C", "N", m, n, m, m, npdt)
    dA, dB = dm.to_device(A), dm.to_device(B)
    dm.trsm(handle, "L", "U", "C", "N", m, n, 0.5 + 2.0j, dA, m, dB, m, alpha_on_device=True)
    torch.cuda.synchronize()
    _check("L", "U", "C", "N", 0.5 + 2.0j, A, B, dm.to_host(dB), npdt, m, n)
    for on_device in (False, True):
        An = dm.to_device(np.full((m, m), np.nan, dtype=npdt, order="F"))
        Bn = dm.to_device(np.full((m, n), np.nan, dtype=npdt, order="F"))
        dm.trsm(handle, "L", "U", "C", "N", m, n, 0.0, An, m, Bn, m, alpha_on_device=on_device)
        torch.cuda.synchronize()
        assert np.all(dm.to_host(Bn) == 0)


@pytest.mark.parametrize("dt", ["z", "c"])
def test_complex_batched_strided_ex_and_64(handle, dt):
    npdt, tdt = DT[dt]
    batch, m, n = 3, 260, 40
    probs = [oracle.nan_triangle_problem(60 + b, "R", "U", "T", "U", m, n, n, m, npdt) for b in range(batch)]
    alpha = -1.0 + 1.0j
    # pointer arrays
    As = [dm.to_device(A) for A, _ in probs]
    Bs = [dm.to_device(B) for _, B in probs]
    dm.trsm_batched(handle, "R", "U", "T", "U", m, n, alpha, As, n, Bs, m)
    for (A, B), dB in zip(probs, Bs):
        _check("R", "U", "T", "U", alpha, A, B, dm.to_host(dB), npdt, m, n)
    # strided (through the _64 form)
    sa, sb = n * n + 3, m * n + 5
    dA = torch.zeros(batch * sa, dtype=tdt, device="cuda")
    dB = torch.zeros(batch * sb, dtype=tdt, device="cuda")
    for b, (A, B) in enumerate(probs):
        dA[b * sa: b * sa + n * n] = torch.from_numpy(A.ravel(order="F")).cuda()
        dB[b * sb: b * sb + m * n] = torch.from_numpy(B.ravel(order="F")).cuda()
    a = torch.tensor([alpha], dtype=tdt)
    st = getattr(rb.lib(), f"rocblas_{dt}trsm_strided_batched_64")(
        handle.value, rb.SIDE["R"], rb.UPLO["U"], rb.TRANS["T"], rb.DIAG["U"], m, n, _ptr(a), _ptr(dA), n,
        sa, _ptr(dB), m, sb, batch)
    assert st == 0
    torch.cuda.synchronize()
    hB = dB.cpu().numpy()
    for b, (A, B) in enumerate(probs):
        out = hB[b * sb: b * sb + m * n].reshape((m, n), order="F")
        _check("R", "U", "T", "U", alpha, A, B, out, npdt, m, n)
    # trsm_ex with the complex compute type; a supplied invA is accepted (and not needed)
    A, B = probs[0]
    dA1, dB1 = dm.to_device(A), dm.to_device(B)
    invA = torch.zeros(128 * n, dtype=tdt, device="cuda")
    dm.trsm_ex(handle, "R", "U", "T", "U", m, n, alpha, dA1, n, dB1, m, invA, 128 * n)
    torch.cuda.synchronize()
    _check("R", "U", "T", "U", alpha, A, B, dm.to_host(dB1), npdt, m, n)


@pytest.mark.parametrize("dt", ["z", "c"])
@pytest.mark.parametrize("uplo,trans,diag", list(itertools.product("UL", "NTC", "NU")))
def test_complex_trsv(handle, dt, uplo, trans, diag):
    npdt, tdt = DT[dt]
    for i, (n, incx) in enumerate([(40, 1), (300, 2), (700, -3)]):
        A, B = oracle.nan_triangle_problem(30 + i, "L", uplo, trans, diag, n, 1, n, n, npdt)
        buf = np.full(1 + (n - 1) * abs(incx), np.nan + 0j, dtype=npdt)
        pos = [(n - 1 - j) * abs(incx) if incx < 0 else j * incx for j in range(n)]
        buf[pos] = B[:, 0]
        dA, dx = dm.to_device(A), torch.from_numpy(buf).cuda()
        st = getattr(rb.lib(), f"rocblas_{dt}trsv")(handle.value, rb.UPLO[uplo], rb.TRANS[trans], rb.DIAG[diag],
                                                    n, _ptr(dA), n, _ptr(dx), incx)
        assert st == 0
        torch.cuda.synchronize()
        got = dx.cpu().numpy()[pos].reshape(n, 1)
        X = oracle.trsm("L", uplo, trans, diag, 1.0, A, np.asfortranarray(B[:, :1]))
        assert oracle.matrix_norm_1(X, np.asfortranarray(got)) <= oracle.trsm_tolerance(npdt, n)


@pytest.mark.parametrize("dt", ["z", "c"])
@pytest.mark.parametrize("side,uplo,trans,diag", COMBOS)
def test_complex_trmm(handle, dt, side, uplo, trans, diag):
    npdt, _ = DT[dt]
    eps = np.finfo(npdt).eps
    for i, (m, n) in enumerate([(33, 21), (200, 90)]):
        k = m if side == "L" else n
        A, B = oracle.nan_triangle_problem(40 + i, side, uplo, trans, diag, m, n, k, m, npdt)
        alpha = 0.5 - 1.5j
        ref = oracle.trmm(side, uplo, trans, diag, alpha, A, np.asfortranarray(B[:m]))
        dA, dB = dm.to_device(A), dm.to_device(B)
        dC = dm.to_device(np.full((m, n), np.nan, dtype=npdt, order="F"))
        dm.trmm(handle, side, uplo, trans, diag, m, n, alpha, dA, k, dB, m, dC, m)
        torch.cuda.synchronize()
        assert oracle.matrix_norm_1(ref, dm.to_host(dC)) <= 4 * eps * k
        # in place
        dm.trmm(handle, side, uplo, trans, diag, m, n, alpha, dA, k, dB, m, dB, m)
        torch.cuda.synchronize()
        assert oracle.matrix_norm_1(ref, dm.to_host(dB)) <= 4 * eps * k


@pytest.mark.parametrize("dt", ["z", "c"])
def test_complex_gemm_entry(handle, dt):
    """rocblas_b200_{z,c}gemm: C := alpha op(A) op(B) + beta C for every op pair (C conjugates),
    against numpy in complex128."""
    npdt, tdt = DT[dt]
    rng = np.random.default_rng(3)
    m, n, k = 150, 97, 133
    eps = np.finfo(npdt).eps
    alpha, beta = 0.75 - 0.5j, -1.25 + 0.25j
    opf = {"N": lambda X: X, "T": lambda X: X.T, "C": lambda X: X.conj().T}
    for ta, tb in itertools.product("NTC", repeat=2):
        Ash = (m, k) if ta == "N" else (k, m)
        Bsh = (k, n) if tb == "N" else (n, k)
        A = (rng.uniform(-1, 1, Ash) + 1j * rng.uniform(-1, 1, Ash)).astype(npdt, order="F")
        B = (rng.uniform(-1, 1, Bsh) + 1j * rng.uniform(-1, 1, Bsh)).astype(npdt, order="F")
        C = (rng.uniform(-1, 1, (m, n)) + 1j * rng.uniform(-1, 1, (m, n))).astype(npdt, order="F")
        ref = alpha * opf[ta](A.astype(np.complex128)) @ opf[tb](B.astype(np.complex128)) + beta * C
        dA, dB, dC = dm.to_device(A), dm.to_device(B), dm.to_device(C)
        a = torch.tensor([alpha], dtype=tdt)
        b = torch.tensor([beta], dtype=tdt)
        st = getattr(rb.lib(), f"rocblas_b200_{dt}gemm")(
            handle.value, rb.TRANS[ta], rb.TRANS[tb], m, n, k, _ptr(a), _ptr(dA), Ash[0], _ptr(dB), Bsh[0],
            _ptr(b), _ptr(dC), m)
        assert st == 0
        torch.cuda.synchronize()
        got = dm.to_host(dC)
        assert np.max(np.abs(got - ref)) <= 8 * eps * k * 4, (ta, tb)


@pytest.mark.parametrize("dt", ["z", "c"])
@pytest.mark.parametrize("uplo,diag", list(itertools.product("UL", "NU")))
def test_complex_trtri(handle, dt, uplo, diag):
    """rocblas_{c,z}trtri: inv(A) with zeros in the opposite triangle, plain and strided batch."""
    npdt, tdt = DT[dt]
    eps = np.finfo(npdt).eps

    def triangle(A, n):
        Tc = np.nan_to_num(np.array(A[:n, :n], dtype=np.complex128))
        Tc = np.tril(Tc) if uplo == "L" else np.triu(Tc)
        if diag == "U":
            np.fill_diagonal(Tc, 1.0)
        return Tc

    for n in (70, 300):
        A, _ = oracle.nan_triangle_problem(90 + n, "L", uplo, "N", diag, n, 1, n + 1, n, npdt)
        T = triangle(A, n)
        dA = dm.to_device(A)
        inv = dm.to_device(np.full((n + 2, n), np.nan, dtype=npdt, order="F"))
        st = getattr(rb.lib(), f"rocblas_{dt}trtri")(handle.value, rb.UPLO[uplo], rb.DIAG[diag], n,
                                                     _ptr(dA), A.shape[0], _ptr(inv), n + 2)
        assert st == 0
        torch.cuda.synchronize()
        X = dm.to_host(inv)
        assert np.isnan(X[n:]).all()
        Xn = X[:n].astype(np.complex128)
        opp = np.triu(Xn, 1) if uplo == "L" else np.tril(Xn, -1)
        assert np.all(opp == 0)
        assert np.max(np.abs(Xn @ T - np.eye(n))) <= 64 * eps * n
    # strided batch of two
    n, batch = 200, 2
    probs = [oracle.nan_triangle_problem(95 + b, "L", uplo, "N", diag, n, 1, n, n, npdt)[0] for b in range(batch)]
    dA = torch.cat([dm.to_device(A).reshape(-1) for A in probs])
    inv = torch.zeros(batch * n * n, dtype=tdt, device="cuda")
    st = getattr(rb.lib(), f"rocblas_{dt}trtri_strided_batched")(handle.value, rb.UPLO[uplo], rb.DIAG[diag], n,
                                                                 _ptr(dA), n, n * n, _ptr(inv), n, n * n, batch)
    assert st == 0
    torch.cuda.synchronize()
    for b, A in enumerate(probs):
        Xb = inv[b * n * n:(b + 1) * n * n].view(n, n).cpu().numpy().T.astype(np.complex128)
        assert np.max(np.abs(Xb @ triangle(A, n) - np.eye(n))) <= 64 * eps * n


@pytest.mark.parametrize("dt", ["z", "c"])
@pytest.mark.parametrize("uplo", ["L", "U"])
def test_complex_trtri_zero_diagonal_reads_as_one(handle, dt, uplo):
    """rocblas_trtri.hpp:128-141: a zero entry on a non-unit diagonal is read as 1 ("the matrix
    is singular"); the complex trtri returns the inverse of the triangle with those entries
    replaced by 1, and the real kernel's rule is the same."""
    npdt, tdt = DT[dt]
    eps = np.finfo(npdt).eps
    n = 300
    A, _ = oracle.nan_triangle_problem(77, "L", uplo, "N", "N", n, 1, n, n, npdt)
    for i in (0, 5, 131, n - 1):
        A[i, i] = 0
    T = np.nan_to_num(np.array(A[:n, :n], dtype=np.complex128))
    T = np.tril(T) if uplo == "L" else np.triu(T)
    d = np.diag(T).copy()
    d[d == 0] = 1
    np.fill_diagonal(T, d)
    dA = dm.to_device(A)
    inv = dm.to_device(np.zeros((n, n), dtype=npdt, order="F"))
    st = getattr(rb.lib(), f"rocblas_{dt}trtri")(handle.value, rb.UPLO[uplo], rb.DIAG["N"], n, _ptr(dA), n,
                                                 _ptr(inv), n)
    assert st == 0
    torch.cuda.synchronize()
    X = dm.to_host(inv).astype(np.complex128)
    assert np.isfinite(X).all()
    assert np.max(np.abs(X @ T - np.eye(n))) <= 64 * eps * n
