"""Seeded synthetic workloads for the TRSM benchmarks and tests.

Column-major matrices are produced as Fortran-ordered numpy arrays (host) or as
``(ncols, ld)`` C-contiguous torch tensors (device), the layout the C ABI reads.
"""
from __future__ import annotations

import numpy as np


def condition_band_lower_torch(m, n, kband, seed, device="cuda", dtype=None):
    """The precision-form workload on the device: lower-triangular A (m x m, lda = m) with
    diagonal d_i = 10^(-kband*i/m) * (1 + U(0, 0.1)), the off-diagonal entries of row i
    d_i * N(0,1)/sqrt(m), the upper triangle NaN; B ~ U(-1, 1) (m x n).

    Off-diagonals are scaled by their row's diagonal: with unscaled N(0,1)/sqrt(m)
    off-diagonals the solution grows like exp((10^(2k)-1)/(2k ln 10)) and overflows double
    for k >= 2 at this size, so those systems have no finite solution.  Returned tensors
    are (ncols, ld) views of column-major storage."""
    import torch

    dtype = dtype or torch.float64
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    # At = A^T in row-major == A in column-major: At[j, i] = A(i, j)
    idx = torch.arange(m, device=device, dtype=torch.float64)
    d = torch.pow(10.0, -kband * idx / m) * (1.0 + 0.1 * torch.rand(m, generator=g, device=device,
                                                                     dtype=torch.float64))
    At = torch.randn(m, m, generator=g, device=device, dtype=torch.float64) / float(np.sqrt(m))
    At.mul_(d.view(1, m))          # row i of A (column i of At) scaled by d_i
    At.triu_(1)                    # At upper (j < i in A terms) == A strictly lower
    At.diagonal().copy_(d)
    nan_mask = torch.ones(m, m, dtype=torch.bool, device=device).tril_(-1)  # A upper = At lower
    At.masked_fill_(nan_mask, float("nan"))
    Bt = torch.rand(n, m, generator=g, device=device, dtype=torch.float64) * 2.0 - 1.0
    return At.to(dtype).contiguous(), Bt.to(dtype).contiguous()


def graded_sigma(m, kband):
    """Singular values graded geometrically from 1 to 10^-kband: kappa_2 = 10^kband."""
    return 10.0 ** (-kband * np.arange(m) / max(m - 1, 1))


def graded_condition_lower_torch(m, n, kband, seed, device="cuda"):
    """Lower-triangular A (m x m, lda = m) with singular values exactly 10^(-kband i/(m-1)),
    i = 0..m-1, so kappa_2(A) = 10^kband, and conditioning that no diagonal scaling removes
    (the construction of LAPACK's dlatms for a triangular factor): A = R^T with R the
    triangular factor of the QR factorisation of U diag(sigma) V^T, U and V Haar-random
    orthogonal (Q factors of Gaussian matrices).  The upper triangle is NaN; B ~ U(-1, 1)
    (m x n).  kband = 0 gives an orthogonal triangle, i.e. a diagonal of +-1.

    Returns (ncols, ld) views of column-major storage, as condition_band_lower_torch does.
    The factorisations run in FP64 on the device (torch.linalg.qr)."""
    return next(graded_condition_bands_torch(m, n, [kband], seed, device))[1:]


def graded_condition_bands_torch(m, n, kbands, seed, device="cuda"):
    """graded_condition_lower_torch for several bands with one pair U, V (two of the
    factorisations shared): yields (kband, At, Bt) in the order of kbands."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(seed)
    U, _ = torch.linalg.qr(torch.randn(m, m, generator=g, device=device, dtype=torch.float64))
    V, _ = torch.linalg.qr(torch.randn(m, m, generator=g, device=device, dtype=torch.float64))
    for kband in kbands:
        sig = torch.from_numpy(graded_sigma(m, kband)).to(device)
        M = (U * sig.view(1, m)) @ V.T
        R = torch.linalg.qr(M, mode="r")[1]
        del M
        # R upper triangular in row-major == At (row-major A^T) with A = R^T lower triangular:
        # At[j, i] = A(i, j) = R(j, i), so At is R itself
        nan_mask = torch.ones(m, m, dtype=torch.bool, device=device).tril_(-1)
        R.masked_fill_(nan_mask, float("nan"))
        del nan_mask
        Bt = torch.rand(n, m, generator=g, device=device, dtype=torch.float64) * 2.0 - 1.0
        yield kband, R.contiguous(), Bt.contiguous()


def graded_condition_problem(seed, m, n, kband, dtype=np.float64):
    """Host (numpy) version of graded_condition_lower_torch's construction (different RNG
    stream), for sizes the CPU oracle handles: column-major A (m x m, NaN upper triangle)
    and B (m x n)."""
    rng = np.random.default_rng(seed)
    U, _ = np.linalg.qr(rng.standard_normal((m, m)))
    V, _ = np.linalg.qr(rng.standard_normal((m, m)))
    M = (U * graded_sigma(m, kband)[None, :]) @ V.T
    R = np.linalg.qr(M, mode="r")
    A = np.array(R.T, order="F")
    A[np.triu_indices(m, 1)] = np.nan
    B = rng.uniform(-1.0, 1.0, size=(m, n))
    return np.asfortranarray(A.astype(dtype)), np.asfortranarray(B.astype(dtype))


def nan_triangle_problem(seed, side, uplo, trans, diag, m, n, lda, ldb, dtype):
    """The drop-in workload recipe: strictly-triangular entries of A ~ U(-1,1)/k, diagonal
    1 + U(0,1), the unused triangle NaN (so stray reads show up as NaN results); with
    diag U the stored diagonal is NaN as well.  B ~ U(-1,1); rows m..ldb-1 of B are NaN."""
    rng = np.random.default_rng(seed)
    k = m if side in ("L", 141) else n
    A = np.full((lda, k), np.nan, dtype=np.float64, order="F")
    vals = rng.uniform(-1.0, 1.0, size=(k, k)) / max(k, 1)
    lower = uplo in ("L", 122)
    mask = np.tril(np.ones((k, k), dtype=bool), -1) if lower else np.triu(np.ones((k, k), dtype=bool), 1)
    blk = np.where(mask, vals, np.nan)
    if diag in ("N", 131):
        blk[np.arange(k), np.arange(k)] = 1.0 + rng.uniform(0.0, 1.0, size=k)
    A[:k, :k] = blk
    B = np.full((ldb, n), np.nan, dtype=np.float64, order="F")
    B[:m, :] = rng.uniform(-1.0, 1.0, size=(m, n))
    if np.issubdtype(np.dtype(dtype), np.complexfloating):
        # complex: the same real parts, then imaginary parts U(-1,1)/k off the diagonal,
        # U(-0.5,0.5) on it and U(-1,1) in B (drawn after, so real streams are unchanged)
        im = np.where(mask, rng.uniform(-1.0, 1.0, size=(k, k)) / max(k, 1), 0.0)
        if diag in ("N", 131):
            im[np.arange(k), np.arange(k)] = rng.uniform(-0.5, 0.5, size=k)
        Ac = A.astype(np.complex128, order="F")
        Ac[:k, :k] += 1j * im
        Bc = B.astype(np.complex128, order="F")
        Bc[:m, :] += 1j * rng.uniform(-1.0, 1.0, size=(m, n))
        return Ac.astype(dtype, order="F"), Bc.astype(dtype, order="F")
    return A.astype(dtype, order="F"), B.astype(dtype, order="F")


def condition_band_problem(seed, m, n, kband, dtype=np.float64):
    """Host (numpy) version of :func:`condition_band_lower_torch`'s recipe (different RNG
    stream), for sizes the CPU oracle handles."""
    rng = np.random.default_rng(seed)
    G = rng.standard_normal((m, m)) / np.sqrt(m)
    d = 10.0 ** (-kband * np.arange(m) / m) * (1.0 + rng.uniform(0.0, 0.1, size=m))
    A = np.tril(G, -1) * d[:, None]
    A[np.arange(m), np.arange(m)] = d
    A[np.triu_indices(m, 1)] = np.nan
    B = rng.uniform(-1.0, 1.0, size=(m, n))
    return np.asfortranarray(A.astype(dtype)), np.asfortranarray(B.astype(dtype))
