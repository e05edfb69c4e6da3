"""Generate the committed golden vectors for the TRSM oracle and parity tests.

The reference ships no golden data for trsm: rocblas-test draws its inputs from a seeded
RNG and checks a GPU result against the host CBLAS it links (ref_trsm ->
cblas_?trsm, clients/common/cblas_interface.cpp:2352-2463) and against the X it built the
right-hand side from (ref_trmm, testing_trsm.hpp:311-315).  This script records exactly
those reference-side answers on fixed inputs so that they travel with the repository:

* ``cblas_<dt>.npz``  -- for every side/uplo/trans/diag combination and both precisions,
  A (unused triangle = NaN, diag-U cases with a NaN diagonal), B, alpha, and
  X = cblas_?trsm(A, B) computed by the host CBLAS (OpenBLAS as bundled with scipy, one of
  the CBLAS builds the reference links, clients/CMakeLists.txt:103-165);
* ``cblas_<c|z>.npz`` -- the same for complex data, trans C included, complex alpha;
* ``protocol_<dt>.npz`` -- rocblas-test's recipe: diagonally dominant integer A, integer X,
  B = op(A) X / alpha via cblas_?trmm; the known X is the answer.

Run from the repository root:  python tests/golden/make_golden.py
"""
import itertools
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402

COMBOS = list(itertools.product("LR", "UL", "NT", "NU"))
# (m, n, lda_pad, ldb_pad): ragged sizes, single rows and columns, a 32-row panel edge
SHAPES = [(37, 29, 3, 2), (1, 5, 0, 1), (5, 1, 1, 0), (33, 20, 0, 0)]


def main():
    oracle.cblas_set_threads(1)
    for dt, name in ((np.float64, "d"), (np.float32, "s")):
        out = {}
        for ci, (side, uplo, trans, diag) in enumerate(COMBOS):
            for si, (m, n, pa, pb) in enumerate(SHAPES):
                k = m if side == "L" else n
                seed = 1000 * ci + si
                A, B = oracle.nan_triangle_problem(seed, side, uplo, trans, diag, m, n, k + pa, m + pb, dt)
                alpha = 0.75 if (ci + si) % 2 else 1.0
                # the host CBLAS must not see NaN where the reference contract says "not read"
                X = oracle.cblas_trsm(side, uplo, trans, diag, alpha, A, np.asfortranarray(B[:m]))
                key = f"{side}{uplo}{trans}{diag}_{m}x{n}"
                out[key + "_A"] = A
                out[key + "_B"] = B
                out[key + "_alpha"] = np.array(alpha)
                out[key + "_X"] = X
        np.savez_compressed(os.path.join(HERE, f"cblas_{name}.npz"), **out)

        out = {}
        for ci, (side, uplo, trans, diag) in enumerate(COMBOS):
            m, n = (24, 33) if ci % 2 else (33, 24)
            k = m if side == "L" else n
            alpha = 2.0 if ci % 3 == 0 else 1.0
            A, B, X = oracle.rocblas_test_problem(7 + ci, side, uplo, trans, diag, m, n, k + 1, m + 1,
                                                  alpha, dt)
            # B = op(A) X / alpha by the host CBLAS trmm (what ref_trmm calls)
            Bc = oracle.cblas_trmm(side, uplo, trans, diag, 1.0 / alpha, A, X)
            key = f"{side}{uplo}{trans}{diag}"
            out[key + "_A"] = A
            out[key + "_B"] = Bc
            out[key + "_X"] = X
            out[key + "_alpha"] = np.array(alpha)
        np.savez_compressed(os.path.join(HERE, f"protocol_{name}.npz"), **out)
    complex_fixtures()
    print("wrote", sorted(f for f in os.listdir(HERE) if f.endswith(".npz")))


# complex: trans C as well (conj(A)), complex alpha
COMBOS_C = list(itertools.product("LR", "UL", "NTC", "NU"))
SHAPES_C = [(21, 13, 3, 2), (5, 1, 1, 0)]


def complex_fixtures():
    """``cblas_<c|z>.npz``: the same recipe with complex A and B (imaginary parts drawn after the
    real ones) and X from cblas_{c,z}trsm."""
    oracle.cblas_set_threads(1)
    for dt, name in ((np.complex128, "z"), (np.complex64, "c")):
        out = {}
        for ci, (side, uplo, trans, diag) in enumerate(COMBOS_C):
            for si, (m, n, pa, pb) in enumerate(SHAPES_C):
                k = m if side == "L" else n
                seed = 5000 + 1000 * ci + si
                A, B = oracle.nan_triangle_problem(seed, side, uplo, trans, diag, m, n, k + pa, m + pb, dt)
                alpha = 0.75 - 0.5j if (ci + si) % 2 else 1.0 + 0.0j
                X = oracle.cblas_trsm(side, uplo, trans, diag, alpha, A, np.asfortranarray(B[:m]))
                key = f"{side}{uplo}{trans}{diag}_{m}x{n}"
                out[key + "_A"] = A
                out[key + "_B"] = B
                out[key + "_alpha"] = np.array(alpha)
                out[key + "_X"] = X
        np.savez_compressed(os.path.join(HERE, f"cblas_{name}.npz"), **out)


if __name__ == "__main__":
    main()
