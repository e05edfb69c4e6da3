/*
 * CPU oracle for the TRSM hot path.  TEST INFRASTRUCTURE ONLY: this file is the checker
 * that tests, smoke() and the bench's CPU-baseline leg compare the CUDA library against.
 * Nothing in the shipped library links or calls it.
 *
 * What it restates.  rocblas-test checks rocblas_?trsm against the host BLAS it links
 * (clients/common/cblas_interface.cpp:2352-2463, ref_trsm -> cblas_?trsm; the forward
 * operator ref_trmm -> cblas_?trmm at :2465-2575).  That host BLAS is third-party and not
 * vendored in the reference (netlib LAPACK v3.9.1 with -DCBLAS=ON per
 * deps/external-lapack.cmake, or AOCL-BLIS / OpenBLAS per clients/CMakeLists.txt:103-165).
 * The functions below restate the published netlib reference-BLAS algorithms for
 * xTRSM / xTRMM (column-oriented substitution, alpha applied per column, zero-skip on
 * B(k,j)/A(k,j)) in C, with the same argument meaning, in three arithmetics:
 *   - s*: float storage, float arithmetic (what cblas_strsm computes),
 *   - d*: double storage, double arithmetic (cblas_dtrsm),
 *   - q*: double storage, __float128 arithmetic (an extended-precision X* used to measure
 *         normwise forward error at the 1e-12 level).
 * The diagonal-block inverse (q/d/s trtri) restates rocblas_trtri semantics
 * (library/src/blas3/rocblas_trtri.hpp:128-141): unit diagonal -> 1, and a zero
 * non-unit diagonal entry is treated as 1 ("means the matrix is singular").
 *
 * Enum values are the rocblas/CBLAS ones (library/include/internal/rocblas-types.h:123-172):
 *   side 141 L / 142 R, uplo 121 U / 122 L, trans 111 N / 112 T / 113 C, diag 131 N / 132 U.
 */
#include <stddef.h>
#include <stdint.h>
#include <string.h>
#include <quadmath.h>
#include <stdlib.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define SIDE_L 141
#define UPLO_U 121
#define TRANS_N 111
#define DIAG_U 132

#define IDX(i, j, ld) ((size_t)(i) + (size_t)(j) * (size_t)(ld))

/* ---------------------------------------------------------------------------------------
 * xTRSM:  op(A) X = alpha B (side L) or X op(A) = alpha B (side R); X overwrites B.
 * TS = storage type, TC = compute type.
 * --------------------------------------------------------------------------------------- */
#define DEFINE_TRSM(NAME, TS, TC)                                                             \
    void NAME(int side, int uplo, int trans, int diag, int64_t m, int64_t n, double alpha_d,  \
              const TS* A, int64_t lda, TS* B, int64_t ldb)                                   \
    {                                                                                         \
        const TC alpha   = (TC)alpha_d;                                                       \
        const int nounit = diag != DIAG_U;                                                    \
        const int upper  = uplo == UPLO_U;                                                    \
        const int notr   = trans == TRANS_N;                                                  \
        if(m <= 0 || n <= 0)                                                                  \
            return;                                                                           \
        if(alpha_d == 0.0)                                                                    \
        {                                                                                     \
            for(int64_t j = 0; j < n; ++j)                                                    \
                for(int64_t i = 0; i < m; ++i)                                                \
                    B[IDX(i, j, ldb)] = (TS)0;                                                \
            return;                                                                           \
        }                                                                                     \
        /* work copy of B in the compute type, ld = m, so that every intermediate */         \
        /* keeps TC precision (matters for the __float128 variant only)          */         \
        TC* W = (TC*)malloc(sizeof(TC) * (size_t)m * (size_t)n);                              \
        for(int64_t j = 0; j < n; ++j)                                                        \
            for(int64_t i = 0; i < m; ++i)                                                    \
                W[IDX(i, j, m)] = (TC)B[IDX(i, j, ldb)];                                      \
        if(side == SIDE_L)                                                                    \
        {                                                                                     \
            /* columns of B are independent solves */                                         \
            _Pragma("omp parallel for schedule(dynamic, 1)")                                  \
            for(int64_t j = 0; j < n; ++j)                                                    \
            {                                                                                 \
                TC* b = W + (size_t)j * (size_t)m;                                            \
                if(notr && upper)                                                             \
                {                                                                             \
                    if(alpha != (TC)1)                                                        \
                        for(int64_t i = 0; i < m; ++i) b[i] = alpha * b[i];                   \
                    for(int64_t k = m - 1; k >= 0; --k)                                       \
                        if(b[k] != (TC)0)                                                     \
                        {                                                                     \
                            if(nounit) b[k] = b[k] / (TC)A[IDX(k, k, lda)];                   \
                            const TC bk = b[k];                                               \
                            for(int64_t i = 0; i < k; ++i)                                    \
                                b[i] -= bk * (TC)A[IDX(i, k, lda)];                           \
                        }                                                                     \
                }                                                                             \
                else if(notr)                                                                 \
                {                                                                             \
                    if(alpha != (TC)1)                                                        \
                        for(int64_t i = 0; i < m; ++i) b[i] = alpha * b[i];                   \
                    for(int64_t k = 0; k < m; ++k)                                            \
                        if(b[k] != (TC)0)                                                     \
                        {                                                                     \
                            if(nounit) b[k] = b[k] / (TC)A[IDX(k, k, lda)];                   \
                            const TC bk = b[k];                                               \
                            for(int64_t i = k + 1; i < m; ++i)                                \
                                b[i] -= bk * (TC)A[IDX(i, k, lda)];                           \
                        }                                                                     \
                }                                                                             \
                else if(upper)                                                                \
                {                                                                             \
                    for(int64_t i = 0; i < m; ++i)                                            \
                    {                                                                         \
                        TC t = alpha * b[i];                                                  \
                        for(int64_t k = 0; k < i; ++k) t -= (TC)A[IDX(k, i, lda)] * b[k];     \
                        if(nounit) t = t / (TC)A[IDX(i, i, lda)];                             \
                        b[i] = t;                                                             \
                    }                                                                         \
                }                                                                             \
                else                                                                          \
                {                                                                             \
                    for(int64_t i = m - 1; i >= 0; --i)                                       \
                    {                                                                         \
                        TC t = alpha * b[i];                                                  \
                        for(int64_t k = i + 1; k < m; ++k) t -= (TC)A[IDX(k, i, lda)] * b[k]; \
                        if(nounit) t = t / (TC)A[IDX(i, i, lda)];                             \
                        b[i] = t;                                                             \
                    }                                                                         \
                }                                                                             \
            }                                                                                 \
        }                                                                                     \
        else                                                                                  \
        {                                                                                     \
            /* side R: the column form of the netlib loops; rows are independent, so */      \
            /* the row range is split across threads                                 */      \
            _Pragma("omp parallel")                                                           \
            {                                                                                 \
                int64_t r0 = 0, r1 = m;                                                       \
                oracle_split_rows(m, &r0, &r1);                                               \
                TRSM_RIGHT_BODY(TC)                                                           \
            }                                                                                 \
        }                                                                                     \
        for(int64_t j = 0; j < n; ++j)                                                        \
            for(int64_t i = 0; i < m; ++i)                                                    \
                B[IDX(i, j, ldb)] = (TS)W[IDX(i, j, m)];                                      \
        free(W);                                                                              \
    }

/* rows [r0, r1) of W, side R, in the netlib loop order */
#define TRSM_RIGHT_BODY(TC)                                                                   \
    if(notr && upper)                                                                         \
    {                                                                                         \
        for(int64_t j = 0; j < n; ++j)                                                        \
        {                                                                                     \
            TC* bj = W + (size_t)j * m;                                                       \
            if(alpha != (TC)1)                                                                \
                for(int64_t i = r0; i < r1; ++i) bj[i] = alpha * bj[i];                       \
            for(int64_t k = 0; k < j; ++k)                                                    \
            {                                                                                 \
                const TC akj = (TC)A[IDX(k, j, lda)];                                         \
                if(akj != (TC)0)                                                              \
                {                                                                             \
                    const TC* bk = W + (size_t)k * m;                                         \
                    for(int64_t i = r0; i < r1; ++i) bj[i] -= akj * bk[i];                    \
                }                                                                             \
            }                                                                                 \
            if(nounit)                                                                        \
            {                                                                                 \
                const TC t = (TC)1 / (TC)A[IDX(j, j, lda)];                                   \
                for(int64_t i = r0; i < r1; ++i) bj[i] = t * bj[i];                           \
            }                                                                                 \
        }                                                                                     \
    }                                                                                         \
    else if(notr)                                                                             \
    {                                                                                         \
        for(int64_t j = n - 1; j >= 0; --j)                                                   \
        {                                                                                     \
            TC* bj = W + (size_t)j * m;                                                       \
            if(alpha != (TC)1)                                                                \
                for(int64_t i = r0; i < r1; ++i) bj[i] = alpha * bj[i];                       \
            for(int64_t k = j + 1; k < n; ++k)                                                \
            {                                                                                 \
                const TC akj = (TC)A[IDX(k, j, lda)];                                         \
                if(akj != (TC)0)                                                              \
                {                                                                             \
                    const TC* bk = W + (size_t)k * m;                                         \
                    for(int64_t i = r0; i < r1; ++i) bj[i] -= akj * bk[i];                    \
                }                                                                             \
            }                                                                                 \
            if(nounit)                                                                        \
            {                                                                                 \
                const TC t = (TC)1 / (TC)A[IDX(j, j, lda)];                                   \
                for(int64_t i = r0; i < r1; ++i) bj[i] = t * bj[i];                           \
            }                                                                                 \
        }                                                                                     \
    }                                                                                         \
    else if(upper)                                                                            \
    {                                                                                         \
        for(int64_t k = n - 1; k >= 0; --k)                                                   \
        {                                                                                     \
            TC* bk = W + (size_t)k * m;                                                       \
            if(nounit)                                                                        \
            {                                                                                 \
                const TC t = (TC)1 / (TC)A[IDX(k, k, lda)];                                   \
                for(int64_t i = r0; i < r1; ++i) bk[i] = t * bk[i];                           \
            }                                                                                 \
            for(int64_t j = 0; j < k; ++j)                                                    \
            {                                                                                 \
                const TC ajk = (TC)A[IDX(j, k, lda)];                                         \
                if(ajk != (TC)0)                                                              \
                {                                                                             \
                    TC* bj = W + (size_t)j * m;                                               \
                    for(int64_t i = r0; i < r1; ++i) bj[i] -= ajk * bk[i];                    \
                }                                                                             \
            }                                                                                 \
            if(alpha != (TC)1)                                                                \
                for(int64_t i = r0; i < r1; ++i) bk[i] = alpha * bk[i];                       \
        }                                                                                     \
    }                                                                                         \
    else                                                                                      \
    {                                                                                         \
        for(int64_t k = 0; k < n; ++k)                                                        \
        {                                                                                     \
            TC* bk = W + (size_t)k * m;                                                       \
            if(nounit)                                                                        \
            {                                                                                 \
                const TC t = (TC)1 / (TC)A[IDX(k, k, lda)];                                   \
                for(int64_t i = r0; i < r1; ++i) bk[i] = t * bk[i];                           \
            }                                                                                 \
            for(int64_t j = k + 1; j < n; ++j)                                                \
            {                                                                                 \
                const TC ajk = (TC)A[IDX(j, k, lda)];                                         \
                if(ajk != (TC)0)                                                              \
                {                                                                             \
                    TC* bj = W + (size_t)j * m;                                               \
                    for(int64_t i = r0; i < r1; ++i) bj[i] -= ajk * bk[i];                    \
                }                                                                             \
            }                                                                                 \
            if(alpha != (TC)1)                                                                \
                for(int64_t i = r0; i < r1; ++i) bk[i] = alpha * bk[i];                       \
        }                                                                                     \
    }

static void oracle_split_rows(int64_t m, int64_t* r0, int64_t* r1)
{
#ifdef _OPENMP
    int nt = omp_get_num_threads(), t = omp_get_thread_num();
#else
    int nt = 1, t = 0;
#endif
    int64_t chunk = (m + nt - 1) / nt;
    *r0 = (int64_t)t * chunk;
    *r1 = *r0 + chunk < m ? *r0 + chunk : m;
    if(*r0 > m)
        *r0 = m;
}

DEFINE_TRSM(oracle_strsm, float, float)
DEFINE_TRSM(oracle_dtrsm, double, double)
DEFINE_TRSM(oracle_qtrsm, double, __float128)

/* ---------------------------------------------------------------------------------------
 * xTRMM: B := alpha op(A) B (side L) or alpha B op(A) (side R).  Used to build the
 * right-hand side from a known X (the rocblas-test protocol,
 * clients/include/blas3/testing_trsm.hpp:311-315) and for residuals.  Computed per
 * output element as a dot product in TC, so it is order-independent of B's update.
 * --------------------------------------------------------------------------------------- */
static inline int tri_has(int upper, int64_t i, int64_t j)
{
    return upper ? (i <= j) : (i >= j);
}

#define DEFINE_TRMM(NAME, TS, TC)                                                             \
    void NAME(int side, int uplo, int trans, int diag, int64_t m, int64_t n, double alpha_d,  \
              const TS* A, int64_t lda, const TS* X, int64_t ldx, TS* C, int64_t ldc)         \
    {                                                                                         \
        const TC alpha  = (TC)alpha_d;                                                        \
        const int unit  = diag == DIAG_U;                                                     \
        const int upper = uplo == UPLO_U;                                                     \
        const int notr  = trans == TRANS_N;                                                   \
        const int64_t k = side == SIDE_L ? m : n;                                             \
        _Pragma("omp parallel for schedule(dynamic, 1)")                                      \
        for(int64_t j = 0; j < n; ++j)                                                        \
            for(int64_t i = 0; i < m; ++i)                                                    \
            {                                                                                 \
                TC s = 0;                                                                     \
                for(int64_t t = 0; t < k; ++t)                                                \
                {                                                                             \
                    /* op(A)(r,c) = A(r,c) or A(c,r) */                                       \
                    int64_t r, c;                                                             \
                    TC xv;                                                                    \
                    if(side == SIDE_L) { r = i; c = t; xv = (TC)X[IDX(t, j, ldx)]; }          \
                    else               { r = t; c = j; xv = (TC)X[IDX(i, t, ldx)]; }          \
                    int64_t ar = notr ? r : c, ac = notr ? c : r;                             \
                    if(!tri_has(upper, ar, ac))                                               \
                        continue;                                                             \
                    TC a = (ar == ac && unit) ? (TC)1 : (TC)A[IDX(ar, ac, lda)];              \
                    s += a * xv;                                                              \
                }                                                                             \
                C[IDX(i, j, ldc)] = (TS)(alpha * s);                                          \
            }                                                                                 \
    }

DEFINE_TRMM(oracle_strmm, float, float)
DEFINE_TRMM(oracle_dtrmm, double, double)
DEFINE_TRMM(oracle_qtrmm, double, __float128)

/* ---------------------------------------------------------------------------------------
 * xTRTRI: invA := inv(A) for a triangular n x n A, computed column by column by
 * substitution in TC.  The opposite triangle of invA is written as 0 (the fill that
 * rocblas_trtri_fill performs for the trsm path, rocblas_trtri.hpp:393-426).
 * --------------------------------------------------------------------------------------- */
#define DEFINE_TRTRI(NAME, TS, TC)                                                            \
    void NAME(int uplo, int diag, int64_t n, const TS* A, int64_t lda, TS* invA,              \
              int64_t ldinv)                                                                  \
    {                                                                                         \
        const int unit  = diag == DIAG_U;                                                     \
        const int upper = uplo == UPLO_U;                                                     \
        _Pragma("omp parallel for schedule(dynamic, 1)")                                      \
        for(int64_t j = 0; j < n; ++j)                                                        \
        {                                                                                     \
            /* column j of inv(A): solve A x = e_j */                                         \
            TC x[n > 0 ? n : 1];                                                              \
            for(int64_t i = 0; i < n; ++i) x[i] = (i == j) ? (TC)1 : (TC)0;                   \
            if(!upper)                                                                        \
            {                                                                                 \
                for(int64_t i = j; i < n; ++i)                                                \
                {                                                                             \
                    TC s = x[i];                                                              \
                    for(int64_t t = j; t < i; ++t) s -= (TC)A[IDX(i, t, lda)] * x[t];         \
                    TC d = unit ? (TC)1 : (TC)A[IDX(i, i, lda)];                              \
                    if(d == (TC)0) d = (TC)1;                                                 \
                    x[i] = s / d;                                                             \
                }                                                                             \
            }                                                                                 \
            else                                                                              \
            {                                                                                 \
                for(int64_t i = j; i >= 0; --i)                                               \
                {                                                                             \
                    TC s = x[i];                                                              \
                    for(int64_t t = i + 1; t <= j; ++t) s -= (TC)A[IDX(i, t, lda)] * x[t];    \
                    TC d = unit ? (TC)1 : (TC)A[IDX(i, i, lda)];                              \
                    if(d == (TC)0) d = (TC)1;                                                 \
                    x[i] = s / d;                                                             \
                }                                                                             \
            }                                                                                 \
            for(int64_t i = 0; i < n; ++i)                                                    \
                invA[IDX(i, j, ldinv)] = tri_has(upper, i, j) ? (TS)x[i] : (TS)0;             \
        }                                                                                     \
    }

DEFINE_TRTRI(oracle_strtri, float, float)
DEFINE_TRTRI(oracle_dtrtri, double, double)
DEFINE_TRTRI(oracle_qtrtri, double, __float128)

/* The reference's forward-error / residual norm (clients/include/norm.hpp:449-492):
 * the running sums err and err_scal are NOT reset per column, so the value returned is
 * max over prefixes, which equals total |gold-x| / total |gold| (both sums are
 * monotone).  Restated as-is so our gate is the gate rocblas-test applies. */
double oracle_matrix_norm_1_d(int64_t M, int64_t N, const double* gold, int64_t ldg,
                              const double* x, int64_t ldx)
{
    double max_err_scal = 0.0, max_err = 0.0, err = 0.0, err_scal = 0.0;
    for(int64_t i = 0; i < N; i++)
    {
        for(int64_t j = 0; j < M; j++)
        {
            double g = gold[IDX(j, i, ldg)];
            double v = x[IDX(j, i, ldx)];
            err += g > v ? g - v : v - g;
            err_scal += g >= 0 ? g : -g;
        }
        max_err_scal = max_err_scal > err_scal ? max_err_scal : err_scal;
        max_err      = max_err > err ? max_err : err;
    }
    return max_err / max_err_scal;
}
