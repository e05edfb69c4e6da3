/*
 * Complex (c / z) part of the CPU oracle.  TEST INFRASTRUCTURE ONLY, like trsm_oracle.c: the
 * checker that tests compare the CUDA library against; nothing in the library links it.
 *
 * What it restates.  For complex types rocblas-test checks rocblas_{c,z}trsm against the host
 * BLAS through ref_trsm -> cblas_{c,z}trsm and builds its right-hand sides with
 * ref_trmm -> cblas_{c,z}trmm (clients/common/cblas_interface.cpp:2352-2575).  The functions
 * below restate the published netlib reference-BLAS CTRSM / ZTRSM and CTRMM / ZTRMM in C99
 * complex arithmetic: column-oriented substitution with alpha applied per column, the zero
 * skips on B(k,j) / A(k,j), the side-right reciprocal-then-scale of the diagonal, and
 * trans = C reading conj(A).  Storage and arithmetic are the same type (float _Complex for c,
 * double _Complex for z), as in the host BLAS.
 *
 * The forward-error norm for complex follows clients/include/norm.hpp:449-492 with
 * rocblas_abs = the complex modulus (library/src/include/utility.hpp:605-610).
 *
 * Enum values are the rocblas/CBLAS ones (library/include/internal/rocblas-types.h:123-172).
 */
#include <complex.h>
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define C_SIDE_L 141
#define C_UPLO_U 121
#define C_TRANS_N 111
#define C_TRANS_C 113
#define C_DIAG_U 132

#define CIDX(i, j, ld) ((size_t)(i) + (size_t)(j) * (size_t)(ld))

/* rows [r0, r1) of an m-row matrix for the calling OpenMP thread */
static void crows(int64_t m, int64_t* r0, int64_t* r1)
{
#ifdef _OPENMP
    const int64_t nt = omp_get_num_threads(), t = omp_get_thread_num();
#else
    const int64_t nt = 1, t = 0;
#endif
    const int64_t per = (m + nt - 1) / nt;
    *r0 = t * per < m ? t * per : m;
    *r1 = *r0 + per < m ? *r0 + per : m;
}

/* op(A) entry reader: A(i,j), conjugated when trans == C (CONJ is conjf or conj, defined
 * before each instantiation) */
#define AV(i, j) (noconj ? A[CIDX(i, j, lda)] : CONJ(A[CIDX(i, j, lda)]))

/* ---- xTRSM: op(A) X = alpha B (side L) or X op(A) = alpha B (side R); X overwrites B --- */
#define DEFINE_CTRSM(NAME, T)                                                                 \
    void NAME(int side, int uplo, int trans, int diag, int64_t m, int64_t n, double ar,       \
              double ai, const T* A, int64_t lda, T* B, int64_t ldb)                          \
    {                                                                                         \
        const T   alpha  = (T)ar + (T)ai * (T)I;                                              \
        const T   one    = (T)1;                                                              \
        const int nounit = diag != C_DIAG_U;                                                  \
        const int upper  = uplo == C_UPLO_U;                                                  \
        const int notr   = trans == C_TRANS_N;                                                \
        const int noconj = trans != C_TRANS_C;                                                \
        if(m <= 0 || n <= 0)                                                                  \
            return;                                                                           \
        if(alpha == (T)0)                                                                     \
        {                                                                                     \
            for(int64_t j = 0; j < n; ++j)                                                    \
                for(int64_t i = 0; i < m; ++i)                                                \
                    B[CIDX(i, j, ldb)] = (T)0;                                                \
            return;                                                                           \
        }                                                                                     \
        if(side == C_SIDE_L)                                                                  \
        {                                                                                     \
            _Pragma("omp parallel for schedule(dynamic, 1)")                                  \
            for(int64_t j = 0; j < n; ++j)                                                    \
            {                                                                                 \
                T* b = B + (size_t)j * (size_t)ldb;                                           \
                if(notr && upper)                                                             \
                {                                                                             \
                    if(alpha != one)                                                          \
                        for(int64_t i = 0; i < m; ++i) b[i] = alpha * b[i];                   \
                    for(int64_t k = m - 1; k >= 0; --k)                                       \
                        if(b[k] != (T)0)                                                      \
                        {                                                                     \
                            if(nounit) b[k] = b[k] / A[CIDX(k, k, lda)];                      \
                            const T bk = b[k];                                                \
                            for(int64_t i = 0; i < k; ++i)                                    \
                                b[i] -= bk * A[CIDX(i, k, lda)];                              \
                        }                                                                     \
                }                                                                             \
                else if(notr)                                                                 \
                {                                                                             \
                    if(alpha != one)                                                          \
                        for(int64_t i = 0; i < m; ++i) b[i] = alpha * b[i];                   \
                    for(int64_t k = 0; k < m; ++k)                                            \
                        if(b[k] != (T)0)                                                      \
                        {                                                                     \
                            if(nounit) b[k] = b[k] / A[CIDX(k, k, lda)];                      \
                            const T bk = b[k];                                                \
                            for(int64_t i = k + 1; i < m; ++i)                                \
                                b[i] -= bk * A[CIDX(i, k, lda)];                              \
                        }                                                                     \
                }                                                                             \
                else if(upper)                                                                \
                {                                                                             \
                    for(int64_t i = 0; i < m; ++i)                                            \
                    {                                                                         \
                        T t = alpha * b[i];                                                   \
                        for(int64_t k = 0; k < i; ++k) t -= AV(k, i) * b[k];                  \
                        if(nounit) t = t / AV(i, i);                                          \
                        b[i] = t;                                                             \
                    }                                                                         \
                }                                                                             \
                else                                                                          \
                {                                                                             \
                    for(int64_t i = m - 1; i >= 0; --i)                                       \
                    {                                                                         \
                        T t = alpha * b[i];                                                   \
                        for(int64_t k = i + 1; k < m; ++k) t -= AV(k, i) * b[k];              \
                        if(nounit) t = t / AV(i, i);                                          \
                        b[i] = t;                                                             \
                    }                                                                         \
                }                                                                             \
            }                                                                                 \
            return;                                                                           \
        }                                                                                     \
        /* side R: rows of B are independent; each thread runs the netlib loops on its */    \
        /* row range                                                                    */    \
        _Pragma("omp parallel")                                                               \
        {                                                                                     \
            int64_t r0, r1;                                                                   \
            crows(m, &r0, &r1);                                                               \
            if(notr && upper)                                                                 \
            {                                                                                 \
                for(int64_t j = 0; j < n; ++j)                                                \
                {                                                                             \
                    if(alpha != one)                                                          \
                        for(int64_t i = r0; i < r1; ++i) B[CIDX(i, j, ldb)] *= alpha;         \
                    for(int64_t k = 0; k < j; ++k)                                            \
                        if(A[CIDX(k, j, lda)] != (T)0)                                        \
                        {                                                                     \
                            const T a = A[CIDX(k, j, lda)];                                   \
                            for(int64_t i = r0; i < r1; ++i)                                  \
                                B[CIDX(i, j, ldb)] -= a * B[CIDX(i, k, ldb)];                 \
                        }                                                                     \
                    if(nounit)                                                                \
                    {                                                                         \
                        const T t = one / A[CIDX(j, j, lda)];                                 \
                        for(int64_t i = r0; i < r1; ++i) B[CIDX(i, j, ldb)] *= t;             \
                    }                                                                         \
                }                                                                             \
            }                                                                                 \
            else if(notr)                                                                     \
            {                                                                                 \
                for(int64_t j = n - 1; j >= 0; --j)                                           \
                {                                                                             \
                    if(alpha != one)                                                          \
                        for(int64_t i = r0; i < r1; ++i) B[CIDX(i, j, ldb)] *= alpha;         \
                    for(int64_t k = j + 1; k < n; ++k)                                        \
                        if(A[CIDX(k, j, lda)] != (T)0)                                        \
                        {                                                                     \
                            const T a = A[CIDX(k, j, lda)];                                   \
                            for(int64_t i = r0; i < r1; ++i)                                  \
                                B[CIDX(i, j, ldb)] -= a * B[CIDX(i, k, ldb)];                 \
                        }                                                                     \
                    if(nounit)                                                                \
                    {                                                                         \
                        const T t = one / A[CIDX(j, j, lda)];                                 \
                        for(int64_t i = r0; i < r1; ++i) B[CIDX(i, j, ldb)] *= t;             \
                    }                                                                         \
                }                                                                             \
            }                                                                                 \
            else if(upper)                                                                    \
            {                                                                                 \
                for(int64_t k = n - 1; k >= 0; --k)                                           \
                {                                                                             \
                    if(nounit)                                                                \
                    {                                                                         \
                        const T t = one / AV(k, k);                                           \
                        for(int64_t i = r0; i < r1; ++i) B[CIDX(i, k, ldb)] *= t;             \
                    }                                                                         \
                    for(int64_t j = 0; j < k; ++j)                                            \
                        if(A[CIDX(j, k, lda)] != (T)0)                                        \
                        {                                                                     \
                            const T t = AV(j, k);                                             \
                            for(int64_t i = r0; i < r1; ++i)                                  \
                                B[CIDX(i, j, ldb)] -= t * B[CIDX(i, k, ldb)];                 \
                        }                                                                     \
                    if(alpha != one)                                                          \
                        for(int64_t i = r0; i < r1; ++i) B[CIDX(i, k, ldb)] *= alpha;         \
                }                                                                             \
            }                                                                                 \
            else                                                                              \
            {                                                                                 \
                for(int64_t k = 0; k < n; ++k)                                                \
                {                                                                             \
                    if(nounit)                                                                \
                    {                                                                         \
                        const T t = one / AV(k, k);                                           \
                        for(int64_t i = r0; i < r1; ++i) B[CIDX(i, k, ldb)] *= t;             \
                    }                                                                         \
                    for(int64_t j = k + 1; j < n; ++j)                                        \
                        if(A[CIDX(j, k, lda)] != (T)0)                                        \
                        {                                                                     \
                            const T t = AV(j, k);                                             \
                            for(int64_t i = r0; i < r1; ++i)                                  \
                                B[CIDX(i, j, ldb)] -= t * B[CIDX(i, k, ldb)];                 \
                        }                                                                     \
                    if(alpha != one)                                                          \
                        for(int64_t i = r0; i < r1; ++i) B[CIDX(i, k, ldb)] *= alpha;         \
                }                                                                             \
            }                                                                                 \
        }                                                                                     \
    }

#define CONJ conjf
DEFINE_CTRSM(oracle_ctrsm, float _Complex)
#undef CONJ
#define CONJ conj
DEFINE_CTRSM(oracle_ztrsm, double _Complex)
#undef CONJ

/* ---- xTRMM, out of place: C := alpha op(A) X (side L) or alpha X op(A) (side R) ---------- */
#define DEFINE_CTRMM(NAME, T)                                                                 \
    void NAME(int side, int uplo, int trans, int diag, int64_t m, int64_t n, double ar,       \
              double ai, const T* A, int64_t lda, const T* X, int64_t ldx, T* B, int64_t ldb) \
    {                                                                                         \
        const T   alpha  = (T)ar + (T)ai * (T)I;                                              \
        const T   one    = (T)1;                                                              \
        const int nounit = diag != C_DIAG_U;                                                  \
        const int upper  = uplo == C_UPLO_U;                                                  \
        const int notr   = trans == C_TRANS_N;                                                \
        const int noconj = trans != C_TRANS_C;                                                \
        if(m <= 0 || n <= 0)                                                                  \
            return;                                                                           \
        for(int64_t j = 0; j < n; ++j)                                                        \
            for(int64_t i = 0; i < m; ++i)                                                    \
                B[CIDX(i, j, ldb)] = alpha == (T)0 ? (T)0 : X[CIDX(i, j, ldx)];               \
        if(alpha == (T)0)                                                                     \
            return;                                                                           \
        if(side == C_SIDE_L)                                                                  \
        {                                                                                     \
            _Pragma("omp parallel for schedule(dynamic, 1)")                                  \
            for(int64_t j = 0; j < n; ++j)                                                    \
            {                                                                                 \
                T* b = B + (size_t)j * (size_t)ldb;                                           \
                if(notr && upper)                                                             \
                {                                                                             \
                    for(int64_t k = 0; k < m; ++k)                                            \
                        if(b[k] != (T)0)                                                      \
                        {                                                                     \
                            T t = alpha * b[k];                                               \
                            for(int64_t i = 0; i < k; ++i) b[i] += t * A[CIDX(i, k, lda)];    \
                            if(nounit) t = t * A[CIDX(k, k, lda)];                            \
                            b[k] = t;                                                         \
                        }                                                                     \
                }                                                                             \
                else if(notr)                                                                 \
                {                                                                             \
                    for(int64_t k = m - 1; k >= 0; --k)                                       \
                        if(b[k] != (T)0)                                                      \
                        {                                                                     \
                            const T t = alpha * b[k];                                         \
                            b[k] = t;                                                         \
                            if(nounit) b[k] = b[k] * A[CIDX(k, k, lda)];                      \
                            for(int64_t i = k + 1; i < m; ++i) b[i] += t * A[CIDX(i, k, lda)]; \
                        }                                                                     \
                }                                                                             \
                else if(upper)                                                                \
                {                                                                             \
                    for(int64_t i = m - 1; i >= 0; --i)                                       \
                    {                                                                         \
                        T t = b[i];                                                           \
                        if(nounit) t = t * AV(i, i);                                          \
                        for(int64_t k = 0; k < i; ++k) t += AV(k, i) * b[k];                  \
                        b[i] = alpha * t;                                                     \
                    }                                                                         \
                }                                                                             \
                else                                                                          \
                {                                                                             \
                    for(int64_t i = 0; i < m; ++i)                                            \
                    {                                                                         \
                        T t = b[i];                                                           \
                        if(nounit) t = t * AV(i, i);                                          \
                        for(int64_t k = i + 1; k < m; ++k) t += AV(k, i) * b[k];              \
                        b[i] = alpha * t;                                                     \
                    }                                                                         \
                }                                                                             \
            }                                                                                 \
            return;                                                                           \
        }                                                                                     \
        _Pragma("omp parallel")                                                               \
        {                                                                                     \
            int64_t r0, r1;                                                                   \
            crows(m, &r0, &r1);                                                               \
            if(notr && upper)                                                                 \
            {                                                                                 \
                for(int64_t j = n - 1; j >= 0; --j)                                           \
                {                                                                             \
                    T t = alpha;                                                              \
                    if(nounit) t = t * A[CIDX(j, j, lda)];                                    \
                    for(int64_t i = r0; i < r1; ++i) B[CIDX(i, j, ldb)] *= t;                 \
                    for(int64_t k = 0; k < j; ++k)                                            \
                        if(A[CIDX(k, j, lda)] != (T)0)                                        \
                        {                                                                     \
                            const T s = alpha * A[CIDX(k, j, lda)];                           \
                            for(int64_t i = r0; i < r1; ++i)                                  \
                                B[CIDX(i, j, ldb)] += s * B[CIDX(i, k, ldb)];                 \
                        }                                                                     \
                }                                                                             \
            }                                                                                 \
            else if(notr)                                                                     \
            {                                                                                 \
                for(int64_t j = 0; j < n; ++j)                                                \
                {                                                                             \
                    T t = alpha;                                                              \
                    if(nounit) t = t * A[CIDX(j, j, lda)];                                    \
                    for(int64_t i = r0; i < r1; ++i) B[CIDX(i, j, ldb)] *= t;                 \
                    for(int64_t k = j + 1; k < n; ++k)                                        \
                        if(A[CIDX(k, j, lda)] != (T)0)                                        \
                        {                                                                     \
                            const T s = alpha * A[CIDX(k, j, lda)];                           \
                            for(int64_t i = r0; i < r1; ++i)                                  \
                                B[CIDX(i, j, ldb)] += s * B[CIDX(i, k, ldb)];                 \
                        }                                                                     \
                }                                                                             \
            }                                                                                 \
            else if(upper)                                                                    \
            {                                                                                 \
                for(int64_t k = 0; k < n; ++k)                                                \
                {                                                                             \
                    for(int64_t j = 0; j < k; ++j)                                            \
                        if(A[CIDX(j, k, lda)] != (T)0)                                        \
                        {                                                                     \
                            const T s = alpha * AV(j, k);                                     \
                            for(int64_t i = r0; i < r1; ++i)                                  \
                                B[CIDX(i, j, ldb)] += s * B[CIDX(i, k, ldb)];                 \
                        }                                                                     \
                    T t = alpha;                                                              \
                    if(nounit) t = t * AV(k, k);                                              \
                    if(t != one)                                                              \
                        for(int64_t i = r0; i < r1; ++i) B[CIDX(i, k, ldb)] *= t;             \
                }                                                                             \
            }                                                                                 \
            else                                                                              \
            {                                                                                 \
                for(int64_t k = n - 1; k >= 0; --k)                                           \
                {                                                                             \
                    for(int64_t j = k + 1; j < n; ++j)                                        \
                        if(A[CIDX(j, k, lda)] != (T)0)                                        \
                        {                                                                     \
                            const T s = alpha * AV(j, k);                                     \
                            for(int64_t i = r0; i < r1; ++i)                                  \
                                B[CIDX(i, j, ldb)] += s * B[CIDX(i, k, ldb)];                 \
                        }                                                                     \
                    T t = alpha;                                                              \
                    if(nounit) t = t * AV(k, k);                                              \
                    if(t != one)                                                              \
                        for(int64_t i = r0; i < r1; ++i) B[CIDX(i, k, ldb)] *= t;             \
                }                                                                             \
            }                                                                                 \
        }                                                                                     \
    }

#define CONJ conjf
DEFINE_CTRMM(oracle_ctrmm, float _Complex)
#undef CONJ
#define CONJ conj
DEFINE_CTRMM(oracle_ztrmm, double _Complex)
#undef CONJ

/* The reference's forward-error / residual norm (clients/include/norm.hpp:449-492) for
 * complex data: |.| is the modulus; the running sums are never reset, as in the reference. */
double oracle_matrix_norm_1_z(int64_t M, int64_t N, const double _Complex* gold, int64_t ldg,
                              const double _Complex* x, int64_t ldx)
{
    double max_err_scal = 0.0, max_err = 0.0, err = 0.0, err_scal = 0.0;
    for(int64_t i = 0; i < N; i++)
    {
        for(int64_t j = 0; j < M; j++)
        {
            const double _Complex g = gold[CIDX(j, i, ldg)];
            const double _Complex v = x[CIDX(j, i, ldx)];
            err += cabs(g - v);
            err_scal += cabs(g);
        }
        max_err_scal = max_err_scal > err_scal ? max_err_scal : err_scal;
        max_err      = max_err > err ? max_err : err;
    }
    return max_err / max_err_scal;
}
