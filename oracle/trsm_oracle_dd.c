/*
 * Double-double residuals for the extended-precision solution X*.  TEST INFRASTRUCTURE ONLY:
 * part of the checker; nothing in the shipped library links or calls it.
 *
 * At m = 16384 the __float128 substitution of trsm_oracle.c costs about 0.3 s per
 * right-hand side on one core, too slow to measure errors on tens of right-hand sides of the
 * precision-form workload.  X* is computed instead by Wilkinson's iterative refinement on top
 * of the host CBLAS solve: X0 = cblas_dtrsm, then twice r = alpha B - T (Xh + Xl) with the
 * residual accumulated in double-double, d = cblas_dtrsm(r), X* = Xh + Xl + d.  The residual
 * here is the published compensated dot product "Dot2" of Ogita, Rump and Oishi (Accurate sum
 * and dot product, SIAM J. Sci. Comput. 26(6), 2005): each product a*x is split exactly into
 * p + e by one FMA (TwoProduct), each running sum s + p exactly into s' + q by Knuth's
 * TwoSum, and the error terms e and q are summed in a second double.  The result is as
 * accurate as if computed in twice the working precision and then rounded: |r - r_exact| <=
 * eps |r| + (2k eps)^2 (|alpha B| + |T| |X|).  The file is compiled without floating-point
 * contraction, which would break the error-free transformations.
 *
 * The triangle T is k x k, column-major, lower (lower != 0) or upper; unit != 0 reads its
 * diagonal as 1.  Only the triangle is read, so the other half may hold anything (NaN).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define TASK_ROWS 8  /* rows per task: two register blocks that share T's cache lines */
#define RB 4         /* rows per register block */
#define CB 4         /* right-hand sides per register block */
#define TCHUNK 512   /* columns of T per pass, kept in cache across the right-hand-side blocks */

/* s + l -= a * (xh + xl) for one register block, a from the RB rows of column t of T */
#define DD_STEP(h, l, a, xht, xlt)                                                            \
    for(int r = 0; r < RB; ++r)                                                               \
        for(int c = 0; c < CB; ++c)                                                           \
        {                                                                                     \
            const double p = -(a)[r] * (xht)[c];                                              \
            const double e = fma(-(a)[r], (xht)[c], -p);                                      \
            const double s = h[r][c] + p;                                                     \
            const double z = s - h[r][c];                                                     \
            const double q = (h[r][c] - (s - z)) + (p - z);                                   \
            h[r][c]        = s;                                                               \
            l[r][c] += (q + e) - (a)[r] * (xlt)[c];                                           \
        }

/* r := alpha B - T (Xh + Xl) for nrhs right-hand sides (columns of B, Xh, Xl, r). */
void oracle_dd_residual(int64_t k, int64_t nrhs, int lower, int unit, const double* T, int64_t ldt,
                        const double* Xh, const double* Xl, int64_t ldx, double alpha, const double* B,
                        int64_t ldb, double* R, int64_t ldr)
{
    if(k <= 0 || nrhs <= 0)
        return;
    /* X row-major (k x ldxr, right-hand sides padded with zeros to a multiple of CB), so that
     * a register block's loads over right-hand sides are contiguous */
    const int64_t ldxr = (nrhs + CB - 1) / CB * CB;
    double*       xh   = (double*)calloc((size_t)k * ldxr, sizeof(double));
    double*       xl   = (double*)calloc((size_t)k * ldxr, sizeof(double));
    for(int64_t c = 0; c < nrhs; ++c)
        for(int64_t t = 0; t < k; ++t)
        {
            xh[t * ldxr + c] = Xh[t + c * ldx];
            xl[t * ldxr + c] = Xl ? Xl[t + c * ldx] : 0.0;
        }
    const int64_t ntask = (k + TASK_ROWS - 1) / TASK_ROWS;
#pragma omp parallel
    {
        double* ah = (double*)malloc(sizeof(double) * TASK_ROWS * ldxr);
        double* al = (double*)malloc(sizeof(double) * TASK_ROWS * ldxr);
        /* the task's rows of T over one chunk of columns, masked to the triangle (zero outside,
         * the unit diagonal as 1) and padded with zero rows past k: [t][row] */
        double* tt = (double*)malloc(sizeof(double) * TASK_ROWS * TCHUNK);
#pragma omp for schedule(dynamic, 1)
        for(int64_t task = 0; task < ntask; ++task)
        {
            /* the lower triangle's long rows first */
            const int64_t i0 = (lower ? ntask - 1 - task : task) * TASK_ROWS;
            for(int r = 0; r < TASK_ROWS; ++r)
                for(int64_t c = 0; c < ldxr; ++c)
                {
                    const int64_t i = i0 + r;
                    const double  b = (i < k && c < nrhs) ? B[i + c * ldb] : 0.0;
                    const double  p = alpha * b;
                    ah[r * ldxr + c] = p;
                    al[r * ldxr + c] = fma(alpha, b, -p);
                }
            /* columns of T that meet the task's rows */
            const int64_t i1 = i0 + TASK_ROWS < k ? i0 + TASK_ROWS : k;
            const int64_t ta = lower ? 0 : i0;
            const int64_t tb = lower ? i1 : k;
            for(int64_t t0 = ta; t0 < tb; t0 += TCHUNK)
            {
                const int64_t nt = t0 + TCHUNK < tb ? TCHUNK : tb - t0;
                for(int64_t u = 0; u < nt; ++u)
                {
                    const int64_t t = t0 + u;
                    for(int r = 0; r < TASK_ROWS; ++r)
                    {
                        const int64_t i  = i0 + r;
                        const int     in = i < k && (lower ? t <= i : t >= i);
                        tt[u * TASK_ROWS + r] = !in ? 0.0 : (i == t && unit) ? 1.0 : T[i + t * ldt];
                    }
                }
                for(int rb = 0; rb < TASK_ROWS; rb += RB)
                    for(int64_t c0 = 0; c0 < ldxr; c0 += CB)
                    {
                        double h[RB][CB], l[RB][CB];
                        for(int r = 0; r < RB; ++r)
                            for(int c = 0; c < CB; ++c)
                            {
                                h[r][c] = ah[(rb + r) * ldxr + c0 + c];
                                l[r][c] = al[(rb + r) * ldxr + c0 + c];
                            }
                        for(int64_t u = 0; u < nt; ++u)
                        {
                            const double* a   = tt + u * TASK_ROWS + rb;
                            const double* xht = xh + (t0 + u) * ldxr + c0;
                            const double* xlt = xl + (t0 + u) * ldxr + c0;
                            DD_STEP(h, l, a, xht, xlt)
                        }
                        for(int r = 0; r < RB; ++r)
                            for(int c = 0; c < CB; ++c)
                            {
                                ah[(rb + r) * ldxr + c0 + c] = h[r][c];
                                al[(rb + r) * ldxr + c0 + c] = l[r][c];
                            }
                    }
            }
            for(int r = 0; r < TASK_ROWS; ++r)
                for(int64_t c = 0; c < nrhs; ++c)
                    if(i0 + r < k)
                        R[(i0 + r) + c * ldr] = ah[r * ldxr + c] + al[r * ldxr + c];
        }
        free(ah);
        free(al);
        free(tt);
    }
    free(xh);
    free(xl);
}
