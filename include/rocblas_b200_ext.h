/*
 * rocblas_b200_ext.h -- functions of librocblas_b200.so that have no counterpart in the
 * reference rocBLAS API.  They extend the drop-in surface of include/rocblas.h and never
 * change the behaviour of the functions declared there.
 */
#ifndef ROCBLAS_B200_EXT_H
#define ROCBLAS_B200_EXT_H

#include "rocblas.h"
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Number of GPU kernels this library has launched in the calling process so far (all
 * handles, all devices).  Benchmarks read it before and after a timed region to state how
 * many of the launches in that region were this library's own kernels. */
ROCBLAS_EXPORT uint64_t rocblas_b200_kernel_launch_count(void);

/* ---- variable-size batched trsm -------------------------------------------------------
 * One entry of a variable-size batch: solve op(A) X = alpha B (side left) or
 * X op(A) = alpha B (side right) for this entry's own sizes, leading dimensions and flags
 * (same meaning and validity rules as rocblas_?trsm).  The array of descriptors lives in
 * device memory; A and B are device pointers of the element type of the call. */
typedef struct rocblas_b200_trsm_problem
{
    const void*       A;
    void*             B;
    rocblas_int       m;
    rocblas_int       n;
    rocblas_int       lda;
    rocblas_int       ldb;
    rocblas_side      side;
    rocblas_fill      uplo;
    rocblas_operation transA;
    rocblas_diagonal  diag;
} rocblas_b200_trsm_problem;

/* Solve `count` independent systems described by `problems` (device array) with one
 * alpha (host or device pointer per the handle's pointer mode) in one persistent kernel.
 * No reference counterpart: rocblas_?trsm_batched needs one m, n for the whole batch, so a
 * reference caller makes one call per system.
 *   max_k: an upper bound of k (m for side left, n for side right) over the batch; at most
 *          512.  Larger bounds return rocblas_status_invalid_size.
 *   invalid_count: optional device pointer; receives the number of descriptors that broke
 *          the trsm argument rules or exceeded max_k (those entries are skipped, their B is
 *          not written).
 * Workspace: 16 * (count + 1) + 32 bytes from the handle (size query supported). */
ROCBLAS_EXPORT rocblas_status rocblas_b200_dtrsm_vbatched(rocblas_handle                   handle,
                                                          const double*                    alpha,
                                                          const rocblas_b200_trsm_problem* problems,
                                                          rocblas_int                      count,
                                                          rocblas_int                      max_k,
                                                          rocblas_int* invalid_count);
ROCBLAS_EXPORT rocblas_status rocblas_b200_strsm_vbatched(rocblas_handle                   handle,
                                                          const float*                     alpha,
                                                          const rocblas_b200_trsm_problem* problems,
                                                          rocblas_int                      count,
                                                          rocblas_int                      max_k,
                                                          rocblas_int* invalid_count);

/* Variable-size batch of any triangle order: as rocblas_b200_?trsm_vbatched, but systems with
 * k > 512 are solved too, by the chain solve (one persistent launch over every such system,
 * items claimed level by level), using the caller's inverted diagonal blocks:
 *   invA: device array of `count` device pointers; entry i holds the 128 x 128 inverses of
 *          system i's diagonal blocks in the rocblas_trsm_ex format (ld 128, stride 128 * 128,
 *          128 * k elements), e.g. from rocblas_?trtri_strided_batched; entries of systems
 *          with k <= 512 are not read (may be NULL);
 *   max_k: upper bound of k over the batch, at most 32768;
 *   max_n: upper bound of the right-hand sides (n for side left, m for side right) of the
 *          systems with k > 512; larger systems are skipped and counted invalid.
 * FP32 systems with k > 512 are computed in FP64 and rounded once.  Workspace from the
 * handle (size query supported): about count * (16 + 64 + 4 * ceil(max_k / 128) *
 * ceil(max_n / 32)) bytes.  No reference counterpart (see rocblas_b200_dtrsm_vbatched). */
ROCBLAS_EXPORT rocblas_status rocblas_b200_dtrsm_vbatched_ex(rocblas_handle                   handle,
                                                             const double*                    alpha,
                                                             const rocblas_b200_trsm_problem* problems,
                                                             const double* const*             invA,
                                                             rocblas_int                      count,
                                                             rocblas_int                      max_k,
                                                             rocblas_int                      max_n,
                                                             rocblas_int* invalid_count);
ROCBLAS_EXPORT rocblas_status rocblas_b200_strsm_vbatched_ex(rocblas_handle                   handle,
                                                             const float*                     alpha,
                                                             const rocblas_b200_trsm_problem* problems,
                                                             const float* const*              invA,
                                                             rocblas_int                      count,
                                                             rocblas_int                      max_k,
                                                             rocblas_int                      max_n,
                                                             rocblas_int* invalid_count);

/* ---- continuous-batching server ------------------------------------------------------------
 * A serving loop for streams of trsm requests (side left, lower, no transpose, non-unit: the
 * serving workload's form) of mixed size and dtype.  The server owns one device arena of
 * `hbm_budget` bytes (resident matrices, each admitted request's data), `n_streams` streams,
 * and a batching window.  rocblas_b200_server_run serves a request list whose arrival times
 * are given relative to the start of the call: requests are admitted in arrival order while
 * their memory fits the budget, collected per dtype until a stream is free and the window has
 * passed, and solved per collection by one variable-size batched call (resident invA reused;
 * a request's own A is copied in and its diagonal blocks inverted).  latency_s[i] receives
 * completion - arrival of request i on the host's steady clock.  A request's result does not
 * depend on the other requests of its collection.  No reference counterpart. */
typedef struct rocblas_b200_server_* rocblas_b200_server;

typedef struct rocblas_b200_request
{
    double           arrival_s; /* seconds after the start of rocblas_b200_server_run */
    rocblas_datatype dtype;     /* rocblas_datatype_f64_r or rocblas_datatype_f32_r */
    rocblas_int      m;         /* order of A and rows of B */
    rocblas_int      n;         /* right-hand sides */
    rocblas_int      resident;  /* index from rocblas_b200_server_add_resident, or -1 */
    const void*      B_src;     /* device: the right-hand sides, m x n, ld m */
    const void*      A_src;     /* device: the request's own lower triangle (resident < 0) */
    rocblas_int      lda_src;   /* its leading dimension (>= m) */
    rocblas_int      reserved;
    void*            X_dst;     /* device: where the solution (m x n, ld m) goes, or NULL */
} rocblas_b200_request;

typedef struct rocblas_b200_server_stats
{
    double  wall_s;             /* duration of the run */
    int64_t peak_bytes;         /* largest arena use during the run */
    int64_t collections;        /* batched solves launched */
    int64_t largest_collection; /* requests in the largest one */
    int64_t kernel_launches;    /* library kernels launched during the run */
} rocblas_b200_server_stats;

ROCBLAS_EXPORT rocblas_status rocblas_b200_server_create(rocblas_b200_server* server,
                                                         size_t               hbm_budget,
                                                         rocblas_int          n_streams,
                                                         double               window_us,
                                                         rocblas_int          max_batch);
ROCBLAS_EXPORT rocblas_status rocblas_b200_server_destroy(rocblas_b200_server server);
/* Copies A (m x m lower triangle, ld lda, device) into the arena and builds its invA. */
ROCBLAS_EXPORT rocblas_status rocblas_b200_server_add_resident(rocblas_b200_server server,
                                                               rocblas_datatype    dtype,
                                                               rocblas_int         m,
                                                               const void*         A,
                                                               rocblas_int         lda,
                                                               rocblas_int*        index);
/* Lowers (or raises, up to the arena) the admission budget; resident matrices count. */
ROCBLAS_EXPORT rocblas_status rocblas_b200_server_set_budget(rocblas_b200_server server,
                                                             size_t              hbm_budget);
ROCBLAS_EXPORT rocblas_status rocblas_b200_server_used_bytes(rocblas_b200_server server,
                                                             size_t*             bytes);
ROCBLAS_EXPORT rocblas_status rocblas_b200_server_run(rocblas_b200_server          server,
                                                      const rocblas_b200_request*  requests,
                                                      rocblas_int                  count,
                                                      double*                      latency_s,
                                                      rocblas_b200_server_stats*   stats);

/* ---- the variable-size batch without any allocation ---------------------------------------
 * No counterpart in the reference.  Same contract and results as
 * rocblas_b200_dtrsm_vbatched, for callers that cannot let a library allocate device memory:
 * applications whose own pool has reserved the GPU's memory up front and which forbid
 * libraries to allocate beside it (the allocation would fail or break the pool's budget), and
 * solver loops on a latency budget that cannot take the device-wide synchronisation a cudaFree
 * implies when the handle's workspace would grow.  Its scratch (queue state and prefix sums)
 * is a fixed device array inside the library, sized for at most 65536 systems (256 KiB +
 * 16 B, held on every GPU that loads the library until exit); count > 65536 returns
 * rocblas_status_invalid_size.  It calls no cudaMalloc or cudaFree and takes nothing from the
 * handle's workspace.  The first call on a device (and the first after that device's context
 * was torn down and made again) sets up: it looks up the array's device address in the
 * current context.  Make that first call before any stream capture.  All calls share the one
 * array and find it as the previous call left it (the call clears what must start at zero):
 * calls that overlap on the GPU (for example on two streams, or two handles at once) race and
 * must be ordered by the caller. */
ROCBLAS_EXPORT rocblas_status rocblas_b200_dtrsm_vbatched_noalloc(rocblas_handle                   handle,
                                                                  const double*                    alpha,
                                                                  const rocblas_b200_trsm_problem* problems,
                                                                  rocblas_int                      count,
                                                                  rocblas_int                      max_k,
                                                                  rocblas_int* invalid_count);

/* ---- FP64 GEMM from integer slices on the tensor cores ------------------------------------
 * C := alpha op(A) op(B) + beta C in FP64 (column-major), computed as exact int8 x int8 ->
 * int32 products of `slices` 7-bit slices of every row of op(A) and every column of op(B)
 * (each scaled by a power of two), combined in FP64.  slices = 7 reproduces FP64 dot
 * products to about 2^-49 relative to K max|row| max|col|; fewer slices are faster and
 * less accurate (about 2^(-7 slices)).  Inputs must be finite.  alpha and beta are host
 * pointers (host pointer mode only; device mode returns rocblas_status_not_implemented).
 * The reference has no counterpart; it is the engine of the precision form of the trsm.
 * Workspace from the handle (size query supported). */
ROCBLAS_EXPORT rocblas_status rocblas_b200_dgemm_sliced(rocblas_handle    handle,
                                                        rocblas_operation transA,
                                                        rocblas_operation transB,
                                                        rocblas_int       m,
                                                        rocblas_int       n,
                                                        rocblas_int       k,
                                                        const double*     alpha,
                                                        const double*     A,
                                                        rocblas_int       lda,
                                                        const double*     B,
                                                        rocblas_int       ldb,
                                                        const double*     beta,
                                                        double*           C,
                                                        rocblas_int       ldc,
                                                        rocblas_int       slices);

/* ---- FP64 GEMM from residues modulo small moduli on the tensor cores ----------------------
 * C := alpha op(A) op(B) + beta C in FP64 (column-major).  Every row of op(A) and column of
 * op(B) is scaled by a power of two and truncated to a b-bit integer (b = 55 for 16 moduli and
 * k <= 4096 per exponent range); the exact integer product is computed modulo `moduli`
 * pairwise coprime moduli <= 256 as int8 x int8 -> int32 tensor-core products and rebuilt by
 * the Chinese remainder theorem, then scaled back and rounded once to FP64.  moduli is 14, 15
 * or 16 (0: 16); fewer moduli keep fewer bits (b drops by about 4 per modulus).  Inputs must be
 * finite.  alpha and beta are host pointers (host pointer mode only; device mode returns
 * rocblas_status_not_implemented).  The reference has no counterpart; it is the second engine
 * of the precision form of the trsm (tuning key mixed_moduli).  Workspace from the handle
 * (size query supported). */
ROCBLAS_EXPORT rocblas_status rocblas_b200_dgemm_crt(rocblas_handle    handle,
                                                     rocblas_operation transA,
                                                     rocblas_operation transB,
                                                     rocblas_int       m,
                                                     rocblas_int       n,
                                                     rocblas_int       k,
                                                     const double*     alpha,
                                                     const double*     A,
                                                     rocblas_int       lda,
                                                     const double*     B,
                                                     rocblas_int       ldb,
                                                     const double*     beta,
                                                     double*           C,
                                                     rocblas_int       ldc,
                                                     rocblas_int       moduli);

/* ---- FP64 GEMM on the DMMA tiles of the trsm updates -----------------------------------------
 * C := alpha op(A) op(B) + beta C (column-major FP64), the engine of rocblas_dtrsm's trailing
 * updates (mma.sync m16n8k8 .f64 tiles fed by cp.async), exposed as a GEMM.  Same argument
 * meaning as rocblas_dgemm (rocblas-functions.h), host pointer mode only (device mode returns
 * rocblas_status_not_implemented); needs no workspace. */
ROCBLAS_EXPORT rocblas_status rocblas_b200_dgemm(rocblas_handle    handle,
                                                 rocblas_operation transA,
                                                 rocblas_operation transB,
                                                 rocblas_int       m,
                                                 rocblas_int       n,
                                                 rocblas_int       k,
                                                 const double*     alpha,
                                                 const double*     A,
                                                 rocblas_int       lda,
                                                 const double*     B,
                                                 rocblas_int       ldb,
                                                 const double*     beta,
                                                 double*           C,
                                                 rocblas_int       ldc);

/* ---- complex GEMM on the complex DMMA tiles of the complex trsm updates --------------------------
 * C := alpha op(A) op(B) + beta C for complex double / complex float, computed in FP64 on the
 * DMMA tensor path (each complex multiply-add as real 2 x 2 blocks; complex float is rounded
 * once at the end).  op C conjugates.  Same argument meaning as rocblas_{z,c}gemm
 * (rocblas-functions.h), host pointer mode only; needs no workspace. */
ROCBLAS_EXPORT rocblas_status rocblas_b200_zgemm(rocblas_handle                handle,
                                                 rocblas_operation             transA,
                                                 rocblas_operation             transB,
                                                 rocblas_int                   m,
                                                 rocblas_int                   n,
                                                 rocblas_int                   k,
                                                 const rocblas_double_complex* alpha,
                                                 const rocblas_double_complex* A,
                                                 rocblas_int                   lda,
                                                 const rocblas_double_complex* B,
                                                 rocblas_int                   ldb,
                                                 const rocblas_double_complex* beta,
                                                 rocblas_double_complex*       C,
                                                 rocblas_int                   ldc);
ROCBLAS_EXPORT rocblas_status rocblas_b200_cgemm(rocblas_handle               handle,
                                                 rocblas_operation            transA,
                                                 rocblas_operation            transB,
                                                 rocblas_int                  m,
                                                 rocblas_int                  n,
                                                 rocblas_int                  k,
                                                 const rocblas_float_complex* alpha,
                                                 const rocblas_float_complex* A,
                                                 rocblas_int                  lda,
                                                 const rocblas_float_complex* B,
                                                 rocblas_int                  ldb,
                                                 const rocblas_float_complex* beta,
                                                 rocblas_float_complex*       C,
                                                 rocblas_int                  ldc);

/* ---- precision form of dtrsm ----------------------------------------------------------------
 * Same contract as rocblas_dtrsm.  The blocked solve keeps the diagonal blocks in FP64
 * (inverted 128 x 128 blocks applied with FP64 tensor-core MMA) and runs every trailing
 * update with K >= sliced_min_k on an integer tensor-core GEMM: slices = 0 takes the tuning
 * table's engine (the residue GEMM rocblas_b200_dgemm_crt with mixed_moduli moduli, or, with
 * mixed_moduli 0, the slice GEMM with mixed_slices slices); slices = 1..8 takes the slice GEMM
 * rocblas_b200_dgemm_sliced with that many slices.  Shorter updates stay on FP64 DMMA.
 * Workspace: the invA blocks plus the operands of the largest update (size query supported). */
ROCBLAS_EXPORT rocblas_status rocblas_b200_dtrsm_mixed(rocblas_handle    handle,
                                                       rocblas_side      side,
                                                       rocblas_fill      uplo,
                                                       rocblas_operation transA,
                                                       rocblas_diagonal  diag,
                                                       rocblas_int       m,
                                                       rocblas_int       n,
                                                       const double*     alpha,
                                                       const double*     A,
                                                       rocblas_int       lda,
                                                       double*           B,
                                                       rocblas_int       ldb,
                                                       rocblas_int       slices);

/* ---- precision form with iterative refinement -------------------------------------------------
 * rocblas_b200_dtrsm_mixed followed by FP64 iterative refinement until the result agrees with
 * the plain FP64 form to `tolerance`.  The reference has no counterpart.  The loop is
 * mixed-precision iterative refinement (Wilkinson; Buttari et al. 2007 for the form LAPACK's
 * dsgesv uses) with the low-precision solve replaced by the sliced tensor-core solve:
 *   X := precision-form solve of op(A) X = alpha B (or X op(A) = alpha B);
 *   test: `check_columns` evenly spaced right-hand sides (columns of B for side left, rows for
 *         side right) are also solved by the plain FP64 form, on a second stream and a few SMs
 *         of their own (tuning keys refine_check_sms, refine_check_pairs: 6 SMs held as SM
 *         pairs) while the precision-form solve runs on the others; the test passes when, for
 *         each of them,
 *         ||x - x_fp64||_inf <= tolerance * ||x_fp64||_inf;
 *   while the test fails and fewer than max_iterations corrections were made:
 *         R := alpha B - op(A) X in FP64 over all right-hand sides (DMMA tiles);
 *         D := precision-form solve of op(A) D = R (the invA blocks of the first solve are
 *         reused);  X := X + D;  test again.
 * If the test still fails and `fallback` is set, B is solved again from its original values by
 * the plain FP64 form (rocblas_dtrsm).  A test on a sample is a statistical check: right-hand
 * sides outside it are not compared.  Everything runs on the GPU; the call reads each test's
 * maxima back to the host and so returns after the solve has completed.  alpha is a host
 * pointer (device pointer mode returns rocblas_status_not_implemented).  Workspace: the
 * precision form's plus two m x n copies (the original B and the residual) and the tested
 * right-hand sides (size query supported).  options may be NULL (all defaults); info may be
 * NULL. */
typedef struct rocblas_b200_refine_options
{
    rocblas_int slices;         /* 0: the tuning table's engine (mixed_moduli / mixed_slices);
                                   1..8: the slice engine with that many slices */
    rocblas_int max_iterations; /* correction solves at most (negative: 10) */
    rocblas_int check_columns;  /* right-hand sides tested (0: 8; >= their count: all) */
    rocblas_int fallback;       /* 1: plain FP64 solve when the test never passes */
    double      tolerance;      /* normwise relative difference allowed (0: 1e-12) */
} rocblas_b200_refine_options;

typedef struct rocblas_b200_refine_info
{
    rocblas_int iterations;           /* correction solves performed */
    rocblas_int converged;            /* 1 if the last test passed */
    rocblas_int fell_back;            /* 1 if the plain FP64 form produced the result */
    rocblas_int checked_columns;      /* right-hand sides in each test */
    double      error_estimate_first; /* max ||x - x_fp64|| / ||x_fp64|| after the first solve */
    double      error_estimate;       /* the same after the last correction */
    double      tolerance;            /* the bound used */
} rocblas_b200_refine_info;

ROCBLAS_EXPORT rocblas_status rocblas_b200_dtrsm_refined(rocblas_handle                     handle,
                                                         rocblas_side                       side,
                                                         rocblas_fill                       uplo,
                                                         rocblas_operation                  transA,
                                                         rocblas_diagonal                   diag,
                                                         rocblas_int                        m,
                                                         rocblas_int                        n,
                                                         const double*                      alpha,
                                                         const double*                      A,
                                                         rocblas_int                        lda,
                                                         double*                            B,
                                                         rocblas_int                        ldb,
                                                         const rocblas_b200_refine_options* options,
                                                         rocblas_b200_refine_info*          info);

/* ---- precision form with A and B in host memory -----------------------------------------------
 * rocblas_b200_dtrsm_mixed for host buffers (pinned memory lets the copies overlap the solve):
 * A (lda x k) and B (ldb x n) are host pointers, alpha a host value whatever the handle's
 * pointer mode, and the call returns when B holds X.  For side left the solve runs
 * left-looking over steps of rows (tuning key host_step_blocks, in 128-row blocks), and the
 * transfer of each step's rows of B and block row of op(A), the solve and the transfer of
 * finished rows of X back to B overlap on the handle's stream and three internal streams;
 * side right copies first and then solves.  Of A only the referenced triangle (with the
 * diagonal blocks of one step) is transferred.  The device copies of A
 * and B are kept by the handle between calls (freed by rocblas_destroy_handle). */
ROCBLAS_EXPORT rocblas_status rocblas_b200_dtrsm_mixed_host(rocblas_handle    handle,
                                                            rocblas_side      side,
                                                            rocblas_fill      uplo,
                                                            rocblas_operation transA,
                                                            rocblas_diagonal  diag,
                                                            rocblas_int       m,
                                                            rocblas_int       n,
                                                            const double*     alpha,
                                                            const double*     A,
                                                            rocblas_int       lda,
                                                            double*           B,
                                                            rocblas_int       ldb,
                                                            rocblas_int       slices);

/* ---- tuning table -----------------------------------------------------------------------
 * Thresholds of the algorithm and tile choices (no reference counterpart beyond its
 * compiled-in block-size tables).  Loaded once from $ROCBLAS_B200_TUNING or tuning.cfg next
 * to the library ("key value" lines, written by rocblas_b200/autotune.py); these two calls
 * read or change one entry in the running process.  Keys: block_max_k, block_always_k,
 * block_min_strips_pct, sliced_min_k, dmma_big_tile_pct, mixed_slices, dmma_force_tile,
 * dmma_big_bk, oz_bn, oz_bk, chain_max_cols, chain_max_cols_f32, chain_w, mixed_chain_blocks,
 * host_step_blocks, sliced_k_chunk, refine_check_sms, refine_check_flag, refine_check_w,
 * refine_check_pairs, wait_cycles_log2,
 * chain_first_item, mixed_moduli, crt_group_m, crt_min_tiles_pct, crt_pair, strsm_slices,
 * strsm_sliced_min_k, trsv_flag_min_n, trsv_flag_nb.  Unknown keys or
 * out-of-range values return rocblas_status_invalid_value. */
/* Per-launch timing of the main kernels with CUDA events on the launching stream, for
 * measuring one kernel's achieved rate inside a larger call.  enable != 0 starts recording
 * (and discards earlier records), 0 stops it.  query sums, over the recorded launches of a
 * kernel class ("sliced": the integer-slice tensor-core GEMM, work = int8 tensor operations;
 * "dmma": the FP64 DMMA GEMM tiles, work = FP64 flops; "chain": the chain solve, work = the
 * trsm flop count k * k * ncols of uniform batches, 0 for variable batches; "trtri": the
 * diagonal-block inversions, work = 128^3 / 3 per block; "strip": the variable batch's
 * strip-solver queues, work = 0), the event time
 * in milliseconds, the work, and the launch count; it waits for the recorded events. */
ROCBLAS_EXPORT rocblas_status rocblas_b200_kernel_timing_enable(rocblas_int enable);
ROCBLAS_EXPORT rocblas_status rocblas_b200_kernel_timing_query(const char* kernel_class,
                                                               double*     total_ms,
                                                               double*     total_work,
                                                               rocblas_int* launches);

ROCBLAS_EXPORT rocblas_status rocblas_b200_set_tuning(const char* key, rocblas_int value);
ROCBLAS_EXPORT rocblas_status rocblas_b200_get_tuning(const char* key, rocblas_int* value);

/* Synchronises the handle's stream and returns (and clears) the error word that kernels
 * with bounded waits set when a wait ran out: 0 = none.  A nonzero value means results of
 * calls since the last check are not valid. */
ROCBLAS_EXPORT rocblas_status rocblas_b200_get_device_error(rocblas_handle handle, rocblas_int* code);

#ifdef __cplusplus
}
#endif

#endif /* ROCBLAS_B200_EXT_H */
