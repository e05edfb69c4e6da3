/*
 * rocblas.h -- the drop-in C ABI of the B200 TRSM library (librocblas_b200.so).
 *
 * This header declares the subset of the rocBLAS C API that the level-3 triangular-solve
 * path uses: handle / stream / pointer-mode / device-memory functions, rocblas_{s,d}trsm
 * and its _batched, _strided_batched and _ex forms, and rocblas_{s,d}trtri (which builds
 * the invA that the _ex forms accept).  Types, enum values, status codes and argument
 * meaning are those of the reference so that existing callers relink unchanged;
 * hipStream_t becomes cudaStream_t.  Each declaration cites the reference declaration it
 * replaces (paths inside the rocBLAS source tree).
 *
 * Conventions (as in the reference):
 *   - column-major storage, leading dimensions in elements;
 *   - A, B, invA and device-mode alpha are device pointers; B is overwritten with X;
 *   - every call is asynchronous on the handle's stream (return != completion);
 *   - no function throws; failures are reported as rocblas_status.
 */
#ifndef ROCBLAS_B200_ROCBLAS_H
#define ROCBLAS_B200_ROCBLAS_H

#include <stddef.h>
#include <stdint.h>
#include <stdbool.h>
#include <cuda_runtime_api.h>

#if defined(__GNUC__)
#define ROCBLAS_EXPORT __attribute__((visibility("default")))
#else
#define ROCBLAS_EXPORT
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- types: library/include/internal/rocblas-types.h:60-245 ---------------------------- */
typedef struct _rocblas_handle* rocblas_handle; /* rocblas-types.h:64 */
typedef int32_t rocblas_int;                    /* rocblas-types.h:80 (LP64 API) */
typedef int64_t rocblas_stride;                 /* rocblas-types.h:84 */
/* complex element types: the C definitions of rocblas-complex-types.h:82-91 */
typedef struct
{
    float x, y;
} rocblas_float_complex;
typedef struct
{
    double x, y;
} rocblas_double_complex;
typedef float   rocblas_float;
typedef double  rocblas_double;

typedef enum rocblas_operation_ /* rocblas-types.h:123-129 */
{
    rocblas_operation_none                = 111,
    rocblas_operation_transpose           = 112,
    rocblas_operation_conjugate_transpose = 113
} rocblas_operation;

typedef enum rocblas_fill_ /* rocblas-types.h:134-139 */
{
    rocblas_fill_upper = 121,
    rocblas_fill_lower = 122,
    rocblas_fill_full  = 123
} rocblas_fill;

typedef enum rocblas_diagonal_ /* rocblas-types.h:144-148 */
{
    rocblas_diagonal_non_unit = 131,
    rocblas_diagonal_unit     = 132
} rocblas_diagonal;

typedef enum rocblas_side_ /* rocblas-types.h:151-157 */
{
    rocblas_side_left  = 141,
    rocblas_side_right = 142,
    rocblas_side_both  = 143
} rocblas_side;

typedef enum rocblas_datatype_ /* rocblas-types.h:164-184 */
{
    rocblas_datatype_f16_r   = 150,
    rocblas_datatype_f32_r   = 151,
    rocblas_datatype_f64_r   = 152,
    rocblas_datatype_f16_c   = 153,
    rocblas_datatype_f32_c   = 154,
    rocblas_datatype_f64_c   = 155,
    rocblas_datatype_i8_r    = 160,
    rocblas_datatype_u8_r    = 161,
    rocblas_datatype_i32_r   = 162,
    rocblas_datatype_u32_r   = 163,
    rocblas_datatype_i8_c    = 164,
    rocblas_datatype_u8_c    = 165,
    rocblas_datatype_i32_c   = 166,
    rocblas_datatype_u32_c   = 167,
    rocblas_datatype_bf16_r  = 168,
    rocblas_datatype_bf16_c  = 169,
    rocblas_datatype_f8_r    = 170,
    rocblas_datatype_bf8_r   = 171,
    rocblas_datatype_invalid = 255
} rocblas_datatype;

typedef enum rocblas_status_ /* rocblas-types.h:203-223 */
{
    rocblas_status_success             = 0,
    rocblas_status_invalid_handle      = 1,
    rocblas_status_not_implemented     = 2,
    rocblas_status_invalid_pointer     = 3,
    rocblas_status_invalid_size        = 4,
    rocblas_status_memory_error        = 5,
    rocblas_status_internal_error      = 6,
    rocblas_status_perf_degraded       = 7,
    rocblas_status_size_query_mismatch = 8,
    rocblas_status_size_increased      = 9,
    rocblas_status_size_unchanged      = 10,
    rocblas_status_invalid_value       = 11,
    rocblas_status_continue            = 12,
    rocblas_status_check_numerics_fail = 13,
    rocblas_status_excluded_from_build = 14,
    rocblas_status_arch_mismatch       = 15
} rocblas_status;

typedef enum rocblas_pointer_mode_ /* rocblas-types.h:228-234 */
{
    rocblas_pointer_mode_host   = 0,
    rocblas_pointer_mode_device = 1
} rocblas_pointer_mode;

typedef enum rocblas_performance_metric_ /* rocblas-types.h:249-258 */
{
    rocblas_default_performance_metric           = 0,
    rocblas_device_efficiency_performance_metric = 1,
    rocblas_cu_efficiency_performance_metric     = 2
} rocblas_performance_metric;

typedef enum rocblas_math_mode_ /* rocblas-types.h:340-347 */
{
    rocblas_default_math     = 0x0,
    rocblas_xf32_xdl_math_op = 0x1
} rocblas_math_mode;

typedef enum rocblas_atomics_mode_ /* rocblas-types.h:239-245 */
{
    rocblas_atomics_not_allowed = 0,
    rocblas_atomics_allowed     = 1
} rocblas_atomics_mode;

/* the bits of ROCBLAS_LAYER and ROCBLAS_CHECK_NUMERICS (rocblas-types.h:261-271, 321-338),
 * read from the environment when a handle is created */
typedef enum rocblas_layer_mode_
{
    rocblas_layer_mode_none        = 0x0,
    rocblas_layer_mode_log_trace   = 0x1,
    rocblas_layer_mode_log_bench   = 0x2,
    rocblas_layer_mode_log_profile = 0x4
} rocblas_layer_mode;

typedef enum rocblas_check_numerics_mode_
{
    rocblas_check_numerics_mode_no_check     = 0x0,
    rocblas_check_numerics_mode_info         = 0x1,
    rocblas_check_numerics_mode_warn         = 0x2,
    rocblas_check_numerics_mode_fail         = 0x4,
    rocblas_check_numerics_mode_only_nan_inf = 0x8
} rocblas_check_numerics_mode;

/* ---- handle / stream / pointer mode: library/include/internal/rocblas-auxiliary.h:40-61 --- */
ROCBLAS_EXPORT rocblas_status rocblas_create_handle(rocblas_handle* handle);
ROCBLAS_EXPORT rocblas_status rocblas_destroy_handle(rocblas_handle handle);
ROCBLAS_EXPORT rocblas_status rocblas_set_stream(rocblas_handle handle, cudaStream_t stream);
ROCBLAS_EXPORT rocblas_status rocblas_get_stream(rocblas_handle handle, cudaStream_t* stream);
ROCBLAS_EXPORT rocblas_status rocblas_set_pointer_mode(rocblas_handle       handle,
                                                       rocblas_pointer_mode pointer_mode);
ROCBLAS_EXPORT rocblas_status rocblas_get_pointer_mode(rocblas_handle        handle,
                                                       rocblas_pointer_mode* pointer_mode);
/* rocblas-auxiliary.h:77-83: the TRSM path uses no atomics either way; the mode is kept and
 * logged */
ROCBLAS_EXPORT rocblas_status rocblas_set_atomics_mode(rocblas_handle       handle,
                                                       rocblas_atomics_mode atomics_mode);
ROCBLAS_EXPORT rocblas_status rocblas_get_atomics_mode(rocblas_handle        handle,
                                                       rocblas_atomics_mode* atomics_mode);
/* rocblas-auxiliary.h: math mode (xf32 is a GEMM-backend mode that this TRSM path does not
 * have: setting it is ignored, as the reference does where its backend lacks it), the GEMM
 * solution-selection metric and the fitness query (kept; no GEMM solution library here, so
 * the fitness stays at the lowest double) */
ROCBLAS_EXPORT rocblas_status rocblas_set_math_mode(rocblas_handle handle, rocblas_math_mode math_mode);
ROCBLAS_EXPORT rocblas_status rocblas_get_math_mode(rocblas_handle handle, rocblas_math_mode* math_mode);
ROCBLAS_EXPORT rocblas_status rocblas_set_performance_metric(rocblas_handle             handle,
                                                             rocblas_performance_metric metric);
ROCBLAS_EXPORT rocblas_status rocblas_get_performance_metric(rocblas_handle              handle,
                                                             rocblas_performance_metric* metric);
ROCBLAS_EXPORT rocblas_status rocblas_set_solution_fitness_query(rocblas_handle handle, double* fitness);
/* rocblas-auxiliary.h:97 */
ROCBLAS_EXPORT rocblas_pointer_mode rocblas_pointer_to_mode(void* ptr);

/* ---- host <-> device copies: rocblas-auxiliary.h (set/get vector and matrix, the _async forms
 * on a stream, the _64 forms with int64_t sizes); library/src/rocblas_auxiliary.cpp:305-790.
 * n == 0 (rows == 0 or cols == 0) returns success; negative sizes, increments <= 0,
 * elem_size <= 0, lda or ldb < rows or <= 0 return invalid_size; null pointers invalid_pointer. */
ROCBLAS_EXPORT rocblas_status rocblas_set_vector(rocblas_int n, rocblas_int elem_size, const void* x_h, rocblas_int incx,
                                              void* y_d, rocblas_int incy);
ROCBLAS_EXPORT rocblas_status rocblas_set_vector_async(rocblas_int n, rocblas_int elem_size, const void* x_h,
                                              rocblas_int incx, void* y_d, rocblas_int incy, cudaStream_t stream);
ROCBLAS_EXPORT rocblas_status rocblas_set_matrix(rocblas_int rows, rocblas_int cols, rocblas_int elem_size, const void* a_h,
                                              rocblas_int lda, void* b_d, rocblas_int ldb);
ROCBLAS_EXPORT rocblas_status rocblas_set_matrix_async(rocblas_int rows, rocblas_int cols, rocblas_int elem_size,
                                              const void* a_h, rocblas_int lda, void* b_d, rocblas_int ldb,
                                              cudaStream_t stream);
ROCBLAS_EXPORT rocblas_status rocblas_get_vector(rocblas_int n, rocblas_int elem_size, const void* x_d, rocblas_int incx,
                                              void* y_h, rocblas_int incy);
ROCBLAS_EXPORT rocblas_status rocblas_get_vector_async(rocblas_int n, rocblas_int elem_size, const void* x_d,
                                              rocblas_int incx, void* y_h, rocblas_int incy, cudaStream_t stream);
ROCBLAS_EXPORT rocblas_status rocblas_get_matrix(rocblas_int rows, rocblas_int cols, rocblas_int elem_size, const void* a_d,
                                              rocblas_int lda, void* b_h, rocblas_int ldb);
ROCBLAS_EXPORT rocblas_status rocblas_get_matrix_async(rocblas_int rows, rocblas_int cols, rocblas_int elem_size,
                                              const void* a_d, rocblas_int lda, void* b_h, rocblas_int ldb,
                                              cudaStream_t stream);
ROCBLAS_EXPORT rocblas_status rocblas_set_vector_64(int64_t n, int64_t elem_size, const void* x_h, int64_t incx,
                                              void* y_d, int64_t incy);
ROCBLAS_EXPORT rocblas_status rocblas_set_vector_async_64(int64_t n, int64_t elem_size, const void* x_h,
                                              int64_t incx, void* y_d, int64_t incy, cudaStream_t stream);
ROCBLAS_EXPORT rocblas_status rocblas_set_matrix_64(int64_t rows, int64_t cols, int64_t elem_size, const void* a_h,
                                              int64_t lda, void* b_d, int64_t ldb);
ROCBLAS_EXPORT rocblas_status rocblas_set_matrix_async_64(int64_t rows, int64_t cols, int64_t elem_size,
                                              const void* a_h, int64_t lda, void* b_d, int64_t ldb,
                                              cudaStream_t stream);
ROCBLAS_EXPORT rocblas_status rocblas_get_vector_64(int64_t n, int64_t elem_size, const void* x_d, int64_t incx,
                                              void* y_h, int64_t incy);
ROCBLAS_EXPORT rocblas_status rocblas_get_vector_async_64(int64_t n, int64_t elem_size, const void* x_d,
                                              int64_t incx, void* y_h, int64_t incy, cudaStream_t stream);
ROCBLAS_EXPORT rocblas_status rocblas_get_matrix_64(int64_t rows, int64_t cols, int64_t elem_size, const void* a_d,
                                              int64_t lda, void* b_h, int64_t ldb);
ROCBLAS_EXPORT rocblas_status rocblas_get_matrix_async_64(int64_t rows, int64_t cols, int64_t elem_size,
                                              const void* a_d, int64_t lda, void* b_h, int64_t ldb,
                                              cudaStream_t stream);

/* ---- device memory: library/include/internal/rocblas-functions.h:25027-25122 ---------- */
ROCBLAS_EXPORT rocblas_status rocblas_start_device_memory_size_query(rocblas_handle handle);
ROCBLAS_EXPORT rocblas_status rocblas_stop_device_memory_size_query(rocblas_handle handle,
                                                                    size_t*        size);
ROCBLAS_EXPORT bool           rocblas_is_device_memory_size_query(rocblas_handle handle);
ROCBLAS_EXPORT rocblas_status rocblas_get_device_memory_size(rocblas_handle handle, size_t* size);
ROCBLAS_EXPORT rocblas_status rocblas_set_device_memory_size(rocblas_handle handle, size_t size);
ROCBLAS_EXPORT rocblas_status rocblas_set_workspace(rocblas_handle handle, void* addr, size_t size);
ROCBLAS_EXPORT bool           rocblas_is_managing_device_memory(rocblas_handle handle);
ROCBLAS_EXPORT bool           rocblas_is_user_managing_device_memory(rocblas_handle handle);

/* ---- trsm: rocblas-functions.h:19388-19412 -------------------------------------------- */
ROCBLAS_EXPORT rocblas_status rocblas_strsm(rocblas_handle    handle,
                                            rocblas_side      side,
                                            rocblas_fill      uplo,
                                            rocblas_operation transA,
                                            rocblas_diagonal  diag,
                                            rocblas_int       m,
                                            rocblas_int       n,
                                            const float*      alpha,
                                            const float*      A,
                                            rocblas_int       lda,
                                            float*            B,
                                            rocblas_int       ldb);

ROCBLAS_EXPORT rocblas_status rocblas_dtrsm(rocblas_handle    handle,
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
                                            rocblas_int       ldb);

/* ---- trsm_batched: rocblas-functions.h:19574-19601 (A, B: device arrays of device
 *      pointers) ----------------------------------------------------------------------- */
ROCBLAS_EXPORT rocblas_status rocblas_strsm_batched(rocblas_handle     handle,
                                                    rocblas_side       side,
                                                    rocblas_fill       uplo,
                                                    rocblas_operation  transA,
                                                    rocblas_diagonal   diag,
                                                    rocblas_int        m,
                                                    rocblas_int        n,
                                                    const float*       alpha,
                                                    const float* const A[],
                                                    rocblas_int        lda,
                                                    float* const       B[],
                                                    rocblas_int        ldb,
                                                    rocblas_int        batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_dtrsm_batched(rocblas_handle      handle,
                                                    rocblas_side        side,
                                                    rocblas_fill        uplo,
                                                    rocblas_operation   transA,
                                                    rocblas_diagonal    diag,
                                                    rocblas_int         m,
                                                    rocblas_int         n,
                                                    const double*       alpha,
                                                    const double* const A[],
                                                    rocblas_int         lda,
                                                    double* const       B[],
                                                    rocblas_int         ldb,
                                                    rocblas_int         batch_count);

/* ---- trsm_strided_batched: rocblas-functions.h:19774-19805 ---------------------------- */
ROCBLAS_EXPORT rocblas_status rocblas_strsm_strided_batched(rocblas_handle    handle,
                                                            rocblas_side      side,
                                                            rocblas_fill      uplo,
                                                            rocblas_operation transA,
                                                            rocblas_diagonal  diag,
                                                            rocblas_int       m,
                                                            rocblas_int       n,
                                                            const float*      alpha,
                                                            const float*      A,
                                                            rocblas_int       lda,
                                                            rocblas_stride    stride_a,
                                                            float*            B,
                                                            rocblas_int       ldb,
                                                            rocblas_stride    stride_b,
                                                            rocblas_int       batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_dtrsm_strided_batched(rocblas_handle    handle,
                                                            rocblas_side      side,
                                                            rocblas_fill      uplo,
                                                            rocblas_operation transA,
                                                            rocblas_diagonal  diag,
                                                            rocblas_int       m,
                                                            rocblas_int       n,
                                                            const double*     alpha,
                                                            const double*     A,
                                                            rocblas_int       lda,
                                                            rocblas_stride    stride_a,
                                                            double*           B,
                                                            rocblas_int       ldb,
                                                            rocblas_stride    stride_b,
                                                            rocblas_int       batch_count);

/* ---- trsm_ex family: rocblas-functions.h:23223-23238, 23404-23420, 23563-23581.
 *      invA: packed 128 x 128 inverses of the diagonal blocks of A (ld 128, stride
 *      128*128) followed by the k % 128 remainder block; invA_size in elements.
 *      compute_type f32_r / f64_r; complex types return rocblas_status_not_implemented. */
ROCBLAS_EXPORT rocblas_status rocblas_trsm_ex(rocblas_handle    handle,
                                              rocblas_side      side,
                                              rocblas_fill      uplo,
                                              rocblas_operation transA,
                                              rocblas_diagonal  diag,
                                              rocblas_int       m,
                                              rocblas_int       n,
                                              const void*       alpha,
                                              const void*       A,
                                              rocblas_int       lda,
                                              void*             B,
                                              rocblas_int       ldb,
                                              const void*       invA,
                                              rocblas_int       invA_size,
                                              rocblas_datatype  compute_type);

ROCBLAS_EXPORT rocblas_status rocblas_trsm_batched_ex(rocblas_handle    handle,
                                                      rocblas_side      side,
                                                      rocblas_fill      uplo,
                                                      rocblas_operation transA,
                                                      rocblas_diagonal  diag,
                                                      rocblas_int       m,
                                                      rocblas_int       n,
                                                      const void*       alpha,
                                                      const void*       A,
                                                      rocblas_int       lda,
                                                      void*             B,
                                                      rocblas_int       ldb,
                                                      rocblas_int       batch_count,
                                                      const void*       invA,
                                                      rocblas_int       invA_size,
                                                      rocblas_datatype  compute_type);

ROCBLAS_EXPORT rocblas_status rocblas_trsm_strided_batched_ex(rocblas_handle    handle,
                                                              rocblas_side      side,
                                                              rocblas_fill      uplo,
                                                              rocblas_operation transA,
                                                              rocblas_diagonal  diag,
                                                              rocblas_int       m,
                                                              rocblas_int       n,
                                                              const void*       alpha,
                                                              const void*       A,
                                                              rocblas_int       lda,
                                                              rocblas_stride    stride_A,
                                                              void*             B,
                                                              rocblas_int       ldb,
                                                              rocblas_stride    stride_B,
                                                              rocblas_int       batch_count,
                                                              const void*       invA,
                                                              rocblas_int       invA_size,
                                                              rocblas_stride    stride_invA,
                                                              rocblas_datatype  compute_type);

/* ---- trtri: rocblas-functions.h:19081-19098, 19159-19177, 19249-19272 ----------------- */
ROCBLAS_EXPORT rocblas_status rocblas_strtri(rocblas_handle   handle,
                                             rocblas_fill     uplo,
                                             rocblas_diagonal diag,
                                             rocblas_int      n,
                                             const float*     A,
                                             rocblas_int      lda,
                                             float*           invA,
                                             rocblas_int      ldinvA);

ROCBLAS_EXPORT rocblas_status rocblas_dtrtri(rocblas_handle   handle,
                                             rocblas_fill     uplo,
                                             rocblas_diagonal diag,
                                             rocblas_int      n,
                                             const double*    A,
                                             rocblas_int      lda,
                                             double*          invA,
                                             rocblas_int      ldinvA);

ROCBLAS_EXPORT rocblas_status rocblas_strtri_batched(rocblas_handle     handle,
                                                     rocblas_fill       uplo,
                                                     rocblas_diagonal   diag,
                                                     rocblas_int        n,
                                                     const float* const A[],
                                                     rocblas_int        lda,
                                                     float* const       invA[],
                                                     rocblas_int        ldinvA,
                                                     rocblas_int        batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_dtrtri_batched(rocblas_handle      handle,
                                                     rocblas_fill        uplo,
                                                     rocblas_diagonal    diag,
                                                     rocblas_int         n,
                                                     const double* const A[],
                                                     rocblas_int         lda,
                                                     double* const       invA[],
                                                     rocblas_int         ldinvA,
                                                     rocblas_int         batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_strtri_strided_batched(rocblas_handle   handle,
                                                             rocblas_fill     uplo,
                                                             rocblas_diagonal diag,
                                                             rocblas_int      n,
                                                             const float*     A,
                                                             rocblas_int      lda,
                                                             rocblas_stride   stride_a,
                                                             float*           invA,
                                                             rocblas_int      ldinvA,
                                                             rocblas_stride   stride_invA,
                                                             rocblas_int      batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_dtrtri_strided_batched(rocblas_handle   handle,
                                                             rocblas_fill     uplo,
                                                             rocblas_diagonal diag,
                                                             rocblas_int      n,
                                                             const double*    A,
                                                             rocblas_int      lda,
                                                             rocblas_stride   stride_a,
                                                             double*          invA,
                                                             rocblas_int      ldinvA,
                                                             rocblas_stride   stride_invA,
                                                             rocblas_int      batch_count);

/* ---- trsv: x := op(A)^-1 x --------------------------------------------------------------
 * rocblas-functions.h:9900-9908 (plain), 10041-10050 (batched), 10198-10209 (strided).
 * Solved as a one-row trsm (side right, transpose flipped); incx < 0 traverses x backwards. */
ROCBLAS_EXPORT rocblas_status rocblas_strsv(rocblas_handle    handle,
                                            rocblas_fill      uplo,
                                            rocblas_operation transA,
                                            rocblas_diagonal  diag,
                                            rocblas_int       n,
                                            const float*      A,
                                            rocblas_int       lda,
                                            float*            x,
                                            rocblas_int       incx);

ROCBLAS_EXPORT rocblas_status rocblas_dtrsv(rocblas_handle    handle,
                                            rocblas_fill      uplo,
                                            rocblas_operation transA,
                                            rocblas_diagonal  diag,
                                            rocblas_int       n,
                                            const double*     A,
                                            rocblas_int       lda,
                                            double*           x,
                                            rocblas_int       incx);

ROCBLAS_EXPORT rocblas_status rocblas_strsv_batched(rocblas_handle     handle,
                                                    rocblas_fill       uplo,
                                                    rocblas_operation  transA,
                                                    rocblas_diagonal   diag,
                                                    rocblas_int        n,
                                                    const float* const A[],
                                                    rocblas_int        lda,
                                                    float* const       x[],
                                                    rocblas_int        incx,
                                                    rocblas_int        batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_dtrsv_batched(rocblas_handle      handle,
                                                    rocblas_fill        uplo,
                                                    rocblas_operation   transA,
                                                    rocblas_diagonal    diag,
                                                    rocblas_int         n,
                                                    const double* const A[],
                                                    rocblas_int         lda,
                                                    double* const       x[],
                                                    rocblas_int         incx,
                                                    rocblas_int         batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_strsv_strided_batched(rocblas_handle    handle,
                                                            rocblas_fill      uplo,
                                                            rocblas_operation transA,
                                                            rocblas_diagonal  diag,
                                                            rocblas_int       n,
                                                            const float*      A,
                                                            rocblas_int       lda,
                                                            rocblas_stride    stride_A,
                                                            float*            x,
                                                            rocblas_int       incx,
                                                            rocblas_stride    stride_x,
                                                            rocblas_int       batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_dtrsv_strided_batched(rocblas_handle    handle,
                                                            rocblas_fill      uplo,
                                                            rocblas_operation transA,
                                                            rocblas_diagonal  diag,
                                                            rocblas_int       n,
                                                            const double*     A,
                                                            rocblas_int       lda,
                                                            rocblas_stride    stride_A,
                                                            double*           x,
                                                            rocblas_int       incx,
                                                            rocblas_stride    stride_x,
                                                            rocblas_int       batch_count);

/* ---- trmm: C := alpha op(A) B (side left) or alpha B op(A) (side right), A triangular ------
 * rocblas-functions.h:18300-18393 (plain), 18630-18644 (batched), 18904-18921 (strided).
 * B == C (in place) requires ldb == ldc (rocblas_trmm.hpp:99-102) and takes m*n*batch
 * elements of workspace from the handle. */
ROCBLAS_EXPORT rocblas_status rocblas_strmm(rocblas_handle    handle,
                                            rocblas_side      side,
                                            rocblas_fill      uplo,
                                            rocblas_operation transA,
                                            rocblas_diagonal  diag,
                                            rocblas_int       m,
                                            rocblas_int       n,
                                            const float*      alpha,
                                            const float*      A,
                                            rocblas_int       lda,
                                            const float*      B,
                                            rocblas_int       ldb,
                                            float*            C,
                                            rocblas_int       ldc);

ROCBLAS_EXPORT rocblas_status rocblas_dtrmm(rocblas_handle    handle,
                                            rocblas_side      side,
                                            rocblas_fill      uplo,
                                            rocblas_operation transA,
                                            rocblas_diagonal  diag,
                                            rocblas_int       m,
                                            rocblas_int       n,
                                            const double*     alpha,
                                            const double*     A,
                                            rocblas_int       lda,
                                            const double*     B,
                                            rocblas_int       ldb,
                                            double*           C,
                                            rocblas_int       ldc);

ROCBLAS_EXPORT rocblas_status rocblas_strmm_batched(rocblas_handle     handle,
                                                    rocblas_side       side,
                                                    rocblas_fill       uplo,
                                                    rocblas_operation  transA,
                                                    rocblas_diagonal   diag,
                                                    rocblas_int        m,
                                                    rocblas_int        n,
                                                    const float*       alpha,
                                                    const float* const A[],
                                                    rocblas_int        lda,
                                                    const float* const B[],
                                                    rocblas_int        ldb,
                                                    float* const       C[],
                                                    rocblas_int        ldc,
                                                    rocblas_int        batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_dtrmm_batched(rocblas_handle      handle,
                                                    rocblas_side        side,
                                                    rocblas_fill        uplo,
                                                    rocblas_operation   transA,
                                                    rocblas_diagonal    diag,
                                                    rocblas_int         m,
                                                    rocblas_int         n,
                                                    const double*       alpha,
                                                    const double* const A[],
                                                    rocblas_int         lda,
                                                    const double* const B[],
                                                    rocblas_int         ldb,
                                                    double* const       C[],
                                                    rocblas_int         ldc,
                                                    rocblas_int         batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_strmm_strided_batched(rocblas_handle    handle,
                                                            rocblas_side      side,
                                                            rocblas_fill      uplo,
                                                            rocblas_operation transA,
                                                            rocblas_diagonal  diag,
                                                            rocblas_int       m,
                                                            rocblas_int       n,
                                                            const float*      alpha,
                                                            const float*      A,
                                                            rocblas_int       lda,
                                                            rocblas_stride    stride_A,
                                                            const float*      B,
                                                            rocblas_int       ldb,
                                                            rocblas_stride    stride_B,
                                                            float*            C,
                                                            rocblas_int       ldc,
                                                            rocblas_stride    stride_C,
                                                            rocblas_int       batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_dtrmm_strided_batched(rocblas_handle    handle,
                                                            rocblas_side      side,
                                                            rocblas_fill      uplo,
                                                            rocblas_operation transA,
                                                            rocblas_diagonal  diag,
                                                            rocblas_int       m,
                                                            rocblas_int       n,
                                                            const double*     alpha,
                                                            const double*     A,
                                                            rocblas_int       lda,
                                                            rocblas_stride    stride_A,
                                                            const double*     B,
                                                            rocblas_int       ldb,
                                                            rocblas_stride    stride_B,
                                                            double*           C,
                                                            rocblas_int       ldc,
                                                            rocblas_stride    stride_C,
                                                            rocblas_int       batch_count);

/* ---- ILP64 (_64) forms: the same functions with 64-bit sizes, leading dimensions,
 * increments and batch counts (trsm: rocblas-functions.h:19441-19492, 19631-19685,
 * 19839-19901; trsv: 9930-9970, 10074-10118, 10237-10290; trmm: 18426-18485, 18679-18741,
 * 18962-19037).  The order of A must fit in 32 bits (A is k x k); a larger one is
 * rocblas_status_invalid_size. --------------------------------------------------------- */

ROCBLAS_EXPORT rocblas_status rocblas_strsm_64(rocblas_handle    handle,
                                               rocblas_side      side,
                                               rocblas_fill      uplo,
                                               rocblas_operation transA,
                                               rocblas_diagonal  diag,
                                               int64_t           m,
                                               int64_t           n,
                                               const float*      alpha,
                                               const float*      A,
                                               int64_t           lda,
                                               float*            B,
                                               int64_t           ldb);

ROCBLAS_EXPORT rocblas_status rocblas_strsm_batched_64(rocblas_handle      handle,
                                                       rocblas_side        side,
                                                       rocblas_fill        uplo,
                                                       rocblas_operation   transA,
                                                       rocblas_diagonal    diag,
                                                       int64_t             m,
                                                       int64_t             n,
                                                       const float*        alpha,
                                                       const float* const* A,
                                                       int64_t             lda,
                                                       float* const*       B,
                                                       int64_t             ldb,
                                                       int64_t             batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_strsm_strided_batched_64(rocblas_handle    handle,
                                                               rocblas_side      side,
                                                               rocblas_fill      uplo,
                                                               rocblas_operation transA,
                                                               rocblas_diagonal  diag,
                                                               int64_t           m,
                                                               int64_t           n,
                                                               const float*      alpha,
                                                               const float*      A,
                                                               int64_t           lda,
                                                               rocblas_stride    stride_a,
                                                               float*            B,
                                                               int64_t           ldb,
                                                               rocblas_stride    stride_b,
                                                               int64_t           batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_strsv_64(rocblas_handle    handle,
                                               rocblas_fill      uplo,
                                               rocblas_operation transA,
                                               rocblas_diagonal  diag,
                                               int64_t           n,
                                               const float*      A,
                                               int64_t           lda,
                                               float*            x,
                                               int64_t           incx);

ROCBLAS_EXPORT rocblas_status rocblas_strsv_batched_64(rocblas_handle      handle,
                                                       rocblas_fill        uplo,
                                                       rocblas_operation   transA,
                                                       rocblas_diagonal    diag,
                                                       int64_t             n,
                                                       const float* const* A,
                                                       int64_t             lda,
                                                       float* const*       x,
                                                       int64_t             incx,
                                                       int64_t             batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_strsv_strided_batched_64(rocblas_handle    handle,
                                                               rocblas_fill      uplo,
                                                               rocblas_operation transA,
                                                               rocblas_diagonal  diag,
                                                               int64_t           n,
                                                               const float*      A,
                                                               int64_t           lda,
                                                               rocblas_stride    stride_A,
                                                               float*            x,
                                                               int64_t           incx,
                                                               rocblas_stride    stride_x,
                                                               int64_t           batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_strmm_64(rocblas_handle    handle,
                                               rocblas_side      side,
                                               rocblas_fill      uplo,
                                               rocblas_operation transA,
                                               rocblas_diagonal  diag,
                                               int64_t           m,
                                               int64_t           n,
                                               const float*      alpha,
                                               const float*      A,
                                               int64_t           lda,
                                               const float*      B,
                                               int64_t           ldb,
                                               float*            C,
                                               int64_t           ldc);

ROCBLAS_EXPORT rocblas_status rocblas_strmm_batched_64(rocblas_handle      handle,
                                                       rocblas_side        side,
                                                       rocblas_fill        uplo,
                                                       rocblas_operation   transA,
                                                       rocblas_diagonal    diag,
                                                       int64_t             m,
                                                       int64_t             n,
                                                       const float*        alpha,
                                                       const float* const* A,
                                                       int64_t             lda,
                                                       const float* const* B,
                                                       int64_t             ldb,
                                                       float* const*       C,
                                                       int64_t             ldc,
                                                       int64_t             batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_strmm_strided_batched_64(rocblas_handle    handle,
                                                               rocblas_side      side,
                                                               rocblas_fill      uplo,
                                                               rocblas_operation transA,
                                                               rocblas_diagonal  diag,
                                                               int64_t           m,
                                                               int64_t           n,
                                                               const float*      alpha,
                                                               const float*      A,
                                                               int64_t           lda,
                                                               rocblas_stride    stride_A,
                                                               const float*      B,
                                                               int64_t           ldb,
                                                               rocblas_stride    stride_B,
                                                               float*            C,
                                                               int64_t           ldc,
                                                               rocblas_stride    stride_C,
                                                               int64_t           batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_dtrsm_64(rocblas_handle    handle,
                                               rocblas_side      side,
                                               rocblas_fill      uplo,
                                               rocblas_operation transA,
                                               rocblas_diagonal  diag,
                                               int64_t           m,
                                               int64_t           n,
                                               const double*     alpha,
                                               const double*     A,
                                               int64_t           lda,
                                               double*           B,
                                               int64_t           ldb);

ROCBLAS_EXPORT rocblas_status rocblas_dtrsm_batched_64(rocblas_handle       handle,
                                                       rocblas_side         side,
                                                       rocblas_fill         uplo,
                                                       rocblas_operation    transA,
                                                       rocblas_diagonal     diag,
                                                       int64_t              m,
                                                       int64_t              n,
                                                       const double*        alpha,
                                                       const double* const* A,
                                                       int64_t              lda,
                                                       double* const*       B,
                                                       int64_t              ldb,
                                                       int64_t              batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_dtrsm_strided_batched_64(rocblas_handle    handle,
                                                               rocblas_side      side,
                                                               rocblas_fill      uplo,
                                                               rocblas_operation transA,
                                                               rocblas_diagonal  diag,
                                                               int64_t           m,
                                                               int64_t           n,
                                                               const double*     alpha,
                                                               const double*     A,
                                                               int64_t           lda,
                                                               rocblas_stride    stride_a,
                                                               double*           B,
                                                               int64_t           ldb,
                                                               rocblas_stride    stride_b,
                                                               int64_t           batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_dtrsv_64(rocblas_handle    handle,
                                               rocblas_fill      uplo,
                                               rocblas_operation transA,
                                               rocblas_diagonal  diag,
                                               int64_t           n,
                                               const double*     A,
                                               int64_t           lda,
                                               double*           x,
                                               int64_t           incx);

ROCBLAS_EXPORT rocblas_status rocblas_dtrsv_batched_64(rocblas_handle       handle,
                                                       rocblas_fill         uplo,
                                                       rocblas_operation    transA,
                                                       rocblas_diagonal     diag,
                                                       int64_t              n,
                                                       const double* const* A,
                                                       int64_t              lda,
                                                       double* const*       x,
                                                       int64_t              incx,
                                                       int64_t              batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_dtrsv_strided_batched_64(rocblas_handle    handle,
                                                               rocblas_fill      uplo,
                                                               rocblas_operation transA,
                                                               rocblas_diagonal  diag,
                                                               int64_t           n,
                                                               const double*     A,
                                                               int64_t           lda,
                                                               rocblas_stride    stride_A,
                                                               double*           x,
                                                               int64_t           incx,
                                                               rocblas_stride    stride_x,
                                                               int64_t           batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_dtrmm_64(rocblas_handle    handle,
                                               rocblas_side      side,
                                               rocblas_fill      uplo,
                                               rocblas_operation transA,
                                               rocblas_diagonal  diag,
                                               int64_t           m,
                                               int64_t           n,
                                               const double*     alpha,
                                               const double*     A,
                                               int64_t           lda,
                                               const double*     B,
                                               int64_t           ldb,
                                               double*           C,
                                               int64_t           ldc);

ROCBLAS_EXPORT rocblas_status rocblas_dtrmm_batched_64(rocblas_handle       handle,
                                                       rocblas_side         side,
                                                       rocblas_fill         uplo,
                                                       rocblas_operation    transA,
                                                       rocblas_diagonal     diag,
                                                       int64_t              m,
                                                       int64_t              n,
                                                       const double*        alpha,
                                                       const double* const* A,
                                                       int64_t              lda,
                                                       const double* const* B,
                                                       int64_t              ldb,
                                                       double* const*       C,
                                                       int64_t              ldc,
                                                       int64_t              batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_dtrmm_strided_batched_64(rocblas_handle    handle,
                                                               rocblas_side      side,
                                                               rocblas_fill      uplo,
                                                               rocblas_operation transA,
                                                               rocblas_diagonal  diag,
                                                               int64_t           m,
                                                               int64_t           n,
                                                               const double*     alpha,
                                                               const double*     A,
                                                               int64_t           lda,
                                                               rocblas_stride    stride_A,
                                                               const double*     B,
                                                               int64_t           ldb,
                                                               rocblas_stride    stride_B,
                                                               double*           C,
                                                               int64_t           ldc,
                                                               rocblas_stride    stride_C,
                                                               int64_t           batch_count);

/* ---- complex (c, z): declarations starting at rocblas-functions.h:19414 (trsm), 19602
 * (trsm_batched), 19806 (trsm_strided_batched), 9910 / 10052 / 10211 (trsv forms) and 18395 /
 * 18646 / 18923 (trmm forms), and their ILP64 forms.  trans C solves with conj(A)^T.  rocblas_trsm_ex and its batched forms take
 * compute_type rocblas_datatype_f32_c / f64_c. ------------------------------------------- */

ROCBLAS_EXPORT rocblas_status rocblas_ctrsm(rocblas_handle               handle,
                                            rocblas_side                 side,
                                            rocblas_fill                 uplo,
                                            rocblas_operation            transA,
                                            rocblas_diagonal             diag,
                                            rocblas_int                  m,
                                            rocblas_int                  n,
                                            const rocblas_float_complex* alpha,
                                            const rocblas_float_complex* A,
                                            rocblas_int                  lda,
                                            rocblas_float_complex*       B,
                                            rocblas_int                  ldb);

ROCBLAS_EXPORT rocblas_status rocblas_ctrsm_batched(rocblas_handle                      handle,
                                                    rocblas_side                        side,
                                                    rocblas_fill                        uplo,
                                                    rocblas_operation                   transA,
                                                    rocblas_diagonal                    diag,
                                                    rocblas_int                         m,
                                                    rocblas_int                         n,
                                                    const rocblas_float_complex*        alpha,
                                                    const rocblas_float_complex* const* A,
                                                    rocblas_int                         lda,
                                                    rocblas_float_complex* const*       B,
                                                    rocblas_int                         ldb,
                                                    rocblas_int                         batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_ctrsm_strided_batched(rocblas_handle               handle,
                                                            rocblas_side                 side,
                                                            rocblas_fill                 uplo,
                                                            rocblas_operation            transA,
                                                            rocblas_diagonal             diag,
                                                            rocblas_int                  m,
                                                            rocblas_int                  n,
                                                            const rocblas_float_complex* alpha,
                                                            const rocblas_float_complex* A,
                                                            rocblas_int                  lda,
                                                            rocblas_stride               stride_a,
                                                            rocblas_float_complex*       B,
                                                            rocblas_int                  ldb,
                                                            rocblas_stride               stride_b,
                                                            rocblas_int                  batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_ctrsv(rocblas_handle               handle,
                                            rocblas_fill                 uplo,
                                            rocblas_operation            transA,
                                            rocblas_diagonal             diag,
                                            rocblas_int                  n,
                                            const rocblas_float_complex* A,
                                            rocblas_int                  lda,
                                            rocblas_float_complex*       x,
                                            rocblas_int                  incx);

ROCBLAS_EXPORT rocblas_status rocblas_ctrsv_batched(rocblas_handle                      handle,
                                                    rocblas_fill                        uplo,
                                                    rocblas_operation                   transA,
                                                    rocblas_diagonal                    diag,
                                                    rocblas_int                         n,
                                                    const rocblas_float_complex* const* A,
                                                    rocblas_int                         lda,
                                                    rocblas_float_complex* const*       x,
                                                    rocblas_int                         incx,
                                                    rocblas_int                         batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_ctrsv_strided_batched(rocblas_handle               handle,
                                                            rocblas_fill                 uplo,
                                                            rocblas_operation            transA,
                                                            rocblas_diagonal             diag,
                                                            rocblas_int                  n,
                                                            const rocblas_float_complex* A,
                                                            rocblas_int                  lda,
                                                            rocblas_stride               stride_A,
                                                            rocblas_float_complex*       x,
                                                            rocblas_int                  incx,
                                                            rocblas_stride               stride_x,
                                                            rocblas_int                  batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_ctrmm(rocblas_handle               handle,
                                            rocblas_side                 side,
                                            rocblas_fill                 uplo,
                                            rocblas_operation            transA,
                                            rocblas_diagonal             diag,
                                            rocblas_int                  m,
                                            rocblas_int                  n,
                                            const rocblas_float_complex* alpha,
                                            const rocblas_float_complex* A,
                                            rocblas_int                  lda,
                                            const rocblas_float_complex* B,
                                            rocblas_int                  ldb,
                                            rocblas_float_complex*       C,
                                            rocblas_int                  ldc);

ROCBLAS_EXPORT rocblas_status rocblas_ctrmm_batched(rocblas_handle                      handle,
                                                    rocblas_side                        side,
                                                    rocblas_fill                        uplo,
                                                    rocblas_operation                   transA,
                                                    rocblas_diagonal                    diag,
                                                    rocblas_int                         m,
                                                    rocblas_int                         n,
                                                    const rocblas_float_complex*        alpha,
                                                    const rocblas_float_complex* const* A,
                                                    rocblas_int                         lda,
                                                    const rocblas_float_complex* const* B,
                                                    rocblas_int                         ldb,
                                                    rocblas_float_complex* const*       C,
                                                    rocblas_int                         ldc,
                                                    rocblas_int                         batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_ctrmm_strided_batched(rocblas_handle               handle,
                                                            rocblas_side                 side,
                                                            rocblas_fill                 uplo,
                                                            rocblas_operation            transA,
                                                            rocblas_diagonal             diag,
                                                            rocblas_int                  m,
                                                            rocblas_int                  n,
                                                            const rocblas_float_complex* alpha,
                                                            const rocblas_float_complex* A,
                                                            rocblas_int                  lda,
                                                            rocblas_stride               stride_A,
                                                            const rocblas_float_complex* B,
                                                            rocblas_int                  ldb,
                                                            rocblas_stride               stride_B,
                                                            rocblas_float_complex*       C,
                                                            rocblas_int                  ldc,
                                                            rocblas_stride               stride_C,
                                                            rocblas_int                  batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_ztrsm(rocblas_handle                handle,
                                            rocblas_side                  side,
                                            rocblas_fill                  uplo,
                                            rocblas_operation             transA,
                                            rocblas_diagonal              diag,
                                            rocblas_int                   m,
                                            rocblas_int                   n,
                                            const rocblas_double_complex* alpha,
                                            const rocblas_double_complex* A,
                                            rocblas_int                   lda,
                                            rocblas_double_complex*       B,
                                            rocblas_int                   ldb);

ROCBLAS_EXPORT rocblas_status rocblas_ztrsm_batched(rocblas_handle                       handle,
                                                    rocblas_side                         side,
                                                    rocblas_fill                         uplo,
                                                    rocblas_operation                    transA,
                                                    rocblas_diagonal                     diag,
                                                    rocblas_int                          m,
                                                    rocblas_int                          n,
                                                    const rocblas_double_complex*        alpha,
                                                    const rocblas_double_complex* const* A,
                                                    rocblas_int                          lda,
                                                    rocblas_double_complex* const*       B,
                                                    rocblas_int                          ldb,
                                                    rocblas_int                          batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_ztrsm_strided_batched(rocblas_handle                handle,
                                                            rocblas_side                  side,
                                                            rocblas_fill                  uplo,
                                                            rocblas_operation             transA,
                                                            rocblas_diagonal              diag,
                                                            rocblas_int                   m,
                                                            rocblas_int                   n,
                                                            const rocblas_double_complex* alpha,
                                                            const rocblas_double_complex* A,
                                                            rocblas_int                   lda,
                                                            rocblas_stride                stride_a,
                                                            rocblas_double_complex*       B,
                                                            rocblas_int                   ldb,
                                                            rocblas_stride                stride_b,
                                                            rocblas_int                   batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_ztrsv(rocblas_handle                handle,
                                            rocblas_fill                  uplo,
                                            rocblas_operation             transA,
                                            rocblas_diagonal              diag,
                                            rocblas_int                   n,
                                            const rocblas_double_complex* A,
                                            rocblas_int                   lda,
                                            rocblas_double_complex*       x,
                                            rocblas_int                   incx);

ROCBLAS_EXPORT rocblas_status rocblas_ztrsv_batched(rocblas_handle                       handle,
                                                    rocblas_fill                         uplo,
                                                    rocblas_operation                    transA,
                                                    rocblas_diagonal                     diag,
                                                    rocblas_int                          n,
                                                    const rocblas_double_complex* const* A,
                                                    rocblas_int                          lda,
                                                    rocblas_double_complex* const*       x,
                                                    rocblas_int                          incx,
                                                    rocblas_int                          batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_ztrsv_strided_batched(rocblas_handle                handle,
                                                            rocblas_fill                  uplo,
                                                            rocblas_operation             transA,
                                                            rocblas_diagonal              diag,
                                                            rocblas_int                   n,
                                                            const rocblas_double_complex* A,
                                                            rocblas_int                   lda,
                                                            rocblas_stride                stride_A,
                                                            rocblas_double_complex*       x,
                                                            rocblas_int                   incx,
                                                            rocblas_stride                stride_x,
                                                            rocblas_int                   batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_ztrmm(rocblas_handle                handle,
                                            rocblas_side                  side,
                                            rocblas_fill                  uplo,
                                            rocblas_operation             transA,
                                            rocblas_diagonal              diag,
                                            rocblas_int                   m,
                                            rocblas_int                   n,
                                            const rocblas_double_complex* alpha,
                                            const rocblas_double_complex* A,
                                            rocblas_int                   lda,
                                            const rocblas_double_complex* B,
                                            rocblas_int                   ldb,
                                            rocblas_double_complex*       C,
                                            rocblas_int                   ldc);

ROCBLAS_EXPORT rocblas_status rocblas_ztrmm_batched(rocblas_handle                       handle,
                                                    rocblas_side                         side,
                                                    rocblas_fill                         uplo,
                                                    rocblas_operation                    transA,
                                                    rocblas_diagonal                     diag,
                                                    rocblas_int                          m,
                                                    rocblas_int                          n,
                                                    const rocblas_double_complex*        alpha,
                                                    const rocblas_double_complex* const* A,
                                                    rocblas_int                          lda,
                                                    const rocblas_double_complex* const* B,
                                                    rocblas_int                          ldb,
                                                    rocblas_double_complex* const*       C,
                                                    rocblas_int                          ldc,
                                                    rocblas_int                          batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_ztrmm_strided_batched(rocblas_handle                handle,
                                                            rocblas_side                  side,
                                                            rocblas_fill                  uplo,
                                                            rocblas_operation             transA,
                                                            rocblas_diagonal              diag,
                                                            rocblas_int                   m,
                                                            rocblas_int                   n,
                                                            const rocblas_double_complex* alpha,
                                                            const rocblas_double_complex* A,
                                                            rocblas_int                   lda,
                                                            rocblas_stride                stride_A,
                                                            const rocblas_double_complex* B,
                                                            rocblas_int                   ldb,
                                                            rocblas_stride                stride_B,
                                                            rocblas_double_complex*       C,
                                                            rocblas_int                   ldc,
                                                            rocblas_stride                stride_C,
                                                            rocblas_int                   batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_ctrsm_64(rocblas_handle               handle,
                                               rocblas_side                 side,
                                               rocblas_fill                 uplo,
                                               rocblas_operation            transA,
                                               rocblas_diagonal             diag,
                                               int64_t                      m,
                                               int64_t                      n,
                                               const rocblas_float_complex* alpha,
                                               const rocblas_float_complex* A,
                                               int64_t                      lda,
                                               rocblas_float_complex*       B,
                                               int64_t                      ldb);

ROCBLAS_EXPORT rocblas_status rocblas_ctrsm_batched_64(rocblas_handle                      handle,
                                                       rocblas_side                        side,
                                                       rocblas_fill                        uplo,
                                                       rocblas_operation                   transA,
                                                       rocblas_diagonal                    diag,
                                                       int64_t                             m,
                                                       int64_t                             n,
                                                       const rocblas_float_complex*        alpha,
                                                       const rocblas_float_complex* const* A,
                                                       int64_t                             lda,
                                                       rocblas_float_complex* const*       B,
                                                       int64_t                             ldb,
                                                       int64_t                             batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_ctrsm_strided_batched_64(rocblas_handle               handle,
                                                               rocblas_side                 side,
                                                               rocblas_fill                 uplo,
                                                               rocblas_operation            transA,
                                                               rocblas_diagonal             diag,
                                                               int64_t                      m,
                                                               int64_t                      n,
                                                               const rocblas_float_complex* alpha,
                                                               const rocblas_float_complex* A,
                                                               int64_t                      lda,
                                                               rocblas_stride               stride_a,
                                                               rocblas_float_complex*       B,
                                                               int64_t                      ldb,
                                                               rocblas_stride               stride_b,
                                                               int64_t                      batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_ctrsv_64(rocblas_handle               handle,
                                               rocblas_fill                 uplo,
                                               rocblas_operation            transA,
                                               rocblas_diagonal             diag,
                                               int64_t                      n,
                                               const rocblas_float_complex* A,
                                               int64_t                      lda,
                                               rocblas_float_complex*       x,
                                               int64_t                      incx);

ROCBLAS_EXPORT rocblas_status rocblas_ctrsv_batched_64(rocblas_handle                      handle,
                                                       rocblas_fill                        uplo,
                                                       rocblas_operation                   transA,
                                                       rocblas_diagonal                    diag,
                                                       int64_t                             n,
                                                       const rocblas_float_complex* const* A,
                                                       int64_t                             lda,
                                                       rocblas_float_complex* const*       x,
                                                       int64_t                             incx,
                                                       int64_t                             batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_ctrsv_strided_batched_64(rocblas_handle               handle,
                                                               rocblas_fill                 uplo,
                                                               rocblas_operation            transA,
                                                               rocblas_diagonal             diag,
                                                               int64_t                      n,
                                                               const rocblas_float_complex* A,
                                                               int64_t                      lda,
                                                               rocblas_stride               stride_A,
                                                               rocblas_float_complex*       x,
                                                               int64_t                      incx,
                                                               rocblas_stride               stride_x,
                                                               int64_t                      batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_ctrmm_64(rocblas_handle               handle,
                                               rocblas_side                 side,
                                               rocblas_fill                 uplo,
                                               rocblas_operation            transA,
                                               rocblas_diagonal             diag,
                                               int64_t                      m,
                                               int64_t                      n,
                                               const rocblas_float_complex* alpha,
                                               const rocblas_float_complex* A,
                                               int64_t                      lda,
                                               const rocblas_float_complex* B,
                                               int64_t                      ldb,
                                               rocblas_float_complex*       C,
                                               int64_t                      ldc);

ROCBLAS_EXPORT rocblas_status rocblas_ctrmm_batched_64(rocblas_handle                      handle,
                                                       rocblas_side                        side,
                                                       rocblas_fill                        uplo,
                                                       rocblas_operation                   transA,
                                                       rocblas_diagonal                    diag,
                                                       int64_t                             m,
                                                       int64_t                             n,
                                                       const rocblas_float_complex*        alpha,
                                                       const rocblas_float_complex* const* A,
                                                       int64_t                             lda,
                                                       const rocblas_float_complex* const* B,
                                                       int64_t                             ldb,
                                                       rocblas_float_complex* const*       C,
                                                       int64_t                             ldc,
                                                       int64_t                             batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_ctrmm_strided_batched_64(rocblas_handle               handle,
                                                               rocblas_side                 side,
                                                               rocblas_fill                 uplo,
                                                               rocblas_operation            transA,
                                                               rocblas_diagonal             diag,
                                                               int64_t                      m,
                                                               int64_t                      n,
                                                               const rocblas_float_complex* alpha,
                                                               const rocblas_float_complex* A,
                                                               int64_t                      lda,
                                                               rocblas_stride               stride_A,
                                                               const rocblas_float_complex* B,
                                                               int64_t                      ldb,
                                                               rocblas_stride               stride_B,
                                                               rocblas_float_complex*       C,
                                                               int64_t                      ldc,
                                                               rocblas_stride               stride_C,
                                                               int64_t                      batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_ztrsm_64(rocblas_handle                handle,
                                               rocblas_side                  side,
                                               rocblas_fill                  uplo,
                                               rocblas_operation             transA,
                                               rocblas_diagonal              diag,
                                               int64_t                       m,
                                               int64_t                       n,
                                               const rocblas_double_complex* alpha,
                                               const rocblas_double_complex* A,
                                               int64_t                       lda,
                                               rocblas_double_complex*       B,
                                               int64_t                       ldb);

ROCBLAS_EXPORT rocblas_status rocblas_ztrsm_batched_64(rocblas_handle                       handle,
                                                       rocblas_side                         side,
                                                       rocblas_fill                         uplo,
                                                       rocblas_operation                    transA,
                                                       rocblas_diagonal                     diag,
                                                       int64_t                              m,
                                                       int64_t                              n,
                                                       const rocblas_double_complex*        alpha,
                                                       const rocblas_double_complex* const* A,
                                                       int64_t                              lda,
                                                       rocblas_double_complex* const*       B,
                                                       int64_t                              ldb,
                                                       int64_t                              batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_ztrsm_strided_batched_64(rocblas_handle                handle,
                                                               rocblas_side                  side,
                                                               rocblas_fill                  uplo,
                                                               rocblas_operation             transA,
                                                               rocblas_diagonal              diag,
                                                               int64_t                       m,
                                                               int64_t                       n,
                                                               const rocblas_double_complex* alpha,
                                                               const rocblas_double_complex* A,
                                                               int64_t                       lda,
                                                               rocblas_stride                stride_a,
                                                               rocblas_double_complex*       B,
                                                               int64_t                       ldb,
                                                               rocblas_stride                stride_b,
                                                               int64_t                       batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_ztrsv_64(rocblas_handle                handle,
                                               rocblas_fill                  uplo,
                                               rocblas_operation             transA,
                                               rocblas_diagonal              diag,
                                               int64_t                       n,
                                               const rocblas_double_complex* A,
                                               int64_t                       lda,
                                               rocblas_double_complex*       x,
                                               int64_t                       incx);

ROCBLAS_EXPORT rocblas_status rocblas_ztrsv_batched_64(rocblas_handle                       handle,
                                                       rocblas_fill                         uplo,
                                                       rocblas_operation                    transA,
                                                       rocblas_diagonal                     diag,
                                                       int64_t                              n,
                                                       const rocblas_double_complex* const* A,
                                                       int64_t                              lda,
                                                       rocblas_double_complex* const*       x,
                                                       int64_t                              incx,
                                                       int64_t                              batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_ztrsv_strided_batched_64(rocblas_handle                handle,
                                                               rocblas_fill                  uplo,
                                                               rocblas_operation             transA,
                                                               rocblas_diagonal              diag,
                                                               int64_t                       n,
                                                               const rocblas_double_complex* A,
                                                               int64_t                       lda,
                                                               rocblas_stride                stride_A,
                                                               rocblas_double_complex*       x,
                                                               int64_t                       incx,
                                                               rocblas_stride                stride_x,
                                                               int64_t                       batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_ztrmm_64(rocblas_handle                handle,
                                               rocblas_side                  side,
                                               rocblas_fill                  uplo,
                                               rocblas_operation             transA,
                                               rocblas_diagonal              diag,
                                               int64_t                       m,
                                               int64_t                       n,
                                               const rocblas_double_complex* alpha,
                                               const rocblas_double_complex* A,
                                               int64_t                       lda,
                                               const rocblas_double_complex* B,
                                               int64_t                       ldb,
                                               rocblas_double_complex*       C,
                                               int64_t                       ldc);

ROCBLAS_EXPORT rocblas_status rocblas_ztrmm_batched_64(rocblas_handle                       handle,
                                                       rocblas_side                         side,
                                                       rocblas_fill                         uplo,
                                                       rocblas_operation                    transA,
                                                       rocblas_diagonal                     diag,
                                                       int64_t                              m,
                                                       int64_t                              n,
                                                       const rocblas_double_complex*        alpha,
                                                       const rocblas_double_complex* const* A,
                                                       int64_t                              lda,
                                                       const rocblas_double_complex* const* B,
                                                       int64_t                              ldb,
                                                       rocblas_double_complex* const*       C,
                                                       int64_t                              ldc,
                                                       int64_t                              batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_ztrmm_strided_batched_64(rocblas_handle                handle,
                                                               rocblas_side                  side,
                                                               rocblas_fill                  uplo,
                                                               rocblas_operation             transA,
                                                               rocblas_diagonal              diag,
                                                               int64_t                       m,
                                                               int64_t                       n,
                                                               const rocblas_double_complex* alpha,
                                                               const rocblas_double_complex* A,
                                                               int64_t                       lda,
                                                               rocblas_stride                stride_A,
                                                               const rocblas_double_complex* B,
                                                               int64_t                       ldb,
                                                               rocblas_stride                stride_B,
                                                               rocblas_double_complex*       C,
                                                               int64_t                       ldc,
                                                               rocblas_stride                stride_C,
                                                               int64_t                       batch_count);

/* ---- complex trtri: rocblas-functions.h:19099-19117, 19179-19198, 19273-19296; inv(A) is the
 * solution of A X = I by the complex solve (a zero non-unit diagonal is not read as 1). ---- */

ROCBLAS_EXPORT rocblas_status rocblas_ctrtri(rocblas_handle               handle,
                                             rocblas_fill                 uplo,
                                             rocblas_diagonal             diag,
                                             rocblas_int                  n,
                                             const rocblas_float_complex* A,
                                             rocblas_int                  lda,
                                             rocblas_float_complex*       invA,
                                             rocblas_int                  ldinvA);

ROCBLAS_EXPORT rocblas_status rocblas_ctrtri_batched(rocblas_handle                      handle,
                                                     rocblas_fill                        uplo,
                                                     rocblas_diagonal                    diag,
                                                     rocblas_int                         n,
                                                     const rocblas_float_complex* const* A,
                                                     rocblas_int                         lda,
                                                     rocblas_float_complex* const*       invA,
                                                     rocblas_int                         ldinvA,
                                                     rocblas_int                         batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_ctrtri_strided_batched(rocblas_handle               handle,
                                                             rocblas_fill                 uplo,
                                                             rocblas_diagonal             diag,
                                                             rocblas_int                  n,
                                                             const rocblas_float_complex* A,
                                                             rocblas_int                  lda,
                                                             rocblas_stride               stride_a,
                                                             rocblas_float_complex*       invA,
                                                             rocblas_int                  ldinvA,
                                                             rocblas_stride               stride_invA,
                                                             rocblas_int                  batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_ztrtri(rocblas_handle                handle,
                                             rocblas_fill                  uplo,
                                             rocblas_diagonal              diag,
                                             rocblas_int                   n,
                                             const rocblas_double_complex* A,
                                             rocblas_int                   lda,
                                             rocblas_double_complex*       invA,
                                             rocblas_int                   ldinvA);

ROCBLAS_EXPORT rocblas_status rocblas_ztrtri_batched(rocblas_handle                       handle,
                                                     rocblas_fill                         uplo,
                                                     rocblas_diagonal                     diag,
                                                     rocblas_int                          n,
                                                     const rocblas_double_complex* const* A,
                                                     rocblas_int                          lda,
                                                     rocblas_double_complex* const*       invA,
                                                     rocblas_int                          ldinvA,
                                                     rocblas_int                          batch_count);

ROCBLAS_EXPORT rocblas_status rocblas_ztrtri_strided_batched(rocblas_handle                handle,
                                                             rocblas_fill                  uplo,
                                                             rocblas_diagonal              diag,
                                                             rocblas_int                   n,
                                                             const rocblas_double_complex* A,
                                                             rocblas_int                   lda,
                                                             rocblas_stride                stride_a,
                                                             rocblas_double_complex*       invA,
                                                             rocblas_int                   ldinvA,
                                                             rocblas_stride                stride_invA,
                                                             rocblas_int                   batch_count);

#ifdef __cplusplus
}
#endif

#endif /* ROCBLAS_B200_ROCBLAS_H */
