/*
 * rocblas_b200_ext.h -- functions of librocblas_b200.so that have no counterpart in the
 * reference rocBLAS API.  They extend the drop-in surface of include/rocblas.h and never
 * change the behaviour of the functions declared there.
 */
#ifndef ROCBLAS_B200_EXT_H
#define ROCBLAS_B200_EXT_H

#include "rocblas.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Number of GPU kernels this library has launched in the calling process so far (all
 * handles, all devices).  Benchmarks read it before and after a timed region to state how
 * many of the launches in that region were this library's own kernels. */
ROCBLAS_EXPORT uint64_t rocblas_b200_kernel_launch_count(void);

#ifdef __cplusplus
}
#endif

#endif /* ROCBLAS_B200_EXT_H */
