// The library context behind rocblas_handle.
//
// Mirrors the state the reference keeps in _rocblas_handle (library/src/include/handle.hpp):
// the stream, the pointer mode, and the device-memory workspace with its three ownership
// modes and the size-query protocol (handle.hpp:374-430, handle.cpp:449-646):
//   - rocblas-managed (default): the workspace grows on demand;
//   - user-managed: rocblas_set_device_memory_size fixed a size the library allocated;
//   - user-owned: rocblas_set_workspace handed in a caller buffer.
// A handle is used by one host thread at a time (as in every reference test); distinct
// handles share nothing.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cuda_runtime.h>

#include "../../include/rocblas.h"

enum class MemOwner
{
    managed,
    user_managed,
    user_owned
};

struct _rocblas_handle
{
    int                  device       = -1;
    int                  sm_count     = 148;
    cudaStream_t         stream       = nullptr;
    rocblas_pointer_mode pointer_mode = rocblas_pointer_mode_host;

    MemOwner owner         = MemOwner::managed;
    void*    mem           = nullptr;
    size_t   mem_size      = 0;
    bool     size_query    = false;
    size_t   query_size    = 0;

    // device word where kernels with bounded waits record a timeout (lazily allocated)
    int* err_dev = nullptr;

    // streams, events and device buffers of the host-buffer entry points (lazily created)
    struct HostPathRes* host_res = nullptr;

    // ROCBLAS_LAYER and ROCBLAS_CHECK_NUMERICS as read at creation, and the log streams
    int   layer_mode     = 0;
    int   check_numerics = 0;
    int   atomics_mode   = 1; // rocblas_atomics_allowed, the reference's default
    int     math_mode          = 0; // rocblas_default_math
    int     performance_metric = 0; // rocblas_default_performance_metric
    double* fitness_query      = nullptr;
    FILE* log_trace_os   = nullptr;
    FILE* log_bench_os   = nullptr;
    FILE* log_profile_os = nullptr;

    // rounding of every workspace request (handle.hpp:56-61)
    static size_t roundup(size_t s) { return (s + 63) / 64 * 64; }

    // size-query bookkeeping: returns size_increased / size_unchanged (handle.hpp:418-431)
    rocblas_status set_optimal_size(size_t s)
    {
        if(!size_query)
            return rocblas_status_size_query_mismatch;
        s = roundup(s);
        if(s > query_size)
        {
            query_size = s;
            return rocblas_status_size_increased;
        }
        return rocblas_status_size_unchanged;
    }

    // Borrow `bytes` of workspace for the duration of one call; nullptr if not available.
    void* borrow(size_t bytes);

    // release the managed allocation (not a user buffer)
    rocblas_status free_mem();
};
