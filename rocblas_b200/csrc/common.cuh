// Shared device-side helpers for the B200 TRSM kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace rb200
{

// One operand of a (possibly batched) call.  Matrix b of the batch starts at
//   arr ? arr[b] : base + b * stride
// and `offset` (elements) is added after that, so sub-blocks of every matrix in a batch are
// addressed by shifting `offset`.  This covers the plain, _strided_batched (stride) and
// _batched (device array of device pointers) forms of the reference API
// (library/src/include/utility.hpp:119-160, load_ptr_batch) with one kernel body.
template <typename T>
struct BatchPtr
{
    T*          base   = nullptr;
    const void* arr    = nullptr;
    int64_t     stride = 0;
    int64_t     offset = 0;

    __device__ __forceinline__ T* get(int b) const
    {
        T* p = arr ? reinterpret_cast<T* const*>(arr)[b] : base + (int64_t)b * stride;
        return p + offset;
    }
    __host__ __device__ BatchPtr shifted(int64_t d) const
    {
        BatchPtr r = *this;
        r.offset += d;
        return r;
    }
    __host__ __device__ bool valid() const { return base != nullptr || arr != nullptr; }
};

// A scalar that is either an immediate (host pointer mode) or read on the device from a
// device pointer (device pointer mode).  Reading on the device means no device-to-host
// synchronisation is needed, unlike the reference launcher
// (library/src/blas3/rocblas_trsm_kernels.hpp:3654-3666), so calls stay capturable in
// device pointer mode too.
template <typename T>
struct Scalar
{
    T        val = T(1);
    const T* ptr = nullptr;
    __device__ __forceinline__ T get() const { return ptr ? __ldg(ptr) : val; }
};

__host__ __device__ constexpr int64_t ceil_div(int64_t a, int64_t b)
{
    return (a + b - 1) / b;
}

// rocblas enum values (library/include/internal/rocblas-types.h:123-157)
enum : int
{
    kOpN    = 111,
    kOpT    = 112,
    kOpC    = 113,
    kUpper  = 121,
    kLower  = 122,
    kNonUnit = 131,
    kUnit   = 132,
    kLeft   = 141,
    kRight  = 142
};

// triangle masks used when an operand is a triangular block (stored coordinates r, c)
enum : int
{
    kTriNone        = 0,
    kTriLower       = 1, // keep r >= c
    kTriUpper       = 2, // keep r <= c
    kTriLowerStrict = 3, // keep r > c
    kTriUpperStrict = 4  // keep r < c
};

__device__ __forceinline__ bool tri_keep(int tri, int64_t r, int64_t c)
{
    switch(tri)
    {
    case kTriLower: return r >= c;
    case kTriUpper: return r <= c;
    case kTriLowerStrict: return r > c;
    case kTriUpperStrict: return r < c;
    default: return true;
    }
}

} // namespace rb200
