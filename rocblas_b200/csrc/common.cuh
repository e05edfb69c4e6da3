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

// ---- complex numbers --------------------------------------------------------------------------
// rocblas_float_complex / rocblas_double_complex are {x, y} pairs of float / double
// (library/include/internal/rocblas-complex-types.h:82-91); cplx<R> has that layout and the
// arithmetic the kernels need.  Complex division uses Smith's scaling (R. L. Smith, "Algorithm
// 116: Complex division", CACM 5(8), 1962) so that |d|^2 is never formed.
template <typename R>
struct cplx
{
    R x, y;
    __host__ __device__ constexpr cplx() : x(0), y(0) {}
    __host__ __device__ constexpr cplx(R re) : x(re), y(0) {}
    __host__ __device__ constexpr cplx(R re, R im) : x(re), y(im) {}
    __host__ __device__ cplx& operator+=(const cplx& b) { x += b.x; y += b.y; return *this; }
    __host__ __device__ cplx& operator-=(const cplx& b) { x -= b.x; y -= b.y; return *this; }
    __host__ __device__ cplx& operator*=(const cplx& b) { *this = *this * b; return *this; }
    friend __host__ __device__ cplx operator+(cplx a, cplx b) { return {a.x + b.x, a.y + b.y}; }
    friend __host__ __device__ cplx operator-(cplx a, cplx b) { return {a.x - b.x, a.y - b.y}; }
    friend __host__ __device__ cplx operator-(cplx a) { return {-a.x, -a.y}; }
    friend __host__ __device__ cplx operator*(cplx a, cplx b)
    {
        return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
    }
    friend __host__ __device__ cplx operator/(cplx n, cplx d)
    {
        const R ax = d.x < R(0) ? -d.x : d.x, ay = d.y < R(0) ? -d.y : d.y;
        if(ax >= ay)
        {
            const R r = d.y / d.x, den = d.x + d.y * r;
            return {(n.x + n.y * r) / den, (n.y - n.x * r) / den};
        }
        const R r = d.x / d.y, den = d.x * r + d.y;
        return {(n.x * r + n.y) / den, (n.y * r - n.x) / den};
    }
    friend __host__ __device__ bool operator==(cplx a, cplx b) { return a.x == b.x && a.y == b.y; }
    friend __host__ __device__ bool operator!=(cplx a, cplx b) { return !(a == b); }
};

template <typename T>
struct is_cplx
{
    static constexpr bool value = false;
};
template <typename R>
struct is_cplx<cplx<R>>
{
    static constexpr bool value = true;
};

// v, or conj(v) when c (real types: v)
template <typename T>
__host__ __device__ __forceinline__ T conj_if(T v, int)
{
    return v;
}
template <typename R>
__host__ __device__ __forceinline__ cplx<R> conj_if(cplx<R> v, int c)
{
    return c ? cplx<R>(v.x, -v.y) : v;
}

// warp broadcast of lane `src`'s value
template <typename T>
__device__ __forceinline__ T shfl_idx(T v, int src)
{
    return __shfl_sync(0xffffffffu, v, src);
}
template <typename R>
__device__ __forceinline__ cplx<R> shfl_idx(cplx<R> v, int src)
{
    return {__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src)};
}

// read-only load
template <typename T>
__device__ __forceinline__ T ldg_val(const T* p)
{
    return __ldg(p);
}
template <typename R>
__device__ __forceinline__ cplx<R> ldg_val(const cplx<R>* p)
{
    return {__ldg(&p->x), __ldg(&p->y)};
}

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
    __device__ __forceinline__ T get() const { return ptr ? ldg_val(ptr) : val; }
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
