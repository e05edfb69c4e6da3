// Tiled GEMM used for the TRSM trailing updates and for applying the inverted diagonal
// blocks (invA) to a block of right-hand sides.
//
//     C := a * op(P) * op(Q) + b * C          (column-major, 64-bit strides, batched)
//
// It replaces the rocblas_internal_gemm calls that the reference makes from
// rocblas_trsm_left / rocblas_trsm_right / special_trsm_template
// (library/src/blas3/rocblas_trsm_kernels.hpp:302-716, 761-1155, 1237-1449) and the
// Tensile/hipBLASLt contraction behind them (blas3/Tensile/gemm_templates.cpp:41-181).
//
// FP64 tiles run on the FP64 tensor path (DMMA, mma.sync m8n8k4 .f64); the Blackwell
// tcgen05 tensor cores have no f64 kind.  FP32 tiles use register-blocked FFMA so that the
// plain strsm keeps IEEE FP32 products (TF32 would not meet the FP32 error bound).
//
// In-place use for the invA application: when op(P) is the (<=128 x <=128) inverse block
// and Q == C (side left), a CTA's tile spans all M rows, so every element of Q the CTA
// reads is read before the epilogue writes the same columns, and no other CTA touches
// them.  The same holds for side right with P == C and N <= BN.  b must be 0 then.
#pragma once
#include "common.cuh"

namespace rb200
{

template <typename T>
struct GemmParams
{
    int         M, N, K;
    BatchPtr<T> P, Q, C;
    int64_t     ldp, ldq, ldc;
    int         transP, transQ; // 0: op(X) = X, 1: op(X) = X^T
    int         conjP, conjQ;   // complex types: op(X) conjugated as well (trans C); else unused
    int         triP, triQ;     // kTri* mask in stored coordinates (triangular invA blocks)
    T           a_imm;          // a = a_user ? ualpha : a_imm
    int         a_user;
    T           b_imm;          // b = b_user ? ualpha : b_imm; b == 0 => C is not read
    int         b_user;
    Scalar<T>   ualpha;         // the caller's alpha
    int         zero_guard;     // ualpha == 0 => C tile := 0 without reading P, Q or C
    int         batch_base;     // first batch index of this launch (grid.z chunking)
};

constexpr int kGemmBM      = 128;
constexpr int kGemmBN      = 128;
constexpr int kGemmBK      = 16;
constexpr int kGemmThreads = 256;
constexpr int kGemmPad     = 4; // smem pitch = 132 elements: conflict-free fragment reads

template <typename T>
constexpr size_t gemm_smem_bytes()
{
    return 2ull * 2ull * kGemmBK * (kGemmBM + kGemmPad) * sizeof(T);
}

// Register staging for one 128 x 16 operand tile.  Logical element (o, k) -- o is the row
// of op(P) or the column of op(Q) -- is stored at ptr[r + c * ld] with
// (r, c) = kc ? (k, o) : (o, k); kc ("k contiguous") picks the thread mapping so that a
// warp always reads consecutive addresses.
template <typename T>
struct TileStage
{
    static constexpr int PER = kGemmBM * kGemmBK / kGemmThreads; // 8
    T v[PER];

    __device__ __forceinline__ void load(const T* ptr, int64_t ld, bool kc, int tri,
                                         int o0, int k0, int O, int K, int tid)
    {
#pragma unroll
        for(int i = 0; i < PER; ++i)
        {
            int o, kk;
            if(kc)
            {
                kk = tid % kGemmBK;
                o  = tid / kGemmBK + (kGemmThreads / kGemmBK) * i;
            }
            else
            {
                o  = tid % kGemmBM;
                kk = tid / kGemmBM + (kGemmThreads / kGemmBM) * i;
            }
            const int go = o0 + o, gk = k0 + kk;
            T         x  = T(0);
            if(go < O && gk < K)
            {
                const int64_t r = kc ? gk : go, c = kc ? go : gk;
                if(tri_keep(tri, r, c))
                    x = ptr[r + c * ld];
            }
            v[i] = x;
        }
    }

    __device__ __forceinline__ void store(T* s, bool kc, int tid) const
    {
#pragma unroll
        for(int i = 0; i < PER; ++i)
        {
            int o, kk;
            if(kc)
            {
                kk = tid % kGemmBK;
                o  = tid / kGemmBK + (kGemmThreads / kGemmBK) * i;
            }
            else
            {
                o  = tid % kGemmBM;
                kk = tid / kGemmBM + (kGemmThreads / kGemmBM) * i;
            }
            s[kk * (kGemmBM + kGemmPad) + o] = v[i];
        }
    }
};

__device__ __forceinline__ void dmma_8x8x4(double (&d)[2], double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

template <typename T>
struct GemmAcc;

// FP64: 8 warps as 2 (M) x 4 (N); warp tile 64 x 32 = 8 x 4 DMMA tiles of 8 x 8.
template <>
struct GemmAcc<double>
{
    double acc[8][4][2];

    __device__ __forceinline__ void zero()
    {
#pragma unroll
        for(int i = 0; i < 8; ++i)
#pragma unroll
            for(int j = 0; j < 4; ++j)
                acc[i][j][0] = acc[i][j][1] = 0.0;
    }

    __device__ __forceinline__ void mac(const double* As, const double* Bs, int tid)
    {
        const int lane = tid & 31, warp = tid >> 5;
        const int wm = warp & 1, wn = warp >> 1;
        const int lr = lane >> 2, lk = lane & 3;
#pragma unroll
        for(int ks = 0; ks < kGemmBK / 4; ++ks)
        {
            double a[8], b[4];
            const double* ap = As + (ks * 4 + lk) * (kGemmBM + kGemmPad) + wm * 64 + lr;
            const double* bp = Bs + (ks * 4 + lk) * (kGemmBN + kGemmPad) + wn * 32 + lr;
#pragma unroll
            for(int i = 0; i < 8; ++i)
                a[i] = ap[i * 8];
#pragma unroll
            for(int j = 0; j < 4; ++j)
                b[j] = bp[j * 8];
#pragma unroll
            for(int i = 0; i < 8; ++i)
#pragma unroll
                for(int j = 0; j < 4; ++j)
                    dmma_8x8x4(acc[i][j], a[i], b[j]);
        }
    }

    template <typename F>
    __device__ __forceinline__ void for_each(int tid, F&& f) const
    {
        const int lane = tid & 31, warp = tid >> 5;
        const int wm = warp & 1, wn = warp >> 1;
#pragma unroll
        for(int i = 0; i < 8; ++i)
#pragma unroll
            for(int j = 0; j < 4; ++j)
#pragma unroll
                for(int e = 0; e < 2; ++e)
                    f(wm * 64 + i * 8 + (lane >> 2), wn * 32 + j * 8 + (lane & 3) * 2 + e,
                      acc[i][j][e]);
    }
};

// FP32: 16 x 16 threads, each an 8 x 8 register tile split as 2 x 2 quads of 4 x 4
// (rows ty*4 and 64+ty*4, columns tx*4 and 64+tx*4) for conflict-free float4 reads.
template <>
struct GemmAcc<float>
{
    float acc[8][8];

    __device__ __forceinline__ void zero()
    {
#pragma unroll
        for(int i = 0; i < 8; ++i)
#pragma unroll
            for(int j = 0; j < 8; ++j)
                acc[i][j] = 0.f;
    }

    __device__ __forceinline__ void mac(const float* As, const float* Bs, int tid)
    {
        const int tx = tid & 15, ty = tid >> 4;
#pragma unroll
        for(int kk = 0; kk < kGemmBK; ++kk)
        {
            const float* ap = As + kk * (kGemmBM + kGemmPad);
            const float* bp = Bs + kk * (kGemmBN + kGemmPad);
            float4 a0 = *reinterpret_cast<const float4*>(ap + ty * 4);
            float4 a1 = *reinterpret_cast<const float4*>(ap + 64 + ty * 4);
            float4 b0 = *reinterpret_cast<const float4*>(bp + tx * 4);
            float4 b1 = *reinterpret_cast<const float4*>(bp + 64 + tx * 4);
            float a[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
            float b[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
            for(int i = 0; i < 8; ++i)
#pragma unroll
                for(int j = 0; j < 8; ++j)
                    acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
    }

    template <typename F>
    __device__ __forceinline__ void for_each(int tid, F&& f) const
    {
        const int tx = tid & 15, ty = tid >> 4;
#pragma unroll
        for(int i = 0; i < 8; ++i)
#pragma unroll
            for(int j = 0; j < 8; ++j)
                f((i < 4 ? ty * 4 + i : 64 + ty * 4 + i - 4),
                  (j < 4 ? tx * 4 + j : 64 + tx * 4 + j - 4), acc[i][j]);
    }
};

template <typename T>
__global__ void __launch_bounds__(kGemmThreads) gemm_tile_kernel(GemmParams<T> p)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* As = reinterpret_cast<T*>(smem_raw);                       // [2][BK][BM+PAD]
    T* Bs = As + 2 * kGemmBK * (kGemmBM + kGemmPad);              // [2][BK][BN+PAD]

    const int tid   = threadIdx.x;
    const int m0    = blockIdx.x * kGemmBM;
    const int n0    = blockIdx.y * kGemmBN;
    const int batch = p.batch_base + blockIdx.z;

    T*       C = p.C.get(batch);
    const T  ua = (p.zero_guard || p.a_user || p.b_user) ? p.ualpha.get() : T(1);
    const bool zero_out = p.zero_guard && ua == T(0);
    const T  a = p.a_user ? ua : p.a_imm;
    const T  b = p.b_user ? ua : p.b_imm;

    GemmAcc<T> acc;
    acc.zero();

    if(!zero_out)
    {
        const T* P = p.P.get(batch);
        const T* Q = p.Q.get(batch);
        // op(P) is M x K: logical (m, k); stored (m, k) when transP == 0 -> k not contiguous
        const bool kcP = p.transP != 0;
        // op(Q) is K x N: logical (n, k) in loader terms; stored (k, n) when transQ == 0
        const bool kcQ = p.transQ == 0;

        TileStage<T> sp, sq;
        const int    nk = (p.K + kGemmBK - 1) / kGemmBK;
        sp.load(P, p.ldp, kcP, p.triP, m0, 0, p.M, p.K, tid);
        sq.load(Q, p.ldq, kcQ, p.triQ, n0, 0, p.N, p.K, tid);
        sp.store(As, kcP, tid);
        sq.store(Bs, kcQ, tid);
        __syncthreads();

        for(int kt = 0; kt < nk; ++kt)
        {
            const int cur = kt & 1;
            if(kt + 1 < nk)
            {
                sp.load(P, p.ldp, kcP, p.triP, m0, (kt + 1) * kGemmBK, p.M, p.K, tid);
                sq.load(Q, p.ldq, kcQ, p.triQ, n0, (kt + 1) * kGemmBK, p.N, p.K, tid);
            }
            acc.mac(As + cur * kGemmBK * (kGemmBM + kGemmPad),
                    Bs + cur * kGemmBK * (kGemmBN + kGemmPad), tid);
            if(kt + 1 < nk)
            {
                sp.store(As + (cur ^ 1) * kGemmBK * (kGemmBM + kGemmPad), kcP, tid);
                sq.store(Bs + (cur ^ 1) * kGemmBK * (kGemmBN + kGemmPad), kcQ, tid);
            }
            __syncthreads();
        }
    }

    const int64_t ldc = p.ldc;
    const int     M = p.M, N = p.N;
    acc.for_each(tid, [&](int r, int c, T v) {
        const int gr = m0 + r, gc = n0 + c;
        if(gr < M && gc < N)
        {
            T* cp = C + gr + (int64_t)gc * ldc;
            T  out;
            if(zero_out)
                out = T(0);
            else if(b == T(0))
                out = a * v;
            else
                out = a * v + b * (*cp);
            *cp = out;
        }
    });
}

} // namespace rb200
