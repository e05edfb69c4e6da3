// Complex GEMM tiles on the FP64 DMMA tensor path (the complex trsm's trailing updates and the
// complex trmm):
//
//     C := a * op(P) * op(Q) + b * C      GemmParams<cplx<R>>, R = float or double
//
// A complex product is a real one of twice the size.  Write each entry p of op(P) as the real
// 2 x 2 block [[pr, -pi], [pi, pr]] and each entry q of op(Q) as the column [qr; qi]: the real
// product of the blocked matrices is the column [Re; Im] of sum_k p q.  One mma.sync m16n8k8
// .f64 then covers 8 complex rows x 8 complex columns x 4 complex k, 1024 real FMAs, the full
// DMMA rate: inside an MMA tile real rows 0-7 are the real parts of 8 complex rows of C and
// rows 8-15 their imaginary parts; real k 0-3 multiply qr and 4-7 multiply qi.  With
// g = lane / 4 and t = lane % 4 the fragments are
//     a = {pr, pi, -pi, pr}      of p = op(P)(g, t)
//     b = {qr, qi}               of q = op(Q)(t, g)
//     c = {Re C(g, 2t), Re C(g, 2t+1), Im C(g, 2t), Im C(g, 2t+1)}
// so a thread reads one complex value of each operand per MMA, and holds the real and
// imaginary parts of its outputs together for the complex epilogue.
//
// Operands are staged in shared memory as stored (cplx<R>) by cp.async copies of one
// component each (the rocblas complex structs are only component-aligned), in the orientation
// that keeps the copies coalesced, and converted to double at fragment load: complex float is
// computed in FP64 and rounded once.  Pitches keep the fragment reads free of bank conflicts.
#pragma once
#include "gemm_dmma.cuh"

namespace rb200
{

__device__ __forceinline__ void cp_async_4(void* smem, const void* gmem, bool valid)
{
    const uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
    const int      n = valid ? 4 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(s), "l"(gmem), "r"(n) : "memory");
}

template <typename R, int BM, int BN, int WM, int WN, int STAGES, bool KCP, bool KCQ, int BK>
struct CdmmaCfg
{
    static constexpr int kWarpsM  = BM / WM;
    static constexpr int kWarpsN  = BN / WN;
    static constexpr int kThreads = kWarpsM * kWarpsN * 32;
    // [o][k] (k contiguous): pitch BK + 4; [k][o]: O + 2 (16-byte elements) or O + 4 (8-byte)
    static constexpr int kPadO    = sizeof(R) == 8 ? 2 : 4;
    static constexpr int kPitchA  = KCP ? (BK + 4) : (BM + kPadO);
    static constexpr int kPitchB  = KCQ ? (BK + 4) : (BN + kPadO);
    static constexpr int kStageA  = KCP ? BM * kPitchA : BK * kPitchA; // elements
    static constexpr int kStageB  = KCQ ? BN * kPitchB : BK * kPitchB;
    static constexpr int kStage   = kStageA + kStageB;
    static constexpr size_t kSmem = (size_t)STAGES * kStage * sizeof(cplx<R>);
};

// One BK-deep stage of an operand tile of O rows: logical (o, k) is stored at
// ptr[r + c * ld] with (r, c) = kc ? (k, o) : (o, k); one cp.async per component.
template <typename R, int O, int NT, bool KC, int BK, int PITCH>
__device__ __forceinline__ void cdmma_load_stage(cplx<R>* s, const cplx<R>* ptr, int64_t ld, int tri,
                                                 int o0, int k0, int Olim, int Klim, int tid)
{
    constexpr int PER = 2 * O * BK / NT;
    static_assert(PER * NT == 2 * O * BK, "tile / thread mismatch");
#pragma unroll
    for(int i = 0; i < PER; ++i)
    {
        const int e = tid + i * NT, comp = e & 1, e2 = e >> 1;
        int       o, kk;
        if(KC)
        {
            kk = e2 % BK;
            o  = e2 / BK;
        }
        else
        {
            o  = e2 % O;
            kk = e2 / O;
        }
        const int     go = o0 + o, gk = k0 + kk;
        const int64_t r = KC ? gk : go, c = KC ? go : gk;
        const bool    valid = go < Olim && gk < Klim && tri_keep(tri, r, c);
        const R*      src   = valid ? &ptr[r + c * ld].x + comp : &ptr->x;
        R*            dst   = &(KC ? s[o * PITCH + kk] : s[kk * PITCH + o]).x + comp;
        if constexpr(sizeof(R) == 8)
            cp_async_8(dst, src, valid);
        else
            cp_async_4(dst, src, valid);
    }
}

template <typename R, int BM, int BN, int WM, int WN, int STAGES, bool KCP, bool KCQ, int BK>
__global__ void __launch_bounds__(CdmmaCfg<R, BM, BN, WM, WN, STAGES, KCP, KCQ, BK>::kThreads)
    gemm_cdmma_kernel(GemmParams<cplx<R>> p)
{
    using Cfg = CdmmaCfg<R, BM, BN, WM, WN, STAGES, KCP, KCQ, BK>;
    using T   = cplx<R>;
    using Z   = cplx<double>;
    constexpr int NT = Cfg::kThreads;
    constexpr int TM = WM / 8, TN = WN / 8;
    static_assert(BK % 4 == 0, "an MMA consumes 4 complex k");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* smem = reinterpret_cast<T*>(smem_raw);

    const int tid   = threadIdx.x;
    const int lane  = tid & 31, warp = tid >> 5;
    const int wm    = warp % Cfg::kWarpsM, wn = warp / Cfg::kWarpsM;
    const int m0    = blockIdx.x * BM;
    const int n0    = blockIdx.y * BN;
    const int batch = p.batch_base + blockIdx.z;

    T*        C  = p.C.get(batch);
    const T   ua = (p.zero_guard || p.a_user || p.b_user) ? p.ualpha.get() : T(1);
    const bool zero_out = p.zero_guard && ua == T(0);
    const T   ta = p.a_user ? ua : p.a_imm;
    const T   tb = p.b_user ? ua : p.b_imm;
    const Z   a(ta.x, ta.y), b(tb.x, tb.y);

    double acc[TM][TN][4];
#pragma unroll
    for(int i = 0; i < TM; ++i)
#pragma unroll
        for(int j = 0; j < TN; ++j)
#pragma unroll
            for(int e = 0; e < 4; ++e)
                acc[i][j][e] = 0.0;

    const int g = lane >> 2, t = lane & 3;
    if(!zero_out)
    {
        const T*  P  = p.P.get(batch);
        const T*  Q  = p.Q.get(batch);
        const int nk = (p.K + BK - 1) / BK;
        auto load = [&](int stage, int kt) {
            T* sA = smem + stage * Cfg::kStage;
            T* sB = sA + Cfg::kStageA;
            cdmma_load_stage<R, BM, NT, KCP, BK, Cfg::kPitchA>(sA, P, p.ldp, p.triP, m0, kt * BK, p.M,
                                                               p.K, tid);
            cdmma_load_stage<R, BN, NT, KCQ, BK, Cfg::kPitchB>(sB, Q, p.ldq, p.triQ, n0, kt * BK, p.N,
                                                               p.K, tid);
        };
        auto ldA = [&](const T* sA, int m, int k) {
            return KCP ? sA[m * Cfg::kPitchA + k] : sA[k * Cfg::kPitchA + m];
        };
        auto ldB = [&](const T* sB, int n, int k) {
            return KCQ ? sB[n * Cfg::kPitchB + k] : sB[k * Cfg::kPitchB + n];
        };
        const double sgnP = p.conjP ? -1.0 : 1.0, sgnQ = p.conjQ ? -1.0 : 1.0;
#pragma unroll
        for(int s = 0; s < STAGES - 1; ++s)
        {
            if(s < nk)
                load(s, s);
            cp_async_commit();
        }
        for(int kt = 0; kt < nk; ++kt)
        {
            cp_async_wait<STAGES - 2>();
            __syncthreads();
            const T* sA = smem + (kt % STAGES) * Cfg::kStage;
            const T* sB = sA + Cfg::kStageA;
#pragma unroll
            for(int ks = 0; ks < BK / 4; ++ks)
            {
                const int k = ks * 4 + t;
                double    fa[TM][4], fb[TN][2];
#pragma unroll
                for(int i = 0; i < TM; ++i)
                {
                    const T      v  = ldA(sA, wm * WM + i * 8 + g, k);
                    const double pr = (double)v.x, pi = sgnP * (double)v.y;
                    fa[i][0] = pr;
                    fa[i][1] = pi;
                    fa[i][2] = -pi;
                    fa[i][3] = pr;
                }
#pragma unroll
                for(int j = 0; j < TN; ++j)
                {
                    const T v = ldB(sB, wn * WN + j * 8 + g, k);
                    fb[j][0]  = (double)v.x;
                    fb[j][1]  = sgnQ * (double)v.y;
                }
#pragma unroll
                for(int i = 0; i < TM; ++i)
#pragma unroll
                    for(int j = 0; j < TN; ++j)
                        dmma_16x8x8(acc[i][j], fa[i], fb[j]);
            }
            const int nxt = kt + STAGES - 1;
            if(nxt < nk)
                load(nxt % STAGES, nxt);
            cp_async_commit();
        }
        cp_async_wait<0>();
    }

    const int64_t ldc = p.ldc;
#pragma unroll
    for(int i = 0; i < TM; ++i)
#pragma unroll
        for(int j = 0; j < TN; ++j)
#pragma unroll
            for(int e = 0; e < 2; ++e)
            {
                const int gr = m0 + wm * WM + i * 8 + g;
                const int gc = n0 + wn * WN + j * 8 + 2 * t + e;
                if(gr < p.M && gc < p.N)
                {
                    T* cp = C + gr + (int64_t)gc * ldc;
                    Z  out(0.0, 0.0);
                    if(!zero_out)
                    {
                        out = a * Z(acc[i][j][e], acc[i][j][2 + e]);
                        if(b != Z(0.0))
                        {
                            const T old = *cp;
                            out += b * Z((double)old.x, (double)old.y);
                        }
                    }
                    *cp = T((R)out.x, (R)out.y);
                }
            }
}

template <typename R, int BM, int BN, int WM, int WN, int STAGES, bool KCP, bool KCQ, int BK>
static void launch_cdmma_cfg(const GemmParams<cplx<R>>& p0, int batch, cudaStream_t s)
{
    using Cfg = CdmmaCfg<R, BM, BN, WM, WN, STAGES, KCP, KCQ, BK>;
    auto kern = gemm_cdmma_kernel<R, BM, BN, WM, WN, STAGES, KCP, KCQ, BK>;
    cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg::kSmem);
    for(int b0 = 0; b0 < batch; b0 += 65535)
    {
        GemmParams<cplx<R>> p = p0;
        p.batch_base = b0;
        dim3 grid((unsigned)ceil_div(p.M, BM), (unsigned)ceil_div(p.N, BN),
                  (unsigned)std::min(65535, batch - b0));
        // work in real FP64 flops: 8 per complex multiply-add
        TimedLaunch tl(KernelClass::dmma, s, 8.0 * p.M * p.N * p.K * grid.z);
        kern<<<grid, Cfg::kThreads, Cfg::kSmem, s>>>(p);
    }
}

// 64 x 64 complex tiles (8 warps of 16 x 32) when they give every SM work, else 32 x 32
// (4 warps of 16 x 16).
template <typename R, bool KCP, bool KCQ>
static void launch_cdmma_tile(const GemmParams<cplx<R>>& p, int batch, cudaStream_t s, int sms)
{
    const int64_t tiles64 = ceil_div(p.M, 64) * ceil_div(p.N, 64) * batch;
    if(tiles64 >= sms)
        launch_cdmma_cfg<R, 64, 64, 16, 32, 4, KCP, KCQ, 8>(p, batch, s);
    else
        launch_cdmma_cfg<R, 32, 32, 16, 16, 4, KCP, KCQ, 8>(p, batch, s);
}

template <typename R>
static void launch_gemm_cdmma(const GemmParams<cplx<R>>& p, int batch, cudaStream_t s, int sms)
{
    if(p.M <= 0 || p.N <= 0)
        return;
    const bool kcP = p.transP != 0, kcQ = p.transQ == 0;
    if(kcP && kcQ)
        launch_cdmma_tile<R, true, true>(p, batch, s, sms);
    else if(kcP)
        launch_cdmma_tile<R, true, false>(p, batch, s, sms);
    else if(kcQ)
        launch_cdmma_tile<R, false, true>(p, batch, s, sms);
    else
        launch_cdmma_tile<R, false, false>(p, batch, s, sms);
}

} // namespace rb200
