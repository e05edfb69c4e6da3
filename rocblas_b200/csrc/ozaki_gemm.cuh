// FP64-accurate GEMM update on the Blackwell tensor cores from exact integer slices.
//
//     C := beta * C + alpha * P * Q            (P: M x K, Q: K x N, C: M x N, FP64)
//
// Used for the trailing updates of the blocked solve: by the precision form of the dtrsm when
// a slice count is asked for, or for updates with fewer output tiles than SMs (the residue
// engine of crt_gemm.cuh takes the others), and by the FP32 trsm with FP32 operands and C (4
// slices); the refinement's FP64 residuals run on the DMMA tiles, gemm_dmma.cuh.  The reference
// computes these updates with FP64 / FP32 GEMMs (rocblas_internal_gemm -> Tensile,
// library/src/blas3/Tensile/gemm_templates.cpp:41-181).
//
// Method (a multi-limb split in the style of Ozaki's error-free matrix product):
//   * every row r of P is scaled by 2^-e_r (e_r = exponent of its largest entry) and cut into
//     S slices of 7 bits: P(r,k) = 2^e_r * sum_s p_s(r,k) 2^-7(s+1) + tail, |p_s| <= 127,
//     stored as int8; every column c of Q the same way with exponents f_c;
//   * the slice products G_d = sum_{s+t=d} p_s q_t (d < S) are computed on the tensor cores
//     with tcgen05.mma kind::i8.  Every product is exact and the int32 accumulation in TMEM
//     is exact while (d+1) * K * 127^2 < 2^31 (K <= 16640 for S = 8); longer K is split;
//   * the epilogue combines P Q ~= 2^(e_r+f_c) * 2^-14 * sum_d 2^-7d G_d in FP64.
// Each entry is represented to 2^-7S relative to its row's (column's) largest entry, and the
// dropped slice pairs (s + t >= S) add about S * 2^-7(S+1) of 2^(e_r+f_c): S = 7 gives 49
// bits, S = 8 gives 56 bits (beyond FP64 rounding of a K-term dot product).
//
// Kernel layout (one CTA per 128 x BN output tile, BN = 64 or 128, 192 threads):
//   warp 0   copy producer: per BK-deep K step (BK = 32 or 64 int8) it brings the slices the
//            pass needs of the P tile (128 x BK) and of the Q tile (BN x BK) into one stage of
//            a ring.  The slicing kernel writes every slice as K panels of BK-byte rows that
//            are already in the tensor cores' swizzled shared-memory order (SWIZZLE_32B /
//            _64B), so each tile is one contiguous block and one bulk copy
//            (cp.async.bulk ... complete_tx) per tile replaces a row-by-row tensor copy;
//   warp 1   TMEM owner and MMA issuer: one 128 x BN int32 accumulator per slice-pair group
//            d = s + t of the pass, group d at TMEM column (d - d_lo) * BN.  The Q slices of
//            a stage sit back to back, so Q slices t0..t0+c-1 form one (c * BN)-row operand and
//            a single MMA with N = c * BN <= 256 computes the products of P slice s with all
//            of them into the adjacent accumulators of groups s+t0 .. s+t0+c-1: per K step
//            and P slice one to two MMAs instead of one per slice pair, and the P tile is read
//            from shared memory once per MMA instead of once per pair.  With BN = 64 all
//            S <= 8 groups fit the 512 TMEM columns in one pass; with BN = 128 and S > 4 the
//            groups are split into two passes (d < 4, then d >= 4; the second adds onto C);
//   warps 2-5 epilogue: tcgen05.ld of the accumulators (lanes = rows), Horner combination in
//            FP64 registers, scaling by the row/column exponents, beta * C + alpha * (...).
// Every mbarrier wait is bounded; on timeout the kernel records the error, drains its
// in-flight copies and MMAs (again bounded), frees TMEM and returns.
#pragma once
#include <cstdint>

#include "common.cuh"

namespace rb200
{

constexpr int kOzBM      = 128;
constexpr int kOzMaxS    = 8;
constexpr int kOzThreads = 192;
constexpr int kOzMmaK    = 32;            // int8 K of one tcgen05.mma
constexpr int kOzMaxN    = 256;           // largest N of one tcgen05.mma with M = 128
constexpr int kOzKMax    = 16384;         // longest exact int32 accumulation run (S <= 8)
constexpr int kOzSmemBudget = 226 * 1024;
constexpr int kOzNPad    = 128;           // row padding of the Q slice buffers
constexpr int kOzExpNone    = -(1 << 30); // exponent of an all-zero row / column

struct OzParams
{
    int      M, N, K;          // logical sizes
    int      S;                // slices (1..8)
    int      d_lo, d_hi;       // slice-pair groups d = s + t computed by this pass
    int      ns;               // slices staged per operand: min(S, d_hi)
    int      M_pad, N_pad;     // slice-buffer row counts (multiples of 128)
    const int8_t* sliceP;      // S panels sets of P: [s][K / BK][M_pad][BK], swizzled rows
    const int8_t* sliceQ;      // the same for Q with N_pad rows
    int      nkc;              // K panels per slice (K_pad / BK)
    const int* exp_rows;       // e_r, M entries
    const int* exp_cols;       // f_c, N entries
    void*    C;                // output (column-major, ldc): double, or float if c_f32
    int64_t  ldc;
    double   alpha, beta;      // C := beta C + alpha P Q ; beta == 0 => C not read
    const void* beta_ptr;      // if set, beta := *beta_ptr (device pointer mode alpha of a trsm;
                               // the element type of C)
    const void* ualpha_ptr;    // if set and *ualpha_ptr == 0: C := 0 (a trsm with alpha == 0)
    int      c_f32;            // C, beta_ptr, ualpha_ptr are float (the FP32 trsm's updates)
    int      ualpha_zero;      // host-side form of the same condition
    int      stages;
    int      tmem_cols;        // power of two >= S * 64
    int*     error;            // set to a nonzero code if a wait timed out
};

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(smem_u32(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}

// Bounded wait: ~2^31 cycles (about a second at boost clock).  Returns false on timeout.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity)
{
    const long long t0 = clock64();
    while(!mbar_try_wait(bar, parity))
    {
        if(clock64() - t0 > (1ll << 31))
            return false;
    }
    return true;
}

// Contiguous global -> shared copy of `bytes` (multiple of 16, both addresses 16-byte
// aligned) that completes on `bar` (transaction count).
__device__ __forceinline__ void bulk_load(void* smem_dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(smem_dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// UMMA shared-memory descriptor: K-major operand with BK-byte rows (BK = 64: SWIZZLE_64B,
// BK = 32: SWIZZLE_32B), 8-row groups 8 * BK bytes apart.
template <int BK>
__device__ __forceinline__ uint64_t oz_smem_desc(uint32_t saddr)
{
    static_assert(BK == 32 || BK == 64, "swizzle span of one K step");
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);       // start address
    d |= (uint64_t)1 << 16;                       // leading byte offset (unused, 16 B)
    d |= (uint64_t)((8 * BK) >> 4) << 32;         // stride byte offset: 8 rows x BK bytes
    d |= (uint64_t)1 << 46;                       // descriptor version (sm_100)
    d |= (uint64_t)(BK == 64 ? 4 : 6) << 61;      // SWIZZLE_64B / SWIZZLE_32B
    return d;
}

// Instruction descriptor, kind::i8: s8 x s8 -> s32, K-major A and B, M = 128, N = n.
__host__ __device__ constexpr uint32_t oz_idesc(int n)
{
    return (2u << 4)                      // D format S32
           | (1u << 7)                    // A format signed int8
           | (1u << 10)                   // B format signed int8
           | ((uint32_t)(n >> 3) << 17)
           | ((uint32_t)(kOzBM >> 4) << 24);
}

__device__ __forceinline__ void oz_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                       uint32_t idesc, uint32_t accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
                 "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

// A scalar of C's element type from device memory, as a double (`dflt` when ptr is null).
__device__ __forceinline__ double oz_read_scalar(const void* ptr, int f32, double dflt)
{
    if(!ptr)
        return dflt;
    return f32 ? (double)*static_cast<const float*>(ptr) : *static_cast<const double*>(ptr);
}

__device__ __forceinline__ void oz_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld_32x32b_x32(uint32_t taddr, uint32_t (&v)[32])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
                 "%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
                   "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
                   "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]),
                   "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
                   "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]),
                   "=r"(v[30]), "=r"(v[31])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Persistent over output tiles: grid = min(tiles, SMs), tile t = blockIdx.x + i * gridDim.x in
// a grouped order (kOzGroupM row tiles side by side, then the next columns) so that the tiles
// in flight share their P and Q slice tiles in L2.  The copy ring runs across tile
// boundaries; the MMA warp starts a tile once the epilogue has drained the previous tile's
// accumulators (tmem_empty), and with BN = 64 the epilogue drains TMEM into registers first,
// releases it, and only then reads and writes C, so the C traffic of one tile overlaps the
// MMAs of the next.
//
// SC > 0: a single pass over all SC slices (d_lo = 0, d_hi = SC) with the slice count known
// at compile time, so the MMA and copy schedules unroll into straight-line code; SC = 0: the
// pass and slice count come from p at run time.
constexpr int kOzGroupM = 8;

__device__ __forceinline__ void oz_tile_coords(int t, int tiles_m, int tiles_n, int& mt, int& nt)
{
    const int per_group = kOzGroupM * tiles_n;
    const int grp = t / per_group, r = t - grp * per_group;
    const int gm  = min(kOzGroupM, tiles_m - grp * kOzGroupM); // rows in this group
    mt = grp * kOzGroupM + r % gm;
    nt = r / gm;
}

template <int BN, int BK, int SC>
__global__ void __launch_bounds__(kOzThreads, 1)
    ozaki_gemm_kernel(const __grid_constant__ OzParams p)
{
    constexpr int  kTileA = kOzBM * BK; // bytes per slice tile of P
    constexpr int  kTileB = BN * BK;    // bytes per slice tile of Q
    constexpr int  kMerge = kOzMaxN / BN; // Q slices per MMA
    constexpr bool kEarlyRelease = BN == 64; // drain TMEM to registers before touching C
    extern __shared__ __align__(1024) unsigned char oz_smem_raw[];
    // 1 KB alignment for the swizzled tiles
    unsigned char* smem = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(oz_smem_raw) + 1023) & ~uintptr_t(1023));
    const int S   = SC > 0 ? SC : p.ns; // slices staged per operand in this pass
    const int DLO = SC > 0 ? 0 : p.d_lo;
    const int DHI = SC > 0 ? SC : p.d_hi;
    const int stage_bytes = S * (kTileA + kTileB);
    const int NS        = p.stages;

    __shared__ uint64_t full_bar[8], empty_bar[8], tmem_full, tmem_empty;
    __shared__ uint32_t tmem_base_sh;
    __shared__ int      abort_flag;
    __shared__ int      issued, consumed; // K steps loaded / handed to the tensor cores

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nk      = (p.K + BK - 1) / BK;
    const int tiles_m = p.M_pad / kOzBM;
    const int tiles_n = (p.N + BN - 1) / BN;
    const int tiles   = tiles_m * tiles_n;

    if(threadIdx.x == 0)
    {
        for(int i = 0; i < NS; ++i)
        {
            mbar_init(&full_bar[i], 1);
            mbar_init(&empty_bar[i], 1);
        }
        mbar_init(&tmem_full, 1);
        mbar_init(&tmem_empty, 4); // one arrival per epilogue warp
        abort_flag = 0;
        issued     = 0;
        consumed   = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if(warp == 1)
    {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_base_sh)),
                     "r"(p.tmem_cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_base_sh;

    if(warp == 0)
    {
        // ---------------- copy producer ----------------
        if(lane == 0)
        {
            const int64_t slP = (int64_t)p.nkc * p.M_pad * BK, slQ = (int64_t)p.nkc * p.N_pad * BK;
            int it = 0; // K steps issued over all tiles
            for(int tile = blockIdx.x; tile < tiles && !*(volatile int*)&abort_flag; tile += gridDim.x)
            {
                int mt, nt;
                oz_tile_coords(tile, tiles_m, tiles_n, mt, nt);
                const int m0 = mt * kOzBM, n0 = nt * BN;
                for(int i = 0; i < nk; ++i, ++it)
                {
                    const int st = it % NS;
                    const uint32_t ph = (uint32_t)((it / NS) & 1);
                    if(!mbar_wait_bounded(&empty_bar[st], ph ^ 1))
                    {
                        atomicExch(p.error, 1);
                        atomicExch(&abort_flag, 1);
                        break;
                    }
                    if(*(volatile int*)&abort_flag)
                        break;
                    unsigned char* base = smem + st * stage_bytes;
                    mbar_expect_tx(&full_bar[st], (uint32_t)stage_bytes);
                    // slice s, K panel i: rows at ((s * nkc + i) * rows_pad + row) * BK
                    const int8_t* srcP = p.sliceP + ((int64_t)i * p.M_pad + m0) * BK;
                    const int8_t* srcQ = p.sliceQ + ((int64_t)i * p.N_pad + n0) * BK;
#pragma unroll
                    for(int s = 0; s < S; ++s)
                        bulk_load(base + s * kTileA, srcP + s * slP, kTileA, &full_bar[st]);
#pragma unroll
                    for(int t = 0; t < S; ++t)
                        bulk_load(base + S * kTileA + t * kTileB, srcQ + t * slQ, kTileB, &full_bar[st]);
                    *(volatile int*)&issued = it + 1;
                }
            }
        }
    }
    else if(warp == 1)
    {
        // ---------------- MMA issuer ----------------
        if(lane == 0)
        {
            // descriptors of stage 0's first P and Q tiles; every other tile is a constant
            // offset (start address field = byte address / 16, no carry out of its 14 bits)
            const uint64_t desc_a0 = oz_smem_desc<BK>(smem_u32(smem));
            const uint64_t desc_b0 = oz_smem_desc<BK>(smem_u32(smem) + S * kTileA);
            int it = 0, tcount = 0;
            bool ok = true;
            for(int tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x, ++tcount)
            {
                // the epilogue has drained the previous tile's accumulators
                if(!mbar_wait_bounded(&tmem_empty, (uint32_t)((tcount & 1) ^ 1)))
                {
                    atomicExch(p.error, 2);
                    atomicExch(&abort_flag, 1);
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;");
                for(int i = 0; i < nk; ++i, ++it)
                {
                    const int st = it % NS;
                    const uint32_t ph = (uint32_t)((it / NS) & 1);
                    if(!mbar_wait_bounded(&full_bar[st], ph) || *(volatile int*)&abort_flag)
                    {
                        atomicExch(p.error, 2);
                        atomicExch(&abort_flag, 1);
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;");
                    *(volatile int*)&consumed = it + 1;
                    const uint64_t soff = (uint64_t)((st * stage_bytes) >> 4);
                    // P slice 0 comes first in every K step and covers every group of the
                    // pass, so only its first MMA of a tile's first K step starts the
                    // accumulators
                    const uint32_t acc0 = i > 0 ? 1u : 0u;
#pragma unroll
                    for(int s = 0; s < S; ++s)
                    {
                        // Q slices t with d_lo <= s + t < d_hi, in runs of at most kMerge
                        const int t_lo = max(0, DLO - s), t_hi = min(S - 1, DHI - 1 - s);
#pragma unroll
                        for(int t0 = t_lo; t0 <= t_hi; t0 += kMerge)
                        {
                            const int      c     = min(kMerge, t_hi - t0 + 1);
                            const uint32_t dcol  = tmem + (uint32_t)((s + t0 - DLO) * BN);
                            const uint32_t idesc = oz_idesc(c * BN);
#pragma unroll
                            for(int kk = 0; kk < BK / kOzMmaK; ++kk)
                            {
                                const uint64_t ad = desc_a0 + soff + (uint64_t)((s * kTileA + kk * kOzMmaK) >> 4);
                                const uint64_t bd = desc_b0 + soff + (uint64_t)((t0 * kTileB + kk * kOzMmaK) >> 4);
                                oz_mma(dcol, ad, bd, idesc, (s == 0 && kk == 0) ? acc0 : 1u);
                            }
                        }
                    }
                    oz_commit(&empty_bar[st]);
                }
                // the tile's accumulators are complete when its MMAs are (also on abort:
                // drains what was issued)
                oz_commit(&tmem_full);
            }
        }
    }
    else
    {
        // ---------------- epilogue (warps 2..5) ----------------
        const int      quarter   = warp & 3; // TMEM lane group this warp may access
        const int      row       = quarter * 32 + lane;
        const uint32_t lane_addr = tmem + ((uint32_t)(quarter * 32) << 16);
        const double   beta      = oz_read_scalar(p.beta_ptr, p.c_f32, p.beta);
        const bool     zero      = p.ualpha_zero || (p.ualpha_ptr && oz_read_scalar(p.ualpha_ptr, p.c_f32, 1.0) == 0.0);
        int            tcount    = 0;
        for(int tile = blockIdx.x; tile < tiles; tile += gridDim.x, ++tcount)
        {
            int mt, nt;
            oz_tile_coords(tile, tiles_m, tiles_n, mt, nt);
            const int m0 = mt * kOzBM, n0 = nt * BN;
            const int gr = m0 + row;
            // warp-uniform outcome: the tcgen05.ld below needs the whole warp
            bool ok = __all_sync(0xffffffffu, mbar_wait_bounded(&tmem_full, (uint32_t)(tcount & 1)));
            if(!ok)
            {
                atomicExch(p.error, 3);
                atomicExch(&abort_flag, 1);
            }
            asm volatile("tcgen05.fence::after_thread_sync;");
            if(!__all_sync(0xffffffffu, ok && !*(volatile int*)&abort_flag))
                break;
            int er = gr < p.M ? p.exp_rows[gr] : 0;
            if(er == kOzExpNone)
                er = 0;
            auto store = [&](const double (&h)[32], int half) {
                if(gr >= p.M)
                    return;
#pragma unroll
                for(int j = 0; j < 32; ++j)
                {
                    const int gc = n0 + half * 32 + j;
                    if(gc < p.N)
                    {
                        const int64_t ci = gr + (int64_t)gc * p.ldc;
                        const int     ec = p.exp_cols[gc] == kOzExpNone ? 0 : p.exp_cols[gc];
                        const double  pq = ldexp(h[j], er + ec - 14 - 7 * DLO);
                        double        out;
                        if(zero)
                            out = 0.0;
                        else if(beta == 0.0)
                            out = p.alpha * pq;
                        else
                            out = fma(p.alpha, pq,
                                      beta * (p.c_f32 ? (double)static_cast<float*>(p.C)[ci]
                                                      : static_cast<double*>(p.C)[ci]));
                        if(p.c_f32)
                            static_cast<float*>(p.C)[ci] = (float)out;
                        else
                            static_cast<double*>(p.C)[ci] = out;
                    }
                }
            };
            auto drain = [&](double (&h)[32], int half) {
#pragma unroll
                for(int j = 0; j < 32; ++j)
                    h[j] = 0.0;
#pragma unroll 1
                for(int d = DHI - 1; d >= DLO; --d)
                {
                    uint32_t v[32];
                    tmem_ld_32x32b_x32(lane_addr + (uint32_t)((d - DLO) * BN + half * 32), v);
#pragma unroll
                    for(int j = 0; j < 32; ++j)
                        h[j] = fma(h[j], 0x1p-7, (double)(int)v[j]);
                }
            };
            auto release = [&]() {
                asm volatile("tcgen05.fence::before_thread_sync;");
                __syncwarp();
                if(lane == 0)
                    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&tmem_empty))
                                 : "memory");
            };
            if constexpr(kEarlyRelease)
            {
                double h0[32], h1[32];
                drain(h0, 0);
                drain(h1, 1);
                release();
                store(h0, 0);
                store(h1, 1);
            }
            else
            {
#pragma unroll 1
                for(int half = 0; half < BN / 32; ++half)
                {
                    double h[32];
                    drain(h, half);
                    store(h, half);
                }
                release();
            }
        }
    }

    // ---------------- teardown ----------------
    __syncthreads();
    if(warp == 0 && lane == 0 && *(volatile int*)&abort_flag)
    {
        // let the copies that were issued but never consumed land before the CTA exits
        for(int i = consumed; i < issued; ++i)
            (void)mbar_wait_bounded(&full_bar[i % NS], (uint32_t)((i / NS) & 1));
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if(warp == 1)
    {
        asm volatile("tcgen05.fence::after_thread_sync;");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(p.tmem_cols));
    }
}

// ---- slicing ----------------------------------------------------------------------------
// Operand element (o, k) lives at src[o * so + k * sk].  exps[o] = 1 + exponent of max_k |x|,
// so that |x| * 2^-exps[o] < 1; rows that are all zero keep kOzExpNone and are sliced as 0.
// exps must be preset to kOzExpNone; partial maxima over K chunks are merged with atomicMax
// (the exponent is monotone in the maximum).
constexpr int kOzExpChunk = 256;

__device__ __forceinline__ void oz_merge_exp(int* exps, int o, double mx)
{
    if(mx > 0.0)
        atomicMax(&exps[o], ilogb(mx) + 1);
}

// one warp per row o and K chunk; lanes stride over k (rows whose k is contiguous)
template <typename TIn>
__global__ void oz_exponent_kernel(const TIn* src, int64_t so, int64_t sk, int O, int K, int* exps)
{
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    const int k0 = blockIdx.y * kOzExpChunk;
    if(w >= O)
        return;
    double    mx   = 0.0;
    const int kend = min(K, k0 + kOzExpChunk);
#pragma unroll 8
    for(int k = k0 + lane; k < kend; k += 32)
        mx = fmax(mx, fabs((double)src[(int64_t)w * so + (int64_t)k * sk]));
#pragma unroll
    for(int off = 16; off; off >>= 1)
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    if(lane == 0)
        oz_merge_exp(exps, w, mx);
}

// one thread per row o and K chunk of kOzExpRowsChunk, for operands whose rows are adjacent
// in memory (so == 1): consecutive threads read consecutive addresses.  The chunk is short so
// that the grid has enough threads to keep HBM busy (rows are few, K is long).
constexpr int kOzExpRowsChunk = 64;

template <typename TIn>
__global__ void oz_exponent_rows_kernel(const TIn* src, int64_t sk, int O, int K, int* exps)
{
    const int o  = blockIdx.x * blockDim.x + threadIdx.x;
    const int k0 = blockIdx.y * kOzExpRowsChunk;
    if(o >= O)
        return;
    // unrolled so that 16 loads are in flight per thread (the maximum does not depend on the
    // order it is taken in, so the exponents are the same)
    double    mx   = 0.0;
    const int kend = min(K, k0 + kOzExpRowsChunk);
#pragma unroll 16
    for(int k = k0; k < kend; ++k)
        mx = fmax(mx, fabs((double)src[o + (int64_t)k * sk]));
    oz_merge_exp(exps, o, mx);
}

// Slices: slice s of row o, k lives in the K panel kc = k / BK as dst[((s * K_pad / BK + kc)
// * O_pad + o) * BK + swizzled(k % BK)]: every panel is the row-major image of O_pad rows of
// BK bytes with the 16-byte chunks of row o permuted the way the tensor cores' shared-memory
// layout (SWIZZLE_64B for BK = 64, SWIZZLE_32B for BK = 32) expects, so a tile of whole
// 8-row groups copies verbatim into 1 KB-aligned shared memory.  Rows o >= O and columns
// k >= K are written as zero.  A 64 x 64 tile goes through shared memory so that both the
// double reads and the int8 writes are coalesced whatever (so, sk) is.
constexpr int kOzSliceTile = 64;

// 16-byte chunk c (of BK / 16) of row o lands at chunk oz_swizzle_chunk<BK>(o, c): the
// address bits [4, 4 + log2(BK / 16)) are XORed with bits [7, ...) of the row's offset
// (row * BK), the 32B / 64B swizzle patterns of the UMMA shared-memory descriptor.
template <int BK>
__host__ __device__ constexpr int oz_swizzle_chunk(int o, int c)
{
    return BK == 64 ? (c ^ ((o >> 1) & 3)) : (c ^ ((o >> 2) & 1));
}

template <int BK, typename TIn>
__global__ void __launch_bounds__(256, 4)
    oz_slice_kernel(const TIn* src, int64_t so, int64_t sk, int O, int K, const int* exps, int S,
                    int8_t* dst, int O_pad, int K_pad)
{
    __shared__ double tile[kOzSliceTile][kOzSliceTile + 1];
    const int o0 = blockIdx.y * kOzSliceTile, k0 = blockIdx.x * kOzSliceTile;
    const int tid = threadIdx.x;
    const bool o_fast = so == 1;
    // all 16 loads of a thread are issued before the first shared-memory store, so that a CTA
    // has its whole 32 KB tile in flight at once
    constexpr int kLoads = kOzSliceTile * kOzSliceTile / 256;
    double        ld[kLoads];
#pragma unroll
    for(int it = 0; it < kLoads; ++it)
    {
        const int idx = tid + it * 256;
        const int oo  = o_fast ? idx % kOzSliceTile : idx / kOzSliceTile;
        const int kk  = o_fast ? idx / kOzSliceTile : idx % kOzSliceTile;
        const int o = o0 + oo, k = k0 + kk;
        ld[it] = (o < O && k < K) ? (double)src[(int64_t)o * so + (int64_t)k * sk] : 0.0;
    }
#pragma unroll
    for(int it = 0; it < kLoads; ++it)
    {
        const int idx = tid + it * 256;
        const int oo  = o_fast ? idx % kOzSliceTile : idx / kOzSliceTile;
        const int kk  = o_fast ? idx / kOzSliceTile : idx % kOzSliceTile;
        tile[oo][kk]  = ld[it];
    }
    __syncthreads();
    // each thread: one row oo, 16 consecutive k (4 words of 4 int8) -> 256 threads = 64 x 64
    const int oo = tid >> 2, kq = (tid & 3) * 16;
    const int o  = o0 + oo;
    if(o >= O_pad)
        return;
    int e = (o < O) ? exps[o] : 0;
    if(e == kOzExpNone)
        e = 0; // all-zero row: every slice is 0
    uint32_t  words[kOzMaxS][4];
#pragma unroll
    for(int s = 0; s < kOzMaxS; ++s)
#pragma unroll
        for(int w = 0; w < 4; ++w)
            words[s][w] = 0;
    // Slice s of x is the s-th base-128 digit of x 2^-e (|x 2^-e| < 1) with x's sign, i.e. what
    // S rounds of v *= 128, q = trunc(v), v -= q produce.  Those digits are the 7-bit fields of
    // the integer W = trunc(|x| 2^(7S - e)) < 2^(7S) <= 2^56, so one exact power-of-two scaling
    // and one conversion replace the S rounds of FP64 arithmetic.
    const int  se     = 7 * S - e;
    const bool direct = se <= 1023; // 2^se is a normal double (se >= 7 - 1025 always)
    const double scale = direct ? __longlong_as_double((long long)(1023 + se) << 52) : 0.0;
#pragma unroll
    for(int j = 0; j < 16; ++j)
    {
        const double x = tile[oo][kq + j];
        // exact (a scaling by a power of two); bits pushed below 2^-1074 are below 1 and would
        // be truncated anyway.  Only rows whose largest entry is tiny take the ldexp path.
        const double             w   = direct ? x * scale : ldexp(x, se);
        const unsigned long long W   = __double2ull_rz(fabs(w));
        const bool               neg = signbit(x);
#pragma unroll
        for(int s = 0; s < kOzMaxS; ++s)
        {
            if(s < S)
            {
                const uint32_t d = (uint32_t)(W >> (7 * (S - 1 - s))) & 127u;
                const uint32_t b = (neg ? 0u - d : d) & 0xFFu;
                words[s][j >> 2] |= b << (8 * (j & 3));
            }
        }
    }
    const int k   = k0 + kq;              // first of this thread's 16 k (one chunk)
    const int kc  = k / BK, c = (k % BK) / 16;
    const int64_t nkc = K_pad / BK;
    const int64_t off = (int64_t)o * BK + oz_swizzle_chunk<BK>(o, c) * 16;
    for(int s = 0; s < S; ++s)
    {
        uint4 w4 = make_uint4(words[s][0], words[s][1], words[s][2], words[s][3]);
        if(k < K_pad)
            *reinterpret_cast<uint4*>(dst + ((int64_t)s * nkc + kc) * O_pad * BK + off) = w4;
    }
}

} // namespace rb200
