// FP64-accurate GEMM update on the Blackwell tensor cores from residues modulo small primes
// (a Chinese-remainder form of the integer emulation of an FP64 product).
//
//     C := beta * C + alpha * P * Q            (P: M x K, Q: K x N, C: M x N, FP64)
//
// Method:
//   * every row r of P is scaled by 2^(b - e_r) (e_r = 1 + exponent of its largest entry) and
//     truncated to the integer P'(r,k) = trunc(P(r,k) 2^(b - e_r)), |P'| < 2^b; every column c
//     of Q the same way with exponents f_c, Q'(k,c);
//   * the exact integer product X = P' Q' (|X| < K 2^2b) is computed modulo NM pairwise
//     coprime moduli p_i <= 256 (crt_modulus): residues P'_i = P' mod p_i, Q'_i = Q' mod p_i in
//     the symmetric range fit int8, and C_i = P'_i Q'_i is one tcgen05.mma kind::i8 GEMM whose
//     int32 accumulation is exact (|C_i| <= K 128^2 <= 2^28 for K <= 16384);
//   * X is rebuilt from its residues r_i = C_i mod p_i (P = prod p_i, M_i = P / p_i,
//     w_i = M_i^-1 mod p_i) as X = sum_i r_i (w_i M_i) - q P with q = rint(sum_i r_i w_i / p_i):
//     the sum is taken modulo 2^128 in four 32-bit limbs, which is exact because |X| < P / 8 by
//     the choice of b (2b + log2 K <= log2 P - 3), and q from a 20-bit fixed-point sum whose
//     error (< 2^-9) is far inside the 3/8 margin that bound leaves;
//   * P Q ~= 2^(e_r + f_c - 2b) X, rounded once to FP64 in the epilogue.
// With 16 moduli (P ~ 2^125.4) and K <= 4096, b = 55: every entry keeps 55 bits relative to its
// row's (column's) largest entry and the product of the truncated operands is exact, at 16 int8
// GEMMs where the 7-bit slice form (ozaki_gemm.cuh) needs 36 slice-pair products for 56 bits.
//
// Kernel layout (persistent, one CTA per SM, 480 threads; output tiles 128 x 256; the tiles of
// a CTA are t = blockIdx.x + j * gridDim.x in a grouped order, so the CTAs in flight work on
// neighbouring tiles and, being in step, on the same modulus, and share its residue panels in L2):
//   warps 0, 14 copy producers (one thread each, alternate stages): per work item (tile,
//             modulus) and 128-deep K stage (two 64-deep panels), one bulk copy of the 2 x 128 x 64
//             P residues and one of the 2 x 256 x 64 Q residues into a 48 KB ring stage (4
//             stages); the residue kernel writes each row tile's panels back to back in the
//             tensor cores' SWIZZLE_64B order.  A single thread issues a stage in a few hundred
//             cycles whatever its size, so stages are large and two threads issue them;
//   warp 1    TMEM owner and MMA issuer: one 128 x 256 int32 accumulator per item, two
//             accumulators (all 512 TMEM columns) so that an item's MMAs overlap the drain of the
//             previous one;
//   warps 2-5 residue epilogue: tcgen05.ld of the accumulator (lanes = rows), r_i as one byte per
//             entry into the CTA's scratch slot in global memory (L2), two slots so that a tile's
//             residues are written while the previous tile is rebuilt;
//   warps 6-13 reconstruction: once all NM residues of a tile are in its slot, each thread takes
//             one row and half the columns, rebuilds X for 16 columns at a time and writes
//             beta C + alpha 2^s X.
// Every mbarrier wait is bounded; on timeout the kernel records the error, drains its in-flight
// copies and MMAs (again bounded), frees TMEM and returns.
#pragma once
#include <cuda.h> // CUtensorMap (the maps are encoded through the runtime's driver entry point)

#include <algorithm>
#include <cstdint>
#include <type_traits>

#include "ozaki_gemm.cuh"

namespace rb200
{

constexpr int kCrtMaxModuli = 16;
constexpr int kCrtBN        = 256;  // output tile width: N of one MMA
constexpr int kCrtBK        = 64;   // int8 K of one ring stage (SWIZZLE_64B rows)
constexpr int kCrtThreads   = 480;  // 15 warps
constexpr int kCrtResWarps  = 4;    // residue epilogue warps (warps 2 ..), a multiple of 4
constexpr int kCrtRebWarps  = 8;    // reconstruction warps (after them), a multiple of 4
constexpr int kCrtProdWarp2 = 2 + kCrtResWarps + kCrtRebWarps; // second copy producer
static_assert(kCrtProdWarp2 < kCrtThreads / 32, "warp roles");
constexpr int kCrtKMax      = 16384; // |C_i| <= K 128^2 <= 2^28 keeps the residue step in int32
constexpr int kCrtMaxBits   = 60;   // W < 2^60: three 20-bit fields in the residue kernel
constexpr int kCrtNPad      = kCrtBN;
constexpr int kCrtSmemBudget = 226 * 1024;
constexpr int kCrtChunks    = kCrtBN / 16; // 16-column chunks of a tile's scratch
constexpr int64_t kCrtSlotBytes = (int64_t)kCrtMaxModuli * kOzBM * kCrtBN; // one tile's residues

// Moduli, largest first: 2^8, 3*5*17, 11*23, 251, 13*19, 241, 239, 233, 229, 227, 223, 7*31, 211,
// 199, 197, 193 are pairwise coprime, so any prefix is a valid set; a symmetric residue of each
// fits int8 ([-128, 127] for 256, [-(p-1)/2, (p-1)/2] for the odd ones).
__host__ __device__ constexpr uint32_t crt_modulus(int i)
{
    return i == 0    ? 256u
           : i == 1  ? 255u
           : i == 2  ? 253u
           : i == 3  ? 251u
           : i == 4  ? 247u
           : i == 5  ? 241u
           : i == 6  ? 239u
           : i == 7  ? 233u
           : i == 8  ? 229u
           : i == 9  ? 227u
           : i == 10 ? 223u
           : i == 11 ? 217u
           : i == 12 ? 211u
           : i == 13 ? 199u
           : i == 14 ? 197u
                     : 193u;
}

// 128-bit unsigned integers for the compile-time CRT constants.
struct CrtU128
{
    unsigned long long lo, hi;
};

__host__ __device__ constexpr uint32_t crt_limb(CrtU128 a, int j)
{
    return (uint32_t)(j == 0 ? a.lo : j == 1 ? a.lo >> 32 : j == 2 ? a.hi : a.hi >> 32);
}

// a * m mod 2^128
__host__ __device__ constexpr CrtU128 crt_mul(CrtU128 a, uint32_t m)
{
    const unsigned long long l0 = (a.lo & 0xffffffffull) * m;
    const unsigned long long l1 = (a.lo >> 32) * m + (l0 >> 32);
    const unsigned long long h0 = (a.hi & 0xffffffffull) * m + (l1 >> 32);
    const unsigned long long h1 = (a.hi >> 32) * m + (h0 >> 32);
    return {(l0 & 0xffffffffull) | (l1 << 32), (h0 & 0xffffffffull) | (h1 << 32)};
}

// floor(a / d) and a mod d for 0 < d < 2^32 (long division by 32-bit limbs)
__host__ __device__ constexpr CrtU128 crt_div(CrtU128 a, uint32_t d)
{
    unsigned long long q[4] = {0, 0, 0, 0};
    unsigned long long r    = 0;
    for(int j = 3; j >= 0; --j)
    {
        const unsigned long long cur = (r << 32) | crt_limb(a, j);
        q[j] = cur / d;
        r    = cur % d;
    }
    return {q[0] | (q[1] << 32), q[2] | (q[3] << 32)};
}

__host__ __device__ constexpr uint32_t crt_rem(CrtU128 a, uint32_t d)
{
    unsigned long long r = 0;
    for(int j = 3; j >= 0; --j)
        r = ((r << 32) | crt_limb(a, j)) % d;
    return (uint32_t)r;
}

// inverse of a modulo p (a, p coprime), by the extended Euclidean algorithm
__host__ __device__ constexpr uint32_t crt_inverse(uint32_t a, uint32_t p)
{
    long long r0 = p, r1 = a % p, t0 = 0, t1 = 1;
    while(r1 != 0)
    {
        const long long q = r0 / r1;
        const long long r2 = r0 - q * r1, t2 = t0 - q * t1;
        r0 = r1;
        r1 = r2;
        t0 = t1;
        t1 = t2;
    }
    return (uint32_t)(((t0 % (long long)p) + (long long)p) % (long long)p);
}

// P = product of the first nm moduli
__host__ __device__ constexpr CrtU128 crt_product(int nm)
{
    CrtU128 p{1, 0};
    for(int i = 0; i < nm; ++i)
        p = crt_mul(p, crt_modulus(i));
    return p;
}

// M_i = P / p_i, w_i = M_i^-1 mod p_i
__host__ __device__ constexpr CrtU128 crt_cofactor(int nm, int i)
{
    return crt_div(crt_product(nm), crt_modulus(i));
}

__host__ __device__ constexpr uint32_t crt_weight(int nm, int i)
{
    return crt_inverse(crt_rem(crt_cofactor(nm, i), crt_modulus(i)), crt_modulus(i));
}

// The reconstruction works on r_i = C_i mod p_i with the weights folded into its constants:
// W_i = w_i M_i (< P, as w_i < p_i) is 1 modulo p_i and 0 modulo the others, so
// X = sum_i r_i W_i - q P with q = rint(sum_i r_i w_i / p_i); R_i = round(2^20 w_i / p_i) gives
// q from sum_i r_i R_i < 16 * 255 * 2^20 < 2^32 with an error below 16 * 128 / 2^20 = 2^-9.
__host__ __device__ constexpr CrtU128 crt_folded(int nm, int i)
{
    return crt_mul(crt_cofactor(nm, i), crt_weight(nm, i));
}

__host__ __device__ constexpr uint32_t crt_recip20(int nm, int i)
{
    return (uint32_t)((((unsigned long long)crt_weight(nm, i) << 20) + crt_modulus(i) / 2) / crt_modulus(i));
}

__host__ __device__ constexpr bool crt_tables_ok(int nm)
{
    for(int i = 0; i < nm; ++i)
    {
        const uint32_t p = crt_modulus(i);
        for(int j = 0; j < i; ++j)
        {
            uint32_t a = p, b = crt_modulus(j);
            while(b)
            {
                const uint32_t t = a % b;
                a = b;
                b = t;
            }
            if(a != 1)
                return false; // not coprime
        }
        if(crt_rem(crt_folded(nm, i), p) != 1)
            return false; // w_i is not the inverse of M_i
        for(int j = 0; j < nm; ++j)
            if(j != i && crt_rem(crt_cofactor(nm, i), crt_modulus(j)) != 0)
                return false; // M_i must vanish modulo the other moduli
    }
    return (crt_product(nm).hi >> 63) == 0; // P < 2^127: X_sym and its limbs stay signed-safe
}
static_assert(crt_tables_ok(8) && crt_tables_ok(12) && crt_tables_ok(14) && crt_tables_ok(15)
                  && crt_tables_ok(16),
              "CRT constants");

// log2 P of the first nm moduli (host side, for the choice of b)
inline double crt_log2_product(int nm)
{
    double s = 0.0;
    for(int i = 0; i < nm; ++i)
        s += __builtin_log2((double)crt_modulus(i));
    return s;
}

// Bits b kept per entry for a pass of depth K: K 2^2b <= P / 8.
inline int crt_bits(int nm, int64_t K)
{
    int lk = 0;
    while((int64_t(1) << lk) < std::max<int64_t>(K, 1))
        ++lk;
    const int b = (int)((crt_log2_product(nm) - 3.0 - lk) / 2.0);
    return std::min(b, kCrtMaxBits);
}

// Compile-time loop: f(std::integral_constant<int, I>) for I in [I0, I1).
template <int I0, int I1, class F>
__host__ __device__ __forceinline__ void crt_static_for(F&& f)
{
    if constexpr(I0 < I1)
    {
        f(std::integral_constant<int, I0>{});
        crt_static_for<I0 + 1, I1>(f);
    }
}

// tcgen05.ld of 32 columns (lanes = rows) without the wait: several loads go out before one
// tcgen05.wait::ld.
__device__ __forceinline__ void tmem_ld_32x32b_x32_nowait(uint32_t taddr, uint32_t* v)
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
}

// ---- residues --------------------------------------------------------------------------------
// Operand element (o, k) at src[o * so + k * sk]; exps[o] from launch_exponents (1 + exponent of
// the row's largest |x|; kOzExpNone for an all-zero row, whose residues are 0).  The rows are
// cut into row tiles of TR rows (the GEMM's tile height: 128 for P, 256 for Q); the residue
// modulo p_i of row o, column k lives in the K panel kc = k / 64 as
// dst[(((i * O_pad / TR + o / TR) * K_pad / 64 + kc) * TR + o % TR) * 64 + swizzled(k % 64)]:
// every (row tile, panel) block is the row-major image of TR rows of 64 bytes with the 16-byte
// chunks of a row permuted for SWIZZLE_64B, and a row tile's panels follow one another, so a
// run of K panels of one tile is one contiguous block.  Rows o >= O and columns k >= K are zero.
//
// Per entry: W = trunc(|x| 2^(bits - e)) < 2^bits (one exact power-of-two scaling and a 64-bit
// conversion), split into three 20-bit fields W = a 2^40 + m 2^20 + c, so that
// W mod p = (a (2^40 mod p) + m (2^20 mod p) + c) mod p is one 32-bit remainder by a constant.
template <int NM>
__global__ void __launch_bounds__(256, 2)
    crt_residue_kernel(const double* src, int64_t so, int64_t sk, int O, int K, const int* exps,
                       int bits, int8_t* dst, int O_pad, int K_pad, int TR)
{
    __shared__ double tile[kOzSliceTile][kOzSliceTile + 1];
    const int  o0 = blockIdx.y * kOzSliceTile, k0 = blockIdx.x * kOzSliceTile;
    const int  tid    = threadIdx.x;
    const bool o_fast = so == 1;
    constexpr int kLoads = kOzSliceTile * kOzSliceTile / 256;
    double        ld[kLoads];
#pragma unroll
    for(int it = 0; it < kLoads; ++it)
    {
        const int idx = tid + it * 256;
        const int oo  = o_fast ? idx % kOzSliceTile : idx / kOzSliceTile;
        const int kk  = o_fast ? idx / kOzSliceTile : idx % kOzSliceTile;
        const int o = o0 + oo, k = k0 + kk;
        ld[it] = (o < O && k < K) ? src[(int64_t)o * so + (int64_t)k * sk] : 0.0;
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
    // each thread: one row oo, 16 consecutive k (one 16-byte chunk per modulus)
    const int oo = tid >> 2, kq = (tid & 3) * 16;
    const int o  = o0 + oo;
    const int k  = k0 + kq;
    if(o >= O_pad || k >= K_pad)
        return;
    int e = (o < O) ? exps[o] : 0;
    if(e == kOzExpNone)
        e = 0; // all-zero row
    const int    se     = bits - e;
    const bool   direct = se <= 1023; // 2^se is a normal double (se >= bits - 1025 > -1022)
    const double scale  = direct ? __longlong_as_double((long long)(1023 + se) << 52) : 0.0;
    // the signed integer Ws = +-trunc(|x| 2^se) as a 2^40 (signed) + m 2^20 + c (m, c in [0, 2^20))
    int32_t  fa[16];
    uint32_t fm[16], fc[16];
#pragma unroll
    for(int j = 0; j < 16; ++j)
    {
        const double x = tile[oo][kq + j];
        // exact scaling; |w| < 2^bits <= 2^60
        const double    w  = direct ? x * scale : ldexp(x, se);
        const long long W  = (long long)__double2ull_rz(fabs(w));
        const long long Ws = signbit(x) ? -W : W;
        fa[j] = (int32_t)(Ws >> 40); // arithmetic shift: in [-2^20, 2^20)
        fm[j] = (uint32_t)(Ws >> 20) & 0xFFFFFu;
        fc[j] = (uint32_t)Ws & 0xFFFFFu;
    }
    const int     kc  = k / kCrtBK, c = (k % kCrtBK) / 16;
    const int64_t nkc = K_pad / kCrtBK;
    const int64_t tiles = O_pad / TR;
    int8_t* out = dst + ((int64_t)(o / TR) * nkc + kc) * TR * kCrtBK + (int64_t)(o % TR) * kCrtBK
                  + oz_swizzle_chunk<kCrtBK>(o, c) * 16;
    crt_static_for<0, NM>([&](auto I) {
        constexpr int      i    = decltype(I)::value;
        constexpr uint32_t p    = crt_modulus(i);
        constexpr int32_t  k40  = (int32_t)((1ull << 40) % p);
        constexpr uint32_t k20  = (uint32_t)((1ull << 20) % p);
        // the symmetric residue of t is ((t + half) mod p) - half for half = (p - 1) / 2 (odd p)
        // or 128 (p = 256); off (>= 2^28, a multiple of p) makes t + half non-negative
        constexpr uint32_t half = p == 256u ? 128u : (p - 1) / 2;
        constexpr uint32_t add  = p * ((1u << 28) / p + 1) + half;
        uint32_t           r[16];
#pragma unroll
        for(int j = 0; j < 16; ++j)
        {
            // in [0, 2^30): |fa k40| < 2^28, fm k20 + fc < 2^28 + 2^20, add < 2^29
            const uint32_t t = (uint32_t)(fa[j] * k40) + fm[j] * k20 + (fc[j] + add);
            r[j] = t % p;
        }
        // bytes r_j - half, four to a word: pack, then one bytewise subtract (wraps mod 256)
        uint32_t words[4];
#pragma unroll
        for(int q = 0; q < 4; ++q)
        {
            const uint32_t lo = __byte_perm(r[4 * q], r[4 * q + 1], 0x0040);
            const uint32_t hi = __byte_perm(r[4 * q + 2], r[4 * q + 3], 0x0040);
            words[q] = __vsub4(__byte_perm(lo, hi, 0x5410), half * 0x01010101u);
        }
        *reinterpret_cast<uint4*>(out + (int64_t)i * tiles * nkc * TR * kCrtBK)
            = make_uint4(words[0], words[1], words[2], words[3]);
    });
}

// ---- GEMM over the residues ------------------------------------------------------------------
struct CrtParams
{
    CUtensorMap   mapP, mapQ;    // CTA-pair form: the residue arrays as 2-D byte arrays [rows][64]
    int           M, N, K;       // logical sizes (K <= kCrtKMax)
    int           M_pad, N_pad;  // residue-panel rows (multiples of 128 (pair: 256) and 256)
    int           nkc;           // 64-deep K panels per modulus (a multiple of kCrtKS)
    const int8_t* resP;          // [NM][M_pad / 128][nkc][128][64], swizzled rows
    const int8_t* resQ;          // [NM][N_pad / 256][nkc][256][64] (pair: [NM][N_pad / 128][nkc][128][64])
    const int*    exp_rows;      // e_r, M entries
    const int*    exp_cols;      // f_c, N entries
    int           shift;         // 2b: P Q ~= 2^(e_r + f_c - shift) X
    double*       C;             // output (column-major, ldc)
    int64_t       ldc;
    double        alpha, beta;   // C := beta C + alpha P Q ; beta == 0 => C not read
    const double* beta_ptr;      // if set, beta := *beta_ptr (device pointer mode alpha of a trsm)
    const double* ualpha_ptr;    // if set and *ualpha_ptr == 0: C := 0 (a trsm with alpha == 0)
    int           ualpha_zero;   // host-side form of the same condition
    uint8_t*      scratch;       // two slots of kCrtSlotBytes per CTA
    int*          error;         // set to a nonzero code if a wait timed out
    int           group_m;       // tile order: group_m row tiles side by side, then the next columns
};

// Bounded wait that also gives up once another role has aborted.
__device__ __forceinline__ bool crt_wait(uint64_t* bar, uint32_t parity, const int* abort_flag)
{
    const long long t0 = clock64();
    while(!mbar_try_wait(bar, parity))
    {
        if(*(volatile const int*)abort_flag)
            return false;
        if(clock64() - t0 > (1ll << 31))
            return false;
    }
    return true;
}

__device__ __forceinline__ void crt_fail(int* error, int* abort_flag, int code)
{
    if(!*(volatile int*)abort_flag)
        atomicCAS(error, 0, code);
    atomicExch(abort_flag, 1);
}

// ---- CTA-pair (cta_group::2) helpers -------------------------------------------------------
__device__ __forceinline__ uint32_t crt_cluster_rank()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

// shared::cluster address of the same shared variable in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t crt_peer_addr(const void* ptr, uint32_t rank)
{
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(ptr)), "r"(rank));
    return r;
}

// every thread of both CTAs
__device__ __forceinline__ void crt_cluster_sync()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

__device__ __forceinline__ void crt_arrive_cluster(uint32_t caddr)
{
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(caddr) : "memory");
}

// try_wait with cluster-scope acquire: the barrier receives arrivals from the peer CTA
__device__ __forceinline__ bool crt_try_wait_cluster(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(smem_u32(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}

template <bool PAIR>
__device__ __forceinline__ bool crt_wait_t(uint64_t* bar, uint32_t parity, const int* abort_flag)
{
    if constexpr(!PAIR)
        return crt_wait(bar, parity, abort_flag);
    const long long t0 = clock64();
    while(!crt_try_wait_cluster(bar, parity))
    {
        if(*(volatile const int*)abort_flag)
            return false;
        if(clock64() - t0 > (1ll << 31))
            return false;
    }
    return true;
}

// One 256-row x 64-byte box of a residue array (2-D tensor map, no swizzle: the rows are stored
// pre-swizzled) into this CTA's shared memory, its bytes counted on the barrier at shared::cluster
// address mbar (the pair's first CTA).  No multicast: each CTA loads its own half of the pair's
// operands from this GPU's memory.
__device__ __forceinline__ void crt_tma_pair(void* dst, const CUtensorMap* map, int y, uint32_t mbar)
{
    asm volatile("cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
                 "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(y), "r"(mbar)
                 : "memory");
}

// M = 256 x N MMA of the pair, issued by one thread of the first CTA: A rows 0-127 and B rows
// (N) 0 .. N/2-1 from its shared memory, the other halves from the peer's at the same offsets;
// D rows 0-127 in its TMEM, 128-255 in the peer's.
__device__ __forceinline__ void crt_mma_pair(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                             uint32_t idesc, uint32_t accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::2.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
                 "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

// arrive on the barrier at this offset in both CTAs once the pair's MMAs so far are done
__device__ __forceinline__ void crt_commit_pair(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
                     smem_u32(bar)),
                 "h"((uint16_t)3)
                 : "memory");
}

// the same, on this CTA's barrier only
__device__ __forceinline__ void crt_commit_pair_local(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// instruction descriptor of the pair's M = 256 MMA
__host__ __device__ constexpr uint32_t crt_idesc_pair(int n)
{
    return (oz_idesc(n) & ~(0x1Fu << 24)) | ((uint32_t)(256 >> 4) << 24);
}

// r_i = C_i mod p_i in [0, p_i) for the int32 accumulator value v (|v| <= 2^28)
template <int I>
__device__ __forceinline__ uint32_t crt_residue_of(uint32_t v)
{
    constexpr uint32_t p = crt_modulus(I);
    if constexpr(p == 256u)
        return v & 255u;
    else
    {
        constexpr uint32_t off = p * ((1u << 28) / p + 1); // >= 2^28, a multiple of p
        return (v + off) % p;                              // v + off in [0, 2^29 + 2p)
    }
}

// X from its residues r_i (byte COL of every modulus' 16-byte chunk); returns X as a double
// (one rounding of the exact 128-bit value).
template <int NM, int COL>
__device__ __forceinline__ double crt_rebuild(const uint4 (&r)[NM])
{
    unsigned long long a0 = 0, a1 = 0, a2 = 0, a3 = 0;
    uint32_t           s20 = 0;
    crt_static_for<0, NM>([&](auto I) {
        constexpr int     i  = decltype(I)::value;
        constexpr CrtU128 Wi = crt_folded(NM, i);
        const uint32_t    wd = (COL >> 2) == 0 ? r[i].x : (COL >> 2) == 1 ? r[i].y : (COL >> 2) == 2 ? r[i].z : r[i].w;
        const uint32_t    y  = (wd >> (8 * (COL & 3))) & 0xFFu;
        s20 += y * crt_recip20(NM, i);
        a0 += (unsigned long long)y * crt_limb(Wi, 0);
        a1 += (unsigned long long)y * crt_limb(Wi, 1);
        a2 += (unsigned long long)y * crt_limb(Wi, 2);
        a3 += (unsigned long long)y * crt_limb(Wi, 3);
    });
    constexpr CrtU128 P = crt_product(NM);
    const unsigned long long q = (s20 + (1u << 19)) >> 20; // rint(sum r_i w_i / p_i)
    long long d0 = (long long)a0 - (long long)(q * crt_limb(P, 0));
    long long d1 = (long long)a1 - (long long)(q * crt_limb(P, 1));
    long long d2 = (long long)a2 - (long long)(q * crt_limb(P, 2));
    long long d3 = (long long)a3 - (long long)(q * crt_limb(P, 3));
    // carries (arithmetic shifts), the value modulo 2^128 in two's complement
    d1 += d0 >> 32;
    d2 += d1 >> 32;
    d3 += d2 >> 32;
    const unsigned long long lo = ((unsigned long long)(uint32_t)d1 << 32) | (uint32_t)d0;
    const unsigned long long hi = ((unsigned long long)(uint32_t)d3 << 32) | (uint32_t)d2;
    const bool               neg = (long long)hi < 0;
    const unsigned long long mlo = neg ? 0ull - lo : lo;
    const unsigned long long mhi = neg ? ~hi + (lo == 0 ? 1ull : 0ull) : hi;
    const double             mag = fma((double)mhi, 0x1p64, (double)mlo);
    return neg ? -mag : mag;
}

// Tile t of the persistent order: groups of g row tiles, within a group row-fastest, so the tiles
// in flight share the residue panels of g row tiles and of a run of column tiles in L2.
__device__ __forceinline__ void crt_tile_coords(int t, int tiles_m, int tiles_n, int g, int& mt, int& nt)
{
    const int per_group = g * tiles_n;
    const int grp = t / per_group, r = t - grp * per_group;
    const int gm  = min(g, tiles_m - grp * g); // rows in this group
    mt = grp * g + r % gm;
    nt = r / gm;
}

// x 2^E for an integer-valued x (|x| >= 1 or 0) by exact power-of-two factors: one factor when
// 2^E is a normal double; else x 2^E1 (E1 clamped to the normal range, exact because |x| >= 1)
// times 2^(E - E1), whose single rounding is the one of x 2^E; products below the smallest
// subnormal become zero and above the largest double infinity, as for ldexp.
__device__ __forceinline__ double crt_scale2(double x, int E)
{
    auto p2 = [](int e) { return __longlong_as_double((long long)(1023 + e) << 52); };
    if(E >= -1022 && E <= 1023)
        return x * p2(E);
    const int E1 = E < 0 ? -1022 : 1023;
    const int E2 = E - E1;
    if(E2 < -1022)
        return x * 0.0;
    return (x * p2(E1)) * p2(E2 > 1023 ? 1023 : E2);
}

// Reconstruction of row `row`'s 16-column chunk ch of output tile (mt, nt) from the residues in
// scratch slot `slot` (called by whole warps whose lanes take 32 consecutive rows of one chunk):
// X rebuilt per entry, scaled by 2^(e_r + f_c - shift) and written as beta C + alpha X.
template <int NM, int kTileRows>
__device__ __forceinline__ void crt_rebuild_chunk(const CrtParams& p, const uint8_t* slots, int slot, int mt,
                                                  int nt, int row, int ch, uint32_t rank, int lane,
                                                  double beta, bool zero)
{
    constexpr int64_t kModBytes = (int64_t)kCrtChunks * kOzBM * 16; // one modulus in a slot
    const int gr = mt * kTileRows + (int)rank * kOzBM + row;
    int       er = gr < p.M ? p.exp_rows[gr] : 0;
    if(er == kOzExpNone)
        er = 0;
    const uint8_t* src    = slots + (int64_t)slot * kCrtSlotBytes + (int64_t)row * 16;
    const bool     read_c = !zero && beta != 0.0;
    const int      c0     = nt * kCrtBN + ch * 16;
    // the chunk's 16 entries of C are loaded before the rebuild, together with the residues, so
    // that their latency (C is usually in DRAM) is paid once per chunk instead of once per entry
    double cin[16];
#pragma unroll
    for(int c = 0; c < 16; ++c)
    {
        const int gc = c0 + c;
        cin[c] = gr < p.M && gc < p.N && read_c ? p.C[gr + (int64_t)gc * p.ldc] : 0.0;
    }
    // lane l holds the exponent of column c0 + (l & 15), read before any store to C
    int ecl = c0 + (lane & 15) < p.N ? p.exp_cols[c0 + (lane & 15)] : 0;
    ecl     = ecl == kOzExpNone ? 0 : ecl;
    uint4 r[NM];
#pragma unroll
    for(int i = 0; i < NM; ++i)
        r[i] = *reinterpret_cast<const uint4*>(src + (int64_t)i * kModBytes + (int64_t)ch * kOzBM * 16);
    crt_static_for<0, 16>([&](auto Cc) {
        constexpr int c    = decltype(Cc)::value;
        const double  x    = crt_rebuild<NM, c>(r);
        const int     gc   = c0 + c;
        const int     ecol = __shfl_sync(0xffffffffu, ecl, c); // every lane, before the bounds test
        if(gr >= p.M || gc >= p.N)
            return;
        const double pq = crt_scale2(x, er + ecol - p.shift);
        double o;
        if(zero)
            o = 0.0;
        else if(beta == 0.0)
            o = p.alpha * pq;
        else
            o = fma(p.alpha, pq, beta * cin[c]);
        p.C[gr + (int64_t)gc * p.ldc] = o;
    });
}

// Stage of the copy ring: kCrtKS consecutive 64-deep K panels of one (tile, modulus) item,
// the P tile (128 x 64 per panel) then the Q tile (256 x 64 per panel; the pair form: this CTA's
// 128 columns); the residue kernel lays a row tile's K panels out back to back, so each operand
// of a stage is one copy.
constexpr int kCrtKS         = 2;
constexpr int kCrtStages     = 4; // 48 KB stages
constexpr int kCrtPairStages = 6; // 32 KB stages of the pair form

// Dynamic shared memory of the kernel (stages + 1 KB for the 1024-byte alignment)
__host__ __device__ constexpr size_t crt_smem_bytes(bool pair)
{
    return pair ? (size_t)kCrtPairStages * kCrtKS * (kOzBM + kCrtBN / 2) * kCrtBK + 1024
                : (size_t)kCrtStages * kCrtKS * (kOzBM + kCrtBN) * kCrtBK + 1024;
}

// PAIR: cta_group::2 form, launched as clusters of two CTAs (the pair) on 256 x 256 output
// tiles.  The pair's first CTA issues M = 256 MMAs whose A rows and B columns come half from
// each CTA's shared memory, so that a CTA streams 32 KB per 128-deep stage where the one-CTA
// form streams 48 KB for the same tensor work on its SM.  Each CTA's producers load its own
// halves by 2-D TMA and count the bytes on the first CTA's full barrier (which that CTA's
// producer arms with both halves); the MMAs' commits arrive on both CTAs' empty and
// accumulator barriers (multicast commit); each CTA drains and rebuilds its own 128 rows, and
// its residue warps free the accumulator on the first CTA's barrier.
template <int NM, bool PAIR>
__global__ void __launch_bounds__(kCrtThreads, 1) crt_gemm_kernel(const __grid_constant__ CrtParams p)
{
    constexpr int kPanelA = kOzBM * kCrtBK;                          // 8 KB of P residues per K panel
    constexpr int kPanelB = (PAIR ? kCrtBN / 2 : kCrtBN) * kCrtBK;   // 8 / 16 KB of Q residues
    constexpr int kStageA = kCrtKS * kPanelA;
    constexpr int kStage  = kCrtKS * (kPanelA + kPanelB);
    constexpr int NS      = PAIR ? kCrtPairStages : kCrtStages;
    constexpr int kTileRows = PAIR ? 2 * kOzBM : kOzBM;              // output tile height
    constexpr int64_t kModBytes = (int64_t)kCrtChunks * kOzBM * 16; // one modulus in a slot
    extern __shared__ __align__(1024) unsigned char crt_smem_raw[];
    unsigned char* smem = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(crt_smem_raw) + 1023) & ~uintptr_t(1023));

    __shared__ uint64_t full_bar[NS], empty_bar[NS], acc_full[2], acc_empty[2], slot_full[2],
        slot_empty[2], mma_done;
    __shared__ uint32_t tmem_base_sh;
    __shared__ int      abort_flag;
    __shared__ int      issued[2], consumed; // stages loaded by each producer / handed to the MMAs

    const int      warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank  = PAIR ? crt_cluster_rank() : 0u;          // CTA in the pair
    const int      unit  = PAIR ? (int)blockIdx.x >> 1 : (int)blockIdx.x;
    const int      units = PAIR ? (int)gridDim.x >> 1 : (int)gridDim.x;
    const int nks      = p.nkc / kCrtKS; // stages per item
    const int tiles_m  = p.M_pad / kTileRows;
    const int tiles_n  = p.N_pad / kCrtBN;
    const int tiles    = tiles_m * tiles_n;
    const int my_tiles = tiles > unit ? (tiles - 1 - unit) / units + 1 : 0;
    const int items    = my_tiles * NM;
    const int total    = items * nks; // stage uses of the whole CTA
    uint8_t*  slots    = p.scratch + (int64_t)blockIdx.x * 2 * kCrtSlotBytes;

    if(threadIdx.x == 0)
    {
        for(int i = 0; i < NS; ++i)
        {
            mbar_init(&full_bar[i], 1);  // the producer's expect_tx (pair: the first CTA's)
            mbar_init(&empty_bar[i], 1); // tcgen05.commit
        }
        for(int b = 0; b < 2; ++b)
        {
            mbar_init(&acc_full[b], 1);                                  // tcgen05.commit
            mbar_init(&acc_empty[b], (PAIR ? 2 : 1) * kCrtResWarps);     // one arrival per residue warp
            mbar_init(&slot_full[b], 32 * kCrtResWarps);  // every residue thread, after its last modulus
            mbar_init(&slot_empty[b], 32 * kCrtRebWarps); // every reconstruction thread
        }
        mbar_init(&mma_done, 1);
        abort_flag = 0;
        issued[0] = issued[1] = 0;
        consumed   = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if(warp == 1)
    {
        if constexpr(PAIR)
        {
            asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                             smem_u32(&tmem_base_sh)),
                         "r"(512));
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
        }
        else
        {
            asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                             smem_u32(&tmem_base_sh)),
                         "r"(512));
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    if constexpr(PAIR)
        crt_cluster_sync(); // both CTAs' barriers initialised and TMEM allocated
    else
        __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_base_sh;

    const double beta = p.beta_ptr ? *p.beta_ptr : p.beta;
    const bool   zero = p.ualpha_zero || (p.ualpha_ptr && *p.ualpha_ptr == 0.0);
    if(warp == 0 || warp == kCrtProdWarp2)
    {
        // ---------------- copy producers ----------------
        // lane 0 of two warps takes alternate stage uses (one thread issues a stage in a few
        // hundred cycles whatever its size, less than the tensor cores need for it at full
        // rate); the whole warps enter this branch so that no lane reaches another role
        const int who = warp == 0 ? 0 : 1;
        for(int it = who; it < total && lane == 0; it += 2)
        {
            const int      st = it % NS;
            const uint32_t ph = (uint32_t)((it / NS) & 1);
            const int      j  = it / nks, ks = it - j * nks;
            const int      jt = j / NM, i = j - jt * NM;
            if(!crt_wait_t<PAIR>(&empty_bar[st], ph ^ 1, &abort_flag))
            {
                crt_fail(p.error, &abort_flag, 11);
                break;
            }
            int mt, nt;
            crt_tile_coords(unit + jt * units, tiles_m, tiles_n, p.group_m, mt, nt);
            unsigned char* base = smem + st * kStage;
            if constexpr(PAIR)
            {
                // this CTA's 128-row P tile and 128-column Q tile, rows of the 2-D maps
                const int64_t yP = (((int64_t)i * (p.M_pad / kOzBM) + 2 * mt + rank) * p.nkc + ks * kCrtKS) * kOzBM;
                const int64_t yQ = (((int64_t)i * (p.N_pad / kOzBM) + 2 * nt + rank) * p.nkc + ks * kCrtKS) * kOzBM;
                if(rank == 0)
                    mbar_expect_tx(&full_bar[st], 2u * (uint32_t)kStage); // both CTAs' bytes
                const uint32_t fb = crt_peer_addr(&full_bar[st], 0);
                crt_tma_pair(base, &p.mapP, (int)yP, fb);
                crt_tma_pair(base + kStageA, &p.mapQ, (int)yQ, fb);
            }
            else
            {
                const int8_t* srcP = p.resP + (((int64_t)i * tiles_m + mt) * p.nkc + ks * kCrtKS) * kPanelA;
                const int8_t* srcQ = p.resQ + (((int64_t)i * tiles_n + nt) * p.nkc + ks * kCrtKS) * kPanelB;
                mbar_expect_tx(&full_bar[st], (uint32_t)kStage);
                bulk_load(base, srcP, kStageA, &full_bar[st]);
                bulk_load(base + kStageA, srcQ, kCrtKS * kPanelB, &full_bar[st]);
            }
            *(volatile int*)&issued[who] = it + 1;
        }
    }
    else if(warp == 1)
    {
        // ---------------- MMA issuer (pair: the first CTA's) ----------------
        if(lane == 0 && rank == 0)
        {
            const uint64_t desc_a0 = oz_smem_desc<kCrtBK>(smem_u32(smem));
            const uint64_t desc_b0 = oz_smem_desc<kCrtBK>(smem_u32(smem) + kStageA);
            constexpr uint32_t idesc = PAIR ? crt_idesc_pair(kCrtBN) : oz_idesc(kCrtBN);
            int  it = 0;
            bool ok = true;
            for(int j = 0; j < items && ok; ++j)
            {
                const int buf = j & 1;
                // the residue warps (pair: of both CTAs) have drained this accumulator's previous item
                if(!crt_wait_t<PAIR>(&acc_empty[buf], (uint32_t)(((j >> 1) & 1) ^ 1), &abort_flag))
                {
                    crt_fail(p.error, &abort_flag, 12);
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;");
                const uint32_t dcol = tmem + (uint32_t)(buf * kCrtBN);
                for(int ks = 0; ks < nks; ++ks, ++it)
                {
                    const int      st = it % NS;
                    const uint32_t ph = (uint32_t)((it / NS) & 1);
                    if(!crt_wait_t<PAIR>(&full_bar[st], ph, &abort_flag))
                    {
                        crt_fail(p.error, &abort_flag, 12);
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;");
                    *(volatile int*)&consumed = it + 1;
                    const uint64_t soff = (uint64_t)((st * kStage) >> 4);
#pragma unroll
                    for(int q = 0; q < kCrtKS; ++q)
#pragma unroll
                        for(int kk = 0; kk < kCrtBK / kOzMmaK; ++kk)
                        {
                            const uint64_t aof = (uint64_t)((q * kPanelA + kk * kOzMmaK) >> 4);
                            const uint64_t bof = (uint64_t)((q * kPanelB + kk * kOzMmaK) >> 4);
                            const uint32_t acc = (ks > 0 || q > 0 || kk > 0) ? 1u : 0u;
                            if constexpr(PAIR)
                                crt_mma_pair(dcol, desc_a0 + soff + aof, desc_b0 + soff + bof, idesc, acc);
                            else
                                oz_mma(dcol, desc_a0 + soff + aof, desc_b0 + soff + bof, idesc, acc);
                        }
                    if constexpr(PAIR)
                        crt_commit_pair(&empty_bar[st]);
                    else
                        oz_commit(&empty_bar[st]);
                }
                if constexpr(PAIR)
                    crt_commit_pair(&acc_full[buf]);
                else
                    oz_commit(&acc_full[buf]);
            }
            // every MMA issued has completed before TMEM is freed
            if constexpr(PAIR)
                crt_commit_pair_local(&mma_done);
            else
                oz_commit(&mma_done);
            (void)mbar_wait_bounded(&mma_done, 0);
        }
    }
    else if(warp < 2 + kCrtResWarps)
    {
        // ---------------- residue epilogue ----------------
        // kCrtResWarps / 4 warps per TMEM lane group (warp & 3), each taking an equal share of
        // the accumulator's columns
        constexpr int  kCols     = kCrtBN / (kCrtResWarps / 4);
        const int      quarter   = warp & 3; // TMEM lane group this warp may access
        const int      col0      = ((warp - 2) >> 2) * kCols;
        const int      row       = quarter * 32 + lane;
        const uint32_t lane_addr = tmem + ((uint32_t)(quarter * 32) << 16);
        for(int j = 0; j < items; ++j)
        {
            const int jt = j / NM, i = j - jt * NM, buf = j & 1, slot = jt & 1;
            bool      ok = true;
            if(i == 0) // the reconstruction warps are done with this slot's previous tile
                ok = crt_wait(&slot_empty[slot], (uint32_t)(((jt >> 1) & 1) ^ 1), &abort_flag);
            ok = ok && crt_wait_t<PAIR>(&acc_full[buf], (uint32_t)((j >> 1) & 1), &abort_flag);
            // warp-uniform outcome: the tcgen05.ld below needs the whole warp
            if(!__all_sync(0xffffffffu, ok))
            {
                crt_fail(p.error, &abort_flag, 13);
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;");
            uint8_t* dst = slots + (int64_t)slot * kCrtSlotBytes + (int64_t)i * kModBytes + (int64_t)row * 16;
            crt_static_for<0, NM>([&](auto I) {
                constexpr int ii = decltype(I)::value;
                if(i != ii)
                    return;
#pragma unroll 1
                for(int cc = col0; cc < col0 + kCols; cc += 64)
                {
                    // two loads in flight before the wait
                    uint32_t v[64];
                    tmem_ld_32x32b_x32_nowait(lane_addr + (uint32_t)(buf * kCrtBN + cc), v);
                    tmem_ld_32x32b_x32_nowait(lane_addr + (uint32_t)(buf * kCrtBN + cc + 32), v + 32);
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                    uint32_t w[16];
#pragma unroll
                    for(int q = 0; q < 16; ++q)
                        w[q] = crt_residue_of<ii>(v[4 * q]) | (crt_residue_of<ii>(v[4 * q + 1]) << 8)
                               | (crt_residue_of<ii>(v[4 * q + 2]) << 16) | (crt_residue_of<ii>(v[4 * q + 3]) << 24);
#pragma unroll
                    for(int c = 0; c < 4; ++c)
                        *reinterpret_cast<uint4*>(dst + (int64_t)(cc / 16 + c) * kOzBM * 16)
                            = make_uint4(w[4 * c], w[4 * c + 1], w[4 * c + 2], w[4 * c + 3]);
                }
            });
            // accumulator free for the item after next
            asm volatile("tcgen05.fence::before_thread_sync;");
            __syncwarp();
            if(lane == 0)
            {
                if constexpr(PAIR)
                    crt_arrive_cluster(crt_peer_addr(&acc_empty[buf], 0)); // the MMA issuer's barrier
                else
                    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&acc_empty[buf])) : "memory");
            }
            if(i == NM - 1) // this thread's residues of the tile are all in the slot
                asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&slot_full[slot])) : "memory");
        }
    }
    else if(warp < 2 + kCrtResWarps + kCrtRebWarps)
    {
        // ---------------- reconstruction ----------------
        // thread t: row t % 128, the t / 128-th share of the tile's 16-column chunks; the
        // CTA's last tile is rebuilt by every warp of the CTA (below)
        constexpr int kChunksPer = kCrtChunks / (kCrtRebWarps / 4);
        const int     t   = (warp - 2 - kCrtResWarps) * 32 + lane;
        const int     row = t & (kOzBM - 1);
        const int     ch0 = (t >> 7) * kChunksPer;
        for(int jt = 0; jt + 1 < my_tiles; ++jt)
        {
            const int slot = jt & 1;
            // warp-uniform outcome: the shuffles of the rebuild need the whole warp
            if(!__all_sync(0xffffffffu, crt_wait(&slot_full[slot], (uint32_t)((jt >> 1) & 1), &abort_flag)))
            {
                crt_fail(p.error, &abort_flag, 14);
                break;
            }
            int mt, nt;
            crt_tile_coords(unit + jt * units, tiles_m, tiles_n, p.group_m, mt, nt);
#pragma unroll 1
            for(int ch = ch0; ch < ch0 + kChunksPer; ++ch)
                crt_rebuild_chunk<NM, kTileRows>(p, slots, slot, mt, nt, row, ch, rank, lane, beta, zero);
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&slot_empty[slot])) : "memory");
        }
    }

    // ---------------- the last tile: every warp rebuilds ----------------
    // After its last MMA nothing else is left for the CTA, so the producer, MMA and residue warps
    // join the reconstruction warps on the last tile's 128 x 16 (row, chunk) units: unit u goes to
    // helper thread u mod (helpers), and the 32 consecutive units of a warp are 32 rows of one
    // chunk.  Each helper reaches this point when at most a few items of the last tile are left
    // (the copies run a few stages ahead of the MMAs, the MMAs two items ahead of the residue
    // warps), so its parity wait cannot see the slot's phase of two tiles before.  The pair's
    // second CTA issues no MMAs: its warp 1 would arrive at the start and stays out.
    __syncwarp(); // the producer and MMA warps' idle lanes wait for their lane 0
    const bool idle_warp = PAIR && rank != 0 && warp == 1;
    if(my_tiles > 0 && !idle_warp)
    {
        const int helpers = kCrtThreads - (PAIR && rank != 0 ? 32 : 0);
        const int hid     = (int)threadIdx.x - (PAIR && rank != 0 && warp > 1 ? 32 : 0);
        const int jt      = my_tiles - 1;
        const int slot    = jt & 1;
        if(__all_sync(0xffffffffu, crt_wait(&slot_full[slot], (uint32_t)((jt >> 1) & 1), &abort_flag)))
        {
            int mt, nt;
            crt_tile_coords(unit + jt * units, tiles_m, tiles_n, p.group_m, mt, nt);
#pragma unroll 1
            for(int u = hid; u < kOzBM * kCrtChunks; u += helpers)
                crt_rebuild_chunk<NM, kTileRows>(p, slots, slot, mt, nt, u & (kOzBM - 1), u / kOzBM, rank, lane,
                                                 beta, zero);
        }
        else
            crt_fail(p.error, &abort_flag, 15);
    }

    // ---------------- teardown ----------------
    __syncthreads();
    if(warp == 0 && lane == 0 && *(volatile int*)&abort_flag)
    {
        if constexpr(PAIR)
        {
            // the copies count on the first CTA's barrier, which this CTA cannot always watch:
            // give the ones still in flight (a few microseconds each) time to land
            const long long t0 = clock64();
            while(clock64() - t0 < 200000)
                __nanosleep(1000);
        }
        else
        {
            // let the copies that were issued but never consumed land before the CTA exits
            for(int it = consumed; it < max(issued[0], issued[1]); ++it)
                if(it < issued[it & 1])
                    (void)mbar_wait_bounded(&full_bar[it % NS], (uint32_t)((it / NS) & 1));
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    if constexpr(PAIR)
        crt_cluster_sync(); // neither CTA leaves while the pair's MMAs or arrivals may touch it
    else
        __syncthreads();
    if(warp == 1)
    {
        asm volatile("tcgen05.fence::after_thread_sync;");
        if constexpr(PAIR)
            asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
        else
            asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
    }
}

} // namespace rb200
