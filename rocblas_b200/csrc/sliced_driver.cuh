// Host side of the sliced (integer-slice, tensor-core) FP64 GEMM and of the precision form
// of the TRSM that uses it for its trailing updates.
#pragma once
#include <climits>
#include <functional>
#include <mutex>

#include "crt_gemm.cuh"
#include "ozaki_gemm.cuh"
#include "trsm_driver.cuh"

namespace rb200
{

// Element (o, k) of an operand at ptr[o * so + k * sk]: doubles, or floats if f32.
struct SliceOperand
{
    const void* ptr;
    int64_t     so, sk;
    int         f32 = 0;
    SliceOperand shifted_k(int64_t k0) const
    {
        const size_t es = f32 ? sizeof(float) : sizeof(double);
        return {static_cast<const char*>(ptr) + k0 * sk * (int64_t)es, so, sk, f32};
    }
    const double* d() const { return static_cast<const double*>(ptr); }
    const float*  f() const { return static_cast<const float*>(ptr); }
};

static inline int64_t round_up(int64_t a, int64_t b)
{
    return (a + b - 1) / b * b;
}

static inline size_t align256(size_t b)
{
    return (b + 255) & ~size_t(255);
}

// Workspace for one sliced GEMM of M x N x K with S slices.
static size_t sliced_gemm_workspace_bytes(int64_t M, int64_t N, int64_t K, int S)
{
    const int64_t Kp = round_up(std::min<int64_t>(std::max<int64_t>(K, 1), kOzKMax), kOzSliceTile);
    const int64_t Mp = round_up(std::max<int64_t>(M, 1), kOzBM), Np = round_up(std::max<int64_t>(N, 1), kOzNPad);
    static_assert(kOzSliceTile % 64 == 0, "slice padding must cover whole K steps");
    return align256((size_t)S * Mp * Kp) + align256((size_t)S * Np * Kp) + align256(4 * Mp)
           + align256(4 * Np);
}

struct SlicedGemm
{
    // C := b * C + a * P Q  (b = b_user ? *ualpha : b_imm; ualpha == 0 with zero_guard => C := 0)
    int64_t       M, N, K;
    int           S;
    SliceOperand  P, Q;
    void*         C;          // double, or float if c_f32 (then P and Q are float too)
    int           c_f32;
    int64_t       ldc;
    double        a;
    double        b_imm;
    const void*   ualpha_dev; // device-mode alpha of the caller, C's element type (or nullptr)
    double        ualpha_host;
    int           b_user;
    int           zero_guard;
    int           sms;        // SMs of the device (persistent grid)
    int           moduli = 0; // > 0: the residue (CRT) engine with this many moduli, else slices
    int           pair_ok = 0; // the sms SMs are whole SM pairs although fewer than the device's
};

__global__ void oz_fill_kernel(int* p, int n, int v)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i < n)
        p[i] = v;
}

static void launch_exponents(SliceOperand X, int O, int K, int* exps, cudaStream_t s)
{
    oz_fill_kernel<<<(unsigned)ceil_div(O, 256), 256, 0, s>>>(exps, O, kOzExpNone);
    count_launch();
    const unsigned kchunks = (unsigned)std::max<int64_t>(1, ceil_div(K, kOzExpChunk));
    if(X.so == 1)
    {
        const unsigned rchunks = (unsigned)std::max<int64_t>(1, ceil_div(K, kOzExpRowsChunk));
        dim3 grid((unsigned)ceil_div(O, 128), rchunks);
        if(X.f32)
            oz_exponent_rows_kernel<float><<<grid, 128, 0, s>>>(X.f(), X.sk, O, K, exps);
        else
            oz_exponent_rows_kernel<double><<<grid, 128, 0, s>>>(X.d(), X.sk, O, K, exps);
    }
    else
    {
        dim3 grid((unsigned)ceil_div((int64_t)O * 32, 256), kchunks);
        if(X.f32)
            oz_exponent_kernel<float><<<grid, 256, 0, s>>>(X.f(), X.so, X.sk, O, K, exps);
        else
            oz_exponent_kernel<double><<<grid, 256, 0, s>>>(X.d(), X.so, X.sk, O, K, exps);
    }
    count_launch();
}

static void launch_slices(SliceOperand X, int O, int K, const int* exps, int S, int8_t* dst, int O_pad,
                          int K_pad, int bk, cudaStream_t s)
{
    dim3 grid((unsigned)(K_pad / kOzSliceTile), (unsigned)(O_pad / kOzSliceTile));
    if(X.f32)
    {
        if(bk == 64)
            oz_slice_kernel<64, float><<<grid, 256, 0, s>>>(X.f(), X.so, X.sk, O, K, exps, S, dst, O_pad, K_pad);
        else
            oz_slice_kernel<32, float><<<grid, 256, 0, s>>>(X.f(), X.so, X.sk, O, K, exps, S, dst, O_pad, K_pad);
    }
    else
    {
        if(bk == 64)
            oz_slice_kernel<64, double><<<grid, 256, 0, s>>>(X.d(), X.so, X.sk, O, K, exps, S, dst, O_pad, K_pad);
        else
            oz_slice_kernel<32, double><<<grid, 256, 0, s>>>(X.d(), X.so, X.sk, O, K, exps, S, dst, O_pad, K_pad);
    }
    count_launch();
}

// One pass of the slice-pair groups [d_lo, d_hi) with output tiles 128 x bn and K steps of bk.
struct OzPass
{
    int d_lo, d_hi, bn, bk, ns, stages;
};

static int oz_stage_bytes(int ns, int bn, int bk)
{
    return ns * (kOzBM + bn) * bk;
}

// Split the S(S+1)/2 slice-pair products into passes whose accumulators fit TMEM (512
// columns of 128 x BN int32) and whose operand stages fit shared memory at least twice.
// Output tile width and K depth come from the tuning table (oz_bn, oz_bk).
static int plan_oz_passes(int S, OzPass* out)
{
    const int bn = tuning().oz_bn == 128 ? 128 : 64;
    int       bk = tuning().oz_bk == 32 ? 32 : 64;
    const int npass = S * bn <= 512 ? 1 : 2;
    const int ns_max = S; // the last pass stages every slice
    // one K depth for all passes (they share the slice panels): 64 if two stages fit
    if(2 * oz_stage_bytes(ns_max, bn, bk) + 1024 > kOzSmemBudget)
        bk = 32;
    auto make = [&](int lo, int hi) {
        OzPass q{lo, hi, bn, bk, std::min(S, hi), 0};
        q.stages = std::min(8, (kOzSmemBudget - 1024) / oz_stage_bytes(q.ns, q.bn, q.bk));
        return q;
    };
    if(npass == 1)
    {
        out[0] = make(0, S);
        return 1;
    }
    out[0] = make(0, 4);
    out[1] = make(4, S);
    return 2;
}

template <int BN, int BK, int SC>
static void launch_oz_kernel(const OzParams& p, int64_t Mp, int64_t Np, int sms, cudaStream_t s)
{
    const size_t smem = (size_t)p.stages * oz_stage_bytes(p.ns, BN, BK) + 1024;
    cudaFuncSetAttribute((const void*)ozaki_gemm_kernel<BN, BK, SC>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    // persistent: one CTA per SM (the stages fill its shared memory), at most one per tile
    const int64_t tiles = (Mp / kOzBM) * ceil_div(p.N, BN);
    const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(tiles, sms));
    (void)Np;
    // algorithmic work: int8 tensor operations of the pass's slice pairs
    int pairs = 0;
    for(int a = 0; a < p.ns; ++a)
        for(int b = 0; b < p.ns; ++b)
            pairs += (a + b >= p.d_lo && a + b < p.d_hi) ? 1 : 0;
    TimedLaunch tl(KernelClass::sliced, s, 2.0 * pairs * (double)p.M * p.N * p.K);
    ozaki_gemm_kernel<BN, BK, SC><<<grid, kOzThreads, smem, s>>>(p);
    count_launch();
}

// A single pass over all slices with BN = 64 uses the schedule unrolled for its slice count.
template <int BN, int BK>
static void launch_oz_pass(const OzParams& p, int64_t Mp, int64_t Np, int sms, cudaStream_t s)
{
    if constexpr(BN == 64)
    {
        if(p.d_lo == 0 && p.d_hi == p.S && p.ns == p.S)
        {
            switch(p.S)
            {
            case 1: return launch_oz_kernel<BN, BK, 1>(p, Mp, Np, sms, s);
            case 2: return launch_oz_kernel<BN, BK, 2>(p, Mp, Np, sms, s);
            case 3: return launch_oz_kernel<BN, BK, 3>(p, Mp, Np, sms, s);
            case 4: return launch_oz_kernel<BN, BK, 4>(p, Mp, Np, sms, s);
            case 5: return launch_oz_kernel<BN, BK, 5>(p, Mp, Np, sms, s);
            case 6: return launch_oz_kernel<BN, BK, 6>(p, Mp, Np, sms, s);
            case 7: return launch_oz_kernel<BN, BK, 7>(p, Mp, Np, sms, s);
            case 8: return launch_oz_kernel<BN, BK, 8>(p, Mp, Np, sms, s);
            default: break;
            }
        }
    }
    launch_oz_kernel<BN, BK, 0>(p, Mp, Np, sms, s);
}

// ---- residue (CRT) engine ------------------------------------------------------------------
// K range per set of row / column exponents (the tuning key shared with the slice engine).
static int64_t crt_k_chunk()
{
    return std::max<int64_t>(64, std::min<int64_t>(kCrtKMax, tuning().sliced_k_chunk / 64 * 64));
}

// CTAs of the persistent grid: at most one per SM; the pair form has 256-row tiles and an even
// number of CTAs
static int64_t crt_grid(int64_t Mp, int64_t Np, int sms, bool pair = false)
{
    if(pair)
    {
        const int64_t tiles = (Mp / (2 * kOzBM)) * (Np / kCrtBN);
        return 2 * std::max<int64_t>(1, std::min<int64_t>(tiles, std::max(sms, 2) / 2));
    }
    const int64_t tiles = (Mp / kOzBM) * (Np / kCrtBN);
    return std::max<int64_t>(1, std::min<int64_t>(tiles, std::max(sms, 1)));
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (the library does not link
// libcuda); null if the driver does not provide it
using CrtEncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                    const cuuint64_t*, const cuuint32_t*, const cuuint32_t*,
                                    CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                    CUtensorMapFloatOOBfill);
static CrtEncodeTiled crt_encode_fn()
{
    static CrtEncodeTiled fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if(cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &f, 12000, cudaEnableDefault, &q) == cudaSuccess
           && q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<CrtEncodeTiled>(f);
        else
            cudaGetLastError();
    });
    return fn;
}

// A residue array of `rows` rows of 64 bytes as a 2-D tensor map with 256-row boxes (no swizzle:
// the rows are stored in the MMA's swizzled order already).  The pair kernel's row coordinates
// are int32, so rows must stay below 2^31.
static bool crt_encode_map(CUtensorMap* m, const void* base, int64_t rows)
{
    const CrtEncodeTiled fn = crt_encode_fn();
    if(!fn || rows <= 0 || rows >= ((int64_t)1 << 31) || (reinterpret_cast<uintptr_t>(base) & 15))
        return false;
    const cuuint64_t dims[2]    = {(cuuint64_t)kCrtBK, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)kCrtBK};
    const cuuint32_t box[2]     = {(cuuint32_t)kCrtBK, (cuuint32_t)(kCrtKS * kOzBM)};
    const cuuint32_t estr[2]    = {1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void*>(base), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE)
           == CUDA_SUCCESS;
}

// K padded to whole ring stages (kCrtKS panels of 64)
static int64_t crt_k_pad(int64_t K)
{
    return round_up(std::max<int64_t>(K, 1), (int64_t)kCrtKS * kCrtBK);
}

// Workspace for one residue-engine GEMM of M x N x K with nm moduli on sms SMs: the residue
// panels of one K range, the exponents and two 512 KB reconstruction slots per CTA.
static size_t crt_gemm_workspace_bytes(int64_t M, int64_t N, int64_t K, int nm, int sms)
{
    const int64_t Kp = crt_k_pad(std::min<int64_t>(std::max<int64_t>(K, 1), crt_k_chunk()));
    // rows padded for either form (the pair form's tiles are 256 rows high)
    const int64_t Mp = round_up(std::max<int64_t>(M, 1), 2 * kOzBM), Np = round_up(std::max<int64_t>(N, 1), kCrtNPad);
    return align256((size_t)nm * Mp * Kp) + align256((size_t)nm * Np * Kp) + align256(4 * Mp)
           + align256(4 * Np) + align256((size_t)crt_grid(Mp, Np, sms) * 2 * kCrtSlotBytes);
}

static bool crt_moduli_supported(int nm)
{
    return nm == 14 || nm == 15 || nm == 16;
}

// pair: the cta_group::2 form (Mp a multiple of 256; the Q residues in 128-column tiles)
template <int NM>
static void launch_crt(SliceOperand P, SliceOperand Q, int M, int N, int K, int* eP, int* eQ,
                       int8_t* rP, int8_t* rQ, int64_t Mp, int64_t Np, int64_t Kp, CrtParams p,
                       int sms, bool pair, cudaStream_t s)
{
    const int bits = crt_bits(NM, K);
    dim3      gP((unsigned)(Kp / kOzSliceTile), (unsigned)(Mp / kOzSliceTile));
    crt_residue_kernel<NM><<<gP, 256, 0, s>>>(P.d(), P.so, P.sk, M, K, eP, bits, rP, (int)Mp, (int)Kp, kOzBM);
    count_launch();
    dim3 gQ((unsigned)(Kp / kOzSliceTile), (unsigned)(Np / kOzSliceTile));
    crt_residue_kernel<NM><<<gQ, 256, 0, s>>>(Q.d(), Q.so, Q.sk, N, K, eQ, bits, rQ, (int)Np, (int)Kp,
                                              pair ? kOzBM : kCrtBN);
    count_launch();
    p.shift = 2 * bits;
    const size_t   smem = crt_smem_bytes(pair);
    const unsigned grid = (unsigned)crt_grid(Mp, Np, sms, pair);
    // algorithmic work: int8 tensor operations of the NM residue products
    TimedLaunch tl(KernelClass::sliced, s, 2.0 * NM * (double)M * N * K);
    if(pair)
    {
        cudaFuncSetAttribute((const void*)crt_gemm_kernel<NM, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
        cudaLaunchConfig_t cfg{};
        cfg.gridDim          = dim3(grid);
        cfg.blockDim         = dim3(kCrtThreads);
        cfg.dynamicSmemBytes = smem;
        cfg.stream           = s;
        cudaLaunchAttribute at[1];
        at[0].id               = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = 2;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs    = at;
        cfg.numAttrs = 1;
        cudaLaunchKernelEx(&cfg, crt_gemm_kernel<NM, true>, p);
    }
    else
    {
        cudaFuncSetAttribute((const void*)crt_gemm_kernel<NM, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
        crt_gemm_kernel<NM, false><<<grid, kCrtThreads, smem, s>>>(p);
    }
    count_launch();
}

// Runs the residue engine; ws must hold crt_gemm_workspace_bytes(M, N, K, moduli, sms).
static bool run_crt_gemm(const SlicedGemm& g, void* ws, int* err_dev, cudaStream_t s)
{
    if(g.M <= 0 || g.N <= 0)
        return true;
    if(!crt_moduli_supported(g.moduli) || g.c_f32 || g.P.f32 || g.Q.f32)
        return false;
    // the pair form: clusters of two CTAs on 256 x 256 tiles (its 2-D maps take int32 rows),
    // only for a GEMM that has every SM of the device: beside another kernel (the refined form's
    // test solve) SM pairs may be split, and a cluster that cannot be placed waits for it
    const int64_t kchunk = crt_k_chunk();
    int           dev = 0, dev_sms = 0;
    if(cudaGetDevice(&dev) != cudaSuccess
       || cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    {
        cudaGetLastError();
        dev_sms = INT_MAX;
    }
    const bool    pair   = tuning().crt_pair != 0 && g.sms >= 2 && (g.sms >= dev_sms || g.pair_ok)
                      && crt_encode_fn() != nullptr
                      && (int64_t)g.moduli * round_up(std::max<int64_t>(g.M, g.N), 2 * kOzBM)
                                 * (crt_k_pad(std::min<int64_t>(std::max<int64_t>(g.K, 1), kchunk)) / kCrtBK)
                             < ((int64_t)1 << 31);
    const int64_t Mp = round_up(g.M, pair ? 2 * kOzBM : kOzBM), Np = round_up(g.N, kCrtNPad);
    const int64_t K  = std::max<int64_t>(g.K, 0);
    for(int64_t k0 = 0; k0 < std::max<int64_t>(K, 1); k0 += kchunk)
    {
        const int64_t kc = std::min<int64_t>(kchunk, K - k0);
        const int64_t Kp = crt_k_pad(kc);
        unsigned char* w = reinterpret_cast<unsigned char*>(ws);
        int8_t* rP = reinterpret_cast<int8_t*>(w);
        w += align256((size_t)g.moduli * Mp * Kp);
        int8_t* rQ = reinterpret_cast<int8_t*>(w);
        w += align256((size_t)g.moduli * Np * Kp);
        int* eP = reinterpret_cast<int*>(w);
        w += align256(4 * Mp);
        int* eQ = reinterpret_cast<int*>(w);
        w += align256(4 * Np);
        uint8_t* scratch = reinterpret_cast<uint8_t*>(w);

        const SliceOperand P = g.P.shifted_k(k0), Q = g.Q.shifted_k(k0);
        if(kc > 0)
        {
            launch_exponents(P, (int)g.M, (int)kc, eP, s);
            launch_exponents(Q, (int)g.N, (int)kc, eQ, s);
        }
        else
        {
            cudaMemsetAsync(eP, 0, 4 * Mp, s);
            cudaMemsetAsync(eQ, 0, 4 * Np, s);
        }
        CrtParams p{};
        p.M = (int)g.M;
        p.N = (int)g.N;
        p.K = (int)std::max<int64_t>(kc, 1);
        p.M_pad = (int)Mp;
        p.N_pad = (int)Np;
        p.nkc = (int)(Kp / kCrtBK);
        p.resP = rP;
        p.resQ = rQ;
        p.exp_rows = eP;
        p.exp_cols = eQ;
        p.C = static_cast<double*>(g.C);
        p.ldc = g.ldc;
        p.alpha = g.a;
        const bool first = k0 == 0;
        p.beta = first ? (g.b_user ? g.ualpha_host : g.b_imm) : 1.0;
        p.beta_ptr = (first && g.b_user) ? static_cast<const double*>(g.ualpha_dev) : nullptr;
        p.ualpha_ptr = g.zero_guard ? static_cast<const double*>(g.ualpha_dev) : nullptr;
        p.ualpha_zero = g.zero_guard && !g.ualpha_dev && g.ualpha_host == 0.0;
        p.scratch = scratch;
        p.error = err_dev;
        p.group_m = std::max(1, tuning().crt_group_m);
        const int kk = (int)std::max<int64_t>(kc, 1);
        if(pair
           && !(crt_encode_map(&p.mapP, rP, (int64_t)g.moduli * Mp * (Kp / kCrtBK))
                && crt_encode_map(&p.mapQ, rQ, (int64_t)g.moduli * Np * (Kp / kCrtBK))))
            return false;
        switch(g.moduli)
        {
        case 14: launch_crt<14>(P, Q, (int)g.M, (int)g.N, kk, eP, eQ, rP, rQ, Mp, Np, Kp, p, g.sms, pair, s); break;
        case 15: launch_crt<15>(P, Q, (int)g.M, (int)g.N, kk, eP, eQ, rP, rQ, Mp, Np, Kp, p, g.sms, pair, s); break;
        default: launch_crt<16>(P, Q, (int)g.M, (int)g.N, kk, eP, eQ, rP, rQ, Mp, Np, Kp, p, g.sms, pair, s); break;
        }
    }
    return true;
}

// Workspace of one update on the engine the tuning table selects (moduli > 0: residues, or
// slices for updates with too few residue tiles, see sliced_trsm_update).
static size_t update_workspace_bytes(int64_t M, int64_t N, int64_t K, int S, int moduli, int sms)
{
    const size_t sl = sliced_gemm_workspace_bytes(M, N, K, S);
    return moduli > 0 ? std::max(crt_gemm_workspace_bytes(M, N, K, moduli, sms), sl) : sl;
}

// Runs the sliced GEMM; ws must hold sliced_gemm_workspace_bytes(M, N, min(K, kOzKMax), S).
static bool run_sliced_gemm(const SlicedGemm& g, void* ws, int* err_dev, cudaStream_t s)
{
    if(g.moduli > 0)
        return run_crt_gemm(g, ws, err_dev, s);
    if(g.M <= 0 || g.N <= 0)
        return true;
    const int64_t Mp = round_up(g.M, kOzBM), Np = round_up(g.N, kOzNPad);
    const int     S  = g.S;
    OzPass        passes[2];
    const int     npass = plan_oz_passes(S, passes);
    const int64_t K = std::max<int64_t>(g.K, 0);
    // K ranges with their own exponents, accumulated in FP64 through C (beta = 1 after the
    // first): at most kOzKMax keeps the int32 sums exact, shorter ones keep more bits of
    // entries far below their row's (column's) maximum
    const int64_t kchunk = std::max<int64_t>(64, std::min<int64_t>(kOzKMax, tuning().sliced_k_chunk / 64 * 64));
    for(int64_t k0 = 0; k0 < std::max<int64_t>(K, 1); k0 += kchunk)
    {
        const int64_t kc = std::min<int64_t>(kchunk, K - k0);
        const int64_t Kp = round_up(std::max<int64_t>(kc, 1), kOzSliceTile);
        unsigned char* w = reinterpret_cast<unsigned char*>(ws);
        int8_t* sP = reinterpret_cast<int8_t*>(w);
        w += align256((size_t)S * Mp * Kp);
        int8_t* sQ = reinterpret_cast<int8_t*>(w);
        w += align256((size_t)S * Np * Kp);
        int* eP = reinterpret_cast<int*>(w);
        w += align256(4 * Mp);
        int* eQ = reinterpret_cast<int*>(w);

        const SliceOperand P = g.P.shifted_k(k0), Q = g.Q.shifted_k(k0);
        if(kc > 0)
        {
            launch_exponents(P, (int)g.M, (int)kc, eP, s);
            launch_exponents(Q, (int)g.N, (int)kc, eQ, s);
        }
        else
        {
            cudaMemsetAsync(eP, 0, 4 * Mp, s);
            cudaMemsetAsync(eQ, 0, 4 * Np, s);
        }
        const int bk = passes[0].bk;
        launch_slices(P, (int)g.M, (int)kc, eP, S, sP, (int)Mp, (int)Kp, bk, s);
        launch_slices(Q, (int)g.N, (int)kc, eQ, S, sQ, (int)Np, (int)Kp, bk, s);

        for(int pi = 0; pi < npass; ++pi)
        {
            const OzPass& q = passes[pi];
            OzParams      p{};
            p.sliceP = sP;
            p.sliceQ = sQ;
            p.nkc    = (int)(Kp / q.bk);
            p.M = (int)g.M;
            p.N = (int)g.N;
            p.K = (int)std::max<int64_t>(kc, 1);
            p.S = S;
            p.d_lo = q.d_lo;
            p.d_hi = q.d_hi;
            p.ns = q.ns;
            p.M_pad = (int)Mp;
            p.N_pad = (int)Np;
            p.exp_rows = eP;
            p.exp_cols = eQ;
            p.C = g.C;
            p.c_f32 = g.c_f32;
            p.ldc = g.ldc;
            p.alpha = g.a;
            const bool first = k0 == 0 && pi == 0;
            p.beta  = first ? (g.b_user ? g.ualpha_host : g.b_imm) : 1.0;
            p.beta_ptr = (first && g.b_user) ? g.ualpha_dev : nullptr;
            p.ualpha_ptr = g.zero_guard ? g.ualpha_dev : nullptr;
            p.ualpha_zero = g.zero_guard && !g.ualpha_dev && g.ualpha_host == 0.0;
            p.stages = q.stages;
            const int cols = (q.d_hi - q.d_lo) * q.bn;
            p.tmem_cols = cols <= 32 ? 32 : cols <= 64 ? 64 : cols <= 128 ? 128 : cols <= 256 ? 256 : 512;
            p.error = err_dev;
            if(q.bn == 128)
            {
                if(q.bk == 64)
                    launch_oz_pass<128, 64>(p, Mp, Np, g.sms, s);
                else
                    launch_oz_pass<128, 32>(p, Mp, Np, g.sms, s);
            }
            else
            {
                if(q.bk == 64)
                    launch_oz_pass<64, 64>(p, Mp, Np, g.sms, s);
                else
                    launch_oz_pass<64, 32>(p, Mp, Np, g.sms, s);
            }
        }
    }
    return true;
}

// One trailing update of a recursive solve of one system on the integer engines:
// C := C - op(A) X (side L) or C - X op(A) (side R), with the caller's alpha applied to C
// (`first`) and alpha == 0 giving C := 0, the way Recursive::update does on the tiles.
template <typename T>
static bool sliced_trsm_update(const TrsmProblem<T>& q, int c_lo, int c_hi, int x_lo, int x_hi,
                               int first, int S, int moduli, void* ws, int* err)
{
    static_assert(std::is_same<T, double>::value || std::is_same<T, float>::value, "real types");
    const int f32 = std::is_same<T, float>::value ? 1 : 0;
    const T*  A   = q.A.base + q.A.offset;
    T*        B   = q.B.base + q.B.offset;
    SlicedGemm g{};
    if(q.side_left)
    {
        g.M = c_hi - c_lo;
        g.N = q.n;
        g.K = x_hi - x_lo;
        g.P = !q.trans ? SliceOperand{A + c_lo + (int64_t)x_lo * q.lda, 1, q.lda, f32}
                       : SliceOperand{A + x_lo + (int64_t)c_lo * q.lda, q.lda, 1, f32};
        g.Q = SliceOperand{B + x_lo, q.ldb, 1, f32};
        g.C = B + c_lo;
    }
    else
    {
        g.M = q.m;
        g.N = c_hi - c_lo;
        g.K = x_hi - x_lo;
        g.P = SliceOperand{B + (int64_t)x_lo * q.ldb, 1, q.ldb, f32};
        g.Q = !q.trans ? SliceOperand{A + x_lo + (int64_t)c_lo * q.lda, q.lda, 1, f32}
                       : SliceOperand{A + c_lo + (int64_t)x_lo * q.lda, 1, q.lda, f32};
        g.C = B + (int64_t)c_lo * q.ldb;
    }
    g.c_f32 = f32;
    g.S = S;
    // the residue engine's 128 x 256 tiles leave SMs idle on updates with fewer tiles than SMs
    // (the host-buffer path's 512-row block rows); the slice engine's 128 x 64 tiles do not
    g.moduli = (int64_t)ceil_div(g.M, kOzBM) * ceil_div(g.N, kCrtBN) * 100
                       >= (int64_t)q.sm_count * tuning().crt_min_tiles_pct
                   ? moduli
                   : 0;
    g.ldc = q.ldb;
    g.a = -1.0;
    g.b_imm = 1.0;
    g.b_user = first;
    g.ualpha_dev = q.alpha.ptr;
    g.ualpha_host = (double)q.alpha.val;
    g.zero_guard = 1;
    g.sms = q.sm_count;
    g.pair_ok = q.crt_pair_ok;
    return run_sliced_gemm(g, ws, err, q.stream);
}

static int mixed_chain_w()
{
    const int t = tuning().chain_w;
    return t == 32 ? 32 : 64;
}

// ---- precision form of the TRSM ---------------------------------------------------------------
// The blocked recursive solve of trsm_driver.cuh with its trailing updates on the sliced
// tensor-core GEMM; the diagonal blocks stay in FP64 (fused trtri + DMMA invA leaves).
struct MixedRecursive : Recursive<double>
{
    int   S;
    int   moduli = 0; // > 0: updates on the residue (CRT) engine with this many moduli
    void* slice_ws;
    int*  err_dev;
    void* chain_ws = nullptr; // flags of the chain sub-solves (nullptr: recursion to the leaves)
    bool  ok = true;
    // optional hooks around every diagonal-block solve of blocks [b0, b1) (a chain sub-solve or
    // a leaf): the host-buffer path waits for A's data before it and copies the finished rows
    // of X out after it
    std::function<void(int, int)> before_diag, after_diag;

    // Updates with a short inner dimension stay on the FP64 DMMA tiles (K < sliced_min_k):
    // slicing costs about as much as a short product and short GEMMs gain nothing from it.
    void update_sliced(int c_lo, int c_hi, int x_lo, int x_hi, int first)
    {
        if(x_hi - x_lo < tuning().sliced_min_k)
        {
            update(c_lo, c_hi, x_lo, x_hi, first);
            return;
        }
        ok = ok && sliced_trsm_update<double>(pr, c_lo, c_hi, x_lo, x_hi, first, S, moduli, slice_ws, err_dev);
    }

    void solve_mixed(int b0, int b1, int first)
    {
        if(b1 - b0 == 1)
        {
            if(before_diag)
                before_diag(b0, b1);
            leaf(b0, first);
            if(after_diag)
                after_diag(b0, b1);
            return;
        }
        // diagonal blocks of at most mixed_chain_blocks x 128 rows: one chain launch in FP64
        if(chain_ws && b1 - b0 <= tuning().mixed_chain_blocks)
        {
            if(before_diag)
                before_diag(b0, b1);
            launch_chain_sub<double>(pr, b0, b1, first, mixed_chain_w(), chain_ws);
            if(after_diag)
                after_diag(b0, b1);
            return;
        }
        const int  bm = (b0 + b1) / 2;
        const int  r0 = row_of(b0), rm = row_of(bm), r1 = row_of(b1);
        const bool forward = pr.side_left ? pr.oplower() : !pr.oplower();
        if(forward)
        {
            solve_mixed(b0, bm, first);
            update_sliced(rm, r1, r0, rm, first);
            solve_mixed(bm, b1, 0);
        }
        else
        {
            solve_mixed(bm, b1, first);
            update_sliced(r0, rm, rm, r1, first);
            solve_mixed(b0, bm, 0);
        }
    }
};

// Flags of the largest chain sub-solve of the precision form (0: no chain sub-solves).
static size_t mixed_chain_workspace_bytes(const TrsmProblem<double>& pr)
{
    const int nbmax = tuning().mixed_chain_blocks;
    if(nbmax < 2)
        return 0;
    const int k = std::min<int64_t>((int64_t)nbmax * kInvNB, pr.k());
    return chain_workspace_bytes(chain_shape(k, pr.side_left ? pr.n : pr.m, pr.batch, mixed_chain_w()));
}

// Largest sliced update of the recursion (the top node's off-diagonal block).
static size_t mixed_slice_workspace_bytes(const TrsmProblem<double>& pr, int S, int moduli)
{
    const int64_t k = pr.k();
    if(k <= kInvNB)
        return 0;
    const int64_t nblk = ceil_div(k, kInvNB);
    const int64_t bm   = nblk / 2;
    const int64_t r_m  = std::min<int64_t>(bm * kInvNB, k);
    const int64_t big  = std::max(r_m, k - r_m);
    return pr.side_left ? update_workspace_bytes(big, pr.n, big, S, moduli, pr.sm_count)
                        : update_workspace_bytes(pr.m, big, big, S, moduli, pr.sm_count);
}

} // namespace rb200
