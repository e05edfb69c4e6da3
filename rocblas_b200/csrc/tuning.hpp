// Tunable thresholds of the algorithm and tile choices.
//
// Defaults are compiled in.  At first use the table is overridden from a text file of
// "key value" lines: $ROCBLAS_B200_TUNING if set, else tuning.cfg next to the shared library
// (written by rocblas_b200/autotune.py, which times the candidates on the GPU).  The
// extension functions rocblas_b200_set_tuning / rocblas_b200_get_tuning change or read an
// entry at run time.  The reference's counterpart is its hand-made block-size tables
// (library/src/blas3/rocblas_trsm_kernels.hpp:39-132) and selection heuristics (:1458-1610).
#pragma once
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <dlfcn.h>
#include <mutex>
#include <string>

namespace rb200
{

struct Tuning
{
    int block_max_k          = 512;  // largest k for the one-CTA block solver (<= 512)
    int block_always_k       = 128;  // block solver at any parallelism up to this k
    int block_min_strips_pct = 100;  // else block solver if strips * batch >= SMs * pct / 100
    int sliced_min_k         = 1024; // precision form: sliced updates only for K >= this
    int dmma_big_tile_pct    = 100000; // 128x128 DMMA tiles if tiles >= SMs * pct / 100
    int mixed_slices         = 7;    // slices of the precision form when the caller passes 0
    int dmma_force_tile      = 0;    // 0: choose; 1..11: force one DMMA tile shape (DmmaTile)
    int dmma_big_bk          = 16;   // k depth of the 128x128 DMMA stage (16 or 32)
    int oz_bn                = 64;   // sliced GEMM output tile width (64: one pass; 128)
    int oz_bk                = 64;   // sliced GEMM K step in int8 (32 or 64)
    int chain_max_cols       = 1 << 30; // FP64 solves (k > 128) with <= this many columns: chain
    int chain_max_cols_f32   = 512;  // the same for FP32 (the chain computes in FP64)
    int chain_w              = 0;    // chain strip width: 0 auto (32 or 64), 32, 64
    int mixed_chain_blocks   = 8;    // precision form: chain solves for diagonal blocks of <= this
                                     // many 128-row blocks (< 2: recursion down to the leaves)
    int host_step_blocks     = 4;    // precision form on host buffers: rows per pipelined step,
                                     // in 128-row blocks
    int sliced_k_chunk       = 16384; // sliced GEMM: K range per set of row / column exponents
                                      // (multiple of 64, at most 16384); shorter ranges keep
                                      // more bits of entries far below their row's maximum
    int refine_check_sms     = 6;    // refined form: SMs of the FP64 solve of the tested
                                     // right-hand sides, which runs beside the sliced solve
    int refine_check_w       = 32;   // refined form: strip width of that solve's chain (16, 32)
    int refine_check_pairs   = 1;    // refined form: that chain in clusters of two CTAs, so the
                                     // sliced solve beside it may run CTA-pair GEMMs
    int refine_check_flag    = 0;    // refined form: that solve as the memory-bound flag
                                     // solve (up to 8 right-hand sides; 0: the chain)
    int wait_cycles_log2     = 31;   // chain solve: a flag wait gives up after 2^this clock
                                     // cycles (2^31: about a second), records error 4, returns
    int trsv_flag_min_n      = 256;  // trsv of one real vector: the flag-synchronised solve from
                                     // this order up
    int trsv_flag_nb         = 128;  // ... its block rows (64 or 128)
    int crt_group_m          = 8;    // residue GEMM tile order: row tiles per group
    int crt_pair             = 1;    // residue GEMM as CTA pairs (cta_group::2, 256 x 256 tiles)
                                     // when it has every SM of the device
    int crt_min_tiles_pct    = 100;  // precision form: residue engine for updates with at least
                                     // SMs * pct / 100 output tiles of 128 x 256, else slices
    int strsm_slices         = 4;    // FP32 solve: slices of its trailing updates on the int8 slice
                                     // engine (0: FFMA tiles)
    int strsm_sliced_min_k   = 1024; // ... for updates with at least this inner dimension
    int mixed_moduli         = 16;   // precision form: 0 updates on the slice engine; 14..16 on
                                     // the residue (CRT) engine with this many moduli
    int chain_first_item     = 0;    // failure injection for tests: uniform chain launches start
                                     // claiming items here, so the flags of the items before it
                                     // are never set and the waits on them run out (0: off)
};

struct TuningEntry
{
    const char* key;
    int Tuning::*field;
    int         lo, hi;
};

static const TuningEntry kTuningEntries[] = {
    {"block_max_k", &Tuning::block_max_k, 0, 512},
    {"block_always_k", &Tuning::block_always_k, 0, 512},
    {"block_min_strips_pct", &Tuning::block_min_strips_pct, 1, 100000},
    {"sliced_min_k", &Tuning::sliced_min_k, 1, 1 << 30},
    {"dmma_big_tile_pct", &Tuning::dmma_big_tile_pct, 1, 100000},
    {"mixed_slices", &Tuning::mixed_slices, 1, 8},
    {"dmma_force_tile", &Tuning::dmma_force_tile, 0, 11},
    {"dmma_big_bk", &Tuning::dmma_big_bk, 16, 32},
    {"oz_bn", &Tuning::oz_bn, 64, 128},
    {"oz_bk", &Tuning::oz_bk, 32, 64},
    {"chain_max_cols", &Tuning::chain_max_cols, 0, 1 << 30},
    {"chain_max_cols_f32", &Tuning::chain_max_cols_f32, 0, 1 << 30},
    {"chain_w", &Tuning::chain_w, 0, 64},
    {"mixed_chain_blocks", &Tuning::mixed_chain_blocks, 0, 1 << 20},
    {"host_step_blocks", &Tuning::host_step_blocks, 1, 1 << 20},
    {"sliced_k_chunk", &Tuning::sliced_k_chunk, 64, 16384},
    {"refine_check_sms", &Tuning::refine_check_sms, 1, 1024},
    {"refine_check_flag", &Tuning::refine_check_flag, 0, 1},
    {"refine_check_w", &Tuning::refine_check_w, 16, 32},
    {"refine_check_pairs", &Tuning::refine_check_pairs, 0, 1},
    {"wait_cycles_log2", &Tuning::wait_cycles_log2, 10, 40},
    {"chain_first_item", &Tuning::chain_first_item, 0, 1 << 30},
    {"mixed_moduli", &Tuning::mixed_moduli, 0, 16},
    {"strsm_slices", &Tuning::strsm_slices, 0, 8},
    {"crt_group_m", &Tuning::crt_group_m, 1, 1024},
    {"crt_pair", &Tuning::crt_pair, 0, 1},
    {"trsv_flag_min_n", &Tuning::trsv_flag_min_n, 1, 1 << 30},
    {"trsv_flag_nb", &Tuning::trsv_flag_nb, 64, 128},
    {"crt_min_tiles_pct", &Tuning::crt_min_tiles_pct, 0, 100000},
    {"strsm_sliced_min_k", &Tuning::strsm_sliced_min_k, 64, 1 << 30},
};

inline bool tuning_set(Tuning& t, const char* key, int value)
{
    for(const auto& e : kTuningEntries)
        if(!std::strcmp(e.key, key))
        {
            if(value < e.lo || value > e.hi)
                return false;
            t.*(e.field) = value;
            return true;
        }
    return false;
}

inline bool tuning_get(const Tuning& t, const char* key, int* value)
{
    for(const auto& e : kTuningEntries)
        if(!std::strcmp(e.key, key))
        {
            *value = t.*(e.field);
            return true;
        }
    return false;
}

inline void tuning_load_file(Tuning& t, const char* path)
{
    FILE* f = std::fopen(path, "r");
    if(!f)
        return;
    char line[256];
    while(std::fgets(line, sizeof(line), f))
    {
        char key[128];
        int  v;
        if(line[0] == '#')
            continue;
        if(std::sscanf(line, "%127s %d", key, &v) == 2)
            tuning_set(t, key, v);
    }
    std::fclose(f);
}

inline Tuning& tuning()
{
    static Tuning         t;
    static std::once_flag once;
    std::call_once(once, [] {
        if(const char* env = std::getenv("ROCBLAS_B200_TUNING"))
        {
            tuning_load_file(t, env);
            return;
        }
        Dl_info info;
        if(dladdr(reinterpret_cast<void*>(&tuning_load_file), &info) && info.dli_fname)
        {
            std::string p(info.dli_fname);
            const size_t slash = p.rfind('/');
            p = (slash == std::string::npos ? std::string(".") : p.substr(0, slash)) + "/tuning.cfg";
            tuning_load_file(t, p.c_str());
        }
    });
    return t;
}

} // namespace rb200
