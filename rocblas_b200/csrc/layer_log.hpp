// Layer logging of the TRSM entry points: the reference's ROCBLAS_LAYER protocol
// (library/src/handle.cpp:856-877 reads the mode, library/src/include/logging.hpp:139-187 and
// library/src/blas3/rocblas_trsm_imp.hpp:74-143 write the lines).
//
//   ROCBLAS_LAYER bit 1 (trace): one comma-separated line per call, the arguments as passed
//                                 (alpha as its value, pointers as addresses) and the atomics mode;
//   bit 2 (bench):               the rocblas-bench command line that repeats the call;
//   bit 4 (profile):             one line per distinct argument set with its call count,
//                                 written when the process exits.
//
// Each kind goes to the file named by ROCBLAS_LOG_TRACE_PATH / ROCBLAS_LOG_BENCH_PATH /
// ROCBLAS_LOG_PROFILE_PATH, else to stderr. The mode and the files are taken when a handle is
// created, as the reference does; a call made for a device-memory size query is not logged.
#pragma once
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

namespace rb200
{

enum : int
{
    kLayerTrace   = 1,
    kLayerBench   = 2,
    kLayerProfile = 4,
};

// One stream per distinct path, opened once per process (so that two handles with the same
// path append to one file instead of truncating each other's lines).
inline FILE* layer_log_stream(const char* env)
{
    static std::mutex                   mu;
    static std::map<std::string, FILE*> files;
    const char*                         path = std::getenv(env);
    if(!path || !*path)
        return stderr;
    std::lock_guard<std::mutex> lock(mu);
    auto                        it = files.find(path);
    if(it != files.end())
        return it->second;
    FILE* f = std::fopen(path, "w");
    if(!f)
        return stderr;
    files[path] = f;
    return f;
}

inline void layer_log_line(FILE* f, const std::string& line)
{
    static std::mutex           mu;
    std::lock_guard<std::mutex> lock(mu);
    std::fputs(line.c_str(), f);
    std::fputc('\n', f);
    std::fflush(f);
}

// Call counts per distinct argument line, written at process exit in first-seen order.
class LayerProfile
{
public:
    void add(FILE* f, const std::string& key)
    {
        std::lock_guard<std::mutex> lock(mu_);
        out_ = f;
        auto it = counts_.find(key);
        if(it == counts_.end())
        {
            counts_.emplace(key, 1);
            order_.push_back(key);
        }
        else
            ++it->second;
    }
    ~LayerProfile()
    {
        if(!out_)
            return;
        for(const auto& k : order_)
            std::fprintf(out_, "- { %s, call_count: %zu }\n", k.c_str(), counts_[k]);
        std::fflush(out_);
    }

private:
    std::mutex                    mu_;
    FILE*                         out_ = nullptr;
    std::map<std::string, size_t> counts_;
    std::vector<std::string>      order_;
};

inline LayerProfile& layer_profile()
{
    static LayerProfile p;
    return p;
}

// rocblas_atomics_mode as the logs print it (utility.hpp:380-383)
inline const char* atomics_mode_string(int mode)
{
    return mode != 0 ? "atomics_allowed" : "atomics_not_allowed";
}

// letters of the enums (rocblas utility.hpp:264-306)
inline char side_letter(int v) { return v == 141 ? 'L' : v == 142 ? 'R' : v == 143 ? 'B' : ' '; }
inline char fill_letter(int v) { return v == 121 ? 'U' : v == 122 ? 'L' : v == 123 ? 'F' : ' '; }
inline char trans_letter(int v) { return v == 111 ? 'N' : v == 112 ? 'T' : v == 113 ? 'C' : ' '; }
inline char diag_letter(int v) { return v == 131 ? 'N' : v == 132 ? 'U' : ' '; }

// What a TRSM entry point adds to its log lines beyond the common arguments.
struct TrsmLogInfo
{
    int     kind     = 0;     // 0 plain, 1 batched (pointer arrays), 2 strided batched
    bool    ilp64    = false; // the _64 entry point
    int64_t stride_a = 0, stride_b = 0;
};

// The arguments of one TRSM call as the log lines print them. alpha_re / alpha_im are the
// scalar's value (NaN for a null pointer); cplx selects the complex spellings.
struct TrsmLogCall
{
    TrsmLogInfo info;
    char        prec; // s, d, c, z
    int         side, uplo, trans, diag;
    int64_t     m, n;
    double      alpha_re, alpha_im;
    const void *A, *B;
    int64_t     lda, ldb, batch;
    bool        atomics; // the handle's atomics mode
};

inline void write_trsm_log(int layer_mode, FILE* trace_os, FILE* bench_os, FILE* profile_os,
                           const TrsmLogCall& c)
{
    const bool  cplx  = c.prec == 'c' || c.prec == 'z';
    const char* kinds[3] = {"", "batched_", "strided_batched_"};
    std::string name = std::string("rocblas_") + kinds[c.info.kind] + c.prec + "trsm";
    if(c.info.ilp64)
        name += "_64";
    const char sl = side_letter(c.side), ul = fill_letter(c.uplo), tl = trans_letter(c.trans),
               dl = diag_letter(c.diag);

    if(layer_mode & kLayerTrace)
    {
        std::ostringstream os;
        os << name << ',' << sl << ',' << ul << ',' << tl << ',' << dl << ',' << c.m << ',' << c.n
           << ',';
        if(cplx)
            os << '(' << c.alpha_re << ',' << c.alpha_im << ')';
        else
            os << c.alpha_re;
        os << ',' << c.A << ',' << c.lda;
        if(c.info.kind == 2)
            os << ',' << c.info.stride_a;
        os << ',' << c.B << ',' << c.ldb;
        if(c.info.kind == 2)
            os << ',' << c.info.stride_b;
        if(c.info.kind != 0)
            os << ',' << c.batch;
        os << ',' << atomics_mode_string(c.atomics);
        layer_log_line(trace_os, os.str());
    }
    if(layer_mode & kLayerBench)
    {
        const char* fn[3]   = {"trsm", "trsm_batched", "trsm_strided_batched"};
        const char* precs[] = {"f32_r", "f64_r", "f32_c", "f64_c"};
        const int   pi      = c.prec == 's' ? 0 : c.prec == 'd' ? 1 : c.prec == 'c' ? 2 : 3;
        std::ostringstream os;
        os << "./rocblas-bench" << (c.info.ilp64 ? " --api 1" : "") << " -f " << fn[c.info.kind]
           << " -r " << precs[pi] << " --side " << sl << " --uplo " << ul << " --transposeA " << tl
           << " --diag " << dl << " -m " << c.m << " -n " << c.n << " --alpha " << c.alpha_re;
        if(cplx && c.alpha_im != 0.0)
            os << " --alphai " << c.alpha_im;
        os << " --lda " << c.lda;
        if(c.info.kind == 2)
            os << " --stride_a " << c.info.stride_a;
        os << " --ldb " << c.ldb;
        if(c.info.kind == 2)
            os << " --stride_b " << c.info.stride_b;
        if(c.info.kind != 0)
            os << " --batch_count " << c.batch;
        if(!c.atomics)
            os << " --atomics_not_allowed";
        layer_log_line(bench_os, os.str());
    }
    if(layer_mode & kLayerProfile)
    {
        std::ostringstream os;
        os << "rocblas_function: \"" << name << "\", atomics_mode: " << atomics_mode_string(c.atomics)
           << ", side: " << sl
           << ", uplo: " << ul << ", transA: " << tl << ", diag: " << dl << ", m: " << c.m
           << ", n: " << c.n << ", lda: " << c.lda;
        if(c.info.kind == 2)
            os << ", stride_A: " << c.info.stride_a;
        os << ", ldb: " << c.ldb;
        if(c.info.kind == 2)
            os << ", stride_B: " << c.info.stride_b;
        if(c.info.kind != 0)
            os << ", batch_count: " << c.batch;
        layer_profile().add(profile_os, os.str());
    }
}

} // namespace rb200
