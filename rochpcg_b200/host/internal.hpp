// Implementation state of the host layer (not part of the public API).
#pragma once

#include <cstdio>
#include <memory>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../csrc/cg.cuh"
#include "../csrc/learned.cuh"
#include "../csrc/mixed.cuh"
#include "../csrc/ops64.cuh"
#include "hpcg.hpp"

namespace hpcg_b200 {

// Errors from CUDA or from the C ABI inside the void-returning reference
// signatures surface as this exception; the C ABI converts it back to a code.
struct Error : std::runtime_error
{
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] void throw_last(int code);
// Records the exception text as the C ABI's last error and returns its code.
inline int report(const Error& e) { return hb::record_error(e.code, "%s", e.what()); }
void check_cuda(cudaError_t e, const char* what);
inline void check(int rc)
{
    if(rc != 0) throw_last(rc);
}
#define HB_HOST_CUDA(call) ::hpcg_b200::check_cuda((call), #call)

// NVTX ranges (the reference's roctx ranges: set-up, optimization, CG, halo
// exchange, allreduce, benchmark phases) for profilers such as Nsight; with
// no tool attached they cost nothing.
struct TraceRange
{
    explicit TraceRange(const char* name) { nvtxRangePushA(name); }
    ~TraceRange() { nvtxRangePop(); }
    TraceRange(const TraceRange&) = delete;
    TraceRange& operator=(const TraceRange&) = delete;
};

// Consecutive phases of one function: phase() closes the previous range.
struct TracePhases
{
    bool open = false;
    void phase(const char* name)
    {
        if(open) nvtxRangePop();
        nvtxRangePushA(name);
        open = true;
    }
    ~TracePhases()
    {
        if(open) nvtxRangePop();
    }
};

struct Runtime
{
    bool initialized = false;
    int device = 0;
    cudaStream_t stream = nullptr;
    hb::ReduceScratch* ws = nullptr;   // reduction scratch (ticket left at zero)
    double* d_scalar = nullptr;        // device result slots
    double* h_scalar = nullptr;        // pinned mirror
};
Runtime& rt();
void ensure_runtime();

// Runs f() (which returns a status code) for a C ABI / operator entry point:
// initialises the runtime and turns a host-layer exception into its code.
template <typename F>
int guarded(F&& f)
{
    try
    {
        ensure_runtime();
        return f();
    }
    catch(const Error& e)
    {
        return report(e);
    }
    catch(const std::bad_alloc&)
    {
        return hb::record_error(HPCGB200_ERR_CUDA, "host allocation failed");
    }
}

template <typename T>
T* dalloc(size_t n)
{
    void* p = nullptr;
    if(n == 0) n = 1;
    HB_HOST_CUDA(cudaMalloc(&p, n * sizeof(T)));
    return static_cast<T*>(p);
}
void dfree(void* p);

// Cached solve graph (one per CG vector set / mode).
struct CGGraph
{
    cudaGraphExec_t exec = nullptr;
    cudaGraph_t graph = nullptr;
    bool conditional = false;          // WHILE node available
    const double* key[6] = {};
    int mode = -1;
    bool precond = true;
    bool flexible = false;
    bool timed = false;                // phase timers between the operators
    int kernels_per_iteration = 0;     // kernel nodes of one iteration body
    const void* smoother = nullptr;    // learned mode: smoother and buffer epoch the body captured
    long long smoother_epoch = -1;
};

// Per-level implementation data (SparseMatrix::optimizationData).
struct LevelOpt
{
    double* diag = nullptr;            // a_ii, read coalesced by the zero-guess backward sweep
    int* colors = nullptr;
    int jpl_blocks = 0;                // the reference's nblocks (2 per JPL round)
    std::vector<int> round_sizes;      // the reference's per-round sizes[]
    hb::ColorChunks cc{};              // colour-interleaved SpMV map
    hb::ZgGroups zg[HPCGB200_MAX_COLORS];  // per colour: slot groups the zero-guess passes need
    bool zg_ok = false;

    // FP32 / implicit-stencil data
    bool stencil_ok = false;
    hb::StencilLevel st{};
    float* diag32 = nullptr;
    float* inv_diag32 = nullptr;
    int* pass_status = nullptr;        // set (3) by a TMA-staged colour pass whose copies timed out (device word;
                                       // never cleared: every later solve on the problem reports it)

    // level-0 solver state
    hb::CGState* cg_state = nullptr;
    int cg_state_iters = 0;
    hb::GridBarrier* step_barrier = nullptr;  // the two-kernel CG step's grid barrier (zeroed per solve)
    std::vector<std::unique_ptr<CGGraph>> graphs;
    double* pap_partial = nullptr;     // per-block partial sums of the stencil SpMV + p.Ap (level 0)
    unsigned int* pap_ticket = nullptr;
    double* spmv_partial = nullptr;    // per-block partial sums of the ELL SpMV + p.Ap (level 0)
    unsigned int* spmv_ticket = nullptr;
    float* r32 = nullptr;              // FP32 right-hand side of the V-cycle (level 0)
    float* z32 = nullptr;              // FP32 V-cycle result (level 0)
    double* vec_scratch = nullptr;     // one FP64 vector of length m (TestCG / TestSymmetry)
    double* x0_saved = nullptr;        // learned CG: the initial guess, for a restart after a non-finite step

    // learned smoother (level 0 holds it for the hierarchy)
    struct Smoother* smoother = nullptr;
    int smoother_first_level = 2;
    int smoother_coarse_steps = 1;     // learned Richardson steps x += N(r - A x) on the coarsest level
    int last_fallback_iter = 0;        // learned CG: iteration at which the last solve fell back (0: none)
    double fb_jump = hb::kFallbackJump;  // learned CG failure rule (CGState)
    double fb_rate = hb::kFallbackRate;
    int fb_stall = hb::kFallbackStall;
    int fb_window = hb::kFallbackWindow;
    hb::PermMap pm{};                  // natural point -> permuted row (stencil levels)
};

// Per-level transfer data (MGData::optimizationData).
struct MGOpt
{
    int* inj_f = nullptr;              // permuted fine row of coarse point i
    int* inj_c = nullptr;              // permuted coarse row of coarse point i
    int* pro_f = nullptr;              // coarse permuted row -> injected fine permuted row (fused prolongation)
    float* rc32 = nullptr;
    float* xc32 = nullptr;
};

// Whether the V-cycles carry the prolongation in the coarse level's final
// smoother passes (HPCGB200_FUSED_PROLONG=1) or run it as a launch of its own
// after the coarse solve (default: measured faster on B200, the scattered
// read-modify-writes in the coarse passes cost more than the launch they
// save: 320^3 mixed V-cycle 1.291 vs 1.318 ms); both give the same bits.
bool fused_prolongation();

inline LevelOpt* opt(const SparseMatrix& A) { return static_cast<LevelOpt*>(A.optimizationData); }
inline const hb::ZgGroups* zg_of(const SparseMatrix& A)
{
    const LevelOpt* o = opt(A);
    return o && o->zg_ok ? o->zg : nullptr;
}
inline MGOpt* mgopt(const SparseMatrix& A) { return A.mgData ? static_cast<MGOpt*>(A.mgData->optimizationData) : nullptr; }

// Operators on raw FP32 level data (mixed V-cycle), defined in operators.cpp.
// pro: where this level's final values are prolongated (the finer level's x),
// fused into the level's last smoother passes; empty on level 0.
int mg_fp32(const SparseMatrix& A, const float* r, float* x, cudaStream_t s, hb::Prolong<float> pro = {});
// Level-0 FP32 V-cycles (mixed, learned) from the FP64 residual r64: the
// result is left in opt(A)->z32, and also written to z64 when it is not null.
int mg_mixed_to(const SparseMatrix& A, const double* r64, double* z64, cudaStream_t s);
int mg_learned_to(const SparseMatrix& A, const double* r64, double* z64, cudaStream_t s);

// Kernel launches of one CG iteration (captures the iteration graph if it
// does not exist yet; nothing is launched), defined in cg.cpp.
int iteration_kernels(const SparseMatrix& A, CGData& data, const Vector& b, Vector& x, bool precond,
                      MGPrecision prec, bool flexible);

// Graph-cached solve, defined in cg.cpp.
// phase_seconds (optional, 4 entries: dot, WAXPBY, SpMV, MG) selects the
// instrumented iteration body and receives the device time of each phase.
int run_cg(const SparseMatrix& A, CGData& data, const Vector& b, Vector& x, int max_iter, double tol, int& niters,
           double& normr, double& normr0, bool precond, MGPrecision prec, bool flexible, double* hist,
           double* seconds, double* phase_seconds = nullptr);

}  // namespace hpcg_b200
