// The benchmark driver's protocol (src/main.cpp:174-563) and its report
// (src/ReportResults.cpp) for one rank on one B200.  Phases, loop bounds and
// the rating formulas follow the reference; the report is a JSON document
// whose sections and field names are those of the reference's YAML so that
// tools reading one can read the other.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "hpcg_b200.h"
#include "internal.hpp"


using namespace hpcg_b200;

namespace hpcg_b200 {
extern bool g_keep_generated;
}

namespace {

double wall() { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); }

void sync() { HB_HOST_CUDA(cudaStreamSynchronize(rt().stream)); }

// src/init.cpp:150-159: a dimension below 16 becomes the largest of the
// other two, and at least 16.
void adjust_dims(int d[3])
{
    for(int i = 0; i < 3; ++i)
    {
        if(d[i] < 16)
            for(int j = 1; j <= 2; ++j)
                if(d[(i + j) % 3] > d[i]) d[i] = d[(i + j) % 3];
        if(d[i] < 16) d[i] = 16;
    }
}

// Device bytes OptimizeProblem allocates (optimize.cpp): per level the
// permutation, colours, ELL (27 x (4 + 8) B per row), diagonal index, 1/a_ii,
// a_ii and their FP32 copies; per coarse row the two transfer indices and the
// FP32 coarse vectors; on level 0 the FP32 V-cycle vectors and one scratch
// vector.
double optimize_problem_bytes(int levels, const long long* rows)
{
    double b = 0.0;
    for(int l = 0; l < levels; ++l)
    {
        const double m = (double)rows[l];
        b += m * (4 + 4 + 27.0 * 12 + 4 + 8 + 8 + 4 + 4);
        if(l + 1 < levels) b += (double)rows[l + 1] * (4 + 4 + 4 + 4);
    }
    return b + (double)rows[0] * (4 + 4 + 8);
}

// ------------------------------------------------------------ JSON output

struct Json
{
    std::string s;
    std::vector<bool> first{true};
    void sep()
    {
        if(!first.back()) s += ",";
        first.back() = false;
        s += "\n";
        s.append(2 * (first.size() - 1), ' ');
    }
    void key(const char* k)
    {
        sep();
        str(k);
        s += ": ";
    }
    void str(const char* v)
    {
        s += '"';
        for(const char* c = v; *c; ++c)
        {
            if(*c == '"' || *c == '\\') s += '\\';
            s += *c;
        }
        s += '"';
    }
    void open(const char* k, char brace = '{')
    {
        if(k) key(k);
        else if(first.size() > 1) sep();
        s += brace;
        first.push_back(true);
    }
    void close(char brace = '}')
    {
        first.pop_back();
        s += "\n";
        s.append(2 * (first.size() - 1), ' ');
        s += brace;
    }
    void num(const char* k, double v)
    {
        key(k);
        if(!std::isfinite(v)) s += "null";
        else
        {
            char buf[40];
            std::snprintf(buf, sizeof buf, "%.17g", v);
            s += buf;
        }
    }
    void integer(const char* k, long long v)
    {
        key(k);
        s += std::to_string(v);
    }
    void text(const char* k, const char* v)
    {
        key(k);
        str(v);
    }
    void boolean(const char* k, bool v)
    {
        key(k);
        s += v ? "true" : "false";
    }
};

// x / t, or NaN (JSON null) when the phase was not timed.
double rate(double x, double t) { return t > 0.0 ? x / t : NAN; }

}  // namespace

extern "C" int hpcgb200_benchmark_report(hpcgb200_benchmark_result* R, char* json, size_t capacity, size_t* length)
{
    if(!R) return hb::record_error(HPCGB200_ERR_ARG, "null result");
    if(R->levels < 1 || R->levels > HPCGB200_BENCH_MAX_LEVELS)
        return hb::record_error(HPCGB200_ERR_ARG, "levels must be 1..%d", HPCGB200_BENCH_MAX_LEVELS);
    const double* times = R->times;
    const int L = R->levels;

    // ======== FLOP count model (src/ReportResults.cpp:134-158)
    const double sets = R->cg_sets;
    const double fniters = sets * (double)R->opt_max_iters;
    const double fnrow = (double)R->rows[0];
    const double fnnz = (double)R->nonzeros[0];
    const double pre = R->presmoother_steps, post = R->postsmoother_steps;
    const double fnops_ddot = (3.0 * fniters + sets) * 2.0 * fnrow;
    const double fnops_waxpby = (3.0 * fniters + sets) * 2.0 * fnrow;
    const double fnops_sparsemv = (fniters + sets) * 2.0 * fnnz;
    double fnops_precond = 0.0;
    for(int i = 0; i + 1 < L; ++i)
    {
        const double nnz = (double)R->nonzeros[i];
        fnops_precond += pre * fniters * 4.0 * nnz;
        fnops_precond += fniters * 2.0 * nnz;
        fnops_precond += post * fniters * 4.0 * nnz;
    }
    fnops_precond += fniters * 4.0 * (double)R->nonzeros[L - 1];
    const double fnops = fnops_ddot + fnops_waxpby + fnops_sparsemv + fnops_precond;
    const double conv = (double)R->ref_max_iters / (double)R->opt_max_iters;
    const double frefnops = fnops * conv;

    // ======== memory traffic model (:160-195): 8 B values, 4 B indices
    const double d8 = 8.0, i4 = 4.0;
    const double fnreads_ddot = (3.0 * fniters + sets) * 2.0 * fnrow * d8;
    const double fnwrites_ddot = (3.0 * fniters + sets) * d8;
    const double fnreads_waxpby = (3.0 * fniters + sets) * 2.0 * fnrow * d8;
    const double fnwrites_waxpby = (3.0 * fniters + sets) * fnrow * d8;
    const double fnreads_sparsemv = (fniters + sets) * (fnnz * (d8 + i4) + fnrow * d8);
    const double fnwrites_sparsemv = (fniters + sets) * fnrow * d8;
    double fnreads_precond = 0.0, fnwrites_precond = 0.0;
    for(int i = 0; i + 1 < L; ++i)
    {
        const double nnz = (double)R->nonzeros[i], nrow = (double)R->rows[i];
        fnreads_precond += pre * fniters * (2.0 * nnz * (d8 + i4) + nrow * d8);
        fnwrites_precond += pre * fniters * nrow * d8;
        fnreads_precond += fniters * (nnz * (d8 + i4) + nrow * d8);
        fnwrites_precond += fniters * nnz * d8;
        fnreads_precond += post * fniters * (2.0 * nnz * (d8 + i4) + nrow * d8);
        fnwrites_precond += post * fniters * nnz * d8;
    }
    {
        const double nnz = (double)R->nonzeros[L - 1], nrow = (double)R->rows[L - 1];
        fnreads_precond += fniters * (2.0 * nnz * (d8 + i4) + nrow * d8);
        fnwrites_precond += fniters * nrow * d8;
    }
    const double fnreads = fnreads_ddot + fnreads_waxpby + fnreads_sparsemv + fnreads_precond;
    const double fnwrites = fnwrites_ddot + fnwrites_waxpby + fnwrites_sparsemv + fnwrites_precond;
    const double frefnreads = fnreads * conv, frefnwrites = fnwrites * conv;

    // ======== memory usage model (:200-262), one rank
    const double nz27 = 27.0, p8 = 8.0;
    double fnbytes = (double)sizeof(Geometry) + d8 * sets;
    fnbytes += fnrow * 1.0 + 4.0 * fnrow * p8;
    fnbytes += fnrow * nz27 * (i4 + d8 + 8.0);
    fnbytes += fnrow * 3.0 * d8;
    fnbytes += fnrow * 2.0 * d8 + fnrow * 2.0 * d8;  // r, Ap; z, p (ncol = nrow at one rank)
    std::vector<double> per_level(L, 0.0);
    per_level[0] = fnbytes;
    fnbytes += R->optimize_problem_bytes;
    for(int i = 1; i < L; ++i)
    {
        const double m = (double)R->rows[i];
        double b = m * i4 + m * d8 + 2.0 * m * d8;
        b += (double)(sizeof(Geometry) + sizeof(SparseMatrix) + 3 * sizeof(Vector) + sizeof(MGData));
        b += m * 1.0 + 4.0 * m * p8 + m * nz27 * (i4 + d8 + 8.0);
        per_level[i] = b;
        fnbytes += b;
    }

    const double overhead = times[0] + sets * (times[7] / 10.0 + times[9] / 10.0);
    const double totalGflops = frefnops / overhead / 1.0e9;
    const double totalGflops24 = frefnops / (times[0] + sets * times[7] / 10.0) / 1.0e9;
    R->fnops = fnops;
    R->frefnops = frefnops;
    R->gflops_raw = rate(fnops, times[0]) / 1e9;
    R->gflops_convergence = rate(frefnops, times[0]) / 1e9;
    R->gflops_final = totalGflops;
    R->gflops_hpcg24 = totalGflops24;
    R->gbs_raw = rate(fnreads + fnwrites, times[0]) / 1e9;
    R->gbs_final = (frefnreads + frefnwrites) / overhead / 1e9;
    R->memory_total_gb = fnbytes / 1e9;
    R->valid = (R->testcg_count_fail == 0) && (R->symmetry_count_fail == 0) && R->norms_pass && !R->global_failure &&
               R->check_problem_errors == 0;

    Json J;
    J.open(nullptr);
    J.text("HPCG-Benchmark version", "3.1");
    J.open("Implementation");
    J.text("Name", "rochpcg_b200 (B200, sm_100a)");
    J.text("Precision", R->mode == HPCGB200_MODE_MIXED
                            ? "mixed: FP64 CG, FP32 V-cycle on the implicit stencil"
                            : (R->mode == HPCGB200_MODE_FP64_STENCIL
                                   ? "FP64 on the implicit stencil (the ELL path's results, no matrix reads)"
                                   : "FP64"));
    J.boolean("Reference phases run", R->verify != 0);
    J.close();
    J.open("Machine Summary");
    J.integer("Distributed Processes", 1);
    J.integer("Threads per processes", 1);
    J.close();
    J.open("Global Problem Dimensions");
    J.integer("Global nx", R->nx);
    J.integer("Global ny", R->ny);
    J.integer("Global nz", R->nz);
    J.close();
    J.open("Processor Dimensions");
    J.integer("npx", 1);
    J.integer("npy", 1);
    J.integer("npz", 1);
    J.close();
    J.open("Local Domain Dimensions");
    J.integer("nx", R->nx);
    J.integer("ny", R->ny);
    J.integer("Lower ipz", 0);
    J.integer("Upper ipz", 0);
    J.integer("nz", R->nz);
    J.close();
    J.open("Setup Information");
    J.num("Setup Time", times[9]);
    J.close();
    J.open("Linear System Information");
    J.integer("Number of Equations", R->rows[0]);
    J.integer("Number of Nonzero Terms", R->nonzeros[0]);
    J.close();
    J.open("Multigrid Information");
    J.integer("Number of coarse grid levels", L - 1);
    J.open("Coarse Grids", '[');
    for(int i = 1; i < L; ++i)
    {
        J.open(nullptr);
        J.integer("Grid Level", i);
        J.integer("Number of Equations", R->rows[i]);
        J.integer("Number of Nonzero Terms", R->nonzeros[i]);
        J.integer("Number of Presmoother Steps", R->presmoother_steps);
        J.integer("Number of Postsmoother Steps", R->postsmoother_steps);
        J.close();
    }
    J.close(']');
    J.close();
    J.open("Memory Use Information");
    J.num("Total memory used for data (Gbytes)", fnbytes / 1e9);
    J.num("Memory used for OptimizeProblem data (Gbytes)", R->optimize_problem_bytes / 1e9);
    J.num("Bytes per equation (Total memory / Number of Equations)", fnbytes / fnrow);
    J.num("Memory used for linear system and CG (Gbytes)", per_level[0] / 1e9);
    J.open("Coarse Grids", '[');
    for(int i = 1; i < L; ++i)
    {
        J.open(nullptr);
        J.integer("Grid Level", i);
        J.num("Memory used", per_level[i] / 1e9);
        J.close();
    }
    J.close(']');
    J.close();
    J.open("Spectral Convergence Tests");
    J.text("Result", R->testcg_count_fail == 0 ? "PASSED" : "FAILED");
    J.open("Unpreconditioned");
    J.integer("Maximum iteration count", R->testcg_niters_max_no_prec);
    J.integer("Expected iteration count", R->testcg_expected_niters_no_prec);
    J.close();
    J.open("Preconditioned");
    J.integer("Maximum iteration count", R->testcg_niters_max_prec);
    J.integer("Expected iteration count", R->testcg_expected_niters_prec);
    J.close();
    J.close();
    J.open("Departure from Symmetry |x'Ay-y'Ax|/(2*||x||*||A||*||y||)/epsilon");
    J.text("Result", R->symmetry_count_fail == 0 ? "PASSED" : "FAILED");
    J.num("Departure for SpMV", R->depsym_spmv);
    J.num("Departure for MG", R->depsym_mg);
    J.close();
    J.open("Iteration Count Information");
    J.text("Result", R->global_failure ? "FAILED" : "PASSED");
    J.integer("Reference CG iterations per set", R->ref_max_iters);
    J.integer("Optimized CG iterations per set", R->opt_max_iters);
    J.integer("Total number of reference iterations", (long long)R->ref_max_iters * R->cg_sets);
    J.integer("Total number of optimized iterations", (long long)R->opt_max_iters * R->cg_sets);
    J.close();
    J.open("Reproducibility Information");
    J.text("Result", R->norms_pass ? "PASSED" : "FAILED");
    J.num("Scaled residual mean", R->norms_mean);
    J.num("Scaled residual variance", R->norms_variance);
    J.close();
    J.open("Benchmark Time Summary");
    J.num("Optimization phase", times[7]);
    J.num("DDOT", times[1]);
    J.num("WAXPBY", times[2]);
    J.num("SpMV", times[3]);
    J.num("MG", times[5]);
    J.num("Total", times[0]);
    J.close();
    J.open("Floating Point Operations Summary");
    J.num("Raw DDOT", fnops_ddot);
    J.num("Raw WAXPBY", fnops_waxpby);
    J.num("Raw SpMV", fnops_sparsemv);
    J.num("Raw MG", fnops_precond);
    J.num("Total", fnops);
    J.num("Total with convergence overhead", frefnops);
    J.close();
    J.open("GB/s Summary");
    J.num("Raw Read B/W", rate(fnreads, times[0]) / 1e9);
    J.num("Raw Write B/W", rate(fnwrites, times[0]) / 1e9);
    J.num("Raw Total B/W", R->gbs_raw);
    J.num("Total with convergence and optimization phase overhead", R->gbs_final);
    J.close();
    // Per-operator times come from device timers between the operators of the
    // graph-resident solve (CG_B200 with times); a rate is null when its time is 0.
    J.open("GFLOP/s Summary");
    J.num("Raw DDOT", rate(fnops_ddot, times[1]) / 1e9);
    J.num("Raw WAXPBY", rate(fnops_waxpby, times[2]) / 1e9);
    J.num("Raw SpMV", rate(fnops_sparsemv, times[3]) / 1e9);
    J.num("Raw MG", rate(fnops_precond, times[5]) / 1e9);
    J.num("Raw Total", R->gflops_raw);
    J.num("Total with convergence overhead", R->gflops_convergence);
    J.num("Total with convergence and optimization phase overhead", totalGflops);
    J.close();
    J.open("User Optimization Overheads");
    J.num("Optimization phase time (sec)", times[7]);
    J.num("Optimization phase time vs reference SpMV+MG time", rate(times[7], times[8]));
    J.close();
    J.open("Validation Details");
    J.integer("CheckProblem mismatching rows", R->check_problem_errors);
    J.num("Reference tolerance (scaled residual after the reference CG)", R->ref_tolerance);
    J.integer("Reference CG iterations run", R->ref_niters);
    J.integer("Optimized CG iterations to reach the reference tolerance", R->opt_setup_niters);
    J.integer("Tolerance failures", R->tolerance_failures);
    J.integer("Errors in CG calls", R->err_count);
    J.num("Worst optimized CG set-up time (sec)", R->opt_worst_time);
    J.integer("Number of CG sets", R->cg_sets);
    J.boolean("QuickPath", R->quick_path != 0);
    J.close();
    J.open("Final Summary");
    if(R->valid)
    {
        J.num("HPCG result is VALID with a GFLOP/s rating of", totalGflops);
        J.num("HPCG 2.4 rating for historical reasons is", totalGflops24);
        if(R->mode == HPCGB200_MODE_MIXED)
            J.text("Mixed precision", "the V-cycle runs in FP32; not an FP64 HPCG rating");
        if(times[0] >= 1800.0) J.boolean("Meets the official minimum execution time", true);
        else
        {
            J.num("Results are valid but execution time (sec) is", times[0]);
            J.num("Official results execution time (sec) must be at least", 1800.0);
        }
    }
    else
    {
        J.text("HPCG result is", "INVALID.");
    }
    J.close();
    J.close();
    J.s += "\n";

    if(length) *length = J.s.size();
    if(!json) return 0;
    if(capacity < J.s.size() + 1)
        return hb::record_error(HPCGB200_ERR_WORKSPACE, "report needs %zu bytes", J.s.size() + 1);
    std::memcpy(json, J.s.c_str(), J.s.size() + 1);
    return 0;
}

namespace {

// A device vector released on every exit path.
struct OwnedVector
{
    Vector v;
    explicit OwnedVector(local_int_t n) { CudaInitializeVector(v, n); }
    ~OwnedVector()
    {
        try
        {
            CudaDeleteVector(v);
        }
        catch(const Error&)
        {
        }
    }
    OwnedVector(const OwnedVector&) = delete;
    OwnedVector& operator=(const OwnedVector&) = delete;
};

struct Hierarchy
{
    Geometry* geom = nullptr;
    SparseMatrix A{};
    Vector b, x, xexact;
    CGData data{};
    ~Hierarchy()
    {
        try
        {
            if(rt().initialized) cudaStreamSynchronize(rt().stream);
            DeleteMatrix(A);
            CudaDeleteVector(b);
            CudaDeleteVector(x);
            CudaDeleteVector(xexact);
            CudaDeleteCGData(data);
            if(geom)
            {
                DeleteGeometry(*geom);
                delete geom;
            }
        }
        catch(const Error&)
        {
        }
    }
};

int run_protocol(const hpcgb200_benchmark_params& P, hpcgb200_benchmark_result& R)
{
    std::memset(&R, 0, sizeof R);
    int d[3] = {P.nx, P.ny, P.nz};
    adjust_dims(d);
    const int numberOfMgLevels = 4;
    const int div = 1 << (numberOfMgLevels - 1);
    if(d[0] % div || d[1] % div || d[2] % div)
        return hb::record_error(HPCGB200_ERR_ARG, "dimensions must be divisible by %d", div);
    if((long long)d[0] * d[1] * d[2] > 0x7fffffffLL) return hb::record_error(HPCGB200_ERR_ARG, "grid exceeds 2^31 rows");
    if(P.mode != HPCGB200_MODE_FP64 && P.mode != HPCGB200_MODE_MIXED && P.mode != HPCGB200_MODE_FP64_STENCIL)
        return hb::record_error(HPCGB200_ERR_ARG, "mode must be HPCGB200_MODE_FP64, _MIXED or _FP64_STENCIL");
    const bool verify = P.verify != 0;
    const bool quickPath = P.running_time == 0;
    const MGPrecision prec = P.mode == HPCGB200_MODE_MIXED
                                 ? MGPrecision::FP32
                                 : (P.mode == HPCGB200_MODE_FP64_STENCIL ? MGPrecision::FP64_STENCIL : MGPrecision::FP64);
    const bool flexible = needs_flexible(prec);
    R.nx = d[0];
    R.ny = d[1];
    R.nz = d[2];
    R.mode = P.mode;
    R.verify = verify;
    R.quick_path = quickPath;
    R.levels = numberOfMgLevels;
    double* times = R.times;

    ensure_runtime();
    Hierarchy H;
    // ---- set-up phase (src/main.cpp:188-215)
    TracePhases trace;
    trace.phase("hpcg:setup");
    sync();
    double t = wall();
    H.geom = new Geometry;
    GenerateGeometry(1, 0, 1, 0, 0, 0, d[0], d[1], d[2], 1, 1, 1, H.geom);
    InitializeSparseMatrix(H.A, H.geom);
    GenerateProblem(H.A, &H.b, &H.x, &H.xexact);
    SetupHalo(H.A);
    SparseMatrix* cur = &H.A;
    for(int level = 1; level < numberOfMgLevels; ++level)
    {
        GenerateCoarseProblem(*cur);
        cur = cur->Ac;
    }
    sync();
    times[9] = wall() - t;
    cur = &H.A;
    for(int l = 0; l < numberOfMgLevels; ++l, cur = cur->Ac)
    {
        R.rows[l] = cur->totalNumberOfRows;
        R.nonzeros[l] = cur->totalNumberOfNonzeros;
    }
    R.presmoother_steps = H.A.mgData->numberOfPresmootherSteps;
    R.postsmoother_steps = H.A.mgData->numberOfPostsmootherSteps;

    // ---- CheckProblem on every level (src/main.cpp:218-246)
    trace.phase("hpcg:CheckProblem");
    if(verify)
    {
        cur = &H.A;
        for(int l = 0; l < numberOfMgLevels; ++l, cur = cur->Ac)
            R.check_problem_errors += CheckProblem_B200(*cur, l == 0 ? &H.b : nullptr, l == 0 ? &H.x : nullptr,
                                                        l == 0 ? &H.xexact : nullptr);
        CudaInitializeSparseCGData(H.A, H.data);
    }

    // ---- reference SpMV+MG timing (src/main.cpp:275-306)
    trace.phase("hpcg:reference SpMV+MG timing");
    const int numberOfCalls = quickPath ? 1 : 10;
    if(verify)
    {
        OwnedVector x_overlap(H.A.localNumberOfColumns), b_computed(H.A.localNumberOfRows);
        CudaFillRandomVector(x_overlap.v);
        int rc = 0;
        sync();
        t = wall();
        for(int i = 0; i < numberOfCalls && !rc; ++i)
        {
            rc = ComputeSPMV_ref(H.A, x_overlap.v, b_computed.v);
            if(!rc) rc = ComputeMG_ref(H.A, b_computed.v, x_overlap.v);
        }
        sync();
        times[8] = (wall() - t) / numberOfCalls;
        if(rc) return rc;
    }

    // ---- reference CG: the residual reduction of 50 iterations (src/main.cpp:312-341)
    trace.phase("hpcg:reference CG");
    const int refMaxIters = 50;
    R.ref_max_iters = refMaxIters;
    double refTolerance = P.tol;
    if(verify)
    {
        std::vector<double> ref_times(9, 0.0);
        int niters = 0;
        double normr = 0.0, normr0 = 0.0;
        CudaZeroVector(H.x);
        if(CG_ref(H.A, H.data, H.b, H.x, refMaxIters, 0.0, niters, normr, normr0, ref_times.data(), true, false))
            ++R.err_count;
        R.ref_niters = niters;
        refTolerance = normr / normr0;
    }
    R.ref_tolerance = refTolerance;

    // ---- OptimizeProblem (src/main.cpp:343-356)
    trace.phase("hpcg:OptimizeProblem");
    sync();
    t = wall();
    check(OptimizeProblem(H.A, H.data, H.b, H.x, H.xexact));
    sync();
    times[7] = wall() - t;
    R.optimize_problem_bytes = optimize_problem_bytes(numberOfMgLevels, R.rows);

    // ---- validation (src/main.cpp:370-386)
    trace.phase("hpcg:TestCG + TestSymmetry");
    if(verify)
    {
        TestCGData tc{};
        check(TestCG_B200(H.A, H.data, H.b, H.x, tc, prec));
        R.testcg_count_pass = tc.count_pass;
        R.testcg_count_fail = tc.count_fail;
        R.testcg_expected_niters_no_prec = tc.expected_niters_no_prec;
        R.testcg_expected_niters_prec = tc.expected_niters_prec;
        R.testcg_niters_max_no_prec = tc.niters_max_no_prec;
        R.testcg_niters_max_prec = tc.niters_max_prec;
        TestSymmetryData ts{};
        check(TestSymmetry_B200(H.A, H.b, H.xexact, ts, prec));
        R.depsym_spmv = ts.depsym_spmv;
        R.depsym_mg = ts.depsym_mg;
        R.symmetry_count_fail = ts.count_fail;
    }

    // ---- optimized CG set-up: iterations to reach the reference residual (src/main.cpp:400-445)
    trace.phase("hpcg:optimized CG set-up");
    int optMaxIters = 10 * refMaxIters;
    int optNiters = refMaxIters;
    double opt_worst_time = 0.0;
    std::vector<double> opt_times(10, 0.0);
    for(int i = 0; i < 1; ++i)
    {
        CudaZeroVector(H.x);
        const double last = opt_times[0];
        int niters = 0;
        double normr = 0.0, normr0 = 0.0;
        if(CG_B200(H.A, H.data, H.b, H.x, optMaxIters, refTolerance, niters, normr, normr0, opt_times.data(), true,
                   prec, flexible, nullptr))
            ++R.err_count;
        if(normr / normr0 > refTolerance) ++R.tolerance_failures;
        if(niters > optNiters) optNiters = niters;
        R.opt_setup_niters = niters;
        const double cur_time = opt_times[0] - last;
        if(cur_time > opt_worst_time) opt_worst_time = cur_time;
    }
    if(R.tolerance_failures) R.global_failure = 1;
    R.opt_worst_time = opt_worst_time;

    // ---- timed CG sets (src/main.cpp:472-530)
    trace.phase("hpcg:timed CG sets");
    const double total_runtime = P.running_time;
    const int numberOfCgSets = int(total_runtime / opt_worst_time) + 1;
    optMaxIters = optNiters;
    R.opt_max_iters = optMaxIters;
    std::vector<double> scaled_residual;
    int actualCgSets = 0;
    while(total_runtime - times[0] > 0.0 || actualCgSets < numberOfCgSets)
    {
        CudaZeroVector(H.x);
        int niters = 0;
        double normr = 0.0, normr0 = 0.0;
        if(CG_B200(H.A, H.data, H.b, H.x, optMaxIters, 0.0, niters, normr, normr0, times, true, prec, flexible,
                   nullptr))
            ++R.err_count;
        scaled_residual.push_back(normr / normr0);
        ++actualCgSets;
    }
    R.cg_sets = actualCgSets;

    // ---- TestNorms (src/main.cpp:532-556)
    trace.phase("hpcg:TestNorms");
    TestNormsData tn{};
    tn.samples = actualCgSets;
    tn.values = scaled_residual.data();
    TestNorms(tn);
    R.norms_mean = tn.mean;
    R.norms_variance = tn.variance;
    R.norms_pass = tn.pass ? 1 : 0;
    return hpcgb200_benchmark_report(&R, nullptr, 0, nullptr);
}

}  // namespace

extern "C" int hpcgb200_benchmark_run(const hpcgb200_benchmark_params* params, hpcgb200_benchmark_result* result)
{
    if(!params || !result) return hb::record_error(HPCGB200_ERR_ARG, "null argument");
    const bool keep = g_keep_generated;
    try
    {
        g_keep_generated = false;
        const int rc = run_protocol(*params, *result);
        g_keep_generated = keep;
        return rc;
    }
    catch(const Error& e)
    {
        g_keep_generated = keep;
        return report(e);
    }
    catch(const std::bad_alloc&)
    {
        g_keep_generated = keep;
        return hb::record_error(HPCGB200_ERR_CUDA, "host allocation failed");
    }
}
