// C ABI problem handle: the benchmark driver's set-up sequence
// (src/main.cpp:198-210 generation, src/main.cpp:355 OptimizeProblem) and
// its calls into CG / TestCG / TestSymmetry, for callers that are not C++.
#include <chrono>
#include <cmath>
#include <cstring>
#include <functional>
#include <string>

#include "hpcg_b200.h"
#include "internal.hpp"
#include "learned.hpp"
#include "problem.hpp"

using namespace hpcg_b200;

namespace hpcg_b200 {
extern bool g_keep_generated;
}



namespace {

MGPrecision prec_of(int mode)
{
    switch(mode)
    {
    case HPCGB200_MODE_MIXED: return MGPrecision::FP32;
    case HPCGB200_MODE_LEARNED: return MGPrecision::LEARNED;
    case HPCGB200_MODE_FP64_STENCIL: return MGPrecision::FP64_STENCIL;
    default: return MGPrecision::FP64;
    }
}

bool mode_ok(int mode)
{
    return mode == HPCGB200_MODE_FP64 || mode == HPCGB200_MODE_MIXED || mode == HPCGB200_MODE_LEARNED ||
           mode == HPCGB200_MODE_FP64_STENCIL;
}

bool flexible_of(int mode) { return needs_flexible(prec_of(mode)); }

// modes TestCG / TestSymmetry run with (the learned V-cycle is not symmetric)
bool test_mode_ok(int mode) { return mode_ok(mode) && mode != HPCGB200_MODE_LEARNED; }

SparseMatrix* level_of(const hpcgb200_problem* p, int level)
{
    if(!p || level < 0 || level >= (int)p->levels.size()) return nullptr;
    return p->levels[level];
}

struct FieldRef
{
    const void* ptr = nullptr;
    size_t bytes = 0;
    bool host = false;
};

FieldRef field_of(const hpcgb200_problem* p, int level, const std::string& f)
{
    FieldRef r;
    SparseMatrix* M = level_of(p, level);
    if(!M) return r;
    const size_t m = (size_t)M->localNumberOfRows;
    const LevelOpt* o = opt(*M);
    const MGOpt* mo = mgopt(*M);
    const size_t nc = M->Ac ? (size_t)M->Ac->localNumberOfRows : 0;
    auto set = [&](const void* ptr, size_t bytes, bool host = false) {
        r.ptr = ptr;
        r.bytes = ptr ? bytes : 0;
        r.host = host;
    };
    if(f == "perm") set(M->perm, m * 4);
    else if(f == "colors") set(o ? o->colors : nullptr, m * 4);
    else if(f == "ell_col") set(M->ell_col_ind, m * 27 * 4);
    else if(f == "ell_val") set(M->ell_val, m * 27 * 8);
    else if(f == "diag_idx") set(M->diag_idx, m * 4);
    else if(f == "inv_diag") set(M->inv_diag, m * 8);
    else if(f == "diag") set(o ? o->diag : nullptr, m * 8);
    else if(f == "diag32") set(o ? o->diag32 : nullptr, m * 4);
    else if(f == "inv_diag32") set(o ? o->inv_diag32 : nullptr, m * 4);
    else if(f == "f2c") set(M->mgData ? M->mgData->d_f2cOperator : nullptr, nc * 4);
    else if(f == "inj_f") set(mo ? mo->inj_f : nullptr, nc * 4);
    else if(f == "inj_c") set(mo ? mo->inj_c : nullptr, nc * 4);
    else if(f == "mtx_ind") set(M->d_mtxIndL, m * 27 * 4);
    else if(f == "values") set(M->d_matrixValues, m * 27 * 8);
    else if(f == "nnz_in_row") set(M->d_nonzerosInRow, m);
    else if(f == "hash") set(M->d_rowHash, m * 4);
    else if(f == "diag_slot") set(M->d_matrixDiagonal, m * 4);
    else if(f == "l2g") set(M->d_localToGlobalMap, m * 8);
    else if(f == "sizes") set(M->sizes, sizeof(int) * HPCGB200_MAX_COLORS, true);
    else if(f == "offsets") set(M->offsets, sizeof(int) * (HPCGB200_MAX_COLORS + 1), true);
    else if(f == "round_sizes") set(o ? o->round_sizes.data() : nullptr, o ? o->round_sizes.size() * 4 : 0, true);
    else if(level == 0 && f == "b") set(p->b.d_values, m * 8);
    else if(level == 0 && f == "xexact") set(p->xexact.d_values, m * 8);
    else if(level == 0 && f == "x") set(p->x.d_values, m * 8);
    return r;
}

}  // namespace

extern "C" int hpcgb200_problem_create_ex(int nx, int ny, int nz, int nlevels, int flags, hpcgb200_problem** out)
{
    if(!out) return hb::record_error(HPCGB200_ERR_ARG, "out is null");
    *out = nullptr;
    if(nx < 2 || ny < 2 || nz < 2 || nlevels < 1 || nlevels > 8)
        return hb::record_error(HPCGB200_ERR_ARG, "need dims >= 2 and 1 <= nlevels <= 8");
    const int div = 1 << (nlevels - 1);
    if(nx % div || ny % div || nz % div)
        return hb::record_error(HPCGB200_ERR_ARG, "dims must be divisible by 2^(nlevels-1) = %d", div);
    if((long long)nx * ny * nz > 0x7fffffffLL) return hb::record_error(HPCGB200_ERR_ARG, "grid exceeds 2^31 rows");
    auto* P = new hpcgb200_problem;
    const int rc = guarded([&] {
        g_keep_generated = (flags & HPCGB200_FLAG_KEEP_GENERATED) != 0;
        TracePhases trace;
        trace.phase("hpcg:GenerateProblem");
        const auto t0 = std::chrono::steady_clock::now();
        P->geom = new Geometry;
        GenerateGeometry(1, 0, 1, 0, 0, 0, nx, ny, nz, 1, 1, 1, P->geom);
        InitializeSparseMatrix(P->A, P->geom);
        GenerateProblem(P->A, &P->b, &P->x, &P->xexact);
        SetupHalo(P->A);
        SparseMatrix* cur = &P->A;
        P->levels.push_back(cur);
        for(int l = 1; l < nlevels; ++l)
        {
            GenerateCoarseProblem(*cur);
            cur = cur->Ac;
            P->levels.push_back(cur);
        }
        HB_HOST_CUDA(cudaStreamSynchronize(rt().stream));
        const auto t1 = std::chrono::steady_clock::now();
        trace.phase("hpcg:OptimizeProblem");
        int r = OptimizeProblem(P->A, P->data, P->b, P->x, P->xexact);
        if(r) return r;
        HB_HOST_CUDA(cudaStreamSynchronize(rt().stream));
        const auto t2 = std::chrono::steady_clock::now();
        P->setup_s = std::chrono::duration<double>(t1 - t0).count();
        P->optimize_s = std::chrono::duration<double>(t2 - t1).count();
        P->nlevels = nlevels;
        P->b_generated = dalloc<double>(P->A.localNumberOfRows);
        HB_HOST_CUDA(cudaMemcpyAsync(P->b_generated, P->b.d_values, sizeof(double) * P->A.localNumberOfRows,
                                     cudaMemcpyDeviceToDevice, rt().stream));
        HB_HOST_CUDA(cudaStreamSynchronize(rt().stream));
        return 0;
    });
    g_keep_generated = false;
    if(rc)
    {
        hpcgb200_problem_destroy(P);
        return rc;
    }
    *out = P;
    return 0;
}

extern "C" int hpcgb200_problem_create(int nx, int ny, int nz, int nlevels, hpcgb200_problem** out)
{
    return hpcgb200_problem_create_ex(nx, ny, nz, nlevels, 0, out);
}

extern "C" int hpcgb200_problem_destroy(hpcgb200_problem* p)
{
    if(!p) return 0;
    try
    {
        if(rt().initialized) cudaStreamSynchronize(rt().stream);
        DeleteMatrix(p->A);
        CudaDeleteVector(p->b);
        CudaDeleteVector(p->x);
        CudaDeleteVector(p->xexact);
        CudaDeleteCGData(p->data);
        dfree(p->b_generated);
        if(p->geom)
        {
            DeleteGeometry(*p->geom);
            delete p->geom;
        }
    }
    catch(const Error&)
    {
    }
    delete p;
    return 0;
}

extern "C" int hpcgb200_problem_info(const hpcgb200_problem* p, int* nlevels, int* dims, int* rows, long long* nnz,
                                     int* nblocks)
{
    if(!p) return hb::record_error(HPCGB200_ERR_ARG, "null problem");
    if(nlevels) *nlevels = (int)p->levels.size();
    for(size_t l = 0; l < p->levels.size(); ++l)
    {
        const SparseMatrix* M = p->levels[l];
        if(dims)
        {
            dims[3 * l] = M->geom->nx;
            dims[3 * l + 1] = M->geom->ny;
            dims[3 * l + 2] = M->geom->nz;
        }
        if(rows) rows[l] = M->localNumberOfRows;
        if(nnz) nnz[l] = M->totalNumberOfNonzeros;
        if(nblocks) nblocks[l] = M->nblocks;
    }
    return 0;
}

extern "C" int hpcgb200_problem_setup_times(const hpcgb200_problem* p, double* setup_s, double* optimize_s)
{
    if(!p) return hb::record_error(HPCGB200_ERR_ARG, "null problem");
    if(setup_s) *setup_s = p->setup_s;
    if(optimize_s) *optimize_s = p->optimize_s;
    return 0;
}

extern "C" int hpcgb200_problem_stream(const hpcgb200_problem* p, void** stream)
{
    if(!p || !stream) return hb::record_error(HPCGB200_ERR_ARG, "null argument");
    *stream = rt().stream;
    return 0;
}

extern "C" int hpcgb200_problem_stencil_ok(const hpcgb200_problem* p, int level, int* ok)
{
    SparseMatrix* M = level_of(p, level);
    if(!M || !ok) return hb::record_error(HPCGB200_ERR_ARG, "bad level");
    *ok = opt(*M) && opt(*M)->stencil_ok ? 1 : 0;
    return 0;
}

extern "C" int hpcgb200_problem_copy_field(const hpcgb200_problem* p, int level, const char* field, void* host,
                                           size_t bytes)
{
    if(!p || !field || !host) return hb::record_error(HPCGB200_ERR_ARG, "null argument");
    return guarded([&] {
        FieldRef r = field_of(p, level, field);
        if(!r.ptr) return hb::record_error(HPCGB200_ERR_ARG, "field '%s' not available on level %d", field, level);
        if(bytes != r.bytes)
            return hb::record_error(HPCGB200_ERR_ARG, "field '%s': %zu bytes requested, %zu available", field, bytes,
                                    r.bytes);
        if(r.host) std::memcpy(host, r.ptr, bytes);
        else
        {
            HB_HOST_CUDA(cudaStreamSynchronize(rt().stream));
            HB_HOST_CUDA(cudaMemcpy(host, r.ptr, bytes, cudaMemcpyDeviceToHost));
        }
        return 0;
    });
}

extern "C" int hpcgb200_problem_field_bytes(const hpcgb200_problem* p, int level, const char* field, size_t* bytes)
{
    if(!p || !field || !bytes) return hb::record_error(HPCGB200_ERR_ARG, "null argument");
    FieldRef r = field_of(p, level, field);
    if(!r.ptr) return hb::record_error(HPCGB200_ERR_ARG, "field '%s' not available on level %d", field, level);
    *bytes = r.bytes;
    return 0;
}

extern "C" int hpcgb200_problem_device_field(const hpcgb200_problem* p, int level, const char* field, void** dev)
{
    if(!p || !field || !dev) return hb::record_error(HPCGB200_ERR_ARG, "null argument");
    FieldRef r = field_of(p, level, field);
    if(!r.ptr || r.host) return hb::record_error(HPCGB200_ERR_ARG, "no device field '%s' on level %d", field, level);
    *dev = const_cast<void*>(r.ptr);
    return 0;
}

extern "C" int hpcgb200_problem_set_rhs(hpcgb200_problem* p, const double* host_b_natural)
{
    if(!p) return hb::record_error(HPCGB200_ERR_ARG, "null problem");
    return guarded([&] {
        const int m = p->A.localNumberOfRows;
        cudaStream_t s = rt().stream;
        if(!host_b_natural)
        {
            HB_HOST_CUDA(cudaMemcpyAsync(p->b.d_values, p->b_generated, sizeof(double) * m, cudaMemcpyDeviceToDevice, s));
        }
        else
        {
            double* tmp = opt(p->A)->vec_scratch;
            HB_HOST_CUDA(cudaMemcpyAsync(tmp, host_b_natural, sizeof(double) * m, cudaMemcpyHostToDevice, s));
            check(hpcgb200_permute_vector(m, p->A.perm, tmp, p->b.d_values, s));
        }
        HB_HOST_CUDA(cudaStreamSynchronize(s));
        return 0;
    });
}

extern "C" int hpcgb200_problem_get_x(hpcgb200_problem* p, double* host_x_natural)
{
    if(!p || !host_x_natural) return hb::record_error(HPCGB200_ERR_ARG, "null argument");
    return guarded([&] {
        const int m = p->A.localNumberOfRows;
        cudaStream_t s = rt().stream;
        double* tmp = opt(p->A)->vec_scratch;
        check(hpcgb200_unpermute_vector(m, p->A.perm, p->x.d_values, tmp, s));
        HB_HOST_CUDA(cudaMemcpyAsync(host_x_natural, tmp, sizeof(double) * m, cudaMemcpyDeviceToHost, s));
        HB_HOST_CUDA(cudaStreamSynchronize(s));
        return 0;
    });
}


// The reference's CG returns 0 whatever the residual became; the problem
// API reports a non-finite end instead (the outputs are filled first).
static int finite_or_error(double normr, double normr0, int niters)
{
    if(std::isfinite(normr) && std::isfinite(normr0)) return 0;
    return hb::record_error(HPCGB200_ERR_NONFINITE, "CG ended with a non-finite residual (normr0 = %g, normr = %g "
                            "after %d iterations): check b and the operator data", normr0, normr, niters);
}

extern "C" int hpcgb200_problem_cg(hpcgb200_problem* p, int mode, int max_iter, double tol, int precond, int* niters,
                                   double* normr, double* normr0, double* normr_hist, double* seconds)
{
    if(!p || !niters || !normr || !normr0) return hb::record_error(HPCGB200_ERR_ARG, "null argument");
    if(!mode_ok(mode)) return hb::record_error(HPCGB200_ERR_ARG, "bad mode");
    return guarded([&] {
        CudaZeroVector(p->x);
        const int r = run_cg(p->A, p->data, p->b, p->x, max_iter, tol, *niters, *normr, *normr0, precond != 0,
                             prec_of(mode), flexible_of(mode), normr_hist, seconds);
        return r ? r : finite_or_error(*normr, *normr0, *niters);
    });
}

extern "C" int hpcgb200_problem_solve_host(hpcgb200_problem* p, int mode, const double* b_natural, double* x_natural,
                                           int max_iter, double tol, int* niters, double* normr, double* normr0,
                                           double* seconds)
{
    if(!p || !b_natural || !x_natural || !niters || !normr || !normr0)
        return hb::record_error(HPCGB200_ERR_ARG, "null argument");
    if(!mode_ok(mode)) return hb::record_error(HPCGB200_ERR_ARG, "bad mode");
    return guarded([&] {
        const auto t0 = std::chrono::steady_clock::now();
        const int m = p->A.localNumberOfRows;
        cudaStream_t s = rt().stream;
        double* tmp = opt(p->A)->vec_scratch;
        HB_HOST_CUDA(cudaMemcpyAsync(tmp, b_natural, sizeof(double) * m, cudaMemcpyHostToDevice, s));
        check(hpcgb200_permute_vector(m, p->A.perm, tmp, p->b.d_values, s));
        HB_HOST_CUDA(cudaMemsetAsync(p->x.d_values, 0, sizeof(double) * m, s));
        int r = run_cg(p->A, p->data, p->b, p->x, max_iter, tol, *niters, *normr, *normr0, true, prec_of(mode),
                       flexible_of(mode), nullptr, nullptr);
        if(r) return r;
        check(hpcgb200_unpermute_vector(m, p->A.perm, p->x.d_values, tmp, s));
        HB_HOST_CUDA(cudaMemcpyAsync(x_natural, tmp, sizeof(double) * m, cudaMemcpyDeviceToHost, s));
        HB_HOST_CUDA(cudaStreamSynchronize(s));
        if(seconds) *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        return finite_or_error(*normr, *normr0, *niters);
    });
}

// src/CG_ref.cpp on the problem's generated arrays (kept with
// HPCGB200_FLAG_KEEP_GENERATED): b is brought back to natural order, x is
// left in natural order.
extern "C" int hpcgb200_problem_cg_ref(hpcgb200_problem* p, int max_iter, double tol, int precond, int* niters,
                                       double* normr, double* normr0, double* seconds)
{
    if(!p || !niters || !normr || !normr0) return hb::record_error(HPCGB200_ERR_ARG, "null argument");
    if(max_iter < 0 || max_iter > 1000000) return hb::record_error(HPCGB200_ERR_ARG, "max_iter out of range");
    return guarded([&] {
        const int m = p->A.localNumberOfRows;
        Vector bn;
        CudaInitializeVector(bn, m);
        int rc = 0;
        try
        {
            check(hpcgb200_unpermute_vector(m, p->A.perm, p->b.d_values, bn.d_values, rt().stream));
            CudaZeroVector(p->x);
            double times[10] = {0};
            rc = CG_ref(p->A, p->data, bn, p->x, max_iter, tol, *niters, *normr, *normr0, times, precond != 0, false);
            if(seconds) *seconds = times[0];
        }
        catch(...)
        {
            CudaDeleteVector(bn);
            throw;
        }
        CudaDeleteVector(bn);
        return rc;
    });
}

// src/ComputeMG_ref.cpp on the problem's generated arrays: z = M^-1 r with
// r and z natural-order device vectors of level 0.
extern "C" int hpcgb200_problem_mg_ref(hpcgb200_problem* p, const double* r_natural, double* z_natural)
{
    if(!p || !r_natural || !z_natural || r_natural == z_natural)
        return hb::record_error(HPCGB200_ERR_ARG, "need distinct device vectors r and z");
    return guarded([&] {
        const int m = p->A.localNumberOfRows;
        Vector r, z;
        r.localLength = z.localLength = m;
        r.d_values = const_cast<double*>(r_natural);
        z.d_values = z_natural;
        const int rc = ComputeMG_ref(p->A, r, z);
        HB_HOST_CUDA(cudaStreamSynchronize(rt().stream));
        return rc;
    });
}

extern "C" int hpcgb200_problem_true_residual(hpcgb200_problem* p, double* rel)
{
    if(!p || !rel) return hb::record_error(HPCGB200_ERR_ARG, "null argument");
    return guarded([&] {
        const int m = p->A.localNumberOfRows;
        cudaStream_t s = rt().stream;
        double* ax = opt(p->A)->vec_scratch;
        HB_RETURN_IF(hb::launch_spmv(m, opt(p->A)->cc, p->A.ell_col_ind, p->A.ell_val, p->x.d_values, ax, s));
        HB_RETURN_IF(hb::launch_waxpby(m, 1.0, p->b.d_values, -1.0, ax, ax, s));
        HB_RETURN_IF(hb::launch_dot(m, ax, ax, rt().ws, rt().d_scalar, s));
        HB_RETURN_IF(hb::launch_dot(m, p->b.d_values, p->b.d_values, rt().ws, rt().d_scalar + 1, s));
        HB_HOST_CUDA(cudaMemcpyAsync(rt().h_scalar, rt().d_scalar, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
        HB_HOST_CUDA(cudaStreamSynchronize(s));
        *rel = std::sqrt(rt().h_scalar[0]) / std::sqrt(rt().h_scalar[1]);
        return 0;
    });
}

extern "C" int hpcgb200_problem_kernels_per_iteration(hpcgb200_problem* p, int mode, int precond, int* kernels)
{
    if(!p || !kernels) return hb::record_error(HPCGB200_ERR_ARG, "null argument");
    if(!mode_ok(mode)) return hb::record_error(HPCGB200_ERR_ARG, "bad mode");
    return guarded([&] {
        *kernels = iteration_kernels(p->A, p->data, p->b, p->x, precond != 0, prec_of(mode), flexible_of(mode));
        return 0;
    });
}

extern "C" int hpcgb200_problem_test_cg(hpcgb200_problem* p, int mode, int* out_niters, int* count_pass,
                                        int* count_fail)
{
    if(!p) return hb::record_error(HPCGB200_ERR_ARG, "null problem");
    if(!test_mode_ok(mode))
        return hb::record_error(HPCGB200_ERR_ARG, "mode must be HPCGB200_MODE_FP64, _MIXED or _FP64_STENCIL");
    TestCGData d{};
    const int rc = TestCG_B200(p->A, p->data, p->b, p->x, d, prec_of(mode));
    if(out_niters)
        for(int i = 0; i < 4; ++i) out_niters[i] = d.niters[i];
    if(count_pass) *count_pass = d.count_pass;
    if(count_fail) *count_fail = d.count_fail;
    return rc;
}

extern "C" int hpcgb200_problem_test_symmetry(hpcgb200_problem* p, int mode, double* depsym_spmv, double* depsym_mg,
                                              double* residual_inf)
{
    if(!p) return hb::record_error(HPCGB200_ERR_ARG, "null problem");
    if(!test_mode_ok(mode))
        return hb::record_error(HPCGB200_ERR_ARG, "mode must be HPCGB200_MODE_FP64, _MIXED or _FP64_STENCIL");
    TestSymmetryData d{};
    const int rc = TestSymmetry_B200(p->A, p->b, p->xexact, d, prec_of(mode));
    if(depsym_spmv) *depsym_spmv = d.depsym_spmv;
    if(depsym_mg) *depsym_mg = d.depsym_mg;
    if(residual_inf) *residual_inf = d.residual_inf;
    return rc;
}

static Vector wrap(const double* d, int n)
{
    Vector v;
    v.localLength = n;
    v.d_values = const_cast<double*>(d);
    return v;
}

extern "C" int hpcgb200_problem_spmv(hpcgb200_problem* p, int level, const double* x, double* y)
{
    SparseMatrix* M = level_of(p, level);
    if(!M || !x || !y) return hb::record_error(HPCGB200_ERR_ARG, "bad arguments");
    Vector xv = wrap(x, M->localNumberOfRows), yv = wrap(y, M->localNumberOfRows);
    return ComputeSPMV(*M, xv, yv);
}

extern "C" int hpcgb200_problem_spmv_stencil(hpcgb200_problem* p, int level, const double* x, double* y)
{
    SparseMatrix* M = level_of(p, level);
    if(!M || !x || !y) return hb::record_error(HPCGB200_ERR_ARG, "bad arguments");
    return guarded([&] {
        const LevelOpt* o = opt(*M);
        if(!o->stencil_ok) return hb::record_error(HPCGB200_ERR_NOT_STENCIL, "level %d is not the verified stencil", level);
        return hb::launch64_spmv_stencil(o->st, o->diag, x, y, rt().stream);
    });
}

extern "C" int hpcgb200_problem_spmv_mixed(hpcgb200_problem* p, int level, const double* x, double* y)
{
    SparseMatrix* M = level_of(p, level);
    if(!M || !x || !y) return hb::record_error(HPCGB200_ERR_ARG, "bad arguments");
    return guarded([&] {
        const LevelOpt* o = opt(*M);
        if(!o->stencil_ok) return hb::record_error(HPCGB200_ERR_NOT_STENCIL, "level %d is not the verified stencil", level);
        return hb::launch64_spmv_sep(o->st, o->diag, x, y, rt().stream);
    });
}

extern "C" int hpcgb200_problem_symgs(hpcgb200_problem* p, int level, const double* r, double* x)
{
    SparseMatrix* M = level_of(p, level);
    if(!M || !r || !x) return hb::record_error(HPCGB200_ERR_ARG, "bad arguments");
    Vector rv = wrap(r, M->localNumberOfRows), xv = wrap(x, M->localNumberOfRows);
    return ComputeSYMGS(*M, rv, xv);
}

extern "C" int hpcgb200_problem_symgs_zero(hpcgb200_problem* p, int level, const double* r, double* x)
{
    SparseMatrix* M = level_of(p, level);
    if(!M || !r || !x) return hb::record_error(HPCGB200_ERR_ARG, "bad arguments");
    Vector rv = wrap(r, M->localNumberOfRows), xv = wrap(x, M->localNumberOfRows);
    return ComputeSYMGSZeroGuess(*M, rv, xv);
}

extern "C" int hpcgb200_problem_mg(hpcgb200_problem* p, int mode, const double* r, double* x)
{
    if(!p || !r || !x) return hb::record_error(HPCGB200_ERR_ARG, "bad arguments");
    Vector rv = wrap(r, p->A.localNumberOfRows), xv = wrap(x, p->A.localNumberOfRows);
    if(!mode_ok(mode)) return hb::record_error(HPCGB200_ERR_ARG, "bad mode");
    if(mode == HPCGB200_MODE_LEARNED) return ComputeMG_Learned(p->A, rv, xv);
    if(mode == HPCGB200_MODE_FP64_STENCIL) return ComputeMG_Stencil(p->A, rv, xv);
    return mode == HPCGB200_MODE_MIXED ? ComputeMG_Mixed(p->A, rv, xv) : ComputeMG(p->A, rv, xv);
}

extern "C" int hpcgb200_problem_restrict(hpcgb200_problem* p, int level, const double* rf, const double* xf,
                                         double* rc)
{
    SparseMatrix* M = level_of(p, level);
    if(!M || !M->mgData || !rf || !xf || !rc) return hb::record_error(HPCGB200_ERR_ARG, "bad arguments");
    return guarded([&] {
        const MGOpt* mo = mgopt(*M);
        return hb::launch_restrict(M->Ac->localNumberOfRows, mo->inj_f, mo->inj_c, M->localNumberOfRows, M->ell_col_ind,
                                   M->ell_val, rf, xf, rc, rt().stream);
    });
}

extern "C" int hpcgb200_problem_prolong(hpcgb200_problem* p, int level, const double* xc, double* xf)
{
    SparseMatrix* M = level_of(p, level);
    if(!M || !M->mgData || !xc || !xf) return hb::record_error(HPCGB200_ERR_ARG, "bad arguments");
    return guarded([&] {
        const MGOpt* mo = mgopt(*M);
        return hb::launch_prolong(M->Ac->localNumberOfRows, mo->inj_f, mo->inj_c, xc, xf, rt().stream);
    });
}

extern "C" int hpcgb200_problem_time_op(hpcgb200_problem* p, const char* op, int n, double* ms_per_launch)
{
    if(!p || !op || n < 1 || !ms_per_launch) return hb::record_error(HPCGB200_ERR_ARG, "bad arguments");
    return guarded([&] {
        // "graph:<op>" captures one call of <op> into a CUDA graph and times
        // launches of that graph (the way the solver runs it)
        std::string o(op);
        const bool as_graph = o.rfind("graph:", 0) == 0;
        if(as_graph) o = o.substr(6);
        SparseMatrix& A = p->A;
        cudaStream_t s = rt().stream;
        Vector& r = p->data.r;
        Vector& z = p->data.z;
        int per_call = 1;
        std::function<int()> f;
        if(o == "spmv") f = [&] { return ComputeSPMV(A, p->data.p, p->data.Ap); };
        else if(o == "symgs" || o == "symgs_sweep")
        {
            f = [&] { return ComputeSYMGS(A, r, z); };
            if(o == "symgs_sweep") per_call = A.nblocks + A.ublocks + 1;
        }
        else if(o == "symgs_zero") f = [&] { return ComputeSYMGSZeroGuess(A, r, z); };
        else if(o == "mg") f = [&] { return ComputeMG(A, r, z); };
        else if(o == "mg_mixed") f = [&] { return ComputeMG_Mixed(A, r, z); };
        else if(o == "mg_stencil") f = [&] { return ComputeMG_Stencil(A, r, z); };
        else if(o == "mg_learned")
        {
            if(!opt(A)->smoother) return hb::record_error(HPCGB200_ERR_ARG, "time_op: no smoother attached");
            HB_RETURN_IF(smoother_ready(A, rt().stream));
            f = [&] { return ComputeMG_Learned(A, r, z); };
        }
        else if(o == "symgs32_sweep" || o == "spmv_stencil" || o == "spmv_mixed")
        {
            const LevelOpt* lo = opt(A);
            if(!lo->stencil_ok) return hb::record_error(HPCGB200_ERR_NOT_STENCIL, "level 0 is not the verified stencil");
            if(o == "spmv_stencil") f = [&, lo] { return hb::launch64_spmv_stencil(lo->st, lo->diag, p->data.p.d_values, p->data.Ap.d_values, s); };
            else if(o == "spmv_mixed") f = [&, lo] { return hb::launch64_spmv_sep(lo->st, lo->diag, p->data.p.d_values, p->data.Ap.d_values, s); };
            else
            {
                // one FP32 SymGS step on level 0 (15 colour launches), averaged per launch
                f = [&, lo] { return hb::launch32_symgs(lo->st, lo->inv_diag32, lo->r32, lo->z32, nullptr, s); };
                per_call = 15;
            }
        }
        else return hb::record_error(HPCGB200_ERR_ARG, "unknown op '%s'", op);
        struct GraphGuard
        {
            cudaGraph_t g = nullptr;
            cudaGraphExec_t exec = nullptr;
            ~GraphGuard()
            {
                if(exec) cudaGraphExecDestroy(exec);
                if(g) cudaGraphDestroy(g);
            }
        } gg;
        if(as_graph)
        {
            HB_HOST_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            const int rc = f();
            const cudaError_t e = cudaStreamEndCapture(s, &gg.g);
            HB_RETURN_IF(rc);
            HB_HOST_CUDA(e);
            HB_HOST_CUDA(cudaGraphInstantiate(&gg.exec, gg.g, 0));
            f = [&] {
                HB_CUDA(cudaGraphLaunch(gg.exec, s));
                return 0;
            };
        }
        HB_RETURN_IF(f());  // warm-up
        cudaEvent_t e0, e1;
        HB_HOST_CUDA(cudaEventCreate(&e0));
        HB_HOST_CUDA(cudaEventCreate(&e1));
        HB_HOST_CUDA(cudaEventRecord(e0, s));
        for(int i = 0; i < n; ++i) HB_RETURN_IF(f());
        HB_HOST_CUDA(cudaEventRecord(e1, s));
        HB_HOST_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        HB_HOST_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        *ms_per_launch = ms / (double)(n * per_call);
        return 0;
    });
}
