// The benchmark's reference routines (src/ComputeSPMV_ref.cpp,
// src/ComputeSYMGS_ref.cpp, src/ComputeMG_ref.cpp,
// src/ComputeRestriction_ref.cpp, src/ComputeProlongation_ref.cpp,
// src/ComputeDotProduct_ref.cpp, src/ComputeWAXPBY_ref.cpp, src/CG_ref.cpp,
// src/CheckProblem.cpp) with their signatures, on the device vectors
// (d_values) in natural row order and the generated row-major arrays -- the
// state the driver calls them in, between GenerateCoarseProblem and
// OptimizeProblem.  The reference runs them on host copies; here the
// Gauss-Seidel sweep runs as wavefronts with the sequential sweep's per-row
// arithmetic (natural.cuh), so the SpMV and SymGS results are bitwise those
// of the sequential C code, and dot products differ from an OpenMP reduction
// only in summation order.
#include <chrono>
#include <cmath>
#include <cstdio>

#include "../csrc/natural.cuh"
#include "hpcg_b200.h"
#include "internal.hpp"

using namespace hpcg_b200;

namespace {

hb::NaturalLevel natural(const SparseMatrix& A)
{
    if(!A.d_mtxIndL || !A.d_matrixValues || !A.d_nonzerosInRow || !A.d_matrixDiagonal)
        throw Error(HPCGB200_ERR_ARG,
                    "reference routine: the generated row-major arrays are gone (they are freed by OptimizeProblem "
                    "unless the problem keeps them)");
    return hb::NaturalLevel{A.geom->nx,      A.geom->ny,
                            A.geom->nz,      A.d_mtxIndL,
                            A.d_matrixValues, reinterpret_cast<const int8_t*>(A.d_nonzerosInRow),
                            A.d_matrixDiagonal};
}

double read_scalar0()
{
    Runtime& R = rt();
    HB_HOST_CUDA(cudaMemcpyAsync(R.h_scalar, R.d_scalar, sizeof(double), cudaMemcpyDeviceToHost, R.stream));
    HB_HOST_CUDA(cudaStreamSynchronize(R.stream));
    return R.h_scalar[0];
}

double now() { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); }

}  // namespace

// src/ComputeSPMV_ref.cpp:48-75
int ComputeSPMV_ref(const SparseMatrix& A, Vector& x, Vector& y)
{
    return guarded([&] {
        if(A.mgData && &y == A.mgData->Axf && !y.d_values) CudaInitializeVector(y, A.localNumberOfColumns);
        return hb::launch_nat_spmv(natural(A), x.d_values, y.d_values, rt().stream);
    });
}

// src/ComputeSYMGS_ref.cpp:51-104
int ComputeSYMGS_ref(const SparseMatrix& A, const Vector& r, Vector& x)
{
    return guarded([&] { return hb::launch_nat_symgs(natural(A), r.d_values, x.d_values, rt().stream); });
}

// src/ComputeRestriction_ref.cpp:41-56
int ComputeRestriction_ref(const SparseMatrix& A, const Vector& rf)
{
    return guarded([&] {
        const MGData* mg = A.mgData;
        if(!mg) throw Error(HPCGB200_ERR_ARG, "ComputeRestriction_ref: level has no coarse grid");
        return hb::launch_nat_restrict(mg->rc->localLength, mg->d_f2cOperator, rf.d_values, mg->Axf->d_values,
                                       mg->rc->d_values, rt().stream);
    });
}

// src/ComputeProlongation_ref.cpp:41-56
int ComputeProlongation_ref(const SparseMatrix& Af, Vector& xf)
{
    return guarded([&] {
        const MGData* mg = Af.mgData;
        if(!mg) throw Error(HPCGB200_ERR_ARG, "ComputeProlongation_ref: level has no coarse grid");
        return hb::launch_nat_prolong(mg->rc->localLength, mg->d_f2cOperator, mg->xc->d_values, xf.d_values,
                                      rt().stream);
    });
}

// src/ComputeMG_ref.cpp:37-62
int ComputeMG_ref(const SparseMatrix& A, const Vector& r, Vector& x)
{
    HB_RETURN_IF(guarded([&] {
        CudaZeroVector(x);
        return 0;
    }));
    int ierr = 0;
    if(A.mgData)
    {
        for(int i = 0; i < A.mgData->numberOfPresmootherSteps; ++i) ierr += ComputeSYMGS_ref(A, r, x);
        if(ierr) return ierr;
        HB_RETURN_IF(ComputeSPMV_ref(A, x, *A.mgData->Axf));
        HB_RETURN_IF(ComputeRestriction_ref(A, r));
        HB_RETURN_IF(ComputeMG_ref(*A.Ac, *A.mgData->rc, *A.mgData->xc));
        HB_RETURN_IF(ComputeProlongation_ref(A, x));
        for(int i = 0; i < A.mgData->numberOfPostsmootherSteps; ++i) ierr += ComputeSYMGS_ref(A, r, x);
        return ierr;
    }
    return ComputeSYMGS_ref(A, r, x);
}

// src/ComputeDotProduct_ref.cpp:46-80 (one rank: no allreduce)
int ComputeDotProduct_ref(local_int_t n, const Vector& x, const Vector& y, double& result, double& time_allreduce)
{
    time_allreduce += 0.0;
    return guarded([&] {
        HB_RETURN_IF(hb::launch_nat_dot(n, x.d_values, y.d_values, rt().ws, rt().d_scalar, rt().stream));
        result = read_scalar0();
        return 0;
    });
}

// src/ComputeWAXPBY_ref.cpp:54-88
int ComputeWAXPBY_ref(local_int_t n, double alpha, const Vector& x, double beta, const Vector& y, Vector& w)
{
    return guarded([&] {
        if(n == 0) return 0;
        return hb::launch_nat_waxpby(n, alpha, x.d_values, beta, y.d_values, w.d_values, rt().stream);
    });
}

// src/CG_ref.cpp:60-160: the recurrence, operator order and timing slots of
// the reference CG (times[1] dots, [2] WAXPBY, [3] SpMV, [5] MG, [0] total;
// every phase is synchronised so the split is meaningful).
int CG_ref(const SparseMatrix& A, CGData& data, const Vector& b, Vector& x, const int max_iter,
           const double tolerance, int& niters, double& normr, double& normr0, double* times, bool doPreconditioning,
           bool verbose)
{
    try
    {
        ensure_runtime();
        cudaStream_t s = rt().stream;
        auto sync = [&] { HB_HOST_CUDA(cudaStreamSynchronize(s)); };
        const double t_begin = now();
        double t0 = 0, t1 = 0, t2 = 0, t3 = 0, t4 = 0, t5 = 0;
        auto tick = [&] { t0 = now(); };
        auto tock = [&](double& t) {
            sync();
            t += now() - t0;
        };
        normr = 0.0;
        double rtz = 0.0, oldrtz = 0.0, alpha = 0.0, beta = 0.0, pAp = 0.0;
        const local_int_t nrow = A.localNumberOfRows;
        Vector& r = data.r;
        Vector& z = data.z;
        Vector& p = data.p;
        Vector& Ap = data.Ap;

        CudaCopyVector(x, p);
        tick();
        HB_RETURN_IF(ComputeSPMV_ref(A, p, Ap));
        tock(t3);
        tick();
        HB_RETURN_IF(ComputeWAXPBY_ref(nrow, 1.0, b, -1.0, Ap, r));
        tock(t2);
        tick();
        HB_RETURN_IF(ComputeDotProduct_ref(nrow, r, r, normr, t4));
        tock(t1);
        normr = std::sqrt(normr);
        if(verbose) std::printf("REFERENCE Initial Residual = %le\n", normr);
        normr0 = normr;
        niters = 0;

        for(int k = 1; k <= max_iter && normr / normr0 > tolerance; k++)
        {
            tick();
            if(doPreconditioning) HB_RETURN_IF(ComputeMG_ref(A, r, z));
            else HB_RETURN_IF(ComputeWAXPBY_ref(nrow, 1.0, r, 0.0, r, z));
            tock(t5);
            if(k == 1)
            {
                CudaCopyVector(z, p);
                tock(t2);
                tick();
                HB_RETURN_IF(ComputeDotProduct_ref(nrow, r, z, rtz, t4));
                tock(t1);
            }
            else
            {
                oldrtz = rtz;
                tick();
                HB_RETURN_IF(ComputeDotProduct_ref(nrow, r, z, rtz, t4));
                tock(t1);
                beta = rtz / oldrtz;
                tick();
                HB_RETURN_IF(ComputeWAXPBY_ref(nrow, 1.0, z, beta, p, p));
                tock(t2);
            }
            tick();
            HB_RETURN_IF(ComputeSPMV_ref(A, p, Ap));
            tock(t3);
            tick();
            HB_RETURN_IF(ComputeDotProduct_ref(nrow, p, Ap, pAp, t4));
            tock(t1);
            alpha = rtz / pAp;
            tick();
            HB_RETURN_IF(ComputeWAXPBY_ref(nrow, 1.0, x, alpha, p, x));
            HB_RETURN_IF(ComputeWAXPBY_ref(nrow, 1.0, r, -alpha, Ap, r));
            tock(t2);
            tick();
            HB_RETURN_IF(ComputeDotProduct_ref(nrow, r, r, normr, t4));
            tock(t1);
            normr = std::sqrt(normr);
            if(verbose) std::printf("REFERENCE Iteration = %d   Scaled Residual = %le\n", k, normr / normr0);
            niters = k;
        }
        if(times)
        {
            times[1] += t1;
            times[2] += t2;
            times[3] += t3;
            times[4] += t4;
            times[5] += t5;
            times[0] += now() - t_begin;
        }
        return 0;
    }
    catch(const Error& e)
    {
        return report(e);
    }
}

// src/CheckProblem.cpp:79-150, counting mismatching rows instead of asserting.
long long CheckProblem_B200(const SparseMatrix& A, const Vector* b, const Vector* x, const Vector* xexact)
{
    ensure_runtime();
    cudaStream_t s = rt().stream;
    const Geometry& g = *A.geom;
    unsigned long long* cnt = dalloc<unsigned long long>(2);
    long long bad = -1;
    try
    {
        HB_HOST_CUDA(cudaMemsetAsync(cnt, 0, 2 * sizeof(unsigned long long), s));
        check(hb::launch_nat_check(natural(A), g.gnx, g.gny, g.gnz, g.gix0, g.giy0, g.giz0, A.d_localToGlobalMap,
                                   b ? b->d_values : nullptr, x ? x->d_values : nullptr,
                                   xexact ? xexact->d_values : nullptr, cnt, cnt + 1, s));
        unsigned long long h[2] = {0, 0};
        HB_HOST_CUDA(cudaMemcpyAsync(h, cnt, sizeof(h), cudaMemcpyDeviceToHost, s));
        HB_HOST_CUDA(cudaStreamSynchronize(s));
        bad = (long long)h[0] + ((long long)h[1] == A.localNumberOfNonzeros ? 0 : 1);
    }
    catch(...)
    {
        dfree(cnt);
        throw;
    }
    dfree(cnt);
    return bad;
}
