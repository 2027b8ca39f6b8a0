// Validation protocol pieces: TestCG (src/TestCG.cpp:111-177), TestSymmetry
// (src/TestSymmetry.cpp:88-166), TestNorms (src/TestNorms.cpp:31-46) and the
// HPCG flop / memory model (src/ReportResults.cpp:134-195).
#include <cfloat>
#include <cmath>

#include "hpcg_b200.h"
#include "internal.hpp"

using namespace hpcg_b200;


int TestCG_B200(SparseMatrix& A, CGData& data, Vector& b, Vector& x, TestCGData& d, MGPrecision prec)
{
    try
    {
        ensure_runtime();
        cudaStream_t s = rt().stream;
        const local_int_t m = A.localNumberOfRows;
        Vector origDiagA, exaggeratedDiagA, origB;
        CudaInitializeVector(origDiagA, m);
        CudaInitializeVector(exaggeratedDiagA, m);
        CudaInitializeVector(origB, m);
        CudaCopyMatrixDiagonal(A, origDiagA);
        CudaCopyVector(b, origB);

        // kernel_scale_vector_values (src/TestCG.cpp:67-95) runs after
        // OptimizeProblem and indexes d_localToGlobalMap -- which is not
        // permuted -- with the permuted row id; reproduced as is, on the device.
        CudaCopyVector(origDiagA, exaggeratedDiagA);
        if(!A.d_localToGlobalMap) throw Error(HPCGB200_ERR_ARG, "TestCG: level has no local-to-global map");
        check(hpcgb200_testcg_scale(m, A.d_localToGlobalMap, exaggeratedDiagA.d_values, b.d_values, s));
        CudaReplaceMatrixDiagonal(A, exaggeratedDiagA);

        int niters = 0;
        double normr = 0.0, normr0 = 0.0;
        const int maxIters = 50;
        const int numberOfCgCalls = 2;
        const double tolerance = 1.0e-12;
        d.expected_niters_no_prec = 12;
        d.expected_niters_prec = 2;
        d.niters_max_no_prec = 0;
        d.niters_max_prec = 0;
        d.count_pass = d.count_fail = 0;
        int rc = 0;
        for(int k = 0; k < 2 && rc == 0; ++k)
        {
            const int expected = k == 0 ? d.expected_niters_no_prec : d.expected_niters_prec;
            for(int i = 0; i < numberOfCgCalls && rc == 0; ++i)
            {
                CudaZeroVector(x);
                rc = CG_B200(A, data, b, x, maxIters, tolerance, niters, normr, normr0, nullptr, k == 1, prec,
                             needs_flexible(prec), nullptr);
                d.niters[k * 2 + i] = niters;
                if(niters <= expected) ++d.count_pass;
                else ++d.count_fail;
                if(k == 0 && niters > d.niters_max_no_prec) d.niters_max_no_prec = niters;
                if(k == 1 && niters > d.niters_max_prec) d.niters_max_prec = niters;
            }
        }
        CudaReplaceMatrixDiagonal(A, origDiagA);
        CudaCopyVector(origB, b);
        HB_HOST_CUDA(cudaStreamSynchronize(s));
        CudaDeleteVector(origDiagA);
        CudaDeleteVector(exaggeratedDiagA);
        CudaDeleteVector(origB);
        d.normr = normr;
        return rc;
    }
    catch(const Error& e)
    {
        return report(e);
    }
}

int TestCG(SparseMatrix& A, CGData& data, Vector& b, Vector& x, TestCGData& d)
{
    return TestCG_B200(A, data, b, x, d, MGPrecision::FP64);
}

int TestSymmetry_B200(SparseMatrix& A, Vector& b, Vector& xexact, TestSymmetryData& d, MGPrecision prec)
{
    const local_int_t nrow = A.localNumberOfRows;
    const local_int_t ncol = A.localNumberOfColumns;
    Vector x_ncol, y_ncol, z_ncol;
    try
    {
        CudaInitializeVector(x_ncol, ncol);
        CudaInitializeVector(y_ncol, ncol);
        CudaInitializeVector(z_ncol, ncol);
    }
    catch(const Error& e)
    {
        return report(e);
    }
    double t4 = 0.0;
    bool opt_flag = true;
    d.count_fail = 0;
    CudaFillRandomVector(x_ncol);
    CudaFillRandomVector(y_ncol);
    double xNorm2, yNorm2;
    const double ANorm = 2 * 26.0;
    int ierr = 0;

    // x'Ay vs y'Ax
    ierr |= ComputeDotProduct(nrow, y_ncol, y_ncol, yNorm2, t4, opt_flag);
    ierr |= ComputeSPMV(A, y_ncol, z_ncol);
    double xtAy = 0.0;
    ierr |= ComputeDotProduct(nrow, x_ncol, z_ncol, xtAy, t4, opt_flag);
    ierr |= ComputeDotProduct(nrow, x_ncol, x_ncol, xNorm2, t4, opt_flag);
    ierr |= ComputeSPMV(A, x_ncol, z_ncol);
    double ytAx = 0.0;
    ierr |= ComputeDotProduct(nrow, y_ncol, z_ncol, ytAx, t4, opt_flag);
    d.depsym_spmv = std::fabs((long double)(xtAy - ytAx)) / ((xNorm2 * ANorm * yNorm2 + yNorm2 * ANorm * xNorm2) * (DBL_EPSILON));
    if(d.depsym_spmv > 1.0) ++d.count_fail;

    // x'M^{-1}y vs y'M^{-1}x
    auto mg = [&](const Vector& r, Vector& z) {
        if(prec == MGPrecision::FP64) return ComputeMG(A, r, z);
        if(prec == MGPrecision::FP64_STENCIL) return ComputeMG_Stencil(A, r, z);
        return ComputeMG_Mixed(A, r, z);
    };
    ierr |= mg(y_ncol, z_ncol);
    double xtMinvy = 0.0;
    ierr |= ComputeDotProduct(nrow, x_ncol, z_ncol, xtMinvy, t4, opt_flag);
    ierr |= mg(x_ncol, z_ncol);
    double ytMinvx = 0.0;
    ierr |= ComputeDotProduct(nrow, y_ncol, z_ncol, ytMinvx, t4, opt_flag);
    d.depsym_mg = std::fabs((long double)(xtMinvy - ytMinvx)) / ((xNorm2 * ANorm * yNorm2 + yNorm2 * ANorm * xNorm2) * (DBL_EPSILON));
    // an FP32 V-cycle is symmetric to single-precision rounding: the same
    // departure (still reported in DBL_EPSILON units) is held to FLT_EPSILON
    const double mg_limit = needs_flexible(prec) ? (double)FLT_EPSILON / DBL_EPSILON : 1.0;
    if(d.depsym_mg > mg_limit) ++d.count_fail;

    // ||A xexact - b||_inf, twice (src/TestSymmetry.cpp:150-160)
    CudaCopyVector(xexact, x_ncol);
    double residual = 0.0;
    for(int i = 0; i < 2; ++i)
    {
        ierr |= ComputeSPMV(A, x_ncol, z_ncol);
        ierr |= ComputeResidual(A.localNumberOfRows, b, z_ncol, residual);
    }
    d.residual_inf = residual;
    cudaStreamSynchronize(rt().stream);
    CudaDeleteVector(x_ncol);
    CudaDeleteVector(y_ncol);
    CudaDeleteVector(z_ncol);
    return ierr;
}

int TestSymmetry(SparseMatrix& A, Vector& b, Vector& xexact, TestSymmetryData& d)
{
    return TestSymmetry_B200(A, b, xexact, d, MGPrecision::FP64);
}

int TestNorms(TestNormsData& t)
{
    double mean_delta = 0.0;
    for(int i = 0; i < t.samples; ++i) mean_delta += (t.values[i] - t.values[0]);
    const double mean = t.values[0] + mean_delta / (double)t.samples;
    t.mean = mean;
    double sumdiff = 0.0;
    for(int i = 0; i < t.samples; ++i) sumdiff += (t.values[i] - mean) * (t.values[i] - mean);
    t.variance = sumdiff / (double)t.samples;
    t.pass = (t.variance < 1.0e-6);
    return 0;
}

HpcgModel ComputeHpcgModel(const SparseMatrix& A, int numberOfMgLevels)
{
    // Per CG iteration: 3 ddots, 3 WAXPBYs, 1 SpMV, MG (1 pre + 1 post SymGS,
    // residual) on levels 0..L-2 and one SymGS on the coarsest level.
    const double fnrow = (double)A.totalNumberOfRows;
    const double fnnz = (double)A.totalNumberOfNonzeros;
    const double dsz = 8.0, isz = 4.0;
    double flops = 3 * 2 * fnrow + 3 * 2 * fnrow + 2 * fnnz;
    double reads = 3 * 2 * fnrow * dsz + 3 * 2 * fnrow * dsz + (fnnz * (dsz + isz) + fnrow * dsz);
    double writes = 3 * dsz + 3 * fnrow * dsz + fnrow * dsz;
    const SparseMatrix* Af = &A;
    for(int i = 1; i < numberOfMgLevels && Af->mgData; ++i)
    {
        const double nnz = (double)Af->totalNumberOfNonzeros, nrow = (double)Af->totalNumberOfRows;
        const double pre = Af->mgData->numberOfPresmootherSteps, post = Af->mgData->numberOfPostsmootherSteps;
        flops += pre * 4 * nnz + 2 * nnz + post * 4 * nnz;
        reads += pre * (2 * nnz * (dsz + isz) + nrow * dsz);
        writes += pre * nrow * dsz;
        reads += nnz * (dsz + isz) + nrow * dsz;
        writes += nnz * dsz;
        reads += post * (2 * nnz * (dsz + isz) + nrow * dsz);
        writes += post * nnz * dsz;
        Af = Af->Ac;
    }
    const double nnz = (double)Af->totalNumberOfNonzeros, nrow = (double)Af->totalNumberOfRows;
    flops += 4 * nnz;
    reads += 2 * nnz * (dsz + isz) + nrow * dsz;
    writes += nrow * dsz;
    return HpcgModel{flops, reads + writes};
}
