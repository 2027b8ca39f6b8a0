// C++ operator API of the B200 HPCG drop-in.
//
// Types and functions keep the reference's names, fields and signatures
// (rocHPCG 0.8.9: src/SparseMatrix.hpp:75-156, src/Vector.hpp:59-69,
// src/MGData.hpp:59-74, src/CGData.hpp:55-60, src/Geometry.hpp:29-72 and the
// Compute*.hpp headers) so that a caller of the reference's hot path -- the
// benchmark driver, TestCG, TestSymmetry -- compiles against this header
// unchanged.  Device work goes through the C ABI in include/hpcg_b200.h.
//
// Conventions that differ from the reference and why:
//  * 1 rank only: local == global column ids, ExchangeHalo is a no-op.
//  * d_mtxIndL holds the generated columns directly (the reference keeps
//    int64 global ids in d_mtxIndG and copies them in SetupHalo).
//  * Implementation state (FP32 copies, transfer indices, cached CUDA graphs)
//    hangs off the `optimizationData` pointers, as HPCG intends.
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

typedef int local_int_t;
typedef long long global_int_t;

struct Geometry_STRUCT
{
    int size;
    int rank;
    int numThreads;
    local_int_t nx, ny, nz;
    int npx, npy, npz;
    int pz;
    int npartz;
    int* partz_ids;
    local_int_t* partz_nz;
    int ipx, ipy, ipz;
    global_int_t gnx, gny, gnz;
    global_int_t gix0, giy0, giz0;
};
typedef struct Geometry_STRUCT Geometry;

struct Vector_STRUCT
{
    local_int_t localLength = 0;
    double* values = nullptr;          // host copy (optional)
    void* optimizationData = nullptr;
    double* d_values = nullptr;        // device values
};
typedef struct Vector_STRUCT Vector;

struct MGData_STRUCT
{
    int numberOfPresmootherSteps;
    int numberOfPostsmootherSteps;
    local_int_t* f2cOperator;          // host copy (optional)
    Vector* rc;
    Vector* xc;
    Vector* Axf;
    void* optimizationData;            // MGOpt (transfer indices, FP32 vectors)
    local_int_t* d_f2cOperator;
    local_int_t* d_c2fOperator;
};
typedef struct MGData_STRUCT MGData;

struct SparseMatrix_STRUCT
{
    char* title;
    Geometry* geom;
    global_int_t totalNumberOfRows;
    global_int_t totalNumberOfNonzeros;
    local_int_t localNumberOfRows;
    local_int_t localNumberOfColumns;
    local_int_t localNumberOfNonzeros;
    local_int_t numberOfNonzerosPerRow;
    mutable bool isDotProductOptimized;
    mutable bool isSpmvOptimized;
    mutable bool isMgOptimized;
    mutable bool isWaxpbyOptimized;
    mutable struct SparseMatrix_STRUCT* Ac;
    mutable MGData* mgData;
    void* optimizationData;            // LevelOpt

    // generated row-major arrays (src/GenerateProblem.cpp)
    char* d_nonzerosInRow;
    local_int_t* d_mtxIndL;
    double* d_matrixValues;
    local_int_t* d_matrixDiagonal;
    global_int_t* d_localToGlobalMap;
    local_int_t* d_rowHash;

    // ELL (src/SparseMatrix.hpp:131-141)
    local_int_t ell_width;
    local_int_t* ell_col_ind;
    double* ell_val;
    local_int_t* diag_idx;
    double* inv_diag;

    // multicoloring (src/SparseMatrix.hpp:143-148)
    int nblocks;
    int ublocks;
    local_int_t* sizes;                // host arrays
    local_int_t* offsets;
    local_int_t* perm;                 // device
};
typedef struct SparseMatrix_STRUCT SparseMatrix;

struct CGData_STRUCT
{
    Vector r, z, p, Ap;
};
typedef struct CGData_STRUCT CGData;

struct TestCGData_STRUCT
{
    int count_pass;
    int count_fail;
    int expected_niters_no_prec;
    int expected_niters_prec;
    int niters_max_no_prec;
    int niters_max_prec;
    double normr;
    int niters[4];                     // per call (extension: lets tests see every count)
};
typedef struct TestCGData_STRUCT TestCGData;

struct TestSymmetryData_STRUCT
{
    double depsym_spmv;
    double depsym_mg;
    int count_fail;
    double residual_inf;               // ||A xexact - b||_inf of the last SpMV call
};
typedef struct TestSymmetryData_STRUCT TestSymmetryData;

struct TestNormsData_STRUCT
{
    double* values;
    double mean;
    double variance;
    int samples;
    bool pass;
};
typedef struct TestNormsData_STRUCT TestNormsData;

// Preconditioner precision of a solve (the FP64 outer recurrence is the same).
enum class MGPrecision
{
    FP64 = 0,    // the reference's optimized path, FP64 ELL
    FP32 = 1,    // FP32 vectors + FP32 accumulation, implicit stencil values
    LEARNED = 2,  // FP32 V-cycle whose coarse levels use the learned conv-net smoother
    FP64_STENCIL = 3  // FP64 V-cycle and SpMV on the implicit stencil: the FP64 path's bits, no matrix reads
};

// Preconditioners that need flexible (Polak-Ribiere) CG.
inline bool needs_flexible(MGPrecision p) { return p == MGPrecision::FP32 || p == MGPrecision::LEARNED; }

// ---------------------------------------------------------------- runtime
// One stream and one reduction workspace per process, like the reference's
// stream_interior / workspace globals (src/utils.hpp:38-45).
int HPCG_B200_Init(int device);
cudaStream_t HPCG_B200_Stream();
void HPCG_B200_SetStream(cudaStream_t s);
int HPCG_B200_Finalize();

// ------------------------------------------------------ problem set-up
void GenerateGeometry(int size, int rank, int numThreads, int pz, local_int_t zl, local_int_t zu, local_int_t nx,
                      local_int_t ny, local_int_t nz, int npx, int npy, int npz, Geometry* geom);
void InitializeSparseMatrix(SparseMatrix& A, Geometry* geom);
void GenerateProblem(SparseMatrix& A, Vector* b, Vector* x, Vector* xexact);
void SetupHalo(SparseMatrix& A);
void GenerateCoarseProblem(const SparseMatrix& Af);
int OptimizeProblem(SparseMatrix& A, CGData& data, Vector& b, Vector& x, Vector& xexact);
void DeleteMatrix(SparseMatrix& A);
void DeleteGeometry(Geometry& geom);

// ------------------------------------------------------------- vectors
void CudaInitializeVector(Vector& v, local_int_t localLength);
void CudaDeleteVector(Vector& v);
void CudaZeroVector(Vector& v);
void CudaCopyVector(const Vector& v, Vector& w);
void CudaFillRandomVector(Vector& v);   // rand()/RAND_MAX + 1, as src/Vector.hpp:134-146
void CudaInitializeSparseCGData(SparseMatrix& A, CGData& data);
void CudaDeleteCGData(CGData& data);
void CudaCopyMatrixDiagonal(const SparseMatrix& A, Vector& diagonal);
void CudaReplaceMatrixDiagonal(SparseMatrix& A, const Vector& diagonal);

// ----------------------------------------------------------- operators
void ExchangeHalo(const SparseMatrix& A, Vector& x);
int ComputeSPMV(const SparseMatrix& A, Vector& x, Vector& y);
int ComputeSYMGS(const SparseMatrix& A, const Vector& r, Vector& x);
int ComputeSYMGSZeroGuess(const SparseMatrix& A, const Vector& r, Vector& x);
int ComputeMG(const SparseMatrix& A, const Vector& r, Vector& x);
int ComputeRestriction(const SparseMatrix& A, const Vector& rf);
int ComputeFusedSpMVRestriction(const SparseMatrix& A, const Vector& rf, Vector& xf);
int ComputeProlongation(const SparseMatrix& Af, Vector& xf);
int ComputeDotProduct(local_int_t n, const Vector& x, const Vector& y, double& result, double& time_allreduce,
                      bool& isOptimized);
int ComputeWAXPBY(local_int_t n, double alpha, const Vector& x, double beta, const Vector& y, Vector& w,
                  bool& isOptimized);
int ComputeFusedWAXPBYDot(local_int_t n, double alpha, const Vector& x, Vector& y, double& result,
                          double& time_allreduce);
int ComputeResidual(local_int_t n, const Vector& v1, const Vector& v2, double& residual);

// FP32 V-cycle on FP64 vectors (no reference counterpart): z = M32^{-1} r.
int ComputeMG_Mixed(const SparseMatrix& A, const Vector& r, Vector& x);
// FP32 V-cycle with the learned smoother attached to A (no reference
// counterpart): on levels >= its first level the conv net replaces the pre-
// and post-smoothing SymGS (x = N(r); ...; x += N(r - A x)) and the coarsest
// solve.  Nonlinear and non-symmetric: use it inside flexible CG.
int ComputeMG_Learned(const SparseMatrix& A, const Vector& r, Vector& x);
// ComputeMG on the implicit stencil (no reference counterpart): the same
// operations in the same order as ComputeMG, so z is bitwise the same, with
// no matrix reads on levels whose colour bricks are 4-aligned (the others
// use the ELL kernels).
int ComputeMG_Stencil(const SparseMatrix& A, const Vector& r, Vector& x);

// --------------------------------------------------------------- solver
int CG(const SparseMatrix& A, CGData& data, const Vector& b, Vector& x, const int max_iter, const double tolerance,
       int& niters, double& normr, double& normr0, double* times, bool doPreconditioning, bool verbose);
// Same recurrence with a selectable preconditioner precision and, for the
// mixed/learned preconditioners, flexible (Polak-Ribiere) beta.  No reference
// counterpart.  normr_hist (optional) gets max_iter+1 entries.
int CG_B200(const SparseMatrix& A, CGData& data, const Vector& b, Vector& x, int max_iter, double tolerance,
            int& niters, double& normr, double& normr0, double* times, bool doPreconditioning, MGPrecision prec,
            bool flexible, double* normr_hist);

// ---------------------------------------------------------- validation
int TestCG(SparseMatrix& A, CGData& data, Vector& b, Vector& x, TestCGData& testcg_data);
int TestCG_B200(SparseMatrix& A, CGData& data, Vector& b, Vector& x, TestCGData& testcg_data, MGPrecision prec);
int TestSymmetry(SparseMatrix& A, Vector& b, Vector& xexact, TestSymmetryData& testsymmetry_data);
int TestSymmetry_B200(SparseMatrix& A, Vector& b, Vector& xexact, TestSymmetryData& testsymmetry_data,
                      MGPrecision prec);
int TestNorms(TestNormsData& testnorms_data);

// -------------------------------------------------- reference routines
// The benchmark's `_ref` routines (src/*_ref.cpp, src/CheckProblem.cpp) on
// the device: natural row order on the generated row-major arrays, so they
// apply between GenerateCoarseProblem and OptimizeProblem (or later on a
// hierarchy that keeps its generated arrays).  SpMV and SymGS results equal
// the sequential C loops bit for bit.
int ComputeSPMV_ref(const SparseMatrix& A, Vector& x, Vector& y);
int ComputeSYMGS_ref(const SparseMatrix& A, const Vector& r, Vector& x);
int ComputeMG_ref(const SparseMatrix& A, const Vector& r, Vector& x);
int ComputeRestriction_ref(const SparseMatrix& A, const Vector& rf);
int ComputeProlongation_ref(const SparseMatrix& Af, Vector& xf);
int ComputeDotProduct_ref(local_int_t n, const Vector& x, const Vector& y, double& result, double& time_allreduce);
int ComputeWAXPBY_ref(local_int_t n, double alpha, const Vector& x, double beta, const Vector& y, Vector& w);
int CG_ref(const SparseMatrix& A, CGData& data, const Vector& b, Vector& x, const int max_iter, const double tolerance,
           int& niters, double& normr, double& normr0, double* times, bool doPreconditioning, bool verbose);
// CheckProblem as a count: rows whose entries, b, x or xexact differ from the
// generated stencil problem, plus one if the nonzero total disagrees.
long long CheckProblem_B200(const SparseMatrix& A, const Vector* b, const Vector* x, const Vector* xexact);

// HPCG flop / memory-traffic model per CG iteration (src/ReportResults.cpp:
// 134-195 with numberOfCgSets = 1, optMaxIters = 1, preamble excluded).
struct HpcgModel
{
    double flops_per_iter;
    double bytes_per_iter;
};
HpcgModel ComputeHpcgModel(const SparseMatrix& A, int numberOfMgLevels);
