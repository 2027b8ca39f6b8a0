/*
 * Test-oracle glue around the reference's own CPU path (HPCG 3.1 `_ref`
 * kernels as shipped in rocHPCG 0.8.9).  TEST INFRASTRUCTURE ONLY: it is
 * linked into oracle/_ref/libhpcg_ref.so by oracle/Makefile together with the
 * unmodified reference sources and is loaded by the tests and by bench.py's
 * CPU-baseline leg, never by the product library.
 *
 * What it restates (because the reference has no CPU version of it):
 *   - the coarse-level builder of src/GenerateCoarseProblem.cpp:98-184
 *     (device code in the reference): f2c[ic] = 2izc*nxf*nyf + 2iyc*nxf + 2ixc
 *     (src/GenerateCoarseProblem.cpp:57-86), GenerateGeometry at half size,
 *     GenerateProblem_ref + SetupHalo_ref on it, rc/xc/Axf host vectors,
 *     1 pre + 1 post smoother step (src/MGData.hpp:85-86).
 * Everything numeric (CG_ref, ComputeMG_ref, ComputeSYMGS_ref, ComputeSPMV_ref,
 * restriction/prolongation, dot, WAXPBY, ComputeResidual_ref, CheckProblem,
 * TestNorms) is the reference's own compiled code.
 */
#include <cstring>
#include <fstream>
#include <vector>
#include <chrono>

#include "hpcg.hpp"
#include "Geometry.hpp"
#include "SparseMatrix.hpp"
#include "Vector.hpp"
#include "MGData.hpp"
#include "CGData.hpp"
#include "GenerateGeometry.hpp"
#include "GenerateProblem_ref.hpp"
#include "SetupHalo_ref.hpp"
#include "CheckProblem.hpp"
#include "CG_ref.hpp"
#include "ComputeSPMV_ref.hpp"
#include "ComputeSYMGS_ref.hpp"
#include "ComputeMG_ref.hpp"
#include "ComputeDotProduct_ref.hpp"
#include "ComputeWAXPBY_ref.hpp"
#include "ComputeResidual_ref.hpp"
#include "ComputeRestriction_ref.hpp"
#include "ComputeProlongation_ref.hpp"
#include "TestNorms.hpp"
#include "ComputeOptimalShapeXYZ.hpp"

// Globals the reference headers declare (src/utils.hpp:38-45, src/hpcg.hpp).
std::ofstream HPCG_fout;
hipStream_t stream_interior = nullptr;
hipStream_t stream_halo = nullptr;
hipEvent_t halo_gather = nullptr;
void* workspace = nullptr;
hipError_t deviceMalloc(void** ptr, size_t) { *ptr = nullptr; return hipSuccess; }
hipError_t deviceFree(void*) { return hipSuccess; }
hipError_t deviceRealloc(void*, size_t) { return hipSuccess; }
hipError_t deviceDefrag(void**, size_t) { return hipSuccess; }
// Device-side diagonal helpers declared in src/SparseMatrix.hpp; the host
// twins (CopyMatrixDiagonal/ReplaceMatrixDiagonal) call them after doing the
// host work, so they are no-ops here.
void HIPCopyMatrixDiagonal(const SparseMatrix&, Vector&) {}
void HIPReplaceMatrixDiagonal(SparseMatrix&, const Vector&) {}

namespace {

struct RefProblem {
    std::vector<SparseMatrix*> levels;  // levels[0] = fine
    std::vector<Geometry*> geoms;
    Vector b, x, xexact;
    CGData data;
};

void build_coarse(SparseMatrix& Af)
{
    const local_int_t nxf = Af.geom->nx, nyf = Af.geom->ny, nzf = Af.geom->nz;
    const local_int_t nxc = nxf / 2, nyc = nyf / 2, nzc = nzf / 2;
    const local_int_t nc = nxc * nyc * nzc;
    local_int_t* f2c = new local_int_t[nc];
    for(local_int_t izc = 0; izc < nzc; ++izc)
        for(local_int_t iyc = 0; iyc < nyc; ++iyc)
            for(local_int_t ixc = 0; ixc < nxc; ++ixc)
                f2c[izc * nxc * nyc + iyc * nxc + ixc] = 2 * izc * nxf * nyf + 2 * iyc * nxf + 2 * ixc;

    Geometry* geomc = new Geometry;
    GenerateGeometry(1, 0, Af.geom->numThreads, 0, 0, 0, nxc, nyc, nzc, 0, 0, 0, geomc);
    SparseMatrix* Ac = new SparseMatrix;
    InitializeSparseMatrix(*Ac, geomc);
    GenerateProblem_ref(*Ac, 0, 0, 0);
    SetupHalo_ref(*Ac);

    Vector* rc = new Vector;
    Vector* xc = new Vector;
    Vector* Axf = new Vector;
    InitializeVector(*rc, Ac->localNumberOfRows);
    InitializeVector(*xc, Ac->localNumberOfColumns);
    InitializeVector(*Axf, Af.localNumberOfColumns);

    MGData* mg = new MGData;
    mg->numberOfPresmootherSteps = 1;
    mg->numberOfPostsmootherSteps = 1;
    mg->f2cOperator = f2c;
    mg->rc = rc;
    mg->xc = xc;
    mg->Axf = Axf;
    mg->optimizationData = nullptr;
    mg->d_f2cOperator = nullptr;
    mg->d_c2fOperator = nullptr;
    Af.Ac = Ac;
    Af.mgData = mg;
}

Vector wrap(double* p, local_int_t n)
{
    Vector v;
    v.localLength = n;
    v.values = p;
    return v;
}

}  // namespace

extern "C" {

void* hpcgref_create(int nx, int ny, int nz, int nlevels)
{
    if(nx <= 0 || ny <= 0 || nz <= 0 || nlevels < 1) return nullptr;
    RefProblem* P = new RefProblem;
    Geometry* geom = new Geometry;
    GenerateGeometry(1, 0, 1, 0, 0, 0, nx, ny, nz, 0, 0, 0, geom);
    SparseMatrix* A = new SparseMatrix;
    InitializeSparseMatrix(*A, geom);
    GenerateProblem_ref(*A, &P->b, &P->x, &P->xexact);
    SetupHalo_ref(*A);
    P->levels.push_back(A);
    SparseMatrix* cur = A;
    for(int l = 1; l < nlevels; ++l)
    {
        build_coarse(*cur);
        cur = cur->Ac;
        P->levels.push_back(cur);
    }
    InitializeSparseCGData(*A, P->data);
    return P;
}

int hpcgref_num_levels(void* h) { return (int)((RefProblem*)h)->levels.size(); }

int hpcgref_level_info(void* h, int level, int* dims, int* nrows, long long* nnz)
{
    RefProblem* P = (RefProblem*)h;
    if(level < 0 || level >= (int)P->levels.size()) return 1;
    SparseMatrix* A = P->levels[level];
    dims[0] = A->geom->nx;
    dims[1] = A->geom->ny;
    dims[2] = A->geom->nz;
    *nrows = A->localNumberOfRows;
    *nnz = A->totalNumberOfNonzeros;
    return 0;
}

// Natural-order matrix, row-major 27 slots; unused slots: col -1, value 0.
int hpcgref_get_matrix(void* h, int level, int* cols, double* vals, signed char* nnz_in_row)
{
    RefProblem* P = (RefProblem*)h;
    if(level < 0 || level >= (int)P->levels.size()) return 1;
    SparseMatrix* A = P->levels[level];
    const local_int_t m = A->localNumberOfRows;
    for(local_int_t i = 0; i < m; ++i)
    {
        const int nnz = A->nonzerosInRow[i];
        nnz_in_row[i] = (signed char)nnz;
        for(int j = 0; j < 27; ++j)
        {
            cols[(size_t)i * 27 + j] = j < nnz ? A->mtxIndL[i][j] : -1;
            vals[(size_t)i * 27 + j] = j < nnz ? A->matrixValues[i][j] : 0.0;
        }
    }
    return 0;
}

int hpcgref_get_f2c(void* h, int level, int* f2c)
{
    RefProblem* P = (RefProblem*)h;
    if(level < 0 || level + 1 >= (int)P->levels.size()) return 1;
    SparseMatrix* A = P->levels[level];
    std::memcpy(f2c, A->mgData->f2cOperator, sizeof(int) * A->mgData->rc->localLength);
    return 0;
}

int hpcgref_get_rhs(void* h, double* b, double* xexact)
{
    RefProblem* P = (RefProblem*)h;
    const local_int_t m = P->levels[0]->localNumberOfRows;
    if(b) std::memcpy(b, P->b.values, sizeof(double) * m);
    if(xexact) std::memcpy(xexact, P->xexact.values, sizeof(double) * m);
    return 0;
}

// CheckProblem (src/CheckProblem.cpp:78) on every level; it asserts on mismatch.
int hpcgref_check_problem(void* h)
{
    RefProblem* P = (RefProblem*)h;
    for(size_t l = 0; l < P->levels.size(); ++l)
    {
        if(l == 0) CheckProblem(*P->levels[0], &P->b, &P->x, &P->xexact);
        else CheckProblem(*P->levels[l], 0, 0, 0);
    }
    return 0;
}

// CG_ref (src/CG_ref.cpp:86) from x0 = 0.  b == nullptr uses the generated b.
int hpcgref_cg(void* h, int max_iter, double tol, const double* b, double* x_out, int precond,
               int* niters, double* normr, double* normr0, double* seconds)
{
    RefProblem* P = (RefProblem*)h;
    SparseMatrix& A = *P->levels[0];
    const local_int_t m = A.localNumberOfRows;
    Vector bb;
    InitializeVector(bb, m);
    std::memcpy(bb.values, b ? b : P->b.values, sizeof(double) * m);
    ZeroVector(P->x);
    std::vector<double> times(9, 0.0);
    int it = 0;
    double nr = 0.0, nr0 = 0.0;
    auto t0 = std::chrono::steady_clock::now();
    int ierr = CG_ref(A, P->data, bb, P->x, max_iter, tol, it, nr, nr0, times.data(), precond != 0, false);
    auto t1 = std::chrono::steady_clock::now();
    if(x_out) std::memcpy(x_out, P->x.values, sizeof(double) * m);
    *niters = it;
    *normr = nr;
    *normr0 = nr0;
    if(seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
    DeleteVector(bb);
    return ierr;
}

int hpcgref_spmv(void* h, int level, double* x, double* y)
{
    RefProblem* P = (RefProblem*)h;
    SparseMatrix& A = *P->levels[level];
    Vector xv = wrap(x, A.localNumberOfColumns), yv = wrap(y, A.localNumberOfRows);
    return ComputeSPMV_ref(A, xv, yv);
}

int hpcgref_symgs(void* h, int level, double* r, double* x)
{
    RefProblem* P = (RefProblem*)h;
    SparseMatrix& A = *P->levels[level];
    Vector rv = wrap(r, A.localNumberOfRows), xv = wrap(x, A.localNumberOfColumns);
    return ComputeSYMGS_ref(A, rv, xv);
}

int hpcgref_mg(void* h, int level, double* r, double* x)
{
    RefProblem* P = (RefProblem*)h;
    SparseMatrix& A = *P->levels[level];
    Vector rv = wrap(r, A.localNumberOfRows), xv = wrap(x, A.localNumberOfColumns);
    return ComputeMG_ref(A, rv, xv);
}

int hpcgref_dot(int n, double* x, double* y, double* result)
{
    Vector xv = wrap(x, n), yv = wrap(y, n);
    double t = 0.0;
    return ComputeDotProduct_ref(n, xv, yv, *result, t);
}

int hpcgref_waxpby(int n, double alpha, double* x, double beta, double* y, double* w)
{
    Vector xv = wrap(x, n), yv = wrap(y, n), wv = wrap(w, n);
    return ComputeWAXPBY_ref(n, alpha, xv, beta, yv, wv);
}

// rc = rf[f2c] - (A xf)[f2c]  (ComputeSPMV_ref into Axf, then ComputeRestriction_ref)
int hpcgref_restriction(void* h, int level, double* rf, double* xf, double* rc)
{
    RefProblem* P = (RefProblem*)h;
    SparseMatrix& A = *P->levels[level];
    if(!A.mgData) return 1;
    Vector xv = wrap(xf, A.localNumberOfColumns), rv = wrap(rf, A.localNumberOfRows);
    int ierr = ComputeSPMV_ref(A, xv, *A.mgData->Axf);
    if(ierr) return ierr;
    ierr = ComputeRestriction_ref(A, rv);
    std::memcpy(rc, A.mgData->rc->values, sizeof(double) * A.mgData->rc->localLength);
    return ierr;
}

int hpcgref_prolongation(void* h, int level, const double* xc, double* xf)
{
    RefProblem* P = (RefProblem*)h;
    SparseMatrix& A = *P->levels[level];
    if(!A.mgData) return 1;
    std::memcpy(A.mgData->xc->values, xc, sizeof(double) * A.mgData->xc->localLength);
    Vector xv = wrap(xf, A.localNumberOfColumns);
    return ComputeProlongation_ref(A, xv);
}

int hpcgref_residual(int n, double* v1, double* v2, double* result)
{
    Vector a = wrap(v1, n), b = wrap(v2, n);
    return ComputeResidual_ref(n, a, b, *result);
}

int hpcgref_test_norms(const double* values, int n, double* mean, double* variance, int* pass)
{
    TestNormsData d;
    d.samples = n;
    d.values = const_cast<double*>(values);
    TestNorms(d);
    *mean = d.mean;
    *variance = d.variance;
    *pass = d.pass ? 1 : 0;
    return 0;
}

// The reference's own process grid for `size` ranks (src/ComputeOptimalShapeXYZ.cpp).
void hpcgref_optimal_shape(int size, int* npx, int* npy, int* npz)
{
    int x = 0, y = 0, z = 0;
    ComputeOptimalShapeXYZ(size, x, y, z);
    *npx = x, *npy = y, *npz = z;
}

// The reference's GenerateGeometry (src/GenerateGeometry.cpp): out[13] =
// {npx, npy, npz, ipx, ipy, ipz, gnx, gny, gnz, gix0, giy0, giz0, npartz}.
void hpcgref_geometry(int size, int rank, int pz, int zl, int zu, int nx, int ny, int nz, int npx, int npy, int npz,
                      long long* out)
{
    Geometry g;
    GenerateGeometry(size, rank, 1, pz, zl, zu, nx, ny, nz, npx, npy, npz, &g);
    const long long v[13] = {g.npx, g.npy, g.npz, g.ipx, g.ipy, g.ipz, g.gnx, g.gny, g.gnz, g.gix0, g.giy0, g.giz0,
                             g.npartz};
    std::memcpy(out, v, sizeof(v));
}

// Rank `rank` of a `size`-rank run with local brick nx*ny*nz, as the
// reference generates it (src/GenerateGeometry.cpp + src/GenerateProblem_ref.cpp
// with the geometry's global offsets): per natural row its GLOBAL column ids
// (row-major 27 slots, -1 padded), values, nonzero count and b; grid[6] =
// {npx, npy, npz, ipx, ipy, ipz}.  The MPI sum of the nonzero count is not
// needed for these arrays.  (The generated problem is not released: a test
// oracle's process memory.)
int hpcgref_rank_problem(int size, int rank, int nx, int ny, int nz, long long* gcols, double* vals,
                         signed char* nnz_in_row, double* b, int* grid)
{
    Geometry* geom = new Geometry;
    GenerateGeometry(size, rank, 1, 0, 0, 0, nx, ny, nz, 0, 0, 0, geom);
    SparseMatrix A;
    InitializeSparseMatrix(A, geom);
    Vector vb, vx, vxe;
    GenerateProblem_ref(A, &vb, &vx, &vxe);
    const local_int_t m = A.localNumberOfRows;
    for(local_int_t i = 0; i < m; ++i)
    {
        const int nnz = A.nonzerosInRow[i];
        nnz_in_row[i] = (signed char)nnz;
        for(int j = 0; j < 27; ++j)
        {
            gcols[(size_t)i * 27 + j] = j < nnz ? (long long)A.mtxIndG[i][j] : -1;
            vals[(size_t)i * 27 + j] = j < nnz ? A.matrixValues[i][j] : 0.0;
        }
        b[i] = vb.values[i];
    }
    grid[0] = geom->npx, grid[1] = geom->npy, grid[2] = geom->npz;
    grid[3] = geom->ipx, grid[4] = geom->ipy, grid[5] = geom->ipz;
    return 0;
}

void hpcgref_destroy(void* h)
{
    // The reference's DeleteMatrix also frees device fields through the shim's
    // no-op deviceFree; releasing the host process memory at exit is enough
    // for a test oracle, so only the handle is dropped here.
    delete (RefProblem*)h;
}

}  // extern "C"
