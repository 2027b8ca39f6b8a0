// Problem construction: src/GenerateGeometry.cpp:49-169,
// src/GenerateProblem.cpp:375-489, src/SetupHalo.cpp:294-327 (single rank),
// src/GenerateCoarseProblem.cpp:98-184 and the deleters of
// src/SparseMatrix.hpp:264-330 / src/MGData.hpp:101-120.
#include <cstring>
#include <string>

#include "dist.hpp"
#include "hpcg_b200.h"
#include "internal.hpp"

using namespace hpcg_b200;

// The process grid (the given one when it fits in size ranks, else the
// least-surface split of size), this rank's coordinates and its brick's
// global offsets; with pz > 0 the process planes below z-index pz hold nz =
// zl points, the others zu (the reference's two z zones).
void GenerateGeometry(int size, int rank, int numThreads, int pz, local_int_t zl, local_int_t zu, local_int_t nx,
                      local_int_t ny, local_int_t nz, int npx, int npy, int npz, Geometry* geom)
{
    if(npx * npy * npz <= 0 || npx * npy * npz > size) optimal_shape(size, npx, npy, npz);
    geom->size = size;
    geom->rank = rank;
    geom->numThreads = numThreads;
    geom->nx = nx;
    geom->ny = ny;
    geom->nz = nz;
    geom->npx = npx;
    geom->npy = npy;
    geom->npz = npz;
    geom->pz = pz;
    if(pz == 0)
    {
        geom->npartz = 1;
        geom->partz_ids = new int[1]{npz};
        geom->partz_nz = new local_int_t[1]{nz};
    }
    else
    {
        geom->npartz = 2;
        geom->partz_ids = new int[2]{pz, npz};
        geom->partz_nz = new local_int_t[2]{zl, zu};
    }
    geom->ipz = rank / (npx * npy);
    geom->ipy = (rank - geom->ipz * npx * npy) / npx;
    geom->ipx = rank % npx;
    geom->gnx = (global_int_t)npx * nx;
    geom->gny = (global_int_t)npy * ny;
    // z extent and offset over the zones: zone i spans process planes
    // [partz_ids[i-1], partz_ids[i]) with partz_nz[i] points each
    global_int_t gnz = 0, giz0 = 0;
    int lo = 0;
    bool placed = false;
    for(int i = 0; i < geom->npartz; ++i)
    {
        const int hi = geom->partz_ids[i];
        gnz += (global_int_t)geom->partz_nz[i] * (hi - lo);
        if(!placed)
        {
            if(geom->ipz < hi)
            {
                giz0 += (global_int_t)(geom->ipz - lo) * geom->partz_nz[i];
                placed = true;
            }
            else
                giz0 += (global_int_t)(hi - lo) * geom->partz_nz[i];
        }
        lo = hi;
    }
    geom->gnz = gnz;
    geom->gix0 = (global_int_t)geom->ipx * nx;
    geom->giy0 = (global_int_t)geom->ipy * ny;
    geom->giz0 = giz0;
}

namespace {

// The C++ operator layer holds one rank; a decomposed problem is built and
// solved through hpcgb200_dist_* (its own halo plan and exchange).
void require_one_rank(const SparseMatrix& A, const char* what)
{
    if(A.geom && A.geom->size > 1)
        throw Error(HPCGB200_ERR_ARG, std::string(what) + ": a geometry of " + std::to_string(A.geom->size) +
                                          " ranks; the C++ operator layer holds one rank, build decomposed problems "
                                          "with hpcgb200_dist_create (include/hpcg_b200.h)");
}

}  // namespace

void DeleteGeometry(Geometry& geom)
{
    delete[] geom.partz_ids;
    delete[] geom.partz_nz;
    geom.partz_ids = nullptr;
    geom.partz_nz = nullptr;
}

void InitializeSparseMatrix(SparseMatrix& A, Geometry* geom)
{
    std::memset(static_cast<void*>(&A), 0, sizeof(SparseMatrix));
    A.geom = geom;
    A.isDotProductOptimized = true;
    A.isSpmvOptimized = true;
    A.isMgOptimized = true;
    A.isWaxpbyOptimized = true;
}

void GenerateProblem(SparseMatrix& A, Vector* b, Vector* x, Vector* xexact)
{
    require_one_rank(A, "GenerateProblem");
    ensure_runtime();
    cudaStream_t s = rt().stream;
    const local_int_t nx = A.geom->nx, ny = A.geom->ny, nz = A.geom->nz;
    if((long long)nx * ny * nz > 0x7fffffffLL)
        throw Error(HPCGB200_ERR_ARG, "local grid exceeds 2^31 rows (local_int_t is int32)");
    const local_int_t m = nx * ny * nz;
    const size_t slots = (size_t)m * 27;

    if(b) CudaInitializeVector(*b, m);
    if(x) CudaInitializeVector(*x, m);
    if(xexact) CudaInitializeVector(*xexact, m);

    A.d_mtxIndL = dalloc<local_int_t>(slots);
    A.d_matrixValues = dalloc<double>(slots);
    A.d_nonzerosInRow = dalloc<char>(m);
    A.d_matrixDiagonal = dalloc<local_int_t>(m);
    A.d_rowHash = dalloc<local_int_t>(m);
    A.d_localToGlobalMap = dalloc<global_int_t>(m);

    check(hpcgb200_generate_problem(nx, ny, nz, A.geom->gnx, A.geom->gny, A.geom->gnz, A.geom->gix0, A.geom->giy0,
                                    A.geom->giz0, A.d_mtxIndL, A.d_matrixValues,
                                    reinterpret_cast<int8_t*>(A.d_nonzerosInRow), A.d_matrixDiagonal,
                                    A.d_localToGlobalMap, A.d_rowHash, b ? b->d_values : nullptr, s));
    if(x) HB_HOST_CUDA(cudaMemsetAsync(x->d_values, 0, sizeof(double) * m, s));
    if(xexact)
    {
        // xexact = 1 (kernel_set_one): fill a host buffer once, copy.
        std::vector<double> ones(m, 1.0);
        HB_HOST_CUDA(cudaMemcpyAsync(xexact->d_values, ones.data(), sizeof(double) * m, cudaMemcpyHostToDevice, s));
        HB_HOST_CUDA(cudaStreamSynchronize(s));
    }

    // Number of nonzeros of the 27-point stencil on an nx x ny x nz box
    // (the reference sums nonzerosInRow on the device; the count is exact).
    const global_int_t nnz = (global_int_t)(3LL * nx - 2) * (3LL * ny - 2) * (3LL * nz - 2);
    A.title = nullptr;
    A.totalNumberOfRows = (global_int_t)A.geom->gnx * A.geom->gny * A.geom->gnz;
    A.totalNumberOfNonzeros = nnz;
    A.localNumberOfRows = m;
    A.localNumberOfColumns = m;
    A.localNumberOfNonzeros = (local_int_t)(nnz > 0x7fffffffLL ? 0x7fffffff : nnz);
    A.ell_width = 27;
    A.numberOfNonzerosPerRow = 27;
}

void SetupHalo(SparseMatrix& A)
{
    // Single rank (src/SetupHalo.cpp:313-327): the local column ids are the
    // global ones, which GenerateProblem already stored in d_mtxIndL with -1
    // pads, so there is nothing left to do.
    A.localNumberOfColumns = A.localNumberOfRows;
}

void GenerateCoarseProblem(const SparseMatrix& Af)
{
    ensure_runtime();
    const local_int_t nxf = Af.geom->nx, nyf = Af.geom->ny, nzf = Af.geom->nz;
    if(nxf % 2 || nyf % 2 || nzf % 2)
        throw Error(HPCGB200_ERR_ARG, "GenerateCoarseProblem: fine dimensions must be even");
    const local_int_t nxc = nxf / 2, nyc = nyf / 2, nzc = nzf / 2;
    const local_int_t nc = nxc * nyc * nzc;
    local_int_t* f2c = dalloc<local_int_t>(nc);
    local_int_t* c2f = dalloc<local_int_t>((size_t)nxf * nyf * nzf);
    check(hpcgb200_f2c_operator(nxf, nyf, nzf, f2c, c2f, rt().stream));

    Geometry* geomc = new Geometry;
    GenerateGeometry(Af.geom->size, Af.geom->rank, Af.geom->numThreads, Af.geom->pz,
                     Af.geom->pz > 0 ? Af.geom->partz_nz[0] / 2 : 0, Af.geom->pz > 0 ? Af.geom->partz_nz[1] / 2 : 0, nxc,
                     nyc, nzc, Af.geom->npx, Af.geom->npy, Af.geom->npz, geomc);
    SparseMatrix* Ac = new SparseMatrix;
    InitializeSparseMatrix(*Ac, geomc);
    GenerateProblem(*Ac, nullptr, nullptr, nullptr);
    SetupHalo(*Ac);

    Vector* rc = new Vector;
    Vector* xc = new Vector;
    Vector* Axf = new Vector;  // allocated on first use by ComputeRestriction
    CudaInitializeVector(*rc, Ac->localNumberOfRows);
    CudaInitializeVector(*xc, Ac->localNumberOfColumns);

    MGData* mg = new MGData;
    mg->numberOfPresmootherSteps = 1;   // src/MGData.hpp:85-86
    mg->numberOfPostsmootherSteps = 1;
    mg->f2cOperator = nullptr;
    mg->rc = rc;
    mg->xc = xc;
    mg->Axf = Axf;
    mg->optimizationData = new MGOpt;
    mg->d_f2cOperator = f2c;
    mg->d_c2fOperator = c2f;
    Af.Ac = Ac;
    Af.mgData = mg;
}

static void delete_level_opt(SparseMatrix& A)
{
    LevelOpt* o = opt(A);
    if(!o) return;
    dfree(o->diag);
    dfree(o->colors);
    dfree(o->diag32);
    dfree(o->inv_diag32);
    dfree(o->pass_status);
    dfree(o->cg_state);
    dfree(o->step_barrier);
    dfree(o->r32);
    dfree(o->pap_partial);
    dfree(o->pap_ticket);
    dfree(o->spmv_partial);
    dfree(o->spmv_ticket);
    dfree(o->z32);
    dfree(o->vec_scratch);
    dfree(o->x0_saved);
    for(auto& g : o->graphs)
    {
        if(g->exec) cudaGraphExecDestroy(g->exec);
        if(g->graph) cudaGraphDestroy(g->graph);
    }
    delete o;
    A.optimizationData = nullptr;
}

void DeleteMatrix(SparseMatrix& A)
{
    if(A.Ac)
    {
        DeleteMatrix(*A.Ac);
        if(A.Ac->geom)
        {
            DeleteGeometry(*A.Ac->geom);
            delete A.Ac->geom;
        }
        delete A.Ac;
        A.Ac = nullptr;
    }
    if(A.mgData)
    {
        MGData* mg = A.mgData;
        CudaDeleteVector(*mg->rc);
        CudaDeleteVector(*mg->xc);
        CudaDeleteVector(*mg->Axf);
        delete mg->rc;
        delete mg->xc;
        delete mg->Axf;
        dfree(mg->d_f2cOperator);
        dfree(mg->d_c2fOperator);
        if(mg->f2cOperator) delete[] mg->f2cOperator;
        if(MGOpt* mo = static_cast<MGOpt*>(mg->optimizationData))
        {
            dfree(mo->inj_f);
            dfree(mo->inj_c);
            dfree(mo->pro_f);
            dfree(mo->rc32);
            dfree(mo->xc32);
            delete mo;
        }
        delete mg;
        A.mgData = nullptr;
    }
    dfree(A.d_nonzerosInRow);
    dfree(A.d_mtxIndL);
    dfree(A.d_matrixValues);
    dfree(A.d_matrixDiagonal);
    dfree(A.d_localToGlobalMap);
    dfree(A.d_rowHash);
    dfree(A.ell_col_ind);
    dfree(A.ell_val);
    dfree(A.diag_idx);
    dfree(A.inv_diag);
    dfree(A.perm);
    delete[] A.sizes;
    delete[] A.offsets;
    delete_level_opt(A);
    A.d_nonzerosInRow = nullptr;
    A.d_mtxIndL = nullptr;
    A.d_matrixValues = nullptr;
    A.d_matrixDiagonal = nullptr;
    A.d_localToGlobalMap = nullptr;
    A.d_rowHash = nullptr;
    A.ell_col_ind = nullptr;
    A.ell_val = nullptr;
    A.diag_idx = nullptr;
    A.inv_diag = nullptr;
    A.perm = nullptr;
    A.sizes = nullptr;
    A.offsets = nullptr;
}
