// Problem construction: src/GenerateGeometry.cpp:49-169 (single rank),
// src/GenerateProblem.cpp:375-489, src/SetupHalo.cpp:294-327 (single rank),
// src/GenerateCoarseProblem.cpp:98-184 and the deleters of
// src/SparseMatrix.hpp:264-330 / src/MGData.hpp:101-120.
#include <cstring>

#include "hpcg_b200.h"
#include "internal.hpp"

using namespace hpcg_b200;

void GenerateGeometry(int size, int rank, int numThreads, int pz, local_int_t zl, local_int_t zu, local_int_t nx,
                      local_int_t ny, local_int_t nz, int npx, int npy, int npz, Geometry* geom)
{
    // One rank (the tier fixes a single GPU): a 1x1x1 process grid.
    (void)npx;
    (void)npy;
    (void)npz;
    (void)zl;
    (void)zu;
    (void)pz;
    geom->size = size;
    geom->rank = rank;
    geom->numThreads = numThreads;
    geom->nx = nx;
    geom->ny = ny;
    geom->nz = nz;
    geom->npx = geom->npy = geom->npz = 1;
    geom->pz = 0;
    geom->npartz = 1;
    geom->partz_ids = new int[1]{1};
    geom->partz_nz = new local_int_t[1]{nz};
    geom->ipx = geom->ipy = geom->ipz = 0;
    geom->gnx = nx;
    geom->gny = ny;
    geom->gnz = nz;
    geom->gix0 = geom->giy0 = geom->giz0 = 0;
}

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
    GenerateGeometry(Af.geom->size, Af.geom->rank, Af.geom->numThreads, 0, 0, 0, nxc, nyc, nzc, 1, 1, 1, geomc);
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
