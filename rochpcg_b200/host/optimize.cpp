// OptimizeProblem (src/OptimizeProblem.cpp:69-160): for every level,
// JPL multicoloring + stable colour sort (src/MultiColoring.cpp:238-353),
// column permutation / ELL conversion / row permutation in one pass
// (src/Permute.cpp:95-218, src/SparseMatrix.cpp:271-359) and diagonal
// extraction (src/SparseMatrix.cpp:361-407); then b and xexact are permuted
// (src/Permute.cpp:237-246).  On top of the reference it prepares the data
// of the B200 kernels: the colour-interleaved SpMV map, the multigrid
// transfer indices, and -- when the level is verified to be the HPCG stencil
// in parity colouring -- the FP32 implicit-stencil description.
#include <cstring>

#include "hpcg_b200.h"
#include "internal.hpp"

using namespace hpcg_b200;

namespace hpcg_b200 {
bool g_keep_generated = false;  // keep the row-major generated arrays (tests inspect them)
}

static void optimize_level(SparseMatrix& A)
{
    cudaStream_t s = rt().stream;
    const local_int_t m = A.localNumberOfRows;
    LevelOpt* o = opt(A);
    if(!o)
    {
        o = new LevelOpt;
        A.optimizationData = o;
    }

    // -- colouring and permutation
    A.perm = dalloc<local_int_t>(m);
    o->colors = dalloc<int>(m);
    const size_t wsb = hpcgb200_coloring_workspace_bytes(m);
    void* ws = dalloc<char>(wsb);
    A.sizes = new local_int_t[HPCGB200_MAX_COLORS];
    A.offsets = new local_int_t[HPCGB200_MAX_COLORS + 1];
    int jpl_blocks = 0;
    std::vector<int> rs(HPCGB200_MAX_COLORS);
    int rc = hpcgb200_jpl_coloring(m, A.d_rowHash, A.d_mtxIndL, o->colors, A.perm, &jpl_blocks, rs.data(), A.sizes,
                                   A.offsets, ws, wsb, s);
    dfree(ws);
    check(rc);
    o->jpl_blocks = jpl_blocks;
    o->round_sizes.assign(rs.begin(), rs.begin() + jpl_blocks);
    int used = 0;
    for(int c = 0; c < HPCGB200_MAX_COLORS; ++c)
        if(A.sizes[c] > 0) used = c + 1;
    A.nblocks = used;
    A.ublocks = used - 2;  // src/MultiColoring.cpp:316,350-352 (optimized build)

    // -- ELL + diagonal
    const size_t slots = (size_t)m * 27;
    A.ell_col_ind = dalloc<local_int_t>(slots);
    A.ell_val = dalloc<double>(slots);
    check(hpcgb200_build_ell(m, A.d_mtxIndL, A.d_matrixValues, A.perm, A.ell_col_ind, A.ell_val, s));
    A.diag_idx = dalloc<local_int_t>(m);
    A.inv_diag = dalloc<double>(m);
    o->diag = dalloc<double>(m);
    check(hpcgb200_extract_diagonal(m, A.ell_col_ind, A.ell_val, A.diag_idx, A.inv_diag, o->diag, s));
    check(hb::zero_guess_groups(m, A.nblocks, A.offsets, A.diag_idx, o->zg, s));
    o->zg_ok = true;
    o->cc = hb::make_chunks(m, A.nblocks, A.offsets);

    // -- FP32 implicit stencil (mixed path): verify before enabling
    o->stencil_ok = false;
    const int nx = A.geom->nx, ny = A.geom->ny, nz = A.geom->nz;
    if(A.nblocks == 8 && nx >= 2 && ny >= 2 && nz >= 2)
    {
        int cop[8];
        bool ok = true;
        for(int p = 0; p < 8; ++p)
        {
            const int ix = (p >> 2) & 1, iy = (p >> 1) & 1, iz = p & 1;
            const size_t nat = (size_t)iz * nx * ny + (size_t)iy * nx + ix;
            HB_HOST_CUDA(cudaMemcpyAsync(&cop[p], o->colors + nat, sizeof(int), cudaMemcpyDeviceToHost, s));
        }
        HB_HOST_CUDA(cudaStreamSynchronize(s));
        ok = hb::make_stencil_level(nx, ny, nz, A.offsets, cop, &o->st);
        if(ok)
        {
            int* bad = dalloc<int>(1);
            HB_HOST_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), s));
            check(hb::launch_stencil_check(o->st, A.perm, A.ell_col_ind, A.ell_val, bad, s));
            int hbad = -1;
            HB_HOST_CUDA(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
            HB_HOST_CUDA(cudaStreamSynchronize(s));
            dfree(bad);
            o->stencil_ok = (hbad == 0);
        }
    }
    if(o->stencil_ok)
    {
        o->pm = hb::make_perm_map(o->st);
        // the TMA-staged colour passes of this level set it when their copies time out
        o->pass_status = dalloc<int>(1);
        HB_HOST_CUDA(cudaMemsetAsync(o->pass_status, 0, sizeof(int), s));
        o->st.status = o->pass_status;
        o->diag32 = dalloc<float>(m);
        o->inv_diag32 = dalloc<float>(m);
        check(hb::launch_diag32(m, o->diag, o->diag32, o->inv_diag32, s));
    }
}

static void free_generated(SparseMatrix& A)
{
    if(g_keep_generated) return;
    dfree(A.d_mtxIndL);
    dfree(A.d_matrixValues);
    dfree(A.d_rowHash);
    A.d_mtxIndL = nullptr;
    A.d_matrixValues = nullptr;
    A.d_rowHash = nullptr;
}

int OptimizeProblem(SparseMatrix& A, CGData& data, Vector& b, Vector& x, Vector& xexact)
{
    (void)x;  // x is zero; the reference does not permute it either
    try
    {
        ensure_runtime();
        cudaStream_t s = rt().stream;
        for(SparseMatrix* M = &A; M; M = M->Ac) optimize_level(*M);

        // multigrid transfer indices (fine permuted row, coarse permuted row)
        for(SparseMatrix* M = &A; M && M->Ac; M = M->Ac)
        {
            MGOpt* mo = mgopt(*M);
            const local_int_t nc = M->Ac->localNumberOfRows;
            mo->inj_f = dalloc<int>(nc);
            mo->inj_c = dalloc<int>(nc);
            check(hpcgb200_transfer_indices(nc, M->mgData->d_f2cOperator, M->perm, M->Ac->perm, mo->inj_f, mo->inj_c,
                                            s));
            mo->pro_f = dalloc<int>(nc);
            check(hb::launch_prolong_map(nc, mo->inj_f, mo->inj_c, mo->pro_f, s));
            if(opt(*M)->stencil_ok && opt(*M->Ac)->stencil_ok)
            {
                mo->rc32 = dalloc<float>(nc);
                mo->xc32 = dalloc<float>(nc);
            }
        }

        // permute b and xexact into the coloured order
        const local_int_t m = A.localNumberOfRows;
        double* tmp = dalloc<double>(m);
        check(hpcgb200_permute_vector(m, A.perm, b.d_values, tmp, s));
        HB_HOST_CUDA(cudaMemcpyAsync(b.d_values, tmp, sizeof(double) * m, cudaMemcpyDeviceToDevice, s));
        check(hpcgb200_permute_vector(m, A.perm, xexact.d_values, tmp, s));
        HB_HOST_CUDA(cudaMemcpyAsync(xexact.d_values, tmp, sizeof(double) * m, cudaMemcpyDeviceToDevice, s));
        HB_HOST_CUDA(cudaStreamSynchronize(s));
        dfree(tmp);

        LevelOpt* o = opt(A);
        if(o->stencil_ok)
        {
            o->r32 = dalloc<float>(m);
            o->z32 = dalloc<float>(m);
            o->pap_partial = dalloc<double>(hb::stencil_pap_partials(o->st));
            o->pap_ticket = dalloc<unsigned int>(1);
            HB_HOST_CUDA(cudaMemsetAsync(o->pap_ticket, 0, sizeof(unsigned int), s));
        }
        o->vec_scratch = dalloc<double>(m);
        o->spmv_partial = dalloc<double>(o->cc.nchunks());
        o->spmv_ticket = dalloc<unsigned int>(1);
        HB_HOST_CUDA(cudaMemsetAsync(o->spmv_ticket, 0, sizeof(unsigned int), s));

        if(!data.r.d_values) CudaInitializeSparseCGData(A, data);
        for(SparseMatrix* M = &A; M; M = M->Ac) free_generated(*M);
        HB_HOST_CUDA(cudaStreamSynchronize(s));
        return 0;
    }
    catch(const Error& e)
    {
        return report(e);
    }
}
