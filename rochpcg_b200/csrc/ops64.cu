// FP64 operators of the plain drop-in path: ELL SpMV, multicolor SymGS
// (full and zero-guess), fused SpMV+restriction, prolongation, dot products
// and WAXPBY.  Matrix data is column-major ELL (slot p of row i at p*m+i), so a
// warp's 32 consecutive rows read 128 B of column indices and 256 B of values
// per slot: fully coalesced streams.  The stencil gathers of x go through L2;
// matrix streams are loaded evict-first so they do not push x out of L2.
//
// Row-wise results are bit-identical to the reference kernels (same fma
// order); reductions use a fixed-shape deterministic tree.
#include <algorithm>
#include <vector>

#include "ops64.cuh"

namespace hb {

ColorChunks make_chunks(int m, int ncolors, const int* offsets)
{
    ColorChunks cc{};
    if(ncolors < 1 || ncolors > kMaxMapColors || offsets == nullptr)
    {
        cc.ncolors = 1;
        cc.offsets[0] = 0;
        cc.offsets[1] = m;
    }
    else
    {
        cc.ncolors = ncolors;
        for(int c = 0; c <= ncolors; ++c) cc.offsets[c] = offsets[c];
    }
    int per = 0;
    for(int c = 0; c < cc.ncolors; ++c)
    {
        const int sz = cc.offsets[c + 1] - cc.offsets[c];
        per = max(per, (sz + kBS - 1) / kBS);
    }
    cc.per_color = per;
    return cc;
}

// src/ComputeSPMV.cpp:130-170.  Blocks are interleaved over colours (block b
// works on colour b % ncolors) so the eight blocks that gather from the same
// neighbourhood of x run together and share it in L2.
__global__ void __launch_bounds__(kBS) k_spmv(int m, ColorChunks cc, const int* __restrict__ ell_col,
                                              const double* __restrict__ ell_val, const double* __restrict__ x,
                                              double* __restrict__ y)
{
    int row;
    if(!cc.row_of(blockIdx.x, threadIdx.x, row)) return;
    y[row] = spmv_row(m, row, ell_col, ell_val, x);
}

// ---------------------------------------------------------------- SymGS

// src/ComputeSYMGS.cpp:113-151 (kernel_symgs_sweep): rows of one colour.
// Columns below ncols take part: the local columns (ncols = m; also
// kernel_symgs_interior, :153-188), or the local and the external ones of a
// rank of a decomposed problem (ncols = m + externals).
__global__ void __launch_bounds__(kBS) k_symgs_sweep(int m, int ncols, int size, int offset,
                                                     const int* __restrict__ ell_col,
                                                     const double* __restrict__ ell_val,
                                                     const double* __restrict__ inv_diag,
                                                     const double* __restrict__ r, double* x, Prolong<double> pro)
{
    const int gid = blockIdx.x * kBS + threadIdx.x;
    if(gid >= size) return;
    const int row = gid + offset;
    const double sum = ell_row_sum(m, row, ell_col, ell_val, x, r[row], -1.0, 0, kWidth,
                                   [ncols, row](int col) { return col >= 0 && col < ncols && col != row; });
    const double v = sum * inv_diag[row];
    x[row] = v;
    pro.add(row, v);
}

// src/ComputeSYMGS.cpp:238-295 (kernel_pointwise_mult + kernel_forward_sweep_0):
// only the slots before the diagonal, only columns of earlier colours.  The
// reference multiplies by __drcp_rn(a_ii); inv_diag = 1/a_ii is the same
// correctly rounded value, read coalesced instead of from the diagonal slot.
template <int GHI>
__global__ void __launch_bounds__(kBS) k_symgs_fwd0(int m, int size, int offset, const int* __restrict__ ell_col,
                                                    const double* __restrict__ ell_val,
                                                    const int* __restrict__ diag_idx,
                                                    const double* __restrict__ inv_diag,
                                                    const double* __restrict__ r, double* x, Prolong<double> pro)
{
    const int gid = blockIdx.x * kBS + threadIdx.x;
    if(gid >= size) return;
    const int row = gid + offset;
    double sum = r[row];
    if(offset > 0)
    {
        const int diag = diag_idx[row];
        sum = ell_row_sum<0, GHI>(m, row, ell_col, ell_val, x, sum, -1.0, 0, diag,
                                  [offset](int col) { return col >= 0 && col < offset; });
    }
    const double v = sum * inv_diag[row];
    x[row] = v;
    pro.add(row, v);
}

// src/ComputeSYMGS.cpp:297-341 (kernel_backward_sweep_0).
template <int GLO>
__global__ void __launch_bounds__(kBS) k_symgs_bwd0(int m, int size, int offset, const int* __restrict__ ell_col,
                                                    const double* __restrict__ ell_val,
                                                    const int* __restrict__ diag_idx, const double* __restrict__ diag,
                                                    const double* __restrict__ inv_diag, double* x,
                                                    Prolong<double> pro)
{
    const int gid = blockIdx.x * kBS + threadIdx.x;
    if(gid >= size) return;
    const int row = gid + offset;
    const int d = diag_idx[row];
    const double sum = ell_row_sum<GLO, 3>(m, row, ell_col, ell_val, x, __dmul_rn(x[row], diag[row]), -1.0, d + 1,
                                           kWidth, [offset, m](int col) { return col >= offset && col < m; });
    const double v = sum * inv_diag[row];
    x[row] = v;
    pro.add(row, v);
}

// ---------------------------------------------------------- restriction

// src/ComputeRestriction.cpp:81-124 (kernel_fused_restrict_spmv).
__global__ void __launch_bounds__(kBS) k_restrict(int nc, const int* __restrict__ inj_f, const int* __restrict__ inj_c,
                                                  int mf, const int* __restrict__ ell_col,
                                                  const double* __restrict__ ell_val, const double* __restrict__ rf,
                                                  const double* __restrict__ xf, double* __restrict__ rc)
{
    const int ic = blockIdx.x * kBS + threadIdx.x;
    if(ic >= nc) return;
    const int row = inj_f[ic];
    const double sum = ell_row_sum(mf, row, ell_col, ell_val, xf, rf[row], -1.0, 0, kWidth,
                                   [mf](int col) { return col >= 0 && col < mf; });
    rc[inj_c[ic]] = sum;
}

// src/ComputeRestriction.cpp:59-79 (kernel_restrict, HPCG_REFERENCE form):
// rc[inj_c[i]] = rf[inj_f[i]] - Axf[inj_f[i]].
__global__ void __launch_bounds__(kBS) k_restrict_axf(int nc, const int* __restrict__ inj_f,
                                                      const int* __restrict__ inj_c, const double* __restrict__ rf,
                                                      const double* __restrict__ axf, double* __restrict__ rc)
{
    const int ic = blockIdx.x * kBS + threadIdx.x;
    if(ic >= nc) return;
    const int row = inj_f[ic];
    rc[inj_c[ic]] = rf[row] - axf[row];
}

// src/ComputeProlongation.cpp:39-59.
__global__ void __launch_bounds__(kBS) k_prolong(int nc, const int* __restrict__ inj_f, const int* __restrict__ inj_c,
                                                 const double* __restrict__ xc, double* __restrict__ xf)
{
    const int ic = blockIdx.x * kBS + threadIdx.x;
    if(ic >= nc) return;
    xf[inj_f[ic]] += xc[inj_c[ic]];
}

// ------------------------------------------------------ vector kernels

// src/ComputeDotProduct.cpp:63-170 (kernel_dot1/dot2 + part2), one launch.
__global__ void __launch_bounds__(kReduceThreads) k_dot(int n, const double* __restrict__ x,
                                                        const double* __restrict__ y, ReduceScratch* ws,
                                                        double* result)
{
    __shared__ double red[32];
    double s = 0.0;
    for(long long i = (long long)blockIdx.x * kReduceThreads + threadIdx.x; i < n; i += kReduceBlocks * kReduceThreads)
        s = fma(y[i], x[i], s);
    s = block_sum(s, red);
    double total;
    if(grid_reduce(s, ws, kReduceBlocks, &total)) *result = total;
}

// src/ComputeWAXPBY.cpp:63-91.
__global__ void __launch_bounds__(kBS) k_waxpby(int n, double alpha, const double* __restrict__ x, double beta,
                                                const double* __restrict__ y, double* __restrict__ w)
{
    const int i = blockIdx.x * kBS + threadIdx.x;
    if(i >= n) return;
    if(alpha == 1.0) w[i] = fma(beta, y[i], x[i]);
    else if(beta == 1.0) w[i] = fma(alpha, x[i], y[i]);
    else w[i] = fma(alpha, x[i], beta * y[i]);
}

// src/ComputeWAXPBY.cpp:137-196.
__global__ void __launch_bounds__(kReduceThreads) k_waxpby_dot(int n, double alpha, const double* __restrict__ x,
                                                               double* __restrict__ y, ReduceScratch* ws,
                                                               double* result)
{
    __shared__ double red[32];
    double s = 0.0;
    for(long long i = (long long)blockIdx.x * kReduceThreads + threadIdx.x; i < n; i += kReduceBlocks * kReduceThreads)
    {
        const double v = fma(alpha, x[i], y[i]);
        y[i] = v;
        s = fma(v, v, s);
    }
    s = block_sum(s, red);
    double total;
    if(grid_reduce(s, ws, kReduceBlocks, &total)) *result = total;
}

// src/ComputeResidual.cpp:77-119.
__global__ void __launch_bounds__(kReduceThreads) k_residual_inf(int n, const double* __restrict__ v1,
                                                                 const double* __restrict__ v2, ReduceScratch* ws,
                                                                 double* result)
{
    __shared__ double red[32];
    double s = 0.0;
    for(long long i = (long long)blockIdx.x * kReduceThreads + threadIdx.x; i < n; i += kReduceBlocks * kReduceThreads)
        s = fmax(s, fabs(v1[i] - v2[i]));
    s = block_max(s, red);
    double total;
    if(grid_reduce<true>(s, ws, kReduceBlocks, &total)) *result = total;
}

// ------------------------------------------------------------ launchers

int launch_spmv(int m, const ColorChunks& cc, const int* ell_col, const double* ell_val, const double* x, double* y,
                cudaStream_t s)
{
    k_spmv<<<cc.nchunks(), kBS, 0, s>>>(m, cc, ell_col, ell_val, x, y);
    HB_LAUNCHED();
    return 0;
}

// A colour's rows are final after its backward pass, or after its forward
// pass when the backward sweep (colours ublocks..0) does not revisit it: the
// passes that carry the fused prolongation.
int launch_symgs(int m, int nblocks, int ublocks, const int* sizes, const int* offsets, const int* ell_col,
                 const double* ell_val, const double* inv_diag, const double* r, double* x, cudaStream_t s,
                 Prolong<double> pro)
{
    for(int i = 0; i < nblocks; ++i)
    {
        if(sizes[i] <= 0) continue;
        k_symgs_sweep<<<(sizes[i] + kBS - 1) / kBS, kBS, 0, s>>>(m, m, sizes[i], offsets[i], ell_col, ell_val,
                                                                 inv_diag, r, x,
                                                                 i > ublocks ? pro : Prolong<double>{});
        HB_LAUNCHED();
    }
    for(int i = ublocks; i >= 0; --i)
    {
        if(sizes[i] <= 0) continue;
        k_symgs_sweep<<<(sizes[i] + kBS - 1) / kBS, kBS, 0, s>>>(m, m, sizes[i], offsets[i], ell_col, ell_val,
                                                                 inv_diag, r, x, pro);
        HB_LAUNCHED();
    }
    return 0;
}

int launch_sweep_color(int m, int ncols, int size, int offset, const int* ell_col, const double* ell_val,
                       const double* inv_diag, const double* r, double* x, cudaStream_t s)
{
    if(size <= 0) return 0;
    k_symgs_sweep<<<(size + kBS - 1) / kBS, kBS, 0, s>>>(m, ncols, size, offset, ell_col, ell_val, inv_diag, r, x,
                                                         Prolong<double>{});
    HB_LAUNCHED();
    return 0;
}

int launch_symgs_zero(int m, int nblocks, int ublocks, const int* sizes, const int* offsets, const int* ell_col,
                      const double* ell_val, const int* diag_idx, const double* diag, const double* inv_diag,
                      const double* r, double* x, cudaStream_t s, Prolong<double> pro, const ZgGroups* zg)
{
    for(int i = 0; i < nblocks; ++i)
    {
        if(sizes[i] <= 0) continue;
        const dim3 g((sizes[i] + kBS - 1) / kBS);
        const Prolong<double> pv = i > ublocks ? pro : Prolong<double>{};
        switch(zg ? zg[i].fhi : 3)
        {
        case 0:
            k_symgs_fwd0<0><<<g, kBS, 0, s>>>(m, sizes[i], offsets[i], ell_col, ell_val, diag_idx, inv_diag, r, x, pv);
            break;
        case 1:
            k_symgs_fwd0<1><<<g, kBS, 0, s>>>(m, sizes[i], offsets[i], ell_col, ell_val, diag_idx, inv_diag, r, x, pv);
            break;
        case 2:
            k_symgs_fwd0<2><<<g, kBS, 0, s>>>(m, sizes[i], offsets[i], ell_col, ell_val, diag_idx, inv_diag, r, x, pv);
            break;
        default:
            k_symgs_fwd0<3><<<g, kBS, 0, s>>>(m, sizes[i], offsets[i], ell_col, ell_val, diag_idx, inv_diag, r, x, pv);
        }
        HB_LAUNCHED();
    }
    for(int i = ublocks; i >= 0; --i)
    {
        if(sizes[i] <= 0) continue;
        const dim3 g((sizes[i] + kBS - 1) / kBS);
        switch(zg ? zg[i].blo : 0)
        {
        case 3:
            k_symgs_bwd0<3><<<g, kBS, 0, s>>>(m, sizes[i], offsets[i], ell_col, ell_val, diag_idx, diag, inv_diag, x,
                                              pro);
            break;
        case 2:
            k_symgs_bwd0<2><<<g, kBS, 0, s>>>(m, sizes[i], offsets[i], ell_col, ell_val, diag_idx, diag, inv_diag, x,
                                              pro);
            break;
        case 1:
            k_symgs_bwd0<1><<<g, kBS, 0, s>>>(m, sizes[i], offsets[i], ell_col, ell_val, diag_idx, diag, inv_diag, x,
                                              pro);
            break;
        default:
            k_symgs_bwd0<0><<<g, kBS, 0, s>>>(m, sizes[i], offsets[i], ell_col, ell_val, diag_idx, diag, inv_diag, x,
                                              pro);
        }
        HB_LAUNCHED();
    }
    return 0;
}

__global__ void k_diag_bounds(int lo, int hi, const int* __restrict__ diag_idx, int* __restrict__ out)
{
    int mn = kWidth, mx = 0;
    for(int i = lo + blockIdx.x * blockDim.x + threadIdx.x; i < hi; i += gridDim.x * blockDim.x)
    {
        const int d = diag_idx[i];
        mn = min(mn, d);
        mx = max(mx, d);
    }
    for(int o = 16; o > 0; o >>= 1)
    {
        mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    if((threadIdx.x & 31) == 0)
    {
        atomicMin(out, mn);
        atomicMax(out + 1, mx);
    }
}

int zero_guess_groups(int m, int nblocks, const int* offsets, const int* diag_idx, ZgGroups* zg, cudaStream_t s)
{
    if(nblocks <= 0) return 0;
    int* d = nullptr;
    HB_CUDA(cudaMallocAsync(&d, sizeof(int) * 2 * nblocks, s));
    std::vector<int> init(2 * nblocks), h(2 * nblocks);
    for(int c = 0; c < nblocks; ++c) init[2 * c] = kWidth, init[2 * c + 1] = 0;
    HB_CUDA(cudaMemcpyAsync(d, init.data(), sizeof(int) * 2 * nblocks, cudaMemcpyHostToDevice, s));
    for(int c = 0; c < nblocks; ++c)
    {
        const int lo = offsets[c], hi = offsets[c + 1];
        if(hi <= lo) continue;
        const int blocks = std::min((hi - lo + kBS - 1) / kBS, kReduceBlocks);
        k_diag_bounds<<<blocks, kBS, 0, s>>>(lo, hi, diag_idx, d + 2 * c);
        HB_LAUNCHED();
    }
    HB_CUDA(cudaMemcpyAsync(h.data(), d, sizeof(int) * 2 * nblocks, cudaMemcpyDeviceToHost, s));
    HB_CUDA(cudaStreamSynchronize(s));
    HB_CUDA(cudaFreeAsync(d, s));
    (void)m;
    for(int c = 0; c < nblocks; ++c)
    {
        const int dmin = h[2 * c], dmax = h[2 * c + 1];
        zg[c].fhi = (dmax + 8) / 9;                      // groups holding slots [0, dmax)
        zg[c].blo = dmin >= kWidth ? 0 : (dmin + 1) / 9; // first group holding slot dmin + 1
    }
    return 0;
}

__global__ void k_prolong_map(int nc, const int* __restrict__ inj_f, const int* __restrict__ inj_c,
                              int* __restrict__ pro_f)
{
    const int ic = blockIdx.x * kBS + threadIdx.x;
    if(ic < nc) pro_f[inj_c[ic]] = inj_f[ic];
}

int launch_prolong_map(int nc, const int* inj_f, const int* inj_c, int* pro_f, cudaStream_t s)
{
    k_prolong_map<<<(nc + kBS - 1) / kBS, kBS, 0, s>>>(nc, inj_f, inj_c, pro_f);
    HB_LAUNCHED();
    return 0;
}

int launch_restrict(int nc, const int* inj_f, const int* inj_c, int mf, const int* ell_col, const double* ell_val,
                    const double* rf, const double* xf, double* rc, cudaStream_t s)
{
    k_restrict<<<(nc + kBS - 1) / kBS, kBS, 0, s>>>(nc, inj_f, inj_c, mf, ell_col, ell_val, rf, xf, rc);
    HB_LAUNCHED();
    return 0;
}

int launch_restrict_axf(int nc, const int* inj_f, const int* inj_c, const double* rf, const double* axf, double* rc,
                        cudaStream_t s)
{
    k_restrict_axf<<<(nc + kBS - 1) / kBS, kBS, 0, s>>>(nc, inj_f, inj_c, rf, axf, rc);
    HB_LAUNCHED();
    return 0;
}

int launch_prolong(int nc, const int* inj_f, const int* inj_c, const double* xc, double* xf, cudaStream_t s)
{
    k_prolong<<<(nc + kBS - 1) / kBS, kBS, 0, s>>>(nc, inj_f, inj_c, xc, xf);
    HB_LAUNCHED();
    return 0;
}

int launch_dot(int n, const double* x, const double* y, ReduceScratch* ws, double* result, cudaStream_t s)
{
    k_dot<<<kReduceBlocks, kReduceThreads, 0, s>>>(n, x, y, ws, result);
    HB_LAUNCHED();
    return 0;
}

int launch_waxpby(int n, double alpha, const double* x, double beta, const double* y, double* w, cudaStream_t s)
{
    k_waxpby<<<(n + kBS - 1) / kBS, kBS, 0, s>>>(n, alpha, x, beta, y, w);
    HB_LAUNCHED();
    return 0;
}

int launch_waxpby_dot(int n, double alpha, const double* x, double* y, ReduceScratch* ws, double* result,
                      cudaStream_t s)
{
    k_waxpby_dot<<<kReduceBlocks, kReduceThreads, 0, s>>>(n, alpha, x, y, ws, result);
    HB_LAUNCHED();
    return 0;
}

int launch_residual_inf(int n, const double* v1, const double* v2, ReduceScratch* ws, double* result, cudaStream_t s)
{
    k_residual_inf<<<kReduceBlocks, kReduceThreads, 0, s>>>(n, v1, v2, ws, result);
    HB_LAUNCHED();
    return 0;
}

}  // namespace hb

using namespace hb;

// ------------------------------------------------------------------ C ABI

extern "C" int hpcgb200_spmv(int m, const int* ell_col, const double* ell_val, const double* x, double* y,
                             void* stream)
{
    HB_CHECK_ARG(m > 0 && ell_col && ell_val && x && y, "bad arguments");
    HB_CHECK_ARG(x != y, "x and y must differ");
    return launch_spmv(m, make_chunks(m, 0, nullptr), ell_col, ell_val, x, y, as_stream(stream));
}

static int check_colors(int m, int nblocks, int ublocks, const int* sizes, const int* offsets)
{
    HB_CHECK_ARG(nblocks >= 1 && nblocks <= HPCGB200_MAX_COLORS && ublocks < nblocks && sizes && offsets,
                 "bad color layout");
    long long total = 0;
    for(int i = 0; i < nblocks; ++i)
    {
        HB_CHECK_ARG(sizes[i] >= 0 && offsets[i] == total, "sizes/offsets inconsistent");
        total += sizes[i];
    }
    HB_CHECK_ARG(total == m, "color sizes do not sum to m");
    return 0;
}

extern "C" int hpcgb200_symgs(int m, int nblocks, int ublocks, const int* sizes, const int* offsets,
                              const int* ell_col, const double* ell_val, const double* inv_diag, const double* r,
                              double* x, void* stream)
{
    HB_CHECK_ARG(m > 0 && ell_col && ell_val && inv_diag && r && x, "bad arguments");
    HB_RETURN_IF(check_colors(m, nblocks, ublocks, sizes, offsets));
    return launch_symgs(m, nblocks, ublocks, sizes, offsets, ell_col, ell_val, inv_diag, r, x, as_stream(stream));
}

extern "C" int hpcgb200_symgs_zero(int m, int nblocks, int ublocks, const int* sizes, const int* offsets,
                                   const int* ell_col, const double* ell_val, const int* diag_idx,
                                   const double* diag, const double* inv_diag, const double* r, double* x,
                                   void* stream)
{
    HB_CHECK_ARG(m > 0 && ell_col && ell_val && diag_idx && diag && inv_diag && r && x, "bad arguments");
    HB_RETURN_IF(check_colors(m, nblocks, ublocks, sizes, offsets));
    return launch_symgs_zero(m, nblocks, ublocks, sizes, offsets, ell_col, ell_val, diag_idx, diag, inv_diag, r, x,
                             as_stream(stream));
}

extern "C" int hpcgb200_restrict_fused(int nc, const int* inj_f, const int* inj_c, int mf, const int* ell_col,
                                       const double* ell_val, const double* rf, const double* xf, double* rc,
                                       void* stream)
{
    HB_CHECK_ARG(nc > 0 && mf >= nc && inj_f && inj_c && ell_col && ell_val && rf && xf && rc, "bad arguments");
    return launch_restrict(nc, inj_f, inj_c, mf, ell_col, ell_val, rf, xf, rc, as_stream(stream));
}

extern "C" int hpcgb200_restrict(int nc, const int* inj_f, const int* inj_c, const double* rf, const double* axf,
                                 double* rc, void* stream)
{
    HB_CHECK_ARG(nc > 0 && inj_f && inj_c && rf && axf && rc, "bad arguments");
    return launch_restrict_axf(nc, inj_f, inj_c, rf, axf, rc, as_stream(stream));
}

extern "C" int hpcgb200_prolong(int nc, const int* inj_f, const int* inj_c, const double* xc, double* xf,
                                void* stream)
{
    HB_CHECK_ARG(nc > 0 && inj_f && inj_c && xc && xf, "bad arguments");
    return launch_prolong(nc, inj_f, inj_c, xc, xf, as_stream(stream));
}

static int check_ws(void* ws, size_t bytes)
{
    if(!ws || bytes < sizeof(ReduceScratch))
        return record_error(HPCGB200_ERR_WORKSPACE, "reduction workspace must be >= %zu bytes",
                            sizeof(ReduceScratch));
    if(reinterpret_cast<uintptr_t>(ws) % 16 != 0)
        return record_error(HPCGB200_ERR_ARG, "reduction workspace must be 16-byte aligned");
    return 0;
}

extern "C" int hpcgb200_dot(int n, const double* x, const double* y, double* result, void* workspace,
                            size_t workspace_bytes, void* stream)
{
    HB_CHECK_ARG(n >= 0 && x && y && result, "bad arguments");
    HB_RETURN_IF(check_ws(workspace, workspace_bytes));
    return launch_dot(n, x, y, reinterpret_cast<ReduceScratch*>(workspace), result, as_stream(stream));
}

extern "C" int hpcgb200_waxpby(int n, double alpha, const double* x, double beta, const double* y, double* w,
                               void* stream)
{
    HB_CHECK_ARG(n >= 0 && x && y && w, "bad arguments");
    if(n == 0) return 0;
    return launch_waxpby(n, alpha, x, beta, y, w, as_stream(stream));
}

extern "C" int hpcgb200_waxpby_dot(int n, double alpha, const double* x, double* y, double* result, void* workspace,
                                   size_t workspace_bytes, void* stream)
{
    HB_CHECK_ARG(n >= 0 && x && y && result, "bad arguments");
    HB_RETURN_IF(check_ws(workspace, workspace_bytes));
    return launch_waxpby_dot(n, alpha, x, y, reinterpret_cast<ReduceScratch*>(workspace), result, as_stream(stream));
}

extern "C" int hpcgb200_residual_inf(int n, const double* v1, const double* v2, double* result, void* workspace,
                                     size_t workspace_bytes, void* stream)
{
    HB_CHECK_ARG(n >= 0 && v1 && v2 && result, "bad arguments");
    HB_RETURN_IF(check_ws(workspace, workspace_bytes));
    return launch_residual_inf(n, v1, v2, reinterpret_cast<ReduceScratch*>(workspace), result, as_stream(stream));
}
