// Kernels of the decomposed problem (see halo.cuh).  The halo kernels touch
// only the surface rows of a rank's brick; their fma order is the
// reference's (ascending external column, sum started at 0), so the halo part
// of every operator is bit-exact like the interior part.
#include "halo.cuh"

namespace hb {

namespace {

constexpr int kHaloBS = 128;

inline unsigned blocks_for(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

__global__ void k_halo_pack(int n, const int* __restrict__ send_perm, const double* __restrict__ x,
                            double* __restrict__ buf)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i < n) buf[i] = x[send_perm[i]];
}

__global__ void k_halo_spmv(int nh, int hw, const int* __restrict__ prow, const int* __restrict__ hcol,
                            const double* __restrict__ hval, const double* __restrict__ x, double* __restrict__ y)
{
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    if(h >= nh) return;
    double s = 0.0;
    for(int p = 0; p < hw; ++p)
    {
        const size_t idx = (size_t)p * nh + h;
        const int col = hcol[idx];
        if(col >= 0) s = fma(hval[idx], x[col], s);
    }
    const int row = prow[h];
    y[row] = y[row] + s;
}

__global__ void k_halo_symgs0(int nh, int hw, const int* __restrict__ prow, const int* __restrict__ hcol,
                              const double* __restrict__ hval, const double* __restrict__ inv_diag, int size0,
                              double* y)
{
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    if(h >= nh) return;
    const int row = prow[h];
    if(row >= size0) return;  // only colour 0 is swept before the exchange completes
    double s = 0.0;
    for(int p = 0; p < hw; ++p)
    {
        const size_t idx = (size_t)p * nh + h;
        const int col = hcol[idx];
        if(col >= 0) s = fma(-hval[idx], y[col], s);
    }
    y[row] = fma(s, inv_diag[row], y[row]);
}

__global__ void k_halo_restrict(int nh, int hw, const int* __restrict__ pc, const int* __restrict__ hcol,
                                const double* __restrict__ hval, const double* __restrict__ xf,
                                double* __restrict__ rc)
{
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    if(h >= nh) return;
    const int c = pc[h];
    if(c < 0) return;  // not an injected row
    double s = 0.0;
    for(int p = 0; p < hw; ++p)
    {
        const size_t idx = (size_t)p * nh + h;
        const int col = hcol[idx];
        if(col >= 0) s = fma(hval[idx], xf[col], s);
    }
    rc[c] = rc[c] - s;
}

__global__ void k_map_perm(int n, const int* __restrict__ in, const int* __restrict__ perm, int* __restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i < n) out[i] = in[i] >= 0 ? perm[in[i]] : -1;
}

__global__ void k_halo_insert(int nh, int hw, int m, const int* __restrict__ halo_rows,
                              const int* __restrict__ halo_ptr, const int* __restrict__ halo_cols,
                              const int* __restrict__ perm, int* __restrict__ ell_col, double* __restrict__ ell_val,
                              int* __restrict__ prow, int* __restrict__ hcol, double* __restrict__ hval,
                              double* __restrict__ b, int* status)
{
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    if(h >= nh) return;
    const int row = perm[halo_rows[h]];
    const int lo = halo_ptr[h], cnt = halo_ptr[h + 1] - lo;
    int nloc = 0;
    while(nloc < kWidth && ell_col[(size_t)nloc * m + row] >= 0) ++nloc;
    if(nloc + cnt > kWidth)
    {
        atomicExch(status, 1);
        return;
    }
    for(int q = nloc; q < kWidth; ++q)
        if(ell_col[(size_t)q * m + row] >= 0)
        {
            atomicExch(status, 2);
            return;
        }
    for(int j = 0; j < cnt; ++j)
    {
        const size_t idx = (size_t)(nloc + j) * m + row;
        ell_col[idx] = halo_cols[lo + j];
        ell_val[idx] = -1.0;
    }
    prow[h] = row;
    for(int j = 0; j < hw; ++j)
    {
        const size_t idx = (size_t)j * nh + h;
        hcol[idx] = j < cnt ? halo_cols[lo + j] : -1;
        hval[idx] = j < cnt ? -1.0 : 0.0;
    }
    if(b) b[row] -= (double)cnt;
}

__global__ void k_group_sum(int n, SlotPtrs ptrs)
{
    if(threadIdx.x != 0 || blockIdx.x != 0) return;
    double s = *ptrs.p[0];
    for(int r = 1; r < n; ++r) s += *ptrs.p[r];
    for(int r = 0; r < n; ++r) *ptrs.p[r] = s;
}

__global__ void k_dist_update_p(int n, int first, const double* __restrict__ z, double* __restrict__ p,
                                const double* __restrict__ sc)
{
    const double beta = first ? 0.0 : sc[kDistRtzNew] / sc[kDistRtz];
    for(long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    {
        const double zi = z[i];
        p[i] = first ? fma(0.0, zi, zi) : fma(beta, p[i], zi);
    }
}

__global__ void __launch_bounds__(kReduceThreads) k_dist_update_xr(int n, const double* __restrict__ p,
                                                                   const double* __restrict__ Ap,
                                                                   double* __restrict__ x, double* __restrict__ r,
                                                                   double* sc, ReduceScratch* ws)
{
    __shared__ double red[32];
    const double alpha = sc[kDistRtzNew] / sc[kDistPap];
    double s = 0.0;
    for(long long i = (long long)blockIdx.x * kReduceThreads + threadIdx.x; i < n;
        i += (long long)kReduceBlocks * kReduceThreads)
    {
        const double ri = fma(-alpha, Ap[i], r[i]);
        r[i] = ri;
        s = fma(ri, ri, s);
        x[i] = fma(alpha, p[i], x[i]);
    }
    s = block_sum(s, red);
    double total;
    if(grid_reduce(s, ws, kReduceBlocks, &total))
    {
        sc[kDistRr] = total;
        sc[kDistRtz] = sc[kDistRtzNew];  // no block reads kDistRtz in this kernel
    }
}

__global__ void __launch_bounds__(kReduceThreads) k_dist_residual(int n, const double* __restrict__ b,
                                                                  const double* __restrict__ Ax,
                                                                  double* __restrict__ r, double* sc,
                                                                  ReduceScratch* ws)
{
    __shared__ double red[32];
    double s = 0.0;
    for(long long i = (long long)blockIdx.x * kReduceThreads + threadIdx.x; i < n;
        i += (long long)kReduceBlocks * kReduceThreads)
    {
        const double ri = fma(-1.0, Ax[i], b[i]);
        r[i] = ri;
        s = fma(ri, ri, s);
    }
    s = block_sum(s, red);
    double total;
    if(grid_reduce(s, ws, kReduceBlocks, &total)) sc[kDistRr] = total;
}

}  // namespace

int launch_halo_pack(int n, const int* send_perm, const double* x, double* buf, cudaStream_t s)
{
    if(n <= 0) return 0;
    k_halo_pack<<<blocks_for(n, kHaloBS), kHaloBS, 0, s>>>(n, send_perm, x, buf);
    HB_LAUNCHED();
    return 0;
}

int launch_halo_spmv(int nh, int hw, const int* prow, const int* hcol, const double* hval, const double* x,
                     double* y, cudaStream_t s)
{
    if(nh <= 0) return 0;
    k_halo_spmv<<<blocks_for(nh, kHaloBS), kHaloBS, 0, s>>>(nh, hw, prow, hcol, hval, x, y);
    HB_LAUNCHED();
    return 0;
}

int launch_halo_symgs0(int nh, int hw, const int* prow, const int* hcol, const double* hval,
                       const double* inv_diag, int size0, double* y, cudaStream_t s)
{
    if(nh <= 0) return 0;
    k_halo_symgs0<<<blocks_for(nh, kHaloBS), kHaloBS, 0, s>>>(nh, hw, prow, hcol, hval, inv_diag, size0, y);
    HB_LAUNCHED();
    return 0;
}

int launch_halo_restrict(int nh, int hw, const int* pc, const int* hcol, const double* hval, const double* xf,
                         double* rc, cudaStream_t s)
{
    if(nh <= 0) return 0;
    k_halo_restrict<<<blocks_for(nh, kHaloBS), kHaloBS, 0, s>>>(nh, hw, pc, hcol, hval, xf, rc);
    HB_LAUNCHED();
    return 0;
}

int launch_map_perm(int n, const int* in, const int* perm, int* out, cudaStream_t s)
{
    if(n <= 0) return 0;
    k_map_perm<<<blocks_for(n, kHaloBS), kHaloBS, 0, s>>>(n, in, perm, out);
    HB_LAUNCHED();
    return 0;
}

int launch_halo_insert(int nh, int hw, int m, const int* halo_rows, const int* halo_ptr, const int* halo_cols,
                       const int* perm, int* ell_col, double* ell_val, int* prow, int* hcol, double* hval, double* b,
                       int* status, cudaStream_t s)
{
    if(nh <= 0) return 0;
    k_halo_insert<<<blocks_for(nh, kHaloBS), kHaloBS, 0, s>>>(nh, hw, m, halo_rows, halo_ptr, halo_cols, perm,
                                                              ell_col, ell_val, prow, hcol, hval, b, status);
    HB_LAUNCHED();
    return 0;
}

int launch_group_sum(int n, const SlotPtrs& ptrs, cudaStream_t s)
{
    if(n <= 0 || n > kMaxGroup) return record_error(HPCGB200_ERR_ARG, "group of %d ranks", n);
    k_group_sum<<<1, 32, 0, s>>>(n, ptrs);
    HB_LAUNCHED();
    return 0;
}

int launch_dist_update_p(int n, int first, const double* z, double* p, const double* sc, cudaStream_t s)
{
    k_dist_update_p<<<kReduceBlocks, kReduceThreads, 0, s>>>(n, first, z, p, sc);
    HB_LAUNCHED();
    return 0;
}

int launch_dist_update_xr(int n, const double* p, const double* Ap, double* x, double* r, double* sc,
                          ReduceScratch* ws, cudaStream_t s)
{
    k_dist_update_xr<<<kReduceBlocks, kReduceThreads, 0, s>>>(n, p, Ap, x, r, sc, ws);
    HB_LAUNCHED();
    return 0;
}

int launch_dist_residual(int n, const double* b, const double* Ax, double* r, double* sc, ReduceScratch* ws,
                         cudaStream_t s)
{
    k_dist_residual<<<kReduceBlocks, kReduceThreads, 0, s>>>(n, b, Ax, r, sc, ws);
    HB_LAUNCHED();
    return 0;
}

}  // namespace hb
