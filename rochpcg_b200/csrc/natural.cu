// Reference kernels in natural order (see natural.cuh).  Products and sums
// use the _rn intrinsics so that nvcc cannot contract them into fma: each
// row rounds exactly like the sequential C loops of the `_ref` sources
// compiled without fma contraction.
#include "natural.cuh"

namespace hb {

namespace {

constexpr int kNatBS = 256;

__global__ void __launch_bounds__(kNatBS) k_nat_spmv(NaturalLevel L, const double* __restrict__ x,
                                                     double* __restrict__ y)
{
    const long long row = (long long)blockIdx.x * kNatBS + threadIdx.x;
    if(row >= L.rows()) return;
    const size_t base = (size_t)row * kWidth;
    const int n = L.nnz[row];
    double sum = 0.0;
    for(int j = 0; j < n; ++j) sum = __dadd_rn(sum, __dmul_rn(L.val[base + j], x[L.ind[base + j]]));
    y[row] = sum;
}

// floor(a / 4) for any sign of a.
__device__ __forceinline__ int floor_div4(int a) { return a >= 0 ? a / 4 : -((3 - a) / 4); }

// One wavefront t of the Gauss-Seidel sweep (src/ComputeSYMGS_ref.cpp:68-85
// for one row).  Thread (iy, j) takes iz = izmin + j, ix = t - 2 iy - 4 iz;
// at most ceil(nx/4) + 1 values of iz meet 0 <= ix < nx for one (t, iy).
__global__ void __launch_bounds__(kNatBS) k_nat_gs_front(NaturalLevel L, int t, int width,
                                                         const double* __restrict__ r, double* x)
{
    const int idx = blockIdx.x * kNatBS + threadIdx.x;
    const int iy = idx / width;
    const int j = idx - iy * width;
    if(iy >= L.ny) return;
    const int u = t - 2 * iy;  // ix + 4 iz
    if(u < 0) return;
    const int izmin = max(0, -floor_div4(L.nx - 1 - u));  // ceil((u - nx + 1) / 4)
    const int iz = izmin + j;
    if(iz >= L.nz || 4 * iz > u) return;
    const int ix = u - 4 * iz;
    const long long row = ((long long)iz * L.ny + iy) * L.nx + ix;
    const size_t base = (size_t)row * kWidth;
    const int n = L.nnz[row];
    double sum = r[row];
    for(int q = 0; q < n; ++q) sum = __dsub_rn(sum, __dmul_rn(L.val[base + q], x[L.ind[base + q]]));
    const double d = L.val[base + L.diag_slot[row]];
    sum = __dadd_rn(sum, __dmul_rn(x[row], d));  // remove the diagonal term of the loop
    x[row] = __ddiv_rn(sum, d);
}

__global__ void k_nat_restrict(int nc, const int* __restrict__ f2c, const double* __restrict__ rf,
                               const double* __restrict__ axf, double* __restrict__ rc)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= nc) return;
    const int f = f2c[i];
    rc[i] = __dsub_rn(rf[f], axf[f]);
}

__global__ void k_nat_prolong(int nc, const int* __restrict__ f2c, const double* __restrict__ xc, double* xf)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= nc) return;
    const int f = f2c[i];
    xf[f] = __dadd_rn(xf[f], xc[i]);
}

// kForm 0: alpha == 1, 1: beta == 1, 2: general (src/ComputeWAXPBY_ref.cpp:65-85)
template <int kForm>
__global__ void k_nat_waxpby(int n, double alpha, const double* __restrict__ x, double beta,
                             const double* __restrict__ y, double* __restrict__ w)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n) return;
    if(kForm == 0) w[i] = __dadd_rn(x[i], __dmul_rn(beta, y[i]));
    else if(kForm == 1) w[i] = __dadd_rn(__dmul_rn(alpha, x[i]), y[i]);
    else w[i] = __dadd_rn(__dmul_rn(alpha, x[i]), __dmul_rn(beta, y[i]));
}

__global__ void __launch_bounds__(kReduceThreads) k_nat_dot(int n, const double* __restrict__ x,
                                                            const double* __restrict__ y, ReduceScratch* ws,
                                                            double* result)
{
    __shared__ double red[32];
    double s = 0.0;
    for(long long i = (long long)blockIdx.x * kReduceThreads + threadIdx.x; i < n; i += kReduceBlocks * kReduceThreads)
        s = __dadd_rn(s, __dmul_rn(x[i], y[i]));
    s = block_sum(s, red);
    double total;
    if(grid_reduce(s, ws, kReduceBlocks, &total)) *result = total;
}

__global__ void __launch_bounds__(kNatBS) k_nat_check(NaturalLevel L, long long gnx, long long gny, long long gnz,
                                                      long long gix0, long long giy0, long long giz0,
                                                      const long long* __restrict__ l2g,
                                                      const double* __restrict__ b, const double* __restrict__ x,
                                                      const double* __restrict__ xexact, unsigned long long* bad,
                                                      unsigned long long* nnz_total)
{
    __shared__ unsigned long long red[32];
    const long long row = (long long)blockIdx.x * kNatBS + threadIdx.x;
    unsigned long long my_bad = 0, my_nnz = 0;
    if(row < L.rows())
    {
        const int nxy = L.nx * L.ny;
        const int iz = (int)(row / nxy);
        const int iy = (int)((row - (long long)iz * nxy) / L.nx);
        const int ix = (int)(row - (long long)iz * nxy - (long long)iy * L.nx);
        const long long giz = giz0 + iz, giy = giy0 + iy, gix = gix0 + ix;
        const long long grow = giz * gnx * gny + giy * gnx + gix;
        const size_t base = (size_t)row * kWidth;
        bool ok = !l2g || l2g[row] == grow;
        int q = 0, dslot = -1;
        for(int sz = -1; sz <= 1; ++sz)
        {
            if(giz + sz < 0 || giz + sz >= gnz) continue;
            for(int sy = -1; sy <= 1; ++sy)
            {
                if(giy + sy < 0 || giy + sy >= gny) continue;
                for(int sx = -1; sx <= 1; ++sx)
                {
                    if(gix + sx < 0 || gix + sx >= gnx) continue;
                    // one rank: the local column is the global one
                    const long long col = grow + sz * gnx * gny + sy * gnx + sx;
                    const bool diag = sz == 0 && sy == 0 && sx == 0;
                    if(diag) dslot = q;
                    ok = ok && L.ind[base + q] == col && L.val[base + q] == (diag ? 26.0 : -1.0);
                    ++q;
                }
            }
        }
        ok = ok && L.nnz[row] == q && L.diag_slot[row] == dslot;
        if(b) ok = ok && b[row] == 26.0 - (double)(q - 1);
        if(x) ok = ok && x[row] == 0.0;
        if(xexact) ok = ok && xexact[row] == 1.0;
        my_bad = ok ? 0 : 1;
        my_nnz = (unsigned long long)L.nnz[row];
    }
    my_bad = block_sum(my_bad, red);
    my_nnz = block_sum(my_nnz, red);
    if(threadIdx.x == 0)
    {
        if(my_bad) atomicAdd(bad, my_bad);
        atomicAdd(nnz_total, my_nnz);
    }
}

unsigned grid_of(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

}  // namespace

int launch_nat_spmv(const NaturalLevel& L, const double* x, double* y, cudaStream_t s)
{
    k_nat_spmv<<<grid_of(L.rows(), kNatBS), kNatBS, 0, s>>>(L, x, y);
    HB_LAUNCHED();
    return 0;
}

int launch_nat_symgs(const NaturalLevel& L, const double* r, double* x, cudaStream_t s)
{
    const int fronts = natural_fronts(L.nx, L.ny, L.nz);
    const int width = (L.nx + 3) / 4 + 1;
    const unsigned grid = grid_of((long long)L.ny * width, kNatBS);
    for(int t = 0; t < fronts; ++t)
    {
        k_nat_gs_front<<<grid, kNatBS, 0, s>>>(L, t, width, r, x);
        HB_LAUNCHED();
    }
    for(int t = fronts - 1; t >= 0; --t)
    {
        k_nat_gs_front<<<grid, kNatBS, 0, s>>>(L, t, width, r, x);
        HB_LAUNCHED();
    }
    return 0;
}

int launch_nat_restrict(int nc, const int* f2c, const double* rf, const double* axf, double* rc, cudaStream_t s)
{
    k_nat_restrict<<<grid_of(nc, kNatBS), kNatBS, 0, s>>>(nc, f2c, rf, axf, rc);
    HB_LAUNCHED();
    return 0;
}

int launch_nat_prolong(int nc, const int* f2c, const double* xc, double* xf, cudaStream_t s)
{
    k_nat_prolong<<<grid_of(nc, kNatBS), kNatBS, 0, s>>>(nc, f2c, xc, xf);
    HB_LAUNCHED();
    return 0;
}

int launch_nat_waxpby(int n, double alpha, const double* x, double beta, const double* y, double* w, cudaStream_t s)
{
    const unsigned g = grid_of(n, kNatBS);
    if(alpha == 1.0) k_nat_waxpby<0><<<g, kNatBS, 0, s>>>(n, alpha, x, beta, y, w);
    else if(beta == 1.0) k_nat_waxpby<1><<<g, kNatBS, 0, s>>>(n, alpha, x, beta, y, w);
    else k_nat_waxpby<2><<<g, kNatBS, 0, s>>>(n, alpha, x, beta, y, w);
    HB_LAUNCHED();
    return 0;
}

int launch_nat_dot(int n, const double* x, const double* y, ReduceScratch* ws, double* result, cudaStream_t s)
{
    k_nat_dot<<<kReduceBlocks, kReduceThreads, 0, s>>>(n, x, y, ws, result);
    HB_LAUNCHED();
    return 0;
}

int launch_nat_check(const NaturalLevel& L, long long gnx, long long gny, long long gnz, long long gix0,
                     long long giy0, long long giz0, const long long* l2g, const double* b, const double* x,
                     const double* xexact, unsigned long long* bad, unsigned long long* nnz_total, cudaStream_t s)
{
    k_nat_check<<<grid_of(L.rows(), kNatBS), kNatBS, 0, s>>>(L, gnx, gny, gnz, gix0, giy0, giz0, l2g, b, x, xexact,
                                                            bad, nnz_total);
    HB_LAUNCHED();
    return 0;
}

// ------------------------------------------------------------------ C ABI

namespace {
int nat_args(int nx, int ny, int nz, const int* ind, const double* val, const signed char* nnz)
{
    if(nx < 1 || ny < 1 || nz < 1 || (long long)nx * ny * nz > 0x7fffffffLL)
        return record_error(HPCGB200_ERR_ARG, "natural-order kernel: bad dimensions %d x %d x %d", nx, ny, nz);
    if(!ind || !val || !nnz) return record_error(HPCGB200_ERR_ARG, "natural-order kernel: null matrix array");
    return 0;
}
}  // namespace

}  // namespace hb

extern "C" int hpcgb200_ref_spmv(int nx, int ny, int nz, const int* mtx_ind, const double* values,
                                 const signed char* nnz_in_row, const double* x, double* y, void* stream)
{
    HB_RETURN_IF(hb::nat_args(nx, ny, nz, mtx_ind, values, nnz_in_row));
    HB_CHECK_ARG(x && y && x != y, "x and y must be distinct device vectors");
    const hb::NaturalLevel L{nx, ny, nz, mtx_ind, values, reinterpret_cast<const int8_t*>(nnz_in_row), nullptr};
    return hb::launch_nat_spmv(L, x, y, hb::as_stream(stream));
}

extern "C" int hpcgb200_ref_symgs(int nx, int ny, int nz, const int* mtx_ind, const double* values,
                                  const signed char* nnz_in_row, const int* diag_slot, const double* r, double* x,
                                  void* stream)
{
    HB_RETURN_IF(hb::nat_args(nx, ny, nz, mtx_ind, values, nnz_in_row));
    HB_CHECK_ARG(diag_slot && r && x && r != x, "need the diagonal slots and distinct r, x");
    const hb::NaturalLevel L{nx, ny, nz, mtx_ind, values, reinterpret_cast<const int8_t*>(nnz_in_row), diag_slot};
    return hb::launch_nat_symgs(L, r, x, hb::as_stream(stream));
}
