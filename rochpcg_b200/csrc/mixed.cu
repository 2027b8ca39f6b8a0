// FP32 implicit-stencil V-cycle kernels (see mixed.cuh).  Per row they read
// the float residual, the float diagonal reciprocal and the 26 gathered
// neighbours, i.e. ~12 B of streamed data instead of 27 x 12 B of ELL.
#include <algorithm>
#include <array>

#include "mixed.cuh"

namespace hb {

constexpr int kBS32 = 256;

bool make_stencil_level(int nx, int ny, int nz, const int* offsets, const int color_of_par[8], StencilLevel* out)
{
    StencilLevel L{};
    L.nx = nx;
    L.ny = ny;
    L.nz = nz;
    L.m = nx * ny * nz;
    L.ncolors = 8;
    bool seen[8] = {};
    for(int p = 0; p < 8; ++p)
    {
        const int v = color_of_par[p];
        if(v < 0 || v >= 8 || seen[v]) return false;
        seen[v] = true;
        L.color_of_par[p] = v;
        L.par[v] = p;
    }
    for(int v = 0; v <= 8; ++v) L.offsets[v] = offsets[v];
    for(int v = 0; v < 8; ++v)
    {
        const int p = L.par[v];
        const int px = (p >> 2) & 1, py = (p >> 1) & 1, pz = p & 1;
        const int bx = (nx - px + 1) / 2, by = (ny - py + 1) / 2, bz = (nz - pz + 1) / 2;
        if(bx <= 0 || by <= 0 || bz <= 0) return false;
        if(L.offsets[v + 1] - L.offsets[v] != bx * by * bz) return false;
        L.bx[v] = bx;
        L.by[v] = by;
        // ELL slot order of colour v: neighbour colour, then (dz,dy,dx)
        std::array<std::array<int, 5>, 27> e{};
        int k = 0;
        for(int dz = -1; dz <= 1; ++dz)
            for(int dy = -1; dy <= 1; ++dy)
                for(int dx = -1; dx <= 1; ++dx)
                {
                    const int p2 = p ^ (((dx & 1) << 2) | ((dy & 1) << 1) | (dz & 1));
                    e[k++] = {L.color_of_par[p2], dz, dy, dx, 0};
                }
        std::sort(e.begin(), e.end());
        for(int j = 0; j < 27; ++j)
        {
            const int v2 = e[j][0], dz = e[j][1], dy = e[j][2], dx = e[j][3];
            L.nb[v][j] = (unsigned short)((dx + 1) | ((dy + 1) << 2) | ((dz + 1) << 4) | (v2 << 8));
            if(dx == 0 && dy == 0 && dz == 0) L.diag_pos[v] = (unsigned char)j;
        }
    }
    *out = L;
    return true;
}

__device__ __forceinline__ void row_coords(const StencilLevel& L, int v, int row, int& ix, int& iy, int& iz)
{
    const int q = row - L.offsets[v];
    const int bx = L.bx[v], by = L.by[v];
    const int kx = q % bx;
    const int t = q / bx;
    const int ky = t % by;
    const int kz = t / by;
    const int p = L.par[v];
    ix = 2 * kx + ((p >> 2) & 1);
    iy = 2 * ky + ((p >> 1) & 1);
    iz = 2 * kz + (p & 1);
}

// Column of neighbour entry e of a row at (ix,iy,iz); false outside the grid.
__device__ __forceinline__ bool nb_col(const StencilLevel& L, unsigned e, int ix, int iy, int iz, int& col)
{
    const int x = ix + (int)(e & 3) - 1;
    const int y = iy + (int)((e >> 2) & 3) - 1;
    const int z = iz + (int)((e >> 4) & 3) - 1;
    if((unsigned)x >= (unsigned)L.nx || (unsigned)y >= (unsigned)L.ny || (unsigned)z >= (unsigned)L.nz) return false;
    const int v2 = (int)(e >> 8);
    col = L.offsets[v2] + ((z >> 1) * L.by[v2] + (y >> 1)) * L.bx[v2] + (x >> 1);
    return true;
}

// Forward zero-guess sweep of colour v: only neighbours of earlier colours,
// which are exactly the slots before the diagonal.
template <bool kFromDouble>
__global__ void __launch_bounds__(kBS32) k32_fwd0(const StencilLevel L, int v, const float* __restrict__ inv_diag32,
                                                  const double* __restrict__ r64, float* __restrict__ r32, float* x)
{
    const int size = L.offsets[v + 1] - L.offsets[v];
    const int gid = blockIdx.x * kBS32 + threadIdx.x;
    if(gid >= size) return;
    const int row = L.offsets[v] + gid;
    float sum;
    if(kFromDouble)
    {
        sum = (float)r64[row];
        r32[row] = sum;
    }
    else
    {
        sum = r32[row];
    }
    if(v > 0)
    {
        int ix, iy, iz;
        row_coords(L, v, row, ix, iy, iz);
        const int dp = L.diag_pos[v];
#pragma unroll
        for(int j = 0; j < 27; ++j)
        {
            if(j >= dp) break;
            int col;
            if(nb_col(L, L.nb[v][j], ix, iy, iz, col)) sum = sum + x[col];
        }
    }
    x[row] = sum * inv_diag32[row];
}

// Backward zero-guess sweep of colour v: x = (d x - sum of later-colour
// neighbours * (-1)) / d.
__global__ void __launch_bounds__(kBS32) k32_bwd0(const StencilLevel L, int v, const float* __restrict__ diag32,
                                                  const float* __restrict__ inv_diag32, float* x)
{
    const int size = L.offsets[v + 1] - L.offsets[v];
    const int gid = blockIdx.x * kBS32 + threadIdx.x;
    if(gid >= size) return;
    const int row = L.offsets[v] + gid;
    int ix, iy, iz;
    row_coords(L, v, row, ix, iy, iz);
    float sum = __fmul_rn(x[row], diag32[row]);
    const int dp = L.diag_pos[v];
#pragma unroll
    for(int j = 0; j < 27; ++j)
    {
        if(j <= dp) continue;
        int col;
        if(nb_col(L, L.nb[v][j], ix, iy, iz, col)) sum = sum + x[col];
    }
    x[row] = sum * inv_diag32[row];
}

// Full sweep of colour v; optionally stores the final value as double.
__global__ void __launch_bounds__(kBS32) k32_sweep(const StencilLevel L, int v, const float* __restrict__ inv_diag32,
                                                   const float* __restrict__ r, float* x, double* __restrict__ z64)
{
    const int size = L.offsets[v + 1] - L.offsets[v];
    const int gid = blockIdx.x * kBS32 + threadIdx.x;
    if(gid >= size) return;
    const int row = L.offsets[v] + gid;
    int ix, iy, iz;
    row_coords(L, v, row, ix, iy, iz);
    float sum = r[row];
    const int dp = L.diag_pos[v];
#pragma unroll
    for(int j = 0; j < 27; ++j)
    {
        if(j == dp) continue;
        int col;
        if(nb_col(L, L.nb[v][j], ix, iy, iz, col)) sum = sum + x[col];
    }
    const float xn = sum * inv_diag32[row];
    x[row] = xn;
    if(z64) z64[row] = (double)xn;
}

// Residual at the injected rows (all of parity class 0, colour v0).
__global__ void __launch_bounds__(kBS32) k32_restrict(const StencilLevel L, int v0, int nc, const int* __restrict__ inj_f,
                                                      const int* __restrict__ inj_c, const float* __restrict__ diag32,
                                                      const float* __restrict__ rf, const float* __restrict__ xf,
                                                      float* __restrict__ rc)
{
    const int ic = blockIdx.x * kBS32 + threadIdx.x;
    if(ic >= nc) return;
    const int row = inj_f[ic];
    int ix, iy, iz;
    row_coords(L, v0, row, ix, iy, iz);
    float sum = rf[row];
    const int dp = L.diag_pos[v0];
#pragma unroll
    for(int j = 0; j < 27; ++j)
    {
        if(j == dp)
        {
            sum = fmaf(-diag32[row], xf[row], sum);
            continue;
        }
        int col;
        if(nb_col(L, L.nb[v0][j], ix, iy, iz, col)) sum = sum + xf[col];
    }
    rc[inj_c[ic]] = sum;
}

__global__ void __launch_bounds__(kBS32) k32_prolong(int nc, const int* __restrict__ inj_f, const int* __restrict__ inj_c,
                                                     const float* __restrict__ xc, float* __restrict__ xf)
{
    const int ic = blockIdx.x * kBS32 + threadIdx.x;
    if(ic >= nc) return;
    xf[inj_f[ic]] += xc[inj_c[ic]];
}

__global__ void k_diag32(int m, const double* __restrict__ diag, float* __restrict__ d32, float* __restrict__ inv32)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= m) return;
    const float d = (float)diag[i];
    d32[i] = d;
    inv32[i] = 1.0f / d;
}

__global__ void k_stencil_check(const StencilLevel L, const int* __restrict__ perm, const int* __restrict__ ell_col,
                                const double* __restrict__ ell_val, int* bad)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= L.m) return;
    int nbad = 0;
    // natural row i -> expected permuted position
    {
        const int iz = i / (L.nx * L.ny);
        const int iy = i / L.nx - L.ny * iz;
        const int ix = i - iz * L.nx * L.ny - iy * L.nx;
        const int p = ((ix & 1) << 2) | ((iy & 1) << 1) | (iz & 1);
        const int v = L.color_of_par[p];
        const int expect = L.offsets[v] + ((iz >> 1) * L.by[v] + (iy >> 1)) * L.bx[v] + (ix >> 1);
        nbad += perm[i] != expect;
    }
    // permuted row i -> its ELL row must be the implicit neighbour list
    {
        int v = 0;
        while(v + 1 < 8 && i >= L.offsets[v + 1]) ++v;
        int ix, iy, iz;
        row_coords(L, v, i, ix, iy, iz);
        int slot = 0;
        for(int j = 0; j < 27; ++j)
        {
            int col;
            if(!nb_col(L, L.nb[v][j], ix, iy, iz, col)) continue;
            const size_t idx = (size_t)slot * L.m + i;
            nbad += ell_col[idx] != col;
            if(j != L.diag_pos[v]) nbad += ell_val[idx] != -1.0;
            ++slot;
        }
        for(; slot < 27; ++slot) nbad += ell_col[(size_t)slot * L.m + i] != -1;
    }
    if(nbad) atomicAdd(bad, nbad);
}

static inline unsigned nblk(int n) { return (unsigned)((n + kBS32 - 1) / kBS32); }

int launch_stencil_check(const StencilLevel& L, const int* perm, const int* ell_col, const double* ell_val, int* bad,
                         cudaStream_t s)
{
    k_stencil_check<<<nblk(L.m), kBS32, 0, s>>>(L, perm, ell_col, ell_val, bad);
    HB_LAUNCHED();
    return 0;
}

int launch_diag32(int m, const double* diag, float* diag32, float* inv_diag32, cudaStream_t s)
{
    k_diag32<<<nblk(m), kBS32, 0, s>>>(m, diag, diag32, inv_diag32);
    HB_LAUNCHED();
    return 0;
}

int launch32_symgs_zero(const StencilLevel& L, const float* diag32, const float* inv_diag32, const double* r64,
                        float* r32, float* x, cudaStream_t s)
{
    const int n = L.ncolors;
    for(int v = 0; v < n; ++v)
    {
        const int size = L.offsets[v + 1] - L.offsets[v];
        if(size <= 0) continue;
        if(r64) k32_fwd0<true><<<nblk(size), kBS32, 0, s>>>(L, v, inv_diag32, r64, r32, x);
        else k32_fwd0<false><<<nblk(size), kBS32, 0, s>>>(L, v, inv_diag32, nullptr, r32, x);
        HB_LAUNCHED();
    }
    for(int v = n - 2; v >= 0; --v)
    {
        const int size = L.offsets[v + 1] - L.offsets[v];
        if(size <= 0) continue;
        k32_bwd0<<<nblk(size), kBS32, 0, s>>>(L, v, diag32, inv_diag32, x);
        HB_LAUNCHED();
    }
    return 0;
}

int launch32_symgs(const StencilLevel& L, const float* inv_diag32, const float* r, float* x, double* z64,
                   cudaStream_t s)
{
    const int n = L.ncolors;
    for(int v = 0; v < n; ++v)
    {
        const int size = L.offsets[v + 1] - L.offsets[v];
        if(size <= 0) continue;
        // colour n-1 is final after the forward sweep (the backward sweep starts at n-2)
        k32_sweep<<<nblk(size), kBS32, 0, s>>>(L, v, inv_diag32, r, x, v == n - 1 ? z64 : nullptr);
        HB_LAUNCHED();
    }
    for(int v = n - 2; v >= 0; --v)
    {
        const int size = L.offsets[v + 1] - L.offsets[v];
        if(size <= 0) continue;
        k32_sweep<<<nblk(size), kBS32, 0, s>>>(L, v, inv_diag32, r, x, z64);
        HB_LAUNCHED();
    }
    return 0;
}

int launch32_restrict(const StencilLevel& Lf, int nc, const int* inj_f, const int* inj_c, const float* diag32,
                      const float* rf, const float* xf, float* rc, cudaStream_t s)
{
    k32_restrict<<<nblk(nc), kBS32, 0, s>>>(Lf, Lf.color_of_par[0], nc, inj_f, inj_c, diag32, rf, xf, rc);
    HB_LAUNCHED();
    return 0;
}

int launch32_prolong(int nc, const int* inj_f, const int* inj_c, const float* xc, float* xf, cudaStream_t s)
{
    k32_prolong<<<nblk(nc), kBS32, 0, s>>>(nc, inj_f, inj_c, xc, xf);
    HB_LAUNCHED();
    return 0;
}

}  // namespace hb
