// Implicit-stencil kernels (see mixed.cuh).  Per row the FP32 sweeps stream
// the float residual and diagonal reciprocal (8 B) and write x (4 B); the 26
// neighbours are gathered with all loads issued before the ordered adds (an
// absent neighbour contributes -0.0f, which leaves any sum unchanged, so the
// rounding sequence is exactly the ELL sweep's).
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <array>
#include <cstdint>
#include <cstdlib>
#include <memory>
#include <mutex>
#include <type_traits>
#include <utility>
#include <vector>

#include "mixed.cuh"
#include "tma.cuh"

namespace hb {

constexpr int kBS32 = 256;

// Slot tables of the colouring the reference's JPL rounds produce (parity
// class p -> colour 7,2,3,6,5,4,1,0, packed in nibbles, class 0 lowest) as
// compile-time constants: per ELL slot j of a row of class `cls`, its
// neighbour offset, the low two bits of its column delta (every other term of
// the delta is a multiple of 4 when the colour bricks are 4-aligned), the
// faces that remove it, and the diagonal slot.
struct KvSlots
{
    int dx[27], dy[27], dz[27];
    int s[27];        // delta & 3
    unsigned bm[27];  // faces that remove the slot (bit order of StencilTab::bmask)
    int dp;
};

__host__ __device__ constexpr int canon_colour(int par) { return (int)((0x01456327u >> (4 * par)) & 15u); }

__host__ __device__ constexpr KvSlots kv_slots(int cls)
{
    KvSlots r{};
    int key[27] = {}, dxs[27] = {}, dys[27] = {}, dzs[27] = {};
    int k = 0;
    for(int dz = -1; dz <= 1; ++dz)
        for(int dy = -1; dy <= 1; ++dy)
            for(int dx = -1; dx <= 1; ++dx)
            {
                const int col = canon_colour(cls ^ (((dx & 1) << 2) | ((dy & 1) << 1) | (dz & 1)));
                key[k] = ((col * 3 + (dz + 1)) * 3 + (dy + 1)) * 3 + (dx + 1);
                dxs[k] = dx;
                dys[k] = dy;
                dzs[k] = dz;
                ++k;
            }
    for(int a = 1; a < 27; ++a)
        for(int b = a; b > 0 && key[b - 1] > key[b]; --b)
        {
            int t = key[b]; key[b] = key[b - 1]; key[b - 1] = t;
            t = dxs[b]; dxs[b] = dxs[b - 1]; dxs[b - 1] = t;
            t = dys[b]; dys[b] = dys[b - 1]; dys[b - 1] = t;
            t = dzs[b]; dzs[b] = dzs[b - 1]; dzs[b - 1] = t;
        }
    const int px = (cls >> 2) & 1;
    for(int j = 0; j < 27; ++j)
    {
        r.dx[j] = dxs[j];
        r.dy[j] = dys[j];
        r.dz[j] = dzs[j];
        r.s[j] = ((px + dxs[j] + 2) / 2 - 1) & 3;
        r.bm[j] = (dxs[j] < 0 ? 1u : 0u) | (dxs[j] > 0 ? 2u : 0u) | (dys[j] < 0 ? 4u : 0u) | (dys[j] > 0 ? 8u : 0u) |
                  (dzs[j] < 0 ? 16u : 0u) | (dzs[j] > 0 ? 32u : 0u);
        if(dxs[j] == 0 && dys[j] == 0 && dzs[j] == 0) r.dp = j;
    }
    return r;
}

template <int kCls>
struct KvTab
{
    static constexpr KvSlots s = kv_slots(kCls);
};

// The level's runtime tables agree with the compile-time ones (canonical
// colouring, 4-aligned bricks): the kernels may use the latter.
static bool kv_tables_match(const StencilLevel& L)
{
    if(!L.even || L.ncolors != 8) return false;
    for(int v = 0; v < 8; ++v)
    {
        if(L.bx[v] % 4 || L.offsets[v] % 4) return false;
        const int p = L.par[v];
        if(canon_colour(p) != v) return false;
        const KvSlots k = kv_slots(p);
        const StencilTab& T = L.tab[v];
        if(T.dp != k.dp) return false;
        for(int j = 0; j < 27; ++j)
        {
            const int dx = (int)(T.nb[j] & 3) - 1, dy = (int)((T.nb[j] >> 2) & 3) - 1, dz = (int)((T.nb[j] >> 4) & 3) - 1;
            if(dx != k.dx[j] || dy != k.dy[j] || dz != k.dz[j]) return false;
            if((T.delta[j] & 3) != k.s[j] || T.bmask[j] != k.bm[j]) return false;
        }
    }
    return true;
}

bool make_stencil_level(int nx, int ny, int nz, const int* offsets, const int color_of_par[8], StencilLevel* out)
{
    StencilLevel L{};
    L.nx = nx;
    L.ny = ny;
    L.nz = nz;
    L.m = nx * ny * nz;
    L.ncolors = 8;
    L.even = (nx % 2 == 0 && ny % 2 == 0 && nz % 2 == 0) ? 1 : 0;
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
    }
    for(int v = 0; v < 8; ++v)
    {
        const int p = L.par[v];
        const int px = (p >> 2) & 1, py = (p >> 1) & 1, pz = p & 1;
        // ELL slot order of colour v: neighbour colour, then (dz,dy,dx)
        std::array<std::array<int, 4>, 27> e{};
        int k = 0;
        for(int dz = -1; dz <= 1; ++dz)
            for(int dy = -1; dy <= 1; ++dy)
                for(int dx = -1; dx <= 1; ++dx)
                {
                    const int p2 = p ^ (((dx & 1) << 2) | ((dy & 1) << 1) | (dz & 1));
                    e[k++] = {L.color_of_par[p2], dz, dy, dx};
                }
        std::sort(e.begin(), e.end());
        StencilTab& T = L.tab[v];
        for(int j = 0; j < 27; ++j)
        {
            const int v2 = e[j][0], dz = e[j][1], dy = e[j][2], dx = e[j][3];
            T.nb[j] = (unsigned short)((dx + 1) | ((dy + 1) << 2) | ((dz + 1) << 4) | (v2 << 8));
            if(dx == 0 && dy == 0 && dz == 0) T.dp = j;
            // brick-coordinate steps: floor((parity + d) / 2)
            const int dkx = (px + dx + 2) / 2 - 1, dky = (py + dy + 2) / 2 - 1, dkz = (pz + dz + 2) / 2 - 1;
            T.delta[j] = (L.offsets[v2] - L.offsets[v]) + (dkz * L.by[v2] + dky) * L.bx[v2] + dkx;
            T.bmask[j] = (unsigned char)((dx < 0 ? 1 : 0) | (dx > 0 ? 2 : 0) | (dy < 0 ? 4 : 0) | (dy > 0 ? 8 : 0) |
                                         (dz < 0 ? 16 : 0) | (dz > 0 ? 32 : 0));
        }
    }
    L.canon = kv_tables_match(L) ? 1 : 0;
    *out = L;
    return true;
}

// Column of neighbour entry e of a row at (ix,iy,iz) for any grid; false outside it.
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

// Everything a launch over the rows of ONE colour needs, passed as its own
// kernel parameter: the unrolled slot loop then reads the table from the
// constant bank at static offsets (a table indexed by a runtime colour would
// cost a constant-cache load per slot and per thread).
struct ColorLaunch
{
    StencilTab tb;
    int v, off, bx, by, bz, par;
    int nx, ny, nz, even;
};

static ColorLaunch color_launch(const StencilLevel& L, int v)
{
    ColorLaunch c{};
    c.tb = L.tab[v];
    c.v = v;
    c.off = L.offsets[v];
    c.bx = L.bx[v];
    c.by = L.by[v];
    c.par = L.par[v];
    c.bz = (L.nz - (c.par & 1) + 1) / 2;
    c.nx = L.nx;
    c.ny = L.ny;
    c.nz = L.nz;
    c.even = L.even;
    return c;
}

// Faces of the grid a point lies on (bit order as StencilTab::bmask).
__device__ __forceinline__ unsigned face_mask(const ColorLaunch& c, int ix, int iy, int iz)
{
    return (ix == 0 ? 1u : 0u) | (ix == c.nx - 1 ? 2u : 0u) | (iy == 0 ? 4u : 0u) | (iy == c.ny - 1 ? 8u : 0u) |
           (iz == 0 ? 16u : 0u) | (iz == c.nz - 1 ? 32u : 0u);
}

struct BrickRow
{
    int row, ix, iy, iz;
    unsigned mask;
    bool in, fast;
};

// Thread (kx, ky) of a 32 x 8 block, brick plane kz: position of the row
// without divisions.  `fast`: even grid and no lane of the warp on a face.
__device__ __forceinline__ BrickRow brick_row(const ColorLaunch& c, int kz)
{
    BrickRow b;
    const int kx = blockIdx.x * 32 + threadIdx.x;
    const int ky = blockIdx.y * 8 + threadIdx.y;
    b.in = kx < c.bx && ky < c.by && kz < c.bz;
    b.ix = 2 * kx + ((c.par >> 2) & 1);
    b.iy = 2 * ky + ((c.par >> 1) & 1);
    b.iz = 2 * kz + (c.par & 1);
    b.mask = b.in ? face_mask(c, b.ix, b.iy, b.iz) : 0x3fu;
    b.fast = c.even && __all_sync(0xffffffffu, b.mask == 0u);
    b.row = c.off + (kz * c.by + ky) * c.bx + kx;
    return b;
}

// Position of a given row of the colour (1-D launches: restriction).
__device__ __forceinline__ BrickRow row_of(const ColorLaunch& c, int row, bool in)
{
    BrickRow b;
    const int q = in ? row - c.off : 0;
    const int t = q / c.bx;
    const int kx = q - t * c.bx;
    const int kz = t / c.by;
    const int ky = t - kz * c.by;
    b.in = in;
    b.row = row;
    b.ix = 2 * kx + ((c.par >> 2) & 1);
    b.iy = 2 * ky + ((c.par >> 1) & 1);
    b.iz = 2 * kz + (c.par & 1);
    b.mask = in ? face_mask(c, b.ix, b.iy, b.iz) : 0x3fu;
    b.fast = c.even && __all_sync(0xffffffffu, b.mask == 0u);
    return b;
}

// Slot selection of the sweeps.
enum Sel
{
    kBefore = 0,  // slots before the diagonal (earlier colours)
    kAfter = 1,   // slots after the diagonal (later colours)
    kOff = 2      // every off-diagonal slot
};

template <int kSel>
__device__ __forceinline__ bool selected(int j, int dp)
{
    return kSel == kBefore ? j < dp : (kSel == kAfter ? j > dp : j != dp);
}

// Neighbour values of slots 0..26 in ELL order; `fill` where the slot is not
// selected or the neighbour does not exist.  Fast path: constant deltas, no
// masks.  Even grids: deltas + per-lane face masks.  Odd grids: per-slot
// brick coordinates.
template <int kSel, bool kEven, typename T>
__device__ __forceinline__ void gather(const StencilLevel& L, const ColorLaunch& c, const BrickRow& b, const T* x,
                                       T fill, T (&val)[27])
{
    if(kEven && b.fast)
    {
#pragma unroll
        for(int j = 0; j < 27; ++j) val[j] = selected<kSel>(j, c.tb.dp) ? x[b.row + c.tb.delta[j]] : fill;
        return;
    }
#pragma unroll
    for(int j = 0; j < 27; ++j)
    {
        int col = b.row;
        bool ok;
        if(kEven)
        {
            col = b.row + c.tb.delta[j];
            ok = selected<kSel>(j, c.tb.dp) && !(b.mask & c.tb.bmask[j]);
        }
        else
        {
            ok = selected<kSel>(j, c.tb.dp) && nb_col(L, c.tb.nb[j], b.ix, b.iy, b.iz, col);
        }
        val[j] = ok ? x[col] : fill;
    }
}

constexpr unsigned kBrickThreads = 256;

inline dim3 brick_grid(const ColorLaunch& c)
{
    return dim3((unsigned)((c.bx + 31) / 32), (unsigned)((c.by + 7) / 8), (unsigned)c.bz);
}

template <bool kEven, bool kFromDouble>
__global__ void __launch_bounds__(kBrickThreads) k32_fwd0(const ColorLaunch c, const StencilLevel L,
                                                          const float* __restrict__ inv_diag32,
                                                          const double* __restrict__ r64, float* __restrict__ r32,
                                                          float* x, Prolong<float> pro)
{
    const BrickRow b = brick_row(c, blockIdx.z);
    if(!b.in) return;
    const int row = b.row;
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
    if(c.tb.dp > 0)
    {
        float val[27];
        gather<kBefore, kEven>(L, c, b, x, -0.0f, val);
#pragma unroll
        for(int j = 0; j < 27; ++j) sum = sum + val[j];
    }
    const float xn = sum * inv_diag32[row];
    x[row] = xn;
    pro.add(row, xn);
}

template <bool kEven>
__global__ void __launch_bounds__(kBrickThreads) k32_bwd0(const ColorLaunch c, const StencilLevel L,
                                                          const float* __restrict__ diag32,
                                                          const float* __restrict__ inv_diag32, float* x,
                                                          Prolong<float> pro)
{
    const BrickRow b = brick_row(c, blockIdx.z);
    if(!b.in) return;
    const int row = b.row;
    float val[27];
    gather<kAfter, kEven>(L, c, b, x, -0.0f, val);
    float sum = __fmul_rn(x[row], diag32[row]);
#pragma unroll
    for(int j = 0; j < 27; ++j) sum = sum + val[j];
    const float xn = sum * inv_diag32[row];
    x[row] = xn;
    pro.add(row, xn);
}

template <bool kEven>
__global__ void __launch_bounds__(kBrickThreads) k32_sweep(const ColorLaunch c, const StencilLevel L,
                                                           const float* __restrict__ inv_diag32,
                                                           const float* __restrict__ r, float* x,
                                                           double* __restrict__ z64, Prolong<float> pro)
{
    const BrickRow b = brick_row(c, blockIdx.z);
    if(!b.in) return;
    const int row = b.row;
    float val[27];
    gather<kOff, kEven>(L, c, b, x, -0.0f, val);
    float sum = r[row];
#pragma unroll
    for(int j = 0; j < 27; ++j) sum = sum + val[j];
    const float xn = sum * inv_diag32[row];
    x[row] = xn;
    if(z64) z64[row] = (double)xn;
    pro.add(row, xn);
}

// Residual at the injected rows (all of parity class 0: launch c is that colour).
template <bool kEven>
__global__ void __launch_bounds__(kBS32) k32_restrict(const ColorLaunch c, const StencilLevel L, int nc,
                                                      const int* __restrict__ inj_f, const int* __restrict__ inj_c,
                                                      const float* __restrict__ diag32, const float* __restrict__ rf,
                                                      const float* __restrict__ xf, float* __restrict__ rc)
{
    const int ic = blockIdx.x * kBS32 + threadIdx.x;
    const bool in = ic < nc;
    const BrickRow b = row_of(c, in ? inj_f[ic] : 0, in);
    if(!in) return;
    const int row = b.row;
    float val[27];
    gather<kOff, kEven>(L, c, b, xf, -0.0f, val);
    const float dterm = -diag32[row];
    const float xr = xf[row];
    float sum = rf[row];
    // ELL order: the diagonal term at slot dp (val[dp] is the no-op -0.0f)
#pragma unroll
    for(int j = 0; j < 27; ++j)
    {
        if(j == c.tb.dp) sum = fmaf(dterm, xr, sum);
        sum = sum + val[j];
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


// ------------------------------------------------ 4-row vector sweeps (even grids)
//
// When every colour brick's x extent is a multiple of 4 (and hence every
// colour's offset), a thread updates four consecutive rows of a brick line.
// Their neighbours in any slot are four consecutive floats of the neighbour's
// brick: one aligned float4 when the slot's column offset is a multiple of 4,
// two otherwise -- instead of four scalar gathers.  Each row keeps the ELL
// slot order and the -0.0f no-op for missing neighbours, so results are the
// same bits as the one-row kernels above.
// block: 8 x 16 threads, 32 rows x 16 lines of a brick plane; a warp spans 4
// lines, whose +-y neighbour rows it shares through L1.  At 320^3 against
// 8 x 32: FP32 sweep 36.1 -> 35.3 us, FP64 stencil V-cycle 2.54 -> 2.35 ms;
// 16 x 16, 32 x 8 and 4 x 32 were slower.
constexpr int kV4X = 8, kV4Y = 16;

inline bool vec4_ok(const StencilLevel& L)
{
    if(!L.even) return false;
    for(int v = 0; v < L.ncolors; ++v)
        if(L.bx[v] % 4 || L.offsets[v] % 4) return false;
    return true;
}

inline dim3 brick_grid4(const ColorLaunch& c)
{
    return dim3((unsigned)((c.bx + 4 * kV4X - 1) / (4 * kV4X)), (unsigned)((c.by + kV4Y - 1) / kV4Y), (unsigned)c.bz);
}

struct Rows4
{
    int row0;
    bool in;
    unsigned mask[4];
    bool fast;
};

__device__ __forceinline__ Rows4 rows4(const ColorLaunch& c, int kz)
{
    Rows4 b;
    const int kx0 = (blockIdx.x * kV4X + threadIdx.x) * 4;
    const int ky = blockIdx.y * kV4Y + threadIdx.y;
    b.in = kx0 < c.bx && ky < c.by && kz < c.bz;  // bx % 4 == 0: all four rows or none
    const int iy = 2 * ky + ((c.par >> 1) & 1), iz = 2 * kz + (c.par & 1);
    unsigned any = 0;
#pragma unroll
    for(int r = 0; r < 4; ++r)
    {
        const int ix = 2 * (kx0 + r) + ((c.par >> 2) & 1);
        b.mask[r] = b.in ? face_mask(c, ix, iy, iz) : 0u;
        any |= b.mask[r];
    }
    b.fast = __all_sync(0xffffffffu, any == 0u);
    b.row0 = c.off + (kz * c.by + ky) * c.bx + kx0;
    return b;
}

// Four consecutive values of a brick line: one float4, or two double2 for
// the FP64 V-cycle (32 bytes, 16-byte aligned halves).
template <typename T>
struct Quad;
template <>
struct Quad<float>
{
    static __device__ __forceinline__ void load(const float* p, float (&v)[4])
    {
        const float4 a = *reinterpret_cast<const float4*>(p);
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    }

    static __device__ __forceinline__ void store(float* p, const float (&v)[4])
    {
        *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
    }
};
template <>
struct Quad<double>
{
    static __device__ __forceinline__ void load(const double* p, double (&v)[4])
    {
        const double2 a = *reinterpret_cast<const double2*>(p);
        const double2 b = *reinterpret_cast<const double2*>(p + 2);
        v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
    }

    static __device__ __forceinline__ void store(double* p, const double (&v)[4])
    {
        *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]);
        *reinterpret_cast<double2*>(p + 2) = make_double2(v[2], v[3]);
    }
};

__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return fma(a, b, c); }

template <typename T>
__device__ __forceinline__ void ld4(const T* x, int i, int m, T (&v)[4])
{
    if(i >= 0 && i + 4 <= m) Quad<T>::load(x + i, v);
    else v[0] = v[1] = v[2] = v[3] = T(0);
}

// x[base .. base+3]; s = base & 3 is the same for every thread of the launch.
template <typename T>
__device__ __forceinline__ void load4(const T* x, int base, int m, int s, T (&v)[4])
{
    if(s == 0)
    {
        ld4(x, base, m, v);
        return;
    }
    const int lo = base - s;
    T a[4], b[4];
    ld4(x, lo, m, a);
    ld4(x, lo + 4, m, b);
    if(s == 1) { v[0] = a[1]; v[1] = a[2]; v[2] = a[3]; v[3] = b[0]; }
    else if(s == 2) { v[0] = a[2]; v[1] = a[3]; v[2] = b[0]; v[3] = b[1]; }
    else { v[0] = a[3]; v[1] = b[0]; v[2] = b[1]; v[3] = b[2]; }
}

// Slots whose loads are issued together before their in-order adds: 5 on
// large levels (keeps registers low, occupancy high; 320^3 mixed V-cycle 1.43
// ms with 3, 1.39 ms with 5, 1.42 ms with 9), all 27 (FP32) or 9 (FP64) on
// small levels (few threads: fewer round trips).
constexpr int kV4GroupLarge = 5, kV4GroupSmall = 27, kV4GroupSmall64 = 9;
constexpr int kV4SmallRows = 1 << 17;  // rows per colour below which a level counts as small

template <int kSel, int kGroup, typename T>
__device__ __forceinline__ void add_slots4(const ColorLaunch& c, const Rows4& b, const T* x, int m, T (&sum)[4])
{
#pragma unroll
    for(int g = 0; g < 27; g += kGroup)
    {
        T v[kGroup][4];
#pragma unroll
        for(int k = 0; k < kGroup; ++k)
        {
            const int j = g + k;
            if(j < 27 && selected<kSel>(j, c.tb.dp)) load4(x, b.row0 + c.tb.delta[j], m, c.tb.delta[j] & 3, v[k]);
        }
#pragma unroll
        for(int k = 0; k < kGroup; ++k)
        {
            const int j = g + k;
            if(j >= 27 || !selected<kSel>(j, c.tb.dp)) continue;
            if(b.fast)
            {
#pragma unroll
                for(int r = 0; r < 4; ++r) sum[r] = sum[r] + v[k][r];
            }
            else
            {
#pragma unroll
                for(int r = 0; r < 4; ++r) sum[r] = sum[r] + ((b.mask[r] & c.tb.bmask[j]) ? T(-0.0) : v[k][r]);
            }
        }
    }
}

// The same slot walk with the canonical colouring's compile-time tables (kCls
// = the colour's parity class): slot selection, the alignment of each
// neighbour quad and the face bits are constants, so no slot costs a runtime
// branch or select; the deltas still come from the launch's table.
template <int kS, typename T>
__device__ __forceinline__ void load4s(const T* x, int base, int m, T (&v)[4])
{
    if constexpr(kS == 0)
    {
        ld4(x, base, m, v);
    }
    else
    {
        T a[4], b[4];
        ld4(x, base - kS, m, a);
        ld4(x, base - kS + 4, m, b);
#pragma unroll
        for(int r = 0; r < 4; ++r) v[r] = (kS + r < 4) ? a[kS + r] : b[kS + r - 4];
    }
}

template <int kSel, int kCls>
__host__ __device__ constexpr bool kv_selected(int j)
{
    return kSel == kBefore ? j < KvTab<kCls>::s.dp : (kSel == kAfter ? j > KvTab<kCls>::s.dp : j != KvTab<kCls>::s.dp);
}

template <int kSel, int kCls, int J, typename T>
__device__ __forceinline__ void kv_load(const ColorLaunch& c, const Rows4& b, const T* x, int m, T (&v)[27][4])
{
    if constexpr(J < 27)
    {
        if constexpr(kv_selected<kSel, kCls>(J)) load4s<KvTab<kCls>::s.s[J]>(x, b.row0 + c.tb.delta[J], m, v[J]);
    }
}

template <int kSel, int kCls, int J, typename T>
__device__ __forceinline__ void kv_add(const Rows4& b, const T (&v)[27][4], T (&sum)[4])
{
    if constexpr(J < 27)
    {
        if constexpr(kv_selected<kSel, kCls>(J))
        {
            constexpr unsigned bj = KvTab<kCls>::s.bm[J];
            if(b.fast)
            {
#pragma unroll
                for(int r = 0; r < 4; ++r) sum[r] = sum[r] + v[J][r];
            }
            else
            {
#pragma unroll
                for(int r = 0; r < 4; ++r) sum[r] = sum[r] + ((b.mask[r] & bj) ? T(-0.0) : v[J][r]);
            }
        }
    }
}

template <int kSel, int kCls, int G0, typename T, int... K>
__device__ __forceinline__ void kv_group(const ColorLaunch& c, const Rows4& b, const T* x, int m, T (&v)[27][4],
                                         T (&sum)[4], std::integer_sequence<int, K...>)
{
    (kv_load<kSel, kCls, G0 + K>(c, b, x, m, v), ...);
    (kv_add<kSel, kCls, G0 + K>(b, v, sum), ...);
}

template <int kSel, int kGroup, int kCls, typename T, int... Gs>
__device__ __forceinline__ void kv_groups(const ColorLaunch& c, const Rows4& b, const T* x, int m, T (&sum)[4],
                                          std::integer_sequence<int, Gs...>)
{
    T v[27][4];
    (kv_group<kSel, kCls, Gs * kGroup>(c, b, x, m, v, sum, std::make_integer_sequence<int, kGroup>{}), ...);
}

// add_slots4 for kCls < 0, its compile-time form otherwise.
template <int kSel, int kGroup, int kCls, typename T>
__device__ __forceinline__ void add_slots(const ColorLaunch& c, const Rows4& b, const T* x, int m, T (&sum)[4])
{
    if constexpr(kCls < 0)
        add_slots4<kSel, kGroup>(c, b, x, m, sum);
    else
        kv_groups<kSel, kGroup, kCls>(c, b, x, m, sum, std::make_integer_sequence<int, (27 + kGroup - 1) / kGroup>{});
}

// Zero-guess forward sweep of one colour.  FP32 with kFromDouble: r comes in
// FP64 (the CG residual) and its float copy is stored for the later sweeps.
template <typename T, bool kFromDouble, int kG, int kCls = -1>
__global__ void __launch_bounds__(kV4X * kV4Y) kv_fwd0(const ColorLaunch c, const StencilLevel L,
                                                       const T* __restrict__ inv_diag, const double* __restrict__ r64,
                                                       T* __restrict__ r, T* x, Prolong<T> pro)
{
    pdl_begin();
    const Rows4 b = rows4(c, blockIdx.z);
    if(!b.in) return;
    T sum[4];
    if constexpr(kFromDouble)
    {
        double a[4];
        Quad<double>::load(r64 + b.row0, a);
#pragma unroll
        for(int q = 0; q < 4; ++q) sum[q] = (T)a[q];
        Quad<T>::store(r + b.row0, sum);
    }
    else
    {
        Quad<T>::load(r + b.row0, sum);
    }
    // FP32: 1/a_ii loaded before the slot sums, in flight while they run
    // (256^3 mixed V-cycle 0.743 -> 0.713 ms with the same in bwd0); FP64
    // keeps it after them (registers: its stencil V-cycle was 3 % slower)
    T inv[4], out[4];
    if constexpr(sizeof(T) == 4) Quad<T>::load(inv_diag + b.row0, inv);
    if(c.tb.dp > 0) add_slots<kBefore, kG, kCls>(c, b, x, L.m, sum);
    if constexpr(sizeof(T) != 4) Quad<T>::load(inv_diag + b.row0, inv);
#pragma unroll
    for(int q = 0; q < 4; ++q) out[q] = sum[q] * inv[q];
    Quad<T>::store(x + b.row0, out);
    pro.add4(b.row0, out);
}

template <typename T, int kG, int kCls = -1>
__global__ void __launch_bounds__(kV4X * kV4Y) kv_bwd0(const ColorLaunch c, const StencilLevel L,
                                                       const T* __restrict__ diag, const T* __restrict__ inv_diag, T* x,
                                                       Prolong<T> pro)
{
    pdl_begin();
    const Rows4 b = rows4(c, blockIdx.z);
    if(!b.in) return;
    T xv[4], dv[4], sum[4];
    Quad<T>::load(x + b.row0, xv);
    Quad<T>::load(diag + b.row0, dv);
#pragma unroll
    for(int q = 0; q < 4; ++q) sum[q] = mul_rn(xv[q], dv[q]);
    T inv[4], out[4];
    if constexpr(sizeof(T) == 4) Quad<T>::load(inv_diag + b.row0, inv);  // as in kv_fwd0
    add_slots<kAfter, kG, kCls>(c, b, x, L.m, sum);
    if constexpr(sizeof(T) != 4) Quad<T>::load(inv_diag + b.row0, inv);
#pragma unroll
    for(int q = 0; q < 4; ++q) out[q] = sum[q] * inv[q];
    Quad<T>::store(x + b.row0, out);
    pro.add4(b.row0, out);
}

// Full sweep of one colour; FP32 with z64: also the FP64 copy of the new x.
template <typename T, int kG, int kCls = -1>
__global__ void __launch_bounds__(kV4X * kV4Y) kv_sweep(const ColorLaunch c, const StencilLevel L,
                                                        const T* __restrict__ inv_diag, const T* __restrict__ r, T* x,
                                                        double* __restrict__ z64, Prolong<T> pro)
{
    pdl_begin();
    const Rows4 b = rows4(c, blockIdx.z);
    if(!b.in) return;
    T sum[4];
    Quad<T>::load(r + b.row0, sum);
    add_slots<kOff, kG, kCls>(c, b, x, L.m, sum);
    T inv[4], out[4];
    Quad<T>::load(inv_diag + b.row0, inv);
#pragma unroll
    for(int q = 0; q < 4; ++q) out[q] = sum[q] * inv[q];
    Quad<T>::store(x + b.row0, out);
    if constexpr(sizeof(T) == 4)
    {
        if(z64)
        {
            const double zo[4] = {(double)out[0], (double)out[1], (double)out[2], (double)out[3]};
            Quad<double>::store(z64 + b.row0, zo);
        }
    }
    pro.add4(b.row0, out);
}

// ------------------------------------------------------------ TMA-staged colour passes
// The colour passes of the FP32 (mixed) and FP64 (stencil) V-cycles on large
// levels with the canonical colouring -- the full sweep (kv_sweep), the
// zero-guess forward and backward passes (kv_fwd0, kv_bwd0) and the
// restriction (kv_restrict) -- with their neighbourhoods staged by TMA.  A CTA
// of 8 x TY x 2 threads takes a 32 x TY x 2 tile of its colour's brick (four
// x-adjacent rows per thread; TY = 16 for float, 8 for double).  One thread
// loads, with one tiled TMA box per colour the pass reads (every other colour
// for the sweep and the restriction, the earlier ones forward, the later ones
// backward), the part of that colour's brick the tile's neighbourhoods cover:
// the tile itself, grown by one brick column along x (4 elements: a box
// starts and spans in 16-byte units), one line along y and one plane along z
// on the axes where that colour's parity differs, on the side the launching
// colour's parity gives.  The boxes complete on one mbarrier (zero fill
// outside the grid); every thread then adds its rows' neighbours out of shared
// memory in the ELL slot order, -0 for the absent ones, with the per-row
// prologue and epilogue of the kernel it replaces -- the same bits.
constexpr int kTmaX = 32, kTmaZ = 2;
template <typename T>
constexpr int kTmaYOf = sizeof(T) == 4 ? 16 : 8;
template <typename T>
constexpr int kTmaThreadsOf = (kTmaX / 4) * kTmaYOf<T> * kTmaZ;
// resident CTAs per SM the register budget is sized for (shared memory allows
// 4-5 of the float tiles' up to 41 KB and the double tiles' up to 43 KB)
template <typename T>
constexpr int kTmaMinBlocksOf = sizeof(T) == 4 ? 4 : 5;

enum : int
{
    kTmaSweep = 0,    // x = (r + sum of all neighbours) / a_ii            (kv_sweep)
    kTmaFwd0 = 1,     // x = (r + sum of the earlier colours) / a_ii         (kv_fwd0)
    kTmaBwd0 = 2,     // x = (x a_ii + sum of the later colours) / a_ii      (kv_bwd0)
    kTmaRestrict = 3  // rc[inj_c] = r - A x on the parity-0 colour         (kv_restrict)
};

__host__ __device__ constexpr int tma_sel(int kind)
{
    return (kind == kTmaSweep || kind == kTmaRestrict) ? kOff : (kind == kTmaFwd0 ? kBefore : kAfter);
}

struct TmaTile
{
    int u;                   // colour of the staged brick
    int bx, by, bz;          // box (elements, lines, planes)
    int sx, sy, sz;          // box start = tile origin - (sx, sy, sz)
    int off;                 // shared-memory offset (elements; a multiple of 128 bytes)
};

struct TmaPlan
{
    int nt;                  // staged colours
    TmaTile t[7];            // in colour order
    int total;               // shared-memory elements
    unsigned bytes;          // bytes the boxes deliver
    int tile[27];            // per ELL slot: staged tile (-1: not read by this pass)
    int ax[27], ay[27], az[27];  // slot's position in its tile relative to the row's (4 tx, ty, tz)
};

__host__ __device__ constexpr int canon_parity(int colour)
{
    int p = 0;
    while(p < 7 && canon_colour(p) != colour) ++p;
    return p;
}

// floor(a / 2) for a >= -2
__host__ __device__ constexpr int half_floor(int a) { return (a + 2) / 2 - 1; }

// colour u is read by a pass of kind `kind` of colour v
__host__ __device__ constexpr bool tma_reads(int kind, int v, int u)
{
    return u != v && (tma_sel(kind) == kOff || (kind == kTmaFwd0 ? u < v : u > v));
}

__host__ __device__ constexpr bool tma_selected(int kind, int j, int dp)
{
    return tma_sel(kind) == kBefore ? j < dp : (tma_sel(kind) == kAfter ? j > dp : j != dp);
}

// ty: tile lines; esize: element bytes
__host__ __device__ constexpr TmaPlan tma_plan(int cls, int kind, int ty, int esize)
{
    TmaPlan P{};
    const int px = (cls >> 2) & 1, py = (cls >> 1) & 1, pz = cls & 1;
    const int v = canon_colour(cls);
    const int align = 128 / esize;
    int idx[8] = {-1, -1, -1, -1, -1, -1, -1, -1};
    int i = 0, off = 0;
    unsigned bytes = 0;
    for(int u = 0; u < 8; ++u)
    {
        if(!tma_reads(kind, v, u)) continue;
        const int d = cls ^ canon_parity(u);
        const int dx = (d >> 2) & 1, dy = (d >> 1) & 1, dz = d & 1;
        TmaTile t{};
        t.u = u;
        t.bx = kTmaX + 4 * dx;
        t.by = ty + dy;
        t.bz = kTmaZ + dz;
        t.sx = (dx && !px) ? 4 : 0;
        t.sy = (dy && !py) ? 1 : 0;
        t.sz = (dz && !pz) ? 1 : 0;
        t.off = off;
        off += (t.bx * t.by * t.bz + align - 1) / align * align;
        bytes += (unsigned)(t.bx * t.by * t.bz * esize);
        idx[u] = i;
        P.t[i++] = t;
    }
    P.nt = i;
    P.total = off;
    P.bytes = bytes;
    const KvSlots k = kv_slots(cls);
    for(int j = 0; j < 27; ++j)
    {
        P.tile[j] = -1;
        if(!tma_selected(kind, j, k.dp)) continue;
        const int u = canon_colour(cls ^ (((k.dx[j] & 1) << 2) | ((k.dy[j] & 1) << 1) | (k.dz[j] & 1)));
        const int ti = idx[u];
        P.tile[j] = ti;
        if(ti < 0) continue;
        P.ax[j] = half_floor(px + k.dx[j]) + P.t[ti].sx;
        P.ay[j] = half_floor(py + k.dy[j]) + P.t[ti].sy;
        P.az[j] = half_floor(pz + k.dz[j]) + P.t[ti].sz;
    }
    return P;
}

template <typename T, int kCls, int kKind>
struct TmaTab
{
    static constexpr TmaPlan p = tma_plan(kCls, kKind, kTmaYOf<T>, (int)sizeof(T));
};

// Every slot a pass reads lies inside its staged tile, every slot of the
// pass's selection has a tile, and the tiles fit the default dynamic shared
// memory (checked at compile time for every class, kind and element size,
// with the largest thread position).
__host__ __device__ constexpr bool tma_plan_ok(int cls, int kind, int ty, int esize)
{
    const TmaPlan P = tma_plan(cls, kind, ty, esize);
    const KvSlots k = kv_slots(cls);
    for(int j = 0; j < 27; ++j)
    {
        if(tma_selected(kind, j, k.dp) != (P.tile[j] >= 0)) return false;
        if(P.tile[j] < 0) continue;
        const TmaTile& t = P.t[P.tile[j]];
        const int lo = P.ax[j] - (P.ax[j] & 3), hi = 4 * (kTmaX / 4 - 1) + lo + ((P.ax[j] & 3) ? 8 : 4);
        if(lo < 0 || hi > t.bx || P.ay[j] < 0 || P.ay[j] + ty > t.by || P.az[j] < 0 || P.az[j] + kTmaZ > t.bz)
            return false;
    }
    return P.total * esize + 128 <= 48 * 1024;
}

__host__ __device__ constexpr bool tma_plans_ok()
{
    for(int cls = 0; cls < 8; ++cls)
        for(int kind = 0; kind < 4; ++kind)
            if(!tma_plan_ok(cls, kind, kTmaYOf<float>, 4) || !tma_plan_ok(cls, kind, kTmaYOf<double>, 8)) return false;
    return true;
}
static_assert(tma_plans_ok(), "TMA colour-pass tiles");

struct NbMaps
{
    CUtensorMap m[7];        // the staged colours' bricks of x, in colour order
};

// Four consecutive elements starting s (0..3) past a 4-aligned position of
// shared memory: float4 loads for float, double2 loads for double.
template <int kS>
__device__ __forceinline__ void sm_quad(const float* q, float (&v)[4])
{
    const float4 a = *reinterpret_cast<const float4*>(q);
    if constexpr(kS == 0)
    {
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    }
    else
    {
        const float4 e = *reinterpret_cast<const float4*>(q + 4);
        const float w[8] = {a.x, a.y, a.z, a.w, e.x, e.y, e.z, e.w};
#pragma unroll
        for(int r = 0; r < 4; ++r) v[r] = w[kS + r];
    }
}

template <int kS>
__device__ __forceinline__ void sm_quad(const double* q, double (&v)[4])
{
    constexpr int p0 = kS / 2, p1 = (kS + 3) / 2;  // double2 pairs covering [kS, kS + 4)
    double w[8];
#pragma unroll
    for(int p = p0; p <= p1; ++p)
    {
        const double2 a = *reinterpret_cast<const double2*>(q + 2 * p);
        w[2 * p] = a.x;
        w[2 * p + 1] = a.y;
    }
#pragma unroll
    for(int r = 0; r < 4; ++r) v[r] = w[kS + r];
}

// Slot J of the rows' ELL walk; the restriction's diagonal slot is
// fma(-a_ii, x_i, sum) with the row's own xo and dg.
template <typename T, int kCls, int kKind, int J>
__device__ __forceinline__ void tma_slot(const T* sm, int tx, int ty, int tz, const Rows4& b, T (&sum)[4],
                                         const T (&xo)[4], const T (&dg)[4])
{
    using Tab = TmaTab<T, kCls, kKind>;
    constexpr int ti = Tab::p.tile[J];
    if constexpr(kKind == kTmaRestrict && J == KvTab<kCls>::s.dp)
    {
#pragma unroll
        for(int r = 0; r < 4; ++r) sum[r] = fma_rn(-dg[r], xo[r], sum[r]);
    }
    else if constexpr(ti >= 0)
    {
        constexpr int bx = Tab::p.t[ti].bx, by = Tab::p.t[ti].by, off = Tab::p.t[ti].off;
        constexpr int ax = Tab::p.ax[J], ay = Tab::p.ay[J], az = Tab::p.az[J];
        constexpr int s = ax & 3;
        T v[4];
        sm_quad<s>(sm + off + ((tz + az) * by + ty + ay) * bx + 4 * tx + (ax - s), v);
        constexpr unsigned bj = KvTab<kCls>::s.bm[J];
        if(b.fast)
        {
#pragma unroll
            for(int r = 0; r < 4; ++r) sum[r] = sum[r] + v[r];
        }
        else
        {
#pragma unroll
            for(int r = 0; r < 4; ++r) sum[r] = sum[r] + ((b.mask[r] & bj) ? T(-0.0) : v[r]);
        }
    }
}

template <typename T, int kCls, int kKind, int... J>
__device__ __forceinline__ void tma_slots(const T* sm, int tx, int ty, int tz, const Rows4& b, T (&sum)[4],
                                          const T (&xo)[4], const T (&dg)[4], std::integer_sequence<int, J...>)
{
    (tma_slot<T, kCls, kKind, J>(sm, tx, ty, tz, b, sum, xo, dg), ...);
}

// One colour pass of kind kKind.  Sweep: r -> x (and, FP32, z64 when given:
// the FP64 copy); forward zero-guess: r -> x, or for FP32 with kFromDouble
// r64 -> x storing the float copy of r64 in r; backward zero-guess: x, diag ->
// x; restriction: r, x, diag -> rc[inj_c] (x is only read).  status (may be
// null) gets 3 when the copies did not arrive in time; the tile's outputs are
// then set to NaN, so the solve ends as non-finite.
template <typename T, int kCls, int kKind, bool kFromDouble>
__global__ void __launch_bounds__(kTmaThreadsOf<T>, kTmaMinBlocksOf<T>)
    kv_pass_tma(const __grid_constant__ NbMaps nb, const ColorLaunch c, const T* __restrict__ inv_diag,
                const T* __restrict__ diag, const double* __restrict__ r64, T* __restrict__ r, T* __restrict__ x,
                double* __restrict__ z64, const int* __restrict__ inj_c, T* __restrict__ rc, int* status)
{
    using Tab = TmaTab<T, kCls, kKind>;
    extern __shared__ unsigned char sm_raw[];
    __shared__ uint64_t mbar;
    T* sm = reinterpret_cast<T*>(sm_raw + ((128u - (tma::smem_u32(sm_raw) & 127u)) & 127u));
    const int tx = threadIdx.x, ty = threadIdx.y, tz = threadIdx.z;
    const int x0 = blockIdx.x * kTmaX, y0 = blockIdx.y * kTmaYOf<T>, z0 = blockIdx.z * kTmaZ;
    pdl_begin();
    const bool leader = tx == 0 && ty == 0 && tz == 0;
    if constexpr(Tab::p.nt > 0)
    {
        if(leader)
        {
            constexpr TmaPlan P = Tab::p;
            tma::mbar_init(&mbar, 1);
            tma::mbar_arrive_expect_tx(&mbar, P.bytes);
#pragma unroll
            for(int i = 0; i < P.nt; ++i)
                tma::load_3d(sm + P.t[i].off, &nb.m[i], x0 - P.t[i].sx, y0 - P.t[i].sy, z0 - P.t[i].sz, &mbar);
        }
    }
    // the rows' own data and face bits while the boxes are in flight
    const int kx0 = x0 + 4 * tx, ky = y0 + ty, kz = z0 + tz;
    Rows4 b;
    b.in = kx0 < c.bx && ky < c.by && kz < c.bz;  // bx % 4 == 0: all four rows or none
    b.row0 = c.off + (kz * c.by + ky) * c.bx + kx0;
    {
        const int iy = 2 * ky + ((c.par >> 1) & 1), iz = 2 * kz + (c.par & 1);
        unsigned any = 0;
#pragma unroll
        for(int q = 0; q < 4; ++q)
        {
            b.mask[q] = b.in ? face_mask(c, 2 * (kx0 + q) + ((c.par >> 2) & 1), iy, iz) : 0u;
            any |= b.mask[q];
        }
        b.fast = __all_sync(0xffffffffu, any == 0u);
    }
    T sum[4], inv[4], xo[4] = {}, dg[4] = {};
    if(b.in)
    {
        if constexpr(kKind == kTmaRestrict)
        {
            Quad<T>::load(r + b.row0, sum);
            Quad<T>::load(x + b.row0, xo);
            Quad<T>::load(diag + b.row0, dg);
        }
        else if constexpr(kKind == kTmaBwd0)
        {
            T xv[4], dv[4];
            Quad<T>::load(x + b.row0, xv);
            Quad<T>::load(diag + b.row0, dv);
#pragma unroll
            for(int q = 0; q < 4; ++q) sum[q] = mul_rn(xv[q], dv[q]);
        }
        else if constexpr(kFromDouble)
        {
            double a[4];
            Quad<double>::load(r64 + b.row0, a);
#pragma unroll
            for(int q = 0; q < 4; ++q) sum[q] = (T)a[q];
            Quad<T>::store(r + b.row0, sum);
        }
        else
        {
            Quad<T>::load(r + b.row0, sum);
        }
        if constexpr(kKind != kTmaRestrict) Quad<T>::load(inv_diag + b.row0, inv);
    }
    if constexpr(Tab::p.nt > 0)
    {
        __syncthreads();  // the barrier is initialised before anyone waits on it
        if(!tma::mbar_wait(&mbar, 0))
        {
            if(leader && status) atomicExch(status, 3);
            if(b.in)
            {
                const T q = (T)__int_as_float(0x7fc00000);
                if constexpr(kKind == kTmaRestrict)
                {
                    const int4 ic = *reinterpret_cast<const int4*>(inj_c + (b.row0 - c.off));
                    rc[ic.x] = q;
                    rc[ic.y] = q;
                    rc[ic.z] = q;
                    rc[ic.w] = q;
                }
                else
                {
                    const T nan[4] = {q, q, q, q};
                    Quad<T>::store(x + b.row0, nan);
                }
            }
            tma::mbar_wait(&mbar, 0);  // the copies still in flight land before the CTA leaves
            return;
        }
    }
    if(!b.in) return;
    tma_slots<T, kCls, kKind>(sm, tx, ty, tz, b, sum, xo, dg, std::make_integer_sequence<int, 27>{});
    if constexpr(kKind == kTmaRestrict)
    {
        const int4 ic = *reinterpret_cast<const int4*>(inj_c + (b.row0 - c.off));
        rc[ic.x] = sum[0];
        rc[ic.y] = sum[1];
        rc[ic.z] = sum[2];
        rc[ic.w] = sum[3];
        return;
    }
    T out[4];
#pragma unroll
    for(int q = 0; q < 4; ++q) out[q] = sum[q] * inv[q];
    Quad<T>::store(x + b.row0, out);
    if constexpr(kKind == kTmaSweep && sizeof(T) == 4)
    {
        if(z64)
        {
            const double zo[4] = {(double)out[0], (double)out[1], (double)out[2], (double)out[3]};
            Quad<double>::store(z64 + b.row0, zo);
        }
    }
}

// Restriction on the 4-row layout: the injected fine points are the parity-0
// colour's brick, whose brick-local index is the coarse natural index, so
// rc[inj_c[row - off]] = (rf - A xf)[row] with the same per-row arithmetic as
// the ELL restriction (slot order, fma(-a_ii, x_i, .) at the diagonal slot).
template <typename T, int kG, int kCls = -1>
__global__ void __launch_bounds__(kV4X * kV4Y) kv_restrict(const ColorLaunch c, const StencilLevel L,
                                                           const int* __restrict__ inj_c, const T* __restrict__ diag,
                                                           const T* __restrict__ rf, const T* __restrict__ xf,
                                                           T* __restrict__ rc)
{
    pdl_begin();
    const Rows4 b = rows4(c, blockIdx.z);
    if(!b.in) return;
    T sum[4];
    Quad<T>::load(rf + b.row0, sum);
    // slots before the diagonal, fma(-a_ii, x_i, .) at it, slots after it
    add_slots<kBefore, kG, kCls>(c, b, xf, L.m, sum);
    T xv[4], dv[4];
    Quad<T>::load(xf + b.row0, xv);
    Quad<T>::load(diag + b.row0, dv);
#pragma unroll
    for(int q = 0; q < 4; ++q) sum[q] = fma_rn(-dv[q], xv[q], sum[q]);
    add_slots<kAfter, kG, kCls>(c, b, xf, L.m, sum);
    const int4 ic = *reinterpret_cast<const int4*>(inj_c + (b.row0 - c.off));
    rc[ic.x] = sum[0];
    rc[ic.y] = sum[1];
    rc[ic.z] = sum[2];
    rc[ic.w] = sum[3];
}

// xf[row] += xc[inj_c[row - off]] over the parity-0 colour's brick.
template <typename T>
__global__ void __launch_bounds__(kV4X * kV4Y) kv_prolong(const ColorLaunch c, const int* __restrict__ inj_c,
                                                          const T* __restrict__ xc, T* __restrict__ xf)
{
    pdl_begin();
    const int kx0 = (blockIdx.x * kV4X + threadIdx.x) * 4;
    const int ky = blockIdx.y * kV4Y + threadIdx.y;
    const int kz = blockIdx.z;
    if(!(kx0 < c.bx && ky < c.by && kz < c.bz)) return;
    const int row0 = c.off + (kz * c.by + ky) * c.bx + kx0;
    const int4 ic = *reinterpret_cast<const int4*>(inj_c + (row0 - c.off));
    T x[4];
    Quad<T>::load(xf + row0, x);
    x[0] += xc[ic.x];
    x[1] += xc[ic.y];
    x[2] += xc[ic.z];
    x[3] += xc[ic.w];
    Quad<T>::store(xf + row0, x);
}

// ----------------------------------------------------- FP64 stencil SpMV
//
// One launch for all colours: a block owns a natural-order tile of
// 32 x 8 x 4 points, stages p on the tile and its one-point halo (34 x 10 x 6
// doubles, 16 KB) in shared memory with coalesced loads from the colour
// bricks, and computes every row of the tile from there.  Each warp holds
// rows of one parity class (= one colour), so the row's ELL slot order --
// that colour's order, read from a per-block table -- is warp-uniform, and
// the sum is formed exactly like the ELL SpMV: sum = fma(a_ii, x_i, sum) at
// the diagonal slot, sum - x_col (= fma(-1, x_col, sum)) at the others, absent
// neighbours (+0.0 in the halo) leave it unchanged.  Bitwise equal to
// k_spmv on the same matrix.

constexpr int kT64X = 32, kT64Y = 8, kT64Z = 4;
constexpr int kH64X = kT64X + 2, kH64Y = kT64Y + 2, kH64Z = kT64Z + 2;
constexpr int kT64Threads = kT64X * kT64Y * kT64Z;  // 1024: 8 parity classes x 128 rows
constexpr int kH64Points = kH64X * kH64Y * kH64Z;   // 2040

__device__ __forceinline__ int natural_to_row(const StencilLevel& L, int z, int y, int x)
{
    const int v = L.color_of_par[((x & 1) << 2) | ((y & 1) << 1) | (z & 1)];
    return L.offsets[v] + ((z >> 1) * L.by[v] + (y >> 1)) * L.bx[v] + (x >> 1);
}

inline dim3 tile64_grid(const StencilLevel& L)
{
    return dim3((unsigned)((L.nx + kT64X - 1) / kT64X), (unsigned)((L.ny + kT64Y - 1) / kT64Y),
                (unsigned)((L.nz + kT64Z - 1) / kT64Z));
}

constexpr int kT64Loads = (kH64Points + kT64Threads - 1) / kT64Threads;  // halo values per thread: 2
// Shared-memory layout of the staged tile: split by parity class into eight
// sub-bricks of (34/2) x (10/2) x (6/2) points, so the rows of one class that a
// warp holds (every other x) read consecutive doubles -- no bank conflicts.
constexpr int kSbX = kH64X / 2, kSbY = kH64Y / 2, kSbZ = kH64Z / 2, kSbN = kSbX * kSbY * kSbZ;
static_assert(kSbN * 8 == kH64Points, "sub-bricks cover the halo'd tile");

// Halo coordinates (h = natural - tile origin + 1; origins are even) -> slot.
__host__ __device__ constexpr int sub_index(int hx, int hy, int hz)
{
    const int par = (((hx + 1) & 1) << 2) | (((hy + 1) & 1) << 1) | ((hz + 1) & 1);
    return par * kSbN + ((hz >> 1) * kSbY + (hy >> 1)) * kSbX + (hx >> 1);
}

struct Tile64
{
    int x0, y0, z0;
};

__device__ __forceinline__ Tile64 tile64_of(const StencilLevel& L, int tile)
{
    const int tx = (L.nx + kT64X - 1) / kT64X, ty = (L.ny + kT64Y - 1) / kT64Y;
    const int bz = tile / (tx * ty), rem = tile - bz * tx * ty;
    const int by = rem / tx, bx = rem - by * tx;
    return Tile64{bx * kT64X, by * kT64Y, bz * kT64Z};
}

// This thread's halo values and its row's diagonal for tile t (loads only).
__device__ __forceinline__ void tile64_load(const StencilLevel& L, const Tile64& t, int tid, int cls_x, int cls_y,
                                            int cls_z, const double* __restrict__ p,
                                            const double* __restrict__ diag, double (&hv)[kT64Loads], double& dv)
{
#pragma unroll
    for(int k = 0; k < kT64Loads; ++k)
    {
        const int e = tid + k * kT64Threads;
        hv[k] = 0.0;
        if(e < kH64Points)
        {
            const int hx = e % kH64X, hy = (e / kH64X) % kH64Y, hz = e / (kH64X * kH64Y);
            const int x = t.x0 + hx - 1, y = t.y0 + hy - 1, z = t.z0 + hz - 1;
            if(x >= 0 && x < L.nx && y >= 0 && y < L.ny && z >= 0 && z < L.nz) hv[k] = p[natural_to_row(L, z, y, x)];
        }
    }
    const int x = t.x0 + cls_x, y = t.y0 + cls_y, z = t.z0 + cls_z;
    dv = (x < L.nx && y < L.ny && z < L.nz) ? diag[natural_to_row(L, z, y, x)] : 0.0;
}

// Persistent: a block walks tiles blockIdx.x, +gridDim.x, ...; the next
// tile's loads are issued before the current tile is computed.
template <bool kPap>
__global__ void __launch_bounds__(kT64Threads, 2) k64_spmv_tile(const StencilLevel L, const double* __restrict__ diag,
                                                                const double* __restrict__ p,
                                                                double* __restrict__ Ap, CGState* st,
                                                                double* partial, unsigned int* ticket)
{
    __shared__ double s_p[kH64Points];
    __shared__ short s_delta[8][27];
    __shared__ int s_dp[8];
    __shared__ double red[32];
    __shared__ bool last;
    const int tid = threadIdx.x;
    const int ntiles = ((L.nx + kT64X - 1) / kT64X) * ((L.ny + kT64Y - 1) / kT64Y) * ((L.nz + kT64Z - 1) / kT64Z);

    // slot order of each parity class (its colour's ELL order) as offsets
    // between sub-brick slots (the same for every point of the class)
    if(tid < 8 * 27)
    {
        const int cls = tid / 27, j = tid - cls * 27;
        const unsigned e = L.tab[L.color_of_par[cls]].nb[j];
        const int dx = (int)(e & 3) - 1, dy = (int)((e >> 2) & 3) - 1, dz = (int)((e >> 4) & 3) - 1;
        const int hx = ((cls >> 2) & 1) + 1, hy = ((cls >> 1) & 1) + 1, hz = (cls & 1) + 1;
        s_delta[cls][j] = (short)(sub_index(hx + dx, hy + dy, hz + dz) - sub_index(hx, hy, hz));
        if(j == 0) s_dp[cls] = L.tab[L.color_of_par[cls]].dp;
    }
    // thread -> (parity class, point of that class in the tile)
    const int cls = tid >> 7, i = tid & 127;
    const int lx = 2 * (i & 15) + ((cls >> 2) & 1);
    const int ly = 2 * ((i >> 4) & 3) + ((cls >> 1) & 1);
    const int lz = 2 * (i >> 6) + (cls & 1);
    const int c = sub_index(lx + 1, ly + 1, lz + 1);

    double hv[kT64Loads], dv = 0.0;
    int tile = blockIdx.x;
    if(tile < ntiles) tile64_load(L, tile64_of(L, tile), tid, lx, ly, lz, p, diag, hv, dv);
    double s = 0.0;
    for(; tile < ntiles; tile += gridDim.x)
    {
        const Tile64 t = tile64_of(L, tile);
        __syncthreads();  // previous tile's reads of s_p are done
#pragma unroll
        for(int k = 0; k < kT64Loads; ++k)
        {
            const int e = tid + k * kT64Threads;
            if(e < kH64Points) s_p[sub_index(e % kH64X, (e / kH64X) % kH64Y, e / (kH64X * kH64Y))] = hv[k];
        }
        const double d = dv;
        __syncthreads();
        if(tile + (int)gridDim.x < ntiles)
            tile64_load(L, tile64_of(L, tile + gridDim.x), tid, lx, ly, lz, p, diag, hv, dv);
        const int x = t.x0 + lx, y = t.y0 + ly, z = t.z0 + lz;
        if(x < L.nx && y < L.ny && z < L.nz)
        {
            const double xr = s_p[c];
            const int dp = s_dp[cls];
            double sum = 0.0;
#pragma unroll
            for(int j = 0; j < 27; ++j)
            {
                if(j == dp) sum = fma(d, xr, sum);
                else sum = sum - s_p[c + s_delta[cls][j]];
            }
            Ap[natural_to_row(L, z, y, x)] = sum;
            if(kPap) s = fma(sum, xr, s);
        }
    }
    if(!kPap) return;
    s = block_sum(s, red);
    if(tid == 0)
    {
        partial[blockIdx.x] = s;
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if(!last) return;
    __threadfence();
    double acc = 0.0;
    for(int k = tid; k < (int)gridDim.x; k += kT64Threads) acc += __ldcg(&partial[k]);
    acc = block_sum(acc, red);
    if(tid == 0)
    {
        *ticket = 0;
        st->pAp = acc;
        st->alpha = st->rtz / acc;
    }
}


// ---- the colouring the reference's JPL rounds produce (parity class ->
// colour 7,2,3,6,5,4,1,0 on every grid it was run on): the plane march below
// compiles the slot order of each class in; levels with any other colour map
// take k64_spmv_tile.
constexpr int kCanonColor[8] = {7, 2, 3, 6, 5, 4, 1, 0};
static_assert(((0x01456327u >> 0) & 15u) == 7 && ((0x01456327u >> 28) & 15u) == 0, "packed canonical colours");

// ---- plane march (canonical colouring): a block owns a 64 x 4 column of the
// grid and walks a chunk of z planes with a ring of four staged planes
// (66 x 6 doubles each, halo included, x split by parity so a warp's reads
// are consecutive).  Per step it stores the prefetched plane z+2, issues the
// loads of plane z+3, computes the rows of plane z with the compile-time slot
// order, and synchronises once.  Each warp holds one x parity and one y row,
// so the parity class (= colour) of its rows is warp-uniform.
constexpr int kMX = 64, kMY = 4, kMZ = 16;                 // column, z chunk
constexpr int kMThreads = (kMX / 2) * 2 * kMY;             // 256: (32 lanes) x (2 x-parities) x (4 rows)
constexpr int kPX = kMX + 2, kPY = kMY + 2;                // staged plane 66 x 6
constexpr int kPXh = kPX / 2;                              // 33 per x parity
constexpr int kPlane = kPX * kPY;                          // 396
constexpr int kMLoads = (kPlane + kMThreads - 1) / kMThreads;  // 2 per thread

// Plane slot of halo coordinates (hx = x - x0 + 1, hy = y - y0 + 1; x0, y0 even).
__host__ __device__ constexpr int plane_slot(int hx, int hy) { return (hy * 2 + ((hx + 1) & 1)) * kPXh + (hx >> 1); }

struct MarchSlots
{
    int off[27];  // plane-slot offset of slot j (same plane index layout for every dz)
    int dz[27];   // plane of slot j relative to the row's plane
    int dp;
};

__host__ __device__ constexpr MarchSlots march_slots(int cls)
{
    MarchSlots r{};
    int key[27] = {}, dxs[27] = {}, dys[27] = {}, dzs[27] = {};
    int k = 0;
    for(int dz = -1; dz <= 1; ++dz)
        for(int dy = -1; dy <= 1; ++dy)
            for(int dx = -1; dx <= 1; ++dx)
            {
                const int col = kCanonColor[cls ^ (((dx & 1) << 2) | ((dy & 1) << 1) | (dz & 1))];
                key[k] = ((col * 3 + (dz + 1)) * 3 + (dy + 1)) * 3 + (dx + 1);
                dxs[k] = dx;
                dys[k] = dy;
                dzs[k] = dz;
                ++k;
            }
    for(int a = 1; a < 27; ++a)
        for(int b = a; b > 0 && key[b - 1] > key[b]; --b)
        {
            int t = key[b]; key[b] = key[b - 1]; key[b - 1] = t;
            t = dxs[b]; dxs[b] = dxs[b - 1]; dxs[b - 1] = t;
            t = dys[b]; dys[b] = dys[b - 1]; dys[b - 1] = t;
            t = dzs[b]; dzs[b] = dzs[b - 1]; dzs[b - 1] = t;
        }
    // any point of the class: x parity (cls>>2)&1, y parity (cls>>1)&1 (x0, y0 even)
    const int hx = ((cls >> 2) & 1) + 1, hy = ((cls >> 1) & 1) + 1;
    for(int j = 0; j < 27; ++j)
    {
        r.off[j] = plane_slot(hx + dxs[j], hy + dys[j]) - plane_slot(hx, hy);
        r.dz[j] = dzs[j];
        if(dxs[j] == 0 && dys[j] == 0 && dzs[j] == 0) r.dp = j;
    }
    return r;
}

template <int kCls>
struct MarchTab
{
    static constexpr MarchSlots s = march_slots(kCls);
};

template <int kCls, int J>
__device__ __forceinline__ void march_step(double& sum, const double* pm, const double* p0, const double* pp, double d,
                                           double xr)
{
    constexpr int off = MarchTab<kCls>::s.off[J];
    constexpr int dz = MarchTab<kCls>::s.dz[J];
    if constexpr(J == MarchTab<kCls>::s.dp) sum = fma(d, xr, sum);
    else sum = sum - (dz < 0 ? pm : (dz == 0 ? p0 : pp))[off];
}

template <int kCls, int... J>
__device__ __forceinline__ double march_row(const double* pm, const double* p0, const double* pp, double d, double xr,
                                            std::integer_sequence<int, J...>)
{
    double sum = 0.0;
    (march_step<kCls, J>(sum, pm, p0, pp, d, xr), ...);  // slots in ELL order, left to right
    return sum;
}

// Colour-permuted row of natural (x, y, z) for the canonical colouring, as
// base + (z >> 1) * stride with base and stride fixed per (x, y, z parity).
struct CanonColumn
{
    int base[2], stride[2];  // indexed by z parity
};

__device__ __forceinline__ CanonColumn canon_column(const StencilLevel& L, int x, int y)
{
    CanonColumn c;
#pragma unroll
    for(int q = 0; q < 2; ++q)
    {
        // kCanonColor packed in nibbles (parity class 0 in the lowest)
        const int v = (int)((0x01456327u >> (4 * (((x & 1) << 2) | ((y & 1) << 1) | q))) & 15u);
        c.base[q] = L.offsets[v] + (y >> 1) * L.bx[v] + (x >> 1);
        c.stride[q] = L.by[v] * L.bx[v];
    }
    return c;
}

template <int kQ>
__device__ __forceinline__ int canon_row(const CanonColumn& c, int z)
{
    return c.base[kQ] + (z >> 1) * c.stride[kQ];
}

template <bool kPap>
__global__ void __launch_bounds__(kMThreads) k64_spmv_march(const StencilLevel L, const double* __restrict__ diag,
                                                            const double* __restrict__ p, double* __restrict__ Ap,
                                                            CGState* st, double* partial, unsigned int* ticket)
{
    __shared__ double ring[4][kPlane];
    __shared__ double red[32];
    __shared__ bool last;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int x0 = blockIdx.x * kMX, y0 = blockIdx.y * kMY, zb = blockIdx.z * kMZ;  // zb even
    const int ze = zb + kMZ < L.nz ? zb + kMZ : L.nz;

    // this thread's staged positions (fixed for every plane), whether they
    // exist, and their rows as functions of z
    int slot[kMLoads];
    bool inxy[kMLoads];
    CanonColumn col[kMLoads];
#pragma unroll
    for(int k = 0; k < kMLoads; ++k)
    {
        const int e = tid + k * kMThreads;
        const int hx = e % kPX, hy = e / kPX;
        const int x = x0 + hx - 1, y = y0 + hy - 1;
        slot[k] = e < kPlane ? plane_slot(hx, hy) : -1;
        inxy[k] = e < kPlane && x >= 0 && x < L.nx && y >= 0 && y < L.ny;
        col[k] = canon_column(L, inxy[k] ? x : 0, inxy[k] ? y : 0);
    }
    auto load_plane = [&](int z, auto zq, double (&v)[kMLoads]) {
        constexpr int q = decltype(zq)::value;  // z & 1
#pragma unroll
        for(int k = 0; k < kMLoads; ++k)
        {
            v[k] = 0.0;
            if(inxy[k] && z >= 0 && z < L.nz) v[k] = p[canon_row<q>(col[k], z)];
        }
    };
    auto store_plane = [&](int z, const double (&v)[kMLoads]) {
        double* dst = ring[(z + 4) & 3];
#pragma unroll
        for(int k = 0; k < kMLoads; ++k)
            if(slot[k] >= 0) dst[slot[k]] = v[k];
    };
    using Q0 = std::integral_constant<int, 0>;
    using Q1 = std::integral_constant<int, 1>;

    // own column: warp -> (x parity, row); lane -> x
    const int px = warp & 1, ly = warp >> 1;
    const int lx = 2 * lane + px;
    const int x = x0 + lx, y = y0 + ly;
    const bool mine = x < L.nx && y < L.ny;
    const int c = plane_slot(lx + 1, ly + 1);
    const CanonColumn own = canon_column(L, mine ? x : 0, mine ? y : 0);

    double hv[kMLoads];
    load_plane(zb - 1, Q1{}, hv);
    store_plane(zb - 1, hv);
    load_plane(zb, Q0{}, hv);
    store_plane(zb, hv);
    load_plane(zb + 1, Q1{}, hv);
    store_plane(zb + 1, hv);
    load_plane(zb + 2, Q0{}, hv);
    double dv = (mine && zb < ze) ? diag[canon_row<0>(own, zb)] : 0.0;
    __syncthreads();
    double s = 0.0;
    // one plane: z & 1 == q
    auto step = [&](int z, auto zq) {
        constexpr int q = decltype(zq)::value;
        using QN = std::integral_constant<int, q ^ 1>;
        store_plane(z + 2, hv);  // ring slot of plane z-2: free since the last step
        const double d = dv;
        if(z + 1 < ze)
        {
            load_plane(z + 3, QN{}, hv);
            dv = mine ? diag[canon_row<q ^ 1>(own, z + 1)] : 0.0;
        }
        if(mine)
        {
            const double* pm = ring[(z + 3) & 3] + c;
            const double* p0 = ring[(z + 4) & 3] + c;
            const double* pp = ring[(z + 5) & 3] + c;
            const double xr = *p0;
            double sum;
            using Seq = std::make_integer_sequence<int, 27>;
            switch((px << 1) | (ly & 1))
            {
                case 0: sum = march_row<0 | q>(pm, p0, pp, d, xr, Seq{}); break;
                case 1: sum = march_row<2 | q>(pm, p0, pp, d, xr, Seq{}); break;
                case 2: sum = march_row<4 | q>(pm, p0, pp, d, xr, Seq{}); break;
                default: sum = march_row<6 | q>(pm, p0, pp, d, xr, Seq{}); break;
            }
            Ap[canon_row<q>(own, z)] = sum;
            if(kPap) s = fma(sum, xr, s);
        }
        __syncthreads();  // plane z+2 stored, plane z-1 no longer read
    };
    for(int z = zb; z < ze; z += 2)
    {
        step(z, Q0{});
        if(z + 1 < ze) step(z + 1, Q1{});
    }
    if(!kPap) return;
    s = block_sum(s, red);
    const unsigned nblocks = gridDim.x * gridDim.y * gridDim.z;
    const unsigned bid = (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
    if(tid == 0)
    {
        partial[bid] = s;
        __threadfence();
        last = atomicAdd(ticket, 1u) == nblocks - 1;
    }
    __syncthreads();
    if(!last) return;
    __threadfence();
    double acc = 0.0;
    for(int k = tid; k < (int)nblocks; k += kMThreads) acc += __ldcg(&partial[k]);
    acc = block_sum(acc, red);
    if(tid == 0)
    {
        *ticket = 0;
        st->pAp = acc;
        st->alpha = st->rtz / acc;
    }
}

inline dim3 march_grid(const StencilLevel& L)
{
    return dim3((unsigned)((L.nx + kMX - 1) / kMX), (unsigned)((L.ny + kMY - 1) / kMY),
                (unsigned)((L.nz + kMZ - 1) / kMZ));
}

// ---- separable product (the mixed path's outer operator, canonical
// colouring).  The outer CG of the mixed path needs A p in FP64, not the ELL
// kernel's summation order, so the 27 neighbours are summed as a separable
// box: per staged plane the x sums sx = x[-1] + x[0] + x[+1] of the tile's
// rows and their y halo go to shared memory, the y sums sxy of those give one
// value per row, and a ring of three sxy values in registers gives the box
// sum S over z.  y = a_ii x - (S - x): about 7 shared-memory reads per row
// instead of the 27 of the ELL-ordered march, which is bound by shared-memory
// bandwidth (27 x 8 B per row).  The result equals the ELL product to FP64
// rounding (a different association of the same 27 terms).  A block owns a
// 64 x 4 column of the grid and kSZ planes; two barriers per plane.
constexpr int kSZ = 32;                                        // z planes per block
constexpr int kSXh = kMX / 2;                                  // sx row: 64 points, x parity split
constexpr int kSRows = kMY + 2;                                // tile rows and their y halo
constexpr int kSPts = kMX * kSRows;                            // 384 x sums per plane
constexpr int kSPer = (kSPts + kMThreads - 1) / kMThreads;     // 2 per thread

// Slot of the x sum of tile column lx (0..63) on halo row hy (0..5).
__host__ __device__ constexpr int sx_slot(int lx, int hy) { return (hy * 2 + (lx & 1)) * kSXh + (lx >> 1); }

// Asynchronous 8-byte global -> shared copy (zero-filled when !valid: the
// source is then not read) and its group fences.
__device__ __forceinline__ void cp_async8(double* smem, const double* gmem, bool valid)
{
    const unsigned saddr = (unsigned)__cvta_generic_to_shared(smem);
    const int n = valid ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(saddr), "l"(gmem), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Planes are staged kSepAhead steps ahead into a ring of kSepRing slots by
// asynchronous copies, so three planes of loads are in flight per block
// without holding them in registers.  (A ring of 8 slots, 6 planes ahead,
// with the diagonal staged too, measured 0.234 against 0.221 ms at 320^3.)
constexpr int kSepRing = 4, kSepAhead = 3;

// TMA staging of the planes (even grids with 4-aligned colour bricks): one
// tiled box per colour brick of the plane's z parity, 36 x 3 x 1 doubles, so
// a plane is four boxes issued by one thread and completing on the ring
// slot's mbarrier instead of 396 eight-byte copies.  Shared layout: block
// (py, px) of 3 lines x 36, the x-odd lines shifted by one (their box starts
// two brick columns left of the tile: a box starts on 16 bytes); blocks are
// padded to 112 doubles so that every box lands on a 128-byte boundary.
constexpr int kSepTmaLine = 36, kSepTmaBlock = 112, kSepTmaPlane = 4 * kSepTmaBlock;
constexpr unsigned kSepTmaBytes = 4 * 3 * kSepTmaLine * 8;  // the four boxes
static_assert(kSepTmaBlock >= 3 * kSepTmaLine && (kSepTmaBlock * 8) % 128 == 0, "TMA plane blocks");

struct SepMaps
{
    CUtensorMap m[8];  // the eight colour bricks of p (box 36 x 3 x 1)
};

// Shared slot of staged point (hx, hy) of the 66 x 6 plane: natural x = x0 + hx - 1, y = y0 + hy - 1.
template <bool kTma>
__host__ __device__ constexpr int sep_slot(int hx, int hy)
{
    if constexpr(!kTma) return plane_slot(hx, hy);
    const int px = (hx + 1) & 1, py = (hy + 1) & 1;
    return (py * 2 + px) * kSepTmaBlock + (hy >> 1) * kSepTmaLine + (hx >> 1) + px;
}

// The ring's mbarriers, initialised once per kernel before the first tile.
__device__ __forceinline__ void sep_tma_init(uint64_t* bars)
{
    if(threadIdx.x == 0)
        for(int i = 0; i < kSepRing; ++i) tma::mbar_init(&bars[i], 1);
    __syncthreads();
}

// One tile (64 x 4 columns, kSZ planes) of the separable product; returns the
// thread's running p.Ap sum.  Called by k64_spmv_sep (one tile per block) and
// by the persistent CG step (a loop over tiles); the staging buffers are
// reused from one tile to the next.  kTma: planes staged by TMA boxes (maps,
// bars, and the ring slots' phase bits in *phase, carried across tiles with
// the x-sum buffer toggle in bit 30; bit 31 records a wait that timed out).
template <bool kPap, bool kTma = false>
__device__ __forceinline__ double sep_tile(const StencilLevel& L, const double* __restrict__ diag,
                                           const double* __restrict__ p, double* __restrict__ Ap, int bx, int by,
                                           int bz, double s, const SepMaps* maps = nullptr,
                                           uint64_t* bars = nullptr, unsigned* phase = nullptr)
{
    constexpr int kSlots = kTma ? kSepTmaPlane : kPlane;
    __shared__ __align__(128) double xs[kSepRing][kSlots];  // staged planes with their one-point halo (66 x 6)
    __shared__ double sxs[kTma ? 2 : 1][kSPts];             // x sums of the 64 x 6 points
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int x0 = bx * kMX, y0 = by * kMY, zb = bz * kSZ;  // zb even
    const int ze = zb + kSZ < L.nz ? zb + kSZ : L.nz;

    // staged positions, as in the march (eight-byte copies)
    int slot[kMLoads];
    bool inxy[kMLoads];
    CanonColumn col[kMLoads];
    if constexpr(!kTma)
    {
#pragma unroll
        for(int k = 0; k < kMLoads; ++k)
        {
            const int e = tid + k * kMThreads;
            const int hx = e % kPX, hy = e / kPX;
            const int x = x0 + hx - 1, y = y0 + hy - 1;
            slot[k] = e < kPlane ? plane_slot(hx, hy) : -1;
            inxy[k] = e < kPlane && x >= 0 && x < L.nx && y >= 0 && y < L.ny;
            col[k] = canon_column(L, inxy[k] ? x : 0, inxy[k] ? y : 0);
        }
    }
    // x-sum positions: a warp takes one halo row and one x parity
    int sdst[kSPer], sm[kSPer], s0[kSPer], sp[kSPer];
#pragma unroll
    for(int k = 0; k < kSPer; ++k)
    {
        const int e = tid + k * kMThreads;
        const int hy = e >> 6, lx = 2 * (e & 31) + ((e >> 5) & 1);
        sdst[k] = e < kSPts ? sx_slot(lx, hy) : -1;
        sm[k] = sep_slot<kTma>(lx, hy);
        s0[k] = sep_slot<kTma>(lx + 1, hy);
        sp[k] = sep_slot<kTma>(lx + 2, hy);
    }
    // own output column: warp -> (x parity, row), lane -> x
    const int px = warp & 1, ly = warp >> 1;
    const int lx = 2 * lane + px;
    const int x = x0 + lx, y = y0 + ly;
    const bool mine = x < L.nx && y < L.ny;
    const int c = sep_slot<kTma>(lx + 1, ly + 1);
    const int cm = sx_slot(lx, ly), c0 = sx_slot(lx, ly + 1), cp = sx_slot(lx, ly + 2);
    const CanonColumn own = canon_column(L, mine ? x : 0, mine ? y : 0);

    // plane z into ring slot z mod kSepRing (zeros outside the grid)
    auto issue = [&](int z, auto zq) {
        constexpr int q = decltype(zq)::value;  // z & 1
        double* dst = xs[(z + kSepRing) & (kSepRing - 1)];
        if constexpr(kTma)
        {
            if(tid == 0)
            {
                uint64_t* bar = &bars[(z + kSepRing) & (kSepRing - 1)];
                // p may have been written by other blocks of this kernel (the
                // CG step's p update): order this thread's view of those
                // generic-proxy writes before its async-proxy reads
                asm volatile("fence.proxy.async.global;" ::: "memory");
                tma::mbar_arrive_expect_tx(bar, kSepTmaBytes);
#pragma unroll
                for(int py = 0; py < 2; ++py)
#pragma unroll
                    for(int pxx = 0; pxx < 2; ++pxx)
                    {
                        const int v = (int)((0x01456327u >> (4 * ((pxx << 2) | (py << 1) | q))) & 15u);
                        tma::load_3d(dst + (py * 2 + pxx) * kSepTmaBlock, &maps->m[v], x0 / 2 - 2 * pxx,
                                     y0 / 2 - py, z >> 1, bar);
                    }
            }
        }
        else
        {
            const bool zin = z >= 0 && z < L.nz;
#pragma unroll
            for(int k = 0; k < kMLoads; ++k)
                if(slot[k] >= 0)
                {
                    const bool v = inxy[k] && zin;
                    cp_async8(dst + slot[k], v ? p + canon_row<q>(col[k], z) : p, v);
                }
        }
    };
    // plane t is in its ring slot: this thread's copies (cp.async) or the
    // slot's mbarrier phase (TMA)
    auto landed = [&](int t) {
        if constexpr(kTma)
        {
            const int sl = (t + kSepRing) & (kSepRing - 1);
            const unsigned ph = (*phase >> sl) & 1u;
            // after a time-out the remaining planes are not waited for (the
            // solve is reported failed; each wait would run its full limit)
            if(!(*phase >> 31) && !tma::mbar_wait(&bars[sl], ph)) *phase |= 1u << 31;
            *phase ^= 1u << sl;
        }
        else
        {
            cp_async_wait<kSepAhead>();
        }
    };
    using Q0 = std::integral_constant<int, 0>;
    using Q1 = std::integral_constant<int, 1>;

    double r0 = 0.0, r1 = 0.0, r2 = 0.0;  // sxy of planes t-2, t-1, t
    double xo0 = 0.0, xo1 = 0.0;          // own x of planes t-1, t
    double dn = 0.0;                       // a_ii of the row plane finished at the next step
    issue(zb - 1, Q1{});
    if constexpr(!kTma) cp_async_commit();
    issue(zb, Q0{});
    if constexpr(!kTma) cp_async_commit();
    issue(zb + 1, Q1{});
    if constexpr(!kTma) cp_async_commit();
    // step t: plane t+3 goes out, plane t is summed, row plane t-1 (of
    // parity q = (t+1)&1 = (t+3)&1) is finished
    auto step = [&](int t, auto zq) {
        constexpr int q = decltype(zq)::value;
        if(t + kSepAhead <= ze) issue(t + kSepAhead, zq);  // its slot held plane t-1, read last step
        if constexpr(!kTma) cp_async_commit();
        const int zo = t - 1;
        const bool out = mine && zo >= zb;
        const double d = dn;
        dn = (mine && t >= zb && t < ze) ? diag[canon_row<q ^ 1>(own, t)] : 0.0;
        landed(t);
        // cp.async: everyone's copies of plane t have landed, and the x sums
        // of the last step are read.  TMA: every thread has waited on the
        // plane's mbarrier itself, and the x sums alternate between two
        // buffers (bit 30 of *phase), so one barrier per plane suffices: the
        // buffer written here was last read two steps ago, before the barrier
        // of the last step.
        if constexpr(!kTma) __syncthreads();
        double* sx = sxs[kTma ? ((*phase >> 30) & 1u) : 0];
        const double* xp = xs[(t + kSepRing) & (kSepRing - 1)];
#pragma unroll
        for(int k = 0; k < kSPer; ++k)
            if(sdst[k] >= 0) sx[sdst[k]] = (xp[sm[k]] + xp[s0[k]]) + xp[sp[k]];
        const double xn = xp[c];
        __syncthreads();  // x sums of plane t stored; plane t no longer read
        if constexpr(kTma) *phase ^= 1u << 30;
        r0 = r1;
        r1 = r2;
        r2 = (sx[cm] + sx[c0]) + sx[cp];
        xo0 = xo1;
        xo1 = xn;
        if(out)
        {
            const double nbr = ((r0 + r1) + r2) - xo0;  // the 26 neighbours of (x, y, zo)
            const double v = fma(d, xo0, -nbr);
            Ap[canon_row<q>(own, zo)] = v;
            if(kPap) s = fma(v, xo0, s);
        }
    };
    for(int t = zb - 1; t <= ze; t += 2)
    {
        step(t, Q0{});
        if(t + 1 <= ze) step(t + 1, Q1{});
    }
    if constexpr(!kTma) cp_async_wait<0>();
    return s;
}

template <bool kPap, bool kTma>
__global__ void __launch_bounds__(kMThreads) k64_spmv_sep(const StencilLevel L, const double* __restrict__ diag,
                                                          const double* __restrict__ p, double* __restrict__ Ap,
                                                          CGState* st, double* partial, unsigned int* ticket,
                                                          const __grid_constant__ SepMaps maps)
{
    __shared__ double red[32];
    __shared__ bool last;
    __shared__ uint64_t bars[kSepRing];
    unsigned phase = 0;
    if constexpr(kTma) sep_tma_init(bars);
    double s = sep_tile<kPap, kTma>(L, diag, p, Ap, blockIdx.x, blockIdx.y, blockIdx.z, 0.0, &maps, bars, &phase);
    if(kTma && (phase >> 31) && st && threadIdx.x == 0) atomicExch(&st->status, 3);
    if(!kPap) return;
    const int tid = threadIdx.x;
    s = block_sum(s, red);
    const unsigned nblocks = gridDim.x * gridDim.y * gridDim.z;
    const unsigned bid = (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
    if(tid == 0)
    {
        partial[bid] = s;
        __threadfence();
        last = atomicAdd(ticket, 1u) == nblocks - 1;
    }
    __syncthreads();
    if(!last) return;
    __threadfence();
    double acc = 0.0;
    for(int k = tid; k < (int)nblocks; k += kMThreads) acc += __ldcg(&partial[k]);
    acc = block_sum(acc, red);
    if(tid == 0)
    {
        *ticket = 0;
        st->pAp = acc;
        st->alpha = st->rtz / acc;
    }
}

// Step 1 of the two-kernel CG step with the separable product (canonical
// colouring): r.z, beta, p update (the rows of n), then the tiles of the
// product in a loop, p.Ap and alpha.  Persistent and cooperative.  kTma: the
// product's planes staged by TMA (the p update's stores are fenced for the
// async proxy before the grid barrier that precedes them).
template <typename Z, bool kTma>
__global__ void __launch_bounds__(kMThreads) k_cg_step1_sep(const StencilLevel L, const double* __restrict__ diag,
                                                            const double* __restrict__ r, const Z* __restrict__ z,
                                                            double* __restrict__ p, double* __restrict__ x,
                                                            double* __restrict__ Ap, CGState* st, double* partial,
                                                            unsigned int* ticket, GridBarrier* gb,
                                                            const __grid_constant__ SepMaps maps)
{
    __shared__ uint64_t bars[kSepRing];
    unsigned phase = 0;
    if constexpr(kTma) sep_tma_init(bars);
    if(!step1_rz_p(L.m, r, z, p, x, st, partial, gb)) return;
    const int tx = (L.nx + kMX - 1) / kMX, ty = (L.ny + kMY - 1) / kMY, tz = (L.nz + kSZ - 1) / kSZ;
    const int ntiles = tx * ty * tz;
    double s = 0.0;
    for(int tile = blockIdx.x; tile < ntiles; tile += gridDim.x)
    {
        const int bz = tile / (tx * ty), rem = tile - bz * tx * ty;
        const int by = rem / tx, bx = rem - by * tx;
        s = sep_tile<true, kTma>(L, diag, p, Ap, bx, by, bz, s, &maps, bars, &phase);
    }
    if(kTma && (phase >> 31) && threadIdx.x == 0) atomicExch(&st->status, 3);
    step1_alpha(s, st, partial, ticket);
}

inline dim3 sep_grid(const StencilLevel& L)
{
    return dim3((unsigned)((L.nx + kMX - 1) / kMX), (unsigned)((L.ny + kMY - 1) / kMY),
                (unsigned)((L.nz + kSZ - 1) / kSZ));
}

// ------------------------------------------------------------ set-up kernels

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
    // permuted row i -> its ELL row must be the implicit neighbour list, and
    // on even grids the constant-delta form must give the same columns
    {
        int v = 0;
        while(v + 1 < 8 && i >= L.offsets[v + 1]) ++v;
        const int q = i - L.offsets[v];
        const int t = q / L.bx[v];
        const int kz = t / L.by[v];
        const int ky = t - kz * L.by[v];
        const int kx = q - t * L.bx[v];
        const int p = L.par[v];
        const int ix = 2 * kx + ((p >> 2) & 1), iy = 2 * ky + ((p >> 1) & 1), iz = 2 * kz + (p & 1);
        const unsigned mask = (ix == 0 ? 1u : 0u) | (ix == L.nx - 1 ? 2u : 0u) | (iy == 0 ? 4u : 0u) |
                              (iy == L.ny - 1 ? 8u : 0u) | (iz == 0 ? 16u : 0u) | (iz == L.nz - 1 ? 32u : 0u);
        const StencilTab& tb = L.tab[v];
        int slot = 0;
        for(int j = 0; j < 27; ++j)
        {
            int col;
            const bool ok = nb_col(L, tb.nb[j], ix, iy, iz, col);
            if(L.even) nbad += ok != !(mask & tb.bmask[j]) || (ok && col != i + tb.delta[j]);
            if(!ok) continue;
            const size_t idx = (size_t)slot * L.m + i;
            nbad += ell_col[idx] != col;
            if(j != tb.dp) nbad += ell_val[idx] != -1.0;
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

// Compile-time parameters of the 4-row kernels: the slot-group size (all
// slots at once on small levels) and the colour's parity class when the level
// has the canonical colouring (compile-time slot tables; -1: the launch's
// runtime tables).
template <int K>
using IntC = std::integral_constant<int, K>;

template <typename F>
cudaError_t by_class(const StencilLevel& L, int par, F&& f)
{
    if(!L.canon) return f(IntC<-1>{});
    switch(par)
    {
        case 0: return f(IntC<0>{});
        case 1: return f(IntC<1>{});
        case 2: return f(IntC<2>{});
        case 3: return f(IntC<3>{});
        case 4: return f(IntC<4>{});
        case 5: return f(IntC<5>{});
        case 6: return f(IntC<6>{});
        default: return f(IntC<7>{});
    }
}

template <typename T>
constexpr int kV4GroupSmallOf = std::is_same<T, float>::value ? kV4GroupSmall : kV4GroupSmall64;

// f(group, class) for colour c of level L.
template <typename T, typename F>
cudaError_t by_shape(const StencilLevel& L, const ColorLaunch& c, F&& f)
{
    if(L.m / 8 < kV4SmallRows) return by_class(L, c.par, [&](auto k) { return f(IntC<kV4GroupSmallOf<T>>{}, k); });
    return by_class(L, c.par, [&](auto k) { return f(IntC<kV4GroupLarge>{}, k); });
}

// f(group, class) for the restriction, which runs on the parity-0 colour.
template <typename T, typename F>
cudaError_t by_shape_restrict(const StencilLevel& Lf, F&& f)
{
    auto cls = [&](auto g) { return Lf.canon ? f(g, IntC<0>{}) : f(g, IntC<-1>{}); };
    return Lf.m / 8 < kV4SmallRows ? cls(IntC<kV4GroupSmallOf<T>>{}) : cls(IntC<kV4GroupLarge>{});
}

// TMA maps of one vector of a level: map[u][d] covers colour u's brick with
// the box a launching colour sees when its parity differs from u's by d.
struct SweepMaps
{
    const void* x = nullptr;
    int esize = 0, m = 0, nx = 0, ny = 0, nz = 0;
    CUtensorMap map[8][8];
};

static int encode_brick_map(CUtensorMap* map, const void* base, int esize, int bx, int by, int bz, int boxx, int boxy,
                            int boxz)
{
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if(!encode)
    {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        HB_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
        if(q != cudaDriverEntryPointSuccess || !fn)
            return record_error(HPCGB200_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
        encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    const cuuint64_t dims[3] = {(cuuint64_t)bx, (cuuint64_t)by, (cuuint64_t)bz};
    const cuuint64_t strides[2] = {(cuuint64_t)bx * esize, (cuuint64_t)bx * by * esize};
    const cuuint32_t box[3] = {(cuuint32_t)boxx, (cuuint32_t)boxy, (cuuint32_t)boxz};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = encode(map, esize == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3,
                              const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if(r != CUDA_SUCCESS) return record_error(HPCGB200_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return 0;
}

// Maps of x on level L, built once per (vector, level) and kept (a V-cycle
// sweeps the same few vectors).
template <typename T>
static std::shared_ptr<const SweepMaps> sweep_maps(const StencilLevel& L, const T* x)
{
    static std::mutex mu;
    static std::vector<std::shared_ptr<SweepMaps>> cache;
    std::lock_guard<std::mutex> lock(mu);
    const int es = (int)sizeof(T);
    for(const auto& e : cache)
        if(e->x == x && e->esize == es && e->m == L.m && e->nx == L.nx && e->ny == L.ny && e->nz == L.nz)
            return e;
    auto e = std::make_shared<SweepMaps>();
    e->x = x;
    e->esize = es;
    e->m = L.m;
    e->nx = L.nx;
    e->ny = L.ny;
    e->nz = L.nz;
    for(int u = 0; u < 8; ++u)
    {
        const int bz = (L.nz - (L.par[u] & 1) + 1) / 2;
        for(int d = 1; d < 8; ++d)
            if(encode_brick_map(&e->map[u][d], x + L.offsets[u], es, L.bx[u], L.by[u], bz, kTmaX + 4 * ((d >> 2) & 1),
                                kTmaYOf<T> + ((d >> 1) & 1), kTmaZ + (d & 1)))
                return nullptr;
    }
    if(cache.size() >= 64) cache.erase(cache.begin());
    cache.push_back(std::move(e));
    return cache.back();
}

// The TMA-staged colour passes serve large even levels with the canonical
// colouring (HPCGB200_SWEEP_TMA=0 keeps the 4-row kernels everywhere).
static bool sweep_tma_enabled()
{
    static const bool on = [] {
        const char* e = getenv("HPCGB200_SWEEP_TMA");
        return !(e && e[0] == '0');
    }();
    return on;
}

// Large even level with the canonical colouring, x 16-byte aligned, no fused
// prolongation: the TMA-staged passes apply.
template <typename T>
static bool pass_tma_ok(const StencilLevel& L, const T* x, const Prolong<T>& pro)
{
    return sweep_tma_enabled() && vec4_ok(L) && L.canon && L.m / 8 >= kV4SmallRows && !pro.xf &&
           (reinterpret_cast<uintptr_t>(x) & 15u) == 0;
}

template <typename T, int C, int K, bool D>
static cudaError_t launch_pass_tma(const StencilLevel& L, const ColorLaunch& c, const SweepMaps& M,
                                   const T* inv_diag, const T* diag, const double* r64, T* r, T* x, double* z64,
                                   const int* inj_c, T* rc, cudaStream_t s)
{
    NbMaps nb;
    for(int u = 0, i = 0; u < 8; ++u)
        if(tma_reads(K, c.v, u)) nb.m[i++] = M.map[u][L.par[c.v] ^ L.par[u]];
    const dim3 grid((unsigned)((c.bx + kTmaX - 1) / kTmaX), (unsigned)((c.by + kTmaYOf<T> - 1) / kTmaYOf<T>),
                    (unsigned)((c.bz + kTmaZ - 1) / kTmaZ));
    const size_t smem = (size_t)TmaTab<T, C, K>::p.total * sizeof(T) + 128;
    return launch_pdl_smem(kv_pass_tma<T, C, K, D>, grid, dim3(kTmaX / 4, kTmaYOf<T>, kTmaZ), smem, s, nb, c,
                           inv_diag, diag, r64, r, x, z64, inj_c, rc, L.status);
}

// One TMA-staged pass of kind K over colour c (canonical colouring: the
// class is a compile-time constant).
template <typename T, int K, bool D = false>
static cudaError_t pass_tma(const StencilLevel& L, const ColorLaunch& c, const SweepMaps& M, const T* inv_diag,
                            const T* diag, const double* r64, T* r, T* x, double* z64, cudaStream_t s,
                            const int* inj_c = nullptr, T* rc = nullptr)
{
    return by_class(L, c.par, [&](auto kc) {
        constexpr int C = decltype(kc)::value;
        if constexpr(C < 0) return cudaErrorInvalidValue;  // L.canon holds on this path
        else return launch_pass_tma<T, C, K, D>(L, c, M, inv_diag, diag, r64, r, x, z64, inj_c, rc, s);
    });
}

// The colour n-1 is final after the forward sweep, the others after the
// backward sweep (n-2..0): those passes carry the fused prolongation `pro`.
int launch32_symgs_zero(const StencilLevel& L, const float* diag32, const float* inv_diag32, const double* r64,
                        float* r32, float* x, cudaStream_t s, Prolong<float> pro)
{
    const int n = L.ncolors;
    const dim3 t(32, 8), t4(kV4X, kV4Y);
    const bool vec = vec4_ok(L);
    const bool tma = pass_tma_ok(L, x, pro);
    const std::shared_ptr<const SweepMaps> maps = tma ? sweep_maps(L, x) : nullptr;
    if(tma && !maps) return HPCGB200_ERR_CUDA;
    for(int v = 0; v < n; ++v)
    {
        if(L.offsets[v + 1] - L.offsets[v] <= 0) continue;
        const ColorLaunch c = color_launch(L, v);
        const dim3 g = brick_grid(c);
        const Prolong<float> pv = v == n - 1 ? pro : Prolong<float>{};
        if(maps)
        {
            HB_CUDA((r64 ? pass_tma<float, kTmaFwd0, true>(L, c, *maps, inv_diag32, nullptr, r64, r32, x, nullptr, s)
                         : pass_tma<float, kTmaFwd0>(L, c, *maps, inv_diag32, nullptr, nullptr, r32, x, nullptr, s)));
        }
        else if(vec)
        {
            HB_CUDA(by_shape<float>(L, c, [&](auto kg, auto kc) {
                constexpr int G = decltype(kg)::value, C = decltype(kc)::value;
                return r64 ? launch_pdl(kv_fwd0<float, true, G, C>, brick_grid4(c), t4, s, c, L, inv_diag32, r64,
                                        r32, x, pv)
                           : launch_pdl(kv_fwd0<float, false, G, C>, brick_grid4(c), t4, s, c, L, inv_diag32, nullptr,
                                        r32, x, pv);
            }));
        }
        else if(L.even)
        {
            if(r64) k32_fwd0<true, true><<<g, t, 0, s>>>(c, L, inv_diag32, r64, r32, x, pv);
            else k32_fwd0<true, false><<<g, t, 0, s>>>(c, L, inv_diag32, nullptr, r32, x, pv);
        }
        else
        {
            if(r64) k32_fwd0<false, true><<<g, t, 0, s>>>(c, L, inv_diag32, r64, r32, x, pv);
            else k32_fwd0<false, false><<<g, t, 0, s>>>(c, L, inv_diag32, nullptr, r32, x, pv);
        }
        HB_LAUNCHED();
    }
    for(int v = n - 2; v >= 0; --v)
    {
        if(L.offsets[v + 1] - L.offsets[v] <= 0) continue;
        const ColorLaunch c = color_launch(L, v);
        if(maps)
        {
            HB_CUDA((pass_tma<float, kTmaBwd0>(L, c, *maps, inv_diag32, diag32, nullptr, nullptr, x, nullptr, s)));
        }
        else if(vec)
        {
            HB_CUDA(by_shape<float>(L, c, [&](auto kg, auto kc) {
                constexpr int G = decltype(kg)::value, C = decltype(kc)::value;
                return launch_pdl(kv_bwd0<float, G, C>, brick_grid4(c), t4, s, c, L, diag32, inv_diag32, x, pro);
            }));
        }
        else if(L.even) k32_bwd0<true><<<brick_grid(c), t, 0, s>>>(c, L, diag32, inv_diag32, x, pro);
        else k32_bwd0<false><<<brick_grid(c), t, 0, s>>>(c, L, diag32, inv_diag32, x, pro);
        HB_LAUNCHED();
    }
    return 0;
}

int launch32_symgs(const StencilLevel& L, const float* inv_diag32, const float* r, float* x, double* z64,
                   cudaStream_t s, Prolong<float> pro)
{
    const int n = L.ncolors;
    const bool vec = vec4_ok(L);
    const bool tma = pass_tma_ok(L, x, pro);
    const std::shared_ptr<const SweepMaps> maps = tma ? sweep_maps(L, x) : nullptr;
    if(tma && !maps) return HPCGB200_ERR_CUDA;
    auto sweep = [&](int v, double* z, Prolong<float> pv) -> int {
        if(L.offsets[v + 1] - L.offsets[v] <= 0) return 0;
        const ColorLaunch c = color_launch(L, v);
        if(maps)
            HB_CUDA((pass_tma<float, kTmaSweep>(L, c, *maps, inv_diag32, nullptr, nullptr, const_cast<float*>(r), x, z,
                                                s)));
        else if(vec)
        {
            HB_CUDA(by_shape<float>(L, c, [&](auto kg, auto kc) {
                constexpr int G = decltype(kg)::value, C = decltype(kc)::value;
                return launch_pdl(kv_sweep<float, G, C>, brick_grid4(c), dim3(kV4X, kV4Y), s, c, L, inv_diag32, r, x,
                                  z, pv);
            }));
        }
        else if(L.even) k32_sweep<true><<<brick_grid(c), dim3(32, 8), 0, s>>>(c, L, inv_diag32, r, x, z, pv);
        else k32_sweep<false><<<brick_grid(c), dim3(32, 8), 0, s>>>(c, L, inv_diag32, r, x, z, pv);
        HB_LAUNCHED();
        return 0;
    };
    // colour n-1 is final after the forward sweep (the backward sweep starts
    // at n-2): it writes z64 and carries the fused prolongation there
    for(int v = 0; v < n; ++v)
        HB_RETURN_IF(sweep(v, v == n - 1 ? z64 : nullptr, v == n - 1 ? pro : Prolong<float>{}));
    for(int v = n - 2; v >= 0; --v) HB_RETURN_IF(sweep(v, z64, pro));
    return 0;
}

int launch32_restrict(const StencilLevel& Lf, int nc, const int* inj_f, const int* inj_c, const float* diag32,
                      const float* rf, const float* xf, float* rc, cudaStream_t s)
{
    const ColorLaunch c = color_launch(Lf, Lf.color_of_par[0]);
    const std::shared_ptr<const SweepMaps> maps =
        pass_tma_ok(Lf, xf, {}) && nc == c.bx * c.by * c.bz ? sweep_maps(Lf, xf) : nullptr;
    if(maps)
    {
        HB_CUDA((pass_tma<float, kTmaRestrict>(Lf, c, *maps, nullptr, diag32, nullptr, const_cast<float*>(rf),
                                                const_cast<float*>(xf), nullptr, s, inj_c, rc)));
    }
    else if(vec4_ok(Lf) && nc == c.bx * c.by * c.bz)
    {
        HB_CUDA(by_shape_restrict<float>(Lf, [&](auto kg, auto kc) {
            constexpr int G = decltype(kg)::value, C = decltype(kc)::value;
            return launch_pdl(kv_restrict<float, G, C>, brick_grid4(c), dim3(kV4X, kV4Y), s, c, Lf, inj_c, diag32, rf,
                              xf, rc);
        }));
    }
    else if(Lf.even) k32_restrict<true><<<nblk(nc), kBS32, 0, s>>>(c, Lf, nc, inj_f, inj_c, diag32, rf, xf, rc);
    else k32_restrict<false><<<nblk(nc), kBS32, 0, s>>>(c, Lf, nc, inj_f, inj_c, diag32, rf, xf, rc);
    HB_LAUNCHED();
    return 0;
}

int launch32_prolong(const StencilLevel& Lf, int nc, const int* inj_f, const int* inj_c, const float* xc, float* xf,
                     cudaStream_t s)
{
    const ColorLaunch c = color_launch(Lf, Lf.color_of_par[0]);
    if(vec4_ok(Lf) && nc == c.bx * c.by * c.bz)
        HB_CUDA(launch_pdl(kv_prolong<float>, brick_grid4(c), dim3(kV4X, kV4Y), s, c, inj_c, xc, xf));
    else
        k32_prolong<<<nblk(nc), kBS32, 0, s>>>(nc, inj_f, inj_c, xc, xf);
    HB_LAUNCHED();
    return 0;
}

// ------------------------------------------ FP64 V-cycle on the implicit stencil
// The same 4-row kernels in double precision: each row performs the ELL
// kernels' operations in the same order (sum + x == fma(1, x, sum) per
// off-diagonal slot, x * (1/a_ii), x_i * a_ii rounded then the later slots,
// fma(-a_ii, x_i, .) in the restriction), so the results are the FP64 ELL
// V-cycle's bits without reading the matrix.

bool stencil_vec4(const StencilLevel& L) { return vec4_ok(L); }

int launch64v_symgs_zero(const StencilLevel& L, const double* diag, const double* inv_diag, const double* r,
                         double* x, cudaStream_t s, Prolong<double> pro)
{
    if(!vec4_ok(L)) return record_error(HPCGB200_ERR_ARG, "FP64 stencil V-cycle: colour bricks not 4-aligned");
    const dim3 t4(kV4X, kV4Y);
    const std::shared_ptr<const SweepMaps> maps = pass_tma_ok(L, x, pro) ? sweep_maps(L, x) : nullptr;
    if(pass_tma_ok(L, x, pro) && !maps) return HPCGB200_ERR_CUDA;
    for(int v = 0; v < L.ncolors; ++v)
    {
        if(L.offsets[v + 1] - L.offsets[v] <= 0) continue;
        const ColorLaunch c = color_launch(L, v);
        const Prolong<double> pv = v == L.ncolors - 1 ? pro : Prolong<double>{};
        if(maps)
        {
            HB_CUDA((pass_tma<double, kTmaFwd0>(L, c, *maps, inv_diag, nullptr, nullptr, const_cast<double*>(r), x,
                                                nullptr, s)));
            continue;
        }
        HB_CUDA(by_shape<double>(L, c, [&](auto kg, auto kc) {
            constexpr int G = decltype(kg)::value, C = decltype(kc)::value;
            return launch_pdl(kv_fwd0<double, false, G, C>, brick_grid4(c), t4, s, c, L, inv_diag, nullptr,
                              const_cast<double*>(r), x, pv);
        }));
    }
    for(int v = L.ncolors - 2; v >= 0; --v)
    {
        if(L.offsets[v + 1] - L.offsets[v] <= 0) continue;
        const ColorLaunch c = color_launch(L, v);
        if(maps)
        {
            HB_CUDA((pass_tma<double, kTmaBwd0>(L, c, *maps, inv_diag, diag, nullptr, nullptr, x, nullptr, s)));
            continue;
        }
        HB_CUDA(by_shape<double>(L, c, [&](auto kg, auto kc) {
            constexpr int G = decltype(kg)::value, C = decltype(kc)::value;
            return launch_pdl(kv_bwd0<double, G, C>, brick_grid4(c), t4, s, c, L, diag, inv_diag, x, pro);
        }));
    }
    return 0;
}

int launch64v_symgs(const StencilLevel& L, const double* inv_diag, const double* r, double* x, cudaStream_t s,
                    Prolong<double> pro)
{
    if(!vec4_ok(L)) return record_error(HPCGB200_ERR_ARG, "FP64 stencil V-cycle: colour bricks not 4-aligned");
    const std::shared_ptr<const SweepMaps> maps = pass_tma_ok(L, x, pro) ? sweep_maps(L, x) : nullptr;
    if(pass_tma_ok(L, x, pro) && !maps) return HPCGB200_ERR_CUDA;
    auto sweep = [&](int v, Prolong<double> pv) -> int {
        if(L.offsets[v + 1] - L.offsets[v] <= 0) return 0;
        const ColorLaunch c = color_launch(L, v);
        if(maps)
        {
            HB_CUDA((pass_tma<double, kTmaSweep>(L, c, *maps, inv_diag, nullptr, nullptr, const_cast<double*>(r), x,
                                                 nullptr, s)));
            return 0;
        }
        HB_CUDA(by_shape<double>(L, c, [&](auto kg, auto kc) {
            constexpr int G = decltype(kg)::value, C = decltype(kc)::value;
            return launch_pdl(kv_sweep<double, G, C>, brick_grid4(c), dim3(kV4X, kV4Y), s, c, L, inv_diag, r, x,
                              nullptr, pv);
        }));
        return 0;
    };
    for(int v = 0; v < L.ncolors; ++v) HB_RETURN_IF(sweep(v, v == L.ncolors - 1 ? pro : Prolong<double>{}));
    for(int v = L.ncolors - 2; v >= 0; --v) HB_RETURN_IF(sweep(v, pro));
    return 0;
}

int launch64v_restrict(const StencilLevel& Lf, int nc, const int* inj_c, const double* diag, const double* rf,
                       const double* xf, double* rc, cudaStream_t s)
{
    const ColorLaunch c = color_launch(Lf, Lf.color_of_par[0]);
    if(!vec4_ok(Lf) || nc != c.bx * c.by * c.bz)
        return record_error(HPCGB200_ERR_ARG, "FP64 stencil restriction: colour bricks not 4-aligned");
    if(pass_tma_ok(Lf, xf, Prolong<double>{}))
    {
        const std::shared_ptr<const SweepMaps> maps = sweep_maps(Lf, xf);
        if(!maps) return HPCGB200_ERR_CUDA;
        HB_CUDA((pass_tma<double, kTmaRestrict>(Lf, c, *maps, nullptr, diag, nullptr, const_cast<double*>(rf),
                                                 const_cast<double*>(xf), nullptr, s, inj_c, rc)));
        return 0;
    }
    HB_CUDA(by_shape_restrict<double>(Lf, [&](auto kg, auto kc) {
        constexpr int G = decltype(kg)::value, C = decltype(kc)::value;
        return launch_pdl(kv_restrict<double, G, C>, brick_grid4(c), dim3(kV4X, kV4Y), s, c, Lf, inj_c, diag, rf, xf,
                          rc);
    }));
    return 0;
}

int launch64v_prolong(const StencilLevel& Lf, int nc, const int* inj_c, const double* xc, double* xf, cudaStream_t s)
{
    const ColorLaunch c = color_launch(Lf, Lf.color_of_par[0]);
    if(!vec4_ok(Lf) || nc != c.bx * c.by * c.bz)
        return record_error(HPCGB200_ERR_ARG, "FP64 stencil prolongation: colour bricks not 4-aligned");
    HB_CUDA(launch_pdl(kv_prolong<double>, brick_grid4(c), dim3(kV4X, kV4Y), s, c, inj_c, xc, xf));
    return 0;
}

// Persistent grid: two 1024-thread blocks per SM (148 SMs on B200), never more
// blocks than tiles.
static int tile64_blocks(const StencilLevel& L)
{
    const dim3 g = tile64_grid(L);
    const long tiles = (long)g.x * g.y * g.z;
    return (int)(tiles < 2 * 148 ? tiles : 2 * 148);
}

size_t stencil_pap_partials(const StencilLevel& L)
{
    const dim3 g = march_grid(L), gs = sep_grid(L);
    size_t n = (size_t)g.x * g.y * g.z;
    n = n > (size_t)gs.x * gs.y * gs.z ? n : (size_t)gs.x * gs.y * gs.z;
    return n > (size_t)tile64_blocks(L) ? n : (size_t)tile64_blocks(L);
}

static bool canonical_colours(const StencilLevel& L)
{
    for(int q = 0; q < 8; ++q)
        if(L.color_of_par[q] != kCanonColor[q]) return false;
    return true;
}

int launch64_spmv_stencil(const StencilLevel& L, const double* diag, const double* x, double* y, cudaStream_t s)
{
    if(canonical_colours(L))
        k64_spmv_march<false><<<march_grid(L), kMThreads, 0, s>>>(L, diag, x, y, nullptr, nullptr, nullptr);
    else
        k64_spmv_tile<false><<<tile64_blocks(L), kT64Threads, 0, s>>>(L, diag, x, y, nullptr, nullptr, nullptr);
    HB_LAUNCHED();
    return 0;
}

// TMA maps of the eight colour bricks of one FP64 vector (box 36 x 3 x 1), for
// the separable product's plane staging; built once per (vector, grid) and
// kept.  The key holds the grid's dimensions, not only its size: a freed
// vector's address can come back for a grid of the same size and another
// shape, whose bricks the old maps would mis-describe.
struct SepMapsEntry
{
    const double* v;
    int nx, ny, nz;
    std::shared_ptr<SepMaps> maps;
};

static std::shared_ptr<const SepMaps> sep_maps(const StencilLevel& L, const double* v)
{
    static std::mutex mu;
    static std::vector<SepMapsEntry> cache;
    std::lock_guard<std::mutex> lock(mu);
    for(const auto& e : cache)
        if(e.v == v && e.nx == L.nx && e.ny == L.ny && e.nz == L.nz) return e.maps;
    auto M = std::make_shared<SepMaps>();
    for(int u = 0; u < 8; ++u)
    {
        const int bz = (L.nz - (L.par[u] & 1) + 1) / 2;
        if(encode_brick_map(&M->m[u], v + L.offsets[u], 8, L.bx[u], L.by[u], bz, kSepTmaLine, 3, 1)) return nullptr;
    }
    if(cache.size() >= 16) cache.erase(cache.begin());
    cache.push_back(SepMapsEntry{v, L.nx, L.ny, L.nz, std::move(M)});
    return cache.back().maps;
}

// The separable product stages its planes by TMA on even grids with 4-aligned
// colour bricks (HPCGB200_SEP_TMA=0: eight-byte asynchronous copies).
static std::shared_ptr<const SepMaps> sep_tma_maps(const StencilLevel& L, const double* v)
{
    static const bool on = [] {
        const char* e = getenv("HPCGB200_SEP_TMA");
        return !(e && e[0] == '0');
    }();
    if(!on || !vec4_ok(L) || (reinterpret_cast<uintptr_t>(v) & 15u)) return nullptr;
    return sep_maps(L, v);
}

int launch64_spmv_sep(const StencilLevel& L, const double* diag, const double* x, double* y, cudaStream_t s)
{
    if(canonical_colours(L))
    {
        const std::shared_ptr<const SepMaps> M = sep_tma_maps(L, x);
        if(M)
            k64_spmv_sep<false, true><<<sep_grid(L), kMThreads, 0, s>>>(L, diag, x, y, nullptr, nullptr, nullptr, *M);
        else
            k64_spmv_sep<false, false><<<sep_grid(L), kMThreads, 0, s>>>(L, diag, x, y, nullptr, nullptr, nullptr,
                                                                          SepMaps{});
    }
    else
        k64_spmv_tile<false><<<tile64_blocks(L), kT64Threads, 0, s>>>(L, diag, x, y, nullptr, nullptr, nullptr);
    HB_LAUNCHED();
    return 0;
}

int launch_cg_step1_sep(const StencilLevel& L, const double* diag, const double* r, const float* z, double* p,
                        double* x, double* Ap, CGState* st, ReduceScratch* ws, GridBarrier* gb, cudaStream_t s)
{
    if(!canonical_colours(L)) return record_error(HPCGB200_ERR_ARG, "CG step: the level is not canonically coloured");
    // each staging runs its own resident grid (the TMA form holds fewer
    // registers: 5 blocks per SM instead of 4); the r.z and p.Ap partitions
    // follow the grid, so the two forms' CG scalars agree to rounding (with
    // equal grids they agree bit for bit)
    static const int grid_tma = resident_grid(k_cg_step1_sep<float, true>, kMThreads, kReduceBlocks);
    static const int grid_cp = resident_grid(k_cg_step1_sep<float, false>, kMThreads, kReduceBlocks);
    const std::shared_ptr<const SepMaps> M = sep_tma_maps(L, p);
    const int grid = M ? grid_tma : grid_cp;
    if(grid <= 0) return record_error(HPCGB200_ERR_CUDA, "CG step: no resident grid");
    if(M)
        HB_CUDA(launch_coop(k_cg_step1_sep<float, true>, grid, kMThreads, s, L, diag, r, z, p, x, Ap, st, ws->partial,
                            &ws->ticket, gb, *M));
    else
        HB_CUDA(launch_coop(k_cg_step1_sep<float, false>, grid, kMThreads, s, L, diag, r, z, p, x, Ap, st,
                            ws->partial, &ws->ticket, gb, SepMaps{}));
    return 0;
}

int launch64_cg_spmv_pap_stencil(const StencilLevel& L, const double* diag, const double* p, double* Ap,
                                 CGState* st, double* partial, unsigned int* ticket, cudaStream_t s)
{
    if(canonical_colours(L))
    {
        const std::shared_ptr<const SepMaps> M = sep_tma_maps(L, p);
        if(M) k64_spmv_sep<true, true><<<sep_grid(L), kMThreads, 0, s>>>(L, diag, p, Ap, st, partial, ticket, *M);
        else
            k64_spmv_sep<true, false><<<sep_grid(L), kMThreads, 0, s>>>(L, diag, p, Ap, st, partial, ticket,
                                                                         SepMaps{});
    }
    else
        k64_spmv_tile<true><<<tile64_blocks(L), kT64Threads, 0, s>>>(L, diag, p, Ap, st, partial, ticket);
    HB_LAUNCHED();
    return 0;
}

}  // namespace hb
