// Device-side problem construction and optimization for libhpcgb200:
// 27-point problem generation, f2c operator, Jones-Plassmann-Luby multicoloring,
// stable color sort, column-sorted column-major ELL, diagonal extraction.
// All index results are bit-identical to the rocHPCG device path (the oracle
// test suite compares every array against the CPU restatement).
#include <cstdlib>
#include <cstring>
#include <vector>

#include "common.cuh"

namespace hb {

// ------------------------------------------------------------ generation
//
// One thread per (row, stencil slot), 32 rows x 27 slots per block, so the
// row-major stores are contiguous across a warp.  Slot order and boundary
// compaction follow src/GenerateProblem.cpp:165-273; the compacted position
// of an existing neighbour (dz,dy,dx) inside the box of existing offsets
// [zlo,zhi]x[ylo,yhi]x[xlo,xhi] is its lexicographic index in that box, which
// is what the reference's 27-lane inclusive scan computes.
constexpr int kGenRows = 32;

__global__ void __launch_bounds__(kGenRows* kWidth)
    k_generate_problem(int m, int nx, int ny, int nz, long long gnx, long long gny, long long gnz, long long gix0,
                       long long giy0, long long giz0, int* __restrict__ mtx_ind, double* __restrict__ values,
                       int8_t* __restrict__ nnz_in_row, int* __restrict__ diag_slot, long long* __restrict__ l2g,
                       int* __restrict__ hash, double* __restrict__ b)
{
    const long long g = (long long)blockIdx.x * (kGenRows * kWidth) + threadIdx.x;
    const int row = (int)(g / kWidth);
    const int s = (int)(g - (long long)row * kWidth);
    if(row >= m) return;
    const int iz = row / (nx * ny);
    const int iy = row / nx - ny * iz;
    const int ix = row - iz * nx * ny - iy * nx;
    const long long giz = giz0 + iz, giy = giy0 + iy, gix = gix0 + ix;
    const int zlo = giz > 0 ? -1 : 0, zhi = giz < gnz - 1 ? 1 : 0;
    const int ylo = giy > 0 ? -1 : 0, yhi = giy < gny - 1 ? 1 : 0;
    const int xlo = gix > 0 ? -1 : 0, xhi = gix < gnx - 1 ? 1 : 0;
    const int cz = zhi - zlo + 1, cy = yhi - ylo + 1, cx = xhi - xlo + 1;
    const int n = cz * cy * cx;
    const int dz = s / 9 - 1, dy = (s % 9) / 3 - 1, dx = s % 3 - 1;
    const size_t base = (size_t)row * kWidth;
    const bool exists = dz >= zlo && dz <= zhi && dy >= ylo && dy <= yhi && dx >= xlo && dx <= xhi;
    if(exists)
    {
        const int pos = ((dz - zlo) * cy + (dy - ylo)) * cx + (dx - xlo);
        // 1 rank: the global column id equals the local one (SetupHalo.cpp:313-327)
        const int col = (iz + dz) * nx * ny + (iy + dy) * nx + (ix + dx);
        mtx_ind[base + pos] = col;
        values[base + pos] = (s == 13) ? 26.0 : -1.0;
    }
    if(s >= n)
    {
        mtx_ind[base + s] = -1;  // kernel_copy_indices pads with -1
        values[base + s] = 0.0;
    }
    if(s == 13)
    {
        nnz_in_row[row] = (int8_t)n;
        diag_slot[row] = ((0 - zlo) * cy + (0 - ylo)) * cx + (0 - xlo);
        if(l2g) l2g[row] = giz * gnx * gny + giy * gnx + gix;
        if(hash)
        {
            // GenerateProblem.cpp:93-96,293-296
            const int h = ((ix & 1) << 2) | ((iy & 1) << 1) | (iz & 1);
            const int crd = iz * nx * ny + iy * (nx << 1) + (ix << 2);
            hash[row] = h * nx * ny * nz + crd;
        }
        if(b) b[row] = 26.0 - (n - 1.0);
    }
}

__global__ void k_f2c(int nxc, int nyc, int nzc, int nxf, int nyf, int* __restrict__ f2c, int* __restrict__ c2f)
{
    const int nc = nxc * nyc * nzc;
    const int ic = blockIdx.x * blockDim.x + threadIdx.x;
    if(ic >= nc) return;
    const int izc = ic / (nxc * nyc);
    const int iyc = ic / nxc - nyc * izc;
    const int ixc = ic - izc * nxc * nyc - iyc * nxc;
    const int f = (izc << 1) * nxf * nyf + (iyc << 1) * nxf + (ixc << 1);
    f2c[ic] = f;
    if(c2f) c2f[f] = ic;
}

// ------------------------------------------------------------ JPL coloring

// src/MultiColoring.cpp:151-236.  A neighbour whose colour is -1, c1 or c2 is
// compared by hash; that set is closed under this round's writes, so reading
// colors[] while other threads update it yields the same decisions as a
// snapshot (the reference relies on the same property).
__global__ void k_jpl_round(int m, const int* __restrict__ hash, int c1, int c2, const int* __restrict__ mtx_ind,
                            int* colors)
{
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if(row >= m) return;
    if(colors[row] != -1) return;
    const int rh = hash[row];
    bool is_max = true, is_min = true;
    const int* cols = mtx_ind + (size_t)row * kWidth;
#pragma unroll
    for(int p = 0; p < kWidth; ++p)
    {
        const int col = cols[p];
        if(col < 0 || col >= m || col == row) continue;
        const int cn = *((volatile int*)colors + col);
        if(cn == -1 || cn == c1 || cn == c2)
        {
            const int ch = hash[col];
            if(ch >= rh) is_max = false;
            if(ch <= rh) is_min = false;
        }
    }
    if(is_max) colors[row] = c1;
    else if(is_min) colors[row] = c2;
}

// Counts of colour value c1 and c2 over all rows (kernel_count_color_part1/2).
__global__ void k_count_two(int m, const int* __restrict__ colors, int c1, int c2, int* __restrict__ counts)
{
    __shared__ int red[32];
    int a = 0, b = 0;
    for(long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (long long)gridDim.x * blockDim.x)
    {
        const int c = colors[i];
        a += c == c1;
        b += c == c2;
    }
    a = block_sum(a, red);
    b = block_sum(b, red);
    if(threadIdx.x == 0)
    {
        atomicAdd(&counts[0], a);
        atomicAdd(&counts[1], b);
    }
}

// ------------------------------------------------- stable counting sort
constexpr int kSortThreads = 256;
constexpr int kSortTile = kSortThreads * 16;
constexpr int kMaxBins = 256;

__global__ void __launch_bounds__(kSortThreads)
    k_color_hist(int m, const int* __restrict__ colors, int mask, int nbins, int* __restrict__ counts)
{
    __shared__ int h[kMaxBins];
    for(int i = threadIdx.x; i < nbins; i += blockDim.x) h[i] = 0;
    __syncthreads();
    const int lo = blockIdx.x * kSortTile;
    const int hi = min(m, lo + kSortTile);
    for(int i = lo + threadIdx.x; i < hi; i += blockDim.x) atomicAdd(&h[colors[i] & mask], 1);
    __syncthreads();
    for(int i = threadIdx.x; i < nbins; i += blockDim.x) counts[(size_t)i * gridDim.x + blockIdx.x] = h[i];
}

// Exclusive scan of counts[nbins][G] (bin-major) in one block.
__global__ void __launch_bounds__(1024) k_color_scan(int n, int* __restrict__ counts)
{
    __shared__ int carry;
    __shared__ int wsum[32];
    if(threadIdx.x == 0) carry = 0;
    __syncthreads();
    for(int base = 0; base < n; base += blockDim.x)
    {
        const int i = base + threadIdx.x;
        const int v = i < n ? counts[i] : 0;
        // block inclusive scan
        int x = v;
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
        for(int o = 1; o < 32; o <<= 1)
        {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if(lane >= o) x += y;
        }
        if(lane == 31) wsum[warp] = x;
        __syncthreads();
        if(warp == 0)
        {
            int w = (lane < (int)(blockDim.x >> 5)) ? wsum[lane] : 0;
#pragma unroll
            for(int o = 1; o < 32; o <<= 1)
            {
                const int y = __shfl_up_sync(0xffffffffu, w, o);
                if(lane >= o) w += y;
            }
            wsum[lane] = w;
        }
        __syncthreads();
        const int incl = x + (warp > 0 ? wsum[warp - 1] : 0) + carry;
        if(i < n) counts[i] = incl - v;
        __syncthreads();
        if(threadIdx.x == blockDim.x - 1) carry = incl;
        __syncthreads();
    }
}

__global__ void k_bin_totals(int nbins, int G, const int* __restrict__ excl, int m, int* __restrict__ totals)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if(b >= nbins) return;
    const int start = excl[(size_t)b * G];
    const int end = (b + 1 < nbins) ? excl[(size_t)(b + 1) * G] : m;
    totals[b] = end - start;
}

// Stable scatter: rows of one tile are ranked in index order within the
// tile, tiles in index order across the grid (offsets from k_color_scan).
__global__ void __launch_bounds__(kSortThreads)
    k_color_scatter(int m, const int* __restrict__ colors, int mask, int nbins, const int* __restrict__ offsets,
                    int* __restrict__ perm)
{
    constexpr int kWarps = kSortThreads / 32;
    __shared__ int running[kMaxBins];
    __shared__ int wcount[kWarps][kMaxBins];
    for(int i = threadIdx.x; i < nbins; i += blockDim.x) running[i] = offsets[(size_t)i * gridDim.x + blockIdx.x];
    for(int i = threadIdx.x; i < kWarps * kMaxBins; i += blockDim.x) (&wcount[0][0])[i] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    const int lo = blockIdx.x * kSortTile;
    const int hi = min(m, lo + kSortTile);
    for(int base = lo; base < hi; base += blockDim.x)
    {
        const int i = base + threadIdx.x;
        const int key = i < hi ? (colors[i] & mask) : -1;
        const unsigned peers = __match_any_sync(0xffffffffu, key);
        const int rank = __popc(peers & lt);
        if(key >= 0 && rank == 0) wcount[warp][key] = __popc(peers);
        __syncthreads();
        if(key >= 0)
        {
            int before = 0;
            for(int w = 0; w < warp; ++w) before += wcount[w][key];
            perm[i] = running[key] + before + rank;
        }
        __syncthreads();
        for(int bn = threadIdx.x; bn < nbins; bn += blockDim.x)
        {
            int t = 0;
            for(int w = 0; w < kWarps; ++w)
            {
                t += wcount[w][bn];
                wcount[w][bn] = 0;
            }
            running[bn] += t;
        }
        __syncthreads();
    }
}

// glibc random_r TYPE_3 (additive feedback, r[i] = r[i-3] + r[i-31], output
// r >> 1, seeded by the Park-Miller LCG and 310 discarded outputs) -- the
// sequence rand() returns after srand(seed) on the reference's platform.
struct GlibcRand
{
    uint32_t state[344 + 4096];
    int n = 0;
    explicit GlibcRand(uint32_t seed)
    {
        int32_t s[344];
        s[0] = (int32_t)seed;
        for(int k = 1; k < 31; ++k)
        {
            const int64_t hi = s[k - 1] / 127773;
            const int64_t lo = s[k - 1] % 127773;
            int64_t w = 16807 * lo - 2836 * hi;
            if(w < 0) w += 2147483647;
            s[k] = (int32_t)w;
        }
        for(int k = 31; k < 34; ++k) s[k] = s[k - 31];
        for(int k = 34; k < 344; ++k) s[k] = (int32_t)((uint32_t)s[k - 31] + (uint32_t)s[k - 3]);
        for(int k = 0; k < 344; ++k) state[k] = (uint32_t)s[k];
        n = 344;
    }
    int next()
    {
        if(n >= 344 + 4096) return -1;
        state[n] = state[n - 31] + state[n - 3];
        const int out = (int)(state[n] >> 1);
        ++n;
        return out;
    }
};

}  // namespace hb

using namespace hb;

// ------------------------------------------------------------- C ABI

extern "C" int hpcgb200_rand_sequence(unsigned int seed, int n, int* out)
{
    HB_CHECK_ARG(n >= 0 && n <= 4096 && (n == 0 || out), "n in [0,4096] and out non-null");
    GlibcRand g(seed);
    for(int k = 0; k < n; ++k) out[k] = g.next();
    return 0;
}

extern "C" int hpcgb200_generate_problem(int nx, int ny, int nz, long long gnx, long long gny, long long gnz,
                                         long long gix0, long long giy0, long long giz0, int* mtx_ind,
                                         double* values, int8_t* nnz_in_row, int* diag_slot, long long* l2g,
                                         int* hash, double* b, void* stream)
{
    HB_CHECK_ARG(nx > 0 && ny > 0 && nz > 0, "grid dimensions must be positive");
    HB_CHECK_ARG((long long)nx * ny * nz <= 0x7fffffffLL, "local rows exceed int32 (local_int_t)");
    HB_CHECK_ARG(mtx_ind && values && nnz_in_row && diag_slot, "null output");
    const int m = nx * ny * nz;
    const long long threads = (long long)m * kWidth;
    const unsigned grid = (unsigned)((threads + kGenRows * kWidth - 1) / (kGenRows * kWidth));
    k_generate_problem<<<grid, kGenRows * kWidth, 0, as_stream(stream)>>>(
        m, nx, ny, nz, gnx, gny, gnz, gix0, giy0, giz0, mtx_ind, values, nnz_in_row, diag_slot, l2g, hash, b);
    HB_LAUNCHED();
    return 0;
}

extern "C" int hpcgb200_f2c_operator(int nxf, int nyf, int nzf, int* f2c, int* c2f, void* stream)
{
    HB_CHECK_ARG(nxf > 1 && nyf > 1 && nzf > 1 && nxf % 2 == 0 && nyf % 2 == 0 && nzf % 2 == 0,
                 "fine dimensions must be even (GenerateCoarseProblem.cpp:108-110)");
    HB_CHECK_ARG(f2c != nullptr, "null f2c");
    const int nxc = nxf / 2, nyc = nyf / 2, nzc = nzf / 2;
    const int nc = nxc * nyc * nzc;
    if(c2f) HB_CUDA(cudaMemsetAsync(c2f, 0xff, sizeof(int) * (size_t)nxf * nyf * nzf, as_stream(stream)));
    k_f2c<<<(nc + 255) / 256, 256, 0, as_stream(stream)>>>(nxc, nyc, nzc, nxf, nyf, f2c, c2f);
    HB_LAUNCHED();
    return 0;
}

static int sort_grid(int m) { return (m + kSortTile - 1) / kSortTile; }

extern "C" size_t hpcgb200_coloring_workspace_bytes(int m)
{
    const size_t G = (size_t)sort_grid(m > 0 ? m : 1);
    return 256 /* counters */ + sizeof(int) * (G * kMaxBins + kMaxBins);
}

extern "C" int hpcgb200_jpl_coloring(int m, const int* hash, const int* mtx_ind, int* colors, int* perm,
                                     int* nblocks_out, int* round_sizes, int* sizes, int* offsets, void* workspace,
                                     size_t workspace_bytes, void* stream)
{
    HB_CHECK_ARG(m > 0 && hash && mtx_ind && colors && perm && nblocks_out && sizes && offsets, "bad arguments");
    if(!workspace || workspace_bytes < hpcgb200_coloring_workspace_bytes(m))
        return record_error(HPCGB200_ERR_WORKSPACE, "hpcgb200_jpl_coloring: workspace too small");
    cudaStream_t s = as_stream(stream);
    int* d_counts = reinterpret_cast<int*>(workspace);
    HB_CUDA(cudaMemsetAsync(colors, 0xff, sizeof(int) * (size_t)m, s));

    GlibcRand rng(0x586744);  // srand(RNG_SEED), src/utils.hpp:47
    int nblocks = 0;
    long long colored = 0;
    int h_counts[2];
    std::vector<int> rsizes;
    int rounds = 0;
    const int block = 256;
    const int grid = (m + block - 1) / block;
    while(colored != m)
    {
        if(++rounds > HPCGB200_MAX_COLORS / 2)
            return record_error(HPCGB200_ERR_COLORING, "JPL coloring did not finish in %d rounds",
                                HPCGB200_MAX_COLORS / 2);
        const int c1 = (nblocks < 8) ? rng.next() % 8 : nblocks;
        const int c2 = (nblocks < 8) ? rng.next() % 8 : nblocks + 1;
        k_jpl_round<<<grid, block, 0, s>>>(m, hash, c1, c2, mtx_ind, colors);
        HB_LAUNCHED();
        HB_CUDA(cudaMemsetAsync(d_counts, 0, 2 * sizeof(int), s));
        k_count_two<<<min(grid, 1184), block, 0, s>>>(m, colors, c1, c2, d_counts);
        HB_LAUNCHED();
        HB_CUDA(cudaMemcpyAsync(h_counts, d_counts, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
        HB_CUDA(cudaStreamSynchronize(s));
        rsizes.push_back(h_counts[0]);
        rsizes.push_back(h_counts[1]);
        colored += h_counts[0];
        colored += h_counts[1];
        nblocks += 2;
    }
    *nblocks_out = nblocks;
    if(round_sizes)
        for(int i = 0; i < nblocks; ++i) round_sizes[i] = rsizes[i];

    // Stable sort of (color, row) on bits [0, 32 - clz(nblocks)) of the colour,
    // exactly the key range rocprim::radix_sort_pairs sees (MultiColoring.cpp:330-340).
    const int endbit = 32 - __builtin_clz((unsigned)nblocks);
    const int nbins = 1 << endbit;
    if(nbins > kMaxBins) return record_error(HPCGB200_ERR_COLORING, "too many colors (%d)", nblocks);
    const int mask = nbins - 1;
    const int G = sort_grid(m);
    int* d_tab = reinterpret_cast<int*>(reinterpret_cast<char*>(workspace) + 256);
    int* d_tot = d_tab + (size_t)G * kMaxBins;
    k_color_hist<<<G, kSortThreads, 0, s>>>(m, colors, mask, nbins, d_tab);
    HB_LAUNCHED();
    k_color_scan<<<1, 1024, 0, s>>>(nbins * G, d_tab);
    HB_LAUNCHED();
    k_bin_totals<<<(nbins + 255) / 256, 256, 0, s>>>(nbins, G, d_tab, m, d_tot);
    HB_LAUNCHED();
    k_color_scatter<<<G, kSortThreads, 0, s>>>(m, colors, mask, nbins, d_tab, perm);
    HB_LAUNCHED();
    std::vector<int> tot(nbins);
    HB_CUDA(cudaMemcpyAsync(tot.data(), d_tot, sizeof(int) * nbins, cudaMemcpyDeviceToHost, s));
    HB_CUDA(cudaStreamSynchronize(s));
    // Blocks of the sweeps = colour values 0 .. (largest used value).  For
    // grids with all dimensions even these equal the reference's round-order
    // sizes[] exactly; for odd dimensions the round order does not match the
    // sorted layout and the by-value sizes are the consistent choice.
    int used = 0;
    for(int bn = 0; bn < nbins; ++bn)
        if(tot[bn] > 0) used = bn + 1;
    if(used > HPCGB200_MAX_COLORS) return record_error(HPCGB200_ERR_COLORING, "too many colors");
    offsets[0] = 0;
    for(int c = 0; c < HPCGB200_MAX_COLORS; ++c)
    {
        sizes[c] = c < used ? tot[c] : 0;
        offsets[c + 1] = offsets[c] + sizes[c];
    }
    return 0;
}

namespace hb {

// PermuteColumns + ConvertToELL + PermuteRows in one pass (Permute.cpp:95-218,
// SparseMatrix.cpp:166-226).  Keys perm[col] of a row are distinct, so the
// output slot of an entry is its rank among the row's keys -- the same order
// the reference's bitonic network produces.  Pads go last with column -1.
__global__ void __launch_bounds__(128) k_build_ell(int m, const int* __restrict__ mtx_ind,
                                                   const double* __restrict__ values, const int* __restrict__ perm,
                                                   int* __restrict__ ell_col, double* __restrict__ ell_val)
{
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if(row >= m) return;
    int key[kWidth];
    const size_t base = (size_t)row * kWidth;
#pragma unroll
    for(int p = 0; p < kWidth; ++p)
    {
        const int col = mtx_ind[base + p];
        key[p] = (col >= 0 && col < m) ? perm[col] : 0x7fffffff;
    }
    const size_t prow = (size_t)perm[row];
    int nvalid = 0;
#pragma unroll
    for(int p = 0; p < kWidth; ++p)
    {
        if(key[p] == 0x7fffffff) continue;
        ++nvalid;
        int rank = 0;
#pragma unroll
        for(int q = 0; q < kWidth; ++q) rank += key[q] < key[p];
        ell_col[(size_t)rank * m + prow] = key[p];
        ell_val[(size_t)rank * m + prow] = values[base + p];
    }
    for(int p = nvalid; p < kWidth; ++p)
    {
        ell_col[(size_t)p * m + prow] = -1;
        ell_val[(size_t)p * m + prow] = 0.0;
    }
}

__global__ void k_extract_diagonal(int m, const int* __restrict__ ell_col, const double* __restrict__ ell_val,
                                   int* __restrict__ diag_idx, double* __restrict__ inv_diag, double* __restrict__ diag)
{
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if(row >= m) return;
    for(int p = 0; p < kWidth; ++p)
    {
        const size_t idx = (size_t)p * m + row;
        if(ell_col[idx] == row)
        {
            const double v = ell_val[idx];
            diag_idx[row] = p;
            inv_diag[row] = 1.0 / v;
            if(diag) diag[row] = v;
            break;
        }
    }
}

__global__ void k_permute(int m, const int* __restrict__ perm, const double* __restrict__ in, double* __restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i < m) out[perm[i]] = in[i];
}

__global__ void k_unpermute(int m, const int* __restrict__ perm, const double* __restrict__ in,
                            double* __restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i < m) out[i] = in[perm[i]];
}

// src/SparseMatrix.cpp:66-101: first slot whose column is the row; stops at a pad.
__global__ void k_copy_diagonal(int m, const int* __restrict__ ell_col, const double* __restrict__ ell_val,
                                double* __restrict__ diagonal)
{
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if(row >= m) return;
    for(int p = 0; p < kWidth; ++p)
    {
        const size_t idx = (size_t)p * m + row;
        const int col = ell_col[idx];
        if(col < 0 || col >= m) break;
        if(col == row)
        {
            diagonal[row] = ell_val[idx];
            break;
        }
    }
}

__global__ void k_replace_diagonal(int m, const double* __restrict__ diagonal, const int* __restrict__ ell_col,
                                   double* __restrict__ ell_val, double* __restrict__ inv_diag, double* __restrict__ diag)
{
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if(row >= m) return;
    const double d = diagonal[row];
    for(int p = 0; p < kWidth; ++p)
    {
        const size_t idx = (size_t)p * m + row;
        const int col = ell_col[idx];
        if(col < 0 || col >= m) break;
        if(col == row)
        {
            ell_val[idx] = d;
            break;
        }
    }
    inv_diag[row] = 1.0 / d;
    if(diag) diag[row] = d;
}

// src/TestCG.cpp:67-95 (kernel_scale_vector_values): TestCG's exaggerated
// diagonal.  Row i's scale comes from its global id l2g[i]: (gid + 2) * 1e6
// for the first nine global rows, 1e6 for all others.  TestCG runs it after
// OptimizeProblem, when rows are colour-permuted but l2g is not, so permuted
// row i takes the scale of natural row i -- kept as the reference does it.
__global__ void k_testcg_scale(int m, const long long* __restrict__ l2g, double* __restrict__ diagonal,
                               double* __restrict__ b)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= m) return;
    const long long gid = l2g[i];
    const double scale = gid < 9 ? (gid + 2) * 1.0e6 : 1.0e6;
    diagonal[i] *= scale;
    b[i] *= scale;
}

__global__ void k_transfer_indices(int nc, const int* __restrict__ f2c, const int* __restrict__ perm_f,
                                   const int* __restrict__ perm_c, int* __restrict__ inj_f, int* __restrict__ inj_c)
{
    const int ic = blockIdx.x * blockDim.x + threadIdx.x;
    if(ic >= nc) return;
    inj_f[ic] = perm_f[f2c[ic]];
    inj_c[ic] = perm_c[ic];
}

}  // namespace hb

static inline unsigned blocks_for(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

extern "C" int hpcgb200_build_ell(int m, const int* mtx_ind, const double* values, const int* perm, int* ell_col,
                                  double* ell_val, void* stream)
{
    HB_CHECK_ARG(m > 0 && mtx_ind && values && perm && ell_col && ell_val, "bad arguments");
    k_build_ell<<<blocks_for(m, 128), 128, 0, as_stream(stream)>>>(m, mtx_ind, values, perm, ell_col, ell_val);
    HB_LAUNCHED();
    return 0;
}

extern "C" int hpcgb200_extract_diagonal(int m, const int* ell_col, const double* ell_val, int* diag_idx,
                                         double* inv_diag, double* diag, void* stream)
{
    HB_CHECK_ARG(m > 0 && ell_col && ell_val && diag_idx && inv_diag, "bad arguments");
    k_extract_diagonal<<<blocks_for(m, 256), 256, 0, as_stream(stream)>>>(m, ell_col, ell_val, diag_idx, inv_diag,
                                                                          diag);
    HB_LAUNCHED();
    return 0;
}

extern "C" int hpcgb200_permute_vector(int m, const int* perm, const double* in, double* out, void* stream)
{
    HB_CHECK_ARG(m > 0 && perm && in && out && in != out, "bad arguments (in-place is not supported)");
    k_permute<<<blocks_for(m, 256), 256, 0, as_stream(stream)>>>(m, perm, in, out);
    HB_LAUNCHED();
    return 0;
}

extern "C" int hpcgb200_unpermute_vector(int m, const int* perm, const double* in, double* out, void* stream)
{
    HB_CHECK_ARG(m > 0 && perm && in && out && in != out, "bad arguments (in-place is not supported)");
    k_unpermute<<<blocks_for(m, 256), 256, 0, as_stream(stream)>>>(m, perm, in, out);
    HB_LAUNCHED();
    return 0;
}

extern "C" int hpcgb200_copy_diagonal(int m, const int* ell_col, const double* ell_val, double* diagonal, void* stream)
{
    HB_CHECK_ARG(m > 0 && ell_col && ell_val && diagonal, "bad arguments");
    k_copy_diagonal<<<blocks_for(m, 256), 256, 0, as_stream(stream)>>>(m, ell_col, ell_val, diagonal);
    HB_LAUNCHED();
    return 0;
}

extern "C" int hpcgb200_replace_diagonal(int m, const double* diagonal, const int* ell_col, double* ell_val,
                                         double* inv_diag, double* diag, void* stream)
{
    HB_CHECK_ARG(m > 0 && diagonal && ell_col && ell_val && inv_diag, "bad arguments");
    k_replace_diagonal<<<blocks_for(m, 256), 256, 0, as_stream(stream)>>>(m, diagonal, ell_col, ell_val, inv_diag,
                                                                         diag);
    HB_LAUNCHED();
    return 0;
}

extern "C" int hpcgb200_testcg_scale(int m, const long long* l2g, double* diagonal, double* b, void* stream)
{
    HB_CHECK_ARG(m > 0 && l2g && diagonal && b, "bad arguments");
    k_testcg_scale<<<blocks_for(m, 256), 256, 0, as_stream(stream)>>>(m, l2g, diagonal, b);
    HB_LAUNCHED();
    return 0;
}

extern "C" int hpcgb200_transfer_indices(int nc, const int* f2c, const int* perm_f, const int* perm_c, int* inj_f,
                                         int* inj_c, void* stream)
{
    HB_CHECK_ARG(nc > 0 && f2c && perm_f && perm_c && inj_f && inj_c, "bad arguments");
    k_transfer_indices<<<blocks_for(nc, 256), 256, 0, as_stream(stream)>>>(nc, f2c, perm_f, perm_c, inj_f, inj_c);
    HB_LAUNCHED();
    return 0;
}
