// Internal launch interface of the FP64 operators (used by the C ABI and by
// the C++ host layer, which captures them into CUDA graphs).
#pragma once

#include "common.cuh"

namespace hb {

constexpr int kBS = 256;            // threads per block of the row kernels
constexpr int kMaxMapColors = 16;   // colours the interleaved SpMV map handles

// Colour-interleaved chunk map for the SpMV: chunk b covers rows
// [offsets[c] + k*kBS, ...) of colour c = b % ncolors, k = b / ncolors.
struct ColorChunks
{
    int ncolors;
    int per_color;
    int offsets[kMaxMapColors + 1];

    __host__ __device__ int nchunks() const { return ncolors * per_color; }
    __device__ __forceinline__ bool row_of(int chunk, int tid, int& row) const
    {
        const int c = chunk % ncolors;
        const int k = chunk / ncolors;
        row = offsets[c] + k * kBS + tid;
        return row < offsets[c + 1];
    }
};

ColorChunks make_chunks(int m, int ncolors, const int* offsets);

// ------------------------------------------------------------ row kernel core

// sum <- fma(s * a_p, x[col_p], sum) over the ELL slots p in [p_lo, p_hi) of
// `row`, in slot order, for the columns with use_col(col).  The slots are
// processed 9 at a time: the column/value loads of a group are issued
// together (predicated), then its gathers, then its fmas, so a row costs 2
// dependent memory round trips per group instead of 2 per slot.  Every group
// is issued, predicated, even when none of its slots is in the range: skipping
// such groups (the zero-guess sweeps need only the slots before or after the
// diagonal) with a branch measured slower (256^3 zero-guess SymGS 1.312 vs
// 1.288 ms), the branch keeping the loads of the next group from starting
// while the current one's fmas wait.
//
// [GLO, GHI) bounds the groups at compile time: a caller that knows every row
// of its launch needs only some groups (the zero-guess sweeps of a colour, from
// the colour's extreme diagonal positions) issues no instructions for the
// others; the sum is the same, since the groups left out hold no slot of the
// range.
template <int GLO = 0, int GHI = kWidth / 9, typename ColPred>
__device__ __forceinline__ double ell_row_sum(int m, int row, const int* __restrict__ ell_col,
                                              const double* __restrict__ ell_val, const double* x, double sum,
                                              double s, int p_lo, int p_hi, ColPred use_col)
{
    constexpr int G = 9;
    static_assert(kWidth == 3 * G && 0 <= GLO && GLO <= GHI && GHI <= 3, "group range");
#pragma unroll
    for(int g = GLO * G; g < GHI * G; g += G)
    {
        int col[G];
        double v[G], xv[G];
#pragma unroll
        for(int q = 0; q < G; ++q)
        {
            const int p = g + q;
            const size_t idx = (size_t)p * m + row;
            const bool u = p >= p_lo && p < p_hi;
            col[q] = u ? ld_stream(ell_col + idx) : -1;
            v[q] = u ? ld_stream(ell_val + idx) : 0.0;
        }
#pragma unroll
        for(int q = 0; q < G; ++q) xv[q] = use_col(col[q]) ? x[col[q]] : 0.0;
#pragma unroll
        for(int q = 0; q < G; ++q)
            if(use_col(col[q])) sum = fma(s * v[q], xv[q], sum);
    }
    return sum;
}

// y_row = sum over the row's slots of a_p x[col_p] (src/ComputeSPMV.cpp:130-170).
__device__ __forceinline__ double spmv_row(int m, int row, const int* __restrict__ ell_col,
                                           const double* __restrict__ ell_val, const double* __restrict__ x)
{
    return ell_row_sum(m, row, ell_col, ell_val, x, 0.0, 1.0, 0, kWidth,
                       [m](int col) { return col >= 0 && col < m; });
}

int launch_spmv(int m, const ColorChunks& cc, const int* ell_col, const double* ell_val, const double* x, double* y,
                cudaStream_t s);
// pro: the prolongation into the finer level fused into the passes that
// finalize rows (used on coarse levels; empty by default).
int launch_symgs(int m, int nblocks, int ublocks, const int* sizes, const int* offsets, const int* ell_col,
                 const double* ell_val, const double* inv_diag, const double* r, double* x, cudaStream_t s,
                 Prolong<double> pro = {});
// One colour of kernel_symgs_sweep with the columns below ncols (the
// decomposed problem's sweeps; launch_symgs uses ncols = m).
int launch_sweep_color(int m, int ncols, int size, int offset, const int* ell_col, const double* ell_val,
                       const double* inv_diag, const double* r, double* x, cudaStream_t s);
// Groups of 9 ELL slots a colour's zero-guess passes need: the forward pass
// groups [0, fhi) (slots before the diagonal), the backward pass [blo, 3).
struct ZgGroups
{
    int fhi = 3;
    int blo = 0;
};
// zg (one entry per colour, optional) narrows each colour's group range.
int launch_symgs_zero(int m, int nblocks, int ublocks, const int* sizes, const int* offsets, const int* ell_col,
                      const double* ell_val, const int* diag_idx, const double* diag, const double* inv_diag,
                      const double* r, double* x, cudaStream_t s, Prolong<double> pro = {},
                      const ZgGroups* zg = nullptr);
// The group ranges of colours [0, nblocks) from their rows' diagonal slots
// (synchronizes the stream).
int zero_guess_groups(int m, int nblocks, const int* offsets, const int* diag_idx, ZgGroups* zg, cudaStream_t s);
// pro_f[inj_c[ic]] = inj_f[ic]: coarse permuted row -> injected fine permuted row.
int launch_prolong_map(int nc, const int* inj_f, const int* inj_c, int* pro_f, cudaStream_t s);
int launch_restrict(int nc, const int* inj_f, const int* inj_c, int mf, const int* ell_col, const double* ell_val,
                    const double* rf, const double* xf, double* rc, cudaStream_t s);
int launch_restrict_axf(int nc, const int* inj_f, const int* inj_c, const double* rf, const double* axf, double* rc,
                        cudaStream_t s);
int launch_prolong(int nc, const int* inj_f, const int* inj_c, const double* xc, double* xf, cudaStream_t s);
int launch_dot(int n, const double* x, const double* y, ReduceScratch* ws, double* result, cudaStream_t s);
int launch_waxpby(int n, double alpha, const double* x, double beta, const double* y, double* w, cudaStream_t s);
int launch_waxpby_dot(int n, double alpha, const double* x, double* y, ReduceScratch* ws, double* result,
                      cudaStream_t s);
int launch_residual_inf(int n, const double* v1, const double* v2, ReduceScratch* ws, double* result, cudaStream_t s);

}  // namespace hb
