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

int launch_spmv(int m, const ColorChunks& cc, const int* ell_col, const double* ell_val, const double* x, double* y,
                cudaStream_t s);
// pro: the prolongation into the finer level fused into the passes that
// finalize rows (used on coarse levels; empty by default).
int launch_symgs(int m, int nblocks, int ublocks, const int* sizes, const int* offsets, const int* ell_col,
                 const double* ell_val, const double* inv_diag, const double* r, double* x, cudaStream_t s,
                 Prolong<double> pro = {});
int launch_symgs_zero(int m, int nblocks, int ublocks, const int* sizes, const int* offsets, const int* ell_col,
                      const double* ell_val, const int* diag_idx, const double* diag, const double* inv_diag,
                      const double* r, double* x, cudaStream_t s, Prolong<double> pro = {});
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
