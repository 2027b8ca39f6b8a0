/*
 * CPU restatement of rocHPCG's OPTIMIZED (multicolored, permuted, ELL) path.
 * TEST INFRASTRUCTURE ONLY: used by tests/ and bench.py's CPU leg as the
 * checker for the CUDA kernels; the product library never links it.
 *
 * Every function cites the reference kernel it restates (paths relative to
 * the rocHPCG source tree).  Floating-point kernels keep the reference
 * kernel's operation order and use fma() where the reference uses fma(), so
 * row-wise results are bit-identical to a device kernel that does the same;
 * only reductions (dot products) differ in summation order.
 */
#ifndef HPCG_ORACLE_COLORED_H
#define HPCG_ORACLE_COLORED_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* GenerateProblem.cpp:98-303 (kernel_generate_problem) + SetupHalo.cpp:107-131
 * (kernel_copy_indices, 1 rank).  Row-major 27 slots in (dz,dy,dx) order,
 * boundary rows compacted; unused slots: col -1, value 0.0. */
void oc_generate(int nx, int ny, int nz, int* cols, double* vals, int8_t* nnz_in_row,
                 int* diag_slot, int* hash, double* b);

/* GenerateCoarseProblem.cpp:57-86 (kernel_f2c_operator). */
void oc_f2c(int nxf, int nyf, int nzf, int* f2c);

/* MultiColoring.cpp:151-236,238-316 (kernel_jpl + JPLColoring round loop),
 * with the host rand() sequence after srand(0x586744).  colors[m] out;
 * round_sizes[] gets the reference's per-round counts (sizes[] in round order);
 * returns nblocks (2 per round) or -1 if it does not terminate in 64 rounds. */
int oc_jpl_coloring(int m, const int* cols, const int8_t* nnz_in_row, const int* hash, int* colors,
                    int* round_colors, int* round_sizes);

/* MultiColoring.cpp:318-344: stable sort of (color, row) by color value and
 * perm[sorted[i]] = i.  sizes/offsets receive the by-value histogram. */
void oc_color_perm(int m, const int* colors, int ncolors, int* perm, int* sizes, int* offsets);

/* Permute.cpp:95-185 (kernel_perm_cols), SparseMatrix.cpp:166-226,271-359
 * (ConvertToELL), Permute.cpp:54-76,187-218 (PermuteRows),
 * SparseMatrix.cpp:361-389 (ExtractDiagonal).  Column-major ELL of width 27,
 * slot index p*m + row. */
void oc_build_ell(int m, const int* cols, const double* vals, const int* perm, int* ell_col,
                  double* ell_val, int* diag_idx, double* inv_diag);

/* Permute.cpp:220-235: out[perm[i]] = in[i]. */
void oc_permute_vector(int m, const int* perm, const double* in, double* out);

/* ComputeSPMV.cpp:130-170 (kernel_spmv_ell). */
void oc_spmv(int m, const int* ell_col, const double* ell_val, const double* x, double* y);

/* ComputeSYMGS.cpp:113-151,369-404 (kernel_symgs_sweep: colors 0..nblocks-1
 * then ublocks..0). */
void oc_symgs(int m, int nblocks, int ublocks, const int* sizes, const int* offsets, const int* ell_col,
              const double* ell_val, const double* inv_diag, const double* r, double* x);

/* ComputeSYMGS.cpp:238-341,406-454 (pointwise_mult, forward_sweep_0,
 * backward_sweep_0). */
void oc_symgs_zero(int m, int nblocks, int ublocks, const int* sizes, const int* offsets, const int* ell_col,
                   const double* ell_val, const int* diag_idx, const double* r, double* x);

/* ComputeRestriction.cpp:81-124 (kernel_fused_restrict_spmv). */
void oc_restrict_fused(int nc, const int* f2c, const int* perm_f, const int* perm_c, int mf, const int* ell_col,
                       const double* ell_val, const double* rf, const double* xf, double* rc);

/* ComputeProlongation.cpp:39-59 (kernel_prolongation). */
void oc_prolong(int nc, const int* f2c, const int* perm_f, const int* perm_c, const double* xc, double* xf);

/* Deterministic dot product (fixed 4096-element blocks, summed in order). */
double oc_dot(int n, const double* x, const double* y);

/* One level of the MG hierarchy as the optimized path holds it. */
typedef struct
{
    int m;
    int nblocks, ublocks;
    const int* sizes;
    const int* offsets;
    const int* ell_col;
    const double* ell_val;
    const int* diag_idx;
    const double* inv_diag;
    /* to next level (NULL on the coarsest) */
    int nc;
    const int* f2c;
    const int* perm;     /* this level's perm */
    const int* perm_c;   /* next level's perm */
    double* rc;          /* next level's residual, length nc */
    double* xc;          /* next level's solution, length nc */
} oc_level;

/* ComputeMG.cpp:64-102 over levels[0..nlevels). */
void oc_mg(const oc_level* levels, int nlevels, const double* r, double* x);

/* CG.cpp:104-200 (non-HPCG_REFERENCE branch) on the permuted system.
 * Work vectors are allocated internally.  normr_hist (optional, length
 * max_iter+1) receives normr after the preamble and after every iteration. */
int oc_cg(const oc_level* levels, int nlevels, const double* b, double* x, int max_iter, double tol,
          int precond, int* niters, double* normr, double* normr0, double* normr_hist);

/* ---- FP32 V-cycle restatement (mixed-precision preconditioner) ----------
 * Same kernels with float vectors, float accumulation and float matrix
 * values (26/-1 are exact in any format), diagonal reciprocal in float. */
void oc_mg_f32(const oc_level* levels, int nlevels, const float* r, float* x);

#ifdef __cplusplus
}
#endif
#endif
