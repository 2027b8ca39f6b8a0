// Implicit-stencil kernels: the FP32 V-cycle of the mixed-precision path and
// the FP64 stencil SpMV of its outer CG.
//
// After the reference's JPL multicoloring of the HPCG grid every colour is
// one parity class (ix&1, iy&1, iz&1) and, because the colour sort is
// stable, the rows of a colour are that class in natural (z,y,x) order: a
// dense brick.  A row's neighbours are therefore computable from its
// position, and their ELL slot order (ascending permuted column) is fixed per
// colour: by neighbour colour, then by (dz,dy,dx).  The kernels walk that
// order, so their sums round exactly like an ELL sweep -- without reading any
// matrix data.  Off-diagonal values are the stencil's -1 (verified on the
// device before these paths are enabled); the diagonal stays an explicit
// array because TestCG rescales it.
//
// When all grid dimensions are even every brick has the same shape and the
// column offset of slot j of a colour-v row is a constant delta[v][j]; a
// 6-bit mask per row (which faces of the grid it touches) decides which
// neighbours exist.  Odd dimensions fall back to computing each neighbour's
// brick coordinates.
#pragma once

#include "cg.cuh"
#include "common.cuh"

namespace hb {

constexpr int kMaxStencilColors = 8;

struct StencilTab
{
    int delta[27];             // col - row of slot j (even grids)
    unsigned char bmask[27];   // boundary faces that remove slot j
    unsigned short nb[27];     // (dx+1) | (dy+1)<<2 | (dz+1)<<4 | colour<<8 (all grids)
    int dp;                    // slot of the diagonal
};

struct StencilLevel
{
    int nx, ny, nz, m;
    int ncolors;
    int even;                  // all dimensions even: deltas are constant
    int offsets[kMaxStencilColors + 1];
    int bx[kMaxStencilColors], by[kMaxStencilColors];
    int par[kMaxStencilColors];           // parity bits (ix&1)<<2 | (iy&1)<<1 | (iz&1) of colour v
    int color_of_par[8];
    int canon;                 // slot tables equal the compile-time ones of the canonical colouring
    StencilTab tab[kMaxStencilColors];
    int* status = nullptr;     // device word the TMA-staged passes set (3) when their copies time out (may be null)
};

// Builds the level description from the grid and the colour of each parity
// class; returns false when some parity class is empty or the colours are not
// a permutation of 0..7.
bool make_stencil_level(int nx, int ny, int nz, const int* offsets, const int color_of_par[8], StencilLevel* out);

// Counts (into *bad, device) rows where perm/ELL differ from the implicit
// stencil: permuted position, column order, off-diagonal value -1.
int launch_stencil_check(const StencilLevel& L, const int* perm, const int* ell_col, const double* ell_val, int* bad,
                         cudaStream_t s);

// diag32 = (float) a_ii, inv_diag32 = 1.0f / diag32.
int launch_diag32(int m, const double* diag, float* diag32, float* inv_diag32, cudaStream_t s);

// Zero-guess symmetric GS (forward colours 0..n-1, backward n-2..0).  When
// r64 is non-null the forward sweeps read the FP64 residual and also store
// its float value into r32 (fusing the down-conversion).
// pro: the prolongation into the finer level, fused into the passes that
// finalize rows (colour n-1's forward pass, every backward pass).
int launch32_symgs_zero(const StencilLevel& L, const float* diag32, const float* inv_diag32, const double* r64,
                        float* r32, float* x, cudaStream_t s, Prolong<float> pro = {});
// Full symmetric GS step.  When z64 is non-null every row's final value is
// also stored as double there (fusing the up-conversion).
int launch32_symgs(const StencilLevel& L, const float* inv_diag32, const float* r, float* x, double* z64,
                   cudaStream_t s, Prolong<float> pro = {});
// rc[inj_c[i]] = rf[inj_f[i]] - (A xf)[inj_f[i]].
int launch32_restrict(const StencilLevel& Lf, int nc, const int* inj_f, const int* inj_c, const float* diag32,
                      const float* rf, const float* xf, float* rc, cudaStream_t s);
// xf[inj_f[i]] += xc[inj_c[i]] (Lf: the fine level).
int launch32_prolong(const StencilLevel& Lf, int nc, const int* inj_f, const int* inj_c, const float* xc, float* xf,
                     cudaStream_t s);

// FP64 V-cycle pieces on the implicit stencil, bitwise equal to the ELL
// kernels (launch_symgs_zero, launch_symgs, launch_restrict, launch_prolong);
// they need stencil_vec4(L): every colour brick's x extent and offset a
// multiple of 4 (else HPCGB200_ERR_ARG).
bool stencil_vec4(const StencilLevel& L);
int launch64v_symgs_zero(const StencilLevel& L, const double* diag, const double* inv_diag, const double* r,
                         double* x, cudaStream_t s, Prolong<double> pro = {});
int launch64v_symgs(const StencilLevel& L, const double* inv_diag, const double* r, double* x, cudaStream_t s,
                    Prolong<double> pro = {});
int launch64v_restrict(const StencilLevel& Lf, int nc, const int* inj_c, const double* diag, const double* rf,
                       const double* xf, double* rc, cudaStream_t s);
int launch64v_prolong(const StencilLevel& Lf, int nc, const int* inj_c, const double* xc, double* xf, cudaStream_t s);

// FP64 y = A x on the implicit stencil (bitwise equal to the ELL SpMV: same
// slot order, fma(-1, x, s) == s - x, fma(a_ii, x_i, s) on the diagonal).
int launch64_spmv_stencil(const StencilLevel& L, const double* diag, const double* x, double* y, cudaStream_t s);
// The mixed path's outer operator: y = A x in FP64 with the 27 terms summed
// as a separable box (x sums, y sums, z sums) -- equal to the ELL product to
// FP64 rounding, not bit for bit; 7 shared-memory reads per row instead of 27.
int launch64_spmv_sep(const StencilLevel& L, const double* diag, const double* x, double* y, cudaStream_t s);
// The separable product fused with p.Ap and alpha = rtz / pAp (the CG step of
// k_cg_spmv_pap) for the mixed and learned paths; one partial sum per block in
// `partial` (stencil_pap_partials(L) entries), `ticket` must start at zero and
// is left at zero.
size_t stencil_pap_partials(const StencilLevel& L);
// Step 1 of the two-kernel CG step (launch_cg_step1_ell) with the separable
// product, for the FP32 V-cycles' output z; canonical colouring only.
int launch_cg_step1_sep(const StencilLevel& L, const double* diag, const double* r, const float* z, double* p,
                        double* x, double* Ap, CGState* st, ReduceScratch* ws, GridBarrier* gb, cudaStream_t s);
int launch64_cg_spmv_pap_stencil(const StencilLevel& L, const double* diag, const double* p, double* Ap,
                                 CGState* st, double* partial, unsigned int* ticket, cudaStream_t s);

}  // namespace hb
