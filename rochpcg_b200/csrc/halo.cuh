// Kernels of the decomposed problem: the halo parts of the operators, the
// send-buffer gather, set-up of the external columns, and the CG vector
// updates whose scalars come from device memory (after the cross-rank sums).
#pragma once

#include "common.cuh"

namespace hb {

// Device-resident scalars of a decomposed CG solve (one array per rank).
enum DistSlot
{
    kDistRtz = 0,     // r.z of the previous iteration (beta's denominator)
    kDistRtzNew = 1,  // r.z of this iteration (summed over ranks)
    kDistPap = 2,     // p.Ap (summed over ranks)
    kDistRr = 3,      // r.r (summed over ranks)
    kDistSlots = 8
};

constexpr int kMaxGroup = 64;  // ranks one process can drive together

struct SlotPtrs
{
    double* p[kMaxGroup];
};

// buf[i] = x[send_perm[i]] (src/ExchangeHalo.cpp:148-186, kernel_gather with
// the permutation folded into send_perm at set-up).
int launch_halo_pack(int n, const int* send_perm, const double* x, double* buf, cudaStream_t s);
// y[prow[h]] += sum_p hval x[hcol] (src/ComputeSPMV.cpp:172-208, kernel_spmv_halo).
int launch_halo_spmv(int nh, int hw, const int* prow, const int* hcol, const double* hval, const double* x,
                     double* y, cudaStream_t s);
// Colour-0 rows: y = fma(-sum_p hval y[hcol], inv_diag, y)
// (src/ComputeSYMGS.cpp:190-236, kernel_symgs_halo).
int launch_halo_symgs0(int nh, int hw, const int* prow, const int* hcol, const double* hval,
                       const double* inv_diag, int size0, double* y, cudaStream_t s);
// Injected rows: rc[pc] -= sum_p hval xf[hcol]
// (src/ComputeRestriction.cpp:126-167, kernel_fused_restrict_spmv_halo).
int launch_halo_restrict(int nh, int hw, const int* pc, const int* hcol, const double* hval, const double* xf,
                         double* rc, cudaStream_t s);

// out[i] = in[i] >= 0 ? perm[in[i]] : -1.
int launch_map_perm(int n, const int* in, const int* perm, int* out, cudaStream_t s);
// Writes each halo row's external columns (value -1, the generated
// off-diagonal) into the ELL slots after its local ones, fills the compact
// halo arrays (prow, column-major hcol/hval of width hw) and, when b is given,
// lowers b by the row's external count (b = 27 - nonzeros, the generated
// right-hand side for an exact solution of ones).  *status: 1 if a row has
// more than 27 entries, 2 if its ELL padding was not empty.
int launch_halo_insert(int nh, int hw, int m, const int* halo_rows, const int* halo_ptr, const int* halo_cols,
                       const int* perm, int* ell_col, double* ell_val, int* prow, int* hcol, double* hval, double* b,
                       int* status, cudaStream_t s);

// Sum of *p[0..n) in rank order, stored back to every p[r] (the cross-rank
// sum of ranks that one process drives on one device).
int launch_group_sum(int n, const SlotPtrs& ptrs, cudaStream_t s);

// p = z (first) or z + beta p with beta = sc[RtzNew] / sc[Rtz] (src/CG.cpp:
// 143-156, WAXPBY(1, z, beta, p)).
int launch_dist_update_p(int n, int first, const double* z, double* p, const double* sc, cudaStream_t s);
// alpha = sc[RtzNew] / sc[Pap]; r -= alpha Ap, x += alpha p, sc[Rr] = r.r
// (this rank's rows; deterministic); sc[Rtz] = sc[RtzNew] for the next beta
// (src/CG.cpp:161-176).
int launch_dist_update_xr(int n, const double* p, const double* Ap, double* x, double* r, double* sc,
                          ReduceScratch* ws, cudaStream_t s);
// r = b - Ax (WAXPBY(1, b, -1, Ax)), sc[Rr] = r.r (src/CG.cpp:129-133).
int launch_dist_residual(int n, const double* b, const double* Ax, double* r, double* sc, ReduceScratch* ws,
                         cudaStream_t s);

}  // namespace hb
