// Reference kernels in natural row order on the generated row-major arrays:
// the arithmetic of the benchmark's `_ref` routines (src/ComputeSPMV_ref.cpp,
// src/ComputeSYMGS_ref.cpp, src/ComputeRestriction_ref.cpp,
// src/ComputeProlongation_ref.cpp, src/ComputeWAXPBY_ref.cpp,
// src/ComputeDotProduct_ref.cpp) on the device.  The benchmark driver runs
// them before OptimizeProblem for the reference timing phase and for the
// 50-iteration reference residual (src/main.cpp:288-341).
#pragma once

#include "common.cuh"

namespace hb {

// One MG level as GenerateProblem leaves it: row i = (iz*ny + iy)*nx + ix,
// 27 slots per row in (dz, dy, dx) order, pads (column -1) at the end.
struct NaturalLevel
{
    int nx, ny, nz;
    const int* ind;           // [m][27] column ids
    const double* val;        // [m][27] values
    const int8_t* nnz;        // nonzeros per row
    const int* diag_slot;     // slot of a_ii in its row
    __host__ __device__ long long rows() const { return (long long)nx * ny * nz; }
};

// Wavefronts of the natural-order Gauss-Seidel sweep: t = ix + 2 iy + 4 iz.
// Every stencil neighbour that precedes a row in natural order has a smaller
// t and every one that follows has a larger t, so sweeping t upwards
// (forward) or downwards (backward), one launch per t, reads exactly the
// values the sequential sweep reads.
__host__ __device__ inline int natural_fronts(int nx, int ny, int nz) { return (nx - 1) + 2 * (ny - 1) + 4 * (nz - 1) + 1; }

// y = A x (sum += a*x, products and sums rounded separately).
int launch_nat_spmv(const NaturalLevel& L, const double* x, double* y, cudaStream_t s);
// One symmetric Gauss-Seidel step in natural order (forward then backward).
int launch_nat_symgs(const NaturalLevel& L, const double* r, double* x, cudaStream_t s);
// rc[i] = rf[f2c[i]] - Axf[f2c[i]].
int launch_nat_restrict(int nc, const int* f2c, const double* rf, const double* axf, double* rc, cudaStream_t s);
// xf[f2c[i]] += xc[i].
int launch_nat_prolong(int nc, const int* f2c, const double* xc, double* xf, cudaStream_t s);
// w = alpha x + beta y with the three forms of src/ComputeWAXPBY_ref.cpp:65-85.
int launch_nat_waxpby(int n, double alpha, const double* x, double beta, const double* y, double* w, cudaStream_t s);
// *result = sum x_i*y_i (products rounded, then summed in a fixed order).
int launch_nat_dot(int n, const double* x, const double* y, ReduceScratch* ws, double* result, cudaStream_t s);

// CheckProblem (src/CheckProblem.cpp:79-150) as a count instead of asserts:
// every row's columns, values, nonzero count and diagonal slot against the
// 27-point stencil on the global grid; b = 26 - (nnz - 1), x = 0 and
// xexact = 1 where given; local-to-global ids where given.  Adds the number
// of mismatching rows to *bad and the row nonzeros to *nnz_total.
int launch_nat_check(const NaturalLevel& L, long long gnx, long long gny, long long gnz, long long gix0,
                     long long giy0, long long giz0, const long long* l2g, const double* b, const double* x,
                     const double* xexact, unsigned long long* bad, unsigned long long* nnz_total, cudaStream_t s);

}  // namespace hb
