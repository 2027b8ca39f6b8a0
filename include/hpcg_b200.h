/*
 * hpcg_b200.h -- C ABI of libhpcgb200.so, the B200 (sm_100a) implementation of
 * HPCG's multigrid-preconditioned conjugate-gradient hot path.
 *
 * Two layers are exported:
 *
 *  1. Kernel entry points (hpcgb200_spmv, hpcgb200_symgs, ...): plain device
 *     pointers, sizes and a cudaStream_t passed as void*.  They replace the
 *     device side of the reference operators named in each comment (paths are
 *     relative to the rocHPCG source tree).  None of them allocates; scratch
 *     space for reductions is passed in by the caller.
 *  2. Problem entry points (hpcgb200_problem_*): an opaque handle that owns a
 *     generated + optimized 4-level hierarchy and runs the reference's
 *     protocol pieces (CG, TestCG, TestSymmetry) on it.  The C++ operator API
 *     with the reference's signatures (CG, ComputeSPMV, ComputeMG, ...) is in
 *     rochpcg_b200/host/hpcg.hpp and is what C++ callers link against.
 *
 * Index conventions: local_int_t is int32 (src/Geometry.hpp:29); ELL storage
 * is column-major with slot p of row i at p*m + i (64-bit offset), width 27;
 * pad slots hold column -1.  After optimization every vector is in the
 * color-permuted order perm[] defines (new = perm[old]).
 *
 * Every function returns 0 on success or one of the HPCGB200_ERR_* codes; it
 * never exits the process.  hpcgb200_last_error() describes the last failure.
 */
#ifndef HPCG_B200_H
#define HPCG_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HPCGB200_OK 0
#define HPCGB200_ERR_ARG 1            /* invalid argument / size */
#define HPCGB200_ERR_CUDA 2           /* CUDA runtime error */
#define HPCGB200_ERR_COLORING 3       /* multicoloring did not terminate */
#define HPCGB200_ERR_WORKSPACE 4      /* workspace too small */
#define HPCGB200_ERR_NOT_STENCIL 5    /* matrix is not the 27-point HPCG stencil (implicit paths) */
#define HPCGB200_ERR_DEVICE_STATUS 6  /* a device-side check failed (status word set) */
#define HPCGB200_ERR_NO_DEVICE 7      /* no CUDA device visible */
#define HPCGB200_ERR_NONFINITE 8      /* a solve ended with a non-finite residual (outputs are filled) */
#define HPCGB200_ERR_COMM 9           /* communication between ranks failed or timed out */

#define HPCGB200_WIDTH 27
#define HPCGB200_MAX_COLORS 128       /* src/utils.hpp:48 */

/* ----------------------------------------------------------------- misc */

/* Text of the last error recorded by this thread. */
const char* hpcgb200_last_error(void);
/* Library version string. */
const char* hpcgb200_version(void);
/* Binds the library's runtime (stream, reduction scratch) to CUDA device
 * `device` (< 0: the current device) -- the reference driver's --dev=
 * (src/init.cpp:196-214 selects the HIP device for one rank).  Call it before
 * any other entry point; once bound, a different device is refused
 * (HPCGB200_ERR_ARG), the same one is a no-op.  HPCGB200_ERR_NO_DEVICE
 * without a device, HPCGB200_ERR_ARG for an index out of range. */
int hpcgb200_init(int device);
/* Bytes of caller-provided scratch the reduction entry points need. */
size_t hpcgb200_reduction_workspace_bytes(void);
/* The first n values rand() returns after srand(seed) with glibc's
 * generator (n <= 4096); the colouring draws its colour pairs from this
 * sequence with seed 0x586744 (src/MultiColoring.cpp:259,283-284). */
int hpcgb200_rand_sequence(unsigned int seed, int n, int* out);

/* ------------------------------------------------ problem construction
 * src/GenerateProblem.cpp:98-303 (kernel_generate_problem) + src/SetupHalo.cpp:
 * 107-131 (kernel_copy_indices, 1 rank).  Row-major 27 slots per row in
 * (dz,dy,dx) order, boundary rows compacted.  mtx_ind gets LOCAL column ids
 * (1 rank: global == local), pads -1; values pads 0.  l2g, hash, b may be NULL. */
int hpcgb200_generate_problem(int nx, int ny, int nz, long long gnx, long long gny, long long gnz,
                              long long gix0, long long giy0, long long giz0, int* mtx_ind, double* values,
                              int8_t* nnz_in_row, int* diag_slot, long long* l2g, int* hash, double* b,
                              void* stream);

/* src/GenerateCoarseProblem.cpp:57-86 (kernel_f2c_operator); c2f (length nxf*nyf*nzf,
 * -1 where no coarse point) may be NULL. */
int hpcgb200_f2c_operator(int nxf, int nyf, int nzf, int* f2c, int* c2f, void* stream);

/* src/MultiColoring.cpp:238-353 (JPLColoring): Jones-Plassmann-Luby rounds
 * with (c1,c2) = rand()%8 after srand(0x586744) (glibc sequence, generated
 * internally so the process's rand() state is untouched), then a stable
 * counting sort by color (replacing rocPRIM radix_sort_pairs on
 * [0, 32-clz(nblocks)) bits) and perm[sorted[i]] = i.
 * Outputs: colors[m], perm[m] (device); *nblocks, round_sizes[nblocks] (the
 * reference's per-round counts), sizes[] / offsets[] (host, by color value,
 * HPCGB200_MAX_COLORS / +1 entries).  workspace: >= hpcgb200_coloring_workspace_bytes(m). */
size_t hpcgb200_coloring_workspace_bytes(int m);
int hpcgb200_jpl_coloring(int m, const int* hash, const int* mtx_ind, int* colors, int* perm, int* nblocks,
                          int* round_sizes, int* sizes, int* offsets, void* workspace, size_t workspace_bytes,
                          void* stream);

/* src/Permute.cpp:95-185 (PermuteColumns) + src/SparseMatrix.cpp:271-359
 * (ConvertToELL) + src/Permute.cpp:187-218 (PermuteRows) in one pass:
 * ell_col[p*m + perm[i]] = p-th smallest perm[col] of natural row i. */
int hpcgb200_build_ell(int m, const int* mtx_ind, const double* values, const int* perm, int* ell_col,
                       double* ell_val, void* stream);

/* src/SparseMatrix.cpp:361-407 (ExtractDiagonal); diag (may be NULL) also gets a_ii. */
int hpcgb200_extract_diagonal(int m, const int* ell_col, const double* ell_val, int* diag_idx, double* inv_diag,
                              double* diag, void* stream);

/* src/Permute.cpp:220-246 (PermuteVector): out[perm[i]] = in[i]. */
int hpcgb200_permute_vector(int m, const int* perm, const double* in, double* out, void* stream);

/* Inverse of the above: out[i] = in[perm[i]] (natural order from permuted). */
int hpcgb200_unpermute_vector(int m, const int* perm, const double* in, double* out, void* stream);

/* src/SparseMatrix.cpp:66-101 (HIPCopyMatrixDiagonal): diagonal[i] = a_ii. */
int hpcgb200_copy_diagonal(int m, const int* ell_col, const double* ell_val, double* diagonal, void* stream);

/* src/SparseMatrix.cpp:103-150 (HIPReplaceMatrixDiagonal): a_ii = diagonal[i],
 * inv_diag = 1/a_ii; diag (may be NULL) mirrors a_ii. */
int hpcgb200_replace_diagonal(int m, const double* diagonal, const int* ell_col, double* ell_val,
                              double* inv_diag, double* diag, void* stream);

/* src/TestCG.cpp:67-95 (kernel_scale_vector_values): TestCG's diagonal
 * exaggeration, diagonal[i] and b[i] scaled by (gid + 2) * 1e6 where
 * gid = l2g[i] < 9, else by 1e6 (l2g: the level's local-to-global map). */
int hpcgb200_testcg_scale(int m, const long long* l2g, double* diagonal, double* b, void* stream);

/* Multigrid transfer indices: inj_f[ic] = perm_f[f2c[ic]], inj_c[ic] = perm_c[ic]
 * (the two gathers src/ComputeRestriction.cpp:100-102 and
 * src/ComputeProlongation.cpp:53-56 do per call, done once). */
int hpcgb200_transfer_indices(int nc, const int* f2c, const int* perm_f, const int* perm_c, int* inj_f,
                              int* inj_c, void* stream);

/* ------------------------------------------------------- FP64 operators */

/* src/ComputeSPMV.cpp:130-170,226-278 (kernel_spmv_ell): y = A x. */
int hpcgb200_spmv(int m, const int* ell_col, const double* ell_val, const double* x, double* y, void* stream);

/* src/ComputeSYMGS.cpp:113-151,369-404: one symmetric multicolor Gauss-Seidel
 * step (colors 0..nblocks-1, then ublocks..0).  sizes/offsets are HOST arrays. */
int hpcgb200_symgs(int m, int nblocks, int ublocks, const int* sizes, const int* offsets, const int* ell_col,
                   const double* ell_val, const double* inv_diag, const double* r, double* x, void* stream);

/* src/ComputeSYMGS.cpp:238-341,406-454 (ComputeSYMGSZeroGuess): the same step
 * from x = 0 without reading x; diag/inv_diag are a_ii and 1/a_ii. */
int hpcgb200_symgs_zero(int m, int nblocks, int ublocks, const int* sizes, const int* offsets,
                        const int* ell_col, const double* ell_val, const int* diag_idx, const double* diag,
                        const double* inv_diag, const double* r, double* x, void* stream);

/* src/ComputeRestriction.cpp:81-124,199-237 (ComputeFusedSpMVRestriction):
 * rc[inj_c[i]] = rf[inj_f[i]] - (A xf)[inj_f[i]]. */
int hpcgb200_restrict_fused(int nc, const int* inj_f, const int* inj_c, int mf, const int* ell_col,
                            const double* ell_val, const double* rf, const double* xf, double* rc, void* stream);

/* src/ComputeRestriction.cpp:59-79,182-197 (ComputeRestriction, the
 * HPCG_REFERENCE form that reads a precomputed Axf = A xf):
 * rc[inj_c[i]] = rf[inj_f[i]] - axf[inj_f[i]]. */
int hpcgb200_restrict(int nc, const int* inj_f, const int* inj_c, const double* rf, const double* axf, double* rc,
                      void* stream);

/* src/ComputeProlongation.cpp:39-86: xf[inj_f[i]] += xc[inj_c[i]]. */
int hpcgb200_prolong(int nc, const int* inj_f, const int* inj_c, const double* xc, double* xf, void* stream);

/* src/ComputeDotProduct.cpp:63-238: *result (DEVICE pointer) = sum x[i]*y[i].
 * Deterministic fixed-shape two-level reduction in one launch; workspace >=
 * hpcgb200_reduction_workspace_bytes(), its counter must start at zero (it is
 * left at zero on return, so a zero-filled workspace can be reused). */
int hpcgb200_dot(int n, const double* x, const double* y, double* result, void* workspace, size_t workspace_bytes,
                 void* stream);

/* No counterpart in the reference.  The dot product for callers that cannot
 * allocate device memory: applications whose device memory belongs to their
 * own pool (a framework's caching allocator, a plugin with a fixed budget)
 * and latency-critical callers for which cudaMalloc -- which can synchronize
 * the device -- is not allowed.  *result (DEVICE pointer) = sum x[i]*y[i],
 * with no workspace argument: the scratch is a 32 KB array inside the library
 * that every GPU loading the library keeps until the process exits.
 * n <= 16,777,216 (4096 partial sums of 4096-element tiles); larger n returns
 * HPCGB200_ERR_ARG.  All calls share that array: calls that overlap on the
 * GPU race, so serialize them.  The first call on a device looks up the
 * array's address (once per CUDA context, so a device reset or a caller's own
 * driver-API context gets a fresh lookup); make it before any stream capture.
 * Allocates nothing.  Deterministic for a given n, but its summation order
 * (one partial per 4096-element tile) is not hpcgb200_dot's, so the two agree
 * to rounding, not bit for bit. */
int hpcgb200_dot_noalloc(long long n, const double* x, const double* y, double* result, void* stream);

/* No reference counterpart: self-test of the bounded grid barrier that the
 * persistent CG step uses.  The blocks of one cooperative launch (a resident
 * grid, reported in *blocks) meet at a barrier; with absent_block >= 0 that
 * block returns without arriving, so the others' waits run out after about a
 * second and set *status = 1 (*passed counts the blocks that got through).
 * With absent_block = -1 every block passes and *status stays 0.  Allocates
 * and synchronizes the device (not for a hot path). */
int hpcgb200_selftest_grid_barrier(int absent_block, int* status, int* passed, int* blocks);

/* src/ComputeWAXPBY.cpp:63-135 (kernel_waxpby): w = alpha x + beta y with the
 * reference's alpha==1 / beta==1 fma forms. */
int hpcgb200_waxpby(int n, double alpha, const double* x, double beta, const double* y, double* w, void* stream);

/* src/ComputeWAXPBY.cpp:137-240 (ComputeFusedWAXPBYDot): y += alpha x and
 * *result (device) = ||y||^2; workspace as for hpcgb200_dot. */
int hpcgb200_waxpby_dot(int n, double alpha, const double* x, double* y, double* result, void* workspace,
                        size_t workspace_bytes, void* stream);

/* src/ComputeResidual.cpp:77-152: *result (device) = max_i |v1[i] - v2[i]|. */
int hpcgb200_residual_inf(int n, const double* v1, const double* v2, double* result, void* workspace,
                          size_t workspace_bytes, void* stream);

/* ------------------------------------------------------ learned smoother kernels
 * No reference counterpart: the conv-net smoother that replaces SymGS on the
 * coarse MG levels (a 3-layer 3x3x3 network, 1 -> 16 -> 16 -> 1 channels,
 * ReLU, BF16 weights and activations, FP32 accumulation).  Tensors are
 * channel-last BF16 [nb][nz][ny][nx][16] (16-byte aligned DEVICE memory);
 * weights w[tap][ci][co] FP32 with tap = (dz+1)*9 + (dy+1)*3 + (dx+1); zero
 * padding outside each sample's grid.  *status (device int) is set non-zero
 * if a tensor-core wait timed out (the launch then returns early). */

/* Bytes of one layer's prepared BF16 operand tiles (27 x 16 x 16 x 2). */
size_t hpcgb200_conv_weight_tile_bytes(void);
/* w (device, 6912 FP32) -> wB (device, tile bytes); flip != 0 prepares the
 * transposed convolution's weights (mirrored taps, swapped channels). */
int hpcgb200_conv_prepare_weights(const float* w, void* wB, int flip, void* stream);
#define HPCGB200_CONV_RELU_BF16 0  /* out = bf16(relu(conv)), 16 channels */
#define HPCGB200_CONV_MASK_BF16 1  /* out = bf16(act > 0 ? conv : 0), 16 channels */
#define HPCGB200_CONV_F32 2        /* out = conv, FP32 16 channels */
#define HPCGB200_CONV_F32_C0 3     /* out = channel 0 of conv, FP32 [nb][nz][ny][nx] */
/* out = conv(in, W) on tcgen05 tensor cores; act is read by the masked mode. */
int hpcgb200_conv16(int nb, int nz, int ny, int nx, const void* in, const void* wB, int out_mode, void* out,
                    const void* act, int* status, void* stream);
/* Workspace of hpcgb200_conv16_wgrad (per-CTA partial sums). */
size_t hpcgb200_conv_wgrad_partial_bytes(int nb, int nz, int ny, int nx);
/* dw[tap][ci][co] (device, 6912 FP32) = sum_p x[p + tap][ci] * g[p][co]
 * (deterministic: fixed partition, fixed-order reduction). */
int hpcgb200_conv16_wgrad(int nb, int nz, int ny, int nx, const void* x, const void* g, float* partial, float* dw,
                          int* status, void* stream);

/* ------------------------------------------------------ problem handle
 * A handle owns the device hierarchy built exactly as src/main.cpp:198-210 +
 * src/OptimizeProblem.cpp:69-160 do (GenerateProblem, SetupHalo,
 * 3x GenerateCoarseProblem, OptimizeProblem), on its own CUDA stream. */
typedef struct hpcgb200_problem hpcgb200_problem;

#define HPCGB200_MODE_FP64 0    /* plain FP64 drop-in (the reference's optimized path) */
#define HPCGB200_MODE_MIXED 1   /* FP64 outer CG, FP32 V-cycle on the implicit stencil */
#define HPCGB200_MODE_LEARNED 2 /* as MIXED, with the attached learned smoother on the coarse levels
                                   (flexible CG; falls back to MIXED for good when the FP64
                                   residual norm jumps, stalls or shrinks too slowly:
                                   hpcgb200_problem_set_fallback) */
#define HPCGB200_MODE_FP64_STENCIL 3 /* FP64 as HPCGB200_MODE_FP64, V-cycle and SpMV on the implicit stencil:
                                        the same residual history bit for bit, no matrix reads (needs the
                                        27-point stencil in parity colouring on level 0; coarse levels
                                        without it, or with colour bricks not 4-aligned, use the ELL
                                        kernels) */

int hpcgb200_problem_create(int nx, int ny, int nz, int nlevels, hpcgb200_problem** out);
/* flags: HPCGB200_FLAG_KEEP_GENERATED keeps the row-major generated arrays
 * (mtx_ind, values, hash ...) that OptimizeProblem otherwise frees. */
#define HPCGB200_FLAG_KEEP_GENERATED 1
int hpcgb200_problem_create_ex(int nx, int ny, int nz, int nlevels, int flags, hpcgb200_problem** out);
int hpcgb200_problem_destroy(hpcgb200_problem* p);
/* dims[3*level..], rows[level], nnz[level], nblocks[level] for every level (host arrays of nlevels). */
int hpcgb200_problem_info(const hpcgb200_problem* p, int* nlevels, int* dims, int* rows, long long* nnz,
                          int* nblocks);
/* Seconds spent in generation (src/main.cpp:190-215) and in OptimizeProblem. */
int hpcgb200_problem_setup_times(const hpcgb200_problem* p, double* setup_s, double* optimize_s);
int hpcgb200_problem_stream(const hpcgb200_problem* p, void** stream);
/* *ok = 1 when the level was verified to be the 27-point stencil in parity
 * colouring (required by HPCGB200_MODE_MIXED). */
int hpcgb200_problem_stencil_ok(const hpcgb200_problem* p, int level, int* ok);

/* Field access for tests and tools: copy a device array of a level to host
 * memory.  field: "perm","colors","ell_col","ell_val","diag_idx","inv_diag",
 * "f2c","inj_f","inj_c","b","xexact","x","sizes","offsets","mtx_ind",
 * "values","nnz_in_row","hash","round_sizes". */
int hpcgb200_problem_copy_field(const hpcgb200_problem* p, int level, const char* field, void* host,
                                size_t bytes);
/* Size in bytes of a field (same names). */
int hpcgb200_problem_field_bytes(const hpcgb200_problem* p, int level, const char* field, size_t* bytes);
/* Device pointer of a field (same names) for zero-copy use. */
int hpcgb200_problem_device_field(const hpcgb200_problem* p, int level, const char* field, void** dev);

/* Right-hand side: b from HOST memory in natural order (it is permuted on
 * upload); NULL restores the generated b (exact solution all ones). */
int hpcgb200_problem_set_rhs(hpcgb200_problem* p, const double* host_b_natural);
/* Current solution to HOST memory in natural order. */
int hpcgb200_problem_get_x(hpcgb200_problem* p, double* host_x_natural);

/* src/CG.cpp:104-200: CG from x = 0 on the problem's b.  mode: HPCGB200_MODE_*.
 * normr_hist (host, may be NULL) gets max_iter+1 entries (normr after the
 * preamble and after each iteration).  seconds: device-timed solve.
 * A residual that turns non-finite (a NaN or Inf in b or in the operator
 * data) ends the iterations at once; the outputs are filled and the call
 * returns HPCGB200_ERR_NONFINITE.  In HPCGB200_MODE_LEARNED a non-finite
 * network step is a smoother failure instead: the solve restarts from x = 0
 * with the plain FP32 V-cycle, counting the abandoned iterations in *niters
 * and reporting the restart as the fallback iteration. */
int hpcgb200_problem_cg(hpcgb200_problem* p, int mode, int max_iter, double tol, int precond, int* niters,
                        double* normr, double* normr0, double* normr_hist, double* seconds);

/* Same, end to end from HOST memory: copies b_natural in, solves, copies x
 * out (natural order); seconds covers the copies too.  Non-finite residual:
 * as above. */
int hpcgb200_problem_solve_host(hpcgb200_problem* p, int mode, const double* b_natural, double* x_natural,
                                int max_iter, double tol, int* niters, double* normr, double* normr0,
                                double* seconds);

/* True residual of the current x, in FP64: *rel = ||b - A x|| / ||b||
 * (independent of the CG recurrence's updated r). */
int hpcgb200_problem_true_residual(hpcgb200_problem* p, double* rel);

/* Number of kernel launches one CG iteration of the given mode issues (the
 * kernel nodes of its iteration graph, captured here if needed). */
int hpcgb200_problem_kernels_per_iteration(hpcgb200_problem* p, int mode, int precond, int* kernels);

/* src/TestCG.cpp:111-177.  out[0..3] = niters of unpreconditioned call 0,1
 * and preconditioned call 0,1; *count_pass / *count_fail as the reference. */
int hpcgb200_problem_test_cg(hpcgb200_problem* p, int mode, int* out_niters, int* count_pass, int* count_fail);

/* src/TestSymmetry.cpp:88-166 with the reference's random vectors
 * (rand()/RAND_MAX + 1 from the process rand() state): depsym_spmv,
 * depsym_mg (mode selects the V-cycle precision), ||A xexact - b||_inf. */
int hpcgb200_problem_test_symmetry(hpcgb200_problem* p, int mode, double* depsym_spmv, double* depsym_mg,
                                   double* residual_inf);

/* Per-operator calls on the handle's level data (vectors are DEVICE
 * pointers in permuted order), used by the operator parity tests. */
int hpcgb200_problem_spmv(hpcgb200_problem* p, int level, const double* x, double* y);
/* y = A x on the implicit stencil in the ELL kernel's summation order (the
 * FP64 stencil mode's operator and every solve's preamble); no reference
 * counterpart; bitwise equal to hpcgb200_problem_spmv. */
int hpcgb200_problem_spmv_stencil(hpcgb200_problem* p, int level, const double* x, double* y);
/* The mixed path's outer FP64 operator on the implicit stencil: y = A x with
 * the 27 terms summed as a separable box (x, then y, then z sums), equal to
 * the ELL product to FP64 rounding (not bit for bit); the product the mixed
 * and learned CG steps use.  No reference counterpart (src/ComputeSPMV.cpp:
 * 226-278 is the operator it stands in for). */
int hpcgb200_problem_spmv_mixed(hpcgb200_problem* p, int level, const double* x, double* y);
int hpcgb200_problem_symgs(hpcgb200_problem* p, int level, const double* r, double* x);
int hpcgb200_problem_symgs_zero(hpcgb200_problem* p, int level, const double* r, double* x);
int hpcgb200_problem_mg(hpcgb200_problem* p, int mode, const double* r, double* x);
int hpcgb200_problem_restrict(hpcgb200_problem* p, int level, const double* rf, const double* xf, double* rc);
int hpcgb200_problem_prolong(hpcgb200_problem* p, int level, const double* xc, double* xf);

/* ------------------------------------------------------ learned smoother
 * No reference counterpart.  A smoother handle owns the conv net's FP32
 * master weights (HPCGB200_SMOOTHER_WEIGHTS floats: layers 1..3 back to back,
 * each w[tap][ci][co]), its BF16 operand tiles, activation buffers and Adam
 * state, all in device memory.  Fields r, e, y are FP32 DEVICE arrays in
 * natural grid order, samples back to back. */
typedef struct hpcgb200_smoother hpcgb200_smoother;
#define HPCGB200_SMOOTHER_WEIGHTS (3 * 27 * 16 * 16)

int hpcgb200_smoother_create(hpcgb200_smoother** out);
/* Detach it from every problem (hpcgb200_problem_set_smoother(p, NULL, 0, 0))
 * before destroying it. */
int hpcgb200_smoother_destroy(hpcgb200_smoother* s);
int hpcgb200_smoother_set_weights(hpcgb200_smoother* s, const float* host_w);
int hpcgb200_smoother_get_weights(hpcgb200_smoother* s, float* host_w);
/* Host-side initial weights: the network computes omega * r / 26 (a damped
 * Jacobi step: channel 0 = relu(r), channel `twin` (1..15; 8 for the tied
 * form) = relu(-r)) plus uniform noise in [-noise, noise] on every other used
 * weight, from a SplitMix64 stream. */
int hpcgb200_smoother_init_jacobi(float* host_w, float omega, float noise, unsigned long long seed, int twin);
/* y = N(r) for nb samples of nz x ny x nx points. */
int hpcgb200_smoother_forward(hpcgb200_smoother* s, int nb, int nz, int ny, int nx, const float* r, float* y,
                              void* stream);
/* Symmetry of the network in r.  0 (default): plain N(r).  1: evaluated as
 * (N(r) - N(-r)) / 2, an odd function (both branches run as one batch of
 * two).  2: tied weights -- hidden channel k+8 is the negated twin of channel
 * k in every layer, enforced on every weight update -- so one evaluation of N
 * is already odd. */
#define HPCGB200_SMOOTHER_PLAIN 0
#define HPCGB200_SMOOTHER_ODD 1
#define HPCGB200_SMOOTHER_TIED 2
int hpcgb200_smoother_configure(hpcgb200_smoother* s, int symmetry);
/* loss = scale * sum_b d_b.M d_b * inv_norm[b], d = y - e with y the network
 * output; kind 0: M = I, kind 1: M = the 27-point stencil A (energy norm).
 * inv_norm (device, nb floats) = 1/(e.e) or 1/(e.Ae): hpcgb200_sample_norms.
 * The gradient with respect to the weights is copied to dw (device,
 * HPCGB200_SMOOTHER_WEIGHTS floats) when not NULL; the handle keeps it for
 * hpcgb200_smoother_adam_step.  *loss (host) may be NULL. */
int hpcgb200_smoother_loss_grad(hpcgb200_smoother* s, int nb, int nz, int ny, int nx, const float* r, const float* e,
                                const float* inv_norm, float scale, int kind, float* dw, double* loss, void* stream);
/* out[b] = 1/(e_b.e_b) (kind 0) or 1/(e_b.A e_b) (kind 1) for nb samples. */
int hpcgb200_sample_norms(int nb, int nz, int ny, int nx, const float* e, int kind, float* out, void* stream);
/* One bias-corrected Adam step with the last gradient. */
int hpcgb200_smoother_adam_step(hpcgb200_smoother* s, float lr, float beta1, float beta2, float eps, void* stream);

/* A set of `count` training pairs of one grid size, trained `batch` samples
 * per step (r, e: count * nz*ny*nx floats; inv_ee: count floats, 1/||e||^2). */
typedef struct
{
    const float* r;
    const float* e;
    const float* inv_ee;
    int count, nz, ny, nx, batch;
} hpcgb200_pair_set;
/* Adam training over the sets for `epochs` passes (batches of all sets in a
 * seeded shuffled order; learning rate geometric from lr0 to lr1; per-sample
 * loss of hpcgb200_smoother_loss_grad with the given kind, relative to the
 * sample's e.e or e.Ae).  epoch_loss (host, may be NULL): mean loss of each
 * epoch. */
int hpcgb200_smoother_train(hpcgb200_smoother* s, const hpcgb200_pair_set* sets, int nsets, int epochs, float lr0,
                            float lr1, int kind, unsigned long long seed, double* epoch_loss, void* stream);
/* Training pairs from the plain FP32 V-cycle: for seeds first_seed ..
 * first_seed+count-1, b ~ N(0,1) (hpcgb200_normal_rhs) on a fine_n^3 grid;
 * r = the residual the V-cycle hands to MG level `level`, e = A_level^-1 r
 * (FP64 MG-PCG to relative residual tol); both in natural order of the
 * (fine_n >> level)^3 level grid, FP32 device arrays of count * points;
 * inv_ee (device, count floats) = 1 / ||e||^2. */
int hpcgb200_make_training_pairs(int fine_n, int level, unsigned long long first_seed, int count, float* r,
                                 float* e, float* inv_ee, double tol);
/* N(0,1) values by natural index (SplitMix64 + Box-Muller, the generator of
 * rochpcg_b200/rhs.py) into out (device, m doubles). */
int hpcgb200_normal_rhs(long long m, unsigned long long seed, double* out, void* stream);

/* Attach a smoother (NULL detaches) to the problem's levels >= first_level
 * for HPCGB200_MODE_LEARNED; the handle must outlive the attachment.  On
 * those levels the V-cycle's pre- and post-smoothing SymGS become x = N(r)
 * and x += N(r - A x); the coarsest level's single SymGS becomes x = N(r)
 * followed by coarse_steps - 1 steps x += N(r - A x) (1..64). */
int hpcgb200_problem_set_smoother(hpcgb200_problem* p, hpcgb200_smoother* s, int first_level, int coarse_steps);
/* The learned solve's failure rule: it falls back to SymGS for good after an
 * iteration that multiplies the residual norm by more than `jump` (>= 1; 1 with
 * the other tests off is "the first iteration that does not reduce it"), after
 * `stall` iterations without a new minimum, with rate > 0 when the norm is above
 * rate times its value `window` iterations earlier, or on a non-finite norm.
 * Defaults: jump 2, stall 16, window 16, rate 0.8 (rate 0 turns that test off). */
int hpcgb200_problem_set_fallback(hpcgb200_problem* p, double jump, int stall, int window, double rate);
/* Iteration at which the last learned solve fell back to SymGS (0: never). */
int hpcgb200_problem_last_fallback(const hpcgb200_problem* p, int* fallback_iter);

/* Time n back-to-back launches of one level-0 operator with CUDA events on
 * the problem's stream; *ms_per_launch = average.  op: "spmv","symgs_sweep"
 * (one full-row color sweep, averaged over the 15 of a SymGS step),
 * "symgs","symgs_zero","mg","mg_mixed", "symgs32_sweep" (one FP32 implicit
 * colour sweep, averaged over a SymGS step), "spmv_stencil", "mg_learned"
 * (the V-cycle with the attached learned smoother), "mg_stencil" (the FP64
 * V-cycle on the implicit stencil).  "graph:<op>" captures one call of <op>
 * into a CUDA graph and times launches of the graph instead. */
int hpcgb200_problem_time_op(hpcgb200_problem* p, const char* op, int n, double* ms_per_launch);

/* ---------------------------------------------- reference routines (natural order)
 * The benchmark's `_ref` kernels on the generated row-major arrays (natural
 * row order, 27 slots per row, nonzero counts as signed char, the diagonal's
 * slot per row), device pointers, nx*ny*nz rows.  Results equal those of the
 * sequential C loops bit for bit (products and sums rounded separately). */
/* src/ComputeSPMV_ref.cpp:48-75: y = A x. */
int hpcgb200_ref_spmv(int nx, int ny, int nz, const int* mtx_ind, const double* values,
                      const signed char* nnz_in_row, const double* x, double* y, void* stream);
/* src/ComputeSYMGS_ref.cpp:51-104: one forward and one backward natural-order
 * Gauss-Seidel sweep on x (in place), run as 2 * (nx + 2 ny + 4 nz - 6)
 * wavefront launches. */
int hpcgb200_ref_symgs(int nx, int ny, int nz, const int* mtx_ind, const double* values,
                       const signed char* nnz_in_row, const int* diag_slot, const double* r, double* x,
                       void* stream);
/* src/CG_ref.cpp:60-160 on a problem created with
 * HPCGB200_FLAG_KEEP_GENERATED: the reference CG in natural order from x = 0
 * on the problem's b (un-permuted), with ComputeMG_ref as preconditioner when
 * precond != 0.  Overwrites the problem's x with the natural-order result
 * (hpcgb200_problem_get_x does not apply to it). */
int hpcgb200_problem_cg_ref(hpcgb200_problem* p, int max_iter, double tol, int precond, int* niters,
                            double* normr, double* normr0, double* seconds);

/* src/ComputeMG_ref.cpp on a problem created with HPCGB200_FLAG_KEEP_GENERATED:
 * z = M^-1 r for natural-order device vectors r, z of level 0 (the V-cycle
 * of the reference CG: natural-order SymGS, injection, 1 pre / 1 post step). */
int hpcgb200_problem_mg_ref(hpcgb200_problem* p, const double* r_natural, double* z_natural);

/* --------------------------------------------------- benchmark protocol
 * src/main.cpp:174-563 with src/ReportResults.cpp: set-up, CheckProblem,
 * reference SpMV+MG timing, the 50-iteration reference CG residual,
 * OptimizeProblem, TestCG, TestSymmetry, the optimized CG set-up run, timed
 * CG sets for running_time seconds, TestNorms and the report (a JSON
 * document with the sections and field names of the reference's YAML).  One
 * rank; the reference phases run on the device in natural order. */
#define HPCGB200_BENCH_MAX_LEVELS 8
typedef struct hpcgb200_benchmark_params
{
    int nx, ny, nz;       /* local = global grid; a dimension < 16 is raised as src/init.cpp:150-159 does */
    int running_time;     /* seconds of timed CG sets (--rt=); 0 selects the QuickPath */
    int verify;           /* 1: reference phases and validation; 0: ref tolerance = tol (--tol=) */
    double tol;
    int mode;             /* HPCGB200_MODE_FP64, HPCGB200_MODE_MIXED or HPCGB200_MODE_FP64_STENCIL */
} hpcgb200_benchmark_params;

typedef struct hpcgb200_benchmark_result
{
    /* filled by hpcgb200_benchmark_run: the inputs of the report */
    int nx, ny, nz, mode, verify, quick_path;
    int levels;
    long long rows[HPCGB200_BENCH_MAX_LEVELS];
    long long nonzeros[HPCGB200_BENCH_MAX_LEVELS];
    int presmoother_steps, postsmoother_steps;
    double times[10];              /* the driver's times[]: 0 timed CG sets, 1 DDOT, 2 WAXPBY, 3 SpMV,
                                      5 MG, 7 optimization, 8 reference SpMV+MG per call, 9 setup */
    double optimize_problem_bytes; /* device bytes OptimizeProblem allocates */
    long long check_problem_errors;
    int ref_max_iters, ref_niters;
    double ref_tolerance;          /* normr/normr0 after the reference CG (or params.tol) */
    int opt_max_iters;             /* iterations per timed set */
    int opt_setup_niters;          /* iterations the set-up run needed to reach ref_tolerance */
    int tolerance_failures, err_count, global_failure;
    double opt_worst_time;
    int cg_sets;
    int testcg_count_pass, testcg_count_fail;
    int testcg_expected_niters_no_prec, testcg_expected_niters_prec;
    int testcg_niters_max_no_prec, testcg_niters_max_prec;
    double depsym_spmv, depsym_mg;
    int symmetry_count_fail;
    double norms_mean, norms_variance;
    int norms_pass;
    /* filled by hpcgb200_benchmark_report */
    double fnops, frefnops;
    double gflops_raw, gflops_convergence, gflops_final, gflops_hpcg24;
    double gbs_raw, gbs_final;
    double memory_total_gb;
    int valid;
} hpcgb200_benchmark_result;

/* Runs the whole protocol on the current device and fills *result (then
 * calls hpcgb200_benchmark_report without a buffer). */
int hpcgb200_benchmark_run(const hpcgb200_benchmark_params* params, hpcgb200_benchmark_result* result);
/* Host only (no device needed): the derived figures of src/ReportResults.cpp
 * :134-195,396-460 from the inputs in *result, and the report as JSON into
 * json[capacity] (NUL-terminated; *length = bytes without the NUL, also when
 * json is NULL or too small, which returns HPCGB200_ERR_WORKSPACE). */
int hpcgb200_benchmark_report(hpcgb200_benchmark_result* result, char* json, size_t capacity, size_t* length);

/* ------------------------------------------------ domain decomposition
 * One rank's sub-brick of a problem split over size = npx*npy*npz ranks (one
 * GPU each), the reference's multi-rank path: src/GenerateGeometry.cpp,
 * src/SetupHalo.cpp, src/ExchangeHalo.cpp and the halo halves of
 * src/ComputeSPMV.cpp, src/ComputeSYMGS.cpp, src/ComputeRestriction.cpp,
 * src/ComputeDotProduct.cpp (FP64 ELL path).  Every rank holds the same local
 * brick nx*ny*nz; the global grid is (npx*nx) x (npy*ny) x (npz*nz). */

/* src/ComputeOptimalShapeXYZ.cpp:94-157: the process grid for size ranks
 * (host only). */
int hpcgb200_dist_shape(int size, int* npx, int* npy, int* npz);

/* src/GenerateGeometry.cpp:49-169 (host only; the C++ GenerateGeometry):
 * out[13] = {npx, npy, npz, ipx, ipy, ipz, gnx, gny, gnz, gix0, giy0, giz0,
 * npartz} of `rank` (npx*npy*npz <= 0 or > size: hpcgb200_dist_shape; pz > 0:
 * process planes below pz hold zl points in z, the others zu). */
int hpcgb200_geometry(int size, int rank, int pz, int zl, int zu, int nx, int ny, int nz, int npx, int npy, int npz,
                      long long* out);

/* src/SetupHalo.cpp:135-651 on the host (no device needed): the halo plan of
 * `rank` for a local brick nx*ny*nz (npx/npy/npz <= 0: hpcgb200_dist_shape).
 * hpcgb200_halo_plan_info fills info[16] = {m, externals, neighbours,
 * send entries, halo rows, halo width, halo entries, npx, npy, npz, ipx,
 * ipy, ipz, nx, ny, nz}; hpcgb200_halo_plan_copy copies one field to the
 * host: "nbr_rank", "nbr_slot", "recv_len", "recv_off", "send_len",
 * "send_off", "send_rows", "halo_rows", "halo_ptr", "halo_cols" (int32) or
 * "recv_gid" (int64), bytes = its exact size. */
typedef struct hpcgb200_halo_plan hpcgb200_halo_plan;
int hpcgb200_halo_plan_create(int nx, int ny, int nz, int size, int rank, int npx, int npy, int npz,
                              hpcgb200_halo_plan** out);
int hpcgb200_halo_plan_info(const hpcgb200_halo_plan* plan, int* info);
int hpcgb200_halo_plan_copy(const hpcgb200_halo_plan* plan, const char* field, void* host, size_t bytes);
int hpcgb200_halo_plan_destroy(hpcgb200_halo_plan* plan);

/* src/main.cpp:183-210 + src/OptimizeProblem.cpp for one rank: generates and
 * optimizes the rank's brick on every level (the single-rank colouring,
 * permutation and ELL of the brick), then adds the external columns after
 * each row's local ones and lowers the generated b by the row's external
 * count.  npx/npy/npz <= 0: hpcgb200_dist_shape(size). */
typedef struct hpcgb200_dist hpcgb200_dist;
int hpcgb200_dist_create(int nx, int ny, int nz, int nlevels, int size, int rank, int npx, int npy, int npz,
                         hpcgb200_dist** out);
int hpcgb200_dist_destroy(hpcgb200_dist* d);
/* info[20]: the 16 plan values of `level`, then size, rank, levels, colours;
 * *nnz = nonzeros of the rank's rows on that level, external ones included. */
int hpcgb200_dist_info(const hpcgb200_dist* d, int level, int* info, long long* nnz);
/* The plan fields above, or device data: "ell_col", "ell_val", "perm",
 * "send_perm", "halo_prow", "halo_col", "halo_pc" (any level), "b", "x"
 * (level 0: b permuted, x permuted with its external tail). */
int hpcgb200_dist_copy_field(const hpcgb200_dist* d, int level, const char* field, void* host, size_t bytes);
/* b in the rank's natural row order (NULL: the generated b again); the
 * rank's part of the solution in natural order. */
int hpcgb200_dist_set_rhs(hpcgb200_dist* d, const double* host_b_natural);
int hpcgb200_dist_get_x(hpcgb200_dist* d, double* host_x_natural);

/* NCCL transport (one process per GPU).  1 if libnccl.so.2 can be opened.
 * Rank 0 makes the communicator id (bytes = 128) and every rank passes it to
 * hpcgb200_dist_attach_nccl (collective over the ranks).  A solve that makes
 * no progress for $HPCGB200_DIST_TIMEOUT_S seconds (600) aborts the
 * communicator and returns HPCGB200_ERR_COMM. */
int hpcgb200_dist_nccl_available(void);
int hpcgb200_dist_nccl_id(void* id, size_t bytes);
int hpcgb200_dist_attach_nccl(hpcgb200_dist* d, const void* id, size_t bytes);

/* Operators and CG over a group of ranks: either every rank of the
 * decomposition in this process (n == size, one device: the exchange is a
 * device copy per neighbour), or one rank with a communicator (n == 1).
 * Vectors are device arrays in each rank's permuted order; x-type vectors
 * (the ones the halo exchange fills) hold the rank's local rows followed by
 * its external columns.  Each call returns when its work is complete.
 *   spmv     y = A x                 (src/ComputeSPMV.cpp:226-278)
 *   symgs    one symmetric sweep     (src/ComputeSYMGS.cpp:369-404)
 *   restrict rc = R(rf - A xf)       (src/ComputeRestriction.cpp:199-237; level < levels-1)
 *   mg       x = M r, the V-cycle    (src/ComputeMG.cpp:64-102)
 *   cg       the preconditioned CG on the ranks' generated (or set) b from
 *            x = 0 (src/CG.cpp:104-200); normr_hist (max_iter+1) may be NULL;
 *            *seconds = device time of the solve on the group's stream. */
int hpcgb200_dist_group_spmv(hpcgb200_dist* const* ranks, int n, int level, double* const* x, double* const* y);
int hpcgb200_dist_group_symgs(hpcgb200_dist* const* ranks, int n, int level, double* const* r, double* const* x);
int hpcgb200_dist_group_restrict(hpcgb200_dist* const* ranks, int n, int level, double* const* rf,
                                 double* const* xf, double* const* rc);
int hpcgb200_dist_group_mg(hpcgb200_dist* const* ranks, int n, double* const* r, double* const* x);
int hpcgb200_dist_group_cg(hpcgb200_dist* const* ranks, int n, int max_iter, double tol, int precond, int* niters,
                           double* normr, double* normr0, double* normr_hist, double* seconds);
/* hpcgb200_dist_group_cg with the one rank d (a communicator attached, or size 1). */
int hpcgb200_dist_cg(hpcgb200_dist* d, int max_iter, double tol, int precond, int* niters, double* normr,
                     double* normr0, double* normr_hist, double* seconds);

#ifdef __cplusplus
}
#endif
#endif /* HPCG_B200_H */
