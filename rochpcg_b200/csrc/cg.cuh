// Device-resident CG recurrence (src/CG.cpp:104-200) for libhpcgb200.
#pragma once

#include "common.cuh"
#include "ops64.cuh"

namespace hb {

// Scalars of one CG solve, kept in device memory so that an iteration needs
// no host round trip: alpha/beta are formed by the last block of the
// reduction that produces their denominator.
struct CGState
{
    double rtz, oldrtz, alpha, beta, pAp;
    double normr, normr0, tol;
    double rtz_flex;      // r_new . z_old (flexible-CG beta numerator term)
    int k;                // iteration about to run (1-based)
    int max_iter;
    int niters;
    int flexible;         // 1: Polak-Ribiere beta (flexible CG); 0: Fletcher-Reeves as the reference
    int status;           // nonzero: a device-side check failed
    int net;              // learned smoother: 0 not used, 1 active, 2 failed (fell back)
    int fallback_iter;    // iteration at which it failed (0: never); the next iteration restarts p = z
    int since_best;       // iterations since normr last reached a new minimum
    double best_normr;    // smallest normr so far
    // learned-smoother failure rule (set by the host): an iteration that
    // multiplies normr by more than fb_jump; fb_stall iterations without a new
    // minimum; with fb_rate > 0, normr above fb_rate times its value fb_window
    // iterations earlier; or a non-finite normr.  PCG residual norms are not
    // monotone, so a single small increase is no failure.
    double fb_jump, fb_rate;
    int fb_stall, fb_window;
    // phase timers of an instrumented solve (k_cg_timer): nanoseconds spent in
    // dot products, vector updates, SpMV and MG, and the last time stamp
    double phase_ns[4];
    unsigned long long t_last;
    double hist[1];       // normr after preamble and after each iteration (max_iter+1 entries)
};

// ---- device helpers of the two-kernel CG step (k_cg_step1_* kernels)
// Per-block row range of the vector phases (a multiple of 32 rows, so that
// no 256-byte line is shared by two blocks' writes).
__device__ __forceinline__ void step_rows(long long n, long long& lo, long long& hi)
{
    const long long per = (((n + gridDim.x - 1) / gridDim.x) + 31) & ~31ll;
    lo = (long long)blockIdx.x * per;
    hi = lo + per < n ? lo + per : n;
}

// Phase 1 and 2 of step 1: beta from r.z, then p = z + beta p.  Returns false
// when a barrier timed out.
template <typename Z>
__device__ __forceinline__ bool step1_rz_p(long long n, const double* __restrict__ r, const Z* __restrict__ z,
                                           double* __restrict__ p, double* __restrict__ x, CGState* st,
                                           double* partial, GridBarrier* gb)
{
    __shared__ double red[32];
    __shared__ double sh_beta;
    const int tid = threadIdx.x;
    long long lo, hi;
    step_rows(n, lo, hi);
    const int k = st->k;
    const bool restart = k == 1 || (st->fallback_iter > 0 && k == st->fallback_iter + 1);
    const double old_rtz = st->rtz, rtz_flex = st->rtz_flex, alpha_prev = st->alpha;
    const bool flex = st->flexible != 0;
    double s = 0.0;
    for(long long i = lo + tid; i < hi; i += blockDim.x) s = fma((double)z[i], r[i], s);
    s = block_sum(s, red);
    if(tid == 0) partial[blockIdx.x] = s;
    if(!grid_barrier(gb, gridDim.x, &st->status)) return false;
    double acc = 0.0;
    for(int i = tid; i < (int)gridDim.x; i += blockDim.x) acc += __ldcg(&partial[i]);
    acc = block_sum(acc, red);
    if(tid == 0)
    {
        const double beta = k == 1 ? 0.0 : (flex ? acc - rtz_flex : acc) / old_rtz;
        sh_beta = beta;
        if(blockIdx.x == 0)
        {
            if(k != 1) st->oldrtz = old_rtz;
            st->rtz = acc;
            st->beta = beta;
        }
    }
    __syncthreads();
    const double beta = sh_beta;
    for(long long i = lo + tid; i < hi; i += blockDim.x)
    {
        const double zi = (double)z[i];
        const double po = k > 1 ? __ldcg(p + i) : 0.0;
        if(k > 1) x[i] = fma(alpha_prev, po, x[i]);  // iteration k-1's x += alpha p, deferred
        __stcg(p + i, restart ? fma(0.0, zi, zi) : fma(beta, po, zi));
    }
    // the product after the next barrier may read p through TMA (the async proxy)
    asm volatile("fence.proxy.async.global;" ::: "memory");
    return grid_barrier(gb, gridDim.x, &st->status);
}

// The last block to arrive forms pAp (partials in block order) and alpha.
__device__ __forceinline__ void step1_alpha(double s, CGState* st, double* partial, unsigned int* ticket)
{
    __shared__ double red[32];
    __shared__ bool last;
    s = block_sum(s, red);
    if(threadIdx.x == 0)
    {
        partial[blockIdx.x] = s;
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if(!last) return;
    __threadfence();
    double acc = 0.0;
    for(int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) acc += __ldcg(&partial[i]);
    acc = block_sum(acc, red);
    if(threadIdx.x == 0)
    {
        *ticket = 0;
        st->pAp = acc;
        st->alpha = st->rtz / acc;
    }
}


// Phases of an instrumented CG iteration (the reference's times[] slots 1, 2, 3, 5).
enum CGPhase
{
    kPhaseDot = 0,
    kPhaseWaxpby = 1,
    kPhaseSpmv = 2,
    kPhaseMG = 3,
    kPhaseStart = -1
};

// Defaults, chosen on the trained smoother (no false fallback at 64^3..256^3
// with N(0,1) right-hand sides) and a planted diverging one (caught at
// iteration 36 of a 64^3 solve): normr must shrink by 20 % every 16 iterations.
constexpr double kFallbackJump = 2.0;
constexpr int kFallbackStall = 16;
constexpr int kFallbackWindow = 16;
constexpr double kFallbackRate = 0.8;

inline size_t cg_state_bytes(int max_iter) { return sizeof(CGState) + sizeof(double) * (size_t)(max_iter + 1); }

// Preamble: r = b - Ap (WAXPBY(1,b,-1,Ap)), normr = ||r||, normr0 = normr,
// k = 1; returns whether iterations are needed through state.
int launch_cg_residual0(int n, const double* b, const double* Ap, double* r, CGState* st, ReduceScratch* ws,
                        cudaStream_t s);
// rtz = r.z, beta = rtz/oldrtz (k>1), oldrtz kept.  The float forms read
// the FP32 V-cycles' output directly (every value widened exactly).
int launch_cg_rtz(int n, const double* r, const double* z, CGState* st, ReduceScratch* ws, cudaStream_t s);
int launch_cg_rtz(int n, const double* r, const float* z, CGState* st, ReduceScratch* ws, cudaStream_t s);
// p = z (k == 1) or p = z + beta p; for k > 1 first the previous iteration's
// x += alpha p (deferred from the r update to this pass, which reads that p
// anyway: one read of p per iteration fewer).  launch_cg_x_final applies the
// last iteration's update after the loop.
int launch_cg_update_p(int n, const double* z, double* p, double* x, const CGState* st, cudaStream_t s);
int launch_cg_update_p(int n, const float* z, double* p, double* x, const CGState* st, cudaStream_t s);
int launch_cg_x_final(int n, const double* p, double* x, const CGState* st, cudaStream_t s);
// Ap = A p and alpha = rtz / (p.Ap); `partial` holds cc.nchunks() per-block
// sums, `ticket` must start at zero and is left at zero.
int launch_cg_spmv_pap(int m, const ColorChunks& cc, const int* ell_col, const double* ell_val, const double* p,
                       double* Ap, CGState* st, double* partial, unsigned int* ticket, cudaStream_t s);
// pAp = p.Ap and alpha from a precomputed Ap, summed with exactly the block
// partition and order of launch_cg_spmv_pap (same partials, same final sum),
// so a solve whose SpMV runs elsewhere keeps the ELL solve's scalars bit for bit.
int launch_cg_pap_chunks(int m, const ColorChunks& cc, const double* p, const double* Ap, CGState* st,
                         double* partial, unsigned int* ticket, cudaStream_t s);
// r -= alpha Ap, normr = ||r||, history; then (own 1-thread kernel) k++ and
// the loop condition (k <= max_iter && normr/normr0 > tol) written to `cond`
// (a graph conditional handle; 0 = none).  While the learned smoother is
// active (net == 1) an iteration that does not reduce normr marks it failed
// (net = 2); with watch_net the loop then also ends.
int launch_cg_update_r(int n, const double* Ap, double* r, const double* z, CGState* st, ReduceScratch* ws,
                       unsigned long long cond, int watch_net, cudaStream_t s);
int launch_cg_update_r(int n, const double* Ap, double* r, const float* z, CGState* st, ReduceScratch* ws,
                       unsigned long long cond, int watch_net, cudaStream_t s);

// Two-kernel CG step (src/CG.cpp:148-184).  Step 1 (persistent, cooperative,
// two bounded grid barriers): rtz = r.z and beta, the previous iteration's
// x += alpha p and p = z + beta p (as launch_cg_update_p), Ap = A p with pAp
// and alpha; it uses ws's partials and ticket (left at zero) and the grid
// barrier gb (count zero before the launch, left at zero).  Step 2:
// r -= alpha Ap, normr, then the loop control (as launch_cg_update_r, in one
// kernel).  A barrier that times out sets st->status.
int launch_cg_step1_ell(int n, const ColorChunks& cc, const int* ell_col, const double* ell_val, const double* r,
                        const double* z, double* p, double* x, double* Ap, CGState* st, ReduceScratch* ws,
                        GridBarrier* gb, cudaStream_t s);
int launch_cg_step2(int n, const double* Ap, double* r, const double* z, CGState* st, ReduceScratch* ws,
                    unsigned long long cond, int watch_net, cudaStream_t s);
int launch_cg_step2(int n, const double* Ap, double* r, const float* z, CGState* st, ReduceScratch* ws,
                    unsigned long long cond, int watch_net, cudaStream_t s);

// One thread: adds the time since the previous stamp to phase_ns[phase]
// (phase kPhaseStart only stamps).  Kernels on one stream run in order, so
// the stamps bracket the kernels launched between them.
int launch_cg_timer(CGState* st, int phase, cudaStream_t s);

// Mixed precision glue: r32 = (float) r and z = (double) z32.
int launch_cast_d2f(int n, const double* in, float* out, cudaStream_t s);
int launch_cast_f2d(int n, const float* in, double* out, cudaStream_t s);

}  // namespace hb
