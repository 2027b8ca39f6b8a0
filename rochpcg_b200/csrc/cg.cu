// Device-resident CG recurrence of src/CG.cpp:104-200.  The reference
// pays 12 device synchronisations and 3 blocking scalar read-backs per
// iteration; here every scalar (rtz, pAp, alpha, beta, normr) is produced by
// the last block of the reduction that needs it, and the loop condition is
// written to a CUDA-graph conditional handle, so a whole solve runs as one
// graph launch.  Vector arithmetic keeps the reference's fma forms.
#include "cg.cuh"

namespace hb {

__global__ void __launch_bounds__(kReduceThreads) k_cg_residual0(int n, const double* __restrict__ b,
                                                                 const double* __restrict__ Ap,
                                                                 double* __restrict__ r, CGState* st,
                                                                 ReduceScratch* ws)
{
    __shared__ double red[32];
    double s = 0.0;
    for(long long i = (long long)blockIdx.x * kReduceThreads + threadIdx.x; i < n; i += kReduceBlocks * kReduceThreads)
    {
        const double v = fma(-1.0, Ap[i], b[i]);  // WAXPBY(1, b, -1, Ap): alpha == 1 form
        r[i] = v;
        s = fma(v, v, s);
    }
    s = block_sum(s, red);
    double total;
    if(grid_reduce(s, ws, kReduceBlocks, &total))
    {
        const double nr = sqrt(total);
        st->normr = nr;
        st->normr0 = nr;
        st->hist[0] = nr;
        st->best_normr = nr;
        st->since_best = 0;
        st->k = 1;
        st->niters = 0;
        st->rtz = 0.0;
        st->oldrtz = 0.0;
        st->rtz_flex = 0.0;
    }
}

// Z: the preconditioner output's type -- double, or float for the FP32
// V-cycles, whose output is read as is ((double)z32 is exact, so the sums are
// the ones an FP64 copy of z would give, without writing or reading that copy).
template <typename Z>
__global__ void __launch_bounds__(kReduceThreads) k_cg_rtz(int n, const double* __restrict__ r,
                                                           const Z* __restrict__ z, CGState* st,
                                                           ReduceScratch* ws)
{
    __shared__ double red[32];
    double s = 0.0;
    for(long long i = (long long)blockIdx.x * kReduceThreads + threadIdx.x; i < n; i += kReduceBlocks * kReduceThreads)
        s = fma((double)z[i], r[i], s);
    s = block_sum(s, red);
    double total;
    if(grid_reduce(s, ws, kReduceBlocks, &total))
    {
        if(st->k == 1)
        {
            st->rtz = total;
            st->beta = 0.0;
        }
        else
        {
            st->oldrtz = st->rtz;
            st->rtz = total;
            // Fletcher-Reeves (the reference) or Polak-Ribiere for flexible CG:
            // beta = r_k.(z_k - z_{k-1}) / r_{k-1}.z_{k-1}
            const double num = st->flexible ? total - st->rtz_flex : total;
            st->beta = num / st->oldrtz;
        }
    }
}

// p = z (k == 1) or z + beta p; first, for k > 1, the previous iteration's
// x += alpha p (src/CG.cpp:174), deferred to this pass, which reads that p
// anyway (launch_cg_x_final applies the last one after the loop).
template <typename Z>
__global__ void __launch_bounds__(kBS) k_cg_update_p(int n, const Z* __restrict__ z, double* __restrict__ p,
                                                     double* __restrict__ x, const CGState* __restrict__ st)
{
    const int i = blockIdx.x * kBS + threadIdx.x;
    if(i >= n) return;
    // first iteration, and the first one after the learned smoother fell
    // back: p = z (a restart: the old directions belong to the other
    // preconditioner)
    const int k = st->k;
    const bool restart = k == 1 || (st->fallback_iter > 0 && k == st->fallback_iter + 1);
    const double zi = (double)z[i];
    const double po = k > 1 ? p[i] : 0.0;
    if(k > 1) x[i] = fma(st->alpha, po, x[i]);     // WAXPBY(1, x, alpha, p) of iteration k-1
    if(restart) p[i] = fma(0.0, zi, zi);            // WAXPBY(1, z, 0, z)
    else p[i] = fma(st->beta, po, zi);             // WAXPBY(1, z, beta, p)
}

// The last iteration's x += alpha p (the deferred update of k_cg_update_p),
// when the solve ran at least one iteration since its preamble.
__global__ void __launch_bounds__(kBS) k_cg_x_final(int n, const double* __restrict__ p, double* __restrict__ x,
                                                    const CGState* __restrict__ st)
{
    const int i = blockIdx.x * kBS + threadIdx.x;
    if(i >= n || st->k <= 1) return;
    x[i] = fma(st->alpha, p[i], x[i]);
}

// Ap = A p (one row per thread, colour-interleaved blocks as k_spmv) and
// pAp: one partial per block, summed in block order by the last block, which
// forms alpha = rtz / pAp.
__global__ void __launch_bounds__(kBS) k_cg_spmv_pap(int m, ColorChunks cc, const int* __restrict__ ell_col,
                                                     const double* __restrict__ ell_val,
                                                     const double* __restrict__ p, double* __restrict__ Ap,
                                                     CGState* st, double* partial, unsigned int* ticket)
{
    __shared__ double red[32];
    __shared__ bool last;
    double s = 0.0;
    int row;
    if(cc.row_of(blockIdx.x, threadIdx.x, row))
    {
        // the SpMV row kernel (its grouped loads; the same fma order, so the same Ap)
        const double sum = spmv_row(m, row, ell_col, ell_val, p);
        Ap[row] = sum;
        s = sum * p[row];
    }
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
    for(unsigned i = threadIdx.x; i < gridDim.x; i += kBS) acc += __ldcg(&partial[i]);
    acc = block_sum(acc, red);
    if(threadIdx.x == 0)
    {
        *ticket = 0;
        st->pAp = acc;
        st->alpha = st->rtz / acc;
    }
}

// The reduction half of k_cg_spmv_pap on a stored Ap: same chunk -> row map,
// same per-block tree, same last-block sum.
__global__ void __launch_bounds__(kBS) k_cg_pap_chunks(ColorChunks cc, const double* __restrict__ p,
                                                       const double* __restrict__ Ap, CGState* st, double* partial,
                                                       unsigned int* ticket)
{
    __shared__ double red[32];
    __shared__ bool last;
    double s = 0.0;
    int row;
    if(cc.row_of(blockIdx.x, threadIdx.x, row)) s = Ap[row] * p[row];
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
    for(unsigned i = threadIdx.x; i < gridDim.x; i += kBS) acc += __ldcg(&partial[i]);
    acc = block_sum(acc, red);
    if(threadIdx.x == 0)
    {
        *ticket = 0;
        st->pAp = acc;
        st->alpha = st->rtz / acc;
    }
}

// r -= alpha Ap and ||r|| (x += alpha p runs in the next p update).
template <typename Z>
__global__ void __launch_bounds__(kReduceThreads) k_cg_update_r(int n, const double* __restrict__ Ap,
                                                                double* __restrict__ r, const Z* __restrict__ z,
                                                                CGState* st, ReduceScratch* ws)
{
    __shared__ double red[32];
    const double alpha = st->alpha;
    const bool flex = st->flexible != 0;
    double s = 0.0, sf = 0.0;
    for(long long i = (long long)blockIdx.x * kReduceThreads + threadIdx.x; i < n; i += kReduceBlocks * kReduceThreads)
    {
        const double v = fma(-alpha, Ap[i], r[i]);   // ComputeFusedWAXPBYDot(-alpha, Ap, r)
        r[i] = v;
        s = fma(v, v, s);
        if(flex) sf = fma((double)z[i], v, sf);
    }
    double t1, t2;
    bool last;
    if(flex)
    {
        s = block_sum(s, red);
        sf = block_sum(sf, red);
        last = grid_reduce2(s, sf, ws, kReduceBlocks, &t1, &t2);
    }
    else
    {
        s = block_sum(s, red);
        last = grid_reduce(s, ws, kReduceBlocks, &t1);
        t2 = 0.0;
    }
    if(last)
    {
        const double nr = sqrt(t1);
        st->normr = nr;
        st->rtz_flex = t2;
        st->hist[st->k] = nr;
    }
}

// Loop control of the device-resident CG, one thread: always advances k, so
// the WHILE node ends after at most max_iter iterations whatever the
// reductions produced.  src/CG.cpp:148: continue while k <= max_iter &&
// normr/normr0 > tol (a NaN residual compares false and ends the loop).
__device__ __forceinline__ void cg_loop_control(CGState* st, unsigned long long cond, int watch_net)
{
    const int k = st->k;
    st->niters = k;
    st->k = k + 1;
    const double nr = st->normr;
    if(nr < st->best_normr)
    {
        st->best_normr = nr;
        st->since_best = 0;
    }
    else
    {
        st->since_best += 1;
    }
    // learned smoother: fall back for good on a jump, a stall or a non-finite residual
    const bool slow = st->fb_rate > 0.0 && k >= st->fb_window && !(nr <= st->fb_rate * st->hist[k - st->fb_window]);
    const bool bad = !(nr <= st->fb_jump * st->hist[k - 1]) || st->since_best >= st->fb_stall || slow;
    if(st->net == 1 && bad)
    {
        st->net = 2;
        st->fallback_iter = k;
    }
    unsigned go = (k + 1 <= st->max_iter) && (st->normr / st->normr0 > st->tol);
    if(watch_net && st->net == 2) go = 0;
    if(cond) cudaGraphSetConditional((cudaGraphConditionalHandle)cond, go);
}

__global__ void k_cg_loop_control(CGState* st, unsigned long long cond, int watch_net)
{
    cg_loop_control(st, cond, watch_net);
}

// ------------------------------------------------------- two-kernel CG step
// src/CG.cpp:148-184 as two kernels.  Step 1 (persistent, cooperative):
// r.z over each block's row range, grid barrier, beta (every block sums the
// per-block partials in index order, so all agree), p = z + beta p, grid
// barrier, Ap = A p with the p.Ap partials, alpha from the last block.  Step
// 2: r -= alpha Ap, x += alpha p, ||r|| (and the flexible-CG term), the last
// block also running the loop control.  p is read and written through L2
// only in the p update, so no SM holds a stale line of it when the product
// gathers it after the barrier.

// Self-test of the bounded grid barrier: the blocks of a cooperative launch
// meet at one barrier; block `absent` (if >= 0) returns without arriving, so
// the others' waits run out (about a second) and set *status.
__global__ void k_barrier_selftest(GridBarrier* gb, int absent, int* status, int* passed)
{
    if((int)blockIdx.x == absent) return;
    const bool ok = grid_barrier(gb, gridDim.x, status);
    if(threadIdx.x == 0 && ok) atomicAdd(passed, 1);
}

// Step 1 with the ELL product (colour-interleaved chunks, one row per thread).
template <typename Z>
__global__ void __launch_bounds__(kBS) k_cg_step1_ell(int n, ColorChunks cc, const int* __restrict__ ell_col,
                                                      const double* __restrict__ ell_val, const double* __restrict__ r,
                                                      const Z* __restrict__ z, double* __restrict__ p,
                                                      double* __restrict__ x, double* __restrict__ Ap, CGState* st,
                                                      double* partial, unsigned int* ticket, GridBarrier* gb)
{
    if(!step1_rz_p(n, r, z, p, x, st, partial, gb)) return;
    double s = 0.0;
    for(int c = blockIdx.x; c < cc.nchunks(); c += gridDim.x)
    {
        int row;
        if(!cc.row_of(c, threadIdx.x, row)) continue;
        const double sum = spmv_row(n, row, ell_col, ell_val, p);
        Ap[row] = sum;
        s = fma(sum, p[row], s);
    }
    step1_alpha(s, st, partial, ticket);
}

// Step 2: the r update of k_cg_update_r with the loop control in its last block.
template <typename Z>
__global__ void __launch_bounds__(kReduceThreads) k_cg_step2(int n, const double* __restrict__ Ap,
                                                             double* __restrict__ r, const Z* __restrict__ z,
                                                             CGState* st, ReduceScratch* ws, unsigned long long cond,
                                                             int watch_net)
{
    __shared__ double red[32];
    const double alpha = st->alpha;
    const bool flex = st->flexible != 0;
    double s = 0.0, sf = 0.0;
    for(long long i = (long long)blockIdx.x * kReduceThreads + threadIdx.x; i < n; i += kReduceBlocks * kReduceThreads)
    {
        const double v = fma(-alpha, Ap[i], r[i]);
        r[i] = v;
        s = fma(v, v, s);
        if(flex) sf = fma((double)z[i], v, sf);
    }
    double t1, t2;
    bool last;
    if(flex)
    {
        s = block_sum(s, red);
        sf = block_sum(sf, red);
        last = grid_reduce2(s, sf, ws, kReduceBlocks, &t1, &t2);
    }
    else
    {
        s = block_sum(s, red);
        last = grid_reduce(s, ws, kReduceBlocks, &t1);
        t2 = 0.0;
    }
    if(last)
    {
        const double nr = sqrt(t1);
        st->normr = nr;
        st->rtz_flex = t2;
        st->hist[st->k] = nr;
        cg_loop_control(st, cond, watch_net);
    }
}

__global__ void k_cg_timer(CGState* st, int phase)
{
    unsigned long long now;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
    if(phase >= 0) st->phase_ns[phase] += (double)(now - st->t_last);
    st->t_last = now;
}

__global__ void k_cast_d2f(int n, const double* __restrict__ in, float* __restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i < n) out[i] = (float)in[i];
}

__global__ void k_cast_f2d(int n, const float* __restrict__ in, double* __restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i < n) out[i] = (double)in[i];
}

int launch_cg_residual0(int n, const double* b, const double* Ap, double* r, CGState* st, ReduceScratch* ws,
                        cudaStream_t s)
{
    k_cg_residual0<<<kReduceBlocks, kReduceThreads, 0, s>>>(n, b, Ap, r, st, ws);
    HB_LAUNCHED();
    return 0;
}

template <typename Z>
static int rtz_impl(int n, const double* r, const Z* z, CGState* st, ReduceScratch* ws, cudaStream_t s)
{
    k_cg_rtz<Z><<<kReduceBlocks, kReduceThreads, 0, s>>>(n, r, z, st, ws);
    HB_LAUNCHED();
    return 0;
}

int launch_cg_rtz(int n, const double* r, const double* z, CGState* st, ReduceScratch* ws, cudaStream_t s)
{
    return rtz_impl(n, r, z, st, ws, s);
}

int launch_cg_rtz(int n, const double* r, const float* z, CGState* st, ReduceScratch* ws, cudaStream_t s)
{
    return rtz_impl(n, r, z, st, ws, s);
}

int launch_cg_update_p(int n, const double* z, double* p, double* x, const CGState* st, cudaStream_t s)
{
    k_cg_update_p<double><<<(n + kBS - 1) / kBS, kBS, 0, s>>>(n, z, p, x, st);
    HB_LAUNCHED();
    return 0;
}

int launch_cg_update_p(int n, const float* z, double* p, double* x, const CGState* st, cudaStream_t s)
{
    k_cg_update_p<float><<<(n + kBS - 1) / kBS, kBS, 0, s>>>(n, z, p, x, st);
    HB_LAUNCHED();
    return 0;
}

int launch_cg_x_final(int n, const double* p, double* x, const CGState* st, cudaStream_t s)
{
    k_cg_x_final<<<(n + kBS - 1) / kBS, kBS, 0, s>>>(n, p, x, st);
    HB_LAUNCHED();
    return 0;
}

int launch_cg_spmv_pap(int m, const ColorChunks& cc, const int* ell_col, const double* ell_val, const double* p,
                       double* Ap, CGState* st, double* partial, unsigned int* ticket, cudaStream_t s)
{
    k_cg_spmv_pap<<<cc.nchunks(), kBS, 0, s>>>(m, cc, ell_col, ell_val, p, Ap, st, partial, ticket);
    HB_LAUNCHED();
    return 0;
}

int launch_cg_pap_chunks(int m, const ColorChunks& cc, const double* p, const double* Ap, CGState* st,
                         double* partial, unsigned int* ticket, cudaStream_t s)
{
    (void)m;
    k_cg_pap_chunks<<<cc.nchunks(), kBS, 0, s>>>(cc, p, Ap, st, partial, ticket);
    HB_LAUNCHED();
    return 0;
}

template <typename Z>
static int update_r_impl(int n, const double* Ap, double* r, const Z* z, CGState* st, ReduceScratch* ws,
                         unsigned long long cond, int watch_net, cudaStream_t s)
{
    k_cg_update_r<Z><<<kReduceBlocks, kReduceThreads, 0, s>>>(n, Ap, r, z, st, ws);
    HB_LAUNCHED();
    k_cg_loop_control<<<1, 1, 0, s>>>(st, cond, watch_net);
    HB_LAUNCHED();
    return 0;
}

int launch_cg_update_r(int n, const double* Ap, double* r, const double* z, CGState* st, ReduceScratch* ws,
                       unsigned long long cond, int watch_net, cudaStream_t s)
{
    return update_r_impl(n, Ap, r, z, st, ws, cond, watch_net, s);
}

int launch_cg_update_r(int n, const double* Ap, double* r, const float* z, CGState* st, ReduceScratch* ws,
                       unsigned long long cond, int watch_net, cudaStream_t s)
{
    return update_r_impl(n, Ap, r, z, st, ws, cond, watch_net, s);
}

// ---- two-kernel CG step
template <typename Z>
static int step1_ell_impl(int n, const ColorChunks& cc, const int* ell_col, const double* ell_val, const double* r,
                          const Z* z, double* p, double* x, double* Ap, CGState* st, ReduceScratch* ws,
                          GridBarrier* gb, cudaStream_t s)
{
    static const int grid = resident_grid(k_cg_step1_ell<Z>, kBS, kReduceBlocks);
    if(grid <= 0) return record_error(HPCGB200_ERR_CUDA, "CG step: no resident grid");
    HB_CUDA(launch_coop(k_cg_step1_ell<Z>, grid, kBS, s, n, cc, ell_col, ell_val, r, z, p, x, Ap, st, ws->partial,
                        &ws->ticket, gb));
    return 0;
}

int launch_cg_step1_ell(int n, const ColorChunks& cc, const int* ell_col, const double* ell_val, const double* r,
                        const double* z, double* p, double* x, double* Ap, CGState* st, ReduceScratch* ws,
                        GridBarrier* gb, cudaStream_t s)
{
    return step1_ell_impl(n, cc, ell_col, ell_val, r, z, p, x, Ap, st, ws, gb, s);
}

template <typename Z>
static int step2_impl(int n, const double* Ap, double* r, const Z* z, CGState* st, ReduceScratch* ws,
                      unsigned long long cond, int watch_net, cudaStream_t s)
{
    k_cg_step2<Z><<<kReduceBlocks, kReduceThreads, 0, s>>>(n, Ap, r, z, st, ws, cond, watch_net);
    HB_LAUNCHED();
    return 0;
}

int launch_cg_step2(int n, const double* Ap, double* r, const double* z, CGState* st, ReduceScratch* ws,
                    unsigned long long cond, int watch_net, cudaStream_t s)
{
    return step2_impl(n, Ap, r, z, st, ws, cond, watch_net, s);
}

int launch_cg_step2(int n, const double* Ap, double* r, const float* z, CGState* st, ReduceScratch* ws,
                    unsigned long long cond, int watch_net, cudaStream_t s)
{
    return step2_impl(n, Ap, r, z, st, ws, cond, watch_net, s);
}

int launch_cg_timer(CGState* st, int phase, cudaStream_t s)
{
    k_cg_timer<<<1, 1, 0, s>>>(st, phase);
    HB_LAUNCHED();
    return 0;
}

int launch_cast_d2f(int n, const double* in, float* out, cudaStream_t s)
{
    k_cast_d2f<<<(n + 255) / 256, 256, 0, s>>>(n, in, out);
    HB_LAUNCHED();
    return 0;
}

int launch_cast_f2d(int n, const float* in, double* out, cudaStream_t s)
{
    k_cast_f2d<<<(n + 255) / 256, 256, 0, s>>>(n, in, out);
    HB_LAUNCHED();
    return 0;
}

}  // namespace hb

using namespace hb;

// ------------------------------------------------------------------ C ABI

extern "C" int hpcgb200_selftest_grid_barrier(int absent_block, int* status, int* passed, int* blocks)
{
    HB_CHECK_ARG(status && passed && blocks, "null argument");
    const int grid = resident_grid(k_barrier_selftest, 128, 2 * 148);
    if(grid <= 0) return record_error(HPCGB200_ERR_CUDA, "no resident grid");
    HB_CHECK_ARG(absent_block < grid, "absent_block beyond the grid");
    struct Scratch
    {
        GridBarrier gb;
        int status, passed;
    };
    Scratch* d = nullptr;
    HB_CUDA(cudaMalloc(&d, sizeof(Scratch)));
    int rc = 0;
    cudaError_t e = cudaMemset(d, 0, sizeof(Scratch));
    if(e == cudaSuccess) e = launch_coop(k_barrier_selftest, grid, 128, nullptr, &d->gb, absent_block, &d->status,
                                         &d->passed);
    if(e == cudaSuccess) e = cudaDeviceSynchronize();
    Scratch h{};
    if(e == cudaSuccess) e = cudaMemcpy(&h, d, sizeof(Scratch), cudaMemcpyDeviceToHost);
    if(e != cudaSuccess) rc = cuda_error(e, "grid barrier self-test", __FILE__, __LINE__);
    cudaFree(d);
    *status = h.status;
    *passed = h.passed;
    *blocks = grid;
    return rc;
}
