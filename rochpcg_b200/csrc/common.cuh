// Shared definitions for the sm_100a kernels of libhpcgb200.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdlib.h>

#include <utility>

#include "hpcg_b200.h"

namespace hb {

constexpr int kWidth = HPCGB200_WIDTH;  // ELL width of the 27-point stencil

// Fixed reduction shape: results do not depend on the device or on timing,
// so every dot product is bit-reproducible run to run.
constexpr int kReduceBlocks = 1184;  // 8 x 148 SMs
constexpr int kReduceThreads = 256;

// Reduction scratch: partial sums then one ticket counter.
struct ReduceScratch
{
    double partial[kReduceBlocks];
    double partial2[kReduceBlocks];  // second sum of two-value reductions
    unsigned int ticket;
    unsigned int pad[3];
};

int record_error(int code, const char* fmt, ...);
int cuda_error(cudaError_t e, const char* what, const char* file, int line);

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Prolongation fused into a coarse level's smoother: the pass that gives a
// row its final value of the coarse solve also adds it into the finer level,
// xf[pro_f[row]] += x_new -- what src/ComputeProlongation.cpp:39-59 does
// after the coarse level returns (the fine vector is not touched while the
// coarse level runs, and each coarse row has one injected fine row).
// xf == nullptr: this pass does no prolongation.
template <typename T>
struct Prolong
{
    T* xf = nullptr;
    const int* pro_f = nullptr;  // coarse permuted row -> fine permuted row
    __device__ __forceinline__ void add(int row, T v) const
    {
        if(xf) xf[pro_f[row]] += v;
    }
    // four consecutive rows (row0 % 4 == 0)
    __device__ __forceinline__ void add4(int row0, const T (&v)[4]) const
    {
        if(!xf) return;
        const int4 f = *reinterpret_cast<const int4*>(pro_f + row0);
        xf[f.x] += v[0];
        xf[f.y] += v[1];
        xf[f.z] += v[2];
        xf[f.w] += v[3];
    }
};

// ---- programmatic dependent launch
// launch_pdl() starts a kernel whose blocks may become resident while the
// previous kernel of the stream is still finishing (once every block of that
// kernel is resident or done), which hides the gap between the short kernels
// of a V-cycle launched one by one (320^3 mixed V-cycle: 1.60 -> 1.43 ms).
// Such a kernel calls pdl_begin() before it touches memory.  Inside stream
// capture the attribute is left off: a graph already launches its kernels
// back to back, and there it cost 2 % (1.37 -> 1.39 ms).  HPCGB200_PDL=0 in
// the environment turns it off everywhere.
inline bool pdl_enabled()
{
    static const bool on = [] {
        const char* e = getenv("HPCGB200_PDL");
        return !(e && e[0] == '0');
    }();
    return on;
}

template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, cudaStream_t s, Args&&... args)
{
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cfg.attrs = attr;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    const bool capturing = cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone;
    cfg.numAttrs = pdl_enabled() && !capturing ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// launch_pdl() with dynamic shared memory.
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl_smem(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                                   Args&&... args)
{
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cfg.attrs = attr;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    const bool capturing = cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone;
    cfg.numAttrs = pdl_enabled() && !capturing ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// Programmatic dependent launch for the learned smoother's kernels, inside
// graphs too: each of them starts its dependents at entry, runs its prologue
// (weights to shared memory, barriers, tensor memory) while the previous
// kernel finishes, and waits (pdl_wait) before it touches that kernel's
// output.  256^3 learned V-cycle 0.784 -> 0.773 ms, solve 0.178 -> 0.176 s
// (A/B on one box); HPCGB200_NET_PDL=0 turns it off.
inline bool net_pdl_enabled()
{
    static const bool on = [] {
        const char* e = getenv("HPCGB200_NET_PDL");
        return !(e && e[0] == '0');
    }();
    return on;
}

template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl_net(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                                  Args&&... args)
{
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = net_pdl_enabled() ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// Cooperative launch (every block resident at once, or the launch fails):
// for the persistent kernels whose blocks meet at grid barriers.  Valid in
// stream capture (the graph's kernel node keeps the attribute).
template <typename... KArgs, typename... Args>
inline cudaError_t launch_coop(void (*kernel)(KArgs...), unsigned grid, unsigned block, cudaStream_t s,
                               Args&&... args)
{
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// Blocks of `kernel` that fit on the device at once (SMs x resident blocks
// per SM), at most `cap`.
template <typename K>
inline int resident_grid(K kernel, int block, int cap)
{
    int dev = 0, sms = 0, per = 0;
    if(cudaGetDevice(&dev) != cudaSuccess) return 0;
    if(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    if(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, block, 0) != cudaSuccess) return 0;
    const int g = sms * per;
    return g < cap ? g : cap;
}

}  // namespace hb

#define HB_CUDA(call)                                                           \
    do                                                                          \
    {                                                                           \
        cudaError_t hb_e_ = (call);                                             \
        if(hb_e_ != cudaSuccess) return hb::cuda_error(hb_e_, #call, __FILE__, __LINE__); \
    } while(0)

#define HB_LAUNCHED() HB_CUDA(cudaGetLastError())

#define HB_CHECK_ARG(cond, msg)                                                 \
    do                                                                          \
    {                                                                           \
        if(!(cond)) return hb::record_error(HPCGB200_ERR_ARG, "%s: %s", __func__, msg); \
    } while(0)

#define HB_RETURN_IF(err)       \
    do                          \
    {                           \
        int hb_r_ = (err);      \
        if(hb_r_ != 0) return hb_r_; \
    } while(0)

// ---------------------------------------------------------------- device helpers

namespace hb {

// First statement of a kernel started by launch_pdl(): wait until the
// previous kernel of the stream has completed and its writes are visible,
// then let the next kernel's blocks start (they wait in turn).  Both are
// no-ops for a kernel launched without the attribute.
__device__ __forceinline__ void pdl_begin()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// The two halves of pdl_begin() for kernels with a prologue that does not
// read the previous kernel's output (no-ops without the launch attribute).
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Streaming (read-once) loads for matrix data: evict-first in L2 so that the
// vectors gathered by the stencil stay resident.
__device__ __forceinline__ int ld_stream(const int* p) { return __ldcs(p); }
__device__ __forceinline__ double ld_stream(const double* p) { return __ldcs(p); }
__device__ __forceinline__ float ld_stream(const float* p) { return __ldcs(p); }

template <typename T>
__device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
    for(int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <typename T>
__device__ __forceinline__ T warp_max(T v)
{
#pragma unroll
    for(int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Linear thread index and size of the block (1-D, 2-D and 3-D blocks).
__device__ __forceinline__ int block_tid()
{
    return (int)(threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z));
}
__device__ __forceinline__ int block_threads() { return (int)(blockDim.x * blockDim.y * blockDim.z); }

// Block-wide sum (block size a multiple of 32, <= 1024); result valid in the
// thread with block_tid() == 0.
template <typename T>
__device__ __forceinline__ T block_sum(T v, T* smem /* >= 32 */)
{
    const int tid = block_tid();
    const int lane = tid & 31, warp = tid >> 5;
    v = warp_sum(v);
    if(lane == 0) smem[warp] = v;
    __syncthreads();
    const int nw = block_threads() >> 5;
    T r = (tid < nw) ? smem[tid] : T(0);
    if(warp == 0) r = warp_sum(r);
    __syncthreads();
    return r;
}

template <typename T>
__device__ __forceinline__ T block_max(T v, T* smem)
{
    const int tid = block_tid();
    const int lane = tid & 31, warp = tid >> 5;
    v = warp_max(v);
    if(lane == 0) smem[warp] = v;
    __syncthreads();
    const int nw = block_threads() >> 5;
    T r = (tid < nw) ? smem[tid] : T(0);
    if(warp == 0) r = warp_max(r);
    __syncthreads();
    return r;
}

// Two-level deterministic reduction epilogue.  Every block of a kernel with
// gridDim.x == nblocks calls this with its block's partial (valid in thread
// 0).  Returns true in thread 0 of the LAST block to arrive, which then holds
// the total in *total (summed over partials in index order).  The ticket is
// reset for the next launch.
template <bool kMax = false>
__device__ __forceinline__ bool grid_reduce(double block_partial, ReduceScratch* ws, int nblocks, double* total)
{
    __shared__ bool last;
    __shared__ double red[32];
    if(threadIdx.x == 0)
    {
        ws->partial[blockIdx.x] = block_partial;
        __threadfence();
        const unsigned int t = atomicAdd(&ws->ticket, 1u);
        last = (t == (unsigned)nblocks - 1);
    }
    __syncthreads();
    if(!last) return false;
    __threadfence();
    double acc = kMax ? 0.0 : 0.0;
    for(int i = threadIdx.x; i < nblocks; i += blockDim.x)
    {
        const double v = __ldcg(&ws->partial[i]);
        acc = kMax ? fmax(acc, v) : acc + v;
    }
    acc = kMax ? block_max(acc, red) : block_sum(acc, red);
    if(threadIdx.x == 0)
    {
        ws->ticket = 0;
        *total = acc;
    }
    return threadIdx.x == 0;
}

// Grid-wide barrier of a persistent kernel launched cooperatively (every
// block resident).  Generation counting: a block reads the generation, then
// arrives; the last to arrive resets the count and bumps the generation; the
// others wait for the bump.  The wait is bounded by time (one second of the
// global timer, and an iteration cap besides): on time-out it sets *status
// and returns false, so a kernel whose blocks cannot all arrive ends with an
// error instead of hanging.  Starts and ends with count == 0.
struct GridBarrier
{
    unsigned int count;
    unsigned int gen;
};

constexpr unsigned long long kBarrierTimeoutNs = 1000000000ull;
constexpr long long kBarrierSpins = 1ll << 26;

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ bool grid_barrier(GridBarrier* gb, unsigned int nblocks, int* status)
{
    __shared__ int ok;
    __syncthreads();
    if(threadIdx.x == 0)
    {
        ok = 1;
        volatile unsigned int* gen = &gb->gen;
        const unsigned int g = *gen;
        __threadfence();
        if(atomicAdd(&gb->count, 1u) == nblocks - 1)
        {
            gb->count = 0;
            __threadfence();
            atomicAdd(&gb->gen, 1u);
        }
        else
        {
            const unsigned long long t0 = global_ns();
            long long spins = 0;
            while(*gen == g)
            {
                if(++spins > kBarrierSpins || global_ns() - t0 > kBarrierTimeoutNs)
                {
                    atomicExch(status, 1);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return ok != 0;
}

// Two sums at once (same protocol as grid_reduce).
__device__ __forceinline__ bool grid_reduce2(double a, double b, ReduceScratch* ws, int nblocks, double* ta,
                                             double* tb)
{
    __shared__ bool last;
    __shared__ double red[32];
    if(threadIdx.x == 0)
    {
        ws->partial[blockIdx.x] = a;
        ws->partial2[blockIdx.x] = b;
        __threadfence();
        const unsigned int t = atomicAdd(&ws->ticket, 1u);
        last = (t == (unsigned)nblocks - 1);
    }
    __syncthreads();
    if(!last) return false;
    __threadfence();
    double sa = 0.0, sb = 0.0;
    for(int i = threadIdx.x; i < nblocks; i += blockDim.x)
    {
        sa += __ldcg(&ws->partial[i]);
        sb += __ldcg(&ws->partial2[i]);
    }
    sa = block_sum(sa, red);
    sb = block_sum(sb, red);
    if(threadIdx.x == 0)
    {
        ws->ticket = 0;
        *ta = sa;
        *tb = sb;
    }
    return threadIdx.x == 0;
}

}  // namespace hb
