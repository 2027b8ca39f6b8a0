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
