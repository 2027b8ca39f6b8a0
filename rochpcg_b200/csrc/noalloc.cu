// hpcgb200_dot_noalloc: the dot product for callers that cannot allocate
// device memory.
//
// Who needs it: code that runs inside a host application which owns all
// device memory through its own pool (a framework's caching allocator, an
// embedded solver plugin with a fixed budget) and forbids cudaMalloc behind
// its back, and latency-critical callers for whom cudaMalloc is not an option
// because it can synchronize the device.  hpcgb200_dot needs a caller-provided
// workspace; this variant needs none: its scratch is one file-scope device
// array, loaded with the library and kept by every GPU that loads it until the
// process exits.
//
// Limits and sharing:
//  * The array holds kNoAllocMaxTiles partial sums, one per tile of
//    kNoAllocTile elements, so n <= kNoAllocMaxTiles * kNoAllocTile =
//    16,777,216 (one 256^3 level-0 vector); larger n is rejected.
//  * Every call, on every stream, uses the same array.  Calls whose kernels
//    overlap on the GPU race on it: serialize them (one stream, or events).
//  * The first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (once per device, with that device current); make
//    that first call before any stream capture.
//  * No cudaMalloc / cudaFree or allocating library call is made.
#include <mutex>

#include "common.cuh"

namespace hb {

constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocTile = kNoAllocThreads * 16;  // elements reduced by one block
constexpr int kNoAllocMaxTiles = 4096;               // partial sums the array holds
constexpr long long kNoAllocMaxN = (long long)kNoAllocTile * kNoAllocMaxTiles;

struct NoAllocScratch
{
    double partial[kNoAllocMaxTiles];
    unsigned int ticket;
};

// 32 KB + 4 B per device.  Zero at load; the ticket is cleared before every
// launch, the partial sums are fully written by each launch before use.
static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

// One block per tile, no grid-stride loop: the tile count is the grid size
// and bounds the scratch it needs.  The last block to finish sums the
// partials in index order (deterministic for a given n).
__global__ void __launch_bounds__(kNoAllocThreads) k_dot_noalloc(long long n, const double* __restrict__ x,
                                                                 const double* __restrict__ y, NoAllocScratch* ws,
                                                                 double* result)
{
    __shared__ double red[32];
    __shared__ bool last;
    const long long base = (long long)blockIdx.x * kNoAllocTile;
    double s = 0.0;
    for(int k = threadIdx.x; k < kNoAllocTile; k += kNoAllocThreads)
    {
        const long long i = base + k;
        if(i < n) s = fma(y[i], x[i], s);
    }
    s = block_sum(s, red);
    if(threadIdx.x == 0)
    {
        ws->partial[blockIdx.x] = s;
        __threadfence();
        last = atomicAdd(&ws->ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if(!last) return;
    __threadfence();
    double acc = 0.0;
    for(int i = threadIdx.x; i < (int)gridDim.x; i += kNoAllocThreads) acc += __ldcg(&ws->partial[i]);
    acc = block_sum(acc, red);
    if(threadIdx.x == 0)
    {
        ws->ticket = 0;
        *result = acc;
    }
}

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_mu;
NoAllocScratch* g_addr[kMaxDevices] = {};

// Device address of the array on the current device, looked up once.
int scratch_address(NoAllocScratch** out)
{
    int dev = -1;
    HB_CUDA(cudaGetDevice(&dev));
    if(dev < 0 || dev >= kMaxDevices) return record_error(HPCGB200_ERR_ARG, "device index %d unsupported", dev);
    std::lock_guard<std::mutex> lock(g_mu);
    if(!g_addr[dev])
    {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if(e != cudaSuccess || p == nullptr) return cuda_error(e, "cudaGetSymbolAddress(g_noalloc_scratch)", __FILE__, __LINE__);
        g_addr[dev] = static_cast<NoAllocScratch*>(p);
    }
    *out = g_addr[dev];
    return 0;
}

}  // namespace

}  // namespace hb

using namespace hb;

extern "C" int hpcgb200_dot_noalloc(long long n, const double* x, const double* y, double* result, void* stream)
{
    HB_CHECK_ARG(n >= 0 && x && y && result, "bad arguments");
    if(n > kNoAllocMaxN)
        return record_error(HPCGB200_ERR_ARG,
                            "hpcgb200_dot_noalloc: n = %lld exceeds the fixed scratch maximum of %lld elements "
                            "(use hpcgb200_dot with a workspace)",
                            n, kNoAllocMaxN);
    NoAllocScratch* ws = nullptr;
    HB_RETURN_IF(scratch_address(&ws));
    cudaStream_t s = as_stream(stream);
    HB_CUDA(cudaMemsetAsync(&ws->ticket, 0, sizeof(unsigned int), s));
    if(n == 0)
    {
        HB_CUDA(cudaMemsetAsync(result, 0, sizeof(double), s));
        return 0;
    }
    const unsigned tiles = (unsigned)((n + kNoAllocTile - 1) / kNoAllocTile);
    k_dot_noalloc<<<tiles, kNoAllocThreads, 0, s>>>(n, x, y, ws, result);
    HB_LAUNCHED();
    return 0;
}
