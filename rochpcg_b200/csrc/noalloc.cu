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
//    cudaGetSymbolAddress (once per CUDA context, with that device current);
//    make that first call before any stream capture.
//  * The result is deterministic for a given n (the tile count follows n),
//    but its summation order differs from hpcgb200_dot's fixed 1184-block
//    grid, so the two agree to rounding, not bit for bit.
//  * No cudaMalloc / cudaFree or allocating library call is made.
#include <cuda.h>

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

// The array's address belongs to the module instance loaded into one CUDA
// context.  It is cached per context (the driver's unique context id), not
// per device index: after cudaDeviceReset, or under a caller's own driver-API
// context, the current context is a different one and gets its own lookup,
// so a cached address never outlives the module it points into.
using PfnCtxGetCurrent = CUresult (*)(CUcontext*);
using PfnCtxGetId = CUresult (*)(CUcontext, unsigned long long*);

constexpr int kMaxContexts = 64;
std::mutex g_mu;
unsigned long long g_ctx_id[kMaxContexts] = {};
NoAllocScratch* g_addr[kMaxContexts] = {};
int g_cached = 0;

// Unique id of the calling thread's current context (false if there is none
// yet or the driver does not report ids; the caller then looks the address up
// without caching it).
bool current_context_id(unsigned long long* id)
{
    static PfnCtxGetCurrent get_current = nullptr;
    static PfnCtxGetId get_id = nullptr;
    static bool resolved = false;
    if(!resolved)
    {
        void* f1 = nullptr;
        void* f2 = nullptr;
        cudaDriverEntryPointQueryResult q1{}, q2{};
        if(cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) == cudaSuccess &&
           q1 == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<PfnCtxGetCurrent>(f1);
        if(cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) == cudaSuccess &&
           q2 == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<PfnCtxGetId>(f2);
        resolved = true;
    }
    if(!get_current || !get_id) return false;
    CUcontext ctx = nullptr;
    if(get_current(&ctx) != CUDA_SUCCESS || ctx == nullptr) return false;
    return get_id(ctx, id) == CUDA_SUCCESS;
}

// Device address of the array in the current context: looked up once per
// context with that context's device current (the first call on a device).
int scratch_address(NoAllocScratch** out)
{
    std::lock_guard<std::mutex> lock(g_mu);
    unsigned long long id = 0;
    if(current_context_id(&id))
        for(int i = 0; i < g_cached; ++i)
            if(g_ctx_id[i] == id)
            {
                *out = g_addr[i];
                return 0;
            }
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if(e != cudaSuccess || p == nullptr)
        return cuda_error(e, "cudaGetSymbolAddress(g_noalloc_scratch)", __FILE__, __LINE__);
    // the lookup above creates the primary context if there was none yet
    if(current_context_id(&id) && g_cached < kMaxContexts)
    {
        g_ctx_id[g_cached] = id;
        g_addr[g_cached] = static_cast<NoAllocScratch*>(p);
        ++g_cached;
    }
    *out = static_cast<NoAllocScratch*>(p);
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
