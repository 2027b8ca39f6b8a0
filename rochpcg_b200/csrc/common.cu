// Error recording and small exported helpers of libhpcgb200.
#include <cstdarg>
#include <cstdio>

#include "common.cuh"

namespace hb {

static thread_local char g_last_error[512] = "";

int record_error(int code, const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
    return code;
}

int cuda_error(cudaError_t e, const char* what, const char* file, int line)
{
    const char* base = file;
    for(const char* c = file; *c; ++c)
        if(*c == '/') base = c + 1;
    return record_error(HPCGB200_ERR_CUDA, "CUDA error %d (%s) in %s at %s:%d", (int)e, cudaGetErrorString(e), what,
                        base, line);
}

}  // namespace hb

extern "C" const char* hpcgb200_last_error(void) { return hb::g_last_error; }

extern "C" const char* hpcgb200_version(void) { return "hpcg-b200 0.1 (sm_100a)"; }

extern "C" size_t hpcgb200_reduction_workspace_bytes(void) { return sizeof(hb::ReduceScratch); }
