// Process-wide runtime (stream, reduction scratch) and vector helpers.
// Mirrors the reference's globals stream_interior / workspace
// (src/utils.hpp:38-45, created in src/init.cpp:200-230) and the vector
// helpers of src/Vector.hpp / src/CGData.hpp.
#include <cstdlib>
#include <cstring>

#include "hpcg_b200.h"
#include "internal.hpp"

namespace hpcg_b200 {

static Runtime g_rt;

Runtime& rt() { return g_rt; }

void throw_last(int code) { throw Error(code, hpcgb200_last_error()); }

void check_cuda(cudaError_t e, const char* what)
{
    if(e != cudaSuccess)
    {
        char buf[256];
        snprintf(buf, sizeof(buf), "CUDA error %d (%s) in %s", (int)e, cudaGetErrorString(e), what);
        throw Error(HPCGB200_ERR_CUDA, buf);
    }
}

void dfree(void* p)
{
    if(p) cudaFree(p);
}

void ensure_runtime()
{
    if(g_rt.initialized) return;
    int n = 0;
    if(cudaGetDeviceCount(&n) != cudaSuccess || n == 0)
        throw Error(HPCGB200_ERR_NO_DEVICE, "no CUDA device visible (libhpcgb200 has no CPU fallback)");
    HB_HOST_CUDA(cudaGetDevice(&g_rt.device));
    HB_HOST_CUDA(cudaStreamCreateWithFlags(&g_rt.stream, cudaStreamNonBlocking));
    void* p = nullptr;
    HB_HOST_CUDA(cudaMalloc(&p, sizeof(hb::ReduceScratch)));
    HB_HOST_CUDA(cudaMemset(p, 0, sizeof(hb::ReduceScratch)));
    g_rt.ws = static_cast<hb::ReduceScratch*>(p);
    HB_HOST_CUDA(cudaMalloc(&g_rt.d_scalar, 16 * sizeof(double)));
    HB_HOST_CUDA(cudaMallocHost(&g_rt.h_scalar, 16 * sizeof(double)));
    g_rt.initialized = true;
}

}  // namespace hpcg_b200

using namespace hpcg_b200;

int HPCG_B200_Init(int device)
{
    try
    {
        if(g_rt.initialized) return 0;
        if(device >= 0) HB_HOST_CUDA(cudaSetDevice(device));
        ensure_runtime();
        return 0;
    }
    catch(const Error& e)
    {
        return report(e);
    }
}

extern "C" int hpcgb200_init(int device)
{
    try
    {
        if(g_rt.initialized)
        {
            if(device >= 0 && device != g_rt.device)
                return hb::record_error(HPCGB200_ERR_ARG, "the library runtime is bound to device %d already",
                                        g_rt.device);
            return 0;
        }
        int n = 0;
        if(cudaGetDeviceCount(&n) != cudaSuccess || n == 0)
            return hb::record_error(HPCGB200_ERR_NO_DEVICE, "no CUDA device visible");
        if(device >= n) return hb::record_error(HPCGB200_ERR_ARG, "device %d out of range (%d visible)", device, n);
        if(device >= 0) HB_HOST_CUDA(cudaSetDevice(device));
        ensure_runtime();
        return 0;
    }
    catch(const Error& e)
    {
        return report(e);
    }
}

cudaStream_t HPCG_B200_Stream()
{
    ensure_runtime();
    return g_rt.stream;
}

void HPCG_B200_SetStream(cudaStream_t s)
{
    ensure_runtime();
    g_rt.stream = s;
}

int HPCG_B200_Finalize()
{
    if(!g_rt.initialized) return 0;
    cudaStreamSynchronize(g_rt.stream);
    dfree(g_rt.ws);
    dfree(g_rt.d_scalar);
    if(g_rt.h_scalar) cudaFreeHost(g_rt.h_scalar);
    g_rt = Runtime{};
    return 0;
}

void CudaInitializeVector(Vector& v, local_int_t localLength)
{
    ensure_runtime();
    v.localLength = localLength;
    v.optimizationData = nullptr;
    v.d_values = dalloc<double>(localLength);
}

void CudaDeleteVector(Vector& v)
{
    dfree(v.d_values);
    v.d_values = nullptr;
    if(v.values) delete[] v.values;
    v.values = nullptr;
    v.localLength = 0;
}

void CudaZeroVector(Vector& v)
{
    ensure_runtime();
    HB_HOST_CUDA(cudaMemsetAsync(v.d_values, 0, sizeof(double) * v.localLength, g_rt.stream));
}

void CudaCopyVector(const Vector& v, Vector& w)
{
    ensure_runtime();
    HB_HOST_CUDA(cudaMemcpyAsync(w.d_values, v.d_values, sizeof(double) * v.localLength, cudaMemcpyDeviceToDevice,
                                 g_rt.stream));
}

void CudaFillRandomVector(Vector& v)
{
    ensure_runtime();
    std::vector<double> h(v.localLength);
    for(local_int_t i = 0; i < v.localLength; ++i) h[i] = rand() / (double)(RAND_MAX) + 1.0;
    HB_HOST_CUDA(cudaMemcpyAsync(v.d_values, h.data(), sizeof(double) * v.localLength, cudaMemcpyHostToDevice,
                                 g_rt.stream));
    HB_HOST_CUDA(cudaStreamSynchronize(g_rt.stream));
}

void CudaInitializeSparseCGData(SparseMatrix& A, CGData& data)
{
    CudaInitializeVector(data.r, A.localNumberOfRows);
    CudaInitializeVector(data.z, A.localNumberOfColumns);
    CudaInitializeVector(data.p, A.localNumberOfColumns);
    CudaInitializeVector(data.Ap, A.localNumberOfRows);
}

void CudaDeleteCGData(CGData& data)
{
    CudaDeleteVector(data.r);
    CudaDeleteVector(data.z);
    CudaDeleteVector(data.p);
    CudaDeleteVector(data.Ap);
}

void CudaCopyMatrixDiagonal(const SparseMatrix& A, Vector& diagonal)
{
    ensure_runtime();
    check(hpcgb200_copy_diagonal(A.localNumberOfRows, A.ell_col_ind, A.ell_val, diagonal.d_values, g_rt.stream));
}

void CudaReplaceMatrixDiagonal(SparseMatrix& A, const Vector& diagonal)
{
    ensure_runtime();
    LevelOpt* o = opt(A);
    check(hpcgb200_replace_diagonal(A.localNumberOfRows, diagonal.d_values, A.ell_col_ind, A.ell_val, A.inv_diag,
                                    o ? o->diag : nullptr, g_rt.stream));
    if(o && o->diag32) check(hb::launch_diag32(A.localNumberOfRows, o->diag, o->diag32, o->inv_diag32, g_rt.stream));
}

void ExchangeHalo(const SparseMatrix&, Vector&)
{
    // One rank: no neighbours, nothing to exchange (src/ExchangeHalo.cpp:67).
}
