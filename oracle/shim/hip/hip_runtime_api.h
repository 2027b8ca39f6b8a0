/*
 * Host-only stand-in for the HIP runtime header, used ONLY to compile the
 * reference's CPU (`*_ref.cpp`) sources into the test oracle under
 * oracle/_ref/.  The reference headers (Vector.hpp, SparseMatrix.hpp,
 * utils.hpp, Memory.hpp) include <hip/hip_runtime_api.h> for a handful of
 * type names and inline helpers; none of the CPU reference kernels issue a
 * HIP call.  Every function here is a no-op that reports success.
 *
 * This file is test infrastructure: nothing in the product library includes it.
 */
#ifndef HPCG_ORACLE_HIP_SHIM_H
#define HPCG_ORACLE_HIP_SHIM_H

#include <stddef.h>

typedef int hipError_t;
enum { hipSuccess = 0 };
typedef void* hipStream_t;
typedef void* hipEvent_t;
typedef enum {
    hipMemcpyHostToHost = 0,
    hipMemcpyHostToDevice = 1,
    hipMemcpyDeviceToHost = 2,
    hipMemcpyDeviceToDevice = 3,
    hipMemcpyDefault = 4
} hipMemcpyKind;

static inline const char* hipGetErrorString(hipError_t) { return "hip shim (no device)"; }
static inline hipError_t hipMemcpy(void*, const void*, size_t, hipMemcpyKind) { return hipSuccess; }
static inline hipError_t hipMemcpyAsync(void*, const void*, size_t, hipMemcpyKind, hipStream_t)
{
    return hipSuccess;
}
static inline hipError_t hipMemsetAsync(void*, int, size_t, hipStream_t) { return hipSuccess; }
static inline hipError_t hipHostUnregister(void*) { return hipSuccess; }

#endif
