// Tensor-memory-access (TMA) helpers for the stencil kernels: an mbarrier
// that counts the bytes of bulk tensor copies, a bounded wait on it, and a
// tiled 3-D load into this CTA's shared memory (no multicast: every copy
// reads this GPU's own memory into its own CTA).
#pragma once

#include <cuda.h>
#include <cstdint>

namespace hb {
namespace tma {

// try_wait rounds before a wait gives up (each round may suspend the thread
// for a while, so this is well beyond any healthy copy).
constexpr uint32_t kSpinLimit = 1u << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// The one arrival of the phase, announcing `bytes` of copies that complete on it.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* mbar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(mbar)), "r"(bytes)
                 : "memory");
}

// Bounded wait for the completion of phase `parity`; false on time-out.
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity)
{
    const uint32_t a = smem_u32(mbar);
    for(uint32_t i = 0; i < kSpinLimit; ++i)
    {
        uint32_t done;
        asm volatile(
            "{\n\t"
            ".reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t"
            "}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if(done) return true;
    }
    return false;
}

// Tiled 3-D box at (c0, c1, c2) of `map` into shared memory at dst (128-byte
// aligned), completing on mbar.  c0 * element size must be a multiple of 16
// bytes; coordinates outside the tensor read as zero.
__device__ __forceinline__ void load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, uint64_t* mbar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(mbar)), "r"(c0), "r"(c1), "r"(c2)
        : "memory");
}

}  // namespace tma
}  // namespace hb
