// Learned smoother kernels on the 5th-generation tensor cores (tcgen05).  No
// reference counterpart: the conv-net smoother is new in this library.
//
// Forward / input-gradient convolution (k_conv16).  Every layer runs as a
// 16 -> 16 channel 3x3x3 convolution (layer 1 has one real input channel and
// layer 3 one real output channel, the other weights are zero), so one kernel
// serves the forward pass and the input gradient (the transposed convolution
// is a convolution with mirrored taps and swapped channels).  A CTA owns a
// brick of 16 x 8 x 2 points = two 128-row M tiles (one per z plane) and
// stages the brick's halo once, as three copies shifted by dx = -1, 0, +1.
// Each copy keeps one 16-byte row (8 BF16 channels) per point, the two
// channel halves in separate regions, so in the no-swizzle K-major operand
// layout every 8-row core matrix is contiguous and consecutive rows are 16
// bytes apart.  A tap (dz, dy, dx) is then only a start-address offset into
// copy dx: 27 taps x 2 tiles = 54 tcgen05.mma (M=128, N=16, K=16) accumulate
// the brick's outputs in 32 TMEM columns, read back with tcgen05.ld.
//
// Weight gradient (k_conv16_wgrad).  dW[tap][ci][co] = sum_p x[p+tap][ci] *
// g[p][co] is a GEMM over points: M = (8 taps x 16 input channels), N = 16
// output channels, K = points.  Both operands are MN-major (8 channels = one
// 16-byte core-matrix row), staged per block of 64 points; four M tiles (taps
// 0-7, 8-15, 16-23, 24-26 + padding) accumulate in 64 TMEM columns.  Per-CTA
// partial sums are reduced in a fixed order, so the gradient is deterministic.
//
// Operand layouts are the canonical no-swizzle ("interleaved") forms, in
// 16-byte units: K-major ((8,m),2):((1,SBO),LBO); MN-major
// ((1,m),(8,k)):((.,SBO),(1,LBO)).
//
// Waits.  The only waits are on an mbarrier completed by tcgen05.commit; each
// is bounded.  On timeout the CTA records an error in *status, waits once more
// (bounded) for its MMAs, leaves its loop as a whole block and still frees its
// TMEM, so the context stays usable.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <cmath>

#include "learned.cuh"

namespace hb {

namespace tc {

constexpr uint32_t kSpinLimit = 1u << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor, no swizzle (layout type 0), sm_100 version.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Descriptor of a K-major operand with 32-byte rows (K = 16 BF16) in the
// 32-byte swizzle (layout type 6): 8-row groups 256 B apart (SBO), the two
// 16-byte halves of a row 16 B apart (LBO).  Start addresses must keep the
// 256-byte atom phase (base offset 0).
__device__ __forceinline__ uint64_t umma_desc_sw32(uint32_t saddr)
{
    return umma_desc(saddr, 16, 256) | ((uint64_t)6 << 61);
}

// Instruction descriptor of kind::f16: BF16 x BF16 -> FP32, M x N.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N, bool a_mn_major, bool b_mn_major)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn_major ? 1u : 0u) << 15) | ((b_mn_major ? 1u : 0u) << 16) |
           ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate)
{
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t"
        "}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint64_t* mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Bounded wait for the completion of phase `parity`; false on timeout.
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

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t* holder, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(holder)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane (32x32b shape: warp
// w of a warpgroup reads lanes 32(w%4) .. 32(w%4)+31).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16])
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for(int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

}  // namespace tc

using namespace tc;

PermMap make_perm_map(const StencilLevel& L)
{
    PermMap pm{};
    for(int v = 0; v <= 8; ++v) pm.offsets[v] = L.offsets[v];
    for(int v = 0; v < 8; ++v)
    {
        pm.bx[v] = L.bx[v];
        pm.by[v] = L.by[v];
        pm.color_of_par[v] = L.color_of_par[v];
    }
    return pm;
}

__device__ __forceinline__ int perm_row(const PermMap& pm, int z, int y, int x)
{
    const int v = pm.color_of_par[((x & 1) << 2) | ((y & 1) << 1) | (z & 1)];
    return pm.offsets[v] + ((z >> 1) * pm.by[v] + (y >> 1)) * pm.bx[v] + (x >> 1);
}

__device__ __forceinline__ uint4 pack_bf16x8(const float* v)
{
    __align__(16) __nv_bfloat162 h[4];
#pragma unroll
    for(int i = 0; i < 4; ++i) h[i] = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
    return *reinterpret_cast<uint4*>(h);
}

// K-major no-swizzle offset (bytes) of row r, 8-element K chunk c, for
// 16-column (K = 16) operands with SBO = 256 B, LBO = 128 B.
__host__ __device__ constexpr uint32_t kmajor_off(int r, int c) { return (uint32_t)((r >> 3) * 256 + c * 128 + (r & 7) * 16); }

// Weight tile slot (16 output-channel rows x 16 input channels, 512 B) of tap
// t = (dz+1)*9 + (dy+1)*3 + (dx+1): ordered [dy][dz = +1, 0, -1][dx], so the
// 9 taps of one dy form one 144-row K-major B operand (SBO 256 B) whose rows
// are (dz, dx, output channel) -- any run of its dz blocks is contiguous.
__host__ __device__ constexpr int weight_slot(int t) { return ((t / 3) % 3) * 9 + (2 - t / 9) * 3 + t % 3; }

// ------------------------------------------------------------ forward conv
//
// Warp-specialised persistent kernel, one CTA per SM.  A brick is 14 x 8 x kTZ
// output points; its input box is 16 x 10 x (kTZ + 2) points (one point of
// halo on every side), one TMA load of 32-byte swizzled rows.  The dx and dz
// taps are stacked in N: for each staged plane q and row shift dy, ONE MMA
// (M = 128 staged points of the plane, K = 16 input channels) multiplies the
// shifted plane by the weights of all (dz, dx) taps it feeds, N = 48 per
// output plane (3 dx x 16 channels) for the 1-3 output planes q - 1 - dz;
// the epilogue adds the dx = -1 / +1 blocks of the x-neighbouring rows (lane
// shuffles), so the two halo columns of the box produce no output.
//   warp 0      TMA producer into kStages shared-memory stages (zero fill
//               outside the grid);
//   warp 1      TMEM owner and MMA issuer: 3 (kTZ + 2) + kTZ - 1 MMAs per
//               brick (21 for kTZ = 4) into one of two accumulators of
//               kTZ x 48 columns;
//   warps 2-5   epilogue: tcgen05.ld of the finished accumulator, the dx
//               combination, ReLU / mask / permuted scatter, global stores.
// Stage and accumulator hand-offs are mbarriers (TMA complete_tx, MMA commit,
// epilogue arrivals), so loads, MMAs and stores of consecutive bricks overlap.

#ifndef HB_CONV_TZ
#define HB_CONV_TZ 4
#endif
#ifndef HB_CONV_STAGES
#define HB_CONV_STAGES 4
#endif
#ifndef HB_CONV_CTAS
#define HB_CONV_CTAS 1
#endif
constexpr int kTX = 16, kTY = 8, kTZ = HB_CONV_TZ;  // staged x width (with halo), output y, output z
constexpr int kOX = kTX - 2;                          // output x per brick
constexpr int kHY = kTY + 2, kHZ = kTZ + 2;
constexpr int kCopyRows = kTX * kHY * kHZ;            // 960 staged points
constexpr int kRowBytes = kNetCh * 2;                 // the 16 BF16 channels of a point: one 32-byte swizzle row
constexpr int kCopyBytes = kCopyRows * kRowBytes;     // 30720 B = one TMA box
constexpr int kStageBytes = kCopyBytes;
constexpr int kStages = HB_CONV_STAGES;
constexpr int kPlaneCols = 3 * kNetCh;                // one output plane: 3 dx blocks of 16 channels
constexpr int kAccCols = kTZ * kPlaneCols;            // FP32 columns of one brick's accumulator (192)
constexpr int kTmemCols = 512;                        // two accumulators, rounded to a power of two
constexpr int kConvThreads = 192;
constexpr int kEpiThreads = 128;
constexpr int kConvSmem = kStages * kStageBytes + kNetWeightTileBytes + 256 + 1024;

static_assert(kRowBytes == 32, "one point per 32-byte swizzle row (K = 16 per MMA)");
static_assert(kTX * kTY == 128, "one z plane of the brick is one 128-row M tile");
static_assert(kStageBytes % 1024 == 0, "stages start on swizzle-atom boundaries");
static_assert(2 * kAccCols <= kTmemCols && kTmemCols <= 512, "TMEM accumulators");
static_assert(3 * kPlaneCols <= 256, "MMA N");
static_assert(kConvSmem <= 227 * 1024, "shared memory per CTA");

struct Brick
{
    int b, x0, y0, z0;
};

__device__ __forceinline__ Brick brick_of(const ConvGrid& g, long tile, int tx, int ty, long per_sample)
{
    Brick r;
    r.b = (int)(tile / per_sample);
    long t2 = tile - (long)r.b * per_sample;
    const int bz = (int)(t2 / ((long)tx * ty));
    t2 -= (long)bz * tx * ty;
    const int by = (int)(t2 / tx), bx = (int)(t2 - (long)by * tx);
    r.x0 = bx * kOX;  // first output x; the box starts one point before
    r.y0 = by * kTY;
    r.z0 = bz * kTZ;
    return r;
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* mbar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(mbar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* mbar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(mbar)) : "memory");
}

// Tiled 5-D TMA load (no multicast) completing on mbar.
__device__ __forceinline__ void tma_load_5d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3, int c4,
                                            uint64_t* mbar)
{
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4, %5, %6, %7}], [%2];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(mbar)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4)
        : "memory");
}

// Bounded wait that also gives up when another role aborted.
__device__ __forceinline__ bool role_wait(uint64_t* mbar, uint32_t parity, volatile int* abort_flag, int* status,
                                          int code)
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
        if((i & 255) == 255 && *abort_flag) return false;
    }
    *abort_flag = 1;
    atomicExch(status, code);
    return false;
}

template <int kOut>
__global__ void __launch_bounds__(kConvThreads, HB_CONV_CTAS)
    k_conv16(const __grid_constant__ CUtensorMap in_map, ConvGrid g, const __nv_bfloat16* __restrict__ wB, void* out,
             const __nv_bfloat16* __restrict__ act, PermMap pm, int* status)
{
    extern __shared__ unsigned char smem_raw[];
    pdl_launch_dependents();  // the next kernel may start its prologue
    unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    unsigned char* sA = smem;                                   // kStages x kStageBytes
    unsigned char* sW = smem + kStages * kStageBytes;           // weights
    uint64_t* full = (uint64_t*)(sW + kNetWeightTileBytes);     // [kStages] TMA -> MMA
    uint64_t* empty = full + kStages;                           // [kStages] MMA -> TMA
    uint64_t* tfull = empty + kStages;                          // [2] MMA -> epilogue
    uint64_t* tempty = tfull + 2;                               // [2] epilogue -> MMA
    uint32_t* tholder = (uint32_t*)(tempty + 2);
    volatile int* abort_flag = (volatile int*)(tholder + 1);

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int tx = (g.nx + kOX - 1) / kOX, ty = (g.ny + kTY - 1) / kTY, tz = (g.nz + kTZ - 1) / kTZ;
    const long per_sample = (long)tx * ty * tz;
    const long ntiles = per_sample * g.nb;

    for(int i = tid; i < kNetWeightTileBytes / 16; i += kConvThreads)
        reinterpret_cast<uint4*>(sW)[i] = reinterpret_cast<const uint4*>(wB)[i];
    if(tid == 0)
    {
        for(int s = 0; s < kStages; ++s)
        {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for(int a = 0; a < 2; ++a)
        {
            mbar_init(&tfull[a], 1);
            mbar_init(&tempty[a], kEpiThreads);
        }
        *abort_flag = 0;
    }
    if(warp == 1) tmem_alloc(tholder, kTmemCols);
    fence_async_smem();  // the weights are read by the tensor cores
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tholder;
    pdl_wait();  // from here on the previous kernel's output is read

    if(warp == 0 && lane == 0)
    {
        // ---- TMA producer
        long issued = 0;
        for(long tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++issued)
        {
            const int st = (int)(issued % kStages);
            const uint32_t ph = (uint32_t)((issued / kStages) & 1);
            if(!role_wait(&empty[st], ph ^ 1u, abort_flag, status, 3)) break;
            const Brick bk = brick_of(g, tile, tx, ty, per_sample);
            mbar_expect_tx(&full[st], (uint32_t)kCopyBytes);
            tma_load_5d(sA + st * kStageBytes, &in_map, 0, bk.x0 - 1, bk.y0 - 1, bk.z0 - 1, bk.b, &full[st]);
        }
        if(*abort_flag)
        {
            // let the loads already issued land before the CTA's shared memory goes away
            for(long k = issued - kStages < 0 ? 0 : issued - kStages; k < issued; ++k)
            {
                uint32_t done = 0;
                const uint32_t a = smem_u32(&full[k % kStages]);
                for(uint32_t i = 0; i < kSpinLimit && !done; ++i)
                    asm volatile(
                        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                        "selp.u32 %0, 1, 0, p;\n\t}\n"
                        : "=r"(done)
                        : "r"(a), "r"((uint32_t)((k / kStages) & 1))
                        : "memory");
            }
        }
    }
    else if(warp == 1 && lane == 0)
    {
        // ---- MMA issuer
        const uint64_t bd0 = umma_desc(smem_u32(sW), 128, 256);
        long i = 0;
        for(long tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++i)
        {
            const int st = (int)(i % kStages);
            const uint32_t ph = (uint32_t)((i / kStages) & 1);
            const int acc = (int)(i & 1);
            const uint32_t aph = (uint32_t)((i >> 1) & 1);
            if(!role_wait(&tempty[acc], aph ^ 1u, abort_flag, status, 4)) break;
            if(!role_wait(&full[st], ph, abort_flag, status, 5)) break;
            tc_fence_after();
            // descriptors = base + compile-time offset (the 14-bit start field
            // holds address / 16 and stays below 2^14 for any smem address)
            const uint64_t ad0 = umma_desc_sw32(smem_u32(sA + st * kStageBytes));
            const uint32_t d0 = tmem + (uint32_t)(acc * kAccCols);
            // staged plane q (z = z0 - 1 + q) feeds output planes mt = q - 1 - dz
            // in [lo, hi]; output plane mt takes dz block j = mt - q + 2 of the
            // row shift's 144-row operand.  Output plane q is first written at
            // (q, dy = -1), with the accumulate flag off, by an MMA of its own.
#pragma unroll
            for(int q = 0; q < kTZ + 2; ++q)
            {
                const int lo = q - 2 < 0 ? 0 : q - 2;
                const int hi = q < kTZ - 1 ? q : kTZ - 1;
#pragma unroll
                for(int dyi = 0; dyi < 3; ++dyi)
                {
                    const int row0 = (q * kHY + dyi) * kTX;
                    const uint64_t ad = ad0 + (uint64_t)((row0 * kRowBytes) >> 4);
                    const uint64_t bs = bd0 + (uint64_t)((dyi * 9 * 512) >> 4);
                    auto mma = [&](int m0, int m1, uint32_t accumulate) {
                        const uint32_t idesc = umma_idesc_bf16(128, (m1 - m0 + 1) * kPlaneCols, false, false);
                        mma_bf16(d0 + m0 * kPlaneCols, ad, bs + (uint64_t)(((m0 - q + 2) * 3 * 512) >> 4), idesc,
                                 accumulate);
                    };
                    if(q <= kTZ - 1 && dyi == 0)
                    {
                        if(hi > lo) mma(lo, hi - 1, 1u);
                        mma(hi, hi, 0u);
                    }
                    else
                    {
                        mma(lo, hi, 1u);
                    }
                }
            }
            mma_commit(&empty[st]);   // stage free once these MMAs have read it
            mma_commit(&tfull[acc]);  // accumulator ready for the epilogue
        }
        if(*abort_flag && i > 0)
        {
            // MMAs in flight must finish before TMEM is released
            const long k = i - 1;
            uint32_t done = 0;
            const uint32_t a = smem_u32(&tfull[k & 1]);
            for(uint32_t j = 0; j < kSpinLimit && !done; ++j)
                asm volatile(
                    "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                    "selp.u32 %0, 1, 0, p;\n\t}\n"
                    : "=r"(done)
                    : "r"(a), "r"((uint32_t)((k >> 1) & 1))
                    : "memory");
        }
    }
    else if(warp >= 2)
    {
        // ---- epilogue: warp w reads TMEM lanes 32 (w % 4) .. +31
        const int qd = warp & 3;
        const int m = qd * 32 + lane;
        long i = 0;
        for(long tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++i)
        {
            const int acc = (int)(i & 1);
            const uint32_t aph = (uint32_t)((i >> 1) & 1);
            if(!role_wait(&tfull[acc], aph, abort_flag, status, 6)) break;
            tc_fence_after();
            const Brick bk = brick_of(g, tile, tx, ty, per_sample);
            // row m is staged point (xi, yi) of the plane; xi = 0 and kTX - 1
            // are the halo columns
            const int xi = m % kTX;
            const int x = bk.x0 - 1 + xi, y = bk.y0 + m / kTX;
            const bool halo = xi == 0 || xi == kTX - 1;
#pragma unroll 1
            for(int mt = 0; mt < kTZ; ++mt)
            {
                // out(x) = D_{dx=-1}[x - 1] + D_{dx=0}[x] + D_{dx=+1}[x + 1]: rows
                // x +- 1 are the neighbouring lanes of the same 16-lane line
                float dm[16], dc[16], dp[16], v[16];
                const uint32_t ta =
                    tmem + ((uint32_t)(qd * 32) << 16) + (uint32_t)(acc * kAccCols + mt * kPlaneCols);
                tmem_ld16(ta, dm);
                tmem_ld16(ta + kNetCh, dc);
                tmem_ld16(ta + 2 * kNetCh, dp);
#pragma unroll
                for(int c = 0; c < 16; ++c)
                {
                    const float left = __shfl_up_sync(0xffffffffu, dm[c], 1);
                    const float right = __shfl_down_sync(0xffffffffu, dp[c], 1);
                    v[c] = (left + dc[c]) + right;
                }
                const int z = bk.z0 + mt;
                if(halo || x >= g.nx || y >= g.ny || z >= g.nz) continue;
                const long p = (((long)bk.b * g.nz + z) * g.ny + y) * g.nx + x;
                if constexpr(kOut == kOutReluBf16 || kOut == kOutMaskBf16)
                {
                    if constexpr(kOut == kOutReluBf16)
                    {
#pragma unroll
                        for(int c = 0; c < 16; ++c) v[c] = v[c] > 0.f ? v[c] : 0.f;
                    }
                    else
                    {
                        const uint4* ap = reinterpret_cast<const uint4*>(act + p * kNetCh);
                        __align__(16) __nv_bfloat16 h[16];
                        *reinterpret_cast<uint4*>(h) = ap[0];
                        *reinterpret_cast<uint4*>(h + 8) = ap[1];
#pragma unroll
                        for(int c = 0; c < 16; ++c) v[c] = __bfloat162float(h[c]) > 0.f ? v[c] : 0.f;
                    }
                    uint4* dst = reinterpret_cast<uint4*>(reinterpret_cast<__nv_bfloat16*>(out) + p * kNetCh);
                    dst[0] = pack_bf16x8(v);
                    dst[1] = pack_bf16x8(v + 8);
                }
                else if constexpr(kOut == kOutF32)
                {
                    float4* dst = reinterpret_cast<float4*>(reinterpret_cast<float*>(out) + p * kNetCh);
#pragma unroll
                    for(int c = 0; c < 4; ++c)
                        dst[c] = make_float4(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
                }
                else if constexpr(kOut == kOutF32C0)
                {
                    reinterpret_cast<float*>(out)[p] = v[0];
                }
                else
                {
                    float* xo = reinterpret_cast<float*>(out) + perm_row(pm, z, y, x);
                    if constexpr(kOut == kOutPermSet) *xo = v[0];
                    else *xo += v[0];
                }
            }
            tc_fence_before();
            mbar_arrive(&tempty[acc]);
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if(warp == 1) tmem_free(tmem, kTmemCols);
}

// ------------------------------------------------------------ layer 3 (16 -> 1)
//
// One output channel: the 27 taps are stacked in N instead of the input being
// shifted.  For each staged input point p, ONE MMA row computes
// D[p][t] = sum_c a2[p][c] w3[t][c] for all taps t (M = 128 points, N = 32,
// K = 16), and the output is y[o] = sum_t D[o + off_t][t], gathered by the
// epilogue from shared memory in tap order (deterministic, no atomics).  In
// the odd evaluation the pair is folded into K: the branch of -r is a second
// MMA into the same accumulator with the weights negated, both halved, so D
// already holds (y(r) - y(-r)) / 2.
//   warp 0      TMA producer: per brick one (two with the pair) box of the
//               halo'd input, 18 x 10 x 4 points of 16 channels, 32-byte
//               swizzled rows, zero fill outside the grid;
//   warp 1      TMEM owner and MMA issuer: 6 MMAs (12 with the pair) per brick
//               into one of two accumulators of 6 x 32 columns;
//   warps 2-5   epilogue: TMEM -> shared memory (27 floats per staged point),
//               then the 27-tap gather for the brick's 16 x 8 x 2 outputs.
constexpr int k3X = 16, k3Y = 8, k3Z = 2;                       // output brick
constexpr int k3HX = k3X + 2, k3HY = k3Y + 2, k3HZ = k3Z + 2;  // staged box 18 x 10 x 4
constexpr int k3Rows = k3HX * k3HY * k3HZ;                      // 720 staged points
constexpr int k3Chunks = (k3Rows + 127) / 128;                  // 6 M tiles per box
constexpr int k3BoxBytes = k3Chunks * 128 * kRowBytes;          // 24 KB (the TMA fills the first 720 rows)
constexpr int k3StageBytes = 2 * k3BoxBytes;                    // the two branches of the pair
constexpr int k3Stages = 2;
constexpr int k3N = 32;                                         // 27 taps + 5 zero columns
constexpr int k3AccCols = k3Chunks * k3N;                       // 192 TMEM columns per brick
constexpr int k3TmemCols = 512;                                 // two accumulators, power of two
constexpr int k3DStride = 27;                                   // floats per staged point (odd: no bank conflicts)
constexpr int k3WTileBytes = k3N * kRowBytes;                   // 32 tap rows x 16 channels, K-major
constexpr int k3Outputs = k3X * k3Y * k3Z;                      // 256 per brick
constexpr int k3Smem = k3Stages * k3StageBytes + 2 * k3WTileBytes + k3Rows * k3DStride * 4 + 256 + 1024;

static_assert(k3BoxBytes % 1024 == 0 && k3Rows * kRowBytes <= k3BoxBytes, "layer-3 box");
static_assert(k3Outputs % kEpiThreads == 0, "whole outputs per epilogue thread");
static_assert(k3Smem <= 227 * 1024, "shared memory per CTA");

// Named barrier 1 of the four epilogue warps (the non-aligned forms: lanes
// may arrive apart); the OR reduction makes a give-up decision of any one
// thread the decision of all, so they take the same barriers.
__device__ __forceinline__ bool epi_any(bool pred)
{
    uint32_t r;
    asm volatile(
        "{\n\t"
        ".reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "barrier.red.or.pred q, 1, 128, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t"
        "}\n"
        : "=r"(r)
        : "r"(pred ? 1u : 0u)
        : "memory");
    return r != 0;
}

__device__ __forceinline__ void epi_sync() { asm volatile("barrier.sync 1, 128;" ::: "memory"); }

template <int kOut, bool kPair>
__global__ void __launch_bounds__(kConvThreads, 1)
    k_layer3_tc(const __grid_constant__ CUtensorMap in_map, ConvGrid g, const float* __restrict__ w3, float* out,
                PermMap pm, int* status)
{
    extern __shared__ unsigned char smem_raw[];
    pdl_launch_dependents();  // the next kernel may start its prologue
    unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    unsigned char* sA = smem;                                       // k3Stages x k3StageBytes
    unsigned char* sW = smem + k3Stages * k3StageBytes;             // + and - weight tiles
    float* sD = (float*)(sW + 2 * k3WTileBytes);                    // k3Rows x k3DStride
    uint64_t* full = (uint64_t*)(sD + k3Rows * k3DStride);
    uint64_t* empty = full + k3Stages;
    uint64_t* tfull = empty + k3Stages;
    uint64_t* tempty = tfull + 2;
    uint32_t* tholder = (uint32_t*)(tempty + 2);
    volatile int* abort_flag = (volatile int*)(tholder + 1);

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int tx = (g.nx + k3X - 1) / k3X, ty = (g.ny + k3Y - 1) / k3Y, tz = (g.nz + k3Z - 1) / k3Z;
    const long per_sample = (long)tx * ty * tz;
    const long ntiles = per_sample * g.nb;

    // weight tiles: row t = tap, 16 channels; the bf16 weight, halved and
    // negated for the pair (exact in bf16)
    for(int i = tid; i < k3N * kNetCh; i += kConvThreads)
    {
        const int t = i / kNetCh, c = i % kNetCh;
        float w = t < 27 ? __bfloat162float(__float2bfloat16_rn(w3[(t * kNetCh + c) * kNetCh])) : 0.f;
        if(kPair) w *= 0.5f;
        const uint32_t off = kmajor_off(t, c >> 3) + (uint32_t)(c & 7) * 2;
        *reinterpret_cast<__nv_bfloat16*>(sW + off) = __float2bfloat16_rn(w);
        *reinterpret_cast<__nv_bfloat16*>(sW + k3WTileBytes + off) = __float2bfloat16_rn(-w);
    }
    if(tid == 0)
    {
        for(int s = 0; s < k3Stages; ++s)
        {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for(int a = 0; a < 2; ++a)
        {
            mbar_init(&tfull[a], 1);
            mbar_init(&tempty[a], kEpiThreads);
        }
        *abort_flag = 0;
    }
    if(warp == 1) tmem_alloc(tholder, k3TmemCols);
    fence_async_smem();  // the weights are read by the tensor cores
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tholder;
    pdl_wait();  // from here on the previous kernel's output is read
    constexpr uint32_t kBoxTx = (uint32_t)(k3Rows * kRowBytes) * (kPair ? 2u : 1u);

    if(warp == 0 && lane == 0)
    {
        // ---- TMA producer
        long issued = 0;
        for(long tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++issued)
        {
            const int st = (int)(issued % k3Stages);
            const uint32_t ph = (uint32_t)((issued / k3Stages) & 1);
            if(!role_wait(&empty[st], ph ^ 1u, abort_flag, status, 3)) break;
            const int b = (int)(tile / per_sample);
            long t2 = tile - (long)b * per_sample;
            const int bz = (int)(t2 / ((long)tx * ty));
            t2 -= (long)bz * tx * ty;
            const int by = (int)(t2 / tx), bx = (int)(t2 - (long)by * tx);
            mbar_expect_tx(&full[st], kBoxTx);
            unsigned char* dst = sA + st * k3StageBytes;
            tma_load_5d(dst, &in_map, 0, bx * k3X - 1, by * k3Y - 1, bz * k3Z - 1, b, &full[st]);
            if(kPair)
                tma_load_5d(dst + k3BoxBytes, &in_map, 0, bx * k3X - 1, by * k3Y - 1, bz * k3Z - 1, b + g.nb,
                            &full[st]);
        }
        if(*abort_flag)
        {
            // let the loads already issued land before the CTA's shared memory goes away
            for(long k = issued - k3Stages < 0 ? 0 : issued - k3Stages; k < issued; ++k)
                mbar_wait(&full[k % k3Stages], (uint32_t)((k / k3Stages) & 1));
        }
    }
    else if(warp == 1 && lane == 0)
    {
        // ---- MMA issuer
        constexpr uint32_t idesc = umma_idesc_bf16(128, k3N, false, false);
        const uint64_t bpos = umma_desc(smem_u32(sW), 128, 256);
        const uint64_t bneg = umma_desc(smem_u32(sW + k3WTileBytes), 128, 256);
        long i = 0;
        for(long tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++i)
        {
            const int st = (int)(i % k3Stages);
            const uint32_t ph = (uint32_t)((i / k3Stages) & 1);
            const int acc = (int)(i & 1);
            const uint32_t aph = (uint32_t)((i >> 1) & 1);
            if(!role_wait(&tempty[acc], aph ^ 1u, abort_flag, status, 4)) break;
            if(!role_wait(&full[st], ph, abort_flag, status, 5)) break;
            tc_fence_after();
            const uint64_t a0 = umma_desc_sw32(smem_u32(sA + st * k3StageBytes));
            const uint32_t d0 = tmem + (uint32_t)(acc * k3AccCols);
#pragma unroll
            for(int c = 0; c < k3Chunks; ++c)
            {
                const uint64_t ac = a0 + (uint64_t)((c * 128 * kRowBytes) >> 4);
                mma_bf16(d0 + c * k3N, ac, bpos, idesc, 0u);
                if(kPair) mma_bf16(d0 + c * k3N, ac + (uint64_t)(k3BoxBytes >> 4), bneg, idesc, 1u);
            }
            mma_commit(&empty[st]);   // stage free once these MMAs have read it
            mma_commit(&tfull[acc]);  // accumulator ready for the epilogue
        }
        if(*abort_flag && i > 0)
        {
            // MMAs in flight must finish before TMEM is released
            const long k = i - 1;
            mbar_wait(&tfull[k & 1], (uint32_t)((k >> 1) & 1));
        }
    }
    else if(warp >= 2)
    {
        // ---- epilogue: warp w reads TMEM lanes 32 (w % 4) .. +31
        const int qd = warp & 3;
        const int et = tid - 64;  // 0 .. 127
        long i = 0;
        for(long tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++i)
        {
            const int acc = (int)(i & 1);
            const uint32_t aph = (uint32_t)((i >> 1) & 1);
            const bool ok = role_wait(&tfull[acc], aph, abort_flag, status, 6);
            if(epi_any(!ok)) break;
            __syncwarp();  // tcgen05.ld is warp-collective
            tc_fence_after();
#pragma unroll 1
            for(int c = 0; c < k3Chunks; ++c)
            {
                float v[32];
                const uint32_t ta = tmem + ((uint32_t)(qd * 32) << 16) + (uint32_t)(acc * k3AccCols + c * k3N);
                tmem_ld16(ta, *reinterpret_cast<float(*)[16]>(v));
                tmem_ld16(ta + 16, *reinterpret_cast<float(*)[16]>(v + 16));
                const int row = c * 128 + qd * 32 + lane;
                if(row < k3Rows)
                {
#pragma unroll
                    for(int t = 0; t < 27; ++t) sD[row * k3DStride + t] = v[t];
                }
            }
            tc_fence_before();
            mbar_arrive(&tempty[acc]);  // the accumulator may take the next brick
            epi_sync();                 // every staged point's taps are in shared memory
            const int b = (int)(tile / per_sample);
            long t2 = tile - (long)b * per_sample;
            const int bz = (int)(t2 / ((long)tx * ty));
            t2 -= (long)bz * tx * ty;
            const int by = (int)(t2 / tx), bx = (int)(t2 - (long)by * tx);
#pragma unroll
            for(int k = 0; k < k3Outputs / kEpiThreads; ++k)
            {
                const int o = et + k * kEpiThreads;
                const int ox = o % k3X, oy = (o / k3X) % k3Y, oz = o / (k3X * k3Y);
                const int x = bx * k3X + ox, y = by * k3Y + oy, z = bz * k3Z + oz;
                if(x >= g.nx || y >= g.ny || z >= g.nz) continue;
                float sum = 0.f;
#pragma unroll
                for(int t = 0; t < 27; ++t)
                {
                    const int dz = t / 9 - 1, dy = (t / 3) % 3 - 1, dx = t % 3 - 1;
                    const int r = ((oz + 1 + dz) * k3HY + (oy + 1 + dy)) * k3HX + (ox + 1 + dx);
                    sum += sD[r * k3DStride + t];
                }
                if constexpr(kOut == 2)
                {
                    out[(((long)b * g.nz + z) * g.ny + y) * g.nx + x] = sum;
                }
                else
                {
                    float* xo = out + perm_row(pm, z, y, x);
                    if constexpr(kOut == 1) *xo += sum;
                    else *xo = sum;
                }
            }
            epi_sync();  // shared memory free for the next brick
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if(warp == 1) tmem_free(tmem, k3TmemCols);
}

// ------------------------------------------------------------ weight gradient

constexpr int kWgK = 64;                  // points per K block
constexpr int kWgATile = 128 * kWgK * 2;  // 16 KB per M tile (8 taps x 16 channels)
constexpr int kWgB = 16 * kWgK * 2;       // 2 KB
constexpr int kWgThreads = 128;
constexpr int kWgSmem = 4 * kWgATile + kWgB + 64 + 128;

// MN-major no-swizzle offsets (bytes) of 8-element M chunk j, K index k.
//   A: SBO (chunk stride) 128 B, LBO (8-k group stride) 16 chunks x 128 B = 2048 B
//   B: SBO 128 B, LBO 2 chunks x 128 B = 256 B
__device__ __forceinline__ uint32_t mn_off_a(int j, int k) { return (uint32_t)(j * 128 + (k & 7) * 16 + (k >> 3) * 2048); }
__device__ __forceinline__ uint32_t mn_off_b(int j, int k) { return (uint32_t)(j * 128 + (k & 7) * 16 + (k >> 3) * 256); }

__global__ void __launch_bounds__(kWgThreads) k_conv16_wgrad(ConvGrid g, const __nv_bfloat16* __restrict__ x,
                                                             const __nv_bfloat16* __restrict__ gr,
                                                             float* __restrict__ partial, int* status)
{
    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
    unsigned char* sA = smem;
    unsigned char* sB = smem + 4 * kWgATile;
    uint64_t* mbar = (uint64_t*)(sB + kWgB);
    uint32_t* tholder = (uint32_t*)(mbar + 1);

    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const long per = (long)g.nz * g.ny * g.nx;
    const long n = per * g.nb;
    const long nblk = (n + kWgK - 1) / kWgK;

    if(tid == 0) mbar_init(mbar, 1);
    if(warp == 0) tmem_alloc(tholder, 64);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tholder;
    constexpr uint32_t idesc = umma_idesc_bf16(128, 16, true, true);
    uint32_t phase = 0;
    bool first = true, ok = true;

    for(long blk = blockIdx.x; blk < nblk; blk += gridDim.x)
    {
        for(int i = tid; i < kWgK * 2; i += kWgThreads)
        {
            const int k = i >> 1, c8 = i & 1;
            const long p = blk * kWgK + k;
            uint4 v = make_uint4(0, 0, 0, 0);
            if(p < n) v = __ldg(reinterpret_cast<const uint4*>(gr + p * kNetCh) + c8);
            *reinterpret_cast<uint4*>(sB + mn_off_b(c8, k)) = v;
        }
        for(int i = tid; i < kWgK * 32 * 2; i += kWgThreads)
        {
            // i -> (k, tap slot 0..31, c8); tap slots >= 27 are zero padding
            const int c8 = i & 1;
            const int ts = (i >> 1) & 31;
            const int k = i >> 6;
            const long p = blk * kWgK + k;
            uint4 v = make_uint4(0, 0, 0, 0);
            if(ts < 27 && p < n)
            {
                const long b = p / per;
                const long rem = p - b * per;
                const int z = (int)(rem / ((long)g.ny * g.nx));
                const long r2 = rem - (long)z * g.ny * g.nx;
                const int y = (int)(r2 / g.nx);
                const int xx = (int)(r2 - (long)y * g.nx);
                const int zz = z + ts / 9 - 1, yy = y + (ts / 3) % 3 - 1, x2 = xx + ts % 3 - 1;
                if(zz >= 0 && zz < g.nz && yy >= 0 && yy < g.ny && x2 >= 0 && x2 < g.nx)
                    v = __ldg(reinterpret_cast<const uint4*>(
                                  x + (((b * g.nz + zz) * g.ny + yy) * g.nx + x2) * kNetCh) +
                              c8);
            }
            const int mt = ts >> 3;
            const int j = (ts & 7) * 2 + c8;
            *reinterpret_cast<uint4*>(sA + mt * kWgATile + mn_off_a(j, k)) = v;
        }
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        if(tid == 0)
        {
            const uint64_t ad0 = umma_desc(smem_u32(sA), 2048, 128);
            const uint64_t bd0 = umma_desc(smem_u32(sB), 256, 128);
#pragma unroll
            for(int s = 0; s < kWgK / 16; ++s)
            {
                const uint64_t bd = bd0 + (uint64_t)(s * 2 * 256 >> 4);
#pragma unroll
                for(int mt = 0; mt < 4; ++mt)
                {
                    const uint64_t ad = ad0 + (uint64_t)((mt * kWgATile + s * 2 * 2048) >> 4);
                    mma_bf16(tmem + (uint32_t)(mt * 16), ad, bd, idesc, (first && s == 0) ? 0u : 1u);
                }
            }
            mma_commit(mbar);
        }
        first = false;
        __syncwarp();
        const bool done = mbar_wait(mbar, phase);
        ok = __syncthreads_and(done) != 0;
        if(!ok)
        {
            if(tid == 0) atomicExch(status, 2);
            if(!done) mbar_wait(mbar, phase);
            break;
        }
        phase ^= 1u;
        tc_fence_after();
        __syncthreads();  // staging consumed before it is rewritten
    }
    tc_fence_after();
    // row m of M tile mt = TMEM lane m: tap mt*8 + m/16, input channel m%16
    for(int mt = 0; mt < 4; ++mt)
    {
        float v[16];
        tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(mt * 16), v);
        const int tap = mt * 8 + (tid >> 4), ci = tid & 15;
        if(tap < 27)
        {
            float4* dst = reinterpret_cast<float4*>(partial + (((size_t)blockIdx.x * 27 + tap) * 16 + ci) * 16);
            const bool zero = first || !ok;
#pragma unroll
            for(int c = 0; c < 4; ++c)
                dst[c] = zero ? make_float4(0.f, 0.f, 0.f, 0.f)
                              : make_float4(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
        }
    }
    tc_fence_before();
    __syncthreads();
    if(warp == 0) tmem_free(tmem, 64);
}

__global__ void k_wgrad_reduce(int nparts, const float* __restrict__ partial, float* __restrict__ dw)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= kNetLayerWeights) return;
    float s = 0.f;
    for(int c = 0; c < nparts; ++c) s += partial[(size_t)c * kNetLayerWeights + i];
    dw[i] = s;
}

// ------------------------------------------------------------ small kernels

// w[tap][ci][co] (FP32) -> per-tap K-major B operand (N = co rows, K = ci).
// flip != 0: W'[t][ci'][co'] = W[26-t][co'][ci'] (transposed convolution).
__global__ void k_prepare_weights(const float* __restrict__ w, __nv_bfloat16* __restrict__ wB, int flip)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= kNetLayerWeights) return;
    const int t = i / 256, nn = (i / 16) % 16, kk = i % 16;
    const float v = flip ? w[((26 - t) * 16 + nn) * 16 + kk] : w[(t * 16 + kk) * 16 + nn];
    unsigned char* base = reinterpret_cast<unsigned char*>(wB) + weight_slot(t) * 512;
    *reinterpret_cast<__nv_bfloat16*>(base + kmajor_off(nn, kk >> 3) + (kk & 7) * 2) = __float2bfloat16_rn(v);
}

__device__ __forceinline__ void store_embed(__nv_bfloat16* a, long p, float r0)
{
    const float v[8] = {r0, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    uint4* dst = reinterpret_cast<uint4*>(a + p * kNetCh);
    dst[0] = pack_bf16x8(v);
    dst[1] = make_uint4(0, 0, 0, 0);
}

// Channel 0 = r (x == nullptr) or the residual r - A x of the 27-point
// stencil (diagonal diag32, off-diagonals -1), read from colour-permuted
// level vectors at natural point p.
__global__ void k_embed_level(PermMap pm, int nz, int ny, int nx, const float* __restrict__ r,
                              const float* __restrict__ x, const float* __restrict__ diag32,
                              __nv_bfloat16* __restrict__ a, int pair)
{
    const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if(p >= (long)nz * ny * nx) return;
    const int z = (int)(p / ((long)ny * nx));
    const long rem = p - (long)z * ny * nx;
    const int y = (int)(rem / nx), xx = (int)(rem - (long)y * nx);
    const int row = perm_row(pm, z, y, xx);
    float v = r[row];
    if(x)
    {
        float off = 0.f;
#pragma unroll
        for(int t = 0; t < 27; ++t)
        {
            const int z2 = z + t / 9 - 1, y2 = y + (t / 3) % 3 - 1, x2 = xx + t % 3 - 1;
            if(t != 13 && z2 >= 0 && z2 < nz && y2 >= 0 && y2 < ny && x2 >= 0 && x2 < nx)
                off += x[perm_row(pm, z2, y2, x2)];
        }
        v = v - (diag32[row] * x[row] - off);
    }
    store_embed(a, p, v);
    if(pair) store_embed(a, p + (long)nz * ny * nx, -v);  // second sample: -v (odd evaluation)
}

// x[row(p)] = (or +=) (y[p] - y[p + n]) / 2: the odd part of the network.
template <bool kAdd>
__global__ void k_odd_combine(PermMap pm, int nz, int ny, int nx, const float* __restrict__ y, float* __restrict__ x)
{
    const long n = (long)nz * ny * nx;
    const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if(p >= n) return;
    const int z = (int)(p / ((long)ny * nx));
    const long rem = p - (long)z * ny * nx;
    const int yy = (int)(rem / nx), xx = (int)(rem - (long)yy * nx);
    const float v = 0.5f * (y[p] - y[p + n]);
    float* o = x + perm_row(pm, z, yy, xx);
    if(kAdd) *o += v;
    else *o = v;
}

// Natural <-> colour-permuted copies of a level vector (training-pair set-up).
template <typename Tin, typename Tout, bool kToNatural>
__global__ void k_perm_copy(PermMap pm, int nz, int ny, int nx, const Tin* __restrict__ in, Tout* __restrict__ out)
{
    const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if(p >= (long)nz * ny * nx) return;
    const int z = (int)(p / ((long)ny * nx));
    const long rem = p - (long)z * ny * nx;
    const int y = (int)(rem / nx), x = (int)(rem - (long)y * nx);
    const int row = perm_row(pm, z, y, x);
    if(kToNatural) out[p] = (Tout)in[row];
    else out[row] = (Tout)in[p];
}

// 1 / sum e^2 (one block, FP64 accumulation).
__global__ void k_inv_sumsq(long n, const float* __restrict__ e, float* __restrict__ out)
{
    __shared__ double red[32];
    double s = 0.0;
    for(long i = threadIdx.x; i < n; i += blockDim.x) s += (double)e[i] * e[i];
    s = block_sum(s, red);
    if(threadIdx.x == 0) *out = (float)(1.0 / s);
}

// Sum of a step's loss partials into acc (one block, fixed order).
__global__ void k_loss_accumulate(int parts, const float* __restrict__ partial, double* __restrict__ acc)
{
    __shared__ double red[32];
    double s = 0.0;
    for(int i = threadIdx.x; i < parts; i += blockDim.x) s += partial[i];
    s = block_sum(s, red);
    if(threadIdx.x == 0) *acc += s;
}

// b ~ N(0,1) by natural row id: SplitMix64 finalizer over (key + 2i, key + 2i + 1)
// with key = mix(seed), 53-bit uniforms u1 in (0,1], u2 in [0,1), Box-Muller
// sqrt(-2 ln u1) cos(2 pi u2).  Stored at out[perm[i]] (perm may be null).
__device__ __forceinline__ unsigned long long splitmix(unsigned long long z)
{
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

__global__ void k_normal_rhs(long long m, unsigned long long seed, const int* __restrict__ perm, double* out64,
                             float* out32)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= m) return;
    const unsigned long long key = splitmix(seed);
    const unsigned long long a = splitmix(key + 2ULL * (unsigned long long)i);
    const unsigned long long b = splitmix(key + 2ULL * (unsigned long long)i + 1ULL);
    const double u1 = ((double)(a >> 11) + 1.0) * (1.0 / 9007199254740992.0);
    const double u2 = (double)(b >> 11) * (1.0 / 9007199254740992.0);
    const double v = sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
    const long long o = perm ? perm[i] : i;
    if(out64) out64[o] = v;
    if(out32) out32[o] = (float)v;
}

__global__ void k_embed_f32(long n, const float* __restrict__ r, __nv_bfloat16* __restrict__ a, int pair)
{
    const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if(p >= n) return;
    store_embed(a, p, r[p]);
    if(pair) store_embed(a, p + n, -r[p]);
}

// 27-point stencil (diagonal 26, off-diagonals -1, zero outside the sample's grid).
__device__ __forceinline__ float stencil_at(const ConvGrid& g, const float* __restrict__ v, long p)
{
    const long per = (long)g.nz * g.ny * g.nx;
    const long b = p / per;
    const long q = p - b * per;
    const int z = (int)(q / ((long)g.ny * g.nx));
    const long rem = q - (long)z * g.ny * g.nx;
    const int y = (int)(rem / g.nx), x = (int)(rem - (long)y * g.nx);
    const float* vb = v + b * per;
    float off = 0.f;
#pragma unroll
    for(int t = 0; t < 27; ++t)
    {
        const int z2 = z + t / 9 - 1, y2 = y + (t / 3) % 3 - 1, x2 = x + t % 3 - 1;
        if(t != 13 && z2 >= 0 && z2 < g.nz && y2 >= 0 && y2 < g.ny && x2 >= 0 && x2 < g.nx)
            off += vb[((long)z2 * g.ny + y2) * g.nx + x2];
    }
    return 26.f * v[p] - off;
}

// out[p] = (y[p] - y[p + n]) / 2 (natural order).
__global__ void k_odd_natural(long n, const float* __restrict__ y, float* __restrict__ out)
{
    const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if(p < n) out[p] = 0.5f * (y[p] - y[p + n]);
}

// ------------------------------------------- layers 1 and 3 on the CUDA cores
// Layer 1 has one real input channel and layer 3 one real output channel, so
// 15/16 of their tensor-core MMA work multiplies zeros.  For evaluation they
// run here instead, in FP32 with the BF16-rounded weights: layer 1 fused with
// the odd pair (the second branch's pre-activation is exactly -z), layer 3
// fused with the odd combination and the scatter into the level vector.

// Bf16 scalar field of a level: r, or the residual r - A x (k_embed_level's
// channel 0 without the 15 zero channels and the negated copy).
__global__ void k_embed_scalar_level(PermMap pm, int nz, int ny, int nx, const float* __restrict__ r,
                                     const float* __restrict__ x, const float* __restrict__ diag32,
                                     __nv_bfloat16* __restrict__ s1)
{
    pdl_begin();
    const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if(p >= (long)nz * ny * nx) return;
    const int z = (int)(p / ((long)ny * nx));
    const long rem = p - (long)z * ny * nx;
    const int y = (int)(rem / nx), xx = (int)(rem - (long)y * nx);
    const int row = perm_row(pm, z, y, xx);
    float v = r[row];
    if(x)
    {
        float off = 0.f;
#pragma unroll
        for(int t = 0; t < 27; ++t)
        {
            const int z2 = z + t / 9 - 1, y2 = y + (t / 3) % 3 - 1, x2 = xx + t % 3 - 1;
            if(t != 13 && z2 >= 0 && z2 < nz && y2 >= 0 && y2 < ny && x2 >= 0 && x2 < nx)
                off += x[perm_row(pm, z2, y2, x2)];
        }
        v = v - (diag32[row] * x[row] - off);
    }
    s1[p] = __float2bfloat16_rn(v);
}

__device__ __forceinline__ float in_value(const __nv_bfloat16* v, long q) { return __bfloat162float(v[q]); }
__device__ __forceinline__ float in_value(const float* v, long q) { return __bfloat162float(__float2bfloat16_rn(v[q])); }


// ------------------------------------------------------------ layer 1 (1 -> 16)
//
// One input channel: the 27 taps are the K dimension.  Per brick of
// 16 x 8 x 4 points the CTA stages the halo'd scalar field (18 x 10 x 6,
// BF16-rounded, zero outside the grid), each thread writes the im2col row of
// its point in every z plane (27 neighbours, 5 zeros: K = 32), and two MMAs
// per plane (M = 128 points, N = 16 channels, K = 16 each) give the 16
// pre-activations in TMEM; the epilogue writes relu(z) and, for the odd pair,
// relu(-z) as BF16.  Several CTAs per SM overlap one CTA's MMA round trip with
// the others' staging.
constexpr int k1X = 16, k1Y = 8, k1Z = 4;
constexpr int k1HX = k1X + 2, k1HY = k1Y + 2, k1HZ = k1Z + 2;
constexpr int k1Halo = k1HX * k1HY * k1HZ;  // 1080 staged scalars
constexpr int k1Threads = 128;              // one thread per point of a plane
constexpr int k1K = 32;                     // 27 taps + 5 zeros
constexpr int k1PlaneBytes = 128 * k1K * 2; // 8 KB of im2col rows per plane
constexpr int k1Cols = k1Z * kNetCh;        // TMEM columns per brick
constexpr int k1WBytes = kNetCh * k1K * 2;  // B: 16 channel rows x 32 taps
constexpr int k1Smem = k1Z * k1PlaneBytes + k1WBytes + k1Halo * 4 + 64 + 1024;
constexpr int k1CtasPerSm = 4;

static_assert(k1X * k1Y == k1Threads, "one plane of the brick is one 128-row M tile");
static_assert(k1Cols * k1CtasPerSm <= 512, "TMEM columns of the co-resident CTAs");

// K-major no-swizzle offset of row r, 8-element K chunk c8 of a 32-wide K
// operand: chunks 128 B apart (LBO), 8-row groups 512 B apart (SBO).
__host__ __device__ constexpr uint32_t k1_off(int r, int c8)
{
    return (uint32_t)((r >> 3) * 512 + c8 * 128 + (r & 7) * 16);
}

template <typename Tin, bool kPair>
__global__ void __launch_bounds__(k1Threads) k_layer1_tc(ConvGrid g, const Tin* __restrict__ in,
                                                         const float* __restrict__ w1,
                                                         __nv_bfloat16* __restrict__ a1, int* status)
{
    extern __shared__ unsigned char smem_raw[];
    pdl_launch_dependents();  // the next kernel may start its prologue
    unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    unsigned char* sA = smem;                           // k1Z im2col planes
    unsigned char* sW = sA + k1Z * k1PlaneBytes;        // weights
    float* sS = (float*)(sW + k1WBytes);                // staged scalars
    uint64_t* mbar = (uint64_t*)(sS + k1Halo);
    uint32_t* tholder = (uint32_t*)(mbar + 1);

    const int tid = threadIdx.x, warp = tid >> 5;
    for(int i = tid; i < kNetCh * k1K; i += k1Threads)
    {
        const int co = i / k1K, t = i % k1K;
        const float w = t < 27 ? w1[t * kNetCh * kNetCh + co] : 0.f;  // w1[t][0][co]
        *reinterpret_cast<__nv_bfloat16*>(sW + k1_off(co, t >> 3) + (t & 7) * 2) = __float2bfloat16_rn(w);
    }
    if(tid == 0) mbar_init(mbar, 1);
    if(warp == 0) tmem_alloc(tholder, k1Cols);
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tholder;
    pdl_wait();  // from here on the previous kernel's output is read

    const long n = g.points();
    const int tx = (g.nx + k1X - 1) / k1X, ty = (g.ny + k1Y - 1) / k1Y, tz = (g.nz + k1Z - 1) / k1Z;
    const long per_sample = (long)tx * ty * tz;
    const long ntiles = per_sample * g.nb;
    constexpr uint32_t idesc = umma_idesc_bf16(128, kNetCh, false, false);
    const uint64_t bd = umma_desc(smem_u32(sW), 128, 512);
    const int mx = tid % k1X, my = tid / k1X;
    uint32_t phase = 0;
    bool failed = false;
    for(long tile = blockIdx.x; tile < ntiles; tile += gridDim.x)
    {
        const int b = (int)(tile / per_sample);
        long t2 = tile - (long)b * per_sample;
        const int bz = (int)(t2 / ((long)tx * ty));
        t2 -= (long)bz * tx * ty;
        const int by = (int)(t2 / tx), bx = (int)(t2 - (long)by * tx);
        const int x0 = bx * k1X, y0 = by * k1Y, z0 = bz * k1Z;
        const long base = (long)b * g.nz * g.ny * g.nx;
        for(int e = tid; e < k1Halo; e += k1Threads)
        {
            const int hx = e % k1HX, hy = (e / k1HX) % k1HY, hz = e / (k1HX * k1HY);
            const int x = x0 + hx - 1, y = y0 + hy - 1, z = z0 + hz - 1;
            float v = 0.f;
            if(x >= 0 && x < g.nx && y >= 0 && y < g.ny && z >= 0 && z < g.nz)
                v = in_value(in, base + ((long)z * g.ny + y) * g.nx + x);
            sS[e] = v;
        }
        __syncthreads();
#pragma unroll 1
        for(int q = 0; q < k1Z; ++q)
        {
            __align__(16) __nv_bfloat16 h[k1K];
#pragma unroll
            for(int t = 0; t < 27; ++t)
            {
                const int dz = t / 9 - 1, dy = (t / 3) % 3 - 1, dx = t % 3 - 1;
                h[t] = __float2bfloat16_rn(sS[((q + 1 + dz) * k1HY + (my + 1 + dy)) * k1HX + (mx + 1 + dx)]);
            }
#pragma unroll
            for(int t = 27; t < k1K; ++t) h[t] = __float2bfloat16_rn(0.f);
            unsigned char* row = sA + q * k1PlaneBytes;
#pragma unroll
            for(int c8 = 0; c8 < k1K / 8; ++c8)
                *reinterpret_cast<uint4*>(row + k1_off(tid, c8)) = *reinterpret_cast<const uint4*>(h + 8 * c8);
        }
        fence_async_smem();  // the im2col rows are read by the tensor cores
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        if(tid == 0)
        {
#pragma unroll
            for(int q = 0; q < k1Z; ++q)
#pragma unroll
                for(int kh = 0; kh < 2; ++kh)
                    mma_bf16(tmem + q * kNetCh, umma_desc(smem_u32(sA + q * k1PlaneBytes + kh * 256), 128, 512),
                             bd + (uint64_t)((kh * 256) >> 4), idesc, (uint32_t)kh);
            mma_commit(mbar);
        }
        const bool ok = mbar_wait(mbar, phase);
        phase ^= 1u;
        if(__syncthreads_or(!ok))
        {
            if(tid == 0) atomicExch(status, 7);
            failed = true;
            break;
        }
        tc_fence_after();
#pragma unroll 1
        for(int q = 0; q < k1Z; ++q)
        {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(q * kNetCh), v);
            const int x = x0 + mx, y = y0 + my, z = z0 + q;
            if(x >= g.nx || y >= g.ny || z >= g.nz) continue;
            const long p = base + ((long)z * g.ny + y) * g.nx + x;
            float pos[16];
#pragma unroll
            for(int c = 0; c < 16; ++c) pos[c] = fmaxf(v[c], 0.f);
            uint4* dst = reinterpret_cast<uint4*>(a1 + p * kNetCh);
            dst[0] = pack_bf16x8(pos);
            dst[1] = pack_bf16x8(pos + 8);
            if(kPair)
            {
#pragma unroll
                for(int c = 0; c < 16; ++c) pos[c] = fmaxf(-v[c], 0.f);
                uint4* d2 = reinterpret_cast<uint4*>(a1 + (p + n) * kNetCh);
                d2[0] = pack_bf16x8(pos);
                d2[1] = pack_bf16x8(pos + 8);
            }
        }
        tc_fence_before();
        __syncthreads();  // TMEM, im2col planes and staged scalars free for the next brick
    }
    if(failed) mbar_wait(mbar, phase ^ 1u);  // the MMAs in flight finish before TMEM is released
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if(warp == 0) tmem_free(tmem, k1Cols);
}


// 1 / (e.e) (kind 0) or 1 / (e.Ae) (kind 1) per sample: one block per sample.
__global__ void k_sample_norm(ConvGrid g, const float* __restrict__ e, int kind, float* __restrict__ out)
{
    __shared__ double red[32];
    const long per = (long)g.nz * g.ny * g.nx;
    const long base = (long)blockIdx.x * per;
    double s = 0.0;
    for(long i = threadIdx.x; i < per; i += blockDim.x)
    {
        const float ev = e[base + i];
        s += (double)ev * (kind ? stencil_at(g, e, base + i) : ev);
    }
    s = block_sum(s, red);
    if(threadIdx.x == 0) out[blockIdx.x] = (float)(1.0 / s);
}

// d = y - e, y the network output (odd: (y[p] - y[p + n]) / 2).
__global__ void k_loss_diff(long n, const float* __restrict__ y, const float* __restrict__ e, int odd,
                            float* __restrict__ d)
{
    const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if(p >= n) return;
    const float yv = odd ? 0.5f * (y[p] - y[p + n]) : y[p];
    d[p] = yv - e[p];
}

constexpr int kLossBlocks = 1184;

// Loss terms d.Md * w (M = I for kind 0, the stencil A for kind 1, i.e. the
// error's energy norm) and the output gradient 2 M d w as BF16 channel 0 of
// G (odd: +/- half of it for the two branches).
__global__ void __launch_bounds__(256) k_loss_grad(ConvGrid g, const float* __restrict__ d,
                                                   const float* __restrict__ wnorm, float scale, int kind, int odd,
                                                   __nv_bfloat16* __restrict__ G, float* __restrict__ loss_partial)
{
    __shared__ float red[32];
    const long per = (long)g.nz * g.ny * g.nx;
    const long n = per * g.nb;
    float acc = 0.f;
    for(long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x)
    {
        const float w = wnorm[p / per] * scale;
        const float md = kind ? stencil_at(g, d, p) : d[p];
        acc += d[p] * md * w;
        const float gv = 2.f * md * w;
        if(odd)
        {
            store_embed(G, p, 0.5f * gv);
            store_embed(G, p + n, -0.5f * gv);
        }
        else
        {
            store_embed(G, p, gv);
        }
    }
    acc = block_sum(acc, red);
    if(threadIdx.x == 0) loss_partial[blockIdx.x] = acc;
}

// Projects the three layers' weights onto the odd-symmetric ("tied") form:
// hidden channels k and k+8 are a +/- pair, so that the network is an odd
// function of its input with one evaluation:
//   w1[t][0][k+8] = -w1[t][0][k]; w2[t][i][j] = w2[t][i^8][j^8]; w3[t][j^8][0] = -w3[t][j][0].
// Unused weights (layer 1 inputs >= 1, layer 3 outputs >= 1) are zeroed.
__global__ void k_tie_odd(float* __restrict__ w)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= kNetLayerWeights) return;
    const int t = i / 256, a = (i / 16) % 16, b = i % 16;
    float* w1 = w;
    float* w2 = w + kNetLayerWeights;
    float* w3 = w + 2 * kNetLayerWeights;
    // each pair/quad is handled by its lowest index
    if(a == 0 && b < 8)
    {
        const int k0 = (t * 16) * 16 + b, k1 = k0 + 8;
        const float v = 0.5f * (w1[k0] - w1[k1]);
        w1[k0] = v;
        w1[k1] = -v;
    }
    if(a != 0) w1[i] = 0.f;
    if(a < 8)
    {
        const int k0 = (t * 16 + a) * 16 + b, k1 = (t * 16 + (a ^ 8)) * 16 + (b ^ 8);
        const float v = 0.5f * (w2[k0] + w2[k1]);
        w2[k0] = v;
        w2[k1] = v;
    }
    if(b == 0 && a < 8)
    {
        const int k0 = (t * 16 + a) * 16, k1 = (t * 16 + (a ^ 8)) * 16;
        const float v = 0.5f * (w3[k0] - w3[k1]);
        w3[k0] = v;
        w3[k1] = -v;
    }
    if(b != 0) w3[i] = 0.f;
}

__global__ void k_adam(int n, float* __restrict__ w, const float* __restrict__ dw, float* __restrict__ m,
                       float* __restrict__ v, float lr, float beta1, float beta2, float eps, float c1, float c2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n) return;
    const float gi = dw[i];
    const float mi = beta1 * m[i] + (1.f - beta1) * gi;
    const float vi = beta2 * v[i] + (1.f - beta2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
}

// ------------------------------------------------------------ launchers

static int sm_count()
{
    static int sms = 0;
    if(sms == 0)
    {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if(sms <= 0) sms = 148;
    }
    return sms;
}

// Tensor map of a channel-last BF16 tensor [nb][nz][ny][nx][16] with a box
// of 16 channels x bx x by x bz points x 1 sample, written in the 32-byte
// swizzle that the A descriptors declare; the driver entry point is looked up
// once through the runtime.
static int bf16_box_map(const ConvGrid& g, const void* in, int bx, int by, int bz, CUtensorMap* map)
{
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if(!encode)
    {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        HB_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
        if(q != cudaDriverEntryPointSuccess || !fn)
            return record_error(HPCGB200_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
        encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    const cuuint64_t dims[5] = {(cuuint64_t)kNetCh, (cuuint64_t)g.nx, (cuuint64_t)g.ny, (cuuint64_t)g.nz,
                                (cuuint64_t)g.nb};
    const cuuint64_t row = (cuuint64_t)kNetCh * 2;
    const cuuint64_t strides[4] = {row, row * g.nx, row * g.nx * g.ny, row * g.nx * g.ny * g.nz};
    const cuuint32_t box[5] = {(cuuint32_t)kNetCh, (cuuint32_t)bx, (cuuint32_t)by, (cuuint32_t)bz, 1};
    const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
    const CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<void*>(in), dims, strides, box,
                              estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_32B,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if(r != CUDA_SUCCESS) return record_error(HPCGB200_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return 0;
}

// The conv brick box: 16 x 10 x 6 points (14 x 8 x 4 outputs and their halo).
static int conv_tensor_map(const ConvGrid& g, const void* in, CUtensorMap* map)
{
    return bf16_box_map(g, in, kTX, kHY, kHZ, map);
}

template <int kOut>
static int conv_launch(const ConvGrid& g, const void* in, const void* wB, void* out, const void* act, const PermMap& pm,
                       int* status, cudaStream_t s)
{
    static bool attr = false;
    if(!attr)
    {
        HB_CUDA(cudaFuncSetAttribute(k_conv16<kOut>, cudaFuncAttributeMaxDynamicSharedMemorySize, kConvSmem));
        attr = true;
    }
    CUtensorMap map;
    HB_RETURN_IF(conv_tensor_map(g, in, &map));
    const long tiles = (long)g.nb * ((g.nx + kOX - 1) / kOX) * ((g.ny + kTY - 1) / kTY) * ((g.nz + kTZ - 1) / kTZ);
    const long cap = (long)HB_CONV_CTAS * sm_count();
    const int grid = (int)(tiles < cap ? tiles : cap);
    HB_CUDA(launch_pdl_net(k_conv16<kOut>, dim3(grid), dim3(kConvThreads), (size_t)kConvSmem, s, map, g,
                           (const __nv_bfloat16*)wB, out, (const __nv_bfloat16*)act, pm, status));
    return 0;
}

int launch_conv16(const ConvGrid& g, const void* in, const void* wB, int out_mode, void* out, const void* act,
                  const PermMap* pm, int* status, cudaStream_t s)
{
    const PermMap none{};
    const PermMap& m = pm ? *pm : none;
    switch(out_mode)
    {
        case kOutReluBf16: return conv_launch<kOutReluBf16>(g, in, wB, out, act, m, status, s);
        case kOutMaskBf16: return conv_launch<kOutMaskBf16>(g, in, wB, out, act, m, status, s);
        case kOutF32: return conv_launch<kOutF32>(g, in, wB, out, act, m, status, s);
        case kOutF32C0: return conv_launch<kOutF32C0>(g, in, wB, out, act, m, status, s);
        case kOutPermSet: return conv_launch<kOutPermSet>(g, in, wB, out, act, m, status, s);
        case kOutPermAdd: return conv_launch<kOutPermAdd>(g, in, wB, out, act, m, status, s);
        default: return record_error(HPCGB200_ERR_ARG, "conv16: unknown output mode %d", out_mode);
    }
}

template <int kOut, bool kPair>
static int layer3_launch(const ConvGrid& g, const void* a2, const float* w3, float* out, const PermMap& pm,
                         int* status, cudaStream_t s)
{
    static bool attr = false;
    if(!attr)
    {
        HB_CUDA(cudaFuncSetAttribute(k_layer3_tc<kOut, kPair>, cudaFuncAttributeMaxDynamicSharedMemorySize, k3Smem));
        attr = true;
    }
    CUtensorMap map;
    const ConvGrid gin{kPair ? 2 * g.nb : g.nb, g.nz, g.ny, g.nx};
    HB_RETURN_IF(bf16_box_map(gin, a2, k3HX, k3HY, k3HZ, &map));
    const long tiles = (long)g.nb * ((g.nx + k3X - 1) / k3X) * ((g.ny + k3Y - 1) / k3Y) * ((g.nz + k3Z - 1) / k3Z);
    const long cap = sm_count();
    const int grid = (int)(tiles < cap ? tiles : cap);
    HB_CUDA(launch_pdl_net(k_layer3_tc<kOut, kPair>, dim3(grid), dim3(kConvThreads), (size_t)k3Smem, s, map, g, w3,
                           out, pm, status));
    return 0;
}

int launch_layer3_tc(const ConvGrid& g, const PermMap* pm, const void* a2, const float* w3, int pair, int mode,
                     float* out, int* status, cudaStream_t s)
{
    if(mode < 0 || mode > 2) return record_error(HPCGB200_ERR_ARG, "layer 3: unknown output mode %d", mode);
    if(mode != 2 && (!pm || g.nb != 1)) return record_error(HPCGB200_ERR_ARG, "layer 3: level output needs one sample");
    const PermMap m = pm ? *pm : PermMap{};
    if(pair)
    {
        if(mode == 0) return layer3_launch<0, true>(g, a2, w3, out, m, status, s);
        if(mode == 1) return layer3_launch<1, true>(g, a2, w3, out, m, status, s);
        return layer3_launch<2, true>(g, a2, w3, out, m, status, s);
    }
    if(mode == 0) return layer3_launch<0, false>(g, a2, w3, out, m, status, s);
    if(mode == 1) return layer3_launch<1, false>(g, a2, w3, out, m, status, s);
    return layer3_launch<2, false>(g, a2, w3, out, m, status, s);
}

int conv16_wgrad_parts(long points)
{
    const long nblk = (points + kWgK - 1) / kWgK;
    const long cap = 3L * sm_count();
    return (int)(nblk < cap ? nblk : cap);
}

int launch_conv16_wgrad(const ConvGrid& g, const void* x, const void* gr, float* partial, float* dw, int* status,
                        cudaStream_t s)
{
    static bool attr = false;
    if(!attr)
    {
        HB_CUDA(cudaFuncSetAttribute(k_conv16_wgrad, cudaFuncAttributeMaxDynamicSharedMemorySize, kWgSmem));
        attr = true;
    }
    const int parts = conv16_wgrad_parts(g.points());
    k_conv16_wgrad<<<parts, kWgThreads, kWgSmem, s>>>(g, (const __nv_bfloat16*)x, (const __nv_bfloat16*)gr, partial,
                                                      status);
    HB_LAUNCHED();
    k_wgrad_reduce<<<(kNetLayerWeights + 255) / 256, 256, 0, s>>>(parts, partial, dw);
    HB_LAUNCHED();
    return 0;
}

int launch_prepare_weights(const float* w, void* wB, int flip, cudaStream_t s)
{
    k_prepare_weights<<<(kNetLayerWeights + 255) / 256, 256, 0, s>>>(w, (__nv_bfloat16*)wB, flip);
    HB_LAUNCHED();
    return 0;
}

int launch_embed_level(const PermMap& pm, int nz, int ny, int nx, const float* r, const float* x,
                       const float* diag32, void* a, int pair, cudaStream_t s)
{
    const long n = (long)nz * ny * nx;
    k_embed_level<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(pm, nz, ny, nx, r, x, diag32, (__nv_bfloat16*)a,
                                                              pair);
    HB_LAUNCHED();
    return 0;
}

int launch_odd_combine(const PermMap& pm, int nz, int ny, int nx, const float* y, float* x, bool add, cudaStream_t s)
{
    const long n = (long)nz * ny * nx;
    if(add) k_odd_combine<true><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(pm, nz, ny, nx, y, x);
    else k_odd_combine<false><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(pm, nz, ny, nx, y, x);
    HB_LAUNCHED();
    return 0;
}

int launch_embed_scalar_level(const PermMap& pm, int nz, int ny, int nx, const float* r, const float* x,
                              const float* diag32, void* s1, cudaStream_t s)
{
    const long n = (long)nz * ny * nx;
    HB_CUDA(launch_pdl_net(k_embed_scalar_level, dim3((unsigned)((n + 255) / 256)), dim3(256), 0, s, pm, nz, ny, nx, r,
                           x, diag32, (__nv_bfloat16*)s1));
    return 0;
}


template <typename Tin, bool kPair>
static int layer1_launch(const ConvGrid& g, const Tin* in, const float* w1, __nv_bfloat16* a1, int* status,
                         cudaStream_t s)
{
    static bool attr = false;
    if(!attr)
    {
        HB_CUDA(cudaFuncSetAttribute(k_layer1_tc<Tin, kPair>, cudaFuncAttributeMaxDynamicSharedMemorySize, k1Smem));
        attr = true;
    }
    const long tiles = (long)g.nb * ((g.nx + k1X - 1) / k1X) * ((g.ny + k1Y - 1) / k1Y) * ((g.nz + k1Z - 1) / k1Z);
    const long cap = (long)k1CtasPerSm * sm_count();
    const int grid = (int)(tiles < cap ? tiles : cap);
    HB_CUDA(launch_pdl_net(k_layer1_tc<Tin, kPair>, dim3(grid), dim3(k1Threads), (size_t)k1Smem, s, g, in, w1, a1,
                           status));
    return 0;
}

int launch_layer1_tc(const ConvGrid& g, const void* in, int in_f32, const float* w1, void* a1, int pair, int* status,
                     cudaStream_t s)
{
    auto* out = (__nv_bfloat16*)a1;
    if(in_f32)
        return pair ? layer1_launch<float, true>(g, (const float*)in, w1, out, status, s)
                    : layer1_launch<float, false>(g, (const float*)in, w1, out, status, s);
    return pair ? layer1_launch<__nv_bfloat16, true>(g, (const __nv_bfloat16*)in, w1, out, status, s)
                : layer1_launch<__nv_bfloat16, false>(g, (const __nv_bfloat16*)in, w1, out, status, s);
}

int launch_odd_natural(long n, const float* y, float* out, cudaStream_t s)
{
    k_odd_natural<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, y, out);
    HB_LAUNCHED();
    return 0;
}

int launch_sample_norm(const ConvGrid& g, const float* e, int kind, float* out, cudaStream_t s)
{
    k_sample_norm<<<g.nb, 512, 0, s>>>(g, e, kind, out);
    HB_LAUNCHED();
    return 0;
}

int launch_natural_from_perm(const PermMap& pm, int nz, int ny, int nx, const float* in, float* out, cudaStream_t s)
{
    const long n = (long)nz * ny * nx;
    k_perm_copy<float, float, true><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(pm, nz, ny, nx, in, out);
    HB_LAUNCHED();
    return 0;
}

int launch_natural_from_perm(const PermMap& pm, int nz, int ny, int nx, const double* in, float* out, cudaStream_t s)
{
    const long n = (long)nz * ny * nx;
    k_perm_copy<double, float, true><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(pm, nz, ny, nx, in, out);
    HB_LAUNCHED();
    return 0;
}

int launch_perm_from_natural(const PermMap& pm, int nz, int ny, int nx, const float* in, double* out, cudaStream_t s)
{
    const long n = (long)nz * ny * nx;
    k_perm_copy<float, double, false><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(pm, nz, ny, nx, in, out);
    HB_LAUNCHED();
    return 0;
}

int launch_inv_sumsq(long n, const float* e, float* out, cudaStream_t s)
{
    k_inv_sumsq<<<1, 1024, 0, s>>>(n, e, out);
    HB_LAUNCHED();
    return 0;
}

int launch_loss_accumulate(const float* partial, double* acc, cudaStream_t s)
{
    k_loss_accumulate<<<1, 1024, 0, s>>>(kLossBlocks, partial, acc);
    HB_LAUNCHED();
    return 0;
}

int launch_normal_rhs(long long m, unsigned long long seed, const int* perm, double* out64, float* out32,
                      cudaStream_t s)
{
    k_normal_rhs<<<(unsigned)((m + 255) / 256), 256, 0, s>>>(m, seed, perm, out64, out32);
    HB_LAUNCHED();
    return 0;
}

int launch_embed_f32(long n, const float* r, void* a, int pair, cudaStream_t s)
{
    k_embed_f32<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, r, (__nv_bfloat16*)a, pair);
    HB_LAUNCHED();
    return 0;
}

int loss_parts(long points)
{
    (void)points;
    return kLossBlocks;
}

int launch_loss_grad(const ConvGrid& g, const float* y, const float* e, float* d, const float* wnorm, float scale,
                     int kind, int odd, void* G, float* loss_partial, cudaStream_t s)
{
    const long n = g.points();
    k_loss_diff<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, y, e, odd, d);
    HB_LAUNCHED();
    k_loss_grad<<<kLossBlocks, 256, 0, s>>>(g, d, wnorm, scale, kind, odd, (__nv_bfloat16*)G, loss_partial);
    HB_LAUNCHED();
    return 0;
}

int launch_tie_odd(float* w, cudaStream_t s)
{
    k_tie_odd<<<(kNetLayerWeights + 255) / 256, 256, 0, s>>>(w);
    HB_LAUNCHED();
    return 0;
}

int launch_adam(int n, float* w, const float* dw, float* m, float* v, float lr, float beta1, float beta2, float eps,
                int t, cudaStream_t s)
{
    const float c1 = 1.f / (1.f - std::pow(beta1, (float)t));
    const float c2 = 1.f / (1.f - std::pow(beta2, (float)t));
    k_adam<<<(n + 255) / 256, 256, 0, s>>>(n, w, dw, m, v, lr, beta1, beta2, eps, c1, c2);
    HB_LAUNCHED();
    return 0;
}

}  // namespace hb

using namespace hb;

// ------------------------------------------------------------------ C ABI

extern "C" size_t hpcgb200_conv_weight_tile_bytes(void) { return kNetWeightTileBytes; }

extern "C" int hpcgb200_conv_prepare_weights(const float* w, void* wB, int flip, void* stream)
{
    HB_CHECK_ARG(w && wB, "bad arguments");
    HB_CHECK_ARG((reinterpret_cast<uintptr_t>(wB) & 15) == 0, "wB must be 16-byte aligned");
    return launch_prepare_weights(w, wB, flip, as_stream(stream));
}

extern "C" int hpcgb200_conv16(int nb, int nz, int ny, int nx, const void* in, const void* wB, int out_mode, void* out,
                               const void* act, int* status, void* stream)
{
    HB_CHECK_ARG(nb > 0 && nz > 0 && ny > 0 && nx > 0 && in && wB && out && status, "bad arguments");
    HB_CHECK_ARG(out_mode >= kOutReluBf16 && out_mode <= kOutF32C0, "out_mode must be 0..3");
    HB_CHECK_ARG(out_mode != kOutMaskBf16 || act, "the masked mode needs the activation tensor");
    HB_CHECK_ARG((reinterpret_cast<uintptr_t>(in) & 15) == 0 && (reinterpret_cast<uintptr_t>(wB) & 15) == 0 &&
                     (reinterpret_cast<uintptr_t>(out) & 15) == 0 && (reinterpret_cast<uintptr_t>(act) & 15) == 0,
                 "tensors must be 16-byte aligned");
    const ConvGrid g{nb, nz, ny, nx};
    return launch_conv16(g, in, wB, out_mode, out, act, nullptr, status, as_stream(stream));
}

extern "C" size_t hpcgb200_conv_wgrad_partial_bytes(int nb, int nz, int ny, int nx)
{
    return sizeof(float) * kNetLayerWeights * (size_t)conv16_wgrad_parts((long)nb * nz * ny * nx);
}

extern "C" int hpcgb200_conv16_wgrad(int nb, int nz, int ny, int nx, const void* x, const void* g, float* partial,
                                     float* dw, int* status, void* stream)
{
    HB_CHECK_ARG(nb > 0 && nz > 0 && ny > 0 && nx > 0 && x && g && partial && dw && status, "bad arguments");
    HB_CHECK_ARG((reinterpret_cast<uintptr_t>(x) & 15) == 0 && (reinterpret_cast<uintptr_t>(g) & 15) == 0 &&
                     (reinterpret_cast<uintptr_t>(partial) & 15) == 0,
                 "tensors must be 16-byte aligned");
    const ConvGrid cg{nb, nz, ny, nx};
    return launch_conv16_wgrad(cg, x, g, partial, dw, status, as_stream(stream));
}

extern "C" int hpcgb200_normal_rhs(long long m, unsigned long long seed, double* out, void* stream)
{
    HB_CHECK_ARG(m >= 0 && (m == 0 || out), "bad arguments");
    if(m == 0) return 0;
    return launch_normal_rhs(m, seed, nullptr, out, nullptr, as_stream(stream));
}

extern "C" int hpcgb200_sample_norms(int nb, int nz, int ny, int nx, const float* e, int kind, float* out, void* stream)
{
    HB_CHECK_ARG(nb > 0 && nz > 0 && ny > 0 && nx > 0 && e && out && (kind == 0 || kind == 1), "bad arguments");
    return launch_sample_norm(ConvGrid{nb, nz, ny, nx}, e, kind, out, as_stream(stream));
}
