// Learned smoother: the conv net's device state, its place in the FP32
// V-cycle, its training (forward, backward, Adam on the device) and the
// generation of its training pairs.  No reference counterpart.
//
// In the V-cycle (ComputeMG_Learned) the levels >= the smoother's first level
// replace SymGS by the network N, which approximates the level's inverse:
//     x = N(r); restrict; coarse cycle; prolong; x += N(r - A x)
// and the coarsest level is x = N(r).  Training pairs (r, e) are the
// residual that the plain FP32 V-cycle hands to that level for a seeded
// N(0,1) right-hand side and the level's exact correction e = A^-1 r (an FP64
// MG-PCG solve on a grid of the level's size).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <utility>

#include "hpcg_b200.h"
#include "learned.hpp"
#include "problem.hpp"

using namespace hpcg_b200;

namespace hpcg_b200 {

Smoother::Smoother()
{
    cudaStream_t s = rt().stream;
    w = dalloc<float>(kNetWeights);
    HB_HOST_CUDA(cudaMemsetAsync(w, 0, sizeof(float) * kNetWeights, s));
    wB = dalloc<unsigned char>(3 * (size_t)hb::kNetWeightTileBytes);
    wT = dalloc<unsigned char>(3 * (size_t)hb::kNetWeightTileBytes);
    status = dalloc<int>(1);
    HB_HOST_CUDA(cudaMemsetAsync(status, 0, sizeof(int), s));
    HB_HOST_CUDA(cudaStreamSynchronize(s));
}

Smoother::~Smoother()
{
    for(void* p : {(void*)w, (void*)wB, (void*)wT, a0, a1, a2, g, d, (void*)y, (void*)dbuf, (void*)dw,
                   (void*)adam_m, (void*)adam_v, (void*)partial, (void*)loss_partial, (void*)loss_acc, (void*)status})
        dfree(p);
}

void smoother_configure(Smoother& S, int symmetry, cudaStream_t s)
{
    const bool odd = symmetry == 1;
    S.tied = symmetry == 2;
    if(S.tied)
    {
        check(hb::launch_tie_odd(S.w, s));
        S.tiles_stale = true;
    }
    if(S.odd == odd) return;
    S.odd = odd;
    S.cap = 0;  // branch count changed: reallocate on next use
}

void smoother_reserve(Smoother& S, long points, bool training)
{
    const long br = S.odd ? 2 : 1;  // network evaluations per grid point
    const bool grow = points > S.cap;
    if(grow)
    {
        for(void** p : {&S.a0, &S.a1, &S.a2, &S.g, &S.d})
        {
            dfree(*p);
            *p = nullptr;
        }
        dfree(S.y);
        dfree(S.dbuf);
        S.y = nullptr;
        S.dbuf = nullptr;
        S.a0 = dalloc<uint4>((size_t)points * br * 2);
        S.a1 = dalloc<uint4>((size_t)points * br * 2);
        S.a2 = dalloc<uint4>((size_t)points * br * 2);
        S.y = dalloc<float>((size_t)points * br);
        S.cap = points;
        S.epoch += 1;  // solve graphs that captured the old buffers are stale
    }
    if(!training) return;
    if(!S.g)
    {
        S.g = dalloc<uint4>((size_t)S.cap * br * 2);
        S.d = dalloc<uint4>((size_t)S.cap * br * 2);
        S.dbuf = dalloc<float>((size_t)S.cap);
    }
    const size_t pf = hb::kNetLayerWeights * (size_t)hb::conv16_wgrad_parts(S.cap * br);
    if(pf > S.partial_floats)
    {
        dfree(S.partial);
        S.partial = dalloc<float>(pf);
        S.partial_floats = pf;
    }
    if(!S.dw)
    {
        cudaStream_t s = rt().stream;
        S.dw = dalloc<float>(kNetWeights);
        S.adam_m = dalloc<float>(kNetWeights);
        S.adam_v = dalloc<float>(kNetWeights);
        HB_HOST_CUDA(cudaMemsetAsync(S.adam_m, 0, sizeof(float) * kNetWeights, s));
        HB_HOST_CUDA(cudaMemsetAsync(S.adam_v, 0, sizeof(float) * kNetWeights, s));
        S.loss_partial = dalloc<float>(hb::loss_parts(0));
        S.loss_acc = dalloc<double>(1);
        HB_HOST_CUDA(cudaMemsetAsync(S.loss_acc, 0, sizeof(double), s));
        HB_HOST_CUDA(cudaStreamSynchronize(s));
    }
}

void smoother_set_weights(Smoother& S, const float* host_w, cudaStream_t s)
{
    HB_HOST_CUDA(cudaMemcpyAsync(S.w, host_w, sizeof(float) * kNetWeights, cudaMemcpyHostToDevice, s));
    if(S.tied) check(hb::launch_tie_odd(S.w, s));
    S.tiles_stale = true;
    S.adam_t = 0;
    if(S.adam_m)
    {
        HB_HOST_CUDA(cudaMemsetAsync(S.adam_m, 0, sizeof(float) * kNetWeights, s));
        HB_HOST_CUDA(cudaMemsetAsync(S.adam_v, 0, sizeof(float) * kNetWeights, s));
    }
    HB_HOST_CUDA(cudaStreamSynchronize(s));
}

int smoother_prepare(Smoother& S, cudaStream_t s)
{
    if(!S.tiles_stale) return 0;
    for(int l = 0; l < 3; ++l)
    {
        const float* wl = S.w + l * hb::kNetLayerWeights;
        HB_RETURN_IF(hb::launch_prepare_weights(wl, S.wB + l * hb::kNetWeightTileBytes, 0, s));
        HB_RETURN_IF(hb::launch_prepare_weights(wl, S.wT + l * hb::kNetWeightTileBytes, 1, s));
    }
    S.tiles_stale = false;
    return 0;
}

static const void* tiles(const Smoother& S, int layer) { return S.wB + layer * hb::kNetWeightTileBytes; }
static const void* tiles_t(const Smoother& S, int layer) { return S.wT + layer * hb::kNetWeightTileBytes; }

int smoother_level_apply(Smoother& S, const LevelOpt& o, const float* r, float* x, bool residual, cudaStream_t s)
{
    const hb::StencilLevel& L = o.st;
    const hb::ConvGrid g{S.odd ? 2 : 1, L.nz, L.ny, L.nx};
    if((long)L.nz * L.ny * L.nx > S.cap)
        return hb::record_error(HPCGB200_ERR_ARG, "learned smoother: buffers not reserved");
    if(S.tiles_stale) return hb::record_error(HPCGB200_ERR_ARG, "learned smoother: weights not prepared");
    // all three layers on the tensor cores: layer 1 with the taps as K (one
    // input channel), layer 2 (16 -> 16), layer 3 with the taps stacked in N
    // and the odd pair folded into K; the scalar input field lives in a0
    const hb::ConvGrid g1{1, L.nz, L.ny, L.nx};
    HB_RETURN_IF(hb::launch_embed_scalar_level(o.pm, L.nz, L.ny, L.nx, r, residual ? x : nullptr, o.diag32, S.a0, s));
    HB_RETURN_IF(hb::launch_layer1_tc(g1, S.a0, 0, S.w, S.a1, S.odd ? 1 : 0, S.status, s));
    HB_RETURN_IF(hb::launch_conv16(g, S.a1, tiles(S, 1), hb::kOutReluBf16, S.a2, nullptr, nullptr, S.status, s));
    return hb::launch_layer3_tc(g1, &o.pm, S.a2, S.w + 2 * hb::kNetLayerWeights, S.odd ? 1 : 0, residual ? 1 : 0, x,
                                S.status, s);
}

// Raw network output of a batch into y (both branches, 2 g.nb samples, when odd).
static int forward_batch(Smoother& S, const hb::ConvGrid& g, const float* r, float* y, cudaStream_t s)
{
    const hb::ConvGrid gg{S.odd ? 2 * g.nb : g.nb, g.nz, g.ny, g.nx};
    HB_RETURN_IF(smoother_prepare(S, s));
    HB_RETURN_IF(hb::launch_embed_f32(g.points(), r, S.a0, S.odd ? 1 : 0, s));
    HB_RETURN_IF(hb::launch_conv16(gg, S.a0, tiles(S, 0), hb::kOutReluBf16, S.a1, nullptr, nullptr, S.status, s));
    HB_RETURN_IF(hb::launch_conv16(gg, S.a1, tiles(S, 1), hb::kOutReluBf16, S.a2, nullptr, nullptr, S.status, s));
    return hb::launch_conv16(gg, S.a2, tiles(S, 2), hb::kOutF32C0, y, nullptr, nullptr, S.status, s);
}

// Evaluation as in the V-cycle (the one-channel forms of layers 1 and 3).
int smoother_forward(Smoother& S, const hb::ConvGrid& g, const float* r, float* y, cudaStream_t s)
{
    smoother_reserve(S, g.points(), false);
    HB_RETURN_IF(smoother_prepare(S, s));
    const hb::ConvGrid gg{S.odd ? 2 * g.nb : g.nb, g.nz, g.ny, g.nx};
    HB_RETURN_IF(hb::launch_layer1_tc(g, r, 1, S.w, S.a1, S.odd ? 1 : 0, S.status, s));
    HB_RETURN_IF(hb::launch_conv16(gg, S.a1, tiles(S, 1), hb::kOutReluBf16, S.a2, nullptr, nullptr, S.status, s));
    return hb::launch_layer3_tc(g, nullptr, S.a2, S.w + 2 * hb::kNetLayerWeights, S.odd ? 1 : 0, 2, y, S.status, s);
}

int smoother_loss_grad(Smoother& S, const hb::ConvGrid& g0, const float* r, const float* e, const float* wnorm,
                       float scale, int kind, cudaStream_t s)
{
    smoother_reserve(S, g0.points(), true);
    HB_RETURN_IF(forward_batch(S, g0, r, S.y, s));
    HB_RETURN_IF(hb::launch_loss_grad(g0, S.y, e, S.dbuf, wnorm, scale, kind, S.odd ? 1 : 0, S.g, S.loss_partial, s));
    HB_RETURN_IF(hb::launch_loss_accumulate(S.loss_partial, S.loss_acc, s));
    const hb::ConvGrid g{S.odd ? 2 * g0.nb : g0.nb, g0.nz, g0.ny, g0.nx};
    float* dw1 = S.dw;
    float* dw2 = S.dw + hb::kNetLayerWeights;
    float* dw3 = S.dw + 2 * hb::kNetLayerWeights;
    // layer 3: dW3 = a2 (x) G; dL/da2 = conv(G, W3^T) where a2 > 0
    HB_RETURN_IF(hb::launch_conv16_wgrad(g, S.a2, S.g, S.partial, dw3, S.status, s));
    HB_RETURN_IF(hb::launch_conv16(g, S.g, tiles_t(S, 2), hb::kOutMaskBf16, S.d, S.a2, nullptr, S.status, s));
    // layer 2
    HB_RETURN_IF(hb::launch_conv16_wgrad(g, S.a1, S.d, S.partial, dw2, S.status, s));
    HB_RETURN_IF(hb::launch_conv16(g, S.d, tiles_t(S, 1), hb::kOutMaskBf16, S.g, S.a1, nullptr, S.status, s));
    // layer 1 (input a0)
    return hb::launch_conv16_wgrad(g, S.a0, S.g, S.partial, dw1, S.status, s);
}

int smoother_adam(Smoother& S, float lr, float beta1, float beta2, float eps, cudaStream_t s)
{
    if(!S.dw) return hb::record_error(HPCGB200_ERR_ARG, "learned smoother: no gradient computed yet");
    S.adam_t += 1;
    HB_RETURN_IF(hb::launch_adam(kNetWeights, S.w, S.dw, S.adam_m, S.adam_v, lr, beta1, beta2, eps, S.adam_t, s));
    if(S.tied) HB_RETURN_IF(hb::launch_tie_odd(S.w, s));
    S.tiles_stale = true;
    return 0;
}

int smoother_status(Smoother& S, cudaStream_t s)
{
    int h = 0;
    HB_HOST_CUDA(cudaMemcpyAsync(&h, S.status, sizeof(int), cudaMemcpyDeviceToHost, s));
    HB_HOST_CUDA(cudaStreamSynchronize(s));
    if(h)
    {
        HB_HOST_CUDA(cudaMemsetAsync(S.status, 0, sizeof(int), s));
        return hb::record_error(HPCGB200_ERR_DEVICE_STATUS, "learned smoother: tensor-core wait timed out (%d)", h);
    }
    return 0;
}

int smoother_ready(const SparseMatrix& A, cudaStream_t s)
{
    LevelOpt* o = opt(A);
    const SparseMatrix* M = &A;
    for(int l = 0; l < o->smoother_first_level && M; ++l) M = M->Ac;
    if(!M) return hb::record_error(HPCGB200_ERR_ARG, "learned smoother: first level beyond the hierarchy");
    smoother_reserve(*o->smoother, M->localNumberOfRows, false);
    return smoother_prepare(*o->smoother, s);
}

// FP32 V-cycle below level 0 with the learned levels (same recursion as
// mg_fp32).  A SymGS level takes the prolongation into the finer level in its
// final passes (`pro`); below a learned level, or from one, it is a launch
// of its own (the network is the level's last operation).
static int mg_fp32_learned(const SparseMatrix& A, int level, Smoother& S, int first, int coarse_steps, const float* r,
                           float* x, cudaStream_t s, hb::Prolong<float> pro = {})
{
    const LevelOpt* o = opt(A);
    const bool learned = level >= first;
    if(learned) HB_RETURN_IF(smoother_level_apply(S, *o, r, x, false, s));
    else
        HB_RETURN_IF(hb::launch32_symgs_zero(o->st, o->diag32, o->inv_diag32, nullptr, const_cast<float*>(r), x, s,
                                             A.mgData ? hb::Prolong<float>{} : pro));
    if(!A.mgData)
    {
        // coarsest level: further learned Richardson steps x += N(r - A x)
        for(int k = 1; learned && k < coarse_steps; ++k) HB_RETURN_IF(smoother_level_apply(S, *o, r, x, true, s));
        return 0;
    }
    const MGOpt* mo = mgopt(A);
    const int nc = A.Ac->localNumberOfRows;
    const bool separate_prolong = level + 1 >= first || !fused_prolongation();
    HB_RETURN_IF(hb::launch32_restrict(o->st, nc, mo->inj_f, mo->inj_c, o->diag32, r, x, mo->rc32, s));
    HB_RETURN_IF(mg_fp32_learned(*A.Ac, level + 1, S, first, coarse_steps, mo->rc32, mo->xc32, s,
                                 separate_prolong ? hb::Prolong<float>{} : hb::Prolong<float>{x, mo->pro_f}));
    if(separate_prolong) HB_RETURN_IF(hb::launch32_prolong(o->st, nc, mo->inj_f, mo->inj_c, mo->xc32, x, s));
    if(learned) return smoother_level_apply(S, *o, r, x, true, s);
    return hb::launch32_symgs(o->st, o->inv_diag32, r, x, nullptr, s, pro);
}

}  // namespace hpcg_b200

namespace hpcg_b200 {

int mg_learned_to(const SparseMatrix& A, const double* r64, double* z64, cudaStream_t s)
{
    {
        const LevelOpt* o = opt(A);
        if(!o || !o->smoother)
            return hb::record_error(HPCGB200_ERR_ARG, "learned V-cycle: no smoother attached to the problem");
        for(const SparseMatrix* M = &A; M; M = M->Ac)
            if(!opt(*M) || !opt(*M)->stencil_ok)
                return hb::record_error(HPCGB200_ERR_NOT_STENCIL,
                                        "learned V-cycle needs the 27-point stencil in parity colouring on every level");
        Smoother& S = *o->smoother;
        const int first = o->smoother_first_level;
        const int m = A.localNumberOfRows;
        if(first <= 0) return hb::record_error(HPCGB200_ERR_ARG, "learned V-cycle: the fine level keeps SymGS");
        // operand tiles are refreshed outside graph capture (a captured cycle
        // reads the tile buffers, which later refreshes update in place)
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        HB_HOST_CUDA(cudaStreamIsCapturing(s, &cs));
        if(cs == cudaStreamCaptureStatusNone) HB_RETURN_IF(smoother_ready(A, s));
        HB_RETURN_IF(hb::launch32_symgs_zero(o->st, o->diag32, o->inv_diag32, r64, o->r32, o->z32, s));
        if(!A.mgData) return z64 ? hb::launch_cast_f2d(m, o->z32, z64, s) : 0;
        const MGOpt* mo = mgopt(A);
        const int nc = A.Ac->localNumberOfRows;
        HB_RETURN_IF(hb::launch32_restrict(o->st, nc, mo->inj_f, mo->inj_c, o->diag32, o->r32, o->z32, mo->rc32, s));
        const bool separate_prolong = first <= 1 || !fused_prolongation();
        HB_RETURN_IF(mg_fp32_learned(*A.Ac, 1, S, first, o->smoother_coarse_steps, mo->rc32, mo->xc32, s,
                                     separate_prolong ? hb::Prolong<float>{} : hb::Prolong<float>{o->z32, mo->pro_f}));
        if(separate_prolong) HB_RETURN_IF(hb::launch32_prolong(o->st, nc, mo->inj_f, mo->inj_c, mo->xc32, o->z32, s));
        return hb::launch32_symgs(o->st, o->inv_diag32, o->r32, o->z32, z64, s);
    }
}

}  // namespace hpcg_b200

int ComputeMG_Learned(const SparseMatrix& A, const Vector& r, Vector& x)
{
    try
    {
        ensure_runtime();
        return mg_learned_to(A, r.d_values, x.d_values, rt().stream);
    }
    catch(const Error& e)
    {
        return report(e);
    }
}

// ------------------------------------------------------------------ C ABI

struct hpcgb200_smoother
{
    Smoother S;
    cudaStream_t stream = nullptr;
};

namespace {

cudaStream_t stream_of(void* s) { return s ? reinterpret_cast<cudaStream_t>(s) : rt().stream; }

// SplitMix64 stream for the initial weights and the batch order.
struct Rng
{
    unsigned long long z;
    unsigned long long next()
    {
        unsigned long long x = (z += 0x9E3779B97F4A7C15ULL);
        x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
        x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
        return x ^ (x >> 31);
    }
    double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }  // [0, 1)
};

}  // namespace

extern "C" int hpcgb200_smoother_create(hpcgb200_smoother** out)
{
    if(!out) return hb::record_error(HPCGB200_ERR_ARG, "out is null");
    *out = nullptr;
    return guarded([&] {
        auto* h = new hpcgb200_smoother;
        h->stream = rt().stream;
        *out = h;
        return 0;
    });
}

extern "C" int hpcgb200_smoother_destroy(hpcgb200_smoother* h)
{
    if(!h) return 0;
    return guarded([&] {
        cudaStreamSynchronize(h->stream);
        delete h;
        return 0;
    });
}

extern "C" int hpcgb200_smoother_set_weights(hpcgb200_smoother* h, const float* host_w)
{
    if(!h || !host_w) return hb::record_error(HPCGB200_ERR_ARG, "bad arguments");
    return guarded([&] {
        smoother_set_weights(h->S, host_w, h->stream);
        return 0;
    });
}

extern "C" int hpcgb200_smoother_get_weights(hpcgb200_smoother* h, float* host_w)
{
    if(!h || !host_w) return hb::record_error(HPCGB200_ERR_ARG, "bad arguments");
    return guarded([&] {
        HB_HOST_CUDA(cudaMemcpyAsync(host_w, h->S.w, sizeof(float) * kNetWeights, cudaMemcpyDeviceToHost, h->stream));
        HB_HOST_CUDA(cudaStreamSynchronize(h->stream));
        return 0;
    });
}

extern "C" int hpcgb200_smoother_init_jacobi(float* host_w, float omega, float noise, unsigned long long seed,
                                             int twin)
{
    if(!host_w || twin < 1 || twin > 15) return hb::record_error(HPCGB200_ERR_ARG, "bad arguments");
    constexpr int W = hb::kNetLayerWeights;
    Rng rng{seed};
    auto at = [](int tap, int ci, int co) { return (tap * 16 + ci) * 16 + co; };
    for(int l = 0; l < 3; ++l)
        for(int i = 0; i < W; ++i)
        {
            const int ci = (i / 16) % 16, co = i % 16;
            const bool used = (l != 0 || ci == 0) && (l != 2 || co == 0);
            host_w[l * W + i] = used ? (float)(noise * (2.0 * rng.uniform() - 1.0)) : 0.f;
        }
    // centre tap: channel 0 = relu(r), channel `twin` = relu(-r), identity, out = omega (c0 - c_twin) / 26
    host_w[0 * W + at(13, 0, 0)] += 1.f;
    host_w[0 * W + at(13, 0, twin)] += -1.f;
    host_w[1 * W + at(13, 0, 0)] += 1.f;
    host_w[1 * W + at(13, twin, twin)] += 1.f;
    host_w[2 * W + at(13, 0, 0)] += omega / 26.f;
    host_w[2 * W + at(13, twin, 0)] += -omega / 26.f;
    return 0;
}

extern "C" int hpcgb200_smoother_forward(hpcgb200_smoother* h, int nb, int nz, int ny, int nx, const float* r,
                                         float* y, void* stream)
{
    if(!h || nb <= 0 || nz <= 0 || ny <= 0 || nx <= 0 || !r || !y)
        return hb::record_error(HPCGB200_ERR_ARG, "bad arguments");
    return guarded([&] {
        cudaStream_t s = stream_of(stream);
        HB_RETURN_IF(smoother_forward(h->S, hb::ConvGrid{nb, nz, ny, nx}, r, y, s));
        return smoother_status(h->S, s);
    });
}

extern "C" int hpcgb200_smoother_configure(hpcgb200_smoother* h, int symmetry)
{
    if(!h || symmetry < 0 || symmetry > 2) return hb::record_error(HPCGB200_ERR_ARG, "bad arguments");
    return guarded([&] {
        HB_HOST_CUDA(cudaStreamSynchronize(h->stream));
        smoother_configure(h->S, symmetry, h->stream);
        HB_HOST_CUDA(cudaStreamSynchronize(h->stream));
        return 0;
    });
}

extern "C" int hpcgb200_smoother_loss_grad(hpcgb200_smoother* h, int nb, int nz, int ny, int nx, const float* r,
                                           const float* e, const float* inv_norm, float scale, int kind, float* dw,
                                           double* loss, void* stream)
{
    if(!h || nb <= 0 || nz <= 0 || ny <= 0 || nx <= 0 || !r || !e || !inv_norm || (kind != 0 && kind != 1))
        return hb::record_error(HPCGB200_ERR_ARG, "bad arguments");
    return guarded([&] {
        cudaStream_t s = stream_of(stream);
        Smoother& S = h->S;
        smoother_reserve(S, (long)nb * nz * ny * nx, true);
        HB_HOST_CUDA(cudaMemsetAsync(S.loss_acc, 0, sizeof(double), s));
        HB_RETURN_IF(smoother_loss_grad(S, hb::ConvGrid{nb, nz, ny, nx}, r, e, inv_norm, scale, kind, s));
        if(dw)
            HB_HOST_CUDA(cudaMemcpyAsync(dw, S.dw, sizeof(float) * kNetWeights, cudaMemcpyDeviceToDevice, s));
        double l = 0.0;
        HB_HOST_CUDA(cudaMemcpyAsync(&l, S.loss_acc, sizeof(double), cudaMemcpyDeviceToHost, s));
        HB_RETURN_IF(smoother_status(S, s));
        if(loss) *loss = l;
        return 0;
    });
}

extern "C" int hpcgb200_smoother_adam_step(hpcgb200_smoother* h, float lr, float beta1, float beta2, float eps,
                                           void* stream)
{
    if(!h) return hb::record_error(HPCGB200_ERR_ARG, "bad arguments");
    return guarded([&] { return smoother_adam(h->S, lr, beta1, beta2, eps, stream_of(stream)); });
}

extern "C" int hpcgb200_smoother_train(hpcgb200_smoother* h, const hpcgb200_pair_set* sets, int nsets, int epochs,
                                       float lr0, float lr1, int kind, unsigned long long seed, double* epoch_loss,
                                       void* stream)
{
    if(!h || !sets || nsets <= 0 || epochs <= 0 || !(lr0 > 0.f) || !(lr1 > 0.f) || (kind != 0 && kind != 1))
        return hb::record_error(HPCGB200_ERR_ARG, "bad arguments");
    for(int i = 0; i < nsets; ++i)
        if(!sets[i].r || !sets[i].e || !sets[i].inv_ee || sets[i].count <= 0 || sets[i].batch <= 0 ||
           sets[i].batch > sets[i].count || sets[i].nz <= 0 || sets[i].ny <= 0 || sets[i].nx <= 0)
            return hb::record_error(HPCGB200_ERR_ARG, "pair set %d is invalid", i);
    return guarded([&] {
        cudaStream_t s = stream_of(stream);
        Smoother& S = h->S;
        long maxpts = 0;
        std::vector<std::pair<int, int>> steps;  // (set, batch index)
        for(int i = 0; i < nsets; ++i)
        {
            const long per = (long)sets[i].nz * sets[i].ny * sets[i].nx;
            maxpts = std::max(maxpts, per * sets[i].batch);
            for(int b = 0; b < sets[i].count / sets[i].batch; ++b) steps.emplace_back(i, b);
        }
        const int nsteps = (int)steps.size();
        smoother_reserve(S, maxpts, true);
        // per-sample loss normalisation 1/(e.e) or 1/(e.Ae)
        std::vector<float*> norms(nsets, nullptr);
        struct Free
        {
            std::vector<float*>& v;
            ~Free()
            {
                for(float* p : v) dfree(p);
            }
        } free_norms{norms};
        for(int i = 0; i < nsets; ++i)
        {
            norms[i] = dalloc<float>(sets[i].count);
            check(hb::launch_sample_norm(hb::ConvGrid{sets[i].count, sets[i].nz, sets[i].ny, sets[i].nx}, sets[i].e,
                                         kind, norms[i], s));
        }
        Rng rng{seed};
        for(int ep = 0; ep < epochs; ++ep)
        {
            const double t = epochs > 1 ? (double)ep / (epochs - 1) : 0.0;
            const float lr = (float)(lr0 * std::pow((double)lr1 / lr0, t));
            for(int i = nsteps - 1; i > 0; --i)
                std::swap(steps[i], steps[(size_t)(rng.next() % (unsigned long long)(i + 1))]);
            HB_HOST_CUDA(cudaMemsetAsync(S.loss_acc, 0, sizeof(double), s));
            for(const auto& st : steps)
            {
                const hpcgb200_pair_set& P = sets[st.first];
                const long per = (long)P.nz * P.ny * P.nx;
                const long off = (long)st.second * P.batch;
                const hb::ConvGrid g{P.batch, P.nz, P.ny, P.nx};
                HB_RETURN_IF(smoother_loss_grad(S, g, P.r + off * per, P.e + off * per, norms[st.first] + off,
                                                1.f / (float)P.batch, kind, s));
                HB_RETURN_IF(smoother_adam(S, lr, 0.9f, 0.999f, 1e-8f, s));
            }
            double l = 0.0;
            HB_HOST_CUDA(cudaMemcpyAsync(&l, S.loss_acc, sizeof(double), cudaMemcpyDeviceToHost, s));
            HB_RETURN_IF(smoother_status(S, s));
            if(epoch_loss) epoch_loss[ep] = l / nsteps;
        }
        return 0;
    });
}

extern "C" int hpcgb200_make_training_pairs(int fine_n, int level, unsigned long long first_seed, int count,
                                            float* r_out, float* e_out, float* inv_ee_out, double tol)
{
    if(fine_n < 8 || level < 1 || level > 3 || count <= 0 || !r_out || !e_out || !inv_ee_out || !(tol > 0.0))
        return hb::record_error(HPCGB200_ERR_ARG, "bad arguments");
    if(fine_n % 8 || (fine_n >> level) < 4)
        return hb::record_error(HPCGB200_ERR_ARG, "fine_n must be a multiple of 8 with fine_n >> level >= 4");
    hpcgb200_problem* P = nullptr;
    hpcgb200_problem* Q = nullptr;
    int rc = hpcgb200_problem_create(fine_n, fine_n, fine_n, 4, &P);
    if(rc) return rc;
    const int nc = fine_n >> level;
    int qlev = 1;
    while(qlev < 4 && nc % (1 << qlev) == 0 && (nc >> qlev) >= 2) ++qlev;
    rc = hpcgb200_problem_create(nc, nc, nc, qlev, &Q);
    if(rc)
    {
        hpcgb200_problem_destroy(P);
        return rc;
    }
    rc = guarded([&] {
        cudaStream_t s = rt().stream;
        for(int l = 0; l <= level; ++l)
            if(!opt(*P->levels[l])->stencil_ok)
                return hb::record_error(HPCGB200_ERR_NOT_STENCIL, "training pairs need stencil levels");
        if(!opt(Q->A)->stencil_ok) return hb::record_error(HPCGB200_ERR_NOT_STENCIL, "training pairs need stencil levels");
        const LevelOpt* o0 = opt(P->A);
        const LevelOpt* ol = opt(*P->levels[level]);
        const LevelOpt* oq = opt(Q->A);
        const long per = (long)nc * nc * nc;
        const int m0 = P->A.localNumberOfRows;
        for(int i = 0; i < count; ++i)
        {
            float* rn = r_out + (size_t)i * per;
            float* en = e_out + (size_t)i * per;
            // b ~ N(0,1) (seed first_seed + i), FP32, coloured order of the fine grid
            check(hb::launch_normal_rhs(m0, first_seed + (unsigned long long)i, P->A.perm, nullptr, o0->r32, s));
            // the plain FP32 V-cycle's descending leg down to `level`
            const float* r = o0->r32;
            float* x = o0->z32;
            for(int l = 0; l < level; ++l)
            {
                const SparseMatrix& M = *P->levels[l];
                const LevelOpt* o = opt(M);
                const MGOpt* mo = mgopt(M);
                check(hb::launch32_symgs_zero(o->st, o->diag32, o->inv_diag32, nullptr, const_cast<float*>(r), x, s));
                check(hb::launch32_restrict(o->st, M.Ac->localNumberOfRows, mo->inj_f, mo->inj_c, o->diag32, r, x,
                                            mo->rc32, s));
                r = mo->rc32;
                x = mo->xc32;
            }
            check(hb::launch_natural_from_perm(ol->pm, nc, nc, nc, r, rn, s));
            // e = A^-1 r on a grid of the level's size (FP64 MG-PCG)
            check(hb::launch_perm_from_natural(oq->pm, nc, nc, nc, rn, Q->b.d_values, s));
            HB_HOST_CUDA(cudaMemsetAsync(Q->x.d_values, 0, sizeof(double) * per, s));
            int it = 0;
            double nr = 0.0, nr0 = 0.0;
            check(run_cg(Q->A, Q->data, Q->b, Q->x, 500, tol, it, nr, nr0, true, MGPrecision::FP64, false, nullptr,
                         nullptr));
            if(!(nr <= tol * nr0 * 1.0000001))
                return hb::record_error(HPCGB200_ERR_DEVICE_STATUS, "training pair %d: level solve did not converge", i);
            check(hb::launch_natural_from_perm(oq->pm, nc, nc, nc, Q->x.d_values, en, s));
            check(hb::launch_inv_sumsq(per, en, inv_ee_out + i, s));
        }
        HB_HOST_CUDA(cudaStreamSynchronize(s));
        return 0;
    });
    hpcgb200_problem_destroy(Q);
    hpcgb200_problem_destroy(P);
    return rc;
}

extern "C" int hpcgb200_problem_set_smoother(hpcgb200_problem* p, hpcgb200_smoother* h, int first_level,
                                             int coarse_steps)
{
    if(!p) return hb::record_error(HPCGB200_ERR_ARG, "bad arguments");
    if(h && (first_level < 1 || first_level >= p->nlevels))
        return hb::record_error(HPCGB200_ERR_ARG, "first_level must be in 1..nlevels-1");
    if(h && (coarse_steps < 1 || coarse_steps > 64))
        return hb::record_error(HPCGB200_ERR_ARG, "coarse_steps must be in 1..64");
    return guarded([&] {
        LevelOpt* o = opt(p->A);
        if(!h)
        {
            o->smoother = nullptr;
            return 0;
        }
        for(int l = first_level; l < p->nlevels; ++l)
            if(!opt(*p->levels[l])->stencil_ok)
                return hb::record_error(HPCGB200_ERR_NOT_STENCIL, "level %d is not a stencil level", l);
        smoother_reserve(h->S, p->levels[first_level]->localNumberOfRows, false);
        // learned solve graphs captured the previous attachment
        for(auto it = o->graphs.begin(); it != o->graphs.end();)
        {
            if((*it)->mode == (int)MGPrecision::LEARNED)
            {
                if((*it)->exec) cudaGraphExecDestroy((*it)->exec);
                if((*it)->graph) cudaGraphDestroy((*it)->graph);
                it = o->graphs.erase(it);
            }
            else
                ++it;
        }
        o->smoother = &h->S;
        o->smoother_first_level = first_level;
        o->smoother_coarse_steps = coarse_steps;
        return 0;
    });
}

extern "C" int hpcgb200_problem_set_fallback(hpcgb200_problem* p, double jump, int stall, int window, double rate)
{
    if(!p || !opt(p->A)) return hb::record_error(HPCGB200_ERR_ARG, "null problem");
    if(!(jump >= 1.0) || stall < 1 || window < 1 || window > 1000 || !(rate >= 0.0))
        return hb::record_error(HPCGB200_ERR_ARG, "fallback rule: need jump >= 1, stall >= 1, 1 <= window <= 1000, "
                                                  "rate >= 0");
    LevelOpt* o = opt(p->A);
    o->fb_jump = jump;
    o->fb_stall = stall;
    o->fb_window = window;
    o->fb_rate = rate;
    return 0;
}

extern "C" int hpcgb200_problem_last_fallback(const hpcgb200_problem* p, int* fallback_iter)
{
    if(!p || !fallback_iter) return hb::record_error(HPCGB200_ERR_ARG, "bad arguments");
    *fallback_iter = opt(p->A) ? opt(p->A)->last_fallback_iter : 0;
    return 0;
}
