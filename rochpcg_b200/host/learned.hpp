// Learned smoother: device state of the conv net and its use on MG levels.
// No reference counterpart.
#pragma once

#include "internal.hpp"

namespace hpcg_b200 {

constexpr int kNetWeights = 3 * hb::kNetLayerWeights;  // layers 1..3 back to back, w[tap][ci][co]

struct Smoother
{
    float* w = nullptr;            // FP32 master weights (device)
    unsigned char* wB = nullptr;   // 3 forward BF16 operand tile sets
    unsigned char* wT = nullptr;   // 3 transposed-convolution tile sets
    bool tiles_stale = true;
    bool odd = false;              // evaluate (N(r) - N(-r)) / 2 (two branches as one batch)
    bool tied = false;             // keep the weights in the tied odd form (one evaluation is odd)

    long cap = 0;                  // grid points the buffers hold (both branches when odd)
    long long epoch = 0;           // bumped when the activation buffers move
    void* a0 = nullptr;            // BF16 x16: layer inputs / activations
    void* a1 = nullptr;
    void* a2 = nullptr;
    void* g = nullptr;             // BF16 x16: output gradient, then dL/da1
    void* d = nullptr;             // BF16 x16: dL/da2
    float* y = nullptr;            // raw network output (both branches when odd)
    float* dbuf = nullptr;         // loss scratch (training)

    float* dw = nullptr;           // gradients (kNetWeights)
    float* adam_m = nullptr;
    float* adam_v = nullptr;
    int adam_t = 0;
    float* partial = nullptr;      // weight-gradient partial sums
    size_t partial_floats = 0;
    float* loss_partial = nullptr;
    double* loss_acc = nullptr;    // running loss sum (device)
    int* status = nullptr;         // tensor-core wait status (device)

    Smoother();
    ~Smoother();
    Smoother(const Smoother&) = delete;
    Smoother& operator=(const Smoother&) = delete;
};

// Buffers for `points` grid points (training adds the gradient buffers).
void smoother_reserve(Smoother& S, long points, bool training);
void smoother_set_weights(Smoother& S, const float* host_w, cudaStream_t s);
// Operand tiles from the master weights when they changed.
int smoother_prepare(Smoother& S, cudaStream_t s);
// Buffers and tiles of the smoother attached to hierarchy A, before a solve
// or an eager V-cycle (never during graph capture).
int smoother_ready(const SparseMatrix& A, cudaStream_t s);
// x = N(r) (residual == false) or x += N(r - A x) on one stencil level
// (colour-permuted FP32 vectors); the tiles must be prepared.
int smoother_level_apply(Smoother& S, const LevelOpt& o, const float* r, float* x, bool residual, cudaStream_t s);
// y = N(r) on natural-order fields of a batch.
int smoother_forward(Smoother& S, const hb::ConvGrid& g, const float* r, float* y, cudaStream_t s);
// Loss scale * sum_b (y_b - e_b).M(y_b - e_b) wnorm[b] (M = I for kind 0,
// the stencil A for kind 1) added to *loss_acc and its weight gradients into S.dw.
int smoother_loss_grad(Smoother& S, const hb::ConvGrid& g, const float* r, const float* e, const float* wnorm,
                       float scale, int kind, cudaStream_t s);
// Symmetry of the network: 0 plain, 1 two-branch odd evaluation, 2 tied
// odd weights (buffers are re-reserved on next use).
void smoother_configure(Smoother& S, int symmetry, cudaStream_t s);
int smoother_adam(Smoother& S, float lr, float beta1, float beta2, float eps, cudaStream_t s);
// Reads and clears the device status word; nonzero: a tensor-core wait timed out.
int smoother_status(Smoother& S, cudaStream_t s);

}  // namespace hpcg_b200
