// Learned smoother kernels: a 3-layer 3x3x3 convolutional network (1 -> 16
// -> 16 -> 1 channels, ReLU, no bias, BF16 weights and activations, FP32
// accumulation) as implicit GEMMs on the tcgen05 tensor cores, with its
// training kernels (input and weight gradients, loss, Adam).
#pragma once

#include "common.cuh"
#include "mixed.cuh"

namespace hb {

constexpr int kNetCh = 16;                     // channels of every layer tensor
constexpr int kNetLayerWeights = 27 * 16 * 16; // w[tap][ci][co], tap = (dz+1)*9 + (dy+1)*3 + (dx+1)
constexpr int kNetWeightTileBytes = 27 * 16 * 16 * 2;  // one layer's BF16 B operands

// Epilogues of the forward convolution.
enum ConvOut : int
{
    kOutReluBf16 = 0,  // out = bf16(relu(v)), 16 channels (hidden layers)
    kOutMaskBf16 = 1,  // out = bf16(act > 0 ? v : 0), 16 channels (ReLU backward)
    kOutF32 = 2,       // out = v, FP32 16 channels
    kOutF32C0 = 3,     // out = v[0], FP32 scalar field
    kOutPermSet = 4,   // x[row(p)] = v[0] on a stencil level's colour-permuted vector
    kOutPermAdd = 5,   // x[row(p)] += v[0]
};

// Natural grid point -> colour-permuted row of a parity-coloured level.
struct PermMap
{
    int offsets[9];
    int bx[8], by[8];
    int color_of_par[8];
};
PermMap make_perm_map(const StencilLevel& L);

// nb samples of nz x ny x nx points, channel-last, samples back to back.
struct ConvGrid
{
    int nb, nz, ny, nx;
    __host__ __device__ long points() const { return (long)nb * nz * ny * nx; }
};

// FP32 weights -> BF16 tensor-core operand tiles (flip != 0: the mirrored-tap,
// swapped-channel weights of the transposed convolution).
int launch_prepare_weights(const float* w, void* wB, int flip, cudaStream_t s);

// out = conv(in, W) with the epilogue `out_mode`; `act` is the activation
// tensor of kOutMaskBf16, `pm` the row map of the permuted modes (nb == 1).
int launch_conv16(const ConvGrid& g, const void* in, const void* wB, int out_mode, void* out, const void* act,
                  const PermMap* pm, int* status, cudaStream_t s);

// Evaluation-only kernels: the scalar input field of a level, and the
// tensor-core forms of the layers with one channel on one side (layer 1: one
// input channel, layer 3: one output channel).
// s1 = bf16 scalar field of a level (r, or r - A x when x is not null).
int launch_embed_scalar_level(const PermMap& pm, int nz, int ny, int nx, const float* r, const float* x,
                              const float* diag32, void* s1, cudaStream_t s);
// a1 = bf16(relu(conv(in, W1))) from a scalar field in (FP32 when in_f32, else
// BF16), 16 channels; pair: also the branch of -in at a1 + 16 * points.  The
// 27 taps are the K dimension (im2col rows built in shared memory), the 16
// channels N; `status` receives the code of a wait that gave up.
int launch_layer1_tc(const ConvGrid& g, const void* in, int in_f32, const float* w1, void* a1, int pair, int* status,
                     cudaStream_t s);
// Channel 0 of conv(a2, W3), odd-combined when pair ((y(a2) - y(a2 + 16 n)) / 2);
// mode 0: set, 1: add into a level vector through pm (g.nb == 1); 2: natural out.
// The 27 taps are stacked in N (one MMA row per staged input point gives its
// contribution to each neighbour), the pair is folded into K, and the 27-tap
// gather runs in the epilogue; `status` receives the code of a wait that gave up.
int launch_layer3_tc(const ConvGrid& g, const PermMap* pm, const void* a2, const float* w3, int pair, int mode,
                     float* out, int* status, cudaStream_t s);

// dw[tap][ci][co] = sum_p x[p + tap][ci] * gr[p][co] (partial: one block of
// conv16_wgrad_parts(points) x 27*256 floats).
int conv16_wgrad_parts(long points);
int launch_conv16_wgrad(const ConvGrid& g, const void* x, const void* gr, float* partial, float* dw, int* status,
                        cudaStream_t s);

// BF16 16-channel tensor whose channel 0 is a scalar field (others zero):
// from colour-permuted FP32 level vectors (r, or the residual r - A x when x
// is not null), or from an FP32 natural field.
// pair != 0 also writes the negated field as a second sample right after the
// first (the odd evaluation N(v) - N(-v) as one batch of two).
int launch_embed_level(const PermMap& pm, int nz, int ny, int nx, const float* r, const float* x,
                       const float* diag32, void* a, int pair, cudaStream_t s);
int launch_embed_f32(long n, const float* r, void* a, int pair, cudaStream_t s);
// x[row(p)] = (or +=) (y[p] - y[p + n]) / 2.
int launch_odd_combine(const PermMap& pm, int nz, int ny, int nx, const float* y, float* x, bool add, cudaStream_t s);
// out[p] = (y[p] - y[p + n]) / 2.
int launch_odd_natural(long n, const float* y, float* out, cudaStream_t s);
// out[b] = 1 / (e_b . e_b) (kind 0) or 1 / (e_b . A e_b) (kind 1, 27-point stencil).
int launch_sample_norm(const ConvGrid& g, const float* e, int kind, float* out, cudaStream_t s);

// Natural <-> colour-permuted copies of level vectors.
int launch_natural_from_perm(const PermMap& pm, int nz, int ny, int nx, const float* in, float* out, cudaStream_t s);
int launch_natural_from_perm(const PermMap& pm, int nz, int ny, int nx, const double* in, float* out, cudaStream_t s);
int launch_perm_from_natural(const PermMap& pm, int nz, int ny, int nx, const float* in, double* out, cudaStream_t s);
// *out = 1 / sum e^2.
int launch_inv_sumsq(long n, const float* e, float* out, cudaStream_t s);
// *acc += sum of the loss partials of launch_loss_grad.
int launch_loss_accumulate(const float* partial, double* acc, cudaStream_t s);
// N(0,1) right-hand side by natural row id (the generator of rochpcg_b200/rhs.py),
// stored at out[perm[i]] (perm may be null) as double and/or float.
int launch_normal_rhs(long long m, unsigned long long seed, const int* perm, double* out64, float* out32,
                      cudaStream_t s);

// Loss of a batch: sum_b d_b.M d_b * wnorm[b] * scale with d = y - e (y the
// odd part (y[p] - y[p+n])/2 when odd), M = I (kind 0) or the stencil A
// (kind 1), as per-block partial sums (`loss_partial`, loss_parts(points)
// floats), and its gradient 2 M d wnorm scale as BF16 channel 0 of G (odd:
// +/- half for the two branches).  d: scratch of g.points() floats.
int loss_parts(long points);
int launch_loss_grad(const ConvGrid& g, const float* y, const float* e, float* d, const float* wnorm, float scale,
                     int kind, int odd, void* G, float* loss_partial, cudaStream_t s);

// Projects the weights (3 layers back to back) onto the tied odd form
// (hidden channel k+8 = the negated twin of channel k): the network is then
// an odd function of its input with a single evaluation.
int launch_tie_odd(float* w, cudaStream_t s);

// One Adam step on n parameters (bias-corrected, step t >= 1).
int launch_adam(int n, float* w, const float* dw, float* m, float* v, float lr, float beta1, float beta2, float eps,
                int t, cudaStream_t s);

}  // namespace hb
