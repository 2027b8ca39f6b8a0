/*
 * CPU restatement of the learned smoother's conv net (test infrastructure
 * only; see conv.c).  No reference counterpart.
 */
#ifndef HPCG_ORACLE_CONV_H
#define HPCG_ORACLE_CONV_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* fp32 -> bf16 (round to nearest even) -> fp32 */
float oc_bf16(float f);
/* out[p][co] = sum_tap sum_ci in[p + tap][ci] * w[tap][ci][co], zero padding,
 * inputs and weights rounded to bf16 when round != 0, fp32 accumulation. */
void oc_conv16(int nz, int ny, int nx, const float* in, const float* w, float* out, int round);
/* mirrored taps, swapped channels: conv(g, W') is the transposed convolution */
void oc_flip_transpose(const float* w, float* wt);
/* dw[tap][ci][co] = sum_p x[p + tap][ci] * g[p][co] */
void oc_conv16_wgrad(int nz, int ny, int nx, const float* x, const float* g, float* dw, int round);
/* y = conv3(relu(conv2(relu(conv1(r))))); a1, a2 = stored hidden activations */
void oc_net_forward(int nz, int ny, int nx, const float* w1, const float* w2, const float* w3, const float* r, float* y,
                    float* a1, float* a2, int round);
/* loss = ||y - e||^2 / ||e||^2 and its weight gradients */
double oc_net_loss_grad(int nz, int ny, int nx, const float* w1, const float* w2, const float* w3, const float* r,
                        const float* e, float* dw1, float* dw2, float* dw3, int round);
/* Same with options: odd != 0 evaluates y = (N(r) - N(-r)) / 2; kind 1 uses
 * the energy norm of the 27-point stencil A: loss = (y-e).A(y-e) / e.Ae. */
double oc_net_loss_grad2(int nz, int ny, int nx, const float* w1, const float* w2, const float* w3, const float* r,
                         const float* e, float* dw1, float* dw2, float* dw3, int round, int odd, int kind);
/* out = A v for the 27-point stencil (diagonal 26, off-diagonals -1). */
void oc_stencil_apply(int nz, int ny, int nx, const float* v, float* out);

#ifdef __cplusplus
}
#endif
#endif
