/*
 * CPU restatement of the learned smoother (3-layer 3x3x3 conv net) -- TEST
 * INFRASTRUCTURE ONLY: the checker for the tcgen05 forward / backward kernels
 * in rochpcg_b200/csrc/learned.cu.  No reference counterpart (the learned
 * smoother is new in this build).
 *
 * Tensors are channel-last on an nz x ny x nx grid: t[((z*ny + y)*nx + x)*C + c].
 * Every layer is computed as 16 -> 16 channels (layer 1 has 1 real input
 * channel, layer 3 one real output channel; the rest are zero weights), zero
 * padding outside the grid.  Weights: w[((tap*16 + ci)*16 + co)], tap =
 * (dz+1)*9 + (dy+1)*3 + (dx+1).
 *
 * Rounding points (bf16 = round-to-nearest-even of fp32) mirror the device:
 * layer inputs and weights are bf16, accumulation fp32, hidden activations
 * stored as bf16(relu(.)), the output fp32.  With round = 0 everything stays
 * fp32 (used for finite-difference gradient checks).
 */
#include "conv.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define CH 16

float oc_bf16(float f)
{
    union
    {
        float f;
        uint32_t u;
    } v = {f};
    if((v.u & 0x7f800000u) == 0x7f800000u) return f; /* inf / nan */
    v.u += 0x7fffu + ((v.u >> 16) & 1u);
    v.u &= 0xffff0000u;
    return v.f;
}

static inline float rnd(float f, int round) { return round ? oc_bf16(f) : f; }

void oc_conv16(int nz, int ny, int nx, const float* in, const float* w, float* out, int round)
{
    const long n = (long)nz * ny * nx;
    float* wr = (float*)malloc(sizeof(float) * 27 * CH * CH);
    for(int i = 0; i < 27 * CH * CH; ++i) wr[i] = rnd(w[i], round);
    float* ir = (float*)malloc(sizeof(float) * (size_t)n * CH);
    for(long i = 0; i < n * CH; ++i) ir[i] = rnd(in[i], round);
#pragma omp parallel for schedule(static)
    for(long p = 0; p < n; ++p)
    {
        const int z = (int)(p / ((long)ny * nx)), y = (int)((p / nx) % ny), x = (int)(p % nx);
        float acc[CH] = {0};
        for(int t = 0; t < 27; ++t)
        {
            const int zz = z + t / 9 - 1, yy = y + (t / 3) % 3 - 1, xx = x + t % 3 - 1;
            if(zz < 0 || zz >= nz || yy < 0 || yy >= ny || xx < 0 || xx >= nx) continue;
            const float* a = ir + (((long)zz * ny + yy) * nx + xx) * CH;
            const float* wt = wr + (size_t)t * CH * CH;
            for(int ci = 0; ci < CH; ++ci)
                for(int co = 0; co < CH; ++co) acc[co] += a[ci] * wt[ci * CH + co];
        }
        for(int co = 0; co < CH; ++co) out[p * CH + co] = acc[co];
    }
    free(wr);
    free(ir);
}

/* W'[t'][co][ci] = W[t][ci][co] with t' the mirrored tap: conv(g, W') is the
 * transposed convolution (the input gradient of conv(., W)). */
void oc_flip_transpose(const float* w, float* wt)
{
    for(int t = 0; t < 27; ++t)
        for(int ci = 0; ci < CH; ++ci)
            for(int co = 0; co < CH; ++co) wt[((26 - t) * CH + co) * CH + ci] = w[(t * CH + ci) * CH + co];
}

void oc_conv16_wgrad(int nz, int ny, int nx, const float* x, const float* g, float* dw, int round)
{
    const long n = (long)nz * ny * nx;
    memset(dw, 0, sizeof(float) * 27 * CH * CH);
#pragma omp parallel
    {
        float loc[27 * CH * CH];
        memset(loc, 0, sizeof(loc));
#pragma omp for schedule(static)
        for(long p = 0; p < n; ++p)
        {
            const int z = (int)(p / ((long)ny * nx)), y = (int)((p / nx) % ny), xx0 = (int)(p % nx);
            for(int t = 0; t < 27; ++t)
            {
                const int zz = z + t / 9 - 1, yy = y + (t / 3) % 3 - 1, xx = xx0 + t % 3 - 1;
                if(zz < 0 || zz >= nz || yy < 0 || yy >= ny || xx < 0 || xx >= nx) continue;
                const float* a = x + (((long)zz * ny + yy) * nx + xx) * CH;
                for(int ci = 0; ci < CH; ++ci)
                {
                    const float av = rnd(a[ci], round);
                    for(int co = 0; co < CH; ++co) loc[(t * CH + ci) * CH + co] += av * rnd(g[p * CH + co], round);
                }
            }
        }
#pragma omp critical
        for(int i = 0; i < 27 * CH * CH; ++i) dw[i] += loc[i];
    }
}

void oc_net_forward(int nz, int ny, int nx, const float* w1, const float* w2, const float* w3, const float* r, float* y,
                    float* a1, float* a2, int round)
{
    const long n = (long)nz * ny * nx;
    float* a0 = (float*)calloc((size_t)n * CH, sizeof(float));
    float* p = (float*)malloc(sizeof(float) * (size_t)n * CH);
    for(long i = 0; i < n; ++i) a0[i * CH] = r[i];
    oc_conv16(nz, ny, nx, a0, w1, p, round);
    for(long i = 0; i < n * CH; ++i) a1[i] = rnd(p[i] > 0.f ? p[i] : 0.f, round);
    oc_conv16(nz, ny, nx, a1, w2, p, round);
    for(long i = 0; i < n * CH; ++i) a2[i] = rnd(p[i] > 0.f ? p[i] : 0.f, round);
    oc_conv16(nz, ny, nx, a2, w3, p, round);
    for(long i = 0; i < n; ++i) y[i] = p[i * CH];
    free(a0);
    free(p);
}

/* Backward of one network evaluation (input r, stored activations a1, a2)
 * for the output gradient g (scalar field): adds the weight gradients. */
static void branch_backward(int nz, int ny, int nx, const float* w2, const float* w3, const float* r,
                            const float* a1, const float* a2, const float* gs, float* dw1, float* dw2, float* dw3,
                            int round)
{
    const long n = (long)nz * ny * nx;
    float* g = (float*)calloc((size_t)n * CH, sizeof(float));
    float* wt = (float*)malloc(sizeof(float) * 27 * CH * CH);
    float* d = (float*)malloc(sizeof(float) * (size_t)n * CH);
    float* d1 = (float*)malloc(sizeof(float) * (size_t)n * CH);
    float* a0 = (float*)calloc((size_t)n * CH, sizeof(float));
    float* dw = (float*)malloc(sizeof(float) * 27 * CH * CH);
    for(long i = 0; i < n; ++i)
    {
        g[i * CH] = gs[i];
        a0[i * CH] = r[i];
    }
    oc_conv16_wgrad(nz, ny, nx, a2, g, dw, round);
    for(int i = 0; i < 27 * CH * CH; ++i) dw3[i] += dw[i];
    oc_flip_transpose(w3, wt);
    oc_conv16(nz, ny, nx, g, wt, d, round); /* dL/da2 */
    for(long i = 0; i < n * CH; ++i) d[i] = a2[i] > 0.f ? d[i] : 0.f;
    oc_conv16_wgrad(nz, ny, nx, a1, d, dw, round);
    for(int i = 0; i < 27 * CH * CH; ++i) dw2[i] += dw[i];
    oc_flip_transpose(w2, wt);
    oc_conv16(nz, ny, nx, d, wt, d1, round); /* dL/da1 */
    for(long i = 0; i < n * CH; ++i) d1[i] = a1[i] > 0.f ? d1[i] : 0.f;
    oc_conv16_wgrad(nz, ny, nx, a0, d1, dw, round);
    for(int i = 0; i < 27 * CH * CH; ++i) dw1[i] += dw[i];
    free(g);
    free(wt);
    free(d);
    free(d1);
    free(a0);
    free(dw);
}

/* 27-point stencil A (diagonal 26, off-diagonals -1, zero outside the grid). */
void oc_stencil_apply(int nz, int ny, int nx, const float* v, float* out)
{
    for(int z = 0; z < nz; ++z)
        for(int y = 0; y < ny; ++y)
            for(int x = 0; x < nx; ++x)
            {
                const long p = ((long)z * ny + y) * nx + x;
                float off = 0.f;
                for(int t = 0; t < 27; ++t)
                {
                    const int z2 = z + t / 9 - 1, y2 = y + (t / 3) % 3 - 1, x2 = x + t % 3 - 1;
                    if(t != 13 && z2 >= 0 && z2 < nz && y2 >= 0 && y2 < ny && x2 >= 0 && x2 < nx)
                        off += v[((long)z2 * ny + y2) * nx + x2];
                }
                out[p] = 26.f * v[p] - off;
            }
}

double oc_net_loss_grad2(int nz, int ny, int nx, const float* w1, const float* w2, const float* w3, const float* r,
                         const float* e, float* dw1, float* dw2, float* dw3, int round, int odd, int kind)
{
    const long n = (long)nz * ny * nx;
    float* yp = (float*)malloc(sizeof(float) * (size_t)n);
    float* ym = (float*)malloc(sizeof(float) * (size_t)n);
    float* rm = (float*)malloc(sizeof(float) * (size_t)n);
    float* a1p = (float*)malloc(sizeof(float) * (size_t)n * CH);
    float* a2p = (float*)malloc(sizeof(float) * (size_t)n * CH);
    float* a1m = (float*)malloc(sizeof(float) * (size_t)n * CH);
    float* a2m = (float*)malloc(sizeof(float) * (size_t)n * CH);
    float* d = (float*)malloc(sizeof(float) * (size_t)n);
    float* md = (float*)malloc(sizeof(float) * (size_t)n);
    float* me = (float*)malloc(sizeof(float) * (size_t)n);
    float* gs = (float*)malloc(sizeof(float) * (size_t)n);
    oc_net_forward(nz, ny, nx, w1, w2, w3, r, yp, a1p, a2p, round);
    if(odd)
    {
        for(long i = 0; i < n; ++i) rm[i] = -r[i];
        oc_net_forward(nz, ny, nx, w1, w2, w3, rm, ym, a1m, a2m, round);
    }
    for(long i = 0; i < n; ++i) d[i] = (odd ? 0.5f * (yp[i] - ym[i]) : yp[i]) - e[i];
    if(kind)
    {
        oc_stencil_apply(nz, ny, nx, d, md);
        oc_stencil_apply(nz, ny, nx, e, me);
    }
    else
    {
        memcpy(md, d, sizeof(float) * (size_t)n);
        memcpy(me, e, sizeof(float) * (size_t)n);
    }
    double num = 0.0, den = 0.0;
    for(long i = 0; i < n; ++i)
    {
        num += (double)d[i] * md[i];
        den += (double)e[i] * me[i];
    }
    memset(dw1, 0, sizeof(float) * 27 * CH * CH);
    memset(dw2, 0, sizeof(float) * 27 * CH * CH);
    memset(dw3, 0, sizeof(float) * 27 * CH * CH);
    /* dL/dy = 2 M d / den, split +/- half over the two branches when odd */
    for(long i = 0; i < n; ++i) gs[i] = (float)((odd ? 1.0 : 2.0) * md[i] / den);
    branch_backward(nz, ny, nx, w2, w3, r, a1p, a2p, gs, dw1, dw2, dw3, round);
    if(odd)
    {
        for(long i = 0; i < n; ++i) gs[i] = -gs[i];
        branch_backward(nz, ny, nx, w2, w3, rm, a1m, a2m, gs, dw1, dw2, dw3, round);
    }
    free(yp);
    free(ym);
    free(rm);
    free(a1p);
    free(a2p);
    free(a1m);
    free(a2m);
    free(d);
    free(md);
    free(me);
    free(gs);
    return num / den;
}

double oc_net_loss_grad(int nz, int ny, int nx, const float* w1, const float* w2, const float* w3, const float* r,
                        const float* e, float* dw1, float* dw2, float* dw3, int round)
{
    return oc_net_loss_grad2(nz, ny, nx, w1, w2, w3, r, e, dw1, dw2, dw3, round, 0, 0);
}
