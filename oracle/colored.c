/*
 * CPU restatement of rocHPCG's optimized (multicolored) MG-PCG path.
 * TEST INFRASTRUCTURE ONLY -- see colored.h.  Compiled with
 * -ffp-contract=off so that only the explicit fma()/fmaf() calls fuse,
 * exactly like the reference kernels (and our CUDA kernels) do.
 */
#include "colored.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define OC_RNG_SEED 0x586744 /* src/utils.hpp:47 */
#define OC_WIDTH 27

/* ------------------------------------------------------------------ setup */

/* GenerateProblem.cpp:93-96 (get_hash) and :293-296 (row hash). */
static int oc_row_hash(int ix, int iy, int iz, int nx, int ny, int nz)
{
    int h = ((ix & 1) << 2) | ((iy & 1) << 1) | (iz & 1);
    int crd = iz * nx * ny + iy * (nx << 1) + (ix << 2);
    return h * nx * ny * nz + crd;
}

void oc_generate(int nx, int ny, int nz, int* cols, double* vals, int8_t* nnz_in_row, int* diag_slot,
                 int* hash, double* b)
{
    const int m = nx * ny * nz;
#pragma omp parallel for schedule(static)
    for(int row = 0; row < m; ++row)
    {
        const int iz = row / (nx * ny);
        const int iy = row / nx - ny * iz;
        const int ix = row - iz * nx * ny - iy * nx;
        int n = 0;
        /* slot order t = 9*(dz+1) + 3*(dy+1) + (dx+1), GenerateProblem.cpp:165-167 */
        for(int t = 0; t < OC_WIDTH; ++t)
        {
            const int dz = t / 9 - 1, dy = (t % 9) / 3 - 1, dx = t % 3 - 1;
            const int z = iz + dz, y = iy + dy, x = ix + dx;
            if(z < 0 || z >= nz || y < 0 || y >= ny || x < 0 || x >= nx) continue;
            const int col = z * nx * ny + y * nx + x;
            cols[(size_t)row * OC_WIDTH + n] = col;
            vals[(size_t)row * OC_WIDTH + n] = (col == row) ? 26.0 : -1.0;
            if(col == row) diag_slot[row] = n;
            ++n;
        }
        for(int t = n; t < OC_WIDTH; ++t)
        {
            cols[(size_t)row * OC_WIDTH + t] = -1;
            vals[(size_t)row * OC_WIDTH + t] = 0.0;
        }
        nnz_in_row[row] = (int8_t)n;
        hash[row] = oc_row_hash(ix, iy, iz, nx, ny, nz);
        if(b) b[row] = 26.0 - (n - 1.0);
    }
}

void oc_f2c(int nxf, int nyf, int nzf, int* f2c)
{
    const int nxc = nxf / 2, nyc = nyf / 2, nzc = nzf / 2;
    for(int izc = 0; izc < nzc; ++izc)
        for(int iyc = 0; iyc < nyc; ++iyc)
            for(int ixc = 0; ixc < nxc; ++ixc)
                f2c[izc * nxc * nyc + iyc * nxc + ixc] = (izc << 1) * nxf * nyf + (iyc << 1) * nxf + (ixc << 1);
}

int oc_jpl_coloring(int m, const int* cols, const int8_t* nnz_in_row, const int* hash, int* colors,
                    int* round_colors, int* round_sizes)
{
    (void)nnz_in_row; /* pads are already -1 (kernel_copy_indices) */
    int* next = (int*)malloc(sizeof(int) * (size_t)m);
    for(int i = 0; i < m; ++i) colors[i] = -1;
    srand(OC_RNG_SEED);
    int nblocks = 0;
    long long colored = 0;
    int rounds = 0;
    while(colored != m)
    {
        if(rounds++ >= 64)
        {
            free(next);
            return -1;
        }
        const int c1 = (nblocks < 8) ? rand() % 8 : nblocks;
        const int c2 = (nblocks < 8) ? rand() % 8 : nblocks + 1;
        round_colors[nblocks] = c1;
        round_colors[nblocks + 1] = c2;
        /* kernel_jpl: a neighbour whose colour is -1, c1 or c2 counts as
         * uncoloured; that set is closed under this round's writes, so the
         * result equals a snapshot evaluation. */
#pragma omp parallel for schedule(static)
        for(int row = 0; row < m; ++row)
        {
            next[row] = colors[row];
            if(colors[row] != -1) continue;
            int is_max = 1, is_min = 1;
            const int rh = hash[row];
            for(int p = 0; p < OC_WIDTH; ++p)
            {
                const int col = cols[(size_t)row * OC_WIDTH + p];
                if(col < 0 || col >= m || col == row) continue;
                const int cn = colors[col];
                if(cn == -1 || cn == c1 || cn == c2)
                {
                    const int ch = hash[col];
                    if(ch >= rh) is_max = 0;
                    if(ch <= rh) is_min = 0;
                }
            }
            if(is_max) next[row] = c1;
            else if(is_min) next[row] = c2;
        }
        memcpy(colors, next, sizeof(int) * (size_t)m);
        /* kernel_count_color_part1/2 count the colour VALUE over all rows */
        int n1 = 0, n2 = 0;
        for(int i = 0; i < m; ++i)
        {
            n1 += colors[i] == c1;
            n2 += colors[i] == c2;
        }
        round_sizes[nblocks] = n1;
        round_sizes[nblocks + 1] = n2;
        colored += n1;
        colored += n2;
        nblocks += 2;
    }
    free(next);
    return nblocks;
}

void oc_color_perm(int m, const int* colors, int ncolors, int* perm, int* sizes, int* offsets)
{
    for(int c = 0; c < ncolors; ++c) sizes[c] = 0;
    for(int i = 0; i < m; ++i) sizes[colors[i]]++;
    offsets[0] = 0;
    for(int c = 0; c < ncolors; ++c) offsets[c + 1] = offsets[c] + sizes[c];
    int* cursor = (int*)malloc(sizeof(int) * (size_t)ncolors);
    memcpy(cursor, offsets, sizeof(int) * (size_t)ncolors);
    /* stable: rows of one colour keep their natural order */
    for(int i = 0; i < m; ++i) perm[i] = cursor[colors[i]]++;
    free(cursor);
}

void oc_build_ell(int m, const int* cols, const double* vals, const int* perm, int* ell_col, double* ell_val,
                  int* diag_idx, double* inv_diag)
{
#pragma omp parallel for schedule(static)
    for(int row = 0; row < m; ++row)
    {
        int key[OC_WIDTH];
        double val[OC_WIDTH];
        int n = 0;
        for(int p = 0; p < OC_WIDTH; ++p)
        {
            const int col = cols[(size_t)row * OC_WIDTH + p];
            if(col >= 0 && col < m)
            {
                key[n] = perm[col];
                val[n] = vals[(size_t)row * OC_WIDTH + p];
                ++n;
            }
        }
        /* keys are distinct, so any correct sort equals the bitonic network */
        for(int i = 1; i < n; ++i)
        {
            const int k = key[i];
            const double v = val[i];
            int j = i - 1;
            while(j >= 0 && key[j] > k)
            {
                key[j + 1] = key[j];
                val[j + 1] = val[j];
                --j;
            }
            key[j + 1] = k;
            val[j + 1] = v;
        }
        const size_t prow = (size_t)perm[row];
        for(int p = 0; p < OC_WIDTH; ++p)
        {
            ell_col[(size_t)p * m + prow] = p < n ? key[p] : -1;
            ell_val[(size_t)p * m + prow] = p < n ? val[p] : 0.0;
        }
    }
#pragma omp parallel for schedule(static)
    for(int row = 0; row < m; ++row)
    {
        for(int p = 0; p < OC_WIDTH; ++p)
        {
            if(ell_col[(size_t)p * m + row] == row)
            {
                diag_idx[row] = p;
                inv_diag[row] = 1.0 / ell_val[(size_t)p * m + row];
                break;
            }
        }
    }
}

void oc_permute_vector(int m, const int* perm, const double* in, double* out)
{
    for(int i = 0; i < m; ++i) out[perm[i]] = in[i];
}

/* ------------------------------------------------------------ FP64 kernels */

void oc_spmv(int m, const int* ell_col, const double* ell_val, const double* x, double* y)
{
#pragma omp parallel for schedule(static)
    for(int row = 0; row < m; ++row)
    {
        double sum = 0.0;
        for(int p = 0; p < OC_WIDTH; ++p)
        {
            const size_t idx = (size_t)p * m + row;
            const int col = ell_col[idx];
            if(col >= 0 && col < m) sum = fma(ell_val[idx], x[col], sum);
        }
        y[row] = sum;
    }
}

static void oc_sweep(int m, int size, int offset, const int* ell_col, const double* ell_val,
                     const double* inv_diag, const double* r, double* x)
{
#pragma omp parallel for schedule(static)
    for(int gid = 0; gid < size; ++gid)
    {
        const int row = gid + offset;
        double sum = r[row];
        for(int p = 0; p < OC_WIDTH; ++p)
        {
            const size_t idx = (size_t)p * m + row;
            const int col = ell_col[idx];
            if(col >= 0 && col < m && col != row) sum = fma(-ell_val[idx], x[col], sum);
        }
        x[row] = sum * inv_diag[row];
    }
}

void oc_symgs(int m, int nblocks, int ublocks, const int* sizes, const int* offsets, const int* ell_col,
              const double* ell_val, const double* inv_diag, const double* r, double* x)
{
    for(int i = 0; i < nblocks; ++i) oc_sweep(m, sizes[i], offsets[i], ell_col, ell_val, inv_diag, r, x);
    for(int i = ublocks; i >= 0; --i) oc_sweep(m, sizes[i], offsets[i], ell_col, ell_val, inv_diag, r, x);
}

void oc_symgs_zero(int m, int nblocks, int ublocks, const int* sizes, const int* offsets, const int* ell_col,
                   const double* ell_val, const int* diag_idx, const double* r, double* x)
{
    /* kernel_pointwise_mult on colour 0: x = r * inv_diag, with inv_diag = 1/a_ii */
    for(int row = 0; row < sizes[0]; ++row)
    {
        const double d = ell_val[(size_t)diag_idx[row] * m + row];
        x[row] = r[row] * (1.0 / d);
    }
    for(int i = 1; i < nblocks; ++i)
    {
        const int offset = offsets[i];
#pragma omp parallel for schedule(static)
        for(int gid = 0; gid < sizes[i]; ++gid)
        {
            const int row = gid + offset;
            const int diag = diag_idx[row];
            double sum = r[row];
            for(int p = 0; p < diag; ++p)
            {
                const size_t idx = (size_t)p * m + row;
                const int col = ell_col[idx];
                if(col >= 0 && col < offset) sum = fma(-ell_val[idx], x[col], sum);
            }
            sum *= 1.0 / ell_val[(size_t)diag * m + row];
            x[row] = sum;
        }
    }
    for(int i = ublocks; i >= 0; --i)
    {
        const int offset = offsets[i];
#pragma omp parallel for schedule(static)
        for(int gid = 0; gid < sizes[i]; ++gid)
        {
            const int row = gid + offset;
            const int diag = diag_idx[row];
            const double dv = ell_val[(size_t)diag * m + row];
            double sum = x[row] * dv;
            for(int p = diag + 1; p < OC_WIDTH; ++p)
            {
                const size_t idx = (size_t)p * m + row;
                const int col = ell_col[idx];
                if(col >= offset && col < m) sum = fma(-ell_val[idx], x[col], sum);
            }
            sum *= 1.0 / dv;
            x[row] = sum;
        }
    }
}

void oc_restrict_fused(int nc, const int* f2c, const int* perm_f, const int* perm_c, int mf, const int* ell_col,
                       const double* ell_val, const double* rf, const double* xf, double* rc)
{
#pragma omp parallel for schedule(static)
    for(int ic = 0; ic < nc; ++ic)
    {
        const int row = perm_f[f2c[ic]];
        double sum = rf[row];
        for(int p = 0; p < OC_WIDTH; ++p)
        {
            const size_t idx = (size_t)p * mf + row;
            const int col = ell_col[idx];
            if(col >= 0 && col < mf) sum = fma(-ell_val[idx], xf[col], sum);
        }
        rc[perm_c[ic]] = sum;
    }
}

void oc_prolong(int nc, const int* f2c, const int* perm_f, const int* perm_c, const double* xc, double* xf)
{
#pragma omp parallel for schedule(static)
    for(int ic = 0; ic < nc; ++ic) xf[perm_f[f2c[ic]]] += xc[perm_c[ic]];
}

double oc_dot(int n, const double* x, const double* y)
{
    const int B = 4096;
    const int nb = (n + B - 1) / B;
    double* part = (double*)malloc(sizeof(double) * (size_t)(nb > 0 ? nb : 1));
#pragma omp parallel for schedule(static)
    for(int k = 0; k < nb; ++k)
    {
        double s = 0.0;
        const int e = (k + 1) * B < n ? (k + 1) * B : n;
        for(int i = k * B; i < e; ++i) s = fma(x[i], y[i], s);
        part[k] = s;
    }
    double s = 0.0;
    for(int k = 0; k < nb; ++k) s += part[k];
    free(part);
    return s;
}

static void oc_mg_level(const oc_level* L, int l, int nlevels, const double* r, double* x)
{
    const oc_level* A = &L[l];
    oc_symgs_zero(A->m, A->nblocks, A->ublocks, A->sizes, A->offsets, A->ell_col, A->ell_val, A->diag_idx, r, x);
    if(l + 1 >= nlevels) return;
    oc_restrict_fused(A->nc, A->f2c, A->perm, A->perm_c, A->m, A->ell_col, A->ell_val, r, x, A->rc);
    oc_mg_level(L, l + 1, nlevels, A->rc, A->xc);
    oc_prolong(A->nc, A->f2c, A->perm, A->perm_c, A->xc, x);
    oc_symgs(A->m, A->nblocks, A->ublocks, A->sizes, A->offsets, A->ell_col, A->ell_val, A->inv_diag, r, x);
}

void oc_mg(const oc_level* levels, int nlevels, const double* r, double* x)
{
    oc_mg_level(levels, 0, nlevels, r, x);
}

int oc_cg(const oc_level* levels, int nlevels, const double* b, double* x, int max_iter, double tol,
          int precond, int* niters, double* normr_out, double* normr0_out, double* normr_hist)
{
    const int m = levels[0].m;
    double* r = (double*)malloc(sizeof(double) * (size_t)m);
    double* z = (double*)malloc(sizeof(double) * (size_t)m);
    double* p = (double*)malloc(sizeof(double) * (size_t)m);
    double* Ap = (double*)malloc(sizeof(double) * (size_t)m);
    memcpy(p, x, sizeof(double) * (size_t)m);
    oc_spmv(m, levels[0].ell_col, levels[0].ell_val, p, Ap);
    for(int i = 0; i < m; ++i) r[i] = fma(-1.0, Ap[i], b[i]); /* WAXPBY(1, b, -1, Ap) */
    double normr = sqrt(oc_dot(m, r, r));
    const double normr0 = normr;
    if(normr_hist) normr_hist[0] = normr;
    double rtz = 0.0, oldrtz = 0.0;
    int k;
    *niters = 0;
    for(k = 1; k <= max_iter && normr / normr0 > tol; ++k)
    {
        if(precond) oc_mg(levels, nlevels, r, z);
        else memcpy(z, r, sizeof(double) * (size_t)m);
        if(k == 1)
        {
            for(int i = 0; i < m; ++i) p[i] = fma(0.0, z[i], z[i]); /* WAXPBY(1, z, 0, z) */
            rtz = oc_dot(m, r, z);
        }
        else
        {
            oldrtz = rtz;
            rtz = oc_dot(m, r, z);
            const double beta = rtz / oldrtz;
            for(int i = 0; i < m; ++i) p[i] = fma(beta, p[i], z[i]); /* WAXPBY(1, z, beta, p) */
        }
        oc_spmv(m, levels[0].ell_col, levels[0].ell_val, p, Ap);
        const double pAp = oc_dot(m, p, Ap);
        const double alpha = rtz / pAp;
        for(int i = 0; i < m; ++i) r[i] = fma(-alpha, Ap[i], r[i]); /* fused WAXPBY+dot */
        normr = sqrt(oc_dot(m, r, r));
        for(int i = 0; i < m; ++i) x[i] = fma(alpha, p[i], x[i]); /* WAXPBY(1, x, alpha, p) */
        if(normr_hist) normr_hist[k] = normr;
        *niters = k;
    }
    *normr_out = normr;
    *normr0_out = normr0;
    free(r);
    free(z);
    free(p);
    free(Ap);
    return 0;
}

/* ------------------------------------------------------------ FP32 V-cycle */

static void oc_symgs_zero_f32(const oc_level* A, const float* r, float* x)
{
    const int m = A->m;
    for(int row = 0; row < A->sizes[0]; ++row)
    {
        const float d = (float)A->ell_val[(size_t)A->diag_idx[row] * m + row];
        x[row] = r[row] * (1.0f / d);
    }
    for(int i = 1; i < A->nblocks; ++i)
    {
        const int offset = A->offsets[i];
#pragma omp parallel for schedule(static)
        for(int gid = 0; gid < A->sizes[i]; ++gid)
        {
            const int row = gid + offset;
            const int diag = A->diag_idx[row];
            float sum = r[row];
            for(int p = 0; p < diag; ++p)
            {
                const size_t idx = (size_t)p * m + row;
                const int col = A->ell_col[idx];
                if(col >= 0 && col < offset) sum = fmaf(-(float)A->ell_val[idx], x[col], sum);
            }
            sum *= 1.0f / (float)A->ell_val[(size_t)diag * m + row];
            x[row] = sum;
        }
    }
    for(int i = A->ublocks; i >= 0; --i)
    {
        const int offset = A->offsets[i];
#pragma omp parallel for schedule(static)
        for(int gid = 0; gid < A->sizes[i]; ++gid)
        {
            const int row = gid + offset;
            const int diag = A->diag_idx[row];
            const float dv = (float)A->ell_val[(size_t)diag * m + row];
            float sum = x[row] * dv;
            for(int p = diag + 1; p < OC_WIDTH; ++p)
            {
                const size_t idx = (size_t)p * m + row;
                const int col = A->ell_col[idx];
                if(col >= offset && col < m) sum = fmaf(-(float)A->ell_val[idx], x[col], sum);
            }
            sum *= 1.0f / dv;
            x[row] = sum;
        }
    }
}

static void oc_sweep_f32(const oc_level* A, int size, int offset, const float* r, float* x)
{
    const int m = A->m;
#pragma omp parallel for schedule(static)
    for(int gid = 0; gid < size; ++gid)
    {
        const int row = gid + offset;
        float sum = r[row];
        for(int p = 0; p < OC_WIDTH; ++p)
        {
            const size_t idx = (size_t)p * m + row;
            const int col = A->ell_col[idx];
            if(col >= 0 && col < m && col != row) sum = fmaf(-(float)A->ell_val[idx], x[col], sum);
        }
        x[row] = sum * (1.0f / (float)A->ell_val[(size_t)A->diag_idx[row] * m + row]);
    }
}

static void oc_mg_level_f32(const oc_level* L, int l, int nlevels, const float* r, float* x, float** rc, float** xc)
{
    const oc_level* A = &L[l];
    oc_symgs_zero_f32(A, r, x);
    if(l + 1 >= nlevels) return;
    const int mf = A->m;
#pragma omp parallel for schedule(static)
    for(int ic = 0; ic < A->nc; ++ic)
    {
        const int row = A->perm[A->f2c[ic]];
        float sum = r[row];
        for(int p = 0; p < OC_WIDTH; ++p)
        {
            const size_t idx = (size_t)p * mf + row;
            const int col = A->ell_col[idx];
            if(col >= 0 && col < mf) sum = fmaf(-(float)A->ell_val[idx], x[col], sum);
        }
        rc[l][A->perm_c[ic]] = sum;
    }
    oc_mg_level_f32(L, l + 1, nlevels, rc[l], xc[l], rc, xc);
#pragma omp parallel for schedule(static)
    for(int ic = 0; ic < A->nc; ++ic) x[A->perm[A->f2c[ic]]] += xc[l][A->perm_c[ic]];
    for(int i = 0; i < A->nblocks; ++i) oc_sweep_f32(A, A->sizes[i], A->offsets[i], r, x);
    for(int i = A->ublocks; i >= 0; --i) oc_sweep_f32(A, A->sizes[i], A->offsets[i], r, x);
}

void oc_mg_f32(const oc_level* levels, int nlevels, const float* r, float* x)
{
    float* rc[16];
    float* xc[16];
    for(int l = 0; l + 1 < nlevels && l < 16; ++l)
    {
        rc[l] = (float*)malloc(sizeof(float) * (size_t)levels[l].nc);
        xc[l] = (float*)malloc(sizeof(float) * (size_t)levels[l].nc);
    }
    oc_mg_level_f32(levels, 0, nlevels, r, x, rc, xc);
    for(int l = 0; l + 1 < nlevels && l < 16; ++l)
    {
        free(rc[l]);
        free(xc[l]);
    }
}
