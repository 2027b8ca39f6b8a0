/*
 * Multi-rank restatement of rocHPCG's optimized path (see distributed.h).
 * TEST INFRASTRUCTURE ONLY.
 */
#include "distributed.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "colored.h"

#define W 27

typedef struct
{
    int nx, ny, nz, m, next, ncols;
    long long gnx, gny, gnz, gix0, giy0, giz0;
    int nblocks, ublocks, ncolors;
    int* sizes;
    int* offsets;
    int* perm;
    int* ell_col;
    double* ell_val;
    int* diag_idx;
    double* inv_diag;
    int* has_ext;          /* per permuted row: 1 if it has external columns */
    int nhalo;
    long long* ext_gid;    /* [next] */
    int* ext_rank;         /* owner of external column m+e */
    int* ext_row;          /* its natural row on the owner */
    double* b;             /* level 0: permuted generated b */
    int nc;                /* to the next level */
    int* f2c;
    double* rc;            /* next level's rhs / x (x with external tail), MG work */
    double* xc;
} od_level;

struct od_problem
{
    int size, npx, npy, npz, nlevels;
    od_level** L; /* L[rank][level] */
};

/* ------------------------------------------------------------ process grid */

static int ipow_(int b, int e)
{
    int v = 1;
    while(e-- > 0) v *= b;
    return v;
}

/* ComputeOptimalShapeXYZ.cpp:47-72 (prime factors), :94-157 (the split). */
void od_shape(int size, int* npx, int* npy, int* npz)
{
    int p[32], c[32], k = 0, n = size;
    const int limit = (int)sqrt((double)size) + 1;
    if(n > 1 && (n & 1) == 0)
    {
        p[k] = 2, c[k] = 0;
        while(n > 1 && (n & 1) == 0) c[k]++, n >>= 1;
        ++k;
    }
    for(int d = 3; d <= limit; d += 2)
        if(n % d == 0)
        {
            p[k] = d, c[k] = 0;
            while(n % d == 0) c[k]++, n /= d;
            ++k;
        }
    if(n > 1 || k == 0) p[k] = n, c[k] = 1, ++k;
    if(k == 1)
    {
        *npz = ipow_(p[0], c[0] / 3);
        *npy = ipow_(p[0], c[0] / 3 + (c[0] % 3 >= 2));
        *npx = ipow_(p[0], c[0] / 3 + (c[0] % 3 >= 1));
        return;
    }
    if(k == 2 && c[0] == 1 && c[1] == 1)
    {
        *npx = p[0], *npy = p[1], *npz = 1;
        return;
    }
    if(k == 2 && c[0] + c[1] == 3)
    {
        *npx = p[0], *npy = p[1], *npz = c[0] == 2 ? p[0] : p[1];
        return;
    }
    if(k == 3 && c[0] == 1 && c[1] == 1 && c[2] == 1)
    {
        *npx = p[0], *npy = p[1], *npz = p[2];
        return;
    }
    /* MixedBaseCounter walk: c1 over nonzero sub-multisets, c2 over nonzero
     * sub-multisets of the rest, first least surface kept */
    int a[32] = {0};
    double best = 2.0 * size + 1.0;
    for(;;)
    {
        int i = 0;
        for(; i < k; ++i)
        {
            if(++a[i] <= c[i]) break;
            a[i] = 0;
        }
        if(i == k) break;
        int b[32] = {0};
        for(;;)
        {
            int j = 0;
            for(; j < k; ++j)
            {
                if(++b[j] <= c[j] - a[j]) break;
                b[j] = 0;
            }
            if(j == k) break;
            int t1 = 1, t2 = 1;
            for(int q = 0; q < k; ++q) t1 *= ipow_(p[q], a[q]), t2 *= ipow_(p[q], b[q]);
            const int t3 = size / t1 / t2;
            const double area = t1 * (double)t2 + t2 * (double)t3 + t1 * (double)t3;
            if(area < best) best = area, *npx = t1, *npy = t2, *npz = t3;
        }
    }
}

/* ------------------------------------------------------------ set-up */

static int cmp_ll(const void* a, const void* b)
{
    const long long x = *(const long long*)a, y = *(const long long*)b;
    return x < y ? -1 : x > y;
}

static int find_ll(const long long* v, int n, long long key)
{
    int lo = 0, hi = n;
    while(lo < hi)
    {
        const int mid = (lo + hi) / 2;
        if(v[mid] < key) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

/* Returns 0, or -1 when the colouring left rows uncoloured: the reference's
 * loop `while(colored != m)` counts colour VALUES, and a round that draws
 * c1 == c2 counts its rows twice, which on a few tiny bricks (4x3x2) ends the
 * loop with rows still at -1; such levels are not restated. */
static int build_level(od_level* A, int rank, int npx, int npy, int npz, int nx, int ny, int nz, int with_b)
{
    /* GenerateGeometry.cpp:84-86,126-166 */
    const int ipz = rank / (npx * npy), ipy = (rank - ipz * npx * npy) / npx, ipx = rank % npx;
    A->nx = nx, A->ny = ny, A->nz = nz;
    const int m = A->m = nx * ny * nz;
    A->gnx = (long long)npx * nx, A->gny = (long long)npy * ny, A->gnz = (long long)npz * nz;
    A->gix0 = (long long)ipx * nx, A->giy0 = (long long)ipy * ny, A->giz0 = (long long)ipz * nz;

    /* colouring and permutation: the local columns only (MultiColoring.cpp:193),
     * i.e. the single-rank problem of the brick */
    int* cols = malloc(sizeof(int) * (size_t)m * W);
    double* vals = malloc(sizeof(double) * (size_t)m * W);
    int8_t* nnz = malloc((size_t)m);
    int* dslot = malloc(sizeof(int) * (size_t)m);
    int* hash = malloc(sizeof(int) * (size_t)m);
    oc_generate(nx, ny, nz, cols, vals, nnz, dslot, hash, NULL);
    int* colors = malloc(sizeof(int) * (size_t)m);
    int rcol[256], rsz[256];
    const int nb = oc_jpl_coloring(m, cols, nnz, hash, colors, rcol, rsz);
    int maxc = 0, minc = 0;
    for(int i = 0; i < m; ++i)
    {
        maxc = colors[i] > maxc ? colors[i] : maxc;
        minc = colors[i] < minc ? colors[i] : minc;
    }
    if(nb < 0 || minc < 0)
    {
        free(colors), free(cols), free(vals), free(nnz), free(dslot), free(hash);
        return -1;
    }
    /* Sweeps over the colour VALUES 0..maxc (the by-value blocks; the
     * reference's nblocks counts JPL rounds, which on bricks that need fewer
     * than 8 colours can be below the largest value drawn -- its round-order
     * sizes[] then straddle colours); ublocks one below the last, as
     * MultiColoring.cpp:316,350-352. */
    A->nblocks = maxc + 1;
    A->ublocks = maxc - 1;
    A->ncolors = nb > maxc + 1 ? nb : maxc + 1;
    A->sizes = calloc((size_t)A->ncolors, sizeof(int));
    A->offsets = calloc((size_t)A->ncolors + 1, sizeof(int));
    A->perm = malloc(sizeof(int) * (size_t)m);
    oc_color_perm(m, colors, A->ncolors, A->perm, A->sizes, A->offsets);
    free(colors);
    free(cols);
    free(vals);
    free(nnz);
    free(dslot);
    free(hash);

    /* global column ids of every row (GenerateProblem.cpp:98-303), external
     * ones classified by the neighbour's relative position (SetupHalo.cpp:
     * 135-257) */
    long long* recv[27];
    int nrecv[27] = {0}, cap[27];
    for(int s = 0; s < 27; ++s) cap[s] = 64, recv[s] = malloc(sizeof(long long) * 64);
    for(int row = 0; row < m; ++row)
    {
        const int iz = row / (nx * ny), iy = (row / nx) % ny, ix = row % nx;
        for(int t = 0; t < W; ++t)
        {
            const int dz = t / 9 - 1, dy = (t / 3) % 3 - 1, dx = t % 3 - 1;
            const long long gx = A->gix0 + ix + dx, gy = A->giy0 + iy + dy, gz = A->giz0 + iz + dz;
            if(gx < 0 || gy < 0 || gz < 0 || gx >= A->gnx || gy >= A->gny || gz >= A->gnz) continue;
            const int px = (int)(gx / nx), py = (int)(gy / ny), pz = (int)(gz / nz);
            const int slot = (pz - ipz + 1) * 9 + (py - ipy + 1) * 3 + (px - ipx + 1);
            if(slot == 13) continue;
            if(nrecv[slot] == cap[slot])
                cap[slot] *= 2, recv[slot] = realloc(recv[slot], sizeof(long long) * (size_t)cap[slot]);
            recv[slot][nrecv[slot]++] = (gz * A->gny + gy) * A->gnx + gx;
        }
    }
    int base[27];
    A->next = 0;
    for(int s = 0; s < 27; ++s)
    {
        qsort(recv[s], (size_t)nrecv[s], sizeof(long long), cmp_ll);
        int u = 0;
        for(int i = 0; i < nrecv[s]; ++i)
            if(u == 0 || recv[s][u - 1] != recv[s][i]) recv[s][u++] = recv[s][i];
        nrecv[s] = u;
        base[s] = A->next;
        A->next += u;
    }
    A->ncols = m + A->next;
    A->ext_gid = malloc(sizeof(long long) * (size_t)(A->next ? A->next : 1));
    A->ext_rank = malloc(sizeof(int) * (size_t)(A->next ? A->next : 1));
    A->ext_row = malloc(sizeof(int) * (size_t)(A->next ? A->next : 1));
    for(int s = 0; s < 27; ++s)
        for(int i = 0; i < nrecv[s]; ++i)
        {
            const long long gid = recv[s][i];
            const long long gx = gid % A->gnx, gy = (gid / A->gnx) % A->gny, gz = gid / (A->gnx * A->gny);
            const int px = (int)(gx / nx), py = (int)(gy / ny), pz = (int)(gz / nz);
            const int e = base[s] + i;
            A->ext_gid[e] = gid;
            A->ext_rank[e] = px + py * npx + pz * npx * npy;
            A->ext_row[e] = (int)(((gz - (long long)pz * nz) * ny + (gy - (long long)py * ny)) * nx +
                                  (gx - (long long)px * nx));
        }

    /* ELL: keys perm[col] (local), m + external id (external), sorted
     * (Permute.cpp:95-185), rows permuted, diagonal extracted */
    A->ell_col = malloc(sizeof(int) * (size_t)m * W);
    A->ell_val = malloc(sizeof(double) * (size_t)m * W);
    A->diag_idx = malloc(sizeof(int) * (size_t)m);
    A->inv_diag = malloc(sizeof(double) * (size_t)m);
    A->has_ext = calloc((size_t)m, sizeof(int));
    if(with_b) A->b = malloc(sizeof(double) * (size_t)m);
    A->nhalo = 0;
    for(int row = 0; row < m; ++row)
    {
        const int iz = row / (nx * ny), iy = (row / nx) % ny, ix = row % nx;
        int key[W], n = 0, ext = 0;
        for(int t = 0; t < W; ++t)
        {
            const int dz = t / 9 - 1, dy = (t / 3) % 3 - 1, dx = t % 3 - 1;
            const long long gx = A->gix0 + ix + dx, gy = A->giy0 + iy + dy, gz = A->giz0 + iz + dz;
            if(gx < 0 || gy < 0 || gz < 0 || gx >= A->gnx || gy >= A->gny || gz >= A->gnz) continue;
            const int px = (int)(gx / nx), py = (int)(gy / ny), pz = (int)(gz / nz);
            const int slot = (pz - ipz + 1) * 9 + (py - ipy + 1) * 3 + (px - ipx + 1);
            if(slot == 13)
                key[n++] = A->perm[(iz + dz) * nx * ny + (iy + dy) * nx + (ix + dx)];
            else
            {
                const long long gid = (gz * A->gny + gy) * A->gnx + gx;
                key[n++] = m + base[slot] + find_ll(recv[slot], nrecv[slot], gid);
                ++ext;
            }
        }
        for(int i = 1; i < n; ++i)
        {
            const int kk = key[i];
            int j = i - 1;
            while(j >= 0 && key[j] > kk) key[j + 1] = key[j], --j;
            key[j + 1] = kk;
        }
        const int prow = A->perm[row];
        for(int p = 0; p < W; ++p)
        {
            const size_t idx = (size_t)p * m + prow;
            A->ell_col[idx] = p < n ? key[p] : -1;
            A->ell_val[idx] = p < n ? (key[p] == prow ? 26.0 : -1.0) : 0.0;
            if(p < n && key[p] == prow)
            {
                A->diag_idx[prow] = p;
                A->inv_diag[prow] = 1.0 / 26.0;
            }
        }
        A->has_ext[prow] = ext > 0;
        A->nhalo += ext > 0;
        if(with_b) A->b[prow] = 26.0 - (n - 1.0); /* GenerateProblem.cpp: row sum for x = 1 */
    }
    for(int s = 0; s < 27; ++s) free(recv[s]);
    return 0;
}

od_problem* od_create(int size, int npx, int npy, int npz, int nx, int ny, int nz, int nlevels)
{
    if(npx <= 0 || npy <= 0 || npz <= 0) od_shape(size, &npx, &npy, &npz);
    if(npx * npy * npz != size || size > 64) return NULL;
    od_problem* P = calloc(1, sizeof(od_problem));
    P->size = size, P->npx = npx, P->npy = npy, P->npz = npz, P->nlevels = nlevels;
    P->L = malloc(sizeof(od_level*) * (size_t)size);
    int bad = 0;
    for(int r = 0; r < size; ++r)
        P->L[r] = calloc((size_t)nlevels, sizeof(od_level));
    for(int r = 0; r < size && !bad; ++r)
    {
        for(int l = 0; l < nlevels && !bad; ++l)
            bad = build_level(&P->L[r][l], r, npx, npy, npz, nx >> l, ny >> l, nz >> l, l == 0);
        if(bad) break;
        for(int l = 0; l + 1 < nlevels; ++l)
        {
            od_level* A = &P->L[r][l];
            const od_level* C = &P->L[r][l + 1];
            A->nc = C->m;
            A->f2c = malloc(sizeof(int) * (size_t)A->nc);
            oc_f2c(A->nx, A->ny, A->nz, A->f2c);
            A->rc = calloc((size_t)C->m, sizeof(double));
            A->xc = calloc((size_t)C->ncols, sizeof(double));
        }
    }
    if(bad)
    {
        od_destroy(P);
        return NULL;
    }
    return P;
}

void od_destroy(od_problem* P)
{
    if(!P) return;
    for(int r = 0; r < P->size; ++r)
    {
        for(int l = 0; l < P->nlevels; ++l)
        {
            od_level* A = &P->L[r][l];
            free(A->sizes), free(A->offsets), free(A->perm), free(A->ell_col), free(A->ell_val);
            free(A->diag_idx), free(A->inv_diag), free(A->has_ext), free(A->ext_gid), free(A->ext_rank);
            free(A->ext_row), free(A->b), free(A->f2c), free(A->rc), free(A->xc);
        }
        free(P->L[r]);
    }
    free(P->L);
    free(P);
}

void od_level_info(const od_problem* P, int rank, int level, int* info)
{
    const od_level* A = &P->L[rank][level];
    info[0] = A->m, info[1] = A->next, info[2] = A->nblocks, info[3] = A->ublocks, info[4] = A->nhalo;
    info[5] = A->nx, info[6] = A->ny, info[7] = A->nz;
}

void od_level_perm(const od_problem* P, int rank, int level, int* out)
{
    const od_level* A = &P->L[rank][level];
    memcpy(out, A->perm, sizeof(int) * (size_t)A->m);
}

void od_level_ell(const od_problem* P, int rank, int level, int* col, double* val)
{
    const od_level* A = &P->L[rank][level];
    memcpy(col, A->ell_col, sizeof(int) * (size_t)A->m * W);
    memcpy(val, A->ell_val, sizeof(double) * (size_t)A->m * W);
}

void od_level_ext_gid(const od_problem* P, int rank, int level, long long* out)
{
    const od_level* A = &P->L[rank][level];
    memcpy(out, A->ext_gid, sizeof(long long) * (size_t)A->next);
}

void od_level_b(const od_problem* P, int rank, double* out)
{
    const od_level* A = &P->L[rank][0];
    memcpy(out, A->b, sizeof(double) * (size_t)A->m);
}

/* ------------------------------------------------------------ operators */

/* ExchangeHalo.cpp:189-275 by its meaning: x[m+e] = the owner's value of the
 * row that external column e names. */
void od_exchange(const od_problem* P, int level, double** xs)
{
    for(int r = 0; r < P->size; ++r)
    {
        const od_level* A = &P->L[r][level];
        for(int e = 0; e < A->next; ++e)
        {
            const od_level* O = &P->L[A->ext_rank[e]][level];
            xs[r][A->m + e] = xs[A->ext_rank[e]][O->perm[A->ext_row[e]]];
        }
    }
}

/* ComputeSPMV.cpp:130-170 (interior, local columns) + :172-208 (halo,
 * external columns from 0, added). */
void od_spmv(const od_problem* P, int level, double** xs, double** ys)
{
    od_exchange(P, level, xs);
    for(int r = 0; r < P->size; ++r)
    {
        const od_level* A = &P->L[r][level];
        const int m = A->m;
        const double* x = xs[r];
        for(int row = 0; row < m; ++row)
        {
            double s = 0.0, t = 0.0;
            for(int p = 0; p < W; ++p)
            {
                const size_t idx = (size_t)p * m + row;
                const int col = A->ell_col[idx];
                if(col >= 0 && col < m) s = fma(A->ell_val[idx], x[col], s);
            }
            if(A->has_ext[row])
            {
                for(int p = 0; p < W; ++p)
                {
                    const size_t idx = (size_t)p * m + row;
                    const int col = A->ell_col[idx];
                    if(col >= m) t = fma(A->ell_val[idx], x[col], t);
                }
                s = s + t;
            }
            ys[r][row] = s;
        }
    }
}

static void sweep(const od_level* A, int c, int ncols, const double* rr, double* x)
{
    const int m = A->m;
    for(int row = A->offsets[c]; row < A->offsets[c] + A->sizes[c]; ++row)
    {
        double s = rr[row];
        for(int p = 0; p < W; ++p)
        {
            const size_t idx = (size_t)p * m + row;
            const int col = A->ell_col[idx];
            if(col >= 0 && col < ncols && col != row) s = fma(-A->ell_val[idx], x[col], s);
        }
        x[row] = s * A->inv_diag[row];
    }
}

/* ComputeSYMGS.cpp:369-404: colour 0 on the local columns (kernel_symgs_interior)
 * then its external part (kernel_symgs_halo), the other colours forward and
 * all colours backward on every column. */
void od_symgs(const od_problem* P, int level, double** rs, double** xs)
{
    od_exchange(P, level, xs);
    for(int r = 0; r < P->size; ++r)
    {
        const od_level* A = &P->L[r][level];
        const int m = A->m;
        double* x = xs[r];
        sweep(A, 0, m, rs[r], x);
        for(int row = A->offsets[0]; row < A->offsets[0] + A->sizes[0]; ++row)
        {
            if(!A->has_ext[row]) continue;
            double t = 0.0;
            for(int p = 0; p < W; ++p)
            {
                const size_t idx = (size_t)p * m + row;
                const int col = A->ell_col[idx];
                if(col >= m) t = fma(-A->ell_val[idx], x[col], t);
            }
            x[row] = fma(t, A->inv_diag[row], x[row]);
        }
        for(int c = 1; c < A->nblocks; ++c) sweep(A, c, A->ncols, rs[r], x);
        for(int c = A->ublocks; c >= 0; --c) sweep(A, c, A->ncols, rs[r], x);
    }
}

void od_symgs_zero(const od_problem* P, int level, double** rs, double** xs)
{
    for(int r = 0; r < P->size; ++r)
    {
        const od_level* A = &P->L[r][level];
        oc_symgs_zero(A->m, A->nblocks, A->ublocks, A->sizes, A->offsets, A->ell_col, A->ell_val, A->diag_idx, rs[r],
                      xs[r]);
    }
}

/* ComputeRestriction.cpp:81-124 (interior) + :126-167 (external part subtracted). */
void od_restrict(const od_problem* P, int level, double** rfs, double** xfs, double** rcs)
{
    od_exchange(P, level, xfs);
    for(int r = 0; r < P->size; ++r)
    {
        const od_level* A = &P->L[r][level];
        const od_level* C = &P->L[r][level + 1];
        const int m = A->m;
        for(int ic = 0; ic < A->nc; ++ic)
        {
            const int row = A->perm[A->f2c[ic]];
            double s = rfs[r][row];
            for(int p = 0; p < W; ++p)
            {
                const size_t idx = (size_t)p * m + row;
                const int col = A->ell_col[idx];
                if(col >= 0 && col < m) s = fma(-A->ell_val[idx], xfs[r][col], s);
            }
            if(A->has_ext[row])
            {
                double t = 0.0;
                for(int p = 0; p < W; ++p)
                {
                    const size_t idx = (size_t)p * m + row;
                    const int col = A->ell_col[idx];
                    if(col >= m) t = fma(A->ell_val[idx], xfs[r][col], t);
                }
                s = s - t;
            }
            rcs[r][C->perm[ic]] = s;
        }
    }
}

static void mg_level(od_problem* P, int l, double** rs, double** xs)
{
    od_symgs_zero(P, l, rs, xs);
    if(l + 1 >= P->nlevels) return;
    double* rc[64];
    double* xc[64];
    for(int r = 0; r < P->size; ++r) rc[r] = P->L[r][l].rc, xc[r] = P->L[r][l].xc;
    od_restrict(P, l, rs, xs, rc);
    mg_level(P, l + 1, rc, xc);
    for(int r = 0; r < P->size; ++r)
    {
        const od_level* A = &P->L[r][l];
        oc_prolong(A->nc, A->f2c, A->perm, P->L[r][l + 1].perm, xc[r], xs[r]);
    }
    od_symgs(P, l, rs, xs);
}

void od_mg(od_problem* P, double** rs, double** xs)
{
    mg_level(P, 0, rs, xs);
}

static double gdot(const od_problem* P, double** a, double** b)
{
    double s = 0.0;
    for(int r = 0; r < P->size; ++r)
    {
        const double d = oc_dot(P->L[r][0].m, a[r], b[r]);
        s = r == 0 ? d : s + d;
    }
    return s;
}

void od_cg(od_problem* P, int max_iter, double tol, int precond, double** bs, double** xs, int* niters,
           double* normr, double* normr0, double* hist)
{
    const int n = P->size;
    double *x[64], *r[64], *z[64], *p[64], *Ap[64], *b[64];
    for(int q = 0; q < n; ++q)
    {
        const od_level* A = &P->L[q][0];
        x[q] = calloc((size_t)A->ncols, sizeof(double));
        p[q] = calloc((size_t)A->ncols, sizeof(double));
        z[q] = calloc((size_t)A->ncols, sizeof(double));
        r[q] = calloc((size_t)A->m, sizeof(double));
        Ap[q] = calloc((size_t)A->m, sizeof(double));
        b[q] = bs ? bs[q] : A->b;
    }
    od_spmv(P, 0, p, Ap);
    for(int q = 0; q < n; ++q)
        for(int i = 0; i < P->L[q][0].m; ++i) r[q][i] = fma(-1.0, Ap[q][i], b[q][i]);
    double nr = sqrt(gdot(P, r, r));
    const double nr0 = nr;
    if(hist) hist[0] = nr;
    double rtz = 0.0;
    *niters = 0;
    for(int k = 1; k <= max_iter && nr / nr0 > tol; ++k)
    {
        if(precond) od_mg(P, r, z);
        else
            for(int q = 0; q < n; ++q) memcpy(z[q], r[q], sizeof(double) * (size_t)P->L[q][0].m);
        const double oldrtz = rtz;
        rtz = gdot(P, r, z);
        const double beta = k == 1 ? 0.0 : rtz / oldrtz;
        for(int q = 0; q < n; ++q)
            for(int i = 0; i < P->L[q][0].m; ++i)
                p[q][i] = k == 1 ? fma(0.0, z[q][i], z[q][i]) : fma(beta, p[q][i], z[q][i]);
        od_spmv(P, 0, p, Ap);
        const double pAp = gdot(P, p, Ap);
        const double alpha = rtz / pAp;
        for(int q = 0; q < n; ++q)
            for(int i = 0; i < P->L[q][0].m; ++i)
            {
                r[q][i] = fma(-alpha, Ap[q][i], r[q][i]);
                x[q][i] = fma(alpha, p[q][i], x[q][i]);
            }
        nr = sqrt(gdot(P, r, r));
        if(hist) hist[k] = nr;
        *niters = k;
    }
    *normr = nr;
    *normr0 = nr0;
    for(int q = 0; q < n; ++q)
    {
        if(xs) memcpy(xs[q], x[q], sizeof(double) * (size_t)P->L[q][0].m);
        free(x[q]), free(p[q]), free(z[q]), free(r[q]), free(Ap[q]);
    }
}
