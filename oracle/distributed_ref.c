/*
 * Multi-rank restatement of rocHPCG's REFERENCE path (the natural-order `_ref`
 * routines that src/test_rochpcg.cpp runs before the optimized CG to fix the
 * tolerance), every rank held in one process.  TEST INFRASTRUCTURE ONLY: the
 * tests use it to hold the decomposed CUDA path to the reference's own
 * multi-rank iteration bounds; the product library never links it.
 *
 * Vectors hold every rank's rows, rank after rank, each rank's rows in natural
 * order.  A column names the row it reads by that concatenated index; for a
 * column owned by another rank the index is stored negative (-(index + 1)).
 * ExchangeHalo (src/ExchangeHalo.cpp:67-187) by its meaning: the external
 * columns take the owner's values at the moment of the exchange.  SpMV reads
 * them from the live vector (nothing changes during an SpMV); the Gauss-Seidel
 * sweeps read them from a copy taken when the sweep starts, since the owner
 * goes on updating its rows while this rank sweeps.
 *
 * The floating-point operations are the reference's, in its order, with no
 * contraction (the file is built with -ffp-contract=off, the reference's
 * `_ref` build emits no fma on x86-64 either).  Dot products: each rank's
 * sum in index order (ComputeDotProduct_ref.cpp:51-63, one thread), then the
 * ranks' sums added in rank order (MPI_Allreduce, :70, whose order MPI leaves
 * to the implementation; with two ranks the sum is the same either way).
 */
#include "distributed.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define W 27
#define MAXL 8

typedef struct
{
    int nx, ny, nz, m;  /* per-rank brick */
    int8_t* nnz;        /* [size*m] */
    int* col;           /* [size*m*W] row-major, in the generation order */
    int* f2c;           /* [m of the next level]: natural fine row of each coarse row */
    double* b;          /* level 0: generated right-hand side */
    double* rc;         /* MG work of the next level: rhs, x */
    double* xc;
    double* Axf;        /* this level's A x (restriction) */
} odr_level;

struct odr_problem
{
    int size, npx, npy, npz, nlevels;
    odr_level L[MAXL];
    double* snap; /* the exchange copy of a Gauss-Seidel sweep */
};

/* src/GenerateGeometry.cpp:126-166 + src/GenerateProblem_ref.cpp:140-201 for
 * every rank: the 27 neighbours in (sz, sy, sx) order, those outside the
 * global grid left out; b = 26 - (nonzeros - 1) (:196). */
static void build(odr_level* A, int size, int npx, int npy, int npz, int nx, int ny, int nz, int with_b)
{
    const int m = nx * ny * nz;
    A->nx = nx, A->ny = ny, A->nz = nz, A->m = m;
    const long long gnx = (long long)npx * nx, gny = (long long)npy * ny, gnz = (long long)npz * nz;
    const size_t rows = (size_t)size * m;
    A->nnz = malloc(rows);
    A->col = malloc(sizeof(int) * rows * W);
    if(with_b) A->b = malloc(sizeof(double) * rows);
#pragma omp parallel for schedule(static)
    for(int q = 0; q < size; ++q)
    {
        const int ipz = q / (npx * npy), ipy = (q - ipz * npx * npy) / npx, ipx = q % npx;
        for(int i = 0; i < m; ++i)
        {
            const int iz = i / (nx * ny), iy = (i / nx) % ny, ix = i % nx;
            const long long gx0 = (long long)ipx * nx + ix, gy0 = (long long)ipy * ny + iy,
                            gz0 = (long long)ipz * nz + iz;
            const size_t g = (size_t)q * m + i;
            int n = 0;
            for(int sz = -1; sz <= 1; ++sz)
            {
                const long long gz = gz0 + sz;
                if(gz < 0 || gz >= gnz) continue;
                for(int sy = -1; sy <= 1; ++sy)
                {
                    const long long gy = gy0 + sy;
                    if(gy < 0 || gy >= gny) continue;
                    for(int sx = -1; sx <= 1; ++sx)
                    {
                        const long long gx = gx0 + sx;
                        if(gx < 0 || gx >= gnx) continue;
                        const int px = (int)(gx / nx), py = (int)(gy / ny), pz = (int)(gz / nz);
                        const int owner = px + py * npx + pz * npx * npy;
                        const int lrow = (int)(((gz - (long long)pz * nz) * ny + (gy - (long long)py * ny)) * nx +
                                               (gx - (long long)px * nx));
                        const int idx = owner * m + lrow;
                        A->col[g * W + n++] = owner == q ? idx : -(idx + 1);
                    }
                }
            }
            A->nnz[g] = (int8_t)n;
            if(with_b) A->b[g] = 26.0 - ((double)(n - 1));
        }
    }
}

/* src/GenerateCoarseProblem.cpp (f2cOperator): coarse (ix, iy, iz) injects
 * the fine row (2 ix, 2 iy, 2 iz) of the same rank. */
static void build_f2c(odr_level* A, const odr_level* C)
{
    A->f2c = malloc(sizeof(int) * (size_t)C->m);
    for(int izc = 0; izc < C->nz; ++izc)
        for(int iyc = 0; iyc < C->ny; ++iyc)
            for(int ixc = 0; ixc < C->nx; ++ixc)
                A->f2c[(izc * C->ny + iyc) * C->nx + ixc] = ((2 * izc) * A->ny + 2 * iyc) * A->nx + 2 * ixc;
}

odr_problem* odr_create(int size, int npx, int npy, int npz, int nx, int ny, int nz, int nlevels)
{
    if(npx <= 0 || npy <= 0 || npz <= 0) od_shape(size, &npx, &npy, &npz);
    if(npx * npy * npz != size || nlevels < 1 || nlevels > MAXL) return NULL;
    for(int l = 0; l < nlevels; ++l)
        if((nx >> l) < 1 || (ny >> l) < 1 || (nz >> l) < 1) return NULL;
    odr_problem* P = calloc(1, sizeof(odr_problem));
    P->size = size, P->npx = npx, P->npy = npy, P->npz = npz, P->nlevels = nlevels;
    for(int l = 0; l < nlevels; ++l) build(&P->L[l], size, npx, npy, npz, nx >> l, ny >> l, nz >> l, l == 0);
    for(int l = 0; l + 1 < nlevels; ++l)
    {
        odr_level* A = &P->L[l];
        const odr_level* C = &P->L[l + 1];
        build_f2c(A, C);
        A->rc = calloc((size_t)size * C->m, sizeof(double));
        A->xc = calloc((size_t)size * C->m, sizeof(double));
    }
    for(int l = 0; l < nlevels; ++l) P->L[l].Axf = calloc((size_t)size * P->L[l].m, sizeof(double));
    P->snap = malloc(sizeof(double) * (size_t)size * P->L[0].m);
    return P;
}

void odr_destroy(odr_problem* P)
{
    if(!P) return;
    for(int l = 0; l < P->nlevels; ++l)
    {
        odr_level* A = &P->L[l];
        free(A->nnz), free(A->col), free(A->f2c), free(A->b), free(A->rc), free(A->xc), free(A->Axf);
    }
    free(P->snap);
    free(P);
}

static double value(int c, size_t g) { return c == (int)g ? 26.0 : -1.0; }

/* src/ComputeSPMV_ref.cpp:48-75 on every rank (after ExchangeHalo). */
void odr_spmv(const odr_problem* P, int level, const double* x, double* y)
{
    const odr_level* A = &P->L[level];
    const long long rows = (long long)P->size * A->m;
#pragma omp parallel for schedule(static)
    for(long long g = 0; g < rows; ++g)
    {
        double sum = 0.0;
        const int* c = A->col + (size_t)g * W;
        for(int j = 0; j < A->nnz[g]; ++j)
        {
            const int k = c[j] >= 0 ? c[j] : -c[j] - 1;
            sum += value(c[j], (size_t)g) * x[k];
        }
        y[g] = sum;
    }
}

/* One row of src/ComputeSYMGS_ref.cpp:73-87 (the same body serves the back
 * sweep, :93-107): local columns from the live x, external ones from the
 * exchange copy. */
static inline void gs_row(const odr_level* A, size_t g, const double* r, double* x, const double* snap)
{
    const int* c = A->col + g * W;
    const double diag = 26.0;
    double sum = r[g];
    for(int j = 0; j < A->nnz[g]; ++j)
    {
        const double xv = c[j] >= 0 ? x[c[j]] : snap[-c[j] - 1];
        sum -= value(c[j], g) * xv;
    }
    sum += x[g] * diag;
    x[g] = sum / diag;
}

/* src/ComputeSYMGS_ref.cpp:51-111 on every rank: ExchangeHalo, then the
 * forward and the backward sweep over the rank's rows. */
void odr_symgs(odr_problem* P, int level, const double* r, double* x)
{
    const odr_level* A = &P->L[level];
    const size_t rows = (size_t)P->size * A->m;
    memcpy(P->snap, x, sizeof(double) * rows);
    const double* snap = P->snap;
#pragma omp parallel for schedule(static, 1)
    for(int q = 0; q < P->size; ++q)
    {
        const size_t g0 = (size_t)q * A->m;
        for(int i = 0; i < A->m; ++i) gs_row(A, g0 + i, r, x, snap);
        for(int i = A->m - 1; i >= 0; --i) gs_row(A, g0 + i, r, x, snap);
    }
}

/* src/ComputeMG_ref.cpp:38-66 (one pre- and one post-smoothing step),
 * ComputeRestriction_ref.cpp:51, ComputeProlongation_ref.cpp:49. */
static void mg(odr_problem* P, int l, const double* r, double* x)
{
    const odr_level* A = &P->L[l];
    const size_t rows = (size_t)P->size * A->m;
    memset(x, 0, sizeof(double) * rows);
    if(l + 1 >= P->nlevels)
    {
        odr_symgs(P, l, r, x);
        return;
    }
    const odr_level* C = &P->L[l + 1];
    odr_symgs(P, l, r, x);
    odr_spmv(P, l, x, A->Axf);
    for(int q = 0; q < P->size; ++q)
        for(int i = 0; i < C->m; ++i)
        {
            const size_t f = (size_t)q * A->m + A->f2c[i];
            A->rc[(size_t)q * C->m + i] = r[f] - A->Axf[f];
        }
    mg(P, l + 1, A->rc, A->xc);
    for(int q = 0; q < P->size; ++q)
        for(int i = 0; i < C->m; ++i) x[(size_t)q * A->m + A->f2c[i]] += A->xc[(size_t)q * C->m + i];
    odr_symgs(P, l, r, x);
}

void odr_mg(odr_problem* P, const double* r, double* x) { mg(P, 0, r, x); }

/* src/ComputeDotProduct_ref.cpp:51-76 per rank, then summed over the ranks. */
static double dot(const odr_problem* P, const double* a, const double* b)
{
    const int m = P->L[0].m;
    double part[64];
#pragma omp parallel for schedule(static, 1)
    for(int q = 0; q < P->size; ++q)
    {
        double s = 0.0;
        const size_t g0 = (size_t)q * m;
        for(int i = 0; i < m; ++i) s += a[g0 + i] * b[g0 + i];
        part[q] = s;
    }
    double s = part[0];
    for(int q = 1; q < P->size; ++q) s += part[q];
    return s;
}

/* src/CG_ref.cpp:86-170 from x = 0 with the generated b; the WAXPBY forms of
 * src/ComputeWAXPBY_ref.cpp:51-67. */
void odr_cg(odr_problem* P, int max_iter, double tol, int precond, int* niters, double* normr, double* normr0,
            double* hist)
{
    const size_t n = (size_t)P->size * P->L[0].m;
    const double* b = P->L[0].b;
    double* x = calloc(n, sizeof(double));
    double* p = calloc(n, sizeof(double));
    double* Ap = calloc(n, sizeof(double));
    double* r = calloc(n, sizeof(double));
    double* z = calloc(n, sizeof(double));
    memcpy(p, x, sizeof(double) * n);                           /* CopyVector(x, p) */
    odr_spmv(P, 0, p, Ap);                                       /* Ap = A p */
    for(size_t i = 0; i < n; ++i) r[i] = b[i] + -1.0 * Ap[i];   /* r = b - Ap (alpha == 1) */
    double nr = sqrt(dot(P, r, r));
    const double nr0 = nr;
    if(hist) hist[0] = nr;
    double rtz = 0.0, oldrtz = 0.0, alpha = 0.0, beta = 0.0, pAp = 0.0;
    *niters = 0;
    for(int k = 1; k <= max_iter && nr / nr0 > tol; ++k)
    {
        if(precond) odr_mg(P, r, z);
        else
            for(size_t i = 0; i < n; ++i) z[i] = r[i] + 0.0 * r[i];
        if(k == 1)
        {
            memcpy(p, z, sizeof(double) * n);
            rtz = dot(P, r, z);
        }
        else
        {
            oldrtz = rtz;
            rtz = dot(P, r, z);
            beta = rtz / oldrtz;
            for(size_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
        }
        odr_spmv(P, 0, p, Ap);
        pAp = dot(P, p, Ap);
        alpha = rtz / pAp;
        for(size_t i = 0; i < n; ++i) x[i] = x[i] + alpha * p[i];
        for(size_t i = 0; i < n; ++i) r[i] = r[i] + -alpha * Ap[i];
        nr = sqrt(dot(P, r, r));
        if(hist) hist[k] = nr;
        *niters = k;
    }
    *normr = nr;
    *normr0 = nr0;
    free(x), free(p), free(Ap), free(r), free(z);
}
