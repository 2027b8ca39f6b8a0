/*
 * CPU restatement of rocHPCG's MULTI-RANK optimized path, every rank held in
 * one process.  TEST INFRASTRUCTURE ONLY: used by tests/ as the checker of
 * the decomposed CUDA path; the product library never links it.
 *
 * Each function cites the reference code it restates (paths relative to the
 * rocHPCG source tree).  The halo plan is rebuilt here from the global
 * column ids the way src/SetupHalo.cpp numbers them, and the exchange is
 * stated by its meaning -- an external column takes the value of the row it
 * names on its owner -- not through send lists, so the CUDA path's send
 * lists are checked rather than reused.
 */
#ifndef HPCG_ORACLE_DISTRIBUTED_H
#define HPCG_ORACLE_DISTRIBUTED_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct od_problem od_problem;

/* src/ComputeOptimalShapeXYZ.cpp:94-157 restated once more (oracle side). */
void od_shape(int size, int* npx, int* npy, int* npz);

/* All ranks of a size = npx*npy*npz decomposition with local brick
 * nx*ny*nz, nlevels MG levels: src/GenerateGeometry.cpp:84-166,
 * src/GenerateProblem.cpp:98-303 (global column ids), src/SetupHalo.cpp:
 * 135-651 (external numbering), src/MultiColoring.cpp (colouring of the local
 * columns), src/Permute.cpp:95-185 + src/SparseMatrix.cpp:166-389 (ELL with
 * the external columns after the local ones), GenerateCoarseProblem. */
od_problem* od_create(int size, int npx, int npy, int npz, int nx, int ny, int nz, int nlevels);
void od_destroy(od_problem* P);

/* info[8] = {m, next, nblocks, ublocks, nhalo_rows, nx, ny, nz} */
void od_level_info(const od_problem* P, int rank, int level, int* info);
/* Copies of a level's arrays: perm[m], ell_col[27*m], ell_val[27*m],
 * ext_gid[next] (int64), b[m] (level 0, permuted). */
void od_level_perm(const od_problem* P, int rank, int level, int* out);
void od_level_ell(const od_problem* P, int rank, int level, int* col, double* val);
void od_level_ext_gid(const od_problem* P, int rank, int level, long long* out);
void od_level_b(const od_problem* P, int rank, double* out);

/* Operators over all ranks; vectors are per-rank arrays in permuted order,
 * x-type ones of length m + next (the external tail is written by the
 * exchange these functions perform). */
void od_exchange(const od_problem* P, int level, double** xs);
void od_spmv(const od_problem* P, int level, double** xs, double** ys);        /* ComputeSPMV.cpp:226-278 */
void od_symgs(const od_problem* P, int level, double** rs, double** xs);       /* ComputeSYMGS.cpp:369-404 */
void od_symgs_zero(const od_problem* P, int level, double** rs, double** xs);  /* ComputeSYMGS.cpp:406-454 */
void od_restrict(const od_problem* P, int level, double** rfs, double** xfs, double** rcs); /* ComputeRestriction.cpp:199-237 */
void od_mg(od_problem* P, double** rs, double** xs);                           /* ComputeMG.cpp:64-102 */
/* CG.cpp:104-200 from x = 0 with b = bs[r] (permuted; NULL: the generated b);
 * dot products: per rank in fixed blocks, then summed in rank order
 * (ComputeDotProduct.cpp:189-238 with MPI_Allreduce).  xs receive the
 * solution (length m each), hist (max_iter+1) the residual norms. */
void od_cg(od_problem* P, int max_iter, double tol, int precond, double** bs, double** xs, int* niters,
           double* normr, double* normr0, double* hist);

/* The REFERENCE (natural-order `_ref`) path over the same decomposition
 * (oracle/distributed_ref.c): vectors hold every rank's rows rank after rank,
 * each rank's in natural order.  src/test_rochpcg.cpp:262-271 runs its CG_ref
 * for 50 iterations to fix the tolerance of the optimized CG. */
typedef struct odr_problem odr_problem;
odr_problem* odr_create(int size, int npx, int npy, int npz, int nx, int ny, int nz, int nlevels);
void odr_destroy(odr_problem* P);
void odr_spmv(const odr_problem* P, int level, const double* x, double* y);  /* ComputeSPMV_ref.cpp:48-75 */
void odr_symgs(odr_problem* P, int level, const double* r, double* x);      /* ComputeSYMGS_ref.cpp:51-111 */
void odr_mg(odr_problem* P, const double* r, double* x);                    /* ComputeMG_ref.cpp:38-66 */
void odr_cg(odr_problem* P, int max_iter, double tol, int precond, int* niters, double* normr, double* normr0,
            double* hist);                                                   /* CG_ref.cpp:86-170 */

#ifdef __cplusplus
}
#endif
#endif
