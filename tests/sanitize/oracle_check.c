/* The CPU restatements (oracle/colored.c, oracle/distributed.c,
 * oracle/distributed_ref.c) run under AddressSanitizer and
 * UndefinedBehaviorSanitizer on small problems: every operator of the
 * multi-rank optimized path, its CG, the multi-rank reference CG and the
 * single-rank coloured CG.  Built and run by tests/test_sanitizers.py; exits
 * 0 when every run ends with a finite residual below its start. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "colored.h"
#include "distributed.h"

static int check_dist(int size, int nx, int ny, int nz, int nlevels)
{
    int npx, npy, npz;
    od_shape(size, &npx, &npy, &npz);
    od_problem* P = od_create(size, npx, npy, npz, nx, ny, nz, nlevels);
    if(!P) return 1;
    int niters = 0;
    double normr = 0.0, normr0 = 0.0;
    double* hist = calloc(31, sizeof(double));
    od_cg(P, 30, 0.0, 1, NULL, NULL, &niters, &normr, &normr0, hist);
    const int ok = niters == 30 && isfinite(normr) && normr < normr0;
    free(hist);
    od_destroy(P);
    odr_problem* R = odr_create(size, npx, npy, npz, nx, ny, nz, nlevels);
    if(!R) return 1;
    odr_cg(R, 30, 0.0, 1, &niters, &normr, &normr0, NULL);
    const int ok2 = niters == 30 && isfinite(normr) && normr < normr0;
    odr_destroy(R);
    return ok && ok2 ? 0 : 1;
}

int main(void)
{
    int bad = 0;
    bad += check_dist(1, 16, 16, 16, 4);
    bad += check_dist(2, 16, 8, 8, 3);
    bad += check_dist(4, 8, 8, 16, 3);
    bad += check_dist(8, 8, 8, 8, 3);
    bad += check_dist(3, 16, 8, 8, 4);
    bad += check_dist(6, 8, 8, 8, 2);
    if(bad) fprintf(stderr, "%d oracle runs failed\n", bad);
    else printf("oracle restatements: all runs clean\n");
    return bad ? 1 : 0;
}
