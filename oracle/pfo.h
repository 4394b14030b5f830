/*
 * ORACLE / TEST INFRASTRUCTURE -- never part of the product path.
 *
 * pfo: a CPU restatement of the reference's exact Fincke-Pohst enumeration
 * (pfvs/fp_kernel/fpk_search_impl.h:217-455, double instantiation, with the
 * kernel contract of pfvs/fp_kernel/fp_kernel.h:25-63), used to check the
 * B200 path.  Returns exactly the c in Z^dim with
 *
 *     q(c) = c^T mat c <= qmax                          (ellipsoid)
 *     linvec . c >= linmin            [if linvec]       (M0 cut)
 *     g == 0 or Q g > q(c)  (Q g >= q(c) if !strict)   (GCD cut)
 *
 * with g = gcd of the `leaf` rows evaluated at c (exact, int128), in DFS
 * order (last coordinate outermost, ascending).  Floating point (U, the
 * M0 bound data) only prunes, widened by the reference's rigorous error
 * model; `prune` rows (any rows whose gcd at c is a multiple of g, grouped
 * by their first nonzero column) only prune.  With leaf_gcd = 0 the exact
 * GCD test is left to the caller.
 */
#ifndef PFO_H
#define PFO_H
#include <stdint.h>

typedef struct {
    int dim;
    int64_t Q, qmax, linmin;
    int strict;
    double eps;                 /* extra absolute pruning slack */
    const double *U;            /* (dim, dim) upper triangular, U^T U ~ mat */
    const int64_t *mat;         /* (dim, dim) exact */
    const int64_t *linvec;      /* (dim,) or NULL */
    const double *m0N, *m0V, *m0Va;   /* M0 bound data (if linvec) */
    int nprune;
    const int64_t *Hp;          /* (nprune, dim) pruning rows */
    int nleaf;
    const int64_t *Hl;          /* (nleaf, dim) exact leaf rows */
    int leaf_gcd;
    long max_out;
} pfo_problem;

/* Status: 0 done; -2 more than max_out points (the first max_out kept);
 * -7 out of memory; -8 a coordinate range beyond int32; -12 an exact leaf
 * value beyond int128 (undecided here). */
int pfo_search(const pfo_problem *P, int32_t **pts, int64_t **qs, long *n, long *nodes);
void pfo_free(void *p);

#endif
