/*
 * C ABI of libpfvs_gpu.so, the B200 (sm_100a) backend of the batched
 * coniZpM search.
 *
 * The first six entry points and the two structs are the interface the
 * reference's ctypes loader binds (pfvs/gpu.py:37-82), declared as the
 * reference's backend declares them (pfvs/fp_kernel/cuda/pfvs_gpu.cu:64-97);
 * a build of this library can be loaded by the reference package unchanged
 * (PFVS_GPU_LIB=/path/to/libpfvs_gpu.so).  Differences in behaviour, all
 * within the reference's own contract:
 *   - pstat is never 1 ("redo on the CPU"): every direction is finished on
 *     the device, or reported with a negative status that the reference's
 *     coniZpM turns into IncompleteSearchError (pfvs/coni.py:446-453):
 *       -8  a coordinate range exceeds int32 (as the reference kernel)
 *       -9  the ellipsoid matrix is not positive definite
 *       -20 an exact setup value exceeds the device's fixed-width integers
 *       -21 the FP64 factor could not be certified (ill-conditioned)
 *       -22 a direction's search ran past its deadline (pfg_options.deadline_s)
 *   - pfg_max_h11() is 64.
 *   - Out of device memory (a shared or partly filled GPU), a call frees its
 *     per-batch buffers, halves the batch and carries on from the batch it
 *     was on, as the reference's backend does (pfvs_gpu.cu:729-747).
 *
 * The remaining entry points are extensions of this library.
 */
#ifndef PFVS_GPU_H
#define PFVS_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Replaces the reference's pfg_input (pfvs/fp_kernel/cuda/pfvs_gpu.cu:66-78). */
typedef struct {
    int            n_geo;
    const int32_t *h;          /* (n_geo,) h11 of each geometry, 3 <= h <= pfg_max_h11() */
    const int64_t *Q, *qmax, *linmin;   /* (n_geo,) tadpole, floor(dil Q), ceil(M0min) */
    const int64_t *kappa;      /* the geometries' kappa (h^3 each), concatenated */
    const int64_t *Mbasis;     /* the geometries' Mbasis (h^2 each, columns = basis), concatenated */
    int64_t        n_p;
    const int64_t *ps;         /* (n_p, pfg_max_h11()) row-major; p (leading 0) in the first h */
    const int32_t *pgeo;       /* (n_p,) geometry of each p */
    int            device;     /* CUDA device ordinal */
    int64_t        batch;      /* p-vectors per device batch (0: all that fit) */
    int            verbose;
} pfg_input;

/* Replaces the reference's pfg_output (pfvs/fp_kernel/cuda/pfvs_gpu.cu:80-88). */
typedef struct {
    int64_t  n;                /* number of lattice points */
    int64_t *M, *Kn;           /* (n, pfg_max_h11()) row-major; first h entries valid, rest 0 */
    int64_t *q;                /* (n,) exact q = c^T mat c */
    int64_t *pidx;             /* (n,) index of the p-vector */
    int8_t  *pstat;            /* (n_p,) 0 done; < 0 a status (see above) */
    double   seconds_gpu;      /* device time of the call */
    char     err[256];
} pfg_output;

/* pfvs_gpu.cu:91 */
int  pfg_max_h11(void);
/* pfvs_gpu.cu:92 -- "cuda" */
const char *pfg_backend(void);
/* pfvs_gpu.cu:93, :476 */
int  pfg_device_count(void);
/* pfvs_gpu.cu:753-758 -- free the device buffers kept between calls */
void pfg_release(int device);
/* pfvs_gpu.cu:489-751 -- the batched pipeline; 0 on success, else err is set */
int  pfg_coni_batch(const pfg_input *in, pfg_output *out);
/* pfvs_gpu.cu:483-487 -- free the arrays of a pfg_output */
void pfg_output_free(pfg_output *out);

/* ---- extensions (no counterpart in the reference's C ABI) ---- */

/* Search form and pruning precision for pfg_coni_batch_ex. */
enum {
    PFG_FORM_BATCHED = 0,      /* persistent work-stealing kernel over all directions */
    PFG_FORM_PLAIN = 1         /* one warp per direction (one block each, one launch), FP64
                                  pruning, no work sharing: the plain form */
};
enum {
    PFG_PREC_AUTO = 0,         /* the library's choice: FP64 on this build (the search is
                                  latency-bound, so FP32 pruning gains nothing and its
                                  FP64 retries cost; measured on B200) */
    PFG_PREC_FP64 = 1,         /* FP64 pruning everywhere */
    PFG_PREC_FP32 = 2          /* FP32 pruning where qmax < 2^22, FP64 retry on -11 */
};

typedef struct {
    int form;                  /* PFG_FORM_* */
    int precision;             /* PFG_PREC_* */
    int blocks_per_sm;         /* persistent search grid (0: default) */
    int warps_per_block;       /* (0: default, 4; at most 4) */
    double gcd_min_tree;       /* GCD-cut rows are built for a direction whose estimated
                                  search tree has at least this many nodes (they only
                                  prune; results are identical either way).  0: the
                                  library default; < 0: always (the reference's pruning) */
    double wait_s;             /* bound on a search warp's wait for work, counted from the
                                  launch: past it the call fails (rc 1, "a bounded device
                                  wait ran out").  0: 30 s */
    double deadline_s;         /* bound on one subtree's search: past it the direction gets
                                  status -22 and the call goes on.  0: 120 s */
    int check_fp32;            /* with PFG_PREC_FP32: run the FP32 pass with an FP64 shadow of
                                  its pruning bounds (one warp per direction, no work
                                  sharing; same points) and report the bound errors in
                                  pfg_stats.fp32_* (a measurement mode, slower) */
    int compact_rows;          /* pfg_coni_batch_ex only: M and Kn rows w entries wide, w the
                                  largest h11 of in->h, instead of pfg_max_h11() (fewer bytes to
                                  copy back when every h11 is small; pfg_coni_batch keeps the
                                  reference's layout) */
} pfg_options;

/* Statistics of one call. */
typedef struct {
    int64_t nodes;             /* search-tree nodes entered (all passes) */
    int64_t candidates;        /* candidate values tested */
    int64_t leaves;            /* leaf candidates decided exactly */
    int64_t points;            /* points emitted by the search (all passes) */
    int64_t donated;           /* subtrees handed between warps */
    int64_t fp64_retries;      /* directions re-searched in FP64 after -11 */
    double  ms_setup, ms_search, ms_output;   /* device time per stage */
    int64_t launches;          /* kernels this library launched */
    int64_t batch_retries;     /* batches redone at half size after a device allocation failed */
    /* with pfg_options.check_fp32: the FP32 pruning bounds against FP64 (the FP64 values
     * standing in for the exact ones), maxima over every node and candidate of the FP32 pass */
    double  fp32_rem_err;      /* |remaining norm (FP32) - (FP64)|, in units of q */
    double  fp32_margin_frac;  /* that error over the FP32 test's safety margin (slack + en) */
    double  fp32_end_err;      /* |interval endpoint (FP32) - (FP64)|, in coordinate units */
    int64_t fp32_narrower;     /* levels whose FP32 integer range misses part of the FP64 one */
} pfg_stats;

/* pfg_coni_batch with options and statistics (opt, stats may be NULL);
 * dir_nodes, if not NULL, receives (n_p,) search-tree nodes per direction. */
int pfg_coni_batch_ex(const pfg_input *in, const pfg_options *opt, pfg_output *out,
                      pfg_stats *stats, int64_t *dir_nodes);

/* PFVs of a pfg_coni_pfvs call (arrays owned by the library). */
typedef struct {
    int64_t n;                 /* PFVs */
    int64_t *K;                /* (n, pfg_max_h11()) row-major, first h11 entries valid */
    int64_t *M;                /* (n, pfg_max_h11()) */
    int64_t *pidx;             /* (n,) p-vector index */
    int64_t n_points;          /* lattice points the post-processing started from */
    int8_t *pstat;             /* (n_p,) 0 done, < 0 status as pfg_output's */
    double seconds_gpu;
    char err[256];
} pfg_pfv_output;

/* The batched pipeline followed by coniZpM's post-processing on the device:
 * lattice points -> coni PFVs (K, M) exactly as the reference's
 * _pfvs_from_points (pfvs/coni.py:275-412) computes them on the host from
 * pfg_coni_batch's points: the strict GCD cut, the expansion over
 * g = 1 .. (Q gcd(Kn[1:]) - 1) // q and K0, the tadpole check (a violation
 * fails the call, as the reference raises), det((kappa.M)[1:, 1:]) != 0
 * decided exactly, and the reference's order (p-vector, g, point, K0).
 * No counterpart in the reference's C ABI.  M0min (linmin) must be > 0.
 * Returns 0, or 1 with out->err set.  opt and stats may be NULL. */
int pfg_coni_pfvs(const pfg_input *in, const pfg_options *opt, pfg_pfv_output *out, pfg_stats *stats);

/* Free a pfg_pfv_output's arrays (safe on a zeroed struct). */
void pfg_pfv_output_free(pfg_pfv_output *out);

/* Non-coni ZpM on the device (the reference runs it on the CPU only:
 * pfvs/nonconi.py:262-514 with its C setup and kernel): for each p-vector
 * (ps rows hold all h11 entries; p in the Kahler cone), the lattice points c
 * with c^T mat c <= qmax and the non-strict GCD cut g == 0 or Q g >= q,
 * g = gcd(K), K = Z M: Z = kappa . p, Binter a basis of {M in the M-lattice :
 * K . p = 0} LLL-reduced w.r.t. mat = -Binter^T Z Binter (pfl_build with
 * coni = 0, pfvs/fp_kernel/pfv_lattice.h:554-680, then pfv_kernel,
 * pfvs/fp_kernel/fp_kernel.pyx:321-352).  in->Q is the search's Qmax and
 * in->qmax = floor(dilation Qmax); in->linmin is ignored (no M0 cut); the
 * rows are pfg_coni_batch_ex's (M = Binter c, Kn = Z M, q, pidx, canonical
 * order) and the options and statistics too.  h11 <= pfg_max_h11() - 1.
 * Returns 0, or 1 with out->err set. */
int pfg_zpm_batch(const pfg_input *in, const pfg_options *opt, pfg_output *out, pfg_stats *stats,
                  int64_t *dir_nodes);

/* The coni dilation bound of n_p directions p_hat = (0, p_r) of one geometry
 * (kappa, h^3): mu0 = min over nonzero K in Z^(h-1) with p_r . K = 0 of
 * -K^T A_rr^-1 K, A = kappa . p_hat, so that every coni PFV with direction
 * p_hat has dilation below Q / mu0 -- the reference's coni_mu0
 * (pfvs/dilation.py:145, its C path pfvs/fp_kernel/coni_bound.h:255, called
 * in batches by _coni_mu0_batch).  p_r: (n_p, h-1) row-major.  Per
 * direction: status 0 with mu0 = mu_num / mu_den in lowest terms and K
 * ((n_p, h-1)) a minimizer; 1 no bound (A_rr singular, s > 0, or the form
 * not positive definite on the lattice); < 0 not decided on the device (an
 * exact value beyond int128, an ill-conditioned form, the search's node
 * budget).  3 <= h <= 32.  Returns 0, or 1 with err (256 chars, may be NULL)
 * set. */
int pfg_coni_mu0_batch(int h, const int64_t *kappa, int64_t n_p, const int64_t *p_r, int device,
                       int32_t *status, int64_t *mu_num, int64_t *mu_den, int64_t *K, char *err);

/* coniZpK above D0 on the device (the reference computes it on the CPU:
 * pfvs/fp_kernel/coni_zpk.h:714 czk_batch, bound by _coni_zpk_batch,
 * pfvs/fp_kernel/fp_kernel.pyx:434, called by coniZpK, pfvs/coni.py:554):
 * for each coni p-vector (rows of ps, (n_p, h) row-major, p[0] = 0) the
 * lattice points c of its coni PFVs with dilation > D0, as M = Binter c,
 * Kn = (Z Binter) c (rows of pfg_max_h11(), first h entries valid), q =
 * c^T mat c and pidx -- the format of pfg_coni_batch -- and per p-vector a
 * status into `status` ((n_p,)): 0 done; 1 no ZpK for the direction (s >= 0,
 * A_rr singular, or S not positive definite on the lattice orthogonal to
 * p); < 0 not decided here (a value beyond int128 / int64, an
 * ill-conditioned form, more than max_out points, the search's step
 * budget), the reference's codes where it has the same failure.  Points of
 * a p-vector with a nonzero status are not returned (out->pstat stays
 * NULL).  3 <= h <= 32 (the reference's C path: h <= 20).  Returns 0, or 1
 * with out->err set; free with pfg_output_free. */
int pfg_coni_zpk_batch(int h, const int64_t *kappa, const int64_t *Mbasis, int64_t n_p, const int64_t *ps,
                       int64_t Q, int64_t M0min, int64_t D0, int64_t max_out, int device,
                       pfg_output *out, int32_t *status);

/* The same followed by coniZpM's post-processing on the device (as
 * pfg_coni_pfvs; coniZpK applies the same _pfvs_from_points to its points,
 * pfvs/coni.py:613): the PFVs (K, M, pidx) of the points, n_points the
 * points they came from; pstat stays NULL (statuses into `status`).  The
 * PFVs are not yet filtered by dilation > D0 (the reference filters after
 * the post-processing, pfvs/coni.py:629-631).  M0min must be > 0.  Returns
 * 0, or 1 with out->err set; free with pfg_pfv_output_free. */
int pfg_coni_zpk_pfvs(int h, const int64_t *kappa, const int64_t *Mbasis, int64_t n_p, const int64_t *ps,
                      int64_t Q, int64_t M0min, int64_t D0, int64_t max_out, int device,
                      pfg_pfv_output *out, int32_t *status);

/* Test hook (no counterpart in the reference): the k-th device allocation
 * this library makes from now on (k >= 1) fails once with
 * cudaErrorMemoryAllocation, without allocating, so that tests can drive the
 * out-of-memory path of the batch loop; k <= 0 cancels. */
void pfg_debug_fail_alloc(int k);

/*
 * No counterpart in the reference.  The coni pipeline for ONE p-vector,
 * for callers that cannot allocate device memory while they run: code in a
 * framework that owns all device memory through its own pool or arena (an
 * XLA custom call, a TensorRT plugin, an inference server with a fixed
 * memory budget), where a cudaMalloc would go around that pool or fail
 * because the pool holds the memory; or a real-time path that may not block
 * on the allocator.  The call allocates nothing: no cudaMalloc/cudaFree, no
 * host allocation.
 *
 * Inputs (device pointers): kappa (h^3), Mbasis (h^2, basis vectors as
 * columns), p (h entries, p[0] = 0); scalars h (3..64), Q, qmax =
 * floor(dilation Q), linmin = ceil(M0min).  Outputs (device pointers, the
 * caller's): M and Kn (cap x 64 int64, rows as pfg_output's), q (cap),
 * n_out (1 int64: the number of rows) and status (1 int32):
 *    0  done
 *   -2  more than cap or PFG_STATIC_MAX_POINTS points (n_out is then 0)
 *   -22 the search ran past its 120 s deadline
 *   else a status of pfg_output's pstat (-8, -9, -20, -21).
 * The rows are exactly pfg_coni_batch's rows for that p-vector, in the same
 * order.  The whole call runs on ONE warp (no work sharing), so a direction
 * with a large search tree takes far longer than in pfg_coni_batch.  The work
 * is queued on `stream` (a cudaStream_t, or NULL); the outputs are valid once
 * it completes.  Returns 0 when queued, 1 on bad arguments (message on
 * stderr): h outside 3..64, cap outside 0..PFG_STATIC_MAX_POINTS.
 *
 * The scratch (about 3 MB) is a static device array that every GPU loading
 * this library holds until the process exits.  All calls share it: calls
 * that overlap on the GPU (other streams, other host threads) race; issue
 * them one after another.  Each call clears what must start at zero; the
 * array otherwise keeps the last call's contents.  The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress) with
 * that device current and keeps it for the process; make that first call
 * before any stream capture.  After cudaDeviceReset the kept address is
 * stale: do not call this entry point in a process that has reset a device
 * it used.
 */
#define PFG_STATIC_MAX_POINTS 2048
int pfg_coni_direction_static(int h, int64_t Q, int64_t qmax, int64_t linmin,
                              const int64_t *kappa, const int64_t *Mbasis, const int64_t *p,
                              int64_t cap, int64_t *M, int64_t *Kn, int64_t *q,
                              int64_t *n_out, int32_t *status, void *stream);

#ifdef __cplusplus
}
#endif

#endif
