/*
 * fln.h — C ABI of the B200 linking-number engine (libfln.so).
 *
 * This is the drop-in boundary for the hot path of antequ/fastlinkingnumbers
 * (`verifycurves`): the Gauss linking integral over every potentially linked
 * loop pair, by direct summation or two-tree Barnes–Hut, plus the host stages
 * that feed it (BCC loading, potential-link search, Discretize) and the
 * certificate built from it. Plain C types only: pointers, sizes, enums.
 * Every entry point returns an fln_status and never throws; on failure
 * fln_last_error() describes the cause (thread-local).
 *
 * Each declaration names the reference interface (file:line in
 * antequ/fastlinkingnumbers) it replaces.
 */
#ifndef FLN_H_
#define FLN_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FLN_ABI_VERSION 3

typedef enum fln_status {
  FLN_OK = 0,
  FLN_ERR_INVALID_ARGUMENT = 1,
  FLN_ERR_IO = 2,              /* file open / short read / write (model.cpp:284-356) */
  FLN_ERR_FORMAT = 3,          /* bad BCC header, type or counts (model.cpp:294-328) */
  FLN_ERR_CUDA = 4,            /* a CUDA runtime call failed */
  FLN_ERR_NO_DEVICE = 5,       /* no CUDA device visible */
  FLN_ERR_OUT_OF_MEMORY = 6,
  FLN_ERR_SEGMENT_TOO_SMALL = 7, /* Discretize: piece < eps * avg coordinate (discretize.cpp:151-160, 219-229) */
  FLN_ERR_MAX_RECURSION = 8,   /* Discretize: more than 55 rounds (discretize.cpp:248-253) */
  FLN_ERR_UNLOOPED = 9,        /* an open curve reached the linking-number stage (curve.cpp:126-128) */
  FLN_ERR_NONFINITE = 10,      /* a pair stayed NaN/inf after the FP64 recompute (lnc.cpp:206-211) */
  FLN_ERR_STACK_OVERFLOW = 11, /* a Barnes–Hut traversal stack exceeded its bound */
  FLN_ERR_TIMEOUT = 12,        /* a bounded device wait ran out */
  FLN_ERR_INTERNAL = 13
} fln_status;

typedef enum fln_method {
  FLN_METHOD_DIRECTSUM = 0, /* --method directsum  (lnc.cpp:241-338) */
  FLN_METHOD_BARNESHUT = 1  /* --method barneshut  (lnc.cpp:102-229) */
} fln_method;

typedef enum fln_precision {
  FLN_PREC_FP64 = 0,  /* every term in FP64: the plain FP64 GPU path */
  FLN_PREC_MIXED = 1  /* FP32 terms, FP64 near-singular terms and per-pair sums, FP64 recompute below margin */
} fln_precision;

typedef enum fln_seg_type {
  FLN_SEG_BSPLINE = 0,    /* BCC "BS" (curve.cpp:20-29) */
  FLN_SEG_CATMULLROM = 1, /* BCC "C0" (curve.cpp:31-36) */
  FLN_SEG_BEZIER = 2,     /* BCC "BZ" (curve.cpp:38-43) */
  FLN_SEG_POLYLINE = 3    /* BCC "PL" */
} fln_seg_type;

/* Per-pair result flags (bit set). */
enum {
  FLN_PAIR_FP64_RECOMPUTED = 1, /* margin below threshold or non-finite: recomputed in FP64 direct sum */
  FLN_PAIR_BETA_RETRIED = 2,    /* Barnes–Hut re-run with the larger beta (lnc.cpp:165-184) */
  FLN_PAIR_NONFINITE = 4,       /* still non-finite after the recompute */
  FLN_PAIR_SWAPPED = 8,         /* evaluated with the loops' roles exchanged (symmetric) */
  FLN_PAIR_BETA_ESCALATED = 16  /* Barnes–Hut re-run with a beta beyond the reference's rule */
};

typedef struct fln_params {
  double barnes_hut_init_beta;  /* 2.0  (define_args.h:50-51) */
  double barnes_hut_beta_limit; /* 10.0 (define_args.h:53-54) */
  double epssq;                 /* 1e-24 CERTIFICATE_EPSSQ (lnc.cpp:24) */
  double target_error;          /* 0.1   TARGET_ERROR (lnc.cpp:25) */
  double error_est_scale;       /* 0.05  ERROR_EST_SCALE (lnc.cpp:26) */
  int32_t precision;            /* fln_precision; default FLN_PREC_MIXED */
  double fp64_margin;           /* recompute in FP64 when 0.5 - |lk - round(lk)| < this; default 0.25 */
  double near_factor;           /* mixed direct sum: a segment pair whose closest endpoint distance is
                                   below near_factor * (longer segment length) is evaluated in FP64; 4.0 */
  int32_t bh_tree;              /* Barnes–Hut tree: 0 = curve-order tree (default), 1 = the reference's
                                   kd-median tree (ModifiedKdBVH.h:207-237) */
  int32_t bh_escalations;       /* after the reference's retry, a pair whose scaled error estimate is still
                                   above bh_err_limit is re-run with twice its beta, up to this many times;
                                   default 2 (0 = the reference's behaviour) */
  double bh_err_limit;          /* default 0.25; a pair still above it is recomputed by FP64 direct sum */
  int32_t bh_schedule;          /* 0 = budgeted rounds, evaluation inside the traversal (default);
                                   1 = one persistent launch with a device work queue;
                                   2 = budgeted rounds, evaluation in separate streaming kernels */
  int32_t host_prepare;         /* fln_certificate_compute: 0 = Discretize and the potential-link searches
                                   on the context's GPU (default), 1 = on the host; same output bit for bit */
  int32_t bh_budget;            /* traversal steps a warp spends on a batch per launch before handing the
                                   rest on; 0 = 128. The node pairs stay the same; only the grouping of
                                   the FP64 partial sums changes (last-bit differences). */
  int32_t bh_bucket;            /* curve-order trees, bh_schedule 0: a node pair that is neither far nor a
                                   leaf pair and has at most this many segments a side is summed exactly,
                                   segment pair by segment pair; 0 = 8, 1 = leaf pairs only (the
                                   reference's traversal), at most 16 */
  int32_t bh_retry_from_roots;  /* 0 (default): bh_schedule 0 continues the beta retry from the first pass's
                                   far node pairs (a node pair opened at beta0 is opened at the larger beta,
                                   an exact one stays exact, so the node pairs and the sums are those of a
                                   run from the roots); 1: the retry re-runs from the roots, as
                                   lnc.cpp:165-184 does */
  int32_t bh_spill_cap;         /* global spill entries per warp of the traversal stacks; 0 = 8192, the
                                   maximum. A traversal that needs more fails with FLN_ERR_STACK_OVERFLOW
                                   (bh_schedule 0 and 1); smaller values exist to test that bound */
  int64_t bh_wait_polls;        /* bh_schedule 1: polls (with a nanosleep back-off of up to 2 us) before
                                   a waiting warp gives up, after which the stage reruns with budgeted
                                   rounds (fln_stats.bh_wait_timeouts); 0 = 2^21, a few seconds; smaller
                                   values exist to test that path */
  int32_t direct_tile;          /* direct sum tile shape (curve-1 segments per item x curve-2 vertices per
                                   shared-memory tile): 0 = 128 x 256 (default), 1 = 128 x 128,
                                   2 = 128 x 512, 3 = 256 x 256, 4 = 256 x 512, 5 = 64 x 256; chosen by
                                   fln_autotune_direct. Sums change only in their rounding. */
  int32_t bh_occupancy;         /* CTAs per SM of the Barnes-Hut traversal kernels: 0 = 5 (96 registers),
                                   5, 6 (80 registers) or 7 (72, some spills); more resident warps hide more of
                                   the traversal's dependent loads. Chosen by fln_autotune; results do not change */
  int32_t bh_exact_serial;      /* bh_schedule 0: 0 = each round's exact list runs on a second stream beside
                                   the next round's traversal (default); 1 = on the context's stream after
                                   its traversal, so that each kernel's CUDA-event time is its own (for
                                   measuring; results are the same bit for bit) */
  int32_t reserved_int;         /* zero */
  double reserved_params[3];    /* zero */
} fln_params;

/* Statistics of the last computation on a context. */
typedef struct fln_stats {
  int64_t pairs;                /* loop pairs evaluated */
  double segment_pairs;         /* sum over pairs of n_i * n_j (direct-sum-equivalent work) */
  int64_t fp64_recomputed;      /* pairs recomputed in FP64 */
  int64_t beta_retried;         /* Barnes–Hut pairs re-run with a larger beta */
  double bh_far_evals;          /* Barnes–Hut far-field node pairs evaluated */
  double bh_leaf_evals;         /* Barnes–Hut segment pairs summed exactly (leaf pairs and the segment
                                   pairs of small node pairs, see bh_bucket) */
  double near_fp64_terms;       /* mixed direct sum: segment pairs evaluated in FP64 */
  double ms_kernels;            /* device time of the linking-number kernels (CUDA events) */
  double ms_total;              /* wall time of the last call */
  double ms_discretize;         /* host Discretize + potential-link search (certificate calls) */
  double mean_off_integer, max_off_integer; /* lnc.cpp:216-225 */
  int32_t discretize_rounds;
  int32_t kernel_launches;      /* kernels launched by the last call */
  double ms_main_kernel;        /* device time of the dominant kernel(s): the Barnes–Hut traversal or the
                                   direct-sum kernel (CUDA events on the launching stream) */
  double ms_tree_build;         /* Barnes–Hut tree topology + FP64 moment build */
  int32_t bh_rounds;            /* Barnes–Hut traversal launches (work is handed on between rounds) */
  int32_t reserved_stats;
  int64_t bh_escalated;         /* pair re-runs with an escalated beta */
  int64_t bh_wait_timeouts;     /* persistent traversals that fell back to rounds */
  double ms_exact;              /* Barnes–Hut: device time of the exact-list kernel (part of ms_main_kernel) */
  double bh_exact_entries;      /* Barnes–Hut: node pairs summed exactly (leaf pairs and small node pairs);
                                   bh_leaf_evals counts their segment pairs */
  double ms_retry;              /* Barnes–Hut: device time of the beta retry and escalation passes (part of
                                   ms_main_kernel) */
  int64_t bh_front_records;     /* Barnes–Hut: frontier records (up to 128 far node pairs each) written by
                                   the first pass for the retry to continue from */
  int64_t bh_retry_from_roots;  /* Barnes–Hut: retried pairs that restarted from the roots (frontier not
                                   kept for them, or bh_retry_from_roots set) */
  double bh_far_reused;         /* Barnes–Hut: frontier node pairs still far at the retry's beta, whose
                                   first-pass values were kept (not evaluated again) */
  double bh_far_subtracted;     /* Barnes–Hut: frontier node pairs opened by the retry, whose first-pass
                                   values were given back */
  double ms_traverse;           /* Barnes–Hut bh_schedule 0: device time of the traversal launches (CUDA
                                   events on the launching stream; the exact-list launches run beside them
                                   on a second stream, so ms_traverse + ms_exact can exceed
                                   ms_main_kernel) */
  double reserved_stats2[1];
} fln_stats;

typedef struct fln_ctx fln_ctx;
typedef struct fln_model fln_model;
typedef struct fln_certificate fln_certificate;

const char *fln_status_string(fln_status s);
const char *fln_last_error(void);
int fln_abi_version(void);
void fln_default_params(fln_params *p);

/* Context: one CUDA device and one stream; owns all device buffers.
 * stream = 0 creates a private stream; otherwise the given cudaStream_t
 * (as an opaque pointer) is used and not destroyed. The context also keeps
 * two internal streams (the pieces of a pinned vertex copy; the Barnes-Hut
 * exact-list launches), joined back to `stream` by events before a call's
 * results are read, so work queued on `stream` after a call sees them. */
fln_status fln_ctx_create(int device, void *stream, fln_ctx **out);
void fln_ctx_destroy(fln_ctx *ctx);
fln_status fln_ctx_stats(const fln_ctx *ctx, fln_stats *out);

/* ---- Kernel-level batched API: replaces the per-pair calls of
 * compute_link.h:62-87 (ComputeLinkingNumberDirectOneArctanPerPair,
 * ComputeLinkingNumberDirectFast) and :95-181 (MakeSegmentTrees,
 * BuildTreeMoments, EvalLinkingNumberBarnesHut) with the per-pair driver
 * loops of linking_number_certificate.cpp:102-229 and :241-338.
 *
 * Closed polylines: loop l owns vertices [loop_offsets[l], loop_offsets[l+1])
 * of xyz (3 doubles per vertex); segment k runs from vertex k to k+1 (mod n).
 * pairs holds npairs (i, j) loop-index pairs. Outputs (any may be NULL
 * except lk_out): lk_out[p] the real-valued linking number, err_out[p] the
 * Barnes–Hut error estimate after ERROR_EST_SCALE (0 for direct sum),
 * flags_out[p] FLN_PAIR_* bits. Host pointers; copies are done inside. */
fln_status fln_linking_numbers(fln_ctx *ctx, const double *xyz, const int64_t *loop_offsets,
                               int32_t nloops, const int32_t *pairs, int64_t npairs,
                               fln_method method, const fln_params *params, double *lk_out,
                               double *err_out, int32_t *flags_out);

/* The same with every array already in device memory (the ctx's device). */
fln_status fln_linking_numbers_device(fln_ctx *ctx, const double *d_xyz,
                                      const int64_t *d_loop_offsets, int32_t nloops,
                                      const int32_t *d_pairs, int64_t npairs, fln_method method,
                                      const fln_params *params, double *d_lk_out,
                                      double *d_err_out, int32_t *d_flags_out);

/* Direct sum that allocates no memory. No counterpart in the reference.
 * For callers that cannot call cudaMalloc — code running while another
 * framework owns the device's memory pool, latency-critical loops that must
 * not take allocator locks, or paths where an allocation failure cannot be
 * handled. Every array is the caller's device memory; the only other memory
 * used is one fixed device array inside libfln.so (about 9.3 MB per GPU,
 * held until the process exits). Limits: npairs <= 65536 and at most 2^20
 * work items (one item = 128 segments of the longer loop of a pair, summed
 * over pairs); larger calls return FLN_ERR_INVALID_ARGUMENT. precision is
 * FLN_PREC_FP64 or FLN_PREC_MIXED; the results are the raw sums of that
 * precision (no margin recompute), the mixed one with the default
 * near_factor, 4.0, so they equal those of fln_linking_numbers_device with
 * the same precision and fp64_margin = 0. Work is queued on `stream` (a
 * cudaStream_t, NULL = default stream) of the current device. Every call
 * reads the plan's size and status back to the host, so it blocks the
 * calling thread until the work queued earlier on `stream` and a small
 * planning kernel have finished; it returns with the sums still in flight
 * on `stream`. Because every call waits on the host, no call can be
 * captured into a CUDA graph (capture the surrounding work around it
 * instead). Calls share the array: calls whose work overlaps on the GPU
 * race, so issue them one at a time. */
fln_status fln_linking_numbers_direct_noalloc(const double *d_xyz, const int64_t *d_loop_offsets,
                                              int32_t nloops, const int32_t *d_pairs, int64_t npairs,
                                              int32_t precision, double *d_lk_out, void *stream);

/* ---- Learned opening criterion for Barnes–Hut. No counterpart in the
 * reference, whose traversal opens a node pair exactly when
 * |dr|^2 + eps^2 <= beta^2 (r1 + r2)^2 + eps^2 (compute_link.cpp:573-574, :608).
 *
 * A small MLP (8 -> 64 -> 64 -> 1, ReLU; BF16 weights, FP32 accumulation)
 * predicts log10 of the true far-field error of a node pair from its
 * separation s = |dr| / (r1 + r2), the radius ratio and the moment norms.
 * With a model set on a context (fln_ctx_set_learned), the traversal accepts
 * as far-field a pair the beta test would open when s >= s_min and the
 * prediction is below log10_tau (tau scaled by (beta0 / beta)^4 in the retry
 * and escalation passes); such a pair adds its Eq. 14 estimate to the error
 * sum like any far-field pair, so the beta retry, the escalation, the margin
 * check and the FP64 recompute keep their meaning and certificates keep
 * their guarantees; only the set of evaluated node pairs changes.
 * Barnes–Hut with bh_schedule 0 only (other schedules return
 * FLN_ERR_INVALID_ARGUMENT while a model is set).
 *
 * Training (fln_learned_train): one Barnes–Hut run over the given loops
 * records node pairs with s in [s_min, 1.25 beta0]; each gets its features
 * and its true error against the FP64 exact sum over the two nodes' segment
 * ranges; the MLP is fitted by our own forward/backward and Adam kernels
 * under the pinball loss at `quantile` (an upper-quantile regression, so the
 * prediction errs high); tau is the tau_quantile of the true errors of the
 * recorded far-field pairs the beta test accepts (s in [beta0, 1.25 beta0]). */
#define FLN_MLP_PARAMS 4801 /* W1[8][64], b1[64], W2[64][64], b2[64], w3[64], b3 (FP32) */

typedef struct fln_learned_options {
  double s_min;           /* 1.5 */
  double sample_keep;     /* fraction of the candidate node pairs recorded: 0.05 */
  int64_t max_samples;    /* 1 << 20 */
  int64_t max_terms;      /* samples whose ranges hold more segment pairs are dropped: 1 << 16 */
  int32_t epochs;         /* 40 */
  int32_t batch;          /* 4096 */
  double learning_rate;   /* 2e-3, cosine decay */
  double quantile;        /* 0.9 */
  double tau_quantile;    /* 0.5 */
  double val_fraction;    /* held-out share of the samples: 0.1 */
  int32_t min_candidates; /* the MLP runs for a warp step with at least this many candidates: 4 */
  int32_t min_node_segments; /* only node pairs whose smaller node holds at least this many segments are
                                candidates (where accepting a pair saves a subtree); 0 = every node */
  uint64_t seed;          /* 1 */
  double reserved[4];
} fln_learned_options;

typedef struct fln_learned_info {
  int64_t recorded;       /* node pairs recorded by the traversal */
  int64_t samples;        /* of them with an exact target */
  int64_t train_samples, val_samples;
  double s_min, log10_tau;
  int32_t min_candidates, epochs;
  double train_loss, val_loss; /* pinball loss */
  double val_coverage;    /* share of held-out samples whose true log10 error is <= the prediction */
  double ms_collect, ms_train;
  int32_t min_node_segments;
  int32_t reserved_i;
  double reserved[3];
} fln_learned_info;

typedef struct fln_learned fln_learned;

void fln_learned_default_options(fln_learned_options *o);
fln_status fln_learned_train(fln_ctx *ctx, const double *xyz, const int64_t *loop_offsets, int32_t nloops,
                             const int32_t *pairs, int64_t npairs, const fln_params *params,
                             const fln_learned_options *options, fln_learned **out);
/* A model from saved parameters (FLN_MLP_PARAMS floats). */
fln_status fln_learned_create(const float *params, double s_min, double log10_tau, int32_t min_candidates,
                              fln_learned **out);
void fln_learned_destroy(fln_learned *m);
/* Changes when the model runs in the traversal (see fln_learned_options:
 * min_candidates >= 1, min_node_segments >= 0); takes effect at the next
 * fln_ctx_set_learned. */
fln_status fln_learned_configure(fln_learned *m, int32_t min_candidates, int32_t min_node_segments);
/* Either output may be NULL. */
fln_status fln_learned_get(const fln_learned *m, float *params_out, fln_learned_info *info_out);
/* NULL turns the criterion off. The context keeps its own device copy. */
fln_status fln_ctx_set_learned(fln_ctx *ctx, const fln_learned *m);
/* Training samples as fln_learned_train records them: up to `cap` rows of
 * features_out[8 * k], target_out[k] (log10 true error), sep_out[k] (the
 * separation s) and est_out[k] (log10 of the Eq. 14 error estimate times
 * error_est_scale, the reference's measure); sep_out and est_out may be NULL.
 * *n_out gets the number written. */
fln_status fln_learned_collect(fln_ctx *ctx, const double *xyz, const int64_t *loop_offsets, int32_t nloops,
                               const int32_t *pairs, int64_t npairs, const fln_params *params, double s_min,
                               double sample_keep, int64_t cap, int64_t max_terms, float *features_out,
                               float *target_out, float *sep_out, float *est_out, int64_t *n_out);
/* MLP outputs for n feature rows: FP32 (use_mma = 0) or the traversal's BF16
 * warp-MMA path (use_mma = 1). */
fln_status fln_learned_predict(fln_ctx *ctx, const float *params, const float *features, int64_t n,
                               int32_t use_mma, float *y_out);
/* Mean pinball loss at `quantile` over n rows and its gradient with respect
 * to the FLN_MLP_PARAMS parameters (the training kernel's backward pass). */
fln_status fln_learned_gradients(fln_ctx *ctx, const float *params, const float *features,
                                 const float *targets, int64_t n, double quantile, float *grad_out,
                                 double *loss_out);

/* ---- Autotuner of the Barnes–Hut stage. No counterpart in the reference.
 * Times the stage (tree build, traversal, retry, escalation, margin check)
 * on a seeded sample of the given pairs, `sample_pairs` of them (0 = 2048;
 * all pairs when there are fewer), for each traversal round budget
 * {128, 256, 512}; with bit 0 of tune_beta, also each initial beta
 * {1.5, 2, 2.5, 3}; then the traversal occupancies 6 and 7 CTAs per SM
 * (fln_params.bh_occupancy) at the best setting; with bit 1 (curve-order
 * trees), then the exact-bucket sizes {4, 6, 10, 12, 16} around it. Beta and the bucket
 * change the real sums within the Barnes-Hut error, never the certificate;
 * the budget changes only their rounding. A setting replaces the best so
 * far only when it is more than 1.5 % faster (timing noise does not choose
 * between ties). *out gets *params with the fastest setting (its budget
 * named explicitly); *result the sample times (device time, best of three
 * runs each). */
typedef struct fln_tune_result {
  double best_ms;     /* sample time of the chosen setting */
  double default_ms;  /* sample time of *params as given */
  int32_t trials;     /* settings timed */
  int32_t sample_pairs;
  int32_t best_budget;
  int32_t best_direct_tile;  /* fln_autotune_direct */
  double best_beta;
  int32_t best_bucket;
  int32_t best_occupancy;
  double reserved[2];
} fln_tune_result;

fln_status fln_autotune(fln_ctx *ctx, const double *xyz, const int64_t *loop_offsets, int32_t nloops,
                        const int32_t *pairs, int64_t npairs, const fln_params *params, int32_t tune_beta,
                        int64_t sample_pairs, fln_params *out, fln_tune_result *result);

/* Autotuner of the direct sum. No counterpart in the reference. Times the
 * direct sum (params->precision, with its margin check) on a seeded sample
 * of the pairs (sample_pairs, 0 = 2048) for each tile shape of
 * fln_params.direct_tile (device time, best of two runs); *out gets *params
 * with the fastest shape, result->best_direct_tile the shape. */
fln_status fln_autotune_direct(fln_ctx *ctx, const double *xyz, const int64_t *loop_offsets, int32_t nloops,
                               const int32_t *pairs, int64_t npairs, const fln_params *params, int64_t sample_pairs,
                               fln_params *out, fln_tune_result *result);

/* One pair, host arrays (compute_link.h:62-64 and :86-87). */
fln_status fln_direct_pair(fln_ctx *ctx, const double *xyz1, int64_t n1, const double *xyz2,
                           int64_t n2, int32_t precision, double *lk_out);

/* ---- Models (model.h:24-75, curve.h:41-195) */
fln_status fln_model_create(fln_model **out);
void fln_model_destroy(fln_model *m);
/* Model::ImportFromFile / ImportBccFile (model.cpp:44-54, :280-364). */
fln_status fln_model_load_bcc(fln_model *m, const char *path);
/* Model::ExportToFile / ExportBccFile (model.cpp:61-71, :367-452). */
fln_status fln_model_save_bcc(const fln_model *m, const char *path);
/* Replace the curves: counts[c] control points (negative = closed loop, the
 * BCC convention), xyz packed 3 doubles per point, one segment type. */
fln_status fln_model_set_curves(fln_model *m, fln_seg_type type, int32_t ncurves,
                                const int32_t *counts, const double *xyz);
int32_t fln_model_num_curves(const fln_model *m);
int64_t fln_model_num_points(const fln_model *m);
/* counts_out[ncurves] (negative = loop), xyz_out[3 * num_points]. */
fln_status fln_model_get_curves(const fln_model *m, int32_t *type_out, int32_t *counts_out,
                                double *xyz_out);

/* ---- Host stages feeding the kernels.
 * PotentialLinkSearch + Discretize + unique PLS (lnc.cpp:61-83;
 * discretize.cpp:103-281; potential_link_search.cpp:88-165): writes the
 * discretized closed polylines and the sorted unique (i < j) pairs into
 * buffers owned by the model (read them with fln_model_get_prepared). */
fln_status fln_model_prepare(fln_model *m, int discretize, int32_t *rounds_out);
/* The same stages with Discretize and both potential-link searches on the
 * context's GPU: bit-identical polylines, pairs and round count (the piece
 * boxes use the host's arithmetic with no fused multiply-add). */
fln_status fln_model_prepare_device(fln_ctx *ctx, fln_model *m, int discretize, int32_t *rounds_out);
fln_status fln_model_prepared_sizes(const fln_model *m, int64_t *num_vertices, int64_t *num_pairs);
fln_status fln_model_get_prepared(const fln_model *m, int64_t *loop_offsets_out, double *xyz_out,
                                  int32_t *pairs_out);

/* ---- Certificates (linking_number_certificate.h:25-131) */
/* LinkingNumberCertificate::ComputeFromModel (lnc.cpp:358-394). */
fln_status fln_certificate_compute(fln_ctx *ctx, const fln_model *m, int force_direct_sum,
                                   int discretize, const fln_params *params,
                                   fln_certificate **out);
/* LinkingNumberCertificate(filename) / ImportFromFile / ReadMatrix (lnc.cpp:43-46, :402-430). */
fln_status fln_certificate_load(const char *path, fln_certificate **out);
void fln_certificate_destroy(fln_certificate *c);
/* ExportToFile / SaveMatrix (lnc.cpp:441-454, :484-486). */
fln_status fln_certificate_save(const fln_certificate *c, const char *path);
/* The certificate text; returns its length (writes at most cap-1 bytes + NUL when buf != NULL). */
int64_t fln_certificate_text(const fln_certificate *c, char *buf, int64_t cap);
int32_t fln_certificate_num_curves(const fln_certificate *c);
int64_t fln_certificate_num_entries(const fln_certificate *c);
/* entries_out[3 * k] = (i, j, lk) with i < j, sorted by (i, j). */
fln_status fln_certificate_entries(const fln_certificate *c, int32_t *entries_out);
/* Per potential pair of the last compute: (i, j), real sum, error estimate, flags. */
int64_t fln_certificate_num_pairs(const fln_certificate *c);
fln_status fln_certificate_pairs(const fln_certificate *c, int32_t *pairs_out, double *lk_out,
                                 double *err_out, int32_t *flags_out);
/* Equals / operator== (linking_number_certificate.h:117-128): 1 if equal. */
int fln_certificate_equals(const fln_certificate *a, const fln_certificate *b);
/* ExportDiffsToFiles (lnc.cpp:520-561); a NULL path or "[none]" skips that file. */
fln_status fln_certificate_export_diffs(const fln_certificate *self, const fln_certificate *other,
                                        const char *diff_pairs_path, const char *diff_curves_path);

#ifdef __cplusplus
}
#endif
#endif /* FLN_H_ */
