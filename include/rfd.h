/*
 * rfd.h - C ABI of the B200 continuous Frechet distance engine (librfd.so).
 *
 * Curves are caller-owned arrays of doubles in interleaved [n][dims] layout
 * (dims 2 or 3), the same flattening the reference performs in
 * Cuda_intersection::Cuda_intersection (src/intersection_algorithm_in_parallel.cu:42-51).
 * Every function returns an rfd_status code; nothing prints.  A context owns one
 * CUDA device, one stream and a cached device workspace; calls on one context
 * are serialised by the caller, distinct contexts may be used from distinct
 * threads.
 */
#ifndef RFD_H
#define RFD_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RFD_ABI_VERSION 1
#define RFD_MAX_ARITY 8    /* rfd_options.search_arity */
#define RFD_ARITY_PAIRS 32 /* pairs per call that get k-ary rounds */
#define RFD_MAX_PROBES 200

/* Status codes (the reference prints CUDA errors and carries on; this ABI reports them). */
enum rfd_status {
  RFD_OK = 0,
  RFD_ERR_ARG = 1,      /* null pointer, dims not 2/3, empty curve, bad option */
  RFD_ERR_CUDA = 2,     /* a CUDA runtime call failed (message: rfd_last_error) */
  RFD_ERR_NOMEM = 3,    /* device or pinned host allocation failed */
  RFD_ERR_TIMEOUT = 4,  /* a bounded inter-warp wait expired; results are not valid */
  RFD_ERR_NODEV = 5,    /* no CUDA device, or the library was built without one */
  RFD_ERR_INTERNAL = 6,
  RFD_ERR_LIMIT = 7     /* a size exceeds a stated maximum */
};

/* Stop rule of the epsilon search. */
enum rfd_stop {
  RFD_STOP_ABS = 0, /* while (ub - lb > tol): the reference rule, tol = FLT_EPSILON
                       (src/frechet.cpp:41, src/compute_distance_wrapper.cpp:6) */
  RFD_STOP_REL = 1  /* while (ub - lb > tol * ub): relative rule for the 1e-9 metric */
};

enum rfd_memory { RFD_MEM_HOST = 0, RFD_MEM_DEVICE = 1 };

/* Free intervals of the decision.  The reference has two decision paths and picks one per
   solve by free device memory (src/intersection_algorithm_in_parallel.cu:87-97): the
   materialised one when 4 (n1-1)(n1+n2-4) doubles of intervals fit, else the fused
   ("oversize") kernel.  They round C of the free-interval quadratic differently
   (interval_calculation .cu:742 forms (sum mi^2) - r^2; reachable .cu:1177-1186 starts the sum
   at -r^2), so a decision within a few ulps of the distance can differ between them. */
enum rfd_formula {
  RFD_FORMULA_FUSED = 0,         /* reachable<d> (.cu:960-1256), forceOversize's path */
  RFD_FORMULA_MATERIALISED = 1,  /* interval_calculation<d> + reachability (.cu:673-958) */
  RFD_FORMULA_REFERENCE = 2      /* per pair, the reference's choice on this device's free
                                    memory at call time (its rule, .cu:92) */
};

enum rfd_precision {
  RFD_PREC_FP64 = 0,       /* every interval in FP64 */
  RFD_PREC_FP32_FILTER = 1 /* FP32 classification with a proven margin, FP64 recheck */
};

/* Result flags. */
enum rfd_flag {
  RFD_FLAG_VEFD_SKIPPED = 1,   /* reference quirk: (int)(n1*n2) <= 10000, lb = endpoint bound */
  RFD_FLAG_LB_GT_UB = 2,       /* VE-FD came out above DFD (the reference asserts here) */
  RFD_FLAG_MAX_PROBES = 4,     /* stopped by max_probes */
  RFD_FLAG_STALLED = 8,        /* (lb+ub)/2 equals lb or ub: no further progress in doubles */
  RFD_FLAG_VEFD_DENSE = 16,    /* VE-FD pruning bound was too tight, recomputed without pruning */
  RFD_FLAG_BRACKET_USED = 32,  /* a proposed bracket was verified and used */
  RFD_FLAG_BRACKET_WIDENED = 64, /* a proposed bracket failed verification and was widened */
  RFD_FLAG_DEGENERATE = 128,   /* a curve of one point: closed form used */
  RFD_FLAG_DFD_COARSE = 256    /* dfd holds the coarse upper bound (rfd_options.coarse_ub) */
};

typedef struct rfd_model rfd_model;

typedef struct rfd_options {
  int32_t stop_mode;        /* enum rfd_stop */
  int32_t reference_quirks; /* 1: reproduce the reference's VE-FD launch rule
                               (src/intersection_algorithm_in_parallel.cu:1343) */
  double tol;               /* see rfd_stop */
  int32_t max_probes;       /* cap on decisions per pair, <= RFD_MAX_PROBES */
  int32_t dense;            /* 1: evaluate every cell (no dead-region skipping) */
  int32_t precision;        /* enum rfd_precision */
  int32_t memory;           /* where curve pointers live: enum rfd_memory */
  const double* bracket;    /* optional, 2 doubles per pair: proposed [lo, hi] containing the
                               distance; verified by two decisions, widened on failure */
  const rfd_model* model;   /* optional learned bracket: proposes [lo, hi] per pair from the
                               curves and the VE-FD bound (ignored when bracket is set) */
  int32_t coarse_ub;        /* 0: the DFD is the upper bound (the reference's method).  k in
                               [2, 4096] (needs reference_quirks = 0): the upper bound is the DFD of
                               every k-th point and the last, each cell weighted by the distance
                               plus both points' inflations (an anchor's inflation: the largest
                               distance to it of the half-blocks it covers, the suffix of the block
                               before it and the prefix of the block after it): a certified bound
                               on the DFD from k*k times fewer cells.  result.dfd then holds that
                               bound (RFD_FLAG_DFD_COARSE).  The FD, within the stop rule, does
                               not depend on it. */
  int32_t drop_repeats;     /* 1: drop consecutive repeated points (all coordinates equal) from
                               both curves before the solve (device-memory curves are counted
                               and compacted on the device, with one read-back of the counts
                               before the call's launches).  The Frechet
                               distance does not change in exact arithmetic, but the reference's
                               free interval of a zero-length segment is [0, 1] at every radius
                               (src/intersection_algorithm_in_parallel.cu:1186-1198: 0 * inf is
                               NaN, which max / min clamp to the whole edge), so a repeated point
                               can make its decisions, and the distance, too small.  The
                               reference's text loaders drop such points (include/txtReader.hpp:
                               36-41); this applies the same rule to curves built in code.
                               0 (default) keeps the reference's behaviour. */
  int32_t graph;            /* 1: capture the call's device work (copies, launches, read-back)
                               as one CUDA graph and keep it in the context; a later call with
                               the same layout (pair sizes, options, workspace, stream) replays
                               it instead of issuing each launch.  Results are identical. */
  int32_t formula;          /* enum rfd_formula, default RFD_FORMULA_FUSED.  The FP32 filter
                               certifies the fused intervals only: it needs RFD_FORMULA_FUSED. */
  int32_t search_arity;     /* 0 or 1 (default): every probe is one decision at the bisection's
                               midpoint (the reference's search, src/frechet.cpp:36-63).  K in
                               [2, RFD_MAX_ARITY]: the pairs whose probe chains are longest (up to
                               RFD_ARITY_PAIRS per call, within a quarter of the free device
                               memory) get K - 1 extra decision workspaces, and once few pairs
                               remain (at most the teams / (2K), or RFD_ARITY_GATE; a single
                               pair always) each of their bisection rounds
                               decides K radii at once, splitting the bracket into K + 1 parts
                               (about log2(K + 1) halvings per round instead of one).  Only the
                               probe sequence changes: every decision is the same function of its
                               radius, the stop rule is the same, and result.probes counts every
                               decision. */
} rfd_options;

typedef struct rfd_result {
  double distance;          /* (lb + ub) / 2 at the stop (src/frechet.cpp:63) */
  double dfd;               /* discrete Frechet distance: the initial upper bound */
  double vefd;              /* vertex-edge Frechet distance: the initial lower bound */
  double endpoint;          /* max(|p0 - q0|, |pn - qm|) (src/frechet.cpp:30) */
  double lb, ub;            /* final bracket */
  int64_t cells_nominal;    /* sum over decisions of (n1-1)(n2-1) */
  int64_t cells_evaluated;  /* decision cells the kernels actually evaluated (includes
                               speculative tiles, so it varies slightly from run to run) */
  int64_t cells_fp64;       /* of those, cells whose intervals were computed in FP64 */
  int64_t cells_vefd;       /* VE-FD cells evaluated (of (n1-1)(n2-1) per pass) */
  int32_t probes;           /* decisions made */
  int32_t flags;            /* enum rfd_flag */
} rfd_result;

typedef struct rfd_context rfd_context;

/* ---- library ---- */
int32_t rfd_abi_version(void);
const char* rfd_status_string(int32_t status);
/* Message of the last failing call on this thread ("" when none). */
const char* rfd_last_error(void);

/* Options of the reference (ABS stop at FLT_EPSILON, quirks on) when precise == 0,
   else the relative rule at tol = 2^-33 with quirks off. */
void rfd_options_init(rfd_options* opt, int32_t precise);

/* ---- context ---- */
int32_t rfd_context_create(int32_t device, rfd_context** out);
int32_t rfd_context_destroy(rfd_context* ctx);
/* Budget of every bounded wait of the context's kernels (a strip waiting for the strip above
   it, a helper warp for its request, the continuous search for a queue entry), in SM clock
   cycles; cycles <= 0 restores the default of about 20 s at the maximum SM clock.  A wait that
   runs out sets an error word, every warp leaves, and the call returns RFD_ERR_TIMEOUT; the next
   call starts afresh.  The environment variable RFD_SPIN_CYCLES sets the initial budget of new
   contexts and the budget of rfd_decide_noalloc.  (The reference's spin-waits are unbounded,
   src/intersection_algorithm_in_parallel.cu:304-306, :332-334.) */
int32_t rfd_context_set_wait_budget(rfd_context* ctx, int64_t cycles);
/* Use a caller stream (cudaStream_t) instead of the context's own; NULL restores it.  A lone
   pair split in two halves (RFD_SPLIT) runs one half on a second stream the context owns,
   forked from and joined back to this stream with events, so the call stays ordered on it. */
int32_t rfd_context_set_stream(rfd_context* ctx, void* stream);
/* Phase timing with CUDA events on the context's stream (off by default; no reference
   counterpart - the reference prints host wall times, src/frechet.cpp:65-71).
   enable: 1 on, 0 off, -1 leave as is.  When out != NULL it receives, for the calls since
   the previous query, out[0] = ms in constants + DFD, out[1] = ms in VE-FD, out[2] = ms in
   decisions, out[3] = calls, out[4] = kernel launches, out[5] = bytes copied host to device,
   out[6] = bytes copied device to host; the counters are then reset. */
int32_t rfd_context_phase_times(rfd_context* ctx, int32_t enable, double* out);

/* Measured FP64 fused multiply-add throughput of the context's device in TFLOP/s (2 flops
   per FMA): independent FMA chains at full occupancy, timed with CUDA events.  The roofline
   denominator for the FP64 wavefront kernels (no reference counterpart). */
int32_t rfd_fp64_peak(rfd_context* ctx, double* tflops);

/* ---- the hot path ---- */

/* One continuous Frechet distance: endpoint bound, DFD and VE-FD bracket, epsilon search.
   Replaces compute_distance_parallel (include/wrapper.hpp:4, src/compute_distance_wrapper.cpp:8)
   and Frechet::Continuous::distance_cuda (include/frechet.hpp:14, src/frechet.cpp:18). */
int32_t rfd_distance(rfd_context* ctx, const double* c1, int64_t n1, const double* c2, int64_t n2,
                     int32_t dims, const rfd_options* opt, rfd_result* out);

/* Many pairs in one persistent launch sequence (no reference counterpart: the reference
   solves one pair per call).  c1s/c2s are arrays of npairs curve pointers; dims may differ
   per pair.  Results are written to out[0..npairs). */
int32_t rfd_distance_batch(rfd_context* ctx, int64_t npairs, const double* const* c1s,
                           const int64_t* n1s, const double* const* c2s, const int64_t* n2s,
                           const int32_t* dims, const rfd_options* opt, rfd_result* out);

/* Autotuner of the DFD sweep (no reference counterpart: the reference fixes its launch shape,
   src/intersection_algorithm_in_parallel.cu:1268-1326).  Times rows per lane (1, 2, 4, 8: the
   strip height) and the row layout (0 stacked, 1 skewed) on the caller's pairs, `reps` timed
   sweeps each after one untimed one, and keeps the fastest in the context for later calls.
   ms_out (optional): 8 doubles, ms per sweep at [rows index * 2 + layout].  best_out
   (optional): 2 ints, the rows and layout kept.  Curves as rfd_distance_batch (opt->memory). */
int32_t rfd_autotune(rfd_context* ctx, int64_t npairs, const double* const* c1s, const int64_t* n1s,
                     const double* const* c2s, const int64_t* n2s, const int32_t* dims,
                     const rfd_options* opt, int32_t reps, double* ms_out, int32_t* best_out);

/* Autotuner of the team strips' shape and of the batched search's split (no reference
   counterpart: the reference fixes its launch shape).  Times every combination of warps per
   team (4 or 8), the switch point from probe rounds run as launches to the continuous queue
   (a quarter of the team count of active pairs, the team count, or the queue from the first
   probe: INT32_MAX) and the continuous search's start window (1, 2 or 4
   strips), on whole solves of the caller's pairs with the caller's options (`reps` timed calls
   each, after one untimed one), and keeps the fastest in the context for later calls.
   ms_out (optional): 18 doubles, ms per solve at [(warps index * 3 + switch index) * 3 +
   window index].  best_out (optional): 3 ints, warps per team, switch point, window kept.
   The strip height is the warp width (32 rows, a lane per row) and is not tuned. */
int32_t rfd_autotune_search(rfd_context* ctx, int64_t npairs, const double* const* c1s,
                            const int64_t* n1s, const double* const* c2s, const int64_t* n2s,
                            const int32_t* dims, const rfd_options* opt, int32_t reps,
                            double* ms_out, int32_t* best_out);

/* All pairwise distances of ncurves curves (no reference counterpart: the many-to-many use of
   the reference's Curves, include/curve.hpp:42-47).  out is ncurves x ncurves, row-major,
   symmetric with a zero diagonal; entry (i, j), i < j, is the distance with curve i as the
   first curve.  results (optional) receives the ncurves (ncurves - 1) / 2 pair results in
   that order.  Pairs go through rfd_distance_batch in chunks whose strip boundary rows
   (n_i n_j / 4 bytes a pair; a pair that alone exceeds the budget runs in launch windows of
   O(n_i + n_j) memory) stay within budget_bytes (<= 0: 8e9).  opt->bracket must be NULL;
   the curves of a pair must have equal dims. */
int32_t rfd_distance_matrix(rfd_context* ctx, int64_t ncurves, const double* const* curves,
                            const int64_t* ns, const int32_t* dims, const rfd_options* opt,
                            double budget_bytes, double* out, rfd_result* results);

/* The two bounds.  *vefd is read as the endpoint lower bound that seeds VE-FD and
   overwritten with VE-FD (left unchanged when the reference rule skips it and
   reference_quirks != 0).  Replaces Cuda_intersection::Bound_call_gpu
   (include/intersection_algorithm_in_parallel.hpp:26, src/intersection_algorithm_in_parallel.cu:1258). */
int32_t rfd_bounds(rfd_context* ctx, const double* c1, int64_t n1, const double* c2, int64_t n2,
                   int32_t dims, int32_t reference_quirks, int32_t dense, double* dfd, double* vefd);

/* One free-space reachability decision at distance `radius`: *reachable = 1 when the
   propagated right interval of the last cell ends at 1.0.  *right_ub receives that
   value (may be NULL).  Replaces Cuda_intersection::intersection_interval_call_gpu
   (include/intersection_algorithm_in_parallel.hpp:19, src/intersection_algorithm_in_parallel.cu:1398). */
int32_t rfd_decide(rfd_context* ctx, const double* c1, int64_t n1, const double* c2, int64_t n2,
                   int32_t dims, double radius, int32_t dense, int32_t* reachable, double* right_ub);

/* rfd_decide with the free intervals of either reference decision path (enum rfd_formula;
   RFD_FORMULA_REFERENCE picks by free device memory as the reference's constructor does,
   src/intersection_algorithm_in_parallel.cu:87-97).  rfd_decide is this with
   RFD_FORMULA_FUSED. */
int32_t rfd_decide_formula(rfd_context* ctx, const double* c1, int64_t n1, const double* c2,
                           int64_t n2, int32_t dims, double radius, int32_t dense, int32_t formula,
                           int32_t* reachable, double* right_ub);

/* One reachability decision that allocates nothing (no counterpart in the reference).
   For callers that cannot allocate device memory once they run: a robot's control loop
   where an allocation could stall for an unbounded time or fail when the GPU is full, or
   a process sharing the GPU under a memory budget fixed at start-up.  The curves (c1, c2)
   and the output (right_ub, one double) are the caller's device memory; all other working
   memory is one file-scope device array of 64 MiB that every GPU loading librfd.so holds
   until exit (pairs needing more return RFD_ERR_LIMIT before anything runs).  The work is
   enqueued on `stream` (a cudaStream_t, NULL for the default stream) and the call returns
   without waiting, so its status covers the arguments and the enqueueing only: what the
   kernels find arrives in *right_ub.  It receives the propagated right UB of the last cell
   (reachable iff it equals 1.0), a value in [-2, 1], or NaN when an inter-warp wait ran out
   of its budget (RFD_SPIN_CYCLES, else about 20 s): NaN means the decision failed and must
   not be read as "not reachable"; the next call starts afresh.  The first call on a device
   looks up the array's address and sets kernel attributes there, so make that first call
   before any stream capture.  All calls share the array and each clears what must start
   at zero; calls whose work overlaps on the GPU race and must not be issued. */
int32_t rfd_decide_noalloc(const double* c1, int64_t n1, const double* c2, int64_t n2,
                           int32_t dims, double radius, void* stream, double* right_ub);

/* ---- learned bracket (no reference counterpart) ----
   A BF16 MLP (400 -> 256 -> 256 -> 256 -> 2, GELU, FP32 accumulation) on the tensor cores,
   predicting the 5% and 95% quantiles of log10(FD / VEFD - 1 + 1e-13) from bracket
   features.  Parameters are one flat FP32 array of rfd_model_num_params() values (layer
   by layer: W[out][in] row-major then b[out]).  x/t/y pointers are device memory.  The
   model works on its own stream: x and t must be complete on the device when a call is
   made (synchronise the producing stream first); each call returns after its work ends. */
int64_t rfd_model_num_params(void);
int32_t rfd_model_create(int32_t device, uint64_t seed, rfd_model** out);
int32_t rfd_model_destroy(rfd_model* model);
int32_t rfd_model_set_params(rfd_model* model, const float* params, int64_t n);
int32_t rfd_model_get_params(rfd_model* model, float* params, int64_t n);
/* y[B][2] = model(x[B][400]) */
int32_t rfd_model_forward(rfd_model* model, const float* x, int64_t B, float* y);
/* pinball loss of x[B][400] against targets t[B]; grads (host, num_params floats) may be NULL */
int32_t rfd_model_gradients(rfd_model* model, const float* x, const float* t, int64_t B,
                            float* grads, float* loss);
/* one Adam step (beta 0.9 / 0.999) on the pinball loss of a minibatch */
int32_t rfd_model_train_step(rfd_model* model, const float* x, const float* t, int64_t B,
                             float lr, float* loss);
/* The network's GEMM kernel on its own (test entry): C[M][N] = A[M][K] B[K][N] with
   A(m,k) = A[m*a_sr + k*a_sc], B(k,n) = B[k*b_sr + n*b_sc], operands rounded to BF16,
   FP32 accumulation; all pointers device memory. */
int32_t rfd_gemm_bf16(int32_t M, int32_t N, int32_t K, const float* A, int64_t a_sr, int64_t a_sc,
                      const float* B, int64_t b_sr, int64_t b_sc, float* C);
/* Bracket features of npairs pairs (host curves, endpoint and VE-FD bounds) into
   out[npairs][400] (host): both curves resampled to 64 points uniform in arc length,
   centred and scaled, then log(endpoint / scale) and log(VEFD / scale), zero padded. */
int32_t rfd_features(rfd_context* ctx, int64_t npairs, const double* const* c1s, const int64_t* n1s,
                     const double* const* c2s, const int64_t* n2s, const int32_t* dims,
                     const double* endpoint, const double* vefd, float* out);

/* ---- loader ----
   Text curve loader: one point per line, comma separated, consecutive duplicates dropped.
   Replaces txtLoader2 / txtLoader3 (include/txtReader.hpp:6, :48).  On success *out is a
   malloc'd [*n][dims] array released with rfd_free. */
int32_t rfd_load_txt(const char* path, int32_t dims, int32_t start, int32_t limit, double** out,
                     int64_t* n);

/* rfd_load_txt with the parsing spread over `threads` host threads (<= 0: all cores); the
   same rules and results (no reference counterpart: the survey's fast loader). */
int32_t rfd_load_txt_fast(const char* path, int32_t dims, int32_t start, int32_t limit,
                          int32_t threads, double** out, int64_t* n);
/* Binary trajectory files: "RFDB", uint32 version 1, int32 dims, int32 0, int64 n, then n*dims
   little-endian doubles.  rfd_load_bin's *out is freed with rfd_free. */
int32_t rfd_save_bin(const char* path, const double* pts, int64_t n, int32_t dims);
int32_t rfd_load_bin(const char* path, double** out, int64_t* n, int32_t* dims);
void rfd_free(void* p);

/* ---- synthetic workloads (seeded; see robotfd_b200/csrc/rfd_gen.cpp) ---- */
int32_t rfd_gen_pair(int32_t style, int32_t dims, int64_t n1, int64_t n2, double scale, double noise,
                     uint64_t seed, uint64_t stream, double* P, int64_t* out_n1, double* Q,
                     int64_t* out_n2);
int32_t rfd_gen_batch_spec(int32_t config, int64_t npairs, uint64_t seed, int32_t* dims, int64_t* n1s,
                           int64_t* n2s, int32_t* styles, double* scales, double* noises);

/* ---- FP32 filter of the free intervals (host-callable copy of the device logic, for
   tests; no reference counterpart) ----
   cls[e] = 1 when the FP64 free interval of the edge a_e -> b_e (di = b - a in FP64) around
   x_e at radius^2 r2 is certainly empty, 2 when it is certainly (0, 1), 0 when it has to be
   computed in FP64.  Arrays are [n][dims]; A[e] = |b_e - a_e|^2 as the engine computes it. */
int32_t rfd_interval_class(int64_t n, const double* x, const double* a, const double* b,
                           const double* A, double r2, int32_t dims, int32_t* cls);

/* ---- search state machine (host-callable copy of the device logic, for tests) ----
   Applies one decision outcome to a bracket search and proposes the next probe.
   state[0..5] = {lb, ub, lo, hi, tol, t}, istate[0..3] = {mode, probes, max_probes, flags},
   stop_mode as in rfd_options.  Returns 1 and *next_eps when another probe is due.  The first
   call (probes 0, no outcome) starts the search as the device does: a finite bracket lo < hi
   enables its checks, and t receives the stop threshold above lb, probed first when lo < t. */
int32_t rfd_search_step(double* state, int32_t* istate, int32_t stop_mode, int32_t have_outcome,
                        double eps, int32_t reachable, double* next_eps);

#ifdef __cplusplus
}
#endif

#endif /* RFD_H */
