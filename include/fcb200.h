/* fcb200.h -- C ABI of the B200-native cross-sectional analysis path.
 *
 * libfcb200.so exports plain C entry points (host pointers + sizes, no torch
 * or pybind types).  Each replaces one native interface of factor-cuda
 * (reference file:line given beside it) with the same argument meaning,
 * preconditions and status codes, so the reference's pybind11 layer -- or the
 * drop-in modules factor_cuda_pybind / factor_corr_pybind built on this ABI --
 * can bind it directly.
 *
 * Status convention (reference src/factor_cuda_pybind.cpp:117-123):
 *   0            success
 *   negative     contract error (caller maps to ValueError)
 *   positive     cudaError_t of the failing CUDA call (RuntimeError)
 * FCB_ERR_DEVICE_WAIT (a positive code outside the cudaError_t range used by
 * these calls) reports a bounded device-side wait that gave up.
 *
 * Host entry points are synchronous: inputs are uploaded, kernels run and
 * results are downloaded before they return.  Host buffers may be pageable or
 * pinned (fcb_host_alloc); pinned buffers make the copies faster.
 * Every entry point is safe to call from any host thread; calls that share a
 * workspace must be serialised by the caller (as in the reference).
 */
#ifndef FCB200_H_
#define FCB200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FCB_DTYPE_F32 0
#define FCB_DTYPE_F64 1

#define FCB_OK 0
#define FCB_ERR_ARG (-1)      /* null pointer or a dimension < 1            */
#define FCB_ERR_CAP2 (-2)     /* op-specific cap, see each entry point      */
#define FCB_ERR_CAP3 (-3)     /* op-specific cap, see each entry point      */
#define FCB_ERR_CAP4 (-4)     /* op-specific (domain / min_valid)           */
#define FCB_ERR_UNSUPPORTED (-5) /* valid request this build cannot serve   */
#define FCB_ERR_NOALLOC_CAP (-6) /* size above a no-allocation entry's maximum */
#define FCB_ERR_DEVICE_WAIT 100000 /* bounded device wait gave up           */

/* parameter_scan group status (reference src/parameter_scan.cuh:35-71) */
#define FCB_GROUP_NOT_EXECUTED (-100)

/* Opaque cached-device-buffer workspace (reference cs_rank_workspace,
 * src/cross_sectional_rank.cuh:38-58, and rolling_ic_workspace,
 * src/rolling_ic.cuh:33-67).  Buffers grow on demand and are reused across
 * calls; they are bound to the device current at allocation time and
 * re-allocated on a device change.  Not thread-safe. */
typedef struct fcb_workspace fcb_workspace;

fcb_workspace* fcb_workspace_create(void);
/* Release all device buffers (idempotent); the handle stays usable.
 * Replaces cs_rank_workspace_clear (src/cross_sectional_rank.cuh:67). */
void fcb_workspace_clear(fcb_workspace* ws);
void fcb_workspace_destroy(fcb_workspace* ws);
/* Allocation accounting: live and high-water device bytes held by the
 * workspace (replaces MemTracker live/peak, src/mem_tracker.h:35-77). */
int fcb_workspace_stats(const fcb_workspace* ws, uint64_t* live_bytes, uint64_t* peak_bytes,
                        uint64_t* n_allocs);

/* Memory budget model (the counterpart of the reference's budget table,
 * docs/memory_budget_v1.json, and of MemTracker's peak, src/mem_tracker.h:
 * 35-77): *bytes = the device bytes the workspace of entry point `op` holds
 * after one call of shape (T, N, F) -- the sum of its buffers, which is the
 * workspace's peak (fcb_workspace_stats) for a fresh workspace.  Buffers the
 * driver rounds up to its allocation granularity can occupy a little more of
 * the device.  flags: FCB_BUDGET_MASK a (first) mask is passed,
 * FCB_BUDGET_MASK2 a second mask (rolling_ic rmask, panel rmask),
 * FCB_BUDGET_RANKS rank outputs (rolling_ic rank_f / rank_r, panel ranks),
 * FCB_BUDGET_FALLBACK factor_corr fallback_out, FCB_BUDGET_R_F64 rolling_ic
 * returns are f64; bits 8-11: parameter_scan active groups (0 = all four).
 * dtype: the input dtype; for FCB_OP_STOCK_CORR_PREC the precision mode.
 * FCB_OP_RANK_IC_PANEL covers method 0; FCB_OP_FACTOR_CORR and
 * FCB_OP_STOCK_CORR count the host entry points' own temporary workspace.
 * Returns -1 unknown op / bad shape, -3 size cap, -5 unsupported shape. */
#define FCB_OP_CS_RANK 1
#define FCB_OP_PARAMETER_SCAN 2
#define FCB_OP_ROLLING_IC 3
#define FCB_OP_FACTOR_CORR 4
#define FCB_OP_DEV_FACTOR_CORR 5
#define FCB_OP_STOCK_CORR 6
#define FCB_OP_DEV_STOCK_CORR 7
#define FCB_OP_FACTOR_CORR_BF16X3 8
#define FCB_OP_STOCK_CORR_PREC 9
#define FCB_OP_RANK_IC_PANEL 10
#define FCB_BUDGET_MASK 1
#define FCB_BUDGET_MASK2 2
#define FCB_BUDGET_RANKS 4
#define FCB_BUDGET_FALLBACK 8
#define FCB_BUDGET_R_F64 16
int fcb_memory_budget(int op, int dtype, int T, int N, int F, int flags, uint64_t* bytes);

/* Learned-splitter state a workspace carries across fcb_rank_ic_panel calls
 * (method 1): ready = a fitted table is in use, fits = refits scheduled so
 * far, learned_chunks = date chunks ranked by the learned kernel so far. */
int fcb_workspace_learned_state(const fcb_workspace* ws, int* ready, int* fits, int* learned_chunks);

/* Library / device helpers. */
int fcb_version(void);
int fcb_device_count(void);
const char* fcb_status_string(int status);
/* Pinned host memory for fast transfers (cudaHostAlloc / cudaFreeHost). */
void* fcb_host_alloc(size_t bytes);
void fcb_host_free(void* p);

/* ---------------------------------------------------------------- rank ---
 * Stable ordinal cross-sectional rank of a (T,N) f32 panel.  Valid cell =
 * finite && mask; ranks 1..K by ascending value (descending: of -x), ties by
 * column; invalid cells get the quiet NaN 0x7fc00000.
 * Replaces cs_rank_gpu (src/cross_sectional_rank.cuh:90-99).
 * Returns -1 null/dim, -2 N > 2^24, -3 T*N > INT32_MAX.
 * Every N up to the cap is served: sections that fit one CTA's shared memory
 * (N <= 16384 for cs_rank, parameter_scan and f32 rank + IC of several
 * factors; about 11000 f32 and 8192 f64 for single-factor rolling_ic) are
 * sorted there, wider ones by a
 * global-memory radix sort per date with the same results (scratch from the
 * workspace, or stream-ordered cudaMallocAsync for the fcb_dev_* variants). */
int fcb_cs_rank_f32(const float* x, const uint8_t* mask, int T, int N, int descending, float* out,
                    fcb_workspace* ws);

/* G=4 parameter scan: out[g] for g = asc-masked, asc-unmasked, desc-masked,
 * desc-unmasked (NULL allowed for inactive groups).  active[4] (NULL = all)
 * selects groups; group_status[g] = 0 ok, -100 not executed, or the
 * whitelisted cudaError_t (9 / 701) of a failed launch.  time_ms / time_gpu_ms
 * (NULL = off) receive per-group host / device time; the four groups are
 * produced by one fused pass whose time is split evenly over the active
 * groups.  Replaces parameter_scan_gpu (src/parameter_scan.cuh:82-90). */
int fcb_parameter_scan_f32(const float* x, const uint8_t* mask, int T, int N, float* const out[4],
                           int group_status[4], double time_ms[4], float time_gpu_ms[4],
                           const int active[4], fcb_workspace* ws);

/* ----------------------------------------------------------- rolling_ic ---
 * Daily Spearman IC between factor f and forward returns r, (T,) f64.
 * Joint valid set = finite(f) & finite(r) & fmask & rmask; fewer than
 * min_valid joint cells, or a constant side on the joint set -> NaN.  f and r
 * are f32 or f64 (FCB_DTYPE_*) and are ranked at that dtype.  rank_f/rank_r
 * (NULL = off) receive the (T,N) joint-set ranks as f64, 0 elsewhere.
 * Replaces rolling_ic_gpu (src/rolling_ic.cuh:102-108).
 * Returns -1 null/dim, -3 T*N > INT32_MAX, -4 min_valid < 2. */
int fcb_rolling_ic(const void* f, int f_dtype, const void* r, int r_dtype, const uint8_t* fmask,
                   const uint8_t* rmask, int T, int N, int min_valid, double* ic, double* rank_f,
                   double* rank_r, fcb_workspace* ws);

/* ---------------------------------------------------------- correlation ---
 * (F,F) pooled pairwise-complete Pearson of a (T,N,F) panel over (t,i) rows,
 * mask (T,N) broadcast to every factor.  x is f32 or f64.  fallback_out
 * (NULL = off) receives F*F bytes, 1 where the pair was recomputed by the
 * two-pass compensated fallback.
 * Replaces factor_corr_gpu (src/factor_corr.cuh:46-49).
 * Returns -1 null/dim, -2 T*N > INT32_MAX, -3 F > 128. */
int fcb_factor_corr(const void* x, int dtype, const uint8_t* mask, int T, int N, int F, double* out,
                    uint8_t* fallback_out);

/* factor_corr on caller-owned DEVICE buffers, asynchronous on `stream` (NULL =
 * legacy stream); same kernels and results as fcb_factor_corr.  planes = 0:
 * d_x is the reference's (T,N,F) panel; planes = 1: F factor planes (F,T,N).
 * Scratch comes from `ws` (required; calls sharing it must be serialised).
 * No reference counterpart (device-pointer variant of factor_corr_gpu). */
int fcb_dev_factor_corr(const void* d_x, int dtype, const uint8_t* d_mask, int T, int N, int F, int planes,
                        double* d_out, fcb_workspace* ws, void* stream);

/* (N,N) pairwise-complete Pearson of a (T,N) panel over t.  selected_path
 * (NULL = off): 0 fully valid panel, 1 masked panel; fallback_count: pairs
 * recomputed by the two-pass fallback.
 * Replaces stock_corr_gpu (src/stock_corr.cuh:66-68).
 * Returns -1 null/dim, -2 T*N > INT32_MAX, -3 N*N > INT32_MAX,
 * -4 domain (max|x| > 1e150 or a nonzero |x| < 1e-150 on a valid cell). */
int fcb_stock_corr(const void* x, int dtype, const uint8_t* mask, int T, int N, double* out,
                   int* selected_path, int* fallback_count);

/* ------------------------------------------------------- batched panels ---
 * Rank + IC over F factor panels sharing one forward-return panel (the
 * reference pipeline's cs_rank -> rolling_ic stages, benchmarks/poc4_e2e_v1.py
 * :80-101, fused).  x (F,T,N) f32, r (T,N) f32, fmask / rmask (T,N) or NULL.
 * ranks (F,T,N) f32 (NULL = off) = cs_rank of each factor under fmask;
 * ic (F,T) f64 = rolling_ic(factor, r, fmask, rmask, min_valid).
 * method: 0 plain radix; 1 learned splitters: the first date chunk is ranked
 * by radix and a CDF model is fitted on it, later chunks use the learned
 * path, and the model is refitted (warm start) on the exact ranks of the
 * latest chunk every 250 dates.
 * Host pointers; the panel is streamed through the device in date chunks
 * with copies overlapping the kernels.  No reference counterpart as one call. */
int fcb_rank_ic_panel(const float* x, const float* r, const uint8_t* fmask, const uint8_t* rmask, int F,
                      int T, int N, int min_valid, float* ranks, double* ic, int method,
                      fcb_workspace* ws);

/* Device-pointer variant (all pointers device-resident, stream = cudaStream_t
 * or NULL for the legacy stream).  Asynchronous; no host synchronisation. */
int fcb_dev_rank_ic_panel(const float* d_x, const float* d_r, const uint8_t* d_fmask, const uint8_t* d_rmask,
                          int F, int T, int N, int min_valid, float* d_ranks, double* d_ic, int method,
                          void* stream);

/* ------------------------------------------- device-resident fc.* calls ---
 * The fc.* operators on caller-owned DEVICE buffers, issued on `stream`
 * (cudaStream_t, NULL = legacy stream), with the same arguments, kernels,
 * results and status codes as the host entry points above.  They remove the
 * device -> host -> device round trip the reference adapter makes for
 * CUDA-resident inputs (fc/_util.py:121-131).  Scratch is either stream-ordered
 * (cudaMallocAsync from a per-device pool) or taken from `ws` where the
 * signature has one; calls sharing a workspace must be serialised. */

/* Bounded device-side waits in the asynchronous entry points (a staged copy
 * that did not land) set a status word of the current device instead of
 * returning a code.  fcb_dev_status synchronises the current device, returns
 * FCB_ERR_DEVICE_WAIT (and clears the word) if any such wait gave up since the
 * last check, else FCB_OK.  The word is allocated on a device's first
 * asynchronous call (before any stream capture on that device).  No reference
 * counterpart: the reference's entry points are all synchronous. */
int fcb_dev_status(void);

/* Self-test of the bounded-wait path (no reference counterpart): one block
 * waits, for at most max_polls polls, on a shared-memory barrier that is
 * completed only when arrive != 0 (otherwise it expects a transfer that is
 * never issued).  Returns FCB_ERR_DEVICE_WAIT when the wait ran out, FCB_OK
 * when it completed; the device stays usable either way.  Synchronous. */
int fcb_selftest_bounded_wait(int arrive, int max_polls);

/* cs_rank (asynchronous). */
int fcb_dev_cs_rank_f32(const float* d_x, const uint8_t* d_mask, int T, int N, int descending, float* d_out,
                        void* stream);

/* parameter_scan (asynchronous).  group_status is filled on the host when
 * the call returns: 0 for every active group that was launched, the
 * whitelisted launch error (9 / 701) for a group whose launch failed, -100 for
 * inactive groups.  Timing is left to the caller (events on `stream`). */
int fcb_dev_parameter_scan_f32(const float* d_x, const uint8_t* d_mask, int T, int N, float* const d_out[4],
                               int group_status[4], const int active[4], void* stream);

/* rolling_ic (asynchronous); f / r f32 or f64; d_rank_f / d_rank_r (NULL =
 * off) receive the (T,N) f64 joint-set ranks, 0 elsewhere. */
int fcb_dev_rolling_ic(const void* d_f, int f_dtype, const void* d_r, int r_dtype, const uint8_t* d_fmask,
                       const uint8_t* d_rmask, int T, int N, int min_valid, double* d_ic, double* d_rank_f,
                       double* d_rank_r, void* stream);

/* stock_corr into a device (N,N) f64 buffer.  Synchronises `stream` twice:
 * the domain check and the path flag are read on the host before the Gram
 * pass, and fallback_count after it.  Scratch from `ws` (required). */
int fcb_dev_stock_corr(const void* d_x, int dtype, const uint8_t* d_mask, int T, int N, double* d_out,
                       int* selected_path, int* fallback_count, fcb_workspace* ws, void* stream);

/* Correlation domain precondition of a device factor_corr panel (layout as
 * fcb_dev_factor_corr): *in_domain = 1 when max|x| <= 1e150 and every nonzero
 * |x| >= 1e-150 over the valid cells (finite, mask true), else 0.  The
 * reference adapter runs this check on the host before factor_corr_gpu
 * (fc/correlation.py:16-49).  Synchronises `stream`. */
int fcb_dev_corr_domain(const void* d_x, int dtype, const uint8_t* d_mask, int T, int N, int F, int planes,
                        int* in_domain, void* stream);

/* ---------------------------------------------------- learned splitters ---
 * No reference counterpart (a new form of the rank path).  A model holds one
 * CDF network per factor (1 -> 32 -> 32 -> 1, tanh, sigmoid output) trained
 * on the GPU by this library's forward/backward kernels, and its tabulated
 * monotone CDF.  The learned rank path scatters each cross-section into
 * buckets by that CDF and ranks each bucket exactly; every date is checked
 * (strictly increasing (value, column) order over the whole output) and any
 * failure, bucket above `cap` or unusable scale falls back to the radix sort,
 * so ranks and IC are bit-identical to the radix path. */
#define FCB_CDF_PARAMS 1153
#define FCB_CDF_KNOTS 1024
typedef struct fcb_cdf_model fcb_cdf_model;
/* F networks, deterministic initialisation from seed; NULL on failure. */
fcb_cdf_model* fcb_cdf_model_create(int F, uint64_t seed);
void fcb_cdf_model_destroy(fcb_cdf_model* m);
/* linear = 1: tabulate a linear ramp over the fitted range instead of the
 * network (the bucket method without the network, for comparisons). */
int fcb_cdf_model_set_linear(fcb_cdf_model* m, int linear);
/* Fit on dates [t0, t0+tcount) of device panels d_x (F,T,N) f32 and their
 * exact cs ranks d_ranks (F,T,N) f32 (NaN = unranked): 64 samples per date
 * (standardised value, (rank-0.5)/m), `steps` Adam steps of 256 samples
 * continuing from the model's previous state, then tabulation.  Async. */
int fcb_cdf_model_fit(fcb_cdf_model* m, const float* d_x, const float* d_ranks, int T, int N, int t0, int tcount,
                      int steps, float lr, void* stream);
/* The two halves of a fit, for refits that overlap ranking (no reference
 * counterpart).  fcb_cdf_model_sample draws the training samples from dates
 * [t0, t0+tcount) of d_x and its exact ranks d_ranks on `stream` (order it
 * after the kernel that wrote the ranks; the ranks buffer may be reused once
 * it has run).  fcb_cdf_model_train runs `steps` Adam steps on the drawn
 * samples and tabulates into the current table slot (into_idle = 0) or into
 * the idle one (into_idle = 1), which rank calls do not read.
 * fcb_cdf_model_swap makes the idle slot current for later rank calls: call
 * it after the training stream has passed the refit (or order the next rank
 * call's stream after it).  Only one refit may be in flight per model. */
int fcb_cdf_model_sample(fcb_cdf_model* m, const float* d_x, const float* d_ranks, int T, int N, int t0,
                         int tcount, void* stream);
int fcb_cdf_model_train(fcb_cdf_model* m, int steps, float lr, int into_idle, void* stream);
int fcb_cdf_model_swap(fcb_cdf_model* m);
/* Save / restore (host buffers): params (F*FCB_CDF_PARAMS), zrange (F*2),
 * table (F*FCB_CDF_KNOTS), last minibatch loss (F); NULL skips a field. */
int fcb_cdf_model_state(const fcb_cdf_model* m, float* params, float* zrange, float* table, float* loss);
int fcb_cdf_model_load(fcb_cdf_model* m, const float* params, const float* zrange, const float* table);
/* Loss (sum of squared errors over samples with u >= 0) and its gradient
 * w.r.t. the FCB_CDF_PARAMS parameters (mean-squared-error normalisation)
 * for one batch of n <= 256 samples, by the training kernel's own
 * forward/backward code.  Host pointers; for checking. */
int fcb_cdf_grad(const float* params, const float* z, const float* u, int n, float* grad, float* loss);
/* Learned rank + IC over device panels (as fcb_dev_rank_ic_panel); d_stats
 * (NULL = off) receives (F,T,4) ints: outcome (1 learned, 2 bucket overflow,
 * 3 order check rejected -- with several factors, a staged CDF table that
 * is not non-decreasing within [0, 1]; with one factor, the ranked keys out
 * of order --, 4 unusable scale; 2-4 fell back to radix), the largest
 * bucket, the sum of squared bucket sizes (the per-date comparison work; m
 * for perfectly even buckets of one) and m, the number of ranked cells.
 * Sections too wide for the shared-memory kernel are ranked by the
 * global-memory radix path (same results); their statistics read 0.  cap:
 * the largest bucket the learned kernel ranks itself; 0 = the default, 256
 * (a bucket of b cells costs each of its cells b comparisons, far less than
 * sending the section to the radix kernel). */
int fcb_dev_rank_ic_panel_learned(const float* d_x, const float* d_r, const uint8_t* d_fmask,
                                  const uint8_t* d_rmask, int F, int T, int N, int min_valid, float* d_ranks,
                                  double* d_ic, const fcb_cdf_model* model, int cap, int* d_stats, void* stream);

/* ------------------------------------------------------ precision forms ---
 * No reference counterpart (a new form of stock_corr).  Pairwise-complete
 * (N,N) Pearson of an f32 (T,N) panel with column-centred moments formed by
 *   FCB_PREC_BF16X3: x' and x'^2 split into three bf16 limbs each, all limb
 *                    products on the tcgen05 tensor cores (7 MMAs per 16
 *                    dates against a stacked B operand, fp32 accumulation
 *                    in TMEM);
 *   FCB_PREC_FP32:   plain fp32 FMA on the CUDA cores;
 * both finalised in f64: cov = sxy - sx sy/n etc., r = (cov/sqrt(vx))/sqrt(vy),
 * NaN for n < 2 or a non-positive variance, diagonal 1.0 iff finite, lower
 * triangle mirrored.  No cancellation fallback: tolerance, not bit parity,
 * against the f64 path (tests state the bound).  The device variant takes
 * its scratch from the workspace (required) and synchronises `stream`. */
#define FCB_PREC_BF16X3 0
#define FCB_PREC_FP32 1
int fcb_stock_corr_prec(const float* x, const uint8_t* mask, int T, int N, int mode, double* out,
                        fcb_workspace* ws);
int fcb_dev_stock_corr_prec(const float* d_x, const uint8_t* d_mask, int T, int N, int mode, double* d_out,
                            fcb_workspace* ws, void* stream);

/* BF16x3 precision form of factor_corr (no reference counterpart; the
 * tensor-core form of factor_corr_gpu, src/factor_corr.cuh:46-49).  The pooled
 * moment products n, sum x', sum x'^2, sum x'x' over the T*N (t,i) rows of an
 * f32 panel (x' = x minus a per-factor shift near its mean) are tcgen05 GEMMs
 * on three bf16 limbs of x' and of x'^2 with fp32 accumulation, split over the
 * SMs and merged in f64; r = (cov/sqrt(vx))/sqrt(vy) in f64, NaN for n < 2 or
 * a non-positive variance, diagonal 1.0 iff finite, lower triangle mirrored.
 * No cancellation fallback: tolerance (|err| <= 1e-6 per output against the
 * f64 path, stated in the tests), not bit parity.  F <= 16 (larger F returns
 * FCB_ERR_UNSUPPORTED; the f64 entry points take F <= 128).
 * fcb_factor_corr_bf16x3: host (T,N,F) panel, synchronous, ws may be NULL.
 * fcb_dev_factor_corr_bf16x3: device buffers, planes = 0 (T,N,F) or 1 (F,T,N)
 * factor planes, asynchronous on `stream`, scratch from `ws` (required);
 * bounded waits report through fcb_dev_status.
 * Returns -1 null/dim, -2 T*N > INT32_MAX, -3 F > 128. */
int fcb_factor_corr_bf16x3(const float* x, const uint8_t* mask, int T, int N, int F, double* out,
                           fcb_workspace* ws);
int fcb_dev_factor_corr_bf16x3(const float* d_x, const uint8_t* d_mask, int T, int N, int F, int planes,
                               double* d_out, fcb_workspace* ws, void* stream);

/* ------------------------------------------------ no-allocation variant ---
 * No counterpart in the reference.  factor_corr for callers that cannot let a
 * library allocate device memory: applications whose device memory belongs to
 * a framework pool or a hard budget, and latency-sensitive loops that cannot
 * take the device-wide synchronisation of cudaMalloc/cudaFree.  The
 * factor_corr kernels of fcb_dev_factor_corr on caller-owned DEVICE buffers:
 * d_x (T,N,F) f32/f64, d_mask (T,N) or NULL, d_out (F,F) f64; asynchronous on
 * `stream` (NULL = legacy stream).  Its row partition is fixed (148 column /
 * 74 Gram blocks) where fcb_dev_factor_corr sizes it from the pool, so partial
 * sums are added in another order: results agree with fcb_factor_corr within
 * 1e-12 per output, not bit for bit.
 * All scratch -- the multi-block fallback's partials included -- lives in one
 * fixed device array of about 4.9 MB inside the library, which every GPU that
 * loads the library holds until exit; no cudaMalloc/cudaFree or allocating
 * library routine is called.  F is limited to FCB_NOALLOC_MAX_F (larger F
 * returns FCB_ERR_NOALLOC_CAP).  Each call resolves the array's device
 * address on the current device (cudaGetSymbolAddress); the first call on a
 * device also loads the library's device image there, so make it before any
 * stream capture.  Every call shares the one array: calls that overlap on the
 * GPU (concurrent streams or threads) race and must be serialised by the
 * caller. */
#define FCB_NOALLOC_MAX_F 32
int fcb_dev_factor_corr_noalloc(const void* d_x, int dtype, const uint8_t* d_mask, int T, int N, int F,
                                double* d_out, void* stream);

/* ------------------------------------------------------ batched panels ---
 * No counterpart in the reference (which processes one panel per call, so a
 * caller with many panels loops over fc.rolling_ic / fc.factor_corr).  One
 * batch holds many panels of uneven T x N on the current device; each run
 * computes, for every panel, what fcb_dev_rank_ic_panel (cs_rank ranks +
 * rolling_ic) and fcb_factor_corr compute for it alone -- bit for bit.
 * Rank + IC of f32 panels runs the single-panel per-(date, factor) kernels in
 * batched form: per kernel variant (N up to 2048 / 5120 / 8192 / 16384), one
 * returns launch over every date of its panels, one rank launch over every
 * (date, factor) section and, with learned splitters, one launch ranking the
 * sections handed back to the radix sort.  f64 panels run persistent kernels
 * taking (panel, date) items from device queues.  factor_corr follows; the
 * sequence is captured once into a CUDA graph and replayed.  All pointers are
 * DEVICE pointers owned by the caller and must stay valid for the batch's
 * lifetime; runs are asynchronous on `stream` (NULL = legacy stream).  Every
 * device buffer a batch needs is allocated by fcb_batch_create (and, for the
 * graph's launch tables, on the first run or the first run after a
 * configuration change), so run it once before capturing it elsewhere. */
typedef struct fcb_batch fcb_batch;

typedef struct fcb_panel {
  int T, N, F;                 /* N within one CTA's shared memory (rank + IC:
                                  16384 f32, about 8192 f64), else
                                  FCB_ERR_UNSUPPORTED                            */
  const void* X;               /* F factor planes, each (T,N), dtype_x           */
  const void* R;               /* (T,N) forward returns, dtype_r                 */
  const uint8_t* fmask;        /* (T,N) factor mask or NULL                      */
  const uint8_t* rmask;        /* (T,N) returns mask or NULL                     */
  float* ranks_out;            /* (F,T,N) cs_rank ranks or NULL                  */
  double* ic_out;              /* (F,T) rolling IC                               */
  double* corr_out;            /* (F,F) factor_corr over the panel's (t,i) rows
                                  (fmask broadcast per column; F <= 128) or NULL */
  const fcb_cdf_model* model;  /* learned splitters for this panel's factors
                                  (f32 only, fitted, model F == F) or NULL       */
} fcb_panel;

/* Scheduling knobs.  None of them changes a result.  f32 panels: a panel of
 * width N runs in the narrowest kernel variant whose range holds it, the
 * first two ranges being N <= min(nt_small_max, 2048) and
 * N <= min(nt_mid_max, 5120) (then 8192, 16384); ctas_per_sm is not used.
 * f64 panels: size classes of 256 / 512 / 1024-thread persistent CTAs. */
typedef struct fcb_batch_config {
  int nt_small_max;  /* f64: largest N ranked by 256-thread CTAs (1..4096)       */
  int nt_mid_max;    /* f64: largest N ranked by 512-thread CTAs (..8192);
                        larger N use 1024-thread CTAs                           */
  int ctas_per_sm;   /* f64: persistent CTAs per SM per class, 0 = all that fit */
  int concurrent;    /* 1: size classes (variants) run side by side; 0: one
                        after another, each on the whole GPU                    */
  int order;         /* 1: longest panels / items first; 0: panel order         */
  int learn_cap;     /* largest learned bucket before the radix fallback         */
} fcb_batch_config;

void fcb_batch_default_config(fcb_batch_config* cfg);
/* dtype pair (F32,F32) or (F64,F64); min_valid >= 2 (else FCB_ERR_CAP4); cfg
 * NULL = defaults.  Same caps as the single-panel entry points. */
int fcb_batch_create(const fcb_panel* panels, int npanels, int dtype_x, int dtype_r, int min_valid,
                     const fcb_batch_config* cfg, fcb_batch** out);
void fcb_batch_destroy(fcb_batch* b);
int fcb_batch_get_config(const fcb_batch* b, fcb_batch_config* cfg);
int fcb_batch_set_config(fcb_batch* b, const fcb_batch_config* cfg);
/* One replay of the batch's graph (captured on first use or after a config
 * change). */
int fcb_batch_run(fcb_batch* b, void* stream);
/* The same work as one launch sequence per panel, no graph: what a caller
 * looping over the single-panel entry points does (the comparison arm). */
int fcb_batch_run_per_panel(fcb_batch* b, void* stream);
/* Synchronises the device; FCB_OK, or FCB_ERR_DEVICE_WAIT if a staged copy
 * in any run since the last call did not land. */
int fcb_batch_status(fcb_batch* b);
/* Measures the batch under alternative configurations (coordinate descent,
 * `reps` replays each) and keeps the fastest; f32: variant boundaries, order,
 * concurrency and the learned bucket cap; f64: the size-class boundaries tried
 * include the occupancy steps of each block size within the batch's range of
 * N.  cache_path (or NULL): a text
 * file of "signature<TAB>config ms" lines; a batch whose signature is found
 * takes that configuration without measuring (returns 1), a measured winner is
 * appended.  Returns 0 after measuring. */
int fcb_batch_autotune(fcb_batch* b, int reps, const char* cache_path, fcb_batch_config* best, float* best_ms);

#ifdef __cplusplus
}
#endif

#endif /* FCB200_H_ */
