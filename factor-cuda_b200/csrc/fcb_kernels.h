// fcb_kernels.h -- internal launch interface between the kernel translation
// units and the C-ABI host drivers (capi.cu).  Not part of the public ABI.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace fcb {

// Largest cross-section the shared-memory rank kernels take (u16 column ids,
// 1024 threads x 16 items).  Larger N goes through the global-memory path.
constexpr int kSmemRankCap = 16384;
// CDF network for learned splitters: hidden width, parameter count, table knots.
constexpr int kCdfHidden = 32;
constexpr int kCdfParams = 1 + 1 * 32 + 32 + 32 * 32 + 32 + 32;  // W1,b1,W2,b2,w3,b3 = 1153
constexpr int kCdfKnots = 1024;
// Share of the buckets the tabulated CDF spreads uniformly over its knots.
constexpr float kCdfLinearShare = 0.03f;
constexpr size_t kMaxSmemPerBlock = 227 * 1024;

struct ScanOut {
  float* out[4];  // group g output panel (T,N) or nullptr when the group is inactive
};

// Default largest bucket the learned rank path ranks itself.  A bucket of b
// cells costs each of its cells b comparisons; above the cap the section goes
// to the radix kernel, whose single-section latency is far larger (C2: cap 64
// sent one section in 14616 there and took 1.215 ms per step, cap 256 none
// and 1.195 ms).
constexpr int kLearnCapDefault = 256;

template <typename TF, typename TR>
struct RankIcArgs {
  const TF* X;              // (F,T,N) factor panels
  const TR* R;              // (T,N) forward returns
  const uint8_t* fmask;     // (T,N) factor mask or nullptr
  const uint8_t* rmask;     // (T,N) forward-return mask or nullptr
  int F, T, N, min_valid;
  float* ranks_out;         // (F,T,N) cs_rank ranks (valid = finite(f) & fmask) or nullptr
  double* ic_out;           // (F,T)
  double* rank_f_out;       // (F,T,N) joint-set ranks, 0 elsewhere, or nullptr
  double* rank_r_out;       // (F,T,N) joint-set ranks of the returns, or nullptr
  // learned splitters (used by the LEARNED instantiation only)
  const float* cdf_table;   // (F, kCdfKnots) tabulated monotone CDF per factor
  const float* cdf_zrange;  // (F, 2) grid range [lo, hi] in standardised units
  int learn_cap;            // largest bucket the learned path accepts
  int* learn_stats;         // (F,T,4): outcome, largest bucket, sum of squared bucket sizes, m; or nullptr
  int ic_ld;                // row stride of ic_out (0 = T)
};

struct ColStat {  // one stock_corr column
  double count, mean, min, max, min_abs, max_abs, s2, s1;
};
struct FcColPart {
  double count, s, c, min, max;
};
struct FcColStat {
  double count, mean, min, max;
};
struct FcWork {
  int nblk_cols, nblk_gram;
  FcColPart* colpart;  // [nblk_cols][F]
  FcColStat* colstat;  // [F]
  double* gram;        // [nblk_gram][4][Fp][Fp]
  int* fb_list;        // [F*F]
  int* fb_count;       // [1]
  double* fb_part;     // fc_fb_part_doubles(R, F) doubles, or nullptr (single-block fallback)
};
// Row blocks of factor_corr's Gram pass: narrow panels (F <= 32) use enough
// blocks to fill the SMs several times over (their staging tile is small);
// the same count everywhere keeps single-panel and batched results identical.
inline int fc_gram_blocks(long long R, int F) {
  const long long cap = F <= 32 ? 888 : 148;
  long long nb = R / 1024;
  if (nb < 1) nb = 1;
  return static_cast<int>(nb < cap ? nb : cap);
}
// Row blocks per flagged pair of the multi-block fallback (at most
// kFcFbMaxNblk), and the partials buffer it needs (doubles): kFcFbPartDoubles
// per pair and block plus 4 per pair.
constexpr int kFcFbMaxNblk = 64;
constexpr int kFcFbPartDoubles = 9;
int fc_fb_nblk(long long R, int F);
size_t fc_fb_part_doubles(long long R, int F);
// One factor-plane panel (rows at unit stride, F planes of R rows) of a
// batched factor_corr launch, with its single-panel launch geometry.
struct FcBatchPanel {
  const void* X;
  const uint8_t* mask;
  long long R;
  int F, Fp;
  long long rpb_cols, rpb_gram;   // rows per column / Gram block
  int tasks_total, tasks_per_block, ytiles;
  int maxpairs, fb_nblk, fb_ysl;  // flagged-pair slots, fallback row blocks, pair slots per row block
  int large;                      // 1: multi-block fallback, 0: one block per flagged pair
  FcWork w;
  double* out;
};
// Kinds of batched grid (prefix offsets are kept per kind).
constexpr int kFcbCols = 0, kFcbColFinal = 1, kFcbGram = 2, kFcbFinal = 3, kFcbFbPass = 4, kFcbFbPair = 5,
              kFcbSmall = 6, kFcbGrids = 7;
FcBatchPanel fc_batch_panel(const void* X, const uint8_t* mask, long long R, int F, const FcWork& w, double* out);
// Blocks the panel contributes to each kind of batched grid.
void fc_batch_grids(const FcBatchPanel& q, int (&blocks)[kFcbGrids]);
// Up to nine launches for every panel: d_off holds kFcbGrids runs of np + 1
// prefix offsets, total the grid sizes (host), gram_smem the largest Gram
// staging of the panels; results equal launch_factor_corr_strided's per panel.
cudaError_t launch_factor_corr_batch(const FcBatchPanel* d_panels, int np, const int* d_off, const int* total,
                                     int dtype, size_t gram_smem, cudaStream_t s);

// rank_kernels.cu
cudaError_t launch_cs_rank(const float* X, const uint8_t* mask, int T, int N, int desc, float* out,
                           int* status, cudaStream_t st);
cudaError_t launch_param_scan(const float* X, const uint8_t* mask, int T, int N, ScanOut outs, int* status,
                              cudaStream_t st);
template <typename TF, typename TR>
size_t rank_ic_smem(int N);
template <typename TF, typename TR>
cudaError_t launch_rank_ic(const RankIcArgs<TF, TR>& a, int* status, cudaStream_t st);
cudaError_t launch_rank_ic_learned(const RankIcArgs<float, float>& a, int* status, cudaStream_t st);

// cdf_mlp.cu
size_t cdf_train_smem();
cudaError_t launch_cdf_features(const float* X, const float* ranks, int F, int T, int N, int t0, int tcount, int S,
                                float2* samples, cudaStream_t s);
cudaError_t launch_cdf_train(float* params, float* adam, const float2* samples, int F, int nsamp, int steps, float lr,
                             int step0, float* loss_out, cudaStream_t s);
cudaError_t launch_cdf_grad(const float* params, const float* z, const float* u, int n, float* grad, float* loss,
                            cudaStream_t s);
cudaError_t launch_cdf_tabulate(const float* params, const float2* samples, int F, int nsamp, float* zrange,
                                float* table, bool linear, cudaStream_t s);

// Operands of the stock_corr precision forms, K-major (Np rows x Tp dates),
// column-centred; unused members are nullptr.
struct PrecOperands {
  __nv_bfloat16* h;  // [7][Np][Tp] bf16: mask, three limbs of x', three limbs of x'^2 (or nullptr)
  int np;            // Np (row count of each plane)
  float *x32, *q32, *m32;        // FP32 x', x'^2, mask
};

// corr_tc.cu
constexpr int kPrecTileTcM = 128, kPrecTileTcN = 64, kPrecTileFp32 = 64;
size_t prec_tc_smem();
// Tile list of a precision form (mode 0 BF16x3, 1 FP32) built on the device;
// prec_tile_count gives its length.
int prec_tile_count(int mode, int N);
cudaError_t launch_prec_tiles(int mode, int N, int2* tiles, cudaStream_t s);
// Column means (two steps; part: prec_colmean_chunks(T) * Np double2 scratch)
// and the split operands.
int prec_colmean_chunks(int T);
cudaError_t launch_prec_prep(const float* X, const uint8_t* mask, int T, int N, int Np, int Tp, float* mu,
                             double2* part, PrecOperands op, cudaStream_t s);
cudaError_t launch_corr_bf16x3(const PrecOperands& op, const int2* tiles, int ntiles, int N, int Np, int Tp,
                               double* out, int* status, cudaStream_t s);
cudaError_t launch_corr_fp32(const PrecOperands& op, const int2* tiles, int ntiles, int N, int Tp, double* out,
                             cudaStream_t s);

// corr_kernels.cu
cudaError_t launch_stock_corr_prep(const void* X, int dtype, const uint8_t* mask, int T, int N, int Tp,
                                   double* Xraw, double* Xc, double* Mc, ColStat* st, double* summary,
                                   cudaStream_t s);
// max |x| and min nonzero |x| over the valid cells (finite, mask true) of a
// factor_corr panel, as IEEE bit patterns in ext[0] / ext[1] (0 and +inf when
// no cell is valid).  planes = 0: (R,F) rows; planes = 1: F planes of R rows.
cudaError_t launch_corr_domain(const void* X, int dtype, const uint8_t* mask, long long R, int F, int planes,
                               unsigned long long* ext, cudaStream_t s);
cudaError_t launch_stock_corr_gram(const double* Xraw, const double* Xc, const double* Mc, const ColStat* st, int T,
                                   int N, int Tp, double* out, int* fb_list, int* fb_count, cudaStream_t s);
size_t fc_gram_smem(int Fp, int tasks_per_block, int elem_bytes);
// Work split of the Gram pass for Fp (factors rounded to 4): tiles or tile
// units in all, per block (blockIdx.y), and the blocks along y.
void fc_gram_plan(int Fp, int* tasks_total, int* tasks_per_block, int* ytiles);
cudaError_t launch_factor_corr(const void* X, int dtype, const uint8_t* mask, long long R, int F, FcWork& w,
                               double* out, uint8_t* flags, cudaStream_t s);
// Returns of each date prepared once for the per-(date, factor) rank + IC
// kernels (rank_ic_bucket.cu).  word[t*ld + i]: bits 0-13 the position of
// stock i in the stable ascending order of the date's valid returns, bits
// 14-27 the position where its tie group starts, bit 28 returns valid, bit 29
// factor mask (N <= 16384; rows 16-byte aligned).  fb_count / fb_items: the
// sections (t*F + f) the learned kernel hands to the radix kernel.
struct RicPrep {
  uint32_t* word;
  int* fb_count;
  int* fb_items;
  int ld;
};
// A device list of sections (item ids) handed from the learned kernel to the
// radix kernel.
struct RicList {
  int* count;
  int* items;
};
size_t ric_prep_bytes(int T, int N, int F);
RicPrep ric_prep_carve(void* base, int T, int N, int F);
// True when the per-(date, factor) kernels take N (f32 factors and returns).
bool ric_items_fit(int N);
// Batched form: the panels of one size variant (variant v serves N up to
// ric_variant_cap(v): 2048, 5120, 8192, 16384) in one returns launch, one rank
// launch and (learned) one fallback launch; items are a panel's dates (returns
// pass) or its (date, factor) sections, in panel order.
constexpr int kRicVariants = 4;
int ric_variant_cap(int variant);
struct RicPanel {
  RankIcArgs<float, float> a;
  RicPrep rp;
};
struct RicBatchVariant {
  const RicPanel* panels;  // device, np entries
  const int* off_dates;    // device, exclusive prefix of the panels' T (np entries)
  const int* off_items;    // device, exclusive prefix of the panels' T*F (np entries)
  int np, dates, items, maxN;
  bool learned;            // some panel has a model (its sections take the learned body)
  RicList fb;              // the variant's fallback list (items entries)
};
cudaError_t launch_rank_ic_items_batch(int variant, const RicBatchVariant& v, cudaStream_t st);
// Rank + IC of F >= 1 f32 factor panels against one f32 returns panel: the
// returns pass, then one CTA per (date, factor) -- learned splitters (with the
// radix kernel taking the sections they hand back) or radix.  Requires
// rank_f_out == rank_r_out == nullptr.
cudaError_t launch_rank_ic_items(const RankIcArgs<float, float>& a, RicPrep rp, bool learned, cudaStream_t st);
// Stream-ordered scratch for the entry points that take no workspace: a
// library-private memory pool per device that keeps freed blocks cached.
cudaError_t scratch_alloc(void** p, size_t bytes, cudaStream_t s);
cudaError_t scratch_free(void* p, cudaStream_t s);
// Per-device status word of the asynchronous entry points (capi.cu).
cudaError_t dev_status_sink(int** out);
// One block waiting (at most max_polls polls) on a barrier that completes
// only if `arrive`; sets *status on timeout (selftest.cu).
cudaError_t launch_wait_probe(bool arrive, uint32_t max_polls, int* status, cudaStream_t s);
// Global-memory rank path for cross-sections the shared-memory kernels cannot
// hold (rank_global.cu).  kind 0 cs_rank, 1 parameter_scan, 2 rank+IC: bytes
// of scratch one date needs; the launchers process dates in chunks that fit
// the scratch they are given (at least one date's worth).
size_t rank_global_bytes_per_date(int kind, int N, int F, int ksz_f, int ksz_r);
cudaError_t launch_cs_rank_global(const float* X, const uint8_t* mask, int T, int N, int desc, float* out,
                                  uint8_t* scratch, size_t bytes, cudaStream_t s);
cudaError_t launch_param_scan_global(const float* X, const uint8_t* mask, int T, int N, ScanOut outs,
                                     uint8_t* scratch, size_t bytes, cudaStream_t s);
template <typename TF, typename TR>
cudaError_t launch_rank_ic_global(const RankIcArgs<TF, TR>& a, uint8_t* scratch, size_t bytes, cudaStream_t s);
// True when the shared-memory rank+IC kernel takes N for these dtypes.
template <typename TF, typename TR>
inline bool rank_ic_fits_smem(int N) {
  return N <= kSmemRankCap && rank_ic_smem<TF, TR>(N) <= kMaxSmemPerBlock;
}
inline size_t rank_global_scratch(size_t per_date, int T) {
  size_t b = per_date * static_cast<size_t>(T);
  if (b > (size_t(1) << 30)) b = size_t(1) << 30;  // chunks of about 1 GiB
  if (b < per_date) b = per_date;
  return b + 8192;
}

// Persistent rank+IC over (panel, date) items; nt in {256, 512, 1024}.  With
// occ != nullptr nothing is launched: *occ receives the CTAs per SM that fit.
template <typename TF, typename TR>
size_t rank_ic_batch_smem(int nt, int maxN);
template <typename TF, typename TR>
cudaError_t launch_rank_ic_batch(int nt, bool learned, const RankIcArgs<TF, TR>* panels, const int2* items,
                                 int nitems, int* counter, int grid, size_t smem, int* status, cudaStream_t st,
                                 int* occ);
// factor_corr precision form (fc_tc.cu): BF16x3 tcgen05 moment products over
// the R pooled rows, split over one CTA per SM, FP64 finalize.  F <= kFcTcMaxF;
// element (r, f) at X[r*sr + f*sf]; work: fc_tc_work_bytes(F) bytes.
constexpr int kFcTcMaxF = 16;
size_t fc_tc_work_bytes(int F);
cudaError_t launch_factor_corr_bf16x3(const float* X, const uint8_t* mask, long long R, int F, long long sr,
                                      long long sf, void* work, double* out, int* status, cudaStream_t s);
// Same with element (r, f) at X[r*sr + f*sf].
cudaError_t launch_factor_corr_strided(const void* X, int dtype, const uint8_t* mask, long long R, int F,
                                       long long sr, long long sf, FcWork& w, double* out, uint8_t* flags,
                                       cudaStream_t s);

}  // namespace fcb
