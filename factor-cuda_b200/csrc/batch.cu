// batch.cu -- many panels of uneven T x N per launch.
//
// Rank + IC of f32 panels: the per-(date, factor) kernels of the single-panel
// entry points in batched form.  Panels are grouped by the kernel variant
// their width needs (N up to 2048 / 5120 / 8192 / 16384; the first two
// boundaries are tunable), and each variant is one returns-preparation
// launch over all its panels' dates, one rank launch over all their
// (date, factor) sections and, with learned splitters, one launch that ranks
// the sections handed back to the radix sort -- the same device bodies, so
// results are those of the single-panel calls bit for bit.
//
// Rank + IC of f64 panels: every (panel, date) pair is one work item.  Items are grouped by
// the block size their cross-section needs (256 / 512 / 1024 threads; the
// thresholds are tunable), each group is a device queue, and one persistent
// kernel per group (k_rank_ic_batch) runs as many CTAs as fit, each taking
// items from its queue until it is empty -- so a short panel does not leave
// SMs idle while a long one finishes, and there is one launch per group
// instead of one per panel.  factor_corr of every panel (its factor planes
// pooled over the panel's (t, i) rows, the factor mask broadcast per column)
// runs as one batched launch per kernel kind (column pass, merge, Gram pass,
// finalize, the fallback passes: launch_factor_corr_batch) on a graph branch
// alongside rank + IC.  The whole sequence is captured once into a CUDA graph
// and replayed by fcb_batch_run.
//
// Outputs do not depend on the scheduling knobs: ranks and IC are exact
// integer/ordinal results, and factor_corr's row blocking is fixed by each
// panel's row count (the same blocking the single-panel entry point uses), so
// fcb_batch_run, fcb_batch_run_per_panel and every autotuned configuration
// agree bit for bit.
//
// The autotuner (fcb_batch_autotune) measures the batch itself: starting
// from the default configuration it tries each knob's alternatives in turn
// (coordinate descent), keeps a change when the graph replay gets faster, and
// can remember the winner per batch signature in a small text cache file.
// Each group's shared memory is sized for its widest section, so one panel
// just above an occupancy step costs the whole group a resident CTA per SM;
// besides fixed steps, the group boundaries tried are those steps (the widest
// N that keeps each occupancy level), found from the occupancy calculator
// over the batch's range of N.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <iterator>
#include <new>
#include <string>
#include <vector>

#include "../../include/fcb200.h"
#include "cdf_model.h"
#include "fcb_kernels.h"

using namespace fcb;

namespace {

inline int rcode(cudaError_t e) { return static_cast<int>(e); }
#define FCB_BTRY(...)                      \
  do {                                     \
    cudaError_t _e = (__VA_ARGS__);        \
    if (_e != cudaSuccess) return rcode(_e); \
  } while (0)

constexpr int kClasses = 3;
constexpr int kClassNt[kClasses] = {256, 512, 1024};

}  // namespace

struct fcb_batch {
  int device = -1;
  int sms = 148;
  std::vector<fcb_panel> p;
  int dtx = 0, dtr = 0, min_valid = 30;
  bool learned = false;
  fcb_batch_config cfg{};
  // device state
  void* d_args = nullptr;          // RankIcArgs<TF,TR>[n]
  size_t args_bytes = 0;
  int2* d_items = nullptr;         // items grouped by class
  size_t items_cap = 0;
  int* d_ctr = nullptr;            // queue heads [kClasses]
  // per-panel arm (f32): each panel's prepared returns for the per-(date,
  // factor) path that the single-panel entry points take with F >= 2
  // (allocated by the first fcb_batch_run_per_panel)
  void* d_prep_mem = nullptr;
  std::vector<RicPrep> preps;
  int* d_status = nullptr;
  // f32 panels: descriptors, item offsets and fallback lists of every variant
  void* d_ric = nullptr;
  size_t ric_cap = 0;
  RicBatchVariant var[kRicVariants] = {};
  std::vector<FcWork> fcw;
  std::vector<void*> fc_mem;
  // factor_corr of every panel with an output, batched: panel descriptors,
  // the prefix offsets of each kind of grid, and the grid sizes
  FcBatchPanel* d_fcb = nullptr;
  int* d_fcb_off = nullptr;
  int fcb_np = 0;
  int fcb_total[kFcbGrids] = {};
  size_t fcb_gram_smem = 0;
  // current schedule
  int cls_off[kClasses] = {}, cls_cnt[kClasses] = {}, cls_maxN[kClasses] = {}, cls_grid[kClasses] = {};
  size_t cls_smem[kClasses] = {};
  double cls_work[kClasses] = {};
  cudaStream_t s[kClasses] = {};
  cudaEvent_t ev_fork = nullptr, ev_join[kClasses] = {}, ev_t0 = nullptr, ev_t1 = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool dirty = true;

  ~fcb_batch() { release(); }
  void drop_graph() {
    if (exec != nullptr) cudaGraphExecDestroy(exec);
    if (graph != nullptr) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
    dirty = true;
  }
  void release() {
    drop_graph();
    cudaFree(d_args);
    cudaFree(d_items);
    cudaFree(d_ctr);
    cudaFree(d_prep_mem);
    cudaFree(d_status);
    cudaFree(d_ric);
    d_ric = nullptr;
    ric_cap = 0;
    for (void* m : fc_mem) cudaFree(m);
    fc_mem.clear();
    cudaFree(d_fcb);
    cudaFree(d_fcb_off);
    d_fcb = nullptr;
    d_fcb_off = nullptr;
    fcb_np = 0;
    for (int k = 0; k < kClasses; ++k) {
      if (s[k] != nullptr) cudaStreamDestroy(s[k]);
      if (ev_join[k] != nullptr) cudaEventDestroy(ev_join[k]);
      s[k] = nullptr;
      ev_join[k] = nullptr;
    }
    if (ev_fork != nullptr) cudaEventDestroy(ev_fork);
    if (ev_t0 != nullptr) cudaEventDestroy(ev_t0);
    if (ev_t1 != nullptr) cudaEventDestroy(ev_t1);
    ev_fork = ev_t0 = ev_t1 = nullptr;
    d_args = nullptr;
    d_items = nullptr;
    d_ctr = nullptr;
    d_prep_mem = nullptr;
    d_status = nullptr;
  }
};

namespace {

int class_of(const fcb_batch& b, int N) {
  if (N <= b.cfg.nt_small_max) return 0;
  if (N <= b.cfg.nt_mid_max) return 1;
  return 2;
}

// Work estimate of one item: cells sorted (the F factor sorts plus the
// returns sort) -- what the queue order and the concurrent grid split use.
double item_work(const fcb_panel& p) { return static_cast<double>(p.N) * (p.F + 1); }

template <typename TF, typename TR>
int upload_args(fcb_batch& b) {
  std::vector<RankIcArgs<TF, TR>> a(b.p.size());
  for (size_t i = 0; i < b.p.size(); ++i) {
    const fcb_panel& q = b.p[i];
    RankIcArgs<TF, TR> r{};
    r.X = static_cast<const TF*>(q.X);
    r.R = static_cast<const TR*>(q.R);
    r.fmask = q.fmask;
    r.rmask = q.rmask;
    r.F = q.F;
    r.T = q.T;
    r.N = q.N;
    r.min_valid = b.min_valid;
    r.ranks_out = q.ranks_out;
    r.ic_out = q.ic_out;
    if (q.model != nullptr) {
      r.cdf_table = q.model->table[q.model->cur];
      r.cdf_zrange = q.model->zrange[q.model->cur];
    }
    r.learn_cap = b.cfg.learn_cap > 0 ? b.cfg.learn_cap : kLearnCapDefault;
    r.ic_ld = 0;
    a[i] = r;
  }
  const size_t bytes = a.size() * sizeof(RankIcArgs<TF, TR>);
  if (b.d_args == nullptr) FCB_BTRY(cudaMalloc(&b.d_args, bytes));
  b.args_bytes = bytes;
  FCB_BTRY(cudaMemcpy(b.d_args, a.data(), bytes, cudaMemcpyHostToDevice));
  return FCB_OK;
}

template <typename TF, typename TR>
int occupancy(const fcb_batch& b, int k, int* occ) {
  return rcode(launch_rank_ic_batch<TF, TR>(kClassNt[k], b.learned, static_cast<const RankIcArgs<TF, TR>*>(b.d_args),
                                            nullptr, 0, nullptr, 0, b.cls_smem[k], nullptr, nullptr, occ));
}

// f32 panels: the kernel variant of a panel of width N under the current
// configuration (a panel may be served by a wider variant than it needs).
int variant_of(const fcb_batch& b, int N) {
  if (N <= std::min(b.cfg.nt_small_max, ric_variant_cap(0))) return 0;
  if (N <= std::min(b.cfg.nt_mid_max, ric_variant_cap(1))) return 1;
  if (N <= ric_variant_cap(2)) return 2;
  return 3;
}

// f32 panels: per variant, the panel descriptors (order 1: widest work
// first), their date and section offsets and the fallback list, uploaded in
// one buffer.
int plan_items(fcb_batch& b) {
  std::vector<int> idx[kRicVariants];
  for (size_t i = 0; i < b.p.size(); ++i) idx[variant_of(b, b.p[i].N)].push_back(static_cast<int>(i));
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  size_t total = 0;
  size_t o_pan[kRicVariants], o_od[kRicVariants], o_oi[kRicVariants], o_cnt[kRicVariants], o_items[kRicVariants];
  long long ndates[kRicVariants] = {}, nitems[kRicVariants] = {};
  for (int k = 0; k < kRicVariants; ++k) {
    if (b.cfg.order == 1)
      std::stable_sort(idx[k].begin(), idx[k].end(), [&](int x, int y) {
        const fcb_panel &px = b.p[x], &py = b.p[y];
        return static_cast<double>(px.T) * px.F * px.N > static_cast<double>(py.T) * py.F * py.N;
      });
    for (int i : idx[k]) {
      ndates[k] += b.p[i].T;
      nitems[k] += static_cast<long long>(b.p[i].T) * b.p[i].F;
    }
    if (nitems[k] > 2147483647LL) return FCB_ERR_CAP3;
    const size_t np = idx[k].size();
    o_pan[k] = total;
    total += al(np * sizeof(RicPanel));
    o_od[k] = total;
    total += al(np * sizeof(int));
    o_oi[k] = total;
    total += al(np * sizeof(int));
    o_cnt[k] = total;
    total += 256;
    o_items[k] = total;
    total += al(static_cast<size_t>(nitems[k]) * sizeof(int));
  }
  if (b.ric_cap < total) {
    cudaFree(b.d_ric);
    b.d_ric = nullptr;
    b.ric_cap = 0;
    FCB_BTRY(cudaMalloc(&b.d_ric, total));
    b.ric_cap = total;
  }
  std::vector<uint8_t> host(total, 0);
  uint8_t* base = static_cast<uint8_t*>(b.d_ric);
  for (int k = 0; k < kRicVariants; ++k) {
    RicBatchVariant& v = b.var[k];
    v = RicBatchVariant{};
    v.np = static_cast<int>(idx[k].size());
    if (v.np == 0) continue;
    RicPanel* hp = reinterpret_cast<RicPanel*>(host.data() + o_pan[k]);
    int* hd = reinterpret_cast<int*>(host.data() + o_od[k]);
    int* hi = reinterpret_cast<int*>(host.data() + o_oi[k]);
    int od = 0, oi = 0;
    for (int j = 0; j < v.np; ++j) {
      const int i = idx[k][j];
      const fcb_panel& q = b.p[i];
      RankIcArgs<float, float> a{};
      a.X = static_cast<const float*>(q.X);
      a.R = static_cast<const float*>(q.R);
      a.fmask = q.fmask;
      a.rmask = q.rmask;
      a.F = q.F;
      a.T = q.T;
      a.N = q.N;
      a.min_valid = b.min_valid;
      a.ranks_out = q.ranks_out;
      a.ic_out = q.ic_out;
      if (q.model != nullptr) {
        a.cdf_table = q.model->table[q.model->cur];
        a.cdf_zrange = q.model->zrange[q.model->cur];
        v.learned = true;
      }
      a.learn_cap = b.cfg.learn_cap > 0 ? b.cfg.learn_cap : kLearnCapDefault;
      hp[j] = RicPanel{a, b.preps[i]};
      hd[j] = od;
      hi[j] = oi;
      od += q.T;
      oi += q.T * q.F;
      v.maxN = std::max(v.maxN, q.N);
    }
    v.dates = od;
    v.items = oi;
    v.panels = reinterpret_cast<const RicPanel*>(base + o_pan[k]);
    v.off_dates = reinterpret_cast<const int*>(base + o_od[k]);
    v.off_items = reinterpret_cast<const int*>(base + o_oi[k]);
    v.fb = RicList{reinterpret_cast<int*>(base + o_cnt[k]), reinterpret_cast<int*>(base + o_items[k])};
  }
  FCB_BTRY(cudaMemcpy(b.d_ric, host.data(), total, cudaMemcpyHostToDevice));
  return FCB_OK;
}

// Items, per-class shared memory and grids for the current configuration.
int plan(fcb_batch& b) {
  if (b.dtx == FCB_DTYPE_F32) return plan_items(b);
  std::vector<std::vector<int2>> items(kClasses);
  for (int k = 0; k < kClasses; ++k) {
    b.cls_maxN[k] = 0;
    b.cls_work[k] = 0.0;
  }
  for (size_t i = 0; i < b.p.size(); ++i) {
    const int k = class_of(b, b.p[i].N);
    b.cls_maxN[k] = std::max(b.cls_maxN[k], b.p[i].N);
    b.cls_work[k] += item_work(b.p[i]) * b.p[i].T;
    for (int t = 0; t < b.p[i].T; ++t) items[k].push_back(make_int2(static_cast<int>(i), t));
  }
  std::vector<int2> all;
  for (int k = 0; k < kClasses; ++k) {
    if (b.cfg.order == 1) {
      // longest items first; ties keep panel order then date order
      std::stable_sort(items[k].begin(), items[k].end(), [&](const int2& x, const int2& y) {
        return item_work(b.p[x.x]) > item_work(b.p[y.x]);
      });
    }
    b.cls_off[k] = static_cast<int>(all.size());
    b.cls_cnt[k] = static_cast<int>(items[k].size());
    all.insert(all.end(), items[k].begin(), items[k].end());
  }
  const size_t bytes = std::max<size_t>(1, all.size()) * sizeof(int2);
  if (b.items_cap < bytes) {
    cudaFree(b.d_items);
    b.d_items = nullptr;
    FCB_BTRY(cudaMalloc(&b.d_items, bytes));
    b.items_cap = bytes;
  }
  if (!all.empty()) FCB_BTRY(cudaMemcpy(b.d_items, all.data(), all.size() * sizeof(int2), cudaMemcpyHostToDevice));
  double wtot = 0.0;
  for (int k = 0; k < kClasses; ++k) wtot += b.cls_work[k];
  for (int k = 0; k < kClasses; ++k) {
    b.cls_grid[k] = 0;
    if (b.cls_cnt[k] == 0) continue;
    b.cls_smem[k] = (b.dtx == FCB_DTYPE_F32) ? rank_ic_batch_smem<float, float>(kClassNt[k], b.cls_maxN[k])
                                             : rank_ic_batch_smem<double, double>(kClassNt[k], b.cls_maxN[k]);
    if (b.cls_smem[k] > kMaxSmemPerBlock) return FCB_ERR_UNSUPPORTED;
    int occ = 0;
    const int r = (b.dtx == FCB_DTYPE_F32) ? occupancy<float, float>(b, k, &occ) : occupancy<double, double>(b, k, &occ);
    if (r != FCB_OK) return r;
    if (occ < 1) return FCB_ERR_UNSUPPORTED;
    if (b.cfg.ctas_per_sm > 0) occ = std::min(occ, b.cfg.ctas_per_sm);
    const int slots = occ * b.sms;
    int g = slots;
    if (b.cfg.concurrent && wtot > 0.0) g = static_cast<int>(std::lround(slots * b.cls_work[k] / wtot));
    b.cls_grid[k] = std::max(1, std::min(g, b.cls_cnt[k]));
  }
  return FCB_OK;
}

// Enqueue one whole batch on s0 (and the batch's side streams).
int enqueue(fcb_batch& b, cudaStream_t s0) {
  if (b.dtx != FCB_DTYPE_F32) FCB_BTRY(cudaMemsetAsync(b.d_ctr, 0, kClasses * sizeof(int), s0));
  FCB_BTRY(cudaEventRecord(b.ev_fork, s0));
  for (int k = 1; k < kClasses; ++k) FCB_BTRY(cudaStreamWaitEvent(b.s[k], b.ev_fork, 0));
  for (int k = 0; k < kRicVariants && b.dtx == FCB_DTYPE_F32; ++k) {
    if (b.var[k].np == 0) continue;
    cudaStream_t st = (b.cfg.concurrent && k > 0) ? b.s[std::min(k, kClasses - 1)] : s0;
    FCB_BTRY(launch_rank_ic_items_batch(k, b.var[k], st));
  }
  for (int k = 0; k < kClasses && b.dtx != FCB_DTYPE_F32; ++k) {
    if (b.cls_cnt[k] == 0) continue;
    cudaStream_t st = (b.cfg.concurrent && k > 0) ? b.s[k] : s0;
    const int2* items = b.d_items + b.cls_off[k];
    if (b.dtx == FCB_DTYPE_F32)
      FCB_BTRY(launch_rank_ic_batch<float, float>(kClassNt[k], b.learned,
                                                  static_cast<const RankIcArgs<float, float>*>(b.d_args), items,
                                                  b.cls_cnt[k], b.d_ctr + k, b.cls_grid[k], b.cls_smem[k],
                                                  b.d_status, st, nullptr));
    else
      FCB_BTRY(launch_rank_ic_batch<double, double>(kClassNt[k], false,
                                                    static_cast<const RankIcArgs<double, double>*>(b.d_args), items,
                                                    b.cls_cnt[k], b.d_ctr + k, b.cls_grid[k], b.cls_smem[k],
                                                    b.d_status, st, nullptr));
  }
  // factor_corr of every panel: one batched launch per kernel kind, on the
  // last branch, alongside the rank + IC kernels (it reads only the factor
  // planes and masks)
  if (b.fcb_np > 0)
    FCB_BTRY(launch_factor_corr_batch(b.d_fcb, b.fcb_np, b.d_fcb_off, b.fcb_total, b.dtx == FCB_DTYPE_F32 ? 0 : 1,
                                      b.fcb_gram_smem, b.s[kClasses - 1]));
  for (int k = 1; k < kClasses; ++k) {
    FCB_BTRY(cudaEventRecord(b.ev_join[k], b.s[k]));
    FCB_BTRY(cudaStreamWaitEvent(s0, b.ev_join[k], 0));
  }
  return FCB_OK;
}

int build_graph(fcb_batch& b) {
  b.drop_graph();
  int r = plan(b);
  if (r != FCB_OK) return r;
  // the scheduling knob learn_cap lives in the panel arguments (f32: in the
  // descriptors plan() uploaded)
  if (b.dtx != FCB_DTYPE_F32 && (r = upload_args<double, double>(b)) != FCB_OK) return r;
  FCB_BTRY(cudaStreamBeginCapture(b.s[0], cudaStreamCaptureModeRelaxed));
  r = enqueue(b, b.s[0]);
  cudaGraph_t g = nullptr;
  const cudaError_t ec = cudaStreamEndCapture(b.s[0], &g);
  if (r != FCB_OK) {
    if (g != nullptr) cudaGraphDestroy(g);
    return r;
  }
  FCB_BTRY(ec);
  b.graph = g;
  FCB_BTRY(cudaGraphInstantiate(&b.exec, b.graph, 0));
  b.dirty = false;
  return FCB_OK;
}

int bind_device(const fcb_batch& b) {
  int dev = -1;
  FCB_BTRY(cudaGetDevice(&dev));
  return dev == b.device ? FCB_OK : FCB_ERR_ARG;
}

// Resident CTAs per SM of the persistent kernel of block size nt with its
// shared memory sized for sections of N cells (0 when it does not fit).
int occ_at(const fcb_batch& b, int nt, int N, int* occ) {
  *occ = 0;
  const size_t smem = (b.dtx == FCB_DTYPE_F32) ? rank_ic_batch_smem<float, float>(nt, N)
                                               : rank_ic_batch_smem<double, double>(nt, N);
  if (smem > kMaxSmemPerBlock) return FCB_OK;
  if (b.dtx == FCB_DTYPE_F32)
    return rcode(launch_rank_ic_batch<float, float>(nt, b.learned,
                                                    static_cast<const RankIcArgs<float, float>*>(b.d_args), nullptr,
                                                    0, nullptr, 0, smem, nullptr, nullptr, occ));
  return rcode(launch_rank_ic_batch<double, double>(nt, false, static_cast<const RankIcArgs<double, double>*>(b.d_args),
                                                    nullptr, 0, nullptr, 0, smem, nullptr, nullptr, occ));
}

// Class boundaries worth measuring: for each occupancy level block size nt
// reaches on [lo, hi], the largest N that still keeps it.  A class sized for
// one cell more runs one resident CTA per SM fewer for all of its items.
int occupancy_cliffs(const fcb_batch& b, int nt, int lo, int hi, std::vector<int>* out) {
  int cur = std::max(1, lo);
  while (cur <= hi) {
    int o = 0;
    int r = occ_at(b, nt, cur, &o);
    if (r != FCB_OK) return r;
    if (o < 1) break;
    int a = cur, z = hi;  // occupancy does not grow with N: bisect for its last N
    while (a < z) {
      const int mid = a + (z - a + 1) / 2;
      int om = 0;
      if ((r = occ_at(b, nt, mid, &om)) != FCB_OK) return r;
      if (om >= o) a = mid; else z = mid - 1;
    }
    out->push_back(a);
    cur = a + 1;
  }
  return FCB_OK;
}

bool valid_cfg(const fcb_batch_config& c) {
  return c.nt_small_max >= 1 && c.nt_small_max <= 4096 && c.nt_mid_max > c.nt_small_max && c.nt_mid_max <= 8192 &&
         c.ctas_per_sm >= 0 && (c.concurrent == 0 || c.concurrent == 1) && (c.order == 0 || c.order == 1) &&
         c.learn_cap >= 0 && c.learn_cap <= 1024;
}

}  // namespace

extern "C" void fcb_batch_default_config(fcb_batch_config* cfg) {
  if (cfg == nullptr) return;
  cfg->nt_small_max = 4096;
  cfg->nt_mid_max = 8192;
  cfg->ctas_per_sm = 0;
  cfg->concurrent = 0;
  cfg->order = 1;
  cfg->learn_cap = kLearnCapDefault;
}

extern "C" int fcb_batch_create(const fcb_panel* panels, int npanels, int dtype_x, int dtype_r, int min_valid,
                                const fcb_batch_config* cfg, fcb_batch** out) {
  if (out == nullptr) return FCB_ERR_ARG;
  *out = nullptr;
  if (panels == nullptr || npanels < 1) return FCB_ERR_ARG;
  if (min_valid < 2) return FCB_ERR_CAP4;
  if (!((dtype_x == FCB_DTYPE_F32 && dtype_r == FCB_DTYPE_F32) ||
        (dtype_x == FCB_DTYPE_F64 && dtype_r == FCB_DTYPE_F64)))
    return FCB_ERR_UNSUPPORTED;
  bool learned = false;
  for (int i = 0; i < npanels; ++i) {
    const fcb_panel& q = panels[i];
    if (q.X == nullptr || q.R == nullptr || q.ic_out == nullptr || q.T < 1 || q.N < 1 || q.F < 1) return FCB_ERR_ARG;
    if (static_cast<long long>(q.T) * q.N > 2147483647LL) return FCB_ERR_CAP3;
    if (q.N > kSmemRankCap) return FCB_ERR_UNSUPPORTED;
    // the cross-section must fit one CTA's shared memory (largest block size)
    if (dtype_x == FCB_DTYPE_F32 ? !ric_items_fit(q.N)
                                 : rank_ic_batch_smem<double, double>(1024, q.N) > kMaxSmemPerBlock)
      return FCB_ERR_UNSUPPORTED;
    if (q.corr_out != nullptr && q.F > 128) return FCB_ERR_CAP3;
    if (q.model != nullptr) {
      if (dtype_x != FCB_DTYPE_F32 || q.model->F != q.F || q.model->table[q.model->cur] == nullptr)
        return FCB_ERR_ARG;
      learned = true;
    }
  }
  fcb_batch_config c;
  fcb_batch_default_config(&c);
  if (cfg != nullptr) c = *cfg;
  if (!valid_cfg(c)) return FCB_ERR_ARG;
  fcb_batch* b = new (std::nothrow) fcb_batch();
  if (b == nullptr) return FCB_ERR_ARG;
  b->p.assign(panels, panels + npanels);
  b->dtx = dtype_x;
  b->dtr = dtype_r;
  b->min_valid = min_valid;
  b->learned = learned;
  b->cfg = c;
  auto fail = [&](int r) {
    delete b;
    return r;
  };
  if (cudaGetDevice(&b->device) != cudaSuccess) return fail(FCB_ERR_ARG);
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, b->device) == cudaSuccess) b->sms = prop.multiProcessorCount;
  cudaError_t e = cudaSuccess;
  for (int k = 0; k < kClasses && e == cudaSuccess; ++k) {
    e = cudaStreamCreateWithFlags(&b->s[k], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_join[k], cudaEventDisableTiming);
  }
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreate(&b->ev_t0);
  if (e == cudaSuccess) e = cudaEventCreate(&b->ev_t1);
  if (e == cudaSuccess) e = cudaMalloc(&b->d_ctr, kClasses * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_status, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(b->d_status, 0, sizeof(int));
  if (e != cudaSuccess) return fail(rcode(e));
  // factor_corr work buffers: same row blocking as the single-panel entry point
  b->fcw.assign(npanels, FcWork{});
  for (int i = 0; i < npanels; ++i) {
    const fcb_panel& q = panels[i];
    if (q.corr_out == nullptr) continue;
    const long long R = static_cast<long long>(q.T) * q.N;
    const int F = q.F, Fp = (F + 3) / 4 * 4;
    FcWork& w = b->fcw[i];
    w.nblk_cols = static_cast<int>(std::min<long long>(592, std::max<long long>(1, R / 2048)));
    w.nblk_gram = fc_gram_blocks(R, F);
    const size_t b_colpart = static_cast<size_t>(w.nblk_cols) * F * sizeof(FcColPart);
    const size_t b_colstat = static_cast<size_t>(F) * sizeof(FcColStat);
    const size_t b_gram = static_cast<size_t>(w.nblk_gram) * 4 * Fp * Fp * sizeof(double);
    const size_t b_fb = static_cast<size_t>(F) * F * sizeof(int) + 16;
    const size_t b_part = fc_fb_part_doubles(R, F) * sizeof(double);
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t total = al(b_colpart) + al(b_colstat) + al(b_gram) + al(b_fb) + 256 + al(b_part);
    void* m = nullptr;
    e = cudaMalloc(&m, total);
    if (e != cudaSuccess) return fail(rcode(e));
    b->fc_mem.push_back(m);
    uint8_t* c8 = static_cast<uint8_t*>(m);
    w.colpart = reinterpret_cast<FcColPart*>(c8);
    c8 += al(b_colpart);
    w.colstat = reinterpret_cast<FcColStat*>(c8);
    c8 += al(b_colstat);
    w.gram = reinterpret_cast<double*>(c8);
    c8 += al(b_gram);
    w.fb_list = reinterpret_cast<int*>(c8);
    c8 += al(b_fb);
    w.fb_count = reinterpret_cast<int*>(c8);
    c8 += 256;
    w.fb_part = reinterpret_cast<double*>(c8);
  }
  {
    // batched factor_corr: descriptors and per-kind prefix offsets
    std::vector<FcBatchPanel> q;
    for (int i = 0; i < npanels; ++i) {
      const fcb_panel& p = panels[i];
      if (p.corr_out == nullptr) continue;
      q.push_back(fc_batch_panel(p.X, p.fmask, static_cast<long long>(p.T) * p.N, p.F, b->fcw[i], p.corr_out));
    }
    const int np = static_cast<int>(q.size());
    if (np > 0) {
      std::vector<int> off(static_cast<size_t>(kFcbGrids) * (np + 1), 0);
      for (int k = 0; k < np; ++k) {
        int blocks[kFcbGrids];
        fc_batch_grids(q[k], blocks);
        for (int g = 0; g < kFcbGrids; ++g)
          off[static_cast<size_t>(g) * (np + 1) + k + 1] = off[static_cast<size_t>(g) * (np + 1) + k] + blocks[g];
        b->fcb_gram_smem = std::max(b->fcb_gram_smem,
                                    fc_gram_smem(q[k].Fp, q[k].tasks_per_block, dtype_x == FCB_DTYPE_F32 ? 4 : 8));
      }
      for (int g = 0; g < kFcbGrids; ++g) b->fcb_total[g] = off[static_cast<size_t>(g) * (np + 1) + np];
      e = cudaMalloc(&b->d_fcb, q.size() * sizeof(FcBatchPanel));
      if (e == cudaSuccess) e = cudaMalloc(&b->d_fcb_off, off.size() * sizeof(int));
      if (e == cudaSuccess)
        e = cudaMemcpy(b->d_fcb, q.data(), q.size() * sizeof(FcBatchPanel), cudaMemcpyHostToDevice);
      if (e == cudaSuccess) e = cudaMemcpy(b->d_fcb_off, off.data(), off.size() * sizeof(int), cudaMemcpyHostToDevice);
      if (e != cudaSuccess) return fail(rcode(e));
      b->fcb_np = np;
    }
  }
  if (dtype_x == FCB_DTYPE_F32) {
    // prepared returns of every panel (ric_prep_bytes each, 256-byte aligned),
    // used by the batched launches and by the per-panel arm
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    size_t total = 0;
    for (const fcb_panel& q : b->p) total += al(ric_prep_bytes(q.T, q.N, q.F));
    e = cudaMalloc(&b->d_prep_mem, total);
    if (e != cudaSuccess) return fail(rcode(e));
    b->preps.resize(b->p.size());
    uint8_t* c8 = static_cast<uint8_t*>(b->d_prep_mem);
    for (size_t i = 0; i < b->p.size(); ++i) {
      b->preps[i] = ric_prep_carve(c8, b->p[i].T, b->p[i].N, b->p[i].F);
      c8 += al(ric_prep_bytes(b->p[i].T, b->p[i].N, b->p[i].F));
    }
  } else {
    const int r = upload_args<double, double>(*b);
    if (r != FCB_OK) return fail(r);
  }
  *out = b;
  return FCB_OK;
}

extern "C" void fcb_batch_destroy(fcb_batch* b) { delete b; }

extern "C" int fcb_batch_get_config(const fcb_batch* b, fcb_batch_config* cfg) {
  if (b == nullptr || cfg == nullptr) return FCB_ERR_ARG;
  *cfg = b->cfg;
  return FCB_OK;
}

extern "C" int fcb_batch_set_config(fcb_batch* b, const fcb_batch_config* cfg) {
  if (b == nullptr || cfg == nullptr || !valid_cfg(*cfg)) return FCB_ERR_ARG;
  b->cfg = *cfg;
  b->drop_graph();
  return FCB_OK;
}

extern "C" int fcb_batch_run(fcb_batch* b, void* stream) {
  if (b == nullptr) return FCB_ERR_ARG;
  int r = bind_device(*b);
  if (r != FCB_OK) return r;
  if (b->dirty) {
    r = build_graph(*b);
    if (r != FCB_OK) return r;
  }
  FCB_BTRY(cudaGraphLaunch(b->exec, static_cast<cudaStream_t>(stream)));
  return FCB_OK;
}

extern "C" int fcb_batch_run_per_panel(fcb_batch* b, void* stream) {
  if (b == nullptr) return FCB_ERR_ARG;
  int r = bind_device(*b);
  if (r != FCB_OK) return r;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  for (size_t i = 0; i < b->p.size(); ++i) {
    const fcb_panel& q = b->p[i];
    if (b->dtx == FCB_DTYPE_F32) {
      RankIcArgs<float, float> a{};
      a.X = static_cast<const float*>(q.X);
      a.R = static_cast<const float*>(q.R);
      a.fmask = q.fmask;
      a.rmask = q.rmask;
      a.F = q.F;
      a.T = q.T;
      a.N = q.N;
      a.min_valid = b->min_valid;
      a.ranks_out = q.ranks_out;
      a.ic_out = q.ic_out;
      const bool lrn = q.model != nullptr;
      if (lrn) {
        a.cdf_table = q.model->table[q.model->cur];
        a.cdf_zrange = q.model->zrange[q.model->cur];
        a.learn_cap = b->cfg.learn_cap > 0 ? b->cfg.learn_cap : kLearnCapDefault;
      }
      // as the single-panel entry points: several factors go through the
      // prepared returns and per-(date, factor) items, one factor per date
      if (a.F >= 2 && ric_items_fit(a.N))
        FCB_BTRY(launch_rank_ic_items(a, b->preps[i], lrn, s));
      else if (lrn)
        FCB_BTRY(launch_rank_ic_learned(a, b->d_status, s));
      else
        FCB_BTRY(launch_rank_ic<float, float>(a, b->d_status, s));
    } else {
      RankIcArgs<double, double> a{};
      a.X = static_cast<const double*>(q.X);
      a.R = static_cast<const double*>(q.R);
      a.fmask = q.fmask;
      a.rmask = q.rmask;
      a.F = q.F;
      a.T = q.T;
      a.N = q.N;
      a.min_valid = b->min_valid;
      a.ranks_out = q.ranks_out;
      a.ic_out = q.ic_out;
      FCB_BTRY(launch_rank_ic<double, double>(a, b->d_status, s));
    }
    if (q.corr_out != nullptr) {
      const long long R = static_cast<long long>(q.T) * q.N;
      FCB_BTRY(launch_factor_corr_strided(q.X, b->dtx, q.fmask, R, q.F, 1, R, b->fcw[i], q.corr_out, nullptr, s));
    }
  }
  return FCB_OK;
}

extern "C" int fcb_batch_status(fcb_batch* b) {
  if (b == nullptr) return FCB_ERR_ARG;
  FCB_BTRY(cudaDeviceSynchronize());
  int h = 0;
  FCB_BTRY(cudaMemcpy(&h, b->d_status, sizeof(int), cudaMemcpyDeviceToHost));
  FCB_BTRY(cudaMemset(b->d_status, 0, sizeof(int)));
  return h != 0 ? FCB_ERR_DEVICE_WAIT : FCB_OK;
}

namespace {

// Mean milliseconds of `reps` graph replays (after one warm-up replay).
int time_config(fcb_batch& b, int reps, float* ms) {
  int r = build_graph(b);
  if (r != FCB_OK) return r;
  FCB_BTRY(cudaGraphLaunch(b.exec, b.s[0]));
  FCB_BTRY(cudaEventRecord(b.ev_t0, b.s[0]));
  for (int i = 0; i < reps; ++i) FCB_BTRY(cudaGraphLaunch(b.exec, b.s[0]));
  FCB_BTRY(cudaEventRecord(b.ev_t1, b.s[0]));
  FCB_BTRY(cudaEventSynchronize(b.ev_t1));
  float t = 0.0f;
  FCB_BTRY(cudaEventElapsedTime(&t, b.ev_t0, b.ev_t1));
  *ms = t / reps;
  return FCB_OK;
}

// Batch signature for the tuning cache: dtypes, learned flag and, per
// default size class, the item count, largest N and total work (3 digits).
std::string signature(const fcb_batch& b) {
  fcb_batch_config d;
  fcb_batch_default_config(&d);
  long long cnt[kClasses] = {}, mx[kClasses] = {};
  double work[kClasses] = {};
  for (const fcb_panel& q : b.p) {
    const int k = q.N <= d.nt_small_max ? 0 : (q.N <= d.nt_mid_max ? 1 : 2);
    cnt[k] += q.T;
    mx[k] = std::max<long long>(mx[k], q.N);
    work[k] += item_work(q) * q.T;
  }
  char buf[512];
  int n = std::snprintf(buf, sizeof(buf), "fcb-batch-v3 n=%zu dt=%d/%d l=%d", b.p.size(), b.dtx, b.dtr,
                        b.learned ? 1 : 0);
  for (int k = 0; k < kClasses; ++k)
    n += std::snprintf(buf + n, sizeof(buf) - n, " c%d=%lld:%lld:%.3e", k, cnt[k], mx[k], work[k]);
  return std::string(buf);
}

bool cache_lookup(const char* path, const std::string& sig, fcb_batch_config* c, float* ms) {
  if (path == nullptr) return false;
  FILE* f = std::fopen(path, "r");
  if (f == nullptr) return false;
  char line[1024];
  bool found = false;
  while (std::fgets(line, sizeof(line), f) != nullptr) {
    const char* tab = std::strchr(line, '\t');
    if (tab == nullptr || static_cast<size_t>(tab - line) != sig.size() || std::strncmp(line, sig.c_str(), sig.size()) != 0)
      continue;
    fcb_batch_config t;
    float m = 0.0f;
    if (std::sscanf(tab + 1, "%d %d %d %d %d %d %f", &t.nt_small_max, &t.nt_mid_max, &t.ctas_per_sm, &t.concurrent,
                    &t.order, &t.learn_cap, &m) == 7 &&
        valid_cfg(t)) {
      *c = t;
      *ms = m;
      found = true;  // the last matching line wins
    }
  }
  std::fclose(f);
  return found;
}

void cache_store(const char* path, const std::string& sig, const fcb_batch_config& c, float ms) {
  if (path == nullptr) return;
  FILE* f = std::fopen(path, "a");
  if (f == nullptr) return;
  std::fprintf(f, "%s\t%d %d %d %d %d %d %.4f\n", sig.c_str(), c.nt_small_max, c.nt_mid_max, c.ctas_per_sm,
               c.concurrent, c.order, c.learn_cap, ms);
  std::fclose(f);
}

}  // namespace

extern "C" int fcb_batch_autotune(fcb_batch* b, int reps, const char* cache_path, fcb_batch_config* best_out,
                                  float* best_ms_out) {
  if (b == nullptr || reps < 1) return FCB_ERR_ARG;
  int r = bind_device(*b);
  if (r != FCB_OK) return r;
  const std::string sig = signature(*b);
  fcb_batch_config best;
  float best_ms = 0.0f;
  if (cache_lookup(cache_path, sig, &best, &best_ms)) {
    b->cfg = best;
    b->drop_graph();
    r = build_graph(*b);
    if (r != FCB_OK) return r;
    if (best_out != nullptr) *best_out = best;
    if (best_ms_out != nullptr) *best_ms_out = best_ms;
    return 1;  // taken from the cache
  }
  best = b->cfg;
  r = time_config(*b, reps, &best_ms);
  if (r != FCB_OK) return r;
  // coordinate descent over the knobs, each alternative tried once
  const int small_opts[] = {1024, 2048, 4096};
  const int cps_opts[] = {0, 1, 2};
  const int cap_opts[] = {64, 128, 256, 512};
  auto consider = [&](const fcb_batch_config& c) -> int {
    if (!valid_cfg(c)) return FCB_OK;
    b->cfg = c;
    float ms = 0.0f;
    const int rr = time_config(*b, reps, &ms);
    if (rr == FCB_ERR_UNSUPPORTED) return FCB_OK;  // e.g. a class that does not fit shared memory
    if (rr != FCB_OK) return rr;
    if (ms < best_ms) {
      best_ms = ms;
      best = c;
    }
    return FCB_OK;
  };
  for (int o = 0; o <= 1; ++o) {
    fcb_batch_config c = best;
    if (c.order == o) continue;
    c.order = o;
    if ((r = consider(c)) != FCB_OK) return r;
  }
  if (b->dtx == FCB_DTYPE_F32) {
    // f32: which kernel variant serves which widths (a narrow panel may run in
    // a wider variant), variants concurrent or in sequence, the bucket cap
    for (int v : {512, 1024, 2048}) {
      fcb_batch_config c = best;
      if (c.nt_small_max == v) continue;
      c.nt_small_max = v;
      if ((r = consider(c)) != FCB_OK) return r;
    }
    for (int v : {2048, 3072, 4096, 5120, 8192}) {
      fcb_batch_config c = best;
      if (c.nt_mid_max == v) continue;
      c.nt_mid_max = v;
      if ((r = consider(c)) != FCB_OK) return r;
    }
    for (int v = 0; v <= 1; ++v) {
      fcb_batch_config c = best;
      if (c.concurrent == v) continue;
      c.concurrent = v;
      if ((r = consider(c)) != FCB_OK) return r;
    }
    if (b->learned) {
      for (int v : cap_opts) {
        fcb_batch_config c = best;
        if (c.learn_cap == v) continue;
        c.learn_cap = v;
        if ((r = consider(c)) != FCB_OK) return r;
      }
    }
    b->cfg = best;
    b->drop_graph();
    r = build_graph(*b);
    if (r != FCB_OK) return r;
    cache_store(cache_path, sig, best, best_ms);
    if (best_out != nullptr) *best_out = best;
    if (best_ms_out != nullptr) *best_ms_out = best_ms;
    return FCB_OK;
  }
  // class boundaries: fixed steps plus the occupancy cliffs inside the
  // batch's range of section widths
  int nmin = 1 << 30, nmax = 0;
  for (const fcb_panel& q : b->p) {
    nmin = std::min(nmin, q.N);
    nmax = std::max(nmax, q.N);
  }
  std::vector<int> small_c(std::begin(small_opts), std::end(small_opts));
  if ((r = occupancy_cliffs(*b, 256, nmin, std::min(nmax, 4096), &small_c)) != FCB_OK) return r;
  std::sort(small_c.begin(), small_c.end());
  small_c.erase(std::unique(small_c.begin(), small_c.end()), small_c.end());
  for (int v : small_c) {
    fcb_batch_config c = best;
    if (c.nt_small_max == v) continue;
    c.nt_small_max = v;
    if ((r = consider(c)) != FCB_OK) return r;
  }
  std::vector<int> mid_c{8192};
  if ((r = occupancy_cliffs(*b, 512, best.nt_small_max + 1, std::min(nmax, 8192), &mid_c)) != FCB_OK) return r;
  std::sort(mid_c.begin(), mid_c.end());
  mid_c.erase(std::unique(mid_c.begin(), mid_c.end()), mid_c.end());
  for (int v : mid_c) {
    fcb_batch_config c = best;
    if (c.nt_mid_max == v) continue;
    c.nt_mid_max = v;
    if ((r = consider(c)) != FCB_OK) return r;
  }
  for (int v : cps_opts) {
    fcb_batch_config c = best;
    if (c.ctas_per_sm == v) continue;
    c.ctas_per_sm = v;
    if ((r = consider(c)) != FCB_OK) return r;
  }
  for (int v = 0; v <= 1; ++v) {
    fcb_batch_config c = best;
    if (c.concurrent == v) continue;
    c.concurrent = v;
    if ((r = consider(c)) != FCB_OK) return r;
  }
  if (b->learned) {
    for (int v : cap_opts) {
      fcb_batch_config c = best;
      if (c.learn_cap == v) continue;
      c.learn_cap = v;
      if ((r = consider(c)) != FCB_OK) return r;
    }
  }
  b->cfg = best;
  b->drop_graph();
  r = build_graph(*b);
  if (r != FCB_OK) return r;
  cache_store(cache_path, sig, best, best_ms);
  if (best_out != nullptr) *best_out = best;
  if (best_ms_out != nullptr) *best_ms_out = best_ms;
  return FCB_OK;
}
