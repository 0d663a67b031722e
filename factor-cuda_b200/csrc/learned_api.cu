// learned_api.cu -- C ABI for the learned-splitter (CDF network) path.
//
// A model holds one CDF network per factor (parameters + Adam state), the
// training samples of its last fit, and the tabulated monotone CDF the rank
// kernel consumes.  Fitting = features from exact ranks of earlier dates ->
// Adam steps (hand-written forward/backward kernels) -> tabulation.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/fcb200.h"
#include "fcb_kernels.h"

using namespace fcb;

#include "cdf_model.h"

namespace {

constexpr int kSamplesPerDate = 64;

// xorshift64* -- deterministic parameter initialisation from a seed
struct Rng {
  uint64_t s;
  explicit Rng(uint64_t seed) : s(seed ? seed : 0x9E3779B97F4A7C15ull) {}
  uint64_t next() {
    s ^= s >> 12;
    s ^= s << 25;
    s ^= s >> 27;
    return s * 2685821657736338717ull;
  }
  float uni(float a, float b) { return a + (b - a) * static_cast<float>((next() >> 40) * (1.0 / 16777216.0)); }
};

void init_params(std::vector<float>& p, int F, uint64_t seed) {
  constexpr int H = kCdfHidden;
  p.assign(static_cast<size_t>(F) * kCdfParams, 0.0f);
  for (int f = 0; f < F; ++f) {
    Rng r(seed * 1000003ull + static_cast<uint64_t>(f) + 1);
    float* q = p.data() + static_cast<size_t>(f) * kCdfParams;
    for (int j = 0; j < H; ++j) q[j] = r.uni(0.5f, 2.5f);             // W1 (positive slopes)
    for (int j = 0; j < H; ++j) q[H + j] = r.uni(-3.0f, 3.0f);        // b1 (spread of centres)
    for (int e = 0; e < H * H; ++e) q[2 * H + e] = r.uni(-0.3f, 0.3f);  // W2
    for (int i = 0; i < H; ++i) q[2 * H + H * H + i] = 0.0f;         // b2
    for (int i = 0; i < H; ++i) q[3 * H + H * H + i] = r.uni(-0.3f, 0.3f);  // w3
    q[4 * H + H * H] = 0.0f;                                           // b3
  }
}

int rc(cudaError_t e) { return static_cast<int>(e); }

#define FCB_TRY(...)                      \
  do {                                    \
    cudaError_t _e = (__VA_ARGS__);       \
    if (_e != cudaSuccess) return rc(_e); \
  } while (0)

}  // namespace

extern "C" fcb_cdf_model* fcb_cdf_model_create(int F, uint64_t seed) {
  if (F < 1 || F > 4096) return nullptr;
  fcb_cdf_model* m = new (std::nothrow) fcb_cdf_model();
  if (m == nullptr) return nullptr;
  m->F = F;
  if (cudaGetDevice(&m->device) != cudaSuccess) {
    delete m;
    return nullptr;
  }
  const size_t P = kCdfParams;
  bool ok = cudaMalloc(&m->params, F * P * 4) == cudaSuccess && cudaMalloc(&m->adam, F * 2 * P * 4) == cudaSuccess &&
            cudaMalloc(&m->table[0], static_cast<size_t>(F) * kCdfKnots * 4) == cudaSuccess &&
            cudaMalloc(&m->table[1], static_cast<size_t>(F) * kCdfKnots * 4) == cudaSuccess &&
            cudaMalloc(&m->zrange[0], F * 2 * 4) == cudaSuccess && cudaMalloc(&m->zrange[1], F * 2 * 4) == cudaSuccess &&
            cudaMalloc(&m->loss, F * 4) == cudaSuccess;
  std::vector<float> p;
  init_params(p, F, seed);
  ok = ok && cudaMemcpy(m->params, p.data(), p.size() * 4, cudaMemcpyHostToDevice) == cudaSuccess &&
       cudaMemset(m->adam, 0, F * 2 * P * 4) == cudaSuccess;
  std::vector<float> zr(static_cast<size_t>(F) * 2);
  std::vector<float> tab(static_cast<size_t>(F) * kCdfKnots);
  for (int f = 0; f < F; ++f) {
    zr[2 * f] = -4.0f;
    zr[2 * f + 1] = 4.0f;
    for (int k = 0; k < kCdfKnots; ++k) tab[static_cast<size_t>(f) * kCdfKnots + k] = k / float(kCdfKnots - 1);
  }
  for (int sl = 0; sl < 2; ++sl)
    ok = ok && cudaMemcpy(m->zrange[sl], zr.data(), zr.size() * 4, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(m->table[sl], tab.data(), tab.size() * 4, cudaMemcpyHostToDevice) == cudaSuccess;
  if (!ok) {
    fcb_cdf_model_destroy(m);
    return nullptr;
  }
  return m;
}

extern "C" void fcb_cdf_model_destroy(fcb_cdf_model* m) {
  if (m == nullptr) return;
  cudaFree(m->params);
  cudaFree(m->adam);
  for (int sl = 0; sl < 2; ++sl) {
    cudaFree(m->table[sl]);
    cudaFree(m->zrange[sl]);
  }
  cudaFree(m->loss);
  cudaFree(m->samples);
  delete m;
}

extern "C" int fcb_cdf_model_set_linear(fcb_cdf_model* m, int linear) {
  if (m == nullptr) return FCB_ERR_ARG;
  m->linear = linear ? 1 : 0;
  return FCB_OK;
}

namespace fcb {

cudaError_t cdf_model_features(fcb_cdf_model* m, const float* d_x, const float* d_ranks, int T, int N, int t0,
                               int tcount, cudaStream_t s) {
  const size_t need = static_cast<size_t>(tcount) * kSamplesPerDate;
  if (need > m->samp_cap) {
    cudaFree(m->samples);
    m->samples = nullptr;
    cudaError_t e = cudaMalloc(&m->samples, need * m->F * sizeof(float2));
    if (e != cudaSuccess) return e;
    m->samp_cap = need;
  }
  m->nsamp = static_cast<int>(need);
  return launch_cdf_features(d_x, d_ranks, m->F, T, N, t0, tcount, kSamplesPerDate, m->samples, s);
}

cudaError_t cdf_model_train_tabulate(fcb_cdf_model* m, int steps, float lr, int slot, cudaStream_t s) {
  if (steps > 0) {
    cudaError_t e = launch_cdf_train(m->params, m->adam, m->samples, m->F, m->nsamp, steps, lr, m->steps_done,
                                     m->loss, s);
    if (e != cudaSuccess) return e;
  }
  m->steps_done += steps;
  return launch_cdf_tabulate(m->params, m->samples, m->F, m->nsamp, m->zrange[slot], m->table[slot],
                             m->linear != 0, s);
}

}  // namespace fcb

extern "C" int fcb_cdf_model_fit(fcb_cdf_model* m, const float* d_x, const float* d_ranks, int T, int N, int t0,
                                 int tcount, int steps, float lr, void* stream) {
  if (m == nullptr || d_x == nullptr || d_ranks == nullptr || T < 1 || N < 1 || tcount < 1 || t0 < 0 ||
      t0 + tcount > T || steps < 0 || !(lr > 0.0f))
    return FCB_ERR_ARG;
  if (static_cast<long long>(T) * N > INT32_MAX) return FCB_ERR_CAP3;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  FCB_TRY(fcb::cdf_model_features(m, d_x, d_ranks, T, N, t0, tcount, s));
  FCB_TRY(fcb::cdf_model_train_tabulate(m, steps, lr, m->cur, s));
  return FCB_OK;
}

// Refits that overlap ranking: the samples are drawn on the ranking stream
// (they read the ranks just produced), the training and the tabulation run on
// another stream into the idle table slot, and the caller makes that slot
// current (fcb_cdf_model_swap) once the training stream has passed it.
extern "C" int fcb_cdf_model_sample(fcb_cdf_model* m, const float* d_x, const float* d_ranks, int T, int N, int t0,
                                    int tcount, void* stream) {
  if (m == nullptr || d_x == nullptr || d_ranks == nullptr || T < 1 || N < 1 || tcount < 1 || t0 < 0 ||
      t0 + tcount > T)
    return FCB_ERR_ARG;
  if (static_cast<long long>(T) * N > INT32_MAX) return FCB_ERR_CAP3;
  FCB_TRY(fcb::cdf_model_features(m, d_x, d_ranks, T, N, t0, tcount, static_cast<cudaStream_t>(stream)));
  return FCB_OK;
}

extern "C" int fcb_cdf_model_train(fcb_cdf_model* m, int steps, float lr, int into_idle, void* stream) {
  if (m == nullptr || steps < 0 || !(lr > 0.0f) || m->nsamp < 1) return FCB_ERR_ARG;
  FCB_TRY(fcb::cdf_model_train_tabulate(m, steps, lr, into_idle ? (m->cur ^ 1) : m->cur,
                                        static_cast<cudaStream_t>(stream)));
  return FCB_OK;
}

extern "C" int fcb_cdf_model_swap(fcb_cdf_model* m) {
  if (m == nullptr) return FCB_ERR_ARG;
  m->cur ^= 1;
  return FCB_OK;
}

extern "C" int fcb_cdf_model_state(const fcb_cdf_model* m, float* params, float* zrange, float* table, float* loss) {
  if (m == nullptr) return FCB_ERR_ARG;
  const size_t P = kCdfParams;
  if (params) FCB_TRY(cudaMemcpy(params, m->params, m->F * P * 4, cudaMemcpyDeviceToHost));
  if (zrange) FCB_TRY(cudaMemcpy(zrange, m->zrange[m->cur], m->F * 2 * 4, cudaMemcpyDeviceToHost));
  if (table)
    FCB_TRY(cudaMemcpy(table, m->table[m->cur], static_cast<size_t>(m->F) * kCdfKnots * 4, cudaMemcpyDeviceToHost));
  if (loss) FCB_TRY(cudaMemcpy(loss, m->loss, m->F * 4, cudaMemcpyDeviceToHost));
  return FCB_OK;
}

extern "C" int fcb_cdf_model_load(fcb_cdf_model* m, const float* params, const float* zrange, const float* table) {
  if (m == nullptr || params == nullptr || zrange == nullptr || table == nullptr) return FCB_ERR_ARG;
  const size_t P = kCdfParams;
  FCB_TRY(cudaMemcpy(m->params, params, m->F * P * 4, cudaMemcpyHostToDevice));
  FCB_TRY(cudaMemcpy(m->zrange[m->cur], zrange, m->F * 2 * 4, cudaMemcpyHostToDevice));
  FCB_TRY(cudaMemcpy(m->table[m->cur], table, static_cast<size_t>(m->F) * kCdfKnots * 4, cudaMemcpyHostToDevice));
  return FCB_OK;
}

extern "C" int fcb_cdf_grad(const float* params, const float* z, const float* u, int n, float* grad, float* loss) {
  if (params == nullptr || z == nullptr || u == nullptr || grad == nullptr || loss == nullptr || n < 1 || n > 256)
    return FCB_ERR_ARG;
  float *dp, *dz, *du, *dg, *dl;
  const size_t P = kCdfParams;
  FCB_TRY(cudaMalloc(&dp, P * 4 + 3 * 256 * 4 + P * 4 + 16));
  dz = dp + P;
  du = dz + 256;
  dg = du + 256;
  dl = dg + P;
  int r = 0;
  cudaError_t e = cudaMemcpy(dp, params, P * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dz, z, n * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(du, u, n * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = launch_cdf_grad(dp, dz, du, n, dg, dl, nullptr);
  if (e == cudaSuccess) e = cudaMemcpy(grad, dg, P * 4, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(loss, dl, 4, cudaMemcpyDeviceToHost);
  r = rc(e);
  cudaFree(dp);
  return r;
}

namespace fcb {
int rank_ic_learned_ld(const float* d_x, const float* d_r, const uint8_t* d_fmask, const uint8_t* d_rmask, int F,
                       int T, int N, int min_valid, float* d_ranks, double* d_ic, int ic_ld,
                       const fcb_cdf_model* model, int cap, int* d_stats, cudaStream_t stream);
}

extern "C" int fcb_dev_rank_ic_panel_learned(const float* d_x, const float* d_r, const uint8_t* d_fmask,
                                             const uint8_t* d_rmask, int F, int T, int N, int min_valid,
                                             float* d_ranks, double* d_ic, const fcb_cdf_model* model, int cap,
                                             int* d_stats, void* stream) {
  return fcb::rank_ic_learned_ld(d_x, d_r, d_fmask, d_rmask, F, T, N, min_valid, d_ranks, d_ic, 0, model, cap,
                                 d_stats, static_cast<cudaStream_t>(stream));
}

int fcb::rank_ic_learned_ld(const float* d_x, const float* d_r, const uint8_t* d_fmask, const uint8_t* d_rmask,
                            int F, int T, int N, int min_valid, float* d_ranks, double* d_ic, int ic_ld,
                            const fcb_cdf_model* model, int cap, int* d_stats, cudaStream_t stream) {
  if (d_x == nullptr || d_r == nullptr || d_ic == nullptr || model == nullptr || F < 1 || T < 1 || N < 1)
    return FCB_ERR_ARG;
  if (F != model->F) return FCB_ERR_ARG;
  if (min_valid < 2) return FCB_ERR_CAP4;
  if (static_cast<long long>(T) * N > INT32_MAX) return FCB_ERR_CAP3;
  if (N > (1 << 24)) return FCB_ERR_CAP2;
  int* d_status = nullptr;
  FCB_TRY(dev_status_sink(&d_status));
  RankIcArgs<float, float> a{d_x, d_r, d_fmask, d_rmask, F, T, N, min_valid, d_ranks, d_ic, nullptr, nullptr,
                             model->table[model->cur], model->zrange[model->cur], cap > 0 ? cap : kLearnCapDefault, d_stats,
                             ic_ld};
  if (F >= 2 && ric_items_fit(N)) {
    // several factors: returns prepared once per date, one CTA per (date, factor)
    void* prep = nullptr;
    FCB_TRY(scratch_alloc(&prep, ric_prep_bytes(T, N, F), stream));
    const cudaError_t e = launch_rank_ic_items(a, ric_prep_carve(prep, T, N, F), true, stream);
    FCB_TRY(scratch_free(prep, stream));
    return rc(e);
  }
  if (rank_ic_fits_smem<float, float>(N)) return rc(launch_rank_ic_learned(a, d_status, stream));
  // too wide for the shared-memory kernel: the global-memory radix path ranks
  // the section (identical results); statistics read outcome 0 (not learned)
  if (d_stats != nullptr)
    FCB_TRY(cudaMemsetAsync(d_stats, 0, static_cast<size_t>(F) * T * 4 * sizeof(int), stream));
  a.cdf_table = nullptr;
  a.cdf_zrange = nullptr;
  a.learn_stats = nullptr;
  const size_t bytes = rank_global_scratch(rank_global_bytes_per_date(2, N, F, 4, 4), T);
  void* scr = nullptr;
  FCB_TRY(scratch_alloc(&scr, bytes, stream));
  const cudaError_t e = launch_rank_ic_global<float, float>(a, static_cast<uint8_t*>(scr), bytes, stream);
  FCB_TRY(scratch_free(scr, stream));
  return rc(e);
}
