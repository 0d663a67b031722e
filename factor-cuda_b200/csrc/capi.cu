// capi.cu -- host drivers behind the C ABI (include/fcb200.h).
//
// Each entry point validates its arguments with the reference's status codes,
// acquires device buffers from a workspace arena (cached across calls when the
// caller passes a workspace, temporary otherwise), uploads, launches, downloads
// and synchronises.  Device buffers are accounted (live / high-water bytes),
// the equivalent of the reference's MemTracker (src/mem_tracker.cu:15-68).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <mutex>
#include <new>
#include <type_traits>
#include <vector>

#include "../../include/fcb200.h"
#include "cdf_model.h"
#include "fcb_kernels.h"

using namespace fcb;

// ---------------------------------------------------------------------------
// workspace arena
// ---------------------------------------------------------------------------
enum Slot : int {
  S_X = 0, S_X2, S_MASK, S_MASK2, S_OUT, S_OUT1, S_OUT2, S_OUT3, S_STATUS, S_IC, S_RF, S_RR,
  S_SC_RAW, S_SC_C, S_SC_M, S_SC_ST, S_SC_SUM, S_FB_LIST, S_FB_CNT,
  S_FC_COLPART, S_FC_COLSTAT, S_FC_GRAM, S_FC_FLAGS, S_FC_FBPART,
  S_PC_MU, S_PC_XH, S_PC_XM, S_PC_XL, S_PC_QH, S_PC_QM, S_PC_QL, S_PC_M16, S_PC_X32, S_PC_Q32, S_PC_M32, S_PC_TILES, S_PC_X, S_PC_MASK,
  S_PC_OUT, S_PC_CPART, S_GSCR, S_RICPREP, S_FCT_WORK,
  // streamed panel: three chunk buffers each (upload / compute / download in flight)
  S_PX0, S_PX1, S_PX2, S_PR0, S_PR1, S_PR2, S_PFM0, S_PFM1, S_PFM2, S_PRM0, S_PRM1, S_PRM2,
  S_PRK0, S_PRK1, S_PRK2, S_PIC,
  S_COUNT
};

// Streams: 0 compute (and every single-shot entry point), 1 uploads,
// 2 downloads, 3 background model refits.
struct fcb_workspace {
  static constexpr int kStreams = 4;
  int device = -1;
  cudaStream_t stream[kStreams] = {};
  void* ptr[S_COUNT] = {};
  size_t cap[S_COUNT] = {};
  uint64_t live = 0, peak = 0, nalloc = 0;
  // learned-splitter state carried across calls
  fcb_cdf_model* model = nullptr;
  bool model_ready = false;   // model->table[model->cur] holds a fitted table
  bool fit_inflight = false;  // a refit runs on stream 3
  int fit_slot = 0;           // table slot the in-flight refit writes
  int since_fit = 0;          // dates ranked since the last refit was scheduled
  int fits = 0;               // refits scheduled
  int learned_chunks = 0;     // chunks ranked by the learned kernel
  cudaEvent_t ev_fit = nullptr;

  cudaError_t bind() {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev != device) {
      release();
      device = dev;
    }
    for (int i = 0; i < kStreams; ++i)
      if (stream[i] == nullptr) {
        e = cudaStreamCreateWithFlags(&stream[i], cudaStreamNonBlocking);
        if (e != cudaSuccess) return e;
      }
    return cudaSuccess;
  }
  template <typename T>
  cudaError_t get(Slot s, size_t bytes, T** out) {
    if (bytes == 0) bytes = 16;
    if (cap[s] < bytes) {
      if (ptr[s] != nullptr) {
        cudaFree(ptr[s]);
        live -= cap[s];
        ptr[s] = nullptr;
        cap[s] = 0;
      }
      cudaError_t e = cudaMalloc(&ptr[s], bytes);
      if (e != cudaSuccess) {
        ptr[s] = nullptr;
        return e;
      }
      cap[s] = bytes;
      live += bytes;
      ++nalloc;
      if (live > peak) peak = live;
    }
    *out = static_cast<T*>(ptr[s]);
    return cudaSuccess;
  }
  // Poll the background refit; when it has finished, the rank kernels switch
  // to the freshly written table slot.
  void poll_fit() {
    if (fit_inflight && cudaEventQuery(ev_fit) == cudaSuccess) {
      model->cur = fit_slot;
      model_ready = true;
      fit_inflight = false;
    }
  }
  void drop_model() {
    if (stream[3] != nullptr) cudaStreamSynchronize(stream[3]);
    if (model != nullptr) fcb_cdf_model_destroy(model);
    model = nullptr;
    model_ready = fit_inflight = false;
    since_fit = 0;
  }
  void release() {
    drop_model();
    if (ev_fit != nullptr) cudaEventDestroy(ev_fit);
    ev_fit = nullptr;
    for (int s = 0; s < S_COUNT; ++s) {
      if (ptr[s] != nullptr) cudaFree(ptr[s]);
      ptr[s] = nullptr;
      cap[s] = 0;
    }
    for (int i = 0; i < kStreams; ++i) {
      if (stream[i] != nullptr) cudaStreamDestroy(stream[i]);
      stream[i] = nullptr;
    }
    live = 0;
  }
};

namespace {

// RAII: the caller's workspace, or a temporary one released on return.
struct WsScope {
  fcb_workspace* ws;
  fcb_workspace tmp;
  explicit WsScope(fcb_workspace* w) : ws(w != nullptr ? w : &tmp) {}
  ~WsScope() {
    if (ws == &tmp) tmp.release();
  }
};

inline int rc(cudaError_t e) { return static_cast<int>(e); }

#define FCB_TRY(...)                           \
  do {                                         \
    cudaError_t _e = (__VA_ARGS__);            \
    if (_e != cudaSuccess) return rc(_e);      \
  } while (0)

// Read and check the device status word after a synchronising copy.
int check_status(const int* h_status) { return *h_status != 0 ? FCB_ERR_DEVICE_WAIT : FCB_OK; }

bool is_group_whitelist(cudaError_t e) {
  return e == cudaErrorInvalidConfiguration || e == cudaErrorLaunchOutOfResources;
}


}  // namespace

// ---------------------------------------------------------------------------
// housekeeping
// ---------------------------------------------------------------------------
namespace fcb {
cudaError_t scratch_alloc(void** p, size_t bytes, cudaStream_t s) {
  static std::mutex mu;
  static cudaMemPool_t pools[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  cudaMemPool_t pool;
  {
    std::lock_guard<std::mutex> g(mu);
    if (pools[dev] == nullptr) {
      cudaMemPoolProps props{};
      props.allocType = cudaMemAllocationTypePinned;
      props.location.type = cudaMemLocationTypeDevice;
      props.location.id = dev;
      e = cudaMemPoolCreate(&pools[dev], &props);
      if (e != cudaSuccess) return e;
      uint64_t keep = ~0ull;  // keep freed blocks for the next call
      e = cudaMemPoolSetAttribute(pools[dev], cudaMemPoolAttrReleaseThreshold, &keep);
      if (e != cudaSuccess) return e;
    }
    pool = pools[dev];
  }
  return cudaMallocFromPoolAsync(p, bytes, pool, s);
}
cudaError_t scratch_free(void* p, cudaStream_t s) { return cudaFreeAsync(p, s); }

// Status word the asynchronous fcb_dev_* entry points hand to kernels with
// bounded waits: one per device, allocated and zeroed on the first call made
// with that device current; kernels only ever set it, fcb_dev_status reads and
// clears it.
cudaError_t dev_status_sink(int** out) {
  static std::mutex mu;
  static int* sinks[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> g(mu);
  if (sinks[dev] == nullptr) {
    int* p = nullptr;
    e = cudaMalloc(&p, 64);
    if (e != cudaSuccess) return e;
    e = cudaMemset(p, 0, 64);
    if (e != cudaSuccess) {
      cudaFree(p);
      return e;
    }
    sinks[dev] = p;
  }
  *out = sinks[dev];
  return cudaSuccess;
}
}  // namespace fcb

extern "C" fcb_workspace* fcb_workspace_create(void) { return new (std::nothrow) fcb_workspace(); }

extern "C" void fcb_workspace_clear(fcb_workspace* ws) {
  if (ws != nullptr) ws->release();
}

extern "C" void fcb_workspace_destroy(fcb_workspace* ws) {
  if (ws == nullptr) return;
  ws->release();
  delete ws;
}

extern "C" int fcb_workspace_stats(const fcb_workspace* ws, uint64_t* live, uint64_t* peak, uint64_t* n) {
  if (ws == nullptr) return FCB_ERR_ARG;
  if (live) *live = ws->live;
  if (peak) *peak = ws->peak;
  if (n) *n = ws->nalloc;
  return FCB_OK;
}

extern "C" int fcb_workspace_learned_state(const fcb_workspace* ws, int* ready, int* fits, int* learned_chunks) {
  if (ws == nullptr) return FCB_ERR_ARG;
  if (ready) *ready = ws->model_ready ? 1 : 0;
  if (fits) *fits = ws->fits;
  if (learned_chunks) *learned_chunks = ws->learned_chunks;
  return FCB_OK;
}

extern "C" int fcb_dev_status(void) {
  int* d = nullptr;
  FCB_TRY(dev_status_sink(&d));
  FCB_TRY(cudaDeviceSynchronize());
  int h = 0;
  FCB_TRY(cudaMemcpy(&h, d, sizeof(int), cudaMemcpyDeviceToHost));
  if (h == 0) return FCB_OK;
  FCB_TRY(cudaMemset(d, 0, sizeof(int)));
  return FCB_ERR_DEVICE_WAIT;
}

extern "C" int fcb_selftest_bounded_wait(int arrive, int max_polls) {
  if (max_polls < 1) return FCB_ERR_ARG;
  int* d = nullptr;
  FCB_TRY(cudaMalloc(&d, sizeof(int)));
  struct Free {
    int* p;
    ~Free() { cudaFree(p); }
  } fr{d};
  FCB_TRY(cudaMemset(d, 0, sizeof(int)));
  FCB_TRY(launch_wait_probe(arrive != 0, static_cast<uint32_t>(max_polls), d, nullptr));
  int h = 0;
  FCB_TRY(cudaMemcpy(&h, d, sizeof(int), cudaMemcpyDeviceToHost));
  return h != 0 ? FCB_ERR_DEVICE_WAIT : FCB_OK;
}

extern "C" int fcb_version(void) { return 10000; }

extern "C" int fcb_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
  return n;
}

extern "C" const char* fcb_status_string(int s) {
  switch (s) {
    case FCB_OK: return "ok";
    case FCB_ERR_ARG: return "null pointer or dimension < 1";
    case FCB_ERR_CAP2: return "size cap exceeded (-2)";
    case FCB_ERR_CAP3: return "size cap exceeded (-3)";
    case FCB_ERR_CAP4: return "domain / min_valid contract violated (-4)";
    case FCB_ERR_UNSUPPORTED: return "request not supported by this build";
    case FCB_ERR_NOALLOC_CAP: return "F above the no-allocation entry point's maximum (FCB_NOALLOC_MAX_F)";
    case FCB_ERR_DEVICE_WAIT: return "a bounded device-side wait gave up";
    default: return s > 0 ? cudaGetErrorString(static_cast<cudaError_t>(s)) : "contract error";
  }
}

extern "C" void* fcb_host_alloc(size_t bytes) {
  void* p = nullptr;
  if (cudaHostAlloc(&p, bytes, cudaHostAllocDefault) != cudaSuccess) return nullptr;
  return p;
}

extern "C" void fcb_host_free(void* p) {
  if (p != nullptr) cudaFreeHost(p);
}

// ---------------------------------------------------------------------------
// cs_rank
// ---------------------------------------------------------------------------
extern "C" int fcb_dev_cs_rank_f32(const float* d_x, const uint8_t* d_mask, int T, int N, int desc, float* d_out,
                                   void* stream) {
  if (d_x == nullptr || d_out == nullptr || T < 1 || N < 1) return FCB_ERR_ARG;
  if (N > (1 << 24)) return FCB_ERR_CAP2;
  if (static_cast<long long>(T) * N > INT32_MAX) return FCB_ERR_CAP3;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (N > kSmemRankCap) {
    // global-memory path; scratch is stream-ordered (no host synchronisation)
    const size_t bytes = rank_global_scratch(rank_global_bytes_per_date(0, N, 1, 4, 4), T);
    void* scr = nullptr;
    FCB_TRY(scratch_alloc(&scr, bytes, s));
    const cudaError_t e = launch_cs_rank_global(d_x, d_mask, T, N, desc, d_out, static_cast<uint8_t*>(scr), bytes, s);
    FCB_TRY(scratch_free(scr, s));
    return rc(e);
  }
  int* d_status;
  FCB_TRY(dev_status_sink(&d_status));
  return rc(launch_cs_rank(d_x, d_mask, T, N, desc, d_out, d_status, s));
}

extern "C" int fcb_cs_rank_f32(const float* x, const uint8_t* mask, int T, int N, int desc, float* out,
                               fcb_workspace* wsp) {
  if (x == nullptr || out == nullptr || T < 1 || N < 1) return FCB_ERR_ARG;
  if (N > (1 << 24)) return FCB_ERR_CAP2;
  if (static_cast<long long>(T) * N > INT32_MAX) return FCB_ERR_CAP3;
  WsScope sc(wsp);
  fcb_workspace& ws = *sc.ws;
  FCB_TRY(ws.bind());
  cudaStream_t s = ws.stream[0];
  const size_t n = static_cast<size_t>(T) * N;
  float *dx, *dout;
  uint8_t* dm = nullptr;
  int* dst;
  FCB_TRY(ws.get(S_X, n * 4, &dx));
  FCB_TRY(ws.get(S_OUT, n * 4, &dout));
  FCB_TRY(ws.get(S_STATUS, 64, &dst));
  if (mask != nullptr) FCB_TRY(ws.get(S_MASK, n, &dm));
  FCB_TRY(cudaMemcpyAsync(dx, x, n * 4, cudaMemcpyHostToDevice, s));
  if (mask != nullptr) FCB_TRY(cudaMemcpyAsync(dm, mask, n, cudaMemcpyHostToDevice, s));
  FCB_TRY(cudaMemsetAsync(dst, 0, sizeof(int), s));
  if (N > kSmemRankCap) {
    const size_t bytes = rank_global_scratch(rank_global_bytes_per_date(0, N, 1, 4, 4), T);
    uint8_t* scr;
    FCB_TRY(ws.get(S_GSCR, bytes, &scr));
    FCB_TRY(launch_cs_rank_global(dx, dm, T, N, desc, dout, scr, bytes, s));
  } else {
    FCB_TRY(launch_cs_rank(dx, dm, T, N, desc, dout, dst, s));
  }
  int hst = 0;
  FCB_TRY(cudaMemcpyAsync(out, dout, n * 4, cudaMemcpyDeviceToHost, s));
  FCB_TRY(cudaMemcpyAsync(&hst, dst, sizeof(int), cudaMemcpyDeviceToHost, s));
  FCB_TRY(cudaStreamSynchronize(s));
  return check_status(&hst);
}

// ---------------------------------------------------------------------------
// parameter_scan
// ---------------------------------------------------------------------------
extern "C" int fcb_parameter_scan_f32(const float* x, const uint8_t* mask, int T, int N, float* const out[4],
                                      int group_status[4], double time_ms[4], float time_gpu_ms[4],
                                      const int active[4], fcb_workspace* wsp) {
  if (group_status != nullptr)
    for (int g = 0; g < 4; ++g) group_status[g] = FCB_GROUP_NOT_EXECUTED;
  if (x == nullptr || out == nullptr || group_status == nullptr || T < 1 || N < 1) return FCB_ERR_ARG;
  int act[4];
  int nact = 0;
  for (int g = 0; g < 4; ++g) {
    act[g] = (active == nullptr || active[g]) ? 1 : 0;
    if (act[g] && out[g] == nullptr) return FCB_ERR_ARG;
    nact += act[g];
  }
  if (N > (1 << 24)) return FCB_ERR_CAP2;
  if (static_cast<long long>(T) * N > INT32_MAX) return FCB_ERR_CAP3;
  for (int g = 0; g < 4; ++g) {
    if (time_ms) time_ms[g] = 0.0;
    if (time_gpu_ms) time_gpu_ms[g] = 0.0f;
  }
  WsScope sc(wsp);
  fcb_workspace& ws = *sc.ws;
  FCB_TRY(ws.bind());
  cudaStream_t s = ws.stream[0];
  const size_t n = static_cast<size_t>(T) * N;
  float* dx;
  uint8_t* dm = nullptr;
  int* dst;
  FCB_TRY(ws.get(S_X, n * 4, &dx));
  FCB_TRY(ws.get(S_STATUS, 64, &dst));
  if (mask != nullptr) FCB_TRY(ws.get(S_MASK, n, &dm));
  ScanOut so{};
  const Slot oslot[4] = {S_OUT, S_OUT1, S_OUT2, S_OUT3};
  for (int g = 0; g < 4; ++g)
    if (act[g]) FCB_TRY(ws.get(oslot[g], n * 4, &so.out[g]));
  FCB_TRY(cudaMemcpyAsync(dx, x, n * 4, cudaMemcpyHostToDevice, s));
  if (mask != nullptr) FCB_TRY(cudaMemcpyAsync(dm, mask, n, cudaMemcpyHostToDevice, s));
  FCB_TRY(cudaMemsetAsync(dst, 0, sizeof(int), s));
  const bool global_path = N > kSmemRankCap;
  uint8_t* scr = nullptr;
  const size_t scr_bytes = rank_global_scratch(rank_global_bytes_per_date(1, N, 1, 4, 4), T);
  if (global_path) FCB_TRY(ws.get(S_GSCR, scr_bytes, &scr));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  FCB_TRY(cudaEventCreate(&e0));
  cudaError_t e = cudaEventCreate(&e1);
  if (e != cudaSuccess) {
    cudaEventDestroy(e0);
    return rc(e);
  }
  auto cleanup = [&]() {
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  };
  e = cudaEventRecord(e0, s);
  const auto t0 = std::chrono::steady_clock::now();
  cudaError_t le = (e != cudaSuccess) ? e
                   : global_path ? launch_param_scan_global(dx, dm, T, N, so, scr, scr_bytes, s)
                                 : launch_param_scan(dx, dm, T, N, so, dst, s);
  if (le != cudaSuccess) {
    cudaError_t se = cudaStreamSynchronize(s);
    cleanup();
    if (is_group_whitelist(le) && se == cudaSuccess) {
      for (int g = 0; g < 4; ++g)
        if (act[g]) group_status[g] = rc(le);
      return FCB_OK;  // every active group failed at launch; results None
    }
    return rc(le);
  }
  e = cudaEventRecord(e1, s);
  int hst = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&hst, dst, sizeof(int), cudaMemcpyDeviceToHost, s);
  for (int g = 0; g < 4 && e == cudaSuccess; ++g)
    if (act[g]) e = cudaMemcpyAsync(out[g], so.out[g], n * 4, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  const auto t1 = std::chrono::steady_clock::now();
  float gpu_ms = 0.0f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&gpu_ms, e0, e1);
  cleanup();
  if (e != cudaSuccess) return rc(e);
  if (hst != 0) return FCB_ERR_DEVICE_WAIT;
  const double host_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
  for (int g = 0; g < 4; ++g) {
    if (!act[g]) continue;
    group_status[g] = 0;
    if (time_ms) time_ms[g] = host_ms / nact;
    if (time_gpu_ms) time_gpu_ms[g] = gpu_ms / static_cast<float>(nact);
  }
  return FCB_OK;
}

extern "C" int fcb_dev_parameter_scan_f32(const float* d_x, const uint8_t* d_mask, int T, int N,
                                          float* const d_out[4], int group_status[4], const int active[4],
                                          void* stream) {
  if (group_status != nullptr)
    for (int g = 0; g < 4; ++g) group_status[g] = FCB_GROUP_NOT_EXECUTED;
  if (d_x == nullptr || d_out == nullptr || group_status == nullptr || T < 1 || N < 1) return FCB_ERR_ARG;
  int act[4];
  ScanOut so{};
  for (int g = 0; g < 4; ++g) {
    act[g] = (active == nullptr || active[g]) ? 1 : 0;
    if (act[g] && d_out[g] == nullptr) return FCB_ERR_ARG;
    so.out[g] = act[g] ? d_out[g] : nullptr;
  }
  if (N > (1 << 24)) return FCB_ERR_CAP2;
  if (static_cast<long long>(T) * N > INT32_MAX) return FCB_ERR_CAP3;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaError_t le;
  if (N > kSmemRankCap) {
    const size_t bytes = rank_global_scratch(rank_global_bytes_per_date(1, N, 1, 4, 4), T);
    void* scr = nullptr;
    FCB_TRY(scratch_alloc(&scr, bytes, s));
    le = launch_param_scan_global(d_x, d_mask, T, N, so, static_cast<uint8_t*>(scr), bytes, s);
    FCB_TRY(scratch_free(scr, s));
  } else {
    int* d_status;
    FCB_TRY(dev_status_sink(&d_status));
    le = launch_param_scan(d_x, d_mask, T, N, so, d_status, s);
  }
  if (le != cudaSuccess) {
    if (!is_group_whitelist(le)) return rc(le);
    for (int g = 0; g < 4; ++g)
      if (act[g]) group_status[g] = rc(le);
    return FCB_OK;  // every active group failed at launch; outputs untouched
  }
  for (int g = 0; g < 4; ++g)
    if (act[g]) group_status[g] = 0;
  return FCB_OK;
}

// ---------------------------------------------------------------------------
// rolling_ic (single factor) and the batched panel
// ---------------------------------------------------------------------------
template <typename TF, typename TR>
static int run_rank_ic(const RankIcArgs<TF, TR>& a, int* dst, cudaStream_t s, fcb_workspace& ws) {
  if constexpr (std::is_same<TF, float>::value && std::is_same<TR, float>::value) {
    if (a.F >= 2 && ric_items_fit(a.N) && a.rank_f_out == nullptr) {
      // several factors: returns prepared once per date, one CTA per (date, factor)
      void* prep;
      FCB_TRY(ws.get(S_RICPREP, ric_prep_bytes(a.T, a.N, a.F), &prep));
      return rc(launch_rank_ic_items(a, ric_prep_carve(prep, a.T, a.N, a.F), false, s));
    }
  }
  if (rank_ic_fits_smem<TF, TR>(a.N)) return rc(launch_rank_ic<TF, TR>(a, dst, s));
  const size_t bytes =
      rank_global_scratch(rank_global_bytes_per_date(2, a.N, a.F, sizeof(TF), sizeof(TR)), a.T);
  uint8_t* scr;
  FCB_TRY(ws.get(S_GSCR, bytes, &scr));
  return rc(launch_rank_ic_global<TF, TR>(a, scr, bytes, s));
}

extern "C" int fcb_rolling_ic(const void* f, int fdt, const void* r, int rdt, const uint8_t* fmask,
                              const uint8_t* rmask, int T, int N, int min_valid, double* ic, double* rank_f,
                              double* rank_r, fcb_workspace* wsp) {
  if (f == nullptr || r == nullptr || ic == nullptr || T < 1 || N < 1) return FCB_ERR_ARG;
  if ((rank_f == nullptr) != (rank_r == nullptr)) return FCB_ERR_ARG;
  if (min_valid < 2) return FCB_ERR_CAP4;
  if (static_cast<long long>(T) * N > INT32_MAX) return FCB_ERR_CAP3;
  if ((fdt != FCB_DTYPE_F32 && fdt != FCB_DTYPE_F64) || (rdt != FCB_DTYPE_F32 && rdt != FCB_DTYPE_F64))
    return FCB_ERR_ARG;
  WsScope sc(wsp);
  fcb_workspace& ws = *sc.ws;
  FCB_TRY(ws.bind());
  cudaStream_t s = ws.stream[0];
  const size_t n = static_cast<size_t>(T) * N;
  const size_t fsz = fdt == FCB_DTYPE_F32 ? 4 : 8, rsz = rdt == FCB_DTYPE_F32 ? 4 : 8;
  void *df, *dr;
  uint8_t *dfm = nullptr, *drm = nullptr;
  double *dic, *drf = nullptr, *drr = nullptr;
  int* dst;
  FCB_TRY(ws.get(S_X, n * fsz, &df));
  FCB_TRY(ws.get(S_X2, n * rsz, &dr));
  FCB_TRY(ws.get(S_IC, static_cast<size_t>(T) * 8, &dic));
  FCB_TRY(ws.get(S_STATUS, 64, &dst));
  if (fmask) FCB_TRY(ws.get(S_MASK, n, &dfm));
  if (rmask) FCB_TRY(ws.get(S_MASK2, n, &drm));
  if (rank_f) {
    FCB_TRY(ws.get(S_RF, n * 8, &drf));
    FCB_TRY(ws.get(S_RR, n * 8, &drr));
  }
  FCB_TRY(cudaMemcpyAsync(df, f, n * fsz, cudaMemcpyHostToDevice, s));
  FCB_TRY(cudaMemcpyAsync(dr, r, n * rsz, cudaMemcpyHostToDevice, s));
  if (fmask) FCB_TRY(cudaMemcpyAsync(dfm, fmask, n, cudaMemcpyHostToDevice, s));
  if (rmask) FCB_TRY(cudaMemcpyAsync(drm, rmask, n, cudaMemcpyHostToDevice, s));
  FCB_TRY(cudaMemsetAsync(dst, 0, sizeof(int), s));
  int e;
  if (fdt == FCB_DTYPE_F32 && rdt == FCB_DTYPE_F32)
    e = run_rank_ic(RankIcArgs<float, float>{static_cast<const float*>(df), static_cast<const float*>(dr), dfm, drm,
                                             1, T, N, min_valid, nullptr, dic, drf, drr},
                    dst, s, ws);
  else if (fdt == FCB_DTYPE_F32)
    e = run_rank_ic(RankIcArgs<float, double>{static_cast<const float*>(df), static_cast<const double*>(dr), dfm,
                                              drm, 1, T, N, min_valid, nullptr, dic, drf, drr},
                    dst, s, ws);
  else if (rdt == FCB_DTYPE_F32)
    e = run_rank_ic(RankIcArgs<double, float>{static_cast<const double*>(df), static_cast<const float*>(dr), dfm,
                                              drm, 1, T, N, min_valid, nullptr, dic, drf, drr},
                    dst, s, ws);
  else
    e = run_rank_ic(RankIcArgs<double, double>{static_cast<const double*>(df), static_cast<const double*>(dr),
                                               dfm, drm, 1, T, N, min_valid, nullptr, dic, drf, drr},
                    dst, s, ws);
  if (e != 0) return e;
  int hst = 0;
  FCB_TRY(cudaMemcpyAsync(ic, dic, static_cast<size_t>(T) * 8, cudaMemcpyDeviceToHost, s));
  if (rank_f) {
    FCB_TRY(cudaMemcpyAsync(rank_f, drf, n * 8, cudaMemcpyDeviceToHost, s));
    FCB_TRY(cudaMemcpyAsync(rank_r, drr, n * 8, cudaMemcpyDeviceToHost, s));
  }
  FCB_TRY(cudaMemcpyAsync(&hst, dst, sizeof(int), cudaMemcpyDeviceToHost, s));
  FCB_TRY(cudaStreamSynchronize(s));
  return check_status(&hst);
}

template <typename TF, typename TR>
static int dev_rank_ic(const RankIcArgs<TF, TR>& a, cudaStream_t s) {
  if (rank_ic_fits_smem<TF, TR>(a.N)) {
    int* d_status;
    FCB_TRY(dev_status_sink(&d_status));
    return rc(launch_rank_ic<TF, TR>(a, d_status, s));
  }
  const size_t bytes =
      rank_global_scratch(rank_global_bytes_per_date(2, a.N, a.F, sizeof(TF), sizeof(TR)), a.T);
  void* scr = nullptr;
  FCB_TRY(scratch_alloc(&scr, bytes, s));
  const cudaError_t e = launch_rank_ic_global<TF, TR>(a, static_cast<uint8_t*>(scr), bytes, s);
  FCB_TRY(scratch_free(scr, s));
  return rc(e);
}

extern "C" int fcb_dev_rolling_ic(const void* d_f, int fdt, const void* d_r, int rdt, const uint8_t* d_fmask,
                                  const uint8_t* d_rmask, int T, int N, int min_valid, double* d_ic,
                                  double* d_rank_f, double* d_rank_r, void* stream) {
  if (d_f == nullptr || d_r == nullptr || d_ic == nullptr || T < 1 || N < 1) return FCB_ERR_ARG;
  if ((d_rank_f == nullptr) != (d_rank_r == nullptr)) return FCB_ERR_ARG;
  if (min_valid < 2) return FCB_ERR_CAP4;
  if (static_cast<long long>(T) * N > INT32_MAX) return FCB_ERR_CAP3;
  if ((fdt != FCB_DTYPE_F32 && fdt != FCB_DTYPE_F64) || (rdt != FCB_DTYPE_F32 && rdt != FCB_DTYPE_F64))
    return FCB_ERR_ARG;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (fdt == FCB_DTYPE_F32 && rdt == FCB_DTYPE_F32)
    return dev_rank_ic(RankIcArgs<float, float>{static_cast<const float*>(d_f), static_cast<const float*>(d_r),
                                                d_fmask, d_rmask, 1, T, N, min_valid, nullptr, d_ic, d_rank_f,
                                                d_rank_r},
                       s);
  if (fdt == FCB_DTYPE_F32)
    return dev_rank_ic(RankIcArgs<float, double>{static_cast<const float*>(d_f), static_cast<const double*>(d_r),
                                                 d_fmask, d_rmask, 1, T, N, min_valid, nullptr, d_ic, d_rank_f,
                                                 d_rank_r},
                       s);
  if (rdt == FCB_DTYPE_F32)
    return dev_rank_ic(RankIcArgs<double, float>{static_cast<const double*>(d_f), static_cast<const float*>(d_r),
                                                 d_fmask, d_rmask, 1, T, N, min_valid, nullptr, d_ic, d_rank_f,
                                                 d_rank_r},
                       s);
  return dev_rank_ic(RankIcArgs<double, double>{static_cast<const double*>(d_f), static_cast<const double*>(d_r),
                                                d_fmask, d_rmask, 1, T, N, min_valid, nullptr, d_ic, d_rank_f,
                                                d_rank_r},
                     s);
}

static int panel_args_check(const void* x, const void* r, const double* ic, int F, int T, int N, int min_valid,
                            int method) {
  if (x == nullptr || r == nullptr || ic == nullptr || F < 1 || T < 1 || N < 1) return FCB_ERR_ARG;
  if (min_valid < 2) return FCB_ERR_CAP4;
  if (static_cast<long long>(T) * N > INT32_MAX) return FCB_ERR_CAP3;
  if (N > (1 << 24)) return FCB_ERR_CAP2;
  if (method != 0 && method != 1) return FCB_ERR_ARG;
  return FCB_OK;
}

extern "C" int fcb_dev_rank_ic_panel(const float* d_x, const float* d_r, const uint8_t* d_fmask,
                                     const uint8_t* d_rmask, int F, int T, int N, int min_valid, float* d_ranks,
                                     double* d_ic, int method, void* stream) {
  const int chk = panel_args_check(d_x, d_r, d_ic, F, T, N, min_valid, method);
  if (chk != FCB_OK) return chk;
  if (method != 0) return FCB_ERR_UNSUPPORTED;  // learned: fcb_dev_rank_ic_panel_learned (needs a model)
  int* d_status;
  FCB_TRY(dev_status_sink(&d_status));
  RankIcArgs<float, float> a{d_x, d_r, d_fmask, d_rmask, F, T, N, min_valid, d_ranks, d_ic, nullptr, nullptr};
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (F >= 2 && ric_items_fit(N)) {
    // several factors: returns prepared once per date, one CTA per (date, factor)
    void* prep = nullptr;
    FCB_TRY(scratch_alloc(&prep, ric_prep_bytes(T, N, F), s));
    const cudaError_t e = launch_rank_ic_items(a, ric_prep_carve(prep, T, N, F), false, s);
    FCB_TRY(scratch_free(prep, s));
    return rc(e);
  }
  if (rank_ic_fits_smem<float, float>(N)) return rc(launch_rank_ic<float, float>(a, d_status, s));
  // global-memory path; scratch is stream-ordered (no host synchronisation)
  const size_t bytes = rank_global_scratch(rank_global_bytes_per_date(2, N, F, 4, 4), T);
  void* scr = nullptr;
  FCB_TRY(scratch_alloc(&scr, bytes, s));
  const cudaError_t e = launch_rank_ic_global<float, float>(a, static_cast<uint8_t*>(scr), bytes, s);
  FCB_TRY(scratch_free(scr, s));
  return rc(e);
}

// Host panel: dates are streamed in chunks through three buffer sets so that
// the upload of chunk k+1, the kernel on chunk k and the download of chunk k-1
// run concurrently (stream 1 uploads, stream 0 computes, stream 2 downloads,
// ordered by events).
// method 1 (learned splitters): the workspace keeps a CDF model across calls.
// Until a fitted table exists, chunks are ranked by radix; after each chunk
// whose date count since the last refit reaches 250 (and after the first
// chunk of a fresh workspace), training samples are taken from that chunk's
// exact ranks on the compute stream and the refit (Adam + tabulation into the
// idle table slot) runs on stream 3 while ranking continues with the current
// slot; the host switches slots once the refit's event has completed.
extern "C" int fcb_rank_ic_panel(const float* x, const float* r, const uint8_t* fmask, const uint8_t* rmask,
                                 int F, int T, int N, int min_valid, float* ranks, double* ic, int method,
                                 fcb_workspace* wsp) {
  const int chk = panel_args_check(x, r, ic, F, T, N, min_valid, method);
  if (chk != FCB_OK) return chk;
  WsScope sc(wsp);
  fcb_workspace& ws = *sc.ws;
  FCB_TRY(ws.bind());
  constexpr int NB = 3;
  constexpr int kRefreshDates = 250;
  // chunk: about 64 MB of factor input per chunk, at least one date (measured
  // optimum of 24 / 40 / 64 / 96 / 160 MB at 1218 x 5000 x 12: larger chunks
  // lengthen the unoverlapped first upload and last download, smaller ones
  // add per-chunk gaps)
  const size_t per_date = static_cast<size_t>(F) * N * 4;
  int Tc = static_cast<int>((64ull << 20) / (per_date > 0 ? per_date : 1));
  if (Tc < 1) Tc = 1;
  if (Tc > T) Tc = T;
  // Chunk schedule: the first upload and the last compute + download overlap
  // nothing, so the chunks ramp up from Tc/8 at the start and back down to
  // Tc/8 at the end (Tc/8, Tc/4, Tc/2, Tc, ..., Tc, Tc/2, Tc/4, Tc/8) when the
  // panel is long enough; shorter panels take uniform chunks of Tc.
  std::vector<int> chunk_t0, chunk_tc;
  {
    const int r1 = std::max(1, Tc / 8), r2 = std::max(1, Tc / 4), r3 = std::max(1, Tc / 2);
    const int ramp = r1 + r2 + r3;
    std::vector<int> sizes;
    if (Tc >= 8 && T >= 2 * ramp + Tc) {
      sizes = {r1, r2, r3};
      int mid = T - 2 * ramp;
      while (mid > 0) {
        const int c = std::min(Tc, mid);
        sizes.push_back(c);
        mid -= c;
      }
      sizes.insert(sizes.end(), {r3, r2, r1});
    } else {
      for (int t = 0; t < T; t += Tc) sizes.push_back(std::min(Tc, T - t));
    }
    int t = 0;
    for (int c : sizes) {
      chunk_t0.push_back(t);
      chunk_tc.push_back(c);
      t += c;
    }
  }
  const int nchunk = static_cast<int>(chunk_tc.size());
  // learned splitters need a shared-memory kernel; wider sections are ranked
  // by the global-memory radix path (identical results)
  const bool learned = (method == 1) && (F >= 2 ? ric_items_fit(N) : rank_ic_fits_smem<float, float>(N));
  const bool need_ranks = ranks != nullptr || learned;
  float* dx[NB];
  float* dr[NB];
  uint8_t* dfm[NB] = {};
  uint8_t* drm[NB] = {};
  float* drk[NB] = {};
  double* dic;  // whole (F,T) IC panel, downloaded once at the end
  int* dst;
  const size_t cn = static_cast<size_t>(Tc) * N;
  FCB_TRY(ws.get(S_STATUS, 64, &dst));
  FCB_TRY(ws.get(S_PIC, static_cast<size_t>(F) * T * 8, &dic));
  for (int b = 0; b < NB; ++b) {
    FCB_TRY(ws.get(static_cast<Slot>(S_PX0 + b), cn * F * 4, &dx[b]));
    FCB_TRY(ws.get(static_cast<Slot>(S_PR0 + b), cn * 4, &dr[b]));
    if (fmask) FCB_TRY(ws.get(static_cast<Slot>(S_PFM0 + b), cn, &dfm[b]));
    if (rmask) FCB_TRY(ws.get(static_cast<Slot>(S_PRM0 + b), cn, &drm[b]));
    if (need_ranks) FCB_TRY(ws.get(static_cast<Slot>(S_PRK0 + b), cn * F * 4, &drk[b]));
  }
  cudaEvent_t ev_in[NB] = {}, ev_comp[NB] = {}, ev_out[NB] = {}, ev_feat = nullptr;
  struct Events {
    cudaEvent_t* a;
    cudaEvent_t* b;
    cudaEvent_t* c;
    cudaEvent_t& f;
    ~Events() {
      for (int i = 0; i < NB; ++i) {
        if (a[i]) cudaEventDestroy(a[i]);
        if (b[i]) cudaEventDestroy(b[i]);
        if (c[i]) cudaEventDestroy(c[i]);
      }
      if (f) cudaEventDestroy(f);
    }
  } evguard{ev_in, ev_comp, ev_out, ev_feat};
  for (int i = 0; i < NB; ++i) {
    FCB_TRY(cudaEventCreateWithFlags(&ev_in[i], cudaEventDisableTiming));
    FCB_TRY(cudaEventCreateWithFlags(&ev_comp[i], cudaEventDisableTiming));
    FCB_TRY(cudaEventCreateWithFlags(&ev_out[i], cudaEventDisableTiming));
  }
  if (learned) {
    if (ws.model != nullptr && ws.model->F != F) ws.drop_model();
    if (ws.model == nullptr) {
      ws.model = fcb_cdf_model_create(F, 20261203ull);
      if (ws.model == nullptr) return rc(cudaErrorMemoryAllocation);
    }
    if (ws.ev_fit == nullptr) FCB_TRY(cudaEventCreateWithFlags(&ws.ev_fit, cudaEventDisableTiming));
    FCB_TRY(cudaEventCreateWithFlags(&ev_feat, cudaEventDisableTiming));
  }
  cudaStream_t s_c = ws.stream[0], s_in = ws.stream[1], s_out = ws.stream[2], s_fit = ws.stream[3];
  FCB_TRY(cudaMemsetAsync(dst, 0, sizeof(int), s_c));
  for (int c = 0; c < nchunk; ++c) {
    const int j = c % NB;
    const int t0 = chunk_t0[c];
    const int tc = chunk_tc[c];
    const size_t cnn = static_cast<size_t>(tc) * N;
    if (c >= NB) FCB_TRY(cudaStreamWaitEvent(s_in, ev_out[j], 0));  // buffer set j drained
    // one strided copy moves this date range of all F factor panels
    FCB_TRY(cudaMemcpy2DAsync(dx[j], cnn * 4, x + static_cast<size_t>(t0) * N, static_cast<size_t>(T) * N * 4, cnn * 4,
                              F, cudaMemcpyHostToDevice, s_in));
    FCB_TRY(cudaMemcpyAsync(dr[j], r + static_cast<size_t>(t0) * N, cnn * 4, cudaMemcpyHostToDevice, s_in));
    if (fmask) FCB_TRY(cudaMemcpyAsync(dfm[j], fmask + static_cast<size_t>(t0) * N, cnn, cudaMemcpyHostToDevice, s_in));
    if (rmask) FCB_TRY(cudaMemcpyAsync(drm[j], rmask + static_cast<size_t>(t0) * N, cnn, cudaMemcpyHostToDevice, s_in));
    FCB_TRY(cudaEventRecord(ev_in[j], s_in));
    FCB_TRY(cudaStreamWaitEvent(s_c, ev_in[j], 0));
    if (learned) ws.poll_fit();
    if (learned && ws.model_ready) {
      const int e = fcb::rank_ic_learned_ld(dx[j], dr[j], dfm[j], drm[j], F, tc, N, min_valid, drk[j], dic + t0, T,
                                            ws.model, 0, nullptr, s_c);
      if (e != 0) return e;
      ++ws.learned_chunks;
    } else {
      RankIcArgs<float, float> a{dx[j], dr[j], dfm[j], drm[j], F, tc, N, min_valid, drk[j], dic + t0, nullptr, nullptr};
      a.ic_ld = T;
      const int e = run_rank_ic(a, dst, s_c, ws);
      if (e != 0) return e;
    }
    if (learned) {
      ws.since_fit += tc;
      if (!ws.fit_inflight && (!ws.model_ready || ws.since_fit >= kRefreshDates)) {
        FCB_TRY(fcb::cdf_model_features(ws.model, dx[j], drk[j], tc, N, 0, tc, s_c));
        FCB_TRY(cudaEventRecord(ev_feat, s_c));
        FCB_TRY(cudaStreamWaitEvent(s_fit, ev_feat, 0));
        ws.fit_slot = ws.model_ready ? (ws.model->cur ^ 1) : ws.model->cur;
        FCB_TRY(fcb::cdf_model_train_tabulate(ws.model, ws.model_ready ? 100 : 1500, ws.model_ready ? 1e-3f : 3e-3f,
                                              ws.fit_slot, s_fit));
        FCB_TRY(cudaEventRecord(ws.ev_fit, s_fit));
        ws.fit_inflight = true;
        ws.since_fit = 0;
        ++ws.fits;
      }
    }
    FCB_TRY(cudaEventRecord(ev_comp[j], s_c));
    FCB_TRY(cudaStreamWaitEvent(s_out, ev_comp[j], 0));
    if (ranks)
      FCB_TRY(cudaMemcpy2DAsync(ranks + static_cast<size_t>(t0) * N, static_cast<size_t>(T) * N * 4, drk[j], cnn * 4,
                                cnn * 4, F, cudaMemcpyDeviceToHost, s_out));
    FCB_TRY(cudaEventRecord(ev_out[j], s_out));
  }
  FCB_TRY(cudaStreamWaitEvent(s_out, ev_comp[(nchunk - 1) % NB], 0));
  FCB_TRY(cudaMemcpyAsync(ic, dic, static_cast<size_t>(F) * T * 8, cudaMemcpyDeviceToHost, s_out));
  int hst = 0;
  FCB_TRY(cudaStreamSynchronize(s_in));
  FCB_TRY(cudaStreamSynchronize(s_c));
  FCB_TRY(cudaStreamSynchronize(s_out));
  if (learned) ws.poll_fit();
  if (&ws == &sc.tmp) ws.drop_model();  // a temporary workspace waits for its refit
  FCB_TRY(cudaMemcpy(&hst, dst, sizeof(int), cudaMemcpyDeviceToHost));
  return check_status(&hst);
}

// ---------------------------------------------------------------------------
// correlations
// ---------------------------------------------------------------------------
static int stock_corr_check(const void* x, int dtype, const void* out, int T, int N) {
  if (x == nullptr || out == nullptr || T < 1 || N < 1) return FCB_ERR_ARG;
  if (dtype != FCB_DTYPE_F32 && dtype != FCB_DTYPE_F64) return FCB_ERR_ARG;
  if (static_cast<long long>(T) * N > INT32_MAX) return FCB_ERR_CAP2;
  if (static_cast<long long>(N) * N > INT32_MAX) return FCB_ERR_CAP3;
  return FCB_OK;
}

extern "C" int fcb_dev_stock_corr(const void* d_x, int dtype, const uint8_t* d_mask, int T, int N, double* d_out,
                                  int* selected_path, int* fallback_count, fcb_workspace* wsp, void* stream) {
  const int chk = stock_corr_check(d_x, dtype, d_out, T, N);
  if (chk != FCB_OK) return chk;
  if (wsp == nullptr) return FCB_ERR_ARG;  // scratch comes from a caller-held workspace
  fcb_workspace& ws = *wsp;
  FCB_TRY(ws.bind());
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int Tp = (T + 31) / 32 * 32;
  double *xraw, *xc, *mc, *sum;
  ColStat* st;
  int *fbl, *fbc;
  FCB_TRY(ws.get(S_SC_RAW, static_cast<size_t>(N) * Tp * 8, &xraw));
  FCB_TRY(ws.get(S_SC_C, static_cast<size_t>(N) * Tp * 8, &xc));
  FCB_TRY(ws.get(S_SC_M, static_cast<size_t>(N) * Tp * 8, &mc));
  FCB_TRY(ws.get(S_SC_ST, static_cast<size_t>(N) * sizeof(ColStat), &st));
  FCB_TRY(ws.get(S_SC_SUM, 64, &sum));
  const size_t upper = static_cast<size_t>(N) * (N - 1) / 2;
  FCB_TRY(ws.get(S_FB_LIST, (upper > 0 ? upper : 1) * 4, &fbl));
  FCB_TRY(ws.get(S_FB_CNT, 64, &fbc));
  FCB_TRY(launch_stock_corr_prep(d_x, dtype, d_mask, T, N, Tp, xraw, xc, mc, st, sum, s));
  // the domain check and the path flag are read on the host before the Gram pass
  double hs[3];
  FCB_TRY(cudaMemcpyAsync(hs, sum, sizeof(hs), cudaMemcpyDeviceToHost, s));
  FCB_TRY(cudaStreamSynchronize(s));
  if (hs[0] > 1e150 || hs[1] < 1e-150) return FCB_ERR_CAP4;
  if (selected_path) *selected_path = hs[2] != 0.0 ? 0 : 1;
  FCB_TRY(cudaMemsetAsync(fbc, 0, sizeof(int), s));
  FCB_TRY(launch_stock_corr_gram(xraw, xc, mc, st, T, N, Tp, d_out, fbl, fbc, s));
  int hfb = 0;
  FCB_TRY(cudaMemcpyAsync(&hfb, fbc, sizeof(int), cudaMemcpyDeviceToHost, s));
  FCB_TRY(cudaStreamSynchronize(s));
  if (fallback_count) *fallback_count = hfb;
  return FCB_OK;
}

extern "C" int fcb_stock_corr(const void* x, int dtype, const uint8_t* mask, int T, int N, double* out,
                              int* selected_path, int* fallback_count) {
  const int chk = stock_corr_check(x, dtype, out, T, N);
  if (chk != FCB_OK) return chk;
  fcb_workspace ws;
  struct Rel {
    fcb_workspace& w;
    ~Rel() { w.release(); }
  } rel{ws};
  FCB_TRY(ws.bind());
  cudaStream_t s = ws.stream[0];
  const size_t n = static_cast<size_t>(T) * N;
  const size_t esz = dtype == FCB_DTYPE_F32 ? 4 : 8;
  void* dx;
  uint8_t* dm = nullptr;
  double* dout;
  FCB_TRY(ws.get(S_X, n * esz, &dx));
  if (mask) FCB_TRY(ws.get(S_MASK, n, &dm));
  FCB_TRY(ws.get(S_OUT, static_cast<size_t>(N) * N * 8, &dout));
  FCB_TRY(cudaMemcpyAsync(dx, x, n * esz, cudaMemcpyHostToDevice, s));
  if (mask) FCB_TRY(cudaMemcpyAsync(dm, mask, n, cudaMemcpyHostToDevice, s));
  const int e = fcb_dev_stock_corr(dx, dtype, dm, T, N, dout, selected_path, fallback_count, &ws, s);
  if (e != FCB_OK) return e;
  FCB_TRY(cudaMemcpyAsync(out, dout, static_cast<size_t>(N) * N * 8, cudaMemcpyDeviceToHost, s));
  FCB_TRY(cudaStreamSynchronize(s));
  return FCB_OK;
}

extern "C" int fcb_dev_corr_domain(const void* d_x, int dtype, const uint8_t* d_mask, int T, int N, int F,
                                   int planes, int* in_domain, void* stream) {
  if (d_x == nullptr || in_domain == nullptr || T < 1 || N < 1 || F < 1) return FCB_ERR_ARG;
  if (dtype != FCB_DTYPE_F32 && dtype != FCB_DTYPE_F64) return FCB_ERR_ARG;
  if (planes != 0 && planes != 1) return FCB_ERR_ARG;
  if (static_cast<long long>(T) * N > INT32_MAX) return FCB_ERR_CAP2;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const long long R = static_cast<long long>(T) * N;
  void* scr = nullptr;
  FCB_TRY(scratch_alloc(&scr, 16, s));
  unsigned long long* d_ext = static_cast<unsigned long long*>(scr);
  unsigned long long h_ext[2] = {0ull, 0ull};
  cudaError_t e = launch_corr_domain(d_x, dtype, d_mask, R, F, planes, d_ext, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(h_ext, d_ext, sizeof(h_ext), cudaMemcpyDeviceToHost, s);
  const cudaError_t fe = scratch_free(scr, s);
  if (e == cudaSuccess) e = fe;
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return rc(e);
  double mx, mn;
  std::memcpy(&mx, &h_ext[0], 8);
  std::memcpy(&mn, &h_ext[1], 8);
  *in_domain = (mx <= 1e150 && mn >= 1e-150) ? 1 : 0;
  return FCB_OK;
}

extern "C" int fcb_dev_factor_corr(const void* d_x, int dtype, const uint8_t* d_mask, int T, int N, int F,
                                   int planes, double* d_out, fcb_workspace* wsp, void* stream) {
  if (d_x == nullptr || d_out == nullptr || T < 1 || N < 1 || F < 1) return FCB_ERR_ARG;
  if (dtype != FCB_DTYPE_F32 && dtype != FCB_DTYPE_F64) return FCB_ERR_ARG;
  if (planes != 0 && planes != 1) return FCB_ERR_ARG;
  if (static_cast<long long>(T) * N > INT32_MAX) return FCB_ERR_CAP2;
  if (F > 128) return FCB_ERR_CAP3;
  if (wsp == nullptr) return FCB_ERR_ARG;  // scratch comes from a caller-held workspace
  fcb_workspace& ws = *wsp;
  FCB_TRY(ws.bind());
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const long long R = static_cast<long long>(T) * N;
  const int Fp = (F + 3) / 4 * 4;
  FcWork w{};
  w.nblk_cols = static_cast<int>(std::min<long long>(592, std::max<long long>(1, R / 2048)));
  w.nblk_gram = fc_gram_blocks(R, F);
  FCB_TRY(ws.get(S_FC_COLPART, static_cast<size_t>(w.nblk_cols) * F * sizeof(FcColPart), &w.colpart));
  FCB_TRY(ws.get(S_FC_COLSTAT, static_cast<size_t>(F) * sizeof(FcColStat), &w.colstat));
  FCB_TRY(ws.get(S_FC_GRAM, static_cast<size_t>(w.nblk_gram) * 4 * Fp * Fp * 8, &w.gram));
  FCB_TRY(ws.get(S_FB_LIST, static_cast<size_t>(F) * F * 4, &w.fb_list));
  FCB_TRY(ws.get(S_FB_CNT, 64, &w.fb_count));
  FCB_TRY(ws.get(S_FC_FBPART, fc_fb_part_doubles(R, F) * sizeof(double), &w.fb_part));
  return rc(launch_factor_corr_strided(d_x, dtype, d_mask, R, F, planes ? 1 : F, planes ? R : 1, w, d_out, nullptr, s));
}

extern "C" int fcb_factor_corr(const void* x, int dtype, const uint8_t* mask, int T, int N, int F, double* out,
                               uint8_t* fallback_out) {
  if (x == nullptr || out == nullptr || T < 1 || N < 1 || F < 1) return FCB_ERR_ARG;
  if (dtype != FCB_DTYPE_F32 && dtype != FCB_DTYPE_F64) return FCB_ERR_ARG;
  if (static_cast<long long>(T) * N > INT32_MAX) return FCB_ERR_CAP2;
  if (F > 128) return FCB_ERR_CAP3;
  fcb_workspace ws;
  struct Rel {
    fcb_workspace& w;
    ~Rel() { w.release(); }
  } rel{ws};
  FCB_TRY(ws.bind());
  cudaStream_t s = ws.stream[0];
  const long long R = static_cast<long long>(T) * N;
  const int Fp = (F + 3) / 4 * 4;
  const size_t esz = dtype == FCB_DTYPE_F32 ? 4 : 8;
  FcWork w{};
  w.nblk_cols = static_cast<int>(std::min<long long>(592, std::max<long long>(1, R / 2048)));
  w.nblk_gram = fc_gram_blocks(R, F);
  void* dx;
  uint8_t* dm = nullptr;
  double* dout;
  uint8_t* dflags = nullptr;
  FCB_TRY(ws.get(S_X, static_cast<size_t>(R) * F * esz, &dx));
  if (mask) FCB_TRY(ws.get(S_MASK, static_cast<size_t>(R), &dm));
  FCB_TRY(ws.get(S_FC_COLPART, static_cast<size_t>(w.nblk_cols) * F * sizeof(FcColPart), &w.colpart));
  FCB_TRY(ws.get(S_FC_COLSTAT, static_cast<size_t>(F) * sizeof(FcColStat), &w.colstat));
  FCB_TRY(ws.get(S_FC_GRAM, static_cast<size_t>(w.nblk_gram) * 4 * Fp * Fp * 8, &w.gram));
  FCB_TRY(ws.get(S_FB_LIST, static_cast<size_t>(F) * F * 4, &w.fb_list));
  FCB_TRY(ws.get(S_FB_CNT, 64, &w.fb_count));
  FCB_TRY(ws.get(S_FC_FBPART, fc_fb_part_doubles(R, F) * sizeof(double), &w.fb_part));
  FCB_TRY(ws.get(S_OUT, static_cast<size_t>(F) * F * 8, &dout));
  if (fallback_out) {
    FCB_TRY(ws.get(S_FC_FLAGS, static_cast<size_t>(F) * F, &dflags));
    FCB_TRY(cudaMemsetAsync(dflags, 0, static_cast<size_t>(F) * F, s));
  }
  FCB_TRY(cudaMemcpyAsync(dx, x, static_cast<size_t>(R) * F * esz, cudaMemcpyHostToDevice, s));
  if (mask) FCB_TRY(cudaMemcpyAsync(dm, mask, static_cast<size_t>(R), cudaMemcpyHostToDevice, s));
  FCB_TRY(launch_factor_corr(dx, dtype, dm, R, F, w, dout, dflags, s));
  FCB_TRY(cudaMemcpyAsync(out, dout, static_cast<size_t>(F) * F * 8, cudaMemcpyDeviceToHost, s));
  if (fallback_out)
    FCB_TRY(cudaMemcpyAsync(fallback_out, dflags, static_cast<size_t>(F) * F, cudaMemcpyDeviceToHost, s));
  FCB_TRY(cudaStreamSynchronize(s));
  return FCB_OK;
}

// ---------------------------------------------------------------------------
// factor_corr precision form (BF16x3 tensor cores, FP64 finalize)
// ---------------------------------------------------------------------------
extern "C" int fcb_dev_factor_corr_bf16x3(const float* d_x, const uint8_t* d_mask, int T, int N, int F, int planes,
                                          double* d_out, fcb_workspace* wsp, void* stream) {
  if (d_x == nullptr || d_out == nullptr || T < 1 || N < 1 || F < 1) return FCB_ERR_ARG;
  if (planes != 0 && planes != 1) return FCB_ERR_ARG;
  if (static_cast<long long>(T) * N > INT32_MAX) return FCB_ERR_CAP2;
  if (F > 128) return FCB_ERR_CAP3;
  if (F > kFcTcMaxF) return FCB_ERR_UNSUPPORTED;
  if (wsp == nullptr) return FCB_ERR_ARG;  // scratch comes from a caller-held workspace
  fcb_workspace& ws = *wsp;
  FCB_TRY(ws.bind());
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const long long R = static_cast<long long>(T) * N;
  void* work;
  int* d_status;
  FCB_TRY(ws.get(S_FCT_WORK, fc_tc_work_bytes(F), &work));
  FCB_TRY(dev_status_sink(&d_status));
  return rc(launch_factor_corr_bf16x3(d_x, d_mask, R, F, planes ? 1 : F, planes ? R : 1, work, d_out, d_status, s));
}

extern "C" int fcb_factor_corr_bf16x3(const float* x, const uint8_t* mask, int T, int N, int F, double* out,
                                      fcb_workspace* wsp) {
  if (x == nullptr || out == nullptr || T < 1 || N < 1 || F < 1) return FCB_ERR_ARG;
  if (static_cast<long long>(T) * N > INT32_MAX) return FCB_ERR_CAP2;
  if (F > 128) return FCB_ERR_CAP3;
  if (F > kFcTcMaxF) return FCB_ERR_UNSUPPORTED;
  WsScope sc(wsp);
  fcb_workspace& ws = *sc.ws;
  FCB_TRY(ws.bind());
  cudaStream_t s = ws.stream[0];
  const long long R = static_cast<long long>(T) * N;
  float* dx;
  uint8_t* dm = nullptr;
  double* dout;
  void* work;
  int* dst;
  FCB_TRY(ws.get(S_X, static_cast<size_t>(R) * F * 4, &dx));
  if (mask) FCB_TRY(ws.get(S_MASK, static_cast<size_t>(R), &dm));
  FCB_TRY(ws.get(S_OUT, static_cast<size_t>(F) * F * 8, &dout));
  FCB_TRY(ws.get(S_FCT_WORK, fc_tc_work_bytes(F), &work));
  FCB_TRY(ws.get(S_STATUS, 64, &dst));
  FCB_TRY(cudaMemsetAsync(dst, 0, sizeof(int), s));
  FCB_TRY(cudaMemcpyAsync(dx, x, static_cast<size_t>(R) * F * 4, cudaMemcpyHostToDevice, s));
  if (mask) FCB_TRY(cudaMemcpyAsync(dm, mask, static_cast<size_t>(R), cudaMemcpyHostToDevice, s));
  FCB_TRY(launch_factor_corr_bf16x3(dx, dm, R, F, F, 1, work, dout, dst, s));
  FCB_TRY(cudaMemcpyAsync(out, dout, static_cast<size_t>(F) * F * 8, cudaMemcpyDeviceToHost, s));
  int hst = 0;
  FCB_TRY(cudaMemcpyAsync(&hst, dst, sizeof(int), cudaMemcpyDeviceToHost, s));
  FCB_TRY(cudaStreamSynchronize(s));
  return check_status(&hst);
}

// ---------------------------------------------------------------------------
// stock_corr precision forms (BF16x3 tensor cores / FP32 SIMT)
// ---------------------------------------------------------------------------
static int prec_check(const void* x, const void* out, int T, int N, int mode) {
  if (x == nullptr || out == nullptr || T < 1 || N < 1) return FCB_ERR_ARG;
  if (mode != FCB_PREC_BF16X3 && mode != FCB_PREC_FP32) return FCB_ERR_ARG;
  if (static_cast<long long>(T) * N > INT32_MAX) return FCB_ERR_CAP2;
  if (static_cast<long long>(N) * N > INT32_MAX) return FCB_ERR_CAP3;
  return FCB_OK;
}

extern "C" int fcb_dev_stock_corr_prec(const float* d_x, const uint8_t* d_mask, int T, int N, int mode, double* d_out,
                                       fcb_workspace* wsp, void* stream) {
  const int chk = prec_check(d_x, d_out, T, N, mode);
  if (chk != FCB_OK) return chk;
  if (wsp == nullptr) return FCB_ERR_ARG;  // scratch must come from a caller-held workspace
  fcb_workspace& ws = *wsp;
  FCB_TRY(ws.bind());
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int Np = (N + 127) / 128 * 128;
  const int Tp = (T + 31) / 32 * 32;
  const size_t e = static_cast<size_t>(Np) * Tp;
  PrecOperands op{};
  float* mu;
  int* dst;
  FCB_TRY(ws.get(S_PC_MU, static_cast<size_t>(Np) * 4, &mu));
  FCB_TRY(ws.get(S_STATUS, 64, &dst));
  if (mode == FCB_PREC_BF16X3) {
    FCB_TRY(ws.get(S_PC_XH, e * 2 * 7, &op.h));
    op.np = Np;
  } else {
    FCB_TRY(ws.get(S_PC_X32, e * 4, &op.x32));
    FCB_TRY(ws.get(S_PC_Q32, e * 4, &op.q32));
    FCB_TRY(ws.get(S_PC_M32, e * 4, &op.m32));
  }
  const int ntiles = prec_tile_count(mode == FCB_PREC_BF16X3 ? 0 : 1, N);
  int2* dt;
  FCB_TRY(ws.get(S_PC_TILES, static_cast<size_t>(ntiles) * sizeof(int2), &dt));
  FCB_TRY(launch_prec_tiles(mode == FCB_PREC_BF16X3 ? 0 : 1, N, dt, s));
  double2* cpart;
  FCB_TRY(ws.get(S_PC_CPART, static_cast<size_t>(prec_colmean_chunks(T)) * Np * sizeof(double2), &cpart));
  FCB_TRY(launch_prec_prep(d_x, d_mask, T, N, Np, Tp, mu, cpart, op, s));
  if (mode == FCB_PREC_BF16X3) {
    FCB_TRY(cudaMemsetAsync(dst, 0, sizeof(int), s));
    FCB_TRY(launch_corr_bf16x3(op, dt, ntiles, N, Np, Tp, d_out, dst, s));
    // the kernel's bounded waits report through dst: read it once the stream is done
    int hst = 0;
    FCB_TRY(cudaMemcpyAsync(&hst, dst, sizeof(int), cudaMemcpyDeviceToHost, s));
    FCB_TRY(cudaStreamSynchronize(s));
    if (hst != 0) return FCB_ERR_DEVICE_WAIT;
  } else {
    FCB_TRY(launch_corr_fp32(op, dt, ntiles, N, Tp, d_out, s));
    FCB_TRY(cudaStreamSynchronize(s));
  }
  return FCB_OK;
}

extern "C" int fcb_stock_corr_prec(const float* x, const uint8_t* mask, int T, int N, int mode, double* out,
                                   fcb_workspace* wsp) {
  const int chk = prec_check(x, out, T, N, mode);
  if (chk != FCB_OK) return chk;
  WsScope sc(wsp);
  fcb_workspace& ws = *sc.ws;
  FCB_TRY(ws.bind());
  cudaStream_t s = ws.stream[0];
  const size_t n = static_cast<size_t>(T) * N;
  float* dx;
  uint8_t* dm = nullptr;
  double* dout;
  FCB_TRY(ws.get(S_PC_X, n * 4, &dx));
  if (mask) FCB_TRY(ws.get(S_PC_MASK, n, &dm));
  FCB_TRY(ws.get(S_PC_OUT, static_cast<size_t>(N) * N * 8, &dout));
  FCB_TRY(cudaMemcpyAsync(dx, x, n * 4, cudaMemcpyHostToDevice, s));
  if (mask) FCB_TRY(cudaMemcpyAsync(dm, mask, n, cudaMemcpyHostToDevice, s));
  const int e = fcb_dev_stock_corr_prec(dx, dm, T, N, mode, dout, &ws, s);
  if (e != FCB_OK) return e;
  FCB_TRY(cudaMemcpyAsync(out, dout, static_cast<size_t>(N) * N * 8, cudaMemcpyDeviceToHost, s));
  FCB_TRY(cudaStreamSynchronize(s));
  return FCB_OK;
}

// ---------------------------------------------------------------------------
// memory budget model
// ---------------------------------------------------------------------------
// Device bytes the workspace of each host / device entry point requests for
// one call of the given shape: the sum of its slots, written next to (and
// checked on a GPU against the high-water accounting of) the entry points
// above.  The counterpart of the reference's memory budget table
// (docs/memory_budget_v1.json, src/mem_tracker.h:35-77).
namespace {
inline uint64_t slot_bytes(size_t b) { return b == 0 ? 16 : b; }

uint64_t budget_dev_factor_corr(int dtype, long long R, int F) {
  (void)dtype;
  const int Fp = (F + 3) / 4 * 4;
  const long long nbc = std::min<long long>(592, std::max<long long>(1, R / 2048));
  const long long nbg = fc_gram_blocks(R, F);
  return slot_bytes(static_cast<size_t>(nbc) * F * sizeof(FcColPart)) + slot_bytes(static_cast<size_t>(F) * sizeof(FcColStat)) +
         slot_bytes(static_cast<size_t>(nbg) * 4 * Fp * Fp * 8) + slot_bytes(static_cast<size_t>(F) * F * 4) + 64 +
         slot_bytes(fc_fb_part_doubles(R, F) * sizeof(double));
}

uint64_t budget_dev_stock_corr(int T, int N) {
  const size_t Tp = static_cast<size_t>((T + 31) / 32 * 32);
  const size_t upper = static_cast<size_t>(N) * (N - 1) / 2;
  return 3 * slot_bytes(static_cast<size_t>(N) * Tp * 8) + slot_bytes(static_cast<size_t>(N) * sizeof(ColStat)) + 64 +
         slot_bytes((upper > 0 ? upper : 1) * 4) + 64;
}
}  // namespace

extern "C" int fcb_memory_budget(int op, int dtype, int T, int N, int F, int flags, uint64_t* bytes) {
  if (bytes == nullptr || T < 1 || N < 1 || F < 1) return FCB_ERR_ARG;
  if (static_cast<long long>(T) * N > INT32_MAX) return FCB_ERR_CAP3;
  const bool m1 = (flags & FCB_BUDGET_MASK) != 0, m2 = (flags & FCB_BUDGET_MASK2) != 0;
  const bool ranks = (flags & FCB_BUDGET_RANKS) != 0;
  const size_t n = static_cast<size_t>(T) * N;
  const long long R = static_cast<long long>(T) * N;
  uint64_t b = 0;
  switch (op) {
    case FCB_OP_CS_RANK:
      b = slot_bytes(n * 4) * 2 + 64 + (m1 ? slot_bytes(n) : 0);
      if (N > kSmemRankCap) b += slot_bytes(rank_global_scratch(rank_global_bytes_per_date(0, N, 1, 4, 4), T));
      break;
    case FCB_OP_PARAMETER_SCAN: {
      const int groups = (flags >> 8) & 0xF;
      const int nact = groups == 0 ? 4 : __builtin_popcount(groups);
      b = slot_bytes(n * 4) + 64 + (m1 ? slot_bytes(n) : 0) + static_cast<uint64_t>(nact) * slot_bytes(n * 4);
      if (N > kSmemRankCap) b += slot_bytes(rank_global_scratch(rank_global_bytes_per_date(1, N, 1, 4, 4), T));
      break;
    }
    case FCB_OP_ROLLING_IC: {
      // dtype: the factor's; FCB_BUDGET_R_F64: the returns are f64
      const int fsz = dtype == FCB_DTYPE_F64 ? 8 : 4, rsz = (flags & FCB_BUDGET_R_F64) ? 8 : 4;
      b = slot_bytes(n * fsz) + slot_bytes(n * rsz) + slot_bytes(static_cast<size_t>(T) * 8) + 64 +
          (m1 ? slot_bytes(n) : 0) + (m2 ? slot_bytes(n) : 0) + (ranks ? 2 * slot_bytes(n * 8) : 0);
      const bool fits = (fsz == 4 && rsz == 4)   ? rank_ic_fits_smem<float, float>(N)
                        : (fsz == 4)             ? rank_ic_fits_smem<float, double>(N)
                        : (rsz == 4)             ? rank_ic_fits_smem<double, float>(N)
                                                 : rank_ic_fits_smem<double, double>(N);
      if (!fits) b += slot_bytes(rank_global_scratch(rank_global_bytes_per_date(2, N, 1, fsz, rsz), T));
      break;
    }
    case FCB_OP_DEV_FACTOR_CORR:
      if (F > 128) return FCB_ERR_CAP3;
      b = budget_dev_factor_corr(dtype, R, F);
      break;
    case FCB_OP_FACTOR_CORR: {
      if (F > 128) return FCB_ERR_CAP3;
      const size_t esz = dtype == FCB_DTYPE_F64 ? 8 : 4;
      b = budget_dev_factor_corr(dtype, R, F) + slot_bytes(static_cast<size_t>(R) * F * esz) +
          (m1 ? slot_bytes(static_cast<size_t>(R)) : 0) + slot_bytes(static_cast<size_t>(F) * F * 8) +
          ((flags & FCB_BUDGET_FALLBACK) ? slot_bytes(static_cast<size_t>(F) * F) : 0);
      break;
    }
    case FCB_OP_DEV_STOCK_CORR:
      if (static_cast<long long>(N) * N > INT32_MAX) return FCB_ERR_CAP3;
      b = budget_dev_stock_corr(T, N);
      break;
    case FCB_OP_STOCK_CORR: {
      if (static_cast<long long>(N) * N > INT32_MAX) return FCB_ERR_CAP3;
      const size_t esz = dtype == FCB_DTYPE_F64 ? 8 : 4;
      b = budget_dev_stock_corr(T, N) + slot_bytes(n * esz) + (m1 ? slot_bytes(n) : 0) +
          slot_bytes(static_cast<size_t>(N) * N * 8);
      break;
    }
    case FCB_OP_FACTOR_CORR_BF16X3:
      if (F > kFcTcMaxF) return FCB_ERR_UNSUPPORTED;
      b = slot_bytes(static_cast<size_t>(R) * F * 4) + (m1 ? slot_bytes(static_cast<size_t>(R)) : 0) +
          slot_bytes(static_cast<size_t>(F) * F * 8) + slot_bytes(fc_tc_work_bytes(F)) + 64;
      break;
    case FCB_OP_STOCK_CORR_PREC: {
      // dtype: the precision mode (FCB_PREC_BF16X3 / FCB_PREC_FP32)
      if (static_cast<long long>(N) * N > INT32_MAX) return FCB_ERR_CAP3;
      const size_t Np = static_cast<size_t>((N + 127) / 128 * 128), Tp = static_cast<size_t>((T + 31) / 32 * 32);
      const size_t e = Np * Tp;
      const int mode = dtype == FCB_PREC_FP32 ? 1 : 0;
      b = slot_bytes(n * 4) + (m1 ? slot_bytes(n) : 0) + slot_bytes(static_cast<size_t>(N) * N * 8) +
          slot_bytes(Np * 4) + 64 + (mode == 0 ? slot_bytes(e * 2 * 7) : 3 * slot_bytes(e * 4)) +
          slot_bytes(static_cast<size_t>(prec_tile_count(mode, N)) * sizeof(int2)) +
          slot_bytes(static_cast<size_t>(prec_colmean_chunks(T)) * Np * sizeof(double2));
      break;
    }
    case FCB_OP_RANK_IC_PANEL: {
      // method 0 (radix); the chunk schedule of fcb_rank_ic_panel
      const size_t per_date = static_cast<size_t>(F) * N * 4;
      int Tc = static_cast<int>((64ull << 20) / per_date);
      Tc = std::max(1, std::min(Tc, T));
      const size_t cn = static_cast<size_t>(Tc) * N;
      b = 64 + slot_bytes(static_cast<size_t>(F) * T * 8) +
          3 * (slot_bytes(cn * F * 4) + slot_bytes(cn * 4) + (m1 ? slot_bytes(cn) : 0) + (m2 ? slot_bytes(cn) : 0) +
               (ranks ? slot_bytes(cn * F * 4) : 0));
      if (F >= 2 && ric_items_fit(N))
        b += slot_bytes(ric_prep_bytes(Tc, N, F));
      else if (!rank_ic_fits_smem<float, float>(N))
        b += slot_bytes(rank_global_scratch(rank_global_bytes_per_date(2, N, F, 4, 4), Tc));
      break;
    }
    default:
      return FCB_ERR_ARG;
  }
  *bytes = b;
  return FCB_OK;
}
