// noalloc.cu -- factor_corr entry point that allocates no device memory.
//
// Some callers cannot let a library call cudaMalloc: applications whose
// device memory is owned by a framework pool or held to a hard per-process
// budget, and latency-sensitive serving loops that cannot afford the implicit
// device-wide synchronisation cudaMalloc/cudaFree perform.  For them,
// fcb_dev_factor_corr_noalloc runs the factor_corr kernels of
// fcb_dev_factor_corr on caller-owned device buffers, with every scratch
// buffer carved out of one fixed-size array that lives in this library's
// device image.  The array is kFcNoallocScratchBytes (about 4.9 MB: column
// partials, Gram partials, the fallback list and the multi-block fallback's
// partials, sized for F <= FCB_NOALLOC_MAX_F at any pool size) and every GPU
// that loads the library holds it until the process exits.
//
// The array fixes the row partition at kColBlocks / kGramBlocks blocks, where
// fcb_dev_factor_corr sizes it from the pool (up to 592 / 888 blocks): the
// partial sums are added in a different order, so the two entry points agree
// within 1e-12 per output rather than bit for bit (and a pair right at the
// cancellation gate may take the two-pass fallback in one and not the other;
// both results are then within the reference's tolerance).
#include <algorithm>

#include "../../include/fcb200.h"
#include "fcb_kernels.h"

namespace {

constexpr int kMaxF = FCB_NOALLOC_MAX_F;
constexpr int kMaxFp = (kMaxF + 3) / 4 * 4;
constexpr int kMaxPairs = kMaxF * (kMaxF - 1) / 2;
constexpr int kColBlocks = 148;  // column-statistics blocks (one per SM)
constexpr int kGramBlocks = 74;  // Gram-partial blocks

constexpr size_t al256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kOffColPart = 0;
constexpr size_t kOffColStat = al256(kOffColPart + size_t(kColBlocks) * kMaxF * sizeof(fcb::FcColPart));
constexpr size_t kOffGram = al256(kOffColStat + size_t(kMaxF) * sizeof(fcb::FcColStat));
constexpr size_t kOffFbList = al256(kOffGram + size_t(kGramBlocks) * 4 * kMaxFp * kMaxFp * sizeof(double));
constexpr size_t kOffFbCount = al256(kOffFbList + size_t(kMaxF) * kMaxF * sizeof(int));
constexpr size_t kOffFbPart = al256(kOffFbCount + sizeof(int));
constexpr size_t kFbPartDoubles =
    size_t(kMaxPairs) * fcb::kFcFbMaxNblk * fcb::kFcFbPartDoubles + size_t(kMaxPairs) * 4;
constexpr size_t kFcNoallocScratchBytes = al256(kOffFbPart + kFbPartDoubles * sizeof(double));

// The scratch array.  Its name is a host-side stand-in, not a device address:
// host code must use the address cudaGetSymbolAddress returns for the
// current device.
static __device__ __align__(256) unsigned char g_fc_scratch[kFcNoallocScratchBytes];

// The device address of g_fc_scratch on the current device.  Resolved on
// every call (a driver lookup that allocates nothing once the library's
// device image is loaded), so a context torn down and created again -- after
// cudaDeviceReset, for instance -- is served its own address.
cudaError_t scratch_for_current_device(unsigned char** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_fc_scratch);
  if (e != cudaSuccess) return e;
  *out = static_cast<unsigned char*>(p);
  return cudaSuccess;
}

}  // namespace

extern "C" int fcb_dev_factor_corr_noalloc(const void* d_x, int dtype, const uint8_t* d_mask, int T, int N, int F,
                                           double* d_out, void* stream) {
  if (d_x == nullptr || d_out == nullptr || T < 1 || N < 1 || F < 1) return FCB_ERR_ARG;
  if (dtype != FCB_DTYPE_F32 && dtype != FCB_DTYPE_F64) return FCB_ERR_ARG;
  if (static_cast<long long>(T) * N > INT32_MAX) return FCB_ERR_CAP2;
  if (F > kMaxF) return FCB_ERR_NOALLOC_CAP;
  unsigned char* base = nullptr;
  cudaError_t e = scratch_for_current_device(&base);
  if (e != cudaSuccess) return static_cast<int>(e);
  const long long R = static_cast<long long>(T) * N;
  fcb::FcWork w{};
  w.nblk_cols = static_cast<int>(std::min<long long>(kColBlocks, std::max<long long>(1, R / 2048)));
  w.nblk_gram = static_cast<int>(std::min<long long>(kGramBlocks, std::max<long long>(1, R / 1024)));
  w.colpart = reinterpret_cast<fcb::FcColPart*>(base + kOffColPart);
  w.colstat = reinterpret_cast<fcb::FcColStat*>(base + kOffColStat);
  w.gram = reinterpret_cast<double*>(base + kOffGram);
  w.fb_list = reinterpret_cast<int*>(base + kOffFbList);
  w.fb_count = reinterpret_cast<int*>(base + kOffFbCount);
  // the large-pool fallback splits each flagged pair's rows over up to
  // kFcFbMaxNblk blocks; its partials fit the fixed region for every R
  if (fcb::fc_fb_part_doubles(R, F) > kFbPartDoubles) return FCB_ERR_NOALLOC_CAP;
  w.fb_part = reinterpret_cast<double*>(base + kOffFbPart);
  // launch_factor_corr zeroes the fallback counter before its first use; every
  // other scratch word is fully written before it is read.
  e = fcb::launch_factor_corr(d_x, dtype, d_mask, R, F, w, d_out, nullptr, static_cast<cudaStream_t>(stream));
  return static_cast<int>(e);
}
