// fcb_common.cuh -- shared device helpers for the sm_100a cross-sectional kernels.
//
// Canonical ordinal keys, Blackwell bulk-copy (TMA engine) row staging with an
// mbarrier, and block-wide scans/reductions built on warp shuffles.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#define FCB_DEV __device__ __forceinline__

namespace fcb {

constexpr uint32_t kInvalidKey32 = 0xFFFFFFFFu;
constexpr unsigned long long kInvalidKey64 = 0xFFFFFFFFFFFFFFFFull;
constexpr uint32_t kQuietNanBits = 0x7fc00000u;
constexpr unsigned kFull = 0xFFFFFFFFu;

// Order-preserving u32 key of an f32 value: +0/-0 fold to 0x80000000,
// negatives -> ~bits, non-negatives -> bits|0x80000000; non-finite -> all ones.
// Same map as the reference's canonical_ordinal_key_f32
// (src/cross_sectional_rank.cu:35-39); computed on the bit pattern so that a
// flush-to-zero compile mode cannot fold subnormals into zero.
FCB_DEV uint32_t key_f32(float v) {
  uint32_t b = __float_as_uint(v);
  if ((b & 0x7f800000u) == 0x7f800000u) return kInvalidKey32;  // inf / nan
  if ((b & 0x7fffffffu) == 0u) b = 0u;                          // -0 -> +0
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

// Order-preserving u64 key of an f64 value (reference src/rolling_ic.cu:34-38).
FCB_DEV unsigned long long key_f64(double v) {
  unsigned long long b = static_cast<unsigned long long>(__double_as_longlong(v));
  if ((b & 0x7ff0000000000000ull) == 0x7ff0000000000000ull) return kInvalidKey64;
  if ((b & 0x7fffffffffffffffull) == 0ull) b = 0ull;
  return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}

FCB_DEV bool finite_f32(float v) { return (__float_as_uint(v) & 0x7f800000u) != 0x7f800000u; }
FCB_DEV bool finite_f64(double v) {
  return (static_cast<unsigned long long>(__double_as_longlong(v)) & 0x7ff0000000000000ull) !=
         0x7ff0000000000000ull;
}

template <typename K> struct KeyOf;
template <> struct KeyOf<float> {
  using type = uint32_t;
  static FCB_DEV uint32_t key(float v) { return key_f32(v); }
  static FCB_DEV bool finite(float v) { return finite_f32(v); }
  static FCB_DEV float max_finite() { return __FLT_MAX__; }
  static constexpr uint32_t invalid = kInvalidKey32;
};
template <> struct KeyOf<double> {
  using type = unsigned long long;
  static FCB_DEV unsigned long long key(double v) { return key_f64(v); }
  static FCB_DEV bool finite(double v) { return finite_f64(v); }
  static FCB_DEV double max_finite() { return __DBL_MAX__; }
  static constexpr unsigned long long invalid = kInvalidKey64;
};

// Spearman IC from exact integer sums.  The joint-set ranks of both sides are
// permutations of 1..m, so sum r = m(m+1)/2 and sum r^2 = m(m+1)(2m+1)/6 and
// only S = sum r_f r_r depends on the data: 4 sxy = 4S - m(m+1)^2 and
// 4 sxx = 4 syy = m(m^2-1)/3 are exact integers.  The reference's two-pass
// f64 Pearson on integer ranks is exact before the same finalize
// (sxy/sqrt(sxx))/sqrt(syy) (src/rolling_ic.cu:232-304), so the results are
// bit-identical.
FCB_DEV double spearman_from_sum(long long m, long long sum_rr) {
  const long long s4 = 4 * sum_rr - m * (m + 1) * (m + 1);  // 4*sxy
  const long long q4 = m * (m * m - 1) / 3;                // 4*sxx == 4*syy
  const double sxy = static_cast<double>(s4) * 0.25;
  const double sxx = static_cast<double>(q4) * 0.25;
  return (sxy / sqrt(sxx)) / sqrt(sxx);
}

FCB_DEV unsigned lane_id() { return threadIdx.x & 31u; }
FCB_DEV unsigned lanemask_lt() {
  unsigned m;
  asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// ----------------------------------------------------------------------------
// Bulk copy global -> shared through the TMA engine (cp.async.bulk), completed
// on an mbarrier.  Used to stage a whole cross-section row into shared memory
// while the issuing warp's siblings proceed.  No cluster multicast anywhere.
// ----------------------------------------------------------------------------
FCB_DEV uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
FCB_DEV void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
FCB_DEV void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
FCB_DEV void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
// Bounded wait on phase `parity`.  Returns false (and gives up) after
// `max_polls` unsuccessful polls, so that a copy that never lands cannot hang
// the GPU; callers turn that into an error status.
FCB_DEV bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t max_polls = (1u << 22)) {
  uint32_t ok = 0;
  for (uint32_t i = 0; i < max_polls; ++i) {
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}
// dst/src 16-byte aligned, bytes a multiple of 16.
// Prefetch [src, src + bytes) into L2 (bulk-copy engine, no shared memory,
// no completion to wait for).  src and bytes are rounded inward to 16 bytes.
FCB_DEV void bulk_prefetch_l2(const void* src, size_t bytes) {
  const uintptr_t a0 = (reinterpret_cast<uintptr_t>(src) + 15) & ~uintptr_t(15);
  const uintptr_t a1 = (reinterpret_cast<uintptr_t>(src) + bytes) & ~uintptr_t(15);
  if (a1 <= a0) return;
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a0), "r"(static_cast<uint32_t>(a1 - a0))
               : "memory");
}

FCB_DEV void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// Row staging through the bulk-copy engine.  `region` is 16-aligned shared
// memory of n*sizeof(T)+16 bytes.  The row is placed at region + (src % 16) so
// that its 16-byte aligned interior lines up with a 16-byte aligned shared
// address; thread 0 arms `bar` and issues one cp.async.bulk for the interior,
// every thread copies part of the ragged head/tail with plain loads.  Returns
// the shared address of element 0.  Must be called by all threads; follow with
// stage_wait(bar, ...) on the same barrier and a __syncthreads().
template <typename T>
FCB_DEV T* stage_issue(uint8_t* region, const T* src, int n, uint64_t* bar, bool& armed) {
  const uintptr_t s = reinterpret_cast<uintptr_t>(src);
  const uint32_t mis = static_cast<uint32_t>(s & 15u);
  T* dst = reinterpret_cast<T*>(region + mis);
  const uintptr_t e = s + static_cast<uintptr_t>(n) * sizeof(T);
  const uintptr_t a0 = (s + 15) & ~uintptr_t(15);
  const uintptr_t a1 = e & ~uintptr_t(15);
  armed = (a1 > a0) && (a1 - a0 >= 64) && (mis % sizeof(T) == 0);
  if (armed) {
    const int i0 = static_cast<int>((a0 - s) / sizeof(T));
    const int i1 = static_cast<int>((a1 - s) / sizeof(T));
    if (threadIdx.x == 0) {
      // the region was last touched by ordinary loads/stores (made visible to
      // this thread by the caller's barrier): order them before the copy's
      // async-proxy writes
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_expect_tx(bar, static_cast<uint32_t>(a1 - a0));
      bulk_g2s(dst + i0, src + i0, static_cast<uint32_t>(a1 - a0), bar);
    }
    for (int i = threadIdx.x; i < i0; i += blockDim.x) dst[i] = src[i];
    for (int i = i1 + threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
  } else {
    for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
  }
  return dst;
}

// Completes a stage_issue: waits (bounded) for the bulk copy if one was
// armed and flips the phase bit.  Returns false if the copy did not land.
FCB_DEV bool stage_wait(uint64_t* bar, uint32_t& phase, bool armed) {
  if (!armed) return true;
  const bool ok = mbar_wait(bar, phase);
  phase ^= 1u;
  return ok;
}

// ----------------------------------------------------------------------------
// Block-wide scans / reductions (warp shuffles + one shared slot per warp).
// `scratch` must hold at least 33 uint32 / 33 uint64 words.
// ----------------------------------------------------------------------------
template <typename T>
FCB_DEV T warp_inclusive_sum(T v) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T u = __shfl_up_sync(kFull, v, o);
    if (lane_id() >= static_cast<unsigned>(o)) v += u;
  }
  return v;
}

template <typename T>
FCB_DEV T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

// Exclusive prefix sum of one value per thread over the block (in thread
// order); also returns the block total.  All threads must call.
template <typename T>
FCB_DEV T block_exclusive_sum(T v, T* scratch, T& total) {
  const int w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  T inc = warp_inclusive_sum(v);
  if (lane_id() == 31) scratch[w] = inc;
  __syncthreads();
  if (w == 0) {
    T s = (lane_id() < static_cast<unsigned>(nw)) ? scratch[lane_id()] : T(0);
    T si = warp_inclusive_sum(s);
    if (lane_id() < static_cast<unsigned>(nw)) scratch[lane_id()] = si - s;
    if (lane_id() == 31) scratch[32] = si;
  }
  __syncthreads();
  T res = scratch[w] + inc - v;
  total = scratch[32];
  __syncthreads();
  return res;
}

template <typename T>
FCB_DEV T block_sum(T v, T* scratch) {
  T total;
  (void)block_exclusive_sum(v, scratch, total);
  return total;
}

FCB_DEV int block_min_int(int v, int* scratch) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(kFull, v, o));
  const int w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  if (lane_id() == 0) scratch[w] = v;
  __syncthreads();
  if (w == 0) {
    int s = (lane_id() < static_cast<unsigned>(nw)) ? scratch[lane_id()] : 0x7fffffff;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s = min(s, __shfl_xor_sync(kFull, s, o));
    if (lane_id() == 0) scratch[32] = s;
  }
  __syncthreads();
  int r = scratch[32];
  __syncthreads();
  return r;
}

FCB_DEV int block_max_int(int v, int* scratch) {
  return -block_min_int(-v, scratch);
}

}  // namespace fcb
