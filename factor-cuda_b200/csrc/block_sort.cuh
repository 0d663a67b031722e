// block_sort.cuh -- stable in-shared-memory LSD radix sort of one cross-section.
//
// One CTA sorts up to NT*MAXIPT (key, column) pairs held in shared memory.
// Each 8-bit pass: every warp ranks a contiguous chunk of the input with
// __match_any_sync (stable: lane order within a 32-wide step, steps in order),
// per-warp digit counters are prefix-summed across warps and digits, and the
// pairs are scattered to the alternate buffer.  Passes over digits on which
// all keys agree are skipped (block-wide AND/OR of the keys).
//
// This replaces the reference's global CUB segmented radix sort
// (src/cross_sectional_rank.cu:152-164): a cross-section of N <= 16K cells fits
// in one SM's shared memory, so no global passes are needed.
#pragma once

#include "fcb_common.cuh"

namespace fcb {

constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;

// Shared-memory words the sorter needs besides the key/index buffers.
template <int NT>
struct SortScratch {
  static_assert(NT >= 256 && NT % 32 == 0, "one thread per digit is needed");
  static constexpr int NW = NT / 32;
  static constexpr size_t hist_bytes = size_t(NW) * kRadix * sizeof(uint16_t);
  static constexpr size_t base_bytes = size_t(kRadix) * sizeof(uint32_t);
  static constexpr size_t scan_bytes = 80 * sizeof(unsigned long long);
  static constexpr size_t bytes = hist_bytes + base_bytes + scan_bytes;
};

template <typename K>
FCB_DEV K shfl_xor_k(K v, int o) { return __shfl_xor_sync(kFull, v, o); }

// Block-wide AND and OR of the keys in [0, n).
template <typename K>
FCB_DEV void block_and_or(const K* keys, int n, K& a, K& o, K* scratch /*>=66*/) {
  K va = ~K(0), vo = K(0);
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    K k = keys[i];
    va &= k;
    vo |= k;
  }
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) {
    va &= shfl_xor_k(va, s);
    vo |= shfl_xor_k(vo, s);
  }
  const int w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  if (lane_id() == 0) {
    scratch[w] = va;
    scratch[32 + w] = vo;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    K ra = ~K(0), ro = K(0);
    for (int i = 0; i < nw; ++i) {
      ra &= scratch[i];
      ro |= scratch[32 + i];
    }
    scratch[64] = ra;
    scratch[65] = ro;
  }
  __syncthreads();
  a = scratch[64];
  o = scratch[65];
  __syncthreads();
}

// One stable 8-bit pass: (ks, is) -> (kd, id) on digit (key >> shift) & 255.
template <int NT, int MAXIPT, typename K>
FCB_DEV void radix_pass(const K* __restrict__ ks, const uint16_t* __restrict__ is, K* __restrict__ kd,
                        uint16_t* __restrict__ id, int n, int shift, uint16_t* whist, uint32_t* dbase,
                        uint32_t* scan) {
  constexpr int NW = NT / 32;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int per_warp = ((n + NW * 32 - 1) / (NW * 32)) * 32;
  const int ipt = per_warp >> 5;
  const int base = w * per_warp;
  uint16_t* wh = whist + w * kRadix;
  for (int d = lane; d < kRadix; d += 32) wh[d] = 0;
  __syncwarp();
  const unsigned lt = lanemask_lt();

  // the keys and the within-warp offsets (two per word) stay in registers
  // between the ranking and the scatter; column ids are re-read for the scatter
  uint32_t loc[(MAXIPT + 1) / 2];
  K kreg[MAXIPT];
#pragma unroll
  for (int k = 0; k < (MAXIPT + 1) / 2; ++k) loc[k] = 0;
#pragma unroll
  for (int k = 0; k < MAXIPT; ++k) {
    kreg[k] = K(0);
    if (k < ipt) {
      const int pos = base + k * 32 + lane;
      const bool v = pos < n;
      const K key = v ? ks[pos] : K(0);
      kreg[k] = key;
      const uint32_t d = v ? static_cast<uint32_t>((key >> shift) & K(kRadix - 1)) : uint32_t(kRadix);
      const unsigned peers = __match_any_sync(kFull, d);
      const uint32_t r = __popc(peers & lt);
      const uint32_t before = v ? wh[d] : 0u;
      __syncwarp();
      if (v && r == 0) wh[d] = static_cast<uint16_t>(before + __popc(peers));
      __syncwarp();
      loc[k >> 1] |= (before + r) << ((k & 1) * 16);
    }
  }
  __syncthreads();
  uint32_t tot = 0;
  if (threadIdx.x < kRadix) {
    const int d = threadIdx.x;
    uint32_t run = 0;
#pragma unroll
    for (int ww = 0; ww < NW; ++ww) {
      const uint32_t c = whist[ww * kRadix + d];
      whist[ww * kRadix + d] = static_cast<uint16_t>(run);
      run += c;
    }
    tot = run;
  }
  uint32_t total;
  const uint32_t ex = block_exclusive_sum(tot, scan, total);
  if (threadIdx.x < kRadix) dbase[threadIdx.x] = ex;
  __syncthreads();
#pragma unroll
  for (int k = 0; k < MAXIPT; ++k) {
    if (k < ipt) {
      const int pos = base + k * 32 + lane;
      if (pos < n) {
        const K key = kreg[k];
        const uint32_t d = static_cast<uint32_t>((key >> shift) & K(kRadix - 1));
        const uint32_t dst = dbase[d] + wh[d] + ((loc[k >> 1] >> ((k & 1) * 16)) & 0xFFFFu);
        kd[dst] = key;
        id[dst] = is[pos];
      }
    }
  }
  __syncthreads();
}

// Sort n <= NT*MAXIPT pairs.  (k0,i0) hold the input; (k1,i1) are scratch of
// the same size.  On return *kout/*iout point at whichever buffer holds the
// sorted sequence.  `scratch` is SortScratch<NT>::bytes of 16-aligned shared
// memory.  All threads of the block must call.
template <int NT, int MAXIPT, typename K>
FCB_DEV void block_radix_sort(K* k0, uint16_t* i0, K* k1, uint16_t* i1, int n, uint8_t* scratch,
                              K** kout, uint16_t** iout) {
  using S = SortScratch<NT>;
  uint16_t* whist = reinterpret_cast<uint16_t*>(scratch);
  uint32_t* dbase = reinterpret_cast<uint32_t*>(scratch + S::hist_bytes);
  unsigned long long* scan64 =
      reinterpret_cast<unsigned long long*>(scratch + S::hist_bytes + S::base_bytes);
  K a, o;
  block_and_or(k0, n, a, o, reinterpret_cast<K*>(scan64));
  const K diff = a ^ o;
  K* ks = k0;
  K* kd = k1;
  uint16_t* is = i0;
  uint16_t* id = i1;
  constexpr int KB = int(sizeof(K) * 8);
  for (int shift = 0; shift < KB; shift += kRadixBits) {
    if (((diff >> shift) & K(kRadix - 1)) == 0) continue;  // uniform across the block
    radix_pass<NT, MAXIPT, K>(ks, is, kd, id, n, shift, whist, dbase,
                              reinterpret_cast<uint32_t*>(scan64));
    K* tk = ks; ks = kd; kd = tk;
    uint16_t* ti = is; is = id; id = ti;
  }
  *kout = ks;
  *iout = is;
}

// Order-preserving compaction: for each i in [0,n) with flag(i) true, writes
// (key(i), i) to (kd[pos], id[pos]) where pos is i's rank among flagged cells.
// Threads own contiguous element chunks.  Returns the flagged count.
template <typename K, typename FlagFn, typename KeyFn>
FCB_DEV int compact_keys(int n, FlagFn flag, KeyFn keyf, K* kd, uint16_t* id, uint32_t* scan) {
  const int per = (n + blockDim.x - 1) / blockDim.x;
  const int b = threadIdx.x * per;
  const int e = min(n, b + per);
  uint32_t c = 0;
  for (int i = b; i < e; ++i) c += flag(i) ? 1u : 0u;
  uint32_t total;
  uint32_t pos = block_exclusive_sum(c, scan, total);
  for (int i = b; i < e; ++i) {
    if (flag(i)) {
      kd[pos] = keyf(i);
      id[pos] = static_cast<uint16_t>(i);
      ++pos;
    }
  }
  __syncthreads();
  return static_cast<int>(total);
}

}  // namespace fcb
