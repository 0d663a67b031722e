// learned_sort.cuh -- bucket sort of one cross-section driven by a tabulated
// CDF network (learned splitters).
//
// bucket(key) = monotone map of the cell's standardised value through the
// network's tabulated CDF u(z) onto [0, B):
//   z = (x - loc) * inv_scale                 (per-date mean / MAD)
//   t = clamp((z - lo) * inv_dz, 0, K-1);  k = min(floor t, K-2);  f = t - k
//   a = floor(B u_k), b = floor(B u_{k+1}),   bucket = a + floor((b - a) f)
// Every step is monotone non-decreasing in x (u is cummax-monotone), so equal
// keys share a bucket and buckets are ordered: sorting each bucket by
// (key, column) gives exactly the stable ascending order.  The per-date judge
// re-checks that order over the whole output; any failure (or a bucket above
// `cap`, or an unusable scale) returns false and the caller uses the radix
// sort for that cross-section.
#pragma once

#include "fcb_common.cuh"
#include "fcb_kernels.h"

namespace fcb {

FCB_DEV float key_to_f32(uint32_t k) {
  const uint32_t b = (k & 0x80000000u) ? (k ^ 0x80000000u) : ~k;
  return __uint_as_float(b);
}

struct BucketMap {
  const float* tab;  // kCdfKnots entries (shared memory)
  float loc, inv_scale, lo, inv_dz, Bf;
  int B;
  FCB_DEV int operator()(uint32_t key) const {
    const float x = key_to_f32(key);
    const float z = (x - loc) * inv_scale;
    float t = (z - lo) * inv_dz;
    t = fminf(fmaxf(t, 0.0f), static_cast<float>(kCdfKnots - 1));
    const int k = min(static_cast<int>(t), kCdfKnots - 2);
    const float fr = fminf(t - static_cast<float>(k), 0.99999994f);
    const int a = min(B - 1, static_cast<int>(Bf * tab[k]));
    const int b = min(B - 1, static_cast<int>(Bf * tab[k + 1]));
    return a + static_cast<int>(static_cast<float>(b - a) * fr);
  }
};

FCB_DEV uint32_t packed_inc(uint16_t* arr, int b) {
  uint32_t* w = reinterpret_cast<uint32_t*>(arr) + (b >> 1);
  const int sh = (b & 1) * 16;
  const uint32_t old = atomicAdd(w, 1u << sh);
  return (old >> sh) & 0xFFFFu;
}

// Block-wide sum by xor shuffles: one shared slot per warp, every thread adds
// the warp totals.  scratch: >= 32 T.  All threads must call.
template <typename T>
FCB_DEV T block_reduce_add(T v, T* scratch) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  const int w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  if (lane_id() == 0) scratch[w] = v;
  __syncthreads();
  T t = T(0);
  for (int i = 0; i < nw; ++i) t += scratch[i];
  __syncthreads();
  return t;
}

// One pass, three block results: the exclusive prefix sum of c (returned),
// and the block maximum of mx and sum of c2 (written back).  Warp shuffles,
// one shared slot per warp and quantity, three barriers.  scan: >= 99 u32.
FCB_DEV uint32_t block_scan_max_sum(uint32_t c, int& mx, uint32_t& c2, uint32_t* scan) {
  const int w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  const unsigned lane = lane_id();
  const uint32_t inc = warp_inclusive_sum(c);
  int wm = mx;
  uint32_t ws = c2;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    wm = max(wm, __shfl_xor_sync(kFull, wm, o));
    ws += __shfl_xor_sync(kFull, ws, o);
  }
  if (lane == 31) scan[w] = inc;
  if (lane == 0) {
    scan[32 + w] = static_cast<uint32_t>(wm);
    scan[64 + w] = ws;
  }
  __syncthreads();
  if (w == 0) {
    const uint32_t sv = lane < static_cast<unsigned>(nw) ? scan[lane] : 0u;
    const uint32_t si = warp_inclusive_sum(sv);
    int mv = lane < static_cast<unsigned>(nw) ? static_cast<int>(scan[32 + lane]) : 0;
    uint32_t cv = lane < static_cast<unsigned>(nw) ? scan[64 + lane] : 0u;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      mv = max(mv, __shfl_xor_sync(kFull, mv, o));
      cv += __shfl_xor_sync(kFull, cv, o);
    }
    if (lane < static_cast<unsigned>(nw)) scan[lane] = si - sv;
    if (lane == 0) {
      scan[96] = static_cast<uint32_t>(mv);
      scan[97] = cv;
    }
  }
  __syncthreads();
  const uint32_t res = scan[w] + inc - c;
  mx = static_cast<int>(scan[96]);
  c2 = scan[97];
  __syncthreads();
  return res;
}

// Outcome codes written to the per-(factor,date) statistics.
constexpr int kLearnOk = 1, kLearnOverflow = 2, kLearnJudge = 3, kLearnScale = 4;

// Sort the m compacted pairs (kA, iA) with the bucket map.  On success the
// sorted sequence is in (kA, iA) and the return is kLearnOk.  kLearnOverflow /
// kLearnScale leave (kA, iA) untouched; kLearnJudge leaves them permuted (the
// caller must rebuild them before falling back).
//   cnt:   u16 array of at least m+2 entries, 4-byte aligned (bucket counters)
//   fscratch: >= 32 doubles; scan: >= 99 u32.
// The bucket of each cell is evaluated once (histogram pass) and parked in iB,
// which is idle until the scatter; the scatter reads it back into registers
// and each thread keeps its cells' buckets and slots there for the ranking.
template <int NT, int MAXIPT>
FCB_DEV int learned_sort(uint32_t* kA, uint16_t* iA, uint32_t* kB, uint16_t* iB, int m, uint16_t* cnt,
                         const float* tab, float lo, float hi, int cap, double* dscratch, uint32_t* scan,
                         int* max_bucket_out, int* sumsq_out) {
  if (m <= 1) return kLearnOk;
  // per-date standardisation: mean and mean absolute deviation of an evenly
  // spaced sample of the compacted cells, one per thread (they only shape the
  // bucket map; the judge below guarantees the order whatever they are)
  const int S = min(m, NT);
  const bool smp = static_cast<int>(threadIdx.x) < S;
  const float sv = smp ? key_to_f32(kA[static_cast<int>((static_cast<long long>(threadIdx.x) * m) / S)]) : 0.0f;
  const float mean = block_reduce_add(sv, reinterpret_cast<float*>(dscratch)) / static_cast<float>(S);
  const float mad = block_reduce_add(smp ? fabsf(sv - mean) : 0.0f, reinterpret_cast<float*>(dscratch)) /
                    static_cast<float>(S);
  BucketMap bm;
  bm.tab = tab;
  bm.loc = mean;
  bm.inv_scale = mad > 0.0f ? 1.0f / mad : 0.0f;
  bm.lo = lo;
  bm.inv_dz = static_cast<float>((kCdfKnots - 1) / static_cast<double>(hi - lo));
  bm.B = m;
  bm.Bf = static_cast<float>(m);
  if (!(mad > 0.0f) || !isfinite(bm.loc) || !isfinite(bm.inv_scale) || !(bm.inv_scale > 0.0f) ||
      !isfinite(bm.inv_dz) || !(bm.inv_dz > 0.0f))
    return kLearnScale;
  // histogram (packed 16-bit counters); each cell's bucket parked in iB
  for (int b = threadIdx.x; b < (m + 2) / 2; b += NT) reinterpret_cast<uint32_t*>(cnt)[b] = 0u;
  __syncthreads();
  for (int p = threadIdx.x; p < m; p += NT) {
    const int b = bm(kA[p]);
    packed_inc(cnt, b);
    iB[p] = static_cast<uint16_t>(b);
  }
  __syncthreads();
  // exclusive scan of the counts -> bucket starts (in place), largest bucket,
  // sum of squared sizes
  {
    const int per = (m + NT - 1) / NT;
    const int b0 = threadIdx.x * per, b1 = min(m, b0 + per);
    uint32_t c = 0, c2 = 0;
    int mx = 0;
    for (int b = b0; b < b1; ++b) {
      const uint32_t v = cnt[b];
      c += v;
      c2 += v * v;
      mx = max(mx, static_cast<int>(v));
    }
    uint32_t run = block_scan_max_sum(c, mx, c2, scan);  // mx, c2 become block totals
    if (max_bucket_out != nullptr) *max_bucket_out = mx;
    if (sumsq_out != nullptr) *sumsq_out = static_cast<int>(c2);
    if (mx > cap) return kLearnOverflow;  // uniform across the block
    for (int b = b0; b < b1; ++b) {
      const uint32_t v = cnt[b];
      cnt[b] = static_cast<uint16_t>(run);
      run += v;
    }
    __syncthreads();
  }
  // scatter into bucket slots (order inside a bucket is arbitrary); each
  // thread keeps the bucket and the slot of each of its cells, two per word
  uint32_t breg[(MAXIPT + 1) / 2], sreg[(MAXIPT + 1) / 2];
#pragma unroll
  for (int j = 0; j < MAXIPT; j += 2) {
    const int p0 = threadIdx.x + j * NT, p1 = p0 + NT;
    const uint32_t b0 = p0 < m ? iB[p0] : 0u;
    const uint32_t b1 = (j + 1 < MAXIPT && p1 < m) ? iB[p1] : 0u;
    breg[j >> 1] = b0 | (b1 << 16);
    sreg[j >> 1] = 0u;
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < MAXIPT; ++j) {
    const int p = threadIdx.x + j * NT;
    if (p < m) {
      const int b = static_cast<int>((breg[j >> 1] >> ((j & 1) * 16)) & 0xFFFFu);
      const uint32_t pos = packed_inc(cnt, b);
      kB[pos] = kA[p];
      iB[pos] = iA[p];
      sreg[j >> 1] |= pos << ((j & 1) * 16);
    }
  }
  __syncthreads();
  // rank inside the bucket by (key, column): keys first, column ids on ties.
  // After the scatter cnt[b] is the end of bucket b, and bucket b starts
  // where bucket b - 1 ends (the buckets tile [0, m) in order).
#pragma unroll
  for (int j = 0; j < MAXIPT; ++j) {
    const int p = threadIdx.x + j * NT;
    if (p < m) {
      const int b = static_cast<int>((breg[j >> 1] >> ((j & 1) * 16)) & 0xFFFFu);
      const int pos = static_cast<int>((sreg[j >> 1] >> ((j & 1) * 16)) & 0xFFFFu);
      const int lo_b = b > 0 ? static_cast<int>(cnt[b - 1]) : 0;
      const int hi_b = static_cast<int>(cnt[b]);
      const uint32_t key = kB[pos];
      const uint16_t id = iB[pos];
      int r = 0;
      for (int s2 = lo_b; s2 < hi_b; ++s2) {
        const uint32_t k2 = kB[s2];
        r += (k2 < key) ? 1 : 0;
        if (k2 == key) r += (iB[s2] < id) ? 1 : 0;
      }
      kA[lo_b + r] = key;
      iA[lo_b + r] = id;
    }
  }
  __syncthreads();
  // judge: strictly increasing (key, column) over the whole row
  int bad = 0;
  for (int p = 1 + threadIdx.x; p < m; p += NT) {
    const uint32_t k0 = kA[p - 1], k1 = kA[p];
    if (!(k0 < k1 || (k0 == k1 && iA[p - 1] < iA[p]))) bad = 1;
  }
  if (__syncthreads_or(bad)) return kLearnJudge;
  return kLearnOk;
}

}  // namespace fcb
