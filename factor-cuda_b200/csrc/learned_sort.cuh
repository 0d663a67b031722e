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

// Outcome codes written to the per-(factor,date) statistics.
constexpr int kLearnOk = 1, kLearnOverflow = 2, kLearnJudge = 3, kLearnScale = 4;

// Sort the m compacted pairs (kA, iA) with the bucket map.  On success the
// sorted sequence is in (kA, iA) and the return is kLearnOk.  kLearnOverflow /
// kLearnScale leave (kA, iA) untouched; kLearnJudge leaves them permuted (the
// caller must rebuild them before falling back).  cnt: u16 array of at least
// m+2 entries, 4-byte aligned.  dscratch: >= 66 doubles; scan: >= 33 u32.
template <int NT>
FCB_DEV int learned_sort(uint32_t* kA, uint16_t* iA, uint32_t* kB, uint16_t* iB, int m, uint16_t* cnt,
                         const float* tab, float lo, float hi, int cap, double* dscratch, uint32_t* scan,
                         int* max_bucket_out, int* sumsq_out) {
  if (m <= 1) return kLearnOk;
  // per-date standardisation: mean and mean absolute deviation of the values
  double s = 0.0;
  for (int p = threadIdx.x; p < m; p += NT) s += key_to_f32(kA[p]);
  s = block_sum(s, dscratch);
  const double mean = s / m;
  double a = 0.0;
  for (int p = threadIdx.x; p < m; p += NT) a += fabs(key_to_f32(kA[p]) - mean);
  a = block_sum(a, dscratch);
  const double mad = a / m;
  BucketMap bm;
  bm.tab = tab;
  bm.loc = static_cast<float>(mean);
  bm.inv_scale = static_cast<float>(1.0 / mad);
  bm.lo = lo;
  bm.inv_dz = static_cast<float>((kCdfKnots - 1) / static_cast<double>(hi - lo));
  bm.B = m;
  bm.Bf = static_cast<float>(m);
  if (!(mad > 0.0) || !isfinite(bm.loc) || !isfinite(bm.inv_scale) || !(bm.inv_scale > 0.0f) ||
      !isfinite(bm.inv_dz) || !(bm.inv_dz > 0.0f))
    return kLearnScale;
  // histogram (packed 16-bit counters)
  for (int b = threadIdx.x; b < (m + 2) / 2; b += NT) reinterpret_cast<uint32_t*>(cnt)[b] = 0u;
  __syncthreads();
  for (int p = threadIdx.x; p < m; p += NT) packed_inc(cnt, bm(kA[p]));
  __syncthreads();
  // largest bucket
  int mx = 0;
  for (int b = threadIdx.x; b < m; b += NT) mx = max(mx, static_cast<int>(cnt[b]));
  mx = block_max_int(mx, reinterpret_cast<int*>(scan));
  if (max_bucket_out != nullptr) *max_bucket_out = mx;
  if (mx > cap) return kLearnOverflow;
  // exclusive scan of the counts -> bucket starts (in place)
  {
    const int per = (m + NT - 1) / NT;
    const int b0 = threadIdx.x * per, b1 = min(m, b0 + per);
    uint32_t c = 0, c2 = 0;
    for (int b = b0; b < b1; ++b) {
      c += cnt[b];
      c2 += static_cast<uint32_t>(cnt[b]) * cnt[b];
    }
    c2 = block_sum(c2, scan);
    if (sumsq_out != nullptr) *sumsq_out = static_cast<int>(c2);
    uint32_t total;
    uint32_t run = block_exclusive_sum(c, scan, total);
    for (int b = b0; b < b1; ++b) {
      const uint32_t v = cnt[b];
      cnt[b] = static_cast<uint16_t>(run);
      run += v;
    }
    __syncthreads();
  }
  // scatter into bucket slots (order inside a bucket is arbitrary)
  for (int p = threadIdx.x; p < m; p += NT) {
    const uint32_t key = kA[p];
    const uint32_t pos = packed_inc(cnt, bm(key));
    kB[pos] = key;
    iB[pos] = iA[p];
  }
  __syncthreads();
  // rank inside the bucket by (key, column); cnt[b] now holds bucket b's end
  for (int q = threadIdx.x; q < m; q += NT) {
    const uint32_t key = kB[q];
    const uint16_t id = iB[q];
    const int b = bm(key);
    const int lo_b = b == 0 ? 0 : cnt[b - 1];
    const int hi_b = cnt[b];
    int r = 0;
    for (int s2 = lo_b; s2 < hi_b; ++s2) {
      const uint32_t k2 = kB[s2];
      r += (k2 < key || (k2 == key && iB[s2] < id)) ? 1 : 0;
    }
    kA[lo_b + r] = key;
    iA[lo_b + r] = id;
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
