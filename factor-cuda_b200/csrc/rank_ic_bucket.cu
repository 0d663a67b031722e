// rank_ic_bucket.cu -- cs_rank + daily Spearman IC of F factor panels against
// one forward-return panel, one CTA per (date, factor), for sm_100a.
//
//  k_ric_prep     one CTA per date: sorts the date's valid forward returns
//                 once (stable radix sort in shared memory) and writes one
//                 32-bit word per stock: its position in that order, the
//                 position where its tie group starts, and the returns-valid
//                 and factor-mask bits.  The rows stay in L2 while the F
//                 factor CTAs of the date read them.
//  k_ric_learned  learned splitters: the factor's tabulated CDF network maps
//                 each valid cell to a bucket; one histogram pass (packed
//                 16-bit counters: all valid cells | joint cells), one scan,
//                 one scatter of (key, column) words into bucket slots, and
//                 each cell's rank is its bucket's start plus the number of
//                 smaller (key, column) words in its bucket.  The joint-set
//                 rank comes from the same counters' second half.  The map
//                 is monotone in the key whenever the table is
//                 non-decreasing, which each CTA checks as it stages the
//                 table; a bucket above the cap, an unusable scale or a
//                 rejected table hands the section to the radix kernel
//                 through a device list.
//  k_ric_radix    the plain path (and the learned path's fallback): the valid
//                 cells are compacted in column order and radix-sorted in
//                 shared memory; ranks are sorted positions.
//
// Both rank kernels keep every cell's state in registers (each thread owns
// four consecutive columns per 128-bit vector, loaded and stored with
// coalesced vector accesses) and share one epilogue: the returns' joint-set
// rank of a cell is its prepared position minus the number of return-valid /
// factor-invalid cells before it in the returns order (a per-CTA bitmap over
// those positions with per-word prefix counts), and the IC follows from the
// exact integer sum of rank products (see spearman_from_sum).
//
// Semantics: cs_rank_gpu (src/cross_sectional_rank.cu:228-372) for the ranks,
// rolling_ic_gpu (src/rolling_ic.cu:306-540) / np_rolling_ic
// (fc/_cpu_core.py:271-293) for the IC; the reference sorts with CUB's global
// segmented radix sort instead.
#include "block_sort.cuh"
#include "fcb_kernels.h"
#include "learned_sort.cuh"

namespace fcb {
namespace {

constexpr uint32_t kPosBits = 0x3FFFu;      // prepared word: bits 0-13 returns position
constexpr int kGidShift = 14;               //                bits 14-27 tie-group start
constexpr uint32_t kRetValid = 1u << 28;    //                bit 28 returns valid
constexpr uint32_t kFacMask = 1u << 29;     //                bit 29 factor mask
// per-cell register flags
constexpr uint32_t kCellValid = 1u << 28;   // factor valid (finite and mask)
constexpr uint32_t kCellJoint = 1u << 29;   // factor and returns valid
constexpr uint32_t kCellDrop = 1u << 30;    // returns valid, factor not

__host__ __device__ inline size_t al16(size_t x) { return (x + 15) & ~size_t(15); }

// Row loads in the vector layout: thread tid owns columns 4*(j*NT + tid) + k.
template <int NT, int V, bool STREAM>
FCB_DEV void load_row_f32(const float* __restrict__ row, int N, float (&x)[4 * V]) {
  const bool al = (reinterpret_cast<uintptr_t>(row) & 15u) == 0;
  const float qnan = __uint_as_float(kQuietNanBits);
#pragma unroll
  for (int j = 0; j < V; ++j) {
    const int i0 = 4 * (j * NT + static_cast<int>(threadIdx.x));
    if (al && i0 + 3 < N) {
      const float4* p = reinterpret_cast<const float4*>(row + i0);
      const float4 q = STREAM ? __ldcs(p) : __ldg(p);
      x[4 * j] = q.x;
      x[4 * j + 1] = q.y;
      x[4 * j + 2] = q.z;
      x[4 * j + 3] = q.w;
    } else {
#pragma unroll
      for (int k = 0; k < 4; ++k) x[4 * j + k] = (i0 + k < N) ? row[i0 + k] : qnan;
    }
  }
}

template <int NT, int V>
FCB_DEV void load_words(const uint32_t* __restrict__ row, int N, uint32_t (&w)[4 * V]) {
#pragma unroll
  for (int j = 0; j < V; ++j) {
    const int i0 = 4 * (j * NT + static_cast<int>(threadIdx.x));
    if (i0 + 3 < N) {
      const uint4 q = __ldg(reinterpret_cast<const uint4*>(row + i0));
      w[4 * j] = q.x;
      w[4 * j + 1] = q.y;
      w[4 * j + 2] = q.z;
      w[4 * j + 3] = q.w;
    } else {
#pragma unroll
      for (int k = 0; k < 4; ++k) w[4 * j + k] = (i0 + k < N) ? row[i0 + k] : 0u;
    }
  }
}

// 0/1 bytes in the vector layout (all ones when there is no mask).
template <int NT, int V>
FCB_DEV void load_mask4(const uint8_t* __restrict__ row, int N, uint32_t (&m)[4 * V]) {
  const bool al = (reinterpret_cast<uintptr_t>(row) & 3u) == 0;
#pragma unroll
  for (int j = 0; j < V; ++j) {
    const int i0 = 4 * (j * NT + static_cast<int>(threadIdx.x));
    if (row == nullptr) {
#pragma unroll
      for (int k = 0; k < 4; ++k) m[4 * j + k] = (i0 + k < N) ? 1u : 0u;
    } else if (al && i0 + 3 < N) {
      const uint32_t q = __ldcs(reinterpret_cast<const unsigned int*>(row + i0));
#pragma unroll
      for (int k = 0; k < 4; ++k) m[4 * j + k] = ((q >> (8 * k)) & 0xFFu) ? 1u : 0u;
    } else {
#pragma unroll
      for (int k = 0; k < 4; ++k) m[4 * j + k] = (i0 + k < N && row[i0 + k] != 0) ? 1u : 0u;
    }
  }
}

template <int NT, int V>
FCB_DEV void store_row_f32v(float* __restrict__ row, int N, const float (&v)[4 * V]) {
  const bool al = (reinterpret_cast<uintptr_t>(row) & 15u) == 0;
#pragma unroll
  for (int j = 0; j < V; ++j) {
    const int i0 = 4 * (j * NT + static_cast<int>(threadIdx.x));
    if (al && i0 + 3 < N) {
      __stcs(reinterpret_cast<float4*>(row + i0), make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]));
    } else {
#pragma unroll
      for (int k = 0; k < 4; ++k)
        if (i0 + k < N) row[i0 + k] = v[4 * j + k];
    }
  }
}

// Order-preserving compaction offsets in the vector layout: the column order
// is the (j, tid, k) order, so cell (j, k) of this thread goes to
//   sum_{j' < j} total_j' + (flagged cells of vector j in threads < tid)
//   + (flagged cells k' < k of this thread's vector j).
// Per-vector counts (0..4 per thread, <= 4*NT per block) are packed into
// 12-bit fields, five per 64-bit word, so one block scan serves five vectors.
// Returns the block total; base[j] receives the first two terms.
template <int NT, int V>
FCB_DEV int compact_bases(uint32_t flags, int (&base)[V], unsigned long long* scratch) {
  static_assert(4 * NT < 4096, "12-bit count fields");
  static_assert(4 * V <= 32, "one flag bit per cell");
  constexpr int PER = 5, K = (V + PER - 1) / PER;
  int run = 0;
#pragma unroll
  for (int q = 0; q < K; ++q) {
    unsigned long long packed = 0;
#pragma unroll
    for (int jj = 0; jj < PER; ++jj) {
      const int j = q * PER + jj;
      if (j < V) packed |= static_cast<unsigned long long>(__popc((flags >> (4 * j)) & 0xFu)) << (12 * jj);
    }
    unsigned long long tot;
    const unsigned long long ex = block_exclusive_sum(packed, scratch, tot);
#pragma unroll
    for (int jj = 0; jj < PER; ++jj) {
      const int j = q * PER + jj;
      if (j < V) {
        base[j] = run + static_cast<int>((ex >> (12 * jj)) & 0xFFFull);
        run += static_cast<int>((tot >> (12 * jj)) & 0xFFFull);
      }
    }
  }
  return run;
}

// Shared-memory layout of the rank kernels (bytes; every region 16-aligned).
struct BucketLayout {  // k_ric_learned
  size_t red, tab, dw, cnt, mem, total;
  __host__ __device__ explicit BucketLayout(int n) {
    size_t o = 0;
    red = o; o += 1024;
    tab = o; o += size_t(kCdfKnots) * 4;
    dw = o; o = al16(o + size_t((n + 31) / 32 + 1) * 8);
    cnt = o; o = al16(o + size_t(n + 2) * 4);
    mem = o; o = al16(o + size_t(n) * 8);
    total = o;
  }
};
template <int NT>
struct SortedLayout {  // k_ric_radix and k_ric_prep
  size_t red, dw, scratch, k0, k1, i0, i1, total;
  __host__ __device__ explicit SortedLayout(int n) {
    size_t o = 0;
    red = o; o += 1024;
    dw = o; o = al16(o + size_t((n + 31) / 32 + 1) * 8);
    scratch = o; o = al16(o + SortScratch<NT>::bytes);
    k0 = o; o = al16(o + size_t(n) * 4 + 16);
    k1 = o; o = al16(o + size_t(n) * 4 + 16);
    i0 = o; o = al16(o + size_t(n) * 2 + 16);
    i1 = o; o = al16(o + size_t(n) * 2 + 16);
    total = o;
  }
};

// Exclusive per-word prefix counts of the drop bitmap: dw[k] low half = the
// bits of returns positions 32k..32k+31, high half = set bits before word k.
// One warp; the bitmap must be complete (a barrier after the last atomicOr).
FCB_DEV void drop_prefix(uint32_t* dw32, int nwd) {
  uint32_t carry = 0;
  for (int base = 0; base < nwd; base += 32) {
    const int k = base + static_cast<int>(lane_id());
    const uint32_t bits = k < nwd ? dw32[2 * k] : 0u;
    const uint32_t c = __popc(bits);
    const uint32_t inc = warp_inclusive_sum(c);
    if (k < nwd) dw32[2 * k + 1] = carry + inc - c;
    carry += __shfl_sync(kFull, inc, 31);
  }
}

// The shared epilogue.  P[c] = cs rank (bits 0-15, 0 = not ranked) | joint
// factor rank (bits 16-31, 0 = not joint).  Writes the rank row, and the IC
// unless `bad` (then the section, item_id, is queued on `fb` for the radix
// kernel).  With
// KEYS the factor-constant test takes the min / max of the joint cells' keys
// (key[]); otherwise fkmin / fkmax are the keys at the first and last joint
// positions of the sorted order, provided by the caller.
template <int NT, int V, bool KEYS>
FCB_DEV void ric_epilogue(const RankIcArgs<float, float>& a, const RicPrep& rp, int t, int f, const uint32_t (&P)[4 * V],
                          const uint32_t (&key)[4 * V], uint32_t fkmin, uint32_t fkmax, uint32_t mj,
                          const unsigned long long* dw, uint32_t* red, int bad, int* stats, int item_id,
                          RicList fb) {
  constexpr int C = 4 * V;
  const int N = a.N;
  const size_t frow = (static_cast<size_t>(f) * a.T + t) * N;
  if (a.ranks_out != nullptr) {
    float v[C];
    const float qnan = __uint_as_float(kQuietNanBits);
#pragma unroll
    for (int c = 0; c < C; ++c) {
      const uint32_t r = P[c] & 0xFFFFu;
      v[c] = r ? static_cast<float>(r) : qnan;
    }
    store_row_f32v<NT, V>(a.ranks_out + frow, N, v);
  }
  uint32_t w[C];
  load_words<NT, V>(rp.word + static_cast<size_t>(t) * rp.ld, N, w);
  unsigned long long sum = 0;
  uint32_t kmin = 0xFFFFFFFFu, kmax = 0u, gmin = 0xFFFFFFFFu, gmax = 0u;
#pragma unroll
  for (int c = 0; c < C; ++c) {
    const uint32_t rfj = P[c] >> 16;
    if (rfj != 0u) {
      const uint32_t pos = w[c] & kPosBits;
      const unsigned long long d = dw[pos >> 5];
      const uint32_t below = static_cast<uint32_t>(d >> 32) +
                             __popc(static_cast<uint32_t>(d) & ((1u << (pos & 31u)) - 1u));
      const uint32_t rrj = pos + 1u - below;
      sum += static_cast<unsigned long long>(rfj) * rrj;
      const uint32_t g = (w[c] >> kGidShift) & kPosBits;
      gmin = min(gmin, g);
      gmax = max(gmax, g);
      if (KEYS) {
        kmin = min(kmin, key[c]);
        kmax = max(kmax, key[c]);
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    sum += __shfl_xor_sync(kFull, sum, o);
    kmin = min(kmin, __shfl_xor_sync(kFull, kmin, o));
    kmax = max(kmax, __shfl_xor_sync(kFull, kmax, o));
    gmin = min(gmin, __shfl_xor_sync(kFull, gmin, o));
    gmax = max(gmax, __shfl_xor_sync(kFull, gmax, o));
  }
  bad = __any_sync(kFull, bad);
  const int wi = static_cast<int>(threadIdx.x >> 5);
  unsigned long long* red64 = reinterpret_cast<unsigned long long*>(red);
  if (lane_id() == 0) {
    red64[wi] = sum;
    red[64 + wi] = kmin;
    red[96 + wi] = kmax;
    red[128 + wi] = gmin;
    red[160 + wi] = gmax;
    red[192 + wi] = static_cast<uint32_t>(bad);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    constexpr int NW = NT / 32;
    unsigned long long s = 0;
    int b = 0;
    for (int i = 0; i < NW; ++i) {
      s += red64[i];
      kmin = min(kmin, red[64 + i]);
      kmax = max(kmax, red[96 + i]);
      gmin = min(gmin, red[128 + i]);
      gmax = max(gmax, red[160 + i]);
      b |= static_cast<int>(red[192 + i]);
    }
    if (!KEYS) {
      kmin = fkmin;
      kmax = fkmax;
    }
    if (b) {
      // the caller's order check failed (bad): the radix kernel redoes the section
      if (stats != nullptr) stats[0] = kLearnJudge;
      fb.items[atomicAdd(fb.count, 1)] = item_id;
    } else {
      double ic = __longlong_as_double(0x7ff8000000000000ll);
      const long long m = static_cast<long long>(mj);
      if (m >= a.min_valid && m >= 2 && kmin != kmax && gmin != gmax)
        ic = spearman_from_sum(m, static_cast<long long>(s));
      a.ic_out[static_cast<size_t>(f) * (a.ic_ld > 0 ? a.ic_ld : a.T) + t] = ic;
    }
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// per-date returns preparation
// ---------------------------------------------------------------------------
// Date t of returns R (T,N) and masks: the prepared words of row t into out.
template <int NT, int V>
FCB_DEV void ric_prep_body(const float* __restrict__ R, const uint8_t* __restrict__ rmask,
                           const uint8_t* __restrict__ fmask, int N, int t, uint32_t* __restrict__ out, uint8_t* sm) {
  constexpr int C = 4 * V;
  const SortedLayout<NT> L(N);
  unsigned long long* scan64 = reinterpret_cast<unsigned long long*>(sm + L.red);
  const size_t row = static_cast<size_t>(t) * N;
  float r[C];
  load_row_f32<NT, V, true>(R + row, N, r);
  uint32_t fmb = 0u, rvb = 0u;  // per-cell bits: factor mask, returns valid
  {
    uint32_t rmk[C], fmk[C];
    load_mask4<NT, V>(rmask != nullptr ? rmask + row : nullptr, N, rmk);
    load_mask4<NT, V>(fmask != nullptr ? fmask + row : nullptr, N, fmk);
#pragma unroll
    for (int c = 0; c < C; ++c) {
      rvb |= ((finite_f32(r[c]) && rmk[c]) ? 1u : 0u) << c;
      fmb |= (fmk[c] ? 1u : 0u) << c;
    }
  }
  int base[V];
  const int mr = compact_bases<NT, V>(rvb, base, scan64);
  uint32_t* k0 = reinterpret_cast<uint32_t*>(sm + L.k0);
  uint32_t* k1 = reinterpret_cast<uint32_t*>(sm + L.k1);
  uint16_t* i0 = reinterpret_cast<uint16_t*>(sm + L.i0);
  uint16_t* i1 = reinterpret_cast<uint16_t*>(sm + L.i1);
#pragma unroll
  for (int j = 0; j < V; ++j) {
    int p = base[j];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int c = 4 * j + k;
      if ((rvb >> c) & 1u) {
        k0[p] = key_f32(r[c]);
        i0[p] = static_cast<uint16_t>(4 * (j * NT + static_cast<int>(threadIdx.x)) + k);
        ++p;
      }
    }
  }
  __syncthreads();
  uint32_t* ks;
  uint16_t* is;
  block_radix_sort<NT, C, uint32_t>(k0, i0, k1, i1, mr, sm + L.scratch, &ks, &is);
  // words of the valid returns, by column: position | tie-group start
  uint32_t* W = (ks == k0) ? k1 : k0;
  const int per = (mr + NT - 1) / NT;
  const int b0 = static_cast<int>(threadIdx.x) * per, b1 = min(mr, b0 + per);
  int last = -1;
  for (int p = b0; p < b1; ++p)
    if (p == 0 || ks[p] != ks[p - 1]) last = p;
  // exclusive max-scan of the chunk's last group start (identity -1)
  int inc = last;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int u = __shfl_up_sync(kFull, inc, o);
    if (lane_id() >= static_cast<unsigned>(o)) inc = max(inc, u);
  }
  int* sc = reinterpret_cast<int*>(scan64);
  const int wi = static_cast<int>(threadIdx.x >> 5);
  if (lane_id() == 31) sc[wi] = inc;
  __syncthreads();
  int carry = -1;
  for (int i = 0; i < wi; ++i) carry = max(carry, sc[i]);
  const int up = __shfl_up_sync(kFull, inc, 1);
  if (lane_id() > 0) carry = max(carry, up);
  for (int p = b0; p < b1; ++p) {
    if (p == 0 || ks[p] != ks[p - 1]) carry = p;
    W[is[p]] = static_cast<uint32_t>(p) | (static_cast<uint32_t>(carry) << kGidShift) | kRetValid;
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < V; ++j) {
    const int i0c = 4 * (j * NT + static_cast<int>(threadIdx.x));
    uint32_t v[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int c = 4 * j + k;
      v[k] = (((rvb >> c) & 1u) ? W[i0c + k] : 0u) | (((fmb >> c) & 1u) ? kFacMask : 0u);
    }
    if (i0c + 3 < N) {
      *reinterpret_cast<uint4*>(out + i0c) = make_uint4(v[0], v[1], v[2], v[3]);
    } else {
#pragma unroll
      for (int k = 0; k < 4; ++k)
        if (i0c + k < N) out[i0c + k] = v[k];
    }
  }
}

// 256-thread sort CTAs keep to 80 registers so that three fit an SM (the
// shared memory of N <= 5120 allows three)
template <int NT, int V>
__global__ void __launch_bounds__(NT, NT == 256 ? 3 : 1) k_ric_prep(const float* __restrict__ R, const uint8_t* __restrict__ rmask,
                                                 const uint8_t* __restrict__ fmask, int N, RicPrep rp) {
  extern __shared__ __align__(16) uint8_t sm[];
  if (blockIdx.x == 0 && threadIdx.x == 0) *rp.fb_count = 0;
  ric_prep_body<NT, V>(R, rmask, fmask, N, blockIdx.x, rp.word + static_cast<size_t>(blockIdx.x) * rp.ld, sm);
}

// ---------------------------------------------------------------------------
// learned splitters
// ---------------------------------------------------------------------------
// Section (t, f); item_id is what a fallback queues on fb.
template <int NT, int V>
FCB_DEV void ric_learned_body(const RankIcArgs<float, float>& a, const RicPrep& rp, const int t, const int f,
                              const int item_id, RicList fb, uint8_t* sm) {
  constexpr int C = 4 * V, NW = NT / 32;
  const int N = a.N;
  const BucketLayout L(N);
  uint32_t* red = reinterpret_cast<uint32_t*>(sm + L.red);
  float* tab = reinterpret_cast<float*>(sm + L.tab);
  uint32_t* dw32 = reinterpret_cast<uint32_t*>(sm + L.dw);
  const unsigned long long* dw = reinterpret_cast<const unsigned long long*>(sm + L.dw);
  uint32_t* cnt = reinterpret_cast<uint32_t*>(sm + L.cnt);
  unsigned long long* mem = reinterpret_cast<unsigned long long*>(sm + L.mem);
  const int tid = static_cast<int>(threadIdx.x), wi = tid >> 5, lane = tid & 31;
  const size_t frow = (static_cast<size_t>(f) * a.T + t) * N;
  int* stats = a.learn_stats != nullptr ? a.learn_stats + (static_cast<size_t>(f) * a.T + t) * 4 : nullptr;
  const int nwd = (N + 31) / 32 + 1;

  // ---- the row and the date's prepared returns words
  float x[C];
  uint32_t w[C];
  load_row_f32<NT, V, true>(a.X + frow, N, x);
  load_words<NT, V>(rp.word + static_cast<size_t>(t) * rp.ld, N, w);
  // warp 0 issues the loads of the location / scale sample (used below) right
  // behind the row's, so that both wait out one memory latency, not two
  float xs[8];
  uint32_t vs = 0u;
  if (wi == 0) {
    const int S = min(N, 256);  // i = s*N/S: s*N/256 when N >= 256, else s
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int s = q * 32 + lane;
      xs[q] = 0.0f;
      if (s < S) {
        const int i = N >= 256 ? (s * N) >> 8 : s;
        const float v = a.X[frow + i];
        if (finite_f32(v) && (rp.word[static_cast<size_t>(t) * rp.ld + i] & kFacMask)) {
          xs[q] = v;
          vs |= 1u << q;
        }
      }
    }
  }
  // ---- stage the table (checking that it is non-decreasing within [0, 1]: a
  // NaN fails every comparison), clear the counters and the drop bitmap --
  // after the row's loads are out, so that their latencies overlap
  int tab_bad = 0;
  {
    const float* tg = a.cdf_table + static_cast<size_t>(f) * kCdfKnots;
    for (int k = tid; k < kCdfKnots / 4; k += NT) {
      const float4 v = __ldg(reinterpret_cast<const float4*>(tg) + k);
      reinterpret_cast<float4*>(tab)[k] = v;
      const float nx = (4 * k + 4 < kCdfKnots) ? __ldg(tg + 4 * k + 4) : 1.0f;
      tab_bad |= (0.0f <= v.x && v.x <= v.y && v.y <= v.z && v.z <= v.w && v.w <= nx && nx <= 1.0f) ? 0 : 1;
    }
  }
  for (int k = tid; k < (N + 2 + 3) / 4; k += NT) reinterpret_cast<uint4*>(cnt)[k] = make_uint4(0u, 0u, 0u, 0u);
  for (int k = tid; k < nwd; k += NT) reinterpret_cast<unsigned long long*>(dw32)[k] = 0ull;

  uint32_t key[C], P[C];
  int nval = 0;
#pragma unroll
  for (int c = 0; c < C; ++c) {
    const bool vf = finite_f32(x[c]) && (w[c] & kFacMask);
    const bool rv = (w[c] & kRetValid) != 0u;
    key[c] = key_f32(x[c]);
    P[c] = (vf ? kCellValid : 0u) | ((vf && rv) ? kCellJoint : 0u) | ((rv && !vf) ? kCellDrop : 0u) |
           (w[c] & kPosBits);
    nval += vf ? 1 : 0;
  }
  // ---- warp 0: location / scale from an evenly spaced sample of the row
  // (mean and mean absolute deviation of up to 256 valid cells; they only
  // shape the bucket map -- the order is exact whatever they are)
  if (wi == 0) {
    int ns = 0;
    float s1 = 0.0f;
#pragma unroll
    for (int q = 0; q < 8; ++q)
      if ((vs >> q) & 1u) {
        s1 += xs[q];
        ++ns;
      }
    const float n_s = static_cast<float>(warp_sum(ns));
    const float mean = warp_sum(s1) / n_s;
    float s2 = 0.0f;
#pragma unroll
    for (int q = 0; q < 8; ++q)
      if ((vs >> q) & 1u) s2 += fabsf(xs[q] - mean);
    const float mad = warp_sum(s2) / n_s;
    if (lane == 0) {
      red[96] = __float_as_uint(mean);
      red[97] = __float_as_uint(mad);
    }
  }
  nval = warp_sum(nval);
  if (lane == 0) red[wi] = static_cast<uint32_t>(nval);
  tab_bad = __syncthreads_or(tab_bad);  // B1
  int m = 0;
  for (int i = 0; i < NW; ++i) m += static_cast<int>(red[i]);
  const float loc = __uint_as_float(red[96]), mad = __uint_as_float(red[97]);
  // drop bits (returns valid, factor not) at their returns positions
#pragma unroll
  for (int c = 0; c < C; ++c)
    if (P[c] & kCellDrop) atomicOr(&dw32[2 * ((P[c] & kPosBits) >> 5)], 1u << (P[c] & 31u));
  BucketMap bm;
  bm.tab = tab;
  bm.loc = loc;
  bm.inv_scale = mad > 0.0f ? 1.0f / mad : 0.0f;
  const float lo = a.cdf_zrange[2 * f], hi = a.cdf_zrange[2 * f + 1];
  bm.lo = lo;
  bm.inv_dz = static_cast<float>((kCdfKnots - 1) / static_cast<double>(hi - lo));
  bm.B = m > 0 ? m : 1;
  bm.Bf = static_cast<float>(bm.B);
  const bool scale_ok = (mad > 0.0f) && isfinite(loc) && isfinite(bm.inv_scale) && (bm.inv_scale > 0.0f) &&
                        isfinite(bm.inv_dz) && (bm.inv_dz > 0.0f);
  if (m >= 2 && (!scale_ok || tab_bad)) {  // uniform across the block
    if (tid == 0) {
      if (stats != nullptr) {
        stats[0] = tab_bad ? kLearnJudge : kLearnScale;
        stats[1] = 0;
        stats[2] = 0;
        stats[3] = m;
      }
      fb.items[atomicAdd(fb.count, 1)] = item_id;
    }
    return;
  }
  // ---- histogram: packed counters (low half all valid cells, high half the
  // joint ones); the returned count is the cell's slot inside its bucket
#pragma unroll
  for (int c = 0; c < C; ++c) {
    if (P[c] & kCellValid) {
      // clamped: a table outside [0, 1] may not index outside the counters
      const uint32_t b = static_cast<uint32_t>(min(max(bm(key[c]), 0), bm.B - 1));
      const uint32_t old = atomicAdd(&cnt[b], (P[c] & kCellJoint) ? 0x10001u : 1u);
      P[c] = b | (min(old & 0xFFFFu, 0xFFFu) << 14) | (P[c] & (kCellValid | kCellJoint));
    } else {
      P[c] = 0u;
    }
  }
  __syncthreads();  // B2
  // ---- scan of the m + 1 counters (the last is the total): each warp takes a
  // segment in 128-counter steps, four counters per lane (one 16-byte access);
  // counters past m + 1 up to the next multiple of four are zero
  const int E4 = (m + 1 + 3) & ~3;
  const int seg = ((E4 + NW - 1) / NW + 127) & ~127;
  const int s0 = min(E4, wi * seg), s1 = min(E4, s0 + seg);
  {
    uint32_t tot = 0, mx = 0, sq = 0;
    for (int i = s0 + 4 * lane; i < s1; i += 128) {
      const uint4 v = *reinterpret_cast<const uint4*>(cnt + i);
      tot += v.x + v.y + v.z + v.w;
      const uint32_t a = v.x & 0xFFFFu, b = v.y & 0xFFFFu, c2 = v.z & 0xFFFFu, d = v.w & 0xFFFFu;
      mx = max(mx, max(max(a, b), max(c2, d)));
      sq += a * a + b * b + c2 * c2 + d * d;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      tot += __shfl_xor_sync(kFull, tot, o);
      mx = max(mx, __shfl_xor_sync(kFull, mx, o));
      sq += __shfl_xor_sync(kFull, sq, o);
    }
    if (lane == 0) {
      red[wi] = tot;
      red[32 + wi] = mx;
      red[64 + wi] = sq;
    }
    if (wi == NW - 1) drop_prefix(dw32, nwd);  // every drop bit is set (B2)
  }
  __syncthreads();  // B3
  uint32_t off = 0, total = 0, mxall = 0, sqall = 0;
  for (int i = 0; i < NW; ++i) {
    const uint32_t v = red[i];
    if (i < wi) off += v;
    total += v;
    mxall = max(mxall, red[32 + i]);
    sqall += red[64 + i];
  }
  const uint32_t mj = total >> 16;
  const int cap = min(a.learn_cap, 0xFFF);
  if (static_cast<int>(mxall) > cap) {  // uniform across the block
    if (tid == 0) {
      if (stats != nullptr) {
        stats[0] = kLearnOverflow;
        stats[1] = static_cast<int>(mxall);
        stats[2] = static_cast<int>(sqall);
        stats[3] = m;
      }
      fb.items[atomicAdd(fb.count, 1)] = item_id;
    }
    return;
  }
  if (tid == 0 && stats != nullptr) {
    stats[0] = kLearnOk;
    stats[1] = static_cast<int>(mxall);
    stats[2] = static_cast<int>(sqall);
    stats[3] = m;
  }
  for (int base = s0; base < s1; base += 128) {
    const int i = base + 4 * lane;
    const bool in = i < s1;
    const uint4 v = in ? *reinterpret_cast<const uint4*>(cnt + i) : make_uint4(0u, 0u, 0u, 0u);
    const uint32_t a0 = v.x, a1 = a0 + v.y, a2 = a1 + v.z, a3 = a2 + v.w;
    const uint32_t inc = warp_inclusive_sum(a3);
    const uint32_t ex = off + inc - a3;
    if (in) *reinterpret_cast<uint4*>(cnt + i) = make_uint4(ex, ex + a0, ex + a1, ex + a2);
    off += __shfl_sync(kFull, inc, 31);
  }
  __syncthreads();  // B4
  // ---- scatter (key, column, joint) words into their bucket slots
#pragma unroll
  for (int c = 0; c < C; ++c) {
    if (P[c] & kCellValid) {
      const uint32_t b = P[c] & kPosBits;
      const uint32_t pos = (cnt[b] & 0xFFFFu) + ((P[c] >> 14) & 0xFFFu);
      const uint32_t i = 4u * ((c >> 2) * NT + tid) + (c & 3);
      mem[pos] = (static_cast<unsigned long long>(key[c]) << 32) | (i << 1) | ((P[c] & kCellJoint) ? 1u : 0u);
    }
  }
  __syncthreads();  // B5
  // ---- ranks: bucket start + smaller words in the bucket
#pragma unroll
  for (int c = 0; c < C; ++c) {
    if (P[c] & kCellValid) {
      const uint32_t b = P[c] & kPosBits;
      const bool joint = (P[c] & kCellJoint) != 0u;
      const uint32_t i = 4u * ((c >> 2) * NT + tid) + (c & 3);
      const unsigned long long mine =
          (static_cast<unsigned long long>(key[c]) << 32) | (i << 1) | (joint ? 1u : 0u);
      const uint32_t s = cnt[b], e = cnt[b + 1];
      uint32_t r = 0, rj = 0;
      // a bucket of one is the cell itself
      if ((e & 0xFFFFu) - (s & 0xFFFFu) > 1u)
      for (uint32_t p = s & 0xFFFFu; p < (e & 0xFFFFu); ++p) {
        const unsigned long long o = mem[p];
        const uint32_t lt = o < mine ? 1u : 0u;
        r += lt;
        rj += lt & static_cast<uint32_t>(o);
      }
      P[c] = ((s & 0xFFFFu) + r + 1u) | (joint ? (((s >> 16) + rj + 1u) << 16) : 0u);
    }
  }
  // No order check is needed: the bucket map is non-decreasing in the key
  // (each step -- the exact key-to-value inverse, the affine standardisation
  // by a positive scale, the clamped knot position, the two knots' buckets
  // of a non-decreasing table and the fraction below one between them -- is
  // monotone under round-to-nearest, and a bucket ends at or below the next
  // knot's), so every bucket holds smaller keys than the next, and the table
  // was checked above.
  ric_epilogue<NT, V, true>(a, rp, t, f, P, key, 0u, 0u, mj, dw, red, 0, stats, item_id, fb);
}

// 256-thread CTAs keep to 80 registers so that three fit an SM (the shared
// memory of N <= 5120 allows three); the 512-thread form of three cells per
// vector (N <= 6144) keeps to 64 so that two fit
template <int NT, int V>
__global__ void __launch_bounds__(NT, NT == 256 ? 3 : (V == 3 ? 2 : 1)) k_ric_learned(RankIcArgs<float, float> a, RicPrep rp) {
  extern __shared__ __align__(16) uint8_t sm[];
  const int item = static_cast<int>(blockIdx.x);
  ric_learned_body<NT, V>(a, rp, item / a.F, item % a.F, item, RicList{rp.fb_count, rp.fb_items}, sm);
}

// ---------------------------------------------------------------------------
// radix (plain path and the learned path's fallback)
// ---------------------------------------------------------------------------
// Section (t, f) by the radix sort.
template <int NT, int V, bool STREAM>
FCB_DEV void ric_radix_body(const RankIcArgs<float, float>& a, const RicPrep& rp, const int t, const int f,
                            uint8_t* sm) {
  constexpr int C = 4 * V;
  const int N = a.N;
  const SortedLayout<NT> L(N);
  uint32_t* red = reinterpret_cast<uint32_t*>(sm + L.red);
  unsigned long long* scan64 = reinterpret_cast<unsigned long long*>(sm + L.red);
  uint32_t* dw32 = reinterpret_cast<uint32_t*>(sm + L.dw);
  const unsigned long long* dw = reinterpret_cast<const unsigned long long*>(sm + L.dw);
  uint32_t* k0 = reinterpret_cast<uint32_t*>(sm + L.k0);
  uint32_t* k1 = reinterpret_cast<uint32_t*>(sm + L.k1);
  uint16_t* i0 = reinterpret_cast<uint16_t*>(sm + L.i0);
  uint16_t* i1 = reinterpret_cast<uint16_t*>(sm + L.i1);
  const int tid = static_cast<int>(threadIdx.x);
  const int nwd = (N + 31) / 32 + 1;
  {
    const size_t frow = (static_cast<size_t>(f) * a.T + t) * N;
    for (int k = tid; k < nwd; k += NT) reinterpret_cast<unsigned long long*>(dw32)[k] = 0ull;
    float x[C];
    uint32_t w[C];
    load_row_f32<NT, V, STREAM>(a.X + frow, N, x);
    load_words<NT, V>(rp.word + static_cast<size_t>(t) * rp.ld, N, w);
    uint32_t valid = 0u, joint = 0u;  // bit c: cell c is factor-valid / in the joint set
#pragma unroll
    for (int c = 0; c < C; ++c) {
      const bool vf = finite_f32(x[c]) && (w[c] & kFacMask);
      valid |= (vf ? 1u : 0u) << c;
      joint |= ((vf && (w[c] & kRetValid)) ? 1u : 0u) << c;
    }
    int base[V];
    const int m = compact_bases<NT, V>(valid, base, scan64);  // barriers: the bitmap clear is visible
#pragma unroll
    for (int c = 0; c < C; ++c)
      if (!((valid >> c) & 1u) && (w[c] & kRetValid))
        atomicOr(&dw32[2 * ((w[c] & kPosBits) >> 5)], 1u << (w[c] & 31u));
#pragma unroll
    for (int j = 0; j < V; ++j) {
      int p = base[j];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int c = 4 * j + k;
        if ((valid >> c) & 1u) {
          k0[p] = key_f32(x[c]);
          i0[p] = static_cast<uint16_t>((4 * (j * NT + tid) + k) | (((joint >> c) & 1u) << 15));
          ++p;
        }
      }
    }
    __syncthreads();
    uint32_t* ks;
    uint16_t* is;
    block_radix_sort<NT, C, uint32_t>(k0, i0, k1, i1, m, sm + L.scratch, &ks, &is);
    if (tid < 32) drop_prefix(dw32, nwd);  // the sort's barriers follow the last atomicOr
    // cs rank = sorted position + 1; joint rank = joint cells before it + 1;
    // first / last joint positions give the factor-constant test
    uint32_t* RK = (ks == k0) ? k1 : k0;
    const int per = (m + NT - 1) / NT;
    const int b0 = tid * per, b1 = min(m, b0 + per);
    uint32_t cj = 0;
    int jfirst = 0x7fffffff, jlast = -1;
    for (int p = b0; p < b1; ++p) {
      if (is[p] & 0x8000u) {
        ++cj;
        jfirst = min(jfirst, p);
        jlast = p;
      }
    }
    uint32_t mj;
    uint32_t ex = block_exclusive_sum(cj, reinterpret_cast<uint32_t*>(scan64), mj);
    for (int p = b0; p < b1; ++p) {
      const uint32_t id = is[p];
      const bool jt = (id & 0x8000u) != 0u;
      if (jt) ++ex;
      RK[id & 0x3FFFu] = static_cast<uint32_t>(p + 1) | (jt ? (ex << 16) : 0u);
    }
    const int jf = block_min_int(jfirst, reinterpret_cast<int*>(scan64));   // barriers publish RK
    const int jl = block_max_int(jlast, reinterpret_cast<int*>(scan64));
    const uint32_t fkmin = jl >= 0 ? ks[jf] : 0u, fkmax = jl >= 0 ? ks[jl] : 0u;
    uint32_t P[C];
#pragma unroll
    for (int c = 0; c < C; ++c) P[c] = ((valid >> c) & 1u) ? RK[4 * ((c >> 2) * NT + tid) + (c & 3)] : 0u;
    ric_epilogue<NT, V, false>(a, rp, t, f, P, P, fkmin, fkmax, mj, dw, red, 0, nullptr, 0, RicList{nullptr, nullptr});
  }
}

// LIST: sections come from the learned kernel's fallback list (persistent
// CTAs stride over it); otherwise blockIdx.x = t * F + f.
template <int NT, int V, bool LIST>
__global__ void __launch_bounds__(NT, NT == 256 ? 3 : 1) k_ric_radix(RankIcArgs<float, float> a, RicPrep rp) {
  extern __shared__ __align__(16) uint8_t sm[];
  if (!LIST) {
    ric_radix_body<NT, V, true>(a, rp, static_cast<int>(blockIdx.x) / a.F, static_cast<int>(blockIdx.x) % a.F, sm);
    return;
  }
  const int nitems = *static_cast<volatile int*>(rp.fb_count);
  for (int it = blockIdx.x; it < nitems; it += static_cast<int>(gridDim.x)) {
    const int item = rp.fb_items[it];
    ric_radix_body<NT, V, false>(a, rp, item / a.F, item % a.F, sm);
    __syncthreads();  // the next section reuses the shared memory
  }
}

// ---------------------------------------------------------------------------
// many panels per launch (the batch)
// ---------------------------------------------------------------------------
// The panels of one size variant share a launch: one CTA per item (a date of
// a panel for the returns pass, a (date, factor) section for the rank pass),
// the item's panel found by binary search over the exclusive prefix `off` of
// the panels' item counts.  Sections handed back by the learned body go on
// the variant's list as global item ids.  Panels without a model are ranked
// by the radix body in the learned launch.
FCB_DEV int panel_of(const int* __restrict__ off, int np, int item) {
  int lo = 0, hi = np - 1;  // the last panel whose first item is <= item
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(off + mid) <= item) lo = mid; else hi = mid - 1;
  }
  return lo;
}

template <int NT, int V>
__global__ void __launch_bounds__(NT) k_ric_prep_batch(const RicPanel* __restrict__ P, const int* __restrict__ off,
                                                       int np, RicList fb) {
  extern __shared__ __align__(16) uint8_t sm[];
  const int item = static_cast<int>(blockIdx.x);
  if (item == 0 && threadIdx.x == 0 && fb.count != nullptr) *fb.count = 0;
  const int q = panel_of(off, np, item);
  const RankIcArgs<float, float> a = P[q].a;
  const RicPrep rp = P[q].rp;
  const int t = item - __ldg(off + q);
  ric_prep_body<NT, V>(a.R, a.rmask, a.fmask, a.N, t, rp.word + static_cast<size_t>(t) * rp.ld, sm);
}

template <int NT, int V, bool LEARNED>
__global__ void __launch_bounds__(NT, NT == 256 ? 3 : 1) k_ric_items_batch(const RicPanel* __restrict__ P, const int* __restrict__ off,
                                                        int np, RicList fb) {
  extern __shared__ __align__(16) uint8_t sm[];
  const int item = static_cast<int>(blockIdx.x);
  const int q = panel_of(off, np, item);
  const RankIcArgs<float, float> a = P[q].a;
  const RicPrep rp = P[q].rp;
  const int l = item - __ldg(off + q);
  if (LEARNED && a.cdf_table != nullptr)
    ric_learned_body<NT, V>(a, rp, l / a.F, l % a.F, item, fb, sm);
  else
    ric_radix_body<NT, V, true>(a, rp, l / a.F, l % a.F, sm);
}

template <int NT, int V>
__global__ void __launch_bounds__(NT) k_ric_list_batch(const RicPanel* __restrict__ P, const int* __restrict__ off,
                                                       int np, RicList fb) {
  extern __shared__ __align__(16) uint8_t sm[];
  const int nitems = *static_cast<volatile int*>(fb.count);
  for (int it = blockIdx.x; it < nitems; it += static_cast<int>(gridDim.x)) {
    const int item = fb.items[it];
    const int q = panel_of(off, np, item);
    const RankIcArgs<float, float> a = P[q].a;
    const RicPrep rp = P[q].rp;
    const int l = item - __ldg(off + q);
    ric_radix_body<NT, V, false>(a, rp, l / a.F, l % a.F, sm);
    __syncthreads();  // the next section reuses the shared memory
  }
}

// ---------------------------------------------------------------------------
// cs_rank and parameter_scan of one plane: one CTA per date
// ---------------------------------------------------------------------------
// cs_rank: valid = finite & mask; the valid cells are compacted in column
// order, radix-sorted by key (of -x for descending), and each cell's rank is
// its sorted position + 1 (replaces cs_rank_gpu, src/cross_sectional_rank.cu:
// 228-372, which runs CUB's global segmented sort).
template <int NT, int V>
__global__ void __launch_bounds__(NT) k_csr(const float* __restrict__ X, const uint8_t* __restrict__ mask, int N,
                                            int desc, float* __restrict__ out) {
  constexpr int C = 4 * V;
  extern __shared__ __align__(16) uint8_t sm[];
  const SortedLayout<NT> L(N);
  unsigned long long* scan64 = reinterpret_cast<unsigned long long*>(sm + L.red);
  uint32_t* k0 = reinterpret_cast<uint32_t*>(sm + L.k0);
  uint32_t* k1 = reinterpret_cast<uint32_t*>(sm + L.k1);
  uint16_t* i0 = reinterpret_cast<uint16_t*>(sm + L.i0);
  uint16_t* i1 = reinterpret_cast<uint16_t*>(sm + L.i1);
  const int tid = static_cast<int>(threadIdx.x);
  const size_t row = static_cast<size_t>(blockIdx.x) * N;
  float x[C];
  uint32_t mk[C];
  load_row_f32<NT, V, true>(X + row, N, x);
  load_mask4<NT, V>(mask != nullptr ? mask + row : nullptr, N, mk);
  uint32_t valid = 0u;
#pragma unroll
  for (int c = 0; c < C; ++c) valid |= ((finite_f32(x[c]) && mk[c]) ? 1u : 0u) << c;
  int base[V];
  const int m = compact_bases<NT, V>(valid, base, scan64);
#pragma unroll
  for (int j = 0; j < V; ++j) {
    int p = base[j];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int c = 4 * j + k;
      if ((valid >> c) & 1u) {
        k0[p] = key_f32(desc ? -x[c] : x[c]);
        i0[p] = static_cast<uint16_t>(4 * (j * NT + tid) + k);
        ++p;
      }
    }
  }
  __syncthreads();
  uint32_t* ks;
  uint16_t* is;
  block_radix_sort<NT, C, uint32_t>(k0, i0, k1, i1, m, sm + L.scratch, &ks, &is);
  uint32_t* RK = (ks == k0) ? k1 : k0;
  for (int p = tid; p < m; p += NT) RK[is[p]] = static_cast<uint32_t>(p + 1);
  __syncthreads();
  const float qnan = __uint_as_float(kQuietNanBits);
  float v[C];
#pragma unroll
  for (int c = 0; c < C; ++c)
    v[c] = ((valid >> c) & 1u) ? static_cast<float>(RK[4 * ((c >> 2) * NT + tid) + (c & 3)]) : qnan;
  store_row_f32v<NT, V>(out + row, N, v);
}

// parameter_scan: one ascending sort of the finite cells serves all four
// groups (asc / desc x masked / unmasked).  With S the start and E the end of
// a cell's tie group in sorted order, C the count of masked-valid cells before
// a sorted position and m / mt the finite / masked-valid totals:
//   asc unmasked  p + 1                  asc masked   C[p] + 1
//   desc unmasked m - E + (p - S) + 1    desc masked  mt - C[E] + (C[p] - C[S]) + 1
// (descending ranks keep ties by ascending column, the contract of
// fc/_cpu_core.py:57-78 / :295-301; replaces the reference's four rank
// pipelines, src/cross_sectional_rank.cu:401-664).  Shared memory stays at
// the sort's 12 bytes per cell: tie-group starts go to a bitmap (the sorted
// keys are then free for C and E), and the ascending and descending pairs of
// ranks pass through one per-column buffer in turn.
template <int NT, int V>
__global__ void __launch_bounds__(NT) k_pscan(const float* __restrict__ X, const uint8_t* __restrict__ mask, int N,
                                              ScanOut outs) {
  constexpr int C = 4 * V;
  extern __shared__ __align__(16) uint8_t sm[];
  const SortedLayout<NT> L(N);
  unsigned long long* scan64 = reinterpret_cast<unsigned long long*>(sm + L.red);
  uint32_t* scan32 = reinterpret_cast<uint32_t*>(sm + L.red);
  uint32_t* bits = reinterpret_cast<uint32_t*>(sm + L.dw);  // tie-group start per sorted position
  uint32_t* k0 = reinterpret_cast<uint32_t*>(sm + L.k0);
  uint32_t* k1 = reinterpret_cast<uint32_t*>(sm + L.k1);
  uint16_t* i0 = reinterpret_cast<uint16_t*>(sm + L.i0);
  uint16_t* i1 = reinterpret_cast<uint16_t*>(sm + L.i1);
  const int tid = static_cast<int>(threadIdx.x);
  const size_t row = static_cast<size_t>(blockIdx.x) * N;
  for (int k = tid; k < (N + 31) / 32 + 1; k += NT) bits[k] = 0u;
  float x[C];
  uint32_t mk[C];
  load_row_f32<NT, V, true>(X + row, N, x);
  load_mask4<NT, V>(mask != nullptr ? mask + row : nullptr, N, mk);
  uint32_t fin = 0u, msk = 0u;
#pragma unroll
  for (int c = 0; c < C; ++c) {
    fin |= (finite_f32(x[c]) ? 1u : 0u) << c;
    msk |= (mk[c] ? 1u : 0u) << c;
  }
  int base[V];
  const int m = compact_bases<NT, V>(fin, base, scan64);  // its barriers publish the bitmap clear
#pragma unroll
  for (int j = 0; j < V; ++j) {
    int p = base[j];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int c = 4 * j + k;
      if ((fin >> c) & 1u) {
        k0[p] = key_f32(x[c]);
        i0[p] = static_cast<uint16_t>((4 * (j * NT + tid) + k) | (((msk >> c) & 1u) << 15));
        ++p;
      }
    }
  }
  __syncthreads();
  uint32_t* ks;
  uint16_t* is;
  block_radix_sort<NT, C, uint32_t>(k0, i0, k1, i1, m, sm + L.scratch, &ks, &is);
  uint16_t* S = (is == i0) ? i1 : i0;                                // group start per sorted position
  uint32_t* O = (ks == k0) ? k1 : k0;                                // two ranks per column
  uint16_t* Cn = reinterpret_cast<uint16_t*>(ks);                    // m + 1 entries, over the sorted keys
  uint16_t* GE = reinterpret_cast<uint16_t*>(ks) + (N + 1);          // group end by group start
  // pass 1: per chunk, masked-valid count, last group start, start bits
  const int per = (m + NT - 1) / NT;
  const int b0 = tid * per, b1 = min(m, b0 + per);
  uint32_t cm = 0;
  int last = -1;
  for (int p = b0; p < b1; ++p) {
    cm += is[p] >> 15;
    if (p == 0 || ks[p] != ks[p - 1]) {
      last = p;
      atomicOr(&bits[p >> 5], 1u << (p & 31));
    }
  }
  uint32_t mt;
  uint32_t c = block_exclusive_sum(cm, scan32, mt);  // barriers: ks reads done, bits complete
  // exclusive max-scan of the chunks' last group starts (identity -1)
  int inc = last;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int u = __shfl_up_sync(kFull, inc, o);
    if (lane_id() >= static_cast<unsigned>(o)) inc = max(inc, u);
  }
  const int wi = tid >> 5;
  int* sc = reinterpret_cast<int*>(scan64);
  if (lane_id() == 31) sc[wi] = inc;
  __syncthreads();
  int carry = -1;
  for (int i = 0; i < wi; ++i) carry = max(carry, sc[i]);
  const int up = __shfl_up_sync(kFull, inc, 1);
  if (lane_id() > 0) carry = max(carry, up);
  // pass 2: S, the masked-valid prefix C and the group ends E
  auto is_start = [&](int p) { return ((bits[p >> 5] >> (p & 31)) & 1u) != 0u; };
  for (int p = b0; p < b1; ++p) {
    if (is_start(p)) carry = p;
    S[p] = static_cast<uint16_t>(carry);
    Cn[p] = static_cast<uint16_t>(c);
    c += is[p] >> 15;
    if (p == m - 1 || is_start(p + 1)) GE[carry] = static_cast<uint16_t>(p + 1);
  }
  if (tid == 0) Cn[m] = static_cast<uint16_t>(mt);
  __syncthreads();
  const float qnan = __uint_as_float(kQuietNanBits);
  // pass 3, twice: the ascending pair (groups 0 | 1), then the descending pair
  // (groups 2 | 3), each stored by column and written out
  for (int half = 0; half < 2; ++half) {
    if (outs.out[2 * half] == nullptr && outs.out[2 * half + 1] == nullptr) continue;  // uniform
    for (int p = tid; p < m; p += NT) {
      const uint32_t id = is[p];
      const uint32_t cp = Cn[p];
      uint32_t lo = 0u, hi;
      if (half == 0) {
        hi = static_cast<uint32_t>(p + 1);
        if (id & 0x8000u) lo = cp + 1u;
      } else {
        const int s0 = S[p], e0 = GE[s0];
        hi = static_cast<uint32_t>(m - e0 + (p - s0) + 1);
        if (id & 0x8000u) lo = mt - Cn[e0] + (cp - Cn[s0]) + 1u;
      }
      O[id & 0x3FFFu] = lo | (hi << 16);
    }
    __syncthreads();
#pragma unroll
    for (int g2 = 0; g2 < 2; ++g2) {
      float* dst = outs.out[2 * half + g2];
      if (dst == nullptr) continue;  // uniform
      const int sh = g2 ? 16 : 0;
      float v[C];
#pragma unroll
      for (int cc = 0; cc < C; ++cc) {
        const uint32_t r =
            ((fin >> cc) & 1u) ? ((O[4 * ((cc >> 2) * NT + tid) + (cc & 3)] >> sh) & 0xFFFFu) : 0u;
        v[cc] = r ? static_cast<float>(r) : qnan;
      }
      store_row_f32v<NT, V>(dst + row, N, v);
    }
    __syncthreads();  // O is rewritten by the second half
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
namespace {
// NT, V: the returns pass and the radix kernel; LT, LV: the learned kernel.
template <int NT, int V, int LT, int LV>
cudaError_t ric_launch(const RankIcArgs<float, float>& a, RicPrep rp, bool learned, cudaStream_t st) {
  const size_t smem_s = SortedLayout<NT>(a.N).total;
  const size_t smem_b = BucketLayout(a.N).total;
  if (smem_s > kMaxSmemPerBlock || smem_b > kMaxSmemPerBlock) return cudaErrorInvalidValue;
  if (a.N > 4 * NT * V || a.N > 4 * LT * LV) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(k_ric_prep<NT, V>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem_s));
  if (e != cudaSuccess) return e;
  k_ric_prep<NT, V><<<a.T, NT, smem_s, st>>>(a.R, a.rmask, a.fmask, a.N, rp);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  const long long grid = static_cast<long long>(a.T) * a.F;
  if (grid > 2147483647LL) return cudaErrorInvalidValue;
  if (!learned) {
    if ((e = cudaFuncSetAttribute(k_ric_radix<NT, V, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(smem_s))) != cudaSuccess)
      return e;
    k_ric_radix<NT, V, false><<<static_cast<unsigned>(grid), NT, smem_s, st>>>(a, rp);
    return cudaGetLastError();
  }
  if ((e = cudaFuncSetAttribute(k_ric_learned<LT, LV>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(smem_b))) != cudaSuccess)
    return e;
  k_ric_learned<LT, LV><<<static_cast<unsigned>(grid), LT, smem_b, st>>>(a, rp);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  // the radix kernel takes the sections the learned kernel handed back;
  // persistent CTAs (one wave) read the list length on the device and exit at
  // once when it is empty
  if ((e = cudaFuncSetAttribute(k_ric_radix<NT, V, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(smem_s))) != cudaSuccess)
    return e;
  int occ = 0, dev = 0, sms = 0;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_ric_radix<NT, V, true>, NT, smem_s)) != cudaSuccess)
    return e;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  long long fb_grid = static_cast<long long>(occ > 0 ? occ : 1) * (sms > 0 ? sms : 1);
  if (fb_grid > grid) fb_grid = grid;
  k_ric_radix<NT, V, true><<<static_cast<unsigned>(fb_grid), NT, smem_s, st>>>(a, rp);
  return cudaGetLastError();
}
}  // namespace

size_t ric_prep_bytes(int T, int N, int F) {
  const size_t ld = (static_cast<size_t>(N) + 3) / 4 * 4;
  return static_cast<size_t>(T) * ld * 4 + 256 + (static_cast<size_t>(T) * F + 64) * 4 + 256;
}

RicPrep ric_prep_carve(void* base, int T, int N, int F) {
  RicPrep rp{};
  rp.ld = (N + 3) / 4 * 4;
  uint8_t* p = static_cast<uint8_t*>(base);
  rp.word = reinterpret_cast<uint32_t*>(p);
  p += (static_cast<size_t>(T) * rp.ld * 4 + 255) & ~size_t(255);
  rp.fb_count = reinterpret_cast<int*>(p);
  p += 256;
  rp.fb_items = reinterpret_cast<int*>(p);
  (void)F;
  return rp;
}


namespace {
template <int NT, int V>
cudaError_t csr_launch(const float* X, const uint8_t* mask, int T, int N, int desc, float* out, cudaStream_t st) {
  const size_t smem = SortedLayout<NT>(N).total;
  cudaError_t e = cudaFuncSetAttribute(k_csr<NT, V>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  k_csr<NT, V><<<T, NT, smem, st>>>(X, mask, N, desc, out);
  return cudaGetLastError();
}
template <int NT, int V>
cudaError_t pscan_launch(const float* X, const uint8_t* mask, int T, int N, ScanOut outs, cudaStream_t st) {
  const size_t smem = SortedLayout<NT>(N).total;
  if (smem > kMaxSmemPerBlock) return cudaErrorInvalidValue;
  cudaError_t e =
      cudaFuncSetAttribute(k_pscan<NT, V>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  k_pscan<NT, V><<<T, NT, smem, st>>>(X, mask, N, outs);
  return cudaGetLastError();
}
}  // namespace


// The per-date rank kernels stage nothing through mbarriers, so `status` has
// nothing to report; it is kept for the callers' uniform interface.
cudaError_t launch_cs_rank(const float* X, const uint8_t* mask, int T, int N, int desc, float* out, int* status,
                           cudaStream_t st) {
  (void)status;
  if (N < 1 || N > kSmemRankCap) return cudaErrorInvalidValue;
  if (N <= 2048) return csr_launch<256, 2>(X, mask, T, N, desc, out, st);
  if (N <= 5120) return csr_launch<256, 5>(X, mask, T, N, desc, out, st);
  if (N <= 8192) return csr_launch<512, 4>(X, mask, T, N, desc, out, st);
  return csr_launch<512, 8>(X, mask, T, N, desc, out, st);
}

cudaError_t launch_param_scan(const float* X, const uint8_t* mask, int T, int N, ScanOut outs, int* status,
                              cudaStream_t st) {
  (void)status;
  if (N < 1 || N > kSmemRankCap) return cudaErrorInvalidValue;
  if (N <= 2048) return pscan_launch<256, 2>(X, mask, T, N, outs, st);
  if (N <= 5120) return pscan_launch<256, 5>(X, mask, T, N, outs, st);
  if (N <= 8192) return pscan_launch<512, 4>(X, mask, T, N, outs, st);
  return pscan_launch<512, 8>(X, mask, T, N, outs, st);
}

namespace {
template <int NT, int V>
cudaError_t ric_batch_launch(const RicBatchVariant& v, cudaStream_t st) {
  const size_t smem_s = SortedLayout<NT>(v.maxN).total;
  const size_t smem_b = BucketLayout(v.maxN).total;
  const size_t smem_l = smem_s > smem_b ? smem_s : smem_b;
  if (smem_l > kMaxSmemPerBlock) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(k_ric_prep_batch<NT, V>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem_s));
  if (e != cudaSuccess) return e;
  k_ric_prep_batch<NT, V><<<v.dates, NT, smem_s, st>>>(v.panels, v.off_dates, v.np, v.fb);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (!v.learned) {
    if ((e = cudaFuncSetAttribute(k_ric_items_batch<NT, V, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(smem_s))) != cudaSuccess)
      return e;
    k_ric_items_batch<NT, V, false><<<v.items, NT, smem_s, st>>>(v.panels, v.off_items, v.np, v.fb);
    return cudaGetLastError();
  }
  if ((e = cudaFuncSetAttribute(k_ric_items_batch<NT, V, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(smem_l))) != cudaSuccess)
    return e;
  k_ric_items_batch<NT, V, true><<<v.items, NT, smem_l, st>>>(v.panels, v.off_items, v.np, v.fb);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = cudaFuncSetAttribute(k_ric_list_batch<NT, V>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(smem_s))) != cudaSuccess)
    return e;
  int occ = 0, dev = 0, sms = 0;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_ric_list_batch<NT, V>, NT, smem_s)) != cudaSuccess)
    return e;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  long long g = static_cast<long long>(occ > 0 ? occ : 1) * (sms > 0 ? sms : 1);
  if (g > v.items) g = v.items;
  k_ric_list_batch<NT, V><<<static_cast<unsigned>(g), NT, smem_s, st>>>(v.panels, v.off_items, v.np, v.fb);
  return cudaGetLastError();
}
}  // namespace

int ric_variant_cap(int variant) {
  static const int caps[kRicVariants] = {2048, 5120, 8192, 16384};
  return (variant >= 0 && variant < kRicVariants) ? caps[variant] : 0;
}

cudaError_t launch_rank_ic_items_batch(int variant, const RicBatchVariant& v, cudaStream_t st) {
  if (v.np < 1 || v.items < 1 || v.maxN > ric_variant_cap(variant)) return cudaErrorInvalidValue;
  switch (variant) {
    case 0: return ric_batch_launch<256, 2>(v, st);
    case 1: return ric_batch_launch<256, 5>(v, st);
    case 2: return ric_batch_launch<512, 4>(v, st);
    default: return ric_batch_launch<512, 8>(v, st);
  }
}

bool ric_items_fit(int N) { return N >= 1 && N <= kSmemRankCap; }

cudaError_t launch_rank_ic_items(const RankIcArgs<float, float>& a, RicPrep rp, bool learned, cudaStream_t st) {
  if (!ric_items_fit(a.N) || a.rank_f_out != nullptr || a.rank_r_out != nullptr) return cudaErrorInvalidValue;
  if (learned && (a.cdf_table == nullptr || a.cdf_zrange == nullptr)) return cudaErrorInvalidValue;
  // the learned kernel runs 512 threads of three cells per vector from 2049 to
  // 6144 columns (shorter per-thread chains than 256 threads of five)
  if (a.N <= 2048) return ric_launch<256, 2, 256, 2>(a, rp, learned, st);
  if (a.N <= 5120) return ric_launch<256, 5, 512, 3>(a, rp, learned, st);
  if (a.N <= 6144) return ric_launch<512, 4, 512, 3>(a, rp, learned, st);
  if (a.N <= 8192) return ric_launch<512, 4, 512, 4>(a, rp, learned, st);
  return ric_launch<512, 8, 512, 8>(a, rp, learned, st);
}

}  // namespace fcb
