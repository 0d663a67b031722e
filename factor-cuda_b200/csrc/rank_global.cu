// rank_global.cu -- cross-sectional ranks for sections too wide for one CTA's
// shared memory (N above the shared-memory kernels' capacity, up to the
// reference's 2^24 cap: src/cross_sectional_rank.cu:233-235).
//
// Same results as the shared-memory kernels (rank_kernels.cu), by the same
// construction: the valid cells of a row are compacted in column order into
// (key, column) pairs, sorted stably by key, and every output is read off the
// sorted order(s).  Here the pairs live in global memory and each row is
// sorted by one CTA with a stable LSD radix sort: per 8-bit digit, a histogram
// of the whole row gives each digit's base; the row then streams through
// shared memory in tiles of 8192 pairs, each tile is partitioned stably by the
// digit (radix_pass of block_sort.cuh) and written to its digits' running
// bases -- tiles in order, positions within a tile in order, so the pass is
// stable.  Digits on which all keys of the row agree are skipped.
//
// Ordered prefix counts over the sorted orders (joint-set ranks, masked ranks,
// tie groups) run as block-wide scans over tiles of 4096 positions with a
// running carry.  The per-chunk scratch (pairs, double buffers, prefix arrays)
// is passed in by the host; dates are processed in chunks that fit it.
#include <algorithm>

#include "block_sort.cuh"
#include "fcb_kernels.h"

namespace fcb {
namespace {

constexpr int GNT = 1024;        // threads per CTA
constexpr int GTILE = GNT * 8;   // pairs per sort tile (radix_pass capacity)
constexpr int GIPT = 4;          // positions per thread per scan tile

template <typename K>
struct GSortSmem {
  static constexpr size_t tk = 0;
  static constexpr size_t tk2 = tk + size_t(GTILE) * sizeof(K);
  static constexpr size_t tidx = tk2 + size_t(GTILE) * sizeof(K);
  static constexpr size_t tp = tidx + size_t(GTILE) * 4;
  static constexpr size_t tp2 = tp + size_t(GTILE) * 2;
  static constexpr size_t scratch = tp2 + size_t(GTILE) * 2;
  static constexpr size_t gbase = scratch + SortScratch<GNT>::bytes;
  static constexpr size_t ghist = gbase + 256 * 4;
  static constexpr size_t red = ghist + 256 * 4;
  static constexpr size_t total = red + 66 * sizeof(unsigned long long) + 16;
};
static_assert(SortScratch<GNT>::bytes % 16 == 0, "scratch keeps 16-byte alignment");

// Stable LSD radix sort of row blockIdx.x: (kA, iA)[0, cnt) -> sorted in A
// (sel = 0) or B (sel = 1).
template <typename K>
__global__ void __launch_bounds__(GNT, 1) k_g_sort(K* __restrict__ kA, uint32_t* __restrict__ iA, K* __restrict__ kB,
                                                   uint32_t* __restrict__ iB, const uint32_t* __restrict__ cnt,
                                                   size_t stride, uint8_t* __restrict__ sel) {
  extern __shared__ __align__(16) uint8_t sm[];
  using L = GSortSmem<K>;
  K* tk = reinterpret_cast<K*>(sm + L::tk);
  K* tk2 = reinterpret_cast<K*>(sm + L::tk2);
  uint32_t* tidx = reinterpret_cast<uint32_t*>(sm + L::tidx);
  uint16_t* tp = reinterpret_cast<uint16_t*>(sm + L::tp);
  uint16_t* tp2 = reinterpret_cast<uint16_t*>(sm + L::tp2);
  uint16_t* whist = reinterpret_cast<uint16_t*>(sm + L::scratch);
  uint32_t* dbase = reinterpret_cast<uint32_t*>(sm + L::scratch + SortScratch<GNT>::hist_bytes);
  uint32_t* scan =
      reinterpret_cast<uint32_t*>(sm + L::scratch + SortScratch<GNT>::hist_bytes + SortScratch<GNT>::base_bytes);
  uint32_t* gbase = reinterpret_cast<uint32_t*>(sm + L::gbase);
  uint32_t* ghist = reinterpret_cast<uint32_t*>(sm + L::ghist);
  K* red = reinterpret_cast<K*>(sm + L::red);
  const size_t off = static_cast<size_t>(blockIdx.x) * stride;
  const int m = static_cast<int>(cnt[blockIdx.x]);
  K* ks = kA + off;
  uint32_t* is = iA + off;
  K* kd = kB + off;
  uint32_t* id = iB + off;
  K a, o;
  block_and_or(ks, m, a, o, red);
  const K diff = a ^ o;
  uint8_t which = 0;
  constexpr int KB = int(sizeof(K) * 8);
  for (int shift = 0; shift < KB; shift += kRadixBits) {
    if (((diff >> shift) & K(kRadix - 1)) == 0) continue;  // uniform across the block
    if (threadIdx.x < kRadix) ghist[threadIdx.x] = 0u;
    __syncthreads();
    for (int p = threadIdx.x; p < m; p += GNT)
      atomicAdd(&ghist[static_cast<uint32_t>((ks[p] >> shift) & K(kRadix - 1))], 1u);
    __syncthreads();
    uint32_t tot;
    const uint32_t v = threadIdx.x < kRadix ? ghist[threadIdx.x] : 0u;
    const uint32_t ex = block_exclusive_sum(v, scan, tot);
    if (threadIdx.x < kRadix) gbase[threadIdx.x] = ex;
    __syncthreads();
    for (int t0 = 0; t0 < m; t0 += GTILE) {
      const int n = min(GTILE, m - t0);
      for (int q = threadIdx.x; q < n; q += GNT) {
        tk[q] = ks[t0 + q];
        tidx[q] = is[t0 + q];
        tp[q] = static_cast<uint16_t>(q);
      }
      __syncthreads();
      radix_pass<GNT, 8, K>(tk, tp, tk2, tp2, n, shift, whist, dbase, scan);
      for (int q = threadIdx.x; q < n; q += GNT) {
        const K k = tk2[q];
        const uint32_t d = static_cast<uint32_t>((k >> shift) & K(kRadix - 1));
        const uint32_t dst = gbase[d] + (static_cast<uint32_t>(q) - dbase[d]);
        kd[dst] = k;
        id[dst] = tidx[tp2[q]];
      }
      __syncthreads();
      if (threadIdx.x < kRadix) {
        const uint32_t e = threadIdx.x < kRadix - 1 ? dbase[threadIdx.x + 1] : static_cast<uint32_t>(n);
        gbase[threadIdx.x] += e - dbase[threadIdx.x];
      }
      __syncthreads();
    }
    K* tkk = ks;
    ks = kd;
    kd = tkk;
    uint32_t* tii = is;
    is = id;
    id = tii;
    which ^= 1;
  }
  if (threadIdx.x == 0) sel[blockIdx.x] = which;
}

// Ordered selection over positions [0, m): body(p, r) for every p with
// pred(p), r = number of selected positions before p.  Returns the total.
// All threads must call.
template <typename Pred, typename Body>
FCB_DEV uint32_t g_select(int m, Pred pred, Body body, uint32_t* scan) {
  uint32_t carry = 0;
  for (int base = 0; base < m; base += GNT * GIPT) {
    const int p0 = base + static_cast<int>(threadIdx.x) * GIPT;
    bool f[GIPT];
    uint32_t c = 0;
#pragma unroll
    for (int j = 0; j < GIPT; ++j) {
      f[j] = (p0 + j < m) && pred(p0 + j);
      c += f[j] ? 1u : 0u;
    }
    uint32_t tot;
    uint32_t r = carry + block_exclusive_sum(c, scan, tot);
#pragma unroll
    for (int j = 0; j < GIPT; ++j)
      if (f[j]) body(p0 + j, r++);
    carry += tot;
  }
  return carry;
}

// Exclusive max-scan of one int per thread in thread order (identity -1).
FCB_DEV int g_excl_max(int v, int* scratch) {
  int inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int u = __shfl_up_sync(kFull, inc, o);
    if (lane_id() >= static_cast<unsigned>(o)) inc = max(inc, u);
  }
  const int w = threadIdx.x >> 5;
  if (lane_id() == 31) scratch[w] = inc;
  __syncthreads();
  if (w == 0) {
    const int s = scratch[lane_id()];
    int si = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(kFull, si, o);
      if (lane_id() >= static_cast<unsigned>(o)) si = max(si, u);
    }
    int ex = __shfl_up_sync(kFull, si, 1);
    if (lane_id() == 0) ex = -1;
    scratch[lane_id()] = ex;
  }
  __syncthreads();
  int el = __shfl_up_sync(kFull, inc, 1);
  if (lane_id() == 0) el = -1;
  const int res = max(scratch[w], el);
  __syncthreads();
  return res;
}

// ---------------------------------------------------------------- cs_rank
__global__ void __launch_bounds__(GNT) k_g_cs_compact(const float* __restrict__ X, const uint8_t* __restrict__ mask,
                                                      int N, int desc, int t0, uint32_t* __restrict__ kA,
                                                      uint32_t* __restrict__ iA, uint32_t* __restrict__ cnt,
                                                      size_t stride) {
  __shared__ uint32_t scan[80];
  const size_t row = static_cast<size_t>(t0 + blockIdx.x) * N;
  const float* x = X + row;
  const uint8_t* mk = mask == nullptr ? nullptr : mask + row;
  uint32_t* k = kA + blockIdx.x * stride;
  uint32_t* ix = iA + blockIdx.x * stride;
  const uint32_t m = g_select(
      N, [&](int i) { return finite_f32(x[i]) && (mk == nullptr || mk[i] != 0); },
      [&](int i, uint32_t r) {
        k[r] = key_f32(desc ? -x[i] : x[i]);
        ix[r] = static_cast<uint32_t>(i);
      },
      scan);
  if (threadIdx.x == 0) cnt[blockIdx.x] = m;
}

__global__ void __launch_bounds__(GNT) k_g_cs_out(const uint32_t* __restrict__ iA, const uint32_t* __restrict__ iB,
                                                  const uint8_t* __restrict__ sel, const uint32_t* __restrict__ cnt,
                                                  size_t stride, int N, int t0, float* __restrict__ out) {
  const uint32_t* is = (sel[blockIdx.x] ? iB : iA) + blockIdx.x * stride;
  const int m = static_cast<int>(cnt[blockIdx.x]);
  float* o = out + static_cast<size_t>(t0 + blockIdx.x) * N;
  const float qnan = __uint_as_float(kQuietNanBits);
  for (int i = threadIdx.x; i < N; i += GNT) o[i] = qnan;
  __syncthreads();
  for (int p = threadIdx.x; p < m; p += GNT) o[is[p]] = static_cast<float>(p + 1);
}

// ---------------------------------------------------------- parameter_scan
__global__ void __launch_bounds__(GNT) k_g_scan_compact(const float* __restrict__ X, int N, int t0,
                                                        uint32_t* __restrict__ kA, uint32_t* __restrict__ iA,
                                                        uint32_t* __restrict__ cnt, size_t stride) {
  __shared__ uint32_t scan[80];
  const float* x = X + static_cast<size_t>(t0 + blockIdx.x) * N;
  uint32_t* k = kA + blockIdx.x * stride;
  uint32_t* ix = iA + blockIdx.x * stride;
  const uint32_t m = g_select(
      N, [&](int i) { return finite_f32(x[i]); },
      [&](int i, uint32_t r) {
        k[r] = key_f32(x[i]);
        ix[r] = static_cast<uint32_t>(i);
      },
      scan);
  if (threadIdx.x == 0) cnt[blockIdx.x] = m;
}

// Groups as in k_param_scan: 0 ascending masked, 1 ascending unmasked,
// 2 descending masked, 3 descending unmasked.  C[p]: masked cells before
// sorted position p (C[m] = their total); S[p]: start of p's tie group;
// GE[s]: one past the end of the group starting at s.
__global__ void __launch_bounds__(GNT) k_g_scan_out(const uint32_t* __restrict__ kA, const uint32_t* __restrict__ kB,
                                                    const uint32_t* __restrict__ iA, const uint32_t* __restrict__ iB,
                                                    const uint8_t* __restrict__ sel, const uint32_t* __restrict__ cnt,
                                                    size_t stride, const uint8_t* __restrict__ mask, int N, int t0,
                                                    uint32_t* __restrict__ Cb, uint32_t* __restrict__ Sb,
                                                    uint32_t* __restrict__ GEb, ScanOut outs) {
  __shared__ uint32_t scan[80];
  const bool b = sel[blockIdx.x] != 0;
  const uint32_t* ks = (b ? kB : kA) + blockIdx.x * stride;
  const uint32_t* is = (b ? iB : iA) + blockIdx.x * stride;
  const int m = static_cast<int>(cnt[blockIdx.x]);
  const size_t row = static_cast<size_t>(t0 + blockIdx.x) * N;
  const uint8_t* mk = mask == nullptr ? nullptr : mask + row;
  uint32_t* C = Cb + blockIdx.x * (stride + 1);
  uint32_t* S = Sb + blockIdx.x * stride;
  uint32_t* GE = GEb + blockIdx.x * stride;
  const bool need_desc = outs.out[2] != nullptr || outs.out[3] != nullptr;
  const bool need_mask = outs.out[0] != nullptr || outs.out[2] != nullptr;
  uint32_t mtot = static_cast<uint32_t>(m);
  if (need_mask) {
    // C[p] for every p: exclusive prefix count of masked cells
    uint32_t carry = 0;
    for (int base = 0; base < m; base += GNT * GIPT) {
      const int p0 = base + static_cast<int>(threadIdx.x) * GIPT;
      uint32_t c = 0;
#pragma unroll
      for (int j = 0; j < GIPT; ++j)
        if (p0 + j < m && (mk == nullptr || mk[is[p0 + j]] != 0)) ++c;
      uint32_t tot;
      uint32_t r = carry + block_exclusive_sum(c, scan, tot);
#pragma unroll
      for (int j = 0; j < GIPT; ++j) {
        const int p = p0 + j;
        if (p < m) {
          C[p] = r;
          if (mk == nullptr || mk[is[p]] != 0) ++r;
        }
      }
      carry += tot;
    }
    mtot = carry;
    if (threadIdx.x == 0) C[m] = carry;
  }
  if (need_desc) {
    // S[p]: running maximum of group starts (start: p == 0 or key change)
    int carry = -1;
    for (int base = 0; base < m; base += GNT * GIPT) {
      const int p0 = base + static_cast<int>(threadIdx.x) * GIPT;
      int last = -1;
#pragma unroll
      for (int j = 0; j < GIPT; ++j) {
        const int p = p0 + j;
        if (p < m && (p == 0 || ks[p] != ks[p - 1])) last = p;
      }
      int run = max(carry, g_excl_max(last, reinterpret_cast<int*>(scan)));
#pragma unroll
      for (int j = 0; j < GIPT; ++j) {
        const int p = p0 + j;
        if (p < m) {
          if (p == 0 || ks[p] != ks[p - 1]) run = p;
          S[p] = static_cast<uint32_t>(run);
        }
      }
      carry = max(carry, block_max_int(last, reinterpret_cast<int*>(scan)));
    }
    __syncthreads();
    for (int p = threadIdx.x; p < m; p += GNT)
      if (p == m - 1 || ks[p] != ks[p + 1]) GE[S[p]] = static_cast<uint32_t>(p + 1);
  }
  __syncthreads();
  const float qnan = __uint_as_float(kQuietNanBits);
  for (int g = 0; g < 4; ++g) {
    float* o = outs.out[g];
    if (o == nullptr) continue;
    o += row;
    for (int i = threadIdx.x; i < N; i += GNT) o[i] = qnan;
    __syncthreads();
    for (int p = threadIdx.x; p < m; p += GNT) {
      const int i = static_cast<int>(is[p]);
      const bool mv = (mk == nullptr || mk[i] != 0);
      switch (g) {
        case 0:
          if (mv) o[i] = static_cast<float>(C[p] + 1);
          break;
        case 1:
          o[i] = static_cast<float>(p + 1);
          break;
        case 2:
          if (mv) {
            const uint32_t s = S[p], e = GE[s];
            o[i] = static_cast<float>(static_cast<long long>(mtot) - C[e] + (C[p] - C[s]) + 1);
          }
          break;
        default: {
          const uint32_t s = S[p], e = GE[s];
          o[i] = static_cast<float>(static_cast<long long>(m) - e + (p - static_cast<int>(s)) + 1);
        }
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------- rank + IC
template <typename TR>
__global__ void __launch_bounds__(GNT) k_g_ric_compact_r(const TR* __restrict__ R, const uint8_t* __restrict__ rmask,
                                                         int N, int t0, typename KeyOf<TR>::type* __restrict__ kA,
                                                         uint32_t* __restrict__ iA, uint32_t* __restrict__ cnt,
                                                         size_t stride) {
  __shared__ uint32_t scan[80];
  const size_t row = static_cast<size_t>(t0 + blockIdx.x) * N;
  const TR* r = R + row;
  const uint8_t* rm = rmask == nullptr ? nullptr : rmask + row;
  auto* k = kA + blockIdx.x * stride;
  uint32_t* ix = iA + blockIdx.x * stride;
  const uint32_t m = g_select(
      N, [&](int i) { return KeyOf<TR>::finite(r[i]) && (rm == nullptr || rm[i] != 0); },
      [&](int i, uint32_t q) {
        k[q] = KeyOf<TR>::key(r[i]);
        ix[q] = static_cast<uint32_t>(i);
      },
      scan);
  if (threadIdx.x == 0) cnt[blockIdx.x] = m;
}

// grid (Tc, F): row = f * Tc + date-in-chunk
template <typename TF>
__global__ void __launch_bounds__(GNT) k_g_ric_compact_f(const TF* __restrict__ X, const uint8_t* __restrict__ fmask,
                                                         int T, int N, int t0, typename KeyOf<TF>::type* __restrict__ kA,
                                                         uint32_t* __restrict__ iA, uint32_t* __restrict__ cnt,
                                                         size_t stride) {
  __shared__ uint32_t scan[80];
  const int rr = blockIdx.y * gridDim.x + blockIdx.x;
  const int t = t0 + blockIdx.x;
  const TF* x = X + (static_cast<size_t>(blockIdx.y) * T + t) * N;
  const uint8_t* fm = fmask == nullptr ? nullptr : fmask + static_cast<size_t>(t) * N;
  auto* k = kA + rr * stride;
  uint32_t* ix = iA + rr * stride;
  const uint32_t m = g_select(
      N, [&](int i) { return KeyOf<TF>::finite(x[i]) && (fm == nullptr || fm[i] != 0); },
      [&](int i, uint32_t q) {
        k[q] = KeyOf<TF>::key(x[i]);
        ix[q] = static_cast<uint32_t>(i);
      },
      scan);
  if (threadIdx.x == 0) cnt[rr] = m;
}

FCB_DEV double g_spearman(long long m, long long sum_rr) {
  const long long s4 = 4 * sum_rr - m * (m + 1) * (m + 1);
  const long long q4 = m * (m * m - 1) / 3;
  const double sxy = static_cast<double>(s4) * 0.25;
  const double sxx = static_cast<double>(q4) * 0.25;
  return (sxy / sqrt(sxx)) / sqrt(sxx);
}

struct GRicBufs {
  void *kRA, *kRB, *kFA, *kFB;
  uint32_t *iRA, *iRB, *iFA, *iFB, *cntR, *cntF, *RR;
  uint8_t *selR, *selF;
  size_t stride;
};

// grid (Tc, F): returns-side joint ranks of factor f at date t0 + x, then the
// factor side (cs ranks, joint ranks, sum of rank products) and the IC.
template <typename TF, typename TR>
__global__ void __launch_bounds__(GNT) k_g_ric_out(RankIcArgs<TF, TR> a, int t0, GRicBufs g) {
  using KF = typename KeyOf<TF>::type;
  using KR = typename KeyOf<TR>::type;
  __shared__ uint32_t scan[80];
  __shared__ unsigned long long scan64[80];
  const int dc = blockIdx.x, f = blockIdx.y, Tc = gridDim.x;
  const int t = t0 + dc;
  const int N = a.N;
  const size_t row = static_cast<size_t>(t) * N;
  const size_t frow = (static_cast<size_t>(f) * a.T + t) * N;
  const TF* x = a.X + frow;
  const TR* r = a.R + row;
  const uint8_t* fm = a.fmask == nullptr ? nullptr : a.fmask + row;
  const uint8_t* rm = a.rmask == nullptr ? nullptr : a.rmask + row;
  auto joint = [&](uint32_t i) {
    return KeyOf<TF>::finite(x[i]) && (fm == nullptr || fm[i] != 0) && KeyOf<TR>::finite(r[i]) &&
           (rm == nullptr || rm[i] != 0);
  };
  const bool rb = g.selR[dc] != 0;
  const KR* kRs = static_cast<const KR*>(rb ? g.kRB : g.kRA) + dc * g.stride;
  const uint32_t* iRs = (rb ? g.iRB : g.iRA) + dc * g.stride;
  const int mr = static_cast<int>(g.cntR[dc]);
  const int fr = f * Tc + dc;
  const bool fb = g.selF[fr] != 0;
  const KF* kFs = static_cast<const KF*>(fb ? g.kFB : g.kFA) + fr * g.stride;
  const uint32_t* iFs = (fb ? g.iFB : g.iFA) + fr * g.stride;
  const int mf = static_cast<int>(g.cntF[fr]);
  uint32_t* RR = g.RR + fr * g.stride;
  // returns side
  int rfirst = 0x7fffffff, rlast = -1;
  const uint32_t mj = g_select(
      mr, [&](int p) { return joint(iRs[p]); },
      [&](int p, uint32_t q) {
        RR[iRs[p]] = q + 1;
        rfirst = min(rfirst, p);
        rlast = max(rlast, p);
      },
      scan);
  rfirst = block_min_int(rfirst, reinterpret_cast<int*>(scan));
  rlast = block_max_int(rlast, reinterpret_cast<int*>(scan));
  // factor side
  if (a.ranks_out != nullptr) {
    const float qnan = __uint_as_float(kQuietNanBits);
    for (int i = threadIdx.x; i < N; i += GNT) a.ranks_out[frow + i] = qnan;
  }
  if (a.rank_f_out != nullptr) {
    for (int i = threadIdx.x; i < N; i += GNT) {
      a.rank_f_out[frow + i] = 0.0;
      a.rank_r_out[frow + i] = 0.0;
    }
  }
  __syncthreads();
  if (a.ranks_out != nullptr)
    for (int p = threadIdx.x; p < mf; p += GNT) a.ranks_out[frow + iFs[p]] = static_cast<float>(p + 1);
  unsigned long long sum = 0;
  int ffirst = 0x7fffffff, flast = -1;
  (void)g_select(
      mf, [&](int p) { return joint(iFs[p]); },
      [&](int p, uint32_t q) {
        const uint32_t i = iFs[p];
        const uint32_t cf = q + 1;
        sum += static_cast<unsigned long long>(cf) * RR[i];
        ffirst = min(ffirst, p);
        flast = max(flast, p);
        if (a.rank_f_out != nullptr) {
          a.rank_f_out[frow + i] = static_cast<double>(cf);
          a.rank_r_out[frow + i] = static_cast<double>(RR[i]);
        }
      },
      scan);
  sum = block_sum<unsigned long long>(sum, scan64);
  ffirst = block_min_int(ffirst, reinterpret_cast<int*>(scan));
  flast = block_max_int(flast, reinterpret_cast<int*>(scan));
  if (threadIdx.x == 0) {
    double ic = __longlong_as_double(0x7ff8000000000000ll);
    const long long m = static_cast<long long>(mj);
    if (m >= a.min_valid && m >= 2) {
      const bool fconst = kFs[ffirst] == kFs[flast];
      const bool rconst = kRs[rfirst] == kRs[rlast];
      if (!fconst && !rconst) ic = g_spearman(m, static_cast<long long>(sum));
    }
    a.ic_out[static_cast<size_t>(f) * (a.ic_ld > 0 ? a.ic_ld : a.T) + t] = ic;
  }
}

inline size_t al256(size_t x) { return (x + 255) & ~size_t(255); }

template <typename K>
cudaError_t sort_rows(K* kA, uint32_t* iA, K* kB, uint32_t* iB, const uint32_t* cnt, size_t stride, uint8_t* sel,
                      int rows, cudaStream_t s) {
  const size_t smem = GSortSmem<K>::total;
  cudaError_t e = cudaFuncSetAttribute(k_g_sort<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  k_g_sort<K><<<rows, GNT, smem, s>>>(kA, iA, kB, iB, cnt, stride, sel);
  return cudaGetLastError();
}

// Bytes per date of the cs_rank / parameter_scan scratch: pairs (A, B) of
// u32 keys and u32 columns, count, buffer flag, and for the scan the prefix
// arrays C, S, GE.
size_t row_bytes(int N, bool scan) {
  const size_t n = static_cast<size_t>(N);
  return 4 * n * 4 + 16 + (scan ? (3 * n + 1) * 4 : 0);
}

int chunk_dates(size_t per_date, int T, size_t bytes) {
  const size_t budget = bytes > 4096 ? bytes - 4096 : 0;  // alignment slack
  const size_t c = per_date > 0 ? budget / per_date : 0;
  return static_cast<int>(std::min<size_t>(c, static_cast<size_t>(T)));
}

}  // namespace

size_t rank_global_bytes_per_date(int kind, int N, int F, int ksz_f, int ksz_r) {
  const size_t n = static_cast<size_t>(N);
  if (kind == 0) return row_bytes(N, false);
  if (kind == 1) return row_bytes(N, true);
  // rank + IC: returns pairs (2 x (key + column)) + F factor pairs + RR
  return 2 * n * (ksz_r + 4) + static_cast<size_t>(F) * n * (2 * (ksz_f + 4) + 4) + 16 * (F + 1) + 4096;
}

cudaError_t launch_cs_rank_global(const float* X, const uint8_t* mask, int T, int N, int desc, float* out,
                                  uint8_t* scratch, size_t bytes, cudaStream_t s) {
  const int Tc = chunk_dates(row_bytes(N, false), T, bytes);
  if (Tc < 1) return cudaErrorInvalidValue;
  const size_t n = static_cast<size_t>(Tc) * N;
  uint8_t* p = scratch;
  auto take = [&](size_t b) {
    uint8_t* q = p;
    p += al256(b);
    return q;
  };
  auto* kA = reinterpret_cast<uint32_t*>(take(n * 4));
  auto* kB = reinterpret_cast<uint32_t*>(take(n * 4));
  auto* iA = reinterpret_cast<uint32_t*>(take(n * 4));
  auto* iB = reinterpret_cast<uint32_t*>(take(n * 4));
  auto* cnt = reinterpret_cast<uint32_t*>(take(static_cast<size_t>(Tc) * 4));
  auto* sel = take(static_cast<size_t>(Tc));
  for (int t0 = 0; t0 < T; t0 += Tc) {
    const int tc = std::min(Tc, T - t0);
    k_g_cs_compact<<<tc, GNT, 0, s>>>(X, mask, N, desc, t0, kA, iA, cnt, N);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if ((e = sort_rows<uint32_t>(kA, iA, kB, iB, cnt, N, sel, tc, s)) != cudaSuccess) return e;
    k_g_cs_out<<<tc, GNT, 0, s>>>(iA, iB, sel, cnt, N, N, t0, out);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_param_scan_global(const float* X, const uint8_t* mask, int T, int N, ScanOut outs,
                                     uint8_t* scratch, size_t bytes, cudaStream_t s) {
  const int Tc = chunk_dates(row_bytes(N, true), T, bytes);
  if (Tc < 1) return cudaErrorInvalidValue;
  const size_t n = static_cast<size_t>(Tc) * N;
  uint8_t* p = scratch;
  auto take = [&](size_t b) {
    uint8_t* q = p;
    p += al256(b);
    return q;
  };
  auto* kA = reinterpret_cast<uint32_t*>(take(n * 4));
  auto* kB = reinterpret_cast<uint32_t*>(take(n * 4));
  auto* iA = reinterpret_cast<uint32_t*>(take(n * 4));
  auto* iB = reinterpret_cast<uint32_t*>(take(n * 4));
  auto* cnt = reinterpret_cast<uint32_t*>(take(static_cast<size_t>(Tc) * 4));
  auto* sel = take(static_cast<size_t>(Tc));
  auto* C = reinterpret_cast<uint32_t*>(take((n + Tc) * 4));
  auto* S = reinterpret_cast<uint32_t*>(take(n * 4));
  auto* GE = reinterpret_cast<uint32_t*>(take(n * 4));
  for (int t0 = 0; t0 < T; t0 += Tc) {
    const int tc = std::min(Tc, T - t0);
    k_g_scan_compact<<<tc, GNT, 0, s>>>(X, N, t0, kA, iA, cnt, N);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if ((e = sort_rows<uint32_t>(kA, iA, kB, iB, cnt, N, sel, tc, s)) != cudaSuccess) return e;
    k_g_scan_out<<<tc, GNT, 0, s>>>(kA, kB, iA, iB, sel, cnt, N, mask, N, t0, C, S, GE, outs);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

template <typename TF, typename TR>
cudaError_t launch_rank_ic_global(const RankIcArgs<TF, TR>& a, uint8_t* scratch, size_t bytes, cudaStream_t s) {
  using KF = typename KeyOf<TF>::type;
  using KR = typename KeyOf<TR>::type;
  const int N = a.N, F = a.F;
  const int Tc = chunk_dates(rank_global_bytes_per_date(2, N, F, sizeof(KF), sizeof(KR)), a.T, bytes);
  if (Tc < 1) return cudaErrorInvalidValue;
  const size_t n = static_cast<size_t>(Tc) * N;
  const size_t nf = n * F;
  uint8_t* p = scratch;
  auto take = [&](size_t b) {
    uint8_t* q = p;
    p += al256(b);
    return q;
  };
  GRicBufs g{};
  g.kRA = take(n * sizeof(KR));
  g.kRB = take(n * sizeof(KR));
  g.iRA = reinterpret_cast<uint32_t*>(take(n * 4));
  g.iRB = reinterpret_cast<uint32_t*>(take(n * 4));
  g.kFA = take(nf * sizeof(KF));
  g.kFB = take(nf * sizeof(KF));
  g.iFA = reinterpret_cast<uint32_t*>(take(nf * 4));
  g.iFB = reinterpret_cast<uint32_t*>(take(nf * 4));
  g.RR = reinterpret_cast<uint32_t*>(take(nf * 4));
  g.cntR = reinterpret_cast<uint32_t*>(take(static_cast<size_t>(Tc) * 4));
  g.cntF = reinterpret_cast<uint32_t*>(take(static_cast<size_t>(Tc) * F * 4));
  g.selR = take(static_cast<size_t>(Tc));
  g.selF = take(static_cast<size_t>(Tc) * F);
  g.stride = static_cast<size_t>(N);
  for (int t0 = 0; t0 < a.T; t0 += Tc) {
    const int tc = std::min(Tc, a.T - t0);
    k_g_ric_compact_r<TR><<<tc, GNT, 0, s>>>(a.R, a.rmask, N, t0, static_cast<KR*>(g.kRA), g.iRA, g.cntR, g.stride);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_g_ric_compact_f<TF><<<dim3(tc, F), GNT, 0, s>>>(a.X, a.fmask, a.T, N, t0, static_cast<KF*>(g.kFA), g.iFA,
                                                      g.cntF, g.stride);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = sort_rows<KR>(static_cast<KR*>(g.kRA), g.iRA, static_cast<KR*>(g.kRB), g.iRB, g.cntR, g.stride, g.selR,
                           tc, s)) != cudaSuccess)
      return e;
    if ((e = sort_rows<KF>(static_cast<KF*>(g.kFA), g.iFA, static_cast<KF*>(g.kFB), g.iFB, g.cntF, g.stride, g.selF,
                           tc * F, s)) != cudaSuccess)
      return e;
    k_g_ric_out<TF, TR><<<dim3(tc, F), GNT, 0, s>>>(a, t0, g);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

template cudaError_t launch_rank_ic_global<float, float>(const RankIcArgs<float, float>&, uint8_t*, size_t,
                                                          cudaStream_t);
template cudaError_t launch_rank_ic_global<float, double>(const RankIcArgs<float, double>&, uint8_t*, size_t,
                                                           cudaStream_t);
template cudaError_t launch_rank_ic_global<double, float>(const RankIcArgs<double, float>&, uint8_t*, size_t,
                                                           cudaStream_t);
template cudaError_t launch_rank_ic_global<double, double>(const RankIcArgs<double, double>&, uint8_t*, size_t,
                                                            cudaStream_t);

}  // namespace fcb
