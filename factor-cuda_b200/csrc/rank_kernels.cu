// rank_kernels.cu -- per-date in-shared-memory rank kernels for sm_100a.
//
//  (cs_rank and parameter_scan of one plane: k_csr / k_pscan in
//   rank_ic_bucket.cu.)
//  k_rank_ic      one CTA per date, looping over F factor panels: the forward
//                 returns are sorted once per date, each factor is sorted once;
//                 cs_rank ranks (own valid set) and the joint-set ranks of the
//                 Spearman IC come from prefix counts over the two sorted
//                 orders; the IC is evaluated in exact integer arithmetic
//                 (sum r_f*r_r in int64) with one f64 finalize.  Semantics of
//                 rolling_ic_gpu (src/rolling_ic.cu:306-540) / np_rolling_ic
//                 (fc/_cpu_core.py:271-293).
#include <type_traits>

#include "block_sort.cuh"
#include "fcb_kernels.h"
#include "learned_sort.cuh"

namespace fcb {

__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

// Exclusive max-scan of one int per thread (in thread order); identity -1.
FCB_DEV int block_exclusive_max(int v, int* scratch) {
  int inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int u = __shfl_up_sync(kFull, inc, o);
    if (lane_id() >= static_cast<unsigned>(o)) inc = max(inc, u);
  }
  const int w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  if (lane_id() == 31) scratch[w] = inc;
  __syncthreads();
  if (w == 0) {
    int s = (lane_id() < static_cast<unsigned>(nw)) ? scratch[lane_id()] : -1;
    int si = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int u = __shfl_up_sync(kFull, si, o);
      if (lane_id() >= static_cast<unsigned>(o)) si = max(si, u);
    }
    int ex = __shfl_up_sync(kFull, si, 1);
    if (lane_id() == 0) ex = -1;
    if (lane_id() < static_cast<unsigned>(nw)) scratch[lane_id()] = ex;
  }
  __syncthreads();
  int excl_lane = __shfl_up_sync(kFull, inc, 1);
  if (lane_id() == 0) excl_lane = -1;
  int res = max(scratch[w], excl_lane);
  __syncthreads();
  return res;
}

// Tie-group start per sorted position: S[p] = largest q <= p with
// q == 0 || key[q] != key[q-1].  Optionally GE[S[p]] = one past the group end.
template <typename K>
FCB_DEV void tie_groups(const K* keys, int m, uint16_t* S, uint16_t* GE, int* scratch) {
  const int per = (m + blockDim.x - 1) / blockDim.x;
  const int b = threadIdx.x * per, e = min(m, b + per);
  int last = -1;
  for (int p = b; p < e; ++p)
    if (p == 0 || keys[p] != keys[p - 1]) last = p;
  int carry = block_exclusive_max(last, scratch);
  for (int p = b; p < e; ++p) {
    if (p == 0 || keys[p] != keys[p - 1]) carry = p;
    S[p] = static_cast<uint16_t>(carry);
  }
  __syncthreads();
  if (GE != nullptr) {
    for (int p = b; p < e; ++p)
      if (p == m - 1 || keys[p] != keys[p + 1]) GE[S[p]] = static_cast<uint16_t>(p + 1);
    __syncthreads();
  }
}

// Blocked exclusive prefix count of pred(p) over p in [0, m): returns the
// count before this thread's chunk [b, e) and the total.
template <typename Pred>
FCB_DEV uint32_t chunk_prefix(int m, Pred pred, int& b, int& e, uint32_t* scan, uint32_t& total) {
  const int per = (m + blockDim.x - 1) / blockDim.x;
  b = threadIdx.x * per;
  e = min(m, b + per);
  uint32_t c = 0;
  for (int p = b; p < e; ++p) c += pred(p) ? 1u : 0u;
  return block_exclusive_sum(c, scan, total);
}

// The rank + IC epilogue's block results in one reduction round: the sum of
// joint rank products and the first / last joint positions on the returns
// and factor sides (integer sums and extrema: any order gives the same
// result).  scratch: >= 32 * 24 bytes, idle between the two barriers' callers.
struct IcEnds {
  unsigned long long sum;
  int rfirst, rlast, ffirst, flast;
};

FCB_DEV IcEnds block_reduce_ends(IcEnds v, uint8_t* scratch) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v.sum += __shfl_xor_sync(kFull, v.sum, o);
    v.rfirst = min(v.rfirst, __shfl_xor_sync(kFull, v.rfirst, o));
    v.rlast = max(v.rlast, __shfl_xor_sync(kFull, v.rlast, o));
    v.ffirst = min(v.ffirst, __shfl_xor_sync(kFull, v.ffirst, o));
    v.flast = max(v.flast, __shfl_xor_sync(kFull, v.flast, o));
  }
  const int w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  unsigned long long* s64 = reinterpret_cast<unsigned long long*>(scratch);
  int* si = reinterpret_cast<int*>(scratch + 32 * sizeof(unsigned long long));
  if (lane_id() == 0) {
    s64[w] = v.sum;
    si[w] = v.rfirst;
    si[32 + w] = v.rlast;
    si[64 + w] = v.ffirst;
    si[96 + w] = v.flast;
  }
  __syncthreads();
  IcEnds r{0ull, 0x7fffffff, -1, 0x7fffffff, -1};
  for (int i = 0; i < nw; ++i) {
    r.sum += s64[i];
    r.rfirst = min(r.rfirst, si[i]);
    r.rlast = max(r.rlast, si[32 + i]);
    r.ffirst = min(r.ffirst, si[64 + i]);
    r.flast = max(r.flast, si[96 + i]);
  }
  __syncthreads();
  return r;
}

FCB_DEV void store_row_f32(float* __restrict__ dst, const float* __restrict__ src, int n) {
  // dst and src share the same 16-byte phase whenever N % 4 == 0 and the
  // panel is 16-aligned; fall back to scalar stores otherwise.
  const uintptr_t d = reinterpret_cast<uintptr_t>(dst), s = reinterpret_cast<uintptr_t>(src);
  if (((d ^ s) & 15u) == 0) {
    const int head = static_cast<int>(((16 - (d & 15u)) & 15u) / 4);
    const int h = min(head, n);
    for (int i = threadIdx.x; i < h; i += blockDim.x) dst[i] = src[i];
    const int nv = (n - h) / 4;
    const float4* s4 = reinterpret_cast<const float4*>(src + h);
    float4* d4 = reinterpret_cast<float4*>(dst + h);
    for (int i = threadIdx.x; i < nv; i += blockDim.x) d4[i] = s4[i];
    for (int i = h + nv * 4 + threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
  } else {
    for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
  }
}

// ---------------------------------------------------------------------------
// rank + IC over F factor panels sharing one forward-return panel
// ---------------------------------------------------------------------------
struct RankIcLayout {
  size_t bars, scratch, k0, k1, i0, i1, flags, ir, gr, rr, total;
  __host__ __device__ RankIcLayout(int n, int ksz, size_t sort_scratch) {
    size_t o = 0;
    bars = o; o += 64;
    scratch = o; o = align16(o + sort_scratch);
    k0 = o; o = align16(o + size_t(n) * ksz + 16);
    k1 = o; o = align16(o + size_t(n) * ksz + 16);
    i0 = o; o = align16(o + size_t(n) * 2 + 16);
    i1 = o; o = align16(o + size_t(n) * 2 + 16);
    flags = o; o = align16(o + size_t(n) + 16);
    ir = o; o = align16(o + size_t(n) * 2);
    gr = o; o = align16(o + size_t(n) * 2);
    rr = o; o = align16(o + size_t(n) * 2 + 16);
    total = o;
  }
};

// The staging barriers (five) sit at the start of every rank+IC layout.
FCB_DEV void rank_ic_cta_init(uint8_t* sm) {
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm);
  if (threadIdx.x == 0) {
    for (int b = 0; b < 5; ++b) mbar_init(&bars[b], 1);
    fence_mbar_init();
  }
  __syncthreads();
}

// One factor f of date t: stage the factor row, rank it (learned splitters or
// radix), then the IC against the returns whose sorted order (column ids) is
// IR[0, mr).  flags (bits 0-1 set by the caller: returns valid, factor mask)
// gain bit 2 (factor finite).  same_ret_group(p, q), called by every thread
// with block-uniform p <= q, tells whether sorted returns positions p and q
// hold equal keys.  Returns false when a staged copy did not land.
// x_staged (or nullptr): the factor row already staged in the k1 region by
// the caller; table_staged: this factor's CDF table already in the histogram
// region.
template <int NT, int MAXIPT, typename TF, typename TR, bool LEARNED, typename SameGroup>
FCB_DEV bool rank_ic_factor(const RankIcArgs<TF, TR>& a, const int t, const int f, uint8_t* sm, const RankIcLayout& L,
                            uint32_t* ph, int* status, uint8_t* flags, const uint16_t* IR, const int mr,
                            SameGroup same_ret_group, const TF* x_staged = nullptr, bool table_staged = false) {
  using KF = typename KeyOf<TF>::type;
  const int N = a.N, T = a.T;
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm + L.bars);
  uint32_t* scan = reinterpret_cast<uint32_t*>(sm + L.scratch + SortScratch<NT>::hist_bytes +
                                               SortScratch<NT>::base_bytes);
  unsigned long long* scan64 = reinterpret_cast<unsigned long long*>(scan);
  uint16_t* RR = reinterpret_cast<uint16_t*>(sm + L.rr);
  uint16_t* i0 = reinterpret_cast<uint16_t*>(sm + L.i0);
  uint16_t* i1 = reinterpret_cast<uint16_t*>(sm + L.i1);
  bool arm[4] = {false, false, false, false};
  bool ok;
  const size_t frow = (static_cast<size_t>(f) * T + t) * N;
  const TF* x = x_staged;
  if (x == nullptr) {
    x = stage_issue(sm + L.k1, a.X + frow, N, &bars[3], arm[3]);
    ok = stage_wait(&bars[3], ph[3], arm[3]);
    if (__syncthreads_or(!ok)) {
      if (threadIdx.x == 0) atomicExch(status, 1);
      return false;
    }
  }
  for (int i = threadIdx.x; i < N; i += NT)
    flags[i] = static_cast<uint8_t>((flags[i] & 3u) | (KeyOf<TF>::finite(x[i]) ? 4u : 0u));
  __syncthreads();
  KF* kf0 = reinterpret_cast<KF*>(sm + L.k0);
  KF* kf1 = reinterpret_cast<KF*>(sm + L.k1);
  const int mf = compact_keys<KF>(
      N, [&](int i) { return (flags[i] & 6u) == 6u; }, [&](int i) { return KeyOf<TF>::key(x[i]); }, kf0, i0,
      scan);
  KF* kfs = kf0;
  uint16_t* ifs = i0;
  bool sorted = false;
  if (LEARNED && a.cdf_table != nullptr) {
    // the radix histogram region is idle here: it holds this factor's table
    float* tab = reinterpret_cast<float*>(sm + L.scratch);
    static_assert(SortScratch<NT>::hist_bytes >= kCdfKnots * sizeof(float), "table must fit the histogram region");
    if (!table_staged) {
      for (int k = threadIdx.x; k < kCdfKnots; k += NT) tab[k] = a.cdf_table[static_cast<size_t>(f) * kCdfKnots + k];
      __syncthreads();
    }
    int mb = 0, ss = 0;
    const int st = learned_sort<NT, MAXIPT>(reinterpret_cast<uint32_t*>(kf0), i0, reinterpret_cast<uint32_t*>(kf1),
                                            i1, mf, RR, tab, a.cdf_zrange[2 * f], a.cdf_zrange[2 * f + 1],
                                            a.learn_cap, reinterpret_cast<double*>(scan64), scan, &mb, &ss);
    if (a.learn_stats != nullptr && threadIdx.x == 0) {
      int* o = a.learn_stats + (static_cast<size_t>(f) * T + t) * 4;
      o[0] = st;
      o[1] = mb;
      o[2] = ss;
      o[3] = mf;
    }
    sorted = (st == kLearnOk);
    if (st == kLearnJudge) {
      // the buffers were permuted: rebuild the compacted input from the row
      x = stage_issue(sm + L.k1, a.X + frow, N, &bars[3], arm[3]);
      ok = stage_wait(&bars[3], ph[3], arm[3]);
      if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0) atomicExch(status, 1);
        return false;
      }
      (void)compact_keys<KF>(
          N, [&](int i) { return (flags[i] & 6u) == 6u; }, [&](int i) { return KeyOf<TF>::key(x[i]); }, kf0, i0,
          scan);
    }
    __syncthreads();
  }
  if (!sorted) block_radix_sort<NT, MAXIPT, KF>(kf0, i0, kf1, i1, mf, sm + L.scratch, &kfs, &ifs);

  // the idle key buffer receives the cs ranks; cells left out of the factor's
  // valid set keep the quiet NaN (the barriers inside the two prefix counts
  // below order these stores before the rank stores)
  float* rbuf = reinterpret_cast<float*>(kfs == kf0 ? kf1 : kf0);
  const bool want_ranks = a.ranks_out != nullptr;
  if (want_ranks) {
    const float qnan = __uint_as_float(kQuietNanBits);
    for (int i = threadIdx.x; i < N; i += NT) rbuf[i] = qnan;
  }
  if (a.rank_f_out != nullptr) {
    for (int i = threadIdx.x; i < N; i += NT) {
      a.rank_f_out[frow + i] = 0.0;
      a.rank_r_out[frow + i] = 0.0;
    }
  }

  // returns side: joint ranks in return order, first/last joint position
  int b, e;
  uint32_t mj;
  uint32_t c = chunk_prefix(mr, [&](int p) { return flags[IR[p]] == 7u; }, b, e, scan, mj);
  IcEnds ends{0ull, 0x7fffffff, -1, 0x7fffffff, -1};
  for (int p = b; p < e; ++p) {
    const int i = IR[p];
    if (flags[i] == 7u) {
      RR[i] = static_cast<uint16_t>(++c);
      ends.rfirst = min(ends.rfirst, p);
      ends.rlast = max(ends.rlast, p);
    }
  }

  // factor side: cs ranks, joint ranks, sum of rank products (the prefix
  // count's barriers also publish RR)
  uint32_t mj2;
  uint32_t cf = chunk_prefix(mf, [&](int p) { return flags[ifs[p]] == 7u; }, b, e, scan, mj2);
  long long sum = 0;
  for (int p = b; p < e; ++p) {
    const int i = ifs[p];
    if (want_ranks) rbuf[i] = static_cast<float>(p + 1);
    if (flags[i] == 7u) {
      ++cf;
      sum += static_cast<long long>(cf) * RR[i];
      ends.ffirst = min(ends.ffirst, p);
      ends.flast = max(ends.flast, p);
      if (a.rank_f_out != nullptr) {
        a.rank_f_out[frow + i] = static_cast<double>(cf);
        a.rank_r_out[frow + i] = static_cast<double>(RR[i]);
      }
    }
  }
  ends.sum = static_cast<unsigned long long>(sum);
  // the sort scratch is idle here (the learned table too)
  ends = block_reduce_ends(ends, sm + L.scratch);
  const int ffirst = ends.ffirst, flast = ends.flast;
  // block-collective: do the joint returns at rfirst and rlast share a key?
  const bool rconst = same_ret_group(ends.rfirst, ends.rlast);
  if (threadIdx.x == 0) {
    double ic = __longlong_as_double(0x7ff8000000000000ll);
    const long long m = static_cast<long long>(mj);
    if (m >= a.min_valid && m >= 2) {
      const bool fconst = kfs[ffirst] == kfs[flast];
      if (!fconst && !rconst) ic = spearman_from_sum(m, static_cast<long long>(ends.sum));
    }
    a.ic_out[static_cast<size_t>(f) * (a.ic_ld > 0 ? a.ic_ld : T) + t] = ic;
  }
  __syncthreads();
  if (want_ranks) store_row_f32(a.ranks_out + frow, rbuf, N);
  __syncthreads();
  return true;
}

// One date t of one panel: sort the returns, then rank every factor and
// evaluate its IC.  `ph` carries the staging barriers' phase bits from one
// call to the next (persistent CTAs process many dates).  Returns false when a
// staged copy did not land (status set); all threads return together.
template <int NT, int MAXIPT, typename TF, typename TR, bool LEARNED>
FCB_DEV bool rank_ic_date(const RankIcArgs<TF, TR>& a, const int t, uint8_t* sm, uint32_t* ph, int* status) {
  using KF = typename KeyOf<TF>::type;
  using KR = typename KeyOf<TR>::type;
  constexpr int KSZ = (sizeof(KF) > sizeof(KR)) ? int(sizeof(KF)) : int(sizeof(KR));
  const int N = a.N, T = a.T;
  const RankIcLayout L(N, KSZ, SortScratch<NT>::bytes);
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm + L.bars);
  uint32_t* scan = reinterpret_cast<uint32_t*>(sm + L.scratch + SortScratch<NT>::hist_bytes +
                                               SortScratch<NT>::base_bytes);
  unsigned long long* scan64 = reinterpret_cast<unsigned long long*>(scan);
  const size_t row = static_cast<size_t>(t) * N;
  uint8_t* flags = sm + L.flags;
  uint16_t* IR = reinterpret_cast<uint16_t*>(sm + L.ir);
  uint16_t* GR = reinterpret_cast<uint16_t*>(sm + L.gr);
  uint16_t* RR = reinterpret_cast<uint16_t*>(sm + L.rr);
  uint16_t* i0 = reinterpret_cast<uint16_t*>(sm + L.i0);
  uint16_t* i1 = reinterpret_cast<uint16_t*>(sm + L.i1);

  bool arm[4] = {false, false, false, false};

  // ---- stage forward returns and both masks; flags bit0 = return valid, bit1 = factor mask
  const TR* r = stage_issue(sm + L.k1, a.R + row, N, &bars[0], arm[0]);
  const uint8_t* rm = nullptr;
  const uint8_t* fm = nullptr;
  if (a.rmask != nullptr) rm = stage_issue(sm + L.i1, a.rmask + row, N, &bars[1], arm[1]);
  if (a.fmask != nullptr) fm = stage_issue(sm + L.i0, a.fmask + row, N, &bars[2], arm[2]);
  bool ok = stage_wait(&bars[0], ph[0], arm[0]);
  ok = stage_wait(&bars[1], ph[1], arm[1]) && ok;
  ok = stage_wait(&bars[2], ph[2], arm[2]) && ok;
  if (__syncthreads_or(!ok)) {
    if (threadIdx.x == 0) atomicExch(status, 1);
    return false;
  }
  for (int i = threadIdx.x; i < N; i += NT) {
    const bool rv = KeyOf<TR>::finite(r[i]) && (rm == nullptr || rm[i] != 0);
    const bool fv = (fm == nullptr) || fm[i] != 0;
    flags[i] = static_cast<uint8_t>((rv ? 1u : 0u) | (fv ? 2u : 0u));
  }
  __syncthreads();

  // ---- sort the forward returns once per date
  KR* kr0 = reinterpret_cast<KR*>(sm + L.k0);
  KR* kr1 = reinterpret_cast<KR*>(sm + L.k1);
  const int mr = compact_keys<KR>(
      N, [&](int i) { return (flags[i] & 1u) != 0; }, [&](int i) { return KeyOf<TR>::key(r[i]); }, kr0, i0,
      scan);
  KR* krs;
  uint16_t* irs;
  block_radix_sort<NT, MAXIPT, KR>(kr0, i0, kr1, i1, mr, sm + L.scratch, &krs, &irs);
  for (int p = threadIdx.x; p < mr; p += NT) IR[p] = irs[p];
  tie_groups(krs, mr, GR, static_cast<uint16_t*>(nullptr), reinterpret_cast<int*>(scan));

  // ---- per factor
  for (int f = 0; f < a.F; ++f) {
    if (!rank_ic_factor<NT, MAXIPT, TF, TR, LEARNED>(a, t, f, sm, L, ph, status, flags, IR, mr,
                                                     [&](int p, int q) { return q <= p || GR[p] == GR[q]; }))
      return false;
  }
  return true;
}

template <int NT, int MAXIPT, typename TF, typename TR, bool LEARNED>
__global__ void __launch_bounds__(NT, (NT >= 1024 ? 1 : 1024 / NT)) k_rank_ic(RankIcArgs<TF, TR> a, int* status) {
  extern __shared__ __align__(16) uint8_t sm[];
  rank_ic_cta_init(sm);
  uint32_t ph[4] = {0, 0, 0, 0};
  (void)rank_ic_date<NT, MAXIPT, TF, TR, LEARNED>(a, blockIdx.x, sm, ph, status);
}

// Persistent rank+IC over many panels: each CTA takes (panel, date) items
// from a device queue until it is empty.  items[k] = (panel index, date); the
// panels' N must all fit this block size (N <= NT * MAXIPT) and the dynamic
// shared memory was sized for the largest of them.
template <int NT, int MAXIPT, typename TF, typename TR, bool LEARNED>
__global__ void __launch_bounds__(NT, (NT >= 1024 ? 1 : 1024 / NT))
    k_rank_ic_batch(const RankIcArgs<TF, TR>* __restrict__ panels, const int2* __restrict__ items, int nitems,
                    int* __restrict__ counter, int* __restrict__ status) {
  extern __shared__ __align__(16) uint8_t sm[];
  __shared__ int s_item;
  rank_ic_cta_init(sm);
  uint32_t ph[4] = {0, 0, 0, 0};
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
    __syncthreads();
    const int it = s_item;
    __syncthreads();
    if (it >= nitems) break;
    const int2 w = items[it];
    const RankIcArgs<TF, TR> a = panels[w.x];
    if (!rank_ic_date<NT, MAXIPT, TF, TR, LEARNED>(a, w.y, sm, ph, status)) break;
  }
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
template <int NT>
constexpr int cap_of() { return NT * 16; }

static int pick_nt(int n) { return n <= 4096 ? 256 : (n <= 8192 ? 512 : 1024); }

template <typename TF, typename TR>
size_t rank_ic_smem(int N) {
  constexpr int KSZ = (sizeof(TF) > sizeof(TR)) ? int(sizeof(TF)) : int(sizeof(TR));
  return RankIcLayout(N, KSZ, SortScratch<1024>::bytes).total;
}
template size_t rank_ic_smem<float, float>(int);
template size_t rank_ic_smem<float, double>(int);
template size_t rank_ic_smem<double, float>(int);
template size_t rank_ic_smem<double, double>(int);

template <int NT, typename TF, typename TR, bool LEARNED>
static cudaError_t launch_rank_ic_nt(const RankIcArgs<TF, TR>& a, int* status, cudaStream_t st) {
  constexpr int KSZ = (sizeof(TF) > sizeof(TR)) ? int(sizeof(TF)) : int(sizeof(TR));
  const size_t smem = RankIcLayout(a.N, KSZ, SortScratch<NT>::bytes).total;
  if (smem > kMaxSmemPerBlock) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(k_rank_ic<NT, 16, TF, TR, LEARNED>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  k_rank_ic<NT, 16, TF, TR, LEARNED><<<a.T, NT, smem, st>>>(a, status);
  return cudaGetLastError();
}

template <typename TF, typename TR>
cudaError_t launch_rank_ic(const RankIcArgs<TF, TR>& a, int* status, cudaStream_t st) {
  if (a.N > kSmemRankCap) return cudaErrorInvalidValue;
  switch (pick_nt(a.N)) {
    case 256: return launch_rank_ic_nt<256, TF, TR, false>(a, status, st);
    case 512: return launch_rank_ic_nt<512, TF, TR, false>(a, status, st);
    default: return launch_rank_ic_nt<1024, TF, TR, false>(a, status, st);
  }
}

cudaError_t launch_rank_ic_learned(const RankIcArgs<float, float>& a, int* status, cudaStream_t st) {
  if (a.N > kSmemRankCap || a.cdf_table == nullptr || a.cdf_zrange == nullptr) return cudaErrorInvalidValue;
  switch (pick_nt(a.N)) {
    case 256: return launch_rank_ic_nt<256, float, float, true>(a, status, st);
    case 512: return launch_rank_ic_nt<512, float, float, true>(a, status, st);
    default: return launch_rank_ic_nt<1024, float, float, true>(a, status, st);
  }
}
template cudaError_t launch_rank_ic<float, float>(const RankIcArgs<float, float>&, int*, cudaStream_t);
template cudaError_t launch_rank_ic<float, double>(const RankIcArgs<float, double>&, int*, cudaStream_t);
template cudaError_t launch_rank_ic<double, float>(const RankIcArgs<double, float>&, int*, cudaStream_t);
template cudaError_t launch_rank_ic<double, double>(const RankIcArgs<double, double>&, int*, cudaStream_t);

// ---------------------------------------------------------------------------
// persistent batch launchers
// ---------------------------------------------------------------------------
template <typename TF, typename TR>
size_t rank_ic_batch_smem(int nt, int maxN) {
  constexpr int KSZ = (sizeof(TF) > sizeof(TR)) ? int(sizeof(TF)) : int(sizeof(TR));
  switch (nt) {
    case 256: return RankIcLayout(maxN, KSZ, SortScratch<256>::bytes).total;
    case 512: return RankIcLayout(maxN, KSZ, SortScratch<512>::bytes).total;
    default: return RankIcLayout(maxN, KSZ, SortScratch<1024>::bytes).total;
  }
}

template <int NT, typename TF, typename TR, bool LEARNED>
static cudaError_t batch_nt(const RankIcArgs<TF, TR>* panels, const int2* items, int nitems, int* counter,
                            int grid, size_t smem, int* status, cudaStream_t st, int* occ) {
  auto* k = k_rank_ic_batch<NT, 16, TF, TR, LEARNED>;
  if (smem > kMaxSmemPerBlock) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  if (occ != nullptr) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, k, NT, smem);
  k<<<grid, NT, smem, st>>>(panels, items, nitems, counter, status);
  return cudaGetLastError();
}

template <typename TF, typename TR>
cudaError_t launch_rank_ic_batch(int nt, bool learned, const RankIcArgs<TF, TR>* panels, const int2* items,
                                 int nitems, int* counter, int grid, size_t smem, int* status, cudaStream_t st,
                                 int* occ) {
  if (learned) {
    if constexpr (std::is_same<TF, float>::value && std::is_same<TR, float>::value) {
      switch (nt) {
        case 256: return batch_nt<256, TF, TR, true>(panels, items, nitems, counter, grid, smem, status, st, occ);
        case 512: return batch_nt<512, TF, TR, true>(panels, items, nitems, counter, grid, smem, status, st, occ);
        default: return batch_nt<1024, TF, TR, true>(panels, items, nitems, counter, grid, smem, status, st, occ);
      }
    } else {
      return cudaErrorInvalidValue;
    }
  }
  switch (nt) {
    case 256: return batch_nt<256, TF, TR, false>(panels, items, nitems, counter, grid, smem, status, st, occ);
    case 512: return batch_nt<512, TF, TR, false>(panels, items, nitems, counter, grid, smem, status, st, occ);
    default: return batch_nt<1024, TF, TR, false>(panels, items, nitems, counter, grid, smem, status, st, occ);
  }
}
template size_t rank_ic_batch_smem<float, float>(int, int);
template size_t rank_ic_batch_smem<double, double>(int, int);
template cudaError_t launch_rank_ic_batch<float, float>(int, bool, const RankIcArgs<float, float>*, const int2*, int,
                                                         int*, int, size_t, int*, cudaStream_t, int*);
template cudaError_t launch_rank_ic_batch<double, double>(int, bool, const RankIcArgs<double, double>*, const int2*,
                                                           int, int*, int, size_t, int*, cudaStream_t, int*);

}  // namespace fcb
