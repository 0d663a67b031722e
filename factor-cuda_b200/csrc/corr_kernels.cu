// corr_kernels.cu -- FP64 pairwise-complete Pearson correlations (drop-in path).
//
// stock_corr (N,N) over t and factor_corr (F,F) over pooled (t,i) rows, with
// the reference's numeric contract (|dr| <= 1e-12 against np.corrcoef on the
// joint subset, serial-Kahan semantics on reduction-sensitive inputs):
//
//  1. column statistics: count, serial-Kahan mean in row order, min/max,
//     |x| extrema for the domain check (stock_corr_gpu's col_stats_kernel,
//     src/stock_corr.cu:73-116, with the demean_kernel's serial Kahan mean,
//     :244-261);
//  2. a Gram pass on column-centred values: n, sum x', sum y', sum x'y',
//     sum x'^2, sum y'^2 over each pair's joint valid set (the six masked
//     products of _masked_gemm_stats, fc/_cpu_core.py:139-169), accumulated
//     hierarchically (per 32-wide k tile, then into the running total);
//  3. finalize: the cancellation gate of _gemm_cancel_mask (ratio 3 on the
//     uncentred sums, reconstructed from the centred ones), |r|>1, the
//     near-zero-variance gate of finalize_cell (src/stock_corr_impl.cuh:102-132);
//     flagged pairs are recomputed by
//  4. the two-pass fallback on the original values: Kahan mean in row order,
//     exact-constant (min==max) gate, centred second pass (Kahan above T=2048),
//     sequential (sxy/sqrt(sxx))/sqrt(syy) (two_pass_centered,
//     src/stock_corr_impl.cuh:150-201; _two_pass_corr, fc/_cpu_core.py:111-137).
// The diagonal is 1.0 iff the column has n>=2, is not constant and its centred
// sum of squares is positive and finite; the lower triangle mirrors the upper
// bitwise.
#include <cmath>

#include <algorithm>

#include "fcb_common.cuh"
#include "fcb_kernels.h"

namespace fcb {

constexpr double kBigPos = 1e300;
constexpr double kCancelRatio = 3.0;
constexpr double kConstVarRel = 1e-10;
constexpr double kTiny = 1e-300;
constexpr int kTwoPassKahanT = 2048;

struct Kahan {
  double s = 0.0, c = 0.0;
  FCB_DEV void add(double x) {
    const double y = x - c;
    const double t = s + y;
    c = (t - s) - y;
    s = t;
  }
  FCB_DEV void merge(const Kahan& o) {
    add(o.s);
    add(-o.c);
  }
};

FCB_DEV double dnan() { return __longlong_as_double(0x7ff8000000000000ll); }

FCB_DEV double safe_pearson(double sxy, double sxx, double syy) {
  if (!(sxx > 0.0 && syy > 0.0) || !isfinite(sxx) || !isfinite(syy) || !isfinite(sxy)) return dnan();
  const double r = (sxy / sqrt(sxx)) / sqrt(syy);
  return isfinite(r) ? r : dnan();
}

// Decide from the centred moment sums of one pair whether the Gram value is
// trustworthy; returns NaN + flag when the pair must go to the fallback.
FCB_DEV double finalize_pair(double n, double sx, double sy, double sxy, double sx2, double sy2, double mux,
                             double muy, bool& flag) {
  flag = false;
  if (n < 2.0) return dnan();
  const double cov = sxy - sx * sy / n;
  const double vx = sx2 - sx * sx / n;
  const double vy = sy2 - sy * sy / n;
  // uncentred sums of the reference's one-pass Gram, reconstructed
  const double sxr = sx + n * mux;
  const double syr = sy + n * muy;
  const double sx2r = sx2 + 2.0 * mux * sx + n * mux * mux;
  const double sy2r = sy2 + 2.0 * muy * sy + n * muy * muy;
  bool fix = (fabs(sxr * syr / n) > kCancelRatio * fabs(cov)) ||
             (fabs(sxr * sxr / n) > kCancelRatio * fabs(vx)) ||
             (fabs(syr * syr / n) > kCancelRatio * fabs(vy));
  const double xmag = fmax(fabs(sx2r), fabs(sxr * sxr / n));
  const double ymag = fmax(fabs(sy2r), fabs(syr * syr / n));
  if (fabs(vx) <= kConstVarRel * (xmag + kTiny) || fabs(vy) <= kConstVarRel * (ymag + kTiny)) fix = true;
  const double r = safe_pearson(cov, vx, vy);
  if (!isfinite(r) || fabs(r) > 1.0) fix = true;
  flag = fix;
  return fix ? dnan() : r;
}

// ---------------------------------------------------------------------------
// stock_corr
// ---------------------------------------------------------------------------

// (T,N) row-major -> column-major Xraw/Xc/Mc (N, Tp), zero padded, tiled.
template <typename TIN>
__global__ void k_sc_transpose(const TIN* __restrict__ X, const uint8_t* __restrict__ mask, int T, int N, int Tp,
                               double* __restrict__ Xraw, double* __restrict__ Mc) {
  __shared__ double tx[32][33];
  __shared__ double tm[32][33];
  const int t0 = blockIdx.x * 32, i0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int t = t0 + r, i = i0 + threadIdx.x;
    double v = 0.0, m = 0.0;
    if (t < T && i < N) {
      const size_t e = static_cast<size_t>(t) * N + i;
      const double x = static_cast<double>(X[e]);
      const bool ok = finite_f64(x) && (mask == nullptr || mask[e] != 0);
      v = ok ? x : 0.0;
      m = ok ? 1.0 : 0.0;
    }
    tx[r][threadIdx.x] = v;
    tm[r][threadIdx.x] = m;
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int i = i0 + r, t = t0 + threadIdx.x;
    if (i < N && t < Tp) {
      Xraw[static_cast<size_t>(i) * Tp + t] = tx[threadIdx.x][r];
      Mc[static_cast<size_t>(i) * Tp + t] = tm[threadIdx.x][r];
    }
  }
}

// One warp per column: serial Kahan mean in row order, extrema, centred
// copy Xc = valid ? x - mu : 0, centred sum of squares for the diagonal.
__global__ void k_sc_colstats(const double* __restrict__ Xraw, const double* __restrict__ Mc, int T, int N, int Tp,
                              double* __restrict__ Xc, ColStat* __restrict__ st) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= N) return;
  const double* x = Xraw + static_cast<size_t>(w) * Tp;
  const double* m = Mc + static_cast<size_t>(w) * Tp;
  Kahan k;
  double cnt = 0.0, mn = kBigPos, mx = -kBigPos, mna = kBigPos, mxa = 0.0;
  for (int t0 = 0; t0 < T; t0 += 32) {
    const int t = t0 + lane;
    const double xv = (t < T) ? x[t] : 0.0;
    const bool ok = (t < T) && m[t] != 0.0;
    const unsigned vb = __ballot_sync(kFull, ok);
    // serial Kahan in row order: lane 0 consumes the 32 values in order
    for (int l = 0; l < 32; ++l) {
      const double v = __shfl_sync(kFull, xv, l);
      if ((vb >> l) & 1u) k.add(v);
    }
    if (ok) {
      cnt += 1.0;
      mn = fmin(mn, xv);
      mx = fmax(mx, xv);
      const double ax = fabs(xv);
      mxa = fmax(mxa, ax);
      if (ax != 0.0) mna = fmin(mna, ax);
    }
  }
  cnt = warp_sum(cnt);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mn = fmin(mn, __shfl_xor_sync(kFull, mn, o));
    mx = fmax(mx, __shfl_xor_sync(kFull, mx, o));
    mna = fmin(mna, __shfl_xor_sync(kFull, mna, o));
    mxa = fmax(mxa, __shfl_xor_sync(kFull, mxa, o));
  }
  const double mu = cnt > 0.0 ? k.s / cnt : 0.0;
  double s2 = 0.0, s1 = 0.0;
  for (int t = lane; t < Tp; t += 32) {
    const bool ok = (t < T) && m[t] != 0.0;
    const double d = ok ? x[t] - mu : 0.0;
    Xc[static_cast<size_t>(w) * Tp + t] = d;
    s2 += d * d;
    s1 += d;
  }
  s2 = warp_sum(s2);
  s1 = warp_sum(s1);
  if (lane == 0) {
    ColStat c;
    c.count = cnt;
    c.mean = mu;
    c.min = mn;
    c.max = mx;
    c.min_abs = mna;
    c.max_abs = mxa;
    c.s2 = s2;
    c.s1 = s1;
    st[w] = c;
  }
}

// Domain check + full-validity over the column stats (single block).
__global__ void k_sc_summary(const ColStat* __restrict__ st, int N, int T, double* __restrict__ out3) {
  double mxa = 0.0, mna = kBigPos;
  int full = 1;
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    mxa = fmax(mxa, st[i].max_abs);
    mna = fmin(mna, st[i].min_abs);
    if (st[i].count < static_cast<double>(T)) full = 0;
  }
  __shared__ double smx[32], smn[32];
  __shared__ int sf[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mxa = fmax(mxa, __shfl_xor_sync(kFull, mxa, o));
    mna = fmin(mna, __shfl_xor_sync(kFull, mna, o));
    full = min(full, __shfl_xor_sync(kFull, full, o));
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    smx[w] = mxa;
    smn[w] = mna;
    sf[w] = full;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 1; i < (blockDim.x + 31) / 32; ++i) {
      mxa = fmax(mxa, smx[i]);
      mna = fmin(mna, smn[i]);
      full = min(full, sf[i]);
    }
    out3[0] = mxa;
    out3[1] = mna;
    out3[2] = full;
  }
}

// Upper-triangle 32x32 tiles; 256 threads, 2x2 cells per thread; six
// accumulators per cell; 32-wide k tiles staged in shared memory.
constexpr int kScTile = 32, kScK = 32;

FCB_DEV void tri_tile(int b, int nt, int& ib, int& jb) {
  int lo = 0, hi = nt - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    const long long pm = static_cast<long long>(mid) * nt - static_cast<long long>(mid) * (mid - 1) / 2;
    if (pm <= b) lo = mid; else hi = mid - 1;
  }
  ib = lo;
  const long long p = static_cast<long long>(ib) * nt - static_cast<long long>(ib) * (ib - 1) / 2;
  jb = ib + static_cast<int>(b - p);
}

__global__ void __launch_bounds__(256, 2)
    k_sc_gram(const double* __restrict__ Xc, const double* __restrict__ Mc, const ColStat* __restrict__ st, int N,
              int Tp, int nt, double* __restrict__ out, int* __restrict__ fb_list, int* __restrict__ fb_count,
              int full) {
  __shared__ double Ax[kScTile][kScK + 1], Am[kScTile][kScK + 1], Bx[kScTile][kScK + 1], Bm[kScTile][kScK + 1];
  int ib, jb;
  tri_tile(blockIdx.x, nt, ib, jb);
  const int i0 = ib * kScTile, j0 = jb * kScTile;
  const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
  double acc[4][6], part[4][6];
#pragma unroll
  for (int c = 0; c < 4; ++c)
#pragma unroll
    for (int q = 0; q < 6; ++q) acc[c][q] = 0.0;
  for (int k0 = 0; k0 < Tp; k0 += kScK) {
    for (int e = threadIdx.x; e < kScTile * kScK; e += 256) {
      const int r = e / kScK, kk = e % kScK;
      const int gi = i0 + r, gj = j0 + r;
      Ax[r][kk] = gi < N ? Xc[static_cast<size_t>(gi) * Tp + k0 + kk] : 0.0;
      Am[r][kk] = gi < N ? Mc[static_cast<size_t>(gi) * Tp + k0 + kk] : 0.0;
      Bx[r][kk] = gj < N ? Xc[static_cast<size_t>(gj) * Tp + k0 + kk] : 0.0;
      Bm[r][kk] = gj < N ? Mc[static_cast<size_t>(gj) * Tp + k0 + kk] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
      for (int q = 0; q < 6; ++q) part[c][q] = 0.0;
#pragma unroll 4
    for (int kk = 0; kk < kScK; ++kk) {
      const double ax0 = Ax[ty * 2][kk], ax1 = Ax[ty * 2 + 1][kk];
      const double am0 = Am[ty * 2][kk], am1 = Am[ty * 2 + 1][kk];
      const double bx0 = Bx[tx * 2][kk], bx1 = Bx[tx * 2 + 1][kk];
      const double bm0 = Bm[tx * 2][kk], bm1 = Bm[tx * 2 + 1][kk];
      const double axs[2] = {ax0, ax1}, ams[2] = {am0, am1}, bxs[2] = {bx0, bx1}, bms[2] = {bm0, bm1};
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) {
          const int c = a * 2 + b;
          const double jx = axs[a] * bms[b];
          const double jy = ams[a] * bxs[b];
          part[c][0] = fma(ams[a], bms[b], part[c][0]);
          part[c][1] += jx;
          part[c][2] += jy;
          part[c][3] = fma(axs[a], bxs[b], part[c][3]);
          part[c][4] = fma(axs[a], jx, part[c][4]);
          part[c][5] = fma(bxs[b], jy, part[c][5]);
        }
    }
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
      for (int q = 0; q < 6; ++q) acc[c][q] += part[c][q];
    __syncthreads();
  }
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      const int i = i0 + ty * 2 + a, j = j0 + tx * 2 + b;
      if (i >= N || j >= N || i > j) continue;
      const double* q = acc[a * 2 + b];
      double r;
      bool flag = false;
      if (i == j) {
        // diagonal: 1.0 iff the column's centred sum of squares is usable
        const ColStat& s = st[i];
        r = (s.count >= 2.0 && s.min != s.max && s.s2 > 0.0 && isfinite(s.s2)) ? 1.0 : dnan();
      } else {
        r = finalize_pair(q[0], q[1], q[2], q[3], q[4], q[5], st[i].mean, st[j].mean, flag);
        if (!flag && q[0] >= 2.0) {
          // an exact-constant column on the joint set has zero centred
          // variance; the gate above catches it, min==max settles it
        }
      }
      out[static_cast<size_t>(i) * N + j] = r;
      out[static_cast<size_t>(j) * N + i] = r;
      if (flag) {
        const int slot = atomicAdd(fb_count, 1);
        fb_list[slot] = i * N + j;  // N*N <= INT32_MAX
      }
    }
  (void)full;
}

// Two-pass Pearson of one pair over its joint valid dates, serial in date
// order (the Kahan-mean two-pass reference's exact sequence of operations).
// One thread per pair: the dates are read kU at a time, all loads issued
// before they are used, so each step does not wait on its own loads; the
// values are then consumed in date order.
template <int kU>
FCB_DEV double two_pass_serial(const double* __restrict__ xi, const double* __restrict__ mi,
                               const double* __restrict__ xj, const double* __restrict__ mj, int T) {
  double n = 0.0, mnx = kBigPos, mxx = -kBigPos, mny = kBigPos, mxy = -kBigPos;
  Kahan kx, ky;
  for (int t0 = 0; t0 < T; t0 += kU) {
    double a[kU], b[kU], x[kU], y[kU];
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      const int t = t0 + u;
      const bool in = t < T;
      a[u] = in ? mi[t] : 0.0;
      b[u] = in ? mj[t] : 0.0;
      x[u] = in ? xi[t] : 0.0;
      y[u] = in ? xj[t] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      if (a[u] != 0.0 && b[u] != 0.0) {
        n += 1.0;
        kx.add(x[u]);
        ky.add(y[u]);
        mnx = fmin(mnx, x[u]);
        mxx = fmax(mxx, x[u]);
        mny = fmin(mny, y[u]);
        mxy = fmax(mxy, y[u]);
      }
    }
  }
  if (n < 2.0) return dnan();
  if (mnx == mxx || mny == mxy) return dnan();
  const double mx = kx.s / n, my = ky.s / n;
  const bool kahan = T > kTwoPassKahanT;
  Kahan ka, kb, kc;
  double sxx = 0.0, syy = 0.0, sxy = 0.0;
  for (int t0 = 0; t0 < T; t0 += kU) {
    double a[kU], b[kU], x[kU], y[kU];
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      const int t = t0 + u;
      const bool in = t < T;
      a[u] = in ? mi[t] : 0.0;
      b[u] = in ? mj[t] : 0.0;
      x[u] = in ? xi[t] : 0.0;
      y[u] = in ? xj[t] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      if (a[u] != 0.0 && b[u] != 0.0) {
        const double dx = x[u] - mx, dy = y[u] - my;
        if (kahan) {
          ka.add(dx * dx);
          kb.add(dy * dy);
          kc.add(dx * dy);
        } else {
          sxx += dx * dx;
          syy += dy * dy;
          sxy += dx * dy;
        }
      }
    }
  }
  if (kahan) {
    sxx = ka.s - ka.c;
    syy = kb.s - kb.c;
    sxy = kc.s - kc.c;
  }
  return safe_pearson(sxy, sxx, syy);
}

__global__ void k_sc_fallback(const double* __restrict__ Xraw, const double* __restrict__ Mc, int T, int N, int Tp,
                              const int* __restrict__ fb_list, const int* __restrict__ fb_count,
                              double* __restrict__ out) {
  const int cnt = *fb_count;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < cnt; k += gridDim.x * blockDim.x) {
    const int cell = fb_list[k];
    const int i = cell / N, j = cell % N;
    const double r = two_pass_serial<8>(Xraw + static_cast<size_t>(i) * Tp, Mc + static_cast<size_t>(i) * Tp,
                                        Xraw + static_cast<size_t>(j) * Tp, Mc + static_cast<size_t>(j) * Tp, T);
    out[static_cast<size_t>(i) * N + j] = r;
    out[static_cast<size_t>(j) * N + i] = r;
  }
}

cudaError_t launch_stock_corr_prep(const void* X, int dtype, const uint8_t* mask, int T, int N, int Tp,
                                   double* Xraw, double* Xc, double* Mc, ColStat* st, double* summary,
                                   cudaStream_t s) {
  dim3 grid((Tp + 31) / 32, (N + 31) / 32), block(32, 8);
  if (dtype == 0)
    k_sc_transpose<float><<<grid, block, 0, s>>>(static_cast<const float*>(X), mask, T, N, Tp, Xraw, Mc);
  else
    k_sc_transpose<double><<<grid, block, 0, s>>>(static_cast<const double*>(X), mask, T, N, Tp, Xraw, Mc);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_sc_colstats<<<(N * 32 + 255) / 256, 256, 0, s>>>(Xraw, Mc, T, N, Tp, Xc, st);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_sc_summary<<<1, 1024, 0, s>>>(st, N, T, summary);
  return cudaGetLastError();
}

cudaError_t launch_stock_corr_gram(const double* Xraw, const double* Xc, const double* Mc, const ColStat* st, int T,
                                   int N, int Tp, double* out, int* fb_list, int* fb_count, cudaStream_t s) {
  const int nt = (N + kScTile - 1) / kScTile;
  const long long tiles = static_cast<long long>(nt) * (nt + 1) / 2;
  k_sc_gram<<<static_cast<unsigned>(tiles), 256, 0, s>>>(Xc, Mc, st, N, Tp, nt, out, fb_list, fb_count, 0);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  // grid-stride over the device-side fallback count (no host round trip)
  k_sc_fallback<<<148 * 4, 128, 0, s>>>(Xraw, Mc, T, N, Tp, fb_list, fb_count, out);
  return cudaGetLastError();
}

// Correlation domain extremes over the valid cells of a factor_corr panel.
// Non-negative doubles order like their bit patterns, so the block results
// merge with 64-bit integer atomics.
__global__ void k_corr_domain_init(unsigned long long* ext) {
  ext[0] = 0ull;                   // +0.0
  ext[1] = 0x7ff0000000000000ull;  // +inf
}

template <typename TIN>
__global__ void __launch_bounds__(256) k_corr_domain(const TIN* __restrict__ X, const uint8_t* __restrict__ mask,
                                                     long long R, int F, int planes,
                                                     unsigned long long* __restrict__ ext) {
  const long long n = R * F;
  double mx = 0.0, mn = __longlong_as_double(0x7ff0000000000000ll);
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < n;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const double v = static_cast<double>(X[e]);
    const long long r = planes ? e % R : e / F;
    if (finite_f64(v) && (mask == nullptr || mask[r] != 0)) {
      const double a = fabs(v);
      mx = fmax(mx, a);
      if (a != 0.0) mn = fmin(mn, a);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mx = fmax(mx, __shfl_xor_sync(kFull, mx, o));
    mn = fmin(mn, __shfl_xor_sync(kFull, mn, o));
  }
  __shared__ double smx[8], smn[8];
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    smx[w] = mx;
    smn[w] = mn;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 1; i < static_cast<int>(blockDim.x >> 5); ++i) {
      mx = fmax(mx, smx[i]);
      mn = fmin(mn, smn[i]);
    }
    atomicMax(&ext[0], static_cast<unsigned long long>(__double_as_longlong(mx)));
    atomicMin(&ext[1], static_cast<unsigned long long>(__double_as_longlong(mn)));
  }
}

cudaError_t launch_corr_domain(const void* X, int dtype, const uint8_t* mask, long long R, int F, int planes,
                               unsigned long long* ext, cudaStream_t s) {
  k_corr_domain_init<<<1, 1, 0, s>>>(ext);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const long long n = R * F;
  const int grid = static_cast<int>(std::max<long long>(1, std::min<long long>(148 * 8, (n + 2047) / 2048)));
  if (dtype == 0)
    k_corr_domain<float><<<grid, 256, 0, s>>>(static_cast<const float*>(X), mask, R, F, planes, ext);
  else
    k_corr_domain<double><<<grid, 256, 0, s>>>(static_cast<const double*>(X), mask, R, F, planes, ext);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// factor_corr: rows r = t*N+i, F <= 128 columns; element (r, f) at
// X[r*sr + f*sf] -- (sr, sf) = (F, 1) for a (T,N,F) panel (the reference's
// layout), (1, T*N) for F stacked (T,N) factor planes.
// ---------------------------------------------------------------------------

// Block coordinates of a factor_corr body: the CUDA block of a single-panel
// launch, or a panel's own block inside a batched launch (see the batched
// kernels below).
struct Blk {
  int x, y, gx;
};
FCB_DEV Blk launch_blk() {
  return Blk{static_cast<int>(blockIdx.x), static_cast<int>(blockIdx.y), static_cast<int>(gridDim.x)};
}

// Per-block column partials over a contiguous row range: count, Kahan sum,
// min, max.  Rows are visited in increasing order within each thread's
// strided slice; partials are merged in a fixed order by k_fc_colfinal.
template <typename TIN, bool UNIT_ROWS>
FCB_DEV void fc_colpart_body(const TIN* __restrict__ X, const uint8_t* __restrict__ mask, long long R, int F,
                             long long sr, long long sf, long long rows_per_block, FcColPart* __restrict__ part,
                             const Blk bk) {
  const long long r0 = bk.x * rows_per_block;
  const long long r1 = min(R, r0 + rows_per_block);
  for (int f = threadIdx.y; f < F; f += blockDim.y) {
    Kahan k;
    // count, min and max in the input's own type (exact: the values are the
    // same after the widening); only the Kahan sum needs FP64
    long long cnt_i = 0;
    TIN mn_t = KeyOf<TIN>::max_finite(), mx_t = -KeyOf<TIN>::max_finite();
    const TIN* col = X + f * sf;
    // rows visited in the same order; kU loads in flight before they are added
    constexpr int kU = 8;
    for (long long rb = r0 + threadIdx.x; rb < r1; rb += static_cast<long long>(kU) * blockDim.x) {
      TIN xv[kU];
      bool ok[kU];
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        const long long r = rb + static_cast<long long>(u) * blockDim.x;
        ok[u] = r < r1;
        xv[u] = ok[u] ? col[UNIT_ROWS ? r : r * sr] : TIN(0);
        ok[u] = ok[u] && (mask == nullptr || mask[r] != 0);
      }
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        if (ok[u] && KeyOf<TIN>::finite(xv[u])) {
          ++cnt_i;
          k.add(static_cast<double>(xv[u]));
          mn_t = xv[u] < mn_t ? xv[u] : mn_t;
          mx_t = xv[u] > mx_t ? xv[u] : mx_t;
        }
      }
    }
    double cnt = static_cast<double>(cnt_i);
    double mn = cnt_i > 0 ? static_cast<double>(mn_t) : kBigPos;
    double mx = cnt_i > 0 ? static_cast<double>(mx_t) : -kBigPos;
    // fixed-order warp merge (lanes are threadIdx.x within one warp row)
    for (int o = 1; o < 32; o <<= 1) {
      const double os = __shfl_down_sync(kFull, k.s, o), oc = __shfl_down_sync(kFull, k.c, o);
      const double on = __shfl_down_sync(kFull, cnt, o);
      const double omn = __shfl_down_sync(kFull, mn, o), omx = __shfl_down_sync(kFull, mx, o);
      if ((threadIdx.x & (2 * o - 1)) == 0) {
        Kahan kk;
        kk.s = os;
        kk.c = oc;
        k.merge(kk);
        cnt += on;
        mn = fmin(mn, omn);
        mx = fmax(mx, omx);
      }
    }
    if (threadIdx.x == 0) {
      FcColPart p;
      p.count = cnt;
      p.s = k.s;
      p.c = k.c;
      p.min = mn;
      p.max = mx;
      part[static_cast<size_t>(bk.x) * F + f] = p;
    }
  }
}

template <typename TIN, bool UNIT_ROWS>
__global__ void k_fc_colpart(const TIN* __restrict__ X, const uint8_t* __restrict__ mask, long long R, int F,
                             long long sr, long long sf, long long rows_per_block, FcColPart* __restrict__ part) {
  fc_colpart_body<TIN, UNIT_ROWS>(X, mask, R, F, sr, sf, rows_per_block, part, launch_blk());
}

// One warp per column: lane l merges partials l, l+32, ... in order, then a
// fixed shuffle tree merges the lanes.
FCB_DEV void fc_colfinal_body(const FcColPart* __restrict__ part, int nblk, int F, FcColStat* __restrict__ st,
                              const Blk bk) {
  const int f = (bk.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (f >= F) return;  // whole warps exit together
  Kahan k;
  double cnt = 0.0, mn = kBigPos, mx = -kBigPos;
  for (int b = lane; b < nblk; b += 32) {
    const FcColPart& p = part[static_cast<size_t>(b) * F + f];
    Kahan o;
    o.s = p.s;
    o.c = p.c;
    k.merge(o);
    cnt += p.count;
    mn = fmin(mn, p.min);
    mx = fmax(mx, p.max);
  }
  for (int o = 1; o < 32; o <<= 1) {
    const double os = __shfl_down_sync(kFull, k.s, o), oc = __shfl_down_sync(kFull, k.c, o);
    const double on = __shfl_down_sync(kFull, cnt, o);
    const double omn = __shfl_down_sync(kFull, mn, o), omx = __shfl_down_sync(kFull, mx, o);
    if ((lane & (2 * o - 1)) == 0) {
      Kahan kk;
      kk.s = os;
      kk.c = oc;
      k.merge(kk);
      cnt += on;
      mn = fmin(mn, omn);
      mx = fmax(mx, omx);
    }
  }
  if (lane != 0) return;
  FcColStat s;
  s.count = cnt;
  s.mean = cnt > 0.0 ? k.s / cnt : 0.0;
  s.min = mn;
  s.max = mx;
  st[f] = s;
}

__global__ void k_fc_colfinal(const FcColPart* __restrict__ part, int nblk, int F, FcColStat* __restrict__ st) {
  fc_colfinal_body(part, nblk, F, st, launch_blk());
}

// Gram partials over a row range.  Products p: 0 n=(m,m), 1 sx=(x',m),
// 2 sx2=(x'^2,m), 3 sxy=(x',x').  Each thread owns a 4x4 (f,g) tile of one
// product and a slice of the staged rows; slices are summed in shared memory
// in a fixed order at the end of the block.
// Rows staged per step: 16 for F > 64, 32 for F in (32, 64], more for
// narrower panels (fewer barriers per row); with the raw-copy double buffer
// the block stays under 75 KB of shared memory for every F <= 128 and both
// input widths, so three blocks fit an SM.
__host__ __device__ inline int fc_rows_chunk(int Fp) {
  return Fp > 64 ? 16 : 32 * (64 / Fp > 8 ? 8 : (64 / Fp < 1 ? 1 : 64 / Fp));
}
// Staged tile layout: column f of the centred values at sx[f * pitch + row],
// the validity tile at the same offsets from sm.  pitch = chunk + 1 is odd, so
// column f starts on bank pair 2f (mod 32) and consecutive rows of a column
// are consecutive words; sm starts 2 doubles past a 16-double boundary (bank
// offset 4), so the columns {c, c+4, c+8} of both tiles that one load of a
// warp touches, on one row or on two adjacent rows, fall in distinct banks.
__host__ __device__ inline int fc_stage_pitch(int Fp) { return fc_rows_chunk(Fp) + 1; }
// Tasks (4x4 tiles) of the Gram pass: the symmetric products n and sxy need
// only the tiles on or above the diagonal (k_fc_final reads (i, j) with
// i <= j), sx and sx2 need all tb x tb tiles (read as (i, j) and (j, i)).
// Order: n upper tiles, sx, sx2, sxy upper tiles.
__host__ __device__ inline int fc_gram_tasks(int tb) { return tb * (tb + 1) + 2 * tb * tb; }
FCB_DEV void fc_gram_task(int tk, int tb, int& p, int& fa, int& ga) {
  const int ntri = tb * (tb + 1) / 2, nsq = tb * tb;
  int k;
  if (tk < ntri) {
    p = 0;
    k = tk;
  } else if (tk < ntri + 2 * nsq) {
    p = tk < ntri + nsq ? 1 : 2;
    const int rem = tk - ntri - (p - 1) * nsq;
    fa = (rem / tb) * 4;
    ga = (rem % tb) * 4;
    return;
  } else {
    p = 3;
    k = tk - ntri - 2 * nsq;
  }
  int a = 0;
  while (k >= tb - a) {  // row a of the upper triangle holds tiles (a, a .. tb-1)
    k -= tb - a;
    ++a;
  }
  fa = a * 4;
  ga = (a + k) * 4;
}
__host__ __device__ inline int fc_stage_sm_offset(int Fp) { return (Fp * fc_stage_pitch(Fp) + 15) / 16 * 16 + 2; }
// Doubles before the raw-copy buffers: the staged tiles, or the slice
// reduction buffer that reuses them after the row loop, whichever is larger.
__host__ __device__ inline size_t fc_gram_raw_offset(int Fp, int tasks_per_block) {
  const size_t stage = static_cast<size_t>(fc_stage_sm_offset(Fp)) + static_cast<size_t>(Fp) * fc_stage_pitch(Fp);
  const size_t red = static_cast<size_t>(256 / tasks_per_block) * tasks_per_block * 16;
  return ((stage > red ? stage : red) + 1) / 2 * 2;  // 16-byte aligned
}

// Gram pass on the FP64 tensor cores (mma.sync m8n8k4 .f64): 8 x 8 output
// tiles of factors, four pooled rows per MMA.  The staged tiles hold Fq =
// Fp rounded up to 8 factor rows (the extra rows stay zero) at a pitch of
// chunk + 4 doubles: a fragment load (factor row lane / 4, pooled row lane % 4)
// then touches 32 distinct banks per half-warp.  A unit of work is one A tile
// (ti) against a group of up to two B tiles (tj); a block's eight warps split
// its units and, when there are fewer than eight, the rows.
constexpr int kFcMmaGroup = 2;
__host__ __device__ inline int fc_mma_fq(int Fp) { return (Fp + 7) / 8 * 8; }
__host__ __device__ inline int fc_mma_pitch(int Fp) { return fc_rows_chunk(Fp) + 4; }
__host__ __device__ inline int fc_mma_units(int Fp) {
  const int nt = fc_mma_fq(Fp) / 8;
  return nt * ((nt + kFcMmaGroup - 1) / kFcMmaGroup);
}
__host__ __device__ inline int fc_mma_units_per_block(int Fp) {
  const int u = fc_mma_units(Fp);
  return u < 8 ? u : 8;
}
// Doubles before the raw-copy buffers: the staged tiles, or the slice
// reduction buffer that reuses them after the row loop, whichever is larger.
__host__ __device__ inline size_t fc_mma_raw_offset(int Fp, int units_per_block) {
  const size_t stage = 2 * static_cast<size_t>(fc_mma_fq(Fp)) * fc_mma_pitch(Fp);
  const size_t red = static_cast<size_t>(units_per_block) * kFcMmaGroup * 4 * 64;
  return ((stage > red ? stage : red) + 1) / 2 * 2;  // 16-byte aligned
}
FCB_DEV void dmma_f64(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

// Asynchronous global -> shared copies of single elements (cp.async, L1
// allocating); each thread waits for its own groups, a barrier publishes them.
template <int BYTES>
FCB_DEV void cp_async_elem(void* smem, const void* gmem) {
  static_assert(BYTES == 4 || BYTES == 8, "element copies are 4 or 8 bytes");
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(smem_u32(smem)), "l"(gmem), "n"(BYTES) : "memory");
}
FCB_DEV void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
FCB_DEV void cp_async_wait_prev() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

template <typename TIN>
FCB_DEV void fc_gram_body_fma(const TIN* __restrict__ X, const uint8_t* __restrict__ mask,
                                                 long long R, int F, long long sr, long long sf, int Fp,
                                                 long long rows_per_block,
                                                 const FcColStat* __restrict__ st, int tasks_total,
                                                 int tasks_per_block, double* __restrict__ part, const Blk bk) {
  extern __shared__ __align__(16) double fsm[];
  const int chunk = fc_rows_chunk(Fp);
  const int pitch = fc_stage_pitch(Fp);
  double* sx = fsm;                                  // [Fp][pitch] centred values
  double* sm = sx + fc_stage_sm_offset(Fp);          // [Fp][pitch] validity
  double* red = fsm;  // [slices][tasks_per_block][16], over the staging tile once it is idle
  const int tb = Fp / 4;
  const int task0 = bk.y * tasks_per_block;
  const int ntask = min(tasks_per_block, tasks_total - task0);
  const int slices = 256 / tasks_per_block;
  const int my_task = threadIdx.x % tasks_per_block;
  const int my_slice = threadIdx.x / tasks_per_block;
  const bool active = (my_slice < slices) && (my_task < ntask);
  int p = 0, fa = 0, ga = 0;
  if (active) fc_gram_task(task0 + my_task, tb, p, fa, ga);
  double acc[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) acc[q] = 0.0;
  const long long r0 = bk.x * rows_per_block;
  const long long r1 = min(R, r0 + rows_per_block);
  // Row chunks are pipelined: while chunk k is centred and multiplied, the raw
  // elements of chunk k + 1 are in flight into the other raw buffer
  // (cp.async) and its mask bytes in a register.
  TIN* raw[2];
  raw[0] = reinterpret_cast<TIN*>(fsm + fc_gram_raw_offset(Fp, tasks_per_block));
  raw[1] = raw[0] + chunk * Fp;
  uint8_t* smask = reinterpret_cast<uint8_t*>(raw[1] + chunk * Fp);
  // Element e of a staged chunk is (row rr, factor f): rr = e / Fp, f = e % Fp
  // for the (rows, F) layout, rr = e % chunk, f = e / chunk for factor planes,
  // so that consecutive threads read consecutive elements of X either way.
  // Each thread walks e = tid, tid + 256, ...: one division up front, then a
  // constant step with a carry.
  const bool planes = sf != 1;
  const int inner = planes ? chunk : Fp;  // extent of the fast index
  const int e0_in = threadIdx.x % inner, e0_out = threadIdx.x / inner;
  const int step_in = 256 % inner, step_out = 256 / inner;
  auto issue = [&](long long cs, TIN* dst) {
    const int nrs = static_cast<int>(min(static_cast<long long>(chunk), r1 - cs));
    const TIN* base = X + cs * sr;
    int a = e0_in, b = e0_out;  // (fast, slow) index of element e
    for (int e = threadIdx.x; e < chunk * Fp; e += 256) {
      const int rr = planes ? a : b;
      const int f = planes ? b : a;
      if (rr < nrs && f < F) cp_async_elem<sizeof(TIN)>(dst + e, base + rr * sr + f * sf);
      a += step_in;
      b += step_out;
      if (a >= inner) {
        a -= inner;
        ++b;
      }
    }
  };
  auto mask_of = [&](long long cs) -> uint8_t {
    const long long r = cs + threadIdx.x;
    return (mask == nullptr || threadIdx.x >= chunk || r >= r1) ? uint8_t(1) : mask[r];
  };
  uint8_t m_cur = 1;
  if (r0 < r1) {
    issue(r0, raw[0]);
    m_cur = mask_of(r0);
  }
  cp_async_commit();
  int it = 0;
  for (long long c0 = r0; c0 < r1; c0 += chunk, ++it) {
    const int nr = static_cast<int>(min(static_cast<long long>(chunk), r1 - c0));
    uint8_t m_next = 1;
    if (c0 + chunk < r1) {
      issue(c0 + chunk, raw[(it + 1) & 1]);
      m_next = mask_of(c0 + chunk);
    }
    cp_async_commit();
    if (threadIdx.x < chunk) smask[threadIdx.x] = m_cur;
    cp_async_wait_prev();  // this thread's copies of chunk `it` have landed
    __syncthreads();
    const TIN* rb = raw[it & 1];
    int a = e0_in, b = e0_out;
    for (int e = threadIdx.x; e < chunk * Fp; e += 256) {
      const int rr = planes ? a : b;
      const int f = planes ? b : a;
      a += step_in;
      b += step_out;
      if (a >= inner) {
        a -= inner;
        ++b;
      }
      const int ei = f * pitch + rr;
      double v = 0.0, mv = 0.0;
      if (rr < nr && f < F) {
        const double x = static_cast<double>(rb[e]);
        if (finite_f64(x) && smask[rr] != 0) {
          v = x - st[f].mean;
          mv = 1.0;
        }
      }
      sx[ei] = v;
      sm[ei] = mv;
    }
    __syncthreads();
    if (active) {
      const double* A = (p == 0) ? sm : sx;  // product 2 squares the centred values below
      const double* B = (p == 3) ? sx : sm;
      for (int rr = my_slice; rr < nr; rr += slices) {
        const double* ar = A + fa * pitch + rr;
        const double* br = B + ga * pitch + rr;
        double a0 = ar[0], a1 = ar[pitch], a2 = ar[2 * pitch], a3 = ar[3 * pitch];
        if (p == 2) {
          a0 *= a0;
          a1 *= a1;
          a2 *= a2;
          a3 *= a3;
        }
        const double b0 = br[0], b1 = br[pitch], b2 = br[2 * pitch], b3 = br[3 * pitch];
        const double av[4] = {a0, a1, a2, a3}, bv[4] = {b0, b1, b2, b3};
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int v = 0; v < 4; ++v) acc[u * 4 + v] = fma(av[u], bv[v], acc[u * 4 + v]);
      }
    }
    __syncthreads();
    m_cur = m_next;
  }
  // reduce slices in fixed order
  if (active) {
    double* dst = red + (static_cast<size_t>(my_slice) * tasks_per_block + my_task) * 16;
#pragma unroll
    for (int q = 0; q < 16; ++q) dst[q] = acc[q];
  }
  __syncthreads();
  for (int e = threadIdx.x; e < ntask * 16; e += 256) {
    const int tk = e / 16, q = e % 16;
    double s = 0.0;
    for (int sl = 0; sl < slices; ++sl) s += red[(static_cast<size_t>(sl) * tasks_per_block + tk) * 16 + q];
    int pp = 0, f0 = 0, g0 = 0;
    fc_gram_task(task0 + tk, tb, pp, f0, g0);
    const int f = f0 + q / 4, g = g0 + q % 4;
    part[((static_cast<size_t>(bk.x) * 4 + pp) * Fp + f) * Fp + g] = s;
  }
}

template <typename TIN>
FCB_DEV void fc_gram_body_mma(const TIN* __restrict__ X, const uint8_t* __restrict__ mask,
                                                 long long R, int F, long long sr, long long sf, int Fp,
                                                 long long rows_per_block,
                                                 const FcColStat* __restrict__ st, int tasks_total,
                                                 int tasks_per_block, double* __restrict__ part, const Blk bk) {
  extern __shared__ __align__(16) double fsm[];
  const int chunk = fc_rows_chunk(Fp);
  const int pitch = fc_mma_pitch(Fp);
  const int Fq = fc_mma_fq(Fp);
  double* sx = fsm;                                  // [Fq][pitch] centred values
  double* sm = sx + static_cast<size_t>(Fq) * pitch; // [Fq][pitch] validity
  double* red = fsm;  // [unit][tj][product][64], over the staging tiles once they are idle
  const int nt = Fq / 8, ng = (nt + kFcMmaGroup - 1) / kFcMmaGroup;
  const int unit0 = bk.y * tasks_per_block;
  const int nunit = min(tasks_per_block, tasks_total - unit0);
  const int warp = static_cast<int>(threadIdx.x >> 5), lane = static_cast<int>(threadIdx.x & 31);
  const int slices = 8 / nunit;
  const int my_unit = warp % nunit, my_slice = warp / nunit;
  const bool active = my_slice < slices;
  const int ti = (unit0 + my_unit) / ng, tj0 = ((unit0 + my_unit) % ng) * kFcMmaGroup;
  const int ntj = min(kFcMmaGroup, nt - tj0);
  double acc[kFcMmaGroup][4][2];  // [tj][product: n, sx, sx2, sxy][lane's two D values]
#pragma unroll
  for (int j = 0; j < kFcMmaGroup; ++j)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[j][q][0] = acc[j][q][1] = 0.0;
  // the factor rows past Fp stay zero for the whole pass
  for (int e = threadIdx.x; e < (Fq - Fp) * pitch; e += 256) {
    sx[static_cast<size_t>(Fp) * pitch + e] = 0.0;
    sm[static_cast<size_t>(Fp) * pitch + e] = 0.0;
  }
  const long long r0 = bk.x * rows_per_block;
  const long long r1 = min(R, r0 + rows_per_block);
  // Row chunks are pipelined: while chunk k is centred and multiplied, the raw
  // elements of chunk k + 1 are in flight into the other raw buffer
  // (cp.async) and its mask bytes in a register.
  TIN* raw[2];
  raw[0] = reinterpret_cast<TIN*>(fsm + fc_mma_raw_offset(Fp, tasks_per_block));
  raw[1] = raw[0] + chunk * Fp;
  uint8_t* smask = reinterpret_cast<uint8_t*>(raw[1] + chunk * Fp);
  // Element e of a staged chunk is (row rr, factor f): rr = e / Fp, f = e % Fp
  // for the (rows, F) layout, rr = e % chunk, f = e / chunk for factor planes,
  // so that consecutive threads read consecutive elements of X either way.
  // Each thread walks e = tid, tid + 256, ...: one division up front, then a
  // constant step with a carry.
  const bool planes = sf != 1;
  const int inner = planes ? chunk : Fp;  // extent of the fast index
  const int e0_in = threadIdx.x % inner, e0_out = threadIdx.x / inner;
  const int step_in = 256 % inner, step_out = 256 / inner;
  auto issue = [&](long long cs, TIN* dst) {
    const int nrs = static_cast<int>(min(static_cast<long long>(chunk), r1 - cs));
    const TIN* base = X + cs * sr;
    int a = e0_in, b = e0_out;  // (fast, slow) index of element e
    for (int e = threadIdx.x; e < chunk * Fp; e += 256) {
      const int rr = planes ? a : b;
      const int f = planes ? b : a;
      if (rr < nrs && f < F) cp_async_elem<sizeof(TIN)>(dst + e, base + rr * sr + f * sf);
      a += step_in;
      b += step_out;
      if (a >= inner) {
        a -= inner;
        ++b;
      }
    }
  };
  auto mask_of = [&](long long cs) -> uint8_t {
    const long long r = cs + threadIdx.x;
    return (mask == nullptr || threadIdx.x >= chunk || r >= r1) ? uint8_t(1) : mask[r];
  };
  uint8_t m_cur = 1;
  if (r0 < r1) {
    issue(r0, raw[0]);
    m_cur = mask_of(r0);
  }
  cp_async_commit();
  int it = 0;
  for (long long c0 = r0; c0 < r1; c0 += chunk, ++it) {
    const int nr = static_cast<int>(min(static_cast<long long>(chunk), r1 - c0));
    uint8_t m_next = 1;
    if (c0 + chunk < r1) {
      issue(c0 + chunk, raw[(it + 1) & 1]);
      m_next = mask_of(c0 + chunk);
    }
    cp_async_commit();
    if (threadIdx.x < chunk) smask[threadIdx.x] = m_cur;
    cp_async_wait_prev();  // this thread's copies of chunk `it` have landed
    __syncthreads();
    const TIN* rb = raw[it & 1];
    int a = e0_in, b = e0_out;
    for (int e = threadIdx.x; e < chunk * Fp; e += 256) {
      const int rr = planes ? a : b;
      const int f = planes ? b : a;
      a += step_in;
      b += step_out;
      if (a >= inner) {
        a -= inner;
        ++b;
      }
      const int ei = f * pitch + rr;
      double v = 0.0, mv = 0.0;
      if (rr < nr && f < F) {
        const double x = static_cast<double>(rb[e]);
        if (finite_f64(x) && smask[rr] != 0) {
          v = x - st[f].mean;
          mv = 1.0;
        }
      }
      sx[ei] = v;
      sm[ei] = mv;
    }
    __syncthreads();
    if (active) {
      // fragments: lane holds factor row lane / 4 of a tile at pooled row
      // r + lane % 4 (A row-major 8 x 4, B column-major 4 x 8: the same address)
      const int fr = lane >> 2, kc = lane & 3;
      const int kend = (nr + 3) & ~3;  // rows past nr are zero
      for (int r = 4 * my_slice; r < kend; r += 4 * slices) {
        const size_t ao = static_cast<size_t>(8 * ti + fr) * pitch + r + kc;
        const double am = sm[ao], ax = sx[ao];
        const double ax2 = ax * ax;
#pragma unroll
        for (int j = 0; j < kFcMmaGroup; ++j) {
          if (j < ntj) {
            const int tj = tj0 + j;
            const size_t bo = static_cast<size_t>(8 * tj + fr) * pitch + r + kc;
            const double bm = sm[bo], bx = sx[bo];
            if (tj >= ti) {  // n and sxy: tiles on or above the diagonal
              dmma_f64(acc[j][0], am, bm);
              dmma_f64(acc[j][3], ax, bx);
            }
            dmma_f64(acc[j][1], ax, bm);
            dmma_f64(acc[j][2], ax2, bm);
          }
        }
      }
    }
    __syncthreads();
    m_cur = m_next;
  }
  // reduce the row slices in slice order (D value e of a lane: tile row
  // lane / 4, column 2 (lane % 4) + e)
  for (int sl = 0; sl < slices; ++sl) {
    if (active && my_slice == sl) {
#pragma unroll
      for (int j = 0; j < kFcMmaGroup; ++j)
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            double* d = red + ((static_cast<size_t>(my_unit) * kFcMmaGroup + j) * 4 + q) * 64 +
                        (lane >> 2) * 8 + 2 * (lane & 3) + e;
            *d = (sl == 0) ? acc[j][q][e] : *d + acc[j][q][e];
          }
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < nunit * kFcMmaGroup * 4 * 64; e += 256) {
    const int idx = e & 63, q = (e >> 6) & 3, j = (e >> 8) % kFcMmaGroup, ul = e / (256 * kFcMmaGroup);
    const int uti = (unit0 + ul) / ng, utj = ((unit0 + ul) % ng) * kFcMmaGroup + j;
    if (utj >= nt || ((q == 0 || q == 3) && utj < uti)) continue;
    const int f = 8 * uti + (idx >> 3), g = 8 * utj + (idx & 7);
    if (f < Fp && g < Fp) part[((static_cast<size_t>(bk.x) * 4 + q) * Fp + f) * Fp + g] = red[e];
  }
}

// The Gram pass takes the FP64 tensor cores when the padded factor count is a
// multiple of 8 (no padded tile rows); otherwise the 4 x 4 FMA tiles, which
// waste less on padding.  tasks_total / tasks_per_block come from
// fc_gram_plan for the same Fp.
__host__ __device__ inline bool fc_gram_use_mma(int Fp) { return Fp % 8 == 0; }
template <typename TIN>
FCB_DEV void fc_gram_body(const TIN* __restrict__ X, const uint8_t* __restrict__ mask, long long R, int F,
                          long long sr, long long sf, int Fp, long long rows_per_block,
                          const FcColStat* __restrict__ st, int tasks_total, int tasks_per_block,
                          double* __restrict__ part, const Blk bk) {
  if (fc_gram_use_mma(Fp))
    fc_gram_body_mma<TIN>(X, mask, R, F, sr, sf, Fp, rows_per_block, st, tasks_total, tasks_per_block, part, bk);
  else
    fc_gram_body_fma<TIN>(X, mask, R, F, sr, sf, Fp, rows_per_block, st, tasks_total, tasks_per_block, part, bk);
}

// Single panel: the path is chosen on the host (MMA = fc_gram_use_mma(Fp)), so
// each instantiation holds one body.
template <typename TIN, bool MMA>
__global__ void __launch_bounds__(256, 3) k_fc_gram(const TIN* __restrict__ X, const uint8_t* __restrict__ mask,
                                                 long long R, int F, long long sr, long long sf, int Fp,
                                                 long long rows_per_block,
                                                 const FcColStat* __restrict__ st, int tasks_total,
                                                 int tasks_per_block, double* __restrict__ part) {
  if (MMA)
    fc_gram_body_mma<TIN>(X, mask, R, F, sr, sf, Fp, rows_per_block, st, tasks_total, tasks_per_block, part,
                          launch_blk());
  else
    fc_gram_body_fma<TIN>(X, mask, R, F, sr, sf, Fp, rows_per_block, st, tasks_total, tasks_per_block, part,
                          launch_blk());
}

// Sum the per-block Gram partials in block order, finalize each pair.
// One warp per (i <= j) pair: lane l sums blocks l, l+32, ..., a fixed
// shuffle tree sums the lanes, lane 0 finalizes.
FCB_DEV void fc_final_body(const double* __restrict__ part, int nblk, int F, int Fp,
                           const FcColStat* __restrict__ st, double* __restrict__ out, int* __restrict__ fb_list,
                           int* __restrict__ fb_count, uint8_t* __restrict__ flags, const Blk bk) {
  const int e = (bk.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (e >= F * F) return;  // whole warps exit together
  const int i = e / F, j = e % F;
  if (i > j) return;
  double q[6] = {0, 0, 0, 0, 0, 0};
  // q: n, sx (x'_i m_j), sy (m_i x'_j), sxy, sx2 (x'^2_i m_j), sy2 (m_i x'^2_j)
  for (int b = lane; b < nblk; b += 32) {
    const double* P = part + static_cast<size_t>(b) * 4 * Fp * Fp;
    q[0] += P[(0 * Fp + i) * Fp + j];
    q[1] += P[(1 * Fp + i) * Fp + j];
    q[2] += P[(1 * Fp + j) * Fp + i];
    q[3] += P[(3 * Fp + i) * Fp + j];
    q[4] += P[(2 * Fp + i) * Fp + j];
    q[5] += P[(2 * Fp + j) * Fp + i];
  }
  for (int o = 1; o < 32; o <<= 1) {
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      const double v = __shfl_down_sync(kFull, q[k], o);
      if ((lane & (2 * o - 1)) == 0) q[k] += v;
    }
  }
  if (lane != 0) return;
  double r;
  bool flag = false;
  if (i == j) {
    const FcColStat& s = st[i];
    const double v = q[4] - q[1] * q[1] / fmax(q[0], 1.0);
    r = (s.count >= 2.0 && s.min != s.max && v > 0.0 && isfinite(v)) ? 1.0 : dnan();
  } else {
    r = finalize_pair(q[0], q[1], q[2], q[3], q[4], q[5], st[i].mean, st[j].mean, flag);
  }
  out[i * F + j] = r;
  out[j * F + i] = r;
  if (flags != nullptr) flags[i * F + j] = flag ? 1 : 0;
  if (flag) {
    const int slot = atomicAdd(fb_count, 1);
    fb_list[slot] = e;
  }
}

__global__ void k_fc_final(const double* __restrict__ part, int nblk, int F, int Fp,
                           const FcColStat* __restrict__ st, double* __restrict__ out, int* __restrict__ fb_list,
                           int* __restrict__ fb_count, uint8_t* __restrict__ flags) {
  fc_final_body(part, nblk, F, Fp, st, out, fb_list, fb_count, flags, launch_blk());
}

// One block per flagged pair: two-pass over the pooled joint rows.  Small
// pools run serially in row order (bit-compatible with the serial-Kahan
// reference); large pools use per-thread Kahan partials merged in a fixed
// tree (the reference's kahan_reduce kernels, src/factor_corr.cu:188-322).
template <typename TIN>
FCB_DEV void fc_fallback_body(const TIN* __restrict__ X, const uint8_t* __restrict__ mask, long long R, int F,
                              long long sr, long long sf, const int* __restrict__ fb_list,
                              const int* __restrict__ fb_count, double* __restrict__ out, const Blk bk) {
  if (static_cast<int>(bk.x) >= *fb_count) return;
  const int e = fb_list[bk.x];
  const int i = e / F, j = e % F;
  __shared__ double sh[6][256];
  __shared__ double res[8];
  const bool serial = R < 4096;
  const int nth = serial ? 1 : blockDim.x;
  const int tid = threadIdx.x;
  if (tid >= nth) {
    // idle threads still take part in the barriers below
  }
  auto valid = [&](long long r, double& x, double& y) {
    x = static_cast<double>(X[r * sr + i * sf]);
    y = static_cast<double>(X[r * sr + j * sf]);
    return finite_f64(x) && finite_f64(y) && (mask == nullptr || mask[r] != 0);
  };
  Kahan kx, ky;
  double n = 0.0, mnx = kBigPos, mxx = -kBigPos, mny = kBigPos, mxy = -kBigPos;
  if (tid < nth) {
    for (long long r = tid; r < R; r += nth) {
      double x, y;
      if (valid(r, x, y)) {
        n += 1.0;
        kx.add(x);
        ky.add(y);
        mnx = fmin(mnx, x);
        mxx = fmax(mxx, x);
        mny = fmin(mny, y);
        mxy = fmax(mxy, y);
      }
    }
  }
  sh[0][tid] = kx.s; sh[1][tid] = kx.c; sh[2][tid] = ky.s; sh[3][tid] = ky.c; sh[4][tid] = n;
  __syncthreads();
  // fixed binary tree merge (thread order)
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (tid < s && tid + s < nth) {
      Kahan a, b, c, d;
      a.s = sh[0][tid]; a.c = sh[1][tid]; b.s = sh[0][tid + s]; b.c = sh[1][tid + s];
      c.s = sh[2][tid]; c.c = sh[3][tid]; d.s = sh[2][tid + s]; d.c = sh[3][tid + s];
      a.merge(b);
      c.merge(d);
      sh[0][tid] = a.s; sh[1][tid] = a.c; sh[2][tid] = c.s; sh[3][tid] = c.c;
      sh[4][tid] += sh[4][tid + s];
    }
    __syncthreads();
  }
  // min / max
  double v0 = mnx, v1 = mxx, v2 = mny, v3 = mxy;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v0 = fmin(v0, __shfl_xor_sync(kFull, v0, o));
    v1 = fmax(v1, __shfl_xor_sync(kFull, v1, o));
    v2 = fmin(v2, __shfl_xor_sync(kFull, v2, o));
    v3 = fmax(v3, __shfl_xor_sync(kFull, v3, o));
  }
  __shared__ double mm[4][8];
  if ((tid & 31) == 0) {
    mm[0][tid >> 5] = v0; mm[1][tid >> 5] = v1; mm[2][tid >> 5] = v2; mm[3][tid >> 5] = v3;
  }
  __syncthreads();
  if (tid == 0) {
    for (int w = 1; w < static_cast<int>(blockDim.x / 32); ++w) {
      v0 = fmin(v0, mm[0][w]); v1 = fmax(v1, mm[1][w]); v2 = fmin(v2, mm[2][w]); v3 = fmax(v3, mm[3][w]);
    }
    const double nn = sh[4][0];
    res[0] = nn;
    res[1] = nn > 0 ? sh[0][0] / nn : 0.0;
    res[2] = nn > 0 ? sh[2][0] / nn : 0.0;
    res[3] = (nn < 2.0 || v0 == v1 || v2 == v3) ? 1.0 : 0.0;
  }
  __syncthreads();
  const double nn = res[0], mx = res[1], my = res[2];
  if (res[3] != 0.0) {
    if (tid == 0) {
      out[i * F + j] = dnan();
      out[j * F + i] = dnan();
    }
    return;
  }
  Kahan a, b, c;
  if (tid < nth) {
    for (long long r = tid; r < R; r += nth) {
      double x, y;
      if (valid(r, x, y)) {
        const double dx = x - mx, dy = y - my;
        if (serial && R <= kTwoPassKahanT) {
          a.s += dx * dx;
          b.s += dy * dy;
          c.s += dx * dy;
        } else {
          a.add(dx * dx);
          b.add(dy * dy);
          c.add(dx * dy);
        }
      }
    }
  }
  sh[0][tid] = a.s; sh[1][tid] = a.c; sh[2][tid] = b.s; sh[3][tid] = b.c; sh[4][tid] = c.s; sh[5][tid] = c.c;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (tid < s && tid + s < nth) {
      for (int q = 0; q < 3; ++q) {
        Kahan u, v;
        u.s = sh[2 * q][tid]; u.c = sh[2 * q + 1][tid]; v.s = sh[2 * q][tid + s]; v.c = sh[2 * q + 1][tid + s];
        u.merge(v);
        sh[2 * q][tid] = u.s;
        sh[2 * q + 1][tid] = u.c;
      }
    }
    __syncthreads();
  }
  if (tid == 0) {
    const double r = safe_pearson(sh[4][0] - sh[5][0], sh[0][0] - sh[1][0], sh[2][0] - sh[3][0]);
    (void)nn;
    out[i * F + j] = r;
    out[j * F + i] = r;
  }
}

template <typename TIN>
__global__ void k_fc_fallback(const TIN* __restrict__ X, const uint8_t* __restrict__ mask, long long R, int F,
                              long long sr, long long sf, const int* __restrict__ fb_list,
                              const int* __restrict__ fb_count, double* __restrict__ out) {
  fc_fallback_body<TIN>(X, mask, R, F, sr, sf, fb_list, fb_count, out, launch_blk());
}

// Multi-block fallback for large pools: the rows are split into `nblk` fixed
// ranges (blockIdx.y); each block forms per-range Kahan partials (threads stride the range,
// a fixed binary tree merges them), a per-pair kernel merges the ranges in
// order.  Two passes as in k_fc_fallback: counts / means / min / max, then the
// centred sums.  Deterministic for a given nblk; agrees with the single-block
// form to rounding (the reference's multi-block kahan_reduce kernels,
// src/factor_corr.cu:188-322, split the rows the same way).
constexpr int kFbThreads = 256;
constexpr int kFbP1 = kFcFbPartDoubles;  // n, sx.s, sx.c, sy.s, sy.c, min x, max x, min y, max y
constexpr int kFbP2 = 6;  // sxx.s, sxx.c, syy.s, syy.c, sxy.s, sxy.c

FCB_DEV void fb_tree_kahan(double (*sh)[kFbThreads], int q0, int nq) {
  const int tid = threadIdx.x;
  for (int st = kFbThreads / 2; st > 0; st >>= 1) {
    if (tid < st) {
      for (int q = q0; q < q0 + nq; ++q) {
        Kahan u, v;
        u.s = sh[2 * q][tid];
        u.c = sh[2 * q + 1][tid];
        v.s = sh[2 * q][tid + st];
        v.c = sh[2 * q + 1][tid + st];
        u.merge(v);
        sh[2 * q][tid] = u.s;
        sh[2 * q + 1][tid] = u.c;
      }
    }
    __syncthreads();
  }
}

template <typename TIN>
FCB_DEV void fc_fb_pass1_body(const TIN* __restrict__ X, const uint8_t* __restrict__ mask,
                                                            long long R, int F, long long sr, long long sf, int nblk,
                                                            const int* __restrict__ fb_list,
                                                            const int* __restrict__ fb_count,
                                                            double* __restrict__ part, const Blk bk) {
  __shared__ double sh[5][kFbThreads];
  __shared__ double mm[4][kFbThreads / 32];
  const long long rpb = (R + nblk - 1) / nblk;
  const long long r0 = bk.y * rpb, r1 = min(R, r0 + rpb);
  const int tid = threadIdx.x;
  for (int slot = bk.x; slot < *fb_count; slot += bk.gx) {
    const int e = fb_list[slot];
    const int i = e / F, j = e % F;
    Kahan kx, ky;
    double n = 0.0, mnx = kBigPos, mxx = -kBigPos, mny = kBigPos, mxy = -kBigPos;
    constexpr int kU = 4;  // rows in flight per thread, added in row order
    for (long long rb = r0 + tid; rb < r1; rb += static_cast<long long>(kU) * kFbThreads) {
      double xv[kU], yv[kU];
      bool ok[kU];
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        const long long r = rb + static_cast<long long>(u) * kFbThreads;
        ok[u] = r < r1;
        xv[u] = ok[u] ? static_cast<double>(X[r * sr + i * sf]) : 0.0;
        yv[u] = ok[u] ? static_cast<double>(X[r * sr + j * sf]) : 0.0;
        ok[u] = ok[u] && (mask == nullptr || mask[r] != 0);
      }
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        if (ok[u] && finite_f64(xv[u]) && finite_f64(yv[u])) {
          n += 1.0;
          kx.add(xv[u]);
          ky.add(yv[u]);
          mnx = fmin(mnx, xv[u]);
          mxx = fmax(mxx, xv[u]);
          mny = fmin(mny, yv[u]);
          mxy = fmax(mxy, yv[u]);
        }
      }
    }
    sh[0][tid] = kx.s;
    sh[1][tid] = kx.c;
    sh[2][tid] = ky.s;
    sh[3][tid] = ky.c;
    sh[4][tid] = n;
    __syncthreads();
    for (int st = kFbThreads / 2; st > 0; st >>= 1) {
      if (tid < st) {
        for (int q = 0; q < 2; ++q) {
          Kahan u, v;
          u.s = sh[2 * q][tid];
          u.c = sh[2 * q + 1][tid];
          v.s = sh[2 * q][tid + st];
          v.c = sh[2 * q + 1][tid + st];
          u.merge(v);
          sh[2 * q][tid] = u.s;
          sh[2 * q + 1][tid] = u.c;
        }
        sh[4][tid] += sh[4][tid + st];
      }
      __syncthreads();
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      mnx = fmin(mnx, __shfl_xor_sync(kFull, mnx, o));
      mxx = fmax(mxx, __shfl_xor_sync(kFull, mxx, o));
      mny = fmin(mny, __shfl_xor_sync(kFull, mny, o));
      mxy = fmax(mxy, __shfl_xor_sync(kFull, mxy, o));
    }
    if ((tid & 31) == 0) {
      mm[0][tid >> 5] = mnx;
      mm[1][tid >> 5] = mxx;
      mm[2][tid >> 5] = mny;
      mm[3][tid >> 5] = mxy;
    }
    __syncthreads();
    if (tid == 0) {
      for (int w = 1; w < kFbThreads / 32; ++w) {
        mnx = fmin(mnx, mm[0][w]);
        mxx = fmax(mxx, mm[1][w]);
        mny = fmin(mny, mm[2][w]);
        mxy = fmax(mxy, mm[3][w]);
      }
      double* P = part + (static_cast<size_t>(slot) * nblk + bk.y) * kFbP1;
      P[0] = sh[4][0];
      P[1] = sh[0][0];
      P[2] = sh[1][0];
      P[3] = sh[2][0];
      P[4] = sh[3][0];
      P[5] = mnx;
      P[6] = mxx;
      P[7] = mny;
      P[8] = mxy;
    }
    __syncthreads();
  }
}

template <typename TIN>
__global__ void __launch_bounds__(kFbThreads) k_fc_fb_pass1(const TIN* __restrict__ X, const uint8_t* __restrict__ mask,
                                                            long long R, int F, long long sr, long long sf, int nblk,
                                                            const int* __restrict__ fb_list,
                                                            const int* __restrict__ fb_count,
                                                            double* __restrict__ part) {
  fc_fb_pass1_body<TIN>(X, mask, R, F, sr, sf, nblk, fb_list, fb_count, part, launch_blk());
}

// Per flagged pair: merge the pass-1 ranges in order -> (n, mean x, mean y,
// degenerate flag) in pair[slot*4 ..]; a degenerate pair is finished here.
// One warp per flagged pair: the lanes load up to 32 range partials at once and
// every lane merges them in range order from shuffled copies (the same
// sequence of operations as a single thread walking the ranges), so the
// merged values do not depend on the warp; lane 0 writes.
FCB_DEV void fc_fb_mid_body(int F, int nblk, const int* __restrict__ fb_list, const int* __restrict__ fb_count,
                            const double* __restrict__ part, double* __restrict__ pair, double* __restrict__ out,
                            const Blk bk) {
  const int slot = (bk.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (slot >= *fb_count) return;  // whole warps exit together
  Kahan kx, ky;
  double n = 0.0, mnx = kBigPos, mxx = -kBigPos, mny = kBigPos, mxy = -kBigPos;
  for (int b0 = 0; b0 < nblk; b0 += 32) {
    double v[kFbP1];
    const int b = b0 + lane;
    const double* P = part + (static_cast<size_t>(slot) * nblk + b) * kFbP1;
#pragma unroll
    for (int q = 0; q < kFbP1; ++q) v[q] = b < nblk ? P[q] : 0.0;
    const int nb = min(32, nblk - b0);
    for (int l = 0; l < nb; ++l) {
      double w[kFbP1];
#pragma unroll
      for (int q = 0; q < kFbP1; ++q) w[q] = __shfl_sync(kFull, v[q], l);
      Kahan o;
      o.s = w[1];
      o.c = w[2];
      kx.merge(o);
      o.s = w[3];
      o.c = w[4];
      ky.merge(o);
      n += w[0];
      mnx = fmin(mnx, w[5]);
      mxx = fmax(mxx, w[6]);
      mny = fmin(mny, w[7]);
      mxy = fmax(mxy, w[8]);
    }
  }
  if (lane != 0) return;
  const bool degenerate = (n < 2.0 || mnx == mxx || mny == mxy);
  double* Q = pair + static_cast<size_t>(slot) * 4;
  Q[0] = n;
  Q[1] = n > 0 ? kx.s / n : 0.0;
  Q[2] = n > 0 ? ky.s / n : 0.0;
  Q[3] = degenerate ? 1.0 : 0.0;
  if (degenerate) {
    const int e = fb_list[slot];
    const int i = e / F, j = e % F;
    out[i * F + j] = dnan();
    out[j * F + i] = dnan();
  }
}

__global__ void k_fc_fb_mid(int F, int nblk, const int* __restrict__ fb_list, const int* __restrict__ fb_count,
                            const double* __restrict__ part, double* __restrict__ pair, double* __restrict__ out) {
  fc_fb_mid_body(F, nblk, fb_list, fb_count, part, pair, out, launch_blk());
}

template <typename TIN>
FCB_DEV void fc_fb_pass2_body(const TIN* __restrict__ X, const uint8_t* __restrict__ mask,
                                                            long long R, int F, long long sr, long long sf, int nblk,
                                                            const int* __restrict__ fb_list,
                                                            const int* __restrict__ fb_count,
                                                            const double* __restrict__ pair,
                                                            double* __restrict__ part, const Blk bk) {
  __shared__ double sh[6][kFbThreads];
  const long long rpb = (R + nblk - 1) / nblk;
  const long long r0 = bk.y * rpb, r1 = min(R, r0 + rpb);
  const int tid = threadIdx.x;
  for (int slot = bk.x; slot < *fb_count; slot += bk.gx) {
    const double* Q = pair + static_cast<size_t>(slot) * 4;
    if (Q[3] != 0.0) continue;  // degenerate: finished by k_fc_fb_mid (uniform per block)
    const int e = fb_list[slot];
    const int i = e / F, j = e % F;
    const double mx = Q[1], my = Q[2];
    Kahan a, b, c;
    constexpr int kU = 4;  // rows in flight per thread, added in row order
    for (long long rb = r0 + tid; rb < r1; rb += static_cast<long long>(kU) * kFbThreads) {
      double xv[kU], yv[kU];
      bool ok[kU];
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        const long long r = rb + static_cast<long long>(u) * kFbThreads;
        ok[u] = r < r1;
        xv[u] = ok[u] ? static_cast<double>(X[r * sr + i * sf]) : 0.0;
        yv[u] = ok[u] ? static_cast<double>(X[r * sr + j * sf]) : 0.0;
        ok[u] = ok[u] && (mask == nullptr || mask[r] != 0);
      }
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        if (ok[u] && finite_f64(xv[u]) && finite_f64(yv[u])) {
          const double dx = xv[u] - mx, dy = yv[u] - my;
          a.add(dx * dx);
          b.add(dy * dy);
          c.add(dx * dy);
        }
      }
    }
    sh[0][tid] = a.s;
    sh[1][tid] = a.c;
    sh[2][tid] = b.s;
    sh[3][tid] = b.c;
    sh[4][tid] = c.s;
    sh[5][tid] = c.c;
    __syncthreads();
    fb_tree_kahan(sh, 0, 3);
    if (tid < kFbP2) part[(static_cast<size_t>(slot) * nblk + bk.y) * kFbP2 + tid] = sh[tid][0];
    __syncthreads();
  }
}

template <typename TIN>
__global__ void __launch_bounds__(kFbThreads) k_fc_fb_pass2(const TIN* __restrict__ X, const uint8_t* __restrict__ mask,
                                                            long long R, int F, long long sr, long long sf, int nblk,
                                                            const int* __restrict__ fb_list,
                                                            const int* __restrict__ fb_count,
                                                            const double* __restrict__ pair,
                                                            double* __restrict__ part) {
  fc_fb_pass2_body<TIN>(X, mask, R, F, sr, sf, nblk, fb_list, fb_count, pair, part, launch_blk());
}

// Pass-2 partials merged per flagged pair, one warp per pair as in k_fc_fb_mid.
FCB_DEV void fc_fb_final_body(int F, int nblk, const int* __restrict__ fb_list, const int* __restrict__ fb_count,
                              const double* __restrict__ pair, const double* __restrict__ part,
                              double* __restrict__ out, const Blk bk) {
  const int slot = (bk.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (slot >= *fb_count) return;  // whole warps exit together
  if (pair[static_cast<size_t>(slot) * 4 + 3] != 0.0) return;
  Kahan a, b, c;
  for (int k0 = 0; k0 < nblk; k0 += 32) {
    double v[kFbP2];
    const int k = k0 + lane;
    const double* P = part + (static_cast<size_t>(slot) * nblk + k) * kFbP2;
#pragma unroll
    for (int q = 0; q < kFbP2; ++q) v[q] = k < nblk ? P[q] : 0.0;
    const int nk = min(32, nblk - k0);
    for (int l = 0; l < nk; ++l) {
      double w[kFbP2];
#pragma unroll
      for (int q = 0; q < kFbP2; ++q) w[q] = __shfl_sync(kFull, v[q], l);
      Kahan o;
      o.s = w[0];
      o.c = w[1];
      a.merge(o);
      o.s = w[2];
      o.c = w[3];
      b.merge(o);
      o.s = w[4];
      o.c = w[5];
      c.merge(o);
    }
  }
  if (lane != 0) return;
  const int e = fb_list[slot];
  const int i = e / F, j = e % F;
  const double r = safe_pearson(c.s - c.c, a.s - a.c, b.s - b.c);
  out[i * F + j] = r;
  out[j * F + i] = r;
}

__global__ void k_fc_fb_final(int F, int nblk, const int* __restrict__ fb_list, const int* __restrict__ fb_count,
                              const double* __restrict__ pair, const double* __restrict__ part,
                              double* __restrict__ out) {
  fc_fb_final_body(F, nblk, fb_list, fb_count, pair, part, out, launch_blk());
}

size_t fc_fb_part_doubles(long long R, int F) {
  const int maxpairs = F * (F - 1) / 2 > 0 ? F * (F - 1) / 2 : 1;
  const int nblk = fc_fb_nblk(R, F);
  return static_cast<size_t>(maxpairs) * nblk * kFbP1 + static_cast<size_t>(maxpairs) * 4;
}

int fc_fb_nblk(long long R, int F) {
  const int maxpairs = F * (F - 1) / 2 > 0 ? F * (F - 1) / 2 : 1;
  long long nb = R / 32768;
  nb = std::min<long long>(nb, kFcFbMaxNblk);
  nb = std::min<long long>(nb, 65536 / maxpairs);
  return static_cast<int>(std::max<long long>(nb, 1));
}

size_t fc_gram_smem(int Fp, int tasks_per_block, int elem_bytes) {
  const size_t raw = 2 * static_cast<size_t>(fc_rows_chunk(Fp)) * Fp * elem_bytes + fc_rows_chunk(Fp);
  const size_t off = fc_gram_use_mma(Fp) ? fc_mma_raw_offset(Fp, tasks_per_block)
                                         : fc_gram_raw_offset(Fp, tasks_per_block);
  return off * sizeof(double) + (raw + 15) / 16 * 16;
}

void fc_gram_plan(int Fp, int* tasks_total, int* tasks_per_block, int* ytiles) {
  if (fc_gram_use_mma(Fp)) {
    *tasks_total = fc_mma_units(Fp);
    *tasks_per_block = fc_mma_units_per_block(Fp);
  } else {
    *tasks_total = fc_gram_tasks(Fp / 4);
    *tasks_per_block = *tasks_total <= 256 ? *tasks_total : 256;
  }
  *ytiles = (*tasks_total + *tasks_per_block - 1) / *tasks_per_block;
}

cudaError_t launch_factor_corr_strided(const void* X, int dtype, const uint8_t* mask, long long R, int F,
                                       long long sr, long long sf, FcWork& w, double* out, uint8_t* flags,
                                       cudaStream_t s) {
  const int Fp = (F + 3) / 4 * 4;
  const int tb = Fp / 4;
  (void)tb;
  int tasks_total = 0, tasks_per_block = 0, ytiles = 0;
  fc_gram_plan(Fp, &tasks_total, &tasks_per_block, &ytiles);
  const long long rpb_cols = (R + w.nblk_cols - 1) / w.nblk_cols;
  const long long rpb_gram = (R + w.nblk_gram - 1) / w.nblk_gram;
  dim3 cb(32, 8);
  // factor planes (rows at unit stride) take the instantiation without the row-stride product
  if (dtype == 0 && sr == 1)
    k_fc_colpart<float, true><<<w.nblk_cols, cb, 0, s>>>(static_cast<const float*>(X), mask, R, F, sr, sf, rpb_cols,
                                                         w.colpart);
  else if (dtype == 0)
    k_fc_colpart<float, false><<<w.nblk_cols, cb, 0, s>>>(static_cast<const float*>(X), mask, R, F, sr, sf,
                                                          rpb_cols, w.colpart);
  else if (sr == 1)
    k_fc_colpart<double, true><<<w.nblk_cols, cb, 0, s>>>(static_cast<const double*>(X), mask, R, F, sr, sf,
                                                          rpb_cols, w.colpart);
  else
    k_fc_colpart<double, false><<<w.nblk_cols, cb, 0, s>>>(static_cast<const double*>(X), mask, R, F, sr, sf,
                                                           rpb_cols, w.colpart);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_fc_colfinal<<<(F * 32 + 127) / 128, 128, 0, s>>>(w.colpart, w.nblk_cols, F, w.colstat);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  const size_t smem = fc_gram_smem(Fp, tasks_per_block, dtype == 0 ? 4 : 8);
  dim3 gg(w.nblk_gram, ytiles);
  auto gram = [&](auto kernel, const auto* x) -> cudaError_t {
    const cudaError_t ge =
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (ge != cudaSuccess) return ge;
    kernel<<<gg, 256, smem, s>>>(x, mask, R, F, sr, sf, Fp, rpb_gram, w.colstat, tasks_total, tasks_per_block, w.gram);
    return cudaSuccess;
  };
  const bool mma = fc_gram_use_mma(Fp);
  if (dtype == 0)
    e = mma ? gram(k_fc_gram<float, true>, static_cast<const float*>(X))
            : gram(k_fc_gram<float, false>, static_cast<const float*>(X));
  else
    e = mma ? gram(k_fc_gram<double, true>, static_cast<const double*>(X))
            : gram(k_fc_gram<double, false>, static_cast<const double*>(X));
  if (e != cudaSuccess) return e;
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(w.fb_count, 0, sizeof(int), s)) != cudaSuccess) return e;
  k_fc_final<<<(F * F * 32 + 255) / 256, 256, 0, s>>>(w.gram, w.nblk_gram, F, Fp, w.colstat, out, w.fb_list,
                                                      w.fb_count, flags);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  const int maxpairs = F * (F - 1) / 2 > 0 ? F * (F - 1) / 2 : 1;
  const int nblk = fc_fb_nblk(R, F);
  if (w.fb_part != nullptr && R >= 4096 && nblk > 1) {
    // large pools, caller-provided partials: rows split over nblk blocks per pair
    double* pair = w.fb_part + static_cast<size_t>(maxpairs) * nblk * kFbP1;
    // pair slots vary fastest, so the blocks of all flagged pairs over one row
    // range run together and share its columns through L2
    const int ysl = std::max(1, std::min(maxpairs, 2048 / nblk));
    dim3 g(ysl, nblk);
    if (dtype == 0)
      k_fc_fb_pass1<float><<<g, kFbThreads, 0, s>>>(static_cast<const float*>(X), mask, R, F, sr, sf, nblk,
                                                     w.fb_list, w.fb_count, w.fb_part);
    else
      k_fc_fb_pass1<double><<<g, kFbThreads, 0, s>>>(static_cast<const double*>(X), mask, R, F, sr, sf, nblk,
                                                      w.fb_list, w.fb_count, w.fb_part);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    k_fc_fb_mid<<<(maxpairs * 32 + 127) / 128, 128, 0, s>>>(F, nblk, w.fb_list, w.fb_count, w.fb_part, pair, out);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (dtype == 0)
      k_fc_fb_pass2<float><<<g, kFbThreads, 0, s>>>(static_cast<const float*>(X), mask, R, F, sr, sf, nblk,
                                                     w.fb_list, w.fb_count, pair, w.fb_part);
    else
      k_fc_fb_pass2<double><<<g, kFbThreads, 0, s>>>(static_cast<const double*>(X), mask, R, F, sr, sf, nblk,
                                                      w.fb_list, w.fb_count, pair, w.fb_part);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    k_fc_fb_final<<<(maxpairs * 32 + 127) / 128, 128, 0, s>>>(F, nblk, w.fb_list, w.fb_count, pair, w.fb_part, out);
    return cudaGetLastError();
  }
  if (dtype == 0)
    k_fc_fallback<float><<<maxpairs, 256, 0, s>>>(static_cast<const float*>(X), mask, R, F, sr, sf, w.fb_list,
                                                  w.fb_count, out);
  else
    k_fc_fallback<double><<<maxpairs, 256, 0, s>>>(static_cast<const double*>(X), mask, R, F, sr, sf, w.fb_list,
                                                   w.fb_count, out);
  return cudaGetLastError();
}

cudaError_t launch_factor_corr(const void* X, int dtype, const uint8_t* mask, long long R, int F, FcWork& w,
                               double* out, uint8_t* flags, cudaStream_t s) {
  return launch_factor_corr_strided(X, dtype, mask, R, F, F, 1, w, out, flags, s);
}

// ---------------------------------------------------------------------------
// batched factor_corr: many factor-plane panels per launch.  Each batched
// kernel's grid is the concatenation of the panels' own grids (prefix offsets
// per kernel kind); a block finds its panel by binary search and runs the
// single-panel body with its block coordinates inside that panel's grid, so
// every panel is computed exactly as by launch_factor_corr_strided.
// ---------------------------------------------------------------------------
namespace {

FCB_DEV int fcb_panel_of(const int* __restrict__ off, int np, int b) {
  int lo = 0, hi = np - 1;  // largest p with off[p] <= b
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= b) lo = mid; else hi = mid - 1;
  }
  return lo;
}

struct FcbAt {
  const FcBatchPanel* q;
  int local;
};
FCB_DEV FcbAt fcb_at(const FcBatchPanel* __restrict__ P, const int* __restrict__ off, int np) {
  const int b = static_cast<int>(blockIdx.x);
  const int p = fcb_panel_of(off, np, b);
  return FcbAt{P + p, b - off[p]};
}

template <typename TIN>
__global__ void k_fcb_colpart(const FcBatchPanel* __restrict__ P, const int* __restrict__ off, int np) {
  const FcbAt a = fcb_at(P, off, np);
  const FcBatchPanel& q = *a.q;
  fc_colpart_body<TIN, true>(static_cast<const TIN*>(q.X), q.mask, q.R, q.F, 1, q.R, q.rpb_cols, q.w.colpart,
                             Blk{a.local, 0, q.w.nblk_cols});
}

__global__ void k_fcb_colfinal(const FcBatchPanel* __restrict__ P, const int* __restrict__ off, int np) {
  const FcbAt a = fcb_at(P, off, np);
  const FcBatchPanel& q = *a.q;
  if (a.local == 0 && threadIdx.x == 0) *q.w.fb_count = 0;  // read by the finalize after the Gram pass
  fc_colfinal_body(q.w.colpart, q.w.nblk_cols, q.F, q.w.colstat, Blk{a.local, 0, 0});
}

template <typename TIN>
__global__ void __launch_bounds__(256, 3) k_fcb_gram(const FcBatchPanel* __restrict__ P, const int* __restrict__ off,
                                                  int np) {
  const FcbAt a = fcb_at(P, off, np);
  const FcBatchPanel& q = *a.q;
  fc_gram_body<TIN>(static_cast<const TIN*>(q.X), q.mask, q.R, q.F, 1, q.R, q.Fp, q.rpb_gram, q.w.colstat,
                    q.tasks_total, q.tasks_per_block, q.w.gram,
                    Blk{a.local % q.w.nblk_gram, a.local / q.w.nblk_gram, q.w.nblk_gram});
}

__global__ void k_fcb_final(const FcBatchPanel* __restrict__ P, const int* __restrict__ off, int np) {
  const FcbAt a = fcb_at(P, off, np);
  const FcBatchPanel& q = *a.q;
  fc_final_body(q.w.gram, q.w.nblk_gram, q.F, q.Fp, q.w.colstat, q.out, q.w.fb_list, q.w.fb_count, nullptr,
                Blk{a.local, 0, 0});
}

template <typename TIN>
__global__ void k_fcb_fallback(const FcBatchPanel* __restrict__ P, const int* __restrict__ off, int np) {
  const FcbAt a = fcb_at(P, off, np);
  const FcBatchPanel& q = *a.q;
  fc_fallback_body<TIN>(static_cast<const TIN*>(q.X), q.mask, q.R, q.F, 1, q.R, q.w.fb_list, q.w.fb_count, q.out,
                        Blk{a.local, 0, 0});
}

FCB_DEV double* fcb_pair(const FcBatchPanel& q) {
  return q.w.fb_part + static_cast<size_t>(q.maxpairs) * q.fb_nblk * kFbP1;
}

template <typename TIN>
__global__ void __launch_bounds__(kFbThreads) k_fcb_fb_pass1(const FcBatchPanel* __restrict__ P,
                                                             const int* __restrict__ off, int np) {
  const FcbAt a = fcb_at(P, off, np);
  const FcBatchPanel& q = *a.q;
  fc_fb_pass1_body<TIN>(static_cast<const TIN*>(q.X), q.mask, q.R, q.F, 1, q.R, q.fb_nblk, q.w.fb_list,
                        q.w.fb_count, q.w.fb_part, Blk{a.local % q.fb_ysl, a.local / q.fb_ysl, q.fb_ysl});
}

__global__ void k_fcb_fb_mid(const FcBatchPanel* __restrict__ P, const int* __restrict__ off, int np) {
  const FcbAt a = fcb_at(P, off, np);
  const FcBatchPanel& q = *a.q;
  fc_fb_mid_body(q.F, q.fb_nblk, q.w.fb_list, q.w.fb_count, q.w.fb_part, fcb_pair(q), q.out, Blk{a.local, 0, 0});
}

template <typename TIN>
__global__ void __launch_bounds__(kFbThreads) k_fcb_fb_pass2(const FcBatchPanel* __restrict__ P,
                                                             const int* __restrict__ off, int np) {
  const FcbAt a = fcb_at(P, off, np);
  const FcBatchPanel& q = *a.q;
  fc_fb_pass2_body<TIN>(static_cast<const TIN*>(q.X), q.mask, q.R, q.F, 1, q.R, q.fb_nblk, q.w.fb_list,
                        q.w.fb_count, fcb_pair(q), q.w.fb_part, Blk{a.local % q.fb_ysl, a.local / q.fb_ysl, q.fb_ysl});
}

__global__ void k_fcb_fb_final(const FcBatchPanel* __restrict__ P, const int* __restrict__ off, int np) {
  const FcbAt a = fcb_at(P, off, np);
  const FcBatchPanel& q = *a.q;
  fc_fb_final_body(q.F, q.fb_nblk, q.w.fb_list, q.w.fb_count, fcb_pair(q), q.w.fb_part, q.out, Blk{a.local, 0, 0});
}

}  // namespace

FcBatchPanel fc_batch_panel(const void* X, const uint8_t* mask, long long R, int F, const FcWork& w, double* out) {
  FcBatchPanel q{};
  q.X = X;
  q.mask = mask;
  q.R = R;
  q.F = F;
  q.Fp = (F + 3) / 4 * 4;
  q.w = w;
  q.out = out;
  const int tb = q.Fp / 4;
  (void)tb;
  fc_gram_plan(q.Fp, &q.tasks_total, &q.tasks_per_block, &q.ytiles);
  q.rpb_cols = (R + w.nblk_cols - 1) / w.nblk_cols;
  q.rpb_gram = (R + w.nblk_gram - 1) / w.nblk_gram;
  q.maxpairs = F * (F - 1) / 2 > 0 ? F * (F - 1) / 2 : 1;
  q.fb_nblk = fc_fb_nblk(R, F);
  // the same choice of fallback as launch_factor_corr_strided
  q.large = (w.fb_part != nullptr && R >= 4096 && q.fb_nblk > 1) ? 1 : 0;
  q.fb_ysl = std::max(1, std::min(q.maxpairs, 2048 / q.fb_nblk));
  return q;
}

void fc_batch_grids(const FcBatchPanel& q, int (&blocks)[kFcbGrids]) {
  blocks[kFcbCols] = q.w.nblk_cols;
  blocks[kFcbColFinal] = (q.F * 32 + 127) / 128;
  blocks[kFcbGram] = q.w.nblk_gram * q.ytiles;
  blocks[kFcbFinal] = (q.F * q.F * 32 + 255) / 256;
  blocks[kFcbFbPass] = q.large ? q.fb_ysl * q.fb_nblk : 0;
  blocks[kFcbFbPair] = q.large ? (q.maxpairs * 32 + 127) / 128 : 0;
  blocks[kFcbSmall] = q.large ? 0 : q.maxpairs;
}

cudaError_t launch_factor_corr_batch(const FcBatchPanel* d_panels, int np, const int* d_off, const int* total,
                                     int dtype, size_t gram_smem, cudaStream_t s) {
  auto off = [&](int g) { return d_off + static_cast<size_t>(g) * (np + 1); };
  cudaError_t e = cudaSuccess;
  auto chk = [&]() { return (e = cudaGetLastError()); };
  const bool f32 = dtype == 0;
  if (total[kFcbCols] > 0) {
    if (f32) k_fcb_colpart<float><<<total[kFcbCols], dim3(32, 8), 0, s>>>(d_panels, off(kFcbCols), np);
    else k_fcb_colpart<double><<<total[kFcbCols], dim3(32, 8), 0, s>>>(d_panels, off(kFcbCols), np);
    if (chk() != cudaSuccess) return e;
  }
  if (total[kFcbColFinal] > 0) {
    k_fcb_colfinal<<<total[kFcbColFinal], 128, 0, s>>>(d_panels, off(kFcbColFinal), np);
    if (chk() != cudaSuccess) return e;
  }
  if (total[kFcbGram] > 0) {
    if (f32) {
      if ((e = cudaFuncSetAttribute(k_fcb_gram<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(gram_smem))) != cudaSuccess)
        return e;
      k_fcb_gram<float><<<total[kFcbGram], 256, gram_smem, s>>>(d_panels, off(kFcbGram), np);
    } else {
      if ((e = cudaFuncSetAttribute(k_fcb_gram<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(gram_smem))) != cudaSuccess)
        return e;
      k_fcb_gram<double><<<total[kFcbGram], 256, gram_smem, s>>>(d_panels, off(kFcbGram), np);
    }
    if (chk() != cudaSuccess) return e;
  }
  if (total[kFcbFinal] > 0) {
    k_fcb_final<<<total[kFcbFinal], 256, 0, s>>>(d_panels, off(kFcbFinal), np);
    if (chk() != cudaSuccess) return e;
  }
  if (total[kFcbSmall] > 0) {
    if (f32) k_fcb_fallback<float><<<total[kFcbSmall], 256, 0, s>>>(d_panels, off(kFcbSmall), np);
    else k_fcb_fallback<double><<<total[kFcbSmall], 256, 0, s>>>(d_panels, off(kFcbSmall), np);
    if (chk() != cudaSuccess) return e;
  }
  if (total[kFcbFbPass] > 0) {
    if (f32) k_fcb_fb_pass1<float><<<total[kFcbFbPass], kFbThreads, 0, s>>>(d_panels, off(kFcbFbPass), np);
    else k_fcb_fb_pass1<double><<<total[kFcbFbPass], kFbThreads, 0, s>>>(d_panels, off(kFcbFbPass), np);
    if (chk() != cudaSuccess) return e;
    k_fcb_fb_mid<<<total[kFcbFbPair], 128, 0, s>>>(d_panels, off(kFcbFbPair), np);
    if (chk() != cudaSuccess) return e;
    if (f32) k_fcb_fb_pass2<float><<<total[kFcbFbPass], kFbThreads, 0, s>>>(d_panels, off(kFcbFbPass), np);
    else k_fcb_fb_pass2<double><<<total[kFcbFbPass], kFbThreads, 0, s>>>(d_panels, off(kFcbFbPass), np);
    if (chk() != cudaSuccess) return e;
    k_fcb_fb_final<<<total[kFcbFbPair], 128, 0, s>>>(d_panels, off(kFcbFbPair), np);
    if (chk() != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace fcb
