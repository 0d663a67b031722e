// cdf_mlp.cu -- per-factor CDF network for learned splitters: features,
// training (hand-written forward/backward + Adam) and tabulation.
//
// Network (one per factor): u(z) = sigmoid(w3 . tanh(W2 tanh(W1 z + b1) + b2) + b3),
// hidden width 32.  z is the cell's value standardised per date by the mean
// and the mean absolute deviation of the date's valid cells; u is trained to
// the empirical quantile (rank - 0.5) / m of the exact ranks the radix path
// produced on earlier dates.  The trained network is tabulated on a uniform
// grid of kCdfKnots z values (cummax-monotone) that the rank kernel turns
// into monotone bucket indices.
#include <cmath>

#include "block_sort.cuh"
#include "fcb_common.cuh"
#include "fcb_kernels.h"

namespace fcb {

constexpr int H = kCdfHidden;  // 32
constexpr int P = kCdfParams;  // 1153
constexpr int BATCH = 256;

// parameter offsets
constexpr int oW1 = 0, oB1 = H, oW2 = 2 * H, oB2 = 2 * H + H * H, oW3 = 3 * H + H * H, oB3 = 4 * H + H * H;
static_assert(oB3 + 1 == P, "parameter layout");

FCB_DEV float sigmoidf_(float o) { return 1.0f / (1.0f + __expf(-o)); }

// ---------------------------------------------------------------------------
// features: per (factor, date) standardise the valid cells and emit S samples
// (z, u) at fixed column positions; invalid positions get u = -1.
// ---------------------------------------------------------------------------
__global__ void k_cdf_features(const float* __restrict__ X, const float* __restrict__ ranks, int T, int N,
                               int t0, int tcount, int S, float2* __restrict__ samples) {
  const int f = blockIdx.y, tl = blockIdx.x;
  const int t = t0 + tl;
  const float* x = X + (static_cast<size_t>(f) * T + t) * N;
  const float* rk = ranks + (static_cast<size_t>(f) * T + t) * N;
  __shared__ double sc[66];
  double s = 0.0, c = 0.0;
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    const float r = rk[i];
    if (r == r) {  // ranked (not NaN)
      s += x[i];
      c += 1.0;
    }
  }
  s = block_sum(s, sc);
  c = block_sum(c, sc);
  const double mean = c > 0 ? s / c : 0.0;
  double a = 0.0;
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    const float r = rk[i];
    if (r == r) a += fabs(x[i] - mean);
  }
  a = block_sum(a, sc);
  const double mad = c > 0 ? a / c : 1.0;
  const float inv = (mad > 0.0 && isfinite(mad)) ? static_cast<float>(1.0 / mad) : 1.0f;
  const float loc = static_cast<float>(mean);
  float2* out = samples + (static_cast<size_t>(f) * tcount + tl) * S;
  const unsigned h = (static_cast<unsigned>(t) * 2654435761u) % static_cast<unsigned>(N);
  for (int j = threadIdx.x; j < S; j += blockDim.x) {
    const int i = static_cast<int>((static_cast<long long>(j) * N / S + h) % N);
    const float r = rk[i];
    float2 v;
    if (r == r && c > 0) {
      v.x = (x[i] - loc) * inv;
      v.y = static_cast<float>((static_cast<double>(r) - 0.5) / c);
    } else {
      v.x = 0.0f;
      v.y = -1.0f;
    }
    out[j] = v;
  }
}

// ---------------------------------------------------------------------------
// one training / gradient step on a minibatch held by the block
// ---------------------------------------------------------------------------
struct TrainSmem {
  float p[P];
  float g[P];
  float h1[BATCH][H + 1];
  float h2[BATCH][H + 1];
  float da2[BATCH][H + 1];
  float gs[BATCH];
  float zs[BATCH];
  float red[64];
};

// Forward + backward of the mean-squared-error loss over the samples held by
// threads (z, u valid iff u >= 0).  Leaves the gradient in S.g and returns
// the summed loss in *loss (thread 0).  All threads must call.
FCB_DEV void cdf_forward_backward(TrainSmem& S, float z, float u, float* loss) {
  const int b = threadIdx.x;
  const bool valid = u >= 0.0f;
  // count valid samples for the mean
  float nv = valid ? 1.0f : 0.0f;
  nv = warp_sum(nv);
  if ((b & 31) == 0) S.red[b >> 5] = nv;
  __syncthreads();
  float nvalid = 0.0f;
  for (int w = 0; w < BATCH / 32; ++w) nvalid += S.red[w];
  __syncthreads();
  float h1[H];
#pragma unroll
  for (int j = 0; j < H; ++j) {
    h1[j] = tanhf(fmaf(S.p[oW1 + j], z, S.p[oB1 + j]));
    S.h1[b][j] = h1[j];
  }
  float o = S.p[oB3];
  float h2[H];
#pragma unroll 4
  for (int i = 0; i < H; ++i) {
    float a = S.p[oB2 + i];
#pragma unroll
    for (int j = 0; j < H; ++j) a = fmaf(S.p[oW2 + i * H + j], h1[j], a);
    h2[i] = tanhf(a);
    S.h2[b][i] = h2[i];
    o = fmaf(S.p[oW3 + i], h2[i], o);
  }
  const float uh = sigmoidf_(o);
  const float diff = valid ? (uh - u) : 0.0f;
  const float g = (nvalid > 0.0f) ? 2.0f * diff * uh * (1.0f - uh) / nvalid : 0.0f;
  S.gs[b] = g;
  S.zs[b] = z;
#pragma unroll
  for (int i = 0; i < H; ++i) S.da2[b][i] = g * S.p[oW3 + i] * (1.0f - h2[i] * h2[i]);
  __syncthreads();
  // dA1 per sample (registers), then overwrite h1 storage after dW2 is formed
  float da1[H];
#pragma unroll
  for (int j = 0; j < H; ++j) {
    float a = 0.0f;
#pragma unroll 8
    for (int i = 0; i < H; ++i) a = fmaf(S.da2[b][i], S.p[oW2 + i * H + j], a);
    da1[j] = a * (1.0f - h1[j] * h1[j]);
  }
  // dW2[i][j] = sum_b da2[b][i] h1[b][j]
  for (int e = b; e < H * H; e += BATCH) {
    const int i = e / H, j = e % H;
    float a = 0.0f;
    for (int s = 0; s < BATCH; ++s) a = fmaf(S.da2[s][i], S.h1[s][j], a);
    S.g[oW2 + e] = a;
  }
  if (b < H) {
    float a = 0.0f, w = 0.0f;
    for (int s = 0; s < BATCH; ++s) {
      a += S.da2[s][b];
      w = fmaf(S.gs[s], S.h2[s][b], w);
    }
    S.g[oB2 + b] = a;
    S.g[oW3 + b] = w;
  } else if (b == H) {
    float a = 0.0f;
    for (int s = 0; s < BATCH; ++s) a += S.gs[s];
    S.g[oB3] = a;
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < H; ++j) S.h1[b][j] = da1[j];
  __syncthreads();
  if (b < H) {
    float a = 0.0f, w = 0.0f;
    for (int s = 0; s < BATCH; ++s) {
      a += S.h1[s][b];
      w = fmaf(S.h1[s][b], S.zs[s], w);
    }
    S.g[oB1 + b] = a;
    S.g[oW1 + b] = w;
  }
  // loss (diagnostic)
  float l = diff * diff;
  l = warp_sum(l);
  if ((b & 31) == 0) S.red[32 + (b >> 5)] = l;
  __syncthreads();
  if (b == 0) {
    float tl = 0.0f;
    for (int w = 0; w < BATCH / 32; ++w) tl += S.red[32 + w];
    *loss = tl;
  }
  __syncthreads();
}

// Gradient only (for checking against the CPU restatement): one block.
__global__ void __launch_bounds__(BATCH) k_cdf_grad(const float* __restrict__ params, const float* __restrict__ z,
                                                    const float* __restrict__ u, int n, float* __restrict__ grad,
                                                    float* __restrict__ loss) {
  extern __shared__ __align__(16) uint8_t smraw[];
  TrainSmem& S = *reinterpret_cast<TrainSmem*>(smraw);
  for (int e = threadIdx.x; e < P; e += BATCH) S.p[e] = params[e];
  __syncthreads();
  const int b = threadIdx.x;
  const float zb = b < n ? z[b] : 0.0f;
  const float ub = b < n ? u[b] : -1.0f;
  float l = 0.0f;
  cdf_forward_backward(S, zb, ub, &l);
  for (int e = threadIdx.x; e < P; e += BATCH) grad[e] = S.g[e];
  if (threadIdx.x == 0) *loss = l;
}

// Training: one block per factor, Adam on minibatches drawn from that
// factor's sample set with a fixed pseudo-random schedule.
__global__ void __launch_bounds__(BATCH) k_cdf_train(float* __restrict__ params, float* __restrict__ adam,
                                                     const float2* __restrict__ samples, int nsamp, int steps,
                                                     float lr, int step0, float* __restrict__ loss_out) {
  extern __shared__ __align__(16) uint8_t smraw[];
  TrainSmem& S = *reinterpret_cast<TrainSmem*>(smraw);
  const int f = blockIdx.x;
  float* pf = params + static_cast<size_t>(f) * P;
  float* mf = adam + static_cast<size_t>(f) * 2 * P;
  float* vf = mf + P;
  const float2* sf = samples + static_cast<size_t>(f) * nsamp;
  for (int e = threadIdx.x; e < P; e += BATCH) S.p[e] = pf[e];
  __syncthreads();
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  float last = 0.0f;
  for (int st = 0; st < steps; ++st) {
    const unsigned long long k =
        (static_cast<unsigned long long>(st + step0) * BATCH + threadIdx.x) * 2654435761ull;
    const float2 smp = sf[k % static_cast<unsigned long long>(nsamp)];
    float l = 0.0f;
    cdf_forward_backward(S, smp.x, smp.y, &l);
    if (threadIdx.x == 0) last = l;
    const int tstep = st + step0 + 1;
    // linear decay to 10% of lr over the steps of this fit
    const float lr_t = lr * (1.0f - 0.9f * static_cast<float>(st) / static_cast<float>(steps > 1 ? steps - 1 : 1));
    const float c1 = 1.0f - powf(b1, static_cast<float>(tstep));
    const float c2 = 1.0f - powf(b2, static_cast<float>(tstep));
    for (int e = threadIdx.x; e < P; e += BATCH) {
      const float g = S.g[e];
      const float m = b1 * mf[e] + (1.0f - b1) * g;
      const float v = b2 * vf[e] + (1.0f - b2) * g * g;
      mf[e] = m;
      vf[e] = v;
      S.p[e] -= lr_t * (m / c1) / (sqrtf(v / c2) + eps);
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < P; e += BATCH) pf[e] = S.p[e];
  if (threadIdx.x == 0 && loss_out != nullptr) loss_out[f] = last;
}

// Grid range of one factor: 0.05% / 99.95% quantiles of (up to 8192) sample
// z values, widened to at least [-4, 4].  One block of 512 threads per
// factor; the quantiles come from the shared-memory radix sort.
__global__ void __launch_bounds__(512) k_cdf_range(const float2* __restrict__ samples, int nsamp,
                                                   float* __restrict__ zrange) {
  extern __shared__ __align__(16) uint8_t sm[];
  constexpr int CAP = 8192;
  const int f = blockIdx.x;
  const float2* sf = samples + static_cast<size_t>(f) * nsamp;
  uint32_t* k0 = reinterpret_cast<uint32_t*>(sm);
  uint32_t* k1 = k0 + CAP;
  uint16_t* i0 = reinterpret_cast<uint16_t*>(k1 + CAP);
  uint16_t* i1 = i0 + CAP;
  uint8_t* scratch = reinterpret_cast<uint8_t*>(i1 + CAP);
  const int stride = nsamp > CAP ? (nsamp + CAP - 1) / CAP : 1;
  uint32_t* scan = reinterpret_cast<uint32_t*>(scratch + SortScratch<512>::hist_bytes + SortScratch<512>::base_bytes);
  const int m = compact_keys<uint32_t>(
      min(nsamp, CAP),
      [&](int j) {
        const long long s = static_cast<long long>(j) * stride;
        return s < nsamp && sf[s].y >= 0.0f && finite_f32(sf[s].x);
      },
      [&](int j) { return key_f32(sf[static_cast<long long>(j) * stride].x); }, k0, i0, scan);
  uint32_t* ks;
  uint16_t* is;
  block_radix_sort<512, 16, uint32_t>(k0, i0, k1, i1, m, scratch, &ks, &is);
  if (threadIdx.x == 0) {
    float lo = -4.0f, hi = 4.0f;
    if (m > 0) {
      const int ql = static_cast<int>(0.0005 * (m - 1)), qh = static_cast<int>(0.9995 * (m - 1));
      const float zl = sf[static_cast<long long>(is[ql]) * stride].x;
      const float zh = sf[static_cast<long long>(is[qh]) * stride].x;
      lo = fminf(lo, fmaxf(zl, -64.0f));
      hi = fmaxf(hi, fminf(zh, 64.0f));
    }
    zrange[2 * f] = lo;
    zrange[2 * f + 1] = hi;
  }
}

// Tabulate u(z) on kCdfKnots uniform knots over [lo, hi]; cummax makes it
// monotone, and a small linear share (kCdfLinearShare of the buckets spread
// uniformly over the knots) keeps a floor of buckets in every knot interval:
// where the network's sigmoid saturates in a heavy tail (u within 1e-3 of 0 or
// 1 over a wide z range) the tail cells would otherwise crowd into one bucket.
// One block per factor.
__global__ void __launch_bounds__(256) k_cdf_tabulate(const float* __restrict__ params, const float* __restrict__ zrange,
                                                      float* __restrict__ table) {
  const int f = blockIdx.x;
  __shared__ float p[P];
  __shared__ float u[kCdfKnots];
  const float* pf = params + static_cast<size_t>(f) * P;
  for (int e = threadIdx.x; e < P; e += blockDim.x) p[e] = pf[e];
  __syncthreads();
  const float lo = zrange[2 * f], hi = zrange[2 * f + 1];
  const float dz = (hi - lo) / (kCdfKnots - 1);
  for (int k = threadIdx.x; k < kCdfKnots; k += blockDim.x) {
    const float z = lo + dz * k;
    float h1[H];
#pragma unroll
    for (int j = 0; j < H; ++j) h1[j] = tanhf(fmaf(p[oW1 + j], z, p[oB1 + j]));
    float o = p[oB3];
    for (int i = 0; i < H; ++i) {
      float a = p[oB2 + i];
#pragma unroll
      for (int j = 0; j < H; ++j) a = fmaf(p[oW2 + i * H + j], h1[j], a);
      o = fmaf(p[oW3 + i], tanhf(a), o);
    }
    const float v = sigmoidf_(o);
    u[k] = fminf(fmaxf(v, 0.0f), 1.0f);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    float run = 0.0f;
    for (int k = 0; k < kCdfKnots; ++k) {
      run = fmaxf(run, u[k]);
      u[k] = (1.0f - kCdfLinearShare) * run + kCdfLinearShare * (static_cast<float>(k) / (kCdfKnots - 1));
    }
  }
  __syncthreads();
  for (int k = threadIdx.x; k < kCdfKnots; k += blockDim.x) table[static_cast<size_t>(f) * kCdfKnots + k] = u[k];
}

// The grid used when no network is trained: u rises linearly over [lo, hi]
// (uniform buckets in standardised value) -- the "method without the network".
__global__ void k_cdf_linear_table(const float* __restrict__ zrange, float* __restrict__ table) {
  const int f = blockIdx.x;
  for (int k = threadIdx.x; k < kCdfKnots; k += blockDim.x)
    table[static_cast<size_t>(f) * kCdfKnots + k] = static_cast<float>(k) / (kCdfKnots - 1);
  (void)zrange;
}

size_t cdf_train_smem() { return sizeof(TrainSmem); }

cudaError_t launch_cdf_features(const float* X, const float* ranks, int F, int T, int N, int t0, int tcount, int S,
                                float2* samples, cudaStream_t s) {
  dim3 g(tcount, F);
  k_cdf_features<<<g, 256, 0, s>>>(X, ranks, T, N, t0, tcount, S, samples);
  return cudaGetLastError();
}

cudaError_t launch_cdf_train(float* params, float* adam, const float2* samples, int F, int nsamp, int steps, float lr,
                             int step0, float* loss_out, cudaStream_t s) {
  const size_t smem = sizeof(TrainSmem);
  cudaError_t e = cudaFuncSetAttribute(k_cdf_train, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  k_cdf_train<<<F, BATCH, smem, s>>>(params, adam, samples, nsamp, steps, lr, step0, loss_out);
  return cudaGetLastError();
}

cudaError_t launch_cdf_grad(const float* params, const float* z, const float* u, int n, float* grad, float* loss,
                            cudaStream_t s) {
  const size_t smem = sizeof(TrainSmem);
  cudaError_t e = cudaFuncSetAttribute(k_cdf_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  k_cdf_grad<<<1, BATCH, smem, s>>>(params, z, u, n, grad, loss);
  return cudaGetLastError();
}

cudaError_t launch_cdf_tabulate(const float* params, const float2* samples, int F, int nsamp, float* zrange,
                                float* table, bool linear, cudaStream_t s) {
  const size_t smem = 8192 * (4 + 4 + 2 + 2) + SortScratch<512>::bytes;
  cudaError_t e = cudaFuncSetAttribute(k_cdf_range, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  k_cdf_range<<<F, 512, smem, s>>>(samples, nsamp, zrange);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (linear)
    k_cdf_linear_table<<<F, 256, 0, s>>>(zrange, table);
  else
    k_cdf_tabulate<<<F, 256, 0, s>>>(params, zrange, table);
  return cudaGetLastError();
}

}  // namespace fcb
