// fc_tc.cu -- factor_corr precision form: the masked moment products of the
// pooled pairwise-complete correlation as BF16x3 tcgen05 GEMMs over the
// R = T*N pooled rows, with an FP64 finalize.
//
// factor_corr pools the (t, i) rows of an (R, F) panel (fc/_cpu_core.py:232-269;
// the reference GPU form is src/factor_corr.cu:392-563, one CTA per pair).  With
// x'_f = x_f - c_f on valid cells (0 elsewhere; c_f a per-factor shift, see
// k_fct_shift) and m_f the validity, a pair needs
//   n = sum m_f m_g,  Sx = sum x'_f m_g,  Sy = sum m_f x'_g,
//   Sxy = sum x'_f x'_g,  Sx2 = sum x'_f^2 m_g,  Sy2 = sum m_f x'_g^2,
// the products M^T M, X'^T M, X'^T X', X'^2^T M of the reference's masked-GEMM
// formulation (fc/_cpu_core.py:139-169).  Every value is split into bf16
// limbs -- x' = H + Mm + L and x'^2 = Qh + Qm + Ql (24 significant bits each,
// exact for f32), m exact -- and the rows of the A operand are the stack
//   [M; H; Mm; L; Qh; Qm; Ql]  (7 blocks of 16 factor rows, 112 of 128 used)
// while B is its first four blocks [M; H; Mm; L] (64 rows, the same shared
// memory).  One 128 x 64 x 16 MMA per 16 pooled rows leaves every limb product
// in its own FP32 accumulator; K = R is split over one persistent CTA per SM,
// and each CTA drains its accumulators into FP64 every 2048 rows (two TMEM
// buffers, so the drain overlaps the next window's MMAs).  Only the limb sums,
// the count / mean / variance correction and the normalisation run in FP64.
//
// The limbs are made in shared memory, not in HBM: converter warps read the
// f32 panel (one pass, 128-bit loads for factor planes) and write the seven
// limb rows of each factor straight into the 128-byte-swizzled K-major layout
// the MMA reads, so the panel is read once and nothing else touches HBM.
//
// Warps: 0-7 converters (warp w fills stage w, 64 pooled rows), 8 TMEM owner
// and MMA issuer, 9-12 epilogue (TMEM lane quadrant = warp % 4).  Every
// mbarrier wait is bounded and reports through the status word.
#include "fcb_common.cuh"
#include "fcb_kernels.h"
#include "tc_common.cuh"

namespace fcb {
namespace {

constexpr int kFtFp = 16;                      // factor rows per limb block
constexpr int kFtRowsA = 7 * kFtFp;            // 112 used A rows (of 128)
constexpr int kFtN = 4 * kFtFp;                // 64 B rows = accumulator columns
constexpr int kFtK = 64;                       // pooled rows per stage (one 128-byte line)
constexpr int kFtConv = 8;                     // converter warps = stages
constexpr int kFtStageBytes = 128 * kFtK * 2;  // 16 KB
constexpr int kFtWindow = 32;                  // stages per accumulator window (2048 rows)
constexpr int kFtThreads = (kFtConv + 1 + 4) * 32;
constexpr int kFtTmemCols = 128;               // two windows of 64 columns
constexpr int kFtPairs = kFtFp * kFtFp;

struct FtSmem {  // after the 1024-aligned stages
  double scr[10][kFtPairs];  // one window's limb partials: n | sx (3) | sxy (3) | sx2 (3)
  double acc[4][kFtPairs];   // running n, Sx, Sxy, Sx2
  uint64_t full[kFtConv], empty[kFtConv], accfull[2], accempty[2];
  uint32_t tmem_slot;
  int err;
};

FCB_DEV uint32_t pack_bf16x2(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&v);
}
FCB_DEV float bf16_lo(uint32_t p) { return __uint_as_float(p << 16); }
FCB_DEV float bf16_hi(uint32_t p) { return __uint_as_float(p & 0xFFFF0000u); }

// Three-limb split of a pair of f32 values: v = h + m + l exactly.
FCB_DEV void split3(float v0, float v1, uint32_t& h, uint32_t& m, uint32_t& l) {
  h = pack_bf16x2(v0, v1);
  const float r0 = v0 - bf16_lo(h), r1 = v1 - bf16_hi(h);
  m = pack_bf16x2(r0, r1);
  l = pack_bf16x2(r0 - bf16_lo(m), r1 - bf16_hi(m));
}

}  // namespace

// Per-factor shift c_f: the mean of the valid cells among 4096 rows spread
// evenly over the pool (the moment formulas are shift invariant; a shift near
// the mean keeps the FP32 sums well conditioned).  One block per factor; each
// thread issues its 16 sample loads before it adds them (row q*R/4096 is a
// shift, not a 64-bit division).
__global__ void __launch_bounds__(256) k_fct_shift(const float* __restrict__ X, const uint8_t* __restrict__ mask,
                                                   long long R, long long sr, long long sf, float* __restrict__ shift) {
  constexpr int kPer = 4096 / 256;
  __shared__ double red[66];
  const int f = blockIdx.x;
  float v[kPer];
  bool ok[kPer];
#pragma unroll
  for (int u = 0; u < kPer; ++u) {
    const long long q = threadIdx.x + 256LL * u;
    ok[u] = q < R;
    const long long r = R >= 4096 ? (q * R) >> 12 : q;
    v[u] = ok[u] ? X[r * sr + f * sf] : 0.0f;
    if (ok[u] && mask != nullptr) ok[u] = mask[r] != 0;
  }
  double s = 0.0, c = 0.0;
#pragma unroll
  for (int u = 0; u < kPer; ++u) {
    if (ok[u] && finite_f32(v[u])) {
      s += v[u];
      c += 1.0;
    }
  }
  s = block_sum(s, red);
  c = block_sum(c, red);
  if (threadIdx.x == 0) shift[f] = c > 0.0 ? static_cast<float>(s / c) : 0.0f;
}

__global__ void __launch_bounds__(kFtThreads, 1)
    k_fct_gram(const float* __restrict__ X, const uint8_t* __restrict__ mask, long long R, int F, long long sr,
               long long sf, const float* __restrict__ shift, double* __restrict__ part, int* __restrict__ status) {
  extern __shared__ __align__(1024) uint8_t sm_raw[];
  uint8_t* stages = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(sm_raw) + 1023) & ~uintptr_t(1023));
  FtSmem& S = *reinterpret_cast<FtSmem*>(stages + kFtConv * kFtStageBytes);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // this CTA's stages (64 pooled rows each)
  const long long nst_all = (R + kFtK - 1) / kFtK;
  const long long k0 = nst_all * blockIdx.x / gridDim.x, k1 = nst_all * (blockIdx.x + 1) / gridDim.x;
  const int nst = static_cast<int>(k1 - k0);
  const int nwin = (nst + kFtWindow - 1) / kFtWindow;

  // zero the stages once (pad rows and pad factors stay zero), the
  // accumulators, and set up the barriers and TMEM
  for (int i = threadIdx.x; i < kFtConv * kFtStageBytes / 16; i += kFtThreads)
    reinterpret_cast<uint4*>(stages)[i] = make_uint4(0u, 0u, 0u, 0u);
  for (int i = threadIdx.x; i < 4 * kFtPairs; i += kFtThreads) (&S.acc[0][0])[i] = 0.0;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kFtConv; ++s) {
      mbar_init(&S.full[s], 1);
      mbar_init(&S.empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&S.accfull[b], 1);
      mbar_init(&S.accempty[b], 4);
    }
    S.err = 0;
    fence_mbar_init();
  }
  if (warp == kFtConv) tmem_alloc(&S.tmem_slot, kFtTmemCols);
  // the zero fill above was written by the generic proxy; the MMAs read the
  // stages through the async proxy
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = S.tmem_slot;

  if (warp < kFtConv) {
    // ---------------- converters: warp w fills stage w for local stages w, w+8, ...
    uint8_t* st = stages + warp * kFtStageBytes;
    const uint32_t st_addr = smem_u32(st);
    const bool planes = (sr == 1);
    for (int j = warp; j < nst; j += kFtConv) {
      const int round = j / kFtConv;
      if (round > 0 && !mbar_wait(&S.empty[warp], (round - 1) & 1)) {
        atomicExch(&S.err, 1);
        break;
      }
      const long long r0 = (k0 + j) * kFtK;
      for (int q = lane; q < 8 * F; q += 32) {
        // planes: 8 lanes per factor walk its 64 rows (32 contiguous bytes each);
        // rows: consecutive lanes take consecutive factors of the same rows
        const int f = planes ? q >> 3 : q % F;
        const int c = planes ? q & 7 : q / F;
        const long long rr = r0 + 8 * c;
        float x[8];
        const float* src = X + rr * sr + f * sf;
        if (planes && rr + 7 < R && (reinterpret_cast<uintptr_t>(src) & 15u) == 0) {
          const float4 a = __ldcs(reinterpret_cast<const float4*>(src));
          const float4 b = __ldcs(reinterpret_cast<const float4*>(src) + 1);
          x[0] = a.x; x[1] = a.y; x[2] = a.z; x[3] = a.w;
          x[4] = b.x; x[5] = b.y; x[6] = b.z; x[7] = b.w;
        } else {
#pragma unroll
          for (int e = 0; e < 8; ++e) x[e] = (rr + e < R) ? __ldcs(src + e * sr) : __uint_as_float(kQuietNanBits);
        }
        uint32_t mk0 = 0xFFFFFFFFu, mk1 = 0xFFFFFFFFu;  // mask bytes (all set without a mask)
        if (mask != nullptr) {
          if (rr + 7 < R && (reinterpret_cast<uintptr_t>(mask + rr) & 7u) == 0) {
            const uint2 mm = __ldg(reinterpret_cast<const uint2*>(mask + rr));
            mk0 = mm.x;
            mk1 = mm.y;
          } else {
            mk0 = mk1 = 0u;
#pragma unroll
            for (int e = 0; e < 8; ++e) {
              const uint32_t b = (rr + e < R && mask[rr + e] != 0) ? 0xFFu : 0u;
              if (e < 4) mk0 |= b << (8 * e); else mk1 |= b << (8 * (e - 4));
            }
          }
        }
        const float cf = shift[f];
        float v[8], one[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          const uint32_t mb = ((e < 4 ? mk0 >> (8 * e) : mk1 >> (8 * (e - 4))) & 0xFFu);
          const bool ok = finite_f32(x[e]) && mb != 0u;
          v[e] = ok ? x[e] - cf : 0.0f;
          one[e] = ok ? 1.0f : 0.0f;
        }
        uint4 lm, lh, lmm, ll, lqh, lqm, lql;
        uint32_t* pm = &lm.x;
        uint32_t* ph = &lh.x;
        uint32_t* pmm = &lmm.x;
        uint32_t* pl = &ll.x;
        uint32_t* pqh = &lqh.x;
        uint32_t* pqm = &lqm.x;
        uint32_t* pql = &lql.x;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          pm[e] = pack_bf16x2(one[2 * e], one[2 * e + 1]);
          split3(v[2 * e], v[2 * e + 1], ph[e], pmm[e], pl[e]);
          split3(v[2 * e] * v[2 * e], v[2 * e + 1] * v[2 * e + 1], pqh[e], pqm[e], pql[e]);
        }
        // row (L, f) = L*16 + f; 16-byte chunk c of the row at chunk c ^ (row & 7)
        const uint4* limbs[7] = {&lm, &lh, &lmm, &ll, &lqh, &lqm, &lql};
#pragma unroll
        for (int L = 0; L < 7; ++L) {
          const int row = L * kFtFp + f;
          *reinterpret_cast<uint4*>(st + row * 128 + ((c ^ (row & 7)) << 4)) = *limbs[L];
        }
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(&S.full[warp]);
    }
    (void)st_addr;
  } else if (warp == kFtConv) {
    // ---------------- MMA issuer
    if (lane == 0) {
      constexpr uint32_t idesc = idesc_bf16(128, kFtN);
      const uint32_t base = smem_u32(stages);
      for (int j = 0; j < nst; ++j) {
        const int s = j % kFtConv;
        const int win = j / kFtWindow, buf = win & 1;
        const bool wfirst = (j % kFtWindow) == 0;
        if (wfirst && win >= 2 && !mbar_wait(&S.accempty[buf], ((win >> 1) - 1) & 1)) {
          atomicExch(&S.err, 1);
          break;
        }
        if (!mbar_wait(&S.full[s], (j / kFtConv) & 1)) {
          atomicExch(&S.err, 1);
          break;
        }
        tc_fence_after();
        const uint32_t a0 = base + s * kFtStageBytes;
        const uint32_t d = tmem + static_cast<uint32_t>(buf * kFtN);
#pragma unroll
        for (int ks = 0; ks < kFtK / 16; ++ks) {
          const uint64_t ad = smem_desc_sw128(a0 + ks * 32);
          mma_bf16(d, ad, ad, idesc, (wfirst && ks == 0) ? 0u : 1u);  // B = the first 64 rows of A
        }
        mma_commit(&S.empty[s]);
        if ((j + 1) % kFtWindow == 0 || j + 1 == nst) mma_commit(&S.accfull[buf]);
      }
    }
    __syncwarp();
  } else {
    // ---------------- epilogue: lane quadrant warp % 4; TMEM row = A row
    const int quad = warp & 3;
    const int row = quad * 32 + lane;
    const int L = row / kFtFp, f = row % kFtFp;
    const int et = threadIdx.x - (kFtConv + 1) * 32;  // 0..127
    const uint32_t lrow = static_cast<uint32_t>(quad * 32) << 16;
    for (int w = 0; w < nwin; ++w) {
      const int buf = w & 1;
      const bool ok = mbar_wait(&S.accfull[buf], (w >> 1) & 1);
      if (!ok) atomicExch(&S.err, 1);
      tc_fence_after();
      float v[kFtN];
#pragma unroll
      for (int c0 = 0; c0 < kFtN; c0 += 16) tmem_ld16(tmem + lrow + buf * kFtN + c0, v + c0);
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&S.accempty[buf]);
      // this row's limb partials: columns [B*16 + g], B in {M, H, Mm, L}
      if (L < 7 && f < F) {
        for (int g = 0; g < F; ++g) {
          const int pr = f * kFtFp + g;
          if (L == 0) {
            S.scr[0][pr] = v[g];
          } else if (L <= 3) {
            S.scr[L][pr] = v[g];
            S.scr[3 + L][pr] = static_cast<double>(v[16 + g]) + static_cast<double>(v[32 + g]) +
                               static_cast<double>(v[48 + g]);
          } else {
            S.scr[3 + L][pr] = v[g];
          }
        }
      }
      named_sync(1, 128);
      // fixed-order merge into the running FP64 sums
      for (int pr = et; pr < kFtPairs; pr += 128) {
        if (pr / kFtFp >= F || pr % kFtFp >= F) continue;
        S.acc[0][pr] += S.scr[0][pr];
        S.acc[1][pr] += (S.scr[1][pr] + S.scr[2][pr]) + S.scr[3][pr];
        S.acc[2][pr] += (S.scr[4][pr] + S.scr[5][pr]) + S.scr[6][pr];
        S.acc[3][pr] += (S.scr[7][pr] + S.scr[8][pr]) + S.scr[9][pr];
      }
      named_sync(1, 128);
    }
    // this CTA's FP64 sums: part[cta][4][16][16]
    double* dst = part + static_cast<size_t>(blockIdx.x) * 4 * kFtPairs;
    for (int i = et; i < 4 * kFtPairs; i += 128) dst[i] = (&S.acc[0][0])[i];
  }
  tc_fence_before();
  __syncthreads();
  if (warp == kFtConv) {
    tc_fence_after();
    tmem_dealloc(tmem, kFtTmemCols);
  }
  if (threadIdx.x == 0 && S.err != 0) atomicExch(status, 1);
}

// Merge of the CTAs' sums and the FP64 finalize, one warp per pair f <= g:
// lane l adds the partials of CTAs l, l + 32, ... in order, then a fixed xor
// tree adds the lanes (the same order on every call).  Then
//   cov = Sxy - Sx Sy / n,  vx = Sx2 - Sx^2 / n,  vy likewise,
//   r = (cov / sqrt(vx)) / sqrt(vy); NaN for n < 2 or a non-positive variance;
// the diagonal is 1.0 iff the self-correlation is finite; the lower triangle
// mirrors the upper.
__global__ void k_fct_final(const double* __restrict__ part, int nblk, int F, double* __restrict__ out) {
  const int p = static_cast<int>((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int lane = static_cast<int>(threadIdx.x & 31);
  if (p >= F * F) return;
  const int f = p / F, g = p % F;
  if (f > g) return;
  const int fg = f * kFtFp + g, gf = g * kFtFp + f;
  double n = 0.0, sx = 0.0, sy = 0.0, sxy = 0.0, sx2 = 0.0, sy2 = 0.0;
  for (int b = lane; b < nblk; b += 32) {
    const double* q = part + static_cast<size_t>(b) * 4 * kFtPairs;
    n += q[fg];
    sx += q[kFtPairs + fg];
    sy += q[kFtPairs + gf];
    sxy += q[2 * kFtPairs + fg];
    sx2 += q[3 * kFtPairs + fg];
    sy2 += q[3 * kFtPairs + gf];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    n += __shfl_xor_sync(kFull, n, o);
    sx += __shfl_xor_sync(kFull, sx, o);
    sy += __shfl_xor_sync(kFull, sy, o);
    sxy += __shfl_xor_sync(kFull, sxy, o);
    sx2 += __shfl_xor_sync(kFull, sx2, o);
    sy2 += __shfl_xor_sync(kFull, sy2, o);
  }
  if (lane != 0) return;
  double r = __longlong_as_double(0x7ff8000000000000ll);
  if (n >= 2.0) {
    const double cov = sxy - sx * sy / n;
    const double vx = sx2 - sx * sx / n;
    const double vy = sy2 - sy * sy / n;
    if (vx > 0.0 && vy > 0.0) {
      const double c = (cov / sqrt(vx)) / sqrt(vy);
      if (isfinite(c)) r = c;
    }
  }
  if (f == g) r = isfinite(r) ? 1.0 : r;
  out[static_cast<size_t>(f) * F + g] = r;
  out[static_cast<size_t>(g) * F + f] = r;
}

size_t fc_tc_smem() { return static_cast<size_t>(kFtConv) * kFtStageBytes + sizeof(FtSmem) + 1024; }

size_t fc_tc_work_bytes(int F) {
  (void)F;
  return 4096 + static_cast<size_t>(1024) * 4 * kFtPairs * sizeof(double);
}

cudaError_t launch_factor_corr_bf16x3(const float* X, const uint8_t* mask, long long R, int F, long long sr,
                                      long long sf, void* work, double* out, int* status, cudaStream_t s) {
  if (F < 1 || F > kFcTcMaxF || R < 1) return cudaErrorInvalidValue;
  int dev = 0, sms = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  // one CTA per SM, each with at least a few windows of rows
  long long grid = sms > 0 ? sms : 1;
  const long long nst = (R + kFtK - 1) / kFtK;
  if (grid > (nst + 3) / 4) grid = (nst + 3) / 4;
  if (grid < 1) grid = 1;
  if (grid > 1024) grid = 1024;
  float* shift = static_cast<float*>(work);
  double* part = reinterpret_cast<double*>(static_cast<uint8_t*>(work) + 4096);
  k_fct_shift<<<F, 256, 0, s>>>(X, mask, R, sr, sf, shift);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  const size_t smem = fc_tc_smem();
  if ((e = cudaFuncSetAttribute(k_fct_gram, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem))) !=
      cudaSuccess)
    return e;
  k_fct_gram<<<static_cast<unsigned>(grid), kFtThreads, smem, s>>>(X, mask, R, F, sr, sf, shift, part, status);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  k_fct_final<<<(F * F + 3) / 4, 128, 0, s>>>(part, static_cast<int>(grid), F, out);
  return cudaGetLastError();
}

}  // namespace fcb
