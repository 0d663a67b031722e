// corr_tc.cu -- precision forms of stock_corr: BF16x3 on the tcgen05 tensor
// cores and a plain FP32 SIMT path, both with an FP64 finalize.
//
// Pairwise-complete Pearson over t needs six moment sums per stock pair
// (i,j) over the joint valid dates: n, sum x, sum y, sum xy, sum x^2, sum y^2
// (the masked products X.M^T, X.X^T, X^2.M^T, M.M^T of the reference's
// masked-GEMM formulation, fc/_cpu_core.py:139-169).  Each column is first
// centred by its own valid-date mean (the pairwise formula is shift
// invariant), so the products stay well conditioned.
//
// BF16x3: x' and x'^2 are each split into three bf16 limbs (hi + mid + lo,
// 24 significant bits -- exact for an f32 value); the mask M is exact in bf16.
// An output tile is 128 stocks i (the A operand) by 64 stocks j (B); the
// operand stage of each side is the stack [M; H; Mm; L; Qh; Qm; Ql] of its
// stocks.  Per 16-deep k step (tcgen05.mma kind::f16, bf16 in, fp32
// accumulate in TMEM), with every limb of a sum accumulated into the same
// TMEM columns:
//   D1  (256 cols) += H_i . [M; H; Mm; L]_j^T, Mm_i . [M; H; Mm]_j^T,
//                     L_i . [M; H]_j^T
//                     -> sx | three column blocks whose sum is sxy
//                     (the limb products Mm.L, L.Mm and L.L are left out: a
//                     limb is below 2^-8 of the one above it, so they are
//                     under 2^-26 of x'_i x'_j, below the FP32 accumulation's
//                     own rounding)
//   Dn|Dsy (128)    = M_i . [M; H]_j^T, then Dsy += M_i . Mm_j^T, M_i . L_j^T
//   Dsy2 (64)      += M_i . q_j^T            for q in {Qh, Qm, Ql}
//   Dsx2 (64)      += q_i . M_j^T            for q in {Qh, Qm, Ql}
// 512 TMEM columns in all.  Each stage's operands (84 KB) serve 8192 outputs.
// Operands are staged by TMA (cp.async.bulk.tensor, no cluster multicast) in
// the canonical K-major 64-byte-swizzle layout: each stock row holds the stage's
// 32 dates as one 64-byte line, 8-row groups 512 bytes apart, and the seven
// matrices of an operand follow one another, so a sub-stack of the B operand
// is a run of consecutive rows.  One 3D box per operand fills a stage with full
// 64-byte row reads (a 16-byte-wide box would fetch a 32-byte sector per 16
// bytes used).
// The FP64 finalize is
//   cov = sxy - sx sy / n, vx = sx2 - sx^2/n, vy = sy2 - sy^2/n,
//   r = (cov/sqrt(vx))/sqrt(vy),  NaN for n < 2 or a non-positive variance.
#include <cuda.h>

#include <cmath>
#include <mutex>

#include "fcb_common.cuh"
#include "fcb_kernels.h"
#include "tc_common.cuh"

namespace fcb {

constexpr int kTcM = kPrecTileTcM;  // output rows per tile (stocks i)
constexpr int kTcN = kPrecTileTcN;  // output columns per tile (stocks j)
constexpr int kTcK = 32;            // k depth per pipeline stage
constexpr int kTcStages = 2;
constexpr int kTcMats = 7;     // operand matrices, order M H Mm L Qh Qm Ql
constexpr int kRowBytes = kTcK * 2;                   // one stock's dates of a stage (64 B)
constexpr int kAMat = kTcM * kRowBytes;               // one A matrix of a stage
constexpr int kBMat = kTcN * kRowBytes;               // one B matrix of a stage
constexpr int kABytesStage = kTcMats * kAMat;
constexpr int kBBytesStage = kTcMats * kBMat;
constexpr int kStageBytes = kABytesStage + kBBytesStage;
// TMEM columns of the accumulators (64 columns = one tile width each)
constexpr int kD1 = 0, kDn = 4 * kTcN, kDsy = 5 * kTcN, kDsy2 = 6 * kTcN, kDsx2 = 7 * kTcN;
constexpr int kTmemCols = 8 * kTcN;
// warps: 0 TMA producer, 1 TMEM owner + MMA issuer, 2..9 epilogue (two per TMEM
// lane quadrant, each reading half of the tile's columns)
constexpr int kTcEpiWarps = 8;
constexpr int kTcThreads = (2 + kTcEpiWarps) * 32;
static_assert(kTmemCols == 512, "the accumulators fill the TMEM of one CTA");

// ---------------------------------------------------------------------------
// prep: (T,N) f32 + mask -> K-major (Np, Tp) operands
// ---------------------------------------------------------------------------
// Column means of the valid cells, in two steps so that enough blocks are in
// flight: k_prec_colpart sums a chunk of dates per block (block (32, 8): 32
// columns, 8 date strides, coalesced row reads) into part[chunk][i] = (sum,
// count); k_prec_colmean adds the chunks in order (deterministic).
__global__ void k_prec_colpart(const float* __restrict__ X, const uint8_t* __restrict__ mask, int T, int N, int Np,
                               int tchunk, double2* __restrict__ part) {
  __shared__ double ss[8][33];
  __shared__ double sc[8][33];
  const int i = blockIdx.x * 32 + threadIdx.x;
  const int t0 = blockIdx.y * tchunk, t1 = min(T, t0 + tchunk);
  double s = 0.0, c = 0.0;
  if (i < N) {
    for (int t = t0 + threadIdx.y; t < t1; t += 8) {
      const size_t e = static_cast<size_t>(t) * N + i;
      const float v = X[e];
      if (finite_f32(v) && (mask == nullptr || mask[e])) {
        s += v;
        c += 1.0;
      }
    }
  }
  ss[threadIdx.y][threadIdx.x] = s;
  sc[threadIdx.y][threadIdx.x] = c;
  __syncthreads();
  if (threadIdx.y == 0 && i < N) {
    for (int y = 1; y < 8; ++y) {
      s += ss[y][threadIdx.x];
      c += sc[y][threadIdx.x];
    }
    part[static_cast<size_t>(blockIdx.y) * Np + i] = make_double2(s, c);
  }
}

__global__ void k_prec_colmean(const double2* __restrict__ part, int nchunk, int N, int Np, float* __restrict__ mu) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double s = 0.0, c = 0.0;
  for (int k = 0; k < nchunk; ++k) {
    const double2 v = part[static_cast<size_t>(k) * Np + i];
    s += v.x;
    c += v.y;
  }
  mu[i] = c > 0 ? static_cast<float>(s / c) : 0.0f;
}

int prec_colmean_chunks(int T) { return T / 64 < 1 ? 1 : (T / 64 > 32 ? 32 : T / 64); }

// Transposing split: one 32x32 (t,i) tile per block.
__global__ void k_prec_split(const float* __restrict__ X, const uint8_t* __restrict__ mask, const float* __restrict__ mu,
                             int T, int N, int Tp, PrecOperands op) {
  __shared__ float tv[32][33];
  __shared__ float tm[32][33];
  const int t0 = blockIdx.x * 32, i0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int t = t0 + r, i = i0 + threadIdx.x;
    float v = 0.0f, m = 0.0f;
    if (t < T && i < N) {
      const size_t e = static_cast<size_t>(t) * N + i;
      const float x = X[e];
      if (finite_f32(x) && (mask == nullptr || mask[e])) {
        v = x - mu[i];
        m = 1.0f;
      }
    }
    tv[r][threadIdx.x] = v;
    tm[r][threadIdx.x] = m;
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int i = i0 + r, t = t0 + threadIdx.x;
    if (t >= Tp) continue;
    const size_t o = static_cast<size_t>(i) * Tp + t;  // rows up to Np (zero pad)
    const float v = tv[threadIdx.x][r];
    const float m = tm[threadIdx.x][r];
    if (op.h != nullptr) {
      const __nv_bfloat16 h = __float2bfloat16_rn(v);
      const float r1 = v - __bfloat162float(h);
      const __nv_bfloat16 mm = __float2bfloat16_rn(r1);
      const __nv_bfloat16 l = __float2bfloat16_rn(r1 - __bfloat162float(mm));
      const float q = v * v;
      const __nv_bfloat16 qh = __float2bfloat16_rn(q);
      const float s1 = q - __bfloat162float(qh);
      const __nv_bfloat16 qm = __float2bfloat16_rn(s1);
      const __nv_bfloat16 ql = __float2bfloat16_rn(s1 - __bfloat162float(qm));
      const size_t plane = static_cast<size_t>(op.np) * Tp;
      __nv_bfloat16* b = op.h;  // [7][Np][Tp]: M H Mm L Qh Qm Ql
      b[o] = __float2bfloat16_rn(m);
      b[plane + o] = h;
      b[2 * plane + o] = mm;
      b[3 * plane + o] = l;
      b[4 * plane + o] = qh;
      b[5 * plane + o] = qm;
      b[6 * plane + o] = ql;
    }
    if (op.x32 != nullptr) {
      op.x32[o] = v;
      op.q32[o] = v * v;
      op.m32[o] = m;
    }
  }
}

FCB_DEV double pearson_from_moments(double n, double sx, double sy, double sxy, double sx2, double sy2) {
  if (n < 2.0) return __longlong_as_double(0x7ff8000000000000ll);
  const double cov = sxy - sx * sy / n;
  const double vx = sx2 - sx * sx / n;
  const double vy = sy2 - sy * sy / n;
  if (!(vx > 0.0 && vy > 0.0)) return __longlong_as_double(0x7ff8000000000000ll);
  const double r = (cov / sqrt(vx)) / sqrt(vy);
  return isfinite(r) ? r : __longlong_as_double(0x7ff8000000000000ll);
}

FCB_DEV void write_pair(double* out, int N, int i, int j, double r) {
  if (i == j) r = isfinite(r) ? 1.0 : r;
  out[static_cast<size_t>(i) * N + j] = r;
  out[static_cast<size_t>(j) * N + i] = r;
}

// ---------------------------------------------------------------------------
// BF16x3 tcgen05 kernel: persistent CTAs over 128 x 64 output tiles
// warps: 0 TMA producer, 1 TMEM owner + MMA issuer, 2..9 epilogue
// ---------------------------------------------------------------------------
// Two 3D views of the [7][Np][Tp] operand buffer (64-byte swizzle): one TMA
// per operand fills a whole stage.
struct TcMaps {
  CUtensorMap a;  // box {32, 128, 7}
  CUtensorMap b;  // box {32, 32, 7}
};

__global__ void __launch_bounds__(kTcThreads, 1)
    k_corr_bf16x3(const __grid_constant__ TcMaps maps, const int2* __restrict__ tiles, int ntiles, int N, int Tp,
                  double* __restrict__ out, int* __restrict__ status) {
  extern __shared__ __align__(1024) uint8_t sm_raw[];
  uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(sm_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(sm + kTcStages * kStageBytes);
  uint64_t* empty = full + kTcStages;
  uint64_t* accb = empty + kTcStages;   // accumulators of a tile complete (MMA commit)
  uint64_t* tfree = accb + 1;           // accumulators read out (one arrival per epilogue warp)
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tfree + 1);
  int* err = reinterpret_cast<int*>(tmem_slot + 1);
  volatile int* verr = err;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nkt = Tp / kTcK;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kTcStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(accb, 1);
    mbar_init(tfree, kTcEpiWarps);
    *err = 0;
    fence_mbar_init();
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  // Persistent CTAs walk the tile list with a stride of the grid.  The stage
  // ring runs on across tiles, so the producer fills the next tile's stages
  // while the epilogue drains this tile's accumulators; the MMA warp starts a
  // tile once the epilogue has read the previous one out of TMEM.
  if (warp == 0) {
    if (lane == 0) {
      int g = 0;
      for (int tl = blockIdx.x; tl < ntiles && *verr == 0; tl += gridDim.x) {
        const int2 tile = tiles[tl];
        const int i0 = tile.x * kTcM, j0 = tile.y * kTcN;
        for (int kt = 0; kt < nkt; ++kt, ++g) {
          const int s = g % kTcStages, round = g / kTcStages;
          if (round > 0 && !mbar_wait(&empty[s], (round - 1) & 1)) {
            atomicExch(err, 1);
            break;
          }
          uint8_t* st = sm + s * kStageBytes;
          mbar_expect_tx(&full[s], kStageBytes);
          tma_load_3d(st, &maps.a, kt * kTcK, i0, 0, &full[s]);
          tma_load_3d(st + kABytesStage, &maps.b, kt * kTcK, j0, 0, &full[s]);
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      constexpr uint32_t id256 = idesc_bf16(kTcM, 4 * kTcN);
      constexpr uint32_t id192 = idesc_bf16(kTcM, 3 * kTcN);
      constexpr uint32_t id128 = idesc_bf16(kTcM, 2 * kTcN);
      constexpr uint32_t id64 = idesc_bf16(kTcM, kTcN);
      int g = 0, it = 0;
      for (int tl = blockIdx.x; tl < ntiles && *verr == 0; tl += gridDim.x, ++it) {
        if (it > 0 && !mbar_wait(tfree, (it - 1) & 1)) {
          atomicExch(err, 1);
          break;
        }
        tc_fence_after();
        for (int kt = 0; kt < nkt; ++kt, ++g) {
          const int s = g % kTcStages, round = g / kTcStages;
          if (!mbar_wait(&full[s], round & 1)) {
            atomicExch(err, 1);
            break;
          }
          tc_fence_after();
          const uint32_t abase = smem_u32(sm + s * kStageBytes);
          const uint32_t bbase = abase + kABytesStage;
#pragma unroll
          for (int ks = 0; ks < kTcK / 16; ++ks) {
            const uint32_t ak = abase + ks * 32, bk = bbase + ks * 32;
            auto A = [&](int m) { return smem_desc_sw64(ak + m * kAMat); };  // rows of matrix m, stocks i
            auto B = [&](int m) { return smem_desc_sw64(bk + m * kBMat); };  // from matrix m on, stocks j
            const uint32_t first = (kt == 0 && ks == 0) ? 0u : 1u;
            // D1: H against [M; H; Mm; L], Mm against [M; H; Mm], L against [M; H]
            mma_bf16(tmem + kD1, A(1), B(0), id256, first);
            mma_bf16(tmem + kD1, A(2), B(0), id192, 1u);
            mma_bf16(tmem + kD1, A(3), B(0), id128, 1u);
            // n | sy: the mask against [M; H], then the other two y limbs into sy
            mma_bf16(tmem + kDn, A(0), B(0), id128, first);
            mma_bf16(tmem + kDsy, A(0), B(2), id64, 1u);
            mma_bf16(tmem + kDsy, A(0), B(3), id64, 1u);
            // sy2: the mask against the y'^2 limbs
            mma_bf16(tmem + kDsy2, A(0), B(4), id64, first);
            mma_bf16(tmem + kDsy2, A(0), B(5), id64, 1u);
            mma_bf16(tmem + kDsy2, A(0), B(6), id64, 1u);
            // sx2: the x'^2 limbs against the mask
            mma_bf16(tmem + kDsx2, A(4), B(0), id64, first);
            mma_bf16(tmem + kDsx2, A(5), B(0), id64, 1u);
            mma_bf16(tmem + kDsx2, A(6), B(0), id64, 1u);
          }
          mma_commit(&empty[s]);  // frees the stage when these MMAs complete
        }
        mma_commit(accb);
      }
    }
  } else {
    // epilogue: warp w reads TMEM lanes 32*(w%4) .. +31 (its row quadrant),
    // columns [half * kTcN/2, (half + 1) * kTcN/2)
    const int quad = warp & 3, half = (warp - 2) >> 2;
    const int row = quad * 32 + lane;
    const int cb = half * (kTcN / 2), ce = cb + kTcN / 2;
    const uint32_t t0 = tmem + (static_cast<uint32_t>(quad * 32) << 16);
    int it = 0;
    for (int tl = blockIdx.x; tl < ntiles; tl += gridDim.x, ++it) {
      const bool ok = mbar_wait(accb, it & 1);
      tc_fence_after();
      if (!ok) {
        atomicExch(err, 1);
        break;
      }
      const int2 tile = tiles[tl];
      const int i = tile.x * kTcM + row, j0 = tile.y * kTcN;
      for (int c0 = cb; c0 < ce; c0 += 16) {
        float sx[16], n[16], sy[16], sy2[16], sx2[16], v[16];
        double sxy[16];
        tmem_ld16(t0 + kD1 + c0, sx);
#pragma unroll
        for (int u = 0; u < 16; ++u) sxy[u] = 0.0;
#pragma unroll
        for (int b = 1; b <= 3; ++b) {
          tmem_ld16(t0 + kD1 + b * kTcN + c0, v);
#pragma unroll
          for (int u = 0; u < 16; ++u) sxy[u] += static_cast<double>(v[u]);
        }
        tmem_ld16(t0 + kDn + c0, n);
        tmem_ld16(t0 + kDsy + c0, sy);
        tmem_ld16(t0 + kDsy2 + c0, sy2);
        tmem_ld16(t0 + kDsx2 + c0, sx2);
        if (c0 + 16 >= ce) {
          // every column of this quadrant is in registers: hand TMEM back
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(tfree);
        }
        if (*verr == 0 && i < N) {
#pragma unroll
          for (int u = 0; u < 16; ++u) {
            const int j = j0 + c0 + u;
            if (j < N && i <= j)
              write_pair(out, N, i, j, pearson_from_moments(n[u], sx[u], sy[u], sxy[u], sx2[u], sy2[u]));
          }
        }
      }
      if (*verr != 0) break;
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
  }
  if (threadIdx.x == 0 && *err != 0) atomicExch(status, 1);
}

// ---------------------------------------------------------------------------
// plain FP32 SIMT path: 64 x 64 tiles, 256 threads, 4x4 cells per thread
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_corr_fp32(const float* __restrict__ X, const float* __restrict__ Q,
                                                   const float* __restrict__ M, const int2* __restrict__ tiles,
                                                   int N, int Tp, double* __restrict__ out) {
  constexpr int TS = 64, KT = 16;
  __shared__ float ax[KT][TS + 4], aq[KT][TS + 4], am[KT][TS + 4];
  __shared__ float bx[KT][TS + 4], bq[KT][TS + 4], bm[KT][TS + 4];
  const int2 tile = tiles[blockIdx.x];
  const int i0 = tile.x * TS, j0 = tile.y * TS;
  const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
  float acc[6][4][4];
#pragma unroll
  for (int q = 0; q < 6; ++q)
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) acc[q][a][b] = 0.0f;
  for (int k0 = 0; k0 < Tp; k0 += KT) {
    for (int e = threadIdx.x; e < TS * KT; e += 256) {
      const int r = e / KT, k = e % KT;
      const size_t oi = static_cast<size_t>(i0 + r) * Tp + k0 + k;
      const size_t oj = static_cast<size_t>(j0 + r) * Tp + k0 + k;
      ax[k][r] = X[oi];
      aq[k][r] = Q[oi];
      am[k][r] = M[oi];
      bx[k][r] = X[oj];
      bq[k][r] = Q[oj];
      bm[k][r] = M[oj];
    }
    __syncthreads();
#pragma unroll 4
    for (int k = 0; k < KT; ++k) {
      float xi[4], qi[4], mi[4], xj[4], qj[4], mj[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        xi[a] = ax[k][ty * 4 + a];
        qi[a] = aq[k][ty * 4 + a];
        mi[a] = am[k][ty * 4 + a];
        xj[a] = bx[k][tx * 4 + a];
        qj[a] = bq[k][tx * 4 + a];
        mj[a] = bm[k][tx * 4 + a];
      }
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          acc[0][a][b] = fmaf(mi[a], mj[b], acc[0][a][b]);
          acc[1][a][b] = fmaf(xi[a], mj[b], acc[1][a][b]);
          acc[2][a][b] = fmaf(mi[a], xj[b], acc[2][a][b]);
          acc[3][a][b] = fmaf(xi[a], xj[b], acc[3][a][b]);
          acc[4][a][b] = fmaf(qi[a], mj[b], acc[4][a][b]);
          acc[5][a][b] = fmaf(mi[a], qj[b], acc[5][a][b]);
        }
    }
    __syncthreads();
  }
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int i = i0 + ty * 4 + a, j = j0 + tx * 4 + b;
      if (i < N && j < N && i <= j)
        write_pair(out, N, i, j,
                   pearson_from_moments(acc[0][a][b], acc[1][a][b], acc[2][a][b], acc[3][a][b], acc[4][a][b],
                                        acc[5][a][b]));
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
// Tile lists on the device (no host vector, no upload).  BF16x3: 128 x 64
// tiles (ti, tj) that reach the upper triangle, tj >= 2 ti, row-major; row ti
// starts at ti*ntj - ti (ti-1).  FP32: 64 x 64 tiles tj >= ti; row ti starts
// at ti*n - ti (ti-1) / 2.  One thread per tile row.
__global__ void k_prec_tiles(int mode, int N, int2* __restrict__ tiles) {
  const int ti = blockIdx.x * blockDim.x + threadIdx.x;
  if (mode == 0) {
    const int nti = (N + kTcM - 1) / kTcM, ntj = (N + kTcN - 1) / kTcN;
    if (ti >= nti) return;
    static_assert(kTcM == 2 * kTcN, "tile row ti starts at column tile 2 ti");
    const long long off = static_cast<long long>(ti) * ntj - static_cast<long long>(ti) * (ti - 1);
    for (int tj = 2 * ti; tj < ntj; ++tj) tiles[off + (tj - 2 * ti)] = make_int2(ti, tj);
  } else {
    const int n = (N + kPrecTileFp32 - 1) / kPrecTileFp32;
    if (ti >= n) return;
    const long long off = static_cast<long long>(ti) * n - static_cast<long long>(ti) * (ti - 1) / 2;
    for (int tj = ti; tj < n; ++tj) tiles[off + (tj - ti)] = make_int2(ti, tj);
  }
}

int prec_tile_count(int mode, int N) {
  if (mode == 0) {
    const long long nti = (N + kTcM - 1) / kTcM, ntj = (N + kTcN - 1) / kTcN;
    return static_cast<int>(nti * ntj - nti * (nti - 1));
  }
  const long long n = (N + kPrecTileFp32 - 1) / kPrecTileFp32;
  return static_cast<int>(n * (n + 1) / 2);
}

cudaError_t launch_prec_tiles(int mode, int N, int2* tiles, cudaStream_t s) {
  const int rows = mode == 0 ? (N + kTcM - 1) / kTcM : (N + kPrecTileFp32 - 1) / kPrecTileFp32;
  k_prec_tiles<<<(rows + 127) / 128, 128, 0, s>>>(mode, N, tiles);
  return cudaGetLastError();
}

size_t prec_tc_smem() { return kTcStages * kStageBytes + 1024 + 256; }

cudaError_t launch_prec_prep(const float* X, const uint8_t* mask, int T, int N, int Np, int Tp, float* mu,
                             double2* part, PrecOperands op, cudaStream_t s) {
  const int nchunk = prec_colmean_chunks(T);
  const int tchunk = (T + nchunk - 1) / nchunk;
  k_prec_colpart<<<dim3((N + 31) / 32, nchunk), dim3(32, 8), 0, s>>>(X, mask, T, N, Np, tchunk, part);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_prec_colmean<<<(N + 255) / 256, 256, 0, s>>>(part, nchunk, N, Np, mu);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  dim3 g((Tp + 31) / 32, (Np + 31) / 32), b(32, 8);
  k_prec_split<<<g, b, 0, s>>>(X, mask, mu, T, N, Tp, op);
  return cudaGetLastError();
}

// cuTensorMapEncodeTiled is a driver-API call; it is resolved at run time
// through the runtime's entry-point query so that the library does not link
// libcuda and loads on hosts without a GPU driver.
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

// 3D map over the [7][Np][Tp] operand block: dims {Tp dates, Np stocks, 7
// matrices}; a box {32, rows, 7} is one stage of one operand, landing as
// (matrix, row, 64-byte swizzled line).
static CUresult make_map3(CUtensorMap* map, const void* base, int Np, int Tp, int box_rows) {
  const cuuint64_t dims[3] = {static_cast<cuuint64_t>(Tp), static_cast<cuuint64_t>(Np),
                              static_cast<cuuint64_t>(kTcMats)};
  const cuuint64_t strides[2] = {static_cast<cuuint64_t>(Tp) * 2,                                 // next stock
                                 static_cast<cuuint64_t>(Np) * static_cast<cuuint64_t>(Tp) * 2};  // next matrix
  const cuuint32_t box[3] = {static_cast<cuuint32_t>(kTcK), static_cast<cuuint32_t>(box_rows),
                             static_cast<cuuint32_t>(kTcMats)};
  const cuuint32_t estr[3] = {1, 1, 1};
  const EncodeTiledFn encode = encode_tiled();
  if (encode == nullptr) return CUDA_ERROR_NOT_SUPPORTED;
  return encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void*>(base), dims, strides, box,
                                estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                                CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
}

cudaError_t launch_corr_bf16x3(const PrecOperands& op, const int2* tiles, int ntiles, int N, int Np, int Tp,
                               double* out, int* status, cudaStream_t s) {
  TcMaps maps;
  if (make_map3(&maps.a, op.h, Np, Tp, kTcM) != CUDA_SUCCESS) return cudaErrorInvalidValue;
  if (make_map3(&maps.b, op.h, Np, Tp, kTcN) != CUDA_SUCCESS) return cudaErrorInvalidValue;
  const size_t smem = prec_tc_smem();
  cudaError_t e = cudaFuncSetAttribute(k_corr_bf16x3, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 0;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  const int grid = ntiles < sms ? ntiles : (sms > 0 ? sms : 1);  // one persistent CTA per SM
  k_corr_bf16x3<<<grid, kTcThreads, smem, s>>>(maps, tiles, ntiles, N, Tp, out, status);
  return cudaGetLastError();
}

cudaError_t launch_corr_fp32(const PrecOperands& op, const int2* tiles, int ntiles, int N, int Tp, double* out,
                             cudaStream_t s) {
  k_corr_fp32<<<ntiles, 256, 0, s>>>(op.x32, op.q32, op.m32, tiles, N, Tp, out);
  return cudaGetLastError();
}

}  // namespace fcb
