// cdf_model.h -- internal layout of the learned-splitter model handle.
#pragma once

#include <cstddef>
#include <cuda_runtime.h>

#include "../../include/fcb200.h"

// One CDF network per factor (parameters + Adam state), the training samples
// of the last fit, and two table slots: rank kernels read slot `cur` while a
// background refit writes the other one.
struct fcb_cdf_model {
  int F = 0;
  int device = -1;
  int linear = 0;           // 1: tabulate a linear ramp instead of the network
  int steps_done = 0;
  int nsamp = 0;            // samples per factor of the last fit
  size_t samp_cap = 0;      // allocated samples per factor
  int cur = 0;              // table slot the rank kernels read
  float* params = nullptr;  // (F, P)
  float* adam = nullptr;    // (F, 2P)
  float* table[2] = {nullptr, nullptr};   // (F, K) per slot
  float* zrange[2] = {nullptr, nullptr};  // (F, 2) per slot
  float* loss = nullptr;    // (F)
  float2* samples = nullptr;
};

namespace fcb {
// Extract training samples from exact ranks (stream-ordered after the kernel
// that produced them).
cudaError_t cdf_model_features(fcb_cdf_model* m, const float* d_x, const float* d_ranks, int T, int N, int t0,
                               int tcount, cudaStream_t s);
// Adam steps on the extracted samples, then tabulate into table slot `slot`.
cudaError_t cdf_model_train_tabulate(fcb_cdf_model* m, int steps, float lr, int slot, cudaStream_t s);
// Learned rank + IC with an explicit IC row stride (ic_ld = 0: T).
int rank_ic_learned_ld(const float* d_x, const float* d_r, const uint8_t* d_fmask, const uint8_t* d_rmask, int F,
                       int T, int N, int min_valid, float* d_ranks, double* d_ic, int ic_ld,
                       const fcb_cdf_model* model, int cap, int* d_stats, cudaStream_t stream);
}  // namespace fcb
