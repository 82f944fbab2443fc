// umma_gemm.h — BF16 GEMM on the sm_100a tensor cores (tcgen05.mma with a
// TMEM accumulator, operands staged by TMA) with the epilogues the power
// proxy network needs.
//
//   C[M, N] = A[M, K] * B[N, K]^T      (both operands K-major, bf16)
//
// followed per element by, in order: + bias[n]; ReLU; ReLU backward
// (keep where mask[m, n] > 0); mean-squared-error gradient against
// target[m, n] (writes the prediction to out_f32 and replaces the value by
// grad_scale * (pred - target) for n < n_valid, 0 beyond); then the stores
// the mode selects and the per-column sum.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace gtpb {
namespace umma {

enum EpiFlags : int {
  EPI_BIAS = 1,
  EPI_RELU = 2,
  EPI_RELU_BWD = 4,
  EPI_MSE = 8,
  EPI_OUT_BF16 = 16,    // out[m * ldo + n]
  EPI_OUT_BF16_T = 32,  // out_t[n * ldt + m]
  EPI_OUT_F32 = 64,     // out_f[m * ldf + n] (the prediction under EPI_MSE)
  EPI_COLSUM = 128,     // colsum[n] += sum over rows m < M
};

struct Epilogue {
  int mode = 0;
  const float* bias = nullptr;
  void* out = nullptr;  // bf16
  int64_t ldo = 0;
  void* out_t = nullptr;  // bf16
  int64_t ldt = 0;
  float* out_f = nullptr;
  int64_t ldf = 0;
  const void* mask = nullptr;  // bf16
  int64_t ldm = 0;
  const float* target = nullptr;
  int64_t ldy = 0;
  int n_valid = 0;
  float grad_scale = 0.f;
  float* colsum = nullptr;
  float* loss = nullptr;  // += sum of squared errors under EPI_MSE
  int* err = nullptr;     // bit 1: a pipeline wait timed out
  // longest spin of one pipeline wait, SM clock cycles; 0 = about one second
  long long spin_limit = 0;
  // test of the timeout path, -1 in normal use: the first CTA's TMA producer
  // skips the loads of its k-th K block (counted over its tiles), so the MMA
  // issuer's wait for them runs out after spin_limit
  int skip_load_block = -1;
  // set by gemm_bf16_tn: the BF16 output goes out by TMA stores of staged
  // 32-row x 64-column boxes (forward modes writing out[] only)
  int tma_store = 0;
};

// Row-major bf16 matrix [rows, ld] whose first `k` columns are the K extent.
struct Operand {
  const void* ptr = nullptr;
  int64_t rows = 0;
  int64_t ld = 0;
};

// Validates shapes and alignment (K % 8 == 0, ld % 8 == 0, 16-byte aligned
// bases and vector stores) and launches. Returns cudaErrorInvalidValue on a
// shape the kernel does not take. bn = 64, 128 or 256 (0: by N).
cudaError_t gemm_bf16_tn(const Operand& a, const Operand& b, int64_t m, int64_t n, int64_t k,
                         const Epilogue& ep, cudaStream_t stream, int bn = 0);

}  // namespace umma
}  // namespace gtpb
