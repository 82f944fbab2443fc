// umma_gemm.cu — BF16 TN GEMM on tcgen05 with TMA-staged operands.
//
// One CTA computes a 128 x BN tile of C with 4 warps:
//   warp 0, one lane : TMA producer. Per 64-wide K block it loads the A
//                      tile (128 rows) and the B tile (BN rows), one box of
//                      64 BF16 (128 bytes) x rows each, with the 128-byte
//                      swizzle: shared memory then holds them in the K-major
//                      SWIZZLE_128B canonical layout (rows 128 bytes apart,
//                      8-row groups 1024 bytes apart).
//   warp 1, one lane : MMA issuer. Four tcgen05.mma (K = 16 each) per K
//                      block into one TMEM accumulator of BN FP32 columns;
//                      tcgen05.commit frees the stage for the producer.
//   warps 0-3        : epilogue. After the last commit every thread reads
//                      its accumulator row (TMEM lane = tile row) 16 columns
//                      at a time and applies the fused epilogue.
// A 4-stage ring of mbarriers (full: TMA bytes landed; empty: MMAs that read
// the stage are done) overlaps loads with math. Every wait is bounded: on
// timeout the kernel records an error bit, lets its own copies in flight
// land, frees TMEM and returns.
#include "tc_sm100.cuh"
#include "umma_gemm.h"

#include <mutex>

namespace gtpb {
namespace umma {
namespace {

constexpr int BM = 128, BK = 64, STAGES = 4, THREADS = 128;
// Guard after the last stage.
constexpr int SLACK = 1024;

template <int BN>
struct Cfg {
  static constexpr int A_BYTES = BM * BK * 2;
  static constexpr int B_BYTES = BN * BK * 2;
  static constexpr int STAGE = A_BYTES + B_BYTES;
  static constexpr int TILES = STAGES * STAGE;
  static constexpr int SMEM = 1024 + TILES + SLACK + 256;
  static constexpr uint32_t TMEM_COLS = BN;
};

__device__ __forceinline__ float bf2f(uint16_t b) { return __uint_as_float(static_cast<uint32_t>(b) << 16); }
__device__ __forceinline__ uint16_t f2bf(float x) {
  return __bfloat16_as_ushort(__float2bfloat16_rn(x));
}
__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
  return static_cast<uint32_t>(f2bf(lo)) | (static_cast<uint32_t>(f2bf(hi)) << 16);
}
__device__ __forceinline__ float warp_sum(float x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

// Loads 16 bf16 of one row starting at column n into v (0 past N).
__device__ __forceinline__ void load16_bf16(const uint16_t* row, int n, int N, bool vec, float (&v)[16]) {
  if (vec && n + 16 <= N) {
    const uint4 q0 = *reinterpret_cast<const uint4*>(row + n);
    const uint4 q1 = *reinterpret_cast<const uint4*>(row + n + 8);
    const uint32_t w[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      v[2 * i] = bf2f(static_cast<uint16_t>(w[i] & 0xFFFF));
      v[2 * i + 1] = bf2f(static_cast<uint16_t>(w[i] >> 16));
    }
  } else {
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = (n + i < N) ? bf2f(row[n + i]) : 0.f;
  }
}

template <int BN>
__global__ void __launch_bounds__(THREADS, 1)
    gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, int M, int N,
                int K, Epilogue ep) {
  using C = Cfg<BN>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + C::TILES + SLACK);
  uint64_t* empty = full + STAGES;
  uint64_t* accb = empty + STAGES;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(accb + 1);
  volatile int* abort_v = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  const int nk = (K + BK - 1) / BK;

  if (threadIdx.x == 0) {
    tc::tma_prefetch_desc(&tmA);
    tc::tma_prefetch_desc(&tmB);
    for (int s = 0; s < STAGES; ++s) {
      tc::mbar_init(&full[s], 1);
      tc::mbar_init(&empty[s], 1);
    }
    tc::mbar_init(accb, 1);
    *abort_v = 0;
    tc::mbar_init_fence();
  }
  if (warp == 2) {
    tc::tmem_alloc(tmem_slot, C::TMEM_COLS);
    tc::tmem_relinquish();
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      int issued = 0;
      for (int kb = 0; kb < nk; ++kb) {
        const int s = kb % STAGES;
        if (kb >= STAGES && !tc::mbar_wait(&empty[s], ((kb / STAGES) - 1) & 1, abort_v)) {
          *abort_v = 1;
          if (ep.err) atomicOr(ep.err, 1);
          break;
        }
        uint8_t* a = smem + s * C::STAGE;
        uint8_t* b = a + C::A_BYTES;
        tc::mbar_expect_tx(&full[s], C::STAGE);
        tc::tma_load_2d(a, &tmA, &full[s], kb * BK, m0);
        tc::tma_load_2d(b, &tmB, &full[s], kb * BK, n0);
        issued = kb + 1;
      }
      if (*abort_v) {  // let this CTA's copies in flight land before exit
        for (int kb = issued > STAGES ? issued - STAGES : 0; kb < issued; ++kb)
          tc::mbar_wait(&full[kb % STAGES], (kb / STAGES) & 1, nullptr);
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc = tc::instr_desc_bf16(BM, BN);
      for (int kb = 0; kb < nk; ++kb) {
        const int s = kb % STAGES;
        if (!tc::mbar_wait(&full[s], (kb / STAGES) & 1, abort_v)) {
          *abort_v = 1;
          if (ep.err) atomicOr(ep.err, 1);
          break;
        }
        tc::tc_fence_after();
        const uint32_t a = tc::smem_u32(smem + s * C::STAGE);
        const uint32_t b = a + C::A_BYTES;
#pragma unroll
        for (int j = 0; j < BK / 16; ++j) {  // K = 16 per MMA: 32 bytes along the swizzled row
          const uint64_t da = tc::smem_desc_kmajor_sw128(a + j * 32);
          const uint64_t db = tc::smem_desc_kmajor_sw128(b + j * 32);
          tc::umma_bf16(tmem, da, db, idesc, (kb | j) != 0 ? 1u : 0u);
        }
        tc::umma_commit(&empty[s]);
      }
      tc::umma_commit(accb);  // arrives once every MMA issued above is done
    }
    __syncwarp();
  }

  // ---- epilogue (all four warps) -------------------------------------------
  int acc_ok = 1;
  if (lane == 0) acc_ok = tc::mbar_wait(accb, 0, nullptr) ? 1 : 0;
  acc_ok = __shfl_sync(0xffffffffu, acc_ok, 0);
  tc::tc_fence_after();
  if (!acc_ok) {
    if (lane == 0 && ep.err) atomicOr(ep.err, 1);
  } else if (!*abort_v) {
    const int mode = ep.mode;
    const int row = m0 + warp * 32 + lane;
    const bool row_ok = row < M;
    const uint32_t lane_base = tmem + (static_cast<uint32_t>(warp * 32) << 16);
    const uint16_t* mrow = static_cast<const uint16_t*>(ep.mask) + static_cast<int64_t>(row) * ep.ldm;
    float sq = 0.f;
    for (int c = 0; c < BN; c += 16) {
      const int nb = n0 + c;
      if (nb >= N) break;
      float v[16];
      tc::tmem_ld16(lane_base + static_cast<uint32_t>(c), v);
      float mk[16];
      if (mode & EPI_RELU_BWD) {
        if (row_ok) load16_bf16(mrow, nb, N, true, mk);
        else {
#pragma unroll
          for (int j = 0; j < 16; ++j) mk[j] = 0.f;
        }
      }
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int n = nb + j;
        const bool ok = row_ok && n < N;
        float x = v[j];
        if (mode & EPI_BIAS) x += (n < N) ? ep.bias[n] : 0.f;
        if (mode & EPI_RELU) x = fmaxf(x, 0.f);
        if (mode & EPI_RELU_BWD) x = mk[j] > 0.f ? x : 0.f;
        if (mode & EPI_MSE) {
          if (ok && (mode & EPI_OUT_F32)) ep.out_f[static_cast<int64_t>(row) * ep.ldf + n] = x;
          float g = 0.f;
          if (ok && n < ep.n_valid) {
            g = x - ep.target[static_cast<int64_t>(row) * ep.ldy + n];
            sq += g * g;
          }
          x = g * ep.grad_scale;
        } else if (ok && (mode & EPI_OUT_F32)) {
          ep.out_f[static_cast<int64_t>(row) * ep.ldf + n] = x;
        }
        v[j] = ok ? x : 0.f;
      }
      if ((mode & EPI_OUT_BF16) && row_ok) {
        uint16_t* orow = static_cast<uint16_t*>(ep.out) + static_cast<int64_t>(row) * ep.ldo;
        if (nb + 16 <= N) {
          uint4 q0, q1;
          q0.x = pack2(v[0], v[1]);
          q0.y = pack2(v[2], v[3]);
          q0.z = pack2(v[4], v[5]);
          q0.w = pack2(v[6], v[7]);
          q1.x = pack2(v[8], v[9]);
          q1.y = pack2(v[10], v[11]);
          q1.z = pack2(v[12], v[13]);
          q1.w = pack2(v[14], v[15]);
          *reinterpret_cast<uint4*>(orow + nb) = q0;
          *reinterpret_cast<uint4*>(orow + nb + 8) = q1;
        } else {
          for (int j = 0; j < 16 && nb + j < N; ++j) orow[nb + j] = f2bf(v[j]);
        }
      }
      if ((mode & EPI_OUT_BF16_T) && row_ok) {
        uint16_t* ot = static_cast<uint16_t*>(ep.out_t);
#pragma unroll
        for (int j = 0; j < 16; ++j)
          if (nb + j < N) ot[static_cast<int64_t>(nb + j) * ep.ldt + row] = f2bf(v[j]);
      }
      if (mode & EPI_COLSUM) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const float s = warp_sum(v[j]);
          if (lane == 0 && nb + j < N) atomicAdd(&ep.colsum[nb + j], s);
        }
      }
    }
    if (mode & EPI_MSE) {
      sq = warp_sum(sq);
      if (lane == 0 && ep.loss) atomicAdd(ep.loss, sq);
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 2) {
    tc::tc_fence_after();
    tc::tmem_dealloc(tmem, C::TMEM_COLS);
  }
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

// Tensor map over a row-major bf16 matrix [rows, ld] reading K columns, box
// of 64 columns (128 bytes) by box_rows rows, 128-byte swizzle.
bool make_map(CUtensorMap* map, const Operand& o, int64_t k, int box_rows) {
  EncodeTiledFn fn = encode_fn();
  if (fn == nullptr) return false;
  const cuuint64_t dims[2] = {static_cast<cuuint64_t>(k), static_cast<cuuint64_t>(o.rows)};
  const cuuint64_t strides[1] = {static_cast<cuuint64_t>(o.ld) * 2};
  const cuuint32_t box[2] = {64, static_cast<cuuint32_t>(box_rows)};
  const cuuint32_t estr[2] = {1, 1};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(o.ptr), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

template <int BN>
cudaError_t launch(const CUtensorMap& ma, const CUtensorMap& mb, int m, int n, int k, const Epilogue& ep,
                   cudaStream_t stream) {
  using C = Cfg<BN>;
  static std::once_flag once;
  static cudaError_t attr = cudaSuccess;
  std::call_once(once, [] {
    attr = cudaFuncSetAttribute(gemm_kernel<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM);
  });
  if (attr != cudaSuccess) return attr;
  const dim3 grid((n + BN - 1) / BN, (m + BM - 1) / BM);
  gemm_kernel<BN><<<grid, THREADS, C::SMEM, stream>>>(ma, mb, m, n, k, ep);
  return cudaGetLastError();
}

}  // namespace

cudaError_t gemm_bf16_tn(const Operand& a, const Operand& b, int64_t m, int64_t n, int64_t k, const Epilogue& ep,
                         cudaStream_t stream, int bn) {
  if (m <= 0 || n <= 0 || k < 8 || (k % 8) != 0) return cudaErrorInvalidValue;
  if (m > (int64_t)65535 * BM || n > (int64_t)1 << 24 || k > (int64_t)1 << 30) return cudaErrorInvalidValue;
  if (a.ptr == nullptr || b.ptr == nullptr || !aligned16(a.ptr) || !aligned16(b.ptr)) return cudaErrorInvalidValue;
  if (a.ld < k || b.ld < k || (a.ld % 8) != 0 || (b.ld % 8) != 0) return cudaErrorInvalidValue;
  if (a.rows < m || b.rows < n) return cudaErrorInvalidValue;
  if ((ep.mode & EPI_OUT_BF16) && (ep.out == nullptr || !aligned16(ep.out) || (ep.ldo % 8) != 0 || ep.ldo < n))
    return cudaErrorInvalidValue;
  if ((ep.mode & EPI_OUT_BF16_T) && (ep.out_t == nullptr || ep.ldt < m)) return cudaErrorInvalidValue;
  if ((ep.mode & EPI_OUT_F32) && (ep.out_f == nullptr || ep.ldf < n)) return cudaErrorInvalidValue;
  if ((ep.mode & EPI_RELU_BWD) && (ep.mask == nullptr || !aligned16(ep.mask) || (ep.ldm % 8) != 0 || ep.ldm < n))
    return cudaErrorInvalidValue;
  if ((ep.mode & EPI_MSE) && (ep.target == nullptr || ep.ldy < ep.n_valid || ep.n_valid > n))
    return cudaErrorInvalidValue;
  if ((ep.mode & EPI_BIAS) && ep.bias == nullptr) return cudaErrorInvalidValue;
  if ((ep.mode & EPI_COLSUM) && ep.colsum == nullptr) return cudaErrorInvalidValue;
  if (bn == 0) bn = n <= 64 ? 64 : (n <= 128 ? 128 : 256);
  if (bn != 64 && bn != 128 && bn != 256) return cudaErrorInvalidValue;
  CUtensorMap ma, mb;
  if (!make_map(&ma, a, k, BM) || !make_map(&mb, b, k, bn)) return cudaErrorInvalidValue;
  if (bn == 64) return launch<64>(ma, mb, static_cast<int>(m), static_cast<int>(n), static_cast<int>(k), ep, stream);
  if (bn == 128) return launch<128>(ma, mb, static_cast<int>(m), static_cast<int>(n), static_cast<int>(k), ep, stream);
  return launch<256>(ma, mb, static_cast<int>(m), static_cast<int>(n), static_cast<int>(k), ep, stream);
}

}  // namespace umma
}  // namespace gtpb
