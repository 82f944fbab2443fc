// umma_gemm.cu — BF16 TN GEMM on tcgen05 with TMA-staged operands.
//
// Persistent: one CTA per SM takes 128 x BN tiles of C in turn, with 6 warps:
//   warp 0, one lane : TMA producer. Per 64-wide K block it loads the A
//                      tile (128 rows) and the B tile (BN rows), one box of
//                      64 BF16 (128 bytes) x rows each, with the 128-byte
//                      swizzle: shared memory then holds them in the K-major
//                      SWIZZLE_128B canonical layout (rows 128 bytes apart,
//                      8-row groups 1024 bytes apart).
//   warp 1, one lane : MMA issuer. Four tcgen05.mma (K = 16 each) per K
//                      block into one of two TMEM accumulators of BN FP32
//                      columns (alternating by tile); tcgen05.commit frees the
//                      stage for the producer and, after a tile's last block,
//                      hands the accumulator to the epilogue.
//   warps 2-5        : epilogue. Warp w reads TMEM lanes (w % 4) * 32 .. +31
//                      (the tile's rows) 16 columns at a time, applies the
//                      fused epilogue and returns the accumulator, so that
//                      the next tile's MMAs overlap this tile's stores.
// A 4-stage ring of mbarriers (full: TMA bytes landed; empty: MMAs that read
// the stage are done) overlaps loads with math. Every wait is bounded (by
// Epilogue::spin_limit): on timeout the kernel records an error bit; before
// it returns, the producer waits for the copies it issued to land and the
// MMA issuer for the MMAs it issued to finish, so that neither shared memory
// nor TMEM (freed last) is released under work in flight.
#include "tc_sm100.cuh"
#include "umma_gemm.h"

#include <algorithm>
#include <mutex>

namespace gtpb {
namespace umma {
namespace {

constexpr int BM = 128, BK = 64, STAGES = 4;
constexpr int EPI_WARPS = 4;                    // one per TMEM lane quarter
constexpr int THREADS = 32 * (2 + EPI_WARPS);   // producer, MMA issuer, epilogue
// Guard after the last stage.
constexpr int SLACK = 1024;

template <int BN>
struct Cfg {
  static constexpr int A_BYTES = BM * BK * 2;
  static constexpr int B_BYTES = BN * BK * 2;
  static constexpr int STAGE = A_BYTES + B_BYTES;
  static constexpr int TILES = STAGES * STAGE;
  // per epilogue warp: one 32-row x 64-column BF16 box staged for a TMA
  // store (128-byte swizzle, 1024-byte aligned), after the barriers
  static constexpr int STG_OFF = TILES + SLACK + 1024;
  static constexpr int STG_BYTES = EPI_WARPS * 32 * 128;
  static constexpr int SMEM = 1024 + STG_OFF + STG_BYTES;
  static constexpr uint32_t TMEM_COLS = 2 * BN;  // two accumulators: the epilogue of one tile
                                                 // overlaps the MMAs of the next
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
    gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                const __grid_constant__ CUtensorMap tmC, int M, int N, int K, Epilogue ep) {
  using C = Cfg<BN>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + C::TILES + SLACK);
  uint64_t* empty = full + STAGES;
  uint64_t* acc_full = empty + STAGES;   // [2] accumulator ready for the epilogue
  uint64_t* acc_empty = acc_full + 2;    // [2] accumulator drained by the epilogue
  uint64_t* mma_done = acc_empty + 2;    // every MMA this CTA issued is complete
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mma_done + 1);
  volatile int* abort_v = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nk = (K + BK - 1) / BK;
  const int tiles_n = (N + BN - 1) / BN;
  const int n_tiles = ((M + BM - 1) / BM) * tiles_n;
  const long long spin = ep.spin_limit > 0 ? ep.spin_limit : tc::kSpinLimit;

  if (threadIdx.x == 0) {
    tc::tma_prefetch_desc(&tmA);
    tc::tma_prefetch_desc(&tmB);
    if (ep.tma_store) tc::tma_prefetch_desc(&tmC);
    for (int s = 0; s < STAGES; ++s) {
      tc::mbar_init(&full[s], 1);
      tc::mbar_init(&empty[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
      tc::mbar_init(&acc_full[a], 1);
      tc::mbar_init(&acc_empty[a], EPI_WARPS);
    }
    tc::mbar_init(mma_done, 1);
    *abort_v = 0;
    tc::mbar_init_fence();
  }
  if (warp == 1) {
    tc::tmem_alloc(tmem_slot, C::TMEM_COLS);
    tc::tmem_relinquish();
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    // TMA producer: one stage ring across all of this CTA's tiles
    if (lane == 0) {
      const int64_t skip = blockIdx.x == 0 ? ep.skip_load_block : -1;
      int64_t g = 0;
      for (int t = blockIdx.x; t < n_tiles && !*abort_v; t += gridDim.x) {
        const int m0 = (t / tiles_n) * BM, n0 = (t % tiles_n) * BN;
        for (int kb = 0; kb < nk; ++kb, ++g) {
          const int s = static_cast<int>(g % STAGES);
          if (g >= STAGES &&
              !tc::mbar_wait(&empty[s], static_cast<uint32_t>(((g / STAGES) - 1) & 1), abort_v, spin)) {
            *abort_v = 1;
            if (ep.err) atomicOr(ep.err, 1);
            break;
          }
          if (g == skip) continue;  // timeout-path test: this stage's bytes never arrive
          uint8_t* a = smem + s * C::STAGE;
          uint8_t* b = a + C::A_BYTES;
          tc::mbar_expect_tx(&full[s], C::STAGE);
          tc::tma_load_2d(a, &tmA, &full[s], kb * BK, m0);
          tc::tma_load_2d(b, &tmB, &full[s], kb * BK, n0);
        }
        if (*abort_v) break;
      }
      // the last copies issued (one per stage at most) must land before the
      // CTA exits; consumed stages pass at once
      for (int64_t q = g > STAGES ? g - STAGES : 0; q < g; ++q)
        if (q != skip) tc::mbar_wait(&full[q % STAGES], static_cast<uint32_t>((q / STAGES) & 1), nullptr, spin);
    }
    __syncwarp();
  } else if (warp == 1) {
    // MMA issuer: accumulator i & 1 for this CTA's i-th tile
    if (lane == 0) {
      const uint32_t idesc = tc::instr_desc_bf16(BM, BN);
      int64_t g = 0;
      int i = 0;
      for (int t = blockIdx.x; t < n_tiles; t += gridDim.x, ++i) {
        const int acc = i & 1;
        const uint32_t d = tmem + static_cast<uint32_t>(acc * BN);
        bool ok = !*abort_v;
        if (ok && i >= 2 &&
            !tc::mbar_wait(&acc_empty[acc], static_cast<uint32_t>(((i / 2) - 1) & 1), abort_v, spin))
          ok = false;
        for (int kb = 0; ok && kb < nk; ++kb, ++g) {
          const int s = static_cast<int>(g % STAGES);
          if (!tc::mbar_wait(&full[s], static_cast<uint32_t>((g / STAGES) & 1), abort_v, spin)) {
            ok = false;
            break;
          }
          tc::tc_fence_after();
          const uint32_t a = tc::smem_u32(smem + s * C::STAGE);
          const uint32_t b = a + C::A_BYTES;
#pragma unroll
          for (int j = 0; j < BK / 16; ++j) {  // K = 16 per MMA: 32 bytes along the swizzled row
            const uint64_t da = tc::smem_desc_kmajor_sw128(a + j * 32);
            const uint64_t db = tc::smem_desc_kmajor_sw128(b + j * 32);
            tc::umma_bf16(d, da, db, idesc, (kb | j) != 0 ? 1u : 0u);
          }
          tc::umma_commit(&empty[s]);
        }
        tc::umma_commit(&acc_full[acc]);  // arrives once every MMA issued so far is done
        if (!ok) {
          *abort_v = 1;
          if (ep.err) atomicOr(ep.err, 1);
          break;
        }
      }
      // TMEM is freed only after every MMA issued here is complete
      tc::umma_commit(mma_done);
      if (!tc::mbar_wait(mma_done, 0u, nullptr, spin) && ep.err) atomicOr(ep.err, 1);
    }
    __syncwarp();
  } else {
    // epilogue warps: warp w reads TMEM lanes (w % 4) * 32 ..., i.e. tile rows
    const int quarter = warp & 3;
    uint8_t* stg = smem + C::STG_OFF + quarter * (32 * 128);   // this warp's staged box
    int i = 0;
    for (int t = blockIdx.x; t < n_tiles; t += gridDim.x, ++i) {
      const int acc = i & 1;
      int acc_ok = 1;
      if (lane == 0) acc_ok = tc::mbar_wait(&acc_full[acc], static_cast<uint32_t>((i / 2) & 1), nullptr, spin) ? 1 : 0;
      acc_ok = __shfl_sync(0xffffffffu, acc_ok, 0);
      tc::tc_fence_after();
      if (!acc_ok) {
        if (lane == 0 && ep.err) atomicOr(ep.err, 1);
        break;
      }
      if (*abort_v) break;
      const int m0 = (t / tiles_n) * BM, n0 = (t % tiles_n) * BN;
      const int mode = ep.mode;
      const int row = m0 + quarter * 32 + lane;
      const bool row_ok = row < M;
      const uint32_t lane_base = tmem + static_cast<uint32_t>(acc * BN) + (static_cast<uint32_t>(quarter * 32) << 16);
      const uint16_t* mrow = static_cast<const uint16_t*>(ep.mask) + static_cast<int64_t>(row) * ep.ldm;
      float sq = 0.f;
      // one 16-column chunk of this thread's row, from registers
      auto chunk = [&](float (&v)[16], const int nb) {
        // the chunk's bias: four 16-byte loads when it lies whole and aligned
        float bv[16];
        if (mode & EPI_BIAS) {
          if (nb + 16 <= N && (reinterpret_cast<uintptr_t>(ep.bias + nb) & 15) == 0) {
            const float4* b4 = reinterpret_cast<const float4*>(ep.bias + nb);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              const float4 w = __ldg(b4 + q);
              bv[4 * q + 0] = w.x; bv[4 * q + 1] = w.y; bv[4 * q + 2] = w.z; bv[4 * q + 3] = w.w;
            }
          } else {
#pragma unroll
            for (int j = 0; j < 16; ++j) bv[j] = (nb + j < N) ? ep.bias[nb + j] : 0.f;
          }
        }
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
          if (mode & EPI_BIAS) x += bv[j];
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
          }
          v[j] = ok ? x : 0.f;
        }
        // the FP32 output (outside the MSE mode, which stores it above):
        // four 16-byte stores when the chunk lies whole and aligned
        if ((mode & EPI_OUT_F32) && !(mode & EPI_MSE) && row_ok) {
          float* frow = ep.out_f + static_cast<int64_t>(row) * ep.ldf;
          if (nb + 16 <= N && (reinterpret_cast<uintptr_t>(frow + nb) & 15) == 0) {
#pragma unroll
            for (int q = 0; q < 4; ++q)
              *reinterpret_cast<float4*>(frow + nb + 4 * q) = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
          } else {
#pragma unroll
            for (int j = 0; j < 16; ++j)
              if (nb + j < N) frow[nb + j] = v[j];
          }
        }
        if ((mode & EPI_OUT_BF16) && row_ok && !ep.tma_store) {
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
#pragma unroll
            for (int j = 0; j < 16; ++j)
              if (nb + j < N) orow[nb + j] = f2bf(v[j]);
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
      };
      // the forward modes read 64 columns per TMEM round trip (four loads in
      // flight, one wait); the others 16
      const bool wide = (mode & (EPI_MSE | EPI_RELU_BWD | EPI_OUT_BF16_T | EPI_COLSUM)) == 0;
      for (int c = 0; c < BN;) {
        const int nb = n0 + c;
        if (nb >= N) break;
        if (wide && c + 64 <= BN) {
          uint32_t r[4][16];
#pragma unroll
          for (int q = 0; q < 4; ++q) tc::tmem_ld16_nowait(lane_base + static_cast<uint32_t>(c + 16 * q), r[q]);
          tc::tmem_wait_ld();
          if (ep.tma_store) {
            // the staged box is free once the previous store has read it
            if (lane == 0) tc::bulk_wait_read();
            __syncwarp();
          }
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            if (nb + 16 * q >= N) break;
            float v[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[q][j]);
            chunk(v, nb + 16 * q);
            if (ep.tma_store) {
              // this row's 16-byte pieces 2q, 2q + 1 of 8, at their 128-byte
              // swizzle positions (piece ^ (row & 7))
              uint8_t* srow = stg + lane * 128;
              const uint4 q0 = make_uint4(pack2(v[0], v[1]), pack2(v[2], v[3]), pack2(v[4], v[5]), pack2(v[6], v[7]));
              const uint4 q1 =
                  make_uint4(pack2(v[8], v[9]), pack2(v[10], v[11]), pack2(v[12], v[13]), pack2(v[14], v[15]));
              *reinterpret_cast<uint4*>(srow + (((2 * q) ^ (lane & 7)) << 4)) = q0;
              *reinterpret_cast<uint4*>(srow + (((2 * q + 1) ^ (lane & 7)) << 4)) = q1;
            }
          }
          if (ep.tma_store) {
            tc::fence_proxy_async_smem();
            __syncwarp();
            if (lane == 0 && m0 + quarter * 32 < M) {   // rows past M are clipped; a box wholly past them is skipped
              tc::tma_store_2d(&tmC, stg, nb, m0 + quarter * 32);
              tc::bulk_commit();
            }
          }
          c += 64;
        } else {
          float v[16];
          tc::tmem_ld16(lane_base + static_cast<uint32_t>(c), v);
          chunk(v, nb);
          c += 16;
        }
      }
      if (mode & EPI_MSE) {
        sq = warp_sum(sq);
        if (lane == 0 && ep.loss) atomicAdd(ep.loss, sq);
      }
      // hand the accumulator back to the MMA issuer
      tc::tc_fence_before();
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&acc_empty[acc]);
    }
    // this warp's stores are complete before the CTA ends
    if (ep.tma_store && lane == 0) tc::bulk_wait_all();
    __syncwarp();
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 1) {
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
cudaError_t launch(const CUtensorMap& ma, const CUtensorMap& mb, const CUtensorMap& mc, int m, int n, int k,
                   const Epilogue& ep, cudaStream_t stream) {
  using C = Cfg<BN>;
  static std::once_flag once;
  static cudaError_t attr = cudaSuccess;
  std::call_once(once, [] {
    attr = cudaFuncSetAttribute(gemm_kernel<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM);
  });
  if (attr != cudaSuccess) return attr;
  static int sms = 0;
  if (sms == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
  }
  const int64_t tiles = ((m + BM - 1) / BM) * ((n + BN - 1) / BN);
  const int grid = static_cast<int>(std::min<int64_t>(tiles, sms));  // persistent: one CTA per SM
  gemm_kernel<BN><<<grid, THREADS, C::SMEM, stream>>>(ma, mb, mc, m, n, k, ep);
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
  CUtensorMap ma, mb, mc;
  if (!make_map(&ma, a, k, BM) || !make_map(&mb, b, k, bn)) return cudaErrorInvalidValue;
  // a forward epilogue writing out[] only stores 32 x 64 boxes by TMA
  Epilogue e2 = ep;
  e2.tma_store = 0;
  mc = ma;
  if ((ep.mode & EPI_OUT_BF16) && !(ep.mode & (EPI_MSE | EPI_RELU_BWD | EPI_OUT_BF16_T | EPI_COLSUM))) {
    Operand o;
    o.ptr = ep.out;
    o.rows = m;
    o.ld = ep.ldo;
    if (make_map(&mc, o, n, 32)) e2.tma_store = 1;
    else mc = ma;
  }
  if (bn == 64) return launch<64>(ma, mb, mc, static_cast<int>(m), static_cast<int>(n), static_cast<int>(k), e2, stream);
  if (bn == 128)
    return launch<128>(ma, mb, mc, static_cast<int>(m), static_cast<int>(n), static_cast<int>(k), e2, stream);
  return launch<256>(ma, mb, mc, static_cast<int>(m), static_cast<int>(n), static_cast<int>(k), e2, stream);
}

}  // namespace umma
}  // namespace gtpb
