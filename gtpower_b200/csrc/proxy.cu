// proxy.cu — the learned per-cycle power proxy of include/gtpb200_proxy.h:
// a 3-layer BF16 MLP trained and evaluated with the tcgen05 GEMM of
// umma_gemm.cu, Adam on FP32 master weights, and the feature kernels that
// read the engine's per-net event CSR.
//
// One training step (all on the proxy's stream; replayed from a CUDA graph
// by gtp_proxy_train):
//   begin     : step counters, zero bias gradients and the step loss
//   gather    : minibatch rows -> Xb [B][I], XbT [I][B], standardised Tb
//   L1        : H1 = relu(Xb W1^T + b1)        -> H1, H1^T   (bf16)
//   L2        : H2 = relu(H1 W2^T + b2)        -> H2, H2^T
//   L3 + loss : Y = H2 W3^T + b3; dY = 2/(B*O) (Y - T); sum (Y - T)^2
//               -> dY, dY^T (bf16), db3 = column sums of dY
//   dW3       = dY^T H2     (A = dY^T [O'][B], B = H2^T [H][B])
//   dH2       = (dY W3) * [H2 > 0]   (A = dY [B][O'], B = W3^T [H][O'])
//               -> dH2, dH2^T, db2
//   dW2       = dH2^T H1
//   dH1       = (dH2 W2) * [H1 > 0] -> dH1^T, db1
//   dW1       = dH1^T Xb    (B = Xb^T [I][B])
//   adam      : FP32 masters, moments; republishes W1, W2, W2^T, W3, W3^T
// O' = n_out rounded up to 8 (the K extent of dY); its padding rows of W3
// and b3 stay zero because their gradients are zero.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <random>
#include <string>
#include <vector>

#include <cuda_bf16.h>

#include "../../include/gtpb200_proxy.h"
#include "umma_gemm.h"

using gtpb::umma::Epilogue;
using gtpb::umma::Operand;
namespace U = gtpb::umma;

namespace {

__device__ __forceinline__ uint16_t f2bf(float x) { return __bfloat16_as_ushort(__float2bfloat16_rn(x)); }

__host__ __device__ inline uint64_t mix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

struct Layout {  // offsets of the internal (padded) parameter vector
  int I, H, O, Op;
  int64_t oW1, ob1, oW2, ob2, oW3, ob3, n;
  int64_t user_n;
  void set(int i, int h, int o) {
    I = i;
    H = h;
    O = o;
    Op = (o + 7) / 8 * 8;
    oW1 = 0;
    ob1 = oW1 + (int64_t)H * I;
    oW2 = ob1 + H;
    ob2 = oW2 + (int64_t)H * H;
    oW3 = ob2 + H;
    ob3 = oW3 + (int64_t)Op * H;
    n = ob3 + Op;
    user_n = (int64_t)H * I + H + (int64_t)H * H + H + (int64_t)O * H + O;
  }
};

// ---- kernels ----------------------------------------------------------------

// He-uniform weights (bound sqrt(6 / fan_in)), zero biases, zero padding.
__global__ void init_params_kernel(float* p, Layout L, uint64_t seed) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < L.n; i += (int64_t)gridDim.x * blockDim.x) {
    float fan_in = 0.f;
    bool w = false;
    if (i < L.ob1) {
      fan_in = (float)L.I;
      w = true;
    } else if (i >= L.oW2 && i < L.ob2) {
      fan_in = (float)L.H;
      w = true;
    } else if (i >= L.oW3 && i < L.ob3) {
      w = ((i - L.oW3) / L.H) < L.O;
      fan_in = (float)L.H;
    }
    float v = 0.f;
    if (w) {
      const uint64_t h = mix64(seed ^ mix64((uint64_t)i));
      const float u = (float)((h >> 40) * (1.0 / 16777216.0));  // [0, 1)
      v = (2.f * u - 1.f) * sqrtf(6.f / fan_in);
    }
    p[i] = v;
  }
}

struct Publish {
  uint16_t *W1, *W2, *W2t, *W3, *W3t;
};

__device__ __forceinline__ void publish_one(const Layout& L, const Publish& P, int64_t i, float v) {
  const uint16_t b = f2bf(v);
  if (i < L.ob1) {
    P.W1[i] = b;
  } else if (i >= L.oW2 && i < L.ob2) {
    const int64_t j = i - L.oW2;
    const int64_t r = j / L.H, c = j % L.H;
    P.W2[j] = b;
    P.W2t[c * L.H + r] = b;
  } else if (i >= L.oW3 && i < L.ob3) {
    const int64_t j = i - L.oW3;
    const int64_t r = j / L.H, c = j % L.H;
    P.W3[j] = b;
    P.W3t[c * L.Op + r] = b;
  }
}

__global__ void publish_kernel(const float* p, Layout L, Publish P) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < L.n; i += (int64_t)gridDim.x * blockDim.x)
    publish_one(L, P, i, p[i]);
}

// counters: [0] Adam steps taken including the current one, [1] minibatch
// index of this step, [2] next minibatch index within the epoch.
__global__ void begin_step_kernel(int64_t* counters, float* grad, Layout L, float* loss_step) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    counters[0] += 1;
    counters[1] = counters[2];
    counters[2] += 1;
    *loss_step = 0.f;
  }
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < L.H; i += gridDim.x * blockDim.x) {
    grad[L.ob1 + i] = 0.f;
    grad[L.ob2 + i] = 0.f;
  }
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < L.Op; i += gridDim.x * blockDim.x) grad[L.ob3 + i] = 0.f;
}

// Minibatch gather. Block (x, y) copies features [64x, 64x+64) of batch rows
// [32y, 32y+32) into Xb and, through a shared tile, into XbT; blocks with
// x == 0 also write the standardised targets.
__global__ void __launch_bounds__(256) gather_kernel(const uint16_t* X, const float* Y, const int32_t* idx_base,
                                                     const int64_t* counters, int B, Layout L, const float* mean,
                                                     const float* inv_std, uint16_t* Xb, uint16_t* XbT, float* Tb) {
  __shared__ uint16_t tile[32][66];
  const int r0 = blockIdx.y * 32, f0 = blockIdx.x * 64;
  const int32_t* idx = counters ? idx_base + counters[1] * (int64_t)B : idx_base;
  for (int e = threadIdx.x; e < 32 * 32; e += 256) {
    const int r = e >> 5, cp = e & 31;
    const int64_t src = idx[r0 + r];
    const uint32_t w = *reinterpret_cast<const uint32_t*>(X + src * L.I + f0 + 2 * cp);
    *reinterpret_cast<uint32_t*>(Xb + (int64_t)(r0 + r) * L.I + f0 + 2 * cp) = w;
    tile[r][2 * cp] = (uint16_t)(w & 0xFFFF);
    tile[r][2 * cp + 1] = (uint16_t)(w >> 16);
  }
  __syncthreads();
  for (int e = threadIdx.x; e < 64 * 32; e += 256) {
    const int f = e >> 5, r = e & 31;
    XbT[(int64_t)(f0 + f) * B + r0 + r] = tile[r][f];
  }
  if (blockIdx.x == 0) {
    for (int e = threadIdx.x; e < 32 * L.Op; e += 256) {
      const int r = e / L.Op, o = e % L.Op;
      const int64_t src = idx[r0 + r];
      Tb[(int64_t)(r0 + r) * L.Op + o] = o < L.O ? (Y[src * L.O + o] - mean[o]) * inv_std[o] : 0.f;
    }
  }
}

struct AdamArgs {
  float *p, *m, *v;
  const float* g;
  Layout L;
  Publish P;
  float lr, b1, b2, eps, wd;
  int64_t* counters;
  const float* loss_step;
  float* loss_epoch;
  float loss_norm;
};

__global__ void adam_kernel(AdamArgs a) {
  const int64_t t = a.counters[0];  // advanced by an earlier kernel of the step
  const float bc1 = 1.f - powf(a.b1, (float)t);
  const float bc2 = 1.f - powf(a.b2, (float)t);
  const Layout& L = a.L;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < L.n; i += (int64_t)gridDim.x * blockDim.x) {
    const float g = a.g[i];
    const float m = a.b1 * a.m[i] + (1.f - a.b1) * g;
    const float v = a.b2 * a.v[i] + (1.f - a.b2) * g * g;
    a.m[i] = m;
    a.v[i] = v;
    float p = a.p[i];
    const bool is_w = i < L.ob1 || (i >= L.oW2 && i < L.ob2) || (i >= L.oW3 && i < L.ob3);
    if (is_w && a.wd > 0.f) p -= a.lr * a.wd * p;
    p -= a.lr * (m / bc1) / (sqrtf(v / bc2) + a.eps);
    a.p[i] = p;
    publish_one(L, a.P, i, p);
  }
  if (a.loss_epoch && blockIdx.x == 0 && threadIdx.x == 0) *a.loss_epoch += *a.loss_step * a.loss_norm;
}

__global__ void bump_kernel(int64_t* counters) { counters[0] += 1; }

// Per-output mean and 1/std of Y [n][O] in FP64; one block per output.
__global__ void colstats_kernel(const float* Y, int64_t n, int O, float* mean, float* inv_std, float* stdv) {
  __shared__ double s1[256], s2[256];
  const int o = blockIdx.x;
  double a = 0, b = 0;
  for (int64_t r = threadIdx.x; r < n; r += blockDim.x) {
    const double y = Y[r * O + o];
    a += y;
    b += y * y;
  }
  s1[threadIdx.x] = a;
  s2[threadIdx.x] = b;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      s1[threadIdx.x] += s1[threadIdx.x + w];
      s2[threadIdx.x] += s2[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double mu = s1[0] / (double)n;
    const double var = fmax(s2[0] / (double)n - mu * mu, 0.0);
    double sd = sqrt(var);
    if (!(sd > 1e-12 * fabs(mu)) || sd == 0.0) sd = fabs(mu) > 0 ? fabs(mu) : 1.0;
    mean[o] = (float)mu;
    stdv[o] = (float)sd;
    inv_std[o] = (float)(1.0 / sd);
  }
}

__global__ void denorm_kernel(const float* py, int64_t n, int O, int Op, const float* mean, const float* stdv,
                              float* y) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n * O; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = i / O;
    const int o = (int)(i % O);
    y[i] = py[r * Op + o] * stdv[o] + mean[o];
  }
}

// floor(t / tpc) for 0 < t < 2^63 with magic = ceil(2^64 / tpc) (0 for
// tpc == 1): umulhi(t, magic) is the quotient or one more.
__device__ __forceinline__ int64_t cycle_of(int64_t t, int64_t tpc, uint64_t magic) {
  if (magic == 0u) return t;
  uint64_t q = __umul64hi(static_cast<uint64_t>(t), magic);
  if (q * static_cast<uint64_t>(tpc) > static_cast<uint64_t>(t)) --q;
  return static_cast<int64_t>(q);
}

uint64_t cycle_magic(int64_t tpc) {
  if (tpc < 2) return 0u;
  const unsigned __int128 one = static_cast<unsigned __int128>(1) << 64;
  return static_cast<uint64_t>(one / static_cast<uint64_t>(tpc) + (one % static_cast<uint64_t>(tpc) != 0));
}

// One warp per selected net.
__global__ void toggle_bits_kernel(const int64_t* off, const int64_t* time, const int32_t* sel, int n_sel,
                                   int64_t tpc, uint64_t magic, int64_t c_lo, int64_t c_hi, uint16_t* x, int64_t ld) {
  const int64_t wid = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (wid >= n_sel) return;
  const int32_t net = sel[wid];
  const int64_t b = off[net], e = off[net + 1];
  for (int64_t i = b + lane; i < e; i += 32) {
    const int64_t t = time[i];
    if (t <= 0) continue;
    const int64_t c = cycle_of(t, tpc, magic);
    if (c < c_lo || c >= c_hi) continue;
    x[(c - c_lo) * ld + wid] = 0x3F80;  // 1.0 in BF16
  }
}

// Dense toggle bits of many windows (gtp_toggle_bits_windows). Block (x, y):
// nets sel[64x .. 64x + 63] over row chunk y (window w, up to kBitsRows
// cycles). 64-bit masks are built with shared atomics, then each warp writes
// whole rows of 64 BF16 entries (128 B).
constexpr int kBitsRows = 2048;
constexpr int kBitsNets = 64;

struct BitsLaunch {
  gtp_bits_window w[GTP_BITS_MAX_WINDOWS];
  int32_t chunk0[GTP_BITS_MAX_WINDOWS + 1];  // first row chunk of each window
  int32_t n_win;
  int32_t pad;
};

__global__ void __launch_bounds__(256) toggle_bits_windows_kernel(const __grid_constant__ BitsLaunch L,
                                                                  const int32_t* __restrict__ sel, int n_sel,
                                                                  int64_t tpc, uint64_t magic, int64_t c_base,
                                                                  uint16_t* __restrict__ x, int64_t ld) {
  __shared__ unsigned long long bits[kBitsRows];
  const int ch = blockIdx.y;
  int wi = 0;
  while (wi + 1 < L.n_win && L.chunk0[wi + 1] <= ch) ++wi;
  const gtp_bits_window& win = L.w[wi];
  const int64_t r_lo = win.c_lo + static_cast<int64_t>(ch - L.chunk0[wi]) * kBitsRows;
  const int64_t r_hi = min(win.c_hi, r_lo + kBitsRows);
  const int rows = static_cast<int>(r_hi - r_lo);
  const int k0 = blockIdx.x * kBitsNets;
  for (int r = threadIdx.x; r < rows; r += blockDim.x) bits[r] = 0ull;
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int j = warp; j < kBitsNets && k0 + j < n_sel; j += nw) {
    const int32_t net = __ldg(sel + k0 + j);
    const int64_t b = __ldg(win.d_net_off + net), e = __ldg(win.d_net_off + net + 1);
    for (int64_t i = b + lane; i < e; i += 32) {
      const int64_t t = __ldg(win.d_time + i);
      if (t <= 0) continue;
      const int64_t c = cycle_of(t, tpc, magic);
      if (c >= r_hi) break;  // a lane's later events are later still
      if (c >= r_lo) atomicOr(bits + (c - r_lo), 1ull << j);
    }
  }
  __syncthreads();
  // a warp writes one row: lane l holds entries 2l and 2l + 1
  const int kc = k0 + 2 * lane;
  const bool pairs = (ld & 1) == 0 && (reinterpret_cast<uintptr_t>(x) & 3) == 0;
  for (int r = warp; r < rows; r += nw) {
    const unsigned long long m = bits[r];
    uint16_t* row = x + (r_lo + r - c_base) * ld;
    const uint16_t v0 = ((m >> (2 * lane)) & 1ull) ? 0x3F80 : 0, v1 = ((m >> (2 * lane + 1)) & 1ull) ? 0x3F80 : 0;
    if (kc + 1 < n_sel && pairs) {
      *reinterpret_cast<uint32_t*>(row + kc) = static_cast<uint32_t>(v0) | (static_cast<uint32_t>(v1) << 16);
    } else {
      if (kc < n_sel) row[kc] = v0;
      if (kc + 1 < n_sel) row[kc + 1] = v1;
    }
  }
}

// One warp per net; a cycle counts once however many events it holds.
__global__ void toggle_stats_kernel(const int64_t* off, const int64_t* time, int n_net, int64_t tpc, uint64_t magic,
                                    int64_t c_lo, int64_t c_hi, const float* y, int64_t* count, double* sum_y) {
  const int64_t wid = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (wid >= n_net) return;
  const int64_t b = off[wid], e = off[wid + 1];
  long long cnt = 0;
  double sy = 0;
  for (int64_t i = b + lane; i < e; i += 32) {
    const int64_t t = time[i];
    if (t <= 0) continue;
    const int64_t c = cycle_of(t, tpc, magic);
    if (c < c_lo || c >= c_hi) continue;
    bool first = true;
    if (i > b) {
      const int64_t tp = time[i - 1];
      first = tp <= 0 || cycle_of(tp, tpc, magic) != c;
    }
    if (first) {
      ++cnt;
      sy += (double)y[c - c_lo];
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    sy += __shfl_xor_sync(0xffffffffu, sy, o);
  }
  if (lane == 0) {
    count[wid] += cnt;
    sum_y[wid] += sy;
  }
}

int grid_for(int64_t n, int threads = 256, int cap = 148 * 16) {
  return (int)std::max<int64_t>(1, std::min<int64_t>(cap, (n + threads - 1) / threads));
}

}  // namespace

struct gtp_proxy {
  gtp_proxy_config cfg{};
  Layout L{};
  int B = 0;
  int device = 0;
  cudaStream_t stream = nullptr, own_stream = nullptr;
  std::string err;
  float *master = nullptr, *grad = nullptr, *mom1 = nullptr, *mom2 = nullptr;
  uint16_t *W1 = nullptr, *W2 = nullptr, *W2t = nullptr, *W3 = nullptr, *W3t = nullptr;
  uint16_t *Xb = nullptr, *XbT = nullptr, *H1 = nullptr, *H1t = nullptr, *H2 = nullptr, *H2t = nullptr;
  uint16_t *dY = nullptr, *dYt = nullptr, *dH2 = nullptr, *dH2t = nullptr, *dH1t = nullptr;
  float *Tb = nullptr, *Yb = nullptr;
  float* scal = nullptr;  // [0] step loss, [1] epoch loss
  int64_t* counters = nullptr;
  int* d_err = nullptr;
  float *mean = nullptr, *inv_std = nullptr, *stdv = nullptr;
  const uint16_t* X_all = nullptr;
  const float* Y_all = nullptr;
  int64_t n_rows = 0;
  int32_t* perm = nullptr;
  int64_t perm_cap = 0;
  int32_t* rows = nullptr;
  uint16_t *P1 = nullptr, *P2 = nullptr;
  float* PY = nullptr;
  int64_t pchunk = 0;
  cudaGraphExec_t gexec = nullptr;
  cudaGraph_t graph = nullptr;
  std::mt19937_64 rng;
};

namespace {

gtp_status fail(gtp_proxy* p, gtp_status s, const std::string& m) {
  if (p) p->err = m;
  return s;
}
gtp_status cuda_fail(gtp_proxy* p, const char* what, cudaError_t e) {
  return fail(p, GTP_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}
#define PX_CUDA(p, call)                                 \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return cuda_fail(p, #call, e_); \
  } while (0)

Publish publish_of(gtp_proxy* p) { return Publish{p->W1, p->W2, p->W2t, p->W3, p->W3t}; }

// Enqueues one forward + backward pass on the gathered minibatch.
gtp_status enqueue_fwd_bwd(gtp_proxy* p) {
  const Layout& L = p->L;
  const int B = p->B;
  cudaStream_t s = p->stream;
  const float* bias1 = p->master + L.ob1;
  const float* bias2 = p->master + L.ob2;
  const float* bias3 = p->master + L.ob3;
  cudaError_t e;
  {  // L1
    Epilogue ep;
    ep.mode = U::EPI_BIAS | U::EPI_RELU | U::EPI_OUT_BF16 | U::EPI_OUT_BF16_T;
    ep.bias = bias1;
    ep.out = p->H1;
    ep.ldo = L.H;
    ep.out_t = p->H1t;
    ep.ldt = B;
    ep.err = p->d_err;
    e = U::gemm_bf16_tn(Operand{p->Xb, B, L.I}, Operand{p->W1, L.H, L.I}, B, L.H, L.I, ep, s);
    if (e != cudaSuccess) return cuda_fail(p, "L1 gemm", e);
  }
  {  // L2
    Epilogue ep;
    ep.mode = U::EPI_BIAS | U::EPI_RELU | U::EPI_OUT_BF16 | U::EPI_OUT_BF16_T;
    ep.bias = bias2;
    ep.out = p->H2;
    ep.ldo = L.H;
    ep.out_t = p->H2t;
    ep.ldt = B;
    ep.err = p->d_err;
    e = U::gemm_bf16_tn(Operand{p->H1, B, L.H}, Operand{p->W2, L.H, L.H}, B, L.H, L.H, ep, s);
    if (e != cudaSuccess) return cuda_fail(p, "L2 gemm", e);
  }
  {  // L3 + MSE gradient
    Epilogue ep;
    ep.mode = U::EPI_BIAS | U::EPI_MSE | U::EPI_OUT_F32 | U::EPI_OUT_BF16 | U::EPI_OUT_BF16_T | U::EPI_COLSUM;
    ep.bias = bias3;
    ep.out_f = p->Yb;
    ep.ldf = L.Op;
    ep.target = p->Tb;
    ep.ldy = L.Op;
    ep.n_valid = L.O;
    ep.grad_scale = 2.f / ((float)B * (float)L.O);
    ep.out = p->dY;
    ep.ldo = L.Op;
    ep.out_t = p->dYt;
    ep.ldt = B;
    ep.colsum = p->grad + L.ob3;
    ep.loss = p->scal;
    ep.err = p->d_err;
    e = U::gemm_bf16_tn(Operand{p->H2, B, L.H}, Operand{p->W3, L.Op, L.H}, B, L.Op, L.H, ep, s);
    if (e != cudaSuccess) return cuda_fail(p, "L3 gemm", e);
  }
  {  // dW3 = dY^T H2
    Epilogue ep;
    ep.mode = U::EPI_OUT_F32;
    ep.out_f = p->grad + L.oW3;
    ep.ldf = L.H;
    ep.err = p->d_err;
    e = U::gemm_bf16_tn(Operand{p->dYt, L.Op, B}, Operand{p->H2t, L.H, B}, L.Op, L.H, B, ep, s);
    if (e != cudaSuccess) return cuda_fail(p, "dW3 gemm", e);
  }
  {  // dH2 = (dY W3) * [H2 > 0]
    Epilogue ep;
    ep.mode = U::EPI_RELU_BWD | U::EPI_OUT_BF16 | U::EPI_OUT_BF16_T | U::EPI_COLSUM;
    ep.mask = p->H2;
    ep.ldm = L.H;
    ep.out = p->dH2;
    ep.ldo = L.H;
    ep.out_t = p->dH2t;
    ep.ldt = B;
    ep.colsum = p->grad + L.ob2;
    ep.err = p->d_err;
    e = U::gemm_bf16_tn(Operand{p->dY, B, L.Op}, Operand{p->W3t, L.H, L.Op}, B, L.H, L.Op, ep, s);
    if (e != cudaSuccess) return cuda_fail(p, "dH2 gemm", e);
  }
  {  // dW2 = dH2^T H1
    Epilogue ep;
    ep.mode = U::EPI_OUT_F32;
    ep.out_f = p->grad + L.oW2;
    ep.ldf = L.H;
    ep.err = p->d_err;
    e = U::gemm_bf16_tn(Operand{p->dH2t, L.H, B}, Operand{p->H1t, L.H, B}, L.H, L.H, B, ep, s);
    if (e != cudaSuccess) return cuda_fail(p, "dW2 gemm", e);
  }
  {  // dH1 = (dH2 W2) * [H1 > 0]
    Epilogue ep;
    ep.mode = U::EPI_RELU_BWD | U::EPI_OUT_BF16_T | U::EPI_COLSUM;
    ep.mask = p->H1;
    ep.ldm = L.H;
    ep.out_t = p->dH1t;
    ep.ldt = B;
    ep.colsum = p->grad + L.ob1;
    ep.err = p->d_err;
    e = U::gemm_bf16_tn(Operand{p->dH2, B, L.H}, Operand{p->W2t, L.H, L.H}, B, L.H, L.H, ep, s);
    if (e != cudaSuccess) return cuda_fail(p, "dH1 gemm", e);
  }
  {  // dW1 = dH1^T Xb
    Epilogue ep;
    ep.mode = U::EPI_OUT_F32;
    ep.out_f = p->grad + L.oW1;
    ep.ldf = L.I;
    ep.err = p->d_err;
    e = U::gemm_bf16_tn(Operand{p->dH1t, L.H, B}, Operand{p->XbT, L.I, B}, L.H, L.I, B, ep, s);
    if (e != cudaSuccess) return cuda_fail(p, "dW1 gemm", e);
  }
  return GTP_OK;
}

AdamArgs adam_args(gtp_proxy* p, bool epoch_loss) {
  AdamArgs a;
  a.p = p->master;
  a.m = p->mom1;
  a.v = p->mom2;
  a.g = p->grad;
  a.L = p->L;
  a.P = publish_of(p);
  a.lr = p->cfg.lr;
  a.b1 = p->cfg.beta1;
  a.b2 = p->cfg.beta2;
  a.eps = p->cfg.eps;
  a.wd = p->cfg.weight_decay;
  a.counters = p->counters;
  a.loss_step = p->scal;
  a.loss_epoch = epoch_loss ? p->scal + 1 : nullptr;
  a.loss_norm = 1.f / ((float)p->B * (float)p->L.O);
  return a;
}

// One full training step reading minibatch counters[1] of `perm`.
gtp_status enqueue_train_step(gtp_proxy* p) {
  const Layout& L = p->L;
  cudaStream_t s = p->stream;
  begin_step_kernel<<<4, 256, 0, s>>>(p->counters, p->grad, L, p->scal);
  gather_kernel<<<dim3(L.I / 64, p->B / 32), 256, 0, s>>>(p->X_all, p->Y_all, p->perm, p->counters, p->B, L,
                                                          p->mean, p->inv_std, p->Xb, p->XbT, p->Tb);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(p, "gather", e);
  gtp_status st = enqueue_fwd_bwd(p);
  if (st != GTP_OK) return st;
  adam_kernel<<<grid_for(L.n), 256, 0, s>>>(adam_args(p, true));
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(p, "adam", e);
  return GTP_OK;
}

gtp_status check_err(gtp_proxy* p) {
  int h = 0;
  PX_CUDA(p, cudaMemcpyAsync(&h, p->d_err, sizeof(int), cudaMemcpyDeviceToHost, p->stream));
  PX_CUDA(p, cudaStreamSynchronize(p->stream));
  if (h != 0) {
    cudaMemsetAsync(p->d_err, 0, sizeof(int), p->stream);
    return fail(p, GTP_ETIMEOUT, "a tensor-core pipeline wait timed out");
  }
  return GTP_OK;
}

template <class T>
cudaError_t dalloc(T** ptr, int64_t n) {
  return cudaMalloc(reinterpret_cast<void**>(ptr), std::max<int64_t>(1, n) * sizeof(T));
}

void free_all(gtp_proxy* p) {
  if (p->gexec) cudaGraphExecDestroy(p->gexec);
  if (p->graph) cudaGraphDestroy(p->graph);
  void* bufs[] = {p->master, p->grad, p->mom1, p->mom2, p->W1, p->W2, p->W2t, p->W3, p->W3t, p->Xb, p->XbT,
                  p->H1, p->H1t, p->H2, p->H2t, p->dY, p->dYt, p->dH2, p->dH2t, p->dH1t, p->Tb, p->Yb, p->scal,
                  p->counters, p->d_err, p->mean, p->inv_std, p->stdv, p->perm, p->rows, p->P1, p->P2, p->PY};
  for (void* b : bufs)
    if (b) cudaFree(b);
  if (p->own_stream) cudaStreamDestroy(p->own_stream);
}

// Maps between the user's flat parameter vector and the padded one.
void user_segments(const Layout& L, int64_t (*seg)[3], int* n_seg) {
  // {internal offset, user offset, count}
  int64_t u = 0;
  int k = 0;
  auto add = [&](int64_t io, int64_t cnt) {
    seg[k][0] = io;
    seg[k][1] = u;
    seg[k][2] = cnt;
    u += cnt;
    ++k;
  };
  add(L.oW1, (int64_t)L.H * L.I);
  add(L.ob1, L.H);
  add(L.oW2, (int64_t)L.H * L.H);
  add(L.ob2, L.H);
  add(L.oW3, (int64_t)L.O * L.H);
  add(L.ob3, L.O);
  *n_seg = k;
}

}  // namespace

extern "C" {

void gtp_proxy_config_default(gtp_proxy_config* c) {
  if (!c) return;
  std::memset(c, 0, sizeof(*c));
  c->cuda_device_id = 0;
  c->n_in = 4096;
  c->n_hidden = 512;
  c->n_out = 33;
  c->batch = 1024;
  c->lr = 1e-3f;
  c->beta1 = 0.9f;
  c->beta2 = 0.999f;
  c->eps = 1e-8f;
  c->weight_decay = 0.f;
  c->seed = 20261203ull;
  c->use_graph = 1;
}

gtp_status gtp_proxy_create(const gtp_proxy_config* cfg, gtp_proxy** out) {
  if (!cfg || !out) return GTP_EINVAL;
  *out = nullptr;
  if (cfg->n_in < 64 || cfg->n_in % 64 || cfg->n_hidden < 64 || cfg->n_hidden % 64 || cfg->n_out < 1 ||
      cfg->n_out > 256 || cfg->batch < 128 || cfg->batch % 128 || cfg->n_in > (1 << 20) ||
      cfg->n_hidden > 8192 || cfg->batch > (1 << 20))
    return GTP_EINVAL;
  if (!(cfg->lr > 0.f) || !(cfg->beta1 >= 0.f && cfg->beta1 < 1.f) || !(cfg->beta2 >= 0.f && cfg->beta2 < 1.f) ||
      !(cfg->eps > 0.f) || cfg->weight_decay < 0.f)
    return GTP_EINVAL;
  gtp_proxy* p = new gtp_proxy();
  p->cfg = *cfg;
  p->L.set(cfg->n_in, cfg->n_hidden, cfg->n_out);
  p->B = cfg->batch;
  p->device = cfg->cuda_device_id;
  p->rng.seed(cfg->seed ^ 0x5EEDull);
  cudaError_t e = cudaSetDevice(p->device);
  if (e != cudaSuccess) {
    delete p;
    return GTP_ECUDA;
  }
  const Layout& L = p->L;
  const int64_t B = p->B;
  e = cudaStreamCreateWithFlags(&p->own_stream, cudaStreamNonBlocking);
  p->stream = p->own_stream;
#define PX_ALLOC(ptr, n) \
  if (e == cudaSuccess) e = dalloc(&(ptr), (n))
  PX_ALLOC(p->master, L.n);
  PX_ALLOC(p->grad, L.n);
  PX_ALLOC(p->mom1, L.n);
  PX_ALLOC(p->mom2, L.n);
  PX_ALLOC(p->W1, (int64_t)L.H * L.I);
  PX_ALLOC(p->W2, (int64_t)L.H * L.H);
  PX_ALLOC(p->W2t, (int64_t)L.H * L.H);
  PX_ALLOC(p->W3, (int64_t)L.Op * L.H);
  PX_ALLOC(p->W3t, (int64_t)L.Op * L.H);
  PX_ALLOC(p->Xb, B * L.I);
  PX_ALLOC(p->XbT, B * L.I);
  PX_ALLOC(p->H1, B * L.H);
  PX_ALLOC(p->H1t, B * L.H);
  PX_ALLOC(p->H2, B * L.H);
  PX_ALLOC(p->H2t, B * L.H);
  PX_ALLOC(p->dY, B * L.Op);
  PX_ALLOC(p->dYt, B * L.Op);
  PX_ALLOC(p->dH2, B * L.H);
  PX_ALLOC(p->dH2t, B * L.H);
  PX_ALLOC(p->dH1t, B * L.H);
  PX_ALLOC(p->Tb, B * L.Op);
  PX_ALLOC(p->Yb, B * L.Op);
  PX_ALLOC(p->scal, 2);
  PX_ALLOC(p->counters, 4);
  PX_ALLOC(p->d_err, 1);
  PX_ALLOC(p->mean, L.Op);
  PX_ALLOC(p->inv_std, L.Op);
  PX_ALLOC(p->stdv, L.Op);
  PX_ALLOC(p->rows, B);
#undef PX_ALLOC
  if (e != cudaSuccess) {
    free_all(p);
    delete p;
    return GTP_ENOMEM;
  }
  cudaStream_t s = p->stream;
  cudaMemsetAsync(p->grad, 0, L.n * sizeof(float), s);
  cudaMemsetAsync(p->mom1, 0, L.n * sizeof(float), s);
  cudaMemsetAsync(p->mom2, 0, L.n * sizeof(float), s);
  cudaMemsetAsync(p->W3, 0, (size_t)L.Op * L.H * 2, s);
  cudaMemsetAsync(p->W3t, 0, (size_t)L.Op * L.H * 2, s);
  cudaMemsetAsync(p->dY, 0, (size_t)B * L.Op * 2, s);
  cudaMemsetAsync(p->scal, 0, 2 * sizeof(float), s);
  cudaMemsetAsync(p->counters, 0, 4 * sizeof(int64_t), s);
  cudaMemsetAsync(p->d_err, 0, sizeof(int), s);
  {
    std::vector<float> ones(L.Op, 1.f), zeros(L.Op, 0.f);
    cudaMemcpy(p->mean, zeros.data(), L.Op * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(p->inv_std, ones.data(), L.Op * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(p->stdv, ones.data(), L.Op * sizeof(float), cudaMemcpyHostToDevice);
  }
  init_params_kernel<<<grid_for(L.n), 256, 0, s>>>(p->master, L, cfg->seed);
  publish_kernel<<<grid_for(L.n), 256, 0, s>>>(p->master, L, publish_of(p));
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    free_all(p);
    delete p;
    return GTP_ECUDA;
  }
  *out = p;
  return GTP_OK;
}

void gtp_proxy_destroy(gtp_proxy* p) {
  if (!p) return;
  cudaSetDevice(p->device);
  if (p->stream) cudaStreamSynchronize(p->stream);
  free_all(p);
  delete p;
}

const char* gtp_proxy_last_error(const gtp_proxy* p) { return p ? p->err.c_str() : "null proxy"; }
void* gtp_proxy_get_stream(gtp_proxy* p) { return p ? (void*)p->stream : nullptr; }
gtp_status gtp_proxy_set_stream(gtp_proxy* p, void* stream) {
  if (!p) return GTP_EINVAL;
  if (p->gexec) {  // the graph was captured on the old stream's work; recapture later
    cudaGraphExecDestroy(p->gexec);
    cudaGraphDestroy(p->graph);
    p->gexec = nullptr;
    p->graph = nullptr;
  }
  p->stream = stream ? static_cast<cudaStream_t>(stream) : p->own_stream;
  return GTP_OK;
}
int64_t gtp_proxy_n_param(const gtp_proxy* p) { return p ? p->L.user_n : 0; }

gtp_status gtp_proxy_set_training_data(gtp_proxy* p, const uint16_t* d_x, const float* d_y, int64_t n_rows) {
  if (!p || !d_x || !d_y || n_rows < p->B) return fail(p, GTP_EINVAL, "training data needs at least `batch` rows");
  if ((reinterpret_cast<uintptr_t>(d_x) & 15) != 0) return fail(p, GTP_EINVAL, "d_x must be 16-byte aligned");
  PX_CUDA(p, cudaSetDevice(p->device));
  if (p->gexec) {  // the captured gather reads the previous data pointers
    PX_CUDA(p, cudaStreamSynchronize(p->stream));
    cudaGraphExecDestroy(p->gexec);
    cudaGraphDestroy(p->graph);
    p->gexec = nullptr;
    p->graph = nullptr;
  }
  p->X_all = d_x;
  p->Y_all = d_y;
  p->n_rows = n_rows;
  if (n_rows > p->perm_cap) {
    if (p->perm) cudaFree(p->perm);
    p->perm = nullptr;
    PX_CUDA(p, dalloc(&p->perm, n_rows));
    p->perm_cap = n_rows;
  }
  colstats_kernel<<<p->L.O, 256, 0, p->stream>>>(d_y, n_rows, p->L.O, p->mean, p->inv_std, p->stdv);
  PX_CUDA(p, cudaGetLastError());
  PX_CUDA(p, cudaStreamSynchronize(p->stream));
  return GTP_OK;
}

gtp_status gtp_proxy_get_norm(gtp_proxy* p, float* mean, float* stdv) {
  if (!p || !mean || !stdv) return GTP_EINVAL;
  PX_CUDA(p, cudaSetDevice(p->device));
  PX_CUDA(p, cudaStreamSynchronize(p->stream));
  PX_CUDA(p, cudaMemcpy(mean, p->mean, p->L.O * sizeof(float), cudaMemcpyDeviceToHost));
  PX_CUDA(p, cudaMemcpy(stdv, p->stdv, p->L.O * sizeof(float), cudaMemcpyDeviceToHost));
  return GTP_OK;
}

gtp_status gtp_proxy_train(gtp_proxy* p, int32_t n_epochs, float* loss_per_epoch) {
  if (!p || n_epochs < 0) return GTP_EINVAL;
  if (!p->X_all) return fail(p, GTP_ESTATE, "no training data");
  PX_CUDA(p, cudaSetDevice(p->device));
  const int64_t steps = p->n_rows / p->B;
  std::vector<int32_t> perm(p->n_rows);
  for (int ep = 0; ep < n_epochs; ++ep) {
    for (int64_t i = 0; i < p->n_rows; ++i) perm[i] = (int32_t)i;
    std::shuffle(perm.begin(), perm.end(), p->rng);
    PX_CUDA(p, cudaMemcpyAsync(p->perm, perm.data(), p->n_rows * sizeof(int32_t), cudaMemcpyHostToDevice, p->stream));
    PX_CUDA(p, cudaMemsetAsync(p->counters + 2, 0, sizeof(int64_t), p->stream));
    PX_CUDA(p, cudaMemsetAsync(p->scal + 1, 0, sizeof(float), p->stream));
    if (p->cfg.use_graph) {
      if (!p->gexec) {
        cudaGraph_t g = nullptr;
        PX_CUDA(p, cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeThreadLocal));
        gtp_status st = enqueue_train_step(p);
        cudaError_t e = cudaStreamEndCapture(p->stream, &g);
        if (st != GTP_OK) {
          if (g) cudaGraphDestroy(g);
          return st;
        }
        if (e != cudaSuccess) return cuda_fail(p, "cudaStreamEndCapture", e);
        e = cudaGraphInstantiate(&p->gexec, g, 0);
        if (e != cudaSuccess) {
          cudaGraphDestroy(g);
          return cuda_fail(p, "cudaGraphInstantiate", e);
        }
        p->graph = g;
      }
      for (int64_t s = 0; s < steps; ++s) PX_CUDA(p, cudaGraphLaunch(p->gexec, p->stream));
    } else {
      for (int64_t s = 0; s < steps; ++s) {
        gtp_status st = enqueue_train_step(p);
        if (st != GTP_OK) return st;
      }
    }
    float el = 0.f;
    PX_CUDA(p, cudaMemcpyAsync(&el, p->scal + 1, sizeof(float), cudaMemcpyDeviceToHost, p->stream));
    gtp_status st = check_err(p);  // synchronises the stream
    if (st != GTP_OK) return st;
    if (loss_per_epoch) loss_per_epoch[ep] = steps > 0 ? el / (float)steps : 0.f;
  }
  return GTP_OK;
}

gtp_status gtp_proxy_compute_grads(gtp_proxy* p, const int32_t* rows, float* loss) {
  if (!p || !rows) return GTP_EINVAL;
  if (!p->X_all) return fail(p, GTP_ESTATE, "no training data");
  for (int i = 0; i < p->B; ++i)
    if (rows[i] < 0 || rows[i] >= p->n_rows) return fail(p, GTP_EINVAL, "row index out of range");
  PX_CUDA(p, cudaSetDevice(p->device));
  cudaStream_t s = p->stream;
  const Layout& L = p->L;
  PX_CUDA(p, cudaMemcpyAsync(p->rows, rows, p->B * sizeof(int32_t), cudaMemcpyHostToDevice, s));
  PX_CUDA(p, cudaMemsetAsync(p->grad + L.ob1, 0, L.H * sizeof(float), s));
  PX_CUDA(p, cudaMemsetAsync(p->grad + L.ob2, 0, L.H * sizeof(float), s));
  PX_CUDA(p, cudaMemsetAsync(p->grad + L.ob3, 0, L.Op * sizeof(float), s));
  PX_CUDA(p, cudaMemsetAsync(p->scal, 0, sizeof(float), s));
  gather_kernel<<<dim3(L.I / 64, p->B / 32), 256, 0, s>>>(p->X_all, p->Y_all, p->rows, nullptr, p->B, L, p->mean,
                                                          p->inv_std, p->Xb, p->XbT, p->Tb);
  PX_CUDA(p, cudaGetLastError());
  gtp_status st = enqueue_fwd_bwd(p);
  if (st != GTP_OK) return st;
  float h = 0.f;
  PX_CUDA(p, cudaMemcpyAsync(&h, p->scal, sizeof(float), cudaMemcpyDeviceToHost, s));
  st = check_err(p);
  if (st != GTP_OK) return st;
  if (loss) *loss = h / ((float)p->B * (float)L.O);
  return GTP_OK;
}

gtp_status gtp_proxy_adam_step(gtp_proxy* p) {
  if (!p) return GTP_EINVAL;
  PX_CUDA(p, cudaSetDevice(p->device));
  bump_kernel<<<1, 1, 0, p->stream>>>(p->counters);
  adam_kernel<<<grid_for(p->L.n), 256, 0, p->stream>>>(adam_args(p, false));
  PX_CUDA(p, cudaGetLastError());
  PX_CUDA(p, cudaStreamSynchronize(p->stream));
  return GTP_OK;
}

static gtp_status copy_params(gtp_proxy* p, float* dev, float* host_out, const float* host_in) {
  int64_t seg[6][3];
  int n = 0;
  user_segments(p->L, seg, &n);
  PX_CUDA(p, cudaSetDevice(p->device));
  PX_CUDA(p, cudaStreamSynchronize(p->stream));
  for (int k = 0; k < n; ++k) {
    if (host_out)
      PX_CUDA(p, cudaMemcpy(host_out + seg[k][1], dev + seg[k][0], seg[k][2] * sizeof(float), cudaMemcpyDeviceToHost));
    else
      PX_CUDA(p, cudaMemcpy(dev + seg[k][0], host_in + seg[k][1], seg[k][2] * sizeof(float), cudaMemcpyHostToDevice));
  }
  return GTP_OK;
}

gtp_status gtp_proxy_get_params(gtp_proxy* p, float* params) {
  if (!p || !params) return GTP_EINVAL;
  return copy_params(p, p->master, params, nullptr);
}

gtp_status gtp_proxy_set_params(gtp_proxy* p, const float* params) {
  if (!p || !params) return GTP_EINVAL;
  gtp_status st = copy_params(p, p->master, nullptr, params);
  if (st != GTP_OK) return st;
  publish_kernel<<<grid_for(p->L.n), 256, 0, p->stream>>>(p->master, p->L, publish_of(p));
  PX_CUDA(p, cudaGetLastError());
  PX_CUDA(p, cudaStreamSynchronize(p->stream));
  return GTP_OK;
}

gtp_status gtp_proxy_get_grads(gtp_proxy* p, float* grads) {
  if (!p || !grads) return GTP_EINVAL;
  return copy_params(p, p->grad, grads, nullptr);
}

gtp_status gtp_proxy_predict(gtp_proxy* p, const uint16_t* d_x, int64_t n_rows, float* d_y) {
  if (!p || !d_x || !d_y || n_rows < 0) return GTP_EINVAL;
  if ((reinterpret_cast<uintptr_t>(d_x) & 15) != 0) return fail(p, GTP_EINVAL, "d_x must be 16-byte aligned");
  if (n_rows == 0) return GTP_OK;
  PX_CUDA(p, cudaSetDevice(p->device));
  const Layout& L = p->L;
  cudaStream_t s = p->stream;
  const int64_t chunk = std::min<int64_t>(65536, (n_rows + 127) / 128 * 128);
  if (chunk > p->pchunk) {
    if (p->P1) cudaFree(p->P1);
    if (p->P2) cudaFree(p->P2);
    if (p->PY) cudaFree(p->PY);
    p->P1 = p->P2 = nullptr;
    p->PY = nullptr;
    p->pchunk = 0;
    PX_CUDA(p, dalloc(&p->P1, chunk * L.H));
    PX_CUDA(p, dalloc(&p->P2, chunk * L.H));
    PX_CUDA(p, dalloc(&p->PY, chunk * L.Op));
    p->pchunk = chunk;
  }
  for (int64_t r0 = 0; r0 < n_rows; r0 += chunk) {
    const int64_t nr = std::min(chunk, n_rows - r0);
    cudaError_t e;
    Epilogue e1;
    e1.mode = U::EPI_BIAS | U::EPI_RELU | U::EPI_OUT_BF16;
    e1.bias = p->master + L.ob1;
    e1.out = p->P1;
    e1.ldo = L.H;
    e1.err = p->d_err;
    e = U::gemm_bf16_tn(Operand{d_x + r0 * L.I, nr, L.I}, Operand{p->W1, L.H, L.I}, nr, L.H, L.I, e1, s);
    if (e != cudaSuccess) return cuda_fail(p, "predict L1", e);
    Epilogue e2 = e1;
    e2.bias = p->master + L.ob2;
    e2.out = p->P2;
    e = U::gemm_bf16_tn(Operand{p->P1, nr, L.H}, Operand{p->W2, L.H, L.H}, nr, L.H, L.H, e2, s);
    if (e != cudaSuccess) return cuda_fail(p, "predict L2", e);
    Epilogue e3;
    e3.mode = U::EPI_BIAS | U::EPI_OUT_F32;
    e3.bias = p->master + L.ob3;
    e3.out_f = p->PY;
    e3.ldf = L.Op;
    e3.err = p->d_err;
    e = U::gemm_bf16_tn(Operand{p->P2, nr, L.H}, Operand{p->W3, L.Op, L.H}, nr, L.Op, L.H, e3, s);
    if (e != cudaSuccess) return cuda_fail(p, "predict L3", e);
    denorm_kernel<<<grid_for(nr * L.O), 256, 0, s>>>(p->PY, nr, L.O, L.Op, p->mean, p->stdv, d_y + r0 * L.O);
    PX_CUDA(p, cudaGetLastError());
  }
  return GTP_OK;
}

gtp_status gtp_toggle_bits(const int64_t* d_net_off, const int64_t* d_time, const int32_t* d_sel, int32_t n_sel,
                           int64_t tpc, int64_t c_lo, int64_t c_hi, uint16_t* d_x, int64_t ld, void* stream) {
  if (!d_net_off || !d_time || !d_sel || !d_x || n_sel < 0 || tpc <= 0 || c_hi < c_lo || ld < n_sel) return GTP_EINVAL;
  if (n_sel == 0 || c_hi == c_lo) return GTP_OK;
  const int64_t threads = (int64_t)n_sel * 32;
  toggle_bits_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      d_net_off, d_time, d_sel, n_sel, tpc, cycle_magic(tpc), c_lo, c_hi, d_x, ld);
  return cudaGetLastError() == cudaSuccess ? GTP_OK : GTP_ECUDA;
}

gtp_status gtp_toggle_bits_windows(const gtp_bits_window* windows, int32_t n_win, const int32_t* d_sel,
                                   int32_t n_sel, int64_t tpc, int64_t c_base, uint16_t* d_x, int64_t ld,
                                   void* stream) {
  if (!windows || n_win < 0 || n_win > GTP_BITS_MAX_WINDOWS || !d_sel || !d_x || n_sel < 0 || tpc <= 0 ||
      ld < n_sel)
    return GTP_EINVAL;
  if (n_sel == 0 || n_win == 0) return GTP_OK;
  BitsLaunch L;
  std::memset(&L, 0, sizeof(L));
  int64_t chunks = 0;
  for (int i = 0; i < n_win; ++i) {
    const gtp_bits_window& w = windows[i];
    if (!w.d_net_off || !w.d_time || w.c_hi < w.c_lo || w.c_lo < c_base) return GTP_EINVAL;
    L.w[i] = w;
    L.chunk0[i] = static_cast<int32_t>(chunks);
    chunks += (w.c_hi - w.c_lo + kBitsRows - 1) / kBitsRows;
    if (chunks > 65535) return GTP_EOVERFLOW;
  }
  L.chunk0[n_win] = static_cast<int32_t>(chunks);
  L.n_win = n_win;
  if (chunks == 0) return GTP_OK;
  dim3 grid(static_cast<unsigned>((n_sel + kBitsNets - 1) / kBitsNets), static_cast<unsigned>(chunks));
  toggle_bits_windows_kernel<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      L, d_sel, n_sel, tpc, cycle_magic(tpc), c_base, d_x, ld);
  return cudaGetLastError() == cudaSuccess ? GTP_OK : GTP_ECUDA;
}

gtp_status gtp_net_toggle_stats(const int64_t* d_net_off, const int64_t* d_time, int32_t n_net, int64_t tpc,
                                int64_t c_lo, int64_t c_hi, const float* d_y, int64_t* d_count, double* d_sum_y,
                                void* stream) {
  if (!d_net_off || !d_time || !d_y || !d_count || !d_sum_y || n_net < 0 || tpc <= 0 || c_hi < c_lo) return GTP_EINVAL;
  if (n_net == 0 || c_hi == c_lo) return GTP_OK;
  const int64_t threads = (int64_t)n_net * 32;
  toggle_stats_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      d_net_off, d_time, n_net, tpc, cycle_magic(tpc), c_lo, c_hi, d_y, d_count, d_sum_y);
  return cudaGetLastError() == cudaSuccess ? GTP_OK : GTP_ECUDA;
}

gtp_status gtp_bf16_gemm(const uint16_t* d_a, int64_t lda, const uint16_t* d_b, int64_t ldb, int64_t m, int64_t n,
                         int64_t k, const float* d_bias, int32_t relu, float* d_c, int64_t ldc, void* stream) {
  Epilogue ep;
  ep.mode = U::EPI_OUT_F32 | (d_bias ? U::EPI_BIAS : 0) | (relu ? U::EPI_RELU : 0);
  ep.bias = d_bias;
  ep.out_f = d_c;
  ep.ldf = ldc;
  cudaError_t e = U::gemm_bf16_tn(Operand{d_a, m, lda}, Operand{d_b, n, ldb}, m, n, k, ep,
                                  static_cast<cudaStream_t>(stream));
  if (e == cudaErrorInvalidValue) return GTP_EINVAL;
  return e == cudaSuccess ? GTP_OK : GTP_ECUDA;
}

gtp_status gtp_bf16_gemm_checked(const uint16_t* d_a, int64_t lda, const uint16_t* d_b, int64_t ldb, int64_t m,
                                 int64_t n, int64_t k, const float* d_bias, int32_t relu, float* d_c, int64_t ldc,
                                 int64_t spin_limit_cycles, int32_t test_skip_load_block, int32_t* d_err,
                                 void* stream) {
  if (d_err == nullptr || spin_limit_cycles < 0 || test_skip_load_block < -1) return GTP_EINVAL;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(d_err, 0, sizeof(int32_t), s) != cudaSuccess) return GTP_ECUDA;
  Epilogue ep;
  ep.mode = U::EPI_OUT_F32 | (d_bias ? U::EPI_BIAS : 0) | (relu ? U::EPI_RELU : 0);
  ep.bias = d_bias;
  ep.out_f = d_c;
  ep.ldf = ldc;
  ep.err = d_err;
  ep.spin_limit = spin_limit_cycles;
  ep.skip_load_block = test_skip_load_block;
  cudaError_t e = U::gemm_bf16_tn(Operand{d_a, m, lda}, Operand{d_b, n, ldb}, m, n, k, ep, s);
  if (e == cudaErrorInvalidValue) return GTP_EINVAL;
  if (e != cudaSuccess) return GTP_ECUDA;
  int32_t h = 0;
  e = cudaMemcpyAsync(&h, d_err, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return GTP_ECUDA;
  return h != 0 ? GTP_ETIMEOUT : GTP_OK;
}

}  // extern "C"
