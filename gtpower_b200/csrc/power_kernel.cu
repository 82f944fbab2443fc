// power_kernel.cu — the fused time-based power walk for sm_100a.
//
// One thread walks one cell over one cycle tile of the event window. It
// merges the cell's pin event lists in time order (the loop of
// findTimeBasedAllPower, power/TimeBasedPower.cc:795-890) and, per step:
//   - leakage: the cell's leakage changes only when its pin state changes.
//     Each change adds its difference to a per-cycle level (a run-difference
//     array, prefix-summed at finalize) and its share of its own cycle, so
//     the per-cycle integral of the state-dependent leakage — what
//     calculatePerCycleLeakagePower (TimeBasedPower.cc:677-701) computes
//     segment by segment — costs O(1) per state change and nothing per
//     idle cycle. Where a tick falls between a cycle's tick boundary and its
//     seconds boundary (c*clk_period), the reference's split departs from
//     the plain overlap; the drift path adds exactly those differences;
//   - glitch: the clock-period grouping of getEventClockCycleBasedGlitchFlags
//     (TimeBasedPower.cc:589-637); an event is isolated in its period unless
//     its neighbours say otherwise (two compares from registers), and only
//     then is the period scanned;
//   - internal energy: the first `when`-matching internal_power group
//     (findInputInternalVal, TimeBasedPower.cc:341-381) — for cells of up to
//     four pins a table lookup by pin state; for an output event, the
//     related input by arc-delay distance from the per-pin last-event
//     registers (findOutputInternalVal, TimeBasedPower.cc:383-509); plus
//     C*V^2 switching per rise.
//
// Per-cycle sums go to shared-memory bins as 64-bit fixed-point energies
// (integer shared atomics: exact, and the per-cycle outputs do not depend on
// accumulation order); a tile flushes its bins once. Per-cell sums stay in
// FP64 registers and are flushed once per tile. Event times are held as
// 32-bit offsets from the tile start.
#include <cstdint>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cuda_runtime.h>

#include "engine.h"

#ifndef WALK_MIN_BLOCKS
#define WALK_MIN_BLOCKS 2   // 2 x 256 threads per SM keeps the walk spill-free
#endif
#ifndef WARP_WALK_MIN_BLOCKS
#define WARP_WALK_MIN_BLOCKS 2
#endif

namespace gtpb {
namespace {

constexpr uint32_t kRelInf = 0xFFFFFFFFu;     // no further event
constexpr uint32_t kRelBeyond = 0xFFFFFFFEu;  // next event at or after the tile end
constexpr int32_t kFarBefore = INT32_MIN / 2;
#ifndef WALK_RING
#define WALK_RING 2
#endif
#ifndef WALK_KEY_CLASS
#define WALK_KEY_CLASS 1    // cells with a periodic clock pin sort apart from the others
#endif
#ifndef WALK_USE_RING
#define WALK_USE_RING 1
#endif
#ifndef WALK_BATCH_RING
#define WALK_BATCH_RING 1   // event buffers in the persistent batched walk too
#endif
#ifndef WALK_STAGE_INST
#define WALK_STAGE_INST 1
#endif
constexpr int kRing = WALK_RING;               // events buffered per pin (RING path)

// floor(t / d) for 0 <= t < 2^63 and d >= 2 with magic = ceil(2^64 / d)
// (0 for d == 1): umulhi(t, magic) is floor(t / d) or one more, since
// t * (magic - 2^64 / d) / 2^64 < 1/2.
__device__ __forceinline__ int64_t div_floor_t(int64_t t, int64_t d, uint64_t magic) {
  if (magic == 0u) return t;
  uint64_t q = __umul64hi(static_cast<uint64_t>(t), magic);
  if (q * static_cast<uint64_t>(d) > static_cast<uint64_t>(t)) --q;
  return static_cast<int64_t>(q);
}

// floor(n / d) for n < 2^31, d < 2^31 with magic = ceil(2^32 / d) (d >= 2):
// umulhi(n, magic) is floor(n / d) or one more.
__device__ __forceinline__ uint32_t udiv32(uint32_t n, uint32_t d, uint32_t magic) {
  if (magic == 0u) return n;  // d == 1
  uint32_t q = __umulhi(n, magic);
  if (q * d > n) --q;
  return q;
}

__device__ __forceinline__ int ev_value(const uint32_t* __restrict__ v, int64_t i) {
  return (__ldg(v + (i >> 4)) >> (2 * (i & 15))) & 3;
}

__device__ __forceinline__ int64_t ev_time(const int64_t* __restrict__ t, int64_t i) {
  return __ldg(t + i);
}

// First index in [lo, hi) whose event time is >= x.
__device__ __forceinline__ int64_t lower_bound_time(const int64_t* __restrict__ t, int64_t lo, int64_t hi, int64_t x) {
  while (lo < hi) {
    const int64_t m = lo + ((hi - lo) >> 1);
    if (ev_time(t, m) < x) lo = m + 1; else hi = m;
  }
  return lo;
}

// getNRise (power/PowerUtils.cc:213-237): returns 2*n_rise (0, 1 or 2).
__device__ __forceinline__ int nrise2(int prev, int cur) {
  if (prev == cur) return 0;
  if (cur == 1) return prev == 0 ? 2 : (prev == 2 ? 1 : 0);
  if (cur == 2) return prev == 0 ? 1 : 0;
  return 0;
}
// getNToggle (power/PowerUtils.cc:247-255): returns 2*n_toggle
__device__ __forceinline__ int ntoggle2(int prev, int cur) {
  if (prev == cur) return 0;
  return (prev == 2 || cur == 2) ? 1 : 2;
}

__device__ __forceinline__ bool when_holds(const uint2* __restrict__ cubes, int off, int n,
                                           uint32_t ones) {
  for (int k = 0; k < n; ++k) {
    const uint2 c = __ldg(cubes + off + k);
    if ((ones & c.x) == c.y) return true;
  }
  return false;
}

__device__ __forceinline__ unsigned long long to_fx(double x, double s) {
  return static_cast<unsigned long long>(__double2ll_rn(x * s));
}

// to_fx of a float energy at the scale fx_dyn: with fs = fx_dyn as a float
// (a power of two >= 1, and |e| * fs <= 2^32), e * fs is exact in FP32 and
// rounds to the same integer as the FP64 product.
__device__ __forceinline__ unsigned long long to_fx_f(float e, float fs, double s) {
  if (fs != 0.0f) return static_cast<unsigned long long>(__float2ll_rn(__fmul_rn(e, fs)));
  return to_fx(static_cast<double>(e), s);
}

// Reads element i of a register array without dynamic indexing.
template <int N, typename T>
__device__ __forceinline__ T sel(const T (&a)[N], int i) {
  T r = a[0];
#pragma unroll
  for (int j = 1; j < N; ++j)
    if (j == i) r = a[j];
  return r;
}

// 64-bit fixed-point add to a shared-memory bin as two 32-bit atomics: the
// low word's add returns the old value, so its carry is known exactly and
// goes to the high word (with the value's own high word) only when that sum
// is non-zero. The bin, read as one 64-bit word, holds the exact sum modulo
// 2^64 in any order of adds. On sm_100 a 32-bit shared atomic costs a small
// fraction of a 64-bit one, and most adds need one.
__device__ __forceinline__ void shared_add64(unsigned long long* a, unsigned long long x) {
  uint32_t* w = reinterpret_cast<uint32_t*>(a);
  const uint32_t xl = static_cast<uint32_t>(x), xh = static_cast<uint32_t>(x >> 32);
  const uint32_t old = atomicAdd(w, xl);
  const uint32_t h = xh + (old + xl < old ? 1u : 0u);
  if (h) atomicAdd(w + 1, h);
}

struct Bins {
  unsigned long long* s;   // [sets][slots][ct] fixed-point energies
  uint32_t* sc;            // [2][ct] counts
  int64_t c_lo;            // first cycle of the tile
  int64_t ct;              // cycles in the tile
  int64_t off;             // this cell's bin set (set * 6 * ct), -1: add to global memory
  int32_t g;               // this cell's group when per-cycle groups are kept
};

// per-cycle accumulator slots
constexpr int kLeakPart = 0;   // leakage inside the cycle of each change
constexpr int kLeakLevel = 1;  // run-difference of the per-cycle leakage level
constexpr int kInt = 2, kGInt = 3, kSw = 4, kGSw = 5;
// shared-memory slots of the clock runs (tile-local run-differences, prefix
// summed into kInt and kLeakPart when the tile is flushed)
constexpr int kIntRun = 6, kLeakRun = 7;

// The global-memory side of add_bin: cycles outside the tile's shared bins
// (kept out of line: rare, and the walks' loops stay small).
__device__ __noinline__ void add_bin_global(const KParams& p, int32_t g, int q, int64_t c, unsigned long long x) {
  const int64_t cc = c < 0 ? p.n_period : (c < p.n_period ? c : p.n_period);
  atomicAdd(p.cyc_acc + q * (p.n_period + 1) + cc, x);
  if (p.cyc_acc_g)
    atomicAdd(p.cyc_acc_g + (static_cast<int64_t>(g) * kNumCycAcc + q) * (p.n_period + 1) + cc, x);
}

__device__ __forceinline__ void add_bin(const KParams& p, const Bins& b, int q, int64_t c,
                                        unsigned long long x) {
  if (x == 0ull) return;
  const int64_t k = c - b.c_lo;
  if (k >= 0 && k < b.ct && b.off >= 0) shared_add64(b.s + b.off + q * b.ct + k, x);
  else add_bin_global(p, b.g, q, c, x);
}

// add_bin for cycle c_lo + k of the tile (k >= 0): the shared bin when k < ct
__device__ __forceinline__ void add_bin_k(const KParams& p, const Bins& b, int q, uint32_t k,
                                          unsigned long long x) {
  if (x == 0ull) return;
  if (k < static_cast<uint32_t>(b.ct) && b.off >= 0)
    shared_add64(b.s + b.off + static_cast<uint32_t>(q) * static_cast<uint32_t>(b.ct) + k, x);
  else
    add_bin_global(p, b.g, q, b.c_lo + k, x);
}

__device__ __forceinline__ void add_cnt(const KParams& p, const Bins& b, int q, int64_t c) {
  const int64_t k = c - b.c_lo;
  if (k >= 0 && k < b.ct) {
    atomicAdd(b.sc + q * b.ct + k, 1u);
  } else {
    const int64_t cc = c < p.n_period ? c : p.n_period;
    atomicAdd(p.cnt_cyc + q * (p.n_period + 1) + cc, 1ull);
  }
}

// In-place inclusive prefix sum of a[0, n) in shared memory, by all threads
// of the block (blockDim.x a multiple of 32); wsum: 32 words of scratch.
__device__ void block_inclusive_scan(unsigned long long* a, int64_t n, unsigned long long* wsum) {
  const int nt = blockDim.x, tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int64_t chunk = (n + nt - 1) / nt;
  const int64_t lo = min(n, static_cast<int64_t>(tid) * chunk), hi = min(n, lo + chunk);
  unsigned long long s = 0;
  for (int64_t k = lo; k < hi; ++k) {
    s += a[k];
    a[k] = s;
  }
  unsigned long long x = s;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const unsigned long long y = __shfl_up_sync(0xffffffffu, x, d);
    if (lane >= d) x += y;
  }
  if (lane == 31) wsum[w] = x;
  __syncthreads();
  if (w == 0) {
    unsigned long long v = lane < (nt >> 5) ? wsum[lane] : 0ull;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const unsigned long long y = __shfl_up_sync(0xffffffffu, v, d);
      if (lane >= d) v += y;
    }
    wsum[lane] = v;
  }
  __syncthreads();
  const unsigned long long off = (x - s) + (w > 0 ? wsum[w - 1] : 0ull);
  for (int64_t k = lo; k < hi; ++k) a[k] += off;
  __syncthreads();
}

// Seconds cycle of tick t: the largest c with c*period <= t*ts (the
// comparison calculatePerCycleLeakagePower's loop makes), given the tick
// cycle c0 of t.
__device__ __forceinline__ int64_t seconds_cycle(const KParams& p, int64_t t, int64_t c0) {
  const double ts = static_cast<double>(t) * p.ts;
  int64_t s = c0;
  while (s > 0 && !(static_cast<double>(s) * p.period_d <= ts)) --s;
  while (static_cast<double>(s + 1) * p.period_d <= ts) ++s;
  return s;
}

// Period-group bounds of event i (global index 0 at g0 never counts).
struct Group {
  int64_t first;
  int64_t last;
};

__device__ __forceinline__ Group period_group(const int64_t* __restrict__ t, int64_t i, int64_t lo,
                                              int64_t hi, int64_t g0, int64_t ps, int64_t pe) {
  Group g;
  int64_t j0 = i;
  while (j0 - 1 >= lo && j0 - 1 != g0 && ev_time(t, j0 - 1) >= ps) --j0;
  int64_t j1 = i;
  while (j1 + 1 < hi && ev_time(t, j1 + 1) < pe) ++j1;
  g.first = j0;
  g.last = j1;
  return g;
}

// Pulse width of event e on a net as float seconds, -1 when the event is not
// a glitch event (getGlitchScalingRatioClockCycleBasedH,
// TimeBasedPower.cc:303-339: flags from whole-waveform period groups, width
// to the previous or next event only when that neighbour is flagged).
__device__ float glitch_pw(const KParams& p, int64_t e, int64_t lo, int64_t hi, int64_t g0,
                           int64_t cur, int64_t cyc_start) {
  if (e == g0) return -1.0f;
  const Group gr = period_group(p.ev_t, e, lo, hi, g0, cyc_start, cyc_start + p.tpc);
  const int64_t k = gr.last - gr.first + 1;
  const int64_t lim = k >= 2 ? (k & ~int64_t(1)) : 0;
  if (!(e - gr.first < lim)) return -1.0f;
  int64_t w = -1;
  if (e - 1 >= lo) {
    bool pflag;
    if (e - 1 >= gr.first) {
      pflag = true;
    } else if (e - 1 == g0) {
      pflag = false;
    } else {
      const int64_t tp = ev_time(p.ev_t, e - 1);
      const int64_t pc = div_floor_t(tp, p.tpc, p.tpc_magic64);
      const Group gp = period_group(p.ev_t, e - 1, lo, hi, g0, pc * p.tpc, pc * p.tpc + p.tpc);
      const int64_t kp = gp.last - gp.first + 1;   // e-1 is the last of its period
      pflag = kp >= 2 && (kp & 1) == 0;
    }
    if (pflag) w = cur - ev_time(p.ev_t, e - 1);
  }
  if (e + 1 < hi) {
    bool nflag;
    const int64_t tn = ev_time(p.ev_t, e + 1);
    if (e + 1 <= gr.last) {
      nflag = (e + 1 - gr.first) < lim;
    } else if (e + 2 < hi) {
      const int64_t nc = div_floor_t(tn, p.tpc, p.tpc_magic64);
      nflag = ev_time(p.ev_t, e + 2) < nc * p.tpc + p.tpc;
    } else {
      nflag = false;
    }
    if (nflag) w = max(w, tn - cur);
  }
  if (w < 0) return -1.0f;
  return __double2float_rn(__dmul_rn(static_cast<double>(w), p.ts));
}

// Glitch scaling ratio for pulse width pw (s) on a pin whose rise and fall
// slews sum to den (getTimeBasedGlitchScalingRatioH, PowerUtils.cc:285-294);
// -1 when pw < 0 (not a glitch event).
// The reference forms the ratio in double, (pw * 2.0) / den, and rounds it
// to float; for float operands that equals the correctly rounded float
// quotient, since double rounding of a quotient through a format of at
// least 2p + 2 bits is innocuous (53 >= 2 * 24 + 2; S. Figueroa, "When is
// double rounding innocuous?", SIGNUM Newsletter 30(3), 1995), and pw * 2
// is exact in float.
__device__ __forceinline__ float glitch_ratio_of(float pw, float den) {
  if (pw < 0.0f) return -1.0f;
  if (den == 0.0f) return 1.0f;
  const float r = __fdiv_rn(__fmul_rn(pw, 2.0f), den);
  return fminf(1.0f, __fmul_rn(r, r));
}

// glitch_pw and glitch_ratio_of in one step.
__device__ __forceinline__ float glitch_ratio(const KParams& p, int64_t e, int64_t lo, int64_t hi, int64_t g0,
                                              int64_t cur, int64_t cyc_start, float den) {
  return glitch_ratio_of(glitch_pw(p, e, lo, hi, g0, cur, cyc_start), den);
}

// One work item of the walk: the cells order[order_begin + gblk * gates_per_block ...]
// of one pin bucket over cycle tile `tile` of the window, with the block's
// dynamic shared memory `smem`. All threads of the block call it together.
// DYN = false walks the leakage alone (the leakage kernel of the separate
// two-kernel evaluation): the merge and the leakage steps, no energies.
template <int MAXP, bool COUNTS, bool FAST, bool DRIFT, bool RUNS, bool RING_EV, bool DYN = true>
__device__ __forceinline__ void walk_block(const KParams& p, const int gblk, const int tile, const int n_blk,
                                           unsigned long long* smem) {
  static_assert(DYN || (!COUNTS && !RUNS), "the leakage-only walk keeps no counts and walks every edge");
  const int64_t ct = p.cycles_per_tile;
  // per-cycle groups: two bin sets, for the block's first group and the next
  const int nset = p.cell_cgroup ? 2 : 1;
  // periodic clock pins (RUNS: cells of up to kFastPins pins, no drift):
  // each set carries the two clock-run slots
  static_assert(!RUNS || (FAST && !DRIFT), "clock runs need the fast walk without drift");
  const bool runs_on = RUNS && p.pclk != nullptr;
  // RUNS: each thread's per-cell FP64 sums live in shared memory (slot q of
  // thread t at s_acc[t * 5 + q]: an odd stride of 8-byte words, free of bank
  // conflicts), ahead of the bins, to leave the registers to the walk
  double* s_acc = nullptr;
  if (RUNS) {
    s_acc = reinterpret_cast<double*>(smem) + threadIdx.x * kNumCellAcc;
    smem += kNumCellAcc * blockDim.x;
  }
  const int nslot = runs_on ? kNumBinSlotsRun : kNumCycAcc;
  __shared__ unsigned long long s_wsum[32];
  Bins bins;
  bins.s = smem;
  bins.sc = reinterpret_cast<uint32_t*>(smem + nset * nslot * ct);
  bins.off = 0;
  bins.g = 0;
  // the tile's cycles [c_lo, c_lo + ct_tile): from the range table, or the
  // window's regular tiling
  const int2 tdesc = p.tiles ? p.tiles[tile] : make_int2(0, 0);
  bins.c_lo = p.tiles ? static_cast<int64_t>(tdesc.x) : p.cyc0 + static_cast<int64_t>(tile) * ct;
  const int64_t ct_tile = p.tiles ? static_cast<int64_t>(tdesc.y) : ct;
  bins.ct = ct;
  for (int64_t k = threadIdx.x; k < nset * nslot * ct; k += blockDim.x) smem[k] = 0ull;
  if (COUNTS)
    for (int64_t k = threadIdx.x; k < 2 * ct; k += blockDim.x) bins.sc[k] = 0u;
  // RING: per-thread event buffers [pin][slot][thread] of times - T0, then
  // the per-type energy-selection and leakage tables when they fit
  static_assert(!RING_EV || FAST, "event buffers are for the fast walk");
  constexpr bool RING = RING_EV;
  constexpr bool STAGE = FAST && WALK_STAGE_INST;
  uint32_t* ring = reinterpret_cast<uint32_t*>(smem + nset * nslot * ct + (COUNTS ? ct : 0));
  const int nt_blk = blockDim.x;
  const int16_t* fast_tab = p.fast_tab;
  const float* leak_pool = p.leak_pool;
  float* s_tabs = reinterpret_cast<float*>(ring + (RING ? MAXP * kRing * nt_blk : 0));
  if (FAST && p.tabs_in_smem) {
    float* s_leak = s_tabs;
    int16_t* s_fast = reinterpret_cast<int16_t*>(s_leak + p.n_leak_pool);
    for (int k = threadIdx.x; k < p.n_leak_pool; k += blockDim.x) s_leak[k] = __ldg(p.leak_pool + k);
    for (int k = threadIdx.x; k < p.n_fast_tab; k += blockDim.x) s_fast[k] = __ldg(p.fast_tab + k);
    leak_pool = s_leak;
    fast_tab = s_fast;
  }
  // STAGE: each thread's copy of its cell's instance block (energies, delays)
  float* s_inst = s_tabs + (FAST && p.tabs_in_smem ? ((p.n_leak_pool * 4 + p.n_fast_tab * 2 + 15) / 16) * 4 : 0)
                  + threadIdx.x * p.fast_inst_stride;
  __syncthreads();

  // tile window in ticks: [T0, T0 + span)
  const int64_t T0 = max(p.t_lo, bins.c_lo * p.tpc);
  // T0's offset within cycle c_lo: event cycles follow from 32-bit offsets
  const uint32_t off0 = static_cast<uint32_t>(T0 - bins.c_lo * p.tpc);
  const uint32_t tpc32 = static_cast<uint32_t>(p.tpc);
  // the tile ends at its last cycle's end, or past time_max (events at
  // time_max belong to the trace) when it reaches the trace's end
  const int64_t t_end = (bins.c_lo + ct_tile) * p.tpc;
  const int64_t T1 = t_end > p.tmax ? min(p.t_hi, p.tmax + 1) : min(p.t_hi, t_end);
  const uint32_t span = static_cast<uint32_t>(T1 > T0 ? T1 - T0 : 0);
  const bool standalone = p.standalone != 0;
  const bool owns_initial = !standalone && bins.c_lo == 0 && (p.t_lo == 0);
  const double P = p.period_d;
  // clock runs: a periodic pin's edges exist from tick max(t_lo, 1) on
  // (r_exist relative to T0); the tile holds those before span
  int32_t r_exist = 0;
  if (runs_on) {
    const int64_t tl = max(p.t_lo, static_cast<int64_t>(1)) - T0;
    r_exist = static_cast<int32_t>(max(tl, -static_cast<int64_t>(INT32_MAX / 2)));
  }

  // The block's work: without a split table, the cells order[g_begin, g_end)
  // of the bucket (one thread each); with one (density split), walk items
  // of the bucket's item space [ib0, ie0) in chunks of gates_per_block:
  // chunk gblk, then gblk + n_blk, ... while items remain. Item it is
  // sub-walk it - item_off[k] of the cell at walk-order position k.
  const bool split = p.item_off != nullptr;
  const int32_t ib0 = split ? __ldg(p.item_off + p.order_begin) : p.order_begin;
  const int32_t ie0 = split ? __ldg(p.item_off + p.order_end) : p.order_end;
  // walk-order position of item it: the last k in [order_begin, order_end)
  // with item_off[k] <= it
  auto pos_of = [&](int32_t it) -> int32_t {
    if (!split) return it;
    int32_t lo = p.order_begin, hi = p.order_end;   // item_off[lo] <= it < item_off[hi]
    while (hi - lo > 1) {
      const int32_t m = lo + ((hi - lo) >> 1);
      if (__ldg(p.item_off + m) <= it) lo = m; else hi = m;
    }
    return lo;
  };
  const int64_t first_item = static_cast<int64_t>(ib0) + static_cast<int64_t>(gblk) * p.gates_per_block;
  // cells are ordered by group within a bucket: the block's first cell has
  // its smallest group
  const int32_t g_first = (p.cell_cgroup && first_item < ie0)
                              ? __ldg(p.cell_cgroup + __ldg(p.order + pos_of(static_cast<int32_t>(first_item))))
                              : 0;

  for (int64_t chunk = gblk;; chunk += n_blk) {
  const int64_t cb = static_cast<int64_t>(ib0) + chunk * p.gates_per_block;
  if (cb >= ie0) break;
  const int32_t ce = static_cast<int32_t>(min(static_cast<int64_t>(ie0), cb + p.gates_per_block));
  for (int32_t it = static_cast<int32_t>(cb) + threadIdx.x; it < ce; it += blockDim.x) {
    const int32_t gi = pos_of(it);
    const int32_t sub = split ? it - __ldg(p.item_off + gi) : 0;
    const int32_t nsub = split ? __ldg(p.item_off + gi + 1) - __ldg(p.item_off + gi) : 1;
    const int32_t cell = __ldg(p.order + gi);
    // this thread's part of the tile: ticks [T0 + s0r, T0 + s1r), the
    // cycles [sub * ct / nsub, (sub + 1) * ct / nsub) of the tile
    uint32_t s0r = 0, s1r = span;
    if (nsub > 1) {
      auto bnd = [&](int64_t k) -> uint32_t {
        const int64_t r = k * static_cast<int64_t>(tpc32) - static_cast<int64_t>(off0);
        return r <= 0 ? 0u : (r >= static_cast<int64_t>(span) ? span : static_cast<uint32_t>(r));
      };
      s0r = bnd(static_cast<int64_t>(sub) * ct / nsub);
      if (sub + 1 < nsub) s1r = bnd(static_cast<int64_t>(sub + 1) * ct / nsub);
    }
    const bool owns_initial_cell = owns_initial && sub == 0;
    if (p.cell_cgroup) {
      bins.g = __ldg(p.cell_cgroup + cell);
      const int32_t set = bins.g - g_first;
      bins.off = (set == 0 || set == 1) ? static_cast<int64_t>(set) * nslot * ct : -1;
    }
    const int32_t p0 = __ldg(p.cell_pin_off + cell);
    const int32_t type = __ldg(p.cell_type + cell);
    const DevType ty = p.types[type];
    const float* __restrict__ blk_g = p.inst + __ldg(p.cell_inst + cell);
    const int n_pin = ty.n_pin, n_in = ty.n_in;
    const int n_state = 1 << (n_pin < 16 ? n_pin : 0);
    const int32_t fo = FAST ? __ldg(p.type_fast_off + type) : 0;
    if (STAGE) {
      // blocks are padded to a multiple of 4 floats and 16-byte aligned
      const float4* src = reinterpret_cast<const float4*>(blk_g);
      for (int k = 0; k < ty.inst_floats / 4; ++k) {
        const float4 v = __ldg(src + k);
        s_inst[4 * k + 0] = v.x; s_inst[4 * k + 1] = v.y; s_inst[4 * k + 2] = v.z; s_inst[4 * k + 3] = v.w;
      }
    }
    const float* blk = STAGE ? s_inst : blk_g;
    // internal energy of input pin i's event (before the rise/fall and
    // toggle factors) under the pre-step pin values oo
    auto in_energy = [&](int i, uint32_t oo, bool rise) -> float {
      float en = 0.0f;
      if (FAST) {
        const int16_t eo = fast_tab[fo + i * n_state + oo];
        if (eo >= 0) en = blk[eo + (rise ? 0 : 1)];
      } else {
        const int32_t s_begin = __ldg(p.pin_slot + ty.pin_slot_off + i);
        const int32_t s_end = __ldg(p.pin_slot + ty.pin_slot_off + i + 1);
        for (int32_t k = s_begin; k < s_end; ++k) {
          const DevSlot sl = p.slots[k];
          if (when_holds(p.cubes, sl.cube_off, sl.n_cube, oo)) {
            en = blk[sl.e_off + (rise ? 0 : 1)];
            break;
          }
        }
      }
      return en;
    };

    int64_t f[MAXP];          // next event index to read (absolute)
    int32_t rem[MAXP];        // events left to read in the accessible range
    uint32_t rs[MAXP];        // RING: head slot | (events held << 8)
    uint32_t rv[MAXP];        // RING: 2-bit values of the held events by slot
    uint32_t nt[MAXP];        // next event time - T0, or kRelBeyond / kRelInf
    int32_t lt[MAXP];         // time of the last event strictly before now - T0
    uint32_t state = 0;       // 2 bits per pin (MAXP <= 16) ...
    uint64_t state_hi = 0;    // ... pins 16..31
    uint32_t ones = 0;        // bit per pin: state == 1
    uint32_t nvals = 0;       // prefetched value of each pin's next event (pins < 16)
    uint64_t nvals_hi = 0;
    uint32_t has_wave = 0, clock_mask = 0, at_lo = 0, last_rise = 0;
    // the cell's periodic clock pin (bit pkbit, at most one), not merged:
    // its edges alternate between phase pA (to 1 - pv0) and pB (back to pv0)
    // of each cycle; edge j of the tile lies in tile cycle j / 2; bit 30 of
    // pBv: the edge at time_max is absent
    uint32_t pkbit = 0, pA = 0, pBv = 0;
    auto get_v = [&](uint32_t s_lo, uint64_t s_hi, int i) -> int {
      return i < 16 ? static_cast<int>((s_lo >> (2 * i)) & 3) : static_cast<int>((s_hi >> (2 * (i - 16))) & 3);
    };
    auto set_v = [&](uint32_t& s_lo, uint64_t& s_hi, int i, int v) {
      if (i < 16) s_lo = (s_lo & ~(3u << (2 * i))) | (static_cast<uint32_t>(v) << (2 * i));
      else s_hi = (s_hi & ~(3ull << (2 * (i - 16)))) | (static_cast<uint64_t>(v) << (2 * (i - 16)));
    };
    auto rel = [&](int64_t t) -> uint32_t {
      const int64_t r = t - T0;
      return (r >= 0 && r < static_cast<int64_t>(s1r)) ? static_cast<uint32_t>(r) : kRelBeyond;
    };
    // RING: read up to kRing events of pin i into its buffer with
    // independent loads (one memory latency per kRing events)
    auto refill = [&](int i) {
      const int32_t rem_i = sel<MAXP>(rem, i);
      const int n = rem_i < kRing ? rem_i : kRing;
      const int64_t a = sel<MAXP>(f, i);
      const int64_t w0 = a >> 4;
      const uint32_t vw0 = __ldg(p.ev_v + w0);
      const uint32_t vw1 = ((a + n - 1) >> 4) != w0 ? __ldg(p.ev_v + w0 + 1) : 0u;
      uint32_t vals = 0;
#pragma unroll 4
      for (int j = 0; j < n; ++j) {
        {
          const int64_t idx = a + j;
          const int64_t tj = ev_time(p.ev_t, idx);
          if (tj > p.tmax) atomicOr(p.status, kErrTimeRange);
          ring[(i * kRing + j) * nt_blk + threadIdx.x] = rel(tj);
          const uint32_t w = (idx >> 4) == w0 ? vw0 : vw1;
          vals |= ((w >> (2 * (idx & 15))) & 3u) << (2 * j);
        }
      }
      const uint32_t head = ring[(i * kRing) * nt_blk + threadIdx.x];
#pragma unroll
      for (int j = 0; j < MAXP; ++j) {
        if (j == i) {
          rv[j] = vals;
          rs[j] = static_cast<uint32_t>(n) << 8;
          f[j] = a + n;
          rem[j] = rem_i - n;
          nt[j] = head;
        }
      }
    };
    // pins whose buffer must be (re)filled before the next merge step
    uint32_t need = 0;
    auto do_refills = [&](int64_t after) {
      while (need) {
        const int i = __ffs(need) - 1;
        need &= need - 1;
        refill(i);
        const uint32_t h = sel<MAXP>(nt, i);
        if (static_cast<int64_t>(h) <= after) atomicOr(p.status, kErrTimeOrder);
      }
    };
#pragma unroll
    for (int i = 0; i < MAXP; ++i) {
      f[i] = 0; rem[i] = 0; nt[i] = kRelInf; lt[i] = kFarBefore; rs[i] = 0; rv[i] = 0;
      if (i < n_pin) {
        const int32_t net = __ldg(p.pin_net + p0 + i);
        const uint8_t pf = __ldg(p.pin_flags + p0 + i);
        if (pf & 4) {
          clock_mask |= 1u << i;
          if (runs_on && !pkbit && net >= 0 && bins.off >= 0) {
            const int2 pc = __ldg(p.pclk + net);
            if (pc.x >= 0) {
              pkbit = 1u << i;
              pA = static_cast<uint32_t>(pc.x);
              pBv = static_cast<uint32_t>(pc.y);
            }
          }
        }
        int v = pf & 3;
        if (net >= 0) {
          const int64_t a = __ldg(p.net_off + net), e = __ldg(p.net_off + net + 1);
          if (a < 0 || e < a || e > p.n_event) {
            atomicOr(p.status, kErrNetRange);
          } else if (e > a) {
            has_wave |= 1u << i;
            const int64_t base = p.net_base ? __ldg(p.net_base + net) : 0;
            // lower_bound(T0 + s0r) in [a, e): the tile's start from the
            // window's per-(tile, net) index when it was built, then (or
            // else) by bisection
            int64_t l = a, r = e;
            const int64_t S0 = T0 + static_cast<int64_t>(s0r);
            if (p.tile_first) l = a + __ldg(p.tile_first + static_cast<int64_t>(tile) * p.n_net + net);
            if (!p.tile_first || s0r > 0) {
              while (l < r) {
                const int64_t m = l + ((r - l) >> 1);
                if (ev_time(p.ev_t, m) < S0) l = m + 1; else r = m;
              }
            }
            // the waveform's first event at tick 0 is the initial condition
            if (l < e && l == a && base == 0 && ev_time(p.ev_t, l) == 0) ++l;
            if (l > a) {
              v = ev_value(p.ev_v, l - 1);
            } else {
              v = 2;
              if (base != 0) atomicOr(p.status, kErrContext);
              at_lo |= 1u << i;
            }
            // last event strictly before T0 (clamped to the first listed one)
            const int64_t re = l > a ? l - 1 : a;
            const int64_t pe = re > a ? re - 1 : a;
            const int64_t tre = ev_time(p.ev_t, re) - T0;
            lt[i] = static_cast<int32_t>(tre < kFarBefore ? kFarBefore : (tre > INT32_MAX / 2 ? INT32_MAX / 2 : tre));
            if (nrise2(ev_value(p.ev_v, pe), ev_value(p.ev_v, re)) > 0) last_rise |= 1u << i;
            f[i] = l;
            rem[i] = static_cast<int32_t>(e - l);
            if (l < e) {
              if (RING) {
                need |= 1u << i;
              } else {
                nt[i] = rel(ev_time(p.ev_t, l));
                if (i < 16) nvals |= static_cast<uint32_t>(ev_value(p.ev_v, l)) << (2 * i);
                else nvals_hi |= static_cast<uint64_t>(ev_value(p.ev_v, l)) << (2 * (i - 16));
              }
            }
          }
        }
        if ((pkbit >> i) & 1) {  // its edges are accounted by runs, not merged
          nt[i] = kRelInf;
          rem[i] = 0;
          need &= ~(1u << i);
        }
        set_v(state, state_hi, i, v);
        if (v == 1) ones |= 1u << i;
      }
    }

    if (RING) do_refills(-1);
    const float leak_const = ty.leak_const;
    const int32_t leak_off = ty.leak_off;
    auto leak_of = [&](uint32_t o) -> float {
      return leak_off >= 0 ? leak_pool[leak_off + o] : leak_const;
    };
    // per-cell sums: internal, glitch internal, switching, glitch switching,
    // leakage (registers, or shared slots with RUNS)
    double acc_r[kNumCellAcc] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (RUNS)
#pragma unroll
      for (int q = 0; q < kNumCellAcc; ++q) s_acc[q] = 0.0;
    auto acc_add = [&](int q, double x) {
      if (RUNS) s_acc[q] += x;
      else acc_r[q] += x;
    };
    uint32_t n_ev = 0, n_gl = 0, n_half = 0, n_rel = 0;
    float leak_cur = leak_of(ones);
    // clock runs: between two changes of the cell's other pins the clock's
    // edges see one state s; the edges to 1 - pv0 (A) and back (B) carry the
    // internal energies eA, eB, and the leakage is lA at pv0, lB at 1 - pv0
    const uint32_t pB = pBv & 0x3fffffffu;
    const int pv0 = static_cast<int>(pBv >> 31);
    uint32_t pj = 0;  // next edge of the tile not yet accounted
    // end of the tile's edges: those before span, or before time_max when the
    // edge there is absent
    auto pclk_jend = [&]() -> uint32_t {
      const int64_t r_end = ((pBv >> 30) & 1u) ? min(static_cast<int64_t>(s1r), p.tmax - T0) : static_cast<int64_t>(s1r);
      if (r_end <= 0) return 0u;
      const uint32_t ce = udiv32(static_cast<uint32_t>(r_end - 1) + off0, tpc32, p.tpc_magic);
      const int32_t he = static_cast<int32_t>(static_cast<uint32_t>(r_end - 1) + off0 - ce * tpc32);
      return 2 * ce + (he >= static_cast<int32_t>(pA) ? 1u : 0u) + (he >= static_cast<int32_t>(pB) ? 1u : 0u);
    };
    // one edge j, with the contributions the merge would give it
    auto pclk_edge = [&](uint32_t j, float eA, float eB, float lA, float lB) {
      const int64_t ce = bins.c_lo + (j >> 1);
      const int64_t te = T0 + static_cast<int64_t>(static_cast<int32_t>((j >> 1) * tpc32) - static_cast<int32_t>(off0) +
                                                   static_cast<int32_t>((j & 1) ? pB : pA));
      const bool ea = !(j & 1);
      const float en = ea ? eA : eB;
      acc_add(0, en);
      add_bin_k(p, bins, kInt, j >> 1, to_fx_f(en, p.fx_dyn_f, p.fx_dyn));
      const double dl = ea ? static_cast<double>(lB) - static_cast<double>(lA)
                           : static_cast<double>(lA) - static_cast<double>(lB);
      if (dl != 0.0) {
        const double cur_s = static_cast<double>(te) * p.ts;
        const double end_s = fmin(static_cast<double>(ce + 1) * P, p.tmax_s);
        add_bin_k(p, bins, kLeakPart, j >> 1, to_fx(dl * (end_s - cur_s), p.fx_leak));
        add_bin_k(p, bins, kLeakLevel, (j >> 1) + 1, to_fx(dl * P, p.fx_leak));
        acc_add(4, dl * static_cast<double>(p.tmax - te));
      }
      if (COUNTS) {
        ++n_ev;
        n_half += 2;
        add_cnt(p, bins, 0, ce);
      }
    };
    // edges [pj, jhi) under state s (the other pins' bits): a lone edge at
    // either end, whole cycles as run-differences (per cycle the sums of the
    // two edges' contributions; the leakage level steps cancel in a cycle)
    auto pclk_close = [&](uint32_t jhi, uint32_t s) {
      if (jhi <= pj) return;
      uint32_t a = pj, b = jhi;
      pj = jhi;
      const int pk = __ffs(pkbit) - 1;
      const uint32_t oA = s | (pv0 ? pkbit : 0u);
      const uint32_t oB = s | (pv0 ? 0u : pkbit);
      const float eA = in_energy(pk, oA, pv0 == 0);
      const float eB = in_energy(pk, oB, pv0 != 0);
      const float lA = leak_of(oA), lB = leak_of(oB);
      if (a & 1) pclk_edge(a++, eA, eB, lA, lB);
      if (b > a && (b & 1)) pclk_edge(--b, eA, eB, lA, lB);
      if (b > a) {
        const uint32_t k1 = a >> 1, k2 = b >> 1;
        const double n = static_cast<double>(k2 - k1);
        const double dl = static_cast<double>(lB) - static_cast<double>(lA);
        const unsigned long long e2 = to_fx_f(eA, p.fx_dyn_f, p.fx_dyn) + to_fx_f(eB, p.fx_dyn_f, p.fx_dyn);
        const unsigned long long l2 = to_fx(dl * (static_cast<double>(pB - pA) * p.ts), p.fx_leak);
        acc_add(0, n * (static_cast<double>(eA) + static_cast<double>(eB)));
        acc_add(4, n * dl * static_cast<double>(pB - pA));
        unsigned long long* run = bins.s + bins.off;
        if (e2) {
          shared_add64(run + kIntRun * ct + k1, e2);
          if (k2 < ct) shared_add64(run + kIntRun * ct + k2, 0ull - e2);
        }
        if (l2) {
          shared_add64(run + kLeakRun * ct + k1, l2);
          if (k2 < ct) shared_add64(run + kLeakRun * ct + k2, 0ull - l2);
        }
        if (COUNTS) {
          n_ev += 2 * (k2 - k1);
          n_half += 4 * (k2 - k1);
          for (uint32_t k = k1; k < k2; ++k) atomicAdd(bins.sc + k, 2u);
        }
      }
    };
    if (pkbit) {
      // first edge at or after max(s0r, r_exist)
      const uint32_t ph0 = off0 + static_cast<uint32_t>(max(static_cast<int32_t>(s0r), r_exist));
      const uint32_t q0 = udiv32(ph0, tpc32, p.tpc_magic);
      const uint32_t h0 = ph0 - q0 * tpc32;
      pj = 2 * q0 + (h0 > pA ? 1u : 0u) + (h0 > pB ? 1u : 0u);
    }
    if (owns_initial_cell) {
      acc_add(4, static_cast<double>(leak_cur) * static_cast<double>(p.tmax));
      add_bin(p, bins, kLeakLevel, 0, to_fx(static_cast<double>(leak_cur) * P, p.fx_leak));
    }
    // per-cell leakage of a level change at tick t: its level times the
    // ticks to the end of what the walk accounts (time_max, or for a
    // standalone window the end of this part of the tile)
    const int64_t leak_end = standalone ? min(T0 + static_cast<int64_t>(s1r), p.tmax) : p.tmax;
    // standalone: the fixed-point level this part has added, removed
    // exactly (integer for integer) at its end
    unsigned long long lvl_fx = 0ull;
    // drift path: a segment whose seconds cycle precedes its tick cycle
    // needs its end before its correction is known
    bool pend = false;
    int64_t pend_p = 0, pend_c0 = 0;
    float pend_v = 0.0f;
    auto apply_pending = [&](int64_t q) {
      const double ps = static_cast<double>(pend_p) * p.ts;
      const double qs = static_cast<double>(q) * p.ts;
      const double b0 = static_cast<double>(pend_c0) * P;
      const double v = static_cast<double>(pend_v);
      if (qs < b0) {
        add_bin(p, bins, kLeakPart, pend_c0 - 1, to_fx(-v * (qs - ps), p.fx_leak));
      } else {
        add_bin(p, bins, kLeakPart, pend_c0 - 1, to_fx(-v * (b0 - ps), p.fx_leak));
        add_bin(p, bins, kLeakPart, pend_c0, to_fx(v * (b0 - ps), p.fx_leak));
      }
      pend = false;
    };
    // the cell's leakage changes from leak_cur to leak_new at tick cur_abs
    // (tick cycle cyc, tile cycle cq): its share of the cycle the tick lies in
    // (in seconds), the level from the next cycle on, and with DRIFT the
    // correction where the tick and seconds cycles differ
    auto level_change = [&](int64_t cur_abs, int64_t cyc, uint32_t cq, float leak_new) {
      const int64_t s = DRIFT ? seconds_cycle(p, cur_abs, cyc) : cyc;
      if (leak_new != leak_cur) {
        const double dl = static_cast<double>(leak_new) - static_cast<double>(leak_cur);
        const double cur_s = static_cast<double>(cur_abs) * p.ts;
        const double end_s = fmin(static_cast<double>(s + 1) * P, p.tmax_s);
        const unsigned long long lv = to_fx(dl * P, p.fx_leak);
        if (DRIFT) {
          add_bin(p, bins, kLeakPart, s, to_fx(dl * (end_s - cur_s), p.fx_leak));
          add_bin(p, bins, kLeakLevel, s + 1, lv);
        } else {  // s is the tick cycle c_lo + cq
          add_bin_k(p, bins, kLeakPart, cq, to_fx(dl * (end_s - cur_s), p.fx_leak));
          add_bin_k(p, bins, kLeakLevel, cq + 1, lv);
        }
        lvl_fx += lv;
        acc_add(4, dl * static_cast<double>(leak_end - cur_abs));
      }
      if (DRIFT && s != cyc) {
        if (s == cyc + 1) {
          const double w = static_cast<double>(cur_abs) * p.ts - static_cast<double>(cyc + 1) * P;
          const double v = static_cast<double>(leak_new);
          add_bin(p, bins, kLeakPart, cyc, to_fx(-v * w, p.fx_leak));
          add_bin(p, bins, kLeakPart, cyc + 1, to_fx(v * w, p.fx_leak));
        } else {
          pend = true;
          pend_p = cur_abs;
          pend_c0 = cyc;
          pend_v = leak_new;
        }
      }
      leak_cur = leak_new;
    };
    if (standalone) {
      // the leakage of a standalone part starts at its first tick
      const uint32_t k0 = udiv32(s0r + off0, tpc32, p.tpc_magic);
      const float l0 = leak_cur;
      leak_cur = 0.0f;
      level_change(T0 + static_cast<int64_t>(s0r), bins.c_lo + k0, k0, l0);
    }

    while (true) {
      uint32_t cur = kRelInf;
#pragma unroll
      for (int i = 0; i < MAXP; ++i)
        if (i < n_pin) cur = min(cur, nt[i]);
      if (cur >= s1r) break;
      const int64_t cur_abs = T0 + cur;
      const uint32_t cq = udiv32(cur + off0, tpc32, p.tpc_magic);     // cycles after c_lo
      const int64_t cyc = bins.c_lo + cq;
      const int32_t cs_rel = static_cast<int32_t>(cq * tpc32) - static_cast<int32_t>(off0);  // cycle start - T0
      const int32_t ce_rel = cs_rel + static_cast<int32_t>(tpc32);
      // periodic clock: its value before cur (edges strictly before cur)
      const int32_t ph = static_cast<int32_t>(cur) - cs_rel;
      if (pkbit) {
        const bool hi = ph > static_cast<int32_t>(pA) && ph <= static_cast<int32_t>(pB);
        ones = (ones & ~pkbit) | ((hi ? pv0 == 0 : pv0 != 0) ? pkbit : 0u);
      }

      // advance every pin with an event at cur
      const uint32_t old_state = state;
      const uint64_t old_state_hi = state_hi;
      const uint32_t old_ones = ones;
      uint32_t trig = 0;
#pragma unroll
      for (int i = 0; i < MAXP; ++i) {
        if (RING && i < n_pin && nt[i] == cur) {
          const uint32_t h = rs[i] & 0xffu, held = rs[i] >> 8;
          const int v = static_cast<int>((rv[i] >> (2 * h)) & 3u);
          set_v(state, state_hi, i, v);
          ones = (ones & ~(1u << i)) | (v == 1 ? (1u << i) : 0u);
          trig |= 1u << i;
          if (held > 1) {
            rs[i] = (h + 1) | ((held - 1) << 8);
            nt[i] = ring[(i * kRing + h + 1) * nt_blk + threadIdx.x];
          } else if (rem[i] > 0) {
            need |= 1u << i;
            nt[i] = kRelInf;
          } else {
            rs[i] = 0;
            nt[i] = kRelInf;
          }
          if (nt[i] <= cur) { atomicOr(p.status, kErrTimeOrder); nt[i] = kRelInf; rem[i] = 0; rs[i] = 0; }
        } else if (!RING && i < n_pin && nt[i] == cur) {
          const int v = get_v(nvals, nvals_hi, i);
          set_v(state, state_hi, i, v);
          ones = (ones & ~(1u << i)) | (v == 1 ? (1u << i) : 0u);
          trig |= 1u << i;
          ++f[i];
          --rem[i];
          if (rem[i] > 0) {
            const int64_t tn = ev_time(p.ev_t, f[i]);
            if (tn <= cur_abs) { atomicOr(p.status, kErrTimeOrder); nt[i] = kRelInf; rem[i] = 0; }
            else {
              nt[i] = rel(tn);
              if (tn > p.tmax) atomicOr(p.status, kErrTimeRange);
              const int nv = ev_value(p.ev_v, f[i]);
              if (i < 16) nvals = (nvals & ~(3u << (2 * i))) | (static_cast<uint32_t>(nv) << (2 * i));
              else nvals_hi = (nvals_hi & ~(3ull << (2 * (i - 16)))) | (static_cast<uint64_t>(nv) << (2 * (i - 16)));
            }
          } else {
            nt[i] = kRelInf;
          }
        }
      }

      if (RING) do_refills(static_cast<int64_t>(cur));

      // periodic clock: its edges up to cur belong to the run of the old
      // state; the leakage step of the other pins is taken at the clock's
      // value after cur
      if (pkbit) {
        // edges at or before cur, but an absent edge at time_max
        const bool at_end = ((pBv >> 30) & 1u) && cur_abs >= p.tmax;
        const bool hi = at_end ? (ph > static_cast<int32_t>(pA) && ph <= static_cast<int32_t>(pB))
                               : (ph >= static_cast<int32_t>(pA) && ph < static_cast<int32_t>(pB));
        const uint32_t cb = (hi ? pv0 == 0 : pv0 != 0) ? pkbit : 0u;
        ones = (ones & ~pkbit) | cb;
        leak_cur = leak_of((old_ones & ~pkbit) | cb);
        if ((ones ^ old_ones) & ~pkbit) {
          uint32_t jhi = 2 * cq + (ph >= static_cast<int32_t>(pA) ? 1u : 0u) + (ph >= static_cast<int32_t>(pB) ? 1u : 0u);
          if (at_end) jhi = min(jhi, pclk_jend());
          pclk_close(jhi, old_ones & ~pkbit);
        }
      }

      // leakage: level change at cur
      if (DRIFT && pend) apply_pending(cur_abs);
      level_change(cur_abs, cyc, cq, leak_of(ones));

      // energies of the triggered pins, in pin order, from the pre-step state
      uint32_t tb = DYN ? trig : 0u;
      while (tb) {
        const int i = __ffs(tb) - 1;
        tb &= tb - 1;
        const int pv = get_v(old_state, old_state_hi, i);
        const int nv = get_v(state, state_hi, i);
        const int tog2 = ntoggle2(pv, nv);
        const int nr2 = nrise2(pv, nv);
        const bool rise = nr2 > 0;

        // glitch: the event is isolated in its period unless its previous
        // event (strictly before) or its next event shares the period
        float g = -1.0f;
        if (!((clock_mask >> i) & 1)) {
          const bool prev_same = !((at_lo >> i) & 1) && sel<MAXP>(lt, i) >= cs_rel;
          const uint32_t nti = sel<MAXP>(nt, i);
          const bool next_same = nti == kRelBeyond || (nti != kRelInf && static_cast<int32_t>(nti) < ce_rel);
          if ((prev_same || next_same) && p.glitch_pw) {
            const int64_t ev_idx = RING ? sel<MAXP>(f, i) - static_cast<int64_t>(sel<MAXP>(rs, i) >> 8) - 1
                                        : sel<MAXP>(f, i) - 1;
            g = glitch_ratio_of(__ldg(p.glitch_pw + ev_idx), __ldg(p.pin_gden + p0 + i));
          } else if (prev_same || next_same) {
            const int32_t net = __ldg(p.pin_net + p0 + i);
            const int64_t lo = __ldg(p.net_off + net), hi = __ldg(p.net_off + net + 1);
            const int64_t base = p.net_base ? __ldg(p.net_base + net) : 0;
            const int64_t ev_idx = RING ? sel<MAXP>(f, i) - static_cast<int64_t>(sel<MAXP>(rs, i) >> 8) - 1
                                        : sel<MAXP>(f, i) - 1;
            g = glitch_ratio(p, ev_idx, lo, hi, base == 0 ? lo : -1, cur_abs,
                             cyc * p.tpc, __ldg(p.pin_gden + p0 + i));
          }
        }

        float energy = 0.0f;
        if (i < n_in) {
          energy = in_energy(i, old_ones, rise);
        } else {
          const int o = i - n_in;
          float best = p.min_diff0;
          int relq = -1;
          bool rel_rise = false;
          const double cur_s = __dmul_rn(static_cast<double>(cur_abs), p.ts);
          const float* dlp = blk + ty.delay_off + o * n_in * 4 + (rise ? 0 : 1);
#pragma unroll
          for (int q = 0; q < (MAXP < 2 ? 1 : MAXP - 1); ++q) {
            if (q >= n_in) break;
            if (!((has_wave >> q) & 1)) continue;
            int32_t tr = lt[q];
            bool fr = (last_rise >> q) & 1;
            if ((pkbit >> q) & 1) {
              // the periodic clock's last edge strictly before cur, when it
              // lies in the window (else the last event before the window)
              const uint32_t jb = 2 * cq + (ph > static_cast<int32_t>(pA) ? 1u : 0u) + (ph > static_cast<int32_t>(pB) ? 1u : 0u);
              if (jb >= 1) {
                const uint32_t jl = jb - 1;
                const int32_t te = static_cast<int32_t>((jl >> 1) * tpc32) - static_cast<int32_t>(off0) +
                                   static_cast<int32_t>((jl & 1) ? pB : pA);
                if (te >= r_exist) {
                  tr = te;
                  fr = (jl & 1) ? (pv0 != 0) : (pv0 == 0);
                }
              }
            }
            if (tr < cs_rel || tr >= ce_rel) continue;  // the related pin's edge lies in this cycle
            const float dl = dlp[q * 4 + (fr ? 0 : 2)];
            if (isnan(dl)) continue;
            const double trs = __dmul_rn(static_cast<double>(T0 + tr), p.ts);
            const float diff = __double2float_rn(fabs(__dsub_rn(__dsub_rn(cur_s, static_cast<double>(dl)), trs)));
            if (diff < best) {
              best = diff;
              relq = q;
              rel_rise = fr;
            }
          }
          if (relq < 0) {
            energy = blk[ty.def_off + 2 * o + (rise ? 0 : 1)];
          } else if (FAST) {
            const int16_t eo = fast_tab[fo + n_in * n_state + (o * n_in + relq) * n_state + old_ones];
            if (eo >= 0) energy = blk[eo + (rel_rise ? 0 : 2) + (rise ? 0 : 1)];
          } else {
            const int32_t s_begin = __ldg(p.pin_slot + ty.pin_slot_off + i);
            const int32_t s_end = __ldg(p.pin_slot + ty.pin_slot_off + i + 1);
            for (int32_t k = s_begin; k < s_end; ++k) {
              const DevSlot sl = p.slots[k];
              if (sl.related != relq) continue;
              if (when_holds(p.cubes, sl.cube_off, sl.n_cube, old_ones)) {
                energy = blk[sl.e_off + (rel_rise ? 0 : 2) + (rise ? 0 : 1)];
                break;
              }
            }
          }
          if (COUNTS) n_rel += static_cast<uint32_t>(relq + 1);
          // switching: n_rise * C * V^2
          if (nr2 > 0) {
            const float esw = __fmul_rn(nr2 == 2 ? 1.0f : 0.5f, __ldg(p.pin_swe + p0 + i));
            if (g > 0.0f) {
              const float x = __fmul_rn(g, esw);
              acc_add(3, x);
              add_bin_k(p, bins, kGSw, cq, to_fx_f(x, p.fx_dyn_f, p.fx_dyn));
            } else {
              acc_add(2, esw);
              add_bin_k(p, bins, kSw, cq, to_fx_f(esw, p.fx_dyn_f, p.fx_dyn));
            }
          }
        }
        energy = __fmul_rn(energy, tog2 == 2 ? 1.0f : (tog2 == 1 ? 0.5f : 0.0f));
        if (g > 0.0f) {
          const float x = __fmul_rn(g, energy);
          acc_add(1, x);
          add_bin_k(p, bins, kGInt, cq, to_fx_f(x, p.fx_dyn_f, p.fx_dyn));
          if (COUNTS) { ++n_gl; add_cnt(p, bins, 1, cyc); }
        } else {
          acc_add(0, energy);
          add_bin_k(p, bins, kInt, cq, to_fx_f(energy, p.fx_dyn_f, p.fx_dyn));
        }
        if (COUNTS) {
          ++n_ev;
          n_half += static_cast<uint32_t>(tog2);
          add_cnt(p, bins, 0, cyc);
        }
      }
      // the triggered pins' last event is now cur
#pragma unroll
      for (int i = 0; i < MAXP; ++i) {
        if ((trig >> i) & 1) {
          const bool r = !((at_lo >> i) & 1) &&
                         nrise2(get_v(old_state, old_state_hi, i), get_v(state, state_hi, i)) > 0;
          last_rise = (last_rise & ~(1u << i)) | (r ? (1u << i) : 0u);
          lt[i] = static_cast<int32_t>(cur);
        }
      }
      at_lo &= ~trig;
    }

    if (pkbit) pclk_close(pclk_jend(), ones & ~pkbit);
    // ... and ends at its last tick, unless that lies past time_max: the
    // level it added is taken back integer for integer, from the cycle the
    // tick starts (without drift, on a cycle boundary) or from the next one,
    // after the rest of the tick's cycle at the final level
    if (standalone && T0 + static_cast<int64_t>(s1r) <= p.tmax) {
      const int64_t t1 = T0 + static_cast<int64_t>(s1r);
      if (DRIFT && pend) apply_pending(t1);
      const uint32_t k = udiv32(s1r + off0, tpc32, p.tpc_magic);
      const uint32_t h = s1r + off0 - k * tpc32;
      const int64_t cyc1 = bins.c_lo + k;
      const int64_t s1 = DRIFT ? seconds_cycle(p, t1, cyc1) : cyc1;
      if (!DRIFT && h == 0) {
        add_bin_k(p, bins, kLeakLevel, k, 0ull - lvl_fx);
      } else {
        const double cur_s = static_cast<double>(t1) * p.ts;
        const double end_s = fmin(static_cast<double>(s1 + 1) * P, p.tmax_s);
        add_bin(p, bins, kLeakPart, s1, to_fx(-static_cast<double>(leak_cur) * (end_s - cur_s), p.fx_leak));
        add_bin(p, bins, kLeakLevel, s1 + 1, 0ull - lvl_fx);
      }
      leak_cur = 0.0f;
    }

    if (DRIFT && pend) {
      // end of the pending segment: the cell's next event, or time_max
      int64_t q = p.tmax;
#pragma unroll
      for (int i = 0; i < MAXP; ++i)
        if (i < n_pin && nt[i] != kRelInf)
          q = min(q, ev_time(p.ev_t, RING ? f[i] - static_cast<int64_t>(rs[i] >> 8) : f[i]));
      apply_pending(q);
    }

    // flush the cell's sums for this tile
    const int64_t nc = p.n_cell;
#pragma unroll
    for (int q = 0; q < kNumCellAcc; ++q) {
      const double a = RUNS ? s_acc[q] : acc_r[q];
      if (a != 0) atomicAdd(p.cell_acc + q * nc + cell, a);
    }
    if (COUNTS) {
      if (n_ev) atomicAdd(p.cnt_cell + 0 * nc + cell, n_ev);
      if (n_gl) atomicAdd(p.cnt_cell + 1 * nc + cell, n_gl);
      if (n_half) atomicAdd(p.cnt_cell + 2 * nc + cell, n_half);
      if (n_rel) atomicAdd(p.cnt_cell + 3 * nc + cell, n_rel);
    }
  }
  if (!split) break;
  }

  __syncthreads();
  // clock runs: run-differences -> per-cycle sums
  if (runs_on) {
    for (int set = 0; set < nset; ++set) {
      block_inclusive_scan(smem + static_cast<int64_t>(set) * nslot * ct + kIntRun * ct, ct, s_wsum);
      block_inclusive_scan(smem + static_cast<int64_t>(set) * nslot * ct + kLeakRun * ct, ct, s_wsum);
    }
  }
  // flush the tile's per-cycle bins
  const int64_t stride = p.n_period + 1;
  for (int64_t k = threadIdx.x; k < ct; k += blockDim.x) {
    const int64_t c = bins.c_lo + k;
    const int64_t cc = c < p.n_period ? c : p.n_period;
#pragma unroll
    for (int q = 0; q < kNumCycAcc; ++q) {
      unsigned long long x0 = smem[q * ct + k];
      unsigned long long x1 = nset == 2 ? smem[(nslot + q) * ct + k] : 0ull;
      if (runs_on && (q == kInt || q == kLeakPart)) {
        const int r = q == kInt ? kIntRun : kLeakRun;
        x0 += smem[r * ct + k];
        if (nset == 2) x1 += smem[(nslot + r) * ct + k];
      }
      if (x0 + x1) atomicAdd(p.cyc_acc + q * stride + cc, x0 + x1);
      if (p.cyc_acc_g) {
        if (x0) atomicAdd(p.cyc_acc_g + (static_cast<int64_t>(g_first) * kNumCycAcc + q) * stride + cc, x0);
        if (x1) atomicAdd(p.cyc_acc_g + (static_cast<int64_t>(g_first + 1) * kNumCycAcc + q) * stride + cc, x1);
      }
    }
    if (COUNTS) {
      const uint32_t a = bins.sc[k], b2 = bins.sc[ct + k];
      if (a) atomicAdd(p.cnt_cyc + 0 * stride + cc, static_cast<unsigned long long>(a));
      if (b2) atomicAdd(p.cnt_cyc + 1 * stride + cc, static_cast<unsigned long long>(b2));
    }
  }
}

// ---- the warp walk: one warp per cell and cycle tile ----
//
// Cells of up to kFastPins pins without drift (most of a standard-cell
// netlist) are walked by one warp each, 32 events at a time in time order,
// so that the per-event work runs on full lanes instead of one lane per
// cell. Per chunk of up to 32 events:
//   - each pin's next 32 events are loaded (coalesced) into a per-warp window
//     in shared memory as keys (t - T0) << 8 | pin << 5 | slot, which order
//     events by time, then by pin (same-time events in pin order);
//   - a merge-path search over the windows gives lane k the cell's k-th
//     next event;
//   - the ticks with several events (time groups) come from a ballot; the
//     pre-step value of each pin for lane k is that of the pin's last event
//     before k's group (a ballot per pin and a shuffle), else the value
//     carried from the previous chunk, and so is the related input's last
//     edge for an output event;
//   - the leakage level changes once per time group (its last lane), the
//     energies once per event, with the walk's fixed-point bins and rules;
//     periodic clock pins are closed as runs by the lanes where the other
//     pins' state changes.
// The results are the per-thread walk's (walk_block): the same integer
// per-cycle terms, per-cell FP64 sums in another order.

constexpr unsigned long long kKeyInf = ~0ull;
// per-warp window: keys [kFastPins][32], merge scratch [2][32], values [kFastPins][32]
constexpr int kWarpWinBytes = kFastPins * 32 * 8 + 2 * 32 * 8 + kFastPins * 32;

__device__ __forceinline__ unsigned lanes_below(int k) { return (1u << k) - 1u; }       // k in [0, 31]
__device__ __forceinline__ unsigned lanes_upto(int k) { return 0xffffffffu >> (31 - k); }  // k in [0, 31]

// Lane k's element of the first 32 of the merge of A[0, 32) and B[0, 32)
// (ascending, distinct keys, padded with kKeyInf): the split a of the
// merge path with A[a - 1] < B[k - a] and B[k - a - 1] < A[a].
__device__ __forceinline__ unsigned long long merge32(const unsigned long long* A, const unsigned long long* B,
                                                      int k) {
  int lo = 0, hi = k;
#pragma unroll
  for (int s = 0; s < 5; ++s) {   // hi - lo <= 31 halves to 0 in 5 steps
    if (lo < hi) {
      const int m = (lo + hi) >> 1;
      if (A[m] < B[k - 1 - m]) lo = m + 1; else hi = m;
    }
  }
  const unsigned long long x = A[lo], y = B[k - lo];
  return x < y ? x : y;
}

// Bytes of one warp's shared-memory region: the window, then its copy of
// the cell's instance block.
__host__ __device__ __forceinline__ int warp_region_bytes(int inst_stride) {
  return kWarpWinBytes + ((inst_stride * 4 + 15) / 16) * 16;
}

// One work item of the warp walk: cells order[order_begin + gblk *
// gates_per_block ...] (one warp each, in turn) over tile `tile`. All
// threads of the block call it together.
template <bool COUNTS, bool RUNS>
__device__ __forceinline__ void warp_walk_block(const KParams& p, const int gblk, const int tile,
                                                unsigned long long* smem) {
  const int64_t ct = p.cycles_per_tile;
  const int nset = p.cell_cgroup ? 2 : 1;
  const bool runs_on = RUNS && p.pclk != nullptr;
  const int nslot = runs_on ? kNumBinSlotsRun : kNumCycAcc;
  __shared__ unsigned long long s_wsum[32];
  Bins bins;
  bins.s = smem;
  bins.sc = reinterpret_cast<uint32_t*>(smem + nset * nslot * ct);
  bins.off = 0;
  bins.g = 0;
  const int2 tdesc = p.tiles ? p.tiles[tile] : make_int2(0, 0);
  bins.c_lo = p.tiles ? static_cast<int64_t>(tdesc.x) : p.cyc0 + static_cast<int64_t>(tile) * ct;
  const int64_t ct_tile = p.tiles ? static_cast<int64_t>(tdesc.y) : ct;
  bins.ct = ct;
  for (int64_t k = threadIdx.x; k < nset * nslot * ct; k += blockDim.x) smem[k] = 0ull;
  if (COUNTS)
    for (int64_t k = threadIdx.x; k < 2 * ct; k += blockDim.x) bins.sc[k] = 0u;
  // the per-type tables when they fit, then the warps' regions
  uint8_t* after_bins = reinterpret_cast<uint8_t*>(smem + nset * nslot * ct + (COUNTS ? ct : 0));
  const int16_t* fast_tab = p.fast_tab;
  const float* leak_pool = p.leak_pool;
  int tab_bytes = 0;
  if (p.tabs_in_smem) {
    float* s_leak = reinterpret_cast<float*>(after_bins);
    int16_t* s_fast = reinterpret_cast<int16_t*>(s_leak + p.n_leak_pool);
    for (int k = threadIdx.x; k < p.n_leak_pool; k += blockDim.x) s_leak[k] = __ldg(p.leak_pool + k);
    for (int k = threadIdx.x; k < p.n_fast_tab; k += blockDim.x) s_fast[k] = __ldg(p.fast_tab + k);
    leak_pool = s_leak;
    fast_tab = s_fast;
    tab_bytes = ((p.n_leak_pool * 4 + p.n_fast_tab * 2 + 15) / 16) * 16;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, n_warp = blockDim.x >> 5;
  uint8_t* wreg = after_bins + tab_bytes + warp * warp_region_bytes(p.fast_inst_stride);
  unsigned long long* wkey = reinterpret_cast<unsigned long long*>(wreg);   // [kFastPins][32]
  unsigned long long* wm0 = wkey + kFastPins * 32;                          // [32]
  unsigned long long* wm1 = wm0 + 32;                                       // [32]
  uint8_t* wval = reinterpret_cast<uint8_t*>(wm1 + 32);                     // [kFastPins][32]
  float* winst = reinterpret_cast<float*>(wreg + kWarpWinBytes);
  __syncthreads();

  // tile window in ticks: [T0, T0 + span)
  const int64_t T0 = max(p.t_lo, bins.c_lo * p.tpc);
  const uint32_t off0 = static_cast<uint32_t>(T0 - bins.c_lo * p.tpc);
  const uint32_t tpc32 = static_cast<uint32_t>(p.tpc);
  const int64_t t_end = (bins.c_lo + ct_tile) * p.tpc;
  const int64_t T1 = t_end > p.tmax ? min(p.t_hi, p.tmax + 1) : min(p.t_hi, t_end);
  const uint32_t span = static_cast<uint32_t>(T1 > T0 ? T1 - T0 : 0);
  const bool standalone = p.standalone != 0;
  const bool owns_initial = !standalone && bins.c_lo == 0 && (p.t_lo == 0);
  const double P = p.period_d;
  int32_t r_exist = 0;
  if (runs_on) {
    const int64_t tl = max(p.t_lo, static_cast<int64_t>(1)) - T0;
    r_exist = static_cast<int32_t>(max(tl, -static_cast<int64_t>(INT32_MAX / 2)));
  }
  const int64_t leak_end = standalone ? min(T0 + static_cast<int64_t>(span), p.tmax) : p.tmax;
  const bool table_next = p.tile_first && !p.tiles && tile + 1 < p.n_tiles;
  const int32_t cb0 = p.order_begin + gblk * p.gates_per_block;
  const int32_t ce0 = min(p.order_end, cb0 + p.gates_per_block);
  const int32_t g_first = (p.cell_cgroup && cb0 < ce0) ? __ldg(p.cell_cgroup + __ldg(p.order + cb0)) : 0;
  const unsigned FULL = 0xffffffffu;

  for (int32_t it = cb0 + warp; it < ce0; it += n_warp) {
    const int32_t cell = __ldg(p.order + it);
    if (p.cell_cgroup) {
      bins.g = __ldg(p.cell_cgroup + cell);
      const int32_t set = bins.g - g_first;
      bins.off = (set == 0 || set == 1) ? static_cast<int64_t>(set) * nslot * ct : -1;
    }
    const int32_t p0 = __ldg(p.cell_pin_off + cell);
    const int32_t type = __ldg(p.cell_type + cell);
    const DevType ty = p.types[type];
    const int n_pin = ty.n_pin, n_in = ty.n_in;
    const int n_state = 1 << n_pin;
    const int32_t fo = __ldg(p.type_fast_off + type);
    {
      const float* __restrict__ src = p.inst + __ldg(p.cell_inst + cell);
      for (int k = lane; k < ty.inst_floats; k += 32) winst[k] = __ldg(src + k);
    }
    __syncwarp();
    const float* blk = winst;

    // pin lanes: lane i < n_pin sets up pin i (the walk's per-pin setup)
    int64_t my_c = 0, my_h = 0;
    int my_v = 0;
    int32_t my_lt = kFarBefore;
    bool my_rise = false, my_atlo = false, my_wave = false, my_clk = false, my_pk = false;
    int2 my_pc = make_int2(-1, 0);
    if (lane < n_pin) {
      const int32_t net = __ldg(p.pin_net + p0 + lane);
      const uint8_t pf = __ldg(p.pin_flags + p0 + lane);
      my_v = pf & 3;
      if (pf & 4) {
        my_clk = true;
        if (runs_on && net >= 0 && bins.off >= 0) {
          my_pc = __ldg(p.pclk + net);
          my_pk = my_pc.x >= 0;
        }
      }
      if (net >= 0) {
        const int64_t a = __ldg(p.net_off + net), e = __ldg(p.net_off + net + 1);
        if (a < 0 || e < a || e > p.n_event) {
          atomicOr(p.status, kErrNetRange);
        } else if (e > a) {
          my_wave = true;
          const int64_t base = p.net_base ? __ldg(p.net_base + net) : 0;
          int64_t l = a;
          if (p.tile_first) {
            l = a + __ldg(p.tile_first + static_cast<int64_t>(tile) * p.n_net + net);
          } else {
            l = lower_bound_time(p.ev_t, a, e, T0);
          }
          if (l < e && l == a && base == 0 && ev_time(p.ev_t, l) == 0) ++l;
          if (l > a) {
            my_v = ev_value(p.ev_v, l - 1);
          } else {
            my_v = 2;
            if (base != 0) atomicOr(p.status, kErrContext);
            my_atlo = true;
          }
          const int64_t re = l > a ? l - 1 : a;
          const int64_t pe = re > a ? re - 1 : a;
          const int64_t tre = ev_time(p.ev_t, re) - T0;
          my_lt = static_cast<int32_t>(tre < kFarBefore ? kFarBefore : (tre > INT32_MAX / 2 ? INT32_MAX / 2 : tre));
          my_rise = nrise2(ev_value(p.ev_v, pe), ev_value(p.ev_v, re)) > 0;
          int64_t h = table_next ? a + __ldg(p.tile_first + static_cast<int64_t>(tile + 1) * p.n_net + net)
                                 : lower_bound_time(p.ev_t, l, e, T1);
          if (h < l) h = l;
          if (h < e && ev_time(p.ev_t, h) > p.tmax) atomicOr(p.status, kErrTimeRange);
          my_c = l;
          my_h = h;
        }
      }
    }
    // the cell's periodic clock pin (at most one, the first): not merged
    const unsigned pk_cand = __ballot_sync(FULL, my_pk);
    const int pk = (RUNS && pk_cand) ? __ffs(pk_cand) - 1 : -1;
    const uint32_t pkbit = (RUNS && pk >= 0) ? (1u << pk) : 0u;
    const int pc_src = pk >= 0 ? pk : 0;
    const uint32_t pA = static_cast<uint32_t>(__shfl_sync(FULL, my_pc.x, pc_src));
    const uint32_t pBv = static_cast<uint32_t>(__shfl_sync(FULL, my_pc.y, pc_src));
    if (lane == pk) my_h = my_c;
    const unsigned has_wave = __ballot_sync(FULL, my_wave);
    const unsigned clock_mask = __ballot_sync(FULL, my_clk);
    unsigned at_lo = __ballot_sync(FULL, my_atlo);
    unsigned last_rise = __ballot_sync(FULL, my_rise);
    // carried 2-bit values of the pins, and the events still to walk
    uint32_t cst = __reduce_or_sync(FULL, lane < n_pin ? static_cast<uint32_t>(my_v) << (2 * lane) : 0u);
    uint32_t n_left = __reduce_add_sync(FULL, lane < n_pin ? static_cast<uint32_t>(my_h - my_c) : 0u);
    // every lane holds each pin's cursor, end and last event time
    int64_t cur_c[kFastPins], end_h[kFastPins];
    int32_t last_t[kFastPins];
#pragma unroll
    for (int j = 0; j < kFastPins; ++j) {
      cur_c[j] = __shfl_sync(FULL, my_c, j);
      end_h[j] = __shfl_sync(FULL, my_h, j);
      last_t[j] = __shfl_sync(FULL, my_lt, j);
    }
    auto ones_of = [&](uint32_t s) -> uint32_t {
      uint32_t o = 0;
#pragma unroll
      for (int j = 0; j < kFastPins; ++j)
        if (((s >> (2 * j)) & 3u) == 1u) o |= 1u << j;
      return o;
    };
    const float leak_const = ty.leak_const;
    const int32_t leak_off = ty.leak_off;
    auto leak_of = [&](uint32_t o) -> float { return leak_off >= 0 ? leak_pool[leak_off + o] : leak_const; };
    auto in_energy = [&](int i, uint32_t oo, bool rise) -> float {
      const int16_t eo = fast_tab[fo + i * n_state + oo];
      return eo >= 0 ? blk[eo + (rise ? 0 : 1)] : 0.0f;
    };
    double acc[kNumCellAcc] = {0.0, 0.0, 0.0, 0.0, 0.0};
    uint32_t n_ev = 0, n_gl = 0, n_half = 0, n_rel = 0;
    unsigned long long lvl = 0ull;   // fixed-point level this lane added (standalone end)
    const uint32_t pB = pBv & 0x3fffffffu;
    const int pv0 = static_cast<int>(pBv >> 31);
    // clock runs, as the per-thread walk's pclk_jend / pclk_edge / pclk_close
    auto pclk_jend = [&]() -> uint32_t {
      const int64_t r_end = ((pBv >> 30) & 1u) ? min(static_cast<int64_t>(span), p.tmax - T0) : static_cast<int64_t>(span);
      if (r_end <= 0) return 0u;
      const uint32_t ce = udiv32(static_cast<uint32_t>(r_end - 1) + off0, tpc32, p.tpc_magic);
      const int32_t he = static_cast<int32_t>(static_cast<uint32_t>(r_end - 1) + off0 - ce * tpc32);
      return 2 * ce + (he >= static_cast<int32_t>(pA) ? 1u : 0u) + (he >= static_cast<int32_t>(pB) ? 1u : 0u);
    };
    auto pclk_edge = [&](uint32_t j, float eA, float eB, float lA, float lB) {
      const int64_t ce = bins.c_lo + (j >> 1);
      const int64_t te = T0 + static_cast<int64_t>(static_cast<int32_t>((j >> 1) * tpc32) - static_cast<int32_t>(off0) +
                                                   static_cast<int32_t>((j & 1) ? pB : pA));
      const bool ea = !(j & 1);
      const float en = ea ? eA : eB;
      acc[0] += en;
      add_bin_k(p, bins, kInt, j >> 1, to_fx_f(en, p.fx_dyn_f, p.fx_dyn));
      const double dl = ea ? static_cast<double>(lB) - static_cast<double>(lA)
                           : static_cast<double>(lA) - static_cast<double>(lB);
      if (dl != 0.0) {
        const double cur_s = static_cast<double>(te) * p.ts;
        const double end_s = fmin(static_cast<double>(ce + 1) * P, p.tmax_s);
        add_bin_k(p, bins, kLeakPart, j >> 1, to_fx(dl * (end_s - cur_s), p.fx_leak));
        add_bin_k(p, bins, kLeakLevel, (j >> 1) + 1, to_fx(dl * P, p.fx_leak));
        acc[4] += dl * static_cast<double>(p.tmax - te);
      }
      if (COUNTS) {
        ++n_ev;
        n_half += 2;
        add_cnt(p, bins, 0, ce);
      }
    };
    // edges [a, b) under the other pins' state s
    auto pclk_run = [&](uint32_t a, uint32_t b, uint32_t s) {
      if (b <= a) return;
      const uint32_t oA = s | (pv0 ? pkbit : 0u);
      const uint32_t oB = s | (pv0 ? 0u : pkbit);
      const float eA = in_energy(pk, oA, pv0 == 0);
      const float eB = in_energy(pk, oB, pv0 != 0);
      const float lA = leak_of(oA), lB = leak_of(oB);
      if (a & 1) pclk_edge(a++, eA, eB, lA, lB);
      if (b > a && (b & 1)) pclk_edge(--b, eA, eB, lA, lB);
      if (b > a) {
        const uint32_t k1 = a >> 1, k2 = b >> 1;
        const double n = static_cast<double>(k2 - k1);
        const double dl = static_cast<double>(lB) - static_cast<double>(lA);
        const unsigned long long e2 = to_fx_f(eA, p.fx_dyn_f, p.fx_dyn) + to_fx_f(eB, p.fx_dyn_f, p.fx_dyn);
        const unsigned long long l2 = to_fx(dl * (static_cast<double>(pB - pA) * p.ts), p.fx_leak);
        acc[0] += n * (static_cast<double>(eA) + static_cast<double>(eB));
        acc[4] += n * dl * static_cast<double>(pB - pA);
        unsigned long long* run = bins.s + bins.off;
        if (e2) {
          shared_add64(run + kIntRun * ct + k1, e2);
          if (k2 < ct) shared_add64(run + kIntRun * ct + k2, 0ull - e2);
        }
        if (l2) {
          shared_add64(run + kLeakRun * ct + k1, l2);
          if (k2 < ct) shared_add64(run + kLeakRun * ct + k2, 0ull - l2);
        }
        if (COUNTS) {
          n_ev += 2 * (k2 - k1);
          n_half += 4 * (k2 - k1);
          for (uint32_t k = k1; k < k2; ++k) atomicAdd(bins.sc + k, 2u);
        }
      }
    };
    uint32_t pj = 0;   // next clock edge of the tile not yet accounted
    if (pkbit) {
      const uint32_t ph0 = off0 + static_cast<uint32_t>(max(0, r_exist));
      const uint32_t q0 = udiv32(ph0, tpc32, p.tpc_magic);
      const uint32_t h0 = ph0 - q0 * tpc32;
      pj = 2 * q0 + (h0 > pA ? 1u : 0u) + (h0 > pB ? 1u : 0u);
    }
    const float leak0 = leak_of(ones_of(cst));
    if (lane == 0) {
      if (owns_initial) {
        acc[4] += static_cast<double>(leak0) * static_cast<double>(p.tmax);
        add_bin(p, bins, kLeakLevel, 0, to_fx(static_cast<double>(leak0) * P, p.fx_leak));
      }
      if (standalone && leak0 != 0.0f) {
        // the leakage of a standalone part starts at its first tick
        const uint32_t k0 = udiv32(off0, tpc32, p.tpc_magic);
        const double dl = static_cast<double>(leak0);
        const double cur_s = static_cast<double>(T0) * p.ts;
        const double end_s = fmin(static_cast<double>(bins.c_lo + k0 + 1) * P, p.tmax_s);
        const unsigned long long lv = to_fx(dl * P, p.fx_leak);
        add_bin_k(p, bins, kLeakPart, k0, to_fx(dl * (end_s - cur_s), p.fx_leak));
        add_bin_k(p, bins, kLeakLevel, k0 + 1, lv);
        lvl += lv;
        acc[4] += dl * static_cast<double>(leak_end - T0);
      }
    }

    while (n_left > 0) {
      // 1. each pin's next 32 events into the window, as ordered keys
#pragma unroll
      for (int i = 0; i < kFastPins; ++i) {
        if (i >= n_pin) break;
        const int64_t ci = cur_c[i];
        const int64_t hi_i = end_h[i];
        const int32_t lt_i = last_t[i];
        const int64_t idx = ci + lane;
        unsigned long long kk = kKeyInf;
        uint8_t vv = 0;
        int32_t rt = 0;
        if (idx < hi_i) {
          rt = static_cast<int32_t>(ev_time(p.ev_t, idx) - T0);
          kk = (static_cast<unsigned long long>(static_cast<uint32_t>(rt)) << 8) |
               (static_cast<unsigned long long>(i) << 5) | static_cast<unsigned long long>(lane);
          vv = static_cast<uint8_t>(ev_value(p.ev_v, idx));
        }
        const int32_t rprev = __shfl_up_sync(FULL, rt, 1);
        if (idx < hi_i && ((lane > 0 && rprev >= rt) || (lane == 0 && !((at_lo >> i) & 1u) && rt <= lt_i)))
          atomicOr(p.status, kErrTimeOrder);
        wkey[i * 32 + lane] = kk;
        wval[i * 32 + lane] = vv;
      }
      __syncwarp();
      // 2. lane k's event: the k-th of the merged windows
      uint32_t am = 0;
      for (int i = 0; i < n_pin; ++i)
        if (wkey[i * 32] != kKeyInf) am |= 1u << i;
      const int na = __popc(am);
      if (na == 0) break;
      const int q0 = __ffs(am) - 1;
      const uint32_t am1 = am & (am - 1);
      const int q1 = am1 ? __ffs(am1) - 1 : q0;
      const uint32_t am2 = am1 & (am1 - 1);
      const int q2 = am2 ? __ffs(am2) - 1 : q0;
      const uint32_t am3 = am2 & (am2 - 1);
      const int q3 = am3 ? __ffs(am3) - 1 : q0;
      // merge rounds: (q0, q1); then (m0, q2), or (q2, q3) and (m0, m1)
      unsigned long long K = wkey[q0 * 32 + lane];
      for (int r = 0; r < na - 1; ++r) {
        const unsigned long long* A = r == 0 ? wkey + q0 * 32 : (na == 4 && r == 1 ? wkey + q2 * 32 : wm0);
        const unsigned long long* B = r == 0 ? wkey + q1 * 32 : (na == 4 ? (r == 1 ? wkey + q3 * 32 : wm1) : wkey + q2 * 32);
        unsigned long long* out = r == na - 2 ? nullptr : (r == 0 ? wm0 : wm1);
        const unsigned long long v = merge32(A, B, lane);
        if (out) {
          out[lane] = v;
          __syncwarp();
        } else {
          K = v;
        }
      }
      const bool valid0 = K != kKeyInf;
      int n_use = __popc(__ballot_sync(FULL, valid0));   // a prefix of the lanes
      const uint32_t rel = valid0 ? static_cast<uint32_t>(K >> 8) : 0u;
      const int pin = valid0 ? static_cast<int>((K >> 5) & 3u) : 0;
      const int slot = static_cast<int>(K & 31u);
      // a time group that continues past lane 31 is left to the next chunk
      if (n_use == 32) {
        const uint32_t t31 = __shfl_sync(FULL, rel, 31);
        bool more = false;
        for (int i = 0; i < n_pin; ++i) {
          const int ui = __popc(__ballot_sync(FULL, pin == i));
          if (ui < 32) {
            const unsigned long long kn = wkey[i * 32 + ui];
            if (kn != kKeyInf && static_cast<uint32_t>(kn >> 8) == t31) more = true;
          }
        }
        if (more) {
          const uint32_t rp = __shfl_up_sync(FULL, rel, 1);
          const unsigned gm = __ballot_sync(FULL, lane == 0 || rel != rp);
          const int k31 = 31 - __clz(gm);
          if (k31 > 0) n_use = k31;
        }
      }
      const bool valid = lane < n_use;
      // 3. time groups: [k0, k1] are the lanes of this lane's tick
      const uint32_t relp = __shfl_up_sync(FULL, rel, 1);
      const unsigned gmask = __ballot_sync(FULL, valid && (lane == 0 || rel != relp));
      const int k0 = valid ? 31 - __clz(gmask & lanes_upto(lane)) : lane;
      const unsigned gafter = gmask & ~lanes_upto(lane);
      const int k1 = valid ? (gafter ? __ffs(gafter) - 2 : n_use - 1) : lane;
      const int nv = valid ? static_cast<int>(wval[pin * 32 + slot]) : 0;
      // pre-step (before the tick) and post-step (after it) pin values
      unsigned pm[kFastPins];
#pragma unroll
      for (int j = 0; j < kFastPins; ++j) pm[j] = __ballot_sync(FULL, valid && pin == j);
      uint32_t opre = 0, opost = 0;
      int pv = 2;
#pragma unroll
      for (int j = 0; j < kFastPins; ++j) {
        const unsigned xj = pm[j] & lanes_below(k0);
        const unsigned yj = pm[j] & lanes_upto(k1);
        const int vx = __shfl_sync(FULL, nv, xj ? 31 - __clz(xj) : 0);
        const int vy = __shfl_sync(FULL, nv, yj ? 31 - __clz(yj) : 0);
        const int cj = static_cast<int>((cst >> (2 * j)) & 3u);
        const int vpre = xj ? vx : cj;
        const int vpost = yj ? vy : cj;
        if (vpre == 1) opre |= 1u << j;
        if (vpost == 1) opost |= 1u << j;
        if (j == pin) pv = vpre;
      }
      const int tog2 = ntoggle2(pv, nv);
      const int nr2 = nrise2(pv, nv);
      const bool rise = nr2 > 0;
      // the rise flag an output's related-pin choice reads: false for a pin's
      // first event after an unknown start
      const bool first_of_pin = (sel<kFastPins>(pm, pin) & lanes_below(lane)) == 0;
      const int rflag = (valid && rise && !(((at_lo >> pin) & 1u) && first_of_pin)) ? 1 : 0;
      // each input's last event strictly before the tick
      int32_t trq[kFastPins - 1];
      int frq[kFastPins - 1];
#pragma unroll
      for (int q = 0; q < kFastPins - 1; ++q) {
        const unsigned xq = pm[q] & lanes_below(k0);
        const int sq = xq ? 31 - __clz(xq) : 0;
        const int32_t tx = __shfl_sync(FULL, static_cast<int32_t>(rel), sq);
        const int rx = __shfl_sync(FULL, rflag, sq);
        trq[q] = xq ? tx : last_t[q];
        frq[q] = xq ? rx : static_cast<int>((last_rise >> q) & 1u);
      }
      const int64_t cpin = sel<kFastPins>(cur_c, pin);
      const uint32_t cq = udiv32(rel + off0, tpc32, p.tpc_magic);
      const int64_t cyc = bins.c_lo + cq;
      const int32_t cs_rel = static_cast<int32_t>(cq * tpc32) - static_cast<int32_t>(off0);
      const int32_t ce_rel = cs_rel + static_cast<int32_t>(tpc32);
      const int64_t cur_abs = T0 + static_cast<int64_t>(rel);
      const int32_t ph = static_cast<int32_t>(rel) - cs_rel;
      // the periodic clock's value before and after the tick, from its phase
      uint32_t o_e = opre;   // the energies' pre-step state
      float l_old, l_new;
      bool closing = false;
      uint32_t jhi = 0;
      if (pkbit) {
        const bool hb = ph > static_cast<int32_t>(pA) && ph <= static_cast<int32_t>(pB);
        const uint32_t cbb = (hb ? pv0 == 0 : pv0 != 0) ? pkbit : 0u;
        const bool at_end = ((pBv >> 30) & 1u) && cur_abs >= p.tmax;
        const bool ha = at_end ? (ph > static_cast<int32_t>(pA) && ph <= static_cast<int32_t>(pB))
                               : (ph >= static_cast<int32_t>(pA) && ph < static_cast<int32_t>(pB));
        const uint32_t cba = (ha ? pv0 == 0 : pv0 != 0) ? pkbit : 0u;
        o_e = (opre & ~pkbit) | cbb;
        l_old = leak_of((opre & ~pkbit) | cba);
        l_new = leak_of((opost & ~pkbit) | cba);
        closing = valid && lane == k1 && ((opost ^ opre) & ~pkbit) != 0;
        jhi = 2 * cq + (ph >= static_cast<int32_t>(pA) ? 1u : 0u) + (ph >= static_cast<int32_t>(pB) ? 1u : 0u);
        if (at_end) jhi = min(jhi, pclk_jend());
      } else {
        l_old = leak_of(opre);
        l_new = leak_of(opost);
      }
      // 4. leakage: the level changes once per tick, at its last lane
      if (valid && lane == k1 && l_new != l_old) {
        const double dl = static_cast<double>(l_new) - static_cast<double>(l_old);
        const double cur_s = static_cast<double>(cur_abs) * p.ts;
        const double end_s = fmin(static_cast<double>(cyc + 1) * P, p.tmax_s);
        const unsigned long long lv = to_fx(dl * P, p.fx_leak);
        add_bin_k(p, bins, kLeakPart, cq, to_fx(dl * (end_s - cur_s), p.fx_leak));
        add_bin_k(p, bins, kLeakLevel, cq + 1, lv);
        lvl += lv;
        acc[4] += dl * static_cast<double>(leak_end - cur_abs);
      }
      // the clock's edges up to a tick where the other pins change belong to
      // the run of their state before it
      if (pkbit) {
        const unsigned cm = __ballot_sync(FULL, closing);
        const unsigned before = cm & lanes_below(lane);
        const uint32_t jprev = __shfl_sync(FULL, jhi, before ? 31 - __clz(before) : 0);
        if (closing) pclk_run(before ? jprev : pj, jhi, opre & ~pkbit);
        if (cm) pj = max(pj, __shfl_sync(FULL, jhi, 31 - __clz(cm)));
      }
      // the periodic clock's last edge strictly before the tick, when it lies
      // in the window (else the last event before the window)
      int32_t tr_clk = 0;
      bool fr_clk = false, has_clk = false;
      if (pkbit) {
        const uint32_t jb = 2 * cq + (ph > static_cast<int32_t>(pA) ? 1u : 0u) + (ph > static_cast<int32_t>(pB) ? 1u : 0u);
        if (jb >= 1) {
          const uint32_t jl = jb - 1;
          const int32_t te = static_cast<int32_t>((jl >> 1) * tpc32) - static_cast<int32_t>(off0) +
                             static_cast<int32_t>((jl & 1) ? pB : pA);
          if (te >= r_exist) {
            tr_clk = te;
            fr_clk = (jl & 1) ? (pv0 != 0) : (pv0 == 0);
            has_clk = true;
          }
        }
      }
      // 5. energies of every event, from the pre-step state
      if (valid) {
        const int64_t ev_idx = cpin + slot;
        float g = -1.0f;
        if (!((clock_mask >> pin) & 1u)) g = glitch_ratio_of(__ldg(p.glitch_pw + ev_idx), __ldg(p.pin_gden + p0 + pin));
        float energy = 0.0f;
        if (pin < n_in) {
          energy = in_energy(pin, o_e, rise);
        } else {
          const int o = pin - n_in;
          float best = p.min_diff0;
          int relq = -1;
          bool rel_rise = false;
          const double cur_s = __dmul_rn(static_cast<double>(cur_abs), p.ts);
          const float* dlp = blk + ty.delay_off + o * n_in * 4 + (rise ? 0 : 1);
#pragma unroll
          for (int q = 0; q < kFastPins - 1; ++q) {
            if (q >= n_in) break;
            if (!((has_wave >> q) & 1u)) continue;
            int32_t tr = trq[q];
            bool fr = frq[q] != 0;
            if (q == pk && has_clk) {
              tr = tr_clk;
              fr = fr_clk;
            }
            if (tr < cs_rel || tr >= ce_rel) continue;   // the related edge lies in this cycle
            const float dl = dlp[q * 4 + (fr ? 0 : 2)];
            if (isnan(dl)) continue;
            const double trs = __dmul_rn(static_cast<double>(T0 + tr), p.ts);
            const float diff = __double2float_rn(fabs(__dsub_rn(__dsub_rn(cur_s, static_cast<double>(dl)), trs)));
            if (diff < best) {
              best = diff;
              relq = q;
              rel_rise = fr;
            }
          }
          if (relq < 0) {
            energy = blk[ty.def_off + 2 * o + (rise ? 0 : 1)];
          } else {
            const int16_t eo = fast_tab[fo + n_in * n_state + (o * n_in + relq) * n_state + o_e];
            if (eo >= 0) energy = blk[eo + (rel_rise ? 0 : 2) + (rise ? 0 : 1)];
          }
          if (COUNTS) n_rel += static_cast<uint32_t>(relq + 1);
          if (nr2 > 0) {
            const float esw = __fmul_rn(nr2 == 2 ? 1.0f : 0.5f, __ldg(p.pin_swe + p0 + pin));
            if (g > 0.0f) {
              const float x = __fmul_rn(g, esw);
              acc[3] += x;
              add_bin_k(p, bins, kGSw, cq, to_fx_f(x, p.fx_dyn_f, p.fx_dyn));
            } else {
              acc[2] += esw;
              add_bin_k(p, bins, kSw, cq, to_fx_f(esw, p.fx_dyn_f, p.fx_dyn));
            }
          }
        }
        energy = __fmul_rn(energy, tog2 == 2 ? 1.0f : (tog2 == 1 ? 0.5f : 0.0f));
        if (g > 0.0f) {
          const float x = __fmul_rn(g, energy);
          acc[1] += x;
          add_bin_k(p, bins, kGInt, cq, to_fx_f(x, p.fx_dyn_f, p.fx_dyn));
          if (COUNTS) { ++n_gl; add_cnt(p, bins, 1, cyc); }
        } else {
          acc[0] += energy;
          add_bin_k(p, bins, kInt, cq, to_fx_f(energy, p.fx_dyn_f, p.fx_dyn));
        }
        if (COUNTS) {
          ++n_ev;
          n_half += static_cast<uint32_t>(tog2);
          add_cnt(p, bins, 0, cyc);
        }
      }
      // 6. carry each pin's last event to the next chunk
#pragma unroll
      for (int j = 0; j < kFastPins; ++j) {
        if (pm[j]) {
          const int l = 31 - __clz(pm[j]);
          const int vl = __shfl_sync(FULL, nv, l);
          const int32_t tl = __shfl_sync(FULL, static_cast<int32_t>(rel), l);
          const int rl = __shfl_sync(FULL, rflag, l);
          cst = (cst & ~(3u << (2 * j))) | (static_cast<uint32_t>(vl) << (2 * j));
          last_rise = (last_rise & ~(1u << j)) | (rl ? (1u << j) : 0u);
          at_lo &= ~(1u << j);
          last_t[j] = tl;
          cur_c[j] += __popc(pm[j]);
        }
      }
      n_left -= static_cast<uint32_t>(n_use);
      __syncwarp();
    }

    if (pkbit && lane == 0) pclk_run(pj, pclk_jend(), ones_of(cst) & ~pkbit);
    // a standalone part ends at its last tick, unless that lies past
    // time_max: the level it added is taken back integer for integer
    unsigned long long lvl_all = lvl;
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) lvl_all += __shfl_xor_sync(FULL, lvl_all, d);
    if (standalone && lane == 0 && T0 + static_cast<int64_t>(span) <= p.tmax) {
      const int64_t t1 = T0 + static_cast<int64_t>(span);
      const uint32_t k = udiv32(span + off0, tpc32, p.tpc_magic);
      const uint32_t h = span + off0 - k * tpc32;
      const int64_t cyc1 = bins.c_lo + k;
      if (h == 0) {
        add_bin_k(p, bins, kLeakLevel, k, 0ull - lvl_all);
      } else {
        const double cur_s = static_cast<double>(t1) * p.ts;
        const double end_s = fmin(static_cast<double>(cyc1 + 1) * P, p.tmax_s);
        const float lf = leak_of(ones_of(cst));
        add_bin(p, bins, kLeakPart, cyc1, to_fx(-static_cast<double>(lf) * (end_s - cur_s), p.fx_leak));
        add_bin(p, bins, kLeakLevel, cyc1 + 1, 0ull - lvl_all);
      }
    }
    // the cell's sums for this tile
    const int64_t nc = p.n_cell;
#pragma unroll
    for (int q = 0; q < kNumCellAcc; ++q) {
      double a = acc[q];
#pragma unroll
      for (int d = 16; d >= 1; d >>= 1) a += __shfl_xor_sync(FULL, a, d);
      if (lane == 0 && a != 0) atomicAdd(p.cell_acc + q * nc + cell, a);
    }
    if (COUNTS) {
      uint32_t c4[4] = {n_ev, n_gl, n_half, n_rel};
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        uint32_t v = __reduce_add_sync(FULL, c4[q]);
        if (lane == 0 && v) atomicAdd(p.cnt_cell + q * nc + cell, v);
      }
    }
    __syncwarp();   // the window and the instance copy are the next cell's
  }
  __syncthreads();
  // clock runs: run-differences -> per-cycle sums
  if (runs_on) {
    for (int set = 0; set < nset; ++set) {
      block_inclusive_scan(smem + static_cast<int64_t>(set) * nslot * ct + kIntRun * ct, ct, s_wsum);
      block_inclusive_scan(smem + static_cast<int64_t>(set) * nslot * ct + kLeakRun * ct, ct, s_wsum);
    }
  }
  // flush the tile's per-cycle bins
  const int64_t stride = p.n_period + 1;
  for (int64_t k = threadIdx.x; k < ct; k += blockDim.x) {
    const int64_t c = bins.c_lo + k;
    const int64_t cc = c < p.n_period ? c : p.n_period;
#pragma unroll
    for (int q = 0; q < kNumCycAcc; ++q) {
      unsigned long long x0 = smem[q * ct + k];
      unsigned long long x1 = nset == 2 ? smem[(nslot + q) * ct + k] : 0ull;
      if (runs_on && (q == kInt || q == kLeakPart)) {
        const int r = q == kInt ? kIntRun : kLeakRun;
        x0 += smem[r * ct + k];
        if (nset == 2) x1 += smem[(nslot + r) * ct + k];
      }
      if (x0 + x1) atomicAdd(p.cyc_acc + q * stride + cc, x0 + x1);
      if (p.cyc_acc_g) {
        if (x0) atomicAdd(p.cyc_acc_g + (static_cast<int64_t>(g_first) * kNumCycAcc + q) * stride + cc, x0);
        if (x1) atomicAdd(p.cyc_acc_g + (static_cast<int64_t>(g_first + 1) * kNumCycAcc + q) * stride + cc, x1);
      }
    }
    if (COUNTS) {
      const uint32_t a = bins.sc[k], b2 = bins.sc[ct + k];
      if (a) atomicAdd(p.cnt_cyc + 0 * stride + cc, static_cast<unsigned long long>(a));
      if (b2) atomicAdd(p.cnt_cyc + 1 * stride + cc, static_cast<unsigned long long>(b2));
    }
  }
}

// One window of one design, cells of up to kFastPins pins without drift:
// block (x, y) walks gate block x over tile y, one warp per cell.
template <bool COUNTS, bool RUNS>
__global__ void __launch_bounds__(256, WARP_WALK_MIN_BLOCKS) power_warp_kernel(const __grid_constant__ KParams p) {
  extern __shared__ unsigned long long smem[];
  warp_walk_block<COUNTS, RUNS>(p, blockIdx.x, blockIdx.y, smem);
}

// One window of one design: block (x, y) walks gate block x over tile y,
// or with p.gate_major gate block y over tile x. Blocks start in the order of
// their linear index, and the walk order puts the heaviest cells first: gate
// major, the launch as a whole runs heaviest first and ends on light blocks.
template <int MAXP, bool COUNTS, bool FAST, bool DRIFT, bool RUNS>
__global__ void __launch_bounds__(256, WALK_MIN_BLOCKS) power_walk_kernel(const __grid_constant__ KParams p) {
  extern __shared__ unsigned long long smem[];
  // one call site: the walk's body is inlined once
  const bool gm = p.gate_major != 0;
  const int gblk = gm ? blockIdx.y : blockIdx.x;
  const int tile = gm ? blockIdx.x : blockIdx.y;
  const int n_blk = gm ? gridDim.y : gridDim.x;
  walk_block<MAXP, COUNTS, FAST, DRIFT, RUNS, FAST && WALK_USE_RING>(p, gblk, tile, n_blk, smem);
}

// Persistent walk over the windows of many designs: each block takes work
// items (x: index into params, one per design and pin bucket; y: gate block;
// z: tile) from a queue in descending order of estimated work until it is
// empty. *n_items and the queue head *counter live in device memory, so a
// captured launch can be replayed with new items.
template <int MAXP, bool COUNTS, bool FAST, bool DRIFT, bool RUNS>
__global__ void __launch_bounds__(256, WALK_MIN_BLOCKS)
    power_walk_batch_kernel(const KParams* __restrict__ params, const int4* __restrict__ items,
                            const int* __restrict__ n_items, int* __restrict__ counter) {
  extern __shared__ unsigned long long smem[];
  __shared__ KParams sp;
  __shared__ int s_item;
  const int n = *n_items;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
    __syncthreads();
    const int it = s_item;
    if (it >= n) break;
    const int4 w = items[it];
    const unsigned long long* src = reinterpret_cast<const unsigned long long*>(params + w.x);
    unsigned long long* dst = reinterpret_cast<unsigned long long*>(&sp);
    for (int k = threadIdx.x; k < static_cast<int>(sizeof(KParams) / 8); k += blockDim.x) dst[k] = src[k];
    __syncthreads();
    walk_block<MAXP, COUNTS, FAST, DRIFT, RUNS, FAST && WALK_BATCH_RING>(sp, w.y, w.z, 1, smem);
    __syncthreads();  // smem and s_item are reused by the next item
  }
}

// ---- first event of every (tile, net) ----

// out[tile * n_net + net] = lower_bound(T0(tile)) - net_off[net] over the
// net's events, T0(tile) = max(t_lo, (cyc0 + tile * cycles_per_tile) * tpc).
// Parameters come from *pd when it is set (device memory, so that a captured
// launch sees each window's values), else from pv.
__global__ void tile_first_kernel(const KParams pv, const KParams* __restrict__ pd, int32_t* __restrict__ out) {
  const KParams& p = pd ? *pd : pv;
  const int64_t nn = p.n_net;
  const int64_t total = static_cast<int64_t>(p.n_tiles) * nn;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t tile = i / nn;
    const int32_t net = static_cast<int32_t>(i - tile * nn);
    const int64_t c_lo = p.tiles ? static_cast<int64_t>(p.tiles[tile].x) : p.cyc0 + tile * p.cycles_per_tile;
    const int64_t T0 = max(p.t_lo, c_lo * p.tpc);
    const int64_t a = p.net_off[net], e = p.net_off[net + 1];
    int64_t l = a, r = e;
    if (a < 0 || e < a || e > p.n_event) {  // reported by the walk
      out[i] = 0;
      continue;
    }
    while (l < r) {
      const int64_t m = l + ((r - l) >> 1);
      if (ev_time(p.ev_t, m) < T0) l = m + 1; else r = m;
    }
    out[i] = static_cast<int32_t>(l - a);
  }
}

// ---- glitch pulse widths of every listed event ----

// out[e] = glitch_pw of event e of its net, one warp per net. Parameters from
// *pd when set (device memory), else from pv.
//
// The warp steps through the net's events 24 at a time: lane l holds event
// e0 - 4 + l, lanes 4..27 own their events and lanes 0-3 and 28-31 show the
// neighbours. Each lane finds its event's period group (the run of events in
// one clock period; the waveform's first event g0 stands alone) from ballots
// of the group starts and ends, and the flags and width of glitch_pw follow
// from the group sizes of the lane and its neighbours. An owned event whose
// group, or previous group, reaches the edge of the 32 events (five or more
// events in one period) takes the per-event routine glitch_pw instead; both
// give the same result.
__global__ void glitch_pw_kernel(const KParams pv, const KParams* __restrict__ pd, float* __restrict__ out) {
  const KParams& p = pd ? *pd : pv;
  const int lane = threadIdx.x & 31;
  const unsigned full = 0xffffffffu;
  const unsigned below = lane == 31 ? full : ((1u << (lane + 1)) - 1u);  // lanes 0..lane
  const unsigned above = ~((1u << lane) - 1u);                            // lanes lane..31
  const bool owner = lane >= 4 && lane < 28;
  const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t net = (blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) >> 5; net < p.n_net;
       net += warps) {
    const int64_t lo = p.net_off[net], hi = p.net_off[net + 1];
    if (lo < 0 || hi < lo || hi > p.n_event) continue;  // reported by the walk
    if (p.net_glitch && !p.net_glitch[net]) continue;   // read by clock pins only: never a glitch
    const int64_t base = p.net_base ? p.net_base[net] : 0;
    const int64_t g0 = base == 0 ? lo : -1;
    for (int64_t e0 = lo; e0 < hi; e0 += 24) {
      const int64_t e = e0 - 4 + lane;
      const bool valid = e >= lo && e < hi;
      const int64_t t = valid ? ev_time(p.ev_t, e) : 0;
      const int64_t c = valid ? div_floor_t(t, p.tpc, p.tpc_magic64) : 0;
      const int64_t t_prev = __shfl_up_sync(full, t, 1), c_prev = __shfl_up_sync(full, c, 1);
      const int64_t t_next = __shfl_down_sync(full, t, 1), c_next = __shfl_down_sync(full, c, 1);
      // period groups: g0 stands alone; past lane 0 and lane 31 a group is
      // taken to go on (unknown)
      const bool has_prev = valid && e != g0 && e - 1 >= lo && e - 1 != g0;
      const bool has_next = valid && e != g0 && e + 1 < hi;
      const bool join_prev = has_prev && (lane == 0 || c_prev == c);
      const bool join_next = has_next && (lane == 31 || c_next == c);
      const unsigned S = __ballot_sync(full, !join_prev);
      const unsigned E = __ballot_sync(full, !join_next);
      // first / last lane of this lane's group, -1 when it reaches outside
      const int first = (S & below) ? 31 - __clz(S & below) : -1;
      const int last = (E & above) ? __ffs(E & above) - 1 : -1;
      const int first_prev = __shfl_up_sync(full, first, 1);
      const int last_prev = __shfl_up_sync(full, last, 1);
      const int last_next = __shfl_down_sync(full, last, 1);
      if (!owner || !valid) continue;
      float res = -1.0f;
      bool slow = first < 0 || last < 0;
      if (!slow && e != g0) {
        const int k = last - first + 1;
        const int lim = k >= 2 ? (k & ~1) : 0;
        const int off = lane - first;
        if (off < lim) {
          int64_t w = -1;
          if (e - 1 >= lo) {
            bool pflag = false;
            if (off > 0) {
              pflag = true;
            } else if (e - 1 != g0) {
              // e - 1 ends the previous group: flagged when that group is even
              if (first_prev <= 0) {
                slow = true;  // it may reach before lane 0
              } else {
                const int kp = last_prev - first_prev + 1;
                pflag = kp >= 2 && (kp & 1) == 0;
              }
            }
            if (pflag) w = t - t_prev;
          }
          if (!slow && e + 1 < hi) {
            bool nflag = false;
            if (lane + 1 <= last) {
              nflag = off + 1 < lim;
            } else if (e + 2 < hi) {
              // e + 1 starts the next group: flagged when it holds two or more
              nflag = last_next < 0 || last_next >= lane + 2;
            }
            if (nflag) w = max(w, t_next - t);
          }
          if (w >= 0) res = __double2float_rn(__dmul_rn(static_cast<double>(w), p.ts));
        }
      }
      if (slow) {
        const int64_t cs = c * p.tpc;
        const bool prev_same = e - 1 >= lo && t_prev >= cs;
        const bool next_same = e + 1 < hi && t_next < cs + p.tpc;
        res = (prev_same || next_same) ? glitch_pw(p, e, lo, hi, g0, t, cs) : -1.0f;
      }
      out[e] = res;
    }
  }
}

// ---- periodic clock patterns ----


// out[nets[w]] = the window's periodic pattern of net nets[w], one block per
// net: its events in [TL, TH) = [max(t_lo, 1), min(t_hi, tmax + 1)) are edge
// k0, k0 + 1, ... of the sequence whose edge k lies at (k / 2) * tpc + (k odd
// ? pb : pa) with value (k odd ? v0 : 1 - v0), no edge of the sequence in
// [TL, TH) is missing but one at exactly time_max (a trace that ends on a
// clock edge it does not list; flagged in bit 30 of y), and the last event
// before TL holds the value before edge k0. Otherwise x = -1 and the walk
// takes the net's events one by one.
__global__ void pclk_kernel(const KParams pv, const KParams* __restrict__ pd, const int32_t* __restrict__ nets,
                            int32_t n, int2* __restrict__ out) {
  // one block per net: every thread reads the header, all check the events
  const KParams& p = pd ? *pd : pv;
  for (int64_t w = blockIdx.x; w < n; w += gridDim.x) {
    const int32_t net = nets[w];
    if (net < 0 || net >= p.n_net) continue;  // uniform over the block
    const int64_t lo = p.net_off[net], hi = p.net_off[net + 1];
    const int64_t tpc = p.tpc;
    bool ok = lo >= 0 && hi >= lo && hi <= p.n_event && tpc >= 2 && tpc < (int64_t(1) << 30);
    const int64_t TL = max(p.t_lo, static_cast<int64_t>(1)), TH = min(p.t_hi, p.tmax + 1);
    int64_t l = lo, u = lo;
    if (ok) {
      l = lower_bound_time(p.ev_t, lo, hi, TL);
      u = lower_bound_time(p.ev_t, l, hi, TH);
      // two edges to read the phases from, a value before them, and no
      // event past time_max inside the window (the walk reports those)
      ok = u - l >= 2 && l > lo && (u == hi || ev_time(p.ev_t, u) >= p.t_hi);
    }
    int64_t pa = 0, pb = 0, k0 = 0;
    int v0 = 0;
    bool end_tmax = false;
    if (ok) {
      const int64_t t0 = ev_time(p.ev_t, l), t1 = ev_time(p.ev_t, l + 1);
      const int64_t c0 = t0 / tpc, c1 = t1 / tpc;
      const int64_t f0 = t0 - c0 * tpc, f1 = t1 - c1 * tpc;
      const int va = ev_value(p.ev_v, l);
      if (c1 == c0) {
        pa = f0; pb = f1; k0 = 2 * c0; v0 = 1 - va;
      } else if (c1 == c0 + 1 && f1 < f0) {
        pa = f1; pb = f0; k0 = 2 * c0 + 1; v0 = va;
      } else {
        ok = false;
      }
      ok = ok && (va == 0 || va == 1) && ev_value(p.ev_v, l - 1) == ((k0 & 1) ? 1 - v0 : v0);
      const int64_t km = k0 - 1, kn = k0 + (u - l);
      const int64_t tn = (kn >> 1) * tpc + ((kn & 1) ? pb : pa);
      end_tmax = tn == p.tmax && p.tmax < TH;
      ok = ok && (km >> 1) * tpc + ((km & 1) ? pb : pa) < TL && (tn >= TH || end_tmax);
    }
    bool good = true;
    if (ok) {
      for (int64_t j = threadIdx.x; j < u - l; j += blockDim.x) {
        const int64_t k = k0 + j;
        good = good && ev_time(p.ev_t, l + j) == (k >> 1) * tpc + ((k & 1) ? pb : pa) &&
               ev_value(p.ev_v, l + j) == ((k & 1) ? v0 : 1 - v0);
      }
    }
    ok = __syncthreads_and(ok && good) != 0;
    if (threadIdx.x == 0)
      out[net] = ok ? make_int2(static_cast<int>(pa),
                                static_cast<int>(static_cast<uint32_t>(pb) | (end_tmax ? (1u << 30) : 0u) |
                                                 (static_cast<uint32_t>(v0) << 31)))
                    : make_int2(-1, 0);
  }
}

// ---- separate dynamic and leakage kernels (the unfused evaluation) ----
//
// The reference's naive baseline (-disable_fusion; GlobalConfig's
// cuda_power_separate_kernels_for_dyn_and_leak, util/GlobalConfig.hh:28;
// kernel1_1 / kernel1_2, power/cuda/CudaPower.cu:730-1039): one kernel with
// a thread per pin event for the dynamic energies, each thread rebuilding
// the cell's pin state at its event's time by searching every pin's event
// list, and one with a thread per cell and cycle tile for the leakage (the
// walk's merge and leakage steps alone, walk_block with DYN = false). The
// contract, and the integer per-cycle terms, are the fused walk's; the pair
// is its comparison point.

// Per net: the first listed event in [max(t_lo, 1), min(t_hi, tmax + 1))
// (the window's events the walk evaluates; tick 0 is the initial
// condition) and their number. Nets with bad offsets count none (the count
// kernel reports them).
__global__ void sep_net_range_kernel(const KParams p, int64_t* __restrict__ net_lo, int64_t* __restrict__ net_cnt) {
  const int64_t S = max(p.t_lo, static_cast<int64_t>(1));
  const int64_t E = min(p.t_hi, p.tmax + 1);
  for (int64_t n = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; n < p.n_net;
       n += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t a = __ldg(p.net_off + n), b = __ldg(p.net_off + n + 1);
    int64_t lo = a, cnt = 0;
    if (a >= 0 && b > a && b <= p.n_event && E > S) {
      lo = lower_bound_time(p.ev_t, a, b, S);
      cnt = lower_bound_time(p.ev_t, lo, b, E) - lo;
    }
    net_lo[n] = lo;
    net_cnt[n] = cnt;
  }
}

// cnt[k] = events of the walked cell at walk-order position k (k < n) over
// its pins; cnt[n] = 0, so that an exclusive scan ends with the total.
// Flags what the walk flags per pin: bad offsets, a listing without the
// event before t_lo, times past time_max.
__global__ void sep_cell_count_kernel(const KParams p, int32_t n, const int64_t* __restrict__ net_lo,
                                      const int64_t* __restrict__ net_cnt, int64_t* __restrict__ cnt) {
  for (int32_t k = blockIdx.x * blockDim.x + threadIdx.x; k <= n; k += gridDim.x * blockDim.x) {
    if (k == n) {
      cnt[n] = 0;
      continue;
    }
    const int32_t cell = __ldg(p.order + k);
    const int32_t p0 = __ldg(p.cell_pin_off + cell), p1 = __ldg(p.cell_pin_off + cell + 1);
    int64_t s = 0;
    for (int32_t q = p0; q < p1; ++q) {
      const int32_t net = __ldg(p.pin_net + q);
      if (net < 0) continue;
      const int64_t a = __ldg(p.net_off + net), b = __ldg(p.net_off + net + 1);
      if (a < 0 || b < a || b > p.n_event) {
        atomicOr(p.status, kErrNetRange);
        continue;
      }
      if (b == a) continue;
      const int64_t base = p.net_base ? __ldg(p.net_base + net) : 0;
      if (base != 0 && __ldg(net_lo + net) == a) atomicOr(p.status, kErrContext);
      if (ev_time(p.ev_t, b - 1) > p.tmax) atomicOr(p.status, kErrTimeRange);
      s += __ldg(net_cnt + net);
    }
    cnt[k] = s;
  }
}

// One thread per pin event g < cell_off[n] (grid-stride): the walk-order
// position and pin that hold it, the pre-step state of every pin of the
// cell (a bisection in each pin's events), the related input of an output
// event, the glitch ratio, the internal and switching energies; per-cell
// FP64 and per-cycle fixed-point sums by global atomics.
template <bool COUNTS>
__global__ void __launch_bounds__(256) sep_dyn_kernel(const KParams p, int32_t n, const int64_t* __restrict__ cell_off,
                                                      const int64_t* __restrict__ net_lo,
                                                      const int64_t* __restrict__ net_cnt) {
  const int64_t total = __ldg(cell_off + n);
  const int64_t nc = p.n_cell;
  const int64_t stride = p.n_period + 1;
  for (int64_t g = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; g < total;
       g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    // the last position k with cell_off[k] <= g
    int32_t lo = 0, hi = n;
    while (hi - lo > 1) {
      const int32_t m = lo + ((hi - lo) >> 1);
      if (__ldg(cell_off + m) <= g) lo = m; else hi = m;
    }
    const int32_t cell = __ldg(p.order + lo);
    int64_t r = g - __ldg(cell_off + lo);
    const int32_t p0 = __ldg(p.cell_pin_off + cell);
    const DevType ty = p.types[__ldg(p.cell_type + cell)];
    const int n_pin = ty.n_pin, n_in = ty.n_in;
    int pin = -1;
    int64_t e = 0;
    for (int i = 0; i < n_pin; ++i) {
      const int32_t net = __ldg(p.pin_net + p0 + i);
      const int64_t c = net >= 0 ? __ldg(net_cnt + net) : 0;
      if (r < c) {
        pin = i;
        e = __ldg(net_lo + net) + r;
        break;
      }
      r -= c;
    }
    if (pin < 0) continue;
    const int32_t net_i = __ldg(p.pin_net + p0 + pin);
    const int64_t a_i = __ldg(p.net_off + net_i), b_i = __ldg(p.net_off + net_i + 1);
    const int64_t cur = ev_time(p.ev_t, e);
    if (e > a_i && ev_time(p.ev_t, e - 1) >= cur) {
      atomicOr(p.status, kErrTimeOrder);
      continue;
    }
    const int nv = ev_value(p.ev_v, e);
    const int pv = e > a_i ? ev_value(p.ev_v, e - 1) : 2;
    const int tog2 = ntoggle2(pv, nv);
    const int nr2 = nrise2(pv, nv);
    const bool rise = nr2 > 0;
    const int64_t cyc = div_floor_t(cur, p.tpc, p.tpc_magic64);
    const int64_t cs = cyc * p.tpc;
    const bool out = pin >= n_in;
    const int o = pin - n_in;
    const float* __restrict__ blk = p.inst + __ldg(p.cell_inst + cell);
    const double cur_s = __dmul_rn(static_cast<double>(cur), p.ts);
    // pre-step state (events strictly before cur) and the related input:
    // its last event strictly before cur, in cur's cycle, nearest to cur
    // less the arc delay
    uint32_t ones = 0;
    float best = p.min_diff0;
    int relq = -1;
    bool rel_rise = false;
    for (int j = 0; j < n_pin; ++j) {
      int v = pv;
      if (j != pin) {
        v = __ldg(p.pin_flags + p0 + j) & 3;
        const int32_t net = __ldg(p.pin_net + p0 + j);
        if (net >= 0) {
          const int64_t a = __ldg(p.net_off + net), b = __ldg(p.net_off + net + 1);
          if (a >= 0 && b > a && b <= p.n_event) {
            const int64_t pos = lower_bound_time(p.ev_t, a, b, cur);
            v = pos > a ? ev_value(p.ev_v, pos - 1) : 2;
            if (out && j < n_in) {
              const int64_t re = pos > a ? pos - 1 : a;
              const int64_t tr = ev_time(p.ev_t, re);
              const bool fr = re > a && nrise2(ev_value(p.ev_v, re - 1), ev_value(p.ev_v, re)) > 0;
              if (tr >= cs && tr < cs + p.tpc) {
                const float dl = blk[ty.delay_off + o * n_in * 4 + (rise ? 0 : 1) + j * 4 + (fr ? 0 : 2)];
                if (!isnan(dl)) {
                  const double trs = __dmul_rn(static_cast<double>(tr), p.ts);
                  const float diff = __double2float_rn(fabs(__dsub_rn(__dsub_rn(cur_s, static_cast<double>(dl)), trs)));
                  if (diff < best) {
                    best = diff;
                    relq = j;
                    rel_rise = fr;
                  }
                }
              }
            }
          }
        }
      }
      if (v == 1) ones |= 1u << j;
    }
    // glitch ratio (clock pins never glitch)
    float gr = -1.0f;
    if (!(__ldg(p.pin_flags + p0 + pin) & 4)) {
      const float den = __ldg(p.pin_gden + p0 + pin);
      if (p.glitch_pw) {
        gr = glitch_ratio_of(__ldg(p.glitch_pw + e), den);
      } else {
        const int64_t base = p.net_base ? __ldg(p.net_base + net_i) : 0;
        gr = glitch_ratio(p, e, a_i, b_i, base == 0 ? a_i : -1, cur, cs, den);
      }
    }
    // internal energy: the first internal_power group whose `when` holds
    // (an output's: of its related input, else the default average)
    float energy = 0.0f;
    const int32_t s_begin = __ldg(p.pin_slot + ty.pin_slot_off + pin);
    const int32_t s_end = __ldg(p.pin_slot + ty.pin_slot_off + pin + 1);
    if (!out) {
      for (int32_t k = s_begin; k < s_end; ++k) {
        const DevSlot sl = p.slots[k];
        if (when_holds(p.cubes, sl.cube_off, sl.n_cube, ones)) {
          energy = blk[sl.e_off + (rise ? 0 : 1)];
          break;
        }
      }
    } else if (relq < 0) {
      energy = blk[ty.def_off + 2 * o + (rise ? 0 : 1)];
    } else {
      for (int32_t k = s_begin; k < s_end; ++k) {
        const DevSlot sl = p.slots[k];
        if (sl.related != relq) continue;
        if (when_holds(p.cubes, sl.cube_off, sl.n_cube, ones)) {
          energy = blk[sl.e_off + (rel_rise ? 0 : 2) + (rise ? 0 : 1)];
          break;
        }
      }
    }
    const int64_t cc = cyc < p.n_period ? cyc : p.n_period;
    const int32_t grp = p.cyc_acc_g ? __ldg(p.cell_cgroup + cell) : 0;
    auto add = [&](int qc, int qy, float x) {
      if (x == 0.0f) return;
      atomicAdd(p.cell_acc + qc * nc + cell, static_cast<double>(x));
      const unsigned long long f = to_fx_f(x, p.fx_dyn_f, p.fx_dyn);
      if (f == 0ull) return;
      atomicAdd(p.cyc_acc + qy * stride + cc, f);
      if (p.cyc_acc_g) atomicAdd(p.cyc_acc_g + (static_cast<int64_t>(grp) * kNumCycAcc + qy) * stride + cc, f);
    };
    if (out && nr2 > 0) {
      // switching: n_rise * C * V^2
      const float esw = __fmul_rn(nr2 == 2 ? 1.0f : 0.5f, __ldg(p.pin_swe + p0 + pin));
      if (gr > 0.0f) add(3, kGSw, __fmul_rn(gr, esw));
      else add(2, kSw, esw);
    }
    energy = __fmul_rn(energy, tog2 == 2 ? 1.0f : (tog2 == 1 ? 0.5f : 0.0f));
    if (gr > 0.0f) add(1, kGInt, __fmul_rn(gr, energy));
    else add(0, kInt, energy);
    if (COUNTS) {
      atomicAdd(p.cnt_cell + 0 * nc + cell, 1u);
      atomicAdd(p.cnt_cyc + 0 * stride + cc, 1ull);
      if (gr > 0.0f) {
        atomicAdd(p.cnt_cell + 1 * nc + cell, 1u);
        atomicAdd(p.cnt_cyc + 1 * stride + cc, 1ull);
      }
      if (tog2) atomicAdd(p.cnt_cell + 2 * nc + cell, static_cast<uint32_t>(tog2));
      if (out && relq >= 0) atomicAdd(p.cnt_cell + 3 * nc + cell, static_cast<uint32_t>(relq + 1));
    }
  }
}

// The leakage kernel: the walk over cell x tile without the energies.
template <int MAXP, bool DRIFT>
__global__ void __launch_bounds__(256, WALK_MIN_BLOCKS) power_leak_kernel(const __grid_constant__ KParams p) {
  extern __shared__ unsigned long long smem[];
  walk_block<MAXP, false, false, DRIFT, false, false, false>(p, blockIdx.x, blockIdx.y, gridDim.x, smem);
}

// ---- walk order by work ----

__global__ void work_keys_kernel(const KParams p, const int32_t* __restrict__ base_order, int32_t n,
                                 int32_t b1, int32_t b2, unsigned long long* __restrict__ keys) {
  const int32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int32_t cell = base_order[k];
  const int32_t a = p.cell_pin_off[cell], e = p.cell_pin_off[cell + 1];
  long long w = 0;
  bool pclk_cell = false;
  for (int32_t q = a; q < e; ++q) {
    const int32_t net = p.pin_net[q];
    if (net < 0) continue;
    // a periodic clock pin of a cell in the first bucket (the fast walk)
    // costs the walk per change of the other pins only
    if (p.pclk && k < b1 && (p.pin_flags[q] & 4) && p.pclk[net].x >= 0) {
      pclk_cell = true;
      continue;
    }
    w += p.net_off[net + 1] - p.net_off[net];
  }
  const unsigned long long bucket = k >= b2 ? 2ull : (k >= b1 ? 1ull : 0ull);
  const unsigned long long cap = (1ull << 39) - 1;
  const unsigned long long wc = w < 0 ? 0ull : (static_cast<unsigned long long>(w) > cap ? cap : static_cast<unsigned long long>(w));
  // bits [0,39): inverted work; bit 39: the cell has a periodic clock pin
  // (its lanes take the clock-run branches, so such cells share warps); then
  // the bucket, or with per-cycle groups the cell group in [40,58) and the
  // bucket in [58,60)
  const unsigned long long cls = (WALK_KEY_CLASS && pclk_cell) ? (1ull << 39) : 0ull;
  if (p.cell_cgroup)
    keys[k] = (bucket << 58) | (static_cast<unsigned long long>(p.cell_cgroup[cell]) << 40) | cls | (cap - wc);
  else
    keys[k] = (bucket << 40) | cls | (cap - wc);
}

// ---- density split ----

// cnt[k] = threads that walk the cell at walk-order position k per tile
// (cnt[n] = 0, the end of the prefix): the events the cell's pins list in
// the window, spread over one tile at the window's mean density, per
// split_events events, within [1, min(kMaxSplit, ct)].
__global__ void split_count_kernel(const unsigned long long* __restrict__ keys, int32_t n, int64_t ct,
                                   int64_t n_cyc, int32_t split_events, int32_t* __restrict__ cnt) {
  const int32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k > n) return;
  if (k == n) {
    cnt[k] = 0;
    return;
  }
  const unsigned long long cap = (1ull << 39) - 1;
  const unsigned long long wc = cap - (keys[k] & cap);
  const double per_tile = static_cast<double>(wc) * static_cast<double>(ct) /
                          static_cast<double>(n_cyc > 0 ? n_cyc : 1);
  const int64_t lim = ct < kMaxSplit ? ct : kMaxSplit;
  int64_t m = static_cast<int64_t>(ceil(per_tile / static_cast<double>(split_events)));
  m = m < 1 ? 1 : (m > lim ? lim : m);
  cnt[k] = static_cast<int32_t>(m);
}

}  // namespace

size_t split_scan_temp_bytes(int32_t n_cell) {
  size_t bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, bytes, static_cast<const int32_t*>(nullptr), static_cast<int32_t*>(nullptr),
                                n_cell + 1);
  return bytes;
}

cudaError_t compute_split(const unsigned long long* keys_sorted, int32_t n_cell, int64_t cycles_per_tile,
                          int64_t n_cyc, int32_t split_events, int32_t* item_off, void* temp, size_t temp_bytes,
                          cudaStream_t stream) {
  if (n_cell <= 0) return cudaSuccess;
  // counts first into the temp area's head, then the scan into item_off
  int32_t* cnt = static_cast<int32_t*>(temp);
  void* scan_temp = static_cast<char*>(temp) + ((static_cast<size_t>(n_cell) + 1) * 4 + 255) / 256 * 256;
  size_t scan_bytes = temp_bytes - (static_cast<char*>(scan_temp) - static_cast<char*>(temp));
  split_count_kernel<<<(n_cell + 1 + 255) / 256, 256, 0, stream>>>(keys_sorted, n_cell, cycles_per_tile, n_cyc,
                                                                    split_events, cnt);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return cub::DeviceScan::ExclusiveSum(scan_temp, scan_bytes, cnt, item_off, n_cell + 1, stream);
}

cudaError_t launch_glitch_pw(const KParams& p, const KParams* d_p, float* out, cudaStream_t stream) {
  if (p.n_net <= 0) return cudaSuccess;
  const int64_t threads = static_cast<int64_t>(p.n_net) * 32;
  const int blocks = static_cast<int>(std::min<int64_t>((threads + 255) / 256, 148 * 32));
  glitch_pw_kernel<<<blocks, 256, 0, stream>>>(p, d_p, out);
  return cudaGetLastError();
}

cudaError_t launch_pclk(const KParams& p, const KParams* d_p, const int32_t* nets, int32_t n, int2* out,
                        cudaStream_t stream) {
  if (n <= 0) return cudaSuccess;
  const int blocks = static_cast<int>(std::min<int64_t>(n, 148 * 8));
  pclk_kernel<<<blocks, 256, 0, stream>>>(p, d_p, nets, n, out);
  return cudaGetLastError();
}

cudaError_t launch_tile_first(const KParams& p, const KParams* d_p, int32_t* out, cudaStream_t stream) {
  const int64_t total = static_cast<int64_t>(p.n_tiles) * p.n_net;
  if (total <= 0) return cudaSuccess;
  const int blocks = static_cast<int>(std::min<int64_t>((total + 255) / 256, 148 * 32));
  tile_first_kernel<<<blocks, 256, 0, stream>>>(p, d_p, out);
  return cudaGetLastError();
}

size_t work_sort_temp_bytes(int32_t n_cell) {
  size_t bytes = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, bytes, static_cast<const unsigned long long*>(nullptr),
                                  static_cast<unsigned long long*>(nullptr),
                                  static_cast<const int32_t*>(nullptr), static_cast<int32_t*>(nullptr),
                                  n_cell, 0, 60);
  return bytes;
}

cudaError_t sort_cells_by_work(const KParams& p, const int32_t* base_order, int32_t n_cell,
                               const int32_t* bucket_begin, unsigned long long* keys_in,
                               unsigned long long* keys_out, int32_t* order_out, void* temp,
                               size_t temp_bytes, cudaStream_t stream) {
  if (n_cell <= 0) return cudaSuccess;
  work_keys_kernel<<<(n_cell + 255) / 256, 256, 0, stream>>>(p, base_order, n_cell, bucket_begin[1],
                                                             bucket_begin[2], keys_in);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const int end_bit = p.cell_cgroup ? 60 : 42;
  return cub::DeviceRadixSort::SortPairs(temp, temp_bytes, keys_in, keys_out, base_order, order_out,
                                         n_cell, 0, end_bit, stream);
}

namespace {

// ---- finalize ----

__global__ void finalize_cells(const KParams p, const uint8_t* __restrict__ group,
                               float* __restrict__ cell5, double* __restrict__ tg) {
  // tg: [0..4] totals, [5 + 5*g + q] groups; order leakage, internal (incl.
  // glitch), glitch internal, switching (incl. glitch), glitch switching
  __shared__ double red[GTP_N_GROUP + 1][5];
  if (threadIdx.x < (GTP_N_GROUP + 1) * 5) (&red[0][0])[threadIdx.x] = 0.0;
  __syncthreads();
  const int64_t nc = p.n_cell;
  const double norm_dyn = static_cast<double>(p.tmax) * p.ts;
  const double norm_leak = static_cast<double>(p.tmax);
  for (int64_t c = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; c < nc;
       c += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double i_r = p.cell_acc[0 * nc + c] / norm_dyn;
    const double i_g = p.cell_acc[1 * nc + c] / norm_dyn;
    const double s_r = p.cell_acc[2 * nc + c] / norm_dyn;
    const double s_g = p.cell_acc[3 * nc + c] / norm_dyn;
    const double lk = p.cell_acc[4 * nc + c] / norm_leak;
    if (cell5) {
      cell5[5 * c + 0] = static_cast<float>(i_r);
      cell5[5 * c + 1] = static_cast<float>(i_g);
      cell5[5 * c + 2] = static_cast<float>(s_r);
      cell5[5 * c + 3] = static_cast<float>(s_g);
      cell5[5 * c + 4] = static_cast<float>(lk);
    }
    const double v5[5] = {lk, i_r + i_g, i_g, s_r + s_g, s_g};
    const int g = group ? group[c] : 0;
    for (int q = 0; q < 5; ++q) {
      atomicAdd(&red[0][q], v5[q]);
      atomicAdd(&red[1 + g][q], v5[q]);
    }
  }
  __syncthreads();
  if (threadIdx.x < (GTP_N_GROUP + 1) * 5) atomicAdd(tg + threadIdx.x, (&red[0][0])[threadIdx.x]);
}

// One block: prefix-sums the leakage level differences and converts the
// fixed-point per-cycle energies to watts. The level of cycle c covers the
// part of the cycle before time_max.
// Block b handles accumulator set b: acc_base + b * 6 * (n_period + 1), with
// its outputs at cycle5_base + b * 5 * n_period.
__global__ void finalize_cycles(const KParams p, const unsigned long long* __restrict__ acc_base,
                                float* __restrict__ cycle5_base,
                                unsigned long long* __restrict__ leak_tmp_base) {
  const int64_t np = p.n_period;
  const int64_t stride = np + 1;
  const unsigned long long* acc = acc_base + static_cast<int64_t>(blockIdx.x) * kNumCycAcc * stride;
  float* cycle5 = cycle5_base + static_cast<int64_t>(blockIdx.x) * 5 * np;
  unsigned long long* leak_tmp = leak_tmp_base + static_cast<int64_t>(blockIdx.x) * np;
  __shared__ unsigned long long carry_s;
  __shared__ unsigned long long warp_sums[32];
  if (threadIdx.x == 0) carry_s = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int64_t base = 0; base < np; base += blockDim.x) {
    const int64_t c = base + threadIdx.x;
    unsigned long long x = c < np ? acc[kLeakLevel * stride + c] : 0ull;
    for (int o = 1; o < 32; o <<= 1) {
      unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[wid] = x;
    __syncthreads();
    if (wid == 0) {
      unsigned long long w = lane < nw ? warp_sums[lane] : 0ull;
      for (int o = 1; o < 32; o <<= 1) {
        unsigned long long y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      if (lane < nw) warp_sums[lane] = w;
    }
    __syncthreads();
    const unsigned long long carry = carry_s;
    const unsigned long long pre = (wid > 0 ? warp_sums[wid - 1] : 0ull) + x + carry;
    if (c < np) leak_tmp[c] = pre;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry_s = pre;
    __syncthreads();
  }
  const double P = p.period_d;
  const double inv_l = 1.0 / (p.fx_leak * P);
  const double inv_d = 1.0 / (p.fx_dyn * P);
  for (int64_t c = threadIdx.x; c < np; c += blockDim.x) {
    const double c0 = static_cast<double>(c) * P;
    double frac = (fmin(static_cast<double>(c + 1) * P, p.tmax_s) - c0) / P;
    frac = frac < 0.0 ? 0.0 : (frac > 1.0 ? 1.0 : frac);
    const double level = static_cast<double>(static_cast<long long>(leak_tmp[c]));
    const double part = static_cast<double>(static_cast<long long>(acc[kLeakPart * stride + c]));
    const long long ir = static_cast<long long>(acc[kInt * stride + c]);
    const long long ig = static_cast<long long>(acc[kGInt * stride + c]);
    const long long sr = static_cast<long long>(acc[kSw * stride + c]);
    const long long sg = static_cast<long long>(acc[kGSw * stride + c]);
    cycle5[0 * np + c] = static_cast<float>((level * frac + part) * inv_l);
    cycle5[1 * np + c] = static_cast<float>(static_cast<double>(ir + ig) * inv_d);
    cycle5[2 * np + c] = static_cast<float>(static_cast<double>(ig) * inv_d);
    cycle5[3 * np + c] = static_cast<float>(static_cast<double>(sr + sg) * inv_d);
    cycle5[4 * np + c] = static_cast<float>(static_cast<double>(sg) * inv_d);
  }
}

template <int MAXP, bool COUNTS, bool FAST, bool DRIFT, bool RUNS = false>
size_t walk_smem_t(const KParams& p, int threads) {
  size_t tabs = (FAST && p.tabs_in_smem) ? ((static_cast<size_t>(p.n_leak_pool) * 4 + static_cast<size_t>(p.n_fast_tab) * 2 + 15) / 16) * 16 : 0;
  if (FAST && WALK_STAGE_INST) tabs += static_cast<size_t>(threads) * p.fast_inst_stride * 4;
  return power_walk_smem_bytes(p.cycles_per_tile, COUNTS, threads, (FAST && WALK_USE_RING) ? MAXP : 0, tabs,
                               p.cell_cgroup ? 2 : 1, RUNS && p.pclk != nullptr) +
         (RUNS ? walk_runs_acc_bytes(threads) : 0);
}

// Blocks of this walk variant resident per SM (0 when the query fails).
template <int MAXP, bool COUNTS, bool FAST, bool DRIFT, bool RUNS = false>
int occupancy_t(const KParams& p, int threads) {
  const size_t smem = walk_smem_t<MAXP, COUNTS, FAST, DRIFT, RUNS>(p, threads);
  auto kern = power_walk_kernel<MAXP, COUNTS, FAST, DRIFT, RUNS>;
  int nb = 0;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, threads, smem);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    return 0;
  }
  return nb;
}

template <int MAXP, bool COUNTS, bool FAST, bool DRIFT, bool RUNS = false>
cudaError_t launch_t(const KParams& p, int threads, cudaStream_t stream) {
  const int32_t n = p.order_end - p.order_begin;
  if (n <= 0) return cudaSuccess;
  const size_t smem = walk_smem_t<MAXP, COUNTS, FAST, DRIFT, RUNS>(p, threads);
  auto kern = power_walk_kernel<MAXP, COUNTS, FAST, DRIFT, RUNS>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  const int32_t n_gblk = (n + p.gates_per_block - 1) / p.gates_per_block;
  KParams q = p;
  // gate major while the gate blocks fit in grid.y
  q.gate_major = n_gblk <= 65535 ? 1 : 0;
  dim3 grid = q.gate_major ? dim3(p.n_tiles, n_gblk) : dim3(n_gblk, p.n_tiles);
  kern<<<grid, threads, smem, stream>>>(q);
  return cudaGetLastError();
}

template <bool COUNTS, bool RUNS>
cudaError_t launch_warp_t(const KParams& p, int threads, cudaStream_t stream) {
  const int32_t n = p.order_end - p.order_begin;
  if (n <= 0) return cudaSuccess;
  size_t tabs = p.tabs_in_smem ? ((static_cast<size_t>(p.n_leak_pool) * 4 + static_cast<size_t>(p.n_fast_tab) * 2 + 15) / 16) * 16 : 0;
  tabs += static_cast<size_t>(threads / 32) * warp_region_bytes(p.fast_inst_stride);
  const size_t smem = power_walk_smem_bytes(p.cycles_per_tile, COUNTS, threads, 0, tabs, p.cell_cgroup ? 2 : 1,
                                            RUNS && p.pclk != nullptr);
  auto kern = power_warp_kernel<COUNTS, RUNS>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  dim3 grid((n + p.gates_per_block - 1) / p.gates_per_block, p.n_tiles);
  kern<<<grid, threads, smem, stream>>>(p);
  return cudaGetLastError();
}

template <int MAXP, bool COUNTS, bool FAST, bool DRIFT, bool RUNS = false>
cudaError_t launch_batch_t(const KParams* d_params, const int4* d_items, const int* d_n_items, int* d_counter,
                           int grid, int threads, size_t smem, cudaStream_t stream) {
  auto kern = power_walk_batch_kernel<MAXP, COUNTS, FAST, DRIFT, RUNS>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  kern<<<grid, threads, smem, stream>>>(d_params, d_items, d_n_items, d_counter);
  return cudaGetLastError();
}

}  // namespace

static_assert(sizeof(KParams) % 8 == 0, "KParams is copied to shared memory in 8-byte words");

cudaError_t launch_power_walk_batch(const KParams* d_params, const int4* d_items, const int* d_n_items,
                                    int* d_counter, int grid, int max_pins, bool counts, bool drift, bool runs,
                                    int threads, size_t smem, cudaStream_t stream) {
#define GTPB_BATCH(MP, C, F, D, R) \
  launch_batch_t<MP, C, F, D, R>(d_params, d_items, d_n_items, d_counter, grid, threads, smem, stream)
  if (max_pins <= kFastPins) {
    if (drift) return counts ? GTPB_BATCH(kFastPins, true, true, true, false) : GTPB_BATCH(kFastPins, false, true, true, false);
    if (runs) return counts ? GTPB_BATCH(kFastPins, true, true, false, true) : GTPB_BATCH(kFastPins, false, true, false, true);
    return counts ? GTPB_BATCH(kFastPins, true, true, false, false) : GTPB_BATCH(kFastPins, false, true, false, false);
  }
  if (max_pins <= 8) {
    if (drift) return counts ? GTPB_BATCH(8, true, false, true, false) : GTPB_BATCH(8, false, false, true, false);
    return counts ? GTPB_BATCH(8, true, false, false, false) : GTPB_BATCH(8, false, false, false, false);
  }
  if (drift) return counts ? GTPB_BATCH(kMaxPins, true, false, true, false) : GTPB_BATCH(kMaxPins, false, false, true, false);
  return counts ? GTPB_BATCH(kMaxPins, true, false, false, false) : GTPB_BATCH(kMaxPins, false, false, false, false);
#undef GTPB_BATCH
}

int walk_blocks_per_sm(int max_pins, bool counts, bool drift, bool runs, int threads, size_t smem) {
  // the kernel that will be launched, with its dynamic shared-memory limit
  // raised first: above 48 KB the occupancy query fails without it
  auto occ = [&](auto kern) -> int {
    int nb = 0;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, threads, smem);
    return e == cudaSuccess && nb > 0 ? nb : 1;
  };
#define GTPB_OCC(MP, F, D, R) (counts ? occ(power_walk_batch_kernel<MP, true, F, D, R>) \
                                      : occ(power_walk_batch_kernel<MP, false, F, D, R>))
  if (max_pins <= kFastPins) {
    if (drift) return GTPB_OCC(kFastPins, true, true, false);
    return runs ? GTPB_OCC(kFastPins, true, false, true) : GTPB_OCC(kFastPins, true, false, false);
  }
  if (max_pins <= 8) return drift ? GTPB_OCC(8, false, true, false) : GTPB_OCC(8, false, false, false);
  return drift ? GTPB_OCC(kMaxPins, false, true, false) : GTPB_OCC(kMaxPins, false, false, false);
#undef GTPB_OCC
}

size_t walk_item_smem_bytes(const KParams& p, int max_pins, bool counts, int threads) {
  const bool fast = max_pins <= kFastPins;
  size_t tabs = (fast && p.tabs_in_smem)
                    ? ((static_cast<size_t>(p.n_leak_pool) * 4 + static_cast<size_t>(p.n_fast_tab) * 2 + 15) / 16) * 16
                    : 0;
  if (fast && WALK_STAGE_INST) tabs += static_cast<size_t>(threads) * p.fast_inst_stride * 4;
  return power_walk_smem_bytes(p.cycles_per_tile, counts, threads, (fast && WALK_BATCH_RING) ? kFastPins : 0, tabs,
                               p.cell_cgroup ? 2 : 1, fast && !p.drift && p.pclk != nullptr);
}

size_t walk_runs_acc_bytes(int threads) { return static_cast<size_t>(kNumCellAcc) * 8 * threads; }

size_t power_walk_smem_bytes(int64_t cycles_per_tile, bool counts, int threads, int ring_pins,
                             size_t tab_bytes, int bin_sets, bool clock_runs) {
  const int slots = clock_runs ? kNumBinSlotsRun : kNumCycAcc;
  return static_cast<size_t>(cycles_per_tile) * (bin_sets * slots * 8 + (counts ? 8 : 0)) +
         static_cast<size_t>(ring_pins) * kRing * threads * 4 + tab_bytes;
}

cudaError_t launch_power_walk(const KParams& p, int max_pins, bool counts, int threads,
                              cudaStream_t stream, bool warp_walk) {
  const bool d = p.drift != 0;
  if (max_pins <= kFastPins && warp_walk && !d && p.glitch_pw && threads % 32 == 0) {
    if (p.pclk) return counts ? launch_warp_t<true, true>(p, threads, stream) : launch_warp_t<false, true>(p, threads, stream);
    return counts ? launch_warp_t<true, false>(p, threads, stream) : launch_warp_t<false, false>(p, threads, stream);
  }
  if (max_pins <= kFastPins) {
    if (d) return counts ? launch_t<kFastPins, true, true, true>(p, threads, stream)
                         : launch_t<kFastPins, false, true, true>(p, threads, stream);
    if (p.pclk) return counts ? launch_t<kFastPins, true, true, false, true>(p, threads, stream)
                              : launch_t<kFastPins, false, true, false, true>(p, threads, stream);
    return counts ? launch_t<kFastPins, true, true, false>(p, threads, stream)
                  : launch_t<kFastPins, false, true, false>(p, threads, stream);
  }
  if (max_pins <= 8) {
    if (d) return counts ? launch_t<8, true, false, true>(p, threads, stream)
                         : launch_t<8, false, false, true>(p, threads, stream);
    return counts ? launch_t<8, true, false, false>(p, threads, stream)
                  : launch_t<8, false, false, false>(p, threads, stream);
  }
  if (d) return counts ? launch_t<kMaxPins, true, false, true>(p, threads, stream)
                       : launch_t<kMaxPins, false, false, true>(p, threads, stream);
  return counts ? launch_t<kMaxPins, true, false, false>(p, threads, stream)
                : launch_t<kMaxPins, false, false, false>(p, threads, stream);
}

int walk_blocks_per_sm_launch(const KParams& p, int max_pins, bool counts, int threads) {
  const bool d = p.drift != 0;
  if (max_pins <= kFastPins) {
    if (d) return counts ? occupancy_t<kFastPins, true, true, true>(p, threads)
                         : occupancy_t<kFastPins, false, true, true>(p, threads);
    if (p.pclk) return counts ? occupancy_t<kFastPins, true, true, false, true>(p, threads)
                              : occupancy_t<kFastPins, false, true, false, true>(p, threads);
    return counts ? occupancy_t<kFastPins, true, true, false>(p, threads)
                  : occupancy_t<kFastPins, false, true, false>(p, threads);
  }
  if (max_pins <= 8) {
    if (d) return counts ? occupancy_t<8, true, false, true>(p, threads) : occupancy_t<8, false, false, true>(p, threads);
    return counts ? occupancy_t<8, true, false, false>(p, threads) : occupancy_t<8, false, false, false>(p, threads);
  }
  if (d) return counts ? occupancy_t<kMaxPins, true, false, true>(p, threads)
                       : occupancy_t<kMaxPins, false, false, true>(p, threads);
  return counts ? occupancy_t<kMaxPins, true, false, false>(p, threads)
                : occupancy_t<kMaxPins, false, false, false>(p, threads);
}

namespace {
template <int MAXP, bool DRIFT>
cudaError_t launch_leak_t(const KParams& p, int threads, cudaStream_t stream) {
  const int32_t n = p.order_end - p.order_begin;
  if (n <= 0) return cudaSuccess;
  const size_t smem = power_walk_smem_bytes(p.cycles_per_tile, false, threads, 0, 0, p.cell_cgroup ? 2 : 1, false);
  auto kern = power_leak_kernel<MAXP, DRIFT>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  dim3 grid((n + p.gates_per_block - 1) / p.gates_per_block, p.n_tiles);
  kern<<<grid, threads, smem, stream>>>(p);
  return cudaGetLastError();
}
}  // namespace

size_t separate_scan_temp_bytes(int32_t n_cell) {
  size_t b = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, b, static_cast<const int64_t*>(nullptr), static_cast<int64_t*>(nullptr),
                                static_cast<int64_t>(n_cell) + 1);
  return b;
}

cudaError_t launch_separate_kernels(const KParams& p, const int32_t* bucket_begin, bool counts, int threads,
                                    const SeparateScratch& s, cudaStream_t stream) {
  const int32_t n = bucket_begin[3];
  int dev = 0, sms = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  auto blocks_for = [&](int64_t work) -> int {
    const int64_t b = (work + 255) / 256;
    return static_cast<int>(b < 1 ? 1 : (b > static_cast<int64_t>(sms) * 16 ? static_cast<int64_t>(sms) * 16 : b));
  };
  // 1. per net: the window's events to evaluate
  if (p.n_net > 0) {
    sep_net_range_kernel<<<blocks_for(p.n_net), 256, 0, stream>>>(p, s.net_lo, s.net_cnt);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  // 2. per walked cell: its pin events, and their exclusive prefix
  sep_cell_count_kernel<<<blocks_for(static_cast<int64_t>(n) + 1), 256, 0, stream>>>(p, n, s.net_lo, s.net_cnt,
                                                                                   s.cell_cnt);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  size_t tb = s.temp_bytes;
  e = cub::DeviceScan::ExclusiveSum(s.temp, tb, s.cell_cnt, s.cell_off, static_cast<int64_t>(n) + 1, stream);
  if (e != cudaSuccess) return e;
  // 3. the dynamic kernel: a thread per pin event, grid-stride over the
  // total the scan left on the device
  {
    auto kern = counts ? sep_dyn_kernel<true> : sep_dyn_kernel<false>;
    int nb = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, 256, 0);
    if (e != cudaSuccess) return e;
    kern<<<sms * (nb > 0 ? nb : 1), 256, 0, stream>>>(p, n, s.cell_off, s.net_lo, s.net_cnt);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  // 4. the leakage kernel: a thread per cell and cycle tile, per pin bucket
  static const int bucket_pins[3] = {kFastPins, 8, kMaxPins};
  for (int b = 0; b < 3; ++b) {
    KParams q = p;
    q.order_begin = bucket_begin[b];
    q.order_end = bucket_begin[b + 1];
    q.item_off = nullptr;
    q.pclk = nullptr;
    if (q.order_end <= q.order_begin) continue;
    const bool d = p.drift != 0;
    if (bucket_pins[b] == kFastPins) e = d ? launch_leak_t<kFastPins, true>(q, threads, stream)
                                           : launch_leak_t<kFastPins, false>(q, threads, stream);
    else if (bucket_pins[b] == 8) e = d ? launch_leak_t<8, true>(q, threads, stream)
                                        : launch_leak_t<8, false>(q, threads, stream);
    else e = d ? launch_leak_t<kMaxPins, true>(q, threads, stream) : launch_leak_t<kMaxPins, false>(q, threads, stream);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_finalize(const KParams& p, const uint8_t* cell_group, float* d_cell5,
                            float* d_cycle5, double* d_tg, unsigned long long* d_leak_tmp,
                            cudaStream_t stream, float* d_cycle5_g, unsigned long long* d_leak_tmp_g) {
  cudaError_t e = cudaMemsetAsync(d_tg, 0, sizeof(double) * (GTP_N_GROUP + 1) * 5, stream);
  if (e != cudaSuccess) return e;
  if (p.n_cell > 0) {
    int blocks = static_cast<int>(std::min<int64_t>((p.n_cell + 255) / 256, 148 * 8));
    finalize_cells<<<blocks, 256, 0, stream>>>(p, cell_group, d_cell5, d_tg);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  if (p.n_period > 0) {
    finalize_cycles<<<1, 1024, 0, stream>>>(p, p.cyc_acc, d_cycle5, d_leak_tmp);
    e = cudaGetLastError();
    if (e == cudaSuccess && p.cyc_acc_g && d_cycle5_g && d_leak_tmp_g && p.n_cgroup > 0) {
      finalize_cycles<<<p.n_cgroup, 1024, 0, stream>>>(p, p.cyc_acc_g, d_cycle5_g, d_leak_tmp_g);
      e = cudaGetLastError();
    }
  }
  return e;
}

}  // namespace gtpb
