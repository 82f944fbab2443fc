// power_kernel.cu — the fused time-based power walk for sm_100a.
//
// One thread walks one cell over one cycle tile of the event window. It
// merges the cell's pin event lists in time order (the loop of
// findTimeBasedAllPower, power/TimeBasedPower.cc:795-890) and, per step:
//   - charges the leakage of the state before the step over the elapsed
//     segment, split into clock cycles exactly as
//     calculatePerCycleLeakagePower does (TimeBasedPower.cc:677-701);
//   - classifies each triggered pin's event as glitch or not with the
//     clock-period grouping of getEventClockCycleBasedGlitchFlags
//     (TimeBasedPower.cc:589-637), evaluated online from the neighbouring
//     events, and scales it with getTimeBasedGlitchScalingRatioH
//     (power/PowerUtils.cc:285-294);
//   - selects the input internal energy (first `when`-matching group) or,
//     for an output event, the related input pin by arc-delay distance
//     (TimeBasedPower.cc:383-509) and its energy, plus C*V^2 switching.
//
// Design for B200:
//   - the CTA owns a cycle tile; per-cycle sums go to shared-memory bins as
//     64-bit fixed-point energies (integer shared atomics: exact, and the
//     final per-cycle values do not depend on accumulation order). Leakage of
//     whole idle cycles is added as a run (+x at the first full cycle, -x
//     after the last) so an idle stretch costs O(1), not O(cycles);
//   - a tile flushes its bins to global memory once;
//   - per-cell sums stay in FP64 registers and are flushed once per tile;
//   - a leakage segment is charged by the tile in which it starts, so a
//     segment that crosses a tile edge is split exactly as the reference
//     splits it (no artificial cut).
#include <cstdint>
#include <cuda_runtime.h>

#include "engine.h"

namespace gtpb {
namespace {

constexpr int64_t kInf = INT64_MAX;

__device__ __forceinline__ int64_t div_floor_pos(int64_t t, int64_t d, double inv) {
  // floor(t / d) for 0 <= t < 2^53 via a double reciprocal and one correction
  int64_t q = static_cast<int64_t>(static_cast<double>(t) * inv);
  int64_t r = t - q * d;
  if (r < 0) --q;
  else if (r >= d) ++q;
  return q;
}

__device__ __forceinline__ int ev_value(const uint32_t* __restrict__ v, int64_t i) {
  return (__ldg(v + (i >> 4)) >> (2 * (i & 15))) & 3;
}

__device__ __forceinline__ int64_t ev_time(const int64_t* __restrict__ t, int64_t i) {
  return __ldg(t + i);
}

// getNRise (power/PowerUtils.cc:213-237) as a 4x4 table packed in bits:
// returns 2*n_rise (0, 1 or 2).
__device__ __forceinline__ int nrise2(int prev, int cur) {
  // prev=0: cur 1 -> 2, cur 2 -> 1 ; prev=2: cur 1 -> 1 ; else 0
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

struct Bins {
  unsigned long long* s;   // [6][ct]
  uint32_t* sc;            // [2][ct] counts
  int64_t c_lo;            // first cycle of the tile
  int64_t ct;              // cycles in the tile
};

template <bool COUNTS>
struct Walker {
  const KParams& p;
  Bins& b;
  __device__ Walker(const KParams& pp, Bins& bb) : p(pp), b(bb) {}

  __device__ __forceinline__ void add_cyc(int q, int64_t c, double joules, double scale) {
    if (joules == 0.0) return;
    const unsigned long long x = to_fx(joules, scale);
    const int64_t k = c - b.c_lo;
    if (k >= 0 && k < b.ct) {
      atomicAdd(b.s + q * b.ct + k, x);
    } else {
      const int64_t cc = c < p.n_period ? c : p.n_period;
      atomicAdd(p.cyc_acc + q * (p.n_period + 1) + cc, x);
    }
  }
  __device__ __forceinline__ void add_cnt(int q, int64_t c) {
    const int64_t k = c - b.c_lo;
    if (k >= 0 && k < b.ct) {
      atomicAdd(b.sc + q * b.ct + k, 1u);
    } else {
      const int64_t cc = c < p.n_period ? c : p.n_period;
      atomicAdd(p.cnt_cyc + q * (p.n_period + 1) + cc, 1ull);
    }
  }

  // calculatePerCycleLeakagePower over [prev, cur) ticks with value val (W).
  __device__ void leak_segment(int64_t prev, int64_t cur, float val) {
    if (val == 0.0f) return;
    const double P = p.period_d;
    const double cur_s = static_cast<double>(cur) * p.ts;
    const double left = static_cast<double>(prev) * p.ts;
    const int64_t c = div_floor_pos(prev, p.tpc, p.inv_tpc);
    if (!(static_cast<double>(c) * P <= cur_s)) return;
    const double r1 = static_cast<double>(c + 1) * P;
    const double v = static_cast<double>(val);
    if (!(r1 <= cur_s)) {
      add_cyc(0, c, v * (cur_s - left), p.fx_leak);
      return;
    }
    add_cyc(0, c, v * (r1 - left), p.fx_leak);
    // last cycle k with k*P <= cur_s; (c+1)*P <= cur_s holds, so k >= c+1.
    // The reciprocal estimate is within one or two of k, so both loops are short.
    int64_t k = static_cast<int64_t>(cur_s * p.inv_period_d);
    if (k < c + 1) k = c + 1;
    while (k > c + 1 && static_cast<double>(k) * P > cur_s) --k;
    while (static_cast<double>(k + 1) * P <= cur_s) ++k;
    if (k >= c + 2) {
      const double full = v * P;
      add_cyc(1, c + 1, full, p.fx_leak);
      add_cyc(1, k, -full, p.fx_leak);
    }
    if (k >= c + 1) add_cyc(0, k, v * (cur_s - static_cast<double>(k) * P), p.fx_leak);
  }
};

// Period-group facts of event i on a net with accessible range [lo, hi) and
// global index 0 at g0 (or -1): the first index of its clock period (never
// g0) and the count k of non-initial events in the period.
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

// Reads element i of a register array without dynamic indexing (keeps the
// array in registers).
template <int N>
__device__ __forceinline__ int64_t sel(const int64_t (&a)[N], int i) {
  int64_t r = a[0];
#pragma unroll
  for (int j = 1; j < N; ++j)
    if (j == i) r = a[j];
  return r;
}

template <int MAXP, bool COUNTS>
__global__ void __launch_bounds__(256) power_walk_kernel(const KParams p) {
  extern __shared__ unsigned long long smem[];
  const int64_t ct = p.cycles_per_tile;
  Bins bins;
  bins.s = smem;
  bins.sc = reinterpret_cast<uint32_t*>(smem + kNumCycAcc * ct);
  const int tile = blockIdx.y;
  bins.c_lo = p.cyc0 + static_cast<int64_t>(tile) * ct;
  bins.ct = ct;
  for (int64_t k = threadIdx.x; k < kNumCycAcc * ct; k += blockDim.x) smem[k] = 0ull;
  if (COUNTS)
    for (int64_t k = threadIdx.x; k < 2 * ct; k += blockDim.x) bins.sc[k] = 0u;
  __syncthreads();

  // tile window in ticks
  const int64_t T0 = max(p.t_lo, bins.c_lo * p.tpc);
  const bool last_tile = (tile == p.n_tiles - 1);
  const int64_t T1 = last_tile ? p.t_hi : min(p.t_hi, (bins.c_lo + ct) * p.tpc);
  const bool owns_initial = (tile == 0) && (p.t_lo == 0);

  Walker<COUNTS> W(p, bins);
  const int32_t g_begin = p.order_begin + blockIdx.x * p.gates_per_block;
  const int32_t g_end = min(p.order_end, g_begin + p.gates_per_block);

  for (int32_t gi = g_begin + threadIdx.x; gi < g_end; gi += blockDim.x) {
    const int32_t cell = __ldg(p.order + gi);
    const int32_t p0 = __ldg(p.cell_pin_off + cell);
    const DevType ty = p.types[__ldg(p.cell_type + cell)];
    const float* __restrict__ blk = p.inst + __ldg(p.cell_inst + cell);
    const int n_pin = ty.n_pin, n_in = ty.n_in;

    int64_t f[MAXP], hi[MAXP], lo[MAXP], nt[MAXP], g0[MAXP];
    uint64_t state = 0;     // 2 bits per pin
    uint32_t ones = 0;      // bit per pin: state == 1
    uint32_t has_wave = 0;
#pragma unroll
    for (int i = 0; i < MAXP; ++i) {
      f[i] = 0; hi[i] = 0; lo[i] = 0; nt[i] = kInf; g0[i] = -1;
      if (i < n_pin) {
        const int32_t net = __ldg(p.pin_net + p0 + i);
        int v;
        bool wave = false;
        if (net >= 0) {
          const int64_t a = __ldg(p.net_off + net), e = __ldg(p.net_off + net + 1);
          if (a < 0 || e < a || e > p.n_event) {
            atomicOr(p.status, kErrNetRange);
          } else if (e > a) {
            wave = true;
            lo[i] = a; hi[i] = e;
            const int64_t base = p.net_base ? __ldg(p.net_base + net) : 0;
            g0[i] = base == 0 ? a : -1;
          }
        }
        if (!wave) {
          v = __ldg(p.pin_flags + p0 + i) & 3;
        } else {
          has_wave |= 1u << i;
          // lower_bound(T0) in [lo, hi)
          int64_t l = lo[i], r = hi[i];
          while (l < r) {
            const int64_t m = l + ((r - l) >> 1);
            if (ev_time(p.ev_t, m) < T0) l = m + 1; else r = m;
          }
          // an event at tick 0 that is the waveform's first is the initial condition
          if (l < hi[i] && l == g0[i] && ev_time(p.ev_t, l) == 0) ++l;
          f[i] = l;
          if (l > lo[i]) {
            v = ev_value(p.ev_v, l - 1);
          } else {
            v = 2;
            if (g0[i] < 0) atomicOr(p.status, kErrContext);
          }
          nt[i] = l < hi[i] ? ev_time(p.ev_t, l) : kInf;
        }
        state |= static_cast<uint64_t>(v) << (2 * i);
        if (v == 1) ones |= 1u << i;
      }
    }

    double acc_int = 0, acc_gint = 0, acc_sw = 0, acc_gsw = 0, acc_leak = 0;
    uint32_t n_ev = 0, n_gl = 0, n_half = 0, n_rel = 0;
    bool owns = owns_initial;
    int64_t prev_time = 0;

    const float leak_const = ty.leak_const;
    const int32_t leak_off = ty.leak_off;
    auto leak_of = [&](uint32_t o) -> float {
      return leak_off >= 0 ? __ldg(p.leak_pool + leak_off + o) : leak_const;
    };

    while (true) {
      int64_t cur = kInf;
#pragma unroll
      for (int i = 0; i < MAXP; ++i)
        if (i < n_pin) cur = min(cur, nt[i]);
      if (cur >= T1) {
        if (owns) {
          const int64_t end = (cur == kInf) ? p.tmax : cur;
          if (end > prev_time) {
            const float lv = leak_of(ones);
            acc_leak += static_cast<double>(lv) * static_cast<double>(end - prev_time);
            W.leak_segment(prev_time, end, lv);
          }
        }
        break;
      }
      if (cur > p.tmax) atomicOr(p.status, kErrTimeRange);
      // advance every pin with an event at cur
      uint64_t new_state = state;
      uint32_t new_ones = ones;
      uint32_t trig = 0;
#pragma unroll
      for (int i = 0; i < MAXP; ++i) {
        if (i < n_pin && nt[i] == cur) {
          const int v = ev_value(p.ev_v, f[i]);
          new_state = (new_state & ~(3ull << (2 * i))) | (static_cast<uint64_t>(v) << (2 * i));
          new_ones = (new_ones & ~(1u << i)) | (v == 1 ? (1u << i) : 0u);
          trig |= 1u << i;
          ++f[i];
          if (f[i] < hi[i]) {
            const int64_t tn = ev_time(p.ev_t, f[i]);
            if (tn <= cur) { atomicOr(p.status, kErrTimeOrder); nt[i] = kInf; }
            else nt[i] = tn;
          } else {
            nt[i] = kInf;
          }
        }
      }
      // leakage of the state before cur
      if (owns) {
        const float lv = leak_of(ones);
        acc_leak += static_cast<double>(lv) * static_cast<double>(cur - prev_time);
        W.leak_segment(prev_time, cur, lv);
      }
      const int64_t cyc = div_floor_pos(cur, p.tpc, p.inv_tpc);
      const int64_t cyc_start = cyc * p.tpc;
      const int64_t cyc_end = cyc_start + p.tpc;

      uint32_t tb = trig;
      while (tb) {
        const int i = __ffs(tb) - 1;
        tb &= tb - 1;
        const int pv = static_cast<int>((state >> (2 * i)) & 3);
        const int nv = static_cast<int>((new_state >> (2 * i)) & 3);
        const int tog2 = ntoggle2(pv, nv);
        const int nr2 = nrise2(pv, nv);
        const bool rise = nr2 > 0;
        const int pin = p0 + i;
        const uint8_t pf = __ldg(p.pin_flags + pin);

        // ---- glitch classification and ratio ----
        float g = -1.0f;
        const int64_t e = sel(f, i) - 1;
        const int64_t lo_i = sel(lo, i), hi_i = sel(hi, i), g0_i = sel(g0, i);
        if (!(pf & 4) && e != g0_i) {
          const Group gr = period_group(p.ev_t, e, lo_i, hi_i, g0_i, cyc_start, cyc_end);
          const int64_t k = gr.last - gr.first + 1;
          const int64_t lim = k >= 2 ? (k & ~int64_t(1)) : 0;
          if (e - gr.first < lim) {
            int64_t w = -1;
            // previous event flagged?
            if (e - 1 >= lo_i && e != g0_i) {
              bool pflag;
              if (e - 1 >= gr.first) {
                pflag = true;
              } else if (e - 1 == g0_i) {
                pflag = false;
              } else {
                const int64_t tp = ev_time(p.ev_t, e - 1);
                const int64_t pc = div_floor_pos(tp, p.tpc, p.inv_tpc);
                const Group gp = period_group(p.ev_t, e - 1, lo_i, hi_i, g0_i, pc * p.tpc,
                                              pc * p.tpc + p.tpc);
                const int64_t kp = gp.last - gp.first + 1;   // e-1 is the last of its period
                pflag = kp >= 2 && (kp & 1) == 0;
              }
              if (pflag) w = cur - ev_time(p.ev_t, e - 1);
            }
            if (e + 1 < hi_i) {
              bool nflag;
              const int64_t tn = ev_time(p.ev_t, e + 1);
              if (e + 1 <= gr.last) {
                nflag = (e + 1 - gr.first) < lim;
              } else if (e + 2 < hi_i) {
                const int64_t nc = div_floor_pos(tn, p.tpc, p.inv_tpc);
                nflag = ev_time(p.ev_t, e + 2) < nc * p.tpc + p.tpc;
              } else {
                nflag = false;
              }
              if (nflag) w = max(w, tn - cur);
            }
            if (w >= 0) {
              const float den = __ldg(p.pin_gden + pin);
              if (den == 0.0f) {
                g = 1.0f;
              } else {
                const float pw = __double2float_rn(__dmul_rn(static_cast<double>(w), p.ts));
                const float r = __double2float_rn(__ddiv_rn(__dmul_rn(static_cast<double>(pw), 2.0),
                                                            static_cast<double>(den)));
                g = fminf(1.0f, __fmul_rn(r, r));
              }
            }
          }
        }

        // ---- internal energy ----
        float energy = 0.0f;
        const int32_t s_begin = __ldg(p.pin_slot + ty.pin_slot_off + i);
        const int32_t s_end = __ldg(p.pin_slot + ty.pin_slot_off + i + 1);
        if (i < n_in) {
          for (int32_t s = s_begin; s < s_end; ++s) {
            const DevSlot sl = p.slots[s];
            if (when_holds(p.cubes, sl.cube_off, sl.n_cube, ones)) {
              energy = __ldg(blk + sl.e_off + (rise ? 0 : 1));
              break;
            }
          }
        } else {
          const int o = i - n_in;
          float best = p.min_diff0;
          int rel = -1;
          bool rel_rise = false;
          const double cur_s = __dmul_rn(static_cast<double>(cur), p.ts);
          for (int q = 0; q < n_in; ++q) {
            if (!((has_wave >> q) & 1)) continue;
            // lower_bound(cur) on pin q: its frontier, minus one if q fired at cur
            const int64_t lb = sel(f, q) - ((trig >> q) & 1);
            const int64_t loq = sel(lo, q);
            const int64_t re = max(loq, lb - 1);
            const int64_t pe = max(loq, re - 1);
            const bool fr = nrise2(ev_value(p.ev_v, pe), ev_value(p.ev_v, re)) > 0;
            const float dl = __ldg(blk + ty.delay_off + (o * n_in + q) * 4 + (fr ? 0 : 2) + (rise ? 0 : 1));
            if (isnan(dl)) continue;
            const int64_t tr = ev_time(p.ev_t, re);
            const double a = __dsub_rn(cur_s, static_cast<double>(dl));
            const float diff = __double2float_rn(fabs(__dsub_rn(a, __dmul_rn(static_cast<double>(tr), p.ts))));
            if (diff < best && tr >= cyc_start && tr < cyc_end) {
              best = diff;
              rel = q;
              rel_rise = fr;
            }
          }
          if (rel < 0) {
            energy = __ldg(blk + ty.def_off + 2 * o + (rise ? 0 : 1));
          } else {
            for (int32_t s = s_begin; s < s_end; ++s) {
              const DevSlot sl = p.slots[s];
              if (sl.related != rel) continue;
              if (when_holds(p.cubes, sl.cube_off, sl.n_cube, ones)) {
                energy = __ldg(blk + sl.e_off + (rel_rise ? 0 : 2) + (rise ? 0 : 1));
                break;
              }
            }
          }
          if (COUNTS) n_rel += static_cast<uint32_t>(rel + 1);
          // switching: n_rise * C * V^2
          if (nr2 > 0) {
            const float esw = __fmul_rn(nr2 == 2 ? 1.0f : 0.5f, __ldg(p.pin_swe + pin));
            if (g > 0.0f) {
              const float x = __fmul_rn(g, esw);
              acc_gsw += x;
              W.add_cyc(5, cyc, x, p.fx_dyn);
            } else {
              acc_sw += esw;
              W.add_cyc(4, cyc, esw, p.fx_dyn);
            }
          }
        }
        energy = __fmul_rn(energy, tog2 == 2 ? 1.0f : (tog2 == 1 ? 0.5f : 0.0f));
        if (g > 0.0f) {
          const float x = __fmul_rn(g, energy);
          acc_gint += x;
          W.add_cyc(3, cyc, x, p.fx_dyn);
          if (COUNTS) { ++n_gl; W.add_cnt(1, cyc); }
        } else {
          acc_int += energy;
          W.add_cyc(2, cyc, energy, p.fx_dyn);
        }
        if (COUNTS) {
          ++n_ev;
          n_half += static_cast<uint32_t>(tog2);
          W.add_cnt(0, cyc);
        }
      }
      state = new_state;
      ones = new_ones;
      prev_time = cur;
      owns = true;
    }

    // flush the cell's sums for this tile
    const int64_t nc = p.n_cell;
    if (acc_int != 0) atomicAdd(p.cell_acc + 0 * nc + cell, acc_int);
    if (acc_gint != 0) atomicAdd(p.cell_acc + 1 * nc + cell, acc_gint);
    if (acc_sw != 0) atomicAdd(p.cell_acc + 2 * nc + cell, acc_sw);
    if (acc_gsw != 0) atomicAdd(p.cell_acc + 3 * nc + cell, acc_gsw);
    if (acc_leak != 0) atomicAdd(p.cell_acc + 4 * nc + cell, acc_leak);
    if (COUNTS) {
      if (n_ev) atomicAdd(p.cnt_cell + 0 * nc + cell, n_ev);
      if (n_gl) atomicAdd(p.cnt_cell + 1 * nc + cell, n_gl);
      if (n_half) atomicAdd(p.cnt_cell + 2 * nc + cell, n_half);
      if (n_rel) atomicAdd(p.cnt_cell + 3 * nc + cell, n_rel);
    }
  }

  __syncthreads();
  // flush the tile's per-cycle bins
  const int64_t stride = p.n_period + 1;
  for (int64_t k = threadIdx.x; k < ct; k += blockDim.x) {
    const int64_t c = bins.c_lo + k;
    const int64_t cc = c < p.n_period ? c : p.n_period;
#pragma unroll
    for (int q = 0; q < kNumCycAcc; ++q) {
      const unsigned long long x = smem[q * ct + k];
      if (x) atomicAdd(p.cyc_acc + q * stride + cc, x);
    }
    if (COUNTS) {
      const uint32_t a = bins.sc[k], b2 = bins.sc[ct + k];
      if (a) atomicAdd(p.cnt_cyc + 0 * stride + cc, static_cast<unsigned long long>(a));
      if (b2) atomicAdd(p.cnt_cyc + 1 * stride + cc, static_cast<unsigned long long>(b2));
    }
  }
}

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

// One block: prefix-sums the leakage run-differences and converts the
// fixed-point per-cycle energies to watts.
__global__ void finalize_cycles(const KParams p, float* __restrict__ cycle5,
                                unsigned long long* __restrict__ leak_tmp) {
  const int64_t np = p.n_period;
  const int64_t stride = np + 1;
  const unsigned long long* acc = p.cyc_acc;
  // block-wide inclusive scan of the run-difference array, chunked
  __shared__ unsigned long long carry_s;
  __shared__ unsigned long long warp_sums[32];
  if (threadIdx.x == 0) carry_s = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int64_t base = 0; base < np; base += blockDim.x) {
    const int64_t c = base + threadIdx.x;
    unsigned long long x = c < np ? acc[1 * stride + c] : 0ull;
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
  const double inv_l = 1.0 / (p.fx_leak * p.period_d);
  const double inv_d = 1.0 / (p.fx_dyn * p.period_d);
  for (int64_t c = threadIdx.x; c < np; c += blockDim.x) {
    const long long lk = static_cast<long long>(acc[0 * stride + c] + leak_tmp[c]);
    const long long ir = static_cast<long long>(acc[2 * stride + c]);
    const long long ig = static_cast<long long>(acc[3 * stride + c]);
    const long long sr = static_cast<long long>(acc[4 * stride + c]);
    const long long sg = static_cast<long long>(acc[5 * stride + c]);
    cycle5[0 * np + c] = static_cast<float>(static_cast<double>(lk) * inv_l);
    cycle5[1 * np + c] = static_cast<float>(static_cast<double>(ir + ig) * inv_d);
    cycle5[2 * np + c] = static_cast<float>(static_cast<double>(ig) * inv_d);
    cycle5[3 * np + c] = static_cast<float>(static_cast<double>(sr + sg) * inv_d);
    cycle5[4 * np + c] = static_cast<float>(static_cast<double>(sg) * inv_d);
  }
}

template <int MAXP, bool COUNTS>
cudaError_t launch_t(const KParams& p, int threads, cudaStream_t stream) {
  const int32_t n = p.order_end - p.order_begin;
  if (n <= 0) return cudaSuccess;
  const size_t smem = power_walk_smem_bytes(p.cycles_per_tile, COUNTS);
  auto kern = power_walk_kernel<MAXP, COUNTS>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  dim3 grid((n + p.gates_per_block - 1) / p.gates_per_block, p.n_tiles);
  kern<<<grid, threads, smem, stream>>>(p);
  return cudaGetLastError();
}

}  // namespace

size_t power_walk_smem_bytes(int64_t cycles_per_tile, bool counts) {
  return static_cast<size_t>(cycles_per_tile) * (kNumCycAcc * 8 + (counts ? 8 : 0));
}

cudaError_t launch_power_walk(const KParams& p, int max_pins, bool counts, int threads,
                              cudaStream_t stream) {
  if (max_pins <= 4) return counts ? launch_t<4, true>(p, threads, stream) : launch_t<4, false>(p, threads, stream);
  if (max_pins <= 8) return counts ? launch_t<8, true>(p, threads, stream) : launch_t<8, false>(p, threads, stream);
  return counts ? launch_t<kMaxPins, true>(p, threads, stream) : launch_t<kMaxPins, false>(p, threads, stream);
}

cudaError_t launch_finalize(const KParams& p, const uint8_t* cell_group, float* d_cell5,
                            float* d_cycle5, double* d_tg, unsigned long long* d_leak_tmp,
                            cudaStream_t stream) {
  cudaError_t e = cudaMemsetAsync(d_tg, 0, sizeof(double) * (GTP_N_GROUP + 1) * 5, stream);
  if (e != cudaSuccess) return e;
  if (p.n_cell > 0) {
    int blocks = static_cast<int>(std::min<int64_t>((p.n_cell + 255) / 256, 148 * 8));
    finalize_cells<<<blocks, 256, 0, stream>>>(p, cell_group, d_cell5, d_tg);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  if (p.n_period > 0) {
    finalize_cycles<<<1, 1024, 0, stream>>>(p, d_cycle5, d_leak_tmp);
    e = cudaGetLastError();
  }
  return e;
}

}  // namespace gtpb
