// synth_rules.h — the counter-based rules of the synthetic traces, shared by
// the host generator (synth.cpp) and the device generator (synth_dev.cu) so
// that both produce the same events bit for bit.
//
// Every (seed, net, cycle) decides independently whether the net toggles in
// the cycle, where, and whether a glitch pulse follows. Double arithmetic
// uses explicitly rounded operations, so that the device compiler cannot
// fuse a multiply and an add into one rounding.
#pragma once

#include <stdint.h>

#if defined(__CUDACC__)
#define SYN_HD __host__ __device__ __forceinline__
#else
#define SYN_HD inline
#endif

namespace gtpb {
namespace syn {

SYN_HD double mul_rn(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dmul_rn(a, b);
#else
  return a * b;
#endif
}
SYN_HD double add_rn(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dadd_rn(a, b);
#else
  return a + b;
#endif
}

SYN_HD uint64_t splitmix(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
SYN_HD uint64_t hash3(uint64_t seed, uint64_t a, uint64_t b, uint64_t c) {
  return splitmix(splitmix(splitmix(seed ^ (a * 0xD6E8FEB86659FD93ull)) ^ (b + 0x632BE59BD9B4E019ull)) ^
                  (c * 0x9E3779B97F4A7C15ull + 1));
}
SYN_HD double u01(uint64_t h) { return mul_rn(static_cast<double>(h >> 11), 1.0 / 9007199254740992.0); }

// Plain view of a trace's parameters and tables (host or device pointers).
struct Rules {
  int32_t mode;        // 0 uniform, 1 zipf + burst, 2 phases, 3 phased units
  int32_t clock_net;
  int32_t n_net;
  int32_t n_unit;      // mode 3
  int64_t n_cycle;
  int64_t tpc;
  uint64_t seed;
  double lo, hi;       // mode 2 rate range
  double glitch_p;
  int64_t w_lo, w_hi;
  const double* net_rate;  // mode 0 / 1 / 3
  const double* burst;     // mode 1, per cycle
  const uint8_t* phase;    // mode 2 / 3, per cycle
  const double* act;       // mode 3, [phase][unit]
};

SYN_HD double prob(const Rules& r, int32_t net, int64_t c) {
  if (r.mode == 0) return r.net_rate[net];
  if (r.mode == 1) {
    const double p = mul_rn(r.net_rate[net], r.burst[c]);
    return p < 1.0 ? p : 1.0;
  }
  if (r.mode == 3) {
    const int64_t u = static_cast<int64_t>(net) * r.n_unit / r.n_net;
    const double p = mul_rn(r.net_rate[net], r.act[static_cast<int64_t>(r.phase[c]) * r.n_unit + u]);
    return p < 0.9 ? p : 0.9;
  }
  const uint64_t h = hash3(r.seed ^ 0x5A5A, static_cast<uint64_t>(net), r.phase[c], 77);
  return add_rn(r.lo, mul_rn(r.hi - r.lo, u01(h)));
}

// Events of one net in cycle c (ticks, ascending); returns how many (0..3).
// Tick 0 holds the net's initial value and is not produced here.
SYN_HD int cycle_events(const Rules& r, int32_t net, int64_t c, int64_t* t) {
  const int64_t base = c * r.tpc;
  if (net == r.clock_net) {  // falls at the cycle boundary, rises mid-cycle
    if (c == 0) {
      t[0] = base + r.tpc / 2;
      return 1;
    }
    t[0] = base;
    t[1] = base + r.tpc / 2;
    return 2;
  }
  const uint64_t h = hash3(r.seed, static_cast<uint64_t>(net), static_cast<uint64_t>(c), 1);
  if (u01(h) >= prob(r, net, c)) return 0;
  const uint64_t h2 = hash3(r.seed, static_cast<uint64_t>(net), static_cast<uint64_t>(c), 2);
  const bool glitch = u01(h2) < r.glitch_p;
  const uint64_t h3 = hash3(r.seed, static_cast<uint64_t>(net), static_cast<uint64_t>(c), 3);
  const int64_t lo0 = (c == 0) ? 1 : 0;
  if (!glitch) {
    t[0] = base + lo0 + static_cast<int64_t>(mul_rn(u01(h3), static_cast<double>(r.tpc - lo0)));
    return 1;
  }
  const uint64_t h4 = hash3(r.seed, static_cast<uint64_t>(net), static_cast<uint64_t>(c), 4);
  int64_t w = r.w_lo + static_cast<int64_t>(mul_rn(u01(h4), static_cast<double>(r.w_hi - r.w_lo + 1)));
  if (2 * w >= r.tpc - lo0) w = ((r.tpc - lo0 - 1) / 2) > 1 ? (r.tpc - lo0 - 1) / 2 : 1;
  const int64_t span = r.tpc - lo0 - 2 * w;
  const int64_t o = lo0 + static_cast<int64_t>(mul_rn(u01(h3), static_cast<double>(span)));
  t[0] = base + o;
  t[1] = base + o + w;
  t[2] = base + o + 2 * w;
  return 3;
}

// Initial net value at tick 0: a seeded coin; the clock starts at 0.
SYN_HD uint8_t initial_value(const Rules& r, int32_t net) {
  return net == r.clock_net ? 0 : static_cast<uint8_t>(hash3(r.seed, static_cast<uint64_t>(net), 0xABCDEFull, 5) & 1);
}

}  // namespace syn
}  // namespace gtpb
