// synth.cpp — seeded synthetic designs and traces for the power engine's
// workloads (host code, no CUDA).
//
// Netlist: n_cell cells drawn from a cell mix, levelized as a DAG. Every
// cell drives one net. A cell's data inputs are wired to nets created
// earlier (primary inputs, flip-flop outputs, earlier combinational
// outputs) that still have free fanout slots; each driver gets a fanout
// target ~ Geometric(p) capped at fanout_cap. Flip-flop clock pins go to
// one clock net. Wire cap per net ~ lognormal with the given mean and sigma.
//
// Trace: a counter-based generator keyed by (seed, net, cycle) so any
// cycle window of any net can be produced independently and in parallel:
//   mode 0 (uniform): per-net toggle probability u ~ U[lo, hi];
//   mode 1 (skew)   : per-net rate ~ Zipf(alpha) over a random net rank,
//                     scaled to mean `rate_mean`, times a per-cycle burst
//                     factor ~ lognormal(0, sigma) normalised to mean 1;
//   mode 2 (phases) : 16-state sticky Markov chain over cycles; each
//                     (phase, net) pair has its own rate ~ U[lo, hi].
//   mode 3 (phased units): the same phase chain; nets are split into n_unit
//                     contiguous id ranges ("units"), each net has a base
//                     rate u ~ U[lo, hi], and each (phase, unit) pair an
//                     activity factor a ~ lognormal(-s^2/2, s) (mean 1); the
//                     toggle probability is min(0.9, u * a).
// A toggle lands at a uniform offset within the cycle; with probability
// glitch_p it is followed by a pulse of width w ~ U[w_lo, w_hi] ticks (two
// extra value flips at +w and +2w, kept inside the cycle). The clock net
// rises at mid-cycle and falls at each later cycle boundary. Every net starts
// with an event at tick 0 (the VCD initial value); time_max = n_cycle*tpc.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "synth_rules.h"

namespace {

using gtpb::syn::hash3;
using gtpb::syn::splitmix;
using gtpb::syn::u01;

struct Rng {  // sequential generator for netlist construction
  uint64_t s;
  explicit Rng(uint64_t seed) : s(seed) {}
  uint64_t next() { s = splitmix(s); return s; }
  double uni() { return u01(next()); }
  int64_t below(int64_t n) { return static_cast<int64_t>(uni() * n) % n; }
  double normal() {
    double a = std::max(uni(), 1e-300), b = uni();
    return std::sqrt(-2.0 * std::log(a)) * std::cos(6.283185307179586 * b);
  }
};

struct Netlist {
  std::vector<int32_t> cell_type, cell_pin_off, pin_net;
  std::vector<double> wire_cap;
  int32_t n_net = 0;
  int32_t clock_net = -1;
  int32_t n_primary_inputs = 0;
};

struct TraceParams {
  int64_t n_cycle;
  int64_t tpc;
  uint64_t seed;
  int32_t mode;
  double lo, hi;             // mode 0 / 2 rate range
  double zipf_alpha, rate_mean, burst_sigma;  // mode 1
  int32_t n_phase;           // mode 2 / 3
  double p_stay;             // mode 2 / 3
  int32_t n_unit;            // mode 3
  double act_sigma;          // mode 3
  double glitch_p;
  int64_t w_lo, w_hi;
  int32_t clock_net;
  int32_t n_net;
};

struct Trace {
  TraceParams tp;
  std::vector<double> net_rate;     // mode 0/1/3
  std::vector<uint32_t> rank;       // mode 1
  std::vector<double> burst;        // mode 1: per cycle factor
  std::vector<uint8_t> phase;       // mode 2 / 3: per cycle phase
  std::vector<double> act;          // mode 3: [phase][unit] activity factor
  gtpb::syn::Rules rules{};         // view of the above, set once the tables are final
  void set_rules() {
    rules.mode = tp.mode;
    rules.clock_net = tp.clock_net;
    rules.n_net = tp.n_net;
    rules.n_unit = tp.n_unit;
    rules.n_cycle = tp.n_cycle;
    rules.tpc = tp.tpc;
    rules.seed = tp.seed;
    rules.lo = tp.lo;
    rules.hi = tp.hi;
    rules.glitch_p = tp.glitch_p;
    rules.w_lo = tp.w_lo;
    rules.w_hi = tp.w_hi;
    rules.net_rate = net_rate.empty() ? nullptr : net_rate.data();
    rules.burst = burst.empty() ? nullptr : burst.data();
    rules.phase = phase.empty() ? nullptr : phase.data();
    rules.act = act.empty() ? nullptr : act.data();
  }
};

// Events of one net in cycle c; writes up to 3 ticks.
inline int cycle_events(const Trace& tr, int32_t net, int64_t c, int64_t* t) {
  return gtpb::syn::cycle_events(tr.rules, net, c, t);
}

}  // namespace

extern "C" {

// cell mix: fraction per type, n_in per type (data inputs, clock counted
// separately through is_ff). Pins of a cell: inputs in type order, then the
// single output.
void* synth_netlist_create(int64_t n_cell, uint64_t seed, int32_t n_type, const double* mix,
                           const int32_t* type_n_in, const int32_t* type_is_ff,
                           double fanout_p, int32_t fanout_cap, double wire_mean,
                           double wire_sigma, double pi_fraction) {
  Netlist* nl = new Netlist();
  Rng rng(seed * 0x2545F4914F6CDD1Dull + 17);
  // exact type counts from the mix, then a seeded shuffle
  std::vector<int32_t> types;
  types.reserve(n_cell);
  double acc = 0;
  int64_t assigned = 0;
  for (int32_t t = 0; t < n_type; ++t) {
    acc += mix[t];
    const int64_t upto = (t == n_type - 1) ? n_cell : static_cast<int64_t>(std::llround(acc * n_cell));
    for (; assigned < upto; ++assigned) types.push_back(t);
  }
  for (int64_t i = n_cell - 1; i > 0; --i) std::swap(types[i], types[rng.below(i + 1)]);
  nl->cell_type = types;

  // nets: clock, primary inputs, then one output net per cell (net id = n_pre + cell)
  const int32_t n_pi = std::max<int32_t>(16, static_cast<int32_t>(pi_fraction * n_cell));
  nl->clock_net = 0;
  nl->n_primary_inputs = n_pi;
  const int32_t n_pre = 1 + n_pi;
  nl->n_net = n_pre + static_cast<int32_t>(n_cell);
  std::vector<int32_t> slots(nl->n_net, 0);
  auto fanout_target = [&]() {
    int k = 1;
    while (k < fanout_cap && rng.uni() >= fanout_p) ++k;
    return k;
  };
  std::vector<int32_t> open;  // nets with free fanout slots
  open.reserve(nl->n_net);
  for (int32_t n = 1; n < n_pre; ++n) { slots[n] = fanout_target(); open.push_back(n); }
  // flip-flop outputs exist from the start (sequential boundary)
  for (int64_t c = 0; c < n_cell; ++c)
    if (type_is_ff[types[c]]) {
      const int32_t net = n_pre + static_cast<int32_t>(c);
      slots[net] = fanout_target();
      open.push_back(net);
    }
  auto take = [&]() -> int32_t {
    if (open.empty()) {  // add a primary input on demand
      const int32_t net = nl->n_net++;
      slots.push_back(fanout_target());
      open.push_back(net);
      ++nl->n_primary_inputs;
    }
    const int64_t k = rng.below(static_cast<int64_t>(open.size()));
    const int32_t net = open[k];
    if (--slots[net] == 0) { open[k] = open.back(); open.pop_back(); }
    return net;
  };
  nl->cell_pin_off.resize(n_cell + 1);
  nl->cell_pin_off[0] = 0;
  // flip-flop data inputs are wired last (they may take any driver)
  std::vector<std::vector<int32_t>> pins(n_cell);
  for (int64_t c = 0; c < n_cell; ++c) {
    const int32_t t = types[c];
    const int32_t n_in = type_n_in[t];
    std::vector<int32_t>& p = pins[c];
    p.assign(n_in + 1, -1);
    if (!type_is_ff[t]) {
      for (int32_t i = 0; i < n_in; ++i) p[i] = take();
      const int32_t net = n_pre + static_cast<int32_t>(c);
      slots[net] = fanout_target();
      open.push_back(net);
    }
    p[n_in] = n_pre + static_cast<int32_t>(c);
  }
  for (int64_t c = 0; c < n_cell; ++c) {
    const int32_t t = types[c];
    if (!type_is_ff[t]) continue;
    const int32_t n_in = type_n_in[t];
    pins[c][0] = nl->clock_net;                    // CLK
    for (int32_t i = 1; i < n_in; ++i) pins[c][i] = take();
  }
  for (int64_t c = 0; c < n_cell; ++c) {
    nl->cell_pin_off[c + 1] = nl->cell_pin_off[c] + static_cast<int32_t>(pins[c].size());
    nl->pin_net.insert(nl->pin_net.end(), pins[c].begin(), pins[c].end());
  }
  // wire caps: lognormal with the requested mean
  nl->wire_cap.resize(nl->n_net);
  const double mu = std::log(wire_mean) - 0.5 * wire_sigma * wire_sigma;
  for (int32_t n = 0; n < nl->n_net; ++n) nl->wire_cap[n] = std::exp(mu + wire_sigma * rng.normal());
  return nl;
}

int64_t synth_netlist_size(void* h, int32_t which) {
  Netlist* nl = static_cast<Netlist*>(h);
  switch (which) {
    case 0: return static_cast<int64_t>(nl->cell_type.size());
    case 1: return static_cast<int64_t>(nl->pin_net.size());
    case 2: return nl->n_net;
    case 3: return nl->clock_net;
    case 4: return nl->n_primary_inputs;
  }
  return -1;
}

void synth_netlist_copy(void* h, int32_t* cell_type, int32_t* cell_pin_off, int32_t* pin_net,
                        double* wire_cap) {
  Netlist* nl = static_cast<Netlist*>(h);
  std::memcpy(cell_type, nl->cell_type.data(), sizeof(int32_t) * nl->cell_type.size());
  std::memcpy(cell_pin_off, nl->cell_pin_off.data(), sizeof(int32_t) * nl->cell_pin_off.size());
  std::memcpy(pin_net, nl->pin_net.data(), sizeof(int32_t) * nl->pin_net.size());
  std::memcpy(wire_cap, nl->wire_cap.data(), sizeof(double) * nl->wire_cap.size());
}

void synth_netlist_free(void* h) { delete static_cast<Netlist*>(h); }

void* synth_trace_create(int32_t n_net, int32_t clock_net, int64_t n_cycle, int64_t tpc,
                         uint64_t seed, int32_t mode, double lo, double hi, double zipf_alpha,
                         double rate_mean, double burst_sigma, int32_t n_phase, double p_stay,
                         double glitch_p, int64_t w_lo, int64_t w_hi) {
  Trace* tr = new Trace();
  TraceParams& tp = tr->tp;
  tp.n_cycle = n_cycle; tp.tpc = tpc; tp.seed = seed; tp.mode = mode;
  tp.lo = lo; tp.hi = hi; tp.zipf_alpha = zipf_alpha; tp.rate_mean = rate_mean;
  tp.burst_sigma = burst_sigma; tp.n_phase = n_phase; tp.p_stay = p_stay;
  tp.glitch_p = glitch_p; tp.w_lo = w_lo; tp.w_hi = w_hi; tp.clock_net = clock_net;
  tp.n_net = n_net;
  tp.n_unit = 1;
  tp.act_sigma = 0.0;
  Rng rng(seed ^ 0x1234567ull);
  if (mode == 0) {
    tr->net_rate.resize(n_net);
    for (int32_t n = 0; n < n_net; ++n)
      tr->net_rate[n] = lo + (hi - lo) * u01(hash3(seed, n, 0xFFFFFFFFull, 9));
  } else if (mode == 1) {
    // Zipf weights over a random rank permutation; per-cycle burst factors
    // normalised to mean 1; the weights' scale k is chosen so that the
    // toggle probability min(1, k * w[net] * burst[c]) averages rate_mean
    // over nets and cycles (clipping included)
    std::vector<uint32_t> perm(n_net);
    for (int32_t n = 0; n < n_net; ++n) perm[n] = n;
    for (int32_t i = n_net - 1; i > 0; --i) std::swap(perm[i], perm[rng.below(i + 1)]);
    tr->net_rate.resize(n_net);
    for (int32_t n = 0; n < n_net; ++n)
      tr->net_rate[n] = 1.0 / std::pow(static_cast<double>(perm[n]) + 1.0, zipf_alpha);
    tr->burst.resize(n_cycle);
    double bs = 0;
    for (int64_t c = 0; c < n_cycle; ++c) {
      tr->burst[c] = std::exp(burst_sigma * rng.normal());
      bs += tr->burst[c];
    }
    const double m = bs / std::max<int64_t>(1, n_cycle);
    for (int64_t c = 0; c < n_cycle; ++c) tr->burst[c] /= m;
    // mean rate for scale k over the sorted weights and (a sample of) the bursts
    std::vector<double> w(tr->net_rate);
    std::sort(w.begin(), w.end());
    std::vector<double> pre(w.size() + 1, 0.0);
    for (size_t i = 0; i < w.size(); ++i) pre[i + 1] = pre[i] + w[i];
    const int64_t stride = std::max<int64_t>(1, n_cycle / 4096);
    auto mean_rate = [&](double k) {
      double acc = 0;
      int64_t cnt = 0;
      for (int64_t c = 0; c < n_cycle; c += stride, ++cnt) {
        const double kb = k * tr->burst[c];
        const size_t j = static_cast<size_t>(std::upper_bound(w.begin(), w.end(), 1.0 / kb) - w.begin());
        acc += kb * pre[j] + static_cast<double>(w.size() - j);
      }
      return acc / (static_cast<double>(w.size()) * std::max<int64_t>(1, cnt));
    };
    double k_lo = 0.0, k_hi = rate_mean * n_net / std::max(pre.back(), 1e-300);
    const double target = std::min(rate_mean, 1.0);
    for (int it = 0; it < 200 && mean_rate(k_hi) < target && target < 1.0; ++it) k_hi *= 2.0;
    for (int it = 0; it < 100; ++it) {
      const double mid = 0.5 * (k_lo + k_hi);
      if (mean_rate(mid) < target) k_lo = mid;
      else k_hi = mid;
    }
    for (int32_t n = 0; n < n_net; ++n) tr->net_rate[n] *= k_hi;
  } else {
    tr->phase.resize(n_cycle);
    uint8_t ph = static_cast<uint8_t>(rng.below(n_phase));
    for (int64_t c = 0; c < n_cycle; ++c) {
      if (rng.uni() >= p_stay) ph = static_cast<uint8_t>(rng.below(n_phase));
      tr->phase[c] = ph;
    }
  }
  tr->set_rules();
  return tr;
}

// Mode 3 trace (phased units); see the header comment.
void* synth_trace_create_phased(int32_t n_net, int32_t clock_net, int64_t n_cycle, int64_t tpc,
                                uint64_t seed, double lo, double hi, int32_t n_phase, double p_stay,
                                int32_t n_unit, double act_sigma, double glitch_p, int64_t w_lo,
                                int64_t w_hi) {
  if (n_phase < 1 || n_phase > 255 || n_unit < 1 || n_net < 1) return nullptr;
  // the phase chain exactly as mode 2 draws it
  Trace* tr = static_cast<Trace*>(synth_trace_create(n_net, clock_net, n_cycle, tpc, seed, 2, lo, hi, 0.0,
                                                     0.0, 0.0, n_phase, p_stay, glitch_p, w_lo, w_hi));
  TraceParams& tp = tr->tp;
  tp.mode = 3;
  tp.n_unit = std::min(n_unit, n_net);
  tp.act_sigma = act_sigma;
  tr->net_rate.resize(n_net);
  for (int32_t n = 0; n < n_net; ++n)
    tr->net_rate[n] = lo + (hi - lo) * u01(hash3(seed, n, 0xFFFFFFFFull, 9));
  tr->act.resize(static_cast<size_t>(n_phase) * tp.n_unit);
  Rng ar(seed ^ 0xAC71u);
  for (double& a : tr->act) a = std::exp(act_sigma * ar.normal() - 0.5 * act_sigma * act_sigma);
  tr->set_rules();
  return tr;
}

void synth_trace_free(void* h) { delete static_cast<Trace*>(h); }

int32_t synth_trace_phase(void* h, int64_t c) {
  Trace* tr = static_cast<Trace*>(h);
  return tr->phase.empty() ? -1 : tr->phase[c];
}

// Events of every net for cycles [c_lo, c_hi), plus the tick-0 initial value
// when c_lo == 0. counts[n] receives the count per net.
void synth_trace_count(void* h, int64_t c_lo, int64_t c_hi, int64_t* counts, int32_t n_threads) {
  Trace* tr = static_cast<Trace*>(h);
  const int32_t nn = tr->tp.n_net;
  if (n_threads < 1) n_threads = 1;
  auto job = [&](int tid) {
    int64_t t[3];
    for (int32_t n = tid; n < nn; n += n_threads) {
      int64_t k = (c_lo == 0) ? 1 : 0;
      for (int64_t c = c_lo; c < c_hi; ++c) k += cycle_events(*tr, n, c, t);
      counts[n] = k;
    }
  };
  std::vector<std::thread> th;
  for (int i = 0; i < n_threads; ++i) th.emplace_back(job, i);
  for (auto& x : th) x.join();
}

// Fills times and one value byte per event (0/1) for cycles [c_lo, c_hi).
// init_value[n] is the net's value before c_lo (updated in place to the
// value after c_hi). off[n] is where net n's events start.
void synth_trace_fill(void* h, int64_t c_lo, int64_t c_hi, const int64_t* off,
                      uint8_t* init_value, int64_t* times, uint8_t* values, int32_t n_threads) {
  Trace* tr = static_cast<Trace*>(h);
  const int32_t nn = tr->tp.n_net;
  if (n_threads < 1) n_threads = 1;
  auto job = [&](int tid) {
    int64_t t[3];
    for (int32_t n = tid; n < nn; n += n_threads) {
      int64_t k = off[n];
      uint8_t v = init_value[n];
      if (c_lo == 0) {
        times[k] = 0;
        values[k] = v;
        ++k;
      }
      for (int64_t c = c_lo; c < c_hi; ++c) {
        const int m = cycle_events(*tr, n, c, t);
        for (int j = 0; j < m; ++j) {
          v ^= 1;
          times[k] = t[j];
          values[k] = v;
          ++k;
        }
      }
      init_value[n] = v;
    }
  };
  std::vector<std::thread> th;
  for (int i = 0; i < n_threads; ++i) th.emplace_back(job, i);
  for (auto& x : th) x.join();
}

// Packs one value per byte into 2-bit fields, 16 per uint32 word, with
// n_threads threads over word ranges.
void synth_pack_values(const uint8_t* values, int64_t n, uint32_t* packed, int32_t n_threads) {
  const int64_t nw = (n + 15) / 16;
  if (n_threads < 1) n_threads = 1;
  auto job = [&](int tid) {
    const int64_t per = (nw + n_threads - 1) / n_threads;
    const int64_t w0 = tid * per, w1 = std::min(nw, w0 + per);
    for (int64_t w = w0; w < w1; ++w) {
      uint32_t x = 0;
      const int64_t b = w * 16;
      const int64_t m = std::min<int64_t>(16, n - b);
      for (int64_t j = 0; j < m; ++j) x |= static_cast<uint32_t>(values[b + j] & 3) << (2 * j);
      packed[w] = x;
    }
  };
  std::vector<std::thread> th;
  for (int i = 0; i < n_threads; ++i) th.emplace_back(job, i);
  for (auto& x : th) x.join();
}

// ---------------------------------------------------------------------------
// Streaming: cycle windows with the context the power walk reads.
//
// Window k covers cycles [c_lo, c_hi). Besides its own events, each net
// lists (a) the events of the last clock period before c_lo that has any
// and the event before that period, and (b) the first events at or after
// c_hi that the glitch look-ahead can read: the next window's events are
// generated one call ahead and supply them; a net with none there is
// scanned further only when its last listed period ends in a glitch event
// (an even count of at least two), the only case in which the look-ahead
// reads past the window.
void synth_trace_initial(void* h, uint8_t* init_value);

namespace {

struct Stream {
  Trace* tr = nullptr;
  int64_t wcyc = 0;
  int32_t n_threads = 1;
  int64_t c_next = 0;                 // first cycle of the next window to emit
  std::vector<uint8_t> value_gen;     // net value after the last generated cycle
  std::vector<int64_t> gcount;        // events emitted in bodies so far, per net
  std::vector<int64_t> ring_t;        // [net][4] head context
  std::vector<uint8_t> ring_v;
  std::vector<uint8_t> ring_n;
  std::vector<uint8_t> ring_g0;       // ring's first event is the waveform's first
  // generated bodies: current (to emit) and next (look-ahead)
  std::vector<int64_t> b_off[2], b_t[2];
  std::vector<uint8_t> b_v[2];
  int64_t b_lo[2] = {0, 0}, b_hi[2] = {0, 0};
  int cur = 0;
  bool have[2] = {false, false};
};

void gen_body(Stream& s, int slot, int64_t c_lo, int64_t c_hi) {
  Trace& tr = *s.tr;
  const int32_t nn = tr.tp.n_net;
  std::vector<int64_t>& off = s.b_off[slot];
  off.assign(nn + 1, 0);
  std::vector<int64_t> cnt(nn);
  synth_trace_count(&tr, c_lo, c_hi, cnt.data(), s.n_threads);
  for (int32_t n = 0; n < nn; ++n) off[n + 1] = off[n] + cnt[n];
  s.b_t[slot].resize(off[nn]);
  s.b_v[slot].resize(off[nn]);
  synth_trace_fill(&tr, c_lo, c_hi, off.data(), s.value_gen.data(), s.b_t[slot].data(),
                   s.b_v[slot].data(), s.n_threads);
  s.b_lo[slot] = c_lo;
  s.b_hi[slot] = c_hi;
  s.have[slot] = true;
}

}  // namespace

void* synth_stream_create(void* trace, int64_t window_cycles, int32_t n_threads) {
  Trace* tr = static_cast<Trace*>(trace);
  Stream* s = new Stream();
  s->tr = tr;
  s->wcyc = std::max<int64_t>(1, window_cycles);
  s->n_threads = std::max(1, n_threads);
  const int32_t nn = tr->tp.n_net;
  s->value_gen.resize(nn);
  synth_trace_initial(tr, s->value_gen.data());
  s->gcount.assign(nn, 0);
  s->ring_t.assign(4 * static_cast<size_t>(nn), 0);
  s->ring_v.assign(4 * static_cast<size_t>(nn), 0);
  s->ring_n.assign(nn, 0);
  s->ring_g0.assign(nn, 0);
  return s;
}

void synth_stream_free(void* h) { delete static_cast<Stream*>(h); }

// Emits the next window into caller buffers (times, one value byte per
// event, net_off [n_net+1], net_base [n_net]) of capacity `cap` events.
// Returns the number of events written, 0 when the trace is exhausted, or
// -(events needed) when cap is too small (nothing is consumed then).
int64_t synth_stream_next(void* h, int64_t* t_lo, int64_t* t_hi, int64_t* net_off, int64_t* times,
                          uint8_t* values, int64_t* net_base, int64_t cap) {
  Stream& s = *static_cast<Stream*>(h);
  Trace& tr = *s.tr;
  const int64_t nc = tr.tp.n_cycle;
  const int32_t nn = tr.tp.n_net;
  if (s.c_next >= nc) return 0;
  const int a = s.cur, b = 1 - s.cur;
  const int64_t c_lo = s.c_next;
  const int64_t c_hi = std::min(nc, c_lo + s.wcyc);
  if (!s.have[a]) gen_body(s, a, c_lo, c_hi);
  if (c_hi < nc && !s.have[b]) gen_body(s, b, c_hi, std::min(nc, c_hi + s.wcyc));
  const int64_t tpc = tr.tp.tpc;
  // per-net layout
  std::vector<int64_t> tail_n(nn, 0);
  std::vector<int64_t> tail_t(2 * static_cast<size_t>(nn));
  std::vector<uint8_t> tail_v(2 * static_cast<size_t>(nn));
  auto period_of = [&](int64_t t) { return t / tpc; };
  auto job = [&](int tid) {
    int64_t tbuf[3];
    for (int32_t n = tid; n < nn; n += s.n_threads) {
      // events of the last listed period: body's last cycle, else the ring
      const int64_t bo = s.b_off[a][n], be = s.b_off[a][n + 1];
      int k_last = 0;
      bool g0_in = false;
      if (be > bo) {
        const int64_t pl = period_of(s.b_t[a][be - 1]);
        int64_t j = be - 1;
        while (j >= bo && period_of(s.b_t[a][j]) == pl) { ++k_last; --j; }
        g0_in = (c_lo == 0 && pl == 0);  // the tick-0 initial value is not counted
      } else if (c_lo > 0 && s.ring_n[n] > 0) {
        const int rn = s.ring_n[n];
        const int64_t pl = period_of(s.ring_t[4 * n + rn - 1]);
        for (int j = rn - 1; j >= 0 && period_of(s.ring_t[4 * n + j]) == pl; --j) ++k_last;
        g0_in = s.ring_g0[n] && period_of(s.ring_t[4 * n]) == pl;
      }
      const int k_eff = k_last - (g0_in ? 1 : 0);
      const bool need_far = k_eff >= 2 && (k_eff % 2) == 0;
      int64_t tn = 0;
      if (c_hi < nc) {
        const int64_t no = s.b_off[b][n], ne = s.b_off[b][n + 1];
        for (int64_t j = no; j < ne && tn < 2; ++j) {
          tail_t[2 * n + tn] = s.b_t[b][j];
          tail_v[2 * n + tn] = s.b_v[b][j];
          ++tn;
        }
        if (tn == 0 && need_far) {
          // scan past the look-ahead window for the next period with events
          uint8_t v = s.value_gen[n];
          for (int64_t c = s.b_hi[b]; c < nc && tn == 0; ++c) {
            const int m = cycle_events(tr, n, c, tbuf);
            for (int j = 0; j < m && tn < 2; ++j) {
              v ^= 1;
              tail_t[2 * n + tn] = tbuf[j];
              tail_v[2 * n + tn] = v;
              ++tn;
            }
          }
        }
      }
      tail_n[n] = tn;
    }
  };
  {
    std::vector<std::thread> th;
    for (int i = 0; i < s.n_threads; ++i) th.emplace_back(job, i);
    for (auto& x : th) x.join();
  }
  net_off[0] = 0;
  for (int32_t n = 0; n < nn; ++n) {
    const int64_t head = c_lo > 0 ? s.ring_n[n] : 0;
    net_off[n + 1] = net_off[n] + head + (s.b_off[a][n + 1] - s.b_off[a][n]) + tail_n[n];
  }
  const int64_t total = net_off[nn];
  if (total > cap) return -total;
  auto fill = [&](int tid) {
    for (int32_t n = tid; n < nn; n += s.n_threads) {
      int64_t k = net_off[n];
      const int64_t head = c_lo > 0 ? s.ring_n[n] : 0;
      for (int64_t j = 0; j < head; ++j) {
        times[k] = s.ring_t[4 * n + j];
        values[k] = s.ring_v[4 * n + j];
        ++k;
      }
      for (int64_t j = s.b_off[a][n]; j < s.b_off[a][n + 1]; ++j) {
        times[k] = s.b_t[a][j];
        values[k] = s.b_v[a][j];
        ++k;
      }
      for (int64_t j = 0; j < tail_n[n]; ++j) {
        times[k] = tail_t[2 * n + j];
        values[k] = tail_v[2 * n + j];
        ++k;
      }
      net_base[n] = s.gcount[n] - head;
      // new ring: last non-empty period of the body plus the event before it
      const int64_t bo = s.b_off[a][n], be = s.b_off[a][n + 1];
      if (be > bo) {
        const int64_t pl = period_of(s.b_t[a][be - 1]);
        int64_t j = be - 1;
        while (j - 1 >= bo && period_of(s.b_t[a][j - 1]) == pl) --j;
        // j = first event of the last period in the body
        int64_t src_t[4];
        uint8_t src_v[4];
        int m = 0;
        bool g0 = false;
        if (j - 1 >= bo) {
          src_t[m] = s.b_t[a][j - 1];
          src_v[m] = s.b_v[a][j - 1];
          ++m;
          g0 = (c_lo == 0 && j - 1 == bo);
        } else if (c_lo > 0 && s.ring_n[n] > 0) {
          src_t[m] = s.ring_t[4 * n + s.ring_n[n] - 1];
          src_v[m] = s.ring_v[4 * n + s.ring_n[n] - 1];
          ++m;
          g0 = s.ring_g0[n] && s.ring_n[n] == 1;
        } else {
          g0 = (c_lo == 0 && j == bo);
        }
        for (int64_t q = j; q < be && m < 4; ++q) {
          src_t[m] = s.b_t[a][q];
          src_v[m] = s.b_v[a][q];
          ++m;
        }
        for (int q = 0; q < m; ++q) {
          s.ring_t[4 * n + q] = src_t[q];
          s.ring_v[4 * n + q] = src_v[q];
        }
        s.ring_n[n] = static_cast<uint8_t>(m);
        s.ring_g0[n] = g0 ? 1 : 0;
        s.gcount[n] += be - bo;
      }
    }
  };
  {
    std::vector<std::thread> th;
    for (int i = 0; i < s.n_threads; ++i) th.emplace_back(fill, i);
    for (auto& x : th) x.join();
  }
  *t_lo = c_lo * tpc;
  *t_hi = c_hi < nc ? c_hi * tpc : INT64_MAX;
  s.have[a] = false;
  s.cur = b;
  s.c_next = c_hi;
  return total;
}

// Initial net values (tick 0): a seeded coin per net; the clock starts at 0.
void synth_trace_initial(void* h, uint8_t* init_value) {
  Trace* tr = static_cast<Trace*>(h);
  for (int32_t n = 0; n < tr->tp.n_net; ++n) init_value[n] = gtpb::syn::initial_value(tr->rules, n);
}

// The trace's parameters and tables, for a generator elsewhere (the device
// generator): fills *rules with host pointers into the trace, valid while the
// trace lives; returns the number of phases (0 when the mode has none).
int32_t synth_trace_rules(void* h, gtpb::syn::Rules* rules) {
  Trace* tr = static_cast<Trace*>(h);
  *rules = tr->rules;
  return tr->tp.n_phase;
}

}  // extern "C"
