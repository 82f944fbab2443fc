// oracle.cpp — CPU restatement of GTPower's time-based power path.
//
// TEST INFRASTRUCTURE ONLY. This file is the checker for the CUDA engine in
// gtpower_b200/csrc: only tests/, __graft_entry__.smoke() and bench.py's
// cpu_baseline / reference arm may load it. The product never calls it.
//
// It restates the reference CPU path line by line:
//   findTimeBasedAllPower            power/TimeBasedPower.cc:703-901
//   getEventClockCycleBasedGlitchFlags power/TimeBasedPower.cc:589-637
//   getGlitchScalingRatioClockCycleBasedH power/TimeBasedPower.cc:303-339
//   findInputInternalVal             power/TimeBasedPower.cc:341-381
//   findOutputInternalVal            power/TimeBasedPower.cc:383-509
//   getDefaultOutputPinInternalEnergyVal power/TimeBasedPower.cc:511-555
//   getLeakagePower / getStateIdx    power/TimeBasedPower.cc:258-301, 557-587
//   calculatePerCycleLeakagePower    power/TimeBasedPower.cc:677-701
//   getEventIdxByTime                power/TimeBasedPower.cc:639-653
//   clkedWaveformIdx, getNToggle, getNRise, getRiseFallEdge,
//   findLeakageVal, getTimeBasedGlitchScalingRatioH
//                                    power/PowerUtils.cc:27-32, 67-90, 213-294
//   Table0/1/2::findValue, findValueIndex
//                                    liberty/TableModel.cc:858-880, 1011-1060,
//                                    1467-1489; InternalPowerModel::power
//                                    liberty/InternalPower.cc:112-156, 186-228
//   Power::power (static thread split, per-thread per-cycle arrays, group
//   classification)                  power/Power.cc:227-386
//
// Two arithmetic modes:
//   Real = double : the FP64 oracle. Every quantity the reference keeps in
//                   float is kept in double; integer decisions (cycle index,
//                   glitch flags, related-pin choice) follow the reference's
//                   exact expressions, including the float rounding of the
//                   related-pin distance (EventTimeVal is float).
//   Real = float  : the reference's own FP32 types (util/Types.hh), used as
//                   the timed CPU baseline ("port" of the reference CPU path).
//
// Parity status: the reference binary cannot be built in this container
// (Tcl, SWIG, flex, bison, Eigen3, CUDD absent). The restatement is pinned
// (a) helper by helper against the reference's own table interpolation,
// toggle, rise, cycle-index and glitch-ratio functions compiled from its
// sources (oracle/Makefile target `ref`, tests/test_oracle_ref.py, and the
// vectors they produced in tests/golden/ref_vectors.npz), (b) on the walk as a
// whole by hand-derived known-answer cases (tests/test_oracle_kat.py) and the
// reference's GCD example report (tests/test_gcd.py).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <thread>
#include <vector>

#include "../include/gtpb200.h"

namespace {

constexpr int64_t kInvalidPulseWidth = -1;    // util/Defines.hh:8
constexpr float kInvalidNToggle = -1.0f;      // util/Defines.hh:9

struct Wave {            // one pin's waveform view (a net's event list)
  const int64_t* t = nullptr;
  const uint32_t* vp = nullptr;
  int64_t off = 0;       // absolute index of event 0 in the packed arrays
  int64_t n = 0;
  inline int64_t time(int64_t i) const { return t[off + i]; }
  inline int value(int64_t i) const {
    const int64_t a = off + i;
    return (vp[a >> 4] >> (2 * (a & 15))) & 3;
  }
};

// getNRise (power/PowerUtils.cc:213-237)
inline float nRise(int prev, int cur) {
  if (prev == cur) return 0.0f;
  if (cur == 2) return prev == 0 ? 0.5f : 0.0f;
  if (cur == 1) {
    if (prev == 2) return 0.5f;
    if (prev == 0) return 1.0f;
  }
  return 0.0f;
}
// getRiseFallEdge: RISE iff n_rise > 0 (power/PowerUtils.cc:239-245)
inline bool isRise(int prev, int cur) { return nRise(prev, cur) > 0; }
// getNToggle (power/PowerUtils.cc:247-255)
inline float nToggle(int prev, int cur) {
  if (prev == cur) return 0.0f;
  return (prev == 2 || cur == 2) ? 0.5f : 1.0f;
}

template <typename Real>
struct Engine {
  const gtp_design& d;
  const gtp_events& ev;
  int max_leak_pins;
  double ts;          // Vcd::timeScale (double)
  float ts_f;         // the same, as EventTimeVal float
  float period_f;     // Power::clk_period_
  double period_d;    // clk_period_ passed as double to calculatePerCycleLeakagePower
  int64_t tpc;        // ticks per cycle
  int64_t tmax;
  int64_t n_period;

  Engine(const gtp_design& design, const gtp_events& events, int mlp)
      : d(design), ev(events), max_leak_pins(mlp) {
    ts = d.timescale;
    ts_f = static_cast<float>(ts);
    period_f = d.clk_period;
    period_d = static_cast<double>(period_f);
    // clkedWaveformIdx: (VcdEventTime)ceil(period / vcd_time_scale), float/float
    tpc = static_cast<int64_t>(std::ceil(period_f / ts_f));
    tmax = d.time_max;
    // Power::power: ceil((timeMax * timeScale) / clk_period_) in double
    n_period = static_cast<int64_t>(std::ceil((static_cast<double>(tmax) * ts) / period_d));
  }

  int64_t cycleOf(int64_t t) const { return t / tpc; }

  // ---- Liberty table lookup (InternalPowerModel::power) ----
  static size_t findValueIndex(float value, const float* axis, int size) {
    if (size <= 1 || value <= axis[0]) return 0;
    if (value >= axis[size - 1]) return size - 2;
    int lower = -1, upper = size;
    while (upper - lower > 1) {
      int mid = (upper + lower) >> 1;
      if (value >= axis[mid]) lower = mid; else upper = mid;
    }
    return lower;
  }

  // Returns the table value at (in_slew, load_cap). In float mode the result
  // is rounded to float as Table*::findValue returns float; in double mode it
  // is kept in double.
  Real tableValue(int32_t ti, float in_slew, float load_cap) const {
    if (ti < 0) return Real(0);
    const gtp_table& tb = d.tables[ti];
    auto axisValue = [&](int var) -> float {
      return var == GTP_AXIS_SLEW ? in_slew : (var == GTP_AXIS_CAP ? load_cap : 0.0f);
    };
    const float* v = d.lut_pool + tb.value_off;
    double r;
    if (tb.order == 0) {
      r = v[0];
    } else if (tb.order == 1) {
      const float* a1 = d.lut_pool + tb.axis1_off;
      const float x = axisValue(tb.axis1_var);
      if (tb.n1 == 1) {
        // Table1::findValue calls value(axis_value1), i.e. an index built from
        // the axis value; for a one-point table that is entry 0.
        r = v[0];
      } else {
        size_t i = findValueIndex(x, a1, tb.n1);
        double x1 = x, x1l = a1[i], x1u = a1[i + 1];
        double y1 = v[i], y2 = v[i + 1];
        double dx1 = (x1 - x1l) / (x1u - x1l);
        r = (1 - dx1) * y1 + dx1 * y2;
      }
    } else {
      const float* a1 = d.lut_pool + tb.axis1_off;
      const float* a2 = d.lut_pool + tb.axis2_off;
      const float x1f = axisValue(tb.axis1_var), x2f = axisValue(tb.axis2_var);
      const int n1 = tb.n1, n2 = tb.n2;
      auto val = [&](size_t i, size_t j) -> double { return v[i * n2 + j]; };
      if (n1 == 1) {
        if (n2 == 1) {
          r = val(0, 0);
        } else {
          size_t j = findValueIndex(x2f, a2, n2);
          double x2 = x2f, y00 = val(0, j), x2l = a2[j], x2u = a2[j + 1];
          double dx2 = (x2 - x2l) / (x2u - x2l);
          double y01 = val(0, j + 1);
          r = (1 - dx2) * y00 + dx2 * y01;
        }
      } else if (n2 == 1) {
        size_t i = findValueIndex(x1f, a1, n1);
        double x1 = x1f, y00 = val(i, 0), x1l = a1[i], x1u = a1[i + 1];
        double dx1 = (x1 - x1l) / (x1u - x1l);
        double y10 = val(i + 1, 0);
        r = (1 - dx1) * y00 + dx1 * y10;
      } else {
        size_t i = findValueIndex(x1f, a1, n1);
        size_t j = findValueIndex(x2f, a2, n2);
        double x1 = x1f, x2 = x2f;
        double y00 = val(i, j);
        double x1l = a1[i], x1u = a1[i + 1];
        double dx1 = (x1 - x1l) / (x1u - x1l);
        double y10 = val(i + 1, j), y11 = val(i + 1, j + 1);
        double x2l = a2[j], x2u = a2[j + 1];
        double dx2 = (x2 - x2l) / (x2u - x2l);
        double y01 = val(i, j + 1);
        r = (1 - dx1) * (1 - dx2) * y00 + dx1 * (1 - dx2) * y10 +
            dx1 * dx2 * y11 + (1 - dx1) * dx2 * y01;
      }
    }
    if (std::is_same<Real, float>::value) {
      return static_cast<Real>(static_cast<float>(r) * tb.scale);
    }
    return static_cast<Real>(r * static_cast<double>(tb.scale));
  }

  // InternalPower::power(rf, pvt, slew, cap): model of the requested edge.
  Real groupPower(const gtp_internal_power& g, bool rise, float slew, float cap) const {
    return tableValue(rise ? g.rise_table : g.fall_table, slew, cap);
  }

  // evalWhen over the ones mask (power/PowerUtils.cc:153-186)
  bool whenHolds(const gtp_when& w, uint32_t ones) const {
    for (int k = 0; k < w.n_cube; ++k) {
      const uint32_t care = d.when_cubes[2 * (w.cube_off + k)];
      const uint32_t val = d.when_cubes[2 * (w.cube_off + k) + 1];
      if ((ones & care) == val) return true;
    }
    return false;
  }

  static uint32_t onesMask(const std::vector<int>& st) {
    uint32_t m = 0;
    for (size_t i = 0; i < st.size() && i < 32; ++i)
      if (st[i] == 1) m |= (1u << i);
    return m;
  }

  // getPinStatesIndex (power/PowerUtils.cc:40-48)
  static size_t stateIndex(const std::vector<int>& st) {
    size_t r = 0;
    for (size_t i = 0; i < st.size(); ++i)
      if (st[i] == 1) r += (size_t(1) << i);
    return r;
  }

  // Power::getLeakagePower (power/TimeBasedPower.cc:258-301)
  void leakageTable(const gtp_cell_type& ty, std::vector<Real>& table, Real& def,
                    bool& def_exists) const {
    def = static_cast<Real>(ty.cell_leakage_power);
    def_exists = ty.has_cell_leakage_power != 0;
    table.clear();
    const int n_pin = ty.n_pin;
    if (n_pin > max_leak_pins) {
      if (ty.n_leak == 1) {
        def = static_cast<Real>(d.leakage_powers[ty.leak_off].power);
        def_exists = true;
      }
      return;
    }
    if (ty.n_leak == 0) return;
    const size_t n_state = size_t(1) << n_pin;
    table.assign(n_state, def_exists ? def : Real(0));
    for (int k = 0; k < ty.n_leak; ++k) {
      const gtp_leakage_power& lp = d.leakage_powers[ty.leak_off + k];
      if (lp.when.n_cube != 1) continue;  // unsupported / unsatisfiable
      const uint32_t care = d.when_cubes[2 * lp.when.cube_off];
      const uint32_t val = d.when_cubes[2 * lp.when.cube_off + 1];
      for (size_t s = 0; s < n_state; ++s)
        if ((static_cast<uint32_t>(s) & care) == val) table[s] = static_cast<Real>(lp.power);
    }
  }

  // getEventClockCycleBasedGlitchFlags(values, 0, n) (TimeBasedPower.cc:589-637)
  void glitchFlags(const Wave& w, std::vector<char>& flags) const {
    flags.assign(static_cast<size_t>(w.n), 0);
    if (w.n == 0) return;
    std::vector<int64_t> cur;
    int64_t cur_period = cycleOf(w.time(0));
    auto close = [&]() {
      const size_t k = cur.size();
      if (k >= 2) {
        const size_t lim = (k % 2 == 0) ? k : k - 1;
        for (size_t i = 0; i < lim; ++i) flags[cur[i]] = 1;
      }
    };
    for (int64_t pos = 1; pos < w.n; ++pos) {
      const int64_t p = cycleOf(w.time(pos));
      if (p != cur_period) {
        close();
        cur_period = p;
        cur.clear();
      }
      cur.push_back(pos);
    }
    close();
  }

  // getTimeBasedGlitchScalingRatioH (power/PowerUtils.cc:285-294)
  Real glitchRatio(int64_t width_ticks, float slew_r, float slew_f) const {
    if (std::is_same<Real, float>::value) {
      const float pulse = static_cast<float>(static_cast<double>(width_ticks) * ts);
      const float sum = slew_r + slew_f;
      if (sum == 0) return Real(1);
      const float ratio = static_cast<float>((pulse * 2.0) / sum);
      return static_cast<Real>(std::min(1.0f, ratio * ratio));
    }
    const double pulse = static_cast<double>(width_ticks) * ts;
    const double sum = static_cast<double>(slew_r) + static_cast<double>(slew_f);
    if (sum == 0) return Real(1);
    const double ratio = (pulse * 2.0) / sum;
    return static_cast<Real>(std::min(1.0, ratio * ratio));
  }

  // getEventIdxByTime (TimeBasedPower.cc:639-653): first index with time >= t
  static int64_t lowerBound(const Wave& w, int64_t t) {
    int64_t left = 0, right = w.n;
    while (left < right) {
      int64_t mid = left + (right - left) / 2;
      if (w.time(mid) < t) left = mid + 1; else right = mid;
    }
    return right;
  }

  struct CellOut {
    Real internal = 0, glitch_internal = 0, switching = 0, glitch_switching = 0, leakage = 0;
    uint32_t events = 0, glitches = 0, half_toggles = 0, related = 0;
  };

  // Census of the reference CPU/CUDA divergences: pin events whose CUDA-path
  // decision (power/cuda/CudaPower.cu:115-315, 317-584) differs from the CPU
  // path's, counted while the CPU path is walked. The CUDA rules are taken
  // for one thread over the whole trace (no cycle-chunk seams).
  struct Census {
    int64_t pin_events = 0;          // every walked pin event
    int64_t toggles = 0;             // events that toggle (the CUDA kernel skips the others)
    int64_t same_tick_state = 0;     // input toggles looked up by the CUDA kernel with the new
                                     // values of pins that toggled earlier at the same tick
                                     // (it walks them in event-index order, updating as it goes)
    int64_t same_tick_energy = 0;    // of those, the ones whose energy differs
    int64_t first_event_state = 0;   // pins whose net's first event is after t=0: the CPU path
                                     // walks it from X, the CUDA kernel takes it as the initial
                                     // state (counted once per pin, compared no further)
    int64_t glitch_class_diff = 0;   // glitch or not differs (online per-period counters,
                                     // unflagged neighbours, the t=0 initial event)
    int64_t glitch_width_diff = 0;   // both glitch, other pulse width
    int64_t related_diff = 0;        // output toggles with another related input (delay rounded
                                     // to ticks, same-cycle rule for logic cells only, ties)
    int64_t no_group_match = 0;      // output toggles with a related input but no matching
                                     // `when` group: 0 on the CPU, the default average on CUDA
    int64_t beyond_cuda_cycles = 0;  // toggles in a cycle at or past ceil(time_max / ticks per
                                     // cycle): the CUDA kernel's last thread ends one tick past
                                     // its last cycle, so it walks those at that tick and adds
                                     // their per-cycle terms past its arrays
    int64_t z_events = 0;            // toggles to or from Z, outside the CUDA 3x3 toggle tables
  };

  struct CycleAcc {
    std::vector<Real> leak, internal, g_internal, sw, g_sw;
    std::vector<int64_t> events, glitches;
    int64_t dropped = 0;
    void init(int64_t n) {
      leak.assign(n, 0); internal.assign(n, 0); g_internal.assign(n, 0);
      sw.assign(n, 0); g_sw.assign(n, 0);
      events.assign(n, 0); glitches.assign(n, 0);
    }
  };

  inline void addCycle(std::vector<Real>& a, int64_t c, Real v, CycleAcc& acc) const {
    if (c >= 0 && c < static_cast<int64_t>(a.size())) a[c] += v; else ++acc.dropped;
  }

  // Power::calculatePerCycleLeakagePower (TimeBasedPower.cc:677-701).
  void perCycleLeakage(Real val, int64_t prev, int64_t cur, CycleAcc& acc) const {
    if (std::is_same<Real, float>::value) {
      float left = static_cast<float>(prev * ts);
      int64_t c = cycleOf(prev);
      while (c * period_d <= cur * ts) {
        float right = static_cast<float>(std::min((c + 1) * period_d, cur * ts));
        float duration = right - left;
        addCycle(acc.leak, c, static_cast<Real>(static_cast<float>(val) * duration / period_d), acc);
        left = static_cast<float>((c + 1) * period_d);
        ++c;
      }
      return;
    }
    double left = prev * ts;
    int64_t c = cycleOf(prev);
    while (c * period_d <= cur * ts) {
      double right = std::min((c + 1) * period_d, cur * ts);
      double duration = right - left;
      addCycle(acc.leak, c, static_cast<Real>(static_cast<double>(val) * duration / period_d), acc);
      left = (c + 1) * period_d;
      ++c;
    }
  }

  // findTimeBasedAllPower for one instance.
  void cell(int32_t ci, CellOut& out, CycleAcc& acc, Census* cen = nullptr) const {
    const int32_t p0 = d.cell_pin_off[ci];
    const gtp_cell_type& ty = d.types[d.cell_type[ci]];
    const int n_pin = ty.n_pin, n_in = ty.n_in;
    const float* arcs = d.arc_delay + d.cell_arc_off[ci];

    std::vector<Wave> waves(n_pin);
    for (int i = 0; i < n_pin; ++i) {
      const int32_t net = d.pin_net[p0 + i];
      if (net >= 0) {
        waves[i].t = ev.time;
        waves[i].vp = ev.value_packed;
        waves[i].off = ev.net_off[net];
        waves[i].n = ev.net_off[net + 1] - ev.net_off[net];
      }
    }
    std::vector<std::vector<char>> gflags(n_pin);
    for (int i = 0; i < n_pin; ++i) {
      if (!d.pin_is_clock[p0 + i]) glitchFlags(waves[i], gflags[i]);
      else gflags[i].assign(static_cast<size_t>(waves[i].n), 0);
    }
    // pin_single_switching_energies: load_cap * volt * volt for outputs
    std::vector<Real> sw_energy(n_pin, Real(0));
    for (int i = n_in; i < n_pin; ++i) {
      const Real cap = d.pin_load_cap[p0 + i];
      const Real v = d.pin_voltage[p0 + i];
      sw_energy[i] = cap * v * v;
    }
    std::vector<Real> leak_tab;
    Real leak_def;
    bool leak_def_exists;
    leakageTable(ty, leak_tab, leak_def, leak_def_exists);
    auto leakVal = [&](const std::vector<int>& st) -> Real {
      if (!leak_tab.empty()) return leak_tab[stateIndex(st)];
      return leak_def_exists ? leak_def : Real(0);
    };

    const int64_t MAX_TIME = tmax + 10;
    std::vector<int64_t> frontier(n_pin, 0);
    std::vector<int> prev_st(n_pin, -1);
    for (int i = 0; i < n_pin; ++i) {
      if (waves[i].n == 0) {
        prev_st[i] = d.pin_default_state[p0 + i];
        continue;
      }
      if (waves[i].time(0) == 0) {
        prev_st[i] = waves[i].value(0);
        frontier[i] = 1;
      } else {
        prev_st[i] = 2;
      }
    }
    int64_t prev_time = 0;
    std::vector<int> st = prev_st;
    std::vector<char> trig(n_pin, 0);
    const double norm_dyn = static_cast<double>(tmax) * ts;  // timeMax * timeScale
    // census: the CUDA kernel's per-pin period counters
    // (getGlitchScalingRatioClockCycleBasedOnDeviceOnly, CudaPower.cu:270-315)
    std::vector<int64_t> cu_period(cen ? n_pin : 0, -1), cu_count(cen ? n_pin : 0, 0);
    const int64_t cuda_cycles = (tmax + tpc - 1) / tpc;   // ceil_div(max_time, ticks), CudaPower.cu:2662
    const bool is_logic = (d.cell_group ? d.cell_group[ci] : 0) == GTP_GROUP_COMBINATIONAL;
    std::vector<uint32_t> seq_ones(cen ? n_pin : 0, 0);
    std::vector<int> order;
    if (cen)
      for (int i = 0; i < n_pin; ++i)
        if (waves[i].n > 0 && waves[i].time(0) != 0) ++cen->first_event_state;

    auto slew = [&](int pin, bool rise) -> float {
      return rise ? d.pin_slew_rise[p0 + pin] : d.pin_slew_fall[p0 + pin];
    };
    auto cap = [&](int pin) -> float { return d.pin_load_cap[p0 + pin]; };

    while (true) {
      int64_t cur = MAX_TIME;
      for (int i = 0; i < n_pin; ++i) {
        if (frontier[i] >= waves[i].n) continue;
        cur = std::min(waves[i].time(frontier[i]), cur);
      }
      if (cur == MAX_TIME) break;
      for (int i = 0; i < n_pin; ++i) {
        if (frontier[i] >= waves[i].n) continue;
        if (waves[i].time(frontier[i]) == cur) {
          st[i] = waves[i].value(frontier[i]);
          trig[i] = 1;
          ++frontier[i];
        }
      }
      const Real lv = leakVal(prev_st);
      perCycleLeakage(lv, prev_time, cur, acc);
      out.leakage += lv * static_cast<Real>(cur - prev_time) / static_cast<Real>(tmax);

      const uint32_t ones = onesMask(prev_st);
      const int64_t cyc = cycleOf(cur);
      if (cen) {
        // the CUDA kernel's order (triggered pins by event index) and the states each
        // lookup sees in it
        order.clear();
        for (int i = 0; i < n_pin; ++i)
          if (trig[i] && frontier[i] - 1 > 0) order.push_back(i);
        std::sort(order.begin(), order.end(), [&](int a, int b) {
          return waves[a].off + frontier[a] < waves[b].off + frontier[b];
        });
        std::vector<int> seq = prev_st;
        for (int i : order) {
          seq_ones[i] = onesMask(seq);
          seq[i] = st[i];
        }
      }
      for (int i = 0; i < n_pin; ++i) {
        if (!trig[i]) continue;
        const float n_tog = nToggle(prev_st[i], st[i]);
        const bool rise = isRise(prev_st[i], st[i]);
        // the CUDA kernel walks this event: it toggles and is not the net's first event (the
        // initial state there)
        const bool cu_walk = cen && n_tog != 0.0f && frontier[i] - 1 > 0;
        if (cen) {
          ++cen->pin_events;
          if (n_tog != 0.0f) {
            ++cen->toggles;
            if (cyc >= cuda_cycles) ++cen->beyond_cuda_cycles;
            if (prev_st[i] == 3 || st[i] == 3) ++cen->z_events;
          }
        }
        // getGlitchScalingRatioClockCycleBasedH
        Real g = kInvalidNToggle;
        {
          const int64_t e = frontier[i] - 1;
          const std::vector<char>& fl = gflags[i];
          if (fl[e]) {
            int64_t pw = kInvalidPulseWidth, nw = kInvalidPulseWidth;
            if (e - 1 >= 0 && fl[e - 1]) pw = waves[i].time(e) - waves[i].time(e - 1);
            if (e + 1 < waves[i].n && fl[e + 1]) nw = waves[i].time(e + 1) - waves[i].time(e);
            const int64_t w = std::max(pw, nw);
            if (w != kInvalidPulseWidth) g = glitchRatio(w, slew(i, true), slew(i, false));
          }
        }
        if (cu_walk && !d.pin_is_clock[p0 + i]) {
          // the CUDA rule for this event (called for toggling events only)
          const Wave& w = waves[i];
          const int64_t e = frontier[i] - 1;
          const int64_t pc = cycleOf(w.time(e));
          if (pc == cu_period[i]) ++cu_count[i];
          else { cu_period[i] = pc; cu_count[i] = 1; }
          int64_t cpw = kInvalidPulseWidth, cnw = kInvalidPulseWidth;
          bool cu_none = false;
          if (e - 1 >= 0 && cycleOf(w.time(e - 1)) == pc) cpw = w.time(e) - w.time(e - 1);
          if (e + 1 < w.n && cycleOf(w.time(e + 1)) == pc) {
            if ((e + 2 < w.n && cycleOf(w.time(e + 2)) == pc) || cu_count[i] % 2 == 1) cnw = w.time(e + 1) - w.time(e);
          } else if (cu_count[i] % 2 == 1) {
            cu_none = true;
          }
          const int64_t cw = cu_none ? kInvalidPulseWidth : std::max(cpw, cnw);
          // the CPU path's width, or invalid
          int64_t qw = kInvalidPulseWidth;
          if (gflags[i][e]) {
            int64_t pw = kInvalidPulseWidth, nw = kInvalidPulseWidth;
            if (e - 1 >= 0 && gflags[i][e - 1]) pw = w.time(e) - w.time(e - 1);
            if (e + 1 < w.n && gflags[i][e + 1]) nw = w.time(e + 1) - w.time(e);
            qw = std::max(pw, nw);
          }
          if ((cw != kInvalidPulseWidth) != (qw != kInvalidPulseWidth)) ++cen->glitch_class_diff;
          else if (cw != qw) ++cen->glitch_width_diff;
        }
        Real energy = 0;
        int related_code = -1;
        if (i < n_in) {
          // findInputInternalVal
          const float s = slew(i, rise);
          if (!std::isinf(s)) {
            for (int k = 0; k < ty.n_ipwr; ++k) {
              const gtp_internal_power& gp = d.internal_powers[ty.ipwr_off + k];
              if (gp.pin != i) continue;
              if (whenHolds(gp.when, ones)) {
                energy = groupPower(gp, rise, s, 0.0f);
                break;
              }
            }
          }
          if (cu_walk && seq_ones[i] != ones) {
            ++cen->same_tick_state;
            Real alt = 0;
            if (!std::isinf(s)) {
              for (int k = 0; k < ty.n_ipwr; ++k) {
                const gtp_internal_power& gp = d.internal_powers[ty.ipwr_off + k];
                if (gp.pin != i) continue;
                if (whenHolds(gp.when, seq_ones[i])) {
                  alt = groupPower(gp, rise, s, 0.0f);
                  break;
                }
              }
            }
            if (alt != energy) ++cen->same_tick_energy;
          }
        } else {
          // findOutputInternalVal
          const int out_local = i - n_in;
          float min_diff = static_cast<float>(static_cast<double>(tmax) * ts);
          int rel = -1;
          int64_t rel_e = -1;
          for (int q = 0; q < n_in; ++q) {
            const Wave& wq = waves[q];
            if (wq.n == 0) continue;
            const int64_t re = std::max<int64_t>(0, lowerBound(wq, cur) - 1);
            const int64_t pe = std::max<int64_t>(0, re - 1);
            const bool from_rise = isRise(wq.value(pe), wq.value(re));
            const float dl = arcs[(static_cast<int64_t>(out_local) * n_in + q) * 4 +
                                  2 * (from_rise ? 0 : 1) + (rise ? 0 : 1)];
            if (std::isnan(dl)) continue;
            const float diff = static_cast<float>(
                std::abs(cur * ts - static_cast<double>(dl) - wq.time(re) * ts));
            if (diff < min_diff && cycleOf(wq.time(re)) == cyc) {
              min_diff = diff;
              rel = q;
              rel_e = re;
            }
          }
          if (cu_walk) {
            // the CUDA rule (getOutputPinInternalEnergyVal, CudaPower.cu:172-235)
            int64_t min_t = tmax;
            int cu_rel = -1;
            int64_t cu_e = -1;
            for (int q = 0; q < n_in; ++q) {
              const Wave& wq = waves[q];
              if (wq.n == 0) continue;
              const int64_t re = std::max<int64_t>(0, lowerBound(wq, cur) - 1);
              const int64_t pe = std::max<int64_t>(0, re - 1);
              const bool from_rise = isRise(wq.value(pe), wq.value(re));
              const float dl = arcs[(static_cast<int64_t>(out_local) * n_in + q) * 4 +
                                    2 * (from_rise ? 0 : 1) + (rise ? 0 : 1)];
              if (std::isnan(dl)) continue;
              const double dt = static_cast<double>(dl) / static_cast<double>(static_cast<float>(ts));
              const int64_t dtk = static_cast<int64_t>(dt >= 0.0 ? dt + 0.5 : dt - 0.5);
              const int64_t delta = cur - (wq.time(re) + dtk);
              const int64_t diff = delta >= 0 ? delta : -delta;
              if (is_logic && cycleOf(wq.time(re)) != cyc) continue;
              const int64_t tie = diff >= min_t ? diff - min_t : min_t - diff;
              const bool near_tie = cu_rel >= 0 && wq.time(re) == waves[cu_rel].time(cu_e) && tie <= 1;
              if (diff < min_t || (near_tie && re + wq.off > cu_e + waves[cu_rel].off)) {
                min_t = diff;
                cu_rel = q;
                cu_e = re;
              }
            }
            if (cu_rel != rel) ++cen->related_diff;
          }
          if (rel < 0) {
            // getDefaultOutputPinInternalEnergyVal
            int n_table = 0;
            Real total = 0;
            for (int q = 0; q < n_in; ++q) {
              for (int fr = 0; fr < 2; ++fr) {
                const float s = slew(q, fr == 0);
                if (std::isinf(s)) continue;
                for (int k = 0; k < ty.n_ipwr; ++k) {
                  const gtp_internal_power& gp = d.internal_powers[ty.ipwr_off + k];
                  if (gp.pin != i || gp.related_pin != q) continue;
                  total += groupPower(gp, rise, s, cap(i));
                  ++n_table;
                }
              }
            }
            energy = n_table == 0 ? Real(0) : total / static_cast<Real>(n_table);
            related_code = 0;
          } else {
            const Wave& wr = waves[rel];
            const int64_t pe = std::max<int64_t>(0, rel_e - 1);
            const bool from_rise = isRise(wr.value(pe), wr.value(rel_e));
            const float s = slew(rel, from_rise);
            bool matched = false;
            if (!std::isinf(s)) {
              for (int k = 0; k < ty.n_ipwr; ++k) {
                const gtp_internal_power& gp = d.internal_powers[ty.ipwr_off + k];
                if (gp.pin != i || gp.related_pin != rel) continue;
                if (whenHolds(gp.when, ones)) {
                  energy = groupPower(gp, rise, s, cap(i));
                  matched = true;
                  break;
                }
              }
            }
            if (cu_walk && !matched) ++cen->no_group_match;
            related_code = rel + 1;
          }
          // switching
          const float nr = nRise(prev_st[i], st[i]);
          if (nr > 0) {
            const Real esw = static_cast<Real>(nr) * sw_energy[i];
            if (g > 0) {
              out.glitch_switching += (g * esw) / static_cast<Real>(norm_dyn);
              addCycle(acc.sw, cyc, (g * esw) / static_cast<Real>(period_f), acc);
              addCycle(acc.g_sw, cyc, (g * esw) / static_cast<Real>(period_f), acc);
            } else {
              out.switching += esw / static_cast<Real>(norm_dyn);
              addCycle(acc.sw, cyc, esw / static_cast<Real>(period_f), acc);
            }
          }
          out.related += static_cast<uint32_t>(related_code);
        }
        energy *= static_cast<Real>(n_tog);
        if (g > 0) {
          out.glitch_internal += g * energy / static_cast<Real>(norm_dyn);
          addCycle(acc.internal, cyc, g * energy / static_cast<Real>(period_f), acc);
          addCycle(acc.g_internal, cyc, g * energy / static_cast<Real>(period_f), acc);
          ++out.glitches;
          if (cyc >= 0 && cyc < static_cast<int64_t>(acc.glitches.size())) ++acc.glitches[cyc];
        } else {
          out.internal += energy / static_cast<Real>(norm_dyn);
          addCycle(acc.internal, cyc, energy / static_cast<Real>(period_f), acc);
        }
        ++out.events;
        out.half_toggles += static_cast<uint32_t>(2.0f * n_tog);
        if (cyc >= 0 && cyc < static_cast<int64_t>(acc.events.size())) ++acc.events[cyc];
      }
      prev_time = cur;
      prev_st = st;
      std::fill(trig.begin(), trig.end(), 0);
    }
    const Real flv = leakVal(prev_st);
    perCycleLeakage(flv, prev_time, tmax, acc);
    out.leakage += flv * static_cast<Real>(tmax - prev_time) / static_cast<Real>(tmax);
  }
};

struct Result {
  double* cell5;
  double* cycle5;
  double* totals;
  double* groups;
  uint32_t* c_events;
  uint32_t* c_glitches;
  uint32_t* c_half;
  uint32_t* c_related;
  int64_t* y_events;
  int64_t* y_glitches;
  int64_t* dropped;
};

template <typename Real>
int runImpl(const gtp_design* d, const gtp_events* ev, const int32_t* cells, int32_t n_cells,
            int n_threads, int max_leak_pins, const Result& r) {
  Engine<Real> eng(*d, *ev, max_leak_pins);
  const int64_t np = eng.n_period;
  std::vector<int32_t> list;
  if (cells) list.assign(cells, cells + n_cells);
  else {
    list.resize(d->n_cell);
    for (int32_t i = 0; i < d->n_cell; ++i) list[i] = i;
  }
  if (n_threads < 1) n_threads = 1;
  const size_t n = list.size();
  using Acc = typename Engine<Real>::CycleAcc;
  using Out = typename Engine<Real>::CellOut;
  std::vector<Acc> accs(n_threads);
  std::vector<Out> outs(n);
  // static split as Power::power (power/Power.cc:284-293)
  const size_t base = n / n_threads, rem = n % n_threads;
  auto job = [&](int tid) {
    accs[tid].init(np);
    const size_t start = tid * base + std::min<size_t>(tid, rem);
    const size_t end = start + base + (static_cast<size_t>(tid) < rem ? 1 : 0);
    for (size_t k = start; k < end; ++k) eng.cell(list[k], outs[k], accs[tid]);
  };
  if (n_threads == 1) job(0);
  else {
    std::vector<std::thread> th;
    for (int t = 0; t < n_threads; ++t) th.emplace_back(job, t);
    for (auto& t : th) t.join();
  }
  // merge (power/Power.cc:318-347)
  if (r.cycle5) std::memset(r.cycle5, 0, sizeof(double) * 5 * np);
  if (r.y_events) std::memset(r.y_events, 0, sizeof(int64_t) * np);
  if (r.y_glitches) std::memset(r.y_glitches, 0, sizeof(int64_t) * np);
  int64_t dropped = 0;
  for (int t = 0; t < n_threads; ++t) {
    const Acc& a = accs[t];
    dropped += a.dropped;
    for (int64_t c = 0; c < np; ++c) {
      if (r.cycle5) {
        r.cycle5[0 * np + c] += a.leak[c];
        r.cycle5[1 * np + c] += a.internal[c];
        r.cycle5[2 * np + c] += a.g_internal[c];
        r.cycle5[3 * np + c] += a.sw[c];
        r.cycle5[4 * np + c] += a.g_sw[c];
      }
      if (r.y_events) r.y_events[c] += a.events[c];
      if (r.y_glitches) r.y_glitches[c] += a.glitches[c];
    }
  }
  if (r.dropped) *r.dropped = dropped;
  double tot[5] = {0, 0, 0, 0, 0};
  double grp[GTP_N_GROUP][5];
  std::memset(grp, 0, sizeof(grp));
  for (size_t k = 0; k < n; ++k) {
    const int32_t ci = list[k];
    const Out& o = outs[k];
    // timeBasedPower folds glitch into internal/switching (TimeBasedPower.cc:203-204)
    const double v5[5] = {static_cast<double>(o.leakage),
                          static_cast<double>(o.internal) + static_cast<double>(o.glitch_internal),
                          static_cast<double>(o.glitch_internal),
                          static_cast<double>(o.switching) + static_cast<double>(o.glitch_switching),
                          static_cast<double>(o.glitch_switching)};
    if (r.cell5) {
      r.cell5[5 * ci + 0] = o.internal;
      r.cell5[5 * ci + 1] = o.glitch_internal;
      r.cell5[5 * ci + 2] = o.switching;
      r.cell5[5 * ci + 3] = o.glitch_switching;
      r.cell5[5 * ci + 4] = o.leakage;
    }
    const int g = d->cell_group ? d->cell_group[ci] : 0;
    for (int q = 0; q < 5; ++q) {
      tot[q] += v5[q];
      grp[g][q] += v5[q];
    }
    if (r.c_events) r.c_events[ci] = o.events;
    if (r.c_glitches) r.c_glitches[ci] = o.glitches;
    if (r.c_half) r.c_half[ci] = o.half_toggles;
    if (r.c_related) r.c_related[ci] = o.related;
  }
  if (r.totals) std::memcpy(r.totals, tot, sizeof(tot));
  if (r.groups) std::memcpy(r.groups, grp, sizeof(grp));
  return 0;
}

}  // namespace

extern "C" {

// Number of per-cycle entries the oracle produces.
int64_t oracle_n_period(const gtp_design* d) {
  const float ts_f = static_cast<float>(d->timescale);
  (void)ts_f;
  return static_cast<int64_t>(std::ceil((static_cast<double>(d->time_max) * d->timescale) /
                                        static_cast<double>(d->clk_period)));
}

int64_t oracle_ticks_per_cycle(const gtp_design* d) {
  const float ts_f = static_cast<float>(d->timescale);
  return static_cast<int64_t>(std::ceil(d->clk_period / ts_f));
}

// Runs the restated CPU path. fp32 = 0: FP64 oracle; fp32 = 1: the
// reference's FP32 arithmetic (timed CPU baseline). cells/n_cells select a
// subset of instances (NULL = all). Output arrays may be NULL. Returns the
// wall time in seconds through *seconds.
int oracle_run(const gtp_design* d, const gtp_events* ev, const int32_t* cells,
               int32_t n_cells, int n_threads, int fp32, int max_leak_pins,
               double* cell5, double* cycle5, double* totals, double* groups,
               uint32_t* c_events, uint32_t* c_glitches, uint32_t* c_half,
               uint32_t* c_related, int64_t* y_events, int64_t* y_glitches,
               int64_t* dropped, double* seconds) {
  if (!d || !ev) return -2;
  Result r{cell5, cycle5, totals, groups, c_events, c_glitches, c_half,
           c_related, y_events, y_glitches, dropped};
  const auto t0 = std::chrono::steady_clock::now();
  int rc = fp32 ? runImpl<float>(d, ev, cells, n_cells, n_threads, max_leak_pins, r)
                : runImpl<double>(d, ev, cells, n_cells, n_threads, max_leak_pins, r);
  const auto t1 = std::chrono::steady_clock::now();
  if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
  return rc;
}

// ---- single helpers of the restatement, checked one by one against the
// reference's own functions compiled from its sources (oracle/_ref) ----

// Engine::tableValue of one table: order 1 over the slew axis, order 2 over
// (slew, load cap); values row-major [n1][n2]; scale 1. fp32 = 0: the FP64
// interpolation; fp32 = 1: rounded to float as Table*::findValue returns.
double oracle_table_value(int32_t order, int32_t n1, const float* axis1, int32_t n2, const float* axis2,
                          const float* values, float slew, float cap, int fp32) {
  std::vector<float> pool;
  gtp_table tb{};
  tb.order = order;
  tb.axis1_var = order >= 1 ? GTP_AXIS_SLEW : GTP_AXIS_NONE;
  tb.axis2_var = order >= 2 ? GTP_AXIS_CAP : GTP_AXIS_NONE;
  tb.n1 = order >= 1 ? n1 : 1;
  tb.n2 = order >= 2 ? n2 : 1;
  tb.axis1_off = 0;
  if (order >= 1) pool.insert(pool.end(), axis1, axis1 + n1);
  tb.axis2_off = static_cast<int64_t>(pool.size());
  if (order >= 2) pool.insert(pool.end(), axis2, axis2 + n2);
  tb.value_off = static_cast<int64_t>(pool.size());
  pool.insert(pool.end(), values, values + static_cast<int64_t>(tb.n1) * tb.n2);
  tb.scale = 1.0f;
  gtp_design d{};
  d.timescale = 1e-12;
  d.clk_period = 1e-9f;
  d.tables = &tb;
  d.n_table = 1;
  d.lut_pool = pool.data();
  d.lut_pool_len = static_cast<int64_t>(pool.size());
  gtp_events ev{};
  if (fp32) return static_cast<double>(Engine<float>(d, ev, 16).tableValue(0, slew, cap));
  return Engine<double>(d, ev, 16).tableValue(0, slew, cap);
}

// findValueIndex over axis[0..n) at x.
int64_t oracle_find_value_index(const float* axis, int32_t n, float x) {
  return static_cast<int64_t>(Engine<double>::findValueIndex(x, axis, n));
}

// Cycle of tick t (clkedWaveformIdx as the oracle evaluates it).
int64_t oracle_cycle_of(int64_t t, double timescale, float clk_period) {
  gtp_design d{};
  d.timescale = timescale;
  d.clk_period = clk_period;
  gtp_events ev{};
  return Engine<double>(d, ev, 16).cycleOf(t);
}

// Divergence census: the Census counters of the FP64 walk over all cells,
// written to out[0..n_out) in declaration order (pin_events, toggles,
// same_tick_state, same_tick_energy, first_event_state, glitch_class_diff,
// glitch_width_diff, related_diff, no_group_match, beyond_cuda_cycles,
// z_events). Returns the number of counters.
int oracle_divergence_census(const gtp_design* d, const gtp_events* ev, int n_threads,
                             int64_t* out, int n_out) {
  if (!d || !ev) return -2;
  using Eng = Engine<double>;
  Eng eng(*d, *ev, 16);
  if (n_threads < 1) n_threads = 1;
  constexpr int kN = static_cast<int>(sizeof(Eng::Census) / sizeof(int64_t));
  std::vector<Eng::Census> cens(n_threads);
  auto job = [&](int tid) {
    Eng::CycleAcc acc;
    acc.init(eng.n_period);
    for (int32_t ci = tid; ci < d->n_cell; ci += n_threads) {
      Eng::CellOut o;
      eng.cell(ci, o, acc, &cens[tid]);
    }
  };
  std::vector<std::thread> th;
  for (int t = 0; t < n_threads; ++t) th.emplace_back(job, t);
  for (auto& t : th) t.join();
  for (int k = 0; k < kN && k < n_out; ++k) {
    int64_t v = 0;
    for (const auto& c : cens) v += reinterpret_cast<const int64_t*>(&c)[k];
    out[k] = v;
  }
  return kN;
}

float oracle_n_rise(int prev, int cur) { return nRise(prev, cur); }
float oracle_n_toggle(int prev, int cur) { return nToggle(prev, cur); }

// Glitch scaling ratio of a pulse of width_ticks ticks on a pin with slews
// slew_r, slew_f (fp32 = 1: the reference's float arithmetic).
double oracle_glitch_ratio(int64_t width_ticks, double timescale, float slew_r, float slew_f, int fp32) {
  gtp_design d{};
  d.timescale = timescale;
  d.clk_period = 1e-9f;
  gtp_events ev{};
  if (fp32) return static_cast<double>(Engine<float>(d, ev, 16).glitchRatio(width_ticks, slew_r, slew_f));
  return Engine<double>(d, ev, 16).glitchRatio(width_ticks, slew_r, slew_f);
}

}  // extern "C"
