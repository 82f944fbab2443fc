// pack.cpp — validates a gtp_design and packs it into the device layout.
//
// Two pieces of the reference's per-event work depend only on per-pin
// constants and are therefore evaluated here once per instance:
//   - the NLDM interpolation of every internal_power table a pin can select
//     (InternalPower::power, liberty/InternalPower.cc:112-156, called per
//     event from findInputInternalVal / findOutputInternalVal,
//     power/TimeBasedPower.cc:341-509). The slew argument is the pin's (or
//     the related input's) rise/fall slew and the load is the output pin's
//     load cap, so for each group only 2 (input) or 4 (output: from x to)
//     values exist per instance. They are computed exactly as the reference
//     does — FP64 interpolation rounded to float, times the float scale
//     factor — so the device sees the same float energies.
//   - the default output energy (getDefaultOutputPinInternalEnergyVal,
//     power/TimeBasedPower.cc:511-555), an average over the same values.
// Leakage tables are expanded per cell type as Power::getLeakagePower does
// (power/TimeBasedPower.cc:258-301, getStateIdx :557-587).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>

#include "engine.h"

namespace gtpb {
namespace {

size_t find_value_index(float value, const float* axis, int size) {
  // findValueIndex (liberty/TableModel.cc:1467-1489)
  if (size <= 1 || value <= axis[0]) return 0;
  if (value >= axis[size - 1]) return size - 2;
  int lower = -1, upper = size;
  while (upper - lower > 1) {
    int mid = (upper + lower) >> 1;
    if (value >= axis[mid]) lower = mid; else upper = mid;
  }
  return lower;
}

// Table0/1/2::findValue (liberty/TableModel.cc:858-880, 1011-1060), returned
// as float and scaled (TableModel::findValue(cell, pvt, ...)).
float table_value(const gtp_design& d, int32_t ti, float slew, float cap) {
  if (ti < 0) return 0.0f;
  const gtp_table& tb = d.tables[ti];
  auto axv = [&](int var) -> float {
    return var == GTP_AXIS_SLEW ? slew : (var == GTP_AXIS_CAP ? cap : 0.0f);
  };
  const float* v = d.lut_pool + tb.value_off;
  double r;
  if (tb.order == 0) {
    r = v[0];
  } else if (tb.order == 1) {
    const float* a1 = d.lut_pool + tb.axis1_off;
    if (tb.n1 == 1) {
      r = v[0];
    } else {
      const float x = axv(tb.axis1_var);
      size_t i = find_value_index(x, a1, tb.n1);
      double x1 = x, x1l = a1[i], x1u = a1[i + 1];
      double dx1 = (x1 - x1l) / (x1u - x1l);
      r = (1 - dx1) * static_cast<double>(v[i]) + dx1 * static_cast<double>(v[i + 1]);
    }
  } else {
    const float* a1 = d.lut_pool + tb.axis1_off;
    const float* a2 = d.lut_pool + tb.axis2_off;
    const float x1f = axv(tb.axis1_var), x2f = axv(tb.axis2_var);
    const int n1 = tb.n1, n2 = tb.n2;
    auto val = [&](size_t i, size_t j) -> double { return v[i * n2 + j]; };
    if (n1 == 1) {
      if (n2 == 1) {
        r = val(0, 0);
      } else {
        size_t j = find_value_index(x2f, a2, n2);
        double x2 = x2f, x2l = a2[j], x2u = a2[j + 1];
        double dx2 = (x2 - x2l) / (x2u - x2l);
        r = (1 - dx2) * val(0, j) + dx2 * val(0, j + 1);
      }
    } else if (n2 == 1) {
      size_t i = find_value_index(x1f, a1, n1);
      double x1 = x1f, x1l = a1[i], x1u = a1[i + 1];
      double dx1 = (x1 - x1l) / (x1u - x1l);
      r = (1 - dx1) * val(i, 0) + dx1 * val(i + 1, 0);
    } else {
      size_t i = find_value_index(x1f, a1, n1);
      size_t j = find_value_index(x2f, a2, n2);
      double x1 = x1f, x2 = x2f;
      double x1l = a1[i], x1u = a1[i + 1];
      double dx1 = (x1 - x1l) / (x1u - x1l);
      double x2l = a2[j], x2u = a2[j + 1];
      double dx2 = (x2 - x2l) / (x2u - x2l);
      r = (1 - dx1) * (1 - dx2) * val(i, j) + dx1 * (1 - dx2) * val(i + 1, j) +
          dx1 * dx2 * val(i + 1, j + 1) + (1 - dx1) * dx2 * val(i, j + 1);
    }
  }
  return static_cast<float>(r) * tb.scale;
}

bool check_table(const gtp_design& d, int32_t ti) {
  if (ti < 0) return true;
  if (ti >= d.n_table) return false;
  const gtp_table& tb = d.tables[ti];
  if (tb.order < 0 || tb.order > 2 || tb.n1 < 1 || tb.n2 < 1) return false;
  const int64_t nv = static_cast<int64_t>(tb.n1) * tb.n2;
  if (tb.value_off < 0 || tb.value_off + nv > d.lut_pool_len) return false;
  if (tb.order >= 1 && (tb.axis1_off < 0 || tb.axis1_off + tb.n1 > d.lut_pool_len)) return false;
  if (tb.order >= 2 && (tb.axis2_off < 0 || tb.axis2_off + tb.n2 > d.lut_pool_len)) return false;
  return true;
}

}  // namespace

gtp_status pack_design(const gtp_design& d, int max_leak_pins, Packed& P, std::string& err) {
  auto fail = [&](const std::string& m) { err = m; return GTP_EINVAL; };
  if (d.n_cell < 0 || d.n_pin < 0 || d.n_net < 0 || d.n_type < 0) return fail("negative sizes");
  if (!(d.timescale > 0) || !(d.clk_period > 0) || d.time_max <= 0)
    return fail("timescale, clk_period and time_max must be positive");
  if (d.time_max >= (int64_t(1) << 53)) return fail("time_max must be below 2^53 ticks");
  if (d.n_cell > 0 && (!d.cell_pin_off || !d.cell_type || !d.cell_arc_off))
    return fail("cell arrays missing");
  if (d.n_pin > 0 && (!d.pin_net || !d.pin_slew_rise || !d.pin_slew_fall || !d.pin_load_cap ||
                      !d.pin_voltage || !d.pin_default_state || !d.pin_is_clock))
    return fail("pin arrays missing");
  if (d.n_type > 0 && !d.types) return fail("types missing");

  P.n_cell = d.n_cell;
  P.n_pin = d.n_pin;
  P.n_net = d.n_net;
  P.ts = d.timescale;
  P.period_f = d.clk_period;
  P.period_d = static_cast<double>(d.clk_period);
  const float ts_f = static_cast<float>(d.timescale);
  P.tpc = static_cast<int64_t>(std::ceil(d.clk_period / ts_f));
  if (P.tpc <= 0) return fail("ticks per cycle must be positive");
  P.tmax = d.time_max;
  P.n_period = static_cast<int64_t>(
      std::ceil((static_cast<double>(d.time_max) * d.timescale) / P.period_d));

  // ---- cell types ----
  for (int32_t t = 0; t < d.n_type; ++t) {
    const gtp_cell_type& ty = d.types[t];
    if (ty.n_pin < 0 || ty.n_pin > kMaxPins) return fail("cell type pin count above 32");
    if (ty.n_in < 0 || ty.n_in > ty.n_pin) return fail("cell type input count invalid");
    if (ty.n_ipwr < 0 || ty.ipwr_off < 0 || ty.ipwr_off + ty.n_ipwr > d.n_internal_power)
      return fail("internal_power range invalid");
    if (ty.n_leak < 0 || ty.leak_off < 0 || ty.leak_off + ty.n_leak > d.n_leakage_power)
      return fail("leakage_power range invalid");
    for (int k = 0; k < ty.n_ipwr; ++k) {
      const gtp_internal_power& g = d.internal_powers[ty.ipwr_off + k];
      if (g.pin < 0 || g.pin >= ty.n_pin) return fail("internal_power pin out of range");
      if (g.related_pin >= ty.n_pin) return fail("internal_power related pin out of range");
      if (g.when.n_cube < 0 || g.when.cube_off < 0 || g.when.cube_off + g.when.n_cube > d.n_when_cube)
        return fail("when range invalid");
      if (!check_table(d, g.rise_table) || !check_table(d, g.fall_table))
        return fail("power table invalid");
    }
    for (int k = 0; k < ty.n_leak; ++k) {
      const gtp_leakage_power& l = d.leakage_powers[ty.leak_off + k];
      if (l.when.n_cube < 0 || l.when.cube_off < 0 || l.when.cube_off + l.when.n_cube > d.n_when_cube)
        return fail("leakage when range invalid");
    }
  }

  P.cubes.assign(d.when_cubes, d.when_cubes + 2 * static_cast<size_t>(d.n_when_cube));

  // per type: slots per pin, instance block layout, leakage table
  P.types.resize(d.n_type);
  std::vector<std::vector<int32_t>> slot_group(d.n_type);  // slot -> internal power index
  for (int32_t t = 0; t < d.n_type; ++t) {
    const gtp_cell_type& ty = d.types[t];
    DevType& dt = P.types[t];
    dt.n_pin = ty.n_pin;
    dt.n_in = ty.n_in;
    dt.pin_slot_off = static_cast<int32_t>(P.pin_slot.size());
    int32_t e = 0;
    for (int pin = 0; pin < ty.n_pin; ++pin) {
      P.pin_slot.push_back(static_cast<int32_t>(P.slots.size()));
      const bool is_in = pin < ty.n_in;
      for (int k = 0; k < ty.n_ipwr; ++k) {
        const gtp_internal_power& g = d.internal_powers[ty.ipwr_off + k];
        if (g.pin != pin) continue;
        // output groups are only ever selected through an input related pin
        if (!is_in && (g.related_pin < 0 || g.related_pin >= ty.n_in)) continue;
        DevSlot s;
        s.related = is_in ? -1 : g.related_pin;
        s.cube_off = g.when.cube_off;
        s.n_cube = g.when.n_cube;
        s.e_off = e;
        e += is_in ? 2 : 4;
        P.slots.push_back(s);
        slot_group[t].push_back(ty.ipwr_off + k);
      }
    }
    P.pin_slot.push_back(static_cast<int32_t>(P.slots.size()));
    const int n_out = ty.n_pin - ty.n_in;
    dt.def_off = e;
    e += 2 * n_out;
    dt.delay_off = e;
    e += 4 * n_out * ty.n_in;
    e = (e + 3) & ~3;   // 16-byte aligned blocks (staged with vector loads)
    dt.inst_floats = e;

    // leakage (Power::getLeakagePower)
    float def = ty.cell_leakage_power;
    bool def_exists = ty.has_cell_leakage_power != 0;
    dt.leak_off = -1;
    if (ty.n_pin > max_leak_pins) {
      if (ty.n_leak == 1) {
        def = d.leakage_powers[ty.leak_off].power;
        def_exists = true;
      }
      dt.leak_const = def_exists ? def : 0.0f;
    } else if (ty.n_leak == 0) {
      dt.leak_const = def_exists ? def : 0.0f;
    } else {
      const size_t n_state = size_t(1) << ty.n_pin;
      dt.leak_off = static_cast<int32_t>(P.leak_pool.size());
      dt.leak_const = 0.0f;
      P.leak_pool.resize(P.leak_pool.size() + n_state, def_exists ? def : 0.0f);
      float* tab = P.leak_pool.data() + dt.leak_off;
      for (int k = 0; k < ty.n_leak; ++k) {
        const gtp_leakage_power& l = d.leakage_powers[ty.leak_off + k];
        if (l.when.n_cube != 1) continue;
        const uint32_t care = d.when_cubes[2 * l.when.cube_off];
        const uint32_t val = d.when_cubes[2 * l.when.cube_off + 1];
        for (size_t s = 0; s < n_state; ++s)
          if ((static_cast<uint32_t>(s) & care) == val) tab[s] = l.power;
      }
    }
    P.max_abs_leak = std::max<double>(P.max_abs_leak, std::fabs(dt.leak_const));
  }
  for (float v : P.leak_pool) P.max_abs_leak = std::max<double>(P.max_abs_leak, std::fabs(v));

  // ---- cells and pins ----
  P.cell_pin_off.assign(d.cell_pin_off, d.cell_pin_off + d.n_cell + 1);
  P.cell_type.assign(d.cell_type, d.cell_type + d.n_cell);
  P.cell_group.resize(d.n_cell, 0);
  if (d.cell_group) {
    for (int32_t c = 0; c < d.n_cell; ++c) {
      if (d.cell_group[c] >= GTP_N_GROUP) return fail("cell group out of range");
      P.cell_group[c] = d.cell_group[c];
    }
  }
  if (d.n_cell > 0 && (P.cell_pin_off[0] != 0 || P.cell_pin_off[d.n_cell] != d.n_pin))
    return fail("cell_pin_off must start at 0 and end at n_pin");
  P.cell_inst.resize(d.n_cell);
  int64_t inst_total = 0;
  for (int32_t c = 0; c < d.n_cell; ++c) {
    const int32_t t = P.cell_type[c];
    if (t < 0 || t >= d.n_type) return fail("cell type out of range");
    if (P.cell_pin_off[c + 1] - P.cell_pin_off[c] != d.types[t].n_pin)
      return fail("cell pin count differs from its type");
    const int n_in = d.types[t].n_in, n_out = d.types[t].n_pin - n_in;
    if (d.cell_arc_off[c] < 0 || d.cell_arc_off[c] + 4LL * n_out * n_in > d.n_arc_delay)
      return fail("arc delay range invalid");
    P.cell_inst[c] = static_cast<int32_t>(inst_total);
    inst_total += P.types[t].inst_floats;
    if (inst_total > INT32_MAX) return fail("instance energy pool above 2^31 floats");
  }
  P.pin_net.assign(d.pin_net, d.pin_net + d.n_pin);
  P.pin_flags.resize(d.n_pin);
  P.pin_gden.resize(d.n_pin);
  P.pin_swe.resize(d.n_pin);
  for (int32_t p = 0; p < d.n_pin; ++p) {
    if (P.pin_net[p] < -1 || P.pin_net[p] >= d.n_net) return fail("pin net out of range");
    if (d.pin_default_state[p] > 2) return fail("pin default state must be 0, 1 or 2");
    P.pin_flags[p] = static_cast<uint8_t>(d.pin_default_state[p] | (d.pin_is_clock[p] ? 4 : 0));
    P.pin_gden[p] = d.pin_slew_rise[p] + d.pin_slew_fall[p];
    // pin_single_switching_energies: load_cap * volt * volt (TimeBasedPower.cc:750-759)
    P.pin_swe[p] = d.pin_load_cap[p] * d.pin_voltage[p] * d.pin_voltage[p];
  }

  // ---- per-instance energies (parallel over cells) ----
  P.inst.assign(static_cast<size_t>(inst_total), 0.0f);
  const int n_threads = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  std::vector<double> max_e(n_threads, 0.0);
  auto work = [&](int tid) {
    const int32_t per = (d.n_cell + n_threads - 1) / n_threads;
    const int32_t c0 = tid * per, c1 = std::min(d.n_cell, c0 + per);
    double me = 0;
    for (int32_t c = c0; c < c1; ++c) {
      const int32_t t = P.cell_type[c];
      const gtp_cell_type& ty = d.types[t];
      const DevType& dt = P.types[t];
      const int32_t p0 = P.cell_pin_off[c];
      float* blk = P.inst.data() + P.cell_inst[c];
      auto slew = [&](int pin, int rf) -> float {
        return rf == 0 ? d.pin_slew_rise[p0 + pin] : d.pin_slew_fall[p0 + pin];
      };
      for (int pin = 0; pin < ty.n_pin; ++pin) {
        const bool is_in = pin < ty.n_in;
        const float cap = d.pin_load_cap[p0 + pin];
        for (int32_t s = P.pin_slot[dt.pin_slot_off + pin]; s < P.pin_slot[dt.pin_slot_off + pin + 1]; ++s) {
          const DevSlot& sl = P.slots[s];
          const int32_t local = s - P.pin_slot[dt.pin_slot_off];
          const gtp_internal_power& g = d.internal_powers[slot_group[t][local]];
          if (is_in) {
            for (int rf = 0; rf < 2; ++rf) {
              const float sw = slew(pin, rf);
              // findInputInternalVal: infinite slew -> 0 (TimeBasedPower.cc:362-365)
              const float v = std::isinf(sw) ? 0.0f
                              : table_value(d, rf == 0 ? g.rise_table : g.fall_table, sw, 0.0f);
              blk[sl.e_off + rf] = v;
              me = std::max<double>(me, std::fabs(v));
            }
          } else {
            for (int fr = 0; fr < 2; ++fr) {
              const float sw = slew(sl.related, fr);
              for (int to = 0; to < 2; ++to) {
                const float v = std::isinf(sw) ? 0.0f
                                : table_value(d, to == 0 ? g.rise_table : g.fall_table, sw, cap);
                blk[sl.e_off + 2 * fr + to] = v;
                me = std::max<double>(me, std::fabs(v));
              }
            }
          }
        }
      }
      // defaults and arc delays per output
      const int n_in = ty.n_in, n_out = ty.n_pin - ty.n_in;
      for (int o = 0; o < n_out; ++o) {
        const int pin = n_in + o;
        const float cap = d.pin_load_cap[p0 + pin];
        for (int to = 0; to < 2; ++to) {
          int n_table = 0;
          float total = 0.0f;
          for (int q = 0; q < n_in; ++q) {
            for (int fr = 0; fr < 2; ++fr) {
              const float sw = slew(q, fr);
              if (std::isinf(sw)) continue;
              for (int k = 0; k < ty.n_ipwr; ++k) {
                const gtp_internal_power& g = d.internal_powers[ty.ipwr_off + k];
                if (g.pin != pin || g.related_pin != q) continue;
                total += table_value(d, to == 0 ? g.rise_table : g.fall_table, sw, cap);
                ++n_table;
              }
            }
          }
          const float v = n_table == 0 ? 0.0f : total / n_table;
          blk[dt.def_off + 2 * o + to] = v;
          me = std::max<double>(me, std::fabs(v));
        }
        for (int q = 0; q < n_in; ++q)
          for (int a = 0; a < 4; ++a)
            blk[dt.delay_off + (o * n_in + q) * 4 + a] =
                d.arc_delay[d.cell_arc_off[c] + (static_cast<int64_t>(o) * n_in + q) * 4 + a];
      }
      for (int pin = n_in; pin < ty.n_pin; ++pin)
        me = std::max<double>(me, std::fabs(static_cast<double>(P.pin_swe[p0 + pin])));
    }
    max_e[tid] = me;
  };
  {
    std::vector<std::thread> th;
    for (int i = 0; i < n_threads; ++i) th.emplace_back(work, i);
    for (auto& x : th) x.join();
  }
  for (double v : max_e) P.max_abs_energy = std::max(P.max_abs_energy, v);

  // ---- fast tables: first matching group per (pin, related, state) ----
  P.type_fast_off.assign(d.n_type, -1);
  for (int32_t t = 0; t < d.n_type; ++t) {
    const DevType& dt = P.types[t];
    if (dt.n_pin > kFastPins) continue;
    const int n_state = 1 << dt.n_pin;
    const int n_in = dt.n_in, n_out = dt.n_pin - dt.n_in;
    P.type_fast_off[t] = static_cast<int32_t>(P.fast_tab.size());
    auto holds = [&](const DevSlot& sl, uint32_t ones) {
      for (int k = 0; k < sl.n_cube; ++k) {
        const uint32_t care = P.cubes[2 * (sl.cube_off + k)];
        const uint32_t val = P.cubes[2 * (sl.cube_off + k) + 1];
        if ((ones & care) == val) return true;
      }
      return false;
    };
    for (int pin = 0; pin < n_in; ++pin)
      for (int s = 0; s < n_state; ++s) {
        int16_t e = -1;
        for (int32_t k = P.pin_slot[dt.pin_slot_off + pin]; k < P.pin_slot[dt.pin_slot_off + pin + 1]; ++k)
          if (holds(P.slots[k], static_cast<uint32_t>(s))) { e = static_cast<int16_t>(P.slots[k].e_off); break; }
        P.fast_tab.push_back(e);
      }
    for (int o = 0; o < n_out; ++o)
      for (int q = 0; q < n_in; ++q)
        for (int s = 0; s < n_state; ++s) {
          int16_t e = -1;
          const int pin = n_in + o;
          for (int32_t k = P.pin_slot[dt.pin_slot_off + pin]; k < P.pin_slot[dt.pin_slot_off + pin + 1]; ++k) {
            if (P.slots[k].related != q) continue;
            if (holds(P.slots[k], static_cast<uint32_t>(s))) { e = static_cast<int16_t>(P.slots[k].e_off); break; }
          }
          P.fast_tab.push_back(e);
        }
    if (dt.inst_floats > INT16_MAX) return fail("instance block too large for the fast tables");
    P.fast_inst_floats = std::max(P.fast_inst_floats, dt.inst_floats);
  }

  // ---- clock drift: does some tick fall between a cycle's tick boundary
  // c*tpc and its seconds boundary c*period (double comparisons as the
  // reference's calculatePerCycleLeakagePower makes them)? ----
  P.drift = false;
  for (int64_t c = 1; c <= P.n_period + 1 && !P.drift; ++c) {
    const double b = static_cast<double>(c) * P.period_d;
    const int64_t t0 = c * P.tpc;
    const bool at = b <= static_cast<double>(t0) * P.ts;
    const bool before = b <= static_cast<double>(t0 - 1) * P.ts;
    if (!at || before) P.drift = true;
  }

  // ---- walk order: bucket by pin count (register footprint), then by type ----
  P.order.resize(d.n_cell);
  for (int32_t c = 0; c < d.n_cell; ++c) P.order[c] = c;
  auto bucket = [&](int32_t c) {
    const int n = d.types[P.cell_type[c]].n_pin;
    return n <= 4 ? 0 : (n <= 8 ? 1 : 2);
  };
  std::stable_sort(P.order.begin(), P.order.end(), [&](int32_t a, int32_t b) {
    const int ba = bucket(a), bb = bucket(b);
    if (ba != bb) return ba < bb;
    return P.cell_type[a] < P.cell_type[b];
  });
  P.bucket_begin[0] = 0;
  for (int b = 1; b <= 3; ++b) {
    int32_t i = P.bucket_begin[b - 1];
    while (i < d.n_cell && bucket(P.order[i]) < b) ++i;
    P.bucket_begin[b] = i;
  }
  P.order_all = P.order;
  for (int b = 0; b < 4; ++b) P.bucket_all[b] = P.bucket_begin[b];
  return GTP_OK;
}

}  // namespace gtpb
