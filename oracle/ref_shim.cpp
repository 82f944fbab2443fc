// ref_shim.cpp — C entry points over the reference's own helpers, compiled
// from the reference sources (TEST INFRASTRUCTURE ONLY; built by
// oracle/Makefile target `ref` into oracle/_ref/libref.so, loaded only by
// tests/ and tests/golden/make_ref_vectors.py).
//
// Each entry point builds the reference's objects and calls the reference
// function unchanged, so that the restatement in oracle.cpp can be checked
// against the reference's arithmetic on many random inputs:
//   Table1::findValue, Table2::findValue, findValueIndex
//                               liberty/TableModel.cc:858-880, 1011-1060, 1467-1489
//   clkedWaveformIdx            power/PowerUtils.cc:27-32
//   getNRise, getNToggle        power/PowerUtils.cc:213-255
//   getTimeBasedGlitchScalingRatioH
//                               power/PowerUtils.cc:285-294
#include <memory>

#include "PowerUtils.hh"
#include "TableModel.hh"

namespace sta {
// defined in liberty/TableModel.cc (declared there, not in a header)
size_t findValueIndex(float value, const FloatSeq* values);
}  // namespace sta

namespace {
sta::FloatSeq* seq(const float* p, int n) {
  auto* s = new sta::FloatSeq;
  s->assign(p, p + n);
  return s;
}
}  // namespace

extern "C" {

// Table1 over axis[0..n) (input_transition_time) with values[0..n), looked up at x.
float ref_table1(const float* axis, int n, const float* values, float x) {
  auto ax = std::make_shared<sta::TableAxis>(sta::TableAxisVariable::input_transition_time, seq(axis, n));
  sta::Table1 t(seq(values, n), ax);
  return t.findValue(x);
}

// Table2 over axis1[0..n1) (input_transition_time) x axis2[0..n2)
// (total_output_net_capacitance), values row-major [n1][n2], looked up at (x1, x2).
float ref_table2(const float* axis1, int n1, const float* axis2, int n2, const float* values, float x1,
                 float x2) {
  auto ax1 = std::make_shared<sta::TableAxis>(sta::TableAxisVariable::input_transition_time, seq(axis1, n1));
  auto ax2 = std::make_shared<sta::TableAxis>(sta::TableAxisVariable::total_output_net_capacitance,
                                              seq(axis2, n2));
  auto* rows = new sta::FloatTable;
  for (int i = 0; i < n1; ++i) rows->push_back(seq(values + i * n2, n2));
  sta::Table2 t(rows, ax1, ax2);
  return t.findValue(x1, x2, 0.0f);
}

// findValueIndex over axis[0..n) at x.
long long ref_find_value_index(const float* axis, int n, float x) {
  sta::FloatSeq v;
  v.assign(axis, axis + n);
  return static_cast<long long>(sta::findValueIndex(x, &v));
}

long long ref_clked_waveform_idx(long long t, float timescale, float period) {
  return gtpower::utils::clkedWaveformIdx(static_cast<VcdEventTime>(t), timescale, period);
}

float ref_n_rise(int prev, int cur) {
  return gtpower::utils::getNRise(static_cast<VcdEventVal>(prev), static_cast<VcdEventVal>(cur));
}

float ref_n_toggle(int prev, int cur) {
  return gtpower::utils::getNToggle(static_cast<VcdEventVal>(prev), static_cast<VcdEventVal>(cur));
}

float ref_glitch_ratio(float pulse_width, float sum_slew) {
  return gtpower::utils::getTimeBasedGlitchScalingRatioH(pulse_width, sum_slew);
}

}  // extern "C"
