// writers.cpp — the reference's result files, written from the engine's
// results with the reference's expressions and stream formatting.
//
//   cuda_cell_power.txt       CudaPower::printCellRes (power/cuda/CudaPower.cu:3134-3165),
//                             Power::printCellRes (power/Power.cc:389-422)
//   cuda_per_cycle_waveform.txt
//                             PowerResult::printPerCycleResults
//                             (include/sta/PowerClass.hh:123-149)
//
// Per instance the reference keeps internal and switching power with their
// glitch parts folded in, in float (CudaPower::recordResult,
// power/cuda/CudaPower.cu:3015-3018; Power::timeBasedPower,
// power/TimeBasedPower.cc:203-204), and writes the regular part back as
// (folded - glitch) and the total as the left-to-right float sum of the five
// columns. Numbers go through std::ostream with its default formatting (six
// significant digits), as the reference's writers do, so that a file written
// here and one written by the reference from the same per-instance values
// are the same bytes.
#include <cstdio>
#include <fstream>
#include <string>

#include "../../include/gtpb200.h"

extern "C" {

gtp_status gtp_write_cell_power(const char* path, int32_t n_cell, const float* cell5, const char* const* cell_names,
                                const int32_t* cell_type, const char* const* type_names, const char* sep) {
  if (!path || n_cell < 0 || (n_cell > 0 && (!cell5 || !cell_names))) return GTP_EINVAL;
  const std::string s = sep ? sep : "\t";
  std::ofstream out(path, std::ios::out);
  if (!out) return GTP_GENERAL_ERROR;
  out << "cell" << s << "Internal_Power" << s << "Glitch_Internal_Power" << s << "Switching_Power" << s
      << "Glitch_Switching_Power" << s << "Leakage_Power" << s << "Total_Power" << s << "Standard_Cell"
      << "\n";
  for (int32_t i = 0; i < n_cell; ++i) {
    const float* v = cell5 + 5 * static_cast<int64_t>(i);
    // the instance's PowerResult: float fields that start at zero and take
    // their values by += (so a -0 entry is written as 0), internal and
    // switching with the glitch part folded in
    float internal = 0.0f, glitch_internal = 0.0f, switching = 0.0f, glitch_switching = 0.0f, leakage = 0.0f;
    leakage += v[4];
    internal += v[0] + v[1];
    glitch_internal += v[1];
    switching += v[2] + v[3];
    glitch_switching += v[3];
    const float regular_internal = internal - glitch_internal;
    const float regular_switching = switching - glitch_switching;
    const float total = regular_internal + glitch_internal + regular_switching + glitch_switching + leakage;
    const char* type_name = "";
    if (cell_type && type_names && cell_type[i] >= 0 && type_names[cell_type[i]]) type_name = type_names[cell_type[i]];
    out << (cell_names[i] ? cell_names[i] : "") << s << regular_internal << s << glitch_internal << s
        << regular_switching << s << glitch_switching << s << leakage << s << total << s << type_name << "\n";
  }
  out.close();
  return out ? GTP_OK : GTP_GENERAL_ERROR;
}

gtp_status gtp_write_per_cycle_waveform(const char* path, int64_t n_period, const float* cycle5, const char* top_name,
                                        const char* sep) {
  if (!path || n_period < 0 || (n_period > 0 && !cycle5)) return GTP_EINVAL;
  const std::string s = sep ? sep : "\t";
  std::ofstream out(path, std::ios::out);
  if (!out) return GTP_GENERAL_ERROR;
  static const char* const titles[5] = {"Per cycle leakage power: ", "Per cycle internal power: ",
                                        "Per cycle glitch internal power: ", "Per cycle switching power: ",
                                        "Per cycle glitch switching power: "};
  for (int q = 0; q < 5; ++q) {
    out << titles[q] << std::endl;
    // one waveform, the design total's (keyed by the top instance)
    out << (top_name ? top_name : "") << s;
    const float* w = cycle5 + static_cast<int64_t>(q) * n_period;
    for (int64_t c = 0; c < n_period; ++c) out << w[c] << s;
    out << std::endl;
  }
  out << "End of per cycle power" << std::endl;
  out.close();
  return out ? GTP_OK : GTP_GENERAL_ERROR;
}

}  // extern "C"
