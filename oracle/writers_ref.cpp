// writers_ref.cpp — restatement of the reference's result-file writers, the
// checker of gtp_write_cell_power / gtp_write_per_cycle_waveform (TEST
// INFRASTRUCTURE ONLY; built by oracle/Makefile, run by tests/test_writers.py).
//
// It keeps the reference's data flow and expressions:
//   per instance, PowerResult's float fields start at zero and take
//   internal += regular + glitch, glitchInternal += glitch (and the same for
//   switching), leakage += leakage       CudaPower::recordResult,
//                                        power/cuda/CudaPower.cu:3011-3019
//   the row: regular = internal - glitchInternal; total = the five columns
//   added left to right, all PowerVal (float), through std::ostream
//                                        CudaPower::printCellRes, :3134-3165
//   per-cycle file: "<title> " << endl, then "<top>" sep, v sep ..., endl,
//   for the five sections, then "End of per cycle power" << endl
//                                        PowerResult::printPerCycleResults,
//                                        include/sta/PowerClass.hh:123-149
//
// Input (binary, little endian): int32 n_cell, int64 n_period,
// float cell_regular[n_cell][5] (regular internal, glitch internal, regular
// switching, glitch switching, leakage), float cycle[5][n_period], then
// NUL-terminated strings: top name, separator, n_cell instance names,
// n_cell Liberty cell names. Usage: writers_ref <in> <cell file> <cycle file>
#include <cstdint>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

typedef float PowerVal;  // util/Types.hh

struct PowerResult {
  PowerVal internal_ = 0, glitch_internal_ = 0, switching_ = 0, glitch_switching_ = 0, leakage_ = 0;
};

static std::string read_str(std::ifstream& in) {
  std::string s;
  std::getline(in, s, '\0');
  return s;
}

int main(int argc, char** argv) {
  if (argc != 4) return 2;
  std::ifstream in(argv[1], std::ios::binary);
  int32_t n_cell = 0;
  int64_t n_period = 0;
  in.read(reinterpret_cast<char*>(&n_cell), 4);
  in.read(reinterpret_cast<char*>(&n_period), 8);
  std::vector<float> cell(5 * static_cast<size_t>(n_cell)), cyc(5 * static_cast<size_t>(n_period));
  in.read(reinterpret_cast<char*>(cell.data()), static_cast<std::streamsize>(cell.size() * 4));
  in.read(reinterpret_cast<char*>(cyc.data()), static_cast<std::streamsize>(cyc.size() * 4));
  const std::string top = read_str(in), sep = read_str(in);
  std::vector<std::string> names(n_cell), types(n_cell);
  for (auto& n : names) n = read_str(in);
  for (auto& t : types) t = read_str(in);
  if (!in) return 3;

  std::ofstream out_file(argv[2], std::ios::out);
  out_file << "cell" << sep << "Internal_Power" << sep << "Glitch_Internal_Power" << sep << "Switching_Power"
           << sep << "Glitch_Switching_Power" << sep << "Leakage_Power" << sep << "Total_Power" << sep
           << "Standard_Cell" << "\n";
  for (int32_t i = 0; i < n_cell; ++i) {
    const float* g = &cell[5 * static_cast<size_t>(i)];
    PowerResult r;
    r.leakage_ += g[4];
    r.internal_ += g[0] + g[1];
    r.glitch_internal_ += g[1];
    r.switching_ += g[2] + g[3];
    r.glitch_switching_ += g[3];
    PowerVal cur_gate_regular_internal = r.internal_ - r.glitch_internal_;
    PowerVal cur_gate_glitch_internal = r.glitch_internal_;
    PowerVal cur_gate_regular_switching = r.switching_ - r.glitch_switching_;
    PowerVal cur_gate_glitch_switching = r.glitch_switching_;
    PowerVal cur_gate_leakage = r.leakage_;
    out_file << names[i] << sep << cur_gate_regular_internal << sep << cur_gate_glitch_internal << sep
             << cur_gate_regular_switching << sep << cur_gate_glitch_switching << sep << cur_gate_leakage << sep
             << cur_gate_regular_internal + cur_gate_glitch_internal + cur_gate_regular_switching +
                    cur_gate_glitch_switching + cur_gate_leakage
             << sep << types[i] << "\n";
  }
  out_file.close();

  std::ofstream wf(argv[3], std::ios::out);
  const char* titles[5] = {"Per cycle leakage power: ", "Per cycle internal power: ",
                           "Per cycle glitch internal power: ", "Per cycle switching power: ",
                           "Per cycle glitch switching power: "};
  for (int q = 0; q < 5; ++q) {
    wf << titles[q] << std::endl;
    wf << top << sep;
    for (int64_t c = 0; c < n_period; ++c) wf << cyc[static_cast<size_t>(q * n_period + c)] << sep;
    wf << std::endl;
  }
  wf << "End of per cycle power" << std::endl;
  return 0;
}
