// engine.h — internal data layout shared by the host packer (pack.cpp), the
// kernels (power_kernel.cu) and the C ABI (abi.cu).
//
// Layout in HBM (one context):
//   static design (uploaded once by gtp_create)
//     cell_pin_off  int32[n_cell+1]   pins of a cell: inputs, then outputs
//     cell_type     int32[n_cell]
//     cell_inst     int32[n_cell]     offset of the cell's energy block in inst[]
//     order         int32[n_cell]     walk order (cells grouped by pin bucket/type)
//     pin_net       int32[n_pin]      -1 = no waveform
//     pin_flags     uint8[n_pin]      bits 0-1 default state, bit 2 is_clock
//     pin_gden      float[n_pin]      slew_rise + slew_fall (glitch ratio divisor)
//     pin_swe       float[n_pin]      load_cap * V * V (switching energy per rise)
//     types/slots/pin_slot/cubes      per-cell-type power program (small)
//     leak_pool     float[]           2^n_pin leakage table per cell type
//     inst          float[]           per-instance interpolated energies and arc
//                                     delays (the NLDM lookups depend only on
//                                     per-pin slews/caps, so they are done once
//                                     per instance at create time, in FP32 from
//                                     FP64 interpolation as the reference does)
//   events (per pushed window): net_off int64[n_net+1], time int64[E],
//     value_packed uint32[E/16], net_base int64[n_net] (optional)
//   accumulators (scratch)
//     cell_acc  double[5][n_cell]       internal, glitch internal, switching,
//                                       glitch switching (J), leakage (W*ticks)
//     cyc_acc   int64[6][n_period+1]    leakage direct, leakage run-difference,
//                                       internal, glitch internal, switching,
//                                       glitch switching — 64-bit fixed point
//                                       energies (J * 2^s), exact and
//                                       order-independent
//     cnt_cell  uint32[4][n_cell], cnt_cyc uint64[2][n_period+1] (optional)
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <vector>
#include <string>

#include "../../include/gtpb200.h"

namespace gtpb {

// Per cell type program (device copy).
struct DevType {
  int32_t n_pin;
  int32_t n_in;
  int32_t leak_off;      // into leak_pool; -1 = constant leak_const
  float   leak_const;
  int32_t pin_slot_off;  // into pin_slot[]: [n_pin+1] slot index bounds
  int32_t def_off;       // float offset in the instance block: defaults [n_out][2]
  int32_t delay_off;     // float offset in the instance block: delays [n_out][n_in][4]
  int32_t inst_floats;   // floats per instance block
};

// One internal_power group usable by the walk, in Liberty order per pin.
struct DevSlot {
  int32_t related;       // cell-local related input pin, -1 for input-pin groups
  int32_t cube_off;      // into cubes[] (uint2 care,value)
  int32_t n_cube;
  int32_t e_off;         // float offset in the instance block:
                         //   input pin : [rise, fall]
                         //   output pin: [from][to] (rise=0, fall=1)
};

constexpr int kMaxPins = 32;      // cell pins supported by the walk
constexpr int kFastPins = 4;      // cells up to this many pins use fast_tab
constexpr int kNumCycAcc = 6;     // per-cycle fixed-point accumulators
constexpr int kNumBinSlotsRun = 8; // shared-memory bin slots per set with clock runs:
                                   // the 6 above, then run-differences of the
                                   // per-cycle clock-edge internal energy and leakage
constexpr int kNumCellAcc = 5;

// Host-side packed design.
struct Packed {
  int32_t n_cell = 0, n_pin = 0, n_net = 0;
  double ts = 0;          // timescale (s/tick)
  float  period_f = 0;    // clk period (float)
  double period_d = 0;
  int64_t tpc = 0;        // ticks per cycle
  int64_t tmax = 0;
  int64_t n_period = 0;
  std::vector<int32_t> cell_pin_off, cell_type, cell_inst, order;
  std::vector<uint8_t> cell_group;
  std::vector<int32_t> pin_net;
  std::vector<uint8_t> pin_flags;
  std::vector<float>   pin_gden, pin_swe;
  std::vector<DevType> types;
  std::vector<DevSlot> slots;
  std::vector<int32_t> pin_slot;
  std::vector<uint32_t> cubes;   // pairs
  std::vector<float>   leak_pool;
  std::vector<float>   inst;
  // per cell type with n_pin <= kFastPins: offset into fast_tab, else -1.
  // fast_tab (int16): for input pin i, [i][ones] = energy offset of the
  // first internal_power group whose `when` holds in pin state `ones` (-1 =
  // none); then for output o and related input q, [o][q][ones] likewise.
  std::vector<int32_t> type_fast_off;
  std::vector<int16_t> fast_tab;
  // true when some tick lies between a cycle's tick boundary and its
  // seconds boundary (c*clk_period), where the reference's per-cycle
  // leakage split departs from the plain overlap (needs the drift path)
  bool drift = false;
  int32_t fast_inst_floats = 0;   // largest instance block of a fast cell type
  // bucket ranges in order[]: cells with n_pin <= 4, <= 8, <= 32; order[]
  // lists the cells the context walks (all, or a shard, gtp_set_cell_range),
  // bucket_begin[3] of them; order_all / bucket_all: the whole design's
  std::vector<int32_t> order_all;
  int32_t bucket_begin[4] = {0, 0, 0, 0};
  int32_t bucket_all[4] = {0, 0, 0, 0};
  double max_abs_energy = 0;     // max |instance energy|, for the fixed-point scale
  double max_abs_leak = 0;
};

// Packs and validates a design. Returns GTP_OK or an error with a message.
gtp_status pack_design(const gtp_design& d, int max_leak_pins, Packed& out, std::string& err);

// Kernel parameter block.
struct KParams {
  const int32_t* cell_pin_off;
  const int32_t* cell_type;
  const int32_t* cell_inst;
  const int32_t* order;
  int32_t order_begin, order_end;
  const int32_t* pin_net;
  const uint8_t* pin_flags;
  const uint8_t* net_glitch;        // [n_net] 1 when some non-clock pin reads the net, or null
  const float* pin_gden;
  const float* pin_swe;
  const DevType* types;
  const DevSlot* slots;
  const int32_t* pin_slot;
  const uint2* cubes;
  const float* leak_pool;
  const float* inst;
  const int32_t* type_fast_off;
  const int16_t* fast_tab;
  int32_t n_fast_tab, n_leak_pool;  // table sizes (for staging in shared memory)
  int32_t tabs_in_smem;
  int32_t fast_inst_stride;         // floats per thread for a staged instance block
  int32_t drift;
  // events
  const int64_t* net_off;
  const int64_t* ev_t;
  const uint32_t* ev_v;
  const int64_t* net_base;   // may be null
  const int32_t* tile_first; // [n_tiles][n_net] first event at or after each tile's start,
                             // relative to net_off; null: the walk bisects
  const float* glitch_pw;    // [n_event] glitch pulse width (s) of each listed event, -1 when
                             // not a glitch event; null: the walk classifies
  const int2* pclk;          // [n_net] for nets read by clock pins: the window's periodic
                             // pattern (x: phase of the cycle's first edge in ticks, -1 =
                             // not periodic; y: phase of the second edge | 1 << 30 when
                             // the edge at time_max is absent | value at the cycle start
                             // << 31); null: every clock edge is walked
  int64_t n_event;
  int64_t t_lo, t_hi;
  int32_t n_net;
  // time base
  int64_t tpc;
  uint32_t tpc_magic;        // ceil(2^32 / tpc) for tpc >= 2 (32-bit division by tpc), 0 for tpc == 1
  uint64_t tpc_magic64;      // ceil(2^64 / tpc) for tpc >= 2 (division of a tick by tpc), 0 for tpc == 1
  double ts;
  double period_d;
  double inv_period_d;
  int64_t tmax;
  int64_t n_period;
  float min_diff0;           // float(time_max * timescale)
  double tmax_s;             // time_max * timescale (s)
  // tiling
  int64_t cyc0;              // first cycle of the window
  int64_t cycles_per_tile;
  int32_t n_tiles;
  int32_t gates_per_block;
  // fixed point scales (J -> int64)
  double fx_dyn;
  double fx_leak;
  float fx_dyn_f;                   // fx_dyn as a float when it is a power of two >= 1 within
                                    // float range (float energies then scale exactly in FP32), else 0
  int32_t fx_pad;
  // accumulators
  double* cell_acc;                 // [5][n_cell]
  unsigned long long* cyc_acc;      // [6][n_period+1]
  uint32_t* cnt_cell;               // [4][n_cell]
  unsigned long long* cnt_cyc;      // [2][n_period+1]
  int32_t n_cell;
  int32_t* status;                  // error bits
  // per-cycle accumulators by cell group (optional)
  const int32_t* cell_cgroup;       // [n_cell] group of each cell, or null
  int32_t n_cgroup;
  unsigned long long* cyc_acc_g;    // [n_cgroup][6][n_period+1]
  // cycle ranges (optional): tile t covers cycles [tiles[t].x, tiles[t].x +
  // tiles[t].y); null = tile t covers cycles cyc0 + t * cycles_per_tile ...
  const int2* tiles;
  // the window is evaluated on its own (after a gap, or over cycle ranges):
  // each tile's leakage starts at its first tick and ends at its last
  // instead of carrying over from the windows before
  int32_t standalone;
  // launch order of power_walk_kernel: 0 = block (x, y) is gate block x of
  // tile y (tile-major); 1 = gate block y of tile x, so that every tile of
  // the heaviest gate blocks starts first (set by the launch)
  int32_t gate_major;
  // density split (optional, one-window walk only): item_off[k] = first walk
  // item of the cell at walk-order position k (exclusive prefix over
  // positions of the number of threads that walk it per tile), n_cell + 1
  // entries; null = one thread per cell and tile
  const int32_t* item_off;
};

// status bits set by the kernel
// largest window whose glitch widths are precomputed (float per event)
constexpr int64_t kGlitchPwMaxEvents = int64_t(1) << 30;

// largest (tile, net) first-event table built per window (int32 entries)
constexpr int64_t kTileFirstMaxEntries = int64_t(1) << 27;

// largest number of per-cycle cell groups (sort keys hold the group in 18 bits)
constexpr int32_t kMaxCycleGroups = 65536;

constexpr int32_t kErrNetRange = 1;
constexpr int32_t kErrTimeOrder = 2;
constexpr int32_t kErrTimeRange = 4;
constexpr int32_t kErrContext = 8;

// Launches the walk over one bucket of cells. shared-memory bytes computed inside.
// warp_walk: cells of up to kFastPins pins without drift are walked by one
// warp each (power_warp_kernel) when the window has its glitch widths.
cudaError_t launch_power_walk(const KParams& p, int max_pins, bool counts, int threads,
                              cudaStream_t stream, bool warp_walk = false);
// Blocks per SM of the per-thread walk launch_power_walk would run for p
// (without warp_walk); 0 when the occupancy query fails.
int walk_blocks_per_sm_launch(const KParams& p, int max_pins, bool counts, int threads);
// Persistent walk over many designs' windows (one launch per pin bucket):
// d_params holds one KParams per (design, bucket), d_items the work items
// (x: params index, y: gate block, z: tile), *d_n_items their count and
// *d_counter the queue head (zeroed before the launch). smem must cover the
// largest item's shared memory.
// runs: the launch walks periodic clock pins as runs (items whose p.pclk is
// set; fast bucket without drift only).
cudaError_t launch_power_walk_batch(const KParams* d_params, const int4* d_items, const int* d_n_items,
                                    int* d_counter, int grid, int max_pins, bool counts, bool drift, bool runs,
                                    int threads, size_t smem, cudaStream_t stream);
// Dynamic shared memory of one walk block for these parameters.
size_t walk_item_smem_bytes(const KParams& p, int max_pins, bool counts, int threads);
// Resident blocks per SM of the persistent walk at this shape.
int walk_blocks_per_sm(int max_pins, bool counts, bool drift, bool runs, int threads, size_t smem);

// bin_sets: 1, or 2 when per-cycle accumulators are kept by cell group;
// clock_runs: the bins carry the two clock-run slots (p.pclk set).
size_t power_walk_smem_bytes(int64_t cycles_per_tile, bool counts, int threads, int ring_pins,
                             size_t tab_bytes, int bin_sets = 1, bool clock_runs = false);

// Shared memory the clock-run walk (RUNS kernels) adds to the bytes above:
// the threads' per-cell sums.
size_t walk_runs_acc_bytes(int threads);

// Fills the pattern table p.pclk (`out`) for the n nets in `nets` over the
// window p describes: a net is periodic when its events in [max(t_lo, 1),
// min(t_hi, tmax + 1)) are exactly one edge at phase x and one at phase y of
// every cycle, alternating between 0 and 1, with a known value before them.
cudaError_t launch_pclk(const KParams& p, const KParams* d_p, const int32_t* nets, int32_t n, int2* out,
                        cudaStream_t stream);

// Fills p.glitch_pw's array (`out`, n_event entries) for the window p
// describes; with d_p set the kernel reads the window from there.
cudaError_t launch_glitch_pw(const KParams& p, const KParams* d_p, float* out, cudaStream_t stream);

// Builds p.tile_first's table (into `out`, n_tiles * n_net entries) for the
// window p describes; with d_p set the kernel reads the window from there.
cudaError_t launch_tile_first(const KParams& p, const KParams* d_p, int32_t* out, cudaStream_t stream);

// Walk order for one window: cells stay grouped by pin bucket and, within a
// bucket, by cell group when groups are set, and are sorted by the number of
// events on their pins (descending) within that.
size_t work_sort_temp_bytes(int32_t n_cell);
cudaError_t sort_cells_by_work(const KParams& p, const int32_t* base_order, int32_t n_cell,
                               const int32_t* bucket_begin, unsigned long long* keys_in,
                               unsigned long long* keys_out, int32_t* order_out, void* temp,
                               size_t temp_bytes, cudaStream_t stream);

// Most threads one cell is split into per tile by the density rule.
constexpr int32_t kMaxSplit = 32;
// Default events per thread and tile above which a cell is split.
constexpr int32_t kDefaultSplitEvents = 2048;

// Density split of one window, after sort_cells_by_work (keys_sorted: the
// sorted keys, whose low 39 bits hold the inverted event count of the cell
// at each walk-order position): the cell at position k is walked by
// n_k = clamp(ceil(work_k * cycles_per_tile / n_cyc / split_events), 1,
// min(kMaxSplit, cycles_per_tile)) threads per tile, each over 1/n_k of the
// tile's cycles; item_off (n_cell + 1 entries) receives the exclusive prefix
// of n_k. n_cyc: cycles of the window. temp: split_temp_bytes(n_cell) bytes.
size_t split_scan_temp_bytes(int32_t n_cell);
inline size_t split_temp_bytes(int32_t n_cell) {
  return ((static_cast<size_t>(n_cell) + 1) * 4 + 255) / 256 * 256 + split_scan_temp_bytes(n_cell);
}
cudaError_t compute_split(const unsigned long long* keys_sorted, int32_t n_cell, int64_t cycles_per_tile,
                          int64_t n_cyc, int32_t split_events, int32_t* item_off, void* temp, size_t temp_bytes,
                          cudaStream_t stream);

// Scratch of the separate dynamic and leakage kernels (gtp_config.
// separate_kernels): per net the first evaluated event and their number,
// per walked cell its pin events and their exclusive prefix, CUB scan
// temporary storage.
struct SeparateScratch {
  int64_t* net_lo;     // [n_net]
  int64_t* net_cnt;    // [n_net]
  int64_t* cell_cnt;   // [n_cell + 1]
  int64_t* cell_off;   // [n_cell + 1]
  void* temp;
  size_t temp_bytes;   // separate_scan_temp_bytes(n_cell)
};
size_t separate_scan_temp_bytes(int32_t n_cell);

// One window by the two unfused kernels: a thread per pin event for the
// dynamic energies, then a thread per cell and tile for the leakage, over
// the walk order p.order[0, bucket_begin[3]) (pin buckets as the walk's).
cudaError_t launch_separate_kernels(const KParams& p, const int32_t* bucket_begin, bool counts, int threads,
                                    const SeparateScratch& s, cudaStream_t stream);

// Finalize kernels: per-cell floats, totals/groups, per-cycle floats.
// With d_cycle5_g (and p.cyc_acc_g), also the per-group per-cycle floats
// [n_cgroup][5][n_period], using d_leak_tmp_g [n_cgroup][n_period].
cudaError_t launch_finalize(const KParams& p, const uint8_t* cell_group, float* d_cell5,
                            float* d_cycle5, double* d_totals_groups,
                            unsigned long long* d_leak_prefix_tmp, cudaStream_t stream,
                            float* d_cycle5_g = nullptr, unsigned long long* d_leak_tmp_g = nullptr);

}  // namespace gtpb
