// abi.cu — implementation of the C ABI declared in include/gtpb200.h.
//
// Replaces the host orchestration of CudaPower::power
// (power/cuda/CudaPower.cu:1227-1337): the reference allocates a fixed
// max_event_num AoS buffer, copies it synchronously in full, launches one
// kernel per interval and merges per-gate tiles. Here a context keeps the
// packed design resident, copies only the events of each pushed window
// (asynchronously, on the context's stream), walks them, and keeps the
// accumulators on the device until gtp_fetch.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "engine.h"

using namespace gtpb;

struct gtp_ctx {
  int device = 0;
  int sm_count = 0;                   // SMs of the device (0: unknown)
  cudaStream_t stream = nullptr;      // stream in use
  cudaStream_t own_stream = nullptr;  // created by the context
  gtp_config cfg;
  Packed P;
  std::string err;
  // static design on device
  int32_t *d_cell_pin_off = nullptr, *d_cell_type = nullptr, *d_cell_inst = nullptr,
          *d_order = nullptr, *d_pin_net = nullptr, *d_pin_slot = nullptr;
  uint8_t *d_pin_flags = nullptr, *d_cell_group = nullptr;
  uint8_t* d_net_glitch = nullptr;  // [n_net] 1 when some non-clock pin reads the net
  // nets read by clock pins, and their per-window periodic patterns
  int32_t* d_clk_nets = nullptr;
  int32_t n_clk_nets = 0;
  std::vector<int32_t> clk_nets;
  int2* d_pclk = nullptr;            // [n_net]
  float *d_pin_gden = nullptr, *d_pin_swe = nullptr, *d_leak_pool = nullptr, *d_inst = nullptr;
  DevType* d_types = nullptr;
  DevSlot* d_slots = nullptr;
  uint2* d_cubes = nullptr;
  int32_t* d_type_fast_off = nullptr;
  int16_t* d_fast_tab = nullptr;
  // per-window walk order sorted by work
  unsigned long long *d_keys_in = nullptr, *d_keys_out = nullptr;
  int32_t* d_order_work = nullptr;
  void* d_sort_temp = nullptr;
  size_t sort_temp_bytes = 0;
  // tiles of a cycle-range push
  int2* d_tiles = nullptr;
  size_t tiles_cap = 0;
  // per-window density split of the walk order (split_events)
  int32_t* d_item_off = nullptr;
  void* d_split_temp = nullptr;
  size_t split_temp_bytes = 0;
  // events (host-pushed windows)
  // events pushed from host memory: two device slots, filled on copy_stream
  // while the walk of the other slot's window runs; slot s's windows walk on
  // walk_stream[s], so the next window's walk may start while this one's
  // last blocks finish
  struct Slot {
    int64_t cap = 0;
    int64_t *d_net_off = nullptr, *d_ev_t = nullptr, *d_net_base = nullptr;
    uint32_t* d_ev_v = nullptr;
    cudaEvent_t free_ev = nullptr;  // the walk that read the slot is done
    bool used = false;
  } slot[2];
  int next_slot = 0;
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t copied_ev = nullptr;
  cudaStream_t walk_stream[2] = {nullptr, nullptr};
  cudaEvent_t walk_done[2] = {nullptr, nullptr};  // the last walk enqueued on walk_stream[s]
  bool walk_pending[2] = {false, false};
  cudaEvent_t stream_tail = nullptr;               // `stream`'s work before a host-pushed walk
  // the context queued work of its own on `stream` (a reset, a device-pushed
  // window, a finalize, ...) that the walk streams have not been ordered after
  bool stream_dirty = true;
  // per-window walk scratch of the other event slot: the first-event table,
  // glitch widths, clock patterns, work order and split offsets of the
  // window that walks on the other stream. The context's own fields hold the
  // set of slot scratch_slot; swap_scratch exchanges the two.
  struct WalkScratch {
    int32_t* tile_first = nullptr;
    int64_t tile_first_cap = 0;
    float* glitch_pw = nullptr;
    int64_t glitch_pw_cap = 0;
    int2* pclk = nullptr;
    unsigned long long *keys_in = nullptr, *keys_out = nullptr;
    int32_t* order_work = nullptr;
    void* sort_temp = nullptr;
    int32_t* item_off = nullptr;
    void* split_temp = nullptr;
    bool ready = false;
  } spare;
  int scratch_slot = 0;
  // accumulators and outputs
  double* d_cell_acc = nullptr;
  unsigned long long* d_cyc_acc = nullptr;
  uint32_t* d_cnt_cell = nullptr;
  unsigned long long* d_cnt_cyc = nullptr;
  int32_t* d_status = nullptr;
  float* d_cell5 = nullptr;
  float* d_cycle5 = nullptr;
  double* d_tg = nullptr;
  unsigned long long* d_leak_tmp = nullptr;
  double fx_dyn = 0, fx_leak = 0;
  int64_t last_t_hi = 0;
  bool any_window = false;
  // per-cycle waveforms by cell group (gtp_set_cycle_groups)
  int32_t n_cgroup = 0;
  int32_t* d_cgroup = nullptr;
  // per-window table of each (tile, net)'s first event
  int32_t* d_tile_first = nullptr;
  int64_t tile_first_cap = 0;
  // per-window glitch pulse width of each listed event
  float* d_glitch_pw = nullptr;
  int64_t glitch_pw_cap = 0;
  unsigned long long* d_cyc_acc_g = nullptr;
  float* d_cycle5_g = nullptr;
  unsigned long long* d_leak_tmp_g = nullptr;
  // the separate dynamic and leakage kernels (cfg.separate_kernels)
  SeparateScratch sep{};
};

namespace {

std::mutex g_err_mu;
std::string g_create_err;

gtp_status cuda_fail(gtp_ctx* c, cudaError_t e, const char* what) {
  if (c) c->err = std::string(what) + ": " + cudaGetErrorString(e);
  return GTP_ECUDA;
}

template <typename T>
cudaError_t upload(T** dst, const std::vector<T>& src, cudaStream_t s) {
  const size_t bytes = std::max<size_t>(1, src.size()) * sizeof(T);
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(dst), bytes);
  if (e != cudaSuccess) return e;
  if (!src.empty()) e = cudaMemcpyAsync(*dst, src.data(), src.size() * sizeof(T),
                                        cudaMemcpyHostToDevice, s);
  return e;
}

// largest power of two s with bound * s <= 2^62
double fixed_point_scale(double bound) {
  if (!(bound > 0) || !std::isfinite(bound)) return std::ldexp(1.0, 60);
  int ex;
  std::frexp(bound, &ex);            // bound < 2^ex
  return std::ldexp(1.0, 62 - ex);
}

void free_all(gtp_ctx* c) {
  void* ptrs[] = {c->d_cell_pin_off, c->d_cell_type, c->d_cell_inst, c->d_order, c->d_pin_net,
                  c->d_pin_slot, c->d_pin_flags, c->d_cell_group, c->d_pin_gden, c->d_pin_swe, c->d_net_glitch,
                  c->d_leak_pool, c->d_inst, c->d_types, c->d_slots, c->d_cubes,
                  c->slot[0].d_net_off, c->slot[0].d_ev_t, c->slot[0].d_net_base, c->slot[0].d_ev_v,
                  c->slot[1].d_net_off, c->slot[1].d_ev_t, c->slot[1].d_net_base, c->slot[1].d_ev_v,
                  c->d_cell_acc, c->d_cyc_acc,
                  c->d_cnt_cell, c->d_cnt_cyc, c->d_status, c->d_cell5, c->d_cycle5, c->d_tg,
                  c->d_leak_tmp, c->d_type_fast_off, c->d_fast_tab, c->d_keys_in,
                  c->d_keys_out, c->d_order_work, c->d_sort_temp, c->d_cgroup, c->d_cyc_acc_g, c->d_tile_first, c->d_glitch_pw,
                  c->d_cycle5_g, c->d_leak_tmp_g, c->d_clk_nets, c->d_pclk, c->d_item_off, c->d_split_temp, c->d_tiles,
                  c->sep.net_lo, c->sep.net_cnt, c->sep.cell_cnt, c->sep.cell_off, c->sep.temp,
                  c->spare.tile_first, c->spare.glitch_pw, c->spare.pclk, c->spare.keys_in, c->spare.keys_out,
                  c->spare.order_work, c->spare.sort_temp, c->spare.item_off, c->spare.split_temp};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  for (int k = 0; k < 2; ++k) {
    if (c->walk_done[k]) cudaEventDestroy(c->walk_done[k]);
    if (c->walk_stream[k]) cudaStreamDestroy(c->walk_stream[k]);
  }
  if (c->stream_tail) cudaEventDestroy(c->stream_tail);
  for (auto& sl : c->slot)
    if (sl.free_ev) cudaEventDestroy(sl.free_ev);
  if (c->copied_ev) cudaEventDestroy(c->copied_ev);
  if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
}

// Makes stream s wait for the walks of host-pushed windows still in flight
// on the walk streams.
cudaError_t join_walks(gtp_ctx* c, cudaStream_t s) {
  // the caller queues work on s next
  if (s == c->stream) c->stream_dirty = true;
  for (int k = 0; k < 2; ++k)
    if (c->walk_pending[k]) {
      cudaError_t e = cudaStreamWaitEvent(s, c->walk_done[k], 0);
      if (e != cudaSuccess) return e;
    }
  return cudaSuccess;
}

void swap_scratch(gtp_ctx* c) {
  auto& w = c->spare;
  std::swap(c->d_tile_first, w.tile_first);
  std::swap(c->tile_first_cap, w.tile_first_cap);
  std::swap(c->d_glitch_pw, w.glitch_pw);
  std::swap(c->glitch_pw_cap, w.glitch_pw_cap);
  std::swap(c->d_pclk, w.pclk);
  std::swap(c->d_keys_in, w.keys_in);
  std::swap(c->d_keys_out, w.keys_out);
  std::swap(c->d_order_work, w.order_work);
  std::swap(c->d_sort_temp, w.sort_temp);
  std::swap(c->d_item_off, w.item_off);
  std::swap(c->d_split_temp, w.split_temp);
  c->scratch_slot ^= 1;
}

// Allocates the second scratch set like the first (the tables that grow
// with the window start empty), on first use.
cudaError_t ready_spare(gtp_ctx* c) {
  auto& w = c->spare;
  if (w.ready) return cudaSuccess;
  const size_t nc = std::max<int32_t>(1, c->P.n_cell);
  cudaError_t e = cudaSuccess;
  auto alloc = [&](auto** p, size_t bytes) {
    if (e == cudaSuccess && !*p) e = cudaMalloc(reinterpret_cast<void**>(p), bytes);
  };
  if (c->d_pclk) {
    alloc(&w.pclk, sizeof(int2) * static_cast<size_t>(c->P.n_net));
    if (e == cudaSuccess) e = cudaMemsetAsync(w.pclk, 0xff, sizeof(int2) * static_cast<size_t>(c->P.n_net), c->stream);
  }
  if (c->d_keys_in) {
    alloc(&w.keys_in, sizeof(unsigned long long) * nc);
    alloc(&w.keys_out, sizeof(unsigned long long) * nc);
    alloc(&w.order_work, sizeof(int32_t) * nc);
    alloc(&w.sort_temp, c->sort_temp_bytes);
  }
  if (c->d_item_off) {
    alloc(&w.item_off, sizeof(int32_t) * (nc + 1));
    alloc(&w.split_temp, c->split_temp_bytes);
  }
  if (e == cudaSuccess) w.ready = true;
  return e;
}

KParams make_params(gtp_ctx* c) {
  const Packed& P = c->P;
  KParams k;
  std::memset(&k, 0, sizeof(k));
  k.cell_pin_off = c->d_cell_pin_off;
  k.cell_type = c->d_cell_type;
  k.cell_inst = c->d_cell_inst;
  k.order = c->d_order;
  k.pin_net = c->d_pin_net;
  k.pin_flags = c->d_pin_flags;
  k.net_glitch = c->d_net_glitch;
  k.pin_gden = c->d_pin_gden;
  k.pin_swe = c->d_pin_swe;
  k.types = c->d_types;
  k.slots = c->d_slots;
  k.pin_slot = c->d_pin_slot;
  k.cubes = c->d_cubes;
  k.leak_pool = c->d_leak_pool;
  k.inst = c->d_inst;
  k.type_fast_off = c->d_type_fast_off;
  k.fast_tab = c->d_fast_tab;
  k.drift = P.drift ? 1 : 0;
  k.n_fast_tab = static_cast<int32_t>(P.fast_tab.size());
  k.n_leak_pool = static_cast<int32_t>(P.leak_pool.size());
  k.tabs_in_smem = (P.fast_tab.size() * 2 + P.leak_pool.size() * 4) <= 16384 ? 1 : 0;
  k.fast_inst_stride = P.fast_inst_floats + 1;   // odd stride: no shared-memory bank conflicts
  k.tmax_s = static_cast<double>(P.tmax) * P.ts;
  k.n_net = P.n_net;
  k.tpc = P.tpc;
  k.tpc_magic = P.tpc >= 2 && P.tpc < (int64_t(1) << 31)
                    ? static_cast<uint32_t>(((uint64_t(1) << 32) + static_cast<uint64_t>(P.tpc) - 1) /
                                            static_cast<uint64_t>(P.tpc))
                    : 0u;
  k.tpc_magic64 = P.tpc >= 2 ? static_cast<uint64_t>((static_cast<unsigned __int128>(1) << 64) / static_cast<uint64_t>(P.tpc) +
                                                     ((static_cast<unsigned __int128>(1) << 64) % static_cast<uint64_t>(P.tpc) != 0))
                              : 0u;
  k.ts = P.ts;
  k.period_d = P.period_d;
  k.inv_period_d = 1.0 / P.period_d;
  k.tmax = P.tmax;
  k.n_period = P.n_period;
  k.min_diff0 = static_cast<float>(static_cast<double>(P.tmax) * P.ts);
  k.fx_dyn = c->fx_dyn;
  k.fx_leak = c->fx_leak;
  k.fx_dyn_f = (c->fx_dyn >= 1.0 && c->fx_dyn <= std::ldexp(1.0, 126)) ? static_cast<float>(c->fx_dyn) : 0.0f;
  k.cell_acc = c->d_cell_acc;
  k.cyc_acc = c->d_cyc_acc;
  k.cnt_cell = c->d_cnt_cell;
  k.cnt_cyc = c->d_cnt_cyc;
  k.n_cell = P.n_cell;
  k.status = c->d_status;
  k.cell_cgroup = c->n_cgroup > 0 ? c->d_cgroup : nullptr;
  k.n_cgroup = c->n_cgroup;
  k.cyc_acc_g = c->n_cgroup > 0 ? c->d_cyc_acc_g : nullptr;
  return k;
}

// Largest cycle tile whose shared memory (bins with counters, event
// buffers, tables, and 1 KB for the walk's static shared memory) stays
// within 227 KB.
int64_t max_cycles_per_tile(int threads, int bin_sets, bool clock_runs = false) {
  const int64_t budget = 226 * 1024 - static_cast<int64_t>(power_walk_smem_bytes(0, false, threads, kFastPins, 16384 + threads * 65 * 4)) -
                         static_cast<int64_t>(clock_runs ? walk_runs_acc_bytes(threads) : 0);
  const int slots = clock_runs ? kNumBinSlotsRun : kNumCycAcc;
  return std::max<int64_t>(1, std::min<int64_t>(3072, budget / (bin_sets * slots * 8 + 8)));
}

// Whether windows of this context walk periodic clock pins as runs.
bool clock_runs_on(const gtp_ctx* c) {
  return c->cfg.clock_runs >= 0 && c->n_clk_nets > 0 && c->d_pclk && !c->P.drift && c->P.tpc >= 2 &&
         c->P.tpc < (int64_t(1) << 30);
}

// Per-tile setup of a cell (first events, initial states, the bin flush), in
// cycles of walk work.
constexpr int64_t kTileSetupCycles = 32;

// Tile count for a window of n_cyc cycles, from nt_min (tiles of at most the
// largest tile) to 3 x nt_min (tiles of at least 64 cycles). The walk of the
// largest pin bucket launches G gate blocks per tile and R blocks fit on the
// device at once, so it runs in ceil(G x nt / R) waves of blocks, each about
// (n_cyc / nt + kTileSetupCycles) cycles long; the count with the shortest
// such time wins, the smallest on ties. q: the window's walk parameters with
// the largest tile (its shared memory bounds the occupancy from below).
int64_t wave_tile_count(const gtp_ctx* c, const KParams& q, int64_t n_cyc, int64_t nt_min) {
  if (c->sm_count <= 0 || nt_min < 1) return nt_min;
  static const int bucket_pins[3] = {4, 8, kMaxPins};
  int b = 0;
  for (int k = 1; k < 3; ++k)
    if (c->P.bucket_begin[k + 1] - c->P.bucket_begin[k] > c->P.bucket_begin[b + 1] - c->P.bucket_begin[b]) b = k;
  const int64_t n_cells = c->P.bucket_begin[b + 1] - c->P.bucket_begin[b];
  const int threads = c->cfg.n_thread_per_block > 0 ? c->cfg.n_thread_per_block : 256;
  const int gpb = c->cfg.gates_per_block > 0 ? c->cfg.gates_per_block : threads;
  if (n_cells <= 0) return nt_min;
  const int per_sm = walk_blocks_per_sm_launch(q, bucket_pins[b], c->cfg.collect_counts != 0, threads);
  if (per_sm <= 0) return nt_min;
  const int64_t g = (n_cells + gpb - 1) / gpb;
  const int64_t r = static_cast<int64_t>(per_sm) * c->sm_count;
  const int64_t nt_max = std::min<int64_t>({3 * nt_min, std::max<int64_t>(nt_min, n_cyc / 64), 65535});
  int64_t best = nt_min, best_cost = -1;
  for (int64_t nt = nt_min; nt <= nt_max; ++nt) {
    const int64_t waves = (g * nt + r - 1) / r;
    const int64_t cost = waves * ((n_cyc + nt - 1) / nt + kTileSetupCycles);
    if (best_cost < 0 || cost < best_cost) {
      best = nt;
      best_cost = cost;
    }
  }
  return best;
}

// Validates one window and sets up its walk parameters *out (sorting the
// walk order by work on `stream` when configured). The context's window
// state advances only when the walk is enqueued (commit_window).
// ranges (pairs of cycles [c0, c1), ascending and disjoint) restrict the
// walk to those cycles of the window.
gtp_status prepare_window(gtp_ctx* c, const int64_t* d_net_off, const int64_t* d_t, const uint32_t* d_v,
                          const int64_t* d_base, int64_t n_event, int64_t t_lo, int64_t t_hi,
                          cudaStream_t stream, KParams* out, bool enqueue_prep = true,
                          const std::vector<int64_t>* ranges = nullptr) {
  if (t_hi <= t_lo) { c->err = "t_hi must exceed t_lo"; return GTP_EINVAL; }
  if (t_lo < 0) { c->err = "t_lo must be >= 0"; return GTP_EINVAL; }
  if (c->any_window && t_lo < c->last_t_hi) {
    c->err = "windows must be pushed in time order without overlap";
    return GTP_ESTATE;
  }
  const Packed& P = c->P;
  // a window that does not continue the last one (a gap, a first window
  // after tick 0, or cycle ranges) is evaluated on its own: its leakage
  // starts at its first tick instead of carrying over
  const bool standalone = ranges != nullptr || (!c->any_window && t_lo > 0) ||
                          (c->any_window && t_lo > c->last_t_hi);
  // the separate kernels walk every clock edge, in the design's cell order
  const bool sep = c->cfg.separate_kernels > 0;

  KParams k = make_params(c);
  k.net_off = d_net_off;
  k.ev_t = d_t;
  k.ev_v = d_v;
  k.net_base = d_base;
  k.n_event = n_event;
  k.t_lo = t_lo;
  k.t_hi = t_hi;
  // cycles of the window: [t_lo/tpc, last cycle that can hold an event)
  const int64_t last_tick = std::min<int64_t>(t_hi - 1, P.tmax);
  k.cyc0 = t_lo / P.tpc;
  const int64_t cyc_end = last_tick / P.tpc + 1;
  const int64_t n_cyc = std::max<int64_t>(1, cyc_end - k.cyc0);
  int64_t ct = c->cfg.cycles_per_tile;
  // 768 cycles keep two blocks per SM with the event buffers; per-group bins
  // double the tile's shared memory
  if (ct <= 0) ct = c->n_cgroup > 0 ? 512 : 768;
  ct = std::min<int64_t>(ct, n_cyc);
  const int threads_ = c->cfg.n_thread_per_block > 0 ? c->cfg.n_thread_per_block : 256;
  // bins + event buffers + tables within 227 KB of shared memory; tile span
  // (ct+1)*tpc within 2^31 ticks, as the walk holds times as 32-bit offsets
  // from the tile start
  const bool runs = clock_runs_on(c);
  const int64_t max_ct = std::min<int64_t>(max_cycles_per_tile(threads_, c->n_cgroup > 0 ? 2 : 1, runs),
                                           (int64_t(INT32_MAX) / P.tpc) - 1);
  ct = std::min(ct, max_ct);
  ct = std::max<int64_t>(ct, (n_cyc + 65534) / 65535);  // grid.y limit
  if (ct > max_ct || ct < 1) { c->err = "window spans too many cycles for one launch"; return GTP_EOVERFLOW; }
  // with the default tile, share the window's cycles evenly among its
  // tiles, so that no tile holds only a few cycles (each tile sets up every
  // cell once), and take the tile count whose blocks fill the SMs' waves best
  if (c->cfg.cycles_per_tile <= 0) {
    int64_t nt = (n_cyc + ct - 1) / ct;
    if (!ranges && !sep && c->cfg.warp_walk <= 0) {
      KParams q = make_params(c);
      q.cycles_per_tile = ct;
      q.pclk = (clock_runs_on(c) && !standalone) ? c->d_pclk : nullptr;
      nt = wave_tile_count(c, q, n_cyc, nt);
    }
    ct = (n_cyc + nt - 1) / nt;
  }
  k.cycles_per_tile = ct;
  k.n_tiles = static_cast<int32_t>((n_cyc + ct - 1) / ct);
  k.standalone = standalone ? 1 : 0;
  if (ranges) {
    // tiles of at most ct cycles over the ranges, within the window
    std::vector<int2> tiles;
    const int64_t cyc_end_w = k.cyc0 + n_cyc;
    for (size_t r = 0; r + 1 < ranges->size(); r += 2) {
      const int64_t c0 = std::max<int64_t>((*ranges)[r], k.cyc0), c1 = std::min<int64_t>((*ranges)[r + 1], cyc_end_w);
      for (int64_t cc = c0; cc < c1; cc += ct)
        tiles.push_back(make_int2(static_cast<int>(cc), static_cast<int>(std::min<int64_t>(ct, c1 - cc))));
    }
    if (tiles.size() > 65535) { c->err = "cycle ranges need more than 65535 tiles"; return GTP_EOVERFLOW; }
    if (tiles.size() > c->tiles_cap) {
      cudaError_t e = cudaStreamSynchronize(c->stream);
      if (e != cudaSuccess) return cuda_fail(c, e, "sync");
      if (c->d_tiles) cudaFree(c->d_tiles);
      c->d_tiles = nullptr;
      c->tiles_cap = 0;
      e = cudaMalloc(&c->d_tiles, sizeof(int2) * tiles.size());
      if (e != cudaSuccess) return cuda_fail(c, e, "range tiles");
      c->tiles_cap = tiles.size();
    }
    if (!tiles.empty()) {
      cudaError_t e = cudaMemcpyAsync(c->d_tiles, tiles.data(), sizeof(int2) * tiles.size(), cudaMemcpyHostToDevice,
                                      stream);
      if (e != cudaSuccess) return cuda_fail(c, e, "range tiles");
    }
    k.tiles = c->d_tiles;
    k.n_tiles = static_cast<int32_t>(tiles.size());
  }
  const int threads = c->cfg.n_thread_per_block > 0 ? c->cfg.n_thread_per_block : 256;
  k.gates_per_block = c->cfg.gates_per_block > 0 ? c->cfg.gates_per_block : threads;
  // the (tile, net) first-event table, when it stays within kTileFirstMaxEntries
  const int64_t entries = static_cast<int64_t>(k.n_tiles) * P.n_net;
  if (entries > 0 && entries <= kTileFirstMaxEntries) {
    if (entries > c->tile_first_cap) {
      cudaError_t e = cudaStreamSynchronize(stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
      if (e != cudaSuccess) return cuda_fail(c, e, "sync");
      if (c->d_tile_first) cudaFree(c->d_tile_first);
      c->d_tile_first = nullptr;
      c->tile_first_cap = 0;
      const int64_t cap = std::min<int64_t>(kTileFirstMaxEntries, entries * 2);
      e = cudaMalloc(&c->d_tile_first, sizeof(int32_t) * cap);
      if (e == cudaSuccess) c->tile_first_cap = cap;
    }
    if (c->d_tile_first) k.tile_first = c->d_tile_first;
  }
  // the glitch widths of the window's events, within kGlitchPwMaxEvents
  // (cycle ranges classify the few events they walk online instead)
  if (!ranges && n_event > 0 && n_event <= kGlitchPwMaxEvents) {
    if (n_event > c->glitch_pw_cap) {
      cudaError_t e = cudaStreamSynchronize(stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
      if (e != cudaSuccess) return cuda_fail(c, e, "sync");
      if (c->d_glitch_pw) cudaFree(c->d_glitch_pw);
      c->d_glitch_pw = nullptr;
      c->glitch_pw_cap = 0;
      const int64_t cap = std::min<int64_t>(kGlitchPwMaxEvents, n_event + n_event / 4 + 1024);
      e = cudaMalloc(&c->d_glitch_pw, sizeof(float) * cap);
      if (e == cudaSuccess) c->glitch_pw_cap = cap;
    }
    if (c->d_glitch_pw) k.glitch_pw = c->d_glitch_pw;
  }
  const bool sorted = c->cfg.sort_by_work && c->d_order_work && !ranges && !sep;
  if (sorted) k.order = c->d_order_work;
  if (runs && !standalone && !sep) k.pclk = c->d_pclk;
  if (enqueue_prep) {
    cudaError_t e = cudaSuccess;
    if (k.tile_first) e = launch_tile_first(k, nullptr, c->d_tile_first, stream);
    if (e == cudaSuccess && k.glitch_pw) e = launch_glitch_pw(k, nullptr, c->d_glitch_pw, stream);
    if (e == cudaSuccess && k.pclk) e = launch_pclk(k, nullptr, c->d_clk_nets, c->n_clk_nets, c->d_pclk, stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "tile index");
    if (sorted) {
      e = sort_cells_by_work(k, c->d_order, P.bucket_begin[3], P.bucket_begin, c->d_keys_in, c->d_keys_out,
                             c->d_order_work, c->d_sort_temp, c->sort_temp_bytes, stream);
      if (e != cudaSuccess) return cuda_fail(c, e, "walk order");
    }
  }
  *out = k;
  return GTP_OK;
}

// The per-window preparation prepare_window(..., enqueue_prep = false) left
// to the caller; d_k: the window's parameters in device memory.
cudaError_t enqueue_window_prep(gtp_ctx* c, const KParams& k, const KParams* d_k, cudaStream_t stream) {
  if (k.tile_first) {
    cudaError_t e = launch_tile_first(k, d_k, c->d_tile_first, stream);
    if (e != cudaSuccess) return e;
  }
  if (k.glitch_pw) {
    cudaError_t e = launch_glitch_pw(k, d_k, c->d_glitch_pw, stream);
    if (e != cudaSuccess) return e;
  }
  if (k.pclk) {
    cudaError_t e = launch_pclk(k, d_k, c->d_clk_nets, c->n_clk_nets, c->d_pclk, stream);
    if (e != cudaSuccess) return e;
  }
  if (!(c->cfg.sort_by_work && c->d_order_work)) return cudaSuccess;
  const Packed& P = c->P;
  return sort_cells_by_work(k, c->d_order, P.bucket_begin[3], P.bucket_begin, c->d_keys_in, c->d_keys_out,
                            c->d_order_work, c->d_sort_temp, c->sort_temp_bytes, stream);
}

void commit_window(gtp_ctx* c, int64_t t_hi) {
  c->any_window = true;
  c->last_t_hi = t_hi;
}

// ws: the stream the window's preparation and walk go on (the context's
// stream, or a walk stream for host-pushed windows).
gtp_status run_window(gtp_ctx* c, const int64_t* d_net_off, const int64_t* d_t,
                      const uint32_t* d_v, const int64_t* d_base, int64_t n_event,
                      int64_t t_lo, int64_t t_hi, const std::vector<int64_t>* ranges = nullptr,
                      cudaStream_t ws = nullptr) {
  if (!ws) ws = c->stream;
  const bool sep = c->cfg.separate_kernels > 0;
  if (sep && ranges) {
    c->err = "separate_kernels: the two-kernel evaluation takes whole windows, not cycle ranges";
    return GTP_EINVAL;
  }
  KParams k;
  gtp_status st = prepare_window(c, d_net_off, d_t, d_v, d_base, n_event, t_lo, t_hi, ws, &k, true, ranges);
  if (st != GTP_OK) return st;
  if (k.n_tiles <= 0) {  // cycle ranges outside the window: nothing to walk
    commit_window(c, t_hi);
    return GTP_OK;
  }
  const Packed& P = c->P;
  const int threads = c->cfg.n_thread_per_block > 0 ? c->cfg.n_thread_per_block : 256;
  const bool counts = c->cfg.collect_counts != 0;
  if (sep) {
    cudaError_t e = launch_separate_kernels(k, P.bucket_begin, counts, threads, c->sep, ws);
    if (e != cudaSuccess) return cuda_fail(c, e, "separate kernels launch");
    commit_window(c, t_hi);
    return GTP_OK;
  }
  // density split: cells whose measured events per tile exceed split_events
  // are walked by several threads, each over part of the tile's cycles
  if (!ranges && c->d_item_off && c->cfg.sort_by_work && c->d_order_work && P.bucket_begin[3] > 0) {
    const int32_t se = c->cfg.split_events > 0 ? c->cfg.split_events : kDefaultSplitEvents;
    const int64_t last_tick = std::min<int64_t>(k.t_hi - 1, k.tmax);
    const int64_t n_cyc = std::max<int64_t>(1, last_tick / k.tpc + 1 - k.cyc0);
    cudaError_t e = compute_split(c->d_keys_out, P.bucket_begin[3], k.cycles_per_tile, n_cyc, se, c->d_item_off,
                                  c->d_split_temp, c->split_temp_bytes, ws);
    if (e != cudaSuccess) return cuda_fail(c, e, "density split");
    k.item_off = c->d_item_off;
  }
  static const int bucket_pins[3] = {4, 8, kMaxPins};
  for (int b = 0; b < 3; ++b) {
    k.order_begin = P.bucket_begin[b];
    k.order_end = P.bucket_begin[b + 1];
    if (k.order_end <= k.order_begin) continue;
    cudaError_t e = launch_power_walk(k, bucket_pins[b], counts, threads, ws, c->cfg.warp_walk > 0);
    if (e != cudaSuccess) return cuda_fail(c, e, "power walk launch");
  }
  commit_window(c, t_hi);
  return GTP_OK;
}

gtp_status check_status(gtp_ctx* c) {
  int32_t st = 0;
  cudaError_t e = join_walks(c, c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&st, c->d_status, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "status read");
  if (st) {
    std::string m = "invalid events:";
    if (st & kErrNetRange) m += " net_off out of range;";
    if (st & kErrTimeOrder) m += " times not strictly increasing within a net;";
    if (st & kErrTimeRange) m += " event time beyond time_max;";
    if (st & kErrContext) m += " window lacks the event before t_lo for some net;";
    c->err = m;
    return GTP_EINVAL;
  }
  return GTP_OK;
}

}  // namespace

extern "C" {

void gtp_config_default(gtp_config* cfg) {
  if (!cfg) return;
  std::memset(cfg, 0, sizeof(*cfg));
  cfg->cuda_device_id = -1;
  cfg->cycles_per_tile = 0;
  cfg->n_thread_per_block = 0;
  cfg->gates_per_block = 0;
  cfg->max_n_pin_for_leakage_power = 16;
  cfg->collect_counts = 0;
  cfg->max_event_num = 0;  // 0 = no cap other than device memory
  cfg->sort_by_work = 1;
}

gtp_status gtp_create(const gtp_design* design, const gtp_config* cfg_in, gtp_ctx** out) {
  if (!out) return GTP_EINVAL;
  *out = nullptr;
  auto set_err = [](const std::string& m) {
    std::lock_guard<std::mutex> g(g_err_mu);
    g_create_err = m;
  };
  if (!design) { set_err("design is NULL"); return GTP_EINVAL; }
  gtp_ctx* c = new (std::nothrow) gtp_ctx();
  if (!c) { set_err("out of host memory"); return GTP_ENOMEM; }
  if (cfg_in) c->cfg = *cfg_in; else gtp_config_default(&c->cfg);
  if (c->cfg.max_n_pin_for_leakage_power <= 0) c->cfg.max_n_pin_for_leakage_power = 16;
  // the walk kernels are compiled for blocks of at most 256 threads, in warps
  if (c->cfg.n_thread_per_block != 0 &&
      (c->cfg.n_thread_per_block < 32 || c->cfg.n_thread_per_block > 256 || c->cfg.n_thread_per_block % 32 != 0)) {
    set_err("n_thread_per_block must be 0 (256) or a multiple of 32 in [32, 256]");
    delete c;
    return GTP_EINVAL;
  }
  std::string err;
  gtp_status st = pack_design(*design, c->cfg.max_n_pin_for_leakage_power, c->P, err);
  if (st != GTP_OK) { set_err(err); delete c; return st; }

  cudaError_t e;
  if (c->cfg.cuda_device_id >= 0) {
    e = cudaSetDevice(c->cfg.cuda_device_id);
    if (e != cudaSuccess) { set_err(std::string("cudaSetDevice: ") + cudaGetErrorString(e)); delete c; return GTP_ECUDA; }
  }
  cudaGetDevice(&c->device);
  if (cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, c->device) != cudaSuccess) {
    (void)cudaGetLastError();
    c->sm_count = 0;
  }
  e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) { set_err(std::string("stream: ") + cudaGetErrorString(e)); delete c; return GTP_ECUDA; }
  c->stream = c->own_stream;

  const Packed& P = c->P;
  std::vector<uint2> cubes(P.cubes.size() / 2);
  for (size_t i = 0; i < cubes.size(); ++i) cubes[i] = make_uint2(P.cubes[2 * i], P.cubes[2 * i + 1]);
#define UP(dst, src) do { e = upload(&c->dst, src, c->stream); if (e != cudaSuccess) goto cuda_err; } while (0)
  UP(d_cell_pin_off, P.cell_pin_off);
  UP(d_cell_type, P.cell_type);
  UP(d_cell_inst, P.cell_inst);
  UP(d_order, P.order);
  UP(d_pin_net, P.pin_net);
  UP(d_pin_slot, P.pin_slot);
  UP(d_pin_flags, P.pin_flags);
  {
    // nets read by some non-clock pin: only those need glitch widths
    std::vector<uint8_t> ng(std::max(1, P.n_net), 0);
    for (size_t q = 0; q < P.pin_net.size(); ++q)
      if (P.pin_net[q] >= 0 && P.pin_net[q] < P.n_net && !(P.pin_flags[q] & 4)) ng[P.pin_net[q]] = 1;
    UP(d_net_glitch, ng);
    // nets read by clock pins: candidates for periodic patterns
    std::vector<uint8_t> isclk(std::max(1, P.n_net), 0);
    for (size_t q = 0; q < P.pin_net.size(); ++q)
      if (P.pin_net[q] >= 0 && P.pin_net[q] < P.n_net && (P.pin_flags[q] & 4)) isclk[P.pin_net[q]] = 1;
    for (int32_t n = 0; n < P.n_net; ++n)
      if (isclk[n]) c->clk_nets.push_back(n);
    c->n_clk_nets = static_cast<int32_t>(c->clk_nets.size());
    if (c->n_clk_nets > 0) {
      UP(d_clk_nets, c->clk_nets);
      e = cudaMalloc(&c->d_pclk, sizeof(int2) * static_cast<size_t>(P.n_net));
      if (e == cudaSuccess) e = cudaMemsetAsync(c->d_pclk, 0xff, sizeof(int2) * static_cast<size_t>(P.n_net), c->stream);
      if (e != cudaSuccess) goto cuda_err;
    }
  }
  UP(d_cell_group, P.cell_group);
  UP(d_pin_gden, P.pin_gden);
  UP(d_pin_swe, P.pin_swe);
  UP(d_leak_pool, P.leak_pool);
  UP(d_inst, P.inst);
  UP(d_types, P.types);
  UP(d_slots, P.slots);
  UP(d_cubes, cubes);
  UP(d_type_fast_off, P.type_fast_off);
  UP(d_fast_tab, P.fast_tab);
#undef UP
  {
    const size_t nc = std::max<int32_t>(1, P.n_cell);
    const size_t ny = static_cast<size_t>(P.n_period + 1);
    e = cudaMalloc(&c->d_cell_acc, sizeof(double) * kNumCellAcc * nc);
    if (e == cudaSuccess) e = cudaMalloc(&c->d_cyc_acc, sizeof(unsigned long long) * kNumCycAcc * ny);
    if (e == cudaSuccess) e = cudaMalloc(&c->d_cnt_cell, sizeof(uint32_t) * 4 * nc);
    if (e == cudaSuccess) e = cudaMalloc(&c->d_cnt_cyc, sizeof(unsigned long long) * 2 * ny);
    if (e == cudaSuccess) e = cudaMalloc(&c->d_status, sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMalloc(&c->d_cell5, sizeof(float) * 5 * nc);
    if (e == cudaSuccess) e = cudaMalloc(&c->d_cycle5, sizeof(float) * 5 * ny);
    if (e == cudaSuccess) e = cudaMalloc(&c->d_tg, sizeof(double) * (GTP_N_GROUP + 1) * 5);
    if (e == cudaSuccess) e = cudaMalloc(&c->d_leak_tmp, sizeof(unsigned long long) * ny);
    if (e == cudaSuccess && c->cfg.sort_by_work && P.n_cell > 0) {
      c->sort_temp_bytes = std::max<size_t>(1, work_sort_temp_bytes(P.n_cell));
      e = cudaMalloc(&c->d_keys_in, sizeof(unsigned long long) * nc);
      if (e == cudaSuccess) e = cudaMalloc(&c->d_keys_out, sizeof(unsigned long long) * nc);
      if (e == cudaSuccess) e = cudaMalloc(&c->d_order_work, sizeof(int32_t) * nc);
      if (e == cudaSuccess) e = cudaMalloc(&c->d_sort_temp, c->sort_temp_bytes);
      if (e == cudaSuccess && c->cfg.split_events >= 0) {
        c->split_temp_bytes = split_temp_bytes(P.n_cell);
        e = cudaMalloc(&c->d_item_off, sizeof(int32_t) * (nc + 1));
        if (e == cudaSuccess) e = cudaMalloc(&c->d_split_temp, c->split_temp_bytes);
      }
    }
    if (e == cudaSuccess && c->cfg.separate_kernels > 0) {
      c->sep.temp_bytes = std::max<size_t>(1, separate_scan_temp_bytes(P.n_cell));
      const size_t nn = static_cast<size_t>(std::max<int32_t>(1, P.n_net));
      e = cudaMalloc(&c->sep.net_lo, sizeof(int64_t) * nn);
      if (e == cudaSuccess) e = cudaMalloc(&c->sep.net_cnt, sizeof(int64_t) * nn);
      if (e == cudaSuccess) e = cudaMalloc(&c->sep.cell_cnt, sizeof(int64_t) * (nc + 1));
      if (e == cudaSuccess) e = cudaMalloc(&c->sep.cell_off, sizeof(int64_t) * (nc + 1));
      if (e == cudaSuccess) e = cudaMalloc(&c->sep.temp, c->sep.temp_bytes);
    }
    if (e != cudaSuccess) goto cuda_err;
  }
  // fixed-point scales: one event's energy, and one level change's leakage
  // over a period, are at most 2^36 units (resolution max|E| * 2^-36 and
  // max|leak| * period * 2^-36, so that terms scaled down by a small glitch
  // ratio keep their precision); a 64-bit bin holds 2^27 of the largest. A
  // shared bin add is one 32-bit atomic, and a second for the high word
  // when the term reaches 2^32 units or the low word carries
  c->fx_dyn = fixed_point_scale(std::max(P.max_abs_energy, 1e-30) * std::ldexp(1.0, 26));
  c->fx_leak = fixed_point_scale(std::max(P.max_abs_leak, 1e-30) * P.period_d * std::ldexp(1.0, 26));
  if (gtp_reset(c) != GTP_OK) { set_err(c->err); free_all(c); delete c; return GTP_ECUDA; }
  e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) goto cuda_err;
  *out = c;
  return GTP_OK;
cuda_err:
  set_err(std::string("device setup: ") + cudaGetErrorString(e));
  free_all(c);
  delete c;
  return e == cudaErrorMemoryAllocation ? GTP_ENOMEM : GTP_ECUDA;
}

void gtp_destroy(gtp_ctx* c) {
  if (!c) return;
  for (int k = 0; k < 2; ++k)
    if (c->walk_stream[k]) cudaStreamSynchronize(c->walk_stream[k]);
  if (c->stream) cudaStreamSynchronize(c->stream);
  free_all(c);
  delete c;
}

const char* gtp_last_error(const gtp_ctx* c) {
  if (c) return c->err.c_str();
  std::lock_guard<std::mutex> g(g_err_mu);
  return g_create_err.c_str();
}

int64_t gtp_n_period(const gtp_ctx* c) { return c ? c->P.n_period : -1; }
int64_t gtp_ticks_per_cycle(const gtp_ctx* c) { return c ? c->P.tpc : -1; }

gtp_status gtp_reset(gtp_ctx* c) {
  if (!c) return GTP_EINVAL;
  const size_t nc = std::max<int32_t>(1, c->P.n_cell);
  const size_t ny = static_cast<size_t>(c->P.n_period + 1);
  cudaError_t e = join_walks(c, c->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->d_cell_acc, 0, sizeof(double) * kNumCellAcc * nc, c->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->d_cyc_acc, 0, sizeof(unsigned long long) * kNumCycAcc * ny, c->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->d_cnt_cell, 0, sizeof(uint32_t) * 4 * nc, c->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->d_cnt_cyc, 0, sizeof(unsigned long long) * 2 * ny, c->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->d_status, 0, sizeof(int32_t), c->stream);
  if (e == cudaSuccess && c->n_cgroup > 0)
    e = cudaMemsetAsync(c->d_cyc_acc_g, 0, sizeof(unsigned long long) * kNumCycAcc * ny * c->n_cgroup, c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "reset");
  c->any_window = false;
  c->last_t_hi = 0;
  return GTP_OK;
}

gtp_status gtp_push_events(gtp_ctx* c, const gtp_events* ev) {
  if (!c || !ev) return GTP_EINVAL;
  if (ev->n_event < 0 || (ev->n_event > 0 && (!ev->time || !ev->value_packed)) || !ev->net_off) {
    c->err = "events: missing arrays";
    return GTP_EINVAL;
  }
  const int32_t nn = c->P.n_net;
  if (ev->net_off[0] != 0 || ev->net_off[nn] != ev->n_event) {
    c->err = "events: net_off must start at 0 and end at n_event";
    return GTP_EINVAL;
  }
  if (c->cfg.max_event_num > 0 && ev->n_event > c->cfg.max_event_num) {
    c->err = "events: window exceeds max_event_num";
    return GTP_EOVERFLOW;
  }
  cudaError_t e = cudaSuccess;
  if (!c->copy_stream) {
    e = cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->copied_ev, cudaEventDisableTiming);
    for (auto& sl : c->slot)
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.free_ev, cudaEventDisableTiming);
    for (int k = 0; k < 2; ++k) {
      if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->walk_stream[k], cudaStreamNonBlocking);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->walk_done[k], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->stream_tail, cudaEventDisableTiming);
    if (e != cudaSuccess) return cuda_fail(c, e, "copy stream");
  }
  const int s_idx = c->next_slot;
  auto& sl = c->slot[s_idx];
  // the walk that last read this slot must be done before it is overwritten
  if (sl.used) {
    e = cudaStreamWaitEvent(c->copy_stream, sl.free_ev, 0);
    if (e != cudaSuccess) return cuda_fail(c, e, "slot order");
  }
  if (ev->n_event > sl.cap || !sl.d_net_off) {
    if (sl.used) {
      e = cudaEventSynchronize(sl.free_ev);
      if (e != cudaSuccess) return cuda_fail(c, e, "sync");
    }
    if (sl.d_ev_t) cudaFree(sl.d_ev_t);
    if (sl.d_ev_v) cudaFree(sl.d_ev_v);
    sl.d_ev_t = nullptr;
    sl.d_ev_v = nullptr;
    const int64_t cap = std::max<int64_t>(ev->n_event, 16);
    e = cudaMalloc(&sl.d_ev_t, sizeof(int64_t) * cap);
    if (e == cudaSuccess) e = cudaMalloc(&sl.d_ev_v, sizeof(uint32_t) * ((cap + 15) / 16));
    if (e != cudaSuccess) {
      sl.cap = 0;
      c->err = std::string("event buffers: ") + cudaGetErrorString(e);
      return e == cudaErrorMemoryAllocation ? GTP_ENOMEM : GTP_ECUDA;
    }
    sl.cap = cap;
    if (!sl.d_net_off) {
      e = cudaMalloc(&sl.d_net_off, sizeof(int64_t) * (nn + 1));
      if (e == cudaSuccess) e = cudaMalloc(&sl.d_net_base, sizeof(int64_t) * std::max(1, nn));
      if (e != cudaSuccess) return cuda_fail(c, e, "net buffers");
    }
  }
  cudaStream_t cs = c->copy_stream;
  e = cudaMemcpyAsync(sl.d_net_off, ev->net_off, sizeof(int64_t) * (nn + 1), cudaMemcpyHostToDevice, cs);
  if (e == cudaSuccess && ev->n_event > 0)
    e = cudaMemcpyAsync(sl.d_ev_t, ev->time, sizeof(int64_t) * ev->n_event, cudaMemcpyHostToDevice, cs);
  if (e == cudaSuccess && ev->n_event > 0)
    e = cudaMemcpyAsync(sl.d_ev_v, ev->value_packed, sizeof(uint32_t) * ((ev->n_event + 15) / 16),
                        cudaMemcpyHostToDevice, cs);
  if (e == cudaSuccess && ev->net_base)
    e = cudaMemcpyAsync(sl.d_net_base, ev->net_base, sizeof(int64_t) * nn, cudaMemcpyHostToDevice, cs);
  if (e == cudaSuccess) e = cudaEventRecord(c->copied_ev, cs);
  // the caller's memory is no longer read once this returns; the walk of the
  // previous window keeps running meanwhile
  if (e == cudaSuccess) e = cudaEventSynchronize(c->copied_ev);
  if (e != cudaSuccess) return cuda_fail(c, e, "event copy");
  // the window walks on its slot's stream with its slot's scratch, after the
  // copy and after the work enqueued on the context's stream so far (a reset,
  // device-pushed windows); the separate kernels keep the context's stream
  cudaStream_t ws = c->stream;
  if (c->cfg.separate_kernels <= 0) {
    ws = c->walk_stream[s_idx];
    if (c->scratch_slot != s_idx) {
      if (!c->spare.ready) c->stream_dirty = true;  // ready_spare clears on the context's stream
      e = ready_spare(c);
      if (e != cudaSuccess) return cuda_fail(c, e, "walk scratch");
      swap_scratch(c);
    }
    // both walk streams follow the context's own work queued so far
    if (c->stream_dirty) {
      e = cudaEventRecord(c->stream_tail, c->stream);
      for (int k = 0; k < 2 && e == cudaSuccess; ++k) e = cudaStreamWaitEvent(c->walk_stream[k], c->stream_tail, 0);
      if (e != cudaSuccess) return cuda_fail(c, e, "walk order");
      c->stream_dirty = false;
    }
  }
  e = cudaStreamWaitEvent(ws, c->copied_ev, 0);
  if (e != cudaSuccess) return cuda_fail(c, e, "event copy");
  gtp_status st = run_window(c, sl.d_net_off, sl.d_ev_t, sl.d_ev_v, ev->net_base ? sl.d_net_base : nullptr,
                             ev->n_event, ev->t_lo, ev->t_hi, nullptr, ws);
  if (st != GTP_OK) return st;
  e = cudaEventRecord(sl.free_ev, ws);
  if (e == cudaSuccess && ws != c->stream) {
    e = cudaEventRecord(c->walk_done[s_idx], ws);
    c->walk_pending[s_idx] = true;
    // work queued on the context's stream from now on follows this walk
    if (e == cudaSuccess) e = cudaStreamWaitEvent(c->stream, c->walk_done[s_idx], 0);
  }
  if (e != cudaSuccess) return cuda_fail(c, e, "slot order");
  sl.used = true;
  c->next_slot ^= 1;
  return GTP_OK;
}

gtp_status gtp_push_events_device(gtp_ctx* c, const gtp_events* ev) {
  if (!c || !ev) return GTP_EINVAL;
  if (ev->n_event < 0 || !ev->net_off || (ev->n_event > 0 && (!ev->time || !ev->value_packed))) {
    c->err = "events: missing arrays";
    return GTP_EINVAL;
  }
  cudaError_t e = join_walks(c, c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "walk order");
  return run_window(c, ev->net_off, ev->time, ev->value_packed, ev->net_base, ev->n_event,
                    ev->t_lo, ev->t_hi);
}

gtp_status gtp_push_events_device_ranges(gtp_ctx* c, const gtp_events* ev, const int64_t* cycle_ranges,
                                         int32_t n_ranges) {
  if (!c || !ev) return GTP_EINVAL;
  if (ev->n_event < 0 || !ev->net_off || (ev->n_event > 0 && (!ev->time || !ev->value_packed)) || n_ranges < 0 ||
      (n_ranges > 0 && !cycle_ranges)) {
    c->err = "events or ranges: missing arrays";
    return GTP_EINVAL;
  }
  std::vector<int64_t> r(cycle_ranges, cycle_ranges + 2 * static_cast<size_t>(n_ranges));
  for (int32_t i = 0; i < n_ranges; ++i) {
    if (r[2 * i] < 0 || r[2 * i + 1] <= r[2 * i] || (i > 0 && r[2 * i] < r[2 * i - 1])) {
      c->err = "cycle ranges must be non-empty, ascending and disjoint";
      return GTP_EINVAL;
    }
  }
  if (n_ranges > 0 && (r[0] * c->P.tpc < ev->t_lo || (ev->t_hi < INT64_MAX / 2 && r.back() * c->P.tpc > ev->t_hi))) {
    c->err = "cycle ranges must lie within the window [t_lo, t_hi)";
    return GTP_EINVAL;
  }
  cudaError_t e = join_walks(c, c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "walk order");
  return run_window(c, ev->net_off, ev->time, ev->value_packed, ev->net_base, ev->n_event, ev->t_lo, ev->t_hi, &r);
}

gtp_status gtp_sync(gtp_ctx* c) {
  if (!c) return GTP_EINVAL;
  cudaError_t e = join_walks(c, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "sync");
  return check_status(c);
}

gtp_status gtp_finalize(gtp_ctx* c) {
  if (!c) return GTP_EINVAL;
  KParams k = make_params(c);
  cudaError_t e = join_walks(c, c->stream);
  if (e == cudaSuccess) e = launch_finalize(k, c->d_cell_group, c->d_cell5, c->d_cycle5, c->d_tg,
                                  c->d_leak_tmp, c->stream, c->d_cycle5_g, c->d_leak_tmp_g);
  if (e != cudaSuccess) return cuda_fail(c, e, "finalize");
  return GTP_OK;
}

void* gtp_get_stream(const gtp_ctx* c) { return c ? static_cast<void*>(c->stream) : nullptr; }

gtp_status gtp_set_stream(gtp_ctx* c, void* stream) {
  if (!c) return GTP_EINVAL;
  cudaError_t e = join_walks(c, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "sync");
  c->stream = stream ? static_cast<cudaStream_t>(stream) : c->own_stream;
  return GTP_OK;
}

gtp_status gtp_fetch(gtp_ctx* c, float* cell5, float* cycle5, double* totals, double* groups,
                     gtp_counts* counts) {
  if (!c) return GTP_EINVAL;
  gtp_status st = check_status(c);
  if (st != GTP_OK) return st;
  KParams k = make_params(c);
  cudaError_t e = launch_finalize(k, c->d_cell_group, c->d_cell5, c->d_cycle5, c->d_tg,
                                  c->d_leak_tmp, c->stream, c->d_cycle5_g, c->d_leak_tmp_g);
  if (e != cudaSuccess) return cuda_fail(c, e, "finalize");
  const Packed& P = c->P;
  const int64_t np = P.n_period;
  double tg[(GTP_N_GROUP + 1) * 5];
  if (cell5 && P.n_cell > 0)
    e = cudaMemcpyAsync(cell5, c->d_cell5, sizeof(float) * 5 * P.n_cell, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess && cycle5 && np > 0)
    e = cudaMemcpyAsync(cycle5, c->d_cycle5, sizeof(float) * 5 * np, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(tg, c->d_tg, sizeof(tg), cudaMemcpyDeviceToHost, c->stream);
  std::vector<unsigned long long> cyc_cnt;
  if (e == cudaSuccess && counts) {
    const int64_t nc = P.n_cell;
    uint32_t* dst[4] = {counts->cell_events, counts->cell_glitches, counts->cell_half_toggles,
                        counts->cell_related};
    for (int q = 0; q < 4 && e == cudaSuccess; ++q)
      if (dst[q] && nc > 0)
        e = cudaMemcpyAsync(dst[q], c->d_cnt_cell + q * nc, sizeof(uint32_t) * nc,
                            cudaMemcpyDeviceToHost, c->stream);
    cyc_cnt.resize(2 * (np + 1));
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(cyc_cnt.data(), c->d_cnt_cyc, sizeof(unsigned long long) * 2 * (np + 1),
                          cudaMemcpyDeviceToHost, c->stream);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "fetch");
  if (totals) std::memcpy(totals, tg, sizeof(double) * 5);
  if (groups) std::memcpy(groups, tg + 5, sizeof(double) * 5 * GTP_N_GROUP);
  if (counts) {
    for (int64_t y = 0; y < np; ++y) {
      if (counts->cycle_events) counts->cycle_events[y] = static_cast<int64_t>(cyc_cnt[y]);
      if (counts->cycle_glitches) counts->cycle_glitches[y] = static_cast<int64_t>(cyc_cnt[np + 1 + y]);
    }
    counts->dropped = static_cast<int64_t>(cyc_cnt[np] + cyc_cnt[np + 1 + np]);
  }
  return GTP_OK;
}

gtp_status gtp_set_cycle_groups(gtp_ctx* c, const int32_t* cell_group, int32_t n_group) {
  if (!c) return GTP_EINVAL;
  if (c->any_window) {
    c->err = "gtp_set_cycle_groups: call before the first window (or after gtp_reset)";
    return GTP_ESTATE;
  }
  const Packed& P = c->P;
  const int32_t nc = P.n_cell;
  if (n_group < 0 || n_group > kMaxCycleGroups || (n_group > 0 && !cell_group)) {
    c->err = "gtp_set_cycle_groups: n_group must be in [0, " + std::to_string(kMaxCycleGroups) + "]";
    return GTP_EINVAL;
  }
  for (int32_t i = 0; i < nc && n_group > 0; ++i)
    if (cell_group[i] < 0 || cell_group[i] >= n_group) {
      c->err = "gtp_set_cycle_groups: cell " + std::to_string(i) + " has group out of range";
      return GTP_EINVAL;
    }
  cudaError_t e = join_walks(c, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "sync");
  void* old[] = {c->d_cgroup, c->d_cyc_acc_g, c->d_cycle5_g, c->d_leak_tmp_g};
  for (void* q : old)
    if (q) cudaFree(q);
  c->d_cgroup = nullptr;
  c->d_cyc_acc_g = nullptr;
  c->d_cycle5_g = nullptr;
  c->d_leak_tmp_g = nullptr;
  c->n_cgroup = 0;
  // base walk order: by pin bucket, then (with groups) by group, then as packed
  std::vector<int32_t> order = P.order;
  if (n_group > 0) {
    for (int b = 0; b < 3; ++b)
      std::stable_sort(order.begin() + P.bucket_begin[b], order.begin() + P.bucket_begin[b + 1],
                       [&](int32_t x, int32_t y) { return cell_group[x] < cell_group[y]; });
  }
  if (!order.empty()) {
    e = cudaMemcpyAsync(c->d_order, order.data(), sizeof(int32_t) * order.size(), cudaMemcpyHostToDevice,
                        c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "walk order upload");
  }
  if (n_group == 0) return GTP_OK;
  const size_t ny = static_cast<size_t>(P.n_period + 1);
  const size_t np = static_cast<size_t>(std::max<int64_t>(1, P.n_period));
  e = cudaMalloc(&c->d_cgroup, sizeof(int32_t) * std::max<int32_t>(1, nc));
  if (e == cudaSuccess) e = cudaMalloc(&c->d_cyc_acc_g, sizeof(unsigned long long) * kNumCycAcc * ny * n_group);
  if (e == cudaSuccess) e = cudaMalloc(&c->d_cycle5_g, sizeof(float) * 5 * np * n_group);
  if (e == cudaSuccess) e = cudaMalloc(&c->d_leak_tmp_g, sizeof(unsigned long long) * np * n_group);
  if (e == cudaSuccess && nc > 0)
    e = cudaMemcpyAsync(c->d_cgroup, cell_group, sizeof(int32_t) * nc, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(c->d_cyc_acc_g, 0, sizeof(unsigned long long) * kNumCycAcc * ny * n_group, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) {
    void* fr[] = {c->d_cgroup, c->d_cyc_acc_g, c->d_cycle5_g, c->d_leak_tmp_g};
    for (void* q : fr)
      if (q) cudaFree(q);
    c->d_cgroup = nullptr;
    c->d_cyc_acc_g = nullptr;
    c->d_cycle5_g = nullptr;
    c->d_leak_tmp_g = nullptr;
    return e == cudaErrorMemoryAllocation ? GTP_ENOMEM : cuda_fail(c, e, "cycle groups");
  }
  c->n_cgroup = n_group;
  return GTP_OK;
}

int32_t gtp_n_cycle_groups(const gtp_ctx* c) { return c ? c->n_cgroup : 0; }

gtp_status gtp_set_cell_range(gtp_ctx* c, int32_t cell_begin, int32_t cell_end) {
  if (!c) return GTP_EINVAL;
  Packed& P = c->P;
  if (c->any_window || c->n_cgroup > 0) {
    c->err = "gtp_set_cell_range: call before the first window (or after gtp_reset) and before "
             "gtp_set_cycle_groups";
    return GTP_ESTATE;
  }
  if (cell_begin < 0 || cell_end < cell_begin || cell_end > P.n_cell) {
    c->err = "gtp_set_cell_range: need 0 <= cell_begin <= cell_end <= n_cell";
    return GTP_EINVAL;
  }
  // the whole design's walk order, keeping the cells of the range (bucket
  // grouping and type order stay as packed)
  std::vector<int32_t> order;
  order.reserve(static_cast<size_t>(cell_end - cell_begin));
  int32_t bb[4] = {0, 0, 0, 0};
  for (int b = 0; b < 3; ++b) {
    bb[b] = static_cast<int32_t>(order.size());
    for (int32_t i = P.bucket_all[b]; i < P.bucket_all[b + 1]; ++i)
      if (P.order_all[i] >= cell_begin && P.order_all[i] < cell_end) order.push_back(P.order_all[i]);
  }
  bb[3] = static_cast<int32_t>(order.size());
  cudaError_t e = join_walks(c, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e == cudaSuccess && !order.empty())
    e = cudaMemcpyAsync(c->d_order, order.data(), sizeof(int32_t) * order.size(), cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "gtp_set_cell_range");
  P.order.swap(order);
  for (int b = 0; b < 4; ++b) P.bucket_begin[b] = bb[b];
  return GTP_OK;
}

int64_t gtp_accumulator_bytes(const gtp_ctx* c) {
  if (!c) return -1;
  const int64_t nc = c->P.n_cell, ny = c->P.n_period + 1;
  int64_t b = 8 * kNumCellAcc * nc + 8 * kNumCycAcc * ny;
  if (c->cfg.collect_counts) b += 8 * 2 * ny + 4 * 4 * nc;
  return b;
}

// Accumulator block layout (gtp_accumulator_bytes): FP64 cell sums
// [5][n_cell] | int64 per-cycle fixed-point bins [6][n_period+1] | with
// collect_counts: uint64 per-cycle counts [2][n_period+1] | uint32 per-cell
// counts [4][n_cell].
namespace {
gtp_status copy_accumulators(gtp_ctx* c, void* dst, const void* src, bool out) {
  if (!c || !dst || !src) return GTP_EINVAL;
  const size_t nc = static_cast<size_t>(c->P.n_cell), ny = static_cast<size_t>(c->P.n_period + 1);
  cudaError_t ej = join_walks(c, c->stream);
  if (ej != cudaSuccess) return cuda_fail(c, ej, "walk order");
  struct Seg {
    void* dev;
    size_t bytes;
  } segs[4] = {{c->d_cell_acc, 8 * kNumCellAcc * nc},
               {c->d_cyc_acc, 8 * kNumCycAcc * ny},
               {c->d_cnt_cyc, c->cfg.collect_counts ? 8 * 2 * ny : 0},
               {c->d_cnt_cell, c->cfg.collect_counts ? 4 * 4 * nc : 0}};
  size_t off = 0;
  for (const Seg& sg : segs) {
    if (sg.bytes == 0) continue;
    cudaError_t e =
        out ? cudaMemcpyAsync(static_cast<char*>(dst) + off, sg.dev, sg.bytes, cudaMemcpyDeviceToDevice, c->stream)
            : cudaMemcpyAsync(sg.dev, static_cast<const char*>(src) + off, sg.bytes, cudaMemcpyDeviceToDevice,
                              c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, out ? "gtp_export_accumulators" : "gtp_import_accumulators");
    off += sg.bytes;
  }
  return GTP_OK;
}
}  // namespace

gtp_status gtp_export_accumulators(gtp_ctx* c, void* d_out) {
  return copy_accumulators(c, d_out, c ? c->d_cell_acc : nullptr, true);
}

gtp_status gtp_import_accumulators(gtp_ctx* c, const void* d_in) {
  gtp_status st = copy_accumulators(c, c ? c->d_cell_acc : nullptr, d_in, false);
  if (st == GTP_OK) c->any_window = true;
  return st;
}

gtp_status gtp_clock_run_nets(gtp_ctx* c, int32_t* n_clock_nets, int32_t* n_periodic) {
  if (!c || !n_clock_nets || !n_periodic) return GTP_EINVAL;
  *n_clock_nets = c->n_clk_nets;
  *n_periodic = 0;
  if (c->n_clk_nets == 0 || !c->d_pclk) return GTP_OK;
  std::vector<int2> tab(static_cast<size_t>(c->P.n_net));
  cudaError_t e = join_walks(c, c->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(tab.data(), c->d_pclk, sizeof(int2) * tab.size(), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "gtp_clock_run_nets");
  int32_t n = 0;
  for (int32_t net : c->clk_nets)
    if (tab[static_cast<size_t>(net)].x >= 0) ++n;
  *n_periodic = n;
  return GTP_OK;
}

gtp_status gtp_walk_items(gtp_ctx* c, int64_t* items) {
  if (!c || !items) return GTP_EINVAL;
  *items = 0;
  const int32_t n_order = c->P.bucket_begin[3];
  if (!c->d_item_off || n_order <= 0 || !c->any_window) return GTP_OK;
  int32_t n = 0;
  cudaError_t e = join_walks(c, c->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&n, c->d_item_off + n_order, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "walk items");
  *items = n;
  return GTP_OK;
}

gtp_status gtp_fetch_cycle_groups(gtp_ctx* c, float* cycle5_groups) {
  if (!c || !cycle5_groups) return GTP_EINVAL;
  if (c->n_cgroup <= 0) {
    c->err = "gtp_fetch_cycle_groups: no cycle groups set";
    return GTP_ESTATE;
  }
  gtp_status st = check_status(c);
  if (st != GTP_OK) return st;
  KParams k = make_params(c);
  cudaError_t e = launch_finalize(k, c->d_cell_group, c->d_cell5, c->d_cycle5, c->d_tg, c->d_leak_tmp,
                                  c->stream, c->d_cycle5_g, c->d_leak_tmp_g);
  const int64_t np = c->P.n_period;
  if (e == cudaSuccess && np > 0)
    e = cudaMemcpyAsync(cycle5_groups, c->d_cycle5_g, sizeof(float) * 5 * np * c->n_cgroup,
                        cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "fetch cycle groups");
  return GTP_OK;
}

}  // extern "C"

// ---- batched evaluation: many contexts' windows in one persistent launch ----

struct gtp_batch {
  std::vector<gtp_ctx*> ctxs;
  gtp_batch_config cfg{};
  int device = 0;
  int sm_count = 148;
  int threads = 256;
  bool counts = false;
  cudaStream_t stream = nullptr;
  std::string err;
  // device and pinned staging copies of the walk parameters and work items
  KParams* d_params = nullptr;
  KParams* h_params = nullptr;
  int params_cap = 0;
  int4* d_items = nullptr;
  int4* h_items = nullptr;
  int64_t items_cap = 0;
  int* d_meta = nullptr;  // per launch group g: [2g] item count, [2g+1] queue head
  int* h_meta = nullptr;
  cudaEvent_t ev = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  std::vector<uint64_t> graph_key;
  int64_t last_items = 0;
  int last_launches = 0;
  int graph_replays = 0;
};

namespace {

constexpr int kBatchGroups = 6;  // pin bucket x drift

void set_create_err(const std::string& m) {
  std::lock_guard<std::mutex> g(g_err_mu);
  g_create_err = m;
}

gtp_status batch_fail(gtp_batch* b, gtp_status st, const std::string& m) {
  b->err = m;
  return st;
}

void batch_release(gtp_batch* b) {
  if (b->gexec) cudaGraphExecDestroy(b->gexec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->gexec = nullptr;
  b->graph = nullptr;
  if (b->d_params) cudaFree(b->d_params);
  if (b->h_params) cudaFreeHost(b->h_params);
  if (b->d_items) cudaFree(b->d_items);
  if (b->h_items) cudaFreeHost(b->h_items);
  if (b->d_meta) cudaFree(b->d_meta);
  if (b->h_meta) cudaFreeHost(b->h_meta);
  if (b->ev) cudaEventDestroy(b->ev);
  if (b->stream) cudaStreamDestroy(b->stream);
}

struct BatchEntry {
  int ctx;
  int group;     // bucket * 2 + drift
  int n_gblk;
  int n_tiles;
  int64_t ct;
  int64_t cycles;  // cycles of the window
  double density;  // events per net and cycle of the window
  int32_t cells;   // cells of the bucket
  int32_t gpb;
};

}  // namespace

extern "C" {

void gtp_batch_config_default(gtp_batch_config* cfg) {
  if (!cfg) return;
  std::memset(cfg, 0, sizeof(*cfg));
  cfg->use_graph = 1;
  cfg->blocks_per_sm = 0;
}

gtp_status gtp_batch_create(gtp_ctx* const* ctxs, int32_t n_ctx, const gtp_batch_config* cfg, gtp_batch** out) {
  if (!ctxs || !out || n_ctx < 1) return GTP_EINVAL;
  *out = nullptr;
  gtp_batch_config def;
  gtp_batch_config_default(&def);
  const gtp_batch_config& C = cfg ? *cfg : def;
  int dev = -1, thr = -1, cnt = -1;
  for (int i = 0; i < n_ctx; ++i) {
    gtp_ctx* c = ctxs[i];
    if (!c) return GTP_EINVAL;
    if (c->cfg.separate_kernels > 0) {
      set_create_err("gtp_batch_create: the batched walk is the fused one; contexts with separate_kernels are "
                     "evaluated one window at a time");
      return GTP_EINVAL;
    }
    const int t = c->cfg.n_thread_per_block > 0 ? c->cfg.n_thread_per_block : 256;
    const int k = c->cfg.collect_counts ? 1 : 0;
    if (i == 0) {
      dev = c->device;
      thr = t;
      cnt = k;
    } else if (c->device != dev || t != thr || k != cnt) {
      set_create_err("gtp_batch_create: contexts must share the device, n_thread_per_block and collect_counts");
      return GTP_EINVAL;
    }
  }
  gtp_batch* b = new gtp_batch();
  b->ctxs.assign(ctxs, ctxs + n_ctx);
  b->cfg = C;
  b->device = dev;
  b->threads = thr;
  b->counts = cnt != 0;
  cudaError_t e = cudaSetDevice(dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&b->sm_count, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaMalloc(&b->d_meta, sizeof(int) * 2 * kBatchGroups);
  if (e == cudaSuccess) e = cudaMallocHost(&b->h_meta, sizeof(int) * 2 * kBatchGroups);
  if (e != cudaSuccess) {
    set_create_err(std::string("gtp_batch_create: ") + cudaGetErrorString(e));
    batch_release(b);
    delete b;
    return GTP_ECUDA;
  }
  *out = b;
  return GTP_OK;
}

void gtp_batch_destroy(gtp_batch* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  batch_release(b);
  delete b;
}

const char* gtp_batch_last_error(const gtp_batch* b) { return b ? b->err.c_str() : "null batch"; }

gtp_status gtp_batch_push_device(gtp_batch* b, const gtp_events* d_ev) {
  if (!b || !d_ev) return GTP_EINVAL;
  cudaError_t e = cudaSetDevice(b->device);
  if (e != cudaSuccess) return batch_fail(b, GTP_ECUDA, cudaGetErrorString(e));
  // staging buffers of the previous push must be consumed
  e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return batch_fail(b, GTP_ECUDA, std::string("sync: ") + cudaGetErrorString(e));
  const int n = static_cast<int>(b->ctxs.size());
  std::vector<KParams> params;
  std::vector<BatchEntry> entries;
  std::vector<int> active;
  std::vector<KParams> kwin(n);
  std::vector<int> first_entry(n, -1);
  static const int bucket_pins[3] = {4, 8, kMaxPins};
  for (int i = 0; i < n; ++i) {
    const gtp_events& ev = d_ev[i];
    if (ev.net_off == nullptr) continue;
    gtp_ctx* c = b->ctxs[i];
    if (ev.n_event < 0 || (ev.n_event > 0 && (!ev.time || !ev.value_packed)))
      return batch_fail(b, GTP_EINVAL, "context " + std::to_string(i) + ": malformed events");
    // the context's host-pushed walks, if any, before its scratch is reused
    e = join_walks(c, b->stream);
    if (e != cudaSuccess) return batch_fail(b, GTP_ECUDA, std::string("walk order: ") + cudaGetErrorString(e));
    gtp_status st = prepare_window(c, ev.net_off, ev.time, ev.value_packed, ev.net_base, ev.n_event, ev.t_lo,
                                   ev.t_hi, b->stream, &kwin[i], false);
    if (st != GTP_OK) return batch_fail(b, st, "context " + std::to_string(i) + ": " + c->err);
    active.push_back(i);
    const KParams& k = kwin[i];
    const Packed& P = c->P;
    const int64_t cyc = static_cast<int64_t>(k.n_tiles) * k.cycles_per_tile;
    const double dens = static_cast<double>(ev.n_event) / (std::max<double>(1.0, P.n_net) * std::max<int64_t>(1, cyc));
    for (int bk = 0; bk < 3; ++bk) {
      const int32_t lo = P.bucket_begin[bk], hi = P.bucket_begin[bk + 1];
      if (hi <= lo) continue;
      if (first_entry[i] < 0) first_entry[i] = static_cast<int>(params.size());
      KParams kp = k;
      kp.order_begin = lo;
      kp.order_end = hi;
      BatchEntry be;
      be.ctx = i;
      be.group = bk * 2 + (k.drift ? 1 : 0);
      be.n_gblk = (hi - lo + k.gates_per_block - 1) / k.gates_per_block;
      be.n_tiles = k.n_tiles;
      be.ct = k.cycles_per_tile;
      be.cycles = cyc;
      be.density = dens;
      be.cells = hi - lo;
      be.gpb = k.gates_per_block;
      params.push_back(kp);
      entries.push_back(be);
    }
  }
  if (active.empty()) return GTP_OK;
  // work items per launch group, heaviest first
  struct Item { double w; int4 v; };
  std::vector<std::vector<Item>> groups(kBatchGroups);
  size_t smem_g[kBatchGroups] = {0, 0, 0, 0, 0, 0};
  bool runs_g[kBatchGroups] = {false, false, false, false, false, false};
  for (size_t q = 0; q < entries.size(); ++q) {
    const BatchEntry& be = entries[q];
    const int bk = be.group / 2;
    if (bk == 0 && !(be.group & 1) && params[q].pclk) runs_g[be.group] = true;
    smem_g[be.group] = std::max(smem_g[be.group], walk_item_smem_bytes(params[q], bucket_pins[bk], b->counts, b->threads));
    for (int g = 0; g < be.n_gblk; ++g) {
      const int32_t cells = std::min<int32_t>(be.gpb, be.cells - g * be.gpb);
      for (int t = 0; t < be.n_tiles; ++t) {
        const int64_t cyc = std::min<int64_t>(be.ct, be.cycles - t * be.ct);
        groups[be.group].push_back(Item{cells * static_cast<double>(cyc) * (be.density + 1e-3),
                                        make_int4(static_cast<int>(q), g, t, 0)});
      }
    }
  }
  int64_t n_items = 0;
  for (auto& g : groups) {
    std::stable_sort(g.begin(), g.end(), [](const Item& x, const Item& y) { return x.w > y.w; });
    n_items += static_cast<int64_t>(g.size());
  }
  if (n_items > INT32_MAX) return batch_fail(b, GTP_EOVERFLOW, "too many work items");
  // staging (grown as needed; a capacity change invalidates the graph)
  bool realloc = false;
  if (static_cast<int>(params.size()) > b->params_cap) {
    if (b->d_params) cudaFree(b->d_params);
    if (b->h_params) cudaFreeHost(b->h_params);
    b->params_cap = static_cast<int>(params.size()) * 2;
    e = cudaMalloc(&b->d_params, sizeof(KParams) * b->params_cap);
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_params, sizeof(KParams) * b->params_cap);
    realloc = true;
  }
  if (e == cudaSuccess && n_items > b->items_cap) {
    if (b->d_items) cudaFree(b->d_items);
    if (b->h_items) cudaFreeHost(b->h_items);
    b->items_cap = n_items * 2;
    e = cudaMalloc(&b->d_items, sizeof(int4) * b->items_cap);
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_items, sizeof(int4) * b->items_cap);
    realloc = true;
  }
  if (e != cudaSuccess) return batch_fail(b, GTP_ENOMEM, std::string("staging: ") + cudaGetErrorString(e));
  std::memcpy(b->h_params, params.data(), sizeof(KParams) * params.size());
  int64_t off = 0;
  int64_t group_off[kBatchGroups];
  for (int g = 0; g < kBatchGroups; ++g) {
    group_off[g] = off;
    for (const Item& it : groups[g]) b->h_items[off++] = it.v;
    b->h_meta[2 * g] = static_cast<int>(groups[g].size());
    b->h_meta[2 * g + 1] = 0;
  }
  // order against earlier work on the contexts' streams
  for (int i : active) {
    e = cudaEventRecord(b->ev, b->ctxs[i]->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(b->stream, b->ev, 0);
    if (e != cudaSuccess) return batch_fail(b, GTP_ECUDA, std::string("stream order: ") + cudaGetErrorString(e));
  }
  e = cudaMemcpyAsync(b->d_params, b->h_params, sizeof(KParams) * params.size(), cudaMemcpyHostToDevice, b->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b->d_items, b->h_items, sizeof(int4) * std::max<int64_t>(1, n_items), cudaMemcpyHostToDevice,
                        b->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b->d_meta, b->h_meta, sizeof(int) * 2 * kBatchGroups, cudaMemcpyHostToDevice, b->stream);
  if (e != cudaSuccess) return batch_fail(b, GTP_ECUDA, std::string("upload: ") + cudaGetErrorString(e));
  // the launch sequence: work sorts of every window, then one persistent
  // walk per launch group. Its shape (contexts, buffers, grid, shared
  // memory) keys the captured graph.
  std::vector<uint64_t> key;
  key.push_back(realloc ? 1u : 0u);
  key.push_back(reinterpret_cast<uint64_t>(b->d_params));
  for (int i : active) {
    key.push_back(static_cast<uint64_t>(i));
    key.push_back(reinterpret_cast<uint64_t>(kwin[i].net_off));
    key.push_back(reinterpret_cast<uint64_t>(kwin[i].tile_first));
    key.push_back(reinterpret_cast<uint64_t>(kwin[i].glitch_pw));
    key.push_back(static_cast<uint64_t>(first_entry[i]));
  }
  // clock-run launches keep the threads' per-cell sums ahead of each item's bins
  for (int g = 0; g < kBatchGroups; ++g)
    if (runs_g[g]) smem_g[g] += walk_runs_acc_bytes(b->threads);
  int grid_g[kBatchGroups];
  for (int g = 0; g < kBatchGroups; ++g) {
    grid_g[g] = 0;
    if (groups[g].empty()) continue;
    const int bk = g / 2;
    const int per_sm = b->cfg.blocks_per_sm > 0
                           ? b->cfg.blocks_per_sm
                           : walk_blocks_per_sm(bucket_pins[bk], b->counts, (g & 1) != 0, runs_g[g], b->threads,
                                                smem_g[g]);
    grid_g[g] = static_cast<int>(std::min<int64_t>(static_cast<int64_t>(b->sm_count) * per_sm,
                                                   static_cast<int64_t>(groups[g].size())));
    key.push_back(static_cast<uint64_t>(g) << 56 | static_cast<uint64_t>(grid_g[g]) << 24 | smem_g[g]);
  }
  auto enqueue = [&]() -> cudaError_t {
    cudaError_t r = cudaSuccess;
    for (int i : active) {
      const KParams* dk = first_entry[i] >= 0 ? b->d_params + first_entry[i] : nullptr;
      r = enqueue_window_prep(b->ctxs[i], kwin[i], dk, b->stream);
      if (r != cudaSuccess) return r;
    }
    for (int g = 0; g < kBatchGroups; ++g) {
      if (!grid_g[g]) continue;
      r = launch_power_walk_batch(b->d_params, b->d_items + group_off[g], b->d_meta + 2 * g, b->d_meta + 2 * g + 1,
                                  grid_g[g], bucket_pins[g / 2], b->counts, (g & 1) != 0, runs_g[g], b->threads,
                                  smem_g[g], b->stream);
      if (r != cudaSuccess) return r;
    }
    return r;
  };
  int launches = 0;
  for (int g = 0; g < kBatchGroups; ++g) launches += grid_g[g] ? 1 : 0;
  if (b->cfg.use_graph) {
    if (!b->gexec || key != b->graph_key) {
      if (b->gexec) cudaGraphExecDestroy(b->gexec);
      if (b->graph) cudaGraphDestroy(b->graph);
      b->gexec = nullptr;
      b->graph = nullptr;
      e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess) {
        cudaError_t r = enqueue();
        cudaGraph_t gr = nullptr;
        e = cudaStreamEndCapture(b->stream, &gr);
        if (r != cudaSuccess) e = r;
        if (e == cudaSuccess) e = cudaGraphInstantiate(&b->gexec, gr, 0);
        if (e == cudaSuccess) {
          b->graph = gr;
          b->graph_key = key;
        } else if (gr) {
          cudaGraphDestroy(gr);
        }
      }
    } else {
      ++b->graph_replays;
    }
    if (e == cudaSuccess) e = cudaGraphLaunch(b->gexec, b->stream);
  } else {
    e = enqueue();
  }
  if (e != cudaSuccess) return batch_fail(b, GTP_ECUDA, std::string("batched walk: ") + cudaGetErrorString(e));
  // later work on each context waits for the batch
  e = cudaEventRecord(b->ev, b->stream);
  for (int i : active) {
    if (e == cudaSuccess) e = cudaStreamWaitEvent(b->ctxs[i]->stream, b->ev, 0);
    commit_window(b->ctxs[i], d_ev[i].t_hi);
  }
  if (e != cudaSuccess) return batch_fail(b, GTP_ECUDA, std::string("stream order: ") + cudaGetErrorString(e));
  b->last_items = n_items;
  b->last_launches = launches;
  return GTP_OK;
}

gtp_status gtp_batch_sync(gtp_batch* b) {
  if (!b) return GTP_EINVAL;
  cudaError_t e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return batch_fail(b, GTP_ECUDA, std::string("sync: ") + cudaGetErrorString(e));
  for (size_t i = 0; i < b->ctxs.size(); ++i) {
    gtp_status st = check_status(b->ctxs[i]);
    if (st != GTP_OK) return batch_fail(b, st, "context " + std::to_string(i) + ": " + b->ctxs[i]->err);
  }
  return GTP_OK;
}

void* gtp_batch_get_stream(const gtp_batch* b) { return b ? static_cast<void*>(b->stream) : nullptr; }

gtp_status gtp_batch_stats(const gtp_batch* b, int64_t* items, int32_t* launches, int32_t* graph_replays) {
  if (!b) return GTP_EINVAL;
  if (items) *items = b->last_items;
  if (launches) *launches = b->last_launches;
  if (graph_replays) *graph_replays = b->graph_replays;
  return GTP_OK;
}

void gtp_pack_values(const uint8_t* values, int64_t n, uint32_t* packed) {
  const int64_t nw = (n + 15) / 16;
  for (int64_t w = 0; w < nw; ++w) {
    uint32_t x = 0;
    const int64_t b = w * 16;
    const int64_t m = std::min<int64_t>(16, n - b);
    for (int64_t j = 0; j < m; ++j) x |= static_cast<uint32_t>(values[b + j] & 3) << (2 * j);
    packed[w] = x;
  }
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free evaluation.
//
// Some callers cannot allocate device memory while they run: an EDA host
// that embeds this engine under its own device-memory arena (reserved once at
// start-up and shared with timing analysis), or a service whose latency
// budget cannot absorb the device-wide synchronization cudaMalloc/cudaFree
// can cause. For them gtp_evaluate_noalloc evaluates a whole trace with its
// accumulators in the fixed static device array below instead of memory the
// context allocates, and writes the results into device buffers the caller
// provides. It calls no cudaMalloc, cudaFree or other allocating routine.
//
// The array is 16 MiB; every GPU that loads this library holds it until the
// process exits. All calls share it and it keeps the last call's contents:
// each call clears the part it uses before the walk, and two calls that
// overlap on the GPU (different streams or contexts on one device) race.
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kNoAllocMaxDevices] = {nullptr};

// Device address of the static array on the current device, looked up once
// per device with that device current.
cudaError_t noalloc_scratch(int dev, unsigned char** out) {
  if (dev < 0 || dev >= kNoAllocMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> g(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_noalloc_ptr[dev] = p;
  }
  *out = static_cast<unsigned char*>(g_noalloc_ptr[dev]);
  return cudaSuccess;
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace

extern "C" gtp_status gtp_evaluate_noalloc(gtp_ctx* c, const gtp_events* ev, float* d_cell5,
                                           float* d_cycle5, double* d_totals) {
  if (!c || !ev) return GTP_EINVAL;
  if (ev->n_event < 0 || !ev->net_off || (ev->n_event > 0 && (!ev->time || !ev->value_packed))) {
    c->err = "noalloc: missing event arrays";
    return GTP_EINVAL;
  }
  if (ev->t_lo != 0 || ev->t_hi <= 0) {
    c->err = "noalloc: evaluates a whole trace; t_lo must be 0 and t_hi > 0";
    return GTP_EINVAL;
  }
  if (c->cfg.separate_kernels > 0) {
    c->err = "noalloc: the fused walk only; the separate kernels need per-window scratch";
    return GTP_EINVAL;
  }
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(c, e, "noalloc: cudaGetDevice");
  if (dev != c->device) {
    c->err = "noalloc: the context's device must be current";
    return GTP_EINVAL;
  }
  const Packed& P = c->P;
  const size_t nc = static_cast<size_t>(std::max<int32_t>(1, P.n_cell));
  const size_t ny = static_cast<size_t>(P.n_period + 1);
  // layout: cell_acc | cyc_acc | tg | leak_tmp
  const size_t off_cell = 0;
  const size_t off_cyc = align256(off_cell + sizeof(double) * kNumCellAcc * nc);
  const size_t off_tg = align256(off_cyc + sizeof(unsigned long long) * kNumCycAcc * ny);
  const size_t off_tmp = align256(off_tg + sizeof(double) * (GTP_N_GROUP + 1) * 5);
  const size_t need = align256(off_tmp + sizeof(unsigned long long) * ny);
  if (need > kNoAllocScratchBytes) {
    c->err = "noalloc: design needs " + std::to_string(need) + " bytes of scratch (40 per cell + 56 per "
             "cycle); the static array holds " + std::to_string(kNoAllocScratchBytes);
    return GTP_EOVERFLOW;
  }
  unsigned char* s = nullptr;
  e = noalloc_scratch(dev, &s);
  if (e != cudaSuccess) return cuda_fail(c, e, "noalloc: cudaGetSymbolAddress");

  // after the context's host-pushed walks, if any (they share its status word)
  e = join_walks(c, c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "noalloc: walk order");
  // accumulators must start at zero
  e = cudaMemsetAsync(s, 0, off_tg, c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "noalloc: clear");
  // the context's status word reports this call's events only (a 4-byte
  // memset of memory the context already holds, not an allocation)
  e = cudaMemsetAsync(c->d_status, 0, sizeof(int32_t), c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "noalloc: status clear");

  KParams k = make_params(c);
  k.cell_acc = reinterpret_cast<double*>(s + off_cell);
  k.cyc_acc = reinterpret_cast<unsigned long long*>(s + off_cyc);
  k.cnt_cell = nullptr;
  k.cnt_cyc = nullptr;
  k.cell_cgroup = nullptr;  // no per-group waveforms on this path
  k.cyc_acc_g = nullptr;
  k.n_cgroup = 0;
  k.net_off = ev->net_off;
  k.ev_t = ev->time;
  k.ev_v = ev->value_packed;
  k.net_base = ev->net_base;
  k.n_event = ev->n_event;
  k.t_lo = 0;
  k.t_hi = ev->t_hi;
  const int64_t last_tick = std::min<int64_t>(ev->t_hi - 1, P.tmax);
  k.cyc0 = 0;
  const int64_t n_cyc = std::max<int64_t>(1, last_tick / P.tpc + 1);
  int64_t ct = c->cfg.cycles_per_tile > 0 ? c->cfg.cycles_per_tile : 512;
  ct = std::min<int64_t>(ct, n_cyc);
  const int64_t max_ct = std::min<int64_t>(
      max_cycles_per_tile(c->cfg.n_thread_per_block > 0 ? c->cfg.n_thread_per_block : 256, 1),
      (int64_t(INT32_MAX) / P.tpc) - 1);
  ct = std::min<int64_t>(ct, max_ct);
  ct = std::max<int64_t>(ct, (n_cyc + 65534) / 65535);
  if (ct > max_ct || ct < 1) { c->err = "noalloc: trace spans too many cycles for one launch"; return GTP_EOVERFLOW; }
  k.cycles_per_tile = ct;
  k.n_tiles = static_cast<int32_t>((n_cyc + ct - 1) / ct);
  const int threads = c->cfg.n_thread_per_block > 0 ? c->cfg.n_thread_per_block : 256;
  k.gates_per_block = c->cfg.gates_per_block > 0 ? c->cfg.gates_per_block : threads * 4;
  static const int bucket_pins[3] = {4, 8, kMaxPins};
  for (int b = 0; b < 3; ++b) {
    k.order_begin = P.bucket_begin[b];
    k.order_end = P.bucket_begin[b + 1];
    if (k.order_end <= k.order_begin) continue;
    e = launch_power_walk(k, bucket_pins[b], false, threads, c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "noalloc: power walk launch");
  }
  double* tg = reinterpret_cast<double*>(s + off_tg);
  e = launch_finalize(k, c->d_cell_group, d_cell5, d_cycle5, tg,
                      reinterpret_cast<unsigned long long*>(s + off_tmp), c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "noalloc: finalize");
  if (d_totals) {
    e = cudaMemcpyAsync(d_totals, tg, sizeof(double) * 5, cudaMemcpyDeviceToDevice, c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "noalloc: totals");
  }
  return GTP_OK;
}
