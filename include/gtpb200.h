/*
 * gtpb200.h — C ABI of the B200 time-based power engine.
 *
 * This is the drop-in boundary for GTPower's time-based power path. The
 * reference exposes that path as the C++ virtual interface
 *
 *   gtpower::Power::power(corner, total, sequential, combinational,
 *                         clock, macro, pad)          power/Power.hh:80-87
 *   gtpower::Power::printCellRes()                    power/Power.hh:109
 *
 * implemented on the CPU by Power::power (power/Power.cc:227-386) and
 * findTimeBasedAllPower (power/TimeBasedPower.cc:703-901), and on CUDA by
 * CudaPower::power (power/cuda/CudaPower.cu:1227-1337). Waveforms reach it
 * through Power::setUserActivity(pin, ..., const VcdValues*, value_bit)
 * (power/Power.cc:138-147).
 *
 * The ABI below carries the same information as plain arrays:
 *   - gtp_design: what CudaPower::initGateData gathers from OpenSTA per pin
 *     and per cell (power/cuda/CudaPower.cu:1601-1816): slews, load caps,
 *     voltages, default states, clock flags, arc delays, and the Liberty
 *     internal_power / leakage_power groups of every cell type;
 *   - gtp_events: the per-net event list (tick, value) that the reference
 *     keeps as VcdValues per var/bit (power/Vcd.hh, power/Vcd.cc:204-277),
 *     as a CSR over nets;
 *   - gtp_fetch: per-cell values (the rows of cuda_cell_power.txt,
 *     power/cuda/CudaPower.cu:3134-3165), per-cycle waveforms (the sections
 *     of cuda_per_cycle_waveform.txt, include/sta/PowerClass.hh:123-149) and
 *     the report_power group totals (power/Power.cc:330-347).
 *
 * All pointers are host pointers unless the name starts with d_. No call
 * keeps a pointer to caller memory after it returns. One context per host
 * thread; a context owns its CUDA streams and device memory.
 */
#ifndef GTPB200_H
#define GTPB200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. GTP_OK and GTP_GENERAL_ERROR keep the values of the
 * reference's ErrorCode (OK=0, GENERAL_ERROR=-1); the reference itself exits
 * the process on errors (util/Log.hh:58-60, util/cuda/CheckCudaRuntime.cu). */
typedef int32_t gtp_status;
#define GTP_OK             0
#define GTP_GENERAL_ERROR (-1)
#define GTP_EINVAL        (-2)   /* malformed design or events            */
#define GTP_ENOMEM        (-3)   /* host or device allocation failed       */
#define GTP_ECUDA         (-4)   /* CUDA runtime error                     */
#define GTP_ETIMEOUT      (-5)   /* a bounded device wait gave up          */
#define GTP_EOVERFLOW     (-6)   /* a size exceeds a documented limit      */
#define GTP_ESTATE        (-7)   /* calls made in the wrong order          */

/* Pin values, as Power::vcd_value_to_int_map_ (power/Power.hh:114). */
#define GTP_V0 0
#define GTP_V1 1
#define GTP_VX 2
#define GTP_VZ 3

/* Report groups, as Power::power classifies instances
 * (power/Power.cc:338-347: macro, pad, clock network, sequential, else
 * combinational). */
#define GTP_GROUP_COMBINATIONAL 0
#define GTP_GROUP_SEQUENTIAL    1
#define GTP_GROUP_CLOCK         2
#define GTP_GROUP_MACRO         3
#define GTP_GROUP_PAD           4
#define GTP_N_GROUP             5

/* Table axis variables (liberty/InternalPower.cc:215-228). */
#define GTP_AXIS_NONE 0
#define GTP_AXIS_SLEW 1   /* input_transition_time          */
#define GTP_AXIS_CAP  2   /* total_output_net_capacitance   */

/* One NLDM power table (rise_power or fall_power of an internal_power
 * group): liberty/TableModel.cc Table0/Table1/Table2. Values are SI (J);
 * axes are SI (s, F). values are row-major [n1][n2]. */
typedef struct gtp_table {
  int32_t order;          /* 0, 1 or 2 */
  int32_t axis1_var;      /* GTP_AXIS_* */
  int32_t axis2_var;
  int32_t n1, n2;         /* axis sizes (1 for unused axes) */
  int64_t axis1_off;      /* offsets into gtp_design.lut_pool */
  int64_t axis2_off;
  int64_t value_off;
  float   scale;          /* TableModel::scaleFactor (1.0 if none) */
  int32_t reserved;
} gtp_table;

/* A `when` condition in disjunctive normal form over the cell's pins: it
 * holds when, for some cube k, (ones & care[k]) == value[k], where bit i of
 * `ones` is set iff pin i is in state 1 (X and Z count as not-one, as
 * evalWhen does in power/PowerUtils.cc:153-186). A group without `when`
 * is one cube with care = 0. Zero cubes = never true. */
typedef struct gtp_when {
  int32_t cube_off;       /* into gtp_design.when_cubes (pairs care,value) */
  int32_t n_cube;
} gtp_when;

/* A Liberty internal_power group of one cell type, in Liberty order
 * (LibertyCell::internalPowers; used by findInputInternalVal and
 * findOutputInternalVal, power/TimeBasedPower.cc:341-509). */
typedef struct gtp_internal_power {
  int32_t  pin;           /* cell-local pin index of the group's port */
  int32_t  related_pin;   /* cell-local related pin index, -1 if none */
  gtp_when when;
  int32_t  rise_table;    /* index into gtp_design.tables, -1 if absent */
  int32_t  fall_table;
} gtp_internal_power;

/* A Liberty leakage_power group, in Liberty order
 * (Power::getLeakagePower, power/TimeBasedPower.cc:258-301). The reference
 * expands only conjunctions (getWhenPinStates, power/PowerUtils.cc:191-201);
 * an unsupported or unsatisfiable `when` is encoded with n_cube = 0. */
typedef struct gtp_leakage_power {
  gtp_when when;
  float    power;         /* W */
  int32_t  reserved;
} gtp_leakage_power;

/* A library cell type. Pins are ordered inputs first, then outputs, in
 * instance pin-iterator order (Power::getPinInformation,
 * power/TimeBasedPower.cc:223-256). */
typedef struct gtp_cell_type {
  int32_t n_pin;
  int32_t n_in;
  int32_t ipwr_off, n_ipwr;   /* into gtp_design.internal_powers */
  int32_t leak_off, n_leak;   /* into gtp_design.leakage_powers  */
  float   cell_leakage_power; /* cell_leakage_power attribute (W) */
  int32_t has_cell_leakage_power;
} gtp_cell_type;

/* The static design: everything the power walk reads besides the events. */
typedef struct gtp_design {
  /* time base */
  double  timescale;      /* seconds per VCD tick (Vcd::timeScale)        */
  float   clk_period;     /* seconds, as float (Power::clk_period_)       */
  int32_t reserved0;
  int64_t time_max;       /* last VCD timestamp (Vcd::timeMax)            */

  int32_t n_cell, n_pin, n_net, n_type;

  /* cells */
  const int32_t* cell_pin_off;   /* [n_cell+1] */
  const int32_t* cell_type;      /* [n_cell]   */
  const uint8_t* cell_group;     /* [n_cell]   GTP_GROUP_*  */
  const int64_t* cell_arc_off;   /* [n_cell]   offset into arc_delay        */

  /* pins */
  const int32_t* pin_net;        /* [n_pin] net id; -1 = no waveform        */
  const float*   pin_slew_rise;  /* [n_pin] s; +inf = no slew (delayInf)    */
  const float*   pin_slew_fall;  /* [n_pin] s                               */
  const float*   pin_load_cap;   /* [n_pin] F (GraphDelayCalc::loadCap)     */
  const float*   pin_voltage;    /* [n_pin] V (Power::portVoltage)          */
  const uint8_t* pin_default_state; /* [n_pin] 0/1/2, for pins w/o events   */
  const uint8_t* pin_is_clock;   /* [n_pin] LibertyPort::isClock            */

  /* arc delays: per cell [n_out][n_in][4] floats (s), arc index
   * 2*(from==fall)+(to==fall) as Gate::cellArcDelay
   * (power/cuda/Gate.cuh:344-348); NaN = no timing arc. */
  const float*   arc_delay;
  int64_t        n_arc_delay;

  /* library */
  const gtp_cell_type*      types;            /* [n_type] */
  const gtp_internal_power* internal_powers;  /* [n_internal_power] */
  const gtp_leakage_power*  leakage_powers;   /* [n_leakage_power] */
  const gtp_table*          tables;           /* [n_table] */
  const float*              lut_pool;         /* [lut_pool_len] */
  const uint32_t*           when_cubes;       /* [2*n_when_cube] */
  int32_t n_internal_power, n_leakage_power, n_table, n_when_cube;
  int64_t lut_pool_len;
} gtp_design;

/* Per-net event lists for one window of time, CSR over nets.
 * Events with time in [t_lo, t_hi) are processed; events outside it are
 * context. A window after the first must list, for every net, all events of
 * the last clock period that has an event before t_lo plus the event before
 * that period, and the first two events at or after t_hi (when they exist):
 * glitch classification and related-pin search look that far. A single
 * window over the whole trace (t_lo = 0, t_hi = INT64_MAX, net_base = NULL)
 * needs no context. */
typedef struct gtp_events {
  int64_t         n_event;
  const int64_t*  net_off;       /* [n_net+1] */
  const int64_t*  time;          /* [n_event] ticks, strictly increasing per net */
  const uint32_t* value_packed;  /* [ceil(n_event/16)] 2 bits per event, event
                                    i in word i/16 at bit 2*(i%16) */
  const int64_t*  net_base;      /* [n_net] index, within the net's whole
                                    waveform, of its first listed event; NULL = 0 */
  int64_t t_lo, t_hi;
} gtp_events;

/* Tunables. Field names follow util/GlobalConfig.hh where one exists. */
typedef struct gtp_config {
  int32_t cuda_device_id;            /* -1 = current device */
  int32_t cycles_per_tile;           /* cycle tile of one CTA; 0 = 768 (512 with cycle groups) */
  int32_t n_thread_per_block;        /* 0 = auto (256); else a multiple of 32 in [32, 256] */
  int32_t gates_per_block;           /* gates one CTA walks per tile; 0 = n_thread_per_block */
  int32_t max_n_pin_for_leakage_power; /* 16 (GlobalConfig.hh:41) */
  int32_t collect_counts;            /* 1 = fill gtp_counts (exact parity) */
  int64_t max_event_num;             /* device event capacity (GlobalConfig.hh:31) */
  int32_t sort_by_work;              /* 1 = per window, walk cells in order of their
                                        event count so a warp's cells carry similar
                                        work (default 1) */
  int32_t clock_runs;                /* clock pins whose net is exactly periodic in a
                                        window (one rise and one fall per cycle at
                                        fixed phases) are walked as runs of whole
                                        cycles between the cell's other events:
                                        0 or 1 = on (default), -1 = edge by edge */
  int32_t split_events;              /* density-aware split, as the reference's
                                        cycles-per-thread rule (Gate::
                                        setNCyclePerThreadByEventCount,
                                        power/cuda/Gate.cuh:354-376): per window,
                                        a cell whose measured event density rho
                                        (its pins' events per cycle, periodic
                                        clock pins excluded) gives more than
                                        split_events events in one cycle tile is
                                        walked by n = ceil(rho * tile /
                                        split_events) threads (at most 32), each
                                        over 1/n of the tile's cycles;
                                        0 = 2048, -1 = off. Needs sort_by_work. */
  int32_t separate_kernels;          /* 1 = evaluate each window with two separate
                                        kernels instead of the fused walk, as the
                                        reference's naive baseline (-disable_fusion,
                                        GlobalConfig cuda_power_separate_kernels_
                                        for_dyn_and_leak, util/GlobalConfig.hh:28;
                                        power/cuda/CudaPower.cu:730-1039): a thread
                                        per pin event for the dynamic energies, a
                                        thread per cell and cycle tile for the
                                        leakage. Same results (per-cycle sums bit
                                        for bit); a comparison point for the fused
                                        walk. Not for cycle-range pushes, batches
                                        or gtp_evaluate_noalloc (GTP_EINVAL).
                                        0 = fused (default). */
  int32_t warp_walk;                 /* 1 = cells of up to 4 pins on a design without
                                        tick/seconds drift are walked by one warp each,
                                        32 events at a time in time order (full lanes,
                                        coalesced event loads; the density split then
                                        applies to the other cells only). Same results
                                        (per-cycle sums bit for bit). 0 = one thread per
                                        cell and tile (default: faster on the traces
                                        measured). */
  int32_t reserved32;
  int64_t reserved[1];
} gtp_config;

/* Integer counters that must match the oracle bit-exactly. */
typedef struct gtp_counts {
  uint32_t* cell_events;       /* [n_cell] pin events walked                 */
  uint32_t* cell_glitches;     /* [n_cell] events classified as glitch       */
  uint32_t* cell_half_toggles; /* [n_cell] sum of 2*n_toggle                 */
  uint32_t* cell_related;      /* [n_cell] sum over output events of
                                  (related input pin + 1), 0 for default     */
  int64_t*  cycle_events;      /* [n_period] pin events per cycle            */
  int64_t*  cycle_glitches;    /* [n_period] glitch events per cycle         */
  int64_t   dropped;           /* contributions past the last cycle          */
} gtp_counts;

typedef struct gtp_ctx gtp_ctx;

void        gtp_config_default(gtp_config* cfg);

/* Validates and packs the design, uploads it to the device. */
gtp_status  gtp_create(const gtp_design* design, const gtp_config* cfg, gtp_ctx** out);
void        gtp_destroy(gtp_ctx* ctx);
const char* gtp_last_error(const gtp_ctx* ctx);

/* Number of per-cycle entries: ceil(time_max*timescale/clk_period), as
 * Power::power sizes its waveforms (power/Power.cc:248). */
int64_t     gtp_n_period(const gtp_ctx* ctx);
/* Ticks per clock cycle: (int64)ceil(float(clk_period)/float(timescale)),
 * as clkedWaveformIdx (power/PowerUtils.cc:27-32). */
int64_t     gtp_ticks_per_cycle(const gtp_ctx* ctx);

/* Clears all accumulators (start of a new trace). */
gtp_status  gtp_reset(gtp_ctx* ctx);

/* Copies one window of events from host memory (pinned or pageable) to the
 * device and evaluates it. Windows must come in time order without overlap.
 * Gaps are allowed: cycles no window covers keep zero per-cycle power, and
 * per-cell values then cover the evaluated windows only (a spot check of
 * selected cycle ranges, e.g. the learned proxy's audit sample). A window
 * after a gap (or a first window with t_lo > 0) is evaluated on its own: its
 * leakage starts at t_lo from the state its context gives and ends at t_hi.
 * Returns once the copy is done (the caller may reuse its buffers); the
 * walk runs on. Consecutive windows alternate between two device buffers
 * and two internal streams, so a window's copy overlaps the walk before it
 * and its walk may start while the last blocks of that walk finish. The
 * context's stream (gtp_get_stream) waits for each walk: work queued on it
 * after this returns runs after the window's walk. */
gtp_status  gtp_push_events(gtp_ctx* ctx, const gtp_events* ev);

/* Same, with events already in device memory (time, value_packed, net_off,
 * net_base are device pointers). Nothing is copied. */
gtp_status  gtp_push_events_device(gtp_ctx* ctx, const gtp_events* d_ev);

/* Evaluates only cycles [cycle_ranges[2k], cycle_ranges[2k+1]) of a device
 * window (ranges ascending, disjoint, within [t_lo, t_hi)), in one pass:
 * spot checks of selected cycles, such as the learned proxy's audit sample
 * and its out-of-range cycles, without walking the rest of the window. The
 * window lists its events as for gtp_push_events_device; the state at each
 * range's start comes from the events before it. Per-cycle power of other
 * cycles stays zero (leakage included: each range is evaluated on its own),
 * per-cell values and counts cover the ranges only, and clock pins are walked
 * edge by edge. The window counts as pushed: later windows follow t_hi.
 * Where the design's tick and seconds cycle boundaries drift apart, the
 * leakage of a cycle that straddles a range's edge in seconds covers only
 * the range's part of it (as for a window pushed after a gap). */
gtp_status  gtp_push_events_device_ranges(gtp_ctx* ctx, const gtp_events* d_ev, const int64_t* cycle_ranges,
                                          int32_t n_ranges);

/* Waits for all queued work. */
gtp_status  gtp_sync(gtp_ctx* ctx);

/* The cudaStream_t (as void*) the context's work is queued on, or waited
 * for: the walks of host-pushed windows run on two internal streams, and
 * this stream waits for each of them (gtp_push_events).
 * gtp_set_stream replaces it with a caller-owned stream (NULL restores the
 * context's own); the caller keeps ownership and must keep it alive. */
void*       gtp_get_stream(const gtp_ctx* ctx);
gtp_status  gtp_set_stream(gtp_ctx* ctx, void* stream);

/* Queues the kernels that turn the accumulators into the outputs of
 * gtp_fetch, without waiting (gtp_fetch runs them too). */
gtp_status  gtp_finalize(gtp_ctx* ctx);

/* Results. Any pointer may be NULL.
 * cell5   [n_cell][5]   : Internal_Power, Glitch_Internal_Power,
 *                         Switching_Power, Glitch_Switching_Power,
 *                         Leakage_Power (W; "Internal"/"Switching" exclude
 *                         glitch, as the columns of cuda_cell_power.txt)
 * cycle5  [5][n_period] : leakage, internal (incl. glitch), glitch internal,
 *                         switching (incl. glitch), glitch switching (W), the
 *                         sections of cuda_per_cycle_waveform.txt
 * totals  [5]           : design totals in FP64, same order as cycle5
 * groups  [GTP_N_GROUP][5] : per report group, FP64, same order as cycle5
 */
gtp_status  gtp_fetch(gtp_ctx* ctx, float* cell5, float* cycle5,
                      double* totals, double* groups, gtp_counts* counts);

/* Per-cycle waveforms by cell group. No counterpart in the reference, whose
 * per-cycle output (cuda_per_cycle_waveform.txt,
 * include/sta/PowerClass.hh:123-149) covers the whole design only. Used to
 * label per-block power for the learned proxy (include/gtpb200_proxy.h).
 * cell_group[i] in [0, n_group) for every cell, n_group <= 65536; n_group = 0
 * turns grouping off. Call before the first window or after gtp_reset. The
 * whole-design waveforms of gtp_fetch are unchanged. */
gtp_status  gtp_set_cycle_groups(gtp_ctx* ctx, const int32_t* cell_group, int32_t n_group);
int32_t     gtp_n_cycle_groups(const gtp_ctx* ctx);
/* cycle5_groups [n_group][5][n_period]: per group, the rows of cycle5. */
gtp_status  gtp_fetch_cycle_groups(gtp_ctx* ctx, float* cycle5_groups);

/* Clock runs (gtp_config.clock_runs); no counterpart in the reference, a
 * diagnostic of this engine. *n_clock_nets = nets read by clock pins,
 * *n_periodic = those whose events in the context's last pushed window
 * (single or batched) were exactly periodic, so that the walk took their
 * clock pins as runs of whole cycles (0 when clock runs are off). Waits for
 * the context's stream. */
gtp_status  gtp_clock_run_nets(gtp_ctx* ctx, int32_t* n_clock_nets, int32_t* n_periodic);

/* Sharding one design across GPUs. No counterpart in the reference, which
 * runs on one device (power/cuda/CudaPower.cu:1227-1337).
 *
 * Cells are independent given their pins' event lists, so N contexts (one
 * per GPU, each created from the whole design so that all share one
 * fixed-point scale) can each walk a contiguous cell range and add their
 * accumulators. gtp_set_cell_range restricts a context to cells
 * [cell_begin, cell_end) (call before the first window or after gtp_reset,
 * and before gtp_set_cycle_groups); its windows need to list only the nets
 * those cells read (other nets may be empty). gtp_export_accumulators copies
 * the context's accumulators (gtp_accumulator_bytes bytes, device to device,
 * on the context's stream) in the layout
 *   double  cell[5][n_cell]          per-cell energy and leakage sums
 *   int64   cycle[6][n_period+1]     per-cycle 64-bit fixed-point bins
 *   uint64  cycle_counts[2][n_period+1]   (with collect_counts)
 *   uint32  cell_counts[4][n_cell]        (with collect_counts)
 * Summed over the shards element-wise (FP64 for the cell sums, which are
 * disjoint, wrap-around integer addition for the rest: exact and
 * order-independent), the block imported into any shard's context with
 * gtp_import_accumulators makes gtp_fetch return the whole design's
 * results. Per-cycle waveforms by cell group are not carried. */
gtp_status  gtp_set_cell_range(gtp_ctx* ctx, int32_t cell_begin, int32_t cell_end);
int64_t     gtp_accumulator_bytes(const gtp_ctx* ctx);
gtp_status  gtp_export_accumulators(gtp_ctx* ctx, void* d_out);
gtp_status  gtp_import_accumulators(gtp_ctx* ctx, const void* d_in);

/* Density split (gtp_config.split_events); a diagnostic of this engine.
 * *items = threads per tile that walked the context's last one-window push
 * (n_cell when no cell was split; n_cell + the extra threads of split cells
 * otherwise; 0 when the split is off). Waits for the context's stream. */
gtp_status  gtp_walk_items(gtp_ctx* ctx, int64_t* items);

/* Allocation-free evaluation. No counterpart in the reference.
 *
 * For callers that cannot allocate device memory while they run, e.g. an
 * EDA host that embeds the engine under its own device-memory arena reserved
 * at start-up, or a service that cannot absorb the device-wide
 * synchronization cudaMalloc/cudaFree may cause. It evaluates one whole
 * trace (t_lo = 0) of device-resident events d_ev against the context's
 * design and writes cell5 [n_cell][5], cycle5 [5][n_period] and totals [5]
 * (layouts as gtp_fetch) into caller device buffers (d_totals may be NULL).
 * It calls no cudaMalloc, cudaFree or other allocating routine: its
 * accumulators live in a 16 MiB static device array that every GPU loading
 * the library holds until exit. Limit: 40 bytes per cell + 56 per cycle
 * within 16 MiB (about 300k cells x 20k cycles); larger designs get
 * GTP_EOVERFLOW. The first call on a device looks up the array's address
 * and keeps it for the life of the process; make that first call before any
 * stream capture, and after a cudaDeviceReset do not call this entry point
 * again on that device in the same process (the kept address is stale). All
 * calls share the array (each clears what it uses first), so calls that
 * overlap on the GPU race. Work is queued on the context's stream; each call
 * first clears the context's status word (dropping any unreported error of
 * earlier work on the context), and gtp_sync then waits and reports this
 * call's invalid events. */
gtp_status  gtp_evaluate_noalloc(gtp_ctx* ctx, const gtp_events* d_ev, float* d_cell5,
                                 float* d_cycle5, double* d_totals);

/* Batched evaluation. No counterpart in the reference, which runs one
 * design per CudaPower::power call (power/cuda/CudaPower.cu:1227-1337).
 *
 * A batch groups contexts (each with its own design, accumulators and
 * windows) that share a device, n_thread_per_block and collect_counts.
 * gtp_batch_push_device takes one device window per context (d_ev[i] as for
 * gtp_push_events_device; d_ev[i].net_off == NULL skips context i) and walks
 * all of them in one persistent launch per pin bucket: blocks take
 * (context, gate block, cycle tile) work items from a device queue, heaviest
 * first. With use_graph the launch sequence (the windows' work sorts and
 * the persistent walks) is captured in a CUDA graph and replayed while the
 * contexts and their window buffers stay the same. Results are read per
 * context with gtp_fetch after gtp_batch_sync. */
typedef struct gtp_batch_config {
  int32_t use_graph;       /* 1 (default): replay captured launches */
  int32_t blocks_per_sm;   /* persistent blocks per SM; 0 = occupancy */
  int64_t reserved[4];
} gtp_batch_config;
typedef struct gtp_batch gtp_batch;

void        gtp_batch_config_default(gtp_batch_config* cfg);
gtp_status  gtp_batch_create(gtp_ctx* const* ctxs, int32_t n_ctx, const gtp_batch_config* cfg,
                             gtp_batch** out);
void        gtp_batch_destroy(gtp_batch* b);
const char* gtp_batch_last_error(const gtp_batch* b);
gtp_status  gtp_batch_push_device(gtp_batch* b, const gtp_events* d_ev);
/* Waits for the batch and reports invalid events of any context. */
gtp_status  gtp_batch_sync(gtp_batch* b);
void*       gtp_batch_get_stream(const gtp_batch* b);
/* Work items and persistent launches of the last push; graph replays so far. */
gtp_status  gtp_batch_stats(const gtp_batch* b, int64_t* items, int32_t* launches,
                            int32_t* graph_replays);

/* The reference's result files, from fetched results (host arrays; no
 * context or device needed), written with the reference's expressions and
 * std::ostream formatting:
 *   gtp_write_cell_power: cuda_cell_power.txt (CudaPower::printCellRes,
 *     power/cuda/CudaPower.cu:3134-3165; the CPU path's cpu_cell_power.txt,
 *     Power::printCellRes, power/Power.cc:389-422, has the same layout).
 *     cell5 [n_cell][5] as gtp_fetch; one row per cell in cell index order,
 *     named cell_names[i], with the Liberty cell name
 *     type_names[cell_type[i]] (both may be NULL: empty names). The
 *     internal and switching columns are formed as the reference forms them:
 *     (regular + glitch) folded in float, then folded - glitch.
 *   gtp_write_per_cycle_waveform: cuda_per_cycle_waveform.txt
 *     (PowerResult::printPerCycleResults, include/sta/PowerClass.hh:123-149):
 *     five sections (leakage, internal, glitch internal, switching, glitch
 *     switching), each the design total's waveform cycle5 [5][n_period]
 *     under top_name.
 * sep: the column separator (NULL: a tab, G_CONFIG's default,
 * util/GlobalConfig.hh:50). GTP_GENERAL_ERROR when the file cannot be
 * written. */
gtp_status  gtp_write_cell_power(const char* path, int32_t n_cell, const float* cell5,
                                 const char* const* cell_names, const int32_t* cell_type,
                                 const char* const* type_names, const char* sep);
gtp_status  gtp_write_per_cycle_waveform(const char* path, int64_t n_period, const float* cycle5,
                                         const char* top_name, const char* sep);

/* VCD value-change ingest on the GPU. Replaces the reference's host parse
 * of the VCD body (VcdReader::parseVarValues, power/VcdReader.cc:247-301),
 * its per-var value store (Vcd::varAppendValue / varAppendBusValue,
 * power/Vcd.cc:204-234; bus bits as VcdValue::value, :271-277) and the
 * per-pin event-buffer build (CudaPower::getGateWaveformRangeMultiThread,
 * power/cuda/CudaPower.cu:1874-2086). The caller parses the header ($var
 * declarations are few) and passes:
 *   the distinct id codes: id_chars[id_off[i] .. id_off[i+1]) for i < n_id;
 *   the sources: net s of the output CSR lists bit src_bit[s] of id
 *     src_id[s] (bit 0 for scalars; for a vector, bit b of its value with
 *     b = 0 the LSB).
 * gtp_vcd_parse then reads a body (host bytes, the text after
 * $enddefinitions ... $end) with the reference's rules: upper-cased first
 * characters; scalar changes 0/1/x/u/z<id> (u read as X); vector changes
 * b<digits> <id>, a value whose first digit is x/u/z being 0, else the
 * leading binary digits as strtol reads them; r<real> <id> skipped; a
 * change equal to the id's previous one dropped; an X (scalars) or 0
 * (vectors) inserted at tick 0 before an id's first change when that comes
 * later; time_max = the last time stamp. It fills *d_out with device
 * arrays (t_lo 0, t_hi INT64_MAX, no net_base) that stay valid until the
 * next parse or gtp_vcd_destroy, ready for gtp_push_events_device.
 * GTP_EINVAL on an undeclared id, a time stamp that is not a decimal number
 * or an id that takes both scalar and vector changes (message in
 * gtp_vcd_last_error). Work runs on the reader's own stream; the call
 * returns when the CSR is complete. */
typedef struct gtp_vcd gtp_vcd;
gtp_status  gtp_vcd_create(const char* id_chars, const int32_t* id_off, int32_t n_id, const int32_t* src_id,
                           const int32_t* src_bit, int32_t n_src, int32_t cuda_device_id, gtp_vcd** out);
gtp_status  gtp_vcd_parse(gtp_vcd* vcd, const char* body, int64_t n_bytes, gtp_events* d_out,
                          int64_t* time_max);
/* Host copies of the last parse's CSR (net_off [n_src+1], time [n_event],
 * packed [ceil(n_event/16)]; any may be NULL). */
gtp_status  gtp_vcd_fetch(gtp_vcd* vcd, int64_t* net_off, int64_t* time, uint32_t* packed);
/* Tokens and value changes (before repeat dropping) of the last parse. */
gtp_status  gtp_vcd_stats(const gtp_vcd* vcd, int64_t* n_token, int64_t* n_change);
const char* gtp_vcd_last_error(const gtp_vcd* vcd);
void        gtp_vcd_destroy(gtp_vcd* vcd);

/* Packs one value per byte (0..3) into the 2-bit layout of value_packed. */
void        gtp_pack_values(const uint8_t* values, int64_t n, uint32_t* packed);

#ifdef __cplusplus
}
#endif
#endif /* GTPB200_H */
