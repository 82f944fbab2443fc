/*
 * gtpb200_proxy.h — learned per-cycle power proxy beside the time-based
 * power engine (include/gtpb200.h).
 *
 * The reference has no counterpart: GTPower evaluates every cycle with the
 * event walk (power/TimeBasedPower.cc:703-901 on the CPU,
 * power/cuda/CudaPower.cu:317-584 on CUDA). This interface adds a small
 * BF16 multilayer perceptron that predicts per-cycle power from the toggle
 * bits of a selected subset of nets:
 *
 *   x[c]  = 1 if net sel[k] changes value in cycle c, else 0   (k < n_in)
 *   h1    = relu(W1 x + b1)      W1: [n_hidden][n_in]
 *   h2    = relu(W2 h1 + b2)     W2: [n_hidden][n_hidden]
 *   y     = W3 h2 + b3           W3: [n_out][n_hidden]
 *
 * trained against per-cycle powers that the engine itself computes (mean
 * squared error on targets standardised per output, Adam). Weights and
 * activations are BF16 with FP32 accumulation on the tcgen05 tensor cores;
 * the master weights and Adam moments are FP32. The engine stays the authority:
 * callers audit a sample of cycles and recompute out-of-range ones with it.
 *
 * Pointers named d_ are device pointers on the proxy's device; all others
 * are host pointers. BF16 arrays are passed as uint16_t bit patterns.
 * Flat parameter order (gtp_proxy_get_params and friends):
 *   W1 [n_hidden][n_in], b1 [n_hidden], W2 [n_hidden][n_hidden],
 *   b2 [n_hidden], W3 [n_out][n_hidden], b3 [n_out].
 */
#ifndef GTPB200_PROXY_H
#define GTPB200_PROXY_H

#include <stdint.h>

#include "gtpb200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gtp_proxy_config {
  int32_t cuda_device_id;
  int32_t n_in;        /* toggle-bit inputs, multiple of 64                */
  int32_t n_hidden;    /* hidden width, multiple of 64                     */
  int32_t n_out;       /* outputs (1..256)                                 */
  int32_t batch;       /* training minibatch rows, multiple of 128         */
  float lr;            /* Adam step size                                   */
  float beta1, beta2, eps;
  float weight_decay;  /* decoupled (AdamW) decay on W1..W3, 0 = none      */
  uint64_t seed;       /* weight initialisation                            */
  int32_t use_graph;   /* 1: replay training steps from a CUDA graph       */
  int32_t reserved32;
  int64_t reserved[4];
} gtp_proxy_config;

typedef struct gtp_proxy gtp_proxy;

/* 4096 -> 512 -> 512 -> 33, batch 1024, lr 1e-3, betas 0.9/0.999, eps 1e-8. */
void        gtp_proxy_config_default(gtp_proxy_config* cfg);
gtp_status  gtp_proxy_create(const gtp_proxy_config* cfg, gtp_proxy** out);
void        gtp_proxy_destroy(gtp_proxy* p);
const char* gtp_proxy_last_error(const gtp_proxy* p);
void*       gtp_proxy_get_stream(gtp_proxy* p);
gtp_status  gtp_proxy_set_stream(gtp_proxy* p, void* stream);
int64_t     gtp_proxy_n_param(const gtp_proxy* p);

/* Training set: d_x [n_rows][n_in] BF16 toggle bits, d_y [n_rows][n_out]
 * FP32 targets. Device memory owned by the caller; it must stay valid until
 * the last gtp_proxy_train / gtp_proxy_compute_grads call that reads it.
 * Computes the per-output standardisation (mean, std) of d_y. */
gtp_status  gtp_proxy_set_training_data(gtp_proxy* p, const uint16_t* d_x, const float* d_y,
                                        int64_t n_rows);
/* Per-output mean and std used to standardise targets (n_out each). */
gtp_status  gtp_proxy_get_norm(gtp_proxy* p, float* mean, float* std);

/* n_epochs passes over the training set in shuffled minibatches
 * (floor(n_rows / batch) steps each). loss_per_epoch (may be NULL) receives
 * the mean squared error on standardised targets of each epoch. */
gtp_status  gtp_proxy_train(gtp_proxy* p, int32_t n_epochs, float* loss_per_epoch);

/* One forward and backward pass over the training rows rows[0..batch),
 * leaving the gradients in place (no update). *loss = mean squared error. */
gtp_status  gtp_proxy_compute_grads(gtp_proxy* p, const int32_t* rows, float* loss);
/* One Adam update from the gradients in place. */
gtp_status  gtp_proxy_adam_step(gtp_proxy* p);

gtp_status  gtp_proxy_get_params(gtp_proxy* p, float* params);
gtp_status  gtp_proxy_set_params(gtp_proxy* p, const float* params);
gtp_status  gtp_proxy_get_grads(gtp_proxy* p, float* grads);

/* d_y [n_rows][n_out] FP32 = de-standardised prediction for d_x. */
gtp_status  gtp_proxy_predict(gtp_proxy* p, const uint16_t* d_x, int64_t n_rows, float* d_y);

/* ---- features from the engine's event CSR (gtp_events layout) ----------
 * Both functions read the events of nets in device memory: d_net_off
 * [n_net+1] and d_time [n_event] as in gtp_events, and consider only
 * events with tick > 0 whose cycle c = tick / ticks_per_cycle lies in
 * [c_lo, c_hi). They run on the stream given (NULL: legacy default stream)
 * and return GTP_ECUDA on a launch error. */

/* d_x[(c - c_lo) * ld + k] = 1.0 (BF16) when net d_sel[k] has an event in
 * cycle c. Entries for other cycles are left unchanged (clear d_x first). */
gtp_status  gtp_toggle_bits(const int64_t* d_net_off, const int64_t* d_time, const int32_t* d_sel,
                            int32_t n_sel, int64_t ticks_per_cycle, int64_t c_lo, int64_t c_hi,
                            uint16_t* d_x, int64_t ld, void* stream);

/* One window for gtp_toggle_bits_windows: its event CSR (device pointers,
 * gtp_events layout) and the cycles [c_lo, c_hi) whose rows it fills. */
typedef struct gtp_bits_window {
  const int64_t* d_net_off;
  const int64_t* d_time;
  int64_t c_lo;
  int64_t c_hi;
} gtp_bits_window;

#define GTP_BITS_MAX_WINDOWS 64

/* Dense toggle bits of many windows in one launch: for every window w (host
 * array, at most GTP_BITS_MAX_WINDOWS, row ranges not overlapping) and every
 * cycle c in [w.c_lo, w.c_hi), d_x[(c - c_base) * ld + k] = 1.0 (BF16) when
 * net d_sel[k] has an event with tick > 0 in cycle c, else 0.0, for all
 * k < n_sel. Rows outside the windows are left unchanged, so d_x needs no
 * clearing first. Each block builds the toggle masks of 64 nets over up to
 * 2048 rows in shared memory and writes whole row segments. */
gtp_status  gtp_toggle_bits_windows(const gtp_bits_window* windows, int32_t n_win, const int32_t* d_sel,
                                    int32_t n_sel, int64_t ticks_per_cycle, int64_t c_base, uint16_t* d_x,
                                    int64_t ld, void* stream);

/* For every net n < n_net: d_count[n] += number of cycles in [c_lo, c_hi)
 * in which it toggles, d_sum_y[n] += sum of d_y[c - c_lo] over those cycles.
 * Accumulates, so that windows of one trace can be added up. */
gtp_status  gtp_net_toggle_stats(const int64_t* d_net_off, const int64_t* d_time, int32_t n_net,
                                 int64_t ticks_per_cycle, int64_t c_lo, int64_t c_hi, const float* d_y,
                                 int64_t* d_count, double* d_sum_y, void* stream);

/* BF16 GEMM on the tensor cores, the building block of the proxy:
 * d_c[m][n] (FP32, row stride ldc) = d_a[m][k] * d_b[n][k]^T (+ d_bias[n]
 * when d_bias is not NULL; then ReLU when relu != 0). Row strides lda, ldb
 * in elements, multiples of 8; k a multiple of 8. */
gtp_status  gtp_bf16_gemm(const uint16_t* d_a, int64_t lda, const uint16_t* d_b, int64_t ldb,
                          int64_t m, int64_t n, int64_t k, const float* d_bias, int32_t relu,
                          float* d_c, int64_t ldc, void* stream);

/* gtp_bf16_gemm that reports its pipeline's health and waits for the result.
 * Every wait inside the kernel (TMA bytes landed, MMAs done, accumulator
 * drained) gives up after spin_limit_cycles SM clock cycles (0: about one
 * second); a wait that gives up sets *d_err (a caller device int32, cleared
 * first), the kernel lets its copies and MMAs in flight finish, frees its
 * TMEM and returns, and the call returns GTP_ETIMEOUT (d_c is then
 * unspecified). The device stays usable. test_skip_load_block >= 0 is a test
 * of that path: the first CTA's TMA producer skips the loads of its K block
 * with that index (counted over its tiles), so that the MMA issuer's wait
 * for them runs out; -1 in normal use. Synchronises `stream`. */
gtp_status  gtp_bf16_gemm_checked(const uint16_t* d_a, int64_t lda, const uint16_t* d_b, int64_t ldb,
                                  int64_t m, int64_t n, int64_t k, const float* d_bias, int32_t relu,
                                  float* d_c, int64_t ldc, int64_t spin_limit_cycles,
                                  int32_t test_skip_load_block, int32_t* d_err, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GTPB200_PROXY_H */
