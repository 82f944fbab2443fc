// synth_dev.cu — the synthetic trace generator on the GPU.
//
// Produces the same cycle windows as the host stream (synth_stream_next in
// synth.cpp), bit for bit, from the shared rules of synth_rules.h, directly
// into device memory: per window a count pass (one thread per net), an
// exclusive scan of the counts into net_off, and a fill pass that writes the
// ticks, the packed 2-bit values and net_base, then advances the per-net
// stream state. Per net and window the listed events are
//   head : the events of the last clock period before c_lo that has any,
//          and the event before that period (the state carried over, at
//          most 4 events; none for the first window);
//   body : the events of cycles [c_lo, c_hi), with the tick-0 initial value
//          in the first window;
//   tail : (c_hi < n_cycle) the first two events of cycles
//          [c_hi, c_hi + window); when there are none and the last listed
//          period holds an even number (>= 2) of counted events, the first
//          events of the next cycle that has any.
// Event i of a net's whole waveform (0 = the initial value) carries the value
// initial ^ (i & 1), as the host generator's toggles do.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdint>

#include "synth_rules.h"

namespace {

using gtpb::syn::Rules;

struct State {
  Rules r{};             // device table pointers
  int64_t wcyc = 1;
  int64_t c_next = 0;    // first cycle of the next window
  int32_t device = 0;
  int32_t n_phase = 0;
  double* net_rate = nullptr;
  double* burst = nullptr;
  double* act = nullptr;
  uint8_t* phase = nullptr;
  int64_t* gcount = nullptr;   // [n_net] events listed in bodies so far (incl. the initial value)
  int64_t* ring_t = nullptr;   // [n_net][4] head for the next window
  uint8_t* ring_n = nullptr;   // [n_net]
  int64_t* tail_t = nullptr;   // [n_net][2] tail of the counted window
  uint8_t* tail_n = nullptr;
  int64_t* counts = nullptr;   // [n_net + 1]
  void* scan_tmp = nullptr;
  size_t scan_bytes = 0;
  int64_t cnt_lo = -1, cnt_hi = -1;  // window counted last
};

__global__ void count_kernel(Rules r, int64_t c_lo, int64_t c_hi, int64_t wcyc, const int64_t* __restrict__ ring_t,
                             const uint8_t* __restrict__ ring_n, int64_t* __restrict__ tail_t,
                             uint8_t* __restrict__ tail_n, int64_t* __restrict__ counts) {
  const int32_t n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= r.n_net) return;
  const int64_t tpc = r.tpc, nc = r.n_cycle;
  int64_t tb[3];
  int64_t n_body = c_lo == 0 ? 1 : 0;
  int64_t last_p = c_lo == 0 ? 0 : -1;
  int k_last = c_lo == 0 ? 1 : 0;
  for (int64_t c = c_lo; c < c_hi; ++c) {
    const int m = gtpb::syn::cycle_events(r, n, c, tb);
    if (m) {
      n_body += m;
      if (c == last_p) k_last += m;
      else {
        last_p = c;
        k_last = m;
      }
    }
  }
  const int hn = c_lo > 0 ? ring_n[n] : 0;
  if (n_body == 0 && hn > 0) {  // last listed period: from the head
    last_p = ring_t[4 * n + hn - 1] / tpc;
    k_last = 0;
    for (int j = hn - 1; j >= 0 && ring_t[4 * n + j] / tpc == last_p; --j) ++k_last;
  }
  const int k_eff = k_last - (last_p == 0 ? 1 : 0);
  const bool need_far = k_eff >= 2 && (k_eff % 2) == 0;
  int tn = 0;
  if (c_hi < nc) {
    const int64_t b_hi = min(nc, c_hi + wcyc);
    for (int64_t c = c_hi; c < b_hi && tn < 2; ++c) {
      const int m = gtpb::syn::cycle_events(r, n, c, tb);
      for (int j = 0; j < m && tn < 2; ++j) tail_t[2 * n + tn++] = tb[j];
    }
    if (tn == 0 && need_far) {
      for (int64_t c = b_hi; c < nc && tn == 0; ++c) {
        const int m = gtpb::syn::cycle_events(r, n, c, tb);
        for (int j = 0; j < m && tn < 2; ++j) tail_t[2 * n + tn++] = tb[j];
      }
    }
  }
  tail_n[n] = static_cast<uint8_t>(tn);
  counts[n] = hn + n_body + tn;
}

__device__ __forceinline__ void put(int64_t k, int64_t t, uint32_t v, int64_t* __restrict__ time,
                                    uint32_t* __restrict__ packed) {
  time[k] = t;
  if (v) atomicOr(packed + (k >> 4), v << (2 * (k & 15)));
}

__global__ void fill_kernel(Rules r, int64_t c_lo, int64_t c_hi, const int64_t* __restrict__ net_off,
                            int64_t* __restrict__ gcount, int64_t* __restrict__ ring_t, uint8_t* __restrict__ ring_n,
                            const int64_t* __restrict__ tail_t, const uint8_t* __restrict__ tail_n,
                            int64_t* __restrict__ time, uint32_t* __restrict__ packed,
                            int64_t* __restrict__ net_base) {
  const int32_t n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= r.n_net) return;
  const int64_t tpc = r.tpc;
  const uint32_t v0 = gtpb::syn::initial_value(r, n);
  int64_t k = net_off[n];
  const int64_t g = gcount[n];
  const int hn = c_lo > 0 ? ring_n[n] : 0;
  // head: the last hn events before c_lo, indices g - hn .. g - 1
  int64_t idx = g - hn;
  net_base[n] = idx;
  int64_t prev_t = -1;  // last listed event before the body
  for (int j = 0; j < hn; ++j, ++idx, ++k) {
    prev_t = ring_t[4 * n + j];
    put(k, prev_t, v0 ^ static_cast<uint32_t>(idx & 1), time, packed);
  }
  // body, tracking the last non-empty period and the event before it
  int64_t per_t[4] = {0, 0, 0, 0};
  int per_n = 0;
  int64_t per_p = -1;
  int64_t before = hn > 0 ? prev_t : -1;
  int64_t cur_before = before;
  auto body_event = [&](int64_t t) {
    const int64_t p = t / tpc;
    if (p != per_p) {
      cur_before = per_n > 0 ? per_t[per_n - 1] : cur_before;
      per_p = p;
      per_n = 0;
    }
    if (per_n < 4) per_t[per_n++] = t;
    put(k, t, v0 ^ static_cast<uint32_t>(idx & 1), time, packed);
    ++k;
    ++idx;
  };
  if (c_lo == 0) body_event(0);
  int64_t tb[3];
  int64_t n_body = c_lo == 0 ? 1 : 0;
  for (int64_t c = c_lo; c < c_hi; ++c) {
    const int m = gtpb::syn::cycle_events(r, n, c, tb);
    for (int j = 0; j < m; ++j) body_event(tb[j]);
    n_body += m;
  }
  // tail
  const int tn = tail_n[n];
  for (int j = 0; j < tn; ++j, ++idx, ++k) put(k, tail_t[2 * n + j], v0 ^ static_cast<uint32_t>(idx & 1), time, packed);
  // next head: the body's last non-empty period and the event before it
  if (n_body > 0) {
    int m = 0;
    if (cur_before >= 0) ring_t[4 * n + m++] = cur_before;
    for (int j = 0; j < per_n && m < 4; ++j) ring_t[4 * n + m++] = per_t[j];
    ring_n[n] = static_cast<uint8_t>(m);
    gcount[n] = g + n_body;
  }
}

template <class T>
cudaError_t dalloc(T** p, size_t n) {
  return cudaMalloc(reinterpret_cast<void**>(p), std::max<size_t>(1, n) * sizeof(T));
}

template <class T>
cudaError_t upload(T** dst, const T* src, size_t n) {
  if (src == nullptr || n == 0) {
    *dst = nullptr;
    return cudaSuccess;
  }
  cudaError_t e = dalloc(dst, n);
  if (e == cudaSuccess) e = cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice);
  return e;
}

void release(State* s) {
  void* p[] = {s->net_rate, s->burst, s->act, s->phase, s->gcount, s->ring_t, s->ring_n,
               s->tail_t, s->tail_n, s->counts, s->scan_tmp};
  for (void* q : p)
    if (q) cudaFree(q);
}

}  // namespace

extern "C" {

// host_rules: the trace's rules with host table pointers (synth_trace_rules);
// n_phase: phases of mode 2/3. Returns null on failure.
void* synthdev_create(const Rules* host_rules, int32_t n_phase, int64_t window_cycles, int32_t device) {
  if (!host_rules || host_rules->n_net < 1 || host_rules->n_cycle < 1 || window_cycles < 1) return nullptr;
  if (cudaSetDevice(device) != cudaSuccess) return nullptr;
  State* s = new State();
  s->r = *host_rules;
  s->wcyc = window_cycles;
  s->device = device;
  s->n_phase = n_phase;
  const Rules& h = *host_rules;
  const size_t nn = static_cast<size_t>(h.n_net);
  cudaError_t e = cudaSuccess;
  const bool rate = h.mode == 0 || h.mode == 1 || h.mode == 3;
  if (e == cudaSuccess && rate) e = upload(&s->net_rate, h.net_rate, nn);
  if (e == cudaSuccess && h.mode == 1) e = upload(&s->burst, h.burst, static_cast<size_t>(h.n_cycle));
  if (e == cudaSuccess && (h.mode == 2 || h.mode == 3)) e = upload(&s->phase, h.phase, static_cast<size_t>(h.n_cycle));
  if (e == cudaSuccess && h.mode == 3) e = upload(&s->act, h.act, static_cast<size_t>(n_phase) * h.n_unit);
  if (e == cudaSuccess) e = dalloc(&s->gcount, nn);
  if (e == cudaSuccess) e = dalloc(&s->ring_t, 4 * nn);
  if (e == cudaSuccess) e = dalloc(&s->ring_n, nn);
  if (e == cudaSuccess) e = dalloc(&s->tail_t, 2 * nn);
  if (e == cudaSuccess) e = dalloc(&s->tail_n, nn);
  if (e == cudaSuccess) e = dalloc(&s->counts, nn + 1);
  if (e == cudaSuccess) e = cudaMemset(s->gcount, 0, nn * sizeof(int64_t));
  if (e == cudaSuccess) e = cudaMemset(s->ring_n, 0, nn);
  if (e == cudaSuccess)
    e = cub::DeviceScan::ExclusiveSum(nullptr, s->scan_bytes, s->counts, s->counts, h.n_net + 1);
  if (e == cudaSuccess) e = cudaMalloc(&s->scan_tmp, std::max<size_t>(1, s->scan_bytes));
  if (e != cudaSuccess) {
    release(s);
    delete s;
    return nullptr;
  }
  s->r.net_rate = s->net_rate;
  s->r.burst = s->burst;
  s->r.phase = s->phase;
  s->r.act = s->act;
  return s;
}

void synthdev_destroy(void* h) {
  if (!h) return;
  State* s = static_cast<State*>(h);
  cudaSetDevice(s->device);
  release(s);
  delete s;
}

// Counts the next window and writes its net_off [n_net + 1] (device).
// Returns the number of events (>= 0) and the window's cycles in *c_lo,
// *c_hi; -1 when the trace is exhausted; -2 on a CUDA error. Synchronises
// the stream.
int64_t synthdev_count(void* h, int64_t* d_net_off, int64_t* c_lo, int64_t* c_hi, void* stream) {
  State* s = static_cast<State*>(h);
  if (!s || !d_net_off || !c_lo || !c_hi) return -2;
  if (s->c_next >= s->r.n_cycle) return -1;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t lo = s->c_next, hi = std::min(s->r.n_cycle, lo + s->wcyc);
  const int nb = (s->r.n_net + 255) / 256;
  count_kernel<<<nb, 256, 0, st>>>(s->r, lo, hi, s->wcyc, s->ring_t, s->ring_n, s->tail_t, s->tail_n, s->counts);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemsetAsync(s->counts + s->r.n_net, 0, sizeof(int64_t), st);
  if (e == cudaSuccess)
    e = cub::DeviceScan::ExclusiveSum(s->scan_tmp, s->scan_bytes, s->counts, d_net_off, s->r.n_net + 1, st);
  int64_t total = 0;
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&total, d_net_off + s->r.n_net, sizeof(int64_t), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return -2;
  s->cnt_lo = lo;
  s->cnt_hi = hi;
  *c_lo = lo;
  *c_hi = hi;
  return total;
}

// Fills the window counted last into d_time [n_event], d_packed
// [ceil(n_event/16)] (cleared here) and d_net_base [n_net], and advances the
// stream. Returns 0, or -2 on a CUDA error, -3 if no window was counted.
int32_t synthdev_fill(void* h, const int64_t* d_net_off, int64_t n_event, int64_t* d_time, uint32_t* d_packed,
                      int64_t* d_net_base, void* stream) {
  State* s = static_cast<State*>(h);
  if (!s || !d_net_off || !d_time || !d_packed || !d_net_base) return -2;
  if (s->cnt_lo != s->c_next) return -3;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(d_packed, 0, sizeof(uint32_t) * std::max<int64_t>(1, (n_event + 15) / 16), st);
  const int nb = (s->r.n_net + 255) / 256;
  if (e == cudaSuccess) {
    fill_kernel<<<nb, 256, 0, st>>>(s->r, s->cnt_lo, s->cnt_hi, d_net_off, s->gcount, s->ring_t, s->ring_n, s->tail_t,
                                    s->tail_n, d_time, d_packed, d_net_base);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) return -2;
  s->c_next = s->cnt_hi;
  s->cnt_lo = s->cnt_hi = -1;
  return 0;
}

}  // extern "C"
