// vcd_gpu.cu — VCD value-change ingest on the GPU: from the body text of a
// VCD file to the per-net event CSR the walk reads (gtp_events).
//
// Replaces the reference's host loops for this step: the char-by-char
// tokenizer VcdReader::parseVarValues (power/VcdReader.cc:247-301), the
// per-var value store with its repeat dropping and initial value
// (Vcd::varAppendValue / varAppendBusValue, power/Vcd.cc:204-234; bus bits
// by VcdValue::value, :271-277) and the per-pin waveform slicing into one
// event buffer (CudaPower::getGateWaveformRangeMultiThread,
// power/cuda/CudaPower.cu:1874-2086). The header (scopes, $var
// declarations, timescale) is small and stays on the host.
//
// Pipeline over the body bytes, all on the device:
//   1. token starts (a non-blank byte after a blank), compacted;
//   2. per token: its kind (time '#', scalar change 0/1/x/u/z<id>, vector
//      change b<digits> <id>, real r<value> <id>, other), its time value;
//      which tokens are ids consumed by the vector/real token before them
//      (a scan of a two-state automaton, so that ids that look like values
//      are read as ids);
//   3. the time of every change (the last time token before it, a max scan)
//      and its id (a hash table of the declared ids), its value (scalar
//      code, or the vector's leading binary digits as strtol reads them);
//   4. changes grouped by id (a stable radix sort keeps file order), a
//      change kept only when it differs from the id's previous change, an
//      initial X (scalars) or 0 (vectors) inserted at tick 0 when an id's
//      first change is later;
//   5. one event list per requested (id, bit) source, as the CSR of the
//      engine's nets: times and 2-bit values (a vector bit is
//      (value >> bit) & 1).
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>
#include <thrust/iterator/counting_iterator.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/gtpb200.h"

namespace {

constexpr uint8_t kTokOther = 0, kTokTime = 1, kTokScalar = 2, kTokVector = 3, kTokReal = 4;
constexpr int32_t kVcdErrUnknownId = 1, kVcdErrBadTime = 2, kVcdErrMixedKinds = 4;
constexpr uint64_t kEmptySlot = ~0ull;

__device__ __forceinline__ bool is_blank(uint8_t c) {
  return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\v' || c == '\f';
}
__device__ __forceinline__ uint8_t upper(uint8_t c) { return (c >= 'a' && c <= 'z') ? c - 32 : c; }

// 64-bit FNV-1a of bytes [a, a + n); the host table uses the same function.
__host__ __device__ __forceinline__ uint64_t fnv1a(const char* a, int64_t n) {
  uint64_t h = 1469598103934665603ull;
  for (int64_t i = 0; i < n; ++i) {
    h ^= static_cast<uint8_t>(a[i]);
    h *= 1099511628211ull;
  }
  return h;
}

// flags[i] = 1 when byte i starts a token
__global__ void token_flags_kernel(const uint8_t* __restrict__ b, int64_t n, uint8_t* __restrict__ flags) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    flags[i] = (!is_blank(b[i]) && (i == 0 || is_blank(b[i - 1]))) ? 1 : 0;
}

// Per token: kind, end, time value (time tokens; -1 when the digits are not
// a decimal number, reported unless the token is read as an id) and its
// automaton step: 1 when the token, read as a value, consumes the next one.
__global__ void token_kind_kernel(const uint8_t* __restrict__ b, int64_t n, const int64_t* __restrict__ start,
                                  int64_t n_tok, uint8_t* __restrict__ kind, int64_t* __restrict__ tend,
                                  int64_t* __restrict__ tval, uint8_t* __restrict__ step) {
  for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < n_tok;
       k += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t s = start[k];
    int64_t e = s + 1;
    while (e < n && !is_blank(b[e])) ++e;
    tend[k] = e;
    const uint8_t c0 = upper(b[s]);
    const int64_t len = e - s;
    uint8_t kd = kTokOther;
    int64_t v = 0;
    if (c0 == '#' && len > 1) {
      kd = kTokTime;
      for (int64_t i = s + 1; i < e; ++i) {
        const uint8_t d = b[i];
        if (d < '0' || d > '9') { v = -1; break; }
        v = v * 10 + (d - '0');
      }
    } else if ((c0 == '0' || c0 == '1' || c0 == 'X' || c0 == 'U' || c0 == 'Z') && len > 1) {
      kd = kTokScalar;
    } else if (c0 == 'B') {
      kd = kTokVector;
    } else if (c0 == 'R') {
      kd = kTokReal;
    }
    kind[k] = kd;
    tval[k] = v;
    step[k] = (kd == kTokVector || kd == kTokReal) ? 1 : 0;
  }
}

// Composition of automaton steps (a, then b) on the 1-bit state "this token
// is consumed": f encodes (f(0) in bit 0, f(1) in bit 1).
struct StepCompose {
  __device__ __forceinline__ uint8_t operator()(uint8_t a, uint8_t b) const {
    const uint8_t x0 = a & 1, x1 = (a >> 1) & 1;
    const uint8_t y0 = (b >> x0) & 1, y1 = (b >> x1) & 1;
    return static_cast<uint8_t>(y0 | (y1 << 1));
  }
};

// A token's step as a function of whether it is consumed: consumed -> the
// next token is not; not consumed -> the next is when this one is a
// vector or real value.
__global__ void step_fn_kernel(const uint8_t* __restrict__ step, int64_t n_tok, uint8_t* __restrict__ fn) {
  for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < n_tok;
       k += static_cast<int64_t>(gridDim.x) * blockDim.x)
    fn[k] = step[k] & 1;  // f(0) = step, f(1) = 0
}

struct MaxOp {
  __device__ __forceinline__ int64_t operator()(int64_t a, int64_t b) const { return a > b ? a : b; }
};

// Device id table: open addressing over FNV-1a hashes of the declared id
// strings; slot = (hash, id index), hash kEmptySlot = empty.
struct IdTable {
  const unsigned long long* hash;
  const int32_t* index;
  uint64_t mask;
  const char* chars;      // id strings, concatenated
  const int32_t* off;     // [n_id + 1]
};

__device__ int32_t lookup_id(const IdTable& t, const char* a, int64_t n) {
  const uint64_t h = fnv1a(a, n);
  for (uint64_t probe = 0; probe <= t.mask; ++probe) {
    const uint64_t s = (h + probe) & t.mask;
    const unsigned long long hs = t.hash[s];
    if (hs == kEmptySlot) return -1;
    if (hs == h) {
      const int32_t id = t.index[s];
      const int32_t a0 = t.off[id], a1 = t.off[id + 1];
      if (a1 - a0 == n) {
        bool same = true;
        for (int64_t i = 0; i < n && same; ++i) same = t.chars[a0 + i] == a[i];
        if (same) return id;
      }
    }
  }
  return -1;
}

}  // namespace

namespace {

// is_change[k]: token k is a scalar or vector change (not an id consumed by
// the token before it); tkey[k]: k for a time token that is not consumed,
// else -1 (the max scan of tkey gives each token its time token).
__global__ void change_flags_kernel(const uint8_t* __restrict__ kind, const uint8_t* __restrict__ pre,
                                    const int64_t* __restrict__ tval, int64_t n_tok, uint8_t* __restrict__ is_change,
                                    int64_t* __restrict__ tkey, int32_t* __restrict__ err) {
  for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < n_tok;
       k += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const bool consumed = (pre[k] & 1) != 0;
    const uint8_t kd = kind[k];
    bool ch = !consumed && (kd == kTokScalar || kd == kTokVector);
    if (ch && kd == kTokVector && k + 1 >= n_tok) {  // a vector value without its id
      atomicOr(err, kVcdErrUnknownId);
      ch = false;
    }
    is_change[k] = ch ? 1 : 0;
    tkey[k] = (!consumed && kd == kTokTime) ? k : -1;
    if (!consumed && kd == kTokTime && tval[k] < 0) atomicOr(err, kVcdErrBadTime);
  }
}

// One record per change: id, time, kind and value (scalar: 0, 1, X, Z, U as
// 0..4, kept apart so that a change from X to U counts as a change, as the
// reference compares characters; vector: the leading binary digits read as
// strtol reads them, LLONG_MAX when they overflow, 0 when the first digit
// is x/u/z).
__global__ void change_records_kernel(const uint8_t* __restrict__ b, const int64_t* __restrict__ start,
                                      const int64_t* __restrict__ tend, const uint8_t* __restrict__ kind,
                                      const int64_t* __restrict__ tval, const int64_t* __restrict__ last_time,
                                      const int64_t* __restrict__ tok, int64_t n_ch, IdTable ids,
                                      int32_t* __restrict__ rec_id, int64_t* __restrict__ rec_time,
                                      int64_t* __restrict__ rec_val, uint8_t* __restrict__ rec_kind,
                                      int32_t* __restrict__ err) {
  for (int64_t j = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; j < n_ch;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t k = tok[j];
    const int64_t s = start[k], e = tend[k];
    const int64_t lt = last_time[k];
    rec_time[j] = lt >= 0 ? tval[lt] : 0;
    const uint8_t kd = kind[k];
    rec_kind[j] = kd;
    int64_t v = 0;
    int32_t id;
    if (kd == kTokScalar) {
      const uint8_t c0 = upper(b[s]);
      v = c0 == '0' ? 0 : (c0 == '1' ? 1 : (c0 == 'X' ? 2 : (c0 == 'Z' ? 3 : 4)));
      id = lookup_id(ids, reinterpret_cast<const char*>(b) + s + 1, e - s - 1);
    } else {
      const uint8_t c1 = e - s > 1 ? upper(b[s + 1]) : '0';
      if (!(c1 == 'X' || c1 == 'U' || c1 == 'Z')) {
        unsigned long long acc = 0;
        bool over = false;
        for (int64_t i = s + 1; i < e; ++i) {
          const uint8_t d = b[i];
          if (d != '0' && d != '1') break;
          if (acc > (static_cast<unsigned long long>(LLONG_MAX) >> 1)) over = true;
          acc = (acc << 1) | static_cast<unsigned long long>(d - '0');
          if (acc > static_cast<unsigned long long>(LLONG_MAX)) over = true;
        }
        v = over ? LLONG_MAX : static_cast<int64_t>(acc);
      }
      const int64_t s2 = start[k + 1], e2 = tend[k + 1];
      id = lookup_id(ids, reinterpret_cast<const char*>(b) + s2, e2 - s2);
    }
    if (id < 0) atomicOr(err, kVcdErrUnknownId);
    rec_id[j] = id < 0 ? INT32_MAX : id;   // unknown ids sort last and are dropped
    rec_val[j] = v;
  }
}

// Over the changes sorted by id (file order within an id): keep a change
// when it starts its id's list or differs from the change before it;
// insert an initial value at tick 0 before an id's first change when that
// is later. cnt[j] = output records of change j (0, 1 or 2).
__global__ void dedup_count_kernel(const int32_t* __restrict__ sid, const int32_t* __restrict__ perm,
                                   const int64_t* __restrict__ rec_time, const int64_t* __restrict__ rec_val,
                                   const uint8_t* __restrict__ rec_kind, int64_t n_ch, int32_t n_id,
                                   int32_t* __restrict__ cnt, int32_t* __restrict__ err) {
  for (int64_t j = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; j < n_ch;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int32_t id = sid[j];
    if (id >= n_id) {
      cnt[j] = 0;
      continue;
    }
    const int32_t r = perm[j];
    const bool first = j == 0 || sid[j - 1] != id;
    int c = 0;
    if (first) {
      c = 1 + (rec_time[r] != 0 ? 1 : 0);
    } else {
      const int32_t q = perm[j - 1];
      if (rec_kind[q] != rec_kind[r]) atomicOr(err, kVcdErrMixedKinds);
      c = rec_val[q] != rec_val[r] ? 1 : 0;
    }
    cnt[j] = c;
  }
}

// Writes the kept records at their positions (pos: exclusive prefix of cnt)
// and each id's first position (id_first[id], -1 when it has none).
__global__ void dedup_fill_kernel(const int32_t* __restrict__ sid, const int32_t* __restrict__ perm,
                                  const int64_t* __restrict__ rec_time, const int64_t* __restrict__ rec_val,
                                  const uint8_t* __restrict__ rec_kind, const int32_t* __restrict__ cnt,
                                  const int64_t* __restrict__ pos, int64_t n_ch, int32_t n_id,
                                  int64_t* __restrict__ st_time, int64_t* __restrict__ st_val,
                                  int64_t* __restrict__ id_first, uint8_t* __restrict__ id_vec) {
  for (int64_t j = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; j < n_ch;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int32_t id = sid[j];
    if (id >= n_id || cnt[j] == 0) continue;
    const int32_t r = perm[j];
    int64_t p = pos[j];
    const bool first = j == 0 || sid[j - 1] != id;
    const bool vec = rec_kind[r] == kTokVector;
    if (first) {
      id_first[id] = p;
      id_vec[id] = vec ? 1 : 0;
      if (cnt[j] == 2) {  // initial X (scalar) or bus value 0 (vector) at tick 0
        st_time[p] = 0;
        st_val[p] = vec ? 0 : 2;
        ++p;
      }
    }
    st_time[p] = rec_time[r];
    st_val[p] = rec_val[r];
  }
}

// id_end[id] = one past the id's last stored record.
__global__ void id_end_kernel(const int32_t* __restrict__ sid, const int32_t* __restrict__ cnt,
                              const int64_t* __restrict__ pos, int64_t n_ch, int32_t n_id,
                              int64_t* __restrict__ id_end) {
  for (int64_t j = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; j < n_ch;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int32_t id = sid[j];
    if (id >= n_id) continue;
    if (j + 1 == n_ch || sid[j + 1] != id) id_end[id] = pos[j] + cnt[j];
  }
}

__global__ void iota_kernel(int32_t* __restrict__ a, int64_t n) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    a[i] = static_cast<int32_t>(i);
}

// Per source (id, bit): its stored event count (scnt[n_src] = 0, the end
// of the prefix).
__global__ void source_count_kernel(const int32_t* __restrict__ src_id, int32_t n_src,
                                    const int64_t* __restrict__ id_first, const int64_t* __restrict__ id_end,
                                    int64_t* __restrict__ scnt) {
  const int32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s > n_src) return;
  if (s == n_src) {
    scnt[s] = 0;
    return;
  }
  const int32_t id = src_id[s];
  scnt[s] = (id >= 0 && id_first[id] >= 0) ? id_end[id] - id_first[id] : 0;
}

// One thread per 16 output events (one packed value word): times and 2-bit
// values of the sources' events.
__global__ void source_fill_kernel(const int32_t* __restrict__ src_id, const int32_t* __restrict__ src_bit,
                                   int32_t n_src, const int64_t* __restrict__ net_off,
                                   const int64_t* __restrict__ id_first, const uint8_t* __restrict__ id_vec,
                                   const int64_t* __restrict__ st_time, const int64_t* __restrict__ st_val,
                                   int64_t n_ev, int64_t* __restrict__ time, uint32_t* __restrict__ packed) {
  const int64_t n_words = (n_ev + 15) / 16;
  for (int64_t w = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; w < n_words;
       w += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t i0 = 16 * w;
    // source of event i0: the last s with net_off[s] <= i0
    int32_t lo = 0, hi = n_src;
    while (hi - lo > 1) {
      const int32_t m = lo + ((hi - lo) >> 1);
      if (net_off[m] <= i0) lo = m; else hi = m;
    }
    int32_t s = lo;
    uint32_t word = 0;
    for (int64_t i = i0; i < i0 + 16 && i < n_ev; ++i) {
      while (i >= net_off[s + 1]) ++s;
      const int32_t id = src_id[s];
      const int64_t q = id_first[id] + (i - net_off[s]);
      time[i] = st_time[q];
      uint32_t v;
      if (id_vec[id]) {
        const int32_t bit = src_bit[s];
        v = (bit >= 0 && bit < 64) ? static_cast<uint32_t>((static_cast<unsigned long long>(st_val[q]) >> bit) & 1ull)
                                   : 0u;
      } else {
        v = st_val[q] == 4 ? 2u : static_cast<uint32_t>(st_val[q]) & 3u;   // U reads as X
      }
      word |= v << (2 * (i - i0));
    }
    packed[w] = word;
  }
}

int grid_for(int64_t n) { return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 16))); }

}  // namespace

struct gtp_vcd {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  int32_t n_id = 0, n_src = 0;
  // id table and sources (device)
  unsigned long long* d_hash = nullptr;
  int32_t* d_index = nullptr;
  uint64_t mask = 0;
  char* d_chars = nullptr;
  int32_t* d_off = nullptr;
  int32_t* d_src_id = nullptr;
  int32_t* d_src_bit = nullptr;
  // outputs of the last parse (in scratch)
  int64_t* d_net_off = nullptr;
  int64_t* d_time = nullptr;
  uint32_t* d_packed = nullptr;
  int64_t n_event = 0, time_max = 0;
  int64_t n_token = 0, n_change = 0;
  std::vector<void*> scratch;   // freed at the next parse
};

namespace {

template <typename T>
cudaError_t dmalloc(gtp_vcd* v, T** p, int64_t n) {
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), sizeof(T) * static_cast<size_t>(std::max<int64_t>(1, n)));
  if (e == cudaSuccess) v->scratch.push_back(*p);
  return e;
}

void free_scratch(gtp_vcd* v) {
  for (void* p : v->scratch) cudaFree(p);
  v->scratch.clear();
  v->d_net_off = nullptr;
  v->d_time = nullptr;
  v->d_packed = nullptr;
}

gtp_status vfail(gtp_vcd* v, cudaError_t e, const char* what) {
  v->err = std::string(what) + ": " + cudaGetErrorString(e);
  return e == cudaErrorMemoryAllocation ? GTP_ENOMEM : GTP_ECUDA;
}

}  // namespace

extern "C" {

void gtp_vcd_destroy(gtp_vcd* v) {
  if (!v) return;
  if (v->stream) cudaStreamSynchronize(v->stream);
  free_scratch(v);
  void* ps[] = {v->d_hash, v->d_index, v->d_chars, v->d_off, v->d_src_id, v->d_src_bit};
  for (void* p : ps)
    if (p) cudaFree(p);
  if (v->stream) cudaStreamDestroy(v->stream);
  delete v;
}

gtp_status gtp_vcd_create(const char* id_chars, const int32_t* id_off, int32_t n_id, const int32_t* src_id,
                          const int32_t* src_bit, int32_t n_src, int32_t device, gtp_vcd** out) {
  if (!out || n_id < 0 || n_src < 0 || (n_id > 0 && (!id_chars || !id_off)) || (n_src > 0 && (!src_id || !src_bit)))
    return GTP_EINVAL;
  *out = nullptr;
  for (int32_t s = 0; s < n_src; ++s)
    if (src_id[s] < 0 || src_id[s] >= n_id) return GTP_EINVAL;
  for (int32_t i = 0; i < n_id; ++i)
    if (id_off[i + 1] < id_off[i]) return GTP_EINVAL;
  gtp_vcd* v = new gtp_vcd();
  if (device >= 0 && cudaSetDevice(device) != cudaSuccess) { delete v; return GTP_ECUDA; }
  cudaGetDevice(&v->device);
  if (cudaStreamCreateWithFlags(&v->stream, cudaStreamNonBlocking) != cudaSuccess) { delete v; return GTP_ECUDA; }
  v->n_id = n_id;
  v->n_src = n_src;
  // the id table: capacity a power of two at least twice the ids
  uint64_t cap = 16;
  while (cap < 2ull * static_cast<uint64_t>(n_id) + 1) cap <<= 1;
  std::vector<unsigned long long> hash(cap, kEmptySlot);
  std::vector<int32_t> index(cap, -1);
  for (int32_t i = 0; i < n_id; ++i) {
    const uint64_t h = fnv1a(id_chars + id_off[i], id_off[i + 1] - id_off[i]);
    uint64_t s = h & (cap - 1);
    bool dup = false;  // a repeated id string keeps its first entry
    while (hash[s] != kEmptySlot) {
      const int32_t j = index[s];
      if (hash[s] == h && id_off[j + 1] - id_off[j] == id_off[i + 1] - id_off[i] &&
          std::equal(id_chars + id_off[j], id_chars + id_off[j + 1], id_chars + id_off[i])) {
        dup = true;
        break;
      }
      s = (s + 1) & (cap - 1);
    }
    if (!dup) {
      hash[s] = h;
      index[s] = i;
    }
  }
  v->mask = cap - 1;
  const size_t n_chars = static_cast<size_t>(n_id > 0 ? id_off[n_id] : 0);
  cudaError_t e = cudaMalloc(&v->d_hash, sizeof(unsigned long long) * cap);
  if (e == cudaSuccess) e = cudaMalloc(&v->d_index, sizeof(int32_t) * cap);
  if (e == cudaSuccess) e = cudaMalloc(&v->d_chars, std::max<size_t>(1, n_chars));
  if (e == cudaSuccess) e = cudaMalloc(&v->d_off, sizeof(int32_t) * (n_id + 1));
  if (e == cudaSuccess) e = cudaMalloc(&v->d_src_id, sizeof(int32_t) * std::max(1, n_src));
  if (e == cudaSuccess) e = cudaMalloc(&v->d_src_bit, sizeof(int32_t) * std::max(1, n_src));
  if (e == cudaSuccess) e = cudaMemcpy(v->d_hash, hash.data(), sizeof(unsigned long long) * cap, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(v->d_index, index.data(), sizeof(int32_t) * cap, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && n_chars > 0) e = cudaMemcpy(v->d_chars, id_chars, n_chars, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && n_id > 0) e = cudaMemcpy(v->d_off, id_off, sizeof(int32_t) * (n_id + 1), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && n_src > 0) e = cudaMemcpy(v->d_src_id, src_id, sizeof(int32_t) * n_src, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && n_src > 0) e = cudaMemcpy(v->d_src_bit, src_bit, sizeof(int32_t) * n_src, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    gtp_vcd_destroy(v);
    return e == cudaErrorMemoryAllocation ? GTP_ENOMEM : GTP_ECUDA;
  }
  *out = v;
  return GTP_OK;
}

const char* gtp_vcd_last_error(const gtp_vcd* v) { return v ? v->err.c_str() : "null VCD reader"; }

gtp_status gtp_vcd_stats(const gtp_vcd* v, int64_t* n_token, int64_t* n_change) {
  if (!v) return GTP_EINVAL;
  if (n_token) *n_token = v->n_token;
  if (n_change) *n_change = v->n_change;
  return GTP_OK;
}

gtp_status gtp_vcd_fetch(gtp_vcd* v, int64_t* net_off, int64_t* time, uint32_t* packed) {
  if (!v) return GTP_EINVAL;
  cudaError_t e = cudaSuccess;
  if (net_off && v->d_net_off)
    e = cudaMemcpyAsync(net_off, v->d_net_off, sizeof(int64_t) * (v->n_src + 1), cudaMemcpyDeviceToHost, v->stream);
  if (e == cudaSuccess && time && v->d_time && v->n_event > 0)
    e = cudaMemcpyAsync(time, v->d_time, sizeof(int64_t) * v->n_event, cudaMemcpyDeviceToHost, v->stream);
  if (e == cudaSuccess && packed && v->d_packed && v->n_event > 0)
    e = cudaMemcpyAsync(packed, v->d_packed, sizeof(uint32_t) * ((v->n_event + 15) / 16), cudaMemcpyDeviceToHost,
                        v->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(v->stream);
  return e == cudaSuccess ? GTP_OK : vfail(v, e, "gtp_vcd_fetch");
}

}  // extern "C"

extern "C" gtp_status gtp_vcd_parse(gtp_vcd* v, const char* body, int64_t n, gtp_events* d_out, int64_t* time_max) {
  if (!v || !d_out || n < 0 || (n > 0 && !body)) return GTP_EINVAL;
  if (n >= (int64_t(1) << 40)) { v->err = "VCD body too large"; return GTP_EOVERFLOW; }
  cudaError_t e = cudaSetDevice(v->device);
  if (e != cudaSuccess) return vfail(v, e, "device");
  if (v->stream) cudaStreamSynchronize(v->stream);
  free_scratch(v);
  v->n_event = v->time_max = v->n_token = v->n_change = 0;
  cudaStream_t st = v->stream;
#define VCHK(call, what) do { e = (call); if (e != cudaSuccess) return vfail(v, e, what); } while (0)
  uint8_t* d_b = nullptr;
  int32_t* d_err = nullptr;
  int64_t* d_cnt1 = nullptr;   // counts written by device selects
  VCHK(dmalloc(v, &d_b, n), "body buffer");
  VCHK(dmalloc(v, &d_err, 1), "status");
  VCHK(dmalloc(v, &d_cnt1, 2), "counts");
  if (n > 0) VCHK(cudaMemcpyAsync(d_b, body, static_cast<size_t>(n), cudaMemcpyHostToDevice, st), "body copy");
  VCHK(cudaMemsetAsync(d_err, 0, sizeof(int32_t), st), "status");
  auto temp = [&](size_t bytes, void** out) -> cudaError_t {
    char* t = nullptr;
    cudaError_t r = dmalloc(v, &t, static_cast<int64_t>(bytes));
    *out = t;
    return r;
  };
  // 1. token starts
  uint8_t* d_flags = nullptr;
  int64_t* d_start = nullptr;
  VCHK(dmalloc(v, &d_flags, n), "token flags");
  VCHK(dmalloc(v, &d_start, n / 2 + 1), "token starts");
  int64_t n_tok = 0;
  if (n > 0) {
    token_flags_kernel<<<grid_for(n), 256, 0, st>>>(d_b, n, d_flags);
    VCHK(cudaGetLastError(), "token flags");
    thrust::counting_iterator<int64_t> it(0);
    size_t tb = 0;
    void* t = nullptr;
    VCHK(cub::DeviceSelect::Flagged(nullptr, tb, it, d_flags, d_start, d_cnt1, n, st), "select");
    VCHK(temp(tb, &t), "select temp");
    VCHK(cub::DeviceSelect::Flagged(t, tb, it, d_flags, d_start, d_cnt1, n, st), "select");
    VCHK(cudaMemcpyAsync(&n_tok, d_cnt1, sizeof(int64_t), cudaMemcpyDeviceToHost, st), "count");
    VCHK(cudaStreamSynchronize(st), "sync");
  }
  v->n_token = n_tok;
  // 2. token kinds and times; the ids that vector and real tokens consume
  uint8_t *d_kind = nullptr, *d_step = nullptr, *d_fn = nullptr, *d_pre = nullptr, *d_isch = nullptr;
  int64_t *d_tend = nullptr, *d_tval = nullptr, *d_tkey = nullptr, *d_last = nullptr, *d_tok = nullptr;
  VCHK(dmalloc(v, &d_kind, n_tok), "tokens");
  VCHK(dmalloc(v, &d_step, n_tok), "tokens");
  VCHK(dmalloc(v, &d_fn, n_tok), "tokens");
  VCHK(dmalloc(v, &d_pre, n_tok), "tokens");
  VCHK(dmalloc(v, &d_isch, n_tok), "tokens");
  VCHK(dmalloc(v, &d_tend, n_tok), "tokens");
  VCHK(dmalloc(v, &d_tval, n_tok), "tokens");
  VCHK(dmalloc(v, &d_tkey, n_tok), "tokens");
  VCHK(dmalloc(v, &d_last, n_tok), "tokens");
  VCHK(dmalloc(v, &d_tok, n_tok), "changes");
  int64_t n_ch = 0;
  if (n_tok > 0) {
    token_kind_kernel<<<grid_for(n_tok), 256, 0, st>>>(d_b, n, d_start, n_tok, d_kind, d_tend, d_tval, d_step);
    step_fn_kernel<<<grid_for(n_tok), 256, 0, st>>>(d_step, n_tok, d_fn);
    VCHK(cudaGetLastError(), "token kinds");
    size_t tb = 0;
    void* t = nullptr;
    const uint8_t ident = 2;  // the identity: f(0) = 0, f(1) = 1
    VCHK(cub::DeviceScan::ExclusiveScan(nullptr, tb, d_fn, d_pre, StepCompose(), ident, n_tok, st), "id scan");
    VCHK(temp(tb, &t), "id scan temp");
    VCHK(cub::DeviceScan::ExclusiveScan(t, tb, d_fn, d_pre, StepCompose(), ident, n_tok, st), "id scan");
    change_flags_kernel<<<grid_for(n_tok), 256, 0, st>>>(d_kind, d_pre, d_tval, n_tok, d_isch, d_tkey, d_err);
    VCHK(cudaGetLastError(), "change flags");
    tb = 0;
    VCHK(cub::DeviceScan::InclusiveScan(nullptr, tb, d_tkey, d_last, MaxOp(), n_tok, st), "time scan");
    VCHK(temp(tb, &t), "time scan temp");
    VCHK(cub::DeviceScan::InclusiveScan(t, tb, d_tkey, d_last, MaxOp(), n_tok, st), "time scan");
    thrust::counting_iterator<int64_t> it(0);
    tb = 0;
    VCHK(cub::DeviceSelect::Flagged(nullptr, tb, it, d_isch, d_tok, d_cnt1 + 1, n_tok, st), "select");
    VCHK(temp(tb, &t), "select temp");
    VCHK(cub::DeviceSelect::Flagged(t, tb, it, d_isch, d_tok, d_cnt1 + 1, n_tok, st), "select");
    VCHK(cudaMemcpyAsync(&n_ch, d_cnt1 + 1, sizeof(int64_t), cudaMemcpyDeviceToHost, st), "count");
    int64_t last_key = -1;
    VCHK(cudaMemcpyAsync(&last_key, d_last + n_tok - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, st), "time");
    VCHK(cudaStreamSynchronize(st), "sync");
    if (last_key >= 0) {
      VCHK(cudaMemcpyAsync(&v->time_max, d_tval + last_key, sizeof(int64_t), cudaMemcpyDeviceToHost, st), "time");
      VCHK(cudaStreamSynchronize(st), "sync");
    }
  }
  if (n_ch >= INT32_MAX) { v->err = "more than 2^31 value changes in one VCD body"; return GTP_EOVERFLOW; }
  v->n_change = n_ch;
  // 3. change records; 4. by id in file order, repeats dropped
  int32_t *d_rid = nullptr, *d_sid = nullptr, *d_iota = nullptr, *d_perm = nullptr, *d_cnt = nullptr;
  int64_t *d_rtime = nullptr, *d_rval = nullptr, *d_pos = nullptr;
  uint8_t* d_rkind = nullptr;
  VCHK(dmalloc(v, &d_rid, n_ch), "changes");
  VCHK(dmalloc(v, &d_sid, n_ch), "changes");
  VCHK(dmalloc(v, &d_iota, n_ch), "changes");
  VCHK(dmalloc(v, &d_perm, n_ch), "changes");
  VCHK(dmalloc(v, &d_cnt, n_ch + 1), "changes");
  VCHK(dmalloc(v, &d_rtime, n_ch), "changes");
  VCHK(dmalloc(v, &d_rval, n_ch), "changes");
  VCHK(dmalloc(v, &d_pos, n_ch + 1), "changes");
  VCHK(dmalloc(v, &d_rkind, n_ch), "changes");
  int64_t *d_first = nullptr, *d_end = nullptr;
  uint8_t* d_vec = nullptr;
  VCHK(dmalloc(v, &d_first, v->n_id), "ids");
  VCHK(dmalloc(v, &d_end, v->n_id), "ids");
  VCHK(dmalloc(v, &d_vec, v->n_id), "ids");
  VCHK(cudaMemsetAsync(d_first, 0xff, sizeof(int64_t) * std::max(1, v->n_id), st), "ids");
  VCHK(cudaMemsetAsync(d_end, 0xff, sizeof(int64_t) * std::max(1, v->n_id), st), "ids");
  VCHK(cudaMemsetAsync(d_vec, 0, std::max(1, v->n_id), st), "ids");
  VCHK(cudaMemsetAsync(d_cnt, 0, sizeof(int32_t) * (n_ch + 1), st), "changes");
  int64_t n_store = 0;
  int64_t* d_stime = nullptr;
  int64_t* d_sval = nullptr;
  if (n_ch > 0) {
    IdTable ids{v->d_hash, v->d_index, v->mask, v->d_chars, v->d_off};
    change_records_kernel<<<grid_for(n_ch), 256, 0, st>>>(d_b, d_start, d_tend, d_kind, d_tval, d_last, d_tok, n_ch,
                                                          ids, d_rid, d_rtime, d_rval, d_rkind, d_err);
    iota_kernel<<<grid_for(n_ch), 256, 0, st>>>(d_iota, n_ch);
    VCHK(cudaGetLastError(), "change records");
    size_t tb = 0;
    void* t = nullptr;
    VCHK(cub::DeviceRadixSort::SortPairs(nullptr, tb, d_rid, d_sid, d_iota, d_perm, n_ch, 0, 31, st), "sort");
    VCHK(temp(tb, &t), "sort temp");
    VCHK(cub::DeviceRadixSort::SortPairs(t, tb, d_rid, d_sid, d_iota, d_perm, n_ch, 0, 31, st), "sort");
    dedup_count_kernel<<<grid_for(n_ch), 256, 0, st>>>(d_sid, d_perm, d_rtime, d_rval, d_rkind, n_ch, v->n_id, d_cnt,
                                                       d_err);
    VCHK(cudaGetLastError(), "dedup");
    tb = 0;
    VCHK(cub::DeviceScan::ExclusiveSum(nullptr, tb, d_cnt, d_pos, n_ch + 1, st), "scan");
    VCHK(temp(tb, &t), "scan temp");
    VCHK(cub::DeviceScan::ExclusiveSum(t, tb, d_cnt, d_pos, n_ch + 1, st), "scan");
    VCHK(cudaMemcpyAsync(&n_store, d_pos + n_ch, sizeof(int64_t), cudaMemcpyDeviceToHost, st), "count");
    VCHK(cudaStreamSynchronize(st), "sync");
    VCHK(dmalloc(v, &d_stime, n_store), "stored values");
    VCHK(dmalloc(v, &d_sval, n_store), "stored values");
    dedup_fill_kernel<<<grid_for(n_ch), 256, 0, st>>>(d_sid, d_perm, d_rtime, d_rval, d_rkind, d_cnt, d_pos, n_ch,
                                                      v->n_id, d_stime, d_sval, d_first, d_vec);
    id_end_kernel<<<grid_for(n_ch), 256, 0, st>>>(d_sid, d_cnt, d_pos, n_ch, v->n_id, d_end);
    VCHK(cudaGetLastError(), "dedup fill");
  }
  // 5. the sources' CSR
  int64_t* d_scnt = nullptr;
  VCHK(dmalloc(v, &d_scnt, v->n_src + 1), "sources");
  VCHK(dmalloc(v, &v->d_net_off, v->n_src + 1), "sources");
  {
    source_count_kernel<<<(v->n_src + 1 + 255) / 256, 256, 0, st>>>(v->d_src_id, v->n_src, d_first, d_end, d_scnt);
    VCHK(cudaGetLastError(), "sources");
    size_t tb = 0;
    void* t = nullptr;
    VCHK(cub::DeviceScan::ExclusiveSum(nullptr, tb, d_scnt, v->d_net_off, v->n_src + 1, st), "scan");
    VCHK(temp(tb, &t), "scan temp");
    VCHK(cub::DeviceScan::ExclusiveSum(t, tb, d_scnt, v->d_net_off, v->n_src + 1, st), "scan");
  }
  int64_t n_ev = 0;
  int32_t h_err = 0;
  VCHK(cudaMemcpyAsync(&n_ev, v->d_net_off + v->n_src, sizeof(int64_t), cudaMemcpyDeviceToHost, st), "count");
  VCHK(cudaMemcpyAsync(&h_err, d_err, sizeof(int32_t), cudaMemcpyDeviceToHost, st), "status");
  VCHK(cudaStreamSynchronize(st), "sync");
  VCHK(dmalloc(v, &v->d_time, n_ev), "events");
  VCHK(dmalloc(v, &v->d_packed, (n_ev + 15) / 16), "events");
  if (n_ev > 0 && v->n_src > 0) {
    source_fill_kernel<<<grid_for((n_ev + 15) / 16), 256, 0, st>>>(v->d_src_id, v->d_src_bit, v->n_src, v->d_net_off,
                                                                    d_first, d_vec, d_stime, d_sval, n_ev, v->d_time,
                                                                    v->d_packed);
    VCHK(cudaGetLastError(), "events");
  }
  VCHK(cudaStreamSynchronize(st), "sync");
#undef VCHK
  if (h_err) {
    v->err = "invalid VCD body:";
    if (h_err & kVcdErrUnknownId) v->err += " a value change names an undeclared id (or a vector value lacks its id);";
    if (h_err & kVcdErrBadTime) v->err += " a time stamp is not a decimal number;";
    if (h_err & kVcdErrMixedKinds) v->err += " an id takes both scalar and vector changes;";
    return GTP_EINVAL;
  }
  v->n_event = n_ev;
  d_out->n_event = n_ev;
  d_out->net_off = v->d_net_off;
  d_out->time = v->d_time;
  d_out->value_packed = v->d_packed;
  d_out->net_base = nullptr;
  d_out->t_lo = 0;
  d_out->t_hi = INT64_MAX;
  if (time_max) *time_max = v->time_max;
  return GTP_OK;
}
