// The event file sink: Prophesee RAW (EVT 2.0, 2.1, 3.0) and DAT files of one camera's events in output order, the
// reference's RawWriter / DatWriter (src/export/raw_writer.h:33-68, raw_writer.cpp; the words of src/export/evt.h
// and dat.h; the T1a time rule of src/export/time_map.h:70-71).
//
// The reference encodes with one streaming state machine per file on one host thread. Every word an event adds
// depends only on that event and the one before it (its time step, address and polarity; EVT 2.1 also on the
// addresses of its open word, at most 32 events back), so here each batch is encoded on the device in three
// passes over the columns, one thread per event:
//   1. check: the first event that breaks the order, the sensor's range, the polarity or the declared sub-us range;
//   2. count: the words each event adds; an exclusive scan gives each event's first word;
//   3. write: each event writes its words at its offset, in output chunks of at most kChunkBytes, each copied out
//      once into pinned memory and appended to the file.
// The encoder state between batches (the last event, EVT 2.1's open word mask) stays on the host, so one append
// and many give the same bytes. Each chunk is hashed (SHA-256, FIPS 180-4) on a second host thread while it is
// written; close() writes EVT 2.1's open word and returns the digest, which is the closed file's: RAW and DAT files
// are written once, never patched (the reference reads the closed file back for the same digest).
#include <cuda_runtime.h>
#include <fcntl.h>
#include <unistd.h>

#include <cerrno>
#include <chrono>
#include <climits>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <cub/device/device_scan.cuh>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <sys/stat.h>

#include <system_error>
#include <thread>
#include <vector>

#include "../../include/ballasim_b200.h"
#include "sha256.h"

namespace bs {

void set_last_error(const char* msg);  // model.cu: the message bs_last_error() returns

namespace sink {

// The exporters' refusal of their input or options (src/export/errors.h): ExportError in Python.
struct Refused : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct SinkCudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

inline void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw SinkCudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

enum Format : int32_t { kEvt2OpenEb = 0, kEvt2OnChange = 1, kEvt21 = 2, kEvt3 = 3, kDat = 4 };

constexpr int32_t kEvtMaxDim = 2048;                                // 11-bit addresses of every EVT format
constexpr int32_t kDatMaxDim = 1 << 14;                             // DAT's 14-bit addresses
constexpr int64_t kEvt2MaxFirstU = (int64_t{1} << 34) - 1;          // EVT 2.0/2.1's first TIME_HIGH is absolute
constexpr int64_t kDatMaxU = (int64_t{1} << 32) - 1;                // DAT's u32 microseconds
constexpr int64_t kKeepaliveSteps = 128;                            // on-change TIME_HIGH keepalive (8.192 ms)
constexpr int64_t kWrapSteps = int64_t{1} << 28;                    // the 28-bit TIME_HIGH value's wrap
constexpr size_t kChunkBytes = size_t{64} << 20;                    // one output chunk (device and pinned)

__host__ __device__ inline int64_t floor_div(int64_t a, int64_t b) {
  const int64_t q = a / b;
  return (a % b < 0) ? q - 1 : q;
}

// T1a: microseconds after the export origin, the sub-microsecond part dropped.
__host__ __device__ inline int64_t t1a_us(int64_t t_ns, int64_t origin_us) { return floor_div(t_ns, 1000) - origin_us; }

// The encoder's state after the last event of the stream: that event, and EVT 2.1's open word mask.
struct Prev {
  int32_t started;
  uint32_t x, y, p;
  int64_t u, t;
  uint32_t mask;
};

struct Cols {
  const uint16_t* x;
  const uint16_t* y;
  const uint8_t* p;
  const int64_t* t;
  uint32_t n;
};

struct Args {
  int32_t format;
  int32_t width, height, rem_min, rem_max;
  int64_t origin_us;
  Prev prev;
  Cols c;
};

// What the host reads back after the counts: the first bad event with its predecessor's time, the first and last
// times, the last event's address and polarity, and EVT 2.1's open word mask after the batch.
struct Info {
  unsigned long long first_bad;
  int64_t t_first, t_last, bad_t, bad_t_prev;
  uint32_t bad_x, bad_y, bad_p, tail_mask;
  uint32_t last_x, last_y, last_p;
};

struct Ev {
  int64_t u;
  uint32_t x, y, p;
};

__device__ inline Ev ev_at(const Args& a, uint32_t i) {
  return {t1a_us(a.c.t[i], a.origin_us), a.c.x[i], a.c.y[i], a.c.p[i]};
}

// The event before i (the batch's, or the last one written): false at the stream's first event.
__device__ inline bool prev_of(const Args& a, uint32_t i, Ev& q) {
  if (i > 0) {
    q = ev_at(a, i - 1);
    return true;
  }
  q = {a.prev.u, a.prev.x, a.prev.y, a.prev.p};
  return a.prev.started != 0;
}

// EVT 2.1 (evt.h:121-129): an event joins its predecessor's open word when (t, y, p, the x base) match and its x is
// greater; the word's last x is always the predecessor's.
__device__ inline bool joins(const Ev& e, const Ev& q) {
  return e.u == q.u && e.y == q.y && e.p == q.p && (e.x & ~31u) == (q.x & ~31u) && e.x > q.x;
}

// The valid mask of EVT 2.1's open word that ends at event i - 1 (its events, back to the one that opened it, or
// the open word carried from earlier batches).
__device__ inline uint32_t mask_before(const Args& a, uint32_t i) {
  uint32_t m = 0;
  for (uint32_t j = i; j-- > 0;) {
    const Ev e = ev_at(a, j);
    m |= 1u << (e.x & 31u);
    Ev q;
    const bool started = prev_of(a, j, q);
    if (!(started && joins(e, q))) return m;
    if (j == 0) return m | a.prev.mask;
  }
  return a.prev.mask;
}

__host__ __device__ inline uint32_t th32(int64_t step64) {
  return 0x80000000u | static_cast<uint32_t>(step64 & 0x0FFFFFFF);
}
__host__ __device__ inline uint64_t th64(int64_t step64) {
  return (uint64_t{0x8} << 60) | (static_cast<uint64_t>(step64 & 0x0FFFFFFF) << 32);
}
__host__ __device__ inline uint64_t cd21(int64_t u, uint32_t x, uint32_t y, uint32_t p, uint32_t mask) {
  return (uint64_t{p} << 60) | (static_cast<uint64_t>(u & 63) << 54) | (uint64_t{x & ~31u} << 43) |
         (uint64_t{y} << 32) | mask;
}
__device__ inline uint64_t word3(uint32_t type, uint32_t content) { return (type << 12) | content; }

// Counting pass: the words an event adds.
struct CountOut {
  unsigned long long n = 0;
  __device__ void put(uint64_t) { ++n; }
  __device__ unsigned long long skippable() const { return ULLONG_MAX; }
  __device__ void skip(unsigned long long k) { n += k; }
  __device__ bool done() const { return false; }
};

// Writing pass: the words of stream positions [w0, w1) into buf (word size ws bytes).
struct WriteOut {
  unsigned long long pos, w0, w1;
  uint8_t* buf;
  int32_t ws;
  __device__ void put(uint64_t v) {
    if (pos >= w0 && pos < w1) {
      const unsigned long long k = pos - w0;
      if (ws == 2) {
        reinterpret_cast<uint16_t*>(buf)[k] = static_cast<uint16_t>(v);
      } else if (ws == 4) {
        reinterpret_cast<uint32_t*>(buf)[k] = static_cast<uint32_t>(v);
      } else {
        reinterpret_cast<uint64_t*>(buf)[k] = v;
      }
    }
    ++pos;
  }
  __device__ unsigned long long skippable() const { return pos < w0 ? w0 - pos : 0; }
  __device__ void skip(unsigned long long k) { pos += k; }
  __device__ bool done() const { return pos >= w1; }
};

// One word per step of [from, to] (none when to < from), skipping the ones before the output range.
template <class Out, class Word>
__device__ void steps(Out& o, int64_t from, int64_t to, Word word) {
  if (to < from) return;
  const unsigned long long n = static_cast<unsigned long long>(to - from) + 1;
  const unsigned long long s = o.skippable() < n ? o.skippable() : n;
  o.skip(s);
  for (int64_t st = from + static_cast<int64_t>(s); st <= to && !o.done(); ++st) o.put(word(st));
}

// The on-change TIME_HIGH steps before an event in 64 us step k (evt.h:31-66): the keepalive multiples of 128 after
// the last emitted step L and below k, then k; with the wrap guard (EVT 2.1) a step that starts a 2^28-step block
// is preceded by the block's last step unless that was the last one emitted. The keepalives between two block
// starts are one word each, taken as one run (steps() skips what lies before the output range), so a gap of any
// length costs one iteration per 2^28-step block.
template <class Out, class Word>
__device__ void on_change(Out& o, bool started, int64_t L, int64_t k, bool wrap, Word word) {
  if (started && k <= L) return;
  if (!started) {  // the stream's first TIME_HIGH
    o.put(word(k));
    return;
  }
  const int64_t base = (L / kKeepaliveSteps + 1) * kKeepaliveSteps;  // the first keepalive
  const int64_t K = k > base ? (k - 1 - base) / kKeepaliveSteps + 1 : 0;  // keepalives base + 128 s, s < K
  int64_t s = 0;
  while (s < K && !o.done()) {
    const int64_t m = base + kKeepaliveSteps * s;
    if (wrap && m % kWrapSteps == 0) {  // a block's first step: its guard unless the last one emitted is m - 1
      if (!(s == 0 && m - 1 == L)) o.put(word(m - 1));
      o.put(word(m));
      ++s;
      continue;
    }
    int64_t end = K;  // the run of plain keepalives up to the next block start
    if (wrap) {
      const int64_t g = (m / kWrapSteps + 1) * kWrapSteps;
      end = (g - base) / kKeepaliveSteps < K ? (g - base) / kKeepaliveSteps : K;
    }
    steps(o, s, end - 1, [&](int64_t j) { return word(base + kKeepaliveSteps * j); });
    s = end;
  }
  if (o.done()) return;
  const int64_t last = K > 0 ? base + kKeepaliveSteps * (K - 1) : L;
  if (wrap && k % kWrapSteps == 0 && k - 1 > last) o.put(word(k - 1));
  o.put(word(k));
}

// The words of event i (evt.h:68-171, dat.h:18-22), in stream order.
template <class Out>
__device__ void encode(const Args& a, uint32_t i, Out& o) {
  const Ev e = ev_at(a, i);
  Ev q;
  const bool started = prev_of(a, i, q);
  switch (a.format) {
    case kDat:
      o.put(static_cast<uint32_t>(e.u));
      o.put(e.x | (e.y << 14) | (e.p << 28));
      return;
    case kEvt2OpenEb: {
      // A TIME_HIGH every 16 us step from the first event's step, each before the first event at or after it.
      const int64_t k = e.u >> 4;
      steps(o, started ? (q.u >> 4) + 1 : k, k, [](int64_t st) { return uint64_t{th32(st >> 2)}; });
      o.put((e.p << 28) | (static_cast<uint32_t>(e.u & 63) << 22) | (e.x << 11) | e.y);
      return;
    }
    case kEvt2OnChange:
      on_change(o, started, started ? q.u >> 6 : 0, e.u >> 6, false, [](int64_t st) { return uint64_t{th32(st)}; });
      o.put((e.p << 28) | (static_cast<uint32_t>(e.u & 63) << 22) | (e.x << 11) | e.y);
      return;
    case kEvt21:
      if (started && joins(e, q)) return;
      if (started) o.put(cd21(q.u, q.x, q.y, q.p, mask_before(a, i)));
      on_change(o, started, started ? q.u >> 6 : 0, e.u >> 6, true, [](int64_t st) { return th64(st); });
      return;
    case kEvt3: {
      // TIME_HIGH at every 4096 us step from u = 0 (the stream's first event) or from the last one; TIME_LOW when
      // t changes; ADDR_Y when y changes; ADDR_X (with the polarity) per event.
      const int64_t hi = e.u >> 12;
      steps(o, started ? (q.u >> 12) + 1 : 0, hi,
            [](int64_t h) { return word3(0x8, static_cast<uint32_t>(h & 0xFFF)); });
      if (!started || e.u != q.u) o.put(word3(0x6, static_cast<uint32_t>(e.u & 0xFFF)));
      if (!started || e.y != q.y) o.put(word3(0x0, e.y));
      o.put(word3(0x2, (e.p << 11) | e.x));
      return;
    }
    default:
      return;
  }
}

// The rules of one event (raw_writer.cpp:91-117): order, range, polarity and the declared sub-us part.
__device__ inline bool bad_event(const Args& a, uint32_t i) {
  const int64_t t = a.c.t[i];
  const int64_t tp = i > 0 ? a.c.t[i - 1] : (a.prev.started ? a.prev.t : INT64_MIN);
  const int64_t rem = t - 1000 * floor_div(t, 1000);
  return t < tp || a.c.x[i] >= a.width || a.c.y[i] >= a.height || a.c.p[i] > 1 || rem < a.rem_min ||
         rem > a.rem_max;
}

// One thread: the batch's ends, the first bad event's columns and EVT 2.1's open word mask after the batch.
__global__ void info_kernel(Args a, const unsigned long long* first_bad, Info* info) {
  Info r{};
  r.first_bad = *first_bad;
  r.t_first = a.c.t[0];
  r.t_last = a.c.t[a.c.n - 1];
  r.last_x = a.c.x[a.c.n - 1];
  r.last_y = a.c.y[a.c.n - 1];
  r.last_p = a.c.p[a.c.n - 1];
  if (r.first_bad < a.c.n) {
    const uint32_t i = static_cast<uint32_t>(r.first_bad);
    r.bad_t = a.c.t[i];
    r.bad_t_prev = i > 0 ? a.c.t[i - 1] : (a.prev.started ? a.prev.t : INT64_MIN);
    r.bad_x = a.c.x[i];
    r.bad_y = a.c.y[i];
    r.bad_p = a.c.p[i];
  } else if (a.format == kEvt21) {
    r.tail_mask = mask_before(a, a.c.n);
  }
  *info = r;
}

// Pass 1: the rules (the first bad event) and the words each event adds (counted whether or not the batch is
// refused: the counts are O(1) per event, or one step per 2^28-step block of an on-change gap).
__global__ void count_kernel(Args a, unsigned long long* words, unsigned long long* first_bad) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > a.c.n) return;
  if (i == a.c.n) {  // the scan's total
    words[i] = 0;
    return;
  }
  if (bad_event(a, i)) atomicMin(first_bad, static_cast<unsigned long long>(i));
  CountOut o;
  encode(a, i, o);
  words[i] = o.n;
}

// The events whose words meet the output range [w0, w1): [range[0], range[1]) by two binary searches over the
// scanned offsets (first, n + 1 entries, non-decreasing).
__global__ void range_kernel(const unsigned long long* first, uint32_t n, unsigned long long w0,
                             unsigned long long w1, uint32_t* range) {
  uint32_t lo = 0, hi = n;  // the last event starting at or before w0
  while (hi - lo > 1) {
    const uint32_t m = lo + (hi - lo) / 2;
    (first[m] <= w0 ? lo : hi) = m;
  }
  uint32_t a = lo, b = n;  // the first event starting at or after w1
  while (a < b) {
    const uint32_t m = a + (b - a) / 2;
    if (first[m] < w1) {
      a = m + 1;
    } else {
      b = m;
    }
  }
  range[0] = lo;
  range[1] = a;
}

// Pass 2: the words of the events in range (range_kernel) that fall in [w0, w1).
__global__ void write_kernel(Args a, const unsigned long long* first, const uint32_t* range, unsigned long long w0,
                             unsigned long long w1, int32_t ws, uint8_t* buf) {
  const uint32_t i = range[0] + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= range[1]) return;
  const unsigned long long b = first[i], e = first[i + 1];
  if (e <= w0 || b >= w1 || b == e) return;
  WriteOut o{b, w0, w1, buf, ws};
  encode(a, i, o);
}

[[noreturn]] void io_error(const std::string& what, const std::string& path) {
  throw std::system_error(errno, std::generic_category(), what + " " + path);
}


// "YYYY-MM-DD HH:MM:SS" (UTC, proleptic Gregorian) of the second that holds ns since the Unix epoch, by the
// days-to-civil conversion of H. Hinnant's "chrono-Compatible Low-Level Date Algorithms".
std::string utc_date(int64_t ns) {
  const int64_t s = floor_div(ns, 1000000000);
  const int64_t days = floor_div(s, 86400);
  const int64_t sec = s - 86400 * days;
  const int64_t z = days + 719468;
  const int64_t era = floor_div(z, 146097);
  const int64_t doe = z - era * 146097;
  const int64_t yoe = (doe - doe / 1460 + doe / 36524 - doe / 146096) / 365;
  const int64_t doy = doe - (365 * yoe + yoe / 4 - yoe / 100);
  const int64_t mp = (5 * doy + 2) / 153;
  const int64_t d = doy - (153 * mp + 2) / 5 + 1;
  const int64_t m = mp < 10 ? mp + 3 : mp - 9;
  const int64_t y = yoe + era * 400 + (m <= 2 ? 1 : 0);
  char buf[64];
  const int n = std::snprintf(buf, sizeof buf, "%04d-%02d-%02d %02d:%02d:%02d", static_cast<int>(y),
                              static_cast<int>(m), static_cast<int>(d), static_cast<int>(sec / 3600),
                              static_cast<int>(sec / 60 % 60), static_cast<int>(sec % 60));
  return std::string(buf, static_cast<size_t>(n));
}

// ---------------------------------------------------------------------------------------------------------------
// The writer
// ---------------------------------------------------------------------------------------------------------------

void need_device() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    throw SinkCudaError("no CUDA device: the event sink encodes on the GPU (there is no CPU path)");
  }
}

template <class T>
struct DBuf {
  T* p = nullptr;
  size_t cap = 0;
  ~DBuf() {
    if (p) cudaFree(p);
  }
  T* ensure(size_t n) {
    if (n <= cap) return p;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    ck(cudaMalloc(&p, n * sizeof(T)), "event sink: device allocation");
    cap = n;
    return p;
  }
};

// A writer's device and pinned buffers, its stream and timing events. A closed writer leaves its set for the next
// one of the process (one spare, per device), so that a file per camera and run does not pay the allocations again.
struct Scratch {
  int device = -1;
  DBuf<unsigned long long> scalars, counts, offsets;
  DBuf<Info> info;
  DBuf<uint8_t> temp, words, stage;
  uint8_t* pin = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  ~Scratch() {
    for (cudaEvent_t e : ev) {
      if (e) cudaEventDestroy(e);
    }
    if (pin) cudaFreeHost(pin);
    if (stream) cudaStreamDestroy(stream);
  }
};

std::mutex g_spare_mutex;
Scratch* g_spare = nullptr;  // released by the process's exit

Scratch* take_scratch() {
  int dev = 0;
  ck(cudaGetDevice(&dev), "event sink: device");
  {
    std::lock_guard<std::mutex> lock(g_spare_mutex);
    if (g_spare && g_spare->device == dev) {
      Scratch* s = g_spare;
      g_spare = nullptr;
      return s;
    }
  }
  auto* s = new Scratch;
  s->device = dev;
  for (cudaEvent_t& e : s->ev) ck(cudaEventCreate(&e), "event sink: event");
  return s;
}

void give_scratch(Scratch* s) {
  if (!s) return;
  std::lock_guard<std::mutex> lock(g_spare_mutex);
  if (!g_spare) {
    g_spare = s;
  } else {
    delete s;
  }
}

class Writer {
 public:
  Writer(const char* what, const std::string& path, int32_t format, int32_t width, int32_t height, int64_t origin_us,
         int64_t epoch_ns, int32_t rem_min, int32_t rem_max, const std::string& version)
      : what_(what), path_(path), format_(format), width_(width), height_(height), origin_(origin_us),
        rem_min_(rem_min), rem_max_(rem_max) {
    const int32_t max_dim = format == kDat ? kDatMaxDim : kEvtMaxDim;
    if (width < 1 || height < 1 || width > max_dim || height > max_dim) {
      throw Refused(what_ + ": width and height must be in [1, " + std::to_string(max_dim) + "], got " +
                    std::to_string(width) + " x " + std::to_string(height));
    }
    if (epoch_ns % 1000 != 0) {
      throw Refused("epoch_ns = " + std::to_string(epoch_ns) + ": must be a multiple of 1000 (every format)");
    }
    int64_t origin_ns = 0, at = 0;
    if (__builtin_mul_overflow(origin_us, int64_t{1000}, &origin_ns) ||
        __builtin_add_overflow(origin_ns, epoch_ns, &at)) {
      throw Refused("epoch_ns + 1000 origin_us overflows int64");
    }
    const bool none = rem_min == -1 && rem_max == -1;
    if (!none && !(0 <= rem_min && rem_min <= rem_max && rem_max <= 999)) {
      throw Refused(what_ + ": t_ns_rem range [" + std::to_string(rem_min) + ", " + std::to_string(rem_max) +
                    "] must lie in [0, 999] (or be -1, -1 for no events)");
    }
    for (const char c : version) {
      if (c < 0x20 || c > 0x7E) throw Refused(what_ + ": version must be printable ASCII");
    }
    max_u_ = format == kDat ? kDatMaxU : INT64_MAX;
    max_first_u_ = (format == kEvt2OpenEb || format == kEvt2OnChange || format == kEvt21) ? kEvt2MaxFirstU : INT64_MAX;
    word_bytes_ = format == kEvt3 ? 2 : format == kEvt21 ? 8 : 4;
    // The header: '% key value' lines (RAW, raw_writer.cpp:53-62) or OpenEB's DAT lines, type and size
    // (:64-72), each with the T1a keys of the origin, the epoch and the dropped sub-us parts.
    const std::string rem = none ? "none" : rem_min == rem_max ? std::to_string(rem_min) : "varies";
    const std::string t1a = "% ballasim_t_offset_us " + std::to_string(origin_us) + "\n% ballasim_epoch_ns " +
                            std::to_string(epoch_ns) + "\n% ballasim_t_ns_rem " + rem + "\n";
    const std::string date = utc_date(epoch_ns + 1000 * origin_us);
    std::string h;
    if (format == kDat) {
      h = "% Data file containing CD events.\n% Version 2\n% Date " + date + "\n% Height " + std::to_string(height) +
          "\n% Width " + std::to_string(width) + "\n" + t1a;
      h.push_back(static_cast<char>(0x0C));  // CD events
      h.push_back(static_cast<char>(8));     // of 8 bytes
    } else {
      const char* name = format == kEvt21 ? "EVT21" : format == kEvt3 ? "EVT3" : "EVT2";
      std::string v = "BallaSim";
      if (!version.empty()) v += " " + version;
      h = std::string("% format ") + name + ";height=" + std::to_string(height) + ";width=" + std::to_string(width) +
          "\n% camera_integrator_name BallaSim\n% plugin_integrator_name BallaSim\n% plugin_version " + v +
          "\n% date " + date + "\n" + t1a + "% end\n";
    }
    fd_ = ::open(path.c_str(), O_WRONLY | O_CREAT | O_TRUNC | O_CLOEXEC, 0644);
    if (fd_ < 0) io_error("cannot create", path);
    write_bytes(h.data(), h.size());
  }

  ~Writer() {
    if (fd_ >= 0) ::close(fd_);
    give_scratch(sc_);
  }

  // A batch of device columns in output order; refused whole (nothing written) when any event breaks a rule.
  void append_device(const uint16_t* x, const uint16_t* y, const uint8_t* p, const int64_t* t, size_t n,
                     cudaStream_t s) {
    const auto t_begin = std::chrono::steady_clock::now();
    if (closed_) throw Refused(what_ + ": append after close");
    if (n == 0) return;
    if (!x || !y || !p || !t) throw std::invalid_argument(what_ + ": null event columns");
    if (n >= (size_t{1} << 32) - 1) throw std::invalid_argument(what_ + ": at most 2^32 - 2 events per batch");
    need_device();
    Args a{format_, width_, height_, rem_min_, rem_max_, origin_, prev_, Cols{x, y, p, t, static_cast<uint32_t>(n)}};
    const int block = 256;
    const unsigned grid = static_cast<unsigned>((n + block) / block);
    if (!sc_) sc_ = take_scratch();
    Scratch& sc = *sc_;
    unsigned long long* bad = sc.scalars.ensure(2);
    uint32_t* range = reinterpret_cast<uint32_t*>(bad + 1);
    Info* info = sc.info.ensure(1);
    unsigned long long* cnt = sc.counts.ensure(n + 1);
    unsigned long long* first = sc.offsets.ensure(n + 1);
    // Pass 1 (the rules and the word counts), the batch's info, the scan; one read-back.
    ck(cudaMemsetAsync(bad, 0xFF, sizeof(unsigned long long), s), "event sink: memset");
    ck(cudaEventRecord(sc.ev[0], s), "event sink: event");
    count_kernel<<<grid, block, 0, s>>>(a, cnt, bad);
    info_kernel<<<1, 1, 0, s>>>(a, bad, info);
    ck(cudaGetLastError(), "event sink: count launch");
    size_t temp_bytes = 0;
    ck(cub::DeviceScan::ExclusiveSum(nullptr, temp_bytes, cnt, first, static_cast<int64_t>(n + 1), s), "scan");
    uint8_t* temp = sc.temp.ensure(temp_bytes + 1);
    ck(cub::DeviceScan::ExclusiveSum(temp, temp_bytes, cnt, first, static_cast<int64_t>(n + 1), s), "scan");
    ck(cudaEventRecord(sc.ev[1], s), "event sink: event");
    Info r{};
    unsigned long long total = 0;
    ck(cudaMemcpyAsync(&r, info, sizeof r, cudaMemcpyDeviceToHost, s), "event sink: copy");
    ck(cudaMemcpyAsync(&total, first + n, sizeof total, cudaMemcpyDeviceToHost, s), "event sink: copy");
    ck(cudaStreamSynchronize(s), "event sink: count");
    refuse_bad(r, n);  // before any byte of the batch is written
    float ms = 0, part = 0;
    ck(cudaEventElapsedTime(&part, sc.ev[0], sc.ev[1]), "event sink: timing");
    ms += part;
    // Pass 2: the words, chunk by chunk, each copied out once through pinned memory and written.
    const unsigned long long chunk_words = kChunkBytes / static_cast<size_t>(word_bytes_);
    uint8_t* dbuf = sc.words.ensure(kChunkBytes);
    double write_ms = 0;
    if (!sc.pin) ck(cudaMallocHost(&sc.pin, kChunkBytes), "event sink: pinned allocation");
    uint64_t chunks = 0;
    for (unsigned long long w0 = 0; w0 < total; w0 += chunk_words, ++chunks) {
      const unsigned long long w1 = total - w0 < chunk_words ? total : w0 + chunk_words;
      ck(cudaEventRecord(sc.ev[0], s), "event sink: event");
      range_kernel<<<1, 1, 0, s>>>(first, static_cast<uint32_t>(n), w0, w1, range);
      write_kernel<<<grid, block, 0, s>>>(a, first, range, w0, w1, word_bytes_, dbuf);
      ck(cudaGetLastError(), "event sink: write launch");
      ck(cudaEventRecord(sc.ev[1], s), "event sink: event");
      const size_t bytes = static_cast<size_t>(w1 - w0) * static_cast<size_t>(word_bytes_);
      ck(cudaMemcpyAsync(sc.pin, dbuf, bytes, cudaMemcpyDeviceToHost, s), "event sink: copy");
      ck(cudaStreamSynchronize(s), "event sink: write");
      ck(cudaEventElapsedTime(&part, sc.ev[0], sc.ev[1]), "event sink: timing");
      ms += part;
      const auto t_w = std::chrono::steady_clock::now();
      write_hashed(sc.pin, bytes);
      write_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_w).count();
    }
    kernel_ms_ = ms;
    words_out_ = total;
    launches_ += 4 + 2 * chunks;  // count, info, the scan's two kernels; range + write per chunk
    // The new state and the stream's counters.
    if (count_ == 0) t_first_u_ = t1a_us(r.t_first, origin_);
    t_last_u_ = t1a_us(r.t_last, origin_);
    count_ += static_cast<int64_t>(n);
    prev_ = Prev{1, r.last_x, r.last_y, r.last_p, t_last_u_, r.t_last, r.tail_mask};
    host_ms_[0] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_begin).count();
    host_ms_[1] = write_ms;
  }

  // A batch of host columns: staged to the device, then as append_device.
  void append_host(const uint16_t* x, const uint16_t* y, const uint8_t* p, const int64_t* t, size_t n) {
    if (closed_) throw Refused(what_ + ": append after close");
    if (n == 0) return;
    if (!x || !y || !p || !t) throw std::invalid_argument(what_ + ": null event columns");
    need_device();
    if (!sc_) sc_ = take_scratch();
    Scratch& sc = *sc_;
    if (!sc.stream) ck(cudaStreamCreateWithFlags(&sc.stream, cudaStreamNonBlocking), "event sink: stream");
    uint8_t* d = sc.stage.ensure(n * 13 + 64);
    int64_t* dt = reinterpret_cast<int64_t*>(d);
    uint16_t* dx = reinterpret_cast<uint16_t*>(d + n * 8);
    uint16_t* dy = dx + n;
    uint8_t* dp = reinterpret_cast<uint8_t*>(dy + n);
    ck(cudaMemcpyAsync(dt, t, n * 8, cudaMemcpyHostToDevice, sc.stream), "event sink: copy in");
    ck(cudaMemcpyAsync(dx, x, n * 2, cudaMemcpyHostToDevice, sc.stream), "event sink: copy in");
    ck(cudaMemcpyAsync(dy, y, n * 2, cudaMemcpyHostToDevice, sc.stream), "event sink: copy in");
    ck(cudaMemcpyAsync(dp, p, n, cudaMemcpyHostToDevice, sc.stream), "event sink: copy in");
    append_device(dx, dy, dp, dt, n, sc.stream);
  }

  // Writes EVT 2.1's open word, closes and hashes the file.
  void close(bs_file_info* out) {
    if (closed_) throw Refused(what_ + ": closed twice");
    if (format_ == kEvt21 && prev_.started) {
      const uint64_t w = cd21(prev_.u, prev_.x, prev_.y, prev_.p, prev_.mask);
      write_bytes(&w, sizeof w);
    }
    closed_ = true;
    const auto t_h = std::chrono::steady_clock::now();
    struct stat st{};
    if (::fstat(fd_, &st) != 0) io_error("cannot stat", path_);
    const int fd = fd_;
    fd_ = -1;
    if (::close(fd) != 0) io_error("cannot close", path_);
    const uint64_t bytes = static_cast<uint64_t>(st.st_size);
    const std::string sha = sha_.hex();
    host_ms_[2] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_h).count();
    if (bytes != written_) {
      throw std::runtime_error(what_ + ": " + path_ + " holds " + std::to_string(bytes) + " bytes after close, " +
                               std::to_string(written_) + " were written");
    }
    out->bytes = bytes;
    std::snprintf(out->sha256, sizeof out->sha256, "%s", sha.c_str());
    out->count = count_;
    out->t_first = count_ ? t_first_u_ : 0;
    out->t_last = count_ ? t_last_u_ : 0;
  }

  uint64_t launches() const { return launches_; }
  double kernel_ms() const { return kernel_ms_; }
  const double* host_ms() const { return host_ms_; }
  uint64_t words_out() const { return words_out_; }
  int32_t word_bytes() const { return word_bytes_; }

 private:
  // The reference's message for the first event that breaks a rule, then the first and last times' rules
  // (raw_writer.cpp:91-129).
  void refuse_bad(const Info& r, size_t n) const {
    if (r.first_bad < n) {
      if (r.bad_t < r.bad_t_prev) {
        throw Refused(what_ + ": events must be in t_reported order (C4): t_ns " + std::to_string(r.bad_t) +
                      " follows " + std::to_string(r.bad_t_prev));
      }
      if (r.bad_x >= static_cast<uint32_t>(width_) || r.bad_y >= static_cast<uint32_t>(height_)) {
        throw Refused(what_ + ": event (" + std::to_string(r.bad_x) + ", " + std::to_string(r.bad_y) +
                      ") outside the " + std::to_string(width_) + " x " + std::to_string(height_) + " sensor");
      }
      if (r.bad_p > 1) throw Refused(what_ + ": polarity must be 0 or 1, got " + std::to_string(r.bad_p));
      const int64_t rem = r.bad_t - 1000 * floor_div(r.bad_t, 1000);
      throw Refused(what_ + ": t_ns_rem " + std::to_string(rem) + " lies outside the declared range [" +
                    std::to_string(rem_min_) + ", " + std::to_string(rem_max_) + "]");
    }
    const int64_t first = t1a_us(r.t_first, origin_), last = t1a_us(r.t_last, origin_);
    if (first < 0) {
      throw Refused(what_ + ": t_ns " + std::to_string(r.t_first) + " lies before the export origin " +
                    std::to_string(origin_) + " us");
    }
    if (!prev_.started && first > max_first_u_) {
      throw Refused(what_ + ": the first event lies u = " + std::to_string(first) +
                    " us after the origin, at or beyond EVT 2.0/2.1's 2^34 us TIME_HIGH loop (readers would decode " +
                    "it modulo 2^34): use raw-evt3, a later --t0 or this camera alone");
    }
    if (last > max_u_) {
      throw Refused(what_ + ": u = " + std::to_string(last) + " us after the origin exceeds " +
                    std::to_string(max_u_) + " (DAT stores u32 microseconds: export a shorter window, --t0/--t1)");
    }
  }

  // A chunk of words: written on this thread while another hashes the same bytes.
  void write_hashed(const void* data, size_t n) {
    std::thread hasher([&] { sha_.update(data, n); });
    try {
      write_raw(data, n);
    } catch (...) {
      hasher.join();
      throw;
    }
    hasher.join();
  }

  // The header and the last word: written and hashed in turn.
  void write_bytes(const void* data, size_t n) {
    write_raw(data, n);
    sha_.update(data, n);
  }

  void write_raw(const void* data, size_t n) {
    const auto* q = static_cast<const char*>(data);
    while (n > 0) {
      const ssize_t r = ::write(fd_, q, n);
      if (r < 0 && errno == EINTR) continue;
      if (r == 0) errno = EIO;
      if (r <= 0) io_error("cannot write", path_);
      q += r;
      n -= static_cast<size_t>(r);
      written_ += static_cast<uint64_t>(r);
    }
  }

  std::string what_, path_;
  int32_t format_, width_, height_;
  int64_t origin_;
  int32_t rem_min_, rem_max_;
  int64_t max_u_ = INT64_MAX, max_first_u_ = INT64_MAX;
  int32_t word_bytes_ = 4;
  int fd_ = -1;
  bool closed_ = false;
  uint64_t written_ = 0, launches_ = 0;
  Prev prev_{};
  int64_t count_ = 0, t_first_u_ = 0, t_last_u_ = 0;
  Scratch* sc_ = nullptr;
  bs::Sha256 sha_;  // of every byte written: RAW and DAT files are never patched, so it is the closed file's hash
  double kernel_ms_ = 0;       // device time of the last append's kernels (check, count + scan, writes)
  uint64_t words_out_ = 0;     // words of the last append
  double host_ms_[3] = {0, 0, 0};  // wall time of the last append, of its file writes, and of close's hash
};

template <class F>
bs_status sink_guarded(F&& f) {
  try {
    f();
    return BS_OK;
  } catch (const Refused& e) {
    set_last_error(e.what());
    return BS_EREFUSED;
  } catch (const std::invalid_argument& e) {
    set_last_error(e.what());
    return BS_EINVAL;
  } catch (const std::system_error& e) {
    set_last_error(e.what());
    return BS_EIO;
  } catch (const SinkCudaError& e) {
    set_last_error(e.what());
    return BS_ECUDA;
  } catch (const std::bad_alloc&) {
    set_last_error("out of host memory");
    return BS_ENOMEM;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return BS_ELOGIC;
  }
}

}  // namespace sink
}  // namespace bs

struct bs_event_writer {
  std::unique_ptr<bs::sink::Writer> w;
};

extern "C" {

bs_status bs_raw_writer_create(const char* path, const char* format, int32_t width, int32_t height, int64_t origin_us,
                               int64_t epoch_ns, const char* evt2_time_high, int32_t t_ns_rem_min,
                               int32_t t_ns_rem_max, const char* version, bs_event_writer** out) {
  using namespace bs::sink;
  return sink_guarded([&] {
    if (!path || !format || !evt2_time_high || !out) throw std::invalid_argument("null argument");
    *out = nullptr;
    const std::string f = format, th = evt2_time_high;
    int32_t code = 0;
    if (f == "evt2") {
      code = kEvt2OpenEb;
    } else if (f == "evt21") {
      code = kEvt21;
    } else if (f == "evt3") {
      code = kEvt3;
    } else {
      throw Refused("unknown RAW format '" + f + "': evt2, evt21 or evt3");
    }
    if (th != "openeb" && th != "change") throw Refused("unknown evt2_time_high '" + th + "': openeb or change");
    if (code == kEvt2OpenEb && th == "change") code = kEvt2OnChange;
    auto* w = new bs_event_writer;
    try {
      w->w = std::make_unique<Writer>("RawWriter", path, code, width, height, origin_us, epoch_ns, t_ns_rem_min,
                                      t_ns_rem_max, version ? version : "");
    } catch (...) {
      delete w;
      throw;
    }
    *out = w;
  });
}

bs_status bs_dat_writer_create(const char* path, int32_t width, int32_t height, int64_t origin_us, int64_t epoch_ns,
                               int32_t t_ns_rem_min, int32_t t_ns_rem_max, const char* version,
                               bs_event_writer** out) {
  using namespace bs::sink;
  return sink_guarded([&] {
    if (!path || !out) throw std::invalid_argument("null argument");
    *out = nullptr;
    auto* w = new bs_event_writer;
    try {
      w->w = std::make_unique<Writer>("DatWriter", path, kDat, width, height, origin_us, epoch_ns, t_ns_rem_min,
                                      t_ns_rem_max, version ? version : "");
    } catch (...) {
      delete w;
      throw;
    }
    *out = w;
  });
}

bs_status bs_event_writer_append(bs_event_writer* w, const uint16_t* x, const uint16_t* y, const uint8_t* p,
                                 const int64_t* t_ns, size_t n) {
  using namespace bs::sink;
  return sink_guarded([&] {
    if (!w) throw std::invalid_argument("null argument");
    w->w->append_host(x, y, p, t_ns, n);
  });
}

bs_status bs_event_writer_append_device(bs_event_writer* w, const uint16_t* x, const uint16_t* y, const uint8_t* p,
                                        const int64_t* t_ns, size_t n, void* stream) {
  using namespace bs::sink;
  return sink_guarded([&] {
    if (!w) throw std::invalid_argument("null argument");
    w->w->append_device(x, y, p, t_ns, n, static_cast<cudaStream_t>(stream));
  });
}

bs_status bs_event_writer_close(bs_event_writer* w, bs_file_info* info) {
  using namespace bs::sink;
  return sink_guarded([&] {
    if (!w || !info) throw std::invalid_argument("null argument");
    w->w->close(info);
  });
}

bs_status bs_event_writer_stats(const bs_event_writer* w, uint64_t* launches, double* kernel_ms,
                                uint64_t* bytes_out, double host_ms[3]) {
  using namespace bs::sink;
  return sink_guarded([&] {
    if (!w) throw std::invalid_argument("null argument");
    if (launches) *launches = w->w->launches();
    if (kernel_ms) *kernel_ms = w->w->kernel_ms();
    if (bytes_out) *bytes_out = w->w->words_out() * static_cast<uint64_t>(w->w->word_bytes());
    if (host_ms) std::memcpy(host_ms, w->w->host_ms(), 3 * sizeof(double));
  });
}

bs_status bs_event_writer_destroy(bs_event_writer* w) {
  using namespace bs::sink;
  return sink_guarded([&] { delete w; });
}

bs_status bs_sha256_hex(const void* data, size_t n, char out[65]) {
  using namespace bs::sink;
  return sink_guarded([&] {
    if ((!data && n > 0) || !out) throw std::invalid_argument("null argument");
    bs::Sha256 s;
    s.update(data, n);
    std::snprintf(out, 65, "%s", s.hex().c_str());
  });
}

}  // extern "C"
