// Event order on the device.
//
// sort_events: SensorModel::finish_events sorts a call's events by (t_cross, pixel) on the host
// (src/sensor/sensor_model.cpp:996-1029); here two stable radix passes over an index permutation (pixel first, then
// t_cross) and one gather put the RawEvent records in that order in device memory, so that the host only copies
// them out. (t_cross, pixel) is unique per event (a pixel fires at most once per ns), so the order is the host
// sort's exactly.
//
// event_columns: the sorted records split into event columns (x, y from the pixel index, the readout's reported time)
// on the device, so that the host copies each column out whole.
//
// output_stage: the engine's output stage (Camera::output, src/engine/engine_impl.h:1761-1847): records with the
// readout's reported time, three stable radix passes (t_cross, (x, y), t_reported) that order them by
// (t_reported, x, y, t_cross) as src/sensor/output_order.h:88-107 does, and the cut of the released prefix.
#include <cub/device/device_radix_sort.cuh>

#include "device.h"

namespace bs {

namespace {

__global__ void pixel_keys_kernel(const RawEvent* ev, uint32_t n, uint32_t* key, uint32_t* idx) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  key[i] = ev[i].pixel;
  idx[i] = i;
}

// t_cross as an unsigned key in the same order: the sign bit flipped.
__global__ void time_keys_kernel(const RawEvent* ev, const uint32_t* idx, uint32_t n, uint64_t* key) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  key[i] = static_cast<uint64_t>(ev[idx[i]].t_cross) ^ (uint64_t{1} << 63);
}

__global__ void gather_events_kernel(const RawEvent* ev, const uint32_t* idx, uint32_t n, RawEvent* out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint4* src = reinterpret_cast<const uint4*>(ev + idx[i]);
  uint4* dst = reinterpret_cast<uint4*>(out + i);
  dst[0] = src[0];
  dst[1] = src[1];
}

struct SortLayout {
  size_t k32_in, k32_out, idx_a, idx_b, k64_in, k64_out, temp, temp_bytes, total;
};

size_t align256(size_t v) { return (v + 255) & ~size_t{255}; }

SortLayout layout(uint32_t n) {
  size_t t32 = 0, t64 = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, t32, static_cast<const uint32_t*>(nullptr), static_cast<uint32_t*>(nullptr),
                                  static_cast<const uint32_t*>(nullptr), static_cast<uint32_t*>(nullptr),
                                  static_cast<int>(n), 0, 32);
  cub::DeviceRadixSort::SortPairs(nullptr, t64, static_cast<const uint64_t*>(nullptr), static_cast<uint64_t*>(nullptr),
                                  static_cast<const uint32_t*>(nullptr), static_cast<uint32_t*>(nullptr),
                                  static_cast<int>(n), 0, 64);
  SortLayout l{};
  size_t at = 0;
  l.k32_in = at;
  at += align256(n * sizeof(uint32_t));
  l.k32_out = at;
  at += align256(n * sizeof(uint32_t));
  l.idx_a = at;
  at += align256(n * sizeof(uint32_t));
  l.idx_b = at;
  at += align256(n * sizeof(uint32_t));
  l.k64_in = at;
  at += align256(n * sizeof(uint64_t));
  l.k64_out = at;
  at += align256(n * sizeof(uint64_t));
  l.temp = at;
  l.temp_bytes = align256(t32 > t64 ? t32 : t64);
  at += l.temp_bytes;
  l.total = at;
  return l;
}

// ---- the output stage ----
__device__ __forceinline__ uint8_t label_s1(uint8_t c3) {
  return (c3 & 3u) == 0u ? 0u : static_cast<uint8_t>((c3 & 3u) + 1u);  // 0 signal, 1 noise, 2 leak, 3 hot -> 0, 2, 3, 4
}

__global__ void build_out_kernel(const RawEvent* raw, uint32_t n, uint32_t width, ReadoutDev rd, OutRecord* out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const RawEvent e = raw[i];
  OutRecord o;
  o.x = static_cast<uint16_t>(e.pixel % width);
  o.y = static_cast<uint16_t>(e.pixel / width);
  o.p = e.polarity;
  o.t_cross = e.t_cross;
  o.t_reported = reported_time(rd, e.t_cross);
  o.label = label_s1(e.label);
  o.flags = e.flags;
  out[i] = o;
}

__global__ void iota_kernel(uint32_t n, uint32_t* idx) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) idx[i] = i;
}

// Pass 0: t_cross, 1: (x, y) x-major, 2: t_reported (order_key); signed times biased to unsigned order.
__global__ void out_keys_kernel(const OutRecord* rec, const uint32_t* idx, uint32_t n, int pass, int y_bits,
                                uint64_t* key) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const OutRecord& r = rec[idx[i]];
  const uint64_t bias = uint64_t{1} << 63;
  key[i] = pass == 0   ? static_cast<uint64_t>(r.t_cross) ^ bias
           : pass == 1 ? (static_cast<uint64_t>(r.x) << y_bits) | r.y
                       : static_cast<uint64_t>(r.t_reported) ^ bias;
}

__global__ void gather_out_kernel(const OutRecord* rec, const uint32_t* idx, uint32_t n, int64_t limit,
                                  OutRecord* out, unsigned long long* ready) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const OutRecord r = rec[idx[i]];
  out[i] = r;
  // sorted by t_reported first: the released records are a prefix; its length is the first index at the limit
  const bool rel = r.t_reported < limit;
  const bool next_rel = i + 1 < n && rec[idx[i + 1]].t_reported < limit;
  if (rel && !next_rel) *ready = i + 1;
}

struct OutLayout {
  size_t idx_a, idx_b, k_in, k_out, temp, temp_bytes, total;
};

OutLayout out_layout(uint32_t n) {
  size_t t64 = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, t64, static_cast<const uint64_t*>(nullptr), static_cast<uint64_t*>(nullptr),
                                  static_cast<const uint32_t*>(nullptr), static_cast<uint32_t*>(nullptr),
                                  static_cast<int>(n), 0, 64);
  OutLayout l{};
  size_t at = 0;
  l.idx_a = at;
  at += align256(n * sizeof(uint32_t));
  l.idx_b = at;
  at += align256(n * sizeof(uint32_t));
  l.k_in = at;
  at += align256(n * sizeof(uint64_t));
  l.k_out = at;
  at += align256(n * sizeof(uint64_t));
  l.temp = at;
  l.temp_bytes = align256(t64);
  at += l.temp_bytes;
  l.total = at;
  return l;
}

}  // namespace

size_t output_scratch_bytes(uint32_t n) { return n == 0 ? 0 : out_layout(n).total; }

cudaError_t output_stage(const OutRecord* held, uint32_t n_held, const RawEvent* raw, uint32_t n_raw, uint32_t width,
                         int y_bits, const ReadoutDev& rd, int64_t limit, OutRecord* all, OutRecord* out,
                         void* scratch, unsigned long long* ready_dev, cudaStream_t stream) {
  const uint32_t n = n_held + n_raw;
  cudaError_t e = cudaMemsetAsync(ready_dev, 0, sizeof(unsigned long long), stream);
  if (e != cudaSuccess || n == 0) return e;
  if (n_held) {
    e = cudaMemcpyAsync(all, held, static_cast<size_t>(n_held) * sizeof(OutRecord), cudaMemcpyDeviceToDevice, stream);
    if (e != cudaSuccess) return e;
  }
  if (n_raw) build_out_kernel<<<(n_raw + 255) / 256, 256, 0, stream>>>(raw, n_raw, width, rd, all + n_held);
  const OutLayout l = out_layout(n);
  unsigned char* base = static_cast<unsigned char*>(scratch);
  uint32_t* idx = reinterpret_cast<uint32_t*>(base + l.idx_a);
  uint32_t* idx_alt = reinterpret_cast<uint32_t*>(base + l.idx_b);
  uint64_t* k_in = reinterpret_cast<uint64_t*>(base + l.k_in);
  uint64_t* k_out = reinterpret_cast<uint64_t*>(base + l.k_out);
  const unsigned grid = (n + 255) / 256;
  iota_kernel<<<grid, 256, 0, stream>>>(n, idx);
  for (int pass = 0; pass < 3; ++pass) {
    out_keys_kernel<<<grid, 256, 0, stream>>>(all, idx, n, pass, y_bits, k_in);
    size_t temp_bytes = l.temp_bytes;
    e = cub::DeviceRadixSort::SortPairs(base + l.temp, temp_bytes, k_in, k_out, idx, idx_alt, static_cast<int>(n), 0,
                                        pass == 1 ? 16 + y_bits : 64, stream);
    if (e != cudaSuccess) return e;
    uint32_t* t = idx;
    idx = idx_alt;
    idx_alt = t;
  }
  gather_out_kernel<<<grid, 256, 0, stream>>>(all, idx, n, limit, out, ready_dev);
  return cudaGetLastError();
}

// ---- event columns: the sorted records split into the caller's columns on the device ----
namespace {
__global__ void columns_kernel(const RawEvent* ev, uint32_t n, uint32_t width, ReadoutDev rd, EventColumnsDev c) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const RawEvent e = ev[i];
  if (c.pixel) c.pixel[i] = e.pixel;
  if (c.x) c.x[i] = static_cast<uint16_t>(e.pixel % width);
  if (c.y) c.y[i] = static_cast<uint16_t>(e.pixel / width);
  if (c.p) c.p[i] = e.polarity;
  if (c.t_cross) c.t_cross[i] = e.t_cross;
  if (c.t_reported) c.t_reported[i] = reported_time(rd, e.t_cross);
  if (c.label) c.label[i] = e.label;
  if (c.flags) c.flags[i] = e.flags;
  if (c.ds) c.ds[i] = e.ds;
  if (c.dn) c.dn[i] = e.dn;
  if (c.dl) c.dl[i] = e.dl;
  if (c.l_first) c.l_first[i] = e.l_first;
}
}  // namespace

cudaError_t event_columns(const RawEvent* ev, uint32_t n, uint32_t width, const ReadoutDev& rd,
                          const EventColumnsDev& cols, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  columns_kernel<<<(n + 255) / 256, 256, 0, stream>>>(ev, n, width, rd, cols);
  return cudaGetLastError();
}

size_t sort_events_scratch_bytes(uint32_t n) { return n == 0 ? 0 : layout(n).total; }

cudaError_t sort_events(const RawEvent* ev, uint32_t n, RawEvent* out, void* scratch, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  const SortLayout l = layout(n);
  unsigned char* base = static_cast<unsigned char*>(scratch);
  uint32_t* k32_in = reinterpret_cast<uint32_t*>(base + l.k32_in);
  uint32_t* k32_out = reinterpret_cast<uint32_t*>(base + l.k32_out);
  uint32_t* idx_a = reinterpret_cast<uint32_t*>(base + l.idx_a);
  uint32_t* idx_b = reinterpret_cast<uint32_t*>(base + l.idx_b);
  uint64_t* k64_in = reinterpret_cast<uint64_t*>(base + l.k64_in);
  uint64_t* k64_out = reinterpret_cast<uint64_t*>(base + l.k64_out);
  void* temp = base + l.temp;
  size_t temp_bytes = l.temp_bytes;
  const unsigned grid = (n + 255) / 256;
  pixel_keys_kernel<<<grid, 256, 0, stream>>>(ev, n, k32_in, idx_a);
  cudaError_t e = cub::DeviceRadixSort::SortPairs(temp, temp_bytes, k32_in, k32_out, idx_a, idx_b,
                                                  static_cast<int>(n), 0, 32, stream);
  if (e != cudaSuccess) return e;
  time_keys_kernel<<<grid, 256, 0, stream>>>(ev, idx_b, n, k64_in);
  temp_bytes = l.temp_bytes;
  e = cub::DeviceRadixSort::SortPairs(temp, temp_bytes, k64_in, k64_out, idx_b, idx_a, static_cast<int>(n), 0, 64,
                                      stream);
  if (e != cudaSuccess) return e;
  gather_events_kernel<<<grid, 256, 0, stream>>>(ev, idx_a, n, out);
  return cudaGetLastError();
}

}  // namespace bs
