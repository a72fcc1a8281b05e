// The output order of a call's events on the device: SensorModel::finish_events sorts the events by
// (t_cross, pixel) on the host (src/sensor/sensor_model.cpp:996-1029); here two stable radix passes over an index
// permutation (pixel first, then t_cross) and one gather put the RawEvent records in that order in device memory,
// so that the host only copies them out. (t_cross, pixel) is unique per event (a pixel fires at most once per ns),
// so the order is the host sort's exactly.
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

}  // namespace

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
