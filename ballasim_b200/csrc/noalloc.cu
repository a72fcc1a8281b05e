// sample_window without any device allocation, for callers that cannot allocate device memory themselves or let a
// library do it: code that runs under an external memory manager with a fixed budget (a framework's caching
// allocator, an embedded renderer that owns the whole card), or that must not call cudaMalloc/cudaFree because
// those calls synchronize the device and would stall its other streams. The caller passes every input and output
// in device memory; the only scratch this entry point needs (the per-pixel sample counts and the scan's block sums)
// lives in one file-scope device array of fixed size that every GPU loading the library keeps until the process
// exits.
#include <cuda_runtime.h>

#include <mutex>
#include <stdexcept>
#include <string>

#include "../../include/ballasim_b200.h"
#include "device.h"

namespace bs {
void set_last_error(const char* msg);  // model.cu: the message bs_last_error() returns

namespace {

// The static scratch: the counts of up to kStaticMaxPixels pixels, the scan's block sums and one error word.
constexpr size_t kStaticMaxPixels = size_t{1} << 20;
constexpr size_t kCountWords = kStaticMaxPixels / 2;                // u32 counts packed two per 8-byte word
constexpr size_t kBlockWords = kStaticMaxPixels / 1024 + 2;         // scan block sums (i64)
constexpr size_t kScratchWords = kCountWords + kBlockWords + 1;     // + the error word
__device__ __align__(256) unsigned long long g_scratch[kScratchWords];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned long long* g_scratch_ptr[kMaxDevices] = {};

// The device address of g_scratch on the current device, looked up once per device. In host code the array's name
// is only a host-side stand-in, so every kernel gets the address this returns.
unsigned long long* scratch_on_current_device() {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) throw std::runtime_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) throw std::runtime_error("device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_mu);
  if (g_scratch_ptr[dev] == nullptr) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess) throw std::runtime_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_scratch_ptr[dev] = static_cast<unsigned long long*>(p);
  }
  return g_scratch_ptr[dev];
}

// Level and pixel-id checks on the device inputs (bit 0: a level above max_level, bit 1: an id outside the field).
__global__ void check_inputs_kernel(const uint32_t* pixel, const uint8_t* level, uint32_t n, uint32_t n_field,
                                    int max_level, unsigned long long* err) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  unsigned long long bits = 0;
  if (level[i] > max_level) bits |= 1ull;
  if (pixel[i] >= n_field) bits |= 2ull;
  if (bits) atomicOr(err, bits);
}

}  // namespace
}  // namespace bs

extern "C" bs_status bs_sample_window_static(const bs_field* field, int64_t t_w, const uint32_t* pixel_ids,
                                              const uint8_t* levels, size_t n, const float* carried_irr,
                                              const uint64_t* carried_sig, const bs_sample_rules* rules,
                                              int64_t* offsets, int64_t* t_ns, float* irr, size_t capacity,
                                              float* carried_irr_out, uint64_t* carried_sig_out, void* stream,
                                              size_t* n_samples) {
  using namespace bs;
  try {
    if (!field || !rules || !offsets || !n_samples) throw std::invalid_argument("null argument");
    if (n > kStaticMaxPixels) {
      throw std::invalid_argument("sample_window_static: " + std::to_string(n) + " pixels exceed its maximum of " +
                                  std::to_string(kStaticMaxPixels) + " (use bs_sample_window)");
    }
    if (n > 0 && (!pixel_ids || !levels || !carried_irr || !carried_sig || !carried_irr_out || !carried_sig_out)) {
      throw std::invalid_argument("null argument");
    }
    if (field->kind != kFieldTanhEdge && field->kind != kFieldBlobs) throw std::invalid_argument("field: unknown kind");
    if (field->width == 0 || field->height == 0) throw std::invalid_argument("field: empty frame");
    if (field->kind == kFieldBlobs && field->n_blobs > 0 && !field->blobs) {
      throw std::invalid_argument("field: null blob table (a device pointer)");
    }
    if (rules->min_dt_ns < 1 || rules->min_dt_ns > kWindowNs || (rules->min_dt_ns & (rules->min_dt_ns - 1)) != 0) {
      throw std::invalid_argument("min_dt_ns must be a power of two in [1, 2^23]");
    }
    if (rules->max_refine_levels < 0) throw std::invalid_argument("max_refine_levels must be >= 0");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned long long* base = scratch_on_current_device();
    uint32_t* counts = reinterpret_cast<uint32_t*>(base);
    int64_t* block_sums = reinterpret_cast<int64_t*>(base + kCountWords);
    unsigned long long* err = base + kCountWords + kBlockWords;

    FieldDev f{};
    f.kind = field->kind;
    f.width = field->width;
    f.height = field->height;
    f.base = field->base;
    f.amp = field->amp;
    f.nx = field->nx;
    f.ny = field->ny;
    f.c = field->c;
    f.speed = field->speed;
    f.width_px = field->width_px;
    f.n_blobs = field->kind == kFieldBlobs ? field->n_blobs : 0;
    f.blobs = field->blobs;
    int shift = 0;
    while ((int64_t{1} << shift) < rules->min_dt_ns) ++shift;
    SamplerRules r{};
    r.tol = rules->tol;
    r.dark = rules->dark;
    r.midpoint = rules->midpoint;
    r.refine_signature = rules->refine_signature;
    r.max_refine_levels = rules->max_refine_levels < 23 ? rules->max_refine_levels : 23;
    r.min_split = static_cast<uint32_t>(2 * rules->min_dt_ns);
    r.l_min = rules->l_min;
    r.l_max = rules->l_max;

    // The error word keeps the last call's value: clear it first.
    cudaError_t e = cudaMemsetAsync(err, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) throw std::runtime_error(std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
    const uint32_t nn = static_cast<uint32_t>(n);
    if (nn > 0) {
      check_inputs_kernel<<<(nn + 255) / 256, 256, 0, s>>>(pixel_ids, levels, nn, f.width * f.height,
                                                           kWindowLog2 - shift, err);
    }
    unsigned long long bits = 0;
    e = cudaMemcpyAsync(&bits, err, sizeof(bits), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) throw std::runtime_error(std::string("check: ") + cudaGetErrorString(e));
    if (bits & 1ull) throw std::invalid_argument("levels must lie in [0, 23 - log2(min_dt_ns)]");
    if (bits & 2ull) throw std::invalid_argument("pixel id outside the field");

    // Pass 0 writes every count it reads back, and the scan rewrites every block sum: nothing else needs clearing.
    launch_sample_window(f, r, t_w, pixel_ids, levels, nn, carried_irr, carried_sig, counts, nullptr, nullptr,
                         nullptr, nullptr, nullptr, 0, s);
    launch_scan(counts, nn, offsets, block_sums, s);
    int64_t total = 0;
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&total, offsets + n, sizeof(total), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) throw std::runtime_error(std::string("sample_window_static: ") + cudaGetErrorString(e));
    *n_samples = static_cast<size_t>(total);
    if (static_cast<size_t>(total) > capacity) {
      throw std::invalid_argument("sample_window_static: the window has " + std::to_string(total) +
                                  " samples, above the output capacity of " + std::to_string(capacity));
    }
    if (total > 0 && (!t_ns || !irr)) throw std::invalid_argument("null output arrays");
    launch_sample_window(f, r, t_w, pixel_ids, levels, nn, carried_irr, carried_sig, counts, offsets, t_ns, irr,
                         carried_irr_out, carried_sig_out, 1, s);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) throw std::runtime_error(std::string("sample_window_static: ") + cudaGetErrorString(e));
    return BS_OK;
  } catch (const std::invalid_argument& ex) {
    bs::set_last_error(ex.what());
    return BS_EINVAL;
  } catch (const std::exception& ex) {
    bs::set_last_error(ex.what());
    return BS_ECUDA;
  }
}
