// Analytic irradiance fields evaluated on the device in place of BallaSim's renderer (the render hook of
// src/engine/window.h:69-84 on this path): a moving tanh edge and a sum of moving Gaussian blobs, fp32 in a
// fixed operation order (bit-identical to any CPU evaluation compiled without contraction).
//
// Blob table rows (kBlobWords floats): a, cx0, cy0, vx, vy, 1/(2 r^2), (6 r)^2, (3 r)^2, |v|, pad. A blob adds
// exactly 0 where d^2 >= (6 r)^2. Per window a warp lists, in shared memory and in blob order, the blobs whose 6 r
// disc can reach its pixels during the window; every lane then runs one loop over that list with a branch-free
// term (a listed blob out of reach adds +0). Skipped and zero terms leave the fp32 sum's bits unchanged, so the
// result is the full definition's.
#pragma once

#include "bs_math.cuh"

namespace bs {

constexpr int kFieldTanhEdge = 1;
constexpr int kFieldBlobs = 2;
constexpr int kBlobWords = 10;
constexpr int kMaxListed = 256;  // tables of up to 256 blobs are culled per warp; larger ones evaluate every blob

struct FieldDev {
  int32_t kind;
  uint32_t width, height;
  float base, amp, nx, ny, c, speed, width_px;
  int32_t n_blobs;
  const float* blobs;  // device memory, n_blobs x kBlobWords
};

// The candidate blobs of one warp and window (indices in blob order), or all blobs (idx null).
struct BlobList {
  const uint16_t* idx;
  int32_t n;
};

BS_HD float t_seconds(int64_t t_ns) { return static_cast<float>(static_cast<double>(t_ns) * 1e-9); }

BS_HD float tanh_det(float u) {
  const float a = fabs_f(u);
  float r = 1.0f;
  if (a <= 9.0f) {
    const float e = exp_f(2.0f * a);
    r = 1.0f - 2.0f / (e + 1.0f);
  }
  return u < 0.0f ? -r : r;
}

BS_HD float edge_eval(const FieldDev& f, float xc, float yc, float ts) {
  const float u = (((f.nx * xc + f.ny * yc) - f.speed * ts) - f.c) / f.width_px;
  return f.base + f.amp * tanh_det(u);
}

// One blob's term, branch-free: A exp(-d^2 / (2 r^2)) inside 6 r, else +0 (the exp then sees a harmless 0).
BS_HD float blob_term(const float* b, float xc, float yc, float ts) {
  const float cx = b[1] + b[3] * ts, cy = b[2] + b[4] * ts;
  const float dx = xc - cx, dy = yc - cy;
  const float d2 = dx * dx + dy * dy;
  const bool in = d2 < b[6];
  const float term = b[0] * exp_f(in ? -(d2 * b[5]) : 0.0f);
  return in ? term : 0.0f;
}

// E(x, y, t) over every blob (the definition).
BS_HD float field_eval_all(const FieldDev& f, uint32_t x, uint32_t y, int64_t t_ns) {
  const float ts = t_seconds(t_ns);
  const float xc = static_cast<float>(x) + 0.5f, yc = static_cast<float>(y) + 0.5f;
  if (f.kind == kFieldTanhEdge) return edge_eval(f, xc, yc, ts);
  float e = f.base;
  for (int32_t k = 0; k < f.n_blobs; ++k) e = e + blob_term(f.blobs + static_cast<size_t>(k) * kBlobWords, xc, yc, ts);
  return e;
}

// E(x, y, t) over a warp's candidate list (bitwise field_eval_all when the list holds every blob in reach). One
// out-of-line copy serves the sampler's render sites (a smaller kernel for the instruction cache); blobs go in
// pairs whose exp chains are independent, summed in list order.
static __host__ __device__ __noinline__ float field_eval(const FieldDev& f, const BlobList& l, uint32_t x, uint32_t y,
                                                         int64_t t_ns) {
  if (f.kind != kFieldBlobs || l.idx == nullptr) return field_eval_all(f, x, y, t_ns);
  const float ts = t_seconds(t_ns);
  const float xc = static_cast<float>(x) + 0.5f, yc = static_cast<float>(y) + 0.5f;
  float e = f.base;
  int32_t i = 0;
  for (; i + 1 < l.n; i += 2) {
    const float t0 = blob_term(f.blobs + static_cast<size_t>(l.idx[i]) * kBlobWords, xc, yc, ts);
    const float t1 = blob_term(f.blobs + static_cast<size_t>(l.idx[i + 1]) * kBlobWords, xc, yc, ts);
    e = e + t0;
    e = e + t1;
  }
  if (i < l.n) e = e + blob_term(f.blobs + static_cast<size_t>(l.idx[i]) * kBlobWords, xc, yc, ts);
  return e;
}

// The level rule at the window start: clamp(ceil(log2(v W / 0.25 px)), l_min, l_max), v the speed of the fastest
// blob whose 3 r support covers the pixel (none, or the tanh edge: l_min).
BS_HD int32_t field_level(const FieldDev& f, const BlobList& l, uint32_t x, uint32_t y, int64_t t_w, int32_t l_min,
                          int32_t l_max) {
  if (f.kind != kFieldBlobs) return l_min;
  const float ts = t_seconds(t_w);
  const float xc = static_cast<float>(x) + 0.5f, yc = static_cast<float>(y) + 0.5f;
  float v = 0.0f;
  const int32_t n = l.idx != nullptr ? l.n : f.n_blobs;
  for (int32_t i = 0; i < n; ++i) {
    const int32_t k = l.idx != nullptr ? l.idx[i] : i;
    const float* b = f.blobs + static_cast<size_t>(k) * kBlobWords;
    const float cx = b[1] + b[3] * ts, cy = b[2] + b[4] * ts;
    const float dx = xc - cx, dy = yc - cy;
    const float d2 = dx * dx + dy * dy;
    v = (d2 <= b[7] && b[8] > v) ? b[8] : v;
  }
  if (!(v > 0.0f)) return l_min;
  const float q = v * 0.033554432f;  // v W / 0.25 px with W = 2^23 ns
  const uint32_t bq = f2u(q);
  const int e = static_cast<int>((bq >> 23) & 0xffu) - 126;  // q = m 2^e, m in [0.5, 1) (q is normal)
  const bool half = (bq & 0x7fffffu) == 0u;                    // m == 0.5: log2 q = e - 1 exactly
  int32_t level = half ? e - 1 : e;
  if (level < l_min) level = l_min;
  if (level > l_max) level = l_max;
  return level;
}

#if defined(__CUDACC__)
// Builds the calling warp's candidate list for [t_a, t_b] in `list` (kMaxListed entries of shared memory): blob k
// is listed when its 6 r disc, swept from t_a to t_b, can reach the bounding box of the active lanes' pixel
// centres (a 1 px margin covers the fp32 rounding of the per-sample test). All 32 lanes call it together.
__device__ inline BlobList warp_blob_list(const FieldDev& f, bool have, uint32_t x, uint32_t y, int64_t t_a,
                                          int64_t t_b, uint16_t* list) {
  if (f.kind != kFieldBlobs || f.n_blobs > kMaxListed) return BlobList{nullptr, f.n_blobs};
  float x0 = have ? static_cast<float>(x) + 0.5f : 3.0e38f, x1 = have ? static_cast<float>(x) + 0.5f : -3.0e38f;
  float y0 = have ? static_cast<float>(y) + 0.5f : 3.0e38f, y1 = have ? static_cast<float>(y) + 0.5f : -3.0e38f;
  for (int o = 16; o > 0; o >>= 1) {
    x0 = fminf(x0, __shfl_xor_sync(0xffffffffu, x0, o));
    x1 = fmaxf(x1, __shfl_xor_sync(0xffffffffu, x1, o));
    y0 = fminf(y0, __shfl_xor_sync(0xffffffffu, y0, o));
    y1 = fmaxf(y1, __shfl_xor_sync(0xffffffffu, y1, o));
  }
  const float ta = t_seconds(t_a), tb = t_seconds(t_b);
  const uint32_t lane = threadIdx.x & 31u;
  int32_t n = 0;
  for (int32_t base = 0; base < f.n_blobs; base += 32) {
    const int32_t k = base + static_cast<int32_t>(lane);
    bool keep = false;
    if (k < f.n_blobs) {
      const float* b = f.blobs + static_cast<size_t>(k) * kBlobWords;
      const float cxa = b[1] + b[3] * ta, cxb = b[1] + b[3] * tb;
      const float cya = b[2] + b[4] * ta, cyb = b[2] + b[4] * tb;
      const float reach = sqrtf(b[6]) + 1.0f;
      const float bx0 = fminf(cxa, cxb) - reach, bx1 = fmaxf(cxa, cxb) + reach;
      const float by0 = fminf(cya, cyb) - reach, by1 = fmaxf(cya, cyb) + reach;
      keep = !(bx1 < x0 || bx0 > x1 || by1 < y0 || by0 > y1);
    }
    const uint32_t bits = __ballot_sync(0xffffffffu, keep);
    if (keep) list[n + __popc(bits & ((1u << lane) - 1u))] = static_cast<uint16_t>(k);
    n += __popc(bits);
  }
  __syncwarp();
  return BlobList{list, n};
}
#endif

}  // namespace bs
