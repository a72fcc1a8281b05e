// Analytic irradiance fields evaluated on the device in place of BallaSim's renderer (the render hook of
// src/engine/window.h:69-84 on this path): a moving tanh edge and a sum of moving Gaussian blobs, fp32 in a
// fixed operation order (bit-identical to any CPU evaluation compiled without contraction).
//
// Blob table rows (kBlobWords floats): a, cx0, cy0, vx, vy, 1/(2 r^2), (6 r)^2, (3 r)^2, |v|, pad. A blob adds
// exactly 0 where d^2 >= (6 r)^2, so a warp evaluates only the blobs whose 6 r disc can reach its pixels during
// the window (a 256-bit candidate mask built once per window with ballots); skipped terms are exact zeros, so the
// sum is the same bits as the full loop.
#pragma once

#include "bs_math.cuh"

namespace bs {

constexpr int kFieldTanhEdge = 1;
constexpr int kFieldBlobs = 2;
constexpr int kBlobWords = 10;
constexpr int kMaskWords = 8;  // candidate masks cover up to 256 blobs; larger tables evaluate every blob

struct FieldDev {
  int32_t kind;
  uint32_t width, height;
  float base, amp, nx, ny, c, speed, width_px;
  int32_t n_blobs;
  const float* blobs;  // device memory, n_blobs x kBlobWords
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

BS_HD float blob_term(const float* b, float xc, float yc, float ts) {
  const float cx = b[1] + b[3] * ts, cy = b[2] + b[4] * ts;
  const float dx = xc - cx, dy = yc - cy;
  const float d2 = dx * dx + dy * dy;
  return d2 < b[6] ? b[0] * exp_f(-(d2 * b[5])) : 0.0f;
}

// E(x, y, t) over every blob (the definition).
BS_HD float field_eval_all(const FieldDev& f, uint32_t x, uint32_t y, int64_t t_ns) {
  const float ts = t_seconds(t_ns);
  const float xc = static_cast<float>(x) + 0.5f, yc = static_cast<float>(y) + 0.5f;
  if (f.kind == kFieldTanhEdge) {
    const float u = (((f.nx * xc + f.ny * yc) - f.speed * ts) - f.c) / f.width_px;
    return f.base + f.amp * tanh_det(u);
  }
  float e = f.base;
  for (int32_t k = 0; k < f.n_blobs; ++k) {
    const float* b = f.blobs + static_cast<size_t>(k) * kBlobWords;
    const float cx = b[1] + b[3] * ts, cy = b[2] + b[4] * ts;
    const float dx = xc - cx, dy = yc - cy;
    const float d2 = dx * dx + dy * dy;
    if (d2 < b[6]) e = e + b[0] * exp_f(-(d2 * b[5]));
  }
  return e;
}

// The blobs a pixel may see in one window, as a bit mask (bit k of word k / 32).
struct BlobMask {
  uint32_t w[kMaskWords];
};

// E(x, y, t) over the candidate blobs only (bitwise field_eval_all when the mask covers every blob the pixel can
// reach at t). Tables over 256 blobs take the full loop.
BS_HD float field_eval(const FieldDev& f, const BlobMask& m, uint32_t x, uint32_t y, int64_t t_ns) {
  if (f.kind != kFieldBlobs || f.n_blobs > 32 * kMaskWords) return field_eval_all(f, x, y, t_ns);
  const float ts = t_seconds(t_ns);
  const float xc = static_cast<float>(x) + 0.5f, yc = static_cast<float>(y) + 0.5f;
  float e = f.base;
#pragma unroll
  for (int wi = 0; wi < kMaskWords; ++wi) {
    uint32_t bits = m.w[wi];
    while (bits != 0u) {
#if defined(__CUDA_ARCH__)
      const int j = __ffs(static_cast<int>(bits)) - 1;
#else
      const int j = __builtin_ctz(bits);
#endif
      bits &= bits - 1u;
      const float* b = f.blobs + static_cast<size_t>(wi * 32 + j) * kBlobWords;
      const float cx = b[1] + b[3] * ts, cy = b[2] + b[4] * ts;
      const float dx = xc - cx, dy = yc - cy;
      const float d2 = dx * dx + dy * dy;
      if (d2 < b[6]) e = e + b[0] * exp_f(-(d2 * b[5]));
    }
  }
  return e;
}

// The level rule at the window start: clamp(ceil(log2(v W / 0.25 px)), l_min, l_max), v the speed of the fastest
// candidate blob whose 3 r support covers the pixel (none, or the tanh edge: l_min).
BS_HD int32_t field_level(const FieldDev& f, const BlobMask& m, uint32_t x, uint32_t y, int64_t t_w, int32_t l_min,
                          int32_t l_max) {
  if (f.kind != kFieldBlobs) return l_min;
  const float ts = t_seconds(t_w);
  const float xc = static_cast<float>(x) + 0.5f, yc = static_cast<float>(y) + 0.5f;
  float v = 0.0f;
  const bool masked = f.n_blobs <= 32 * kMaskWords;
  for (int32_t k = 0; k < f.n_blobs; ++k) {
    if (masked && ((m.w[k >> 5] >> (k & 31)) & 1u) == 0u) continue;
    const float* b = f.blobs + static_cast<size_t>(k) * kBlobWords;
    const float cx = b[1] + b[3] * ts, cy = b[2] + b[4] * ts;
    const float dx = xc - cx, dy = yc - cy;
    const float d2 = dx * dx + dy * dy;
    if (d2 <= b[7] && b[8] > v) v = b[8];
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
// The candidate blobs of the calling warp's pixels for the window [t_w, t_w + W]: blob k is kept when its 6 r disc,
// swept over the window, can reach the bounding box of the active lanes' pixel centres (a 1 px margin covers the
// fp32 rounding of the per-sample test). Every lane of `active` must call it; all get the same mask.
__device__ inline BlobMask warp_blob_mask(const FieldDev& f, uint32_t active, bool have, uint32_t x, uint32_t y,
                                          int64_t t_w) {
  BlobMask m;
#pragma unroll
  for (int i = 0; i < kMaskWords; ++i) m.w[i] = 0xffffffffu;
  if (f.kind != kFieldBlobs || f.n_blobs > 32 * kMaskWords) return m;
  float x0 = have ? static_cast<float>(x) + 0.5f : 3.0e38f, x1 = have ? static_cast<float>(x) + 0.5f : -3.0e38f;
  float y0 = have ? static_cast<float>(y) + 0.5f : 3.0e38f, y1 = have ? static_cast<float>(y) + 0.5f : -3.0e38f;
  for (int o = 16; o > 0; o >>= 1) {
    x0 = fminf(x0, __shfl_xor_sync(active, x0, o));
    x1 = fmaxf(x1, __shfl_xor_sync(active, x1, o));
    y0 = fminf(y0, __shfl_xor_sync(active, y0, o));
    y1 = fmaxf(y1, __shfl_xor_sync(active, y1, o));
  }
  const float ta = t_seconds(t_w), tb = t_seconds(t_w + kWindowNs);
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int wi = 0; wi < kMaskWords; ++wi) {
    const int k = wi * 32 + lane;
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
    m.w[wi] = __ballot_sync(active, keep);
  }
  return m;
}
#endif

}  // namespace bs
