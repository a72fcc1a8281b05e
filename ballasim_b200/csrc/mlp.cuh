// The learned step proposal: an MLP 16 -> 64 -> 64 -> 1 (ReLU) that predicts a pixel's next sample interval from
// its recent log-irradiance history. This part has no reference counterpart (BallaSim's sampler is the plain
// lattice + midpoint rule, src/engine/sampling.h); the plain rule stays both the judge of every proposed step and
// its fallback.
//
// Arithmetic: BF16 weights and activations, FP32 accumulate, on the tensor cores through warp-level
// mma.sync.m16n8k16 (one warp proposes for its 32 pixels at once, inside the per-pixel loop of the engine, so the
// operand tiles are 32 rows: a CTA-wide tcgen05 tile of 128 rows has no place there). Biases stay FP32; the last
// layer (64 -> 1) is an FP32 dot product of the BF16 activations with the BF16 weights.
//
// Inputs of one proposal at walk point i (x = log irradiance at the walk points, t their times):
//   f[k]     = asinh((x[i-1-k] - x[i]) * 1e4) / 4                       k = 0..7 (the last 8 points, newest first)
//   f[8 + k] = (log2(t[i-k] - t[i-1-k]) - 13) / 10                      their gaps (powers of two, >= 2^13 ns)
// Output: log2(step / min_dt). asinh is log(|z| + sqrt(z^2 + 1)) with this project's deterministic log, so the
// features are bit-identical on the host and the device.
#pragma once

#include "bs_math.cuh"

namespace bs {

constexpr int kMlpIn = 16, kMlpHid = 64;
// FP32 parameter vector: W1 [16 in][64 out], b1 [64], W2 [64 in][64 out], b2 [64], W3 [64], b3.
constexpr int kOffW1 = 0, kOffB1 = 1024, kOffW2 = 1088, kOffB2 = 5184, kOffW3 = 5248, kOffB3 = 5312;
constexpr int kMlpParams = 5313;
constexpr int kMlpParamsPad = 5316;  // row stride of the per-CTA gradient partials
// BF16 operand block (u16 words), in the layouts the mma fragments load with one 32-bit access per register:
// W1t [64 out][16 in], W2t [64 out][64 in] (forward), W2n [64 in][64 out] (backward), W3 [64].
constexpr int kOpW1t = 0, kOpW2t = 1024, kOpW2n = 5120, kOpW3 = 9216, kOpWords = 9280;
// Shared-memory row strides (u16) that make the fragment loads of a warp hit 32 distinct banks.
constexpr int kSW1 = 24, kSW2 = 72, kSF = 24;
constexpr uint32_t kPurposeWalk = 0x0090;   // walk perturbation of the training pairs
constexpr uint32_t kPurposeBatch = 0x0091;  // training batch rows
constexpr uint32_t kPurposeInit = 0x0092;   // initial weights

// FP32 -> BF16, round to nearest even (NaN kept quiet); the same bits on the host and the device.
BS_HD uint16_t bf16_rn(float f) {
  uint32_t u = f2u(f);
  if ((u & 0x7fffffffu) > 0x7f800000u) return static_cast<uint16_t>((u >> 16) | 0x40u);
  u += 0x7fffu + ((u >> 16) & 1u);
  return static_cast<uint16_t>(u >> 16);
}
BS_HD float bf16_f(uint16_t h) { return u2f(static_cast<uint32_t>(h) << 16); }
BS_HD float bf16_round(float f) { return bf16_f(bf16_rn(f)); }

BS_HD float asinh_quarter(float z) {
  const float a = fabs_f(z);
  const float r = log_f(a + sqrtf(a * a + 1.0f)) * 0.25f;
  return z < 0.0f ? -r : r;
}

// The 16 features of walk point (t_i, x_i): hx[k] = x at the k-th previous point (newest first), gaps byte k =
// log2 of the k-th previous gap (byte 0 the newest).
BS_HD void step_features(const float* hx, uint64_t gaps, float x, float* out) {
  for (int k = 0; k < 8; ++k) out[k] = asinh_quarter((hx[k] - x) * 1e4f);
  for (int k = 0; k < 8; ++k) {
    const int g = static_cast<int>((gaps >> (8 * k)) & 0xffu);
    out[8 + k] = static_cast<float>(g - 13) * 0.1f;
  }
}

// log2(step / min_dt) predicted -> the step's log2 in ns: round down after the safety margin, clamp to
// [sh, 23], raise to the plain lattice's step 2^s_floor, and lower until the step starts on its own lattice.
BS_HD int proposal_log2(float y, float margin, int sh, int s_floor, uint32_t cur) {
  float k = y + 0.5f - margin;
  int s;
  if (!(k >= 0.0f)) s = sh;  // NaN or negative
  else if (k >= static_cast<float>(kWindowLog2 - sh)) s = kWindowLog2;
  else s = sh + static_cast<int>(k);
  if (s < s_floor) s = s_floor;
  while (s > 0 && (cur & ((1u << s) - 1u)) != 0u) --s;
  return s;
}

#ifdef __CUDACC__
// D = A B + D for one m16n8k16 tile: A 16 x 16 (row), B 16 x 8 (col), BF16 operands, FP32 accumulators.
// Fragments (g = lane / 4, q = lane % 4): a0 (row g, k 2q..2q+1), a1 (row g + 8, k 2q..), a2 (row g, k 2q+8..),
// a3 (row g + 8, k 2q+8..); b0 (k 2q..2q+1, col g), b1 (k 2q+8.., col g); c0, c1 (row g, cols 2q, 2q+1),
// c2, c3 (row g + 8, cols 2q, 2q+1). The lower k (or column) sits in the low half of each 32-bit register.
__device__ __forceinline__ void mma_bf16(float* c, const uint32_t* a, uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
__device__ __forceinline__ uint32_t ld32(const uint16_t* p) { return *reinterpret_cast<const uint32_t*>(p); }
__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
  return static_cast<uint32_t>(bf16_rn(lo)) | (static_cast<uint32_t>(bf16_rn(hi)) << 16);
}
__device__ __forceinline__ float lo_f(uint32_t r) { return bf16_f(static_cast<uint16_t>(r & 0xffffu)); }
__device__ __forceinline__ float hi_f(uint32_t r) { return bf16_f(static_cast<uint16_t>(r >> 16)); }

// The weights in shared memory, loaded once per CTA.
struct MlpShared {
  uint16_t w1t[kMlpHid * kSW1];
  uint16_t w2t[kMlpHid * kSW2];
  float b1[kMlpHid], b2[kMlpHid], w3[kMlpHid];
  float b3;
};

// All threads of the block call (it ends with __syncthreads).
__device__ inline void mlp_load_shared(MlpShared& s, const uint16_t* ops, const float* params) {
  for (int i = threadIdx.x; i < kMlpHid * kMlpIn; i += blockDim.x) {
    s.w1t[(i / kMlpIn) * kSW1 + i % kMlpIn] = ops[kOpW1t + i];
  }
  for (int i = threadIdx.x; i < kMlpHid * kMlpHid; i += blockDim.x) {
    s.w2t[(i / kMlpHid) * kSW2 + i % kMlpHid] = ops[kOpW2t + i];
  }
  for (int i = threadIdx.x; i < kMlpHid; i += blockDim.x) {
    s.b1[i] = params[kOffB1 + i];
    s.b2[i] = params[kOffB2 + i];
    s.w3[i] = bf16_f(ops[kOpW3 + i]);
  }
  if (threadIdx.x == 0) s.b3 = params[kOffB3];
  __syncthreads();
}

// Forward pass of 32 rows (the warp's feature tile, stride kSF u16) into y[32]. All 32 lanes call.
__device__ inline void mlp_forward_warp(const MlpShared& w, const uint16_t* rows, float* y) {
  const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
#pragma unroll 1
  for (int mt = 0; mt < 2; ++mt) {
    const uint16_t* R = rows + mt * 16 * kSF;
    uint32_t a[4];
    a[0] = ld32(R + g * kSF + 2 * q);
    a[1] = ld32(R + (g + 8) * kSF + 2 * q);
    a[2] = ld32(R + g * kSF + 2 * q + 8);
    a[3] = ld32(R + (g + 8) * kSF + 2 * q + 8);
    uint32_t h1[4][4];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const float b0 = w.b1[8 * j + 2 * q], b1 = w.b1[8 * j + 2 * q + 1];
      float c[4] = {b0, b1, b0, b1};
      mma_bf16(c, a, ld32(w.w1t + (8 * j + g) * kSW1 + 2 * q), ld32(w.w1t + (8 * j + g) * kSW1 + 2 * q + 8));
      h1[j >> 1][(j & 1) * 2 + 0] = pack2(fmaxf(c[0], 0.0f), fmaxf(c[1], 0.0f));
      h1[j >> 1][(j & 1) * 2 + 1] = pack2(fmaxf(c[2], 0.0f), fmaxf(c[3], 0.0f));
    }
    // h1[kk] is the A fragment of k-tile kk: regs (row g, 16kk + 2q), (row g + 8, ...), (row g, 16kk + 8 + 2q), ...
    float y0 = 0.0f, y1 = 0.0f;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const float b0 = w.b2[8 * j + 2 * q], b1 = w.b2[8 * j + 2 * q + 1];
      float c[4] = {b0, b1, b0, b1};
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) {
        const uint32_t a2[4] = {h1[kk][0], h1[kk][1], h1[kk][2], h1[kk][3]};
        mma_bf16(c, a2, ld32(w.w2t + (8 * j + g) * kSW2 + 16 * kk + 2 * q),
                 ld32(w.w2t + (8 * j + g) * kSW2 + 16 * kk + 2 * q + 8));
      }
      const float w30 = w.w3[8 * j + 2 * q], w31 = w.w3[8 * j + 2 * q + 1];
      y0 = y0 + bf16_round(fmaxf(c[0], 0.0f)) * w30;
      y0 = y0 + bf16_round(fmaxf(c[1], 0.0f)) * w31;
      y1 = y1 + bf16_round(fmaxf(c[2], 0.0f)) * w30;
      y1 = y1 + bf16_round(fmaxf(c[3], 0.0f)) * w31;
    }
    y0 += __shfl_xor_sync(0xffffffffu, y0, 1);
    y1 += __shfl_xor_sync(0xffffffffu, y1, 1);
    y0 += __shfl_xor_sync(0xffffffffu, y0, 2);
    y1 += __shfl_xor_sync(0xffffffffu, y1, 2);
    if (q == 0) {
      y[mt * 16 + g] = y0 + w.b3;
      y[mt * 16 + g + 8] = y1 + w.b3;
    }
  }
  __syncwarp();
}
#endif

}  // namespace bs
