// Training of the learned step proposal on the GPU: the walk that turns the plain sampler's runs into
// (history, step) pairs, the fused forward + backward pass on the tensor cores (mma.sync m16n8k16, BF16 operands,
// FP32 accumulators), Adam, and the batch forward pass. No reference counterpart (this project's own method).
//
// One training step = train_partials_kernel (grid = rows / 128 CTAs of 4 warps; each warp runs 32 rows forward
// and back, then the CTA forms its weight gradients over its 128 rows with two more mma passes and writes them as
// one partial row) + adam_kernel (sums the partial rows in a fixed order, so a step is deterministic, and updates
// the FP32 masters and their BF16 operand copies). The step counter lives in device memory, so a run of steps can
// be replayed from a CUDA graph.
#include <cooperative_groups.h>

#include "device.h"

namespace cg = cooperative_groups;

namespace bs {

namespace {

// ---------------------------------------------------------------------------------------------
// training pairs
// ---------------------------------------------------------------------------------------------
struct RunView {
  const int64_t* t;
  const float* v;
  int64_t t_w;
  __device__ uint32_t t_rel(int i) const { return static_cast<uint32_t>(t[i] - t_w); }
};
struct RunAcc {
  const RunView* r;
  __device__ uint32_t t(int i) const { return r->t_rel(i); }
  __device__ float v(int i) const { return r->v[i]; }
};

__device__ __forceinline__ unsigned long long warp_slot(unsigned long long* count) {
  cg::coalesced_group g = cg::coalesced_threads();
  unsigned long long base = 0;
  if (g.thread_rank() == 0) base = atomicAdd(count, static_cast<unsigned long long>(g.size()));
  return g.shfl(base, 0) + g.thread_rank();
}

__device__ __forceinline__ void load_walk(const LearnedSoA& a, uint32_t p, uint32_t n, LearnedPixel& L) {
  for (int k = 0; k < 8; ++k) L.hx[k] = a.hx[static_cast<size_t>(k) * n + p];
  L.gaps = a.gaps[p];
  L.pv = a.pv[p];
  L.valid = a.valid[p];
}
__device__ __forceinline__ void store_walk(const LearnedSoA& a, uint32_t p, uint32_t n, const LearnedPixel& L) {
  for (int k = 0; k < 8; ++k) a.hx[static_cast<size_t>(k) * n + p] = L.hx[k];
  a.gaps[p] = L.gaps;
  a.pv[p] = L.pv;
  a.valid[p] = static_cast<uint8_t>(L.valid);
}

__global__ void __launch_bounds__(128) walk_pairs_kernel(WalkArgs a) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t p = i * a.stride;
  if (p >= a.n_pixels) return;
  const int64_t o0 = a.offsets[p];
  const int n = static_cast<int>(a.offsets[p + 1] - o0);
  RunView rv{a.t + o0, a.irr + o0, a.t_w};
  RunAcc run{&rv};
  LearnedPixel L;
  if (a.reset) learned_reset(L, run.v(0));
  else load_walk(a.st, p, a.n_pixels, L);
  const int s_floor = kWindowLog2 - static_cast<int>(a.level[p]);
  uint32_t cur = 0;
  int i_cur = 0;
  uint32_t step_no = 0;
  while (cur < static_cast<uint32_t>(kWindowNs) && i_cur < n - 1) {
    const float v_cur = run.v(i_cur);
    const float x_cur = log_f(v_cur);
    const int s_star = walk_target(run, n, i_cur, cur, s_floor, a.eps);
    float f[16];
    step_features(L.hx, L.gaps, x_cur, f);
    const unsigned long long slot = warp_slot(a.count);
    if (slot < a.capacity) {
      uint32_t w[8];
      for (int k = 0; k < 8; ++k) {
        w[k] = static_cast<uint32_t>(bf16_rn(f[2 * k])) | (static_cast<uint32_t>(bf16_rn(f[2 * k + 1])) << 16);
      }
      uint4* dst = reinterpret_cast<uint4*>(a.x + slot * kMlpIn);
      dst[0] = make_uint4(w[0], w[1], w[2], w[3]);
      dst[1] = make_uint4(w[4], w[5], w[6], w[7]);
      a.y[slot] = static_cast<float>(s_star - a.sh);
      if (a.key) {
        a.key[slot] = (static_cast<uint64_t>(p) << 32) | (static_cast<uint64_t>(a.window) << 11) | step_no;
      }
    }
    int s_step = s_star - walk_drop(a.seed, p, a.window, step_no);
    if (s_step < s_floor) s_step = s_floor;
    const uint32_t hi = cur + (1u << s_step);
    while (i_cur < n - 1 && run.t(i_cur) < hi) ++i_cur;
    learned_push(L, x_cur, v_cur, s_step);
    cur = hi;
    ++step_no;
  }
  store_walk(a.st, p, a.n_pixels, L);
}

// ---------------------------------------------------------------------------------------------
// training step
// ---------------------------------------------------------------------------------------------
constexpr int kRowsPerCta = 128;
constexpr int kST = kRowsPerCta + 8;  // stride (u16) of the transposed activation tiles [feature][row]

struct TrainShared {
  uint16_t w1t[kMlpHid * kSW1];
  uint16_t w2t[kMlpHid * kSW2];
  uint16_t w2n[kMlpHid * kSW2];
  float b1[kMlpHid], b2[kMlpHid], w3[kMlpHid];
  float b3;
  uint16_t xt[kMlpIn * kST];
  uint16_t h1t[kMlpHid * kST];
  uint16_t dh2t[kMlpHid * kST];
  uint16_t dh1t[kMlpHid * kST];
  float wsum[4][3][kMlpHid];  // per warp: db1, db2, dW3 column sums
  float wdb3[4];
  double wloss[4];
};

__device__ __forceinline__ uint16_t lo16(uint32_t r) { return static_cast<uint16_t>(r & 0xffffu); }
__device__ __forceinline__ uint16_t hi16(uint32_t r) { return static_cast<uint16_t>(r >> 16); }

__global__ void __launch_bounds__(128) train_partials_kernel(TrainArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TrainShared& S = *reinterpret_cast<TrainShared*>(smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, g = lane >> 2, q = lane & 3;
  for (int i = tid; i < kMlpHid * kMlpIn; i += blockDim.x) S.w1t[(i / kMlpIn) * kSW1 + i % kMlpIn] = a.ops[kOpW1t + i];
  for (int i = tid; i < kMlpHid * kMlpHid; i += blockDim.x) {
    S.w2t[(i / kMlpHid) * kSW2 + i % kMlpHid] = a.ops[kOpW2t + i];
    S.w2n[(i / kMlpHid) * kSW2 + i % kMlpHid] = a.ops[kOpW2n + i];
  }
  for (int i = tid; i < kMlpHid; i += blockDim.x) {
    S.b1[i] = a.params[kOffB1 + i];
    S.b2[i] = a.params[kOffB2 + i];
    S.w3[i] = bf16_f(a.ops[kOpW3 + i]);
  }
  if (tid == 0) S.b3 = a.params[kOffB3];
  __syncthreads();

  // This lane's row: local row 32 warp + lane of the CTA.
  const uint32_t gi = blockIdx.x * kRowsPerCta + warp * 32 + lane;
  uint64_t idx = 0;
  bool valid = false;
  if (a.sampled) {
    valid = gi < a.rows;
    if (valid) {
      const U4 u = draw(a.seed, kPurposeBatch, 0u, gi, static_cast<uint64_t>(*a.step));
      idx = ((static_cast<uint64_t>(u.v[0]) << 32) | u.v[1]) % a.n;
    }
  } else {
    valid = gi < a.n;
    idx = gi;
  }
  float dw3[8][2], db2[8][2], db1[8][2];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    dw3[j][0] = dw3[j][1] = db2[j][0] = db2[j][1] = db1[j][0] = db1[j][1] = 0.0f;
  }
  float sdy = 0.0f;
  double sloss = 0.0;
#pragma unroll 1
  for (int mt = 0; mt < 2; ++mt) {
    const int r0 = mt * 16 + g, r1 = r0 + 8;  // warp-local rows
    const uint64_t i0 = __shfl_sync(0xffffffffu, idx, r0), i1 = __shfl_sync(0xffffffffu, idx, r1);
    const bool v0 = __shfl_sync(0xffffffffu, valid, r0), v1 = __shfl_sync(0xffffffffu, valid, r1);
    const int c0 = warp * 32 + r0, c1 = warp * 32 + r1;  // CTA-local rows
    uint32_t ax[4];
    ax[0] = v0 ? ld32(a.x + i0 * kMlpIn + 2 * q) : 0u;
    ax[1] = v1 ? ld32(a.x + i1 * kMlpIn + 2 * q) : 0u;
    ax[2] = v0 ? ld32(a.x + i0 * kMlpIn + 2 * q + 8) : 0u;
    ax[3] = v1 ? ld32(a.x + i1 * kMlpIn + 2 * q + 8) : 0u;
    S.xt[(2 * q) * kST + c0] = lo16(ax[0]);
    S.xt[(2 * q + 1) * kST + c0] = hi16(ax[0]);
    S.xt[(2 * q) * kST + c1] = lo16(ax[1]);
    S.xt[(2 * q + 1) * kST + c1] = hi16(ax[1]);
    S.xt[(2 * q + 8) * kST + c0] = lo16(ax[2]);
    S.xt[(2 * q + 9) * kST + c0] = hi16(ax[2]);
    S.xt[(2 * q + 8) * kST + c1] = lo16(ax[3]);
    S.xt[(2 * q + 9) * kST + c1] = hi16(ax[3]);
    // layer 1
    uint32_t h1[4][4];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const float bb0 = S.b1[8 * j + 2 * q], bb1 = S.b1[8 * j + 2 * q + 1];
      float c[4] = {bb0, bb1, bb0, bb1};
      mma_bf16(c, ax, ld32(S.w1t + (8 * j + g) * kSW1 + 2 * q), ld32(S.w1t + (8 * j + g) * kSW1 + 2 * q + 8));
      const uint32_t top = pack2(fmaxf(c[0], 0.0f), fmaxf(c[1], 0.0f));
      const uint32_t bot = pack2(fmaxf(c[2], 0.0f), fmaxf(c[3], 0.0f));
      h1[j >> 1][(j & 1) * 2 + 0] = top;
      h1[j >> 1][(j & 1) * 2 + 1] = bot;
      S.h1t[(8 * j + 2 * q) * kST + c0] = lo16(top);
      S.h1t[(8 * j + 2 * q + 1) * kST + c0] = hi16(top);
      S.h1t[(8 * j + 2 * q) * kST + c1] = lo16(bot);
      S.h1t[(8 * j + 2 * q + 1) * kST + c1] = hi16(bot);
    }
    // layer 2 and the output
    uint32_t h2[8][2];
    float y0 = 0.0f, y1 = 0.0f;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const float bb0 = S.b2[8 * j + 2 * q], bb1 = S.b2[8 * j + 2 * q + 1];
      float c[4] = {bb0, bb1, bb0, bb1};
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) {
        mma_bf16(c, h1[kk], ld32(S.w2t + (8 * j + g) * kSW2 + 16 * kk + 2 * q),
                 ld32(S.w2t + (8 * j + g) * kSW2 + 16 * kk + 2 * q + 8));
      }
      h2[j][0] = pack2(fmaxf(c[0], 0.0f), fmaxf(c[1], 0.0f));
      h2[j][1] = pack2(fmaxf(c[2], 0.0f), fmaxf(c[3], 0.0f));
      const float w30 = S.w3[8 * j + 2 * q], w31 = S.w3[8 * j + 2 * q + 1];
      y0 = y0 + lo_f(h2[j][0]) * w30;
      y0 = y0 + hi_f(h2[j][0]) * w31;
      y1 = y1 + lo_f(h2[j][1]) * w30;
      y1 = y1 + hi_f(h2[j][1]) * w31;
    }
    y0 += __shfl_xor_sync(0xffffffffu, y0, 1);
    y1 += __shfl_xor_sync(0xffffffffu, y1, 1);
    y0 += __shfl_xor_sync(0xffffffffu, y0, 2);
    y1 += __shfl_xor_sync(0xffffffffu, y1, 2);
    y0 += S.b3;
    y1 += S.b3;
    const float e0 = v0 ? y0 - a.y[i0] : 0.0f, e1 = v1 ? y1 - a.y[i1] : 0.0f;
    const float w0 = 2.0f * (e0 < 0.0f ? a.tau : 1.0f - a.tau), w1 = 2.0f * (e1 < 0.0f ? a.tau : 1.0f - a.tau);
    const float dy0 = w0 * e0 * a.inv_rows, dy1 = w1 * e1 * a.inv_rows;
    if (q == 0) {
      sloss += static_cast<double>(w0) * e0 * e0 + static_cast<double>(w1) * e1 * e1;
      sdy += dy0 + dy1;
    }
    // dH2 = dy W3^T masked by ReLU; the dW3 and db2 column sums
    uint32_t da[4][4];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const float w30 = S.w3[8 * j + 2 * q], w31 = S.w3[8 * j + 2 * q + 1];
      const float h00 = lo_f(h2[j][0]), h01 = hi_f(h2[j][0]), h10 = lo_f(h2[j][1]), h11 = hi_f(h2[j][1]);
      const float d00 = h00 > 0.0f ? dy0 * w30 : 0.0f, d01 = h01 > 0.0f ? dy0 * w31 : 0.0f;
      const float d10 = h10 > 0.0f ? dy1 * w30 : 0.0f, d11 = h11 > 0.0f ? dy1 * w31 : 0.0f;
      dw3[j][0] += h00 * dy0 + h10 * dy1;
      dw3[j][1] += h01 * dy0 + h11 * dy1;
      db2[j][0] += d00 + d10;
      db2[j][1] += d01 + d11;
      const uint32_t top = pack2(d00, d01), bot = pack2(d10, d11);
      da[j >> 1][(j & 1) * 2 + 0] = top;
      da[j >> 1][(j & 1) * 2 + 1] = bot;
      S.dh2t[(8 * j + 2 * q) * kST + c0] = lo16(top);
      S.dh2t[(8 * j + 2 * q + 1) * kST + c0] = hi16(top);
      S.dh2t[(8 * j + 2 * q) * kST + c1] = lo16(bot);
      S.dh2t[(8 * j + 2 * q + 1) * kST + c1] = hi16(bot);
    }
    // dH1 = dH2 W2^T masked by ReLU; the db1 column sums
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      float c[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) {
        mma_bf16(c, da[kk], ld32(S.w2n + (8 * j + g) * kSW2 + 16 * kk + 2 * q),
                 ld32(S.w2n + (8 * j + g) * kSW2 + 16 * kk + 2 * q + 8));
      }
      const uint32_t ht = h1[j >> 1][(j & 1) * 2 + 0], hb = h1[j >> 1][(j & 1) * 2 + 1];
      const float m00 = lo_f(ht) > 0.0f ? c[0] : 0.0f, m01 = hi_f(ht) > 0.0f ? c[1] : 0.0f;
      const float m10 = lo_f(hb) > 0.0f ? c[2] : 0.0f, m11 = hi_f(hb) > 0.0f ? c[3] : 0.0f;
      db1[j][0] += m00 + m10;
      db1[j][1] += m01 + m11;
      S.dh1t[(8 * j + 2 * q) * kST + c0] = bf16_rn(m00);
      S.dh1t[(8 * j + 2 * q + 1) * kST + c0] = bf16_rn(m01);
      S.dh1t[(8 * j + 2 * q) * kST + c1] = bf16_rn(m10);
      S.dh1t[(8 * j + 2 * q + 1) * kST + c1] = bf16_rn(m11);
    }
  }
  // Column sums over the warp's rows: reduce over g (lanes q, q + 4, ..., q + 28).
#pragma unroll
  for (int j = 0; j < 8; ++j) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      float s0 = db1[j][h], s1 = db2[j][h], s2 = dw3[j][h];
#pragma unroll
      for (int o = 4; o < 32; o <<= 1) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, o);
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
        s2 += __shfl_xor_sync(0xffffffffu, s2, o);
      }
      if (g == 0) {
        S.wsum[warp][0][8 * j + 2 * q + h] = s0;
        S.wsum[warp][1][8 * j + 2 * q + h] = s1;
        S.wsum[warp][2][8 * j + 2 * q + h] = s2;
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    sdy += __shfl_xor_sync(0xffffffffu, sdy, o);
    sloss += __shfl_xor_sync(0xffffffffu, sloss, o);
  }
  if (lane == 0) {
    S.wdb3[warp] = sdy;
    S.wloss[warp] = sloss;
  }
  __syncthreads();

  float* out = a.partial + static_cast<size_t>(blockIdx.x) * kMlpParamsPad;
  // dW2 [i][o] = sum_r H1[r][i] dH2[r][o]: warp w takes rows i in [16w, 16w + 16).
#pragma unroll 1
  for (int j = 0; j < 8; ++j) {
    float c[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int kk = 0; kk < kRowsPerCta / 16; ++kk) {
      uint32_t aa[4];
      aa[0] = ld32(S.h1t + (16 * warp + g) * kST + 16 * kk + 2 * q);
      aa[1] = ld32(S.h1t + (16 * warp + g + 8) * kST + 16 * kk + 2 * q);
      aa[2] = ld32(S.h1t + (16 * warp + g) * kST + 16 * kk + 2 * q + 8);
      aa[3] = ld32(S.h1t + (16 * warp + g + 8) * kST + 16 * kk + 2 * q + 8);
      mma_bf16(c, aa, ld32(S.dh2t + (8 * j + g) * kST + 16 * kk + 2 * q),
               ld32(S.dh2t + (8 * j + g) * kST + 16 * kk + 2 * q + 8));
    }
    const int i0 = 16 * warp + g, o0 = 8 * j + 2 * q;
    out[kOffW2 + i0 * kMlpHid + o0] = c[0];
    out[kOffW2 + i0 * kMlpHid + o0 + 1] = c[1];
    out[kOffW2 + (i0 + 8) * kMlpHid + o0] = c[2];
    out[kOffW2 + (i0 + 8) * kMlpHid + o0 + 1] = c[3];
  }
  // dW1 [f][h] = sum_r X[r][f] dH1[r][h]: warp w takes columns h in [16w, 16w + 16).
#pragma unroll 1
  for (int jj = 0; jj < 2; ++jj) {
    const int j = 2 * warp + jj;
    float c[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int kk = 0; kk < kRowsPerCta / 16; ++kk) {
      uint32_t aa[4];
      aa[0] = ld32(S.xt + g * kST + 16 * kk + 2 * q);
      aa[1] = ld32(S.xt + (g + 8) * kST + 16 * kk + 2 * q);
      aa[2] = ld32(S.xt + g * kST + 16 * kk + 2 * q + 8);
      aa[3] = ld32(S.xt + (g + 8) * kST + 16 * kk + 2 * q + 8);
      mma_bf16(c, aa, ld32(S.dh1t + (8 * j + g) * kST + 16 * kk + 2 * q),
               ld32(S.dh1t + (8 * j + g) * kST + 16 * kk + 2 * q + 8));
    }
    const int h0 = 8 * j + 2 * q;
    out[kOffW1 + g * kMlpHid + h0] = c[0];
    out[kOffW1 + g * kMlpHid + h0 + 1] = c[1];
    out[kOffW1 + (g + 8) * kMlpHid + h0] = c[2];
    out[kOffW1 + (g + 8) * kMlpHid + h0 + 1] = c[3];
  }
  if (tid < kMlpHid) {
    out[kOffB1 + tid] = ((S.wsum[0][0][tid] + S.wsum[1][0][tid]) + S.wsum[2][0][tid]) + S.wsum[3][0][tid];
    out[kOffB2 + tid] = ((S.wsum[0][1][tid] + S.wsum[1][1][tid]) + S.wsum[2][1][tid]) + S.wsum[3][1][tid];
    out[kOffW3 + tid] = ((S.wsum[0][2][tid] + S.wsum[1][2][tid]) + S.wsum[2][2][tid]) + S.wsum[3][2][tid];
  }
  if (tid == 0) {
    out[kOffB3] = ((S.wdb3[0] + S.wdb3[1]) + S.wdb3[2]) + S.wdb3[3];
    a.partial_loss[blockIdx.x] = ((S.wloss[0] + S.wloss[1]) + S.wloss[2]) + S.wloss[3];
  }
}

// The BF16 operand copies of parameter p (FP32 master value v).
__device__ __forceinline__ void write_operand(uint16_t* ops, int p, float v) {
  const uint16_t h = bf16_rn(v);
  if (p < kOffB1) {
    const int i = p / kMlpHid, o = p % kMlpHid;
    ops[kOpW1t + o * kMlpIn + i] = h;
  } else if (p >= kOffW2 && p < kOffB2) {
    const int i = (p - kOffW2) / kMlpHid, o = (p - kOffW2) % kMlpHid;
    ops[kOpW2t + o * kMlpHid + i] = h;
    ops[kOpW2n + i * kMlpHid + o] = h;
  } else if (p >= kOffW3 && p < kOffB3) {
    ops[kOpW3 + p - kOffW3] = h;
  }
}

__global__ void operands_kernel(const float* params, uint16_t* ops) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < kMlpParams) write_operand(ops, p, params[p]);
}

__global__ void adam_kernel(float* params, float* m, float* v, uint16_t* ops, const float* partial,
                            const double* partial_loss, int ctas, float lr, float inv_rows, int64_t* step,
                            float* losses, int64_t loss_cap, unsigned int* done) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t s = *step;  // completed steps before this one
  if (p < kMlpParams) {
    float gsum = 0.0f;
    for (int c = 0; c < ctas; ++c) gsum += partial[static_cast<size_t>(c) * kMlpParamsPad + p];
    const float b1 = 0.9f, b2 = 0.999f;
    const float mm = b1 * m[p] + (1.0f - b1) * gsum;
    const float vv = b2 * v[p] + (1.0f - b2) * gsum * gsum;
    m[p] = mm;
    v[p] = vv;
    const double t = static_cast<double>(s + 1);
    const float c1 = static_cast<float>(1.0 - pow(0.9, t)), c2 = static_cast<float>(1.0 - pow(0.999, t));
    const float np = params[p] - lr * (mm / c1) / (sqrtf(vv / c2) + 1e-8f);
    params[p] = np;
    write_operand(ops, p, np);
  }
  // The last block to finish records the loss and advances the step counter (every block has read it).
  __syncthreads();
  __shared__ bool last;
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(done, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    double l = 0.0;
    for (int c = 0; c < ctas; ++c) l += partial_loss[c];
    if (losses && s < loss_cap) losses[s] = static_cast<float>(l * 0.5 * inv_rows);
    *step = s + 1;
    *done = 0u;
    __threadfence();
  }
}

__global__ void reduce_partials_kernel(const float* partial, const double* partial_loss, int ctas, float inv_rows,
                                       double* grad, double* loss) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < kMlpParams) {
    double s = 0.0;
    for (int c = 0; c < ctas; ++c) s += partial[static_cast<size_t>(c) * kMlpParamsPad + p];
    grad[p] = s;
  }
  if (p == 0) {
    double l = 0.0;
    for (int c = 0; c < ctas; ++c) l += partial_loss[c];
    *loss = l * 0.5 * inv_rows;
  }
}

__global__ void __launch_bounds__(128) mlp_forward_kernel(const uint16_t* ops, const float* params, const uint16_t* x,
                                                          uint64_t n, float* y) {
  __shared__ MlpShared W;
  __shared__ __align__(16) uint16_t rows[4][32 * kSF];
  __shared__ float ys[4][32];
  mlp_load_shared(W, ops, params);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint64_t r = static_cast<uint64_t>(blockIdx.x) * 128 + warp * 32 + lane;
  uint4* dst = reinterpret_cast<uint4*>(rows[warp] + lane * kSF);
  if (r < n) {
    const uint4* src = reinterpret_cast<const uint4*>(x + r * kMlpIn);
    dst[0] = src[0];
    dst[1] = src[1];
  } else {
    dst[0] = make_uint4(0u, 0u, 0u, 0u);
    dst[1] = make_uint4(0u, 0u, 0u, 0u);
  }
  __syncwarp();
  mlp_forward_warp(W, rows[warp], ys[warp]);
  if (r < n) y[r] = ys[warp][lane];
}

}  // namespace

void launch_walk_pairs(const WalkArgs& a, cudaStream_t stream) {
  const uint32_t walkers = (a.n_pixels + a.stride - 1) / a.stride;
  if (walkers == 0) return;
  walk_pairs_kernel<<<(walkers + 127) / 128, 128, 0, stream>>>(a);
}

int train_grid(uint32_t rows) { return static_cast<int>((rows + kRowsPerCta - 1) / kRowsPerCta); }

void launch_train_partials(const TrainArgs& a, cudaStream_t stream) {
  static bool configured = false;
  const int bytes = static_cast<int>(sizeof(TrainShared));
  if (!configured) {
    cudaFuncSetAttribute(train_partials_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    configured = true;
  }
  train_partials_kernel<<<train_grid(a.rows), kRowsPerCta, bytes, stream>>>(a);
}

void launch_adam(float* params, float* m, float* v, uint16_t* ops, const float* partial, const double* partial_loss,
                 int ctas, float lr, float inv_rows, int64_t* step, float* losses, int64_t loss_cap,
                 unsigned int* done, cudaStream_t stream) {
  adam_kernel<<<(kMlpParams + 255) / 256, 256, 0, stream>>>(params, m, v, ops, partial, partial_loss, ctas, lr,
                                                             inv_rows, step, losses, loss_cap, done);
}

void launch_reduce_partials(const float* partial, const double* partial_loss, int ctas, float inv_rows,
                            double* grad, double* loss, cudaStream_t stream) {
  reduce_partials_kernel<<<(kMlpParams + 255) / 256, 256, 0, stream>>>(partial, partial_loss, ctas, inv_rows, grad,
                                                                       loss);
}

void launch_operands(const float* params, uint16_t* ops, cudaStream_t stream) {
  operands_kernel<<<(kMlpParams + 255) / 256, 256, 0, stream>>>(params, ops);
}

void launch_mlp_forward(const uint16_t* ops, const float* params, const uint16_t* x, uint64_t n, float* y,
                        cudaStream_t stream) {
  if (n == 0) return;
  mlp_forward_kernel<<<static_cast<unsigned>((n + 127) / 128), 128, 0, stream>>>(ops, params, x, n, y);
}

}  // namespace bs
