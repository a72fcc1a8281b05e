// Training of the learned step proposal on the GPU: the walk that turns the plain sampler's runs into
// (history, step) pairs, the fused forward + backward pass on the 5th-generation tensor cores (tcgen05.mma, BF16
// operands from shared memory, FP32 accumulators in tensor memory), Adam, and the batch forward pass. No reference
// counterpart (this project's own method).
//
// One training step = train_partials_kernel (grid = rows / 128 CTAs of 4 warps, one thread per row; the CTA runs
// its 128 rows forward and back and forms its weight gradients over them, five tcgen05 chains in all, and writes them
// as one partial row) + adam_kernel (sums the partial rows in a fixed order, so a step is deterministic, and updates
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
// training step on the 5th-generation tensor cores
// ---------------------------------------------------------------------------------------------
// A CTA takes 128 rows of the batch, one thread per row; each of its five contractions is one tcgen05.mma chain of
// M = 128 (the rows, or for the weight gradients the weight's rows padded to 128), N = 64, K = 16 per instruction,
// BF16 operands from shared memory and an FP32 accumulator in tensor memory (TMEM lane t = the tile's row t, so
// thread t reads its own row back with tcgen05.ld):
//   H1 = relu(X W1 + b1)          X [128 x 16],   W1^T [64 x 16]   (both K-major)
//   H2 = relu(H1 W2 + b2)         H1 [128 x 64],  W2^T [64 x 64]   (K-major); y = H2 w3 + b3 per thread
//   dH1 = (dH2 W2^T) * [H1 > 0]   dH2 [128 x 64], W2 [64 x 64]     (K-major)
//   dW2 = H1^T dH2, dW1 = X^T dH1 over the 128 rows               (the same tiles read MN-major)
// One thread (tid 0) issues each chain and commits it to an mbarrier that the CTA waits on; the bias and w3
// gradients and the loss are column sums over the rows, taken in a fixed order (shuffles within each warp, then
// the four warps), so a step is deterministic. BF16 rounding happens where the mma.sync form rounded (X, H1, dH2, dH1 and the weights).
//
// Tiles use the tensor core's canonical no-swizzle layout: a [rows][cols] BF16 matrix in core matrices of 8 rows x 8
// columns (16 bytes a row, 128 contiguous bytes), core (rb, cb) at byte (rb * cols / 8 + cb) * 128. Read with K
// along the columns (K-major) the descriptor's leading offset is 128 (the next 8 columns) and its stride offset
// cols * 16 (the next 8 rows); read with K along the rows (MN-major, for the transposed operands) the same bytes have
// stride offset 128 and leading offset cols * 16.
constexpr int kRowsPerCta = 128;
constexpr int kMmaWaitLimit = 1 << 20;  // mbarrier polls before a wait gives up (the step's error word is set)

__host__ __device__ constexpr uint32_t tile_off(int r, int c, int cols) {
  return static_cast<uint32_t>(((r >> 3) * (cols >> 3) + (c >> 3)) * 128 + (r & 7) * 16 + (c & 7) * 2);
}

// The transposed reads with M = 128 run past a tile whose M is smaller (X^T: 16 rows, H1^T: 64 rows) into the next
// member, which is why x is followed by w1t and h1 by dh2; those accumulator rows are never read.
struct __align__(128) TrainTiles {
  uint8_t x[kRowsPerCta * kMlpIn * 2];    // X [r][f]
  uint8_t w1t[kMlpHid * kMlpIn * 2];      // W1^T [h][f]
  uint8_t h1[kRowsPerCta * kMlpHid * 2];  // H1 [r][h]
  uint8_t dh2[kRowsPerCta * kMlpHid * 2]; // dH2 [r][o]
  uint8_t dh1[kRowsPerCta * kMlpHid * 2]; // dH1 [r][h]
  uint8_t w2t[kMlpHid * kMlpHid * 2];     // W2^T [o][h]
  uint8_t w2n[kMlpHid * kMlpHid * 2];     // W2 [h][o]
  float part[3][4][kMlpHid];             // per warp: the db2, dW3 and db1 column sums of its 32 rows
  float b1[kMlpHid], b2[kMlpHid], w3[kMlpHid];
  float b3;
  float wdb3[4];
  double wloss[4];
  unsigned long long bar;
  uint32_t tmem;
};
static_assert(offsetof(TrainTiles, w1t) == sizeof(TrainTiles::x) && offsetof(TrainTiles, dh2) ==
              offsetof(TrainTiles, h1) + sizeof(TrainTiles::h1), "the transposed reads' overrun targets");
static_assert(offsetof(TrainTiles, w1t) + sizeof(TrainTiles::w1t) >= 15 * 128 + 7 * 512 + 256 + 128,
              "X^T's overrun stays inside w1t");
static_assert(offsetof(TrainTiles, h1) % 128 == 0 && offsetof(TrainTiles, dh1) % 128 == 0 &&
              offsetof(TrainTiles, w2t) % 128 == 0 && offsetof(TrainTiles, w2n) % 128 == 0 &&
              offsetof(TrainTiles, bar) % 8 == 0, "tile alignment");

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// A shared-memory matrix descriptor: no swizzle, version 1 (bits 46-47), the start and both offsets in 16-byte
// units.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return static_cast<uint64_t>((saddr >> 4) & 0x3FFFu) | (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) |
         (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (uint64_t{1} << 46);
}

// The instruction descriptor of kind::f16: FP32 accumulator (bits 4-5 = 1), BF16 A and B (bits 7-9, 10-12 = 1),
// A and B major (bits 15, 16: 0 K-major, 1 MN-major), N / 8 (bits 17-22), M / 16 (bits 24-28); M = 128, N = 64.
__host__ __device__ constexpr uint32_t umma_idesc(bool mn_major) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (mn_major ? (1u << 15) | (1u << 16) : 0u) | ((64u >> 3) << 17) |
         ((128u >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      :
      : "r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}

__device__ __forceinline__ void umma_commit(unsigned long long* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// This thread's shared-memory writes made visible to the tensor core (the async proxy).
__device__ __forceinline__ void proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Polls the barrier's phase of the given parity; false after kMmaWaitLimit polls.
__device__ __forceinline__ bool bar_wait(unsigned long long* bar, uint32_t parity) {
  const uint32_t b = smem_u32(bar);
  for (int i = 0; i < kMmaWaitLimit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(b), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// Waits for the chain committed to the barrier's phase; a wait that gives up sets the error word and waits once more
// (the chain's TMEM must not be freed under it).
__device__ __forceinline__ void chain_wait(unsigned long long* bar, uint32_t parity, unsigned int* err) {
  if (!bar_wait(bar, parity)) {
    if (threadIdx.x == 0) atomicOr(err, 1u);
    bar_wait(bar, parity);
  }
  tc_fence_after();
}

// 16 FP32 columns of this thread's TMEM lane (the warp's 32 lanes, starting at column col of taddr).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
      "[%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
// 64 FP32 columns of this thread's lane.
__device__ __forceinline__ void tmem_ld64(uint32_t taddr, float (&v)[64]) {
  tmem_ld16(taddr, v);
  tmem_ld16(taddr + 16, v + 16);
  tmem_ld16(taddr + 32, v + 32);
  tmem_ld16(taddr + 48, v + 48);
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Row t of a [rows][64] tile from 32 packed BF16 pairs.
__device__ __forceinline__ void store_row64(uint8_t* tile, int t, const uint32_t (&p)[32]) {
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    *reinterpret_cast<uint4*>(tile + tile_off(t, 8 * j, kMlpHid)) =
        make_uint4(p[4 * j], p[4 * j + 1], p[4 * j + 2], p[4 * j + 3]);
  }
}

// The warp's column sums of v (64 columns, one row per lane), reduced and scattered: halving exchanges with the
// lanes 16, 8, 4, 2 and 1 apart, each lane keeping the half its lane bit selects, leave lane l the sums of columns
// 2l and 2l + 1 in v[0] and v[1] (a fixed order, so the sums are deterministic).
__device__ __forceinline__ void warp_column_sums(float (&v)[64], int lane) {
#pragma unroll
  for (int s = 16, n = 64; s >= 1; s >>= 1, n >>= 1) {
    const bool up = (lane & s) != 0;
#pragma unroll
    for (int i = 0; i < n / 2; ++i) {
      const float keep = up ? v[i + n / 2] : v[i], send = up ? v[i] : v[i + n / 2];
      v[i] = keep + __shfl_xor_sync(0xffffffffu, send, s);
    }
  }
}

__global__ void __launch_bounds__(128, 1) train_partials_kernel(TrainArgs a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  TrainTiles& S = *reinterpret_cast<TrainTiles*>(smem_raw);
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  if (warp == 0) {  // 128 TMEM columns: two 64-column accumulators
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S.tmem)),
                 "r"(128u)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (t == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&S.bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // The operands of the weights (BF16, row-major in ops) into their tiles.
  {
    const int h = t >> 1, j = t & 1;
    *reinterpret_cast<uint4*>(S.w1t + tile_off(h, 8 * j, kMlpIn)) =
        *reinterpret_cast<const uint4*>(a.ops + kOpW1t + h * kMlpIn + 8 * j);
  }
  for (int q = t; q < kMlpHid * 8; q += kRowsPerCta) {
    const int r = q >> 3, j = q & 7;
    *reinterpret_cast<uint4*>(S.w2t + tile_off(r, 8 * j, kMlpHid)) =
        *reinterpret_cast<const uint4*>(a.ops + kOpW2t + r * kMlpHid + 8 * j);
    *reinterpret_cast<uint4*>(S.w2n + tile_off(r, 8 * j, kMlpHid)) =
        *reinterpret_cast<const uint4*>(a.ops + kOpW2n + r * kMlpHid + 8 * j);
  }
  if (t < kMlpHid) {
    S.b1[t] = a.params[kOffB1 + t];
    S.b2[t] = a.params[kOffB2 + t];
    S.w3[t] = bf16_f(a.ops[kOpW3 + t]);
  }
  if (t == 0) S.b3 = a.params[kOffB3];

  // This thread's row.
  const uint32_t gi = blockIdx.x * kRowsPerCta + t;
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
  {
    uint32_t xw[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) xw[k] = valid ? ld32(a.x + idx * kMlpIn + 2 * k) : 0u;
    *reinterpret_cast<uint4*>(S.x + tile_off(t, 0, kMlpIn)) = make_uint4(xw[0], xw[1], xw[2], xw[3]);
    *reinterpret_cast<uint4*>(S.x + tile_off(t, 8, kMlpIn)) = make_uint4(xw[4], xw[5], xw[6], xw[7]);
  }
  proxy_fence();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = S.tmem;
  const uint32_t lane_base = static_cast<uint32_t>(32 * warp) << 16;  // this warp's TMEM lanes
  const uint32_t acc_a = tmem, acc_b = tmem + 64;                      // the two accumulators (columns)
  constexpr uint32_t kK = umma_idesc(false), kMN = umma_idesc(true);
  const uint32_t sx = smem_u32(S.x), sw1 = smem_u32(S.w1t), sh1 = smem_u32(S.h1), sdh2 = smem_u32(S.dh2),
                 sdh1 = smem_u32(S.dh1), sw2t = smem_u32(S.w2t), sw2n = smem_u32(S.w2n);

  // Layer 1 into accumulator a.
  if (t == 0) {
    umma_bf16(acc_a, umma_desc(sx, 128, 256), umma_desc(sw1, 128, 256), kK, 0u);
    umma_commit(&S.bar);
  }
  chain_wait(&S.bar, 0, a.err);
  float acc[64];
  uint32_t h1p[32];
  tmem_ld64(acc_a + lane_base, acc);
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    h1p[j] = pack2(fmaxf(acc[2 * j] + S.b1[2 * j], 0.0f), fmaxf(acc[2 * j + 1] + S.b1[2 * j + 1], 0.0f));
  }
  store_row64(S.h1, t, h1p);
  proxy_fence();
  tc_fence_before();
  __syncthreads();

  // Layer 2 into accumulator b.
  if (t == 0) {
    tc_fence_after();
#pragma unroll
    for (int s = 0; s < kMlpHid / 16; ++s) {
      umma_bf16(acc_b, umma_desc(sh1 + 256 * s, 128, 1024), umma_desc(sw2t + 256 * s, 128, 1024), kK, s > 0);
    }
    umma_commit(&S.bar);
  }
  chain_wait(&S.bar, 1, a.err);
  tmem_ld64(acc_b + lane_base, acc);
  float y = 0.0f;
#pragma unroll
  for (int o = 0; o < kMlpHid; ++o) y = y + bf16_round(fmaxf(acc[o] + S.b2[o], 0.0f)) * S.w3[o];
  y += S.b3;
  const float e = valid ? y - a.y[idx] : 0.0f;
  const float wgt = 2.0f * (e < 0.0f ? a.tau : 1.0f - a.tau);
  const float dy = wgt * e * a.inv_rows;
  // dH2 = dy w3 masked by ReLU: the tile (BF16); its FP32 values summed down the columns for db2.
  {
    uint32_t dp[32];
    float v[64];
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      const float h0 = bf16_round(fmaxf(acc[2 * j] + S.b2[2 * j], 0.0f));
      const float h1v = bf16_round(fmaxf(acc[2 * j + 1] + S.b2[2 * j + 1], 0.0f));
      const float d0 = h0 > 0.0f ? dy * S.w3[2 * j] : 0.0f, d1 = h1v > 0.0f ? dy * S.w3[2 * j + 1] : 0.0f;
      v[2 * j] = d0;
      v[2 * j + 1] = d1;
      dp[j] = pack2(d0, d1);
    }
    store_row64(S.dh2, t, dp);
    warp_column_sums(v, lane);
    S.part[0][warp][2 * lane] = v[0];
    S.part[0][warp][2 * lane + 1] = v[1];
  }
  // db3 and the loss: the warp's rows, then the warps in order.
  {
    float sdy = dy;
    double sl = static_cast<double>(wgt) * e * e;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      sdy += __shfl_xor_sync(0xffffffffu, sdy, o);
      sl += __shfl_xor_sync(0xffffffffu, sl, o);
    }
    if (lane == 0) {
      S.wdb3[warp] = sdy;
      S.wloss[warp] = sl;
    }
  }
  proxy_fence();
  tc_fence_before();
  __syncthreads();

  // dH1 into accumulator a, while the CTA sums db2 and dW3.
  if (t == 0) {
    tc_fence_after();
#pragma unroll
    for (int s = 0; s < kMlpHid / 16; ++s) {
      umma_bf16(acc_a, umma_desc(sdh2 + 256 * s, 128, 1024), umma_desc(sw2n + 256 * s, 128, 1024), kK, s > 0);
    }
    umma_commit(&S.bar);
  }
#pragma unroll
  for (int o = 0; o < kMlpHid; ++o) acc[o] = bf16_round(fmaxf(acc[o] + S.b2[o], 0.0f)) * dy;
  warp_column_sums(acc, lane);
  S.part[1][warp][2 * lane] = acc[0];
  S.part[1][warp][2 * lane + 1] = acc[1];
  chain_wait(&S.bar, 0, a.err);
  tmem_ld64(acc_a + lane_base, acc);
  {
    uint32_t dp[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      const float m0 = lo_f(h1p[j]) > 0.0f ? acc[2 * j] : 0.0f, m1 = hi_f(h1p[j]) > 0.0f ? acc[2 * j + 1] : 0.0f;
      acc[2 * j] = m0;
      acc[2 * j + 1] = m1;
      dp[j] = pack2(m0, m1);
    }
    store_row64(S.dh1, t, dp);
  }
  proxy_fence();
  tc_fence_before();
  __syncthreads();

  // dW2 = H1^T dH2 into accumulator b, dW1 = X^T dH1 into accumulator a (K = the 128 rows, MN-major reads).
  if (t == 0) {
    tc_fence_after();
#pragma unroll
    for (int s = 0; s < kRowsPerCta / 16; ++s) {
      umma_bf16(acc_b, umma_desc(sh1 + 2048 * s, 1024, 128), umma_desc(sdh2 + 2048 * s, 1024, 128), kMN, s > 0);
    }
#pragma unroll
    for (int s = 0; s < kRowsPerCta / 16; ++s) {
      umma_bf16(acc_a, umma_desc(sx + 512 * s, 256, 128), umma_desc(sdh1 + 2048 * s, 1024, 128), kMN, s > 0);
    }
    umma_commit(&S.bar);
  }
  warp_column_sums(acc, lane);
  S.part[2][warp][2 * lane] = acc[0];
  S.part[2][warp][2 * lane + 1] = acc[1];
  __syncthreads();
  float* out = a.partial + static_cast<size_t>(blockIdx.x) * kMlpParamsPad;
  if (t < kMlpHid) {  // the column sums: the four warps' in order
    out[kOffB2 + t] = ((S.part[0][0][t] + S.part[0][1][t]) + S.part[0][2][t]) + S.part[0][3][t];
    out[kOffW3 + t] = ((S.part[1][0][t] + S.part[1][1][t]) + S.part[1][2][t]) + S.part[1][3][t];
    out[kOffB1 + t] = ((S.part[2][0][t] + S.part[2][1][t]) + S.part[2][2][t]) + S.part[2][3][t];
  }
  chain_wait(&S.bar, 1, a.err);
  if (warp < 2) {  // dW2 [h][o]: rows 0-63 of accumulator b
    tmem_ld64(acc_b + lane_base, acc);
    float4* dst = reinterpret_cast<float4*>(out + kOffW2 + t * kMlpHid);
#pragma unroll
    for (int o = 0; o < kMlpHid / 4; ++o) {
      dst[o] = make_float4(acc[4 * o], acc[4 * o + 1], acc[4 * o + 2], acc[4 * o + 3]);
    }
  }
  if (warp == 0) {  // dW1 [f][h]: rows 0-15 of accumulator a
    tmem_ld64(acc_a + lane_base, acc);
    if (lane < kMlpIn) {
      float4* dst = reinterpret_cast<float4*>(out + kOffW1 + lane * kMlpHid);
#pragma unroll
      for (int h = 0; h < kMlpHid / 4; ++h) {
        dst[h] = make_float4(acc[4 * h], acc[4 * h + 1], acc[4 * h + 2], acc[4 * h + 3]);
      }
    }
  }
  if (t == 0) {
    out[kOffB3] = ((S.wdb3[0] + S.wdb3[1]) + S.wdb3[2]) + S.wdb3[3];
    a.partial_loss[blockIdx.x] = ((S.wloss[0] + S.wloss[1]) + S.wloss[2]) + S.wloss[3];
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128u) : "memory");
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
  const int bytes = static_cast<int>(sizeof(TrainTiles));
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
