// The device kernels of the path (sm_100a): sensor init, the pixel model over CSR sample runs (the
// SensorModel::advance_device boundary, src/sensor/sensor_model.h:157-167), the window sampler writing CSR runs
// (sample_window, src/engine/bindings/engine_module.cpp:311-355), and the fused engine that samples and senses
// every window of every sensor with each pixel's state in registers (the reference's Camera::sample_and_sense,
// src/engine/engine_impl.h:1253-1357, without the runs ever reaching HBM).
//
// Events leave through warp-aggregated atomics: the lanes that emit together take one slot range with one atomic
// (coalesced group rank), and a call whose events exceed the buffer is re-run from its unchanged input state.
#include <cooperative_groups.h>

#include "device.h"

namespace cg = cooperative_groups;

namespace bs {

namespace {

// Appends events to one sensor's buffer; the lanes of a warp that push together share one atomic, so every lane of
// the warp must push to the same buffer (a warp works on one tile of one sensor).
struct GlobalSink {
  EventBuf ev;
  unsigned long long* count;
  __device__ __forceinline__ void push(const RawEvent& e) {
    cg::coalesced_group g = cg::coalesced_threads();
    unsigned long long base = 0;
    if (g.thread_rank() == 0) base = atomicAdd(count, static_cast<unsigned long long>(g.size()));
    base = g.shfl(base, 0);
    const unsigned long long i = base + g.thread_rank();
    if (i < ev.capacity) {
      const uint4* src = reinterpret_cast<const uint4*>(&e);
      uint4* dst = reinterpret_cast<uint4*>(ev.data + i);
      dst[0] = src[0];
      dst[1] = src[1];
    }
  }
};

// Appends each event with the pushing thread's own atomic: for a kernel whose lanes serve pixels of different
// sensors (engine_rest_kernel).
struct ThreadSink {
  EventBuf ev;
  unsigned long long* count;
  __device__ __forceinline__ void push(const RawEvent& e) {
    const unsigned long long i = atomicAdd(count, 1ull);
    if (i < ev.capacity) {
      const uint4* src = reinterpret_cast<const uint4*>(&e);
      uint4* dst = reinterpret_cast<uint4*>(ev.data + i);
      dst[0] = src[0];
      dst[1] = src[1];
    }
  }
};

__device__ __forceinline__ void load_state(const StateSoA& a, uint32_t p, bool noise, PixelRegs& s) {
  s.t_ref = a.t_ref[p];
  s.t_search = a.t_search[p];
  s.blind_until = a.blind_until[p];
  s.s3_ref = a.s3_ref[p];
  s.n3_ref = a.n3_ref[p];
  s.dr_ref = a.dr_ref[p];
  s.i_scale = a.i_scale[p];
  s.held = a.held[p];
  s.flags = a.flags[p];
  if (noise) {
    s.t_shot = a.t_shot[p];
    s.t_ba = a.t_ba[p];
    s.n_shot = a.n_shot[p];
    s.n_ba = a.n_ba[p];
  } else {
    s.t_shot = s.t_ba = kForever;
    s.n_shot = s.n_ba = 0;
  }
}

__device__ __forceinline__ void store_state(const StateSoA& a, uint32_t p, bool noise, const PixelRegs& s) {
  a.t_ref[p] = s.t_ref;
  a.t_search[p] = s.t_search;
  a.blind_until[p] = s.blind_until;
  a.s3_ref[p] = s.s3_ref;
  a.n3_ref[p] = s.n3_ref;
  a.dr_ref[p] = s.dr_ref;
  a.i_scale[p] = s.i_scale;
  a.held[p] = s.held;
  a.flags[p] = s.flags;
  if (noise) {
    a.t_shot[p] = s.t_shot;
    a.t_ba[p] = s.t_ba;
    a.n_shot[p] = s.n_shot;
    a.n_ba[p] = s.n_ba;
  }
}

__device__ __forceinline__ void load_cascade(const StateSoA& a, uint32_t p, CascadeRegs& q) {
  q.z = a.z[p];
  q.x1 = a.x1[p];
  q.s2 = a.s2[p];
  q.s3 = a.s3[p];
  q.tv = a.tv[p];
}

__device__ __forceinline__ void store_cascade(const StateSoA& a, uint32_t p, const CascadeRegs& q) {
  a.z[p] = q.z;
  a.x1[p] = q.x1;
  a.s2[p] = q.s2;
  a.s3[p] = q.s3;
  a.tv[p] = q.tv;
}

__device__ __forceinline__ void load_lattice(const StateSoA& a, uint32_t p, uint32_t n, LatticeRegs& L) {
  for (int i = 0; i < 3; ++i) {
    L.nk[i] = a.lat[static_cast<size_t>(i) * n + p];
    L.nk1[i] = a.lat[static_cast<size_t>(3 + i) * n + p];
  }
  L.ln_a1 = a.lat[static_cast<size_t>(6) * n + p];
  L.rho = a.lat[static_cast<size_t>(7) * n + p];
  L.cell = a.cell[p];
  L.have_k1 = a.have_k1[p];
}

__device__ __forceinline__ void store_lattice(const StateSoA& a, uint32_t p, uint32_t n, const LatticeRegs& L) {
  for (int i = 0; i < 3; ++i) {
    a.lat[static_cast<size_t>(i) * n + p] = L.nk[i];
    a.lat[static_cast<size_t>(3 + i) * n + p] = L.nk1[i];
  }
  a.lat[static_cast<size_t>(6) * n + p] = L.ln_a1;
  a.lat[static_cast<size_t>(7) * n + p] = L.rho;
  a.cell[p] = L.cell;
  a.have_k1[p] = L.have_k1;
}

// Drops events (the init of the noise lattice fires nothing).
struct NullSink {
  __device__ void push(const RawEvent&) {}
};

__device__ __forceinline__ void load_map(const MapSoA& m, uint32_t p, PixelMapRegs& r) {
  r.theta_on = m.theta_on[p];
  r.theta_off = m.theta_off[p];
  r.leak = m.leak[p];
  r.dark = m.dark[p];
  r.scale = m.scale[p];
  r.ba_rate_hz = m.ba_rate[p];
  r.shot_max_hz = m.shot_max[p];
}

// Sums a value over the warp and adds it to a counter from lane 0 (all 32 lanes must call).
__device__ __forceinline__ void warp_add(unsigned long long* dst, unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0 && v != 0ull) atomicAdd(dst, v);
}
__device__ __forceinline__ void warp_or(unsigned long long* dst, unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v |= __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0 && v != 0ull) atomicOr(dst, v);
}

// ---------------------------------------------------------------------------------------------
// init
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(128) init_kernel(SensorConsts k, CascadeConsts cc, NoiseTableDev tab, MapSoA map,
                                                   StateSoA st, uint32_t n_pixels, int64_t t0, const float* irr0,
                                                   const uint32_t* pixel_ids, unsigned long long* counters) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long clamps = 0, err = 0;
  if (p < n_pixels) {
    const float raw = irr0[p];
    if (!isfinite(raw)) err |= kErrNonFinite;
    const float v = clamp_irr(raw, k.irr_max);
    if (!(v == raw)) ++clamps;
    PixelMapRegs m;
    load_map(map, p, m);
    PixelRegs s;
    pixel_init(s, m, k, pixel_ids ? pixel_ids[p] : p, t0, v, map.phi0[p]);
    store_state(st, p, true, s);
    if (k.cascade) {
      CascadeRegs q;
      cascade_init(q, s);
      if (tab.data != nullptr) {
        // The noise lattice's init (the noise at the cell's first node, the part of the cell before t0): its
        // look-ahead sees the held input.
        LatticeRegs L;
        NullSink none;
        PixelCounters c;
        CascadeCounters cn;
        const RunInput in{t0, v, nullptr, nullptr, 0, 0, k.irr_max};
        LatticeProc<NullSink> proc{s, q, L, m, k, cc, tab, pixel_ids ? pixel_ids[p] : p, none, c, cn, in};
        proc.init(t0, map.phi0[p]);
        store_state(st, p, true, s);
        store_lattice(st, p, n_pixels, L);
      }
      store_cascade(st, p, q);
    }
  }
  warp_add(&counters[kCntClamps], clamps);
  warp_or(&counters[kCntErrors], err);
}

// ---------------------------------------------------------------------------------------------
// CSR runs -> pixel model
// ---------------------------------------------------------------------------------------------
__global__ void scatter_rows_kernel(const uint32_t* pixel, uint32_t n, int32_t* row_of, uint32_t n_pixels,
                                    unsigned long long* counters) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t p = pixel[i];
  if (p >= n_pixels) {
    atomicOr(&counters[kCntErrors], kErrPixelRange);
    return;
  }
  if (atomicExch(&row_of[p], static_cast<int32_t>(i)) != -1) atomicOr(&counters[kCntErrors], kErrDuplicate);
}

struct RunArgs {
  SensorConsts k;
  CascadeConsts cc;
  NoiseTableDev tab;
  MapSoA map;
  StateSoA in, out;
  uint32_t n_pixels;
  const uint32_t* pixel_ids;
  const int32_t* row_of;
  const int64_t* row_start;
  const int32_t* row_count;
  const int64_t* t;
  const float* irr;
  uint64_t n_samples;
  int64_t t_state, t_end;
  EventBuf ev;
  unsigned long long* counters;
};

__global__ void __launch_bounds__(128) advance_runs_kernel(RunArgs a) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  PixelCounters c;
  unsigned long long clamps = 0, samples = 0, err = 0;
  if (p < a.n_pixels) {
    const bool noise = a.k.noise != 0;
    PixelRegs s;
    load_state(a.in, p, noise, s);
    PixelMapRegs m;
    load_map(a.map, p, m);
    GlobalSink sink{a.ev, &a.counters[kCntEvents]};
    PixelProc<GlobalSink> proc{s, m, a.k, a.pixel_ids ? a.pixel_ids[p] : p, sink, c};
    int64_t prev_t = a.t_state;
    float prev_v = s.held;
    const int32_t row = a.row_of != nullptr ? a.row_of[p] : -1;
    int32_t cnt = 0;
    if (row >= 0) {
      const int64_t s0 = a.row_start[row];
      cnt = a.row_count[row];
      if (cnt < 0 || s0 < 0 || static_cast<uint64_t>(s0) + static_cast<uint64_t>(cnt) > a.n_samples) {
        err |= kErrRunRange;
        cnt = 0;
      } else {
        const int64_t* tp = a.t + s0;
        const float* vp = a.irr + s0;
        float x_prev = 0.0f;
        bool have_x = false;
        for (int32_t i = 0; i < cnt; ++i) {
          const int64_t ti = __ldg(tp + i);
          const float raw = __ldg(vp + i);
          if (!isfinite(raw)) err |= kErrNonFinite;
          const float vi = clamp_irr(raw, a.k.irr_max);
          if (!(vi == raw)) ++clamps;
          if (i == 0 ? ti < a.t_state : ti <= prev_t) {
            err |= kErrOrder;
            break;
          }
          if (ti > a.t_end) {
            err |= kErrAfterEnd;
            break;
          }
          if (i == 0 && ti == a.t_state) {  // a sample at the model time replaces the held one (pixel.h:777)
            prev_v = vi;
            continue;
          }
          // A segment inside one 2^23 ns piece takes the fast path with x at both ends (each computed once).
          if (((ti - 1) >> kWindowLog2) == (prev_t >> kWindowLog2)) {
            if (!have_x) x_prev = proc.x_at_sample(prev_v);
            const float x1 = proc.x_at_sample(vi);
            proc.segment_fast(Segment{prev_t, ti, prev_v, vi}, x_prev, x1);
            x_prev = x1;
            have_x = true;
          } else {
            proc.segment(Segment{prev_t, ti, prev_v, vi}, prev_t, ti);
            have_x = false;
          }
          prev_t = ti;
          prev_v = vi;
        }
        samples = static_cast<unsigned long long>(cnt);
      }
    }
    proc.segment(Segment{prev_t, kForever, prev_v, prev_v}, prev_t, a.t_end);
    if (row >= 0 && cnt > 0) s.held = prev_v;
    store_state(a.out, p, noise, s);
  }
  __syncwarp();
  warp_add(&a.counters[kCntClamps], clamps);
  warp_add(&a.counters[kCntPieces], c.pieces);
  warp_add(&a.counters[kCntLeaves], c.leaves);
  warp_add(&a.counters[kCntSamples], samples);
  warp_add(&a.counters[kCntNoise], c.noise_candidates);
  warp_or(&a.counters[kCntErrors], err);
}

// ---------------------------------------------------------------------------------------------
// CSR runs -> the instantaneous pixel model, row-major, long runs walked by the whole warp
// ---------------------------------------------------------------------------------------------
// A warp takes 32 consecutive runs (lane = run; its pixel p = pixel[run]): the run arrays and, for runs listed in
// pixel order, the state and map planes are read as contiguous segments. A run's time is set by its serial chain
// (each segment's comparator state depends on the one before), so the longest run of a window bounds the call; here
// runs longer than long_row samples are walked by all 32 lanes together, one after another:
//  - the lanes load 32 consecutive samples (coalesced) and each computes its sample's x = ln(I / i_scale), the
//    pixel's state broadcast to every lane;
//  - each lane tests its segment (from the previous sample) for the fast path's clean outcome: the pixel not blind,
//    the search armed at or before the segment's start, no noise candidate before its end, Delta at its start below
//    both levels and the rest of it excluded by the exact bound (PixelProc::segment_fast, whose only effects there are
//    the search time and the piece / node counters);
//  - a ballot finds the first segment that is not clean: those before it take their effects at once, it runs through
//    the pixel model on every lane with the same values (the state stays warp-uniform; lane 0 alone appends its
//    events), and the lanes after it are tested again with the new state.
// So a run of n samples with d segments that can fire costs about n / 32 + d steps instead of n. Runs of at most
// long_row samples are walked one per lane, as advance_runs_kernel does. Every lane then advances its own pixel on its
// last sample to t_end.
//
// Listed pixels are marked in a bitmap (one bit per pixel, cleared per call): a pixel listed twice is refused
// (kErrDuplicate) as the reference does; pixels no run lists are advanced to t_end by advance_unlisted_kernel.
constexpr int kRowsWarps = 4;

struct RowsArgs {
  SensorConsts k;
  MapSoA map;
  StateSoA in, out;
  uint32_t n_pixels;
  const uint32_t* pixel;
  uint32_t n_rows;
  const int64_t* row_start;
  const int32_t* row_count;
  const int64_t* t;
  const float* irr;
  uint64_t n_samples;
  int64_t t_state, t_end;
  int32_t long_row;
  uint32_t* listed;
  EventBuf ev;
  unsigned long long* counters;
  const SensorConsts* kd;  // a device copy of k, for the cold calls (a kernel parameter's address is not taken)
};

// Marks the warp's pixels listed; returns kErrDuplicate if some pixel was listed before (in this warp or another).
__device__ __forceinline__ unsigned long long mark_listed(uint32_t* listed, bool valid, uint32_t p) {
  const unsigned full = 0xffffffffu;
  unsigned long long err = 0;
  const uint32_t key = valid ? p : 0xFFFFFFFFu;
  const unsigned same = __match_any_sync(full, key);
  if (valid && __popc(same) > 1) err |= kErrDuplicate;
  const uint32_t word = valid ? (p >> 5) : 0xFFFFFFFFu;
  const unsigned group = __match_any_sync(full, word);
  const uint32_t bit = valid ? (1u << (p & 31u)) : 0u;
  const uint32_t bits = __reduce_or_sync(group, bit);
  if (valid && (threadIdx.x & 31u) == static_cast<uint32_t>(__ffs(group) - 1)) {
    const uint32_t old = atomicOr(listed + word, bits);
    if (old & bits) err |= kErrDuplicate;
  }
  return err;
}

// Inside warp-uniform processing every lane pushes the same event: lane 0 alone appends it.
struct LaneZeroSink {
  GlobalSink inner;
  __device__ __forceinline__ void push(const RawEvent& e) {
    if ((threadIdx.x & 31u) == 0u) inner.push(e);
  }
};

__device__ __forceinline__ PixelRegs shfl_regs(const PixelRegs& s, int src) {
  const unsigned full = 0xffffffffu;
  PixelRegs o;
  o.t_ref = __shfl_sync(full, s.t_ref, src);
  o.t_search = __shfl_sync(full, s.t_search, src);
  o.blind_until = __shfl_sync(full, s.blind_until, src);
  o.s3_ref = __shfl_sync(full, s.s3_ref, src);
  o.n3_ref = __shfl_sync(full, s.n3_ref, src);
  o.dr_ref = __shfl_sync(full, s.dr_ref, src);
  o.i_scale = __shfl_sync(full, s.i_scale, src);
  o.held = __shfl_sync(full, s.held, src);
  o.flags = __shfl_sync(full, s.flags, src);
  o.t_shot = __shfl_sync(full, s.t_shot, src);
  o.t_ba = __shfl_sync(full, s.t_ba, src);
  o.n_shot = __shfl_sync(full, s.n_shot, src);
  o.n_ba = __shfl_sync(full, s.n_ba, src);
  return o;
}

__device__ __forceinline__ PixelMapRegs shfl_map(const PixelMapRegs& m, int src) {
  const unsigned full = 0xffffffffu;
  PixelMapRegs o;
  o.theta_on = __shfl_sync(full, m.theta_on, src);
  o.theta_off = __shfl_sync(full, m.theta_off, src);
  o.leak = __shfl_sync(full, m.leak, src);
  o.dark = __shfl_sync(full, m.dark, src);
  o.scale = __shfl_sync(full, m.scale, src);
  o.ba_rate_hz = __shfl_sync(full, m.ba_rate_hz, src);
  o.shot_max_hz = __shfl_sync(full, m.shot_max_hz, src);
  return o;
}

// Would PixelProc::segment_fast pass segment [t0, e) with nothing but its clean effects (the piece counted, the
// search moved to e, a node counted when e - t0 > 2)? Only where it takes that branch: one 2^23 ns piece, the pixel
// not blind, its search armed at or before t0, no noise candidate before e, Delta(t0) below both levels, and the
// node (t0, e - 1] a single integer or excluded. Inline code on the caller's registers.
__device__ __forceinline__ bool clean_segment(const PixelRegs& s, const PixelMapRegs& m, const SensorConsts& k,
                                              int64_t t0, int64_t e, float v0, float v1, float x0, float x1) {
  if (((e - 1) >> kWindowLog2) != (t0 >> kWindowLog2)) return false;
  if (s.blind_until != kNotBlind || s.t_search > t0) return false;
  const int64_t tn = k.noise ? mini(s.t_shot, s.t_ba) : kForever;
  if (tn < e) return false;
  NullSink ns;
  PixelCounters nc;
  const PixelProc<NullSink> hp{const_cast<PixelRegs&>(s), m, k, 0u, ns, nc};
  const float D0 = hp.delta(t0, x0);
  if (D0 >= m.theta_on || D0 <= -m.theta_off) return false;
  if (e - t0 == 1) return true;
  return hp.excluded(Segment{t0, e, v0, v1}, t0, e, x0, x1);
}

// clean_segment's other case, for a segment it refused: the search armed after t0 (the first segment after init, or
// the segment of an event), where PixelProc::piece searches [t_search, e) alone, without Delta(t0); clean when
// nothing is left to search or the node (t0, e - 1] around it is excluded (the same effects).
__device__ __forceinline__ bool clean_after_start(const PixelRegs& s, const PixelMapRegs& m, const SensorConsts& k,
                                                  int64_t t0, int64_t e, float v0, float v1, float x0, float x1) {
  if (((e - 1) >> kWindowLog2) != (t0 >> kWindowLog2)) return false;
  if (s.blind_until != kNotBlind || s.t_search <= t0) return false;
  const int64_t tn = k.noise ? mini(s.t_shot, s.t_ba) : kForever;
  if (tn < e) return false;
  if (s.t_search >= e) return true;
  NullSink ns;
  PixelCounters nc;
  const PixelProc<NullSink> hp{const_cast<PixelRegs&>(s), m, k, 0u, ns, nc};
  return hp.excluded(Segment{t0, e, v0, v1}, t0, e, x0, x1);
}

// The noise candidates of a stretch [t_from, t_end) of every lane's pixel, computed with all 32 lanes together.
// A candidate that thinning rejects changes nothing but its chain (PixelProc::noise_candidate), and its acceptance
// depends only on its draw and the irradiance at its time, which the stretch's samples give: so each lane's chains
// move past their rejected candidates here, and stop at their first accepted candidate in the stretch (or at their
// first candidate after it). The pixel model then meets only accepted candidates, at which it runs its own noise
// path (the draw and the thinning test again, the refractory drop, the event) and follows the chains from there as
// usual. Events and the chains' end state are those of the pixel model meeting every candidate; only the count of
// the crossing search's nodes differs, since the search is no longer cut at rejected candidates (the first crossing
// is the same: a time-ordered search over [lo, e) finds what searches over [lo, tn) then [tn, e) find).
// active: this lane's stretch is in `run` (run.n samples after the one held at t_from, run.t(j) / run.v_at(j), raw
// values clamped here as the pixel model clamps them). All lanes of the warp call it.
template <class Run>
__device__ __forceinline__ void noise_ahead(PixelRegs& s, const PixelMapRegs& m, const SensorConsts& k,
                                            uint32_t pixel, bool active, int64_t t_from, float v_held,
                                            int64_t t_end, const Run& run, PixelCounters& c) {
  bool done_shot = !active, done_ba = !active;
  for (;;) {
    const bool p_shot = !done_shot && s.t_shot < t_end, p_ba = !done_ba && s.t_ba < t_end;
    if (!__any_sync(0xffffffffu, p_shot || p_ba)) break;
    if (!(p_shot || p_ba)) continue;
    const bool shot = p_shot && (!p_ba || s.t_shot <= s.t_ba);
    const int64_t tn = shot ? s.t_shot : s.t_ba;
    const uint32_t purpose = shot ? kPurposeShot : kPurposeBackground;
    const uint32_t nidx = shot ? s.n_shot : s.n_ba;
    // The segment holding tn: [t_a, t_b) between consecutive samples, or held after the last one.
    int64_t ta = t_from;
    float va = v_held;
    int64_t tb = kForever;
    float vb = va;
    for (int j = 0; j < run.n; ++j) {
      const int64_t tj = run.t(j);
      const float vj = clamp_irr(run.v_at(j), k.irr_max);
      if (tj > tn) {
        tb = tj;
        vb = vj;
        break;
      }
      ta = tj;
      va = vj;
    }
    if (tb == kForever) vb = va;
    const U4 w = draw(k.seed, purpose, k.camera, pixel, nidx);
    NullSink ns;
    PixelCounters nc;
    const PixelProc<NullSink> hp{s, m, k, pixel, ns, nc};
    const float I = hp.current(Segment{ta, tb, va, vb}, tn);
    const double accept = shot ? sqrt(static_cast<double>(m.dark) / static_cast<double>(I)) : 1.0;
    if (open_uniform_d(w.v[1]) < accept) {
      if (shot) done_shot = true;
      else done_ba = true;
      continue;
    }
    ++c.noise_candidates;
    const int64_t next = noise_next(k.seed, purpose, k.camera, pixel, nidx + 1, tn, shot ? m.shot_max_hz : m.ba_rate_hz);
    if (shot) {
      s.n_shot = nidx + 1;
      s.t_shot = next;
    } else {
      s.n_ba = nidx + 1;
      s.t_ba = next;
    }
  }
}

// A lane's window staged in shared memory (dt / v strided by 32 lanes) as noise_ahead's run.
struct StagedRun {
  int64_t t_w;
  const uint32_t* dt;
  const float* v;
  int n;
  __device__ __forceinline__ int64_t t(int j) const { return t_w + dt[j * 32]; }
  __device__ __forceinline__ float v_at(int j) const { return v[j * 32]; }
};
// A CSR run in device memory as noise_ahead's run.
struct GlobalRun {
  const int64_t* tp;
  const float* vp;
  int n;
  __device__ __forceinline__ int64_t t(int j) const { return __ldg(tp + j); }
  __device__ __forceinline__ float v_at(int j) const { return __ldg(vp + j); }
};

// x = ln(I / i_scale) at a sample of value v (PixelProc::x_at_sample on the caller's registers).
__device__ __forceinline__ float x_sample(const PixelRegs& s, const PixelMapRegs& m, float v) {
  return log_f((m.dark + m.scale * v) / s.i_scale);
}

// The pixel model's full path on a state in memory, out of line: the hot loops keep the state in registers and copy
// it here only for a segment that is not clean. fast: PixelProc::segment_fast with x at both ends; else
// PixelProc::segment over [from, to).
// kFlat: the processor's rare paths inline here, on copies the compiler can keep in registers (one large function:
// the CSR kernel and the streaming engine); else they stay separate out-of-line functions working on the state in
// memory (smaller code: the staged engine, whose instruction footprint sets its speed).
template <class Sink, bool kFlat>
__device__ __noinline__ void cold_segment(PixelRegs* s, const PixelMapRegs* m, const SensorConsts* k, uint32_t pixel,
                                          Sink sink, PixelCounters* c, Segment g, int64_t from, int64_t to, bool fast,
                                          float x0, float x1) {
  PixelRegs sl = *s;
  const PixelMapRegs ml = *m;
  PixelCounters cl = *c;
  PixelProc<Sink, kFlat> proc{sl, ml, *k, pixel, sink, cl};
  if (fast) proc.segment_fast(g, x0, x1);
  else proc.segment(g, from, to);
  *s = sl;
  *c = cl;
}

// One segment [t0, t1) of a pixel whose state is in registers: the clean outcome in place, anything else out of line.
template <bool kFlat = true, class Sink>
__device__ __forceinline__ void feed_segment(PixelRegs& s, const PixelMapRegs& m, const SensorConsts& k,
                                             const SensorConsts* kd, uint32_t pixel, const Sink& sink,
                                             PixelCounters& c, int64_t t0, int64_t t1, float v0, float v1, float x0,
                                             float x1) {
  if (clean_segment(s, m, k, t0, t1, v0, v1, x0, x1)) {
    ++c.pieces;
    if (t1 - t0 > 2) ++c.leaves;
    s.t_search = maxi(s.t_search, t1);
    return;
  }
  const Segment g{t0, t1, v0, v1};
  const bool fast = ((t1 - 1) >> kWindowLog2) == (t0 >> kWindowLog2);
  PixelRegs ts = s;
  PixelMapRegs tm = m;
  PixelCounters tc = c;
  cold_segment<Sink, kFlat>(&ts, &tm, kd, pixel, sink, &tc, g, t0, t1, fast, x0, x1);
  s = ts;
  c = tc;
}

// The held sample from t_from to t_end (the end of a call), out of line where there is such a stretch.
template <class Sink>
__device__ __forceinline__ void feed_held(PixelRegs& s, const PixelMapRegs& m, const SensorConsts* kd, uint32_t pixel,
                                          const Sink& sink, PixelCounters& c, int64_t t_from, float v,
                                          int64_t t_end) {
  if (t_from >= t_end) return;
  PixelRegs ts = s;
  PixelMapRegs tm = m;
  PixelCounters tc = c;
  cold_segment<Sink, true>(&ts, &tm, kd, pixel, sink, &tc, Segment{t_from, kForever, v, v}, t_from, t_end, false, 0.0f,
                           0.0f);
  s = ts;
  c = tc;
}

// The warp-cooperative walk of one run (cnt samples at tp / vp) of a pixel whose state u every lane holds alike.
// prev_t / prev_v / x_prev: the last sample fed (at entry the held one at the model time, x_prev its x), updated.
// Stops at the first sample out of order or after t_end (the call is refused then).
__device__ __forceinline__ void coop_run(PixelRegs& u, const PixelMapRegs& um, const RowsArgs& a, uint32_t pixel,
                                         const LaneZeroSink& lz, PixelCounters& cu, const int64_t* tp,
                                         const float* vp, int32_t cnt, uint32_t lane, int64_t& prev_t,
                                         float& prev_v, float& x_prev, unsigned long long& err,
                                         unsigned long long& clamps) {
  const unsigned full = 0xffffffffu;
  for (int32_t b = 0; b < cnt; b += 32) {
    const int32_t i = b + static_cast<int32_t>(lane);
    const bool in = i < cnt;
    const int64_t ti = in ? __ldg(tp + i) : kForever;
    const float raw = in ? __ldg(vp + i) : 0.0f;
    if (in && !isfinite(raw)) err |= kErrNonFinite;
    const float vi = clamp_irr(raw, a.k.irr_max);
    if (in && !(vi == raw)) ++clamps;
    const float xi = in ? x_sample(u, um, vi) : 0.0f;
    int64_t tq = __shfl_up_sync(full, ti, 1);
    float vq = __shfl_up_sync(full, vi, 1), xq = __shfl_up_sync(full, xi, 1);
    if (lane == 0u) {
      tq = prev_t;
      vq = prev_v;
      xq = x_prev;
    }
    const bool bad_order = in && (i == 0 ? ti < a.t_state : ti <= tq);
    const bool after = in && ti > a.t_end;
    if (bad_order) err |= kErrOrder;
    if (after) err |= kErrAfterEnd;
    const unsigned bad = __ballot_sync(full, bad_order || after);
    const int32_t left = cnt - b < 32 ? cnt - b : 32;
    const int32_t limit = bad ? mini(__ffs(bad) - 1, left) : left;
    int32_t j = 0;
    // The run's first sample at the model time replaces the held one (pixel.h:777): no segment.
    if (b == 0 && limit > 0 && __shfl_sync(full, ti, 0) == a.t_state) j = 1;
    const unsigned upto = limit == 32 ? full : ((1u << limit) - 1u);
    while (j < limit) {
      const bool mine = static_cast<int32_t>(lane) >= j && static_cast<int32_t>(lane) < limit;
      const bool clean = !mine || clean_segment(u, um, a.k, tq, ti, vq, vi, xq, xi);
      const unsigned range = upto & ~((1u << j) - 1u);
      const unsigned dirty = __ballot_sync(full, !clean) & range;
      const int32_t f = dirty ? __ffs(dirty) - 1 : limit;
      if (f > j) {  // segments j .. f - 1 are clean: their effects at once
        const unsigned cm = range & (f == 32 ? full : ((1u << f) - 1u));
        cu.pieces += static_cast<uint32_t>(__popc(cm));
        cu.leaves += static_cast<uint32_t>(__popc(__ballot_sync(full, ti - tq > 2) & cm));
        u.t_search = maxi(u.t_search, __shfl_sync(full, ti, f - 1));
      }
      if (f < limit) {  // segment f through the pixel model, the same on every lane
        const int64_t t0 = __shfl_sync(full, tq, f), e = __shfl_sync(full, ti, f);
        const float v0 = __shfl_sync(full, vq, f), v1 = __shfl_sync(full, vi, f);
        const float x0 = __shfl_sync(full, xq, f), x1 = __shfl_sync(full, xi, f);
        PixelRegs ts = u;
        PixelMapRegs tm = um;
        PixelCounters tc = cu;
        const bool fast = ((e - 1) >> kWindowLog2) == (t0 >> kWindowLog2);
        cold_segment<LaneZeroSink, true>(&ts, &tm, a.kd, pixel, lz, &tc, Segment{t0, e, v0, v1}, t0, e, fast, x0, x1);
        u = ts;
        cu = tc;
      }
      j = f + 1;
    }
    if (limit > 0) {
      prev_t = __shfl_sync(full, ti, limit - 1);
      prev_v = __shfl_sync(full, vi, limit - 1);
      x_prev = __shfl_sync(full, xi, limit - 1);
    }
    if (bad) break;
  }
}

__global__ void __launch_bounds__(32 * kRowsWarps) advance_rows_kernel(RowsArgs a) {
  const unsigned full = 0xffffffffu;
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t row = (blockIdx.x * kRowsWarps + warp) * 32u + lane;
  const bool in_rows = row < a.n_rows;
  const uint32_t p = in_rows ? __ldg(a.pixel + row) : 0u;
  unsigned long long err = 0, clamps = 0, samples = 0;
  const bool valid = in_rows && p < a.n_pixels;
  if (in_rows && !valid) err |= kErrPixelRange;
  err |= mark_listed(a.listed, valid, p);
  int64_t beg = 0;
  int32_t cnt = 0;
  if (valid) {
    beg = __ldg(a.row_start + row);
    cnt = __ldg(a.row_count + row);
    if (cnt < 0 || beg < 0 || static_cast<uint64_t>(beg) + static_cast<uint64_t>(cnt) > a.n_samples) {
      err |= kErrRunRange;
      cnt = 0;
      beg = 0;
    }
  }
  const bool noise = a.k.noise != 0;
  PixelRegs s{};
  PixelMapRegs m{};
  if (valid) {
    load_state(a.in, p, noise, s);
    load_map(a.map, p, m);
  }
  PixelCounters c;
  const GlobalSink sink{a.ev, &a.counters[kCntEvents]};
  int64_t prev_t = a.t_state;
  float prev_v = s.held;
  const bool longrun = cnt > a.long_row;

  // The short runs' noise candidates, all lanes together (a long run meets its candidates in the pixel model).
  if (noise) {
    const GlobalRun run{a.t + beg, a.irr + beg, cnt};
    noise_ahead(s, m, a.k, p, valid && !longrun, a.t_state, s.held, a.t_end, run, c);
  }
  // Short runs: one lane each.
  if (cnt > 0 && !longrun) {
    const int64_t* tp = a.t + beg;
    const float* vp = a.irr + beg;
    float x_prev = 0.0f;
    bool have_x = false;
    for (int32_t i = 0; i < cnt; ++i) {
      const int64_t ti = __ldg(tp + i);
      const float raw = __ldg(vp + i);
      if (!isfinite(raw)) err |= kErrNonFinite;
      const float vi = clamp_irr(raw, a.k.irr_max);
      if (!(vi == raw)) ++clamps;
      if (i == 0 ? ti < a.t_state : ti <= prev_t) {
        err |= kErrOrder;
        break;
      }
      if (ti > a.t_end) {
        err |= kErrAfterEnd;
        break;
      }
      if (i == 0 && ti == a.t_state) {  // a sample at the model time replaces the held one (pixel.h:777)
        prev_v = vi;
        continue;
      }
      if (!have_x) x_prev = x_sample(s, m, prev_v);
      const float x1 = x_sample(s, m, vi);
      feed_segment(s, m, a.k, a.kd, p, sink, c, prev_t, ti, prev_v, vi, x_prev, x1);
      x_prev = x1;
      have_x = true;
      prev_t = ti;
      prev_v = vi;
    }
  }

  // Long runs: the whole warp on each, one after another.
  for (unsigned pend = __ballot_sync(full, longrun); pend != 0u; pend &= pend - 1u) {
    const int r = __ffs(pend) - 1;
    PixelRegs u = shfl_regs(s, r);
    const PixelMapRegs um = shfl_map(m, r);
    const uint32_t pr = __shfl_sync(full, p, r);
    const int64_t br = __shfl_sync(full, beg, r);
    const int32_t nr = __shfl_sync(full, cnt, r);
    PixelCounters cu;
    const LaneZeroSink lz{sink};
    int64_t pt = a.t_state;
    float pv = u.held, px = x_sample(u, um, u.held);
    coop_run(u, um, a, pr, lz, cu, a.t + br, a.irr + br, nr, lane, pt, pv, px, err, clamps);
    if (static_cast<int>(lane) == r) {
      s = u;
      c.pieces += cu.pieces;
      c.leaves += cu.leaves;
      c.noise_candidates += cu.noise_candidates;
      prev_t = pt;
      prev_v = pv;
    }
  }

  if (valid) {
    samples = static_cast<unsigned long long>(cnt);
    feed_held(s, m, a.kd, p, sink, c, prev_t, prev_v, a.t_end);
    if (cnt > 0) s.held = prev_v;
    store_state(a.out, p, noise, s);
  }
  __syncwarp();
  warp_add(&a.counters[kCntClamps], clamps);
  warp_add(&a.counters[kCntPieces], c.pieces);
  warp_add(&a.counters[kCntLeaves], c.leaves);
  warp_add(&a.counters[kCntSamples], samples);
  warp_add(&a.counters[kCntNoise], c.noise_candidates);
  warp_or(&a.counters[kCntErrors], err);
}

// The row-major kernel split like the split engine: advance_rows_split_kernel runs what advance_rows_kernel runs
// except the pixel model's paths for a short run's segment that is not clean (and the held stretch after its last
// sample): there the lane stops and posts its row (the state, the feed, the next sample's index), and
// advance_rows_rest_kernel finishes the posted rows one thread each, reading their samples in place with the same
// checks. A row's samples meet the same state in the same order, so the events and the refusals are the same.
struct RowRest {
  PixelRegs s;
  int64_t prev_t;
  float prev_v, x_prev;
  uint32_t row;
  int32_t next;     // the first sample not yet fed (cnt: only the held stretch to t_end is left)
  uint32_t have_x;  // x_prev holds x at prev_v
};

struct RowRestList {
  RowRest* rec;
  unsigned int* count;
  unsigned int capacity;
};

// kFirst: the model's first call after init, where every pixel's search is armed after its first segment's start:
// such a segment is also taken in place when clean (clean_after_start) rather than posted; the other calls' kernel
// leaves that test out of its loop.
template <bool kFirst>
// At most 64 registers (8 blocks of 4 warps per SM): the kernel waits on its rows' loads, and the extra warps hide
// more than the spills cost (pixel-model kernels 97.0 ms per six-sensor runs step at 128 registers, 82.0 at 80,
// 78.1 at 64).
__global__ void __launch_bounds__(32 * kRowsWarps, 8) advance_rows_split_kernel(RowsArgs a, RowRestList rl) {
  const unsigned full = 0xffffffffu;
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t row = (blockIdx.x * kRowsWarps + warp) * 32u + lane;
  const bool in_rows = row < a.n_rows;
  const uint32_t p = in_rows ? __ldg(a.pixel + row) : 0u;
  unsigned long long err = 0, clamps = 0, samples = 0;
  const bool valid = in_rows && p < a.n_pixels;
  if (in_rows && !valid) err |= kErrPixelRange;
  err |= mark_listed(a.listed, valid, p);
  int64_t beg = 0;
  int32_t cnt = 0;
  if (valid) {
    beg = __ldg(a.row_start + row);
    cnt = __ldg(a.row_count + row);
    if (cnt < 0 || beg < 0 || static_cast<uint64_t>(beg) + static_cast<uint64_t>(cnt) > a.n_samples) {
      err |= kErrRunRange;
      cnt = 0;
      beg = 0;
    }
  }
  const bool noise = a.k.noise != 0;
  PixelRegs s{};
  PixelMapRegs m{};
  if (valid) {
    load_state(a.in, p, noise, s);
    load_map(a.map, p, m);
  }
  PixelCounters c;
  const GlobalSink sink{a.ev, &a.counters[kCntEvents]};
  int64_t prev_t = a.t_state;
  float prev_v = s.held;
  const bool longrun = cnt > a.long_row;

  // The short runs' noise candidates, all lanes together (a long run meets its candidates in the pixel model).
  if (noise) {
    const GlobalRun run{a.t + beg, a.irr + beg, cnt};
    noise_ahead(s, m, a.k, p, valid && !longrun, a.t_state, s.held, a.t_end, run, c);
  }
  // Short runs: one lane each, the clean segments in place; the first other one stops the lane there.
  bool post = false;
  int32_t next = 0;
  float x_prev = 0.0f;
  bool have_x = false;
  if (cnt > 0 && !longrun) {
    const int64_t* tp = a.t + beg;
    const float* vp = a.irr + beg;
    int64_t t_next = __ldg(tp);  // each sample loaded one iteration ahead of its use
    float v_next = __ldg(vp);
    for (int32_t i = 0; i < cnt; ++i) {
      const int64_t ti = t_next;
      const float raw = v_next;
      if (i + 1 < cnt) {
        t_next = __ldg(tp + i + 1);
        v_next = __ldg(vp + i + 1);
      }
      if (!isfinite(raw)) err |= kErrNonFinite;
      const float vi = clamp_irr(raw, a.k.irr_max);
      if (!(vi == raw)) ++clamps;
      if (i == 0 ? ti < a.t_state : ti <= prev_t) {
        err |= kErrOrder;
        break;
      }
      if (ti > a.t_end) {
        err |= kErrAfterEnd;
        break;
      }
      if (i == 0 && ti == a.t_state) {  // a sample at the model time replaces the held one (pixel.h:777)
        prev_v = vi;
        continue;
      }
      if (!have_x) x_prev = x_sample(s, m, prev_v);
      const float x1 = x_sample(s, m, vi);
      have_x = true;
      if (!clean_segment(s, m, a.k, prev_t, ti, prev_v, vi, x_prev, x1) &&
          !(kFirst && clean_after_start(s, m, a.k, prev_t, ti, prev_v, vi, x_prev, x1))) {
        if (!(vi == raw)) --clamps;  // the rest kernel counts this sample's clamp (and checks it) again
        post = true;
        next = i;
        break;
      }
      ++c.pieces;
      if (ti - prev_t > 2) ++c.leaves;
      s.t_search = maxi(s.t_search, ti);
      x_prev = x1;
      prev_t = ti;
      prev_v = vi;
    }
  }

  // Long runs: the whole warp on each, one after another.
  for (unsigned pend = __ballot_sync(full, longrun); pend != 0u; pend &= pend - 1u) {
    const int r = __ffs(pend) - 1;
    PixelRegs u = shfl_regs(s, r);
    const PixelMapRegs um = shfl_map(m, r);
    const uint32_t pr = __shfl_sync(full, p, r);
    const int64_t br = __shfl_sync(full, beg, r);
    const int32_t nr = __shfl_sync(full, cnt, r);
    PixelCounters cu;
    const LaneZeroSink lz{sink};
    int64_t pt = a.t_state;
    float pv = u.held, px = x_sample(u, um, u.held);
    coop_run(u, um, a, pr, lz, cu, a.t + br, a.irr + br, nr, lane, pt, pv, px, err, clamps);
    if (static_cast<int>(lane) == r) {
      s = u;
      c.pieces += cu.pieces;
      c.leaves += cu.leaves;
      c.noise_candidates += cu.noise_candidates;
      prev_t = pt;
      prev_v = pv;
    }
  }

  if (valid) {
    samples = static_cast<unsigned long long>(cnt);
    if (!post && prev_t < a.t_end) {  // the held stretch to t_end goes to the rest kernel
      post = true;
      next = cnt;
    }
    if (!post) {
      if (cnt > 0) s.held = prev_v;
      store_state(a.out, p, noise, s);
    }
  }
  // One record per stopped row, the warp's records reserved together.
  __syncwarp();
  const unsigned posting = __ballot_sync(full, post);
  if (posting != 0u) {
    const int leader = __ffs(posting) - 1;
    unsigned int base = 0;
    if (static_cast<int>(lane) == leader) base = atomicAdd(rl.count, static_cast<unsigned int>(__popc(posting)));
    base = __shfl_sync(full, base, leader);
    if (post) {
      const unsigned int i = base + static_cast<unsigned int>(__popc(posting & ((1u << lane) - 1u)));
      if (i >= rl.capacity) {
        err |= kErrRestList;
      } else {
        RowRest& r = rl.rec[i];
        r.s = s;
        r.prev_t = prev_t;
        r.prev_v = prev_v;
        r.x_prev = x_prev;
        r.row = row;
        r.next = next;
        r.have_x = have_x ? 1u : 0u;
      }
    }
  }
  __syncwarp();
  warp_add(&a.counters[kCntClamps], clamps);
  warp_add(&a.counters[kCntPieces], c.pieces);
  warp_add(&a.counters[kCntLeaves], c.leaves);
  warp_add(&a.counters[kCntSamples], samples);
  warp_add(&a.counters[kCntNoise], c.noise_candidates);
  warp_or(&a.counters[kCntErrors], err);
}

// The posted rows, one thread each: the rest of the row through the full pixel model with advance_rows_kernel's
// checks, the held stretch to t_end, the state stored.
__global__ void __launch_bounds__(128) advance_rows_rest_kernel(RowsArgs a, RowRestList rl) {
  const unsigned int count = min(*rl.count, rl.capacity);
  const bool noise = a.k.noise != 0;
  for (unsigned int q = blockIdx.x * blockDim.x + threadIdx.x; q < count; q += gridDim.x * blockDim.x) {
    const RowRest& r = rl.rec[q];
    const uint32_t p = __ldg(a.pixel + r.row);
    const int64_t beg = __ldg(a.row_start + r.row);
    const int32_t cnt = __ldg(a.row_count + r.row);
    PixelRegs s = r.s;
    PixelMapRegs m;
    load_map(a.map, p, m);
    PixelCounters c;
    const ThreadSink sink{a.ev, &a.counters[kCntEvents]};
    unsigned long long err = 0, clamps = 0;
    int64_t prev_t = r.prev_t;
    float prev_v = r.prev_v, x_prev = r.x_prev;
    bool have_x = r.have_x != 0u;
    const int64_t* tp = a.t + beg;
    const float* vp = a.irr + beg;
    for (int32_t i = r.next; i < cnt; ++i) {
      const int64_t ti = __ldg(tp + i);
      const float raw = __ldg(vp + i);
      if (!isfinite(raw)) err |= kErrNonFinite;
      const float vi = clamp_irr(raw, a.k.irr_max);
      if (!(vi == raw)) ++clamps;
      if (i == 0 ? ti < a.t_state : ti <= prev_t) {
        err |= kErrOrder;
        break;
      }
      if (ti > a.t_end) {
        err |= kErrAfterEnd;
        break;
      }
      if (i == 0 && ti == a.t_state) {
        prev_v = vi;
        continue;
      }
      if (!have_x) x_prev = x_sample(s, m, prev_v);
      const float x1 = x_sample(s, m, vi);
      feed_segment(s, m, a.k, a.kd, p, sink, c, prev_t, ti, prev_v, vi, x_prev, x1);
      x_prev = x1;
      have_x = true;
      prev_t = ti;
      prev_v = vi;
    }
    feed_held(s, m, a.kd, p, sink, c, prev_t, prev_v, a.t_end);
    if (cnt > 0) s.held = prev_v;
    store_state(a.out, p, noise, s);
    if (clamps) atomicAdd(&a.counters[kCntClamps], clamps);
    if (c.pieces) atomicAdd(&a.counters[kCntPieces], static_cast<unsigned long long>(c.pieces));
    if (c.leaves) atomicAdd(&a.counters[kCntLeaves], static_cast<unsigned long long>(c.leaves));
    if (c.noise_candidates) atomicAdd(&a.counters[kCntNoise], static_cast<unsigned long long>(c.noise_candidates));
    if (err) atomicOr(&a.counters[kCntErrors], err);
  }
}

// The pixels no run lists: each advances on its held sample to t_end.
__global__ void __launch_bounds__(128) advance_unlisted_kernel(RowsArgs a) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  PixelCounters c;
  if (p < a.n_pixels && !((__ldg(a.listed + (p >> 5)) >> (p & 31u)) & 1u)) {
    const bool noise = a.k.noise != 0;
    PixelRegs s;
    load_state(a.in, p, noise, s);
    PixelMapRegs m;
    load_map(a.map, p, m);
    const GlobalSink sink{a.ev, &a.counters[kCntEvents]};
    feed_held(s, m, a.kd, p, sink, c, a.t_state, s.held, a.t_end);
    store_state(a.out, p, noise, s);
  }
  __syncwarp();
  warp_add(&a.counters[kCntPieces], c.pieces);
  warp_add(&a.counters[kCntLeaves], c.leaves);
  warp_add(&a.counters[kCntNoise], c.noise_candidates);
}

// The cascade with its noise lattice on CSR runs: the row is checked first (the same errors as advance_runs_kernel),
// then the processor reads it with random access (the lattice's look-ahead).
__global__ void __launch_bounds__(128) advance_runs_lattice_kernel(RunArgs a) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  PixelCounters c;
  CascadeCounters cn;
  unsigned long long clamps = 0, samples = 0, err = 0;
  if (p < a.n_pixels) {
    PixelRegs s;
    load_state(a.in, p, false, s);
    CascadeRegs q;
    load_cascade(a.in, p, q);
    LatticeRegs L;
    load_lattice(a.in, p, a.n_pixels, L);
    PixelMapRegs m;
    load_map(a.map, p, m);
    const int32_t row = a.row_of != nullptr ? a.row_of[p] : -1;
    int32_t cnt = 0;
    const int64_t* tp = nullptr;
    const float* vp = nullptr;
    if (row >= 0) {
      const int64_t s0 = a.row_start[row];
      cnt = a.row_count[row];
      if (cnt < 0 || s0 < 0 || static_cast<uint64_t>(s0) + static_cast<uint64_t>(cnt) > a.n_samples) {
        err |= kErrRunRange;
        cnt = 0;
      } else {
        tp = a.t + s0;
        vp = a.irr + s0;
        int64_t prev_t = a.t_state;
        for (int32_t i = 0; i < cnt; ++i) {
          const int64_t ti = __ldg(tp + i);
          const float raw = __ldg(vp + i);
          if (!isfinite(raw)) err |= kErrNonFinite;
          if (!(clamp_irr(raw, a.k.irr_max) == raw)) ++clamps;
          if (i == 0 ? ti < a.t_state : ti <= prev_t) err |= kErrOrder;
          if (ti > a.t_end) err |= kErrAfterEnd;
          prev_t = ti;
        }
        samples = static_cast<unsigned long long>(cnt);
      }
    }
    if (err == 0) {
      GlobalSink sink{a.ev, &a.counters[kCntEvents]};
      const int32_t skip = cnt > 0 && tp[0] == a.t_state ? 1 : 0;
      const RunInput in{a.t_state, s.held, tp, vp, cnt, skip, a.k.irr_max};
      LatticeProc<GlobalSink> proc{s, q, L, m, a.k, a.cc, a.tab, a.pixel_ids ? a.pixel_ids[p] : p, sink, c, cn, in};
      proc.resume();
      proc.advance(a.t_end);
    }
    store_state(a.out, p, false, s);
    store_cascade(a.out, p, q);
    store_lattice(a.out, p, a.n_pixels, L);
  }
  __syncwarp();
  warp_add(&a.counters[kCntClamps], clamps);
  warp_add(&a.counters[kCntPieces], c.pieces);
  warp_add(&a.counters[kCntLeaves], c.leaves);
  warp_add(&a.counters[kCntSamples], samples);
  warp_add(&a.counters[kCntSubsteps], cn.substeps);
  warp_or(&a.counters[kCntErrors], err);
}

// The cascade on CSR runs: the same run checks as advance_runs_kernel, every segment through CascadeProc.
__global__ void __launch_bounds__(128) advance_runs_cascade_kernel(RunArgs a) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  PixelCounters c;
  CascadeCounters cn;
  unsigned long long clamps = 0, samples = 0, err = 0;
  if (p < a.n_pixels) {
    PixelRegs s;
    load_state(a.in, p, false, s);
    CascadeRegs q;
    load_cascade(a.in, p, q);
    PixelMapRegs m;
    load_map(a.map, p, m);
    GlobalSink sink{a.ev, &a.counters[kCntEvents]};
    CascadeProc<GlobalSink> proc{s, q, m, a.k, a.cc, a.pixel_ids ? a.pixel_ids[p] : p, sink, c, cn};
    int64_t prev_t = a.t_state;
    float prev_v = s.held;
    const int32_t row = a.row_of != nullptr ? a.row_of[p] : -1;
    int32_t cnt = 0;
    if (row >= 0) {
      const int64_t s0 = a.row_start[row];
      cnt = a.row_count[row];
      if (cnt < 0 || s0 < 0 || static_cast<uint64_t>(s0) + static_cast<uint64_t>(cnt) > a.n_samples) {
        err |= kErrRunRange;
        cnt = 0;
      } else {
        const int64_t* tp = a.t + s0;
        const float* vp = a.irr + s0;
        for (int32_t i = 0; i < cnt; ++i) {
          const int64_t ti = __ldg(tp + i);
          const float raw = __ldg(vp + i);
          if (!isfinite(raw)) err |= kErrNonFinite;
          const float vi = clamp_irr(raw, a.k.irr_max);
          if (!(vi == raw)) ++clamps;
          if (i == 0 ? ti < a.t_state : ti <= prev_t) {
            err |= kErrOrder;
            break;
          }
          if (ti > a.t_end) {
            err |= kErrAfterEnd;
            break;
          }
          if (i == 0 && ti == a.t_state) {  // a sample at the model time replaces the held one (pixel.h:777)
            prev_v = vi;
            continue;
          }
          proc.segment(Segment{prev_t, ti, prev_v, vi}, prev_t, ti);
          prev_t = ti;
          prev_v = vi;
        }
        samples = static_cast<unsigned long long>(cnt);
      }
    }
    proc.segment(Segment{prev_t, kForever, prev_v, prev_v}, prev_t, a.t_end);
    if (row >= 0 && cnt > 0) s.held = prev_v;
    store_state(a.out, p, false, s);
    store_cascade(a.out, p, q);
  }
  __syncwarp();
  warp_add(&a.counters[kCntClamps], clamps);
  warp_add(&a.counters[kCntPieces], c.pieces);
  warp_add(&a.counters[kCntLeaves], c.leaves);
  warp_add(&a.counters[kCntSamples], samples);
  warp_add(&a.counters[kCntSubsteps], cn.substeps);
  warp_or(&a.counters[kCntErrors], err);
}

// ---------------------------------------------------------------------------------------------
// sample_window
// ---------------------------------------------------------------------------------------------
struct WindowArgs {
  FieldDev f;
  SamplerRules r;
  int64_t t_w;
  const uint32_t* pixel;
  const uint8_t* level;
  uint32_t n;
  const float* carried_in;
  const uint64_t* sig_in;
  uint32_t* counts;
  const int64_t* offsets;
  int64_t* t_out;
  float* irr_out;
  float* carried_out;
  uint64_t* sig_out;
};

template <int kPass>
__global__ void __launch_bounds__(128) sample_window_kernel(WindowArgs a) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool have = i < a.n;
  const uint32_t px = have ? a.pixel[i] : 0u;
  const uint32_t x = a.f.width > 0 ? px % a.f.width : 0u, y = a.f.width > 0 ? px / a.f.width : 0u;
  __shared__ uint16_t lists[4][kMaxListed];
  const BlobList list = warp_blob_list(a.f, have, x, y, a.t_w, a.t_w + kWindowNs, lists[threadIdx.x >> 5]);
  if (!have) return;
  const float carried = a.carried_in[i];
  const bool flip = a.sig_in[i] != 0ull;
  const FieldDev& f = a.f;
  const int64_t t_w = a.t_w;
  auto render = [&](uint32_t dt) { return field_eval(f, list, x, y, t_w + dt); };
  if (kPass == 0) {
    const uint32_t n = sample_pixel_window(a.r, a.level[i], carried, flip, render, [](uint32_t, float) {});
    a.counts[i] = n;
  } else {
    int64_t* t_out = a.t_out + a.offsets[i];
    float* irr_out = a.irr_out + a.offsets[i];
    t_out[0] = t_w;  // slot 0: the carried sample
    irr_out[0] = carried;
    uint32_t k = 1;
    float last = carried;
    sample_pixel_window(a.r, a.level[i], carried, flip, render, [&](uint32_t dt, float v) {
      t_out[k] = t_w + dt;
      irr_out[k] = v;
      ++k;
      last = v;
    });
    a.carried_out[i] = last;
    a.sig_out[i] = 0ull;
  }
}

// sample_window in one walk (the device-runs path): sample_window_stage_kernel checks each pixel's id and level (a
// bad one is flagged in *err, 1: level, 2: id, and not walked), walks every pixel once, stages its samples after slot
// 0 in shared memory (up to kSampStage), writes its count and keeps its carried sample and signature in scratch, and
// copies the staged samples to a scratch list (each warp's reserved with one atomic; stage_at[i] their start, or
// kStageNone). After the scan of the counts (and only when nothing was flagged), sample_window_place_kernel writes
// each row at its offset from the list, or walks a pixel whose window overflowed the stage (or the list) again, and
// the carried samples and signatures. The runs equal the two-pass form's. 16 staged samples a lane (18 KB of shared
// memory a block) leave the registers to bound the blocks per SM; 32 (35 KB) held them to 6 and measured slower.
constexpr int kSampStage = 16;
constexpr uint32_t kStageNone = 0xFFFFFFFFu;

struct StageArgs {
  WindowArgs w;
  uint32_t* stage_dt;
  float* stage_v;
  uint32_t* stage_at;
  unsigned int* stage_used;
  uint32_t stage_cap;
  float* stage_carried;  // each pixel's carried sample and signature, written out by the place kernel
  uint64_t* stage_sig;
  uint32_t n_field;
  int max_level;
  unsigned long long* err;
};

// At most 64 registers, so that 8 blocks fit an SM (68 held it to 7: 142.8 against 134.2 ms per six-sensor runs step).
__global__ void __launch_bounds__(128, 8) sample_window_stage_kernel(StageArgs sa) {
  const WindowArgs& a = sa.w;
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool have = i < a.n;
  const uint32_t px = have ? a.pixel[i] : 0u;
  const uint32_t x = a.f.width > 0 ? px % a.f.width : 0u, y = a.f.width > 0 ? px / a.f.width : 0u;
  __shared__ uint16_t lists[4][kMaxListed];
  __shared__ uint32_t st_dt[4][kSampStage][32];
  __shared__ float st_v[4][kSampStage][32];
  unsigned long long bad = 0;
  if (have && px >= sa.n_field) bad |= 2ull;
  if (have && a.level[i] > sa.max_level) bad |= 1ull;
  const BlobList list = warp_blob_list(a.f, have && bad == 0ull, x, y, a.t_w, a.t_w + kWindowNs, lists[warp]);
  warp_or(sa.err, bad);
  uint32_t n = 0;
  if (have && bad != 0ull) {
    n = 1;
    a.counts[i] = n;
  } else if (have) {
    const float carried = a.carried_in[i];
    const bool flip = a.sig_in[i] != 0ull;
    const FieldDev& f = a.f;
    const int64_t t_w = a.t_w;
    auto render = [&](uint32_t dt) { return field_eval(f, list, x, y, t_w + dt); };
    uint32_t k = 0;
    float last = carried;
    n = sample_pixel_window(a.r, a.level[i], carried, flip, render, [&](uint32_t dt, float v) {
      if (k < static_cast<uint32_t>(kSampStage)) {
        st_dt[warp][k][lane] = dt;
        st_v[warp][k][lane] = v;
      }
      ++k;
      last = v;
    });
    a.counts[i] = n;
    sa.stage_carried[i] = last;
    sa.stage_sig[i] = 0ull;
  }
  __syncwarp();
  const uint32_t m = have && n >= 1u && n - 1u <= static_cast<uint32_t>(kSampStage) ? n - 1u : 0u;
  const bool staged = have && n >= 1u && n - 1u <= static_cast<uint32_t>(kSampStage);
  // The warp's staged samples reserved together: lane l's start is the base plus the lanes before it.
  uint32_t before = m;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y2 = __shfl_up_sync(0xffffffffu, before, o);
    if (static_cast<int>(lane) >= o) before += y2;
  }
  const uint32_t total = __shfl_sync(0xffffffffu, before, 31);
  before -= m;
  unsigned int base = 0;
  if (lane == 0u && total > 0u) base = atomicAdd(sa.stage_used, total);
  base = __shfl_sync(0xffffffffu, base, 0);
  if (have) {
    const bool fits = staged && static_cast<uint64_t>(base) + total <= sa.stage_cap;
    if (fits) {
      const uint32_t at = base + before;
      for (uint32_t q = 0; q < m; ++q) {
        sa.stage_dt[at + q] = st_dt[warp][q][lane];
        sa.stage_v[at + q] = st_v[warp][q][lane];
      }
      sa.stage_at[i] = at;
    } else {
      sa.stage_at[i] = kStageNone;
    }
  }
}

__global__ void __launch_bounds__(128) sample_window_place_kernel(StageArgs sa) {
  const WindowArgs& a = sa.w;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool have = i < a.n;
  const uint32_t at = have ? sa.stage_at[i] : 0u;
  const bool walk = have && at == kStageNone;
  const uint32_t px = have ? a.pixel[i] : 0u;
  const uint32_t x = a.f.width > 0 ? px % a.f.width : 0u, y = a.f.width > 0 ? px / a.f.width : 0u;
  __shared__ uint16_t lists[4][kMaxListed];
  BlobList list{nullptr, a.f.n_blobs};
  if (__any_sync(0xffffffffu, walk)) {
    list = warp_blob_list(a.f, have, x, y, a.t_w, a.t_w + kWindowNs, lists[threadIdx.x >> 5]);
  }
  if (!have) return;
  const int64_t t_w = a.t_w;
  const float carried = a.carried_in[i];
  a.carried_out[i] = sa.stage_carried[i];
  a.sig_out[i] = sa.stage_sig[i];
  int64_t* t_out = a.t_out + a.offsets[i];
  float* irr_out = a.irr_out + a.offsets[i];
  t_out[0] = t_w;  // slot 0: the carried sample
  irr_out[0] = carried;
  if (!walk) {
    const uint32_t m = a.counts[i] - 1u;
    for (uint32_t q = 0; q < m; ++q) {
      t_out[1 + q] = t_w + sa.stage_dt[at + q];
      irr_out[1 + q] = sa.stage_v[at + q];
    }
    return;
  }
  const FieldDev& f = a.f;
  auto render = [&](uint32_t dt) { return field_eval(f, list, x, y, t_w + dt); };
  uint32_t k = 1;
  sample_pixel_window(a.r, a.level[i], carried, a.sig_in[i] != 0ull, render, [&](uint32_t dt, float v) {
    t_out[k] = t_w + dt;
    irr_out[k] = v;
    ++k;
  });
}

__global__ void levels_kernel(FieldDev f, int64_t t_w, int32_t l_min, int32_t l_max, uint32_t n_pixels,
                              uint8_t* level) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  const bool have = p < n_pixels;
  const uint32_t x = have ? p % f.width : 0u, y = have ? p / f.width : 0u;
  __shared__ uint16_t lists[4][kMaxListed];
  const BlobList list = warp_blob_list(f, have, x, y, t_w, t_w, lists[threadIdx.x >> 5]);
  if (have) level[p] = static_cast<uint8_t>(field_level(f, list, x, y, t_w, l_min, l_max));
}

__global__ void field_frame_kernel(FieldDev f, int64_t t, uint32_t n_pixels, float* out) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n_pixels) out[p] = field_eval_all(f, p % f.width, p / f.width, t);
}

// ---------------------------------------------------------------------------------------------
// Exclusive scan (counts u32 -> offsets i64): per-block scan, a scan of the block sums, then the fix-up.
// ---------------------------------------------------------------------------------------------
constexpr int kScanBlock = 1024;

__device__ __forceinline__ int64_t block_exclusive_scan(int64_t v, int64_t* total) {
  __shared__ int64_t warp_sums[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int64_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    int64_t w = lane < nw ? warp_sums[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < nw) warp_sums[lane] = w;
  }
  __syncthreads();
  const int64_t before = warp == 0 ? 0 : warp_sums[warp - 1];
  *total = warp_sums[(blockDim.x >> 5) - 1];
  __syncthreads();
  return before + x - v;
}

__global__ void __launch_bounds__(kScanBlock) scan_blocks_kernel(const uint32_t* counts, uint32_t n, int64_t* out,
                                                                 int64_t* block_sums) {
  const uint32_t i = blockIdx.x * kScanBlock + threadIdx.x;
  const int64_t v = i < n ? counts[i] : 0;
  int64_t total;
  const int64_t ex = block_exclusive_scan(v, &total);
  if (i < n) out[i] = ex;
  if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanBlock) scan_sums_kernel(int64_t* block_sums, uint32_t n_blocks,
                                                               int64_t* out, uint32_t n) {
  __shared__ int64_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (uint32_t b = 0; b < n_blocks; b += kScanBlock) {
    const uint32_t i = b + threadIdx.x;
    const int64_t v = i < n_blocks ? block_sums[i] : 0;
    int64_t total;
    const int64_t ex = block_exclusive_scan(v, &total);
    if (i < n_blocks) block_sums[i] = ex + carry;
    __syncthreads();
    if (threadIdx.x == 0) carry += total;
    __syncthreads();
  }
  if (threadIdx.x == 0) out[n] = carry;
}

__global__ void scan_fix_kernel(int64_t* out, uint32_t n, const int64_t* block_sums) {
  const uint32_t i = blockIdx.x * kScanBlock + threadIdx.x;
  if (i < n) out[i] += block_sums[blockIdx.x];
}

// ---------------------------------------------------------------------------------------------
// The fused engine
// ---------------------------------------------------------------------------------------------
struct EngineArgs {
  const EngineSensor* sensors;
  int n_sensors;
  uint32_t total_tiles;
  const int64_t* t0;  // the model time, in device memory (a captured launch replays at any time)
  int32_t w0, w1;
  SamplerRules r;
  unsigned int* tile_counter;
  uint32_t tile_lw;   // log2 of the tile width: tiles of 2^lw x 2^(5 - lw) pixels, one warp each
};

// The pixel of `lane` in tile `local` of a sensor with tiles_x tiles per row.
__device__ __forceinline__ void tile_xy(uint32_t local, uint32_t tiles_x, uint32_t lw, uint32_t lane, uint32_t& x,
                                        uint32_t& y) {
  x = (local % tiles_x) * (1u << lw) + (lane & ((1u << lw) - 1u));
  y = (local / tiles_x) * (32u >> lw) + (lane >> lw);
}

// Feeds a window's samples, in time order, to the pixel model: every segment lies inside the window, so each
// takes the fast path with x at both ends, each x computed once.
struct WindowFeed {
  PixelProc<GlobalSink>* proc;
  int64_t t_w;
  float irr_max;
  int64_t prev_t;
  float prev_v;
  float last_raw;
  float x_prev;
  // Slot 0, the carried sample, sits at the model time: it replaces the held one.
  __device__ __forceinline__ void start(float carried) {
    last_raw = carried;
    prev_v = clamp_irr(carried, irr_max);
    x_prev = proc->x_at_sample(prev_v);
  }
  __device__ __forceinline__ void operator()(uint32_t dt, float v) {
    last_raw = v;
    const float vc = clamp_irr(v, irr_max);
    const int64_t t = t_w + dt;
    const float x1 = proc->x_at_sample(vc);
    proc->segment_fast(Segment{prev_t, t, prev_v, vc}, x_prev, x1);
    prev_t = t;
    prev_v = vc;
    x_prev = x1;
  }
};

// WindowFeed for a pixel whose state stays in the caller's registers (s, m, c): each segment's clean outcome is taken
// in place, anything else out of line (feed_segment<kFlat>); the same samples and state as WindowFeed's.
template <bool kFlat, class Sink = GlobalSink>
struct RegFeed {
  PixelRegs& s;
  const PixelMapRegs& m;
  PixelCounters& c;
  const SensorConsts& k;
  const SensorConsts* kd;
  uint32_t pixel;
  Sink sink;
  int64_t t_w;
  int64_t prev_t;
  float prev_v;
  float last_raw;
  float x_prev;
  __device__ __forceinline__ void start(float carried) {
    last_raw = carried;
    prev_v = clamp_irr(carried, k.irr_max);
    x_prev = x_sample(s, m, prev_v);
  }
  __device__ __forceinline__ void operator()(uint32_t dt, float v) {
    last_raw = v;
    const float vc = clamp_irr(v, k.irr_max);
    const int64_t t = t_w + dt;
    const float x1 = x_sample(s, m, vc);
    feed_segment<kFlat>(s, m, k, kd, pixel, sink, c, prev_t, t, prev_v, vc, x_prev, x1);
    prev_t = t;
    prev_v = vc;
    x_prev = x1;
  }
};

// At most 128 registers (168 uncapped): 7.79 against 7.93 ms per step on 346x260 (102 registers: 8.58).
__global__ void __launch_bounds__(128, 4) engine_kernel(EngineArgs a) {
  const uint32_t lane = threadIdx.x & 31u;
  const int64_t t0 = *a.t0;
  for (;;) {
    uint32_t tile = 0;
    if (lane == 0) tile = atomicAdd(a.tile_counter, 1u);
    tile = __shfl_sync(0xffffffffu, tile, 0);
    if (tile >= a.total_tiles) break;
    int si = 0;
    while (si + 1 < a.n_sensors && a.sensors[si + 1].tile0 <= tile) ++si;
    const EngineSensor& S = a.sensors[si];
    const uint32_t local = tile - S.tile0;
    uint32_t x, y;
    tile_xy(local, S.tiles_x, a.tile_lw, lane, x, y);
    const bool have = x < S.width && y < S.height;
    const uint32_t p = have ? y * S.width + x : 0u;
    const bool noise = S.consts.noise != 0;
    PixelRegs s;
    PixelMapRegs m;
    float carried = 0.0f;
    if (have) {
      load_state(S.in, p, noise, s);
      load_map(S.map, p, m);
      carried = S.carried_in[p];
    }
    PixelCounters c;
    unsigned long long samples = 0;
    const GlobalSink sink{S.ev, &S.counters[kCntEvents]};
    const FieldDev& f = S.field;
    __shared__ uint16_t lists[4][kMaxListed];
    uint16_t* my_list = lists[threadIdx.x >> 5];
    for (int32_t w = a.w0; w < a.w1; ++w) {
      const int64_t t_w = t0 + static_cast<int64_t>(w) * kWindowNs;
      const BlobList list = warp_blob_list(f, have, x, y, t_w, t_w + kWindowNs, my_list);
      if (have) {
        const int level = field_level(f, list, x, y, t_w, a.r.l_min, a.r.l_max);
        RegFeed<true> feed{s, m, c, S.consts, &S.consts, p, sink, t_w, t_w, s.held, carried, 0.0f};
        feed.start(carried);
        auto render = [&](uint32_t dt) { return field_eval(f, list, x, y, t_w + dt); };
        samples += sample_pixel_window(a.r, level, carried, false, render, feed);
        s.held = feed.prev_v;
        carried = feed.last_raw;
      }
      __syncwarp();
    }
    if (have) {
      store_state(S.out, p, noise, s);
      S.carried_out[p] = carried;
    }
    warp_add(&S.counters[kCntPieces], c.pieces);
    warp_add(&S.counters[kCntLeaves], c.leaves);
    warp_add(&S.counters[kCntSamples], samples);
    warp_add(&S.counters[kCntNoise], c.noise_candidates);
  }
}

// The fused engine with the cascade photoreceptor (noise lattice off): the tile loop of engine_kernel, each window's
// samples fed as segments to CascadeProc (a segment never crosses the window, so each is one piece).
struct CascadeFeed {
  CascadeProc<GlobalSink>* proc;
  int64_t t_w;
  float irr_max;
  int64_t prev_t;
  float prev_v;
  float last_raw;
  __device__ __forceinline__ void start(float carried) {
    last_raw = carried;
    prev_v = clamp_irr(carried, irr_max);
  }
  __device__ __forceinline__ void operator()(uint32_t dt, float v) {
    last_raw = v;
    const float vc = clamp_irr(v, irr_max);
    const int64_t t = t_w + dt;
    proc->segment(Segment{prev_t, t, prev_v, vc}, prev_t, t);
    prev_t = t;
    prev_v = vc;
  }
};

// At most 128 registers (168 uncapped): on the 346x260 cascade workload 36.6 against 38.2 ms per step, spills
// included (the lattice engine, capped alike, ran 1,936 against 1,870 ms and stays uncapped).
__global__ void __launch_bounds__(128, 4) engine_cascade_kernel(EngineArgs a) {
  const uint32_t lane = threadIdx.x & 31u;
  const int64_t t0 = *a.t0;
  for (;;) {
    uint32_t tile = 0;
    if (lane == 0) tile = atomicAdd(a.tile_counter, 1u);
    tile = __shfl_sync(0xffffffffu, tile, 0);
    if (tile >= a.total_tiles) break;
    int si = 0;
    while (si + 1 < a.n_sensors && a.sensors[si + 1].tile0 <= tile) ++si;
    const EngineSensor& S = a.sensors[si];
    const uint32_t local = tile - S.tile0;
    uint32_t x, y;
    tile_xy(local, S.tiles_x, a.tile_lw, lane, x, y);
    const bool have = x < S.width && y < S.height;
    const uint32_t p = have ? y * S.width + x : 0u;
    PixelRegs s;
    CascadeRegs q;
    PixelMapRegs m;
    float carried = 0.0f;
    if (have) {
      load_state(S.in, p, false, s);
      load_cascade(S.in, p, q);
      load_map(S.map, p, m);
      carried = S.carried_in[p];
    }
    PixelCounters c;
    CascadeCounters cn;
    unsigned long long samples = 0;
    GlobalSink sink{S.ev, &S.counters[kCntEvents]};
    CascadeProc<GlobalSink> proc{s, q, m, S.consts, S.cc, p, sink, c, cn};
    const FieldDev& f = S.field;
    __shared__ uint16_t lists[4][kMaxListed];
    uint16_t* my_list = lists[threadIdx.x >> 5];
    for (int32_t w = a.w0; w < a.w1; ++w) {
      const int64_t t_w = t0 + static_cast<int64_t>(w) * kWindowNs;
      const BlobList list = warp_blob_list(f, have, x, y, t_w, t_w + kWindowNs, my_list);
      if (have) {
        const int level = field_level(f, list, x, y, t_w, a.r.l_min, a.r.l_max);
        CascadeFeed feed{&proc, t_w, S.consts.irr_max, t_w, s.held, carried};
        feed.start(carried);
        auto render = [&](uint32_t dt) { return field_eval(f, list, x, y, t_w + dt); };
        samples += sample_pixel_window(a.r, level, carried, false, render, feed);
        s.held = feed.prev_v;
        carried = feed.last_raw;
      }
      __syncwarp();
    }
    if (have) {
      store_state(S.out, p, false, s);
      store_cascade(S.out, p, q);
      S.carried_out[p] = carried;
    }
    warp_add(&S.counters[kCntPieces], c.pieces);
    warp_add(&S.counters[kCntLeaves], c.leaves);
    warp_add(&S.counters[kCntSamples], samples);
    warp_add(&S.counters[kCntSubsteps], cn.substeps);
  }
}

// The fused engine with the cascade's noise lattice. A cell's look-ahead needs the cell's input up to its end, so
// the window's samples are buffered from the last one at or before the current time to the first one at or after
// the cell's end, and the cell then runs on that buffer. A window's last sample is at its end, so each window is
// one call, as in the reference's engine (a cell that crosses the window end sees the held input beyond it).
// kCellBuf bounds the buffer: the engine refuses min_dt_ns < 4096 with the lattice (a cell then holds at most 16
// sample intervals).
constexpr int kCellBuf = 20;

struct CellInput {
  int64_t t_w;
  const uint32_t* dt;  // offsets from t_w, the first at or before the processed range
  const float* v;      // clamped values
  int32_t count;
  BS_HD int n_aug() const { return count; }
  BS_HD int64_t time(int i) const { return t_w + dt[i]; }
  BS_HD float value(int i) const { return v[i]; }
  BS_HD int segment_at(int64_t tt) const {
    int lo = 0, hi = count - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) / 2;
      if (time(mid) <= tt) lo = mid;
      else hi = mid - 1;
    }
    return lo;
  }
  BS_HD int segment_of(int seg, int64_t tt) const {
    while (seg < count - 1 && time(seg + 1) <= tt) ++seg;
    return seg;
  }
  BS_HD int64_t segment_end(int seg) const { return seg + 1 < count ? time(seg + 1) : kForever; }
  BS_HD float group_value(int seg, int64_t tt) const {
    if (seg + 1 >= count) return v[seg];
    const int64_t t0 = time(seg), t1 = time(seg + 1);
    const float f = static_cast<float>(tt - t0) / static_cast<float>(t1 - t0);
    return v[seg] + (v[seg + 1] - v[seg]) * f;
  }
};

struct LatticeFeed {
  LatticeProc<GlobalSink, CellInput>* proc;
  CellInput* in;
  uint32_t* dt;
  float* v;
  int64_t t_w, t_cur, t_end;
  float irr_max;
  float last_raw;
  bool overflow;
  __device__ __forceinline__ void start(float carried) {
    last_raw = carried;
    dt[0] = 0;
    v[0] = clamp_irr(carried, irr_max);
    in->count = 1;
    t_cur = t_w;
  }
  // Runs [t_cur, t_to) on the buffer, then drops the samples before the last one at or before t_to.
  __device__ __forceinline__ void run_to(int64_t t_to) {
    proc->advance_range(t_cur, t_to);
    t_cur = t_to;
    int keep = 0;
    while (keep + 1 < in->count && t_w + dt[keep + 1] <= t_to) ++keep;
    if (keep > 0) {
      for (int i = keep; i < in->count; ++i) {
        dt[i - keep] = dt[i];
        v[i - keep] = v[i];
      }
      in->count -= keep;
    }
  }
  __device__ __forceinline__ void operator()(uint32_t d, float val) {
    last_raw = val;
    if (in->count == kCellBuf) {
      overflow = true;
      return;
    }
    dt[in->count] = d;
    v[in->count] = clamp_irr(val, irr_max);
    ++in->count;
    const int64_t t = t_w + d;
    while (t_cur < t_end) {
      const int64_t tc1 = ((t_cur >> kNoiseCellLog2) + 1) * kNoiseCellNs;
      if (t < tc1) break;
      run_to(mini(tc1, t_end));
    }
  }
  __device__ __forceinline__ void finish() {
    if (t_cur < t_end) run_to(t_end);
  }
};

__global__ void __launch_bounds__(128) engine_lattice_kernel(EngineArgs a) {
  const uint32_t lane = threadIdx.x & 31u;
  const int64_t t0 = *a.t0;
  for (;;) {
    uint32_t tile = 0;
    if (lane == 0) tile = atomicAdd(a.tile_counter, 1u);
    tile = __shfl_sync(0xffffffffu, tile, 0);
    if (tile >= a.total_tiles) break;
    int si = 0;
    while (si + 1 < a.n_sensors && a.sensors[si + 1].tile0 <= tile) ++si;
    const EngineSensor& S = a.sensors[si];
    const uint32_t local = tile - S.tile0;
    uint32_t x, y;
    tile_xy(local, S.tiles_x, a.tile_lw, lane, x, y);
    const bool have = x < S.width && y < S.height;
    const uint32_t n_px = S.width * S.height;
    const uint32_t p = have ? y * S.width + x : 0u;
    PixelRegs s;
    CascadeRegs q;
    LatticeRegs L;
    PixelMapRegs m;
    float carried = 0.0f;
    if (have) {
      load_state(S.in, p, false, s);
      load_cascade(S.in, p, q);
      load_lattice(S.in, p, n_px, L);
      load_map(S.map, p, m);
      carried = S.carried_in[p];
    }
    PixelCounters c;
    CascadeCounters cn;
    unsigned long long samples = 0, err = 0;
    GlobalSink sink{S.ev, &S.counters[kCntEvents]};
    uint32_t buf_dt[kCellBuf];
    float buf_v[kCellBuf];
    CellInput in{0, buf_dt, buf_v, 0};
    LatticeProc<GlobalSink, CellInput> proc{s, q, L, m, S.consts, S.cc, S.tab, p, sink, c, cn, in};
    if (have) proc.resume();
    const FieldDev& f = S.field;
    __shared__ uint16_t lists[4][kMaxListed];
    uint16_t* my_list = lists[threadIdx.x >> 5];
    for (int32_t w = a.w0; w < a.w1; ++w) {
      const int64_t t_w = t0 + static_cast<int64_t>(w) * kWindowNs;
      const BlobList list = warp_blob_list(f, have, x, y, t_w, t_w + kWindowNs, my_list);
      if (have && err == 0) {
        const int level = field_level(f, list, x, y, t_w, a.r.l_min, a.r.l_max);
        in.t_w = t_w;
        LatticeFeed feed{&proc, &in, buf_dt, buf_v, t_w, t_w, t_w + kWindowNs, S.consts.irr_max, carried, false};
        feed.start(carried);
        auto render = [&](uint32_t dt) { return field_eval(f, list, x, y, t_w + dt); };
        samples += sample_pixel_window(a.r, level, carried, false, render, feed);
        if (feed.overflow) {
          err |= kErrRunRange;
        } else {
          feed.finish();
          s.held = buf_v[in.count - 1];
        }
        carried = feed.last_raw;
      }
      __syncwarp();
    }
    if (have) {
      store_state(S.out, p, false, s);
      store_cascade(S.out, p, q);
      store_lattice(S.out, p, n_px, L);
      S.carried_out[p] = carried;
    }
    warp_add(&S.counters[kCntPieces], c.pieces);
    warp_add(&S.counters[kCntLeaves], c.leaves);
    warp_add(&S.counters[kCntSamples], samples);
    warp_add(&S.counters[kCntSubsteps], cn.substeps);
    warp_or(&S.counters[kCntErrors], err);
  }
}

// The lattice engine in two phases per window, so that a warp's lanes run the lattice's code together: phase A runs
// every lane's sampler walk and stages its window's samples in shared memory (kLatStage per lane, lane-minor, slot 0
// the carried sample); phase B runs every lane's 128 cells from its staged samples. A window with more samples than
// kLatStage is redone by its lane in the streaming form (the same samples: the walk is deterministic).
constexpr int kLatStage = 32;

struct StagedInput {
  int64_t t_w;
  const uint32_t* dt;  // entry i at dt[i * 32]
  const float* v;      // clamped values, entry i at v[i * 32]
  int32_t count;
  BS_HD int n_aug() const { return count; }
  BS_HD int64_t time(int i) const { return t_w + dt[i * 32]; }
  BS_HD float value(int i) const { return v[i * 32]; }
  BS_HD int segment_at(int64_t tt) const {
    int lo = 0, hi = count - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) / 2;
      if (time(mid) <= tt) lo = mid;
      else hi = mid - 1;
    }
    return lo;
  }
  BS_HD int segment_of(int seg, int64_t tt) const {
    while (seg < count - 1 && time(seg + 1) <= tt) ++seg;
    return seg;
  }
  BS_HD int64_t segment_end(int seg) const { return seg + 1 < count ? time(seg + 1) : kForever; }
  BS_HD float group_value(int seg, int64_t tt) const {
    if (seg + 1 >= count) return value(seg);
    const int64_t t0 = time(seg), t1 = time(seg + 1);
    const float f = static_cast<float>(tt - t0) / static_cast<float>(t1 - t0);
    const float v0 = value(seg), v1 = value(seg + 1);
    return v0 + (v1 - v0) * f;
  }
};

struct LatticeStageFeed {
  uint32_t* dt;
  float* v;
  float irr_max;
  int32_t n;
  bool overflow;
  float last_raw;
  __device__ __forceinline__ void start(float carried) {
    last_raw = carried;
    dt[0] = 0;
    v[0] = clamp_irr(carried, irr_max);
    n = 1;
  }
  __device__ __forceinline__ void operator()(uint32_t d, float val) {
    last_raw = val;
    if (n == kLatStage) {
      overflow = true;
      return;
    }
    dt[n * 32] = d;
    v[n * 32] = clamp_irr(val, irr_max);
    ++n;
  }
};

__global__ void __launch_bounds__(128) engine_lattice_kernel_staged(EngineArgs a) {
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const int64_t t0 = *a.t0;
  __shared__ uint16_t lists[4][kMaxListed];
  __shared__ uint32_t st_dt[4][kLatStage][32];
  __shared__ float st_v[4][kLatStage][32];
  uint16_t* my_list = lists[warp];
  for (;;) {
    uint32_t tile = 0;
    if (lane == 0) tile = atomicAdd(a.tile_counter, 1u);
    tile = __shfl_sync(0xffffffffu, tile, 0);
    if (tile >= a.total_tiles) break;
    int si = 0;
    while (si + 1 < a.n_sensors && a.sensors[si + 1].tile0 <= tile) ++si;
    const EngineSensor& S = a.sensors[si];
    const uint32_t local = tile - S.tile0;
    uint32_t x, y;
    tile_xy(local, S.tiles_x, a.tile_lw, lane, x, y);
    const bool have = x < S.width && y < S.height;
    const uint32_t n_px = S.width * S.height;
    const uint32_t p = have ? y * S.width + x : 0u;
    PixelRegs s;
    CascadeRegs q;
    LatticeRegs L;
    PixelMapRegs m;
    float carried = 0.0f;
    if (have) {
      load_state(S.in, p, false, s);
      load_cascade(S.in, p, q);
      load_lattice(S.in, p, n_px, L);
      load_map(S.map, p, m);
      carried = S.carried_in[p];
    }
    PixelCounters c;
    CascadeCounters cn;
    unsigned long long samples = 0, err = 0;
    GlobalSink sink{S.ev, &S.counters[kCntEvents]};
    const FieldDev& f = S.field;
    uint32_t* my_dt = &st_dt[warp][0][lane];
    float* my_v = &st_v[warp][0][lane];
    for (int32_t w = a.w0; w < a.w1; ++w) {
      const int64_t t_w = t0 + static_cast<int64_t>(w) * kWindowNs;
      const BlobList list = warp_blob_list(f, have, x, y, t_w, t_w + kWindowNs, my_list);
      auto render = [&](uint32_t dt) { return field_eval(f, list, x, y, t_w + dt); };
      int level = 0;
      LatticeStageFeed stage{my_dt, my_v, S.consts.irr_max, 0, false, carried};
      if (have && err == 0) {
        level = field_level(f, list, x, y, t_w, a.r.l_min, a.r.l_max);
        stage.start(carried);
        samples += sample_pixel_window(a.r, level, carried, false, render, stage);
      }
      __syncwarp();
      if (have && err == 0) {
        if (!stage.overflow) {
          const StagedInput in{t_w, my_dt, my_v, stage.n};
          LatticeProc<GlobalSink, StagedInput> proc{s, q, L, m, S.consts, S.cc, S.tab, p, sink, c, cn, in};
          proc.resume();
          proc.advance_range(t_w, t_w + kWindowNs);
          s.held = my_v[(stage.n - 1) * 32];
        } else {
          uint32_t buf_dt[kCellBuf];
          float buf_v[kCellBuf];
          CellInput in{t_w, buf_dt, buf_v, 0};
          LatticeProc<GlobalSink, CellInput> proc{s, q, L, m, S.consts, S.cc, S.tab, p, sink, c, cn, in};
          proc.resume();
          LatticeFeed feed{&proc, &in, buf_dt, buf_v, t_w, t_w, t_w + kWindowNs, S.consts.irr_max, carried, false};
          feed.start(carried);
          sample_pixel_window(a.r, level, carried, false, render, feed);
          if (feed.overflow) {
            err |= kErrRunRange;
          } else {
            feed.finish();
            s.held = buf_v[in.count - 1];
          }
        }
        carried = stage.last_raw;
      }
      __syncwarp();
    }
    if (have) {
      store_state(S.out, p, false, s);
      store_cascade(S.out, p, q);
      store_lattice(S.out, p, n_px, L);
      S.carried_out[p] = carried;
    }
    warp_add(&S.counters[kCntPieces], c.pieces);
    warp_add(&S.counters[kCntLeaves], c.leaves);
    warp_add(&S.counters[kCntSamples], samples);
    warp_add(&S.counters[kCntSubsteps], cn.substeps);
    warp_or(&S.counters[kCntErrors], err);
  }
}

// The engine in two phases per window: phase A runs every lane's sampler walk and stages its samples (dt, v) in
// shared memory, kStage per lane (lane-minor, so a warp's stores and loads hit 32 banks); phase B feeds every lane's
// staged samples to its pixel model. Each phase is one compact loop that all lanes run together, instead of the
// sampler and the pixel model alternating per sample across diverged lanes. A window with more samples than kStage
// is redone by its lane in the streaming form (the same samples: the walk is deterministic).
template <int kStage>
__global__ void __launch_bounds__(128) engine_kernel_staged(EngineArgs a) {
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const int64_t t0 = *a.t0;
  __shared__ uint16_t lists[4][kMaxListed];
  __shared__ uint32_t st_dt[4][kStage][32];
  __shared__ float st_v[4][kStage][32];
  uint16_t* my_list = lists[warp];
  for (;;) {
    uint32_t tile = 0;
    if (lane == 0) tile = atomicAdd(a.tile_counter, 1u);
    tile = __shfl_sync(0xffffffffu, tile, 0);
    if (tile >= a.total_tiles) break;
    int si = 0;
    while (si + 1 < a.n_sensors && a.sensors[si + 1].tile0 <= tile) ++si;
    const EngineSensor& S = a.sensors[si];
    const uint32_t local = tile - S.tile0;
    uint32_t x, y;
    tile_xy(local, S.tiles_x, a.tile_lw, lane, x, y);
    const bool have = x < S.width && y < S.height;
    const uint32_t p = have ? y * S.width + x : 0u;
    const bool noise = S.consts.noise != 0;
    PixelRegs s;
    PixelMapRegs m;
    float carried = 0.0f;
    if (have) {
      load_state(S.in, p, noise, s);
      load_map(S.map, p, m);
      carried = S.carried_in[p];
    }
    PixelCounters c;
    unsigned long long samples = 0;
    const GlobalSink sink{S.ev, &S.counters[kCntEvents]};
    const FieldDev& f = S.field;
    for (int32_t w = a.w0; w < a.w1; ++w) {
      const int64_t t_w = t0 + static_cast<int64_t>(w) * kWindowNs;
      const BlobList list = warp_blob_list(f, have, x, y, t_w, t_w + kWindowNs, my_list);
      auto render = [&](uint32_t dt) { return field_eval(f, list, x, y, t_w + dt); };
      // Phase A: the walk, its first kStage samples after slot 0 staged.
      uint32_t n = 0;
      int level = 0;
      if (have) {
        level = field_level(f, list, x, y, t_w, a.r.l_min, a.r.l_max);
        uint32_t k = 0;
        n = sample_pixel_window(a.r, level, carried, false, render, [&](uint32_t dt, float v) {
          if (k < static_cast<uint32_t>(kStage)) {
            st_dt[warp][k][lane] = dt;
            st_v[warp][k][lane] = v;
          }
          ++k;
        });
      }
      __syncwarp();
      // Phase N: the window's noise candidates of all lanes together; the rejected ones leave the pixel model.
      if (noise) {
        const StagedRun run{t_w, &st_dt[warp][0][lane], &st_v[warp][0][lane], static_cast<int>(n) - 1};
        noise_ahead(s, m, S.consts, p, have && n - 1 <= static_cast<uint32_t>(kStage), t_w,
                    clamp_irr(carried, S.consts.irr_max), t_w + kWindowNs, run, c);
      }
      // Phase B: the pixel model over the staged samples.
      if (have) {
        RegFeed<false> feed{s, m, c, S.consts, &S.consts, p, sink, t_w, t_w, s.held, carried, 0.0f};
        feed.start(carried);
        if (n - 1 <= static_cast<uint32_t>(kStage)) {
          for (uint32_t k = 0; k + 1 < n; ++k) feed(st_dt[warp][k][lane], st_v[warp][k][lane]);
        } else {
          sample_pixel_window(a.r, level, carried, false, render, feed);
        }
        samples += n;
        s.held = feed.prev_v;
        carried = feed.last_raw;
      }
      __syncwarp();
    }
    if (have) {
      store_state(S.out, p, noise, s);
      S.carried_out[p] = carried;
    }
    warp_add(&S.counters[kCntPieces], c.pieces);
    warp_add(&S.counters[kCntLeaves], c.leaves);
    warp_add(&S.counters[kCntSamples], samples);
    warp_add(&S.counters[kCntNoise], c.noise_candidates);
  }
}

// ---------------------------------------------------------------------------------------------
// The split engine: per window, the common path in one kernel and the rare one in another
// ---------------------------------------------------------------------------------------------
// A pixel's rare paths (a segment where a crossing may occur, an accepted noise candidate, the refractory interval,
// the first segment after the start) run one or two lanes at a time while the rest of the warp waits, and their code
// competes with the hot loop's for the instruction cache: on the six sensors they took most of the staged engine's
// time. Here each window is two launches. engine_window_kernel runs the staged engine's phases for every pixel (the
// walk with its first kSplitStage samples staged, the noise pass, the pixel model's clean segments in registers)
// and, at a pixel's first segment that is not clean, stops that pixel and posts it (its state, its feed and the
// staged samples left) to a list; a window that overflows the stage is posted whole. engine_rest_kernel then
// finishes the posted pixels' windows, one thread per pixel, through the full pixel model, so its lanes all run the
// rare paths together. A pixel's samples are fed in the same order to the same state either way, so events and
// state are the staged engine's; the state passes from one window to the next through HBM.
constexpr int kSplitStage = 16;
constexpr uint32_t kRestWhole = 0xFF;  // the samples left of a window that overflowed the stage

// The posted pixels, as planes (structure of arrays): field k of record i at plane k, entry i, so that the window
// kernel's posting lanes (consecutive records) store and the rest kernel's threads load with coalesced accesses.
// Per record: the state where the pixel stopped (after the noise pass and its clean segments); the feed (the last
// sample fed: time, clamped value, x; the last raw value); the pixel, its sensor, the samples left in dt / v
// (kRestWhole: the window from its start, the carried sample in last_raw) and the window's lattice level (for a
// whole window); the staged samples left.
enum : int { kR64TRef, kR64TSearch, kR64Blind, kR64TShot, kR64TBa, kR64PrevT, kRest64 };
enum : int {
  kR32S3Ref, kR32N3Ref, kR32DrRef, kR32IScale, kR32Held, kR32Flags, kR32NShot, kR32NBa, kR32PrevV, kR32XPrev,
  kR32LastRaw, kR32Pixel, kR32Tag, kR32Dt, kR32V = kR32Dt + kSplitStage, kRest32 = kR32V + kSplitStage
};
constexpr size_t kRestRecordBytes = kRest64 * 8 + kRest32 * 4;

struct RestList {
  unsigned char* base;  // kRest64 planes of 8 bytes, then kRest32 planes of 4, each `capacity` entries
  unsigned int* count;
  unsigned int capacity;
  __device__ __forceinline__ int64_t* p64(int k) const {
    return reinterpret_cast<int64_t*>(base) + static_cast<size_t>(k) * capacity;
  }
  __device__ __forceinline__ uint32_t* p32(int k) const {
    return reinterpret_cast<uint32_t*>(base + static_cast<size_t>(kRest64) * 8 * capacity) +
           static_cast<size_t>(k) * capacity;
  }
  __device__ __forceinline__ void put_state(unsigned int i, const PixelRegs& s) const {
    p64(kR64TRef)[i] = s.t_ref;
    p64(kR64TSearch)[i] = s.t_search;
    p64(kR64Blind)[i] = s.blind_until;
    p64(kR64TShot)[i] = s.t_shot;
    p64(kR64TBa)[i] = s.t_ba;
    p32(kR32S3Ref)[i] = __float_as_uint(s.s3_ref);
    p32(kR32N3Ref)[i] = __float_as_uint(s.n3_ref);
    p32(kR32DrRef)[i] = __float_as_uint(s.dr_ref);
    p32(kR32IScale)[i] = __float_as_uint(s.i_scale);
    p32(kR32Held)[i] = __float_as_uint(s.held);
    p32(kR32Flags)[i] = s.flags;
    p32(kR32NShot)[i] = s.n_shot;
    p32(kR32NBa)[i] = s.n_ba;
  }
  __device__ __forceinline__ PixelRegs state(unsigned int i) const {
    PixelRegs s;
    s.t_ref = p64(kR64TRef)[i];
    s.t_search = p64(kR64TSearch)[i];
    s.blind_until = p64(kR64Blind)[i];
    s.t_shot = p64(kR64TShot)[i];
    s.t_ba = p64(kR64TBa)[i];
    s.s3_ref = __uint_as_float(p32(kR32S3Ref)[i]);
    s.n3_ref = __uint_as_float(p32(kR32N3Ref)[i]);
    s.dr_ref = __uint_as_float(p32(kR32DrRef)[i]);
    s.i_scale = __uint_as_float(p32(kR32IScale)[i]);
    s.held = __uint_as_float(p32(kR32Held)[i]);
    s.flags = p32(kR32Flags)[i];
    s.n_shot = p32(kR32NShot)[i];
    s.n_ba = p32(kR32NBa)[i];
    return s;
  }
};

// Window a.w0 of every tile (a.t0 the model time at the call's start). kFirst: the call's first window, where the
// pixels' searches can be armed after their first segment's start (after init): such a segment is also taken in
// place when clean (clean_after_start), instead of being posted; the other windows' kernel leaves that test out (in
// the hot loop it cost more than it saves there).
template <bool kFirst>
__global__ void __launch_bounds__(128) engine_window_kernel(EngineArgs a, RestList rl) {
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const int64_t t_w = *a.t0 + static_cast<int64_t>(a.w0) * kWindowNs;
  __shared__ uint16_t lists[4][kMaxListed];
  __shared__ uint32_t st_dt[4][kSplitStage][32];
  __shared__ float st_v[4][kSplitStage][32];
  uint16_t* my_list = lists[warp];
  for (;;) {
    uint32_t tile = 0;
    if (lane == 0) tile = atomicAdd(a.tile_counter, 1u);
    tile = __shfl_sync(0xffffffffu, tile, 0);
    if (tile >= a.total_tiles) break;
    int si = 0;
    while (si + 1 < a.n_sensors && a.sensors[si + 1].tile0 <= tile) ++si;
    const EngineSensor& S = a.sensors[si];
    const uint32_t local = tile - S.tile0;
    uint32_t x, y;
    tile_xy(local, S.tiles_x, a.tile_lw, lane, x, y);
    const bool have = x < S.width && y < S.height;
    const uint32_t p = have ? y * S.width + x : 0u;
    const bool noise = S.consts.noise != 0;
    const float irr_max = S.consts.irr_max;
    PixelRegs s;
    PixelMapRegs m;
    float carried = 0.0f;
    if (have) {
      load_state(S.in, p, noise, s);
      load_map(S.map, p, m);
      carried = S.carried_in[p];
    }
    PixelCounters c;
    const FieldDev& f = S.field;
    const BlobList list = warp_blob_list(f, have, x, y, t_w, t_w + kWindowNs, my_list);
    auto render = [&](uint32_t dt) { return field_eval(f, list, x, y, t_w + dt); };
    // The walk, its first kSplitStage samples after slot 0 staged.
    uint32_t n = 0;
    int level = 0;
    if (have) {
      level = field_level(f, list, x, y, t_w, a.r.l_min, a.r.l_max);
      uint32_t k = 0;
      n = sample_pixel_window(a.r, level, carried, false, render, [&](uint32_t dt, float v) {
        if (k < static_cast<uint32_t>(kSplitStage)) {
          st_dt[warp][k][lane] = dt;
          st_v[warp][k][lane] = v;
        }
        ++k;
      });
    }
    __syncwarp();
    const bool staged = have && n - 1 <= static_cast<uint32_t>(kSplitStage);
    // The window's noise candidates of all lanes together; the rejected ones leave the pixel model.
    if (noise) {
      const StagedRun run{t_w, &st_dt[warp][0][lane], &st_v[warp][0][lane], static_cast<int>(n) - 1};
      noise_ahead(s, m, S.consts, p, staged, t_w, clamp_irr(carried, irr_max), t_w + kWindowNs, run, c);
    }
    // The clean segments in place; the first other one stops the pixel there (a window that overflowed the stage
    // stops at its start).
    bool post = have && !staged;
    uint32_t j = 0;
    int64_t prev_t = t_w;
    float prev_v = 0.0f, last_raw = carried, x_prev = 0.0f;
    if (staged) {
      prev_v = clamp_irr(carried, irr_max);
      x_prev = x_sample(s, m, prev_v);
      for (; j + 1 < n; ++j) {
        const float v = st_v[warp][j][lane];
        const int64_t t = t_w + st_dt[warp][j][lane];
        const float vc = clamp_irr(v, irr_max);
        const float x1 = x_sample(s, m, vc);
        if (!clean_segment(s, m, S.consts, prev_t, t, prev_v, vc, x_prev, x1) &&
            !(kFirst && clean_after_start(s, m, S.consts, prev_t, t, prev_v, vc, x_prev, x1))) {
          break;
        }
        ++c.pieces;
        if (t - prev_t > 2) ++c.leaves;
        s.t_search = maxi(s.t_search, t);
        last_raw = v;
        prev_t = t;
        prev_v = vc;
        x_prev = x1;
      }
      post = j + 1 < n;
      if (!post) {
        s.held = prev_v;
        store_state(S.out, p, noise, s);
        S.carried_out[p] = last_raw;
      }
    }
    // One record per stopped pixel, the warp's records reserved together.
    __syncwarp();
    const unsigned posting = __ballot_sync(0xffffffffu, post);
    if (posting != 0u) {
      const int leader = __ffs(posting) - 1;
      unsigned int base = 0;
      if (static_cast<int>(lane) == leader) base = atomicAdd(rl.count, static_cast<unsigned int>(__popc(posting)));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (post) {
        const unsigned int i = base + static_cast<unsigned int>(__popc(posting & ((1u << lane) - 1u)));
        if (i >= rl.capacity) {
          atomicOr(&S.counters[kCntErrors], kErrRestList);
        } else {
          rl.put_state(i, s);
          rl.p64(kR64PrevT)[i] = prev_t;
          rl.p32(kR32PrevV)[i] = __float_as_uint(prev_v);
          rl.p32(kR32XPrev)[i] = __float_as_uint(x_prev);
          rl.p32(kR32LastRaw)[i] = __float_as_uint(last_raw);
          rl.p32(kR32Pixel)[i] = p;
          const uint32_t left = staged ? n - 1 - j : kRestWhole;
          rl.p32(kR32Tag)[i] = static_cast<uint32_t>(si) | left << 16 | static_cast<uint32_t>(level) << 24;
          if (staged) {  // by plane, so that the posting lanes write each plane together
            for (uint32_t u = 0; u < left; ++u) {
              rl.p32(kR32Dt + static_cast<int>(u))[i] = st_dt[warp][j + u][lane];
              rl.p32(kR32V + static_cast<int>(u))[i] = __float_as_uint(st_v[warp][j + u][lane]);
            }
          }
        }
      }
    }
    __syncwarp();
    warp_add(&S.counters[kCntPieces], c.pieces);
    warp_add(&S.counters[kCntLeaves], c.leaves);
    warp_add(&S.counters[kCntSamples], have ? n : 0u);
    warp_add(&S.counters[kCntNoise], c.noise_candidates);
  }
}

// The posted pixels of window a.w0, one thread each: the rest of the window through the full pixel model (a window
// posted whole is walked again from its start, every blob of the field evaluated: the same values as the warp's
// culled list gives), then the state and the carried sample stored. Capped for 5 blocks per SM (at most 102
// registers): more spills, but 20 warps per SM; on the six sensors 68.5 ms per step against 70.1 at 4 blocks (128
// registers) and 69.0 at 6 (4 blocks had measured 0.5 % faster than 3, uncapped).
__global__ void __launch_bounds__(128, 5) engine_rest_kernel(EngineArgs a, RestList rl) {
  const int64_t t_w = *a.t0 + static_cast<int64_t>(a.w0) * kWindowNs;
  const unsigned int count = min(*rl.count, rl.capacity);
  for (unsigned int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const uint32_t tag = rl.p32(kR32Tag)[i], pixel = rl.p32(kR32Pixel)[i];
    const uint32_t left = tag >> 16 & 0xFFu;
    const float raw0 = __uint_as_float(rl.p32(kR32LastRaw)[i]);
    const EngineSensor& S = a.sensors[tag & 0xFFFFu];
    PixelRegs s = rl.state(i);
    PixelMapRegs m;
    load_map(S.map, pixel, m);
    PixelCounters c;
    const ThreadSink sink{S.ev, &S.counters[kCntEvents]};
    float held, last_raw;
    if (left == kRestWhole) {
      const FieldDev& f = S.field;
      const BlobList all{nullptr, f.n_blobs};
      const uint32_t x = pixel % S.width, y = pixel / S.width;
      auto render = [&](uint32_t dt) { return field_eval(f, all, x, y, t_w + dt); };
      RegFeed<true, ThreadSink> feed{s, m, c, S.consts, &S.consts, pixel, sink, t_w, t_w, s.held, raw0, 0.0f};
      feed.start(raw0);
      sample_pixel_window(a.r, static_cast<int>(tag >> 24), raw0, false, render, feed);
      held = feed.prev_v;
      last_raw = feed.last_raw;
    } else {
      RegFeed<true, ThreadSink> feed{s, m, c, S.consts, &S.consts, pixel, sink, t_w, rl.p64(kR64PrevT)[i],
                                     __uint_as_float(rl.p32(kR32PrevV)[i]), raw0,
                                     __uint_as_float(rl.p32(kR32XPrev)[i])};
      for (uint32_t q = 0; q < left; ++q) {
        feed(rl.p32(kR32Dt + static_cast<int>(q))[i], __uint_as_float(rl.p32(kR32V + static_cast<int>(q))[i]));
      }
      held = feed.prev_v;
      last_raw = feed.last_raw;
    }
    s.held = held;
    store_state(S.out, pixel, S.consts.noise != 0, s);
    S.carried_out[pixel] = last_raw;
    if (c.pieces) atomicAdd(&S.counters[kCntPieces], static_cast<unsigned long long>(c.pieces));
    if (c.leaves) atomicAdd(&S.counters[kCntLeaves], static_cast<unsigned long long>(c.leaves));
    if (c.noise_candidates) atomicAdd(&S.counters[kCntNoise], static_cast<unsigned long long>(c.noise_candidates));
  }
}

// ---------------------------------------------------------------------------------------------
// The fused engine with the warp-cooperative crossing search
// ---------------------------------------------------------------------------------------------

// One pixel's crossing search as every lane of the warp needs it: the piece and the comparator's state.
struct SearchReq {
  int64_t g_t0, g_t1, lo, hi, t_ref;
  float g_v0, g_v1, i_scale, s3_ref, n3_ref, dr_ref, leak, theta_on, theta_off, dark, scale;
};

__device__ __forceinline__ SearchReq request_of(const PixelProc<GlobalSink>& p) {
  return SearchReq{p.pg.t0, p.pg.t1, p.p_lo, p.p_stop, p.s.t_ref, p.pg.v0, p.pg.v1, p.s.i_scale, p.s.s3_ref,
                   p.s.n3_ref, p.s.dr_ref, p.m.leak, p.m.theta_on, p.m.theta_off, p.m.dark, p.m.scale};
}

__device__ __forceinline__ SearchReq shfl_req(const SearchReq& r, int src) {
  const unsigned full = 0xffffffffu;
  SearchReq o;
  o.g_t0 = __shfl_sync(full, r.g_t0, src);
  o.g_t1 = __shfl_sync(full, r.g_t1, src);
  o.lo = __shfl_sync(full, r.lo, src);
  o.hi = __shfl_sync(full, r.hi, src);
  o.t_ref = __shfl_sync(full, r.t_ref, src);
  o.g_v0 = __shfl_sync(full, r.g_v0, src);
  o.g_v1 = __shfl_sync(full, r.g_v1, src);
  o.i_scale = __shfl_sync(full, r.i_scale, src);
  o.s3_ref = __shfl_sync(full, r.s3_ref, src);
  o.n3_ref = __shfl_sync(full, r.n3_ref, src);
  o.dr_ref = __shfl_sync(full, r.dr_ref, src);
  o.leak = __shfl_sync(full, r.leak, src);
  o.theta_on = __shfl_sync(full, r.theta_on, src);
  o.theta_off = __shfl_sync(full, r.theta_off, src);
  o.dark = __shfl_sync(full, r.dark, src);
  o.scale = __shfl_sync(full, r.scale, src);
  return o;
}

// The first integer t in [lo, hi) where Delta fires, searched by the whole warp (all 32 lanes, uniform control
// flow): the time-ordered search of PixelProc::search with 32-way splits. A node (a, c] with x at its ends splits
// at a + len j / 32; lane j takes sub-interval j (the exact node test, or Delta itself at a single integer), a ballot
// picks the earliest candidate, and the rest of the node after it (when a later sub-interval is a candidate too)
// waits on a stack; a node of at most 32 integers is tested integer by integer, one per lane. Every evaluation is
// PixelProc's own, and any time-ordered exhaustive search with a sound node test finds the same first integer.
// Returns false when no integer fires. *leaves counts the nodes tested with the node test (32 per split round, one
// per sub-interval longer than one integer): they are this search's nodes, not the serial search's.
//
// The round bound is derived from the piece: every round that removes no integer from the unexplored set (the node
// and the stack) descends one 32-fold level, at most 5 levels below the node it started from, so a search of
// hi - lo integers ends within 6 (hi - lo) + 6 rounds. (Where Delta stays just under a level over a long piece, most
// sub-intervals stay candidates and the search really visits about (hi - lo) / 32 leaves, like the serial one.) The
// stack holds one entry per level. *err is set only if either bound is passed, which the argument above excludes.
__device__ bool coop_search(const SearchReq& r, const SensorConsts& k, uint32_t lane, int64_t& t_hit, bool& on,
                            float& x_hit, uint32_t* leaves, unsigned long long* err) {
  const unsigned full = 0xffffffffu;
  PixelRegs rs{};
  rs.t_ref = r.t_ref;
  rs.s3_ref = r.s3_ref;
  rs.n3_ref = r.n3_ref;
  rs.dr_ref = r.dr_ref;
  rs.i_scale = r.i_scale;
  PixelMapRegs rm{r.theta_on, r.theta_off, r.leak, r.dark, r.scale, 0.0, 0.0};
  NullSink ns;
  PixelCounters pc;
  const PixelProc<NullSink> ev{rs, rm, k, 0u, ns, pc};
  const Segment g{r.g_t0, r.g_t1, r.g_v0, r.g_v1};
  const auto fires = [&](float D) { return D >= r.theta_on || D <= -r.theta_off; };
  const float x_lo = ev.log_ratio(ev.current(g, r.lo));
  const float D_lo = ev.delta(r.lo, x_lo);
  if (fires(D_lo)) {
    t_hit = r.lo;
    on = D_lo >= r.theta_on;
    x_hit = x_lo;
    return true;
  }
  if (r.hi - r.lo == 1) return false;
  constexpr int kStack = 16;  // one entry per nesting level: 2^23 integers need 5
  int64_t sa[kStack], sc[kStack];
  float sxa[kStack], sxc[kStack];
  int sp = 0;
  int64_t a = r.lo, c = r.hi - 1;
  float xa = x_lo, xc = ev.log_ratio(ev.current(g, c));
  const int64_t max_rounds = 6 * (r.hi - r.lo) + 64;
  for (int64_t round = 0; round < max_rounds; ++round) {
    const int64_t len = c - a;
    if (len <= 32) {
      const int64_t t = a + 1 + lane;
      bool f = false, ont = false;
      float xt = 0.0f;
      if (t <= c) {
        xt = t == c ? xc : ev.log_ratio(ev.current(g, t));
        const float Dt = ev.delta(t, xt);
        f = fires(Dt);
        ont = Dt >= r.theta_on;
      }
      const unsigned b = __ballot_sync(full, f);
      if (b != 0u) {
        const int j = __ffs(b) - 1;
        t_hit = a + 1 + j;
        on = __shfl_sync(full, ont, j);
        x_hit = __shfl_sync(full, xt, j);
        return true;
      }
    } else {
      const int64_t bl = a + (len * lane) / 32, br = a + (len * (lane + 1)) / 32;
      const float xr = lane == 31 ? xc : ev.log_ratio(ev.current(g, br));
      float xl = __shfl_up_sync(full, xr, 1);
      if (lane == 0) xl = xa;
      bool may;
      if (br - bl == 1) {
        may = fires(ev.delta(br, xr));
      } else {
        may = ev.may_fire_exact(bl, br, xl, xr);
      }
      *leaves += __popc(__ballot_sync(full, br - bl > 1));
      const unsigned b = __ballot_sync(full, may);
      if (b != 0u) {
        const int j = __ffs(b) - 1;
        const int64_t nl = a + (len * j) / 32, nr = a + (len * (j + 1)) / 32;
        const float nxl = __shfl_sync(full, xl, j), nxr = __shfl_sync(full, xr, j);
        if ((b >> j) > 1u) {  // a later sub-interval is a candidate too: the rest of the node waits
          if (sp == kStack) {
            *err |= kErrSearchBound;
            return false;
          }
          sa[sp] = nr;
          sc[sp] = c;
          sxa[sp] = nxr;
          sxc[sp] = xc;
          ++sp;
        }
        a = nl;
        c = nr;
        xa = nxl;
        xc = nxr;
        continue;
      }
    }
    if (sp == 0) return false;
    --sp;
    a = sa[sp];
    c = sc[sp];
    xa = sxa[sp];
    xc = sxc[sp];
  }
  *err |= kErrSearchBound;
  return false;
}

// The staged engine (engine_kernel_staged<32>) with the crossing search taken by the whole warp. Phase B is one
// warp-uniform loop: every lane feeds its staged samples with the search deferred, up to its first search or the
// window's end; the warp then runs the posted searches one by one, 32 lanes each; the lanes apply the outcomes
// (the event, or the search cleared to its stop) and resume their pieces. Where many lanes search at once (dense
// events with noise and leak: C3, C4) the searches queue behind one another and the autotuner keeps another stage. Lanes whose window overflowed the stage
// run it alone afterwards, searching as the other engines do.
__global__ void __launch_bounds__(128) engine_kernel_coop(EngineArgs a) {
  constexpr int kStage = 32;
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const unsigned full = 0xffffffffu;
  const int64_t t0 = *a.t0;
  __shared__ uint16_t lists[4][kMaxListed];
  __shared__ uint32_t st_dt[4][kStage][32];
  __shared__ float st_v[4][kStage][32];
  uint16_t* my_list = lists[warp];
  for (;;) {
    uint32_t tile = 0;
    if (lane == 0) tile = atomicAdd(a.tile_counter, 1u);
    tile = __shfl_sync(full, tile, 0);
    if (tile >= a.total_tiles) break;
    int si = 0;
    while (si + 1 < a.n_sensors && a.sensors[si + 1].tile0 <= tile) ++si;
    const EngineSensor& S = a.sensors[si];
    const uint32_t local = tile - S.tile0;
    uint32_t x, y;
    tile_xy(local, S.tiles_x, a.tile_lw, lane, x, y);
    const bool have = x < S.width && y < S.height;
    const uint32_t p = have ? y * S.width + x : 0u;
    const bool noise = S.consts.noise != 0;
    PixelRegs s;
    PixelMapRegs m;
    float carried = 0.0f;
    if (have) {
      load_state(S.in, p, noise, s);
      load_map(S.map, p, m);
      carried = S.carried_in[p];
    }
    PixelCounters c;
    unsigned long long samples = 0, err = 0;
    GlobalSink sink{S.ev, &S.counters[kCntEvents]};
    PixelProc<GlobalSink> proc{s, m, S.consts, p, sink, c};
    const FieldDev& f = S.field;
    for (int32_t w = a.w0; w < a.w1; ++w) {
      const int64_t t_w = t0 + static_cast<int64_t>(w) * kWindowNs;
      const BlobList list = warp_blob_list(f, have, x, y, t_w, t_w + kWindowNs, my_list);
      auto render = [&](uint32_t dt) { return field_eval(f, list, x, y, t_w + dt); };
      // Phase A: the walk, its first kStage samples after slot 0 staged.
      uint32_t n = 0;
      int level = 0;
      if (have) {
        level = field_level(f, list, x, y, t_w, a.r.l_min, a.r.l_max);
        uint32_t kk = 0;
        n = sample_pixel_window(a.r, level, carried, false, render, [&](uint32_t dt, float v) {
          if (kk < static_cast<uint32_t>(kStage)) {
            st_dt[warp][kk][lane] = dt;
            st_v[warp][kk][lane] = v;
          }
          ++kk;
        });
      }
      __syncwarp();
      const bool staged = have && n - 1 <= static_cast<uint32_t>(kStage);
      // The window's noise candidates of all lanes together; the rejected ones leave the pixel model.
      if (noise) {
        const StagedRun run{t_w, &st_dt[warp][0][lane], &st_v[warp][0][lane], static_cast<int>(n) - 1};
        noise_ahead(s, m, S.consts, p, staged, t_w, clamp_irr(carried, S.consts.irr_max), t_w + kWindowNs, run, c);
      }
      // Phase B, the warp together.
      WindowFeed feed{&proc, t_w, S.consts.irr_max, t_w, s.held, carried, 0.0f};
      if (staged) feed.start(carried);
      proc.defer = true;
      uint32_t next = 0;
      for (int64_t iter = 0;; ++iter) {
        if (staged && !proc.pending) {
          while (next + 1 < n) {
            feed(st_dt[warp][next][lane], st_v[warp][next][lane]);
            ++next;
            if (proc.pending) break;
          }
        }
        unsigned mask = __ballot_sync(full, staged && proc.pending);
        if (mask == 0u) break;
        // Every outcome moves the lane's search at least 1 ns on (an event re-arms it after the event's ns), so a
        // lane posts at most one search per ns of the window and per piece: 2^25 rounds cannot be reached.
        if (iter >= (int64_t{1} << 25)) {
          err |= kErrSearchBound;
          break;
        }
        bool found = false, on = false;
        int64_t th = 0;
        float xh = 0.0f;
        const SearchReq mine = request_of(proc);
        while (mask != 0u) {
          const int src = __ffs(mask) - 1;
          mask &= mask - 1u;
          const SearchReq r = shfl_req(mine, src);
          int64_t t_hit = 0;
          bool o = false;
          float xv = 0.0f;
          uint32_t lv = 0;
          const bool fnd = coop_search(r, S.consts, lane, t_hit, o, xv, &lv, &err);
          if (static_cast<int>(lane) == src) {
            c.leaves += lv;
            found = fnd;
            th = t_hit;
            on = o;
            xh = xv;
          }
        }
        if (staged && proc.pending) proc.resume_search(found, th, on, xh);
      }
      proc.defer = false;
      if (have) {
        if (staged) {
          samples += n;
          s.held = feed.prev_v;
          carried = feed.last_raw;
        } else {  // the window overflowed the stage: this lane alone, the walk again with the model fed inline
          WindowFeed alone{&proc, t_w, S.consts.irr_max, t_w, s.held, carried, 0.0f};
          alone.start(carried);
          sample_pixel_window(a.r, level, carried, false, render, alone);
          samples += n;
          s.held = alone.prev_v;
          carried = alone.last_raw;
        }
      }
      __syncwarp();
    }
    if (have) {
      store_state(S.out, p, noise, s);
      S.carried_out[p] = carried;
    }
    warp_add(&S.counters[kCntPieces], c.pieces);
    warp_add(&S.counters[kCntLeaves], c.leaves);
    warp_add(&S.counters[kCntSamples], samples);
    warp_add(&S.counters[kCntNoise], c.noise_candidates);
    warp_or(&S.counters[kCntErrors], err);
  }
}

// ---------------------------------------------------------------------------------------------
// The fused engine with the learned step proposal
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ void load_learned(const LearnedSoA& a, uint32_t p, uint32_t n, LearnedPixel& L) {
#pragma unroll
  for (int k = 0; k < 8; ++k) L.hx[k] = a.hx[static_cast<size_t>(k) * n + p];
  L.gaps = a.gaps[p];
  L.pv = a.pv[p];
  L.valid = a.valid[p];
}
__device__ __forceinline__ void store_learned(const LearnedSoA& a, uint32_t p, uint32_t n, const LearnedPixel& L) {
#pragma unroll
  for (int k = 0; k < 8; ++k) a.hx[static_cast<size_t>(k) * n + p] = L.hx[k];
  a.gaps[p] = L.gaps;
  a.pv[p] = L.pv;
  a.valid[p] = static_cast<uint8_t>(L.valid);
}

__device__ __forceinline__ void rec_push(const RecBuf& r, int64_t t, uint32_t pixel, float v) {
  cg::coalesced_group g = cg::coalesced_threads();
  unsigned long long base = 0;
  if (g.thread_rank() == 0) base = atomicAdd(r.count, static_cast<unsigned long long>(g.size()));
  base = g.shfl(base, 0);
  const unsigned long long i = base + g.thread_rank();
  if (i < r.capacity) r.data[i] = RecRow{t, pixel, v};
}

__global__ void learned_reset_kernel(LearnedSoA st, uint32_t n, const float* irr0) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  LearnedPixel L;
  learned_reset(L, irr0[p]);
  store_learned(st, p, n, L);
}

// Per window and warp: every lane with its walk inside the window writes its 16 features, the warp runs the MLP on
// the tensor cores (32 rows), and each lane takes its proposed step (judge, fallback and pixel model on its own);
// the loop ends when every lane has reached the window's end.
// At most 64 registers (8 blocks per SM; 128 uncapped held it to 4): on the 1280x720 held-out field 170.5 against
// 198.7 ms (186.3 at 6 blocks, 177.2 at 7), the proposals and the events unchanged.
__global__ void __launch_bounds__(128, 8) learned_engine_kernel(EngineArgs a, LearnedLaunch l) {
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const int64_t t0 = *a.t0;
  __shared__ MlpShared W;
  __shared__ __align__(16) uint16_t rows[4][32 * kSF];
  __shared__ float ys[4][32];
  __shared__ uint16_t lists[4][kMaxListed];
  mlp_load_shared(W, l.ops, l.params);
  uint16_t* my_list = lists[warp];
  uint16_t* my_rows = rows[warp];
  float* my_y = ys[warp];
  const bool rec_s = l.rec_samples.capacity > 0, rec_p = l.rec_steps.capacity > 0;
  for (;;) {
    uint32_t tile = 0;
    if (lane == 0) tile = atomicAdd(a.tile_counter, 1u);
    tile = __shfl_sync(0xffffffffu, tile, 0);
    if (tile >= a.total_tiles) break;
    int si = 0;
    while (si + 1 < a.n_sensors && a.sensors[si + 1].tile0 <= tile) ++si;
    const EngineSensor& S = a.sensors[si];
    const uint32_t local = tile - S.tile0;
    uint32_t x, y;
    tile_xy(local, S.tiles_x, a.tile_lw, lane, x, y);
    const bool have = x < S.width && y < S.height;
    const uint32_t np = S.width * S.height;
    const uint32_t p = have ? y * S.width + x : 0u;
    const uint32_t tag = (static_cast<uint32_t>(si) << 24) | p;
    const bool noise = S.consts.noise != 0;
    PixelRegs s;
    PixelMapRegs m;
    LearnedPixel L;
    float carried = 0.0f;
    if (have) {
      load_state(S.in, p, noise, s);
      load_map(S.map, p, m);
      load_learned(S.lin, p, np, L);
      carried = S.carried_in[p];
    }
    PixelCounters c;
    unsigned long long samples = 0;
    GlobalSink sink{S.ev, &S.counters[kCntEvents]};
    PixelProc<GlobalSink> proc{s, m, S.consts, p, sink, c};
    const FieldDev& f = S.field;
    for (int32_t w = a.w0; w < a.w1; ++w) {
      const int64_t t_w = t0 + static_cast<int64_t>(w) * kWindowNs;
      const BlobList list = warp_blob_list(f, have, x, y, t_w, t_w + kWindowNs, my_list);
      auto render = [&](uint32_t dt) { return field_eval(f, list, x, y, t_w + dt); };
      WindowFeed feed{&proc, t_w, S.consts.irr_max, t_w, s.held, carried, 0.0f};
      int s_floor = kWindowLog2;
      uint32_t cur = 0;
      float v_cur = carried, x_cur = 0.0f;
      if (have) {
        s_floor = kWindowLog2 - field_level(f, list, x, y, t_w, a.r.l_min, a.r.l_max);
        feed.start(carried);
        x_cur = log_f(carried);
      }
      auto emit = [&](uint32_t dt, float v) {
        feed(dt, v);
        if (rec_s) rec_push(l.rec_samples, t_w + dt, tag, v);
      };
      for (;;) {
        const bool act = have && cur < static_cast<uint32_t>(kWindowNs);
        if (!__any_sync(0xffffffffu, act)) break;
        float feat[16];
        if (act) {
          step_features(L.hx, L.gaps, x_cur, feat);
        } else {
#pragma unroll
          for (int k = 0; k < 16; ++k) feat[k] = 0.0f;
        }
        uint32_t packed[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) packed[k] = pack2(feat[2 * k], feat[2 * k + 1]);
        uint4* dst = reinterpret_cast<uint4*>(my_rows + lane * kSF);
        dst[0] = make_uint4(packed[0], packed[1], packed[2], packed[3]);
        dst[1] = make_uint4(packed[4], packed[5], packed[6], packed[7]);
        __syncwarp();
        mlp_forward_warp(W, my_rows, my_y);
        if (act) {
          const int sl = proposal_log2(my_y[lane], l.margin, l.sh, s_floor, cur);
          if (rec_p) rec_push(l.rec_steps, t_w + cur, tag, static_cast<float>(sl));
          float v_end = 0.0f;
          samples += learned_step(a.r, cur, sl, v_cur, x_cur, L, v_end, render, emit);
          cur += 1u << sl;
          v_cur = v_end;
          x_cur = log_f(v_end);
        }
        __syncwarp();
      }
      if (have) {
        ++samples;  // the carried slot, as in the plain engine's count
        s.held = feed.prev_v;
        carried = feed.last_raw;
      }
      __syncwarp();
    }
    if (have) {
      store_state(S.out, p, noise, s);
      store_learned(S.lout, p, np, L);
      S.carried_out[p] = carried;
    }
    warp_add(&S.counters[kCntPieces], c.pieces);
    warp_add(&S.counters[kCntLeaves], c.leaves);
    warp_add(&S.counters[kCntSamples], samples);
    warp_add(&S.counters[kCntNoise], c.noise_candidates);
  }
}

// MidpointTest.eta (sampling.h:36-53): per group in order, dev = |(a + b) * -0.5 + m|, num += m_max dev,
// den += m_min min(a, m, b), the mediant max(dev / low) when some group is modulated; eta = num / den.
struct MidArgs {
  float tol, dark;
  int32_t g;
  float m_min[8], m_max[8];
  bool mediant;
};

__global__ void midpoint_eta_kernel(MidArgs p, const float* ea, const float* em, const float* eb, uint32_t n,
                                    float* eta, uint8_t* exceeds) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float num = 0.0f, den = p.dark, mediant = 0.0f;
  for (int32_t k = 0; k < p.g; ++k) {
    const float a = ea[static_cast<size_t>(i) * p.g + k], m = em[static_cast<size_t>(i) * p.g + k];
    const float b = eb[static_cast<size_t>(i) * p.g + k];
    const float dev = fabs_f((a + b) * -0.5f + m);
    const float low = np_min(np_min(a, m), b);
    num = num + p.m_max[k] * dev;
    den = den + p.m_min[k] * low;
    if (p.mediant) {
      const float q = dev == 0.0f ? 0.0f : dev / low;
      mediant = (mediant >= q || mediant != mediant) ? mediant : q;  // NumPy maximum
    }
  }
  float e = num / den;
  if (p.mediant) e = np_min(e, mediant);
  eta[i] = e;
  exceeds[i] = e > p.tol ? 1 : 0;
}

}  // namespace

void launch_midpoint_eta(float tol, float dark, int32_t g, const float* m_min, const float* m_max, const float* ea,
                         const float* em, const float* eb, uint32_t n, float* eta, uint8_t* exceeds,
                         cudaStream_t stream) {
  MidArgs p{};
  p.tol = tol;
  p.dark = dark;
  p.g = g;
  p.mediant = false;
  for (int32_t k = 0; k < g; ++k) {
    p.m_min[k] = m_min[k];
    p.m_max[k] = m_max[k];
    p.mediant = p.mediant || m_min[k] != m_max[k];
  }
  if (n == 0) return;
  midpoint_eta_kernel<<<(n + 255) / 256, 256, 0, stream>>>(p, ea, em, eb, n, eta, exceeds);
}

void launch_init_counted(const SensorConsts& k, const CascadeConsts& cc, const NoiseTableDev& tab, const MapSoA& map,
                         StateSoA st, uint32_t n_pixels, int64_t t0, const float* irr0, unsigned long long* counters,
                         cudaStream_t stream) {
  const int block = 128;
  const unsigned grid = (n_pixels + block - 1) / block;
  init_kernel<<<grid, block, 0, stream>>>(k, cc, tab, map, st, n_pixels, t0, irr0, nullptr, counters);
}

void launch_scatter_rows(const uint32_t* pixel, uint32_t n, int32_t* row_of, uint32_t n_pixels,
                         unsigned long long* counters, cudaStream_t stream) {
  if (n == 0) return;
  scatter_rows_kernel<<<(n + 255) / 256, 256, 0, stream>>>(pixel, n, row_of, n_pixels, counters);
}

void launch_advance_runs(const SensorConsts& k, const CascadeConsts& cc, const NoiseTableDev& tab, const MapSoA& map,
                         StateSoA in, StateSoA out, uint32_t n_pixels, const uint32_t* pixel_ids, const int32_t* row_of,
                         const int64_t* row_start, const int32_t* row_count, const int64_t* t, const float* irr,
                         uint64_t n_samples, int64_t t_state, int64_t t_end, EventBuf ev, unsigned long long* counters,
                         int block, cudaStream_t stream) {
  RunArgs a{k, cc, tab, map, in, out, n_pixels, pixel_ids, row_of, row_start, row_count, t, irr, n_samples, t_state,
            t_end, ev, counters};
  if (block <= 0) block = 128;
  const unsigned grid = (n_pixels + block - 1) / block;
  if (k.cascade && tab.data != nullptr) advance_runs_lattice_kernel<<<grid, block, 0, stream>>>(a);
  else if (k.cascade) advance_runs_cascade_kernel<<<grid, block, 0, stream>>>(a);
  else advance_runs_kernel<<<grid, block, 0, stream>>>(a);
}

void launch_advance_rows(const SensorConsts& k, const MapSoA& map, StateSoA in, StateSoA out, uint32_t n_pixels,
                         const uint32_t* pixel, uint32_t n_rows, const int64_t* row_start, const int32_t* row_count,
                         const int64_t* t, const float* irr, uint64_t n_samples, int64_t t_state, int64_t t_end,
                         int32_t long_row, uint32_t* listed, EventBuf ev, unsigned long long* counters,
                         const SensorConsts* k_dev, void* rest, unsigned int* rest_count, int rest_blocks,
                         bool first_call, cudaStream_t stream) {
  RowsArgs a{k, map, in, out, n_pixels, pixel, n_rows, row_start, row_count, t, irr, n_samples, t_state, t_end,
             long_row, listed, ev, counters, k_dev};
  if (n_rows > 0) {
    const unsigned grid = (n_rows + 32 * kRowsWarps - 1) / (32 * kRowsWarps);
    if (rest != nullptr) {
      const RowRestList rl{static_cast<RowRest*>(rest), rest_count, n_rows};
      if (first_call) advance_rows_split_kernel<true><<<grid, 32 * kRowsWarps, 0, stream>>>(a, rl);
      else advance_rows_split_kernel<false><<<grid, 32 * kRowsWarps, 0, stream>>>(a, rl);
      advance_rows_rest_kernel<<<rest_blocks, 128, 0, stream>>>(a, rl);
    } else {
      advance_rows_kernel<<<grid, 32 * kRowsWarps, 0, stream>>>(a);
    }
  }
  if (n_rows < n_pixels) advance_unlisted_kernel<<<(n_pixels + 127) / 128, 128, 0, stream>>>(a);
}

void launch_sample_window(const FieldDev& f, const SamplerRules& r, int64_t t_w, const uint32_t* pixel,
                          const uint8_t* level, uint32_t n, const float* carried_in, const uint64_t* sig_in,
                          uint32_t* counts, const int64_t* offsets, int64_t* t_out, float* irr_out,
                          float* carried_out, uint64_t* sig_out, int pass, cudaStream_t stream) {
  if (n == 0) return;
  WindowArgs a{f, r, t_w, pixel, level, n, carried_in, sig_in, counts, offsets, t_out, irr_out, carried_out, sig_out};
  const unsigned grid = (n + 127) / 128;
  if (pass == 0) sample_window_kernel<0><<<grid, 128, 0, stream>>>(a);
  else sample_window_kernel<1><<<grid, 128, 0, stream>>>(a);
}

void launch_sample_window_staged(const FieldDev& f, const SamplerRules& r, int64_t t_w, const uint32_t* pixel,
                                 const uint8_t* level, uint32_t n, const float* carried_in, const uint64_t* sig_in,
                                 uint32_t* counts, const int64_t* offsets, int64_t* t_out, float* irr_out,
                                 float* carried_out, uint64_t* sig_out, uint32_t* stage_dt, float* stage_v,
                                 uint32_t* stage_at, unsigned int* stage_used, uint32_t stage_cap, float* stage_carried,
                                 uint64_t* stage_sig, uint32_t n_field, int max_level, unsigned long long* err,
                                 int pass, cudaStream_t stream) {
  if (n == 0) return;
  const StageArgs a{WindowArgs{f, r, t_w, pixel, level, n, carried_in, sig_in, counts, offsets, t_out, irr_out,
                               carried_out, sig_out},
                    stage_dt, stage_v, stage_at, stage_used, stage_cap, stage_carried, stage_sig, n_field, max_level,
                    err};
  const unsigned grid = (n + 127) / 128;
  if (pass == 0) sample_window_stage_kernel<<<grid, 128, 0, stream>>>(a);
  else sample_window_place_kernel<<<grid, 128, 0, stream>>>(a);
}

size_t scan_scratch_words(uint32_t n) { return (n + kScanBlock - 1) / kScanBlock + 1; }

void launch_scan(const uint32_t* counts, uint32_t n, int64_t* offsets, int64_t* scratch, cudaStream_t stream) {
  const uint32_t blocks = n == 0 ? 1 : (n + kScanBlock - 1) / kScanBlock;
  scan_blocks_kernel<<<blocks, kScanBlock, 0, stream>>>(counts, n, offsets, scratch);
  scan_sums_kernel<<<1, kScanBlock, 0, stream>>>(scratch, blocks, offsets, n);
  scan_fix_kernel<<<blocks, kScanBlock, 0, stream>>>(offsets, n, scratch);
}

void launch_levels(const FieldDev& f, int64_t t_w, int32_t l_min, int32_t l_max, uint32_t n_pixels, uint8_t* level,
                   cudaStream_t stream) {
  levels_kernel<<<(n_pixels + 127) / 128, 128, 0, stream>>>(f, t_w, l_min, l_max, n_pixels, level);
}

void launch_field_frame(const FieldDev& f, int64_t t, uint32_t n_pixels, float* out, cudaStream_t stream) {
  field_frame_kernel<<<(n_pixels + 255) / 256, 256, 0, stream>>>(f, t, n_pixels, out);
}

void launch_engine(const EngineSensor* sensors_dev, int n_sensors, uint32_t total_tiles, const int64_t* t0,
                   int32_t w0, int32_t w1, const SamplerRules& r, unsigned int* tile_counter, int blocks,
                   int warps_per_block, int stage, int tile_lw, int cascade, cudaStream_t stream) {
  EngineArgs a{sensors_dev, n_sensors, total_tiles, t0, w0, w1, r, tile_counter, static_cast<uint32_t>(tile_lw)};
  if (cascade == 2 && stage != 0) engine_lattice_kernel_staged<<<blocks, warps_per_block * 32, 0, stream>>>(a);
  else if (cascade == 2) engine_lattice_kernel<<<blocks, warps_per_block * 32, 0, stream>>>(a);
  else if (cascade == 1) engine_cascade_kernel<<<blocks, warps_per_block * 32, 0, stream>>>(a);
  else if (stage == 64) engine_kernel_coop<<<blocks, warps_per_block * 32, 0, stream>>>(a);
  else if (stage == 16) engine_kernel_staged<16><<<blocks, warps_per_block * 32, 0, stream>>>(a);
  else if (stage == 32) engine_kernel_staged<32><<<blocks, warps_per_block * 32, 0, stream>>>(a);
  else engine_kernel<<<blocks, warps_per_block * 32, 0, stream>>>(a);
}

void launch_engine_split(const EngineSensor* sensors_dev, int n_sensors, uint32_t total_tiles, const int64_t* t0,
                         int32_t w, const SamplerRules& r, unsigned int* tile_counter, void* rest, unsigned int* rest_count,
                         unsigned int rest_capacity, int blocks, int warps_per_block, int tile_lw, int rest_blocks,
                         cudaStream_t stream) {
  const EngineArgs a{sensors_dev, n_sensors, total_tiles, t0, w, w + 1, r, tile_counter, static_cast<uint32_t>(tile_lw)};
  const RestList rl{static_cast<unsigned char*>(rest), rest_count, rest_capacity};
  if (w == 0) engine_window_kernel<true><<<blocks, warps_per_block * 32, 0, stream>>>(a, rl);
  else engine_window_kernel<false><<<blocks, warps_per_block * 32, 0, stream>>>(a, rl);
  engine_rest_kernel<<<rest_blocks, 128, 0, stream>>>(a, rl);
}

size_t rest_record_bytes() { return kRestRecordBytes; }
size_t row_rest_bytes() { return sizeof(RowRest); }
int rows_rest_blocks_per_sm() {
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, advance_rows_rest_kernel, 128, 0);
  return n;
}

int engine_rest_blocks_per_sm() {
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, engine_rest_kernel, 128, 0);
  return n;
}

int engine_max_blocks_per_sm(int warps_per_block, int stage, int cascade) {
  int n = 0;
  if (stage == kStageSplit) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, engine_window_kernel<false>, warps_per_block * 32, 0);
    return n;
  }
  if (cascade == 2 && stage != 0) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, engine_lattice_kernel_staged, warps_per_block * 32, 0);
  } else if (cascade == 2) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, engine_lattice_kernel, warps_per_block * 32, 0);
  } else if (cascade == 1) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, engine_cascade_kernel, warps_per_block * 32, 0);
  } else if (stage == 64) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, engine_kernel_coop, warps_per_block * 32, 0);
  } else if (stage == 16) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, engine_kernel_staged<16>, warps_per_block * 32, 0);
  } else if (stage == 32) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, engine_kernel_staged<32>, warps_per_block * 32, 0);
  } else {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, engine_kernel, warps_per_block * 32, 0);
  }
  return n;
}

}  // namespace bs

namespace bs {

void launch_learned_engine(const EngineSensor* sensors_dev, int n_sensors, uint32_t total_tiles, const int64_t* t0,
                           int32_t w0, int32_t w1, const SamplerRules& r, const LearnedLaunch& l,
                           unsigned int* tile_counter, int blocks, int warps_per_block, int tile_lw,
                           cudaStream_t stream) {
  EngineArgs a{sensors_dev, n_sensors, total_tiles, t0, w0, w1, r, tile_counter, static_cast<uint32_t>(tile_lw)};
  (void)warps_per_block;  // 4 warps: the shared tiles are sized for them
  learned_engine_kernel<<<blocks, 128, 0, stream>>>(a, l);
}

int learned_engine_max_blocks_per_sm(int warps_per_block) {
  (void)warps_per_block;
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, learned_engine_kernel, 128, 0);
  return n;
}

void launch_learned_reset(LearnedSoA st, uint32_t n, const float* irr0, cudaStream_t stream) {
  if (n == 0) return;
  learned_reset_kernel<<<(n + 255) / 256, 256, 0, stream>>>(st, n, irr0);
}

}  // namespace bs
