// The learned-proposal sampler of one pixel and the training walk over the plain sampler's runs (this project's
// own method; no reference counterpart). Steps are powers of two, 2^s ns with s in [log2 min_dt, 23], each starting
// on its own lattice inside the window, so every sample lies on the plain sampler's dyadic lattice of the window
// (src/engine/sampling.h:355-414) and a step never crosses a window boundary.
//
// Judge and fallback are the plain rules (src/engine/sampling.h:26-69, 638-678):
//  - a step of the same length as the previous one is judged by the triple (previous point, current point, step
//    end), whose middle is its midpoint: no extra render (the plain round-0 triple, sampling.h:490-523);
//  - any other step renders its midpoint and is judged by (start, midpoint, end);
//  - a step shorter than min_split (2 min_dt) cannot be split and is taken as it is, like the plain lattice;
//  - a rejected step is refined exactly as the plain sampler refines a selected interval: each half whose triple
//    exceeds is split again, depth-first, down to min_split and for at most max_refine_levels levels.
// Every rendered point is a sample.
#pragma once

#include "mlp.cuh"
#include "sampler.cuh"

namespace bs {

// A pixel's walk state: the last 8 walk points before the current one.
struct LearnedPixel {
  float hx[8];      // log irradiance, newest first
  uint64_t gaps;    // byte k: log2 of the gap after the k-th previous point (byte 0 the newest)
  float pv;         // irradiance at the previous walk point
  uint32_t valid;   // a previous walk point exists (the history starts as a flat virtual one)
};

// The history at the start of a run: 8 virtual points one window apart with the initial value.
BS_HD void learned_reset(LearnedPixel& L, float v0) {
  const float x = log_f(v0);
  for (int k = 0; k < 8; ++k) L.hx[k] = x;
  L.gaps = 0x1717171717171717ull;  // 23
  L.pv = v0;
  L.valid = 0u;
}

BS_HD void learned_push(LearnedPixel& L, float x_cur, float v_cur, int s) {
  for (int k = 7; k > 0; --k) L.hx[k] = L.hx[k - 1];
  L.hx[0] = x_cur;
  L.gaps = (L.gaps << 8) | static_cast<uint64_t>(s);
  L.pv = v_cur;
  L.valid = 1u;
}

// The plain refinement of an interval (lo, hi) whose midpoint vm is rendered and whose triple decided `bad`:
// emits every sample strictly inside (lo, hi) in time order; returns their number.
template <class Render, class Emit>
BS_HD uint32_t refine_interval(const SamplerRules& r, uint32_t lo, uint32_t hi, float vlo, float vm, float vhi,
                               Render&& render, Emit&& emit) {
  struct Frame {
    uint32_t lo, hi;
    float vlo, vg, vhi;
    int32_t depth;
    uint32_t phase;  // 0: mid not rendered; 1: rendered, left not started; 2: left done
    bool bad;
  };
  constexpr int kMaxDepth = 24;
  Frame st[kMaxDepth];
  int sp = 1;
  st[0] = Frame{lo, hi, vlo, vm, vhi, 0, 1u, false};
  uint32_t n = 0;
  while (sp > 0) {
    Frame& f = st[sp - 1];
    const uint32_t g = (f.lo + f.hi) >> 1;
    if (f.phase == 0u) {
      f.vg = render(g);
      f.phase = 1u;
    }
    if (f.phase == 1u) {
      f.phase = 2u;
      f.bad = exceeds(r, f.vlo, f.vg, f.vhi);
      if (f.bad && g - f.lo >= r.min_split && f.depth + 1 < r.max_refine_levels && sp < kMaxDepth) {
        st[sp] = Frame{f.lo, g, f.vlo, 0.0f, f.vg, f.depth + 1, 0u, false};
        ++sp;
        continue;
      }
    }
    emit(g, f.vg);
    ++n;
    if (f.bad && f.hi - g >= r.min_split && f.depth + 1 < r.max_refine_levels) {
      f = Frame{g, f.hi, f.vg, 0.0f, f.vhi, f.depth + 1, 0u, false};
    } else {
      --sp;
    }
  }
  return n;
}

// One step of 2^s ns from walk point cur (ns after the window start) with value v_cur and log x_cur: emits the
// step's samples (cur, cur + 2^s] in time order, moves the history on and returns the sample count; v_end gets
// the value at the step's end.
template <class Render, class Emit>
BS_HD uint32_t learned_step(const SamplerRules& r, uint32_t cur, int s, float v_cur, float x_cur, LearnedPixel& L,
                            float& v_end, Render&& render, Emit&& emit) {
  const uint32_t dt = 1u << s, hi = cur + dt;
  const float vb = render(hi);
  uint32_t n = 0;
  if (dt >= r.min_split &&
      !(L.valid != 0u && static_cast<int>(L.gaps & 0xffu) == s && !exceeds(r, L.pv, v_cur, vb))) {
    const float vm = render(cur + (dt >> 1));
    n += refine_interval(r, cur, hi, v_cur, vm, vb, render, emit);
  }
  emit(hi, vb);
  ++n;
  learned_push(L, x_cur, v_cur, s);
  v_end = vb;
  return n;
}

// ---- training pairs from the plain sampler's runs ----

// The target at walk point cur of a window's plain run (times ts[i] relative to the window start, values vs[i],
// n samples, ts[0] = 0 and ts[n - 1] = 2^23): the largest s >= s_floor such that every step 2^s' (s_floor < s' <= s)
// from cur is aligned and its chord stays within eps of the run's log irradiance at every run sample inside it.
// The walk points are multiples of 2^s_floor, i.e. run samples; i_cur is cur's index in the run.
template <class Run>
BS_HD int walk_target(const Run& run, int n, int i_cur, uint32_t cur, int s_floor, float eps) {
  int best = s_floor;
  const float va = run.v(i_cur);
  int j = i_cur;
  for (int s = s_floor + 1; s <= kWindowLog2; ++s) {
    if ((cur & ((1u << s) - 1u)) != 0u) break;
    const uint32_t hi = cur + (1u << s);
    while (j < n - 1 && run.t(j) < hi) ++j;
    if (run.t(j) != hi) break;  // not on the run (cannot happen for s >= s_floor)
    const float vb = run.v(j);
    const float step = static_cast<float>(1u << s);
    bool ok = true;
    for (int k = i_cur + 1; k < j; ++k) {
      const float lin = va + (vb - va) * (static_cast<float>(run.t(k) - cur) / step);
      if (!(fabs_f(log_f(run.v(k)) - log_f(lin)) <= eps)) {
        ok = false;
        break;
      }
    }
    if (!ok) break;
    best = s;
  }
  return best;
}

// The walk's perturbation: the step taken is the target lowered by 0 (half the time), 1, 2 or 3 octaves, never
// below the plain lattice, so that the pairs also hold the shorter histories a proposal meets.
BS_HD int walk_drop(uint64_t seed, uint32_t pixel, int32_t window, uint32_t step_no) {
  const U4 u = draw(seed, kPurposeWalk, 0u, pixel, (static_cast<uint64_t>(window) << 11) | step_no);
  const uint32_t t = u.v[0] & 7u;
  return t < 4u ? 0 : (t < 6u ? 1 : static_cast<int>(t) - 4);
}

}  // namespace bs
