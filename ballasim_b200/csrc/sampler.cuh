// BallaSim's window sampler (src/engine/sampling.h:355-839, src/engine/window_impl.h:461-713) restated per
// pixel: the dyadic lattice of 2^level + 1 slots (slot 0 the carried sample at t_w, never rendered), the round-0
// flags of each lattice interval from its two covering triples, then refinement of the selected intervals while
// the eta_L midpoint test exceeds the tolerance, down to min_split and for at most max_refine_levels rounds.
//
// The reference refines breadth-first over a batch of pixels, one render call per round; a half's flag depends
// only on its own triple (lo, mid, hi) and the round it is in, so the same set of samples comes out of a
// depth-first walk per pixel. Walking in order emits the samples in time order, which is the order the runs
// (PoolKeys / stable sort / ScatterSlots, sampling.h:764-839) put them in: the generator feeds a consumer
// directly, either a CSR writer or the pixel model on the same thread.
#pragma once

#include "bs_math.cuh"

namespace bs {

struct SamplerRules {
  float tol, dark;           // eta_L > tol flags (MidpointTest(tol, dark, [1], [1]))
  int32_t midpoint;          // the midpoint test is on
  int32_t refine_signature;  // signature flips flag (analytic samples have signature 0)
  int32_t max_refine_levels;
  uint32_t min_split;        // 2 min_dt_ns
  int32_t l_min, l_max;      // level rule clamp (fused engine)
};

// NumPy's float minimum: a NaN operand propagates (sampling.h:26).
BS_HD float np_min(float a, float b) { return (a <= b || a != a) ? a : b; }

// eta_L of one light group with m_min = m_max = 1 (midpoint_eta, sampling.h:36-53, in its operation order).
BS_HD float midpoint_eta1(float dark, float a, float m, float b) {
  float num = 0.0f, den = dark;
  const float dev = fabs_f((a + b) * -0.5f + m);
  const float low = np_min(np_min(a, m), b);
  num = num + 1.0f * dev;
  den = den + 1.0f * low;
  return num / den;
}

BS_HD bool exceeds(const SamplerRules& r, float a, float m, float b) {
  return r.midpoint != 0 && midpoint_eta1(r.dark, a, m, b) > r.tol;
}

// Walks one pixel's window: render(dt) -> irradiance; emit(dt, v) for every sample after slot 0 in time order (one
// call site). carried: the slot-0 value (the caller's to take); carried_flip: its signature differs from the
// rendered ones (0). Returns the number of samples, slot 0 included.
template <class Render, class Emit>
BS_HD uint32_t sample_pixel_window(const SamplerRules& r, int level, float carried, bool carried_flip,
                                   Render&& render, Emit&& emit) {
  struct Frame {
    uint32_t lo, hi, g;
    float vlo, vhi, vg;
    int32_t depth;
    uint32_t phase;  // 0: mid not yet rendered; 1: left half done
    bool flip, bad;
  };
  // A selected interval halves at most 22 times above min_split >= 2 (2^23 ns down to 2 ns), and the rules clamp
  // max_refine_levels to 23, so the walk never holds more than kMaxDepth frames.
  constexpr int kMaxDepth = 24;
  Frame st[kMaxDepth];
  const uint32_t count = (1u << level) + 1u, step = 1u << (kWindowLog2 - level);
  uint32_t n = 1;
  // Sliding lattice values v[j - 2], v[j - 1], v[j], v[j + 1].
  float vm2 = 0.0f, vm1 = carried, v0 = render(step), vp1 = count > 2 ? render(2 * step) : 0.0f;
  uint32_t j = 1;
  bool opened = false;  // interval (j - 1, j) flagged and its refinement started
  int sp = 0;
  while (j < count) {
    uint32_t dt;
    float v;
    if (sp > 0) {
      Frame& f = st[sp - 1];
      if (f.phase == 0u) {
        f.g = (f.lo + f.hi) >> 1;
        f.vg = render(f.g);
        // HalfFlags (sampling.h:638-678): the triple (lo, mid, hi) flags both halves.
        f.bad = exceeds(r, f.vlo, f.vg, f.vhi);
        f.phase = 1u;
        if ((f.flip || f.bad) && f.g - f.lo >= r.min_split && f.depth + 1 < r.max_refine_levels &&
            sp < kMaxDepth) {
          st[sp] = Frame{f.lo, f.g, 0u, f.vlo, f.vg, 0.0f, f.depth + 1, 0u, f.flip, false};
          ++sp;
        }
        continue;
      }
      dt = f.g;
      v = f.vg;
      if (f.bad && f.hi - f.g >= r.min_split && f.depth + 1 < r.max_refine_levels) {
        f = Frame{f.g, f.hi, 0u, f.vg, f.vhi, 0.0f, f.depth + 1, 0u, false, false};
      } else {
        --sp;
      }
    } else if (!opened) {
      // Round0Flags (sampling.h:490-523) of interval (j - 1, j): triples (j - 1, j, j + 1) and (j - 2, j - 1, j).
      opened = true;
      const bool flip = r.refine_signature != 0 && j == 1 && carried_flip;
      const bool m = (j + 1 < count && exceeds(r, vm1, v0, vp1)) || (j >= 2 && exceeds(r, vm2, vm1, v0));
      if ((flip || m) && step >= r.min_split && r.max_refine_levels > 0) {
        st[0] = Frame{(j - 1) * step, j * step, 0u, vm1, v0, 0.0f, 0, 0u, flip, false};
        sp = 1;
      }
      continue;
    } else {
      dt = j * step;
      v = v0;
      opened = false;
      vm2 = vm1;
      vm1 = v0;
      v0 = vp1;
      if (j + 2 < count) vp1 = render((j + 2) * step);
      ++j;
    }
    emit(dt, v);
    ++n;
  }
  return n;
}

}  // namespace bs
