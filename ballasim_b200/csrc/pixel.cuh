// The instantaneous pixel model of BallaSim (src/sensor/pixel.h: advance_instant :876-907, instant_search
// :1886-1916, instant_may_fire :1853-1876, fire :1534-1588, init :792-818), restated for the device as a
// streaming processor: the pixel's state lives in registers and is fed one linear sample segment at a time,
// in time order, from wherever the samples come from (a CSR run in HBM, or the sampler on the same thread).
//
// Input model: one constant light group. Between consecutive samples (t0, v0), (t1, v1) the irradiance is
// v0 + (v1 - v0) ((t - t0) / (t1 - t0)) (fp32, that operation order) and after the last sample it is held;
// the photocurrent is I = I_dk + s v (s = illuminance_scale x gain); x(t) = ln(I / i_scale).
// Comparator: Delta(t) = (x - s3_ref) + (0 - n3_ref) + (leak (t - t_ref) 1e-9 + dr_ref) fires at the first
// integer ns of each piece where Delta >= theta_on or <= -theta_off, found by the reference's time-ordered
// depth-first bisection, whose nodes are pruned here by an exact (margin-free) bound instead of the reference's
// margins: the same first crossing, far fewer nodes where Delta lingers near a level; pieces never cross a
// multiple of 2^23 ns.
//
// Noise (this project's, no reference counterpart): two Poisson chains of candidate times per pixel, keyed by
// (pixel, candidate number) in Philox streams 0x0080 (shot) and 0x0081 (background activity). Candidate n's
// gap from n - 1 is ceil(-ln(u0) / lambda_max 1e9) ns (>= 1), it is accepted when u1 < lambda(t) / lambda_max
// and u2's low bit is its polarity (u_i = open uniform of word i of draw n). Shot noise: lambda = r sqrt(100 fA / I)
// with lambda_max = r sqrt(100 fA / I_dk); background activity: lambda = lambda_max = the pixel's drawn rate. An
// accepted candidate outside the refractory time fires as a comparator event of its polarity (label NOISE, the
// pixel's reset applied); one inside it (or during an ideal reset's dead time) is dropped.
#pragma once

#include "bs_math.cuh"

namespace bs {

// Device copy of the reference's RawEvent (src/sensor/pixel.h:123-135), 32 bytes.
struct RawEvent {
  uint32_t pixel;
  uint8_t polarity;
  uint8_t label;
  uint16_t flags;
  int64_t t_cross;
  float ds, dn, dl, l_first;
};
static_assert(sizeof(RawEvent) == 32, "RawEvent is 32 bytes");

// Per-model constants of the kernel (KernelConstants<float>, src/sensor/pixel.h:215-252, on this path).
struct SensorConsts {
  float irr_max;
  float eps_ci;
  float label_cut;
  int32_t ideal_reset;
  int64_t refractory_ns;
  int32_t noise;          // shot or background-activity noise on
  int32_t cascade;        // the cascade photoreceptor (cascade.cuh) instead of the instantaneous response
  double shot_rate_hz;    // r of lambda = r sqrt(100 fA / I); 0: no shot noise
  uint64_t seed;
  uint32_t camera;
};

// The state of one pixel between calls (SoA in HBM; see SensorDev).
struct PixelRegs {
  int64_t t_ref, t_search, blind_until;
  float s3_ref, n3_ref, dr_ref, i_scale, held;
  uint32_t flags;
  int64_t t_shot, t_ba;
  uint32_t n_shot, n_ba;
};

// The pixel's frozen map, fp32 as the kernel takes it (PixelMap's fp64 values cast once).
struct PixelMapRegs {
  float theta_on, theta_off, leak, dark, scale;
  double ba_rate_hz;
  double shot_max_hz;
};

struct PixelCounters {
  uint32_t pieces = 0, leaves = 0, noise_candidates = 0;
};

BS_HOT float clamp_irr(float v, float v_max) { return v >= 0.0f ? (v <= v_max ? v : v_max) : 0.0f; }
BS_HOT float since_ref(int64_t t, int64_t t_ref) { return static_cast<float>(static_cast<double>(t - t_ref) * 1e-9); }

BS_HD uint8_t split_label(float ds, float dl, float D, float cut) {
  const float a_s = ds / D, a_l = dl / D;
  if (a_s >= cut && a_s >= a_l) return kLabelSignal;
  if (a_l >= cut && a_l > a_s) return kLabelLeak;
  return kLabelNoise;
}
BS_HD uint8_t first_label(bool on, float ds, float dn, float l, float cut) {
  const float D = ds + dn + l;
  return (on ? D > 0.0f : D < 0.0f) ? split_label(ds, l, D, cut) : kLabelNoise;
}

// The candidate after one at t whose successor's draw is w (word 0 its gap): kForever without a rate.
BS_HD int64_t noise_after(const U4& w, int64_t t, double rate_hz) {
  if (!(rate_hz > 0.0)) return kForever;
  const double dt = -log_d(open_uniform_d(w.v[0])) / rate_hz * 1e9;
  const double step = ceil(dt);
  if (!(step < 9.0e18)) return kForever;
  return t + static_cast<int64_t>(step < 1.0 ? 1.0 : step);
}

// The next candidate of a noise chain after t (kForever without a rate): candidate n's draw gives its gap.
static BS_COLD int64_t noise_next(uint64_t seed, uint32_t purpose, uint32_t camera, uint32_t pixel, uint32_t n,
                                  int64_t t, double rate_hz) {
  if (!(rate_hz > 0.0)) return kForever;
  return noise_after(draw(seed, purpose, camera, pixel, n), t, rate_hz);
}

// One linear sample segment: [t0, t1) between two samples, or held from t0 on (t1 = kForever).
struct Segment {
  int64_t t0, t1;
  float v0, v1;
};

// kFlat: the rare paths (fire, the search, the noise candidates, piece) inline into the caller, for a caller that is
// itself out of line (cold_segment): there the state can stay in registers. Otherwise each is one out-of-line copy.
// The input at t on segment g: linear between its samples in that operation order, held after the last one.
BS_HOT float segment_value(const Segment& g, int64_t t) {
  if (g.t1 == kForever) return g.v0;
  const float f = static_cast<float>(t - g.t0) / static_cast<float>(g.t1 - g.t0);
  return g.v0 + (g.v1 - g.v0) * f;
}

template <class Sink, bool kFlat = false>
struct PixelProc {
  PixelRegs& s;
  const PixelMapRegs& m;
  const SensorConsts& k;
  uint32_t pixel;  // the frame's pixel id (events, noise keys)
  Sink& sink;
  PixelCounters& c;
  // The deferred search (the warp-cooperative engine): with defer set, piece() records the search it needs
  // (pending; the piece g, [p_t, p_e) and the search's [p_lo, p_stop)) and returns; resume_search applies the
  // outcome as piece() would have and resumes the piece.
  bool defer = false;
  bool pending = false;
  Segment pg{};
  int64_t p_t = 0, p_e = 0, p_lo = 0, p_stop = 0;

  BS_HOT float value(const Segment& g, int64_t t) const { return segment_value(g, t); }
  BS_HOT float current(const Segment& g, int64_t t) const { return m.dark + m.scale * value(g, t); }
  BS_HOT float log_ratio(float I) const { return log_f(I / s.i_scale); }

  BS_HOT float delta(int64_t t, float x) const {
    const float ds = x - s.s3_ref;
    const float dn = 0.0f - s.n3_ref;
    const float dl = m.leak * since_ref(t, s.t_ref) + s.dr_ref;
    return ds + dn + dl;
  }

  BS_HOT void set_reference(int64_t t, float s3, float offset) {
    s.t_ref = t;
    s.s3_ref = s3;
    s.n3_ref = 0.0f;
    s.dr_ref = offset;
  }

  // The event and the reset (pixel.h:1534-1588); label_override >= 0 labels a noise event.
  BS_HD void fire(int64_t t, bool on, float x, int label_override) {
    if constexpr (kFlat) {
      fire_body(t, on, x, label_override);
    } else {
      fire_out(t, on, x, label_override);
    }
  }
  BS_COLD void fire_out(int64_t t, bool on, float x, int label_override) { fire_body(t, on, x, label_override); }
  BS_HD void fire_body(int64_t t, bool on, float x, int label_override) {
    const float ds = x - s.s3_ref;
    const float dn = 0.0f - s.n3_ref;
    const float l = m.leak * since_ref(t, s.t_ref);
    const float dl = l + s.dr_ref;
    const float D = ds + dn + dl;
    const bool first = (s.flags & kFlagFirstAfterInit) != 0u;
    uint8_t label = first ? first_label(on, ds, dn, l, k.label_cut) : split_label(ds, dl, D, k.label_cut);
    if (label_override >= 0) label = static_cast<uint8_t>(label_override);
    RawEvent ev;
    ev.pixel = pixel;
    ev.polarity = on ? 1 : 0;
    ev.label = label;
    ev.flags = static_cast<uint16_t>(s.flags);
    ev.t_cross = t;
    ev.ds = ds;
    ev.dn = dn;
    ev.dl = dl;
    ev.l_first = first ? l : 0.0f;
    sink.push(ev);
    s.flags = 0;
    if (k.ideal_reset) {
      set_reference(t, x, D - (on ? m.theta_on : -m.theta_off));
      s.t_search = t + 1 + k.refractory_ns;
    } else if (k.refractory_ns == 0) {
      set_reference(t, x, -k.eps_ci);
      s.t_search = t + 1;
    } else {
      s.blind_until = t + k.refractory_ns;
      s.t_search = s.blind_until + 1;
    }
  }

  // Can Delta reach a level at an integer of (a, c], given x at both ends? Exact for constant light: I(t) is a
  // monotone fp32 interpolation between the samples, I / i_scale and this build's log_f are monotone (log_f is
  // checked over every positive float), the leak term is non-decreasing in t (leak >= 0), and fp32 additions round
  // monotonically; so Delta over (a, c] lies between its value formed from min(x) and dl(a) and its value formed
  // from max(x) and dl(c), with no margin. It answers "no" only where no integer of (a, c] fires, and so prunes
  // at least what instant_may_fire prunes; the time-ordered search then finds the same first crossing.
  BS_HOT bool may_fire_exact(int64_t a, int64_t cc, float xa, float xc) const {
    const float dn = 0.0f - s.n3_ref;
    const float dl_a = m.leak * since_ref(a, s.t_ref) + s.dr_ref;
    const float dl_c = m.leak * since_ref(cc, s.t_ref) + s.dr_ref;
    const float hi = ((maxr(xa, xc) - s.s3_ref) + dn) + dl_c;
    const float lo = ((minr(xa, xc) - s.s3_ref) + dn) + dl_a;
    return hi >= m.theta_on || lo <= -m.theta_off;
  }

  // The first integer t in [lo, hi) where Delta fires (instant_search's time-ordered depth-first bisection,
  // pixel.h:1886-1916, with the exact node test above; each node carries x at its ends, one log per split).
  BS_HD bool search(const Segment& g, int64_t lo, int64_t hi, int64_t& t_hit, bool& on, float& x_hit) {
    if constexpr (kFlat) {
      return search_body(g, lo, hi, t_hit, on, x_hit);
    } else {
      return search_out(g, lo, hi, t_hit, on, x_hit);
    }
  }
  BS_COLD bool search_out(const Segment& g, int64_t lo, int64_t hi, int64_t& t_hit, bool& on, float& x_hit) { return search_body(g, lo, hi, t_hit, on, x_hit); }
  BS_HD bool search_body(const Segment& g, int64_t lo, int64_t hi, int64_t& t_hit, bool& on, float& x_hit) {
    float x = log_ratio(current(g, lo));
    float D = delta(lo, x);
    if (D >= m.theta_on || D <= -m.theta_off) {
      t_hit = lo;
      on = D >= m.theta_on;
      x_hit = x;
      return true;
    }
    if (hi - lo == 1) return false;
    int64_t sa[32], sc[32];
    float sxa[32], sxc[32];
    int sp = 1;
    sa[0] = lo;
    sc[0] = hi - 1;
    sxa[0] = x;
    sxc[0] = log_ratio(current(g, hi - 1));
    while (sp > 0) {
      --sp;
      const int64_t a = sa[sp], cc = sc[sp];
      const float xa = sxa[sp], xc = sxc[sp];
      if (cc - a == 1) {
        D = delta(cc, xc);
        if (D >= m.theta_on || D <= -m.theta_off) {
          t_hit = cc;
          on = D >= m.theta_on;
          x_hit = xc;
          return true;
        }
        continue;
      }
      ++c.leaves;
      if (!may_fire_exact(a, cc, xa, xc)) continue;
      const int64_t mid = a + (cc - a) / 2;
      const float xm = log_ratio(current(g, mid));
      sa[sp] = mid;
      sc[sp] = cc;
      sxa[sp] = xm;
      sxc[sp] = xc;
      ++sp;
      sa[sp] = a;
      sc[sp] = mid;
      sxa[sp] = xa;
      sxc[sp] = xm;
      ++sp;
    }
    return false;
  }

  // Is the earliest noise candidate (at tn) accepted by thinning (u1 < lambda(t) / lambda_max)? on: its polarity,
  // I: the photocurrent at tn. No side effects.
  BS_HD bool candidate_accepted(const Segment& g, int64_t tn, bool& on, float& I) const {
    if constexpr (kFlat) {
      return candidate_accepted_body(g, tn, on, I);
    } else {
      return candidate_accepted_out(g, tn, on, I);
    }
  }
  BS_COLD bool candidate_accepted_out(const Segment& g, int64_t tn, bool& on, float& I) const { return candidate_accepted_body(g, tn, on, I); }
  BS_HD bool candidate_accepted_body(const Segment& g, int64_t tn, bool& on, float& I) const {
    const bool shot = s.t_shot <= s.t_ba;
    const U4 w = draw(k.seed, shot ? kPurposeShot : kPurposeBackground, k.camera, pixel, shot ? s.n_shot : s.n_ba);
    I = current(g, tn);
    const double accept = shot ? sqrt(static_cast<double>(m.dark) / static_cast<double>(I)) : 1.0;
    on = (w.v[2] & 1u) != 0u;
    return open_uniform_d(w.v[1]) < accept;
  }

  // Moves the earliest candidate's chain (the one at tn) on to its next candidate.
  BS_HD void advance_chain(int64_t tn) {
    if constexpr (kFlat) {
      advance_chain_body(tn);
    } else {
      advance_chain_out(tn);
    }
  }
  BS_COLD void advance_chain_out(int64_t tn) { advance_chain_body(tn); }
  BS_HD void advance_chain_body(int64_t tn) {
    ++c.noise_candidates;
    const bool shot = s.t_shot <= s.t_ba;
    const uint32_t purpose = shot ? kPurposeShot : kPurposeBackground;
    const uint32_t n = shot ? s.n_shot : s.n_ba;
    const double rate = shot ? m.shot_max_hz : m.ba_rate_hz;
    const int64_t next = noise_next(k.seed, purpose, k.camera, pixel, n + 1, tn, rate);
    if (shot) {
      s.n_shot = n + 1;
      s.t_shot = next;
    } else {
      s.n_ba = n + 1;
      s.t_ba = next;
    }
  }

  // Drops the earliest noise candidate (refractory or dead time) or tests and fires it; advances its chain.
  BS_HD void noise_candidate(const Segment& g, int64_t tn, bool blind) {
    if constexpr (kFlat) {
      noise_candidate_body(g, tn, blind);
    } else {
      noise_candidate_out(g, tn, blind);
    }
  }
  BS_COLD void noise_candidate_out(const Segment& g, int64_t tn, bool blind) { noise_candidate_body(g, tn, blind); }
  BS_HD void noise_candidate_body(const Segment& g, int64_t tn, bool blind) {
    bool on = false;
    float I = 0.0f;
    const bool fires = !blind && candidate_accepted(g, tn, on, I);
    advance_chain(tn);
    if (fires) fire(tn, on, log_ratio(I), kLabelNoise);
  }

  // One piece [t, e) inside segment g (advance_instant's inner loop), with the noise candidates it holds.
  BS_HD void piece(const Segment& g, int64_t t, int64_t e) {
    if constexpr (kFlat) {
      piece_body(g, t, e);
    } else {
      piece_out(g, t, e);
    }
  }
  BS_COLD void piece_out(const Segment& g, int64_t t, int64_t e) { piece_body(g, t, e); }
  BS_HD void piece_body(const Segment& g, int64_t t, int64_t e) {
    ++c.pieces;
    for (;;) {
      const int64_t tn = k.noise ? mini(s.t_shot, s.t_ba) : kForever;
      if (s.blind_until != kNotBlind) {
        if (s.blind_until >= e) {
          if (tn < e) {
            noise_candidate(g, tn, true);
            continue;
          }
          break;
        }
        if (tn <= s.blind_until) {
          noise_candidate(g, tn, true);
          continue;
        }
        const int64_t tb = s.blind_until;  // the release (M3 A.16): a new reference at x(t_rel) - eps_ci
        set_reference(tb, log_ratio(current(g, tb)), -k.eps_ci);
        s.blind_until = kNotBlind;
      }
      const int64_t lo = maxi(s.t_search, t);
      const int64_t stop = mini(e, tn);
      if (lo < stop) {
        if (defer) {
          pending = true;
          pg = g;
          p_t = t;
          p_e = e;
          p_lo = lo;
          p_stop = stop;
          return;
        }
        int64_t th;
        bool on;
        float x;
        if (search(g, lo, stop, th, on, x)) {
          fire(th, on, x, -1);
          continue;
        }
        s.t_search = maxi(s.t_search, stop);
      }
      if (tn >= e) break;
      noise_candidate(g, tn, tn < s.t_search);
    }
  }

  // [t_from, t_to) of segment g (t_from >= g.t0), cut into pieces at multiples of 2^23 ns.
  BS_HD void segment(const Segment& g, int64_t t_from, int64_t t_to) {
    const int64_t end = mini(g.t1, t_to);
    int64_t t = t_from;
    while (t < end) {
      const int64_t e = mini(end, ((t >> kWindowLog2) + 1) * kWindowNs);
      piece(g, t, e);
      t = e;
    }
  }

  // x(t) = ln(I / i_scale) at a sample of value v (the start of the segment it opens).
  BS_HOT float x_at_sample(float v) const { return log_ratio(m.dark + m.scale * v); }

  // A whole segment g = [t0, t1) that is one piece (no multiple of 2^23 ns inside), with x0 = x(t0) and
  // x1 = x(t1) (the next segment's start, x_at_sample(g.v1)). Bitwise piece(g, t0, t1): where the pixel is not
  // blind and nothing is pending before t0, Delta(t0) is tested exactly as the reference does; then the node
  // (t0, t1 - 1] is excluded here when bounds from x0 and x1 prove that no integer of it fires, and only otherwise
  // is the reference's search run.
  //
  // Noise candidates inside the segment: when Delta(t0) and the whole node are excluded, no crossing can occur in
  // [t0, t1) while the reference stays put, so the candidates are the only events possible. A rejected candidate
  // changes nothing but its chain; the first accepted one hands over to the reference's loop at its time (which
  // handles a candidate before the comparator at the same ns), with the search known clear up to it.
  BS_HD void segment_fast(const Segment& g, float x0, float x1) {
    const int64_t t0 = g.t0, e = g.t1;
    if (s.blind_until != kNotBlind || s.t_search > t0) {
      piece(g, t0, e);
      return;
    }
    int64_t tn = k.noise ? mini(s.t_shot, s.t_ba) : kForever;
    if (tn < e) {
      if (tn < t0) {  // a candidate left before the segment (none is, by construction): the reference's loop
        piece(g, t0, e);
        return;
      }
      const float D0 = delta(t0, x0);
      if (D0 >= m.theta_on || D0 <= -m.theta_off || (e - t0 > 1 && !excluded(g, t0, e, x0, x1))) {
        piece(g, t0, e);
        return;
      }
      ++c.pieces;
      do {
        bool on;
        float I;
        if (candidate_accepted(g, tn, on, I)) {
          s.t_search = maxi(s.t_search, tn);
          piece_rest(g, tn, e);
          return;
        }
        advance_chain(tn);
        tn = mini(s.t_shot, s.t_ba);
      } while (tn < e);
      s.t_search = maxi(s.t_search, e);
      return;
    }
    ++c.pieces;
    const float D0 = delta(t0, x0);
    if (D0 >= m.theta_on || D0 <= -m.theta_off) {
      fire(t0, D0 >= m.theta_on, x0, -1);
      piece_rest(g, t0, e);
      return;
    }
    if (e - t0 == 1) {
      s.t_search = maxi(s.t_search, e);
      return;
    }
    if (!excluded(g, t0, e, x0, x1)) {
      piece_rest_from_search(g, t0, e);
      return;
    }
    if (e - t0 > 2) ++c.leaves;
    s.t_search = maxi(s.t_search, e);
  }

  // True when instant_may_fire(t0, t1 - 1, I(t0), I(t1 - 1)) and Delta(t1 - 1) are provably both false.
  BS_HOT bool excluded(const Segment& g, int64_t t0, int64_t e, float x0, float x1) const {
    // The interpolation reaches v1 exactly (v0 + (v1 - v0) == v1 in fp32): I over [t0, t1] then lies between its
    // end values, and the exact bounds of may_fire_exact hold with x0, x1 (dl(t1) >= dl(t1 - 1)).
    if (g.v0 + (g.v1 - g.v0) == g.v1) {
      const float dn = 0.0f - s.n3_ref;
      const float dl0 = m.leak * since_ref(t0, s.t_ref) + s.dr_ref;
      const float dl1 = m.leak * since_ref(e, s.t_ref) + s.dr_ref;
      const float hi = ((maxr(x0, x1) - s.s3_ref) + dn) + dl1;
      const float lo = ((minr(x0, x1) - s.s3_ref) + dn) + dl0;
      return hi < m.theta_on && lo > -m.theta_off;
    }
    const float eps = 0x1p-23f;
    const float xa = minr(x0, x1), xb = maxr(x0, x1);
    const float dl0 = m.leak * since_ref(t0, s.t_ref) + s.dr_ref;
    const float dl1 = m.leak * since_ref(e, s.t_ref) + s.dr_ref;
    const float mag = 1.0f + fabs_f(xa) + fabs_f(xb) + fabs_f(s.s3_ref) + fabs_f(dl0) + fabs_f(dl1);
    if (!(mag < 1.0e3f)) return false;
    const float slack = 1.0e-5f + 64.0f * eps * mag;
    const float hi = (((xb + slack) - s.s3_ref) + (0.0f - s.n3_ref)) + dl1;
    if (!(hi < m.theta_on - slack)) return false;
    const float lo_x = (((xa - slack) - s.s3_ref) + (0.0f - s.n3_ref)) + dl0;
    if (m.leak == 0.0f || g.v1 >= g.v0) {
      // leak 0: may_fire is Delta(t1 - 1) against both levels; v1 >= v0 (I non-decreasing): against theta_on only.
      return lo_x > -m.theta_off + slack;
    }
    // leak > 0 and I decreasing: the exclusion test bounds I from below by min(I) - 64 eps max(I), whose log lies
    // below xa by at most 64 eps I(t0) / I(t1) (relative) plus rounding.
    const float I0 = m.dark + m.scale * g.v0, I1 = m.dark + m.scale * g.v1;
    if (!(I1 > 1024.0f * eps * I0)) return false;  // keeps -ln(1 - u) <= 1.1 u for the correction below
    const float corr = 1.1f * (8.0f * eps + 64.0f * eps * (I0 / I1));
    const float lo = ((((xa - corr) - slack) - s.s3_ref) + (0.0f - s.n3_ref)) + dl0;
    return lo > -m.theta_off + slack;
  }

  // The outcome of the deferred search (found: the first firing integer th, its polarity and x), applied as piece()
  // applies its search's, then the piece resumed from its start (its loop holds no state but the pixel's).
  BS_HD void resume_search(bool found, int64_t th, bool on, float x) {
    pending = false;
    if (found) {
      fire(th, on, x, -1);
    } else {
      s.t_search = maxi(s.t_search, p_stop);
    }
    --c.pieces;  // piece() counts the piece again
    piece(pg, p_t, p_e);
  }

  // The rest of piece(g, t, e) after an event inside it (the reference's loop with the new state).
  BS_HD void piece_rest(const Segment& g, int64_t t, int64_t e) {
    --c.pieces;  // piece() counts the piece again
    piece(g, t, e);
  }

  // piece(g, t0, e) whose Delta(t0) is known not to fire: the reference's search from t0, then its loop.
  BS_HD void piece_rest_from_search(const Segment& g, int64_t t0, int64_t e) {
    --c.pieces;
    piece(g, t0, e);
  }
};

// The init of the instantaneous response (pixel.h:792-818) for a pixel whose irradiance at t0 is v (clamped).
BS_HD void pixel_init(PixelRegs& s, const PixelMapRegs& m, const SensorConsts& k, uint32_t pixel, int64_t t0,
                      float v_clamped, float phi0) {
  s.held = v_clamped;
  s.i_scale = m.dark + m.scale * v_clamped;
  const float I = m.dark + m.scale * v_clamped;
  s.t_ref = t0;
  s.s3_ref = log_f(I / s.i_scale);
  s.n3_ref = 0.0f;
  s.dr_ref = phi0;
  s.blind_until = kNotBlind;
  s.t_search = t0 + 1;
  s.flags = kFlagFirstAfterInit;
  s.n_shot = s.n_ba = 0;
  s.t_shot = s.t_ba = kForever;
  if (k.noise) {
    s.t_shot = noise_next(k.seed, kPurposeShot, k.camera, pixel, 0, t0, m.shot_max_hz);
    s.t_ba = noise_next(k.seed, kPurposeBackground, k.camera, pixel, 0, t0, m.ba_rate_hz);
  }
}

}  // namespace bs
