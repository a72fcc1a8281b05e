// The cascade photoreceptor of BallaSim without its noise lattice (photoreceptor = cascade, noise = false), restated
// for the device as a streaming processor like PixelProc: the pixel's state lives in registers and is fed one
// linear sample segment at a time, in time order.
//
// Model (src/sensor/stage1.h, substep.h, expcubic.h; the noise-free paths of pixel.h):
//   stage 1: dz/dt = k (1 - I(t) z), x1 = -ln(z i_scale), solved exactly on each linear piece of the photocurrent
//     (z_step: 8-point Gauss-Legendre, a first-order small-slope form, the zero-order hold, Dawson's integral or
//     erfcx, by the integrated pole P and the slope);
//   stages 2-3: tau_o s2' + s2 = x1, tau_sf s3' + s3 = s2, solved exactly for the cubic Hermite of x1 on each
//     accepted sub-step (try_substep: the midpoint residual and boundary-layer bounds accept a dyadic halving of
//     the rest of the piece; the plain or the residual-exponential split);
//   comparator: Delta = (s3 - s3_ref) + leak (t - t_ref) + dr_ref, a cubic plus two exponentials on each sub-step
//     (ExpCubic), whose first integer-ns crossing of theta_on or -theta_off is found exactly (Polya-Rolle
//     isolation of the monotone pieces with ITP roots, then an interpolation search on the integers).
// Pieces are cut at sample times and at multiples of 2^23 ns (pixel.h:920-941 without noise); events and resets
// are PixelProc::fire's with x = s3 and n3 = 0. Every fp32 operation keeps the reference's order (--fmad=false on
// the device), so states and events are bitwise the reference's fp32 CPU kernel's.
#pragma once

#include "pixel.cuh"
#include "special.cuh"

namespace bs {

constexpr float kNsF = static_cast<float>(1e-9);
constexpr uint16_t kFlagQuarantined = 1u << 9, kFlagSolverFallback = 1u << 10;

// Finite in the reference's sense (x - x == 0: false for inf and NaN).
BS_HD bool finite_f(float x) { return x - x == 0.0f; }

// CascadeConstants<float> and eps_pl_base (src/sensor/sensor_model.cpp:376-397): k in (fA s)^-1, rates in s^-1.
struct CascadeConsts {
  float k, a2, a3, tau_o, tau_sf, eps_accept, eps_drop, eps_pl_base;
};

// The cascade's part of a pixel's state (PixelState z, x1, s2, s3, tv; fp32 values, as the fp32 kernel keeps them).
struct CascadeRegs {
  float z, x1, s2, s3, tv;
};

// ---------------------------------------------------------------------------------------------
// Stage 1 (stage1.h)
// ---------------------------------------------------------------------------------------------
BS_HD float integrated_pole(float I0, float I1, float h, float k) { return k * h * (0.5f * (I0 + I1)); }

// One Gauss-Legendre node pair (u_lo, u_hi, weight w) of int_0^1 e^{-(P(h) - P(u h))} du.
BS_HD float gl8_pair(float kh, float I0, float dI, float u_lo, float u_hi, float w) {
  const float g_lo = kh * (1.0f - u_lo) * (I0 + 0.5f * dI * (1.0f + u_lo));
  const float g_hi = kh * (1.0f - u_hi) * (I0 + 0.5f * dI * (1.0f + u_hi));
  return w * (exp_f(-g_lo) + exp_f(-g_hi));
}
BS_HD float gl8_sum(float, float, float, float J) { return J; }
template <class... R>
BS_HD float gl8_sum(float kh, float I0, float dI, float J, float u_lo, float u_hi, float w, R... rest) {
  return gl8_sum(kh, I0, dI, J + gl8_pair(kh, I0, dI, u_lo, u_hi, w), rest...);
}
template <class... R>
BS_HD float gl8_start(float kh, float I0, float dI, float u_lo, float u_hi, float w, R... rest) {
  return gl8_sum(kh, I0, dI, gl8_pair(kh, I0, dI, u_lo, u_hi, w), rest...);
}

// Exact z(h) from z0 under the photocurrent I0 -> I1 (fA) over h seconds.
static BS_COLD float z_step(float z0, float I0, float I1, float h, float k) {
  const float kh = k * h;
  const float Im = 0.5f * (I0 + I1);
  const float P = kh * Im;
  const float eP = exp_f(-P);
  const float dI = I1 - I0;
  if (P <= 0.5f) {
    if (P > 0.0f && P * fabs_f(dI) <= static_cast<float>(2.4e-4) * Im) {
      // First order in the curvature of the exponent: (1 - e^{-a h}) / a + b h^3 g(a h).
      const float x = kh * I1;
      const float b = 0.5f * k * dI / h;
      const float one_m_E = -expm1_f(-x);
      const float g = 1.0f / 3.0f +
                      x * (-0.25f + x * (static_cast<float>(0.1) + x * (-1.0f / 36.0f + x * (1.0f / 168.0f))));
      const float J = one_m_E / x * h + b * h * h * h * g;
      return z0 * eP + k * J;
    }
    const float J = gl8_start(kh, I0, dI, BS_GL8);
    return z0 * eP + kh * J;
  }
  if (fabs_f(dI) <= 0x1p-23f * Im) return 1.0f / Im + (z0 - 1.0f / Im) * eP;
  const float s = fabs_f(dI) / h;
  const float r = sqrt_f(k / (2.0f * s));
  const float k_over_beta = sqrt_f(2.0f * k / s);
  if (dI > 0.0f) return z0 * eP + k_over_beta * (dawson_f(r * I1) - dawson_f(r * I0) * eP);
  return z0 * eP + k_over_beta * kHalfSqrtPi * (erfcx_f(r * I1) - erfcx_f(r * I0) * eP);
}

// ---------------------------------------------------------------------------------------------
// The comparator input on an interval (expcubic.h): g(u) = c0 + c1 u + c2 u^2 + c3 u^3 + C0 R_j(a0 u) + C1 R_j(a1 u)
// ---------------------------------------------------------------------------------------------
struct ExpCubic {
  float c[4];
  float C[2];
  float a[2];
  int order;  // 0: plain exponentials; 4: residual exponentials R_4

  BS_HD float poly(float u) const { return c[0] + u * (c[1] + u * (c[2] + u * c[3])); }
  BS_HD float term(int i, float u) const { return C[i] == 0.0f ? 0.0f : C[i] * resid_exp_f(order, a[i] * u); }
  BS_HD float operator()(float u) const { return poly(u) + term(0, u) + term(1, u); }
  BS_HD float at(float u, float r0, float r1) const {
    return poly(u) + (C[0] == 0.0f ? 0.0f : C[0] * r0) + (C[1] == 0.0f ? 0.0f : C[1] * r1);
  }
};

BS_HD ExpCubic constant_expcubic(float v, float a2, float a3) { return ExpCubic{{v, 0.0f, 0.0f, 0.0f}, {0.0f, 0.0f}, {a2, a3}, 0}; }

// n-th derivative: d^n/du^n C R_j(a u) = C (-a)^n R_{max(j - n, 0)}(a u).
BS_HD ExpCubic derivative(const ExpCubic& g, int n) {
  ExpCubic d = g;
  for (int i = 0; i < n; ++i) {
    d.c[0] = d.c[1];
    d.c[1] = 2.0f * d.c[2];
    d.c[2] = 3.0f * d.c[3];
    d.c[3] = 0.0f;
    d.C[0] = -d.a[0] * d.C[0];
    d.C[1] = -d.a[1] * d.C[1];
  }
  d.order = g.order > n ? g.order - n : 0;
  return d;
}

// g(d + u) in u (d >= 0): R_j(a (d + u)) = e^{-a d} R_j(a u) + sum_{m<j} ((-a)^m / m!) R_{j-m}(a d) u^m.
static BS_COLD ExpCubic shifted(const ExpCubic& g, float d) {
  ExpCubic s = g;
  s.c[0] = g.c[0] + d * (g.c[1] + d * (g.c[2] + d * g.c[3]));
  s.c[1] = g.c[1] + d * (2.0f * g.c[2] + d * (3.0f * g.c[3]));
  s.c[2] = g.c[2] + d * (3.0f * g.c[3]);
  s.c[3] = g.c[3];
  for (int i = 0; i < 2; ++i) {
    if (g.C[i] == 0.0f) continue;
    const float ad = g.a[i] * d;
    s.C[i] = g.C[i] * exp_f(-ad);
    float coef = g.C[i];
    for (int m = 0; m < g.order; ++m) {
      s.c[m] = s.c[m] + coef * resid_exp_f(g.order - m, ad);
      coef = coef * (-g.a[i]) / static_cast<float>(m + 1);
    }
  }
  return s;
}

struct RangeF {
  float lo, hi;
};

// Bernstein hull of the cubic on [u0, u1], plus the endpoint values of each monotone exponential term.
BS_HD RangeF cubic_range(const float* c, float u0, float u1) {
  const float w = u1 - u0;
  const float q0 = c[0] + u0 * (c[1] + u0 * (c[2] + u0 * c[3]));
  const float q1 = (c[1] + u0 * (2.0f * c[2] + u0 * (3.0f * c[3]))) * w;
  const float q2 = (c[2] + u0 * (3.0f * c[3])) * (w * w);
  const float q3 = c[3] * (w * w * w);
  const float b0 = q0;
  const float b1 = q0 + q1 / 3.0f;
  const float b2 = q0 + (2.0f * q1 + q2) / 3.0f;
  const float b3 = q0 + q1 + q2 + q3;
  return {minr(minr(b0, b1), minr(b2, b3)), maxr(maxr(b0, b1), maxr(b2, b3))};
}
BS_HD RangeF range(const ExpCubic& g, float u0, float u1) {
  RangeF r = cubic_range(g.c, u0, u1);
  for (int i = 0; i < 2; ++i) {
    if (g.C[i] == 0.0f) continue;
    const float e0 = g.term(i, u0), e1 = g.term(i, u1);
    r.lo = r.lo + minr(e0, e1);
    r.hi = r.hi + maxr(e0, e1);
  }
  return r;
}

struct Roots {
  float v[6];
  int n = 0;
  BS_HD void push(float x) { v[n++] = x; }
};

BS_HD float root_tolerance(float hi) { return maxr(static_cast<float>(1e-11), 16.0f * 0x1p-23f * fabs_f(hi)); }

// ITP root of f on [a, b], f(a) f(b) < 0 (Oliveira and Takahashi 2020; kappa1 = 0.2 / (b - a), kappa2 = 2, n0 = 1).
static BS_COLD float itp_root(const ExpCubic& f, float a, float b, float fa, float fb, float tol) {
  const float width0 = b - a;
  const float k1 = static_cast<float>(0.2) / width0;
  int n_half = 0;
  for (float w = width0; w > 2.0f * tol && n_half < 200; w = w * 0.5f) ++n_half;
  const int n_max = n_half + 1;
  float scale = tol;
  for (int j = 0; j < n_max; ++j) scale = scale * 2.0f;
  for (int j = 0; j < 400 && b - a > 2.0f * tol; ++j) {
    const float xh = 0.5f * (a + b);
    const float r = scale - 0.5f * (b - a);
    const float xf = (fb * a - fa * b) / (fb - fa);
    const float sg = xh - xf >= 0.0f ? 1.0f : -1.0f;
    const float delta = k1 * (b - a) * (b - a);
    const float xt = delta <= fabs_f(xh - xf) ? xf + sg * delta : xh;
    const float xi = fabs_f(xt - xh) <= r ? xt : xh - sg * r;
    if (!(xi > a && xi < b)) break;
    const float yi = f(xi);
    if (yi == 0.0f) return xi;
    if ((yi > 0.0f) == (fa > 0.0f)) {
      a = xi;
      fa = yi;
    } else {
      b = xi;
      fb = yi;
    }
    scale = scale * 0.5f;
  }
  return 0.5f * (a + b);
}

// The zero of g's fourth derivative C0 a0^4 e^{-a0 u} + C1 a1^4 e^{-a1 u} in (lo, hi), in log space.
BS_HD void fourth_derivative_root(const ExpCubic& g, float lo, float hi, Roots& out) {
  if (g.C[0] == 0.0f || g.C[1] == 0.0f) return;
  if ((g.C[0] > 0.0f) == (g.C[1] > 0.0f)) return;
  if (g.a[0] == g.a[1]) return;
  const float ln_ratio = log_f(fabs_f(g.C[1]) / fabs_f(g.C[0])) + 4.0f * log_f(g.a[1] / g.a[0]);
  const float u = ln_ratio / (g.a[1] - g.a[0]);
  if (u > lo && u < hi) out.push(u);
}

// Sign-change zeros of g^(N) in (lo, hi), sorted: each derivative is monotone between the zeros of the next.
template <int N>
BS_HD void level_roots(const ExpCubic& g, float lo, float hi, float tol, Roots& out) {
  if constexpr (N >= 4) {
    fourth_derivative_root(g, lo, hi, out);
  } else {
    const ExpCubic f = derivative(g, N);
    const ExpCubic fd = derivative(g, N + 1);
    Roots pts;
    pts.push(lo);
    const RangeF rd = range(fd, lo, hi);
    if (rd.lo < 0.0f && rd.hi > 0.0f) {
      Roots crit;
      level_roots<N + 1>(g, lo, hi, tol, crit);
      for (int i = 0; i < crit.n; ++i) pts.push(crit.v[i]);
    }
    pts.push(hi);
    float fa = f(pts.v[0]);
    for (int i = 0; i + 1 < pts.n; ++i) {
      const float a = pts.v[i], b = pts.v[i + 1];
      const float fb = f(b);
      if ((fa < 0.0f && fb > 0.0f) || (fa > 0.0f && fb < 0.0f)) out.push(itp_root(f, a, b, fa, fb, tol));
      fa = fb;
    }
  }
}

static BS_COLD Roots critical_points(const ExpCubic& g, float lo, float hi) {
  Roots crit;
  level_roots<1>(g, lo, hi, root_tolerance(hi), crit);
  return crit;
}

// First integer k in [k_lo, k_hi] (ns from the interval start) with G(k 1e-9) >= 0, or -1: per monotone piece
// between the critical points, an interpolation search alternating with bisection.
static BS_COLD int64_t first_firing(const ExpCubic& G, const Roots& crit, int64_t k_lo, int64_t k_hi) {
  if (k_lo > k_hi) return -1;
  int64_t piece_lo = k_lo;
  for (int i = 0; i <= crit.n && piece_lo <= k_hi; ++i) {
    const int64_t piece_hi = i < crit.n ? mini(static_cast<int64_t>(floor_f(crit.v[i] / kNsF)), k_hi) : k_hi;
    if (piece_hi < piece_lo) continue;
    int64_t a = piece_lo, b = piece_hi;
    piece_lo = piece_hi + 1;
    float ga = G(static_cast<float>(a) * kNsF);
    if (ga >= 0.0f) return a;
    if (b == a) continue;
    float gb = G(static_cast<float>(b) * kNsF);
    if (gb >= 0.0f) {
      bool interpolate = true;
      while (b - a > 1) {
        int64_t m;
        if (interpolate) {
          const float frac = (-ga) / (gb - ga);
          m = a + static_cast<int64_t>(frac * static_cast<float>(b - a));
          m = mini(maxi(m, a + 1), b - 1);
        } else {
          m = a + (b - a) / 2;
        }
        const int64_t width = b - a;
        const float gm = G(static_cast<float>(m) * kNsF);
        if (gm >= 0.0f) {
          b = m;
          gb = gm;
        } else {
          a = m;
          ga = gm;
        }
        interpolate = (b - a) * 2 <= width;
      }
      return b;
    }
  }
  return -1;
}

struct CascadeHit {
  bool found, on;
  int64_t t;
};

// The first crossing of Delta (from e0) on the integers [max(lo, e0), e1) (pixel.h:386-414).
static BS_COLD CascadeHit cascade_search(const ExpCubic& delta, int64_t e0, int64_t e1, int64_t lo, float theta_on,
                                         float theta_off) {
  const CascadeHit none{false, false, 0};
  const int64_t k_lo = maxi(lo, e0) - e0, k_hi = e1 - 1 - e0;
  if (k_lo > k_hi) return none;
  const float u_lo = static_cast<float>(k_lo) * kNsF, u_hi = static_cast<float>(k_hi) * kNsF;
  const RangeF r = range(delta, u_lo, u_hi);
  const bool on = r.hi >= theta_on, off = r.lo <= -theta_off;
  if (!(on || off)) return none;
  ExpCubic gon = delta, goff = delta;
  gon.c[0] = gon.c[0] - theta_on;
  for (int m = 0; m < 4; ++m) goff.c[m] = -goff.c[m];
  goff.C[0] = -goff.C[0];
  goff.C[1] = -goff.C[1];
  goff.c[0] = goff.c[0] - theta_off;
  Roots crit;
  if (u_hi > u_lo) crit = critical_points(delta, u_lo, u_hi);
  const int64_t k_on = on ? first_firing(gon, crit, k_lo, k_hi) : -1;
  const int64_t k_off = off ? first_firing(goff, crit, k_lo, k_hi) : -1;
  if (k_on < 0 && k_off < 0) return none;
  if (k_off < 0 || (k_on >= 0 && k_on <= k_off)) return {true, true, e0 + k_on};
  return {true, false, e0 + k_off};
}

// ---------------------------------------------------------------------------------------------
// Sub-steps (substep.h)
// ---------------------------------------------------------------------------------------------
struct SubStep {
  int64_t t_a, t_b;
  ExpCubic s3;
  float x1_a, x1_b, int_ku;
  bool fallback;
};

struct CascadeState3 {
  float z, s2, s3;
};

// Particular polynomial solution b of tau y' + y = sum c_m s^m.
BS_HD void particular(const float* c, float tau, float* b) {
  b[3] = c[3];
  b[2] = c[2] - 3.0f * tau * b[3];
  b[1] = c[1] - 2.0f * tau * b[2];
  b[0] = c[0] - tau * b[1];
}

BS_HD float boundary_layer_factor(float P) {
  const float p2 = P * P;
  return minr(p2 * p2 / 384.0f, static_cast<float>(0.15) * P + 1.0f);
}

// The sub-step [0, h] under the photocurrent I_a -> I_b from st; true (and sub, next filled) when accepted or at_floor.
static BS_COLD bool try_substep(const CascadeConsts& cc, const CascadeState3& st, float i_scale, float I_a, float I_b,
                                float h, bool at_floor, SubStep& sub, CascadeState3& next) {
  const float k = cc.k;
  const float z_a = st.z;
  const float z_b = z_step(z_a, I_a, I_b, h, k);
  const float I_m = 0.5f * (I_a + I_b);
  const float z_m = z_step(z_a, I_a, I_m, 0.5f * h, k);
  const float x1a = -log_f(z_a * i_scale), x1b = -log_f(z_b * i_scale), x1m = -log_f(z_m * i_scale);
  const float da = k * (I_a - 1.0f / z_a), db = k * (I_b - 1.0f / z_b);
  float c[4];
  const float delta = (x1b - x1a) / h;
  c[0] = x1a;
  c[1] = da;
  c[2] = (3.0f * delta - 2.0f * da - db) / h;
  c[3] = (da + db - 2.0f * delta) / (h * h);
  const float hh = 0.5f * h;
  const float mid_residual = (c[0] + hh * (c[1] + hh * (c[2] + hh * c[3]))) - x1m;
  const float P = integrated_pole(I_a, I_b, h, k);
  const float int_ku = log_f(z_b / z_a) + P;
  const float xi0 = -log_f(z_a * I_a) + (I_b - I_a) / (h * k * I_a * I_a);
  const float P_star = maxr(P, int_ku);
  const bool accurate =
      fabs_f(mid_residual) <= cc.eps_accept && fabs_f(xi0) * boundary_layer_factor(P_star) <= cc.eps_accept;
  const bool linear = fabs_f(c[2]) * h * h + fabs_f(c[3]) * h * h * h <= cc.eps_drop;
  const bool residual_form = maxr(cc.a2, cc.a3) * h <= 1.0f;
  const bool conditioned = residual_form || linear || 2.0f * minr(cc.a2, cc.a3) * h >= 1.0f;
  if (!at_floor && !(accurate && conditioned)) return false;

  float p2[4], p3[4];
  particular(c, cc.tau_o, p2);
  particular(p2, cc.tau_sf, p3);
  const float A2 = st.s2 - p2[0];
  const float A3 = st.s3 - p3[0];
  const float C_o = A2 * cc.a3 / (cc.a3 - cc.a2);
  const float C_s = A3 - C_o;
  float r2, r3 = 0.0f;
  ExpCubic& g = sub.s3;
  g.a[0] = cc.a2;
  g.a[1] = cc.a3;
  g.C[0] = C_o;
  g.C[1] = C_s;
  if (residual_form) {
    // The exact cubic Taylor polynomials of s2 and s3 at 0 from the cascade equations.
    const float d1[4] = {c[0], c[1], 2.0f * c[2], 6.0f * c[3]};
    float d2[4], d3[4];
    d2[0] = st.s2;
    d3[0] = st.s3;
    for (int j = 0; j < 3; ++j) {
      d2[j + 1] = cc.a2 * (d1[j] - d2[j]);
      d3[j + 1] = cc.a3 * (d2[j] - d3[j]);
    }
    g.c[0] = d3[0];
    g.c[1] = d3[1];
    g.c[2] = d3[2] / 2.0f;
    g.c[3] = d3[3] / 6.0f;
    g.order = 4;
    r2 = resid_exp_f(4, cc.a2 * h);
    r3 = resid_exp_f(4, cc.a3 * h);
    next.s2 = d2[0] + h * (d2[1] + h * (d2[2] / 2.0f + h * (d2[3] / 6.0f))) + A2 * r2;
  } else {
    for (int m = 0; m < 4; ++m) g.c[m] = p3[m];
    g.order = 0;
    r2 = exp_f(-cc.a2 * h);
    if (C_s != 0.0f) r3 = exp_f(-cc.a3 * h);
    next.s2 = p2[0] + h * (p2[1] + h * (p2[2] + h * p2[3])) + A2 * r2;
  }
  next.s3 = g.at(h, r2, r3);
  next.z = z_b;
  // The comparator's copy drops free modes that stay below eps_drop over the whole step (the state keeps them).
  if (fabs_f(g.C[0]) * (residual_form ? r2 : 1.0f) <= cc.eps_drop &&
      fabs_f(g.C[1]) * (residual_form ? r3 : 1.0f) <= cc.eps_drop) {
    g.C[0] = 0.0f;
    g.C[1] = 0.0f;
  }
  sub.x1_a = x1a;
  sub.x1_b = x1b;
  sub.int_ku = int_ku;
  sub.fallback = at_floor && !(accurate && conditioned);
  return true;
}

// A linear piece [t_a, t_b] of photocurrent I_a -> I_b (fA).
struct LinearPiece {
  int64_t t_a, t_b;
  float I_a, I_b;
  BS_HD float at(int64_t t) const {
    if (t == t_b) return I_b;
    return I_a + (I_b - I_a) * (static_cast<float>(t - t_a) / static_cast<float>(t_b - t_a));
  }
};

BS_HD bool cascade_settled(const CascadeConsts& cc, const CascadeState3& st, float x1, float I) {
  return fabs_f(st.z * I - 1.0f) <= cc.eps_drop && fabs_f(st.s2 - x1) <= cc.eps_drop &&
         fabs_f(st.s3 - x1) <= cc.eps_drop;
}

struct CascadeCounters {
  uint32_t substeps = 0, attempts = 0, fallbacks = 0, quarantines = 0;
};

// The next accepted sub-step from ta inside piece pc (substep.h next_substep with pixel.h make_substep :1477-1502 and
// quarantine :1506-1515): the rest of the piece when the cascade is settled under constant input, else the longest
// dyadic halving that try_substep accepts; the state advances to its end (a non-finite one restarts at the steady
// state of the current input, flagged QUARANTINED).
BS_HD int64_t cascade_substep(const CascadeConsts& cc, CascadeRegs& q, uint32_t& flags, float i_scale,
                              const LinearPiece& pc, int64_t ta, int64_t& h_hint, SubStep& sub, CascadeCounters& cn) {
  const CascadeState3 st{q.z, q.s2, q.s3};
  const float I_a = pc.at(ta);
  ++cn.substeps;
  sub.t_a = ta;
  if (pc.I_a == pc.I_b && cascade_settled(cc, st, q.x1, I_a)) {
    sub.t_b = pc.t_b;
    const float h = static_cast<float>(pc.t_b - ta) * kNsF;
    sub.s3 = constant_expcubic(st.s3, cc.a2, cc.a3);
    sub.x1_a = sub.x1_b = q.x1;
    sub.int_ku = cc.k * h / st.z;
    sub.fallback = false;
    if (q.tv != 0.0f) q.tv = q.tv * exp_f(-sub.int_ku);
    return pc.t_b;
  }
  CascadeState3 next{};
  int64_t tb = h_hint > 0 ? mini(pc.t_b, ta + 2 * h_hint) : pc.t_b;
  while (true) {
    const int64_t h_ns = tb - ta;
    ++cn.attempts;
    if (try_substep(cc, st, i_scale, I_a, pc.at(tb), static_cast<float>(h_ns) * kNsF, h_ns <= 1, sub, next)) break;
    tb = ta + h_ns / 2;
  }
  if (tb < pc.t_b || h_hint > 0) h_hint = tb - ta;
  sub.t_b = tb;
  if (sub.fallback) {
    flags |= kFlagSolverFallback;
    ++cn.fallbacks;
  }
  if (!(finite_f(next.z) && next.z > 0.0f && finite_f(next.s2) && finite_f(next.s3))) {
    const float I = pc.at(tb);
    q.z = 1.0f / I;
    q.x1 = -log_f(q.z * i_scale);
    q.s2 = q.s3 = q.x1;
    q.tv = 0.0f;
    sub.s3 = constant_expcubic(q.s3, cc.a2, cc.a3);
    sub.x1_a = sub.x1_b = q.x1;
    flags |= kFlagQuarantined;
    ++cn.quarantines;
  } else {
    q.z = next.z;
    q.s2 = next.s2;
    q.s3 = next.s3;
    q.x1 = sub.x1_b;
    q.tv = q.tv * exp_f(-sub.int_ku) + fabs_f(sub.x1_b - sub.x1_a);
  }
  return tb;
}

// ---------------------------------------------------------------------------------------------
// The processor
// ---------------------------------------------------------------------------------------------

template <class Sink>
struct CascadeProc {
  PixelRegs& s;
  CascadeRegs& q;
  const PixelMapRegs& m;
  const SensorConsts& k;
  const CascadeConsts& cc;
  uint32_t pixel;
  Sink& sink;
  PixelCounters& c;
  CascadeCounters& cn;

  BS_HD float current(const Segment& g, int64_t t) const {
    if (g.t1 == kForever) return m.dark + m.scale * g.v0;
    const float f = static_cast<float>(t - g.t0) / static_cast<float>(g.t1 - g.t0);
    return m.dark + m.scale * (g.v0 + (g.v1 - g.v0) * f);
  }

  // [t_from, t_to) of segment g: pieces cut at the segment's end and at multiples of 2^23 ns (pixel.h:920-941,
  // 1458-1474).
  BS_HD void segment(const Segment& g, int64_t t_from, int64_t t_to) {
    const int64_t end = mini(g.t1, t_to);
    int64_t t = t_from;
    while (t < end) {
      const int64_t e = mini(end, ((t >> kWindowLog2) + 1) * kWindowNs);
      ++c.pieces;
      run_piece(LinearPiece{t, e, current(g, t), current(g, e)});
      t = e;
    }
  }

  BS_HD void run_piece(const LinearPiece& pc) {
    int64_t ta = pc.t_a, h_hint = 0;
    while (ta < pc.t_b) {
      SubStep sub;
      ta = make_substep(pc, ta, h_hint, sub);
      comparator(sub);
    }
  }

  BS_HD int64_t make_substep(const LinearPiece& pc, int64_t ta, int64_t& h_hint, SubStep& sub) {
    return cascade_substep(cc, q, s.flags, s.i_scale, pc, ta, h_hint, sub, cn);
  }

  BS_HD float s3_at(const SubStep& sub, int64_t t) const { return sub.s3(static_cast<float>(t - sub.t_a) * kNsF); }

  // Delta from e0 on the sub-step (pixel.h:322-340 without noise).
  BS_HD ExpCubic delta_from(const SubStep& sub, int64_t e0) const {
    ExpCubic g = e0 == sub.t_a ? sub.s3 : shifted(sub.s3, static_cast<float>(e0 - sub.t_a) * kNsF);
    const float c0 = g.c[0] - s.s3_ref;
    g.c[0] = c0 + (m.leak * since_ref(e0, s.t_ref) + s.dr_ref);
    g.c[1] = g.c[1] + m.leak;
    return g;
  }

  // comparator_plain with handle_blind (pixel.h:1601-1630).
  BS_HD void comparator(const SubStep& sub) {
    PixelProc<Sink> fire_proc{s, m, k, pixel, sink, c};
    while (true) {
      if (s.blind_until != kNotBlind) {
        if (s.blind_until >= sub.t_b) return;
        const int64_t t = s.blind_until;
        fire_proc.set_reference(t, s3_at(sub, t), -k.eps_ci);
        s.blind_until = kNotBlind;
      }
      const int64_t lo = maxi(s.t_search, sub.t_a);
      if (lo >= sub.t_b) return;
      ++c.leaves;
      const CascadeHit hit = cascade_search(delta_from(sub, lo), lo, sub.t_b, lo, m.theta_on, m.theta_off);
      if (!hit.found) {
        s.t_search = maxi(s.t_search, sub.t_b);
        return;
      }
      fire_proc.fire(hit.t, hit.on, s3_at(sub, hit.t), -1);
    }
  }
};

// The cascade's init (pixel.h:792-818 and :836-845 without noise): the steady state at the input held at t0.
BS_HD void cascade_init(CascadeRegs& q, const PixelRegs& s) {
  q.z = 1.0f / s.i_scale;
  q.x1 = 0.0f;
  q.s2 = q.s3 = 0.0f;
  q.tv = 0.0f;
}

}  // namespace bs
