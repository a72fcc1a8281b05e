// fp32 special functions of the cascade photoreceptor: e^x - 1, the residual exponentials R_j, erfcx and
// Dawson's integral, with the same methods and operation order as BallaSim's deterministic maths
// (src/core/pmath/explog.h:232-236 expm1, src/core/pmath/special.h:29-51 resid_exp, :177-186 erfcx, :189-208
// dawson), so that every result is bitwise the reference's fp32 value on the host and on the device.
//
// Methods (published; the constants come from gen_special.py, which evaluates each construction):
//   expm1: degree-8 Taylor polynomial for |x| < 0.35, else e^x - 1.
//   R_j(y) = e^{-y} - sum_{i<j} (-y)^i / i!: the direct form for y > 1, else ((-y)^j / j!) times the nested
//     series 1 - y/(j+1) (1 - y/(j+2) (...)) with 10 terms.
//   erfcx(x) = e^{x^2} erfc(x): Weideman's rational approximation with N = 24.
//   dawson(x): the Taylor series x (1 - 2x^2/3 (1 - 2x^2/5 (...))) with 12 terms below |x| = 1, Rybicki's sum
//     with h = 1/4 and 13 terms above, 1/(2x) beyond 1e8.
// Every operation is an IEEE +, -, *, /, sqrt or an exact one; the device build passes --fmad=false.
#pragma once

#include "bs_math.cuh"

namespace bs {

// Weideman's p(Z) for N = 24, highest degree first; L = sqrt(24 / sqrt 2); 1 / sqrt(pi); sqrt(pi) / 2.
#define BS_WEIDEMAN_P24                                                                                         \
  -0x1.4ce060p-33f, 0x1.510e84p-28f, 0x1.6ddffcp-30f, -0x1.0268d4p-25f, -0x1.488496p-26f, 0x1.926722p-23f,      \
      0x1.13c3e8p-22f, -0x1.236d22p-20f, -0x1.97df94p-19f, 0x1.15cb6ap-18f, 0x1.ff383cp-16f, 0x1.9836a2p-16f,   \
      -0x1.b3204cp-13f, -0x1.99d134p-11f, -0x1.02cf9ap-11f, 0x1.974e82p-8f, 0x1.144306p-5f, 0x1.bbf440p-4f,     \
      0x1.0fde4ap-2f, 0x1.127d88p-1f, 0x1.d9f67ep-1f, 0x1.6512e6p+0f, 0x1.db3598p+0f, 0x1.195372p+1f
constexpr float kWeidemanL24 = 0x1.07a674p+2f;
constexpr float kInvSqrtPi = 0x1.20dd76p-1f;
constexpr float kHalfSqrtPi = 0x1.c5bf8ap-1f;
// Rybicki's weights e^{-((2i + 1) / 4)^2}, i = 0..12.
#define BS_RYBICKI_C                                                                                           \
  0x1.e0fac0p-1f, 0x1.23ba94p-1f, 0x1.ad48bcp-3f, 0x1.7f251ap-5f, 0x1.9ed300p-8f, 0x1.106822p-11f,             \
      0x1.b1fea4p-16f, 0x1.a3604ap-21f, 0x1.eb97d4p-27f, 0x1.5d82c2p-33f, 0x1.2d7026p-40f, 0x1.3b5e5cp-48f,     \
      0x1.903daep-57f
// 8-point Gauss-Legendre on [0, 1]: per node pair (u_lo, u_hi, weight), in the order the integral sums them.
#define BS_GL8                                                                                                 \
  0x1.a214dap-2f, 0x1.2ef592p-1f, 0x1.736360p-3f, 0x1.e5dad4p-3f, 0x1.86894ap-1f, 0x1.413c50p-3f,              \
      0x1.a06d54p-4f, 0x1.cbf256p-1f, 0x1.c76fb6p-4f, 0x1.454e34p-6f, 0x1.f5d58ep-1f, 0x1.9ea1d0p-5f

BS_HD float sqrt_f(float x) {
#if defined(__CUDA_ARCH__)
  return __fsqrt_rn(x);
#else
  return std::sqrt(x);
#endif
}
BS_HD float floor_f(float x) {
#if defined(__CUDA_ARCH__)
  return floorf(x);
#else
  return std::floor(x);
#endif
}
BS_HD float copysign_f(float x, float s) { return u2f((f2u(x) & 0x7fffffffu) | (f2u(s) & 0x80000000u)); }

// p = c0, then p = p z + c_k for each following coefficient.
BS_HD float horner_f(float p, float) { return p; }
template <class... R>
BS_HD float horner_f(float p, float z, float c, R... rest) {
  return horner_f(p * z + c, z, rest...);
}
template <class... R>
BS_HD float horner_start(float z, float c0, R... rest) {
  return horner_f(c0, z, rest...);
}

BS_HD float expm1_f(float x) {
  if (fabs_f(x) < 0.35f) {
    float p = 1.0f / 40320.0f;
    p = p * x + 1.0f / 5040.0f;
    p = p * x + 1.0f / 720.0f;
    p = p * x + 1.0f / 120.0f;
    p = p * x + 1.0f / 24.0f;
    p = p * x + 1.0f / 6.0f;
    p = p * x + 0.5f;
    return (p * x) * x + x;
  }
  return exp_f(x) - 1.0f;
}

// R_j(y) for y >= 0, j = 0..4 (j <= 0: e^{-y}).
static BS_COLD float resid_exp_f(int j, float y) {
  if (j <= 0) return exp_f(-y);
  float yj = 1.0f, jfact = 1.0f;
  for (int i = 1; i <= j; ++i) {
    yj = yj * (-y);
    jfact = jfact * static_cast<float>(i);
  }
  if (y > 1.0f) {
    float t = 1.0f, s = 1.0f;
    for (int i = 1; i < j; ++i) {
      t = t * (-y) / static_cast<float>(i);
      s = s + t;
    }
    return exp_f(-y) - s;
  }
  float q = 1.0f;
  for (int i = 10; i >= 1; --i) q = 1.0f - y * q / static_cast<float>(j + i);
  return yj * (q / jfact);
}

// erfcx(x) for x >= 0 (x <= 0 gives 1, +inf gives 0, NaN propagates).
static BS_COLD float erfcx_f(float x) {
  if (!(x > 0.0f && x < kInfF)) return x > 0.0f ? 0.0f : (x == x ? 1.0f : x);
  const float lx = kWeidemanL24 + x;
  const float Z = (kWeidemanL24 - x) / lx;
  const float p = horner_start(Z, BS_WEIDEMAN_P24);
  return 2.0f * p / (lx * lx) + kInvSqrtPi / lx;
}

// One term of Rybicki's sum, c (e1 / d1 + 1 / (d2 e1)), then the next odd n.
BS_HD void rybicki_step(float, float&, float&, float&, float&) {}
template <class... R>
BS_HD void rybicki_step(float e2, float& sum, float& e1, float& d1, float& d2, float c, R... rest) {
  sum = sum + c * (e1 / d1 + 1.0f / (d2 * e1));
  d1 = d1 + 2.0f;
  d2 = d2 - 2.0f;
  e1 = e1 * e2;
  rybicki_step(e2, sum, e1, d1, d2, rest...);
}

// Dawson's integral F(x) = e^{-x^2} int_0^x e^{t^2} dt (odd).
static BS_COLD float dawson_f(float x) {
  const float ax = fabs_f(x);
  if (ax < 1.0f) {
    const float two_x2 = 2.0f * x * x;
    float q = 1.0f;
    for (int n = 12; n >= 1; --n) q = 1.0f - two_x2 * q / static_cast<float>(2 * n + 1);
    return x * q;
  }
  if (!(ax <= 1e8f)) return ax == ax ? copysign_f(0.5f / ax, x) : x;
  const float h = 0.25f;
  const int n0 = 2 * static_cast<int>(0.5f * ax / h + 0.5f);
  const float xp = ax - static_cast<float>(n0) * h;
  float e1 = exp_f(2.0f * xp * h);
  const float e2 = e1 * e1;
  float sum = 0.0f, d1 = static_cast<float>(n0 + 1), d2 = static_cast<float>(n0 - 1);
  rybicki_step(e2, sum, e1, d1, d2, BS_RYBICKI_C);
  return copysign_f(kInvSqrtPi * exp_f(-xp * xp) * sum, x);
}

}  // namespace bs
