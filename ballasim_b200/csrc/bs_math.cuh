// Deterministic scalar maths shared by the device kernels and the host-side model set-up.
//
// The event times of the pixel model depend on the last bit of ln I, so this build evaluates the
// logarithm with the same published method as BallaSim's own deterministic maths
// (src/core/pmath/explog.h:137-225): x = m 2^e with m in [sqrt(1/2), sqrt(2)), ln(1 + f) = f - s (f - R(s^2)),
// s = f / (2 + f), R the first terms of the atanh series, and ln 2 split hi/lo (Cody-Waite). The fp64 sin/cos
// of the map draws follow the same reduction and Taylor kernels (trig.h:57-155). Every operation is a plain
// IEEE +, -, *, / or an exact bit operation; the build passes --fmad=false (device) and -ffp-contract=off
// (host), so no multiply-add is fused and host and device round identically.
#pragma once

#include <stdint.h>

// BS_HD: shared host/device code, inlined where the compiler finds it worth it. BS_COLD: a rare path kept out of
// line on the device, one copy per kernel, so that the hot loops' code stays small enough for the instruction cache.
// BS_HOT: a small function of the per-sample path, always inlined: a call would need the caller's pixel state in
// memory (a PixelProc holds references to it), which on the device means local memory on every access.
#if defined(__CUDACC__)
#define BS_HD __host__ __device__ inline
#define BS_HOT __host__ __device__ __forceinline__
#define BS_D __device__ __forceinline__
#define BS_COLD __host__ __device__ __noinline__
#else
#define BS_HD inline
#define BS_HOT inline
#define BS_D inline
#define BS_COLD
#endif

#if !defined(__CUDA_ARCH__)
#include <cmath>
#include <cstring>
#endif

namespace bs {

constexpr int kWindowLog2 = 23;
constexpr int64_t kWindowNs = int64_t{1} << kWindowLog2;
constexpr int64_t kNotBlind = INT64_MIN;
constexpr int64_t kForever = INT64_MAX;
constexpr uint16_t kFlagFirstAfterInit = 1u << 12;
constexpr uint8_t kLabelSignal = 0, kLabelNoise = 1, kLabelLeak = 2, kLabelHot = 3;

BS_HD float u2f(uint32_t u) {
#if defined(__CUDA_ARCH__)
  return __uint_as_float(u);
#else
  float f;
  std::memcpy(&f, &u, 4);
  return f;
#endif
}
BS_HD uint32_t f2u(float f) {
#if defined(__CUDA_ARCH__)
  return __float_as_uint(f);
#else
  uint32_t u;
  std::memcpy(&u, &f, 4);
  return u;
#endif
}
BS_HD double u2d(uint64_t u) {
#if defined(__CUDA_ARCH__)
  return __longlong_as_double(static_cast<long long>(u));
#else
  double d;
  std::memcpy(&d, &u, 8);
  return d;
#endif
}
BS_HD uint64_t d2u(double d) {
#if defined(__CUDA_ARCH__)
  return static_cast<uint64_t>(__double_as_longlong(d));
#else
  uint64_t u;
  std::memcpy(&u, &d, 8);
  return u;
#endif
}
BS_HD float rint_f(float x) {
#if defined(__CUDA_ARCH__)
  return rintf(x);
#else
  return std::rint(x);
#endif
}
BS_HD double rint_d(double x) {
#if defined(__CUDA_ARCH__)
  return rint(x);
#else
  return std::rint(x);
#endif
}
BS_HD float fabs_f(float x) { return u2f(f2u(x) & 0x7fffffffu); }

// min / max with the reference's operand order (a NaN operand is not propagated symmetrically).
BS_HOT float minr(float a, float b) { return b < a ? b : a; }
BS_HOT float maxr(float a, float b) { return a < b ? b : a; }
BS_HOT int64_t mini(int64_t a, int64_t b) { return b < a ? b : a; }
BS_HOT int64_t maxi(int64_t a, int64_t b) { return a < b ? b : a; }

constexpr float kInfF = __builtin_huge_valf();

// ---------------------------------------------------------------------------------------------
// fp32 natural logarithm
// ---------------------------------------------------------------------------------------------
BS_HOT float log_f(float x) {
  if (!(x > 0.0f)) return x == 0.0f ? -kInfF : u2f(0x7fc00000u);
  if (x == kInfF) return x;
  int bias = 0;
  if (x < 0x1p-126f) {
    x = x * 0x1p25f;
    bias = 25;
  }
  uint32_t b = f2u(x);
  int e = static_cast<int>((b >> 23) & 0xffu) - 126 - bias;
  float m = u2f((b & 0x807fffffu) | (126u << 23));  // [0.5, 1)
  if (m < 0x1.6a09e6p-1f) {
    m = m + m;
    e -= 1;
  }
  const float f = m - 1.0f;
  const float s = f / (2.0f + f);
  const float z = s * s;
  float p = 2.0f / 9.0f;
  p = p * z + 2.0f / 7.0f;
  p = p * z + 2.0f / 5.0f;
  p = p * z + 2.0f / 3.0f;
  const float r = p * z;
  const float logm = f - s * (f - r);
  const float ef = static_cast<float>(e);
  return ef * 0x1.62e400p-1f + (logm + ef * 0x1.7f7d1cp-20f);
}

// fp32 e^x for the analytic fields: k = rint(x log2 e), Cody-Waite r, degree-7 Taylor, exact scaling by 2^k;
// 0 below -87.33 (no subnormal results).
BS_HOT float exp_f(float x) {
  if (!(x >= -87.33f)) return x != x ? x : 0.0f;
  if (x > 88.72f) return kInfF;
  const float k = rint_f(x * 0x1.715476p+0f);
  const float r = (x - k * 0x1.62e400p-1f) - k * 0x1.7f7d1cp-20f;
  float p = 1.0f / 5040.0f;
  p = p * r + 1.0f / 720.0f;
  p = p * r + 1.0f / 120.0f;
  p = p * r + 1.0f / 24.0f;
  p = p * r + 1.0f / 6.0f;
  p = p * r + 0.5f;
  p = p * r + 1.0f;
  p = p * r + 1.0f;
  const int ki = static_cast<int>(k);
  const int e1 = ki > 127 ? 127 : (ki < -126 ? -126 : ki);
  const int e2 = ki - e1;
  const float p1 = u2f(static_cast<uint32_t>(e1 + 127) << 23), p2 = u2f(static_cast<uint32_t>(e2 + 127) << 23);
  return e2 == 0 ? p * p1 : (p * p1) * p2;
}

// ---------------------------------------------------------------------------------------------
// fp64 log / exp / sincos (map draws)
// ---------------------------------------------------------------------------------------------
BS_HD double log_d(double x) {
  if (!(x > 0.0)) return x == 0.0 ? -__builtin_huge_val() : u2d(0x7ff8000000000000ull);
  if (x == __builtin_huge_val()) return x;
  int bias = 0;
  if (x < 0x1p-1022) {
    x = x * 0x1p54;
    bias = 54;
  }
  uint64_t b = d2u(x);
  int e = static_cast<int>((b >> 52) & 0x7ff) - 1022 - bias;
  double m = u2d((b & 0x800fffffffffffffull) | (uint64_t{1022} << 52));
  if (m < 0x1.6a09e667f3bcdp-1) {
    m = m + m;
    e -= 1;
  }
  const double f = m - 1.0;
  const double s = f / (2.0 + f);
  const double z = s * s;
  double p = 2.0 / 19.0;
  p = p * z + 2.0 / 17.0;
  p = p * z + 2.0 / 15.0;
  p = p * z + 2.0 / 13.0;
  p = p * z + 2.0 / 11.0;
  p = p * z + 2.0 / 9.0;
  p = p * z + 2.0 / 7.0;
  p = p * z + 2.0 / 5.0;
  p = p * z + 2.0 / 3.0;
  const double r = p * z;
  const double logm = f - s * (f - r);
  const double ef = static_cast<double>(e);
  return ef * 0x1.62e42fee00000p-1 + (logm + ef * 0x1.a39ef35793c76p-33);
}

BS_HD double exp_d(double x) {
  if (!(x >= -708.39)) return x != x ? x : 0.0;
  if (x > 709.78) return __builtin_huge_val();
  const double k = rint_d(x * 0x1.71547652b82fep+0);
  const double r = (x - k * 0x1.62e42fee00000p-1) - k * 0x1.a39ef35793c76p-33;
  double p = 1.0 / 6227020800.0;
  p = p * r + 1.0 / 479001600.0;
  p = p * r + 1.0 / 39916800.0;
  p = p * r + 1.0 / 3628800.0;
  p = p * r + 1.0 / 362880.0;
  p = p * r + 1.0 / 40320.0;
  p = p * r + 1.0 / 5040.0;
  p = p * r + 1.0 / 720.0;
  p = p * r + 1.0 / 120.0;
  p = p * r + 1.0 / 24.0;
  p = p * r + 1.0 / 6.0;
  p = p * r + 0.5;
  p = p * r + 1.0;
  p = p * r + 1.0;
  const int ki = static_cast<int>(k);
  const int e1 = ki > 1023 ? 1023 : (ki < -1022 ? -1022 : ki);
  const int e2 = ki - e1;
  const double p1 = u2d(static_cast<uint64_t>(e1 + 1023) << 52), p2 = u2d(static_cast<uint64_t>(e2 + 1023) << 52);
  return e2 == 0 ? p * p1 : (p * p1) * p2;
}

BS_HD void sincos_d(double x, double* s, double* c) {
  const double ax = x < 0 ? -x : x;
  if (!(ax <= 1.0e6)) {
    *s = *c = u2d(0x7ff8000000000000ull);
    return;
  }
  if (x == 0.0) {
    *s = x;
    *c = 1.0;
    return;
  }
  const double k = rint_d(x * 0x1.45f306dc9c883p-1);
  const double r = k == 0.0 ? x : ((x - k * 0x1.921fb544p+0) - k * 0x1.0b4611a6p-34) - k * 0x1.3198a2e037073p-69;
  const double z = r * r;
  double ps = 2.8114572543455207632e-15;
  ps = ps * z - 7.6471637318198164759e-13;
  ps = ps * z + 1.6059043836821614599e-10;
  ps = ps * z - 2.5052108385441718775e-08;
  ps = ps * z + 2.7557319223985890653e-06;
  ps = ps * z - 1.9841269841269841270e-04;
  ps = ps * z + 8.3333333333333333333e-03;
  ps = ps * z - 1.6666666666666666667e-01;
  const double sr = r + (r * z) * ps;
  double pc = -1.5619206968586225e-16;
  pc = pc * z + 4.7794773323873852974e-14;
  pc = pc * z - 1.1470745597729724714e-11;
  pc = pc * z + 2.0876756987868098979e-09;
  pc = pc * z - 2.7557319223985890653e-07;
  pc = pc * z + 2.4801587301587301587e-05;
  pc = pc * z - 1.3888888888888888889e-03;
  pc = pc * z + 4.1666666666666666667e-02;
  const double cr = (1.0 - 0.5 * z) + (z * z) * pc;
  switch (static_cast<int>(k) & 3) {
    case 0: *s = sr; *c = cr; break;
    case 1: *s = cr; *c = -sr; break;
    case 2: *s = -sr; *c = -cr; break;
    default: *s = -cr; *c = sr; break;
  }
}

// ---------------------------------------------------------------------------------------------
// Philox4x32-10 (Salmon et al., SC'11) and BallaSim's counter layout for every draw:
// counter (purpose << 8 | camera, pixel, index lo, index hi), key = the 64-bit seed (src/core/rng/purpose.h:47-53).
// ---------------------------------------------------------------------------------------------
struct U4 {
  uint32_t v[4];
};

BS_HD uint32_t mulhi(uint32_t a, uint32_t b) {
#if defined(__CUDA_ARCH__)
  return __umulhi(a, b);
#else
  return static_cast<uint32_t>((static_cast<uint64_t>(a) * b) >> 32);
#endif
}

BS_HD U4 philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int round = 0; round < 10; ++round) {
    const uint32_t hi0 = mulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
    const uint32_t hi1 = mulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
    c0 = hi1 ^ c1 ^ k0;
    c1 = lo1;
    c2 = hi0 ^ c3 ^ k1;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return U4{{c0, c1, c2, c3}};
}

BS_HD U4 draw(uint64_t seed, uint32_t purpose, uint32_t camera, uint32_t pixel, uint64_t index) {
  return philox((purpose << 8) | (camera & 0xFFu), pixel, static_cast<uint32_t>(index),
                static_cast<uint32_t>(index >> 32), static_cast<uint32_t>(seed), static_cast<uint32_t>(seed >> 32));
}

// Philox word -> (0, 1) in fp64 (all 32 bits).
BS_HD double open_uniform_d(uint32_t u) { return (static_cast<double>(u) + 0.5) * 0x1p-32; }

// Purpose tags: the reference's map tag, and this build's noise tags (new, unused by the reference's registry).
constexpr uint32_t kPurposeSensorMap = 0x0002;
constexpr uint32_t kPurposeReadoutPhase = 0x0022;
constexpr uint32_t kPurposeShot = 0x0080;
constexpr uint32_t kPurposeBackground = 0x0081;
constexpr uint32_t kPurposeBackgroundMap = 0x0082;

}  // namespace bs
