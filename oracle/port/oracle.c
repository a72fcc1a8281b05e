/* CPU restatement of BallaSim's per-pixel event-generation path. TEST INFRASTRUCTURE ONLY: see
 * oracle.h. Every function cites the reference file:line it restates; paths are relative to the
 * reference project root. Compiled with -ffp-contract=off so that no multiply-add is fused: each
 * expression below is evaluated in the operation order the reference's policy fixes
 * (cmake/FloatingPoint.cmake:8-13). */
#include "oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static char g_error[512];
const char* orc_last_error(void) { return g_error; }
static int fail(const char* msg) {
  snprintf(g_error, sizeof g_error, "%s", msg);
  return -1;
}

/* ======================================================================================== */
/* Philox4x32-10 (Salmon et al., SC'11; src/core/rng/philox.h:29-53)                         */
/* ======================================================================================== */
static uint32_t mulhi32(uint32_t a, uint32_t b) { return (uint32_t)(((uint64_t)a * b) >> 32); }

void orc_philox(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]) {
  uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
  uint32_t k0 = key_in[0], k1 = key_in[1];
  for (int round = 0; round < 10; ++round) {
    if (round > 0) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    const uint32_t hi0 = mulhi32(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
    const uint32_t hi1 = mulhi32(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
    const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

/* Counter (purpose << 8 | camera, pixel, index lo, index hi), key = the 64-bit seed (purpose.h:47-53). */
void orc_draw(uint64_t seed, uint32_t purpose, uint32_t camera, uint32_t pixel, uint64_t index, uint32_t out[4]) {
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  const uint32_t ctr[4] = {(purpose << 8) | (camera & 0xFFu), pixel, (uint32_t)index, (uint32_t)(index >> 32)};
  orc_philox(ctr, key, out);
}

/* Philox word -> open (0, 1): fp64 uses all 32 bits (src/sensor/noise.h:24-27). */
static double open_uniform64(uint32_t u) { return ((double)u + 0.5) * 0x1p-32; }

/* ======================================================================================== */
/* Deterministic exp / log / sincos (src/core/pmath/explog.h, trig.h)                        */
/* ======================================================================================== */
static float bits_f(uint32_t u) {
  float f;
  memcpy(&f, &u, 4);
  return f;
}
static uint32_t f_bits(float f) {
  uint32_t u;
  memcpy(&u, &f, 4);
  return u;
}

/* Exact mantissa/exponent split, m in [0.5, 1) (explog.h:72-96). */
static float frexp_exactf(float x, int* e) {
  int bias = 0;
  if (x < 0x1p-126f) {
    x = x * 0x1p25f;
    bias = 25;
  }
  uint32_t b = f_bits(x);
  *e = (int)((b >> 23) & 0xff) - 126 - bias;
  b = (b & 0x807fffffu) | (126u << 23);
  return bits_f(b);
}
static double frexp_exact(double x, int* e) {
  int bias = 0;
  if (x < 0x1p-1022) {
    x = x * 0x1p54;
    bias = 54;
  }
  uint64_t b;
  memcpy(&b, &x, 8);
  *e = (int)((b >> 52) & 0x7ff) - 1022 - bias;
  b = (b & 0x800fffffffffffffull) | ((uint64_t)1022 << 52);
  double m;
  memcpy(&m, &b, 8);
  return m;
}
static float ldexp_exactf(float x, int e) {
  const int e1 = e > 127 ? 127 : (e < -126 ? -126 : e);
  const int e2 = e - e1;
  const float p1 = bits_f((uint32_t)(e1 + 127) << 23), p2 = bits_f((uint32_t)(e2 + 127) << 23);
  return e2 == 0 ? x * p1 : (x * p1) * p2;
}
static double ldexp_exact(double x, int e) {
  const int e1 = e > 1023 ? 1023 : (e < -1022 ? -1022 : e);
  const int e2 = e - e1;
  uint64_t b1 = (uint64_t)(e1 + 1023) << 52, b2 = (uint64_t)(e2 + 1023) << 52;
  double p1, p2;
  memcpy(&p1, &b1, 8);
  memcpy(&p2, &b2, 8);
  return e2 == 0 ? x * p1 : (x * p1) * p2;
}

/* ln(m) for x = m 2^e, m in [sqrt(1/2), sqrt(2)), by log(1 + f) = f - s (f - R(s^2)), s = f / (2 + f), with
 * the atanh series R = 2 z/3 + 2 z^2/5 + ... (explog.h:137-153, 157-168). */
static float log_reducedf(float x, int* e) {
  float m = frexp_exactf(x, e);
  if (m < 0x1.6a09e6p-1f) {
    m = m + m;
    *e -= 1;
  }
  const float f = m - 1.0f;
  const float s = f / (2.0f + f);
  const float z = s * s;
  float p = 2.0f / 9.0f;
  p = p * z + 2.0f / 7.0f;
  p = p * z + 2.0f / 5.0f;
  p = p * z + 2.0f / 3.0f;
  const float R = p * z;
  return f - s * (f - R);
}
static double log_reduced(double x, int* e) {
  double m = frexp_exact(x, e);
  if (m < 0x1.6a09e667f3bcdp-1) {
    m = m + m;
    *e -= 1;
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
  const double R = p * z;
  return f - s * (f - R);
}

/* log with ln 2 split hi/lo (Cody-Waite; explog.h:214-225). */
float orc_logf(float x) {
  if (!(x > 0.0f)) return x == 0.0f ? -INFINITY : NAN;
  if (x == INFINITY) return x;
  int e = 0;
  const float logm = log_reducedf(x, &e);
  const float ef = (float)e;
  return ef * 0x1.62e400p-1f + (logm + ef * 0x1.7f7d1cp-20f);
}
double orc_log(double x) {
  if (!(x > 0.0)) return x == 0.0 ? -INFINITY : NAN;
  if (x == INFINITY) return x;
  int e = 0;
  const double logm = log_reduced(x, &e);
  const double ef = (double)e;
  return ef * 0x1.62e42fee00000p-1 + (logm + ef * 0x1.a39ef35793c76p-33);
}

/* e^x: k = rint(x log2 e), r = x - k ln2 (hi/lo), Taylor polynomial, exact scaling; 0 below the underflow
 * cut (explog.h:203-211, 100-131). */
float orc_expf(float x) {
  if (!(x >= -87.33f)) return x != x ? x : 0.0f;
  if (x > 88.72f) return INFINITY;
  const float k = rintf(x * 0x1.715476p+0f);
  const float r = (x - k * 0x1.62e400p-1f) - k * 0x1.7f7d1cp-20f;
  float p = 1.0f / 5040.0f;
  p = p * r + 1.0f / 720.0f;
  p = p * r + 1.0f / 120.0f;
  p = p * r + 1.0f / 24.0f;
  p = p * r + 1.0f / 6.0f;
  p = p * r + 0.5f;
  p = p * r + 1.0f;
  p = p * r + 1.0f;
  return ldexp_exactf(p, (int)k);
}
double orc_exp(double x) {
  if (!(x >= -708.39)) return x != x ? x : 0.0;
  if (x > 709.78) return INFINITY;
  const double k = rint(x * 0x1.71547652b82fep+0);
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
  return ldexp_exact(p * r + 1.0, (int)k);
}

/* sin and cos by a three-part Cody-Waite reduction by pi/2 and Taylor polynomials on |r| <= pi/4
 * (trig.h:57-80, 130-155). The coefficients are 1/n! rounded to double. */
void orc_sincos(double x, double* s, double* c) {
  if (!(fabs(x) <= 1.0e6)) {
    *s = *c = NAN;
    return;
  }
  if (x == 0.0) {
    *s = x;
    *c = 1.0;
    return;
  }
  const double k = rint(x * 0x1.45f306dc9c883p-1);
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
  switch ((int)k & 3) {
    case 0: *s = sr; *c = cr; break;
    case 1: *s = cr; *c = -sr; break;
    case 2: *s = -sr; *c = -cr; break;
    default: *s = -cr; *c = sr; break;
  }
}

/* ======================================================================================== */
/* Analytic fields (the project's renderer stand-in; fp32, fixed operation order)             */
/* ======================================================================================== */
static float t_seconds(int64_t t_ns) { return (float)((double)t_ns * 1e-9); }

/* tanh(u) = sign(u) (1 - 2 / (e^{2|u|} + 1)), exactly +-1 beyond |u| = 9. */
static float tanh_det(float u) {
  const float a = fabsf(u);
  float r = 1.0f;
  if (a <= 9.0f) {
    const float e = orc_expf(2.0f * a);
    r = 1.0f - 2.0f / (e + 1.0f);
  }
  return u < 0.0f ? -r : r;
}

float orc_field_eval(const orc_field* f, uint32_t x, uint32_t y, int64_t t_ns) {
  const float ts = t_seconds(t_ns);
  const float xc = (float)x + 0.5f, yc = (float)y + 0.5f;
  if (f->kind == ORC_FIELD_TANH_EDGE) {
    const float u = (((f->nx * xc + f->ny * yc) - f->speed * ts) - f->c) / f->width_px;
    return f->base + f->amp * tanh_det(u);
  }
  float e = f->base;
  for (int32_t k = 0; k < f->n_blobs; ++k) {
    const float* b = f->blobs + (size_t)k * ORC_BLOB_WORDS;
    const float cx = b[1] + b[3] * ts, cy = b[2] + b[4] * ts;
    const float dx = xc - cx, dy = yc - cy;
    const float d2 = dx * dx + dy * dy;
    if (d2 < b[6]) e = e + b[0] * orc_expf(-(d2 * b[5]));
  }
  return e;
}

int32_t orc_field_level(const orc_field* f, uint32_t x, uint32_t y, int64_t t_w, int32_t l_min, int32_t l_max) {
  if (f->kind != ORC_FIELD_BLOBS) return l_min;
  const float ts = t_seconds(t_w);
  const float xc = (float)x + 0.5f, yc = (float)y + 0.5f;
  float v = 0.0f;
  for (int32_t k = 0; k < f->n_blobs; ++k) {
    const float* b = f->blobs + (size_t)k * ORC_BLOB_WORDS;
    const float cx = b[1] + b[3] * ts, cy = b[2] + b[4] * ts;
    const float dx = xc - cx, dy = yc - cy;
    const float d2 = dx * dx + dy * dy;
    if (d2 <= b[7] && b[8] > v) v = b[8];
  }
  if (!(v > 0.0f)) return l_min;
  /* v W / d_px with W = 2^23 ns and d_px = 0.25 px: v * 2^-23... in seconds, 0.008388608 / 0.25 */
  const float q = v * 0.033554432f;
  int e = 0;
  const float m = frexp_exactf(q, &e);
  int32_t level = m == 0.5f ? e - 1 : e; /* ceil(log2 q) */
  if (level < l_min) level = l_min;
  if (level > l_max) level = l_max;
  return level;
}

void orc_field_frame(const orc_field* f, int64_t t_ns, float* out) {
  for (uint32_t y = 0; y < f->height; ++y)
    for (uint32_t x = 0; x < f->width; ++x) out[(size_t)y * f->width + x] = orc_field_eval(f, x, y, t_ns);
}

void orc_field_samples(const orc_field* f, const uint32_t* pixel, const int64_t* t_ns, size_t n, float* out) {
  for (size_t i = 0; i < n; ++i) out[i] = orc_field_eval(f, pixel[i] % f->width, pixel[i] / f->width, t_ns[i]);
}

void orc_field_levels(const orc_field* f, int64_t t_w, int32_t l_min, int32_t l_max, uint8_t* out) {
  for (uint32_t y = 0; y < f->height; ++y)
    for (uint32_t x = 0; x < f->width; ++x)
      out[(size_t)y * f->width + x] = (uint8_t)orc_field_level(f, x, y, t_w, l_min, l_max);
}

/* ======================================================================================== */
/* Sensor maps (src/sensor/maps.cpp:26-39, 78-156): fp64, Philox purpose kSensorMap (2)       */
/* ======================================================================================== */
typedef struct {
  double theta_on, theta_off, leak, dark_fA, phi0;
  double ba_rate_hz; /* background-activity rate of the pixel (noise on) */
} orc_map;

static void normals4(uint64_t seed, uint32_t camera, uint32_t pixel, uint64_t block, double* out) {
  uint32_t r[4];
  orc_draw(seed, 2, camera, pixel, block, r);
  const double u0 = open_uniform64(r[0]), u1 = open_uniform64(r[1]);
  const double u2 = open_uniform64(r[2]), u3 = open_uniform64(r[3]);
  const double two_pi = 0x1.921fb54442d18p+2;
  const double r0 = sqrt(-2.0 * orc_log(u0)), r1 = sqrt(-2.0 * orc_log(u2));
  double s0, c0, s1, c1;
  orc_sincos(two_pi * u1, &s0, &c0);
  orc_sincos(two_pi * u3, &s1, &c1);
  out[0] = r0 * c0;
  out[1] = r0 * s0;
  out[2] = r1 * c1;
  out[3] = r1 * s1;
}

/* exp(-Ea / kB (1/T - 1/T0)) (maps.cpp:41-43). */
static double arrhenius(double ea, double t, double t0) {
  return orc_exp(-ea / 8.617333262e-5 * (1.0 / t - 1.0 / t0));
}
static double dmax(double a, double b) { return a < b ? b : a; } /* std::max */

/* Purpose tag of the background-activity rate map (new; no reference counterpart). */
#define ORC_PURPOSE_BA_MAP 0x0082u
#define ORC_PURPOSE_SHOT 0x0080u
#define ORC_PURPOSE_BA 0x0081u

static void draw_map(const orc_params* p, uint64_t seed, uint32_t camera, uint32_t px, orc_map* m) {
  const double leak_temp = arrhenius(p->leak_ea_eV, p->temperature_K, p->reference_temperature_K);
  const double dark_temp = arrhenius(p->dark_ea_eV, p->temperature_K, p->reference_temperature_K);
  const double rho = p->theta_onoff_corr, rho_c = sqrt(1.0 - rho * rho);
  const double ln10 = orc_log(10.0);
  double xi[4];
  normals4(seed, camera, px, 0, xi);
  uint32_t u[4];
  orc_draw(seed, 2, camera, px, 1, u);
  const double u_phase = open_uniform64(u[0]);
  const double xi_off = rho == 0.0 ? xi[1] : rho * xi[0] + rho_c * xi[1];
  m->theta_on = dmax(p->theta_floor, p->theta_on + p->sigma_theta_on * xi[0]);
  m->theta_off = dmax(p->theta_floor, p->theta_off + p->sigma_theta_off * xi_off);
  const double leak_rate = p->leak_rate_hz * orc_exp(p->leak_sigma_log10 * xi[2] * ln10) * leak_temp;
  m->dark_fA = p->dark_current_fA * orc_exp(p->dark_sigma_ln * xi[3]) * dark_temp;
  m->leak = m->theta_on * leak_rate;
  m->phi0 = p->initial_phase == 0   ? u_phase * m->theta_on
            : p->initial_phase == 1 ? -m->theta_off + u_phase * (m->theta_on + m->theta_off)
                                    : 0.0;
  m->ba_rate_hz = 0.0;
  if (p->noise) {
    /* The pixel's background-activity rate, log-normal: median exp(sigma xi) with xi from its own block. */
    double z[4];
    uint32_t w[4];
    orc_draw(seed, ORC_PURPOSE_BA_MAP, camera, px, 0, w);
    const double a = open_uniform64(w[0]), b = open_uniform64(w[1]);
    double s, c;
    orc_sincos(0x1.921fb54442d18p+2 * b, &s, &c);
    z[0] = sqrt(-2.0 * orc_log(a)) * c;
    m->ba_rate_hz = p->ba_median_hz * orc_exp(p->ba_sigma_ln * z[0]);
  }
}

/* ======================================================================================== */
/* The instantaneous pixel kernel (src/sensor/pixel.h:760-1054, 1519-1588, 1779-1924), fp32  */
/* ======================================================================================== */
#define NOT_BLIND INT64_MIN
#define NO_BREAKPOINT INT64_MAX
#define SEG_LOG2 23
#define FLAG_FIRST_AFTER_INIT (1u << 12)
#define MAX_GROUPS 8

typedef struct {
  int64_t t_ref, t_search, blind_until;
  float s3_ref, n3_ref, dr_ref, i_scale;
  float held[MAX_GROUPS];
  uint16_t flags;
  /* noise chains (new): the next candidate time and count of each */
  int64_t t_shot, t_ba;
  uint32_t n_shot, n_ba;
} orc_state;

struct orc_model {
  orc_params p;
  uint32_t width, height, camera;
  int32_t groups;
  uint64_t seed;
  orc_map* maps;
  orc_state* st;
  /* kernel constants (KernelConstants<float>, sensor_model.cpp:394-433) */
  float scale, irr_max, eps_ci, label_cut;
  int ideal_reset;
  int64_t refractory_ns;
  int64_t t_state;
  int initialized;
  orc_event* ev;
  size_t n_ev, cap_ev;
  uint64_t pieces, leaves, clamps;
};

static void push_event(orc_model* m, const orc_event* e) {
  if (m->n_ev == m->cap_ev) {
    m->cap_ev = m->cap_ev ? 2 * m->cap_ev : 1024;
    m->ev = (orc_event*)realloc(m->ev, m->cap_ev * sizeof(orc_event));
  }
  m->ev[m->n_ev++] = *e;
}

static float clamp_irr(float v, float v_max) { return v >= 0.0f ? (v <= v_max ? v : v_max) : 0.0f; }
static float fmaxr(float a, float b) { return a < b ? b : a; } /* balla::max */
static float fminr(float a, float b) { return b < a ? b : a; } /* balla::min */
static int64_t imin(int64_t a, int64_t b) { return b < a ? b : a; }
static int64_t imax(int64_t a, int64_t b) { return a < b ? b : a; }

/* One pixel and call: PixelKernel's instantaneous members. */
typedef struct {
  orc_model* m;
  uint32_t pixel;
  orc_state* s;
  const orc_map* map;
  const int64_t* t; /* the run */
  const float* irr;
  int32_t n, skip;
  int64_t t_state;
  uint32_t live;
  float theta_on, theta_off, leak, dark, scale;
} kern;

static int n_aug(const kern* k) { return 1 + k->n - k->skip; }
static int64_t sample_time(const kern* k, int i) { return i == 0 ? k->t_state : k->t[i - 1 + k->skip]; }
static float sample_value(const kern* k, int i, int g) {
  if (i == 0 && k->skip == 0) return k->s->held[g];
  return clamp_irr(k->irr[(int64_t)(i - 1 + k->skip) * k->m->groups + g], k->m->irr_max);
}

/* Live groups: a non-zero value somewhere in the augmented samples (pixel.h:1070-1091). */
static void scan_input(kern* k) {
  const int G = k->m->groups;
  const uint32_t all = (1u << G) - 1u;
  uint32_t live = 0;
  if (k->skip == 0) {
    for (int g = 0; g < G; ++g)
      if (k->s->held[g] != 0.0f) live |= 1u << g;
  }
  for (int i = 0; i < k->n && live != all; ++i)
    for (int g = 0; g < G; ++g)
      if (clamp_irr(k->irr[(int64_t)i * G + g], k->m->irr_max) != 0.0f) live |= 1u << g;
  k->live = live;
}

static int segment_at(const kern* k, int64_t t) { /* pixel.h:1097-1105 */
  int lo = 0, hi = n_aug(k) - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (sample_time(k, mid) <= t) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}
static int segment_of(const kern* k, int seg, int64_t t) { /* pixel.h:1108-1112 */
  const int last = n_aug(k) - 1;
  while (seg < last && sample_time(k, seg + 1) <= t) ++seg;
  return seg;
}
static int64_t segment_end(const kern* k, int seg) {
  return seg + 1 < n_aug(k) ? sample_time(k, seg + 1) : NO_BREAKPOINT;
}

/* Linear between samples, held after the last (pixel.h:1119-1130; constant waveforms, no glare). */
static float group_value(const kern* k, int seg, int64_t t, int g) {
  if (seg + 1 >= n_aug(k)) return sample_value(k, seg, g);
  const int64_t t0 = sample_time(k, seg), t1 = sample_time(k, seg + 1);
  const float f = (float)(t - t0) / (float)(t1 - t0);
  const float v0 = sample_value(k, seg, g), v1 = sample_value(k, seg + 1, g);
  return v0 + (v1 - v0) * f;
}

/* I(t) = I_dk + sum_g m_g s v_g(t) with m_g = 1 (pixel.h:1782-1790). */
static float photocurrent(const kern* k, int seg, int64_t t) {
  float I = k->dark;
  for (int g = 0; g < k->m->groups; ++g) {
    if (!((k->live >> g) & 1u)) continue;
    I = I + 1.0f * k->scale * group_value(k, seg, t, g);
  }
  return I;
}

static float log_ratio(const kern* k, float I) { return orc_logf(I / k->s->i_scale); } /* pixel.h:1793 */

static float since_ref(int64_t t, int64_t t_ref) { return (float)((double)(t - t_ref) * 1e-9); }

/* Delta at t for x = log_ratio(I(t)) (pixel.h:1797-1802). */
static float instant_delta(const kern* k, int64_t t, float x) {
  const orc_state* s = k->s;
  const float ds = x - s->s3_ref;
  const float dn = 0.0f - s->n3_ref;
  const float dl = k->leak * since_ref(t, s->t_ref) + s->dr_ref;
  return ds + dn + dl;
}

static void set_reference(orc_state* s, int64_t t, float s3, float n3, float offset) { /* pixel.h:1520-1529 */
  s->t_ref = t;
  s->s3_ref = s3;
  s->n3_ref = n3;
  s->dr_ref = offset;
}

/* Labels by the increment split (pixel.h:291-307). */
static uint8_t split_label(float ds, float dl, float D, float cut) {
  const float a_s = ds / D, a_l = dl / D;
  if (a_s >= cut && a_s >= a_l) return 0;
  if (a_l >= cut && a_l > a_s) return 2;
  return 1;
}
static uint8_t first_label(int on, float ds, float dn, float l, float cut) {
  const float D = ds + dn + l;
  return (on ? D > 0.0f : D < 0.0f) ? split_label(ds, l, D, cut) : 1;
}

/* An event and the reset (pixel.h:1534-1588). label_override >= 0 marks a noise event's label. */
static void fire(kern* k, int64_t t, int on, float s3, float n3, int label_override) {
  orc_state* s = k->s;
  const float ds = s3 - s->s3_ref;
  const float dn = n3 - s->n3_ref;
  const float l = k->leak * since_ref(t, s->t_ref);
  const float dl = l + s->dr_ref;
  const float D = ds + dn + dl;
  uint8_t label = (s->flags & FLAG_FIRST_AFTER_INIT) != 0 ? first_label(on, ds, dn, l, k->m->label_cut)
                                                           : split_label(ds, dl, D, k->m->label_cut);
  if (label_override >= 0) label = (uint8_t)label_override;
  orc_event ev;
  ev.pixel = k->pixel;
  ev.polarity = on ? 1 : 0;
  ev.label = label;
  ev.flags = s->flags;
  ev.t_cross = t;
  ev.ds = ds;
  ev.dn = dn;
  ev.dl = dl;
  ev.l_first = (s->flags & FLAG_FIRST_AFTER_INIT) != 0 ? l : 0.0f;
  push_event(k->m, &ev);
  s->flags = 0;
  if (k->m->ideal_reset) {
    set_reference(s, t, s3, n3, D - (on ? k->theta_on : -k->theta_off));
    s->t_search = t + 1 + k->m->refractory_ns;
  } else if (k->m->refractory_ns == 0) {
    set_reference(s, t, s3, n3, -k->m->eps_ci);
    s->t_search = t + 1;
  } else {
    s->blind_until = t + k->m->refractory_ns;
    s->t_search = s->blind_until + 1;
  }
}

/* Can Delta reach a level at an integer of (a, c]? Constant light: curvature 0, no range cap
 * (pixel.h:1853-1876 with instant_curvature's linear case, :1815). */
static int instant_may_fire(const kern* k, int64_t a, int64_t c, float Ia, float Ic) {
  const float eps = 0x1p-23f;
  float hi = fmaxr(Ia, Ic), lo = fminr(Ia, Ic);
  const float h = (float)(c - a) * 1e-9f;
  const float curv = 0.0f, mod = 0.0f, i_lo = k->dark, i_hi = INFINITY;
  const float hh = h * h * curv;
  const float margin = 64.0f * eps * (hi + 2.0f * mod);
  const orc_state* s = k->s;
  if (k->leak == 0.0f && hi - lo >= 0.5f * hh) {
    const float D = instant_delta(k, c, log_ratio(k, Ic));
    return D >= k->theta_on || D <= -k->theta_off;
  }
  if (Ic >= Ia && (curv == 0.0f || hi - lo > hh + 2.0f * margin)) {
    return instant_delta(k, c, log_ratio(k, Ic)) >= k->theta_on;
  }
  hi = fminr(hi + 0.125f * hh, i_hi) + margin;
  lo = fmaxr(lo - 0.125f * hh, i_lo) - margin;
  const float dl_a = k->leak * since_ref(a, s->t_ref) + s->dr_ref;
  const float dl_c = k->leak * since_ref(c, s->t_ref) + s->dr_ref;
  const float base = 0.0f - s->n3_ref - s->s3_ref;
  const float x_hi = log_ratio(k, hi);
  if (x_hi + base + dl_c + 16.0f * eps * (1.0f + fabsf(x_hi) + fabsf(s->s3_ref) + fabsf(dl_c)) >= k->theta_on) return 1;
  if (!(lo > 0.0f)) return 1;
  const float x_lo = log_ratio(k, lo);
  return x_lo + base + dl_a - 16.0f * eps * (1.0f + fabsf(x_lo) + fabsf(s->s3_ref) + fabsf(dl_a)) <= -k->theta_off;
}

typedef struct {
  int found, on;
  int64_t t;
  float x;
} hit_t;

static int instant_fires(const kern* k, int64_t t, hit_t* h) { /* pixel.h:1918-1924 */
  const float D = instant_delta(k, t, h->x);
  h->found = D >= k->theta_on || D <= -k->theta_off;
  h->on = D >= k->theta_on;
  h->t = t;
  return h->found;
}

/* First integer t in [lo, hi) of a piece where Delta fires: time-ordered depth-first bisection
 * (pixel.h:1886-1916). */
static hit_t instant_search(kern* k, int seg, int64_t lo, int64_t hi) {
  typedef struct {
    int64_t a, c;
    float Ia, Ic;
  } node;
  const float I_lo = photocurrent(k, seg, lo);
  hit_t out = {0, 0, lo, log_ratio(k, I_lo)};
  if (instant_fires(k, lo, &out)) return out;
  if (hi - lo == 1) return out;
  node stack[32];
  int sp = 0;
  stack[sp].a = lo;
  stack[sp].c = hi - 1;
  stack[sp].Ia = I_lo;
  stack[sp].Ic = photocurrent(k, seg, hi - 1);
  ++sp;
  while (sp > 0) {
    const node nd = stack[--sp];
    if (nd.c - nd.a == 1) {
      out.t = nd.c;
      out.x = log_ratio(k, nd.Ic);
      if (instant_fires(k, nd.c, &out)) return out;
      continue;
    }
    ++k->m->leaves;
    if (!instant_may_fire(k, nd.a, nd.c, nd.Ia, nd.Ic)) continue;
    const int64_t mid = nd.a + (nd.c - nd.a) / 2;
    const float Im = photocurrent(k, seg, mid);
    stack[sp].a = mid;
    stack[sp].c = nd.c;
    stack[sp].Ia = Im;
    stack[sp].Ic = nd.Ic;
    ++sp;
    stack[sp].a = nd.a;
    stack[sp].c = mid;
    stack[sp].Ia = nd.Ia;
    stack[sp].Ic = Im;
    ++sp;
  }
  out.found = 0;
  return out;
}

/* ---- noise of the new model (no reference counterpart) ----
 * Two Poisson streams per pixel, each a chain of candidate times keyed by (pixel, candidate number):
 * candidate n + 1 follows n after ceil(-ln(u) / lambda_max s) ns, u = open_uniform of word 0 of
 * draw(seed, purpose, camera, pixel, n); a candidate at t is accepted with probability
 * lambda(t) / lambda_max against word 1, and word 2's low bit is the polarity. Background activity
 * has lambda = lambda_max = the pixel's rate; shot noise has lambda(I) = r_shot sqrt(100 fA / I),
 * lambda_max = r_shot sqrt(100 / I_dk) (I >= I_dk). An accepted candidate fires as a crossing of its
 * polarity (label NOISE) unless the pixel is blind. */
static double shot_max(const kern* k) { return k->m->p.shot_rate_hz * sqrt(100.0 / (double)k->dark); }

static int64_t next_candidate(uint64_t seed, uint32_t purpose, uint32_t camera, uint32_t pixel, uint32_t n,
                              int64_t t, double rate_hz) {
  if (!(rate_hz > 0.0)) return INT64_MAX;
  uint32_t w[4];
  orc_draw(seed, purpose, camera, pixel, n, w);
  const double u = open_uniform64(w[0]);
  const double dt = -orc_log(u) / rate_hz * 1e9;
  const double step = ceil(dt);
  if (!(step < 9.0e18)) return INT64_MAX;
  return t + (int64_t)(step < 1.0 ? 1.0 : step);
}

/* The earliest noise candidate at tn: dropped when the pixel is blind (refractory) or inside the dead time,
 * else accepted with probability lambda(t) / lambda_max and fired as a comparator event of its polarity;
 * its chain advances either way. */
static void noise_candidate(kern* k, int seg, int64_t tn, int blind) {
  orc_state* s = k->s;
  const int shot = s->t_shot <= s->t_ba;
  const uint32_t purpose = shot ? ORC_PURPOSE_SHOT : ORC_PURPOSE_BA;
  const uint32_t n = shot ? s->n_shot : s->n_ba;
  const double rate = shot ? shot_max(k) : k->map->ba_rate_hz;
  const int64_t next = next_candidate(k->m->seed, purpose, k->m->camera, k->pixel, n + 1, tn, rate);
  if (shot) {
    s->n_shot = n + 1;
    s->t_shot = next;
  } else {
    s->n_ba = n + 1;
    s->t_ba = next;
  }
  if (blind) return;
  uint32_t w[4];
  orc_draw(k->m->seed, purpose, k->m->camera, k->pixel, n, w);
  const float I = photocurrent(k, seg, tn);
  const double accept = shot ? sqrt((double)k->dark / (double)I) : 1.0;
  if (open_uniform64(w[1]) < accept) fire(k, tn, (int)(w[2] & 1u), log_ratio(k, I), 0.0f, 1);
}

/* Advances from t_from to t_to (pixel.h:876-907); with noise on, the candidates are handled at their times
 * inside the pieces (blind ones dropped). */
static void advance_instant(kern* k, int64_t t_from, int64_t t_to) {
  orc_state* s = k->s;
  int seg = segment_at(k, t_from);
  int64_t t = t_from;
  while (t < t_to) {
    seg = segment_of(k, seg, t);
    const int64_t e = imin(imin(t_to, segment_end(k, seg)), ((t >> SEG_LOG2) + 1) * ((int64_t)1 << SEG_LOG2));
    ++k->m->pieces;
    for (;;) {
      const int64_t tn = k->m->p.noise ? imin(s->t_shot, s->t_ba) : INT64_MAX;
      if (s->blind_until != NOT_BLIND) {
        if (s->blind_until >= e) {
          if (tn < e) {
            noise_candidate(k, seg, tn, 1);
            continue;
          }
          break;
        }
        if (tn <= s->blind_until) {
          noise_candidate(k, seg, tn, 1);
          continue;
        }
        set_reference(s, s->blind_until, log_ratio(k, photocurrent(k, seg, s->blind_until)), 0.0f, -k->m->eps_ci);
        s->blind_until = NOT_BLIND;
      }
      const int64_t lo = imax(s->t_search, t);
      const int64_t stop = imin(e, tn);
      if (lo < stop) {
        const hit_t hit = instant_search(k, seg, lo, stop);
        if (hit.found) {
          fire(k, hit.t, hit.on, hit.x, 0.0f, -1);
          continue;
        }
        s->t_search = imax(s->t_search, stop);
      }
      if (tn >= e) break;
      noise_candidate(k, seg, tn, tn < s->t_search);
    }
    t = e;
  }
  if (k->n > 0) {
    for (int g = 0; g < k->m->groups; ++g) s->held[g] = sample_value(k, n_aug(k) - 1, g);
  }
}

static void kern_setup(kern* k, orc_model* m, uint32_t p, const int64_t* t, const float* irr, int32_t n) {
  k->m = m;
  k->pixel = p;
  k->s = &m->st[p];
  k->map = &m->maps[p];
  k->t = t;
  k->irr = irr;
  k->n = n;
  k->t_state = m->t_state;
  k->skip = n > 0 && t[0] == m->t_state ? 1 : 0;
  k->theta_on = (float)k->map->theta_on;
  k->theta_off = (float)k->map->theta_off;
  k->leak = (float)k->map->leak;
  k->dark = (float)k->map->dark_fA;
  k->scale = m->scale * 1.0f; /* gain 1 */
  scan_input(k);
}

orc_model* orc_model_create(const orc_params* p, uint32_t width, uint32_t height, uint64_t seed, uint32_t camera,
                            int32_t groups) {
  if (groups < 1 || groups > MAX_GROUPS || width == 0 || height == 0 || camera > 255) {
    fail("orc_model_create: bad shape");
    return NULL;
  }
  orc_model* m = (orc_model*)calloc(1, sizeof(orc_model));
  m->p = *p;
  m->width = width;
  m->height = height;
  m->camera = camera;
  m->groups = groups;
  m->seed = seed;
  const size_t n = (size_t)width * height;
  m->maps = (orc_map*)calloc(n, sizeof(orc_map));
  m->st = (orc_state*)calloc(n, sizeof(orc_state));
  for (size_t i = 0; i < n; ++i) draw_map(p, seed, camera, (uint32_t)i, &m->maps[i]);
  /* make_constants (sensor_model.cpp:394-433), fp32, gain 1 */
  m->scale = (float)p->illuminance_scale;
  m->irr_max = (float)(1e9 / (p->illuminance_scale * 1.0));
  m->ideal_reset = p->reset_mode == 1;
  m->refractory_ns = llround(p->refractory_s * 1e9);
  m->eps_ci = (float)p->eps_ci;
  m->label_cut = (float)p->label_share_cut;
  return m;
}

void orc_model_destroy(orc_model* m) {
  if (!m) return;
  free(m->maps);
  free(m->st);
  free(m->ev);
  free(m);
}

/* init's instantaneous branch (pixel.h:792-818). */
int orc_model_init(orc_model* m, int64_t t0, const float* irr0) {
  const size_t n = (size_t)m->width * m->height;
  const int G = m->groups;
  for (size_t i = 0; i < n * (size_t)G; ++i)
    if (!isfinite(irr0[i])) return fail("init: non-finite irradiance");
  m->t_state = t0;
  for (size_t p = 0; p < n; ++p) {
    orc_state* s = &m->st[p];
    memset(s, 0, sizeof *s);
    kern k;
    kern_setup(&k, m, (uint32_t)p, NULL, NULL, 0);
    float mean_I = k.dark;
    for (int g = 0; g < G; ++g) {
      const float v = clamp_irr(irr0[p * G + g], m->irr_max);
      if (!(v == irr0[p * G + g])) ++m->clamps;
      s->held[g] = v;
      mean_I = mean_I + k.scale * v;
    }
    scan_input(&k);
    s->i_scale = mean_I;
    set_reference(s, t0, log_ratio(&k, photocurrent(&k, 0, t0)), 0.0f, (float)m->maps[p].phi0);
    s->blind_until = NOT_BLIND;
    s->t_search = t0 + 1;
    s->flags = FLAG_FIRST_AFTER_INIT;
    s->t_shot = s->t_ba = INT64_MAX;
    s->n_shot = s->n_ba = 0;
    if (m->p.noise) {
      s->t_shot = next_candidate(m->seed, ORC_PURPOSE_SHOT, m->camera, (uint32_t)p, 0, t0, shot_max(&k));
      s->t_ba = next_candidate(m->seed, ORC_PURPOSE_BA, m->camera, (uint32_t)p, 0, t0, m->maps[p].ba_rate_hz);
    }
  }
  m->initialized = 1;
  return 0;
}

int orc_model_advance_runs(orc_model* m, const uint32_t* ids, size_t n, const int64_t* t, const float* irr,
                           size_t n_samples, const int64_t* row_start, const int32_t* row_count, int64_t t_end) {
  if (!m->initialized) return fail("advance: not initialized");
  if (t_end < m->t_state) return fail("advance: t_end before the model time");
  const size_t np = (size_t)m->width * m->height;
  int32_t* row_of = (int32_t*)malloc(np * sizeof(int32_t));
  for (size_t i = 0; i < np; ++i) row_of[i] = -1;
  /* The run rules of SensorModel::advance_raw (sensor_model.cpp:1075-1103). */
  for (size_t i = 0; i < n; ++i) {
    const uint32_t p = ids[i];
    if (p >= np || row_of[p] >= 0) {
      free(row_of);
      return fail("advance: pixel id out of range or duplicate");
    }
    row_of[p] = (int32_t)i;
    const int64_t s = row_start[i];
    const int32_t c = row_count[i];
    if (c < 0 || s < 0 || (size_t)s + (size_t)c > n_samples) {
      free(row_of);
      return fail("advance: sample run out of range");
    }
    for (int32_t j = 0; j < c; ++j) {
      if (j == 0 ? t[s] < m->t_state : t[s + j] <= t[s + j - 1]) {
        free(row_of);
        return fail("advance: sample times must be strictly increasing from the model time");
      }
    }
    if (c > 0 && t[s + c - 1] > t_end) {
      free(row_of);
      return fail("advance: sample after t_end");
    }
    for (size_t j = 0; j < (size_t)c * m->groups; ++j) {
      const float v = irr[(size_t)s * m->groups + j];
      if (!isfinite(v)) {
        free(row_of);
        return fail("advance: non-finite irradiance");
      }
      if (clamp_irr(v, m->irr_max) != v) ++m->clamps;
    }
  }
  for (size_t p = 0; p < np; ++p) {
    const int32_t row = row_of[p];
    kern k;
    if (row >= 0) {
      kern_setup(&k, m, (uint32_t)p, t + row_start[row], irr + (size_t)row_start[row] * m->groups, row_count[row]);
    } else {
      kern_setup(&k, m, (uint32_t)p, NULL, NULL, 0);
    }
    advance_instant(&k, m->t_state, t_end);
  }
  free(row_of);
  m->t_state = t_end;
  return 0;
}

size_t orc_model_event_count(const orc_model* m) { return m->n_ev; }

static int cmp_event(const void* a, const void* b) {
  const orc_event* x = (const orc_event*)a;
  const orc_event* y = (const orc_event*)b;
  if (x->t_cross != y->t_cross) return x->t_cross < y->t_cross ? -1 : 1;
  return x->pixel < y->pixel ? -1 : (x->pixel > y->pixel ? 1 : 0);
}

void orc_model_take_events(orc_model* m, orc_event* out) {
  qsort(m->ev, m->n_ev, sizeof(orc_event), cmp_event);
  if (out) memcpy(out, m->ev, m->n_ev * sizeof(orc_event));
  m->n_ev = 0;
}

void orc_model_maps(const orc_model* m, double* on, double* off, double* leak, double* dark, double* phi0) {
  const size_t n = (size_t)m->width * m->height;
  for (size_t i = 0; i < n; ++i) {
    if (on) on[i] = m->maps[i].theta_on;
    if (off) off[i] = m->maps[i].theta_off;
    if (leak) leak[i] = m->maps[i].leak;
    if (dark) dark[i] = m->maps[i].dark_fA;
    if (phi0) phi0[i] = m->maps[i].phi0;
  }
}

void orc_model_state(const orc_model* m, int64_t* t_ref, int64_t* t_search, float* s3_ref, float* dr_ref,
                     float* held) {
  const size_t n = (size_t)m->width * m->height;
  for (size_t i = 0; i < n; ++i) {
    if (t_ref) t_ref[i] = m->st[i].t_ref;
    if (t_search) t_search[i] = m->st[i].t_search;
    if (s3_ref) s3_ref[i] = m->st[i].s3_ref;
    if (dr_ref) dr_ref[i] = m->st[i].dr_ref;
    if (held) held[i] = m->st[i].held[0];
  }
}

void orc_model_noise_maps(const orc_model* m, double* ba_rate_hz) {
  const size_t n = (size_t)m->width * m->height;
  for (size_t i = 0; i < n; ++i) ba_rate_hz[i] = m->maps[i].ba_rate_hz;
}

uint64_t orc_model_stat(const orc_model* m, int32_t which) {
  return which == 0 ? m->pieces : which == 1 ? m->leaves : m->clamps;
}

/* ======================================================================================== */
/* The window sampler (src/engine/sampling.h:26-69, 355-839; window_impl.h:461-713)           */
/* ======================================================================================== */
static float np_min(float a, float b) { return (a <= b || a != a) ? a : b; } /* sampling.h:26-27 */

float orc_midpoint_eta(float tol, float dark, float a, float m, float b) {
  (void)tol;
  float num = 0.0f, den = dark;
  const float dev = fabsf((a + b) * -0.5f + m);
  const float low = np_min(np_min(a, m), b);
  num += 1.0f * dev;
  den += 1.0f * low;
  return num / den;
}
static int exceeds(const orc_rules* r, float a, float m, float b) {
  return r->midpoint && orc_midpoint_eta(r->tol, r->dark, a, m, b) > r->tol;
}

typedef struct {
  const orc_field* f;
  const orc_rules* r;
  int64_t t_w;
  uint32_t x, y;
  int64_t* t_out;
  float* irr_out;
  size_t cap, n;
} sampler_ctx;

static void emit(sampler_ctx* c, uint32_t dt, float v) {
  if (c->n < c->cap) {
    c->t_out[c->n] = c->t_w + dt;
    c->irr_out[c->n] = v;
  }
  ++c->n;
}

/* Refinement of one selected interval below the lattice, depth-first and in time order: the interval's
 * midpoint is rendered while depth < max_refine_levels, and each half whose triple (lo, mid, hi) exceeds is
 * split again if it is at least min_split long (Midpoints, HalfFlags; sampling.h:591-678, window_impl.h:574-652).
 * The breadth-first rounds of the reference render the same set: a half's flag depends on its own triple only. */
static void refine(sampler_ctx* c, uint32_t lo, uint32_t hi, float vlo, float vhi, int32_t depth, int flip_lo) {
  if (depth >= c->r->max_refine_levels) return;
  const uint32_t g = (lo + hi) >> 1;
  const float vg = orc_field_eval(c->f, c->x, c->y, c->t_w + g);
  const int bad = exceeds(c->r, vlo, vg, vhi);
  /* Rendered samples of an analytic field have signature 0: only an interval that starts at a carried sample
   * of another signature flips (its left half keeps the flip). */
  if ((flip_lo || bad) && (int64_t)(g - lo) >= 2 * c->r->min_dt_ns) refine(c, lo, g, vlo, vg, depth + 1, flip_lo);
  emit(c, g, vg);
  if (bad && (int64_t)(hi - g) >= 2 * c->r->min_dt_ns) refine(c, g, hi, vg, vhi, depth + 1, 0);
}

int64_t orc_sample_window(const orc_field* f, const orc_rules* r, int64_t t_w, const uint32_t* pixel,
                          const uint8_t* level, size_t n, float* carried_irr, uint64_t* carried_sig,
                          int64_t* offsets, int64_t* t_out, float* irr_out, size_t cap) {
  sampler_ctx c = {f, r, t_w, 0, 0, t_out, irr_out, cap, 0};
  float v[(1 << 13) + 1];
  for (size_t a = 0; a < n; ++a) {
    offsets[a] = (int64_t)c.n;
    const uint32_t px = pixel[a];
    c.x = px % f->width;
    c.y = px / f->width;
    const int L = level[a];
    const uint32_t count = (1u << L) + 1u, step = 1u << (23 - L);
    v[0] = carried_irr[a];
    for (uint32_t j = 1; j < count; ++j) v[j] = orc_field_eval(f, c.x, c.y, t_w + (int64_t)j * step);
    emit(&c, 0, v[0]);
    for (uint32_t j = 1; j < count; ++j) {
      /* Round0Flags (sampling.h:490-523): triples (j-1, j, j+1) and (j-2, j-1, j); the carried signature
       * flips against the rendered ones (0) when it is not 0. */
      const int flip = r->refine_signature && j == 1 && carried_sig[a] != 0;
      const int m = (j + 1 < count && exceeds(r, v[j - 1], v[j], v[j + 1])) ||
                    (j >= 2 && exceeds(r, v[j - 2], v[j - 1], v[j]));
      if ((flip || m) && (int64_t)step >= 2 * r->min_dt_ns) refine(&c, (j - 1) * step, j * step, v[j - 1], v[j], 0, flip);
      emit(&c, j * step, v[j]);
    }
    carried_irr[a] = v[count - 1];
    carried_sig[a] = 0;
  }
  offsets[n] = (int64_t)c.n;
  return c.n <= cap ? (int64_t)c.n : -(int64_t)c.n;
}

/* ======================================================================================== */
/* The learned step proposal: features, training walk and the sampler's judge / fallback.     */
/* This project's own method (no reference counterpart); restated here from its definition:   */
/* steps of 2^s ns aligned on their own lattice inside the window, judged by the plain        */
/* midpoint rule and refined by it when rejected (sampling.h:26-69, 490-523, 638-678).        */
/* ======================================================================================== */
uint16_t orc_bf16(float f) {
  uint32_t u;
  memcpy(&u, &f, 4);
  if ((u & 0x7fffffffu) > 0x7f800000u) return (uint16_t)((u >> 16) | 0x40u);
  u += 0x7fffu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}

static float quarter_asinh(float z) {
  const float a = fabsf(z);
  const float r = orc_logf(a + sqrtf(a * a + 1.0f)) * 0.25f;
  return z < 0.0f ? -r : r;
}

void orc_step_features(const float hx[8], uint64_t gaps, float x, float out[16]) {
  for (int k = 0; k < 8; ++k) out[k] = quarter_asinh((hx[k] - x) * 1e4f);
  for (int k = 0; k < 8; ++k) out[8 + k] = (float)((int)((gaps >> (8 * k)) & 0xffu) - 13) * 0.1f;
}

void orc_walk_reset(orc_walk* w, float v0) {
  const float x = orc_logf(v0);
  for (int k = 0; k < 8; ++k) w->hx[k] = x;
  w->gaps = 0x1717171717171717ull;
  w->pv = v0;
  w->valid = 0;
}

static void walk_push(orc_walk* w, float x, float v, int s) {
  for (int k = 7; k > 0; --k) w->hx[k] = w->hx[k - 1];
  w->hx[0] = x;
  w->gaps = (w->gaps << 8) | (uint64_t)s;
  w->pv = v;
  w->valid = 1;
}

int orc_walk_window(const int64_t* t, const float* v, int n, int64_t t_w, int level, int sh, float eps, uint64_t seed,
                    uint32_t pixel, int32_t window, orc_walk* w, uint16_t* x_out, float* y_out, uint64_t* key_out,
                    int cap) {
  const int s_floor = 23 - level;
  uint32_t cur = 0;
  int i = 0, np = 0;
  uint32_t step_no = 0;
  while (cur < (1u << 23) && i < n - 1) {
    const float va = v[i], xa = orc_logf(va);
    /* the target: the longest aligned step whose chord holds within eps at every run sample it spans */
    int best = s_floor, j = i;
    for (int s = s_floor + 1; s <= 23; ++s) {
      if (cur & ((1u << s) - 1u)) break;
      const uint32_t hi = cur + (1u << s);
      while (j < n - 1 && (uint32_t)(t[j] - t_w) < hi) ++j;
      if ((uint32_t)(t[j] - t_w) != hi) break;
      const float vb = v[j], step = (float)(1u << s);
      int ok = 1;
      for (int k = i + 1; k < j && ok; ++k) {
        const float lin = va + (vb - va) * ((float)((uint32_t)(t[k] - t_w) - cur) / step);
        if (!(fabsf(orc_logf(v[k]) - orc_logf(lin)) <= eps)) ok = 0;
      }
      if (!ok) break;
      best = s;
    }
    if (np < cap) {
      float f[16];
      orc_step_features(w->hx, w->gaps, xa, f);
      for (int k = 0; k < 16; ++k) x_out[np * 16 + k] = orc_bf16(f[k]);
      y_out[np] = (float)(best - sh);
      key_out[np] = ((uint64_t)pixel << 32) | ((uint64_t)window << 11) | step_no;
    }
    ++np;
    uint32_t d[4];
    orc_draw(seed, 0x0090u, 0u, pixel, ((uint64_t)window << 11) | step_no, d);
    const uint32_t u = d[0] & 7u;
    int s_step = best - (u < 4u ? 0 : (u < 6u ? 1 : (int)u - 4));
    if (s_step < s_floor) s_step = s_floor;
    const uint32_t hi = cur + (1u << s_step);
    while (i < n - 1 && (uint32_t)(t[i] - t_w) < hi) ++i;
    walk_push(w, xa, va, s_step);
    cur = hi;
    ++step_no;
  }
  return np;
}

int64_t orc_learned_window(const orc_field* f, const orc_rules* r, int64_t t_w, uint32_t x, uint32_t y, int level,
                           float carried, orc_walk* w, const int32_t* steps, int n_steps, int64_t* t_out,
                           float* v_out, size_t cap) {
  sampler_ctx c = {f, r, t_w, x, y, t_out, v_out, cap, 0};
  const int s_floor = 23 - level;
  const uint32_t min_split = (uint32_t)(2 * r->min_dt_ns);
  uint32_t cur = 0;
  float vc = carried;
  int k = 0;
  while (cur < (1u << 23)) {
    if (k >= n_steps) return -1;
    const int s = steps[k++];
    if (s < s_floor || s > 23 || (cur & ((1u << s) - 1u)) != 0u) return -2;
    const uint32_t dt = 1u << s, hi = cur + dt;
    const float vb = orc_field_eval(f, x, y, t_w + hi);
    if (dt >= min_split && !(w->valid && (int)(w->gaps & 0xffu) == s && !exceeds(r, w->pv, vc, vb))) {
      const uint32_t g = cur + (dt >> 1);
      const float vm = orc_field_eval(f, x, y, t_w + g);
      const int bad = exceeds(r, vc, vm, vb);
      if (bad && (int64_t)(g - cur) >= 2 * r->min_dt_ns) refine(&c, cur, g, vc, vm, 1, 0);
      emit(&c, g, vm);
      if (bad && (int64_t)(hi - g) >= 2 * r->min_dt_ns) refine(&c, g, hi, vm, vb, 1, 0);
    }
    emit(&c, hi, vb);
    walk_push(w, orc_logf(vc), vc, s);
    cur = hi;
    vc = vb;
  }
  return k == n_steps ? (int64_t)c.n : -3;
}
