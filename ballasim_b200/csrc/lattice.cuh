// The cascade photoreceptor with its in-path noise lattice (photoreceptor = cascade, noise = true; frozen or transient
// diffusion):
// BallaSim's default sensor model, restated for the device.
//
// The linearized noise n = (n1, n2, n3) lives on a lattice of cells of 2^16 ns (src/sensor/noise.h,
// src/sensor/pixel.h:1266-1455): on entering a cell its frozen rate a1 is the exact cell average of k u, from a
// z-only look-ahead over the cell's input (held after the last sample); n at the cell's end is drawn from n at its
// start with the tabulated transition (lattice_step), and the cell's n3 is the cubic Hermite of its nodes. Each
// sub-step is tested against the cell's level-0 exclusion hull (Delta widened by the tabulated margin); where that
// cannot exclude a crossing, a time-ordered depth-first walk refines the cell's Gaussian bridge tree (midpoints
// drawn from their parents' endpoints, keyed by the absolute node time) down to the leaf level, whose leaves are
// searched exactly (cascade_search). Events carry the noise's share dn = n3(t) - n3_ref. Every draw is
// Philox(seed, purpose, camera, pixel, node time): noise and events do not depend on the sample schedule.
//
// The processor reads its input as the reference's kernel does (a run with the held sample at the model time,
// random access for the look-ahead) and runs the general path for every cell: the reference's quiet-cell shortcut
// performs the same operations (pixel.h:1399-1406, the same bits), but on the device it splits a warp between two
// code paths, which measured slower. Like the reference's device kernels, the table blocks are interpolated at every
// draw rather than kept per rate (keeping them raised the kernel to 255 registers and measured slower); the settled
// rate of the last z is kept (settled_rate's memo, pixel.h:1320-1333).
#pragma once

#include "cascade.cuh"
#include "noise_build.h"

namespace bs {

constexpr uint32_t kPurposeNoise = 0x0010, kPurposeNoiseInit = 0x0011;

// NoiseTableView<float> (noise_tables.h:99-107): the tables in device (or host) memory.
struct NoiseTableDev {
  const float* data;
  int32_t n_nodes, stride, levels;
  float ln_a1_min, inv_dln, margin_z;
  int32_t transient;  // accuracy.noise_diffusion transient: the tables hold the split blocks
};

// The lattice's part of a pixel's state (PixelState nk, nk1, ln_a1, cell, have_k1 and rho = 1 + rho_m1; fp32 values).
struct LatticeRegs {
  float nk[3], nk1[3];
  float ln_a1;
  int64_t cell;
  uint32_t have_k1;
  float rho;  // the cell's diffusion ratio (1 under frozen diffusion; rho - 1 is exact in fp32)
};

// ---------------------------------------------------------------------------------------------
// Draws (noise.h:26-45) and fp32 sincos (src/core/pmath/trig.h:81-156)
// ---------------------------------------------------------------------------------------------
BS_HD void sincos_f(float x, float* s, float* c) {
  if (!(fabs_f(x) <= 6000.0f)) {
    *s = *c = u2f(0x7fc00000u);
    return;
  }
  if (x == 0.0f) {
    *s = x;
    *c = 1.0f;
    return;
  }
  const float k = rint_f(x * 0x1.45f306p-1f);
  const float r = k == 0.0f ? x : ((x - k * 0x1.922p+0f) - k * -0x1.2aep-18f) - k * -0x1.de973ep-31f;
  const float z = r * r;
  // Taylor coefficients 1/9!, 1/7!, 1/5!, 1/3! and 1/10!, 1/8!, 1/6!, 1/4! as the reference's fp32 kernel has them
  // (its 1/5! is one float below the nearest).
  float ps = 0x1.71de3ap-19f;
  ps = ps * z - 0x1.a01a02p-13f;
  ps = ps * z + 0x1.111110p-7f;
  ps = ps * z - 0x1.555556p-3f;
  const float sr = r + (r * z) * ps;
  float pc = -0x1.27e4fcp-22f;
  pc = pc * z + 0x1.a01a02p-16f;
  pc = pc * z - 0x1.6c16c2p-10f;
  pc = pc * z + 0x1.555556p-5f;
  const float cr = (1.0f - 0.5f * z) + (z * z) * pc;
  switch (static_cast<int>(k) & 3) {
    case 0: *s = sr; *c = cr; break;
    case 1: *s = cr; *c = -sr; break;
    case 2: *s = -sr; *c = -cr; break;
    default: *s = -cr; *c = sr; break;
  }
}

BS_HD float open_uniform_f(uint32_t u) { return (static_cast<float>(u >> 9) + 0.5f) * 0x1p-23f; }

// Three standard normals from one Philox draw (Box-Muller).
static BS_COLD void normals3_f(uint64_t seed, uint32_t purpose, uint32_t camera, uint32_t pixel, uint64_t index,
                               float* out) {
  const U4 r = draw(seed, purpose, camera, pixel, index);
  const float u0 = open_uniform_f(r.v[0]), u1 = open_uniform_f(r.v[1]);
  const float u2 = open_uniform_f(r.v[2]), u3 = open_uniform_f(r.v[3]);
  const float two_pi = static_cast<float>(0x1.921fb54442d18p+2);
  const float r0 = sqrt_f(-2.0f * log_f(u0)), r1 = sqrt_f(-2.0f * log_f(u2));
  float s0, c0, s1, c1;
  sincos_f(two_pi * u1, &s0, &c0);
  sincos_f(two_pi * u3, &s1, &c1);
  out[0] = r0 * c0;
  out[1] = r0 * s0;
  out[2] = r1 * c1;
}

// ---------------------------------------------------------------------------------------------
// Table lookups and the lattice's linear algebra (noise_tables.h:113-136, noise.h:48-189)
// ---------------------------------------------------------------------------------------------
struct NoisePosF {
  int i;
  float f;
};

BS_HD NoisePosF noise_pos(const NoiseTableDev& v, float ln_a1) {
  float x = (ln_a1 - v.ln_a1_min) * v.inv_dln;
  const float x_max = static_cast<float>(v.n_nodes - 1);
  x = x > 0.0f ? (x < x_max ? x : x_max) : 0.0f;
  int i = static_cast<int>(x);
  if (i > v.n_nodes - 2) i = v.n_nodes - 2;
  return {i, x - static_cast<float>(i)};
}

BS_HD void noise_lookup(const NoiseTableDev& v, NoisePosF p, int offset, int count, float* out) {
  const float* a = v.data + static_cast<int64_t>(p.i) * v.stride + offset;
  const float* b = a + v.stride;
  for (int j = 0; j < count; ++j) out[j] = a[j] + p.f * (b[j] - a[j]);
}

BS_HD void lower3_mul(const float* L, const float* x, float* y) {
  y[0] = L[0] * x[0];
  y[1] = L[1] * x[0] + L[2] * x[1];
  y[2] = L[3] * x[0] + L[4] * x[1] + L[5] * x[2];
}

BS_HD void lattice_step(const float* phi, const float* chol, const float* x, const float* xi, float* x_next) {
  float a[3], b[3];
  lower3_mul(phi, x, a);
  lower3_mul(chol, xi, b);
  for (int i = 0; i < 3; ++i) x_next[i] = a[i] + b[i];
}

// x_m = A x_L + B x_R + L xi; blk = A (9), B (9), L (6).
BS_HD void bridge_midpoint(const float* blk, const float* xl, const float* xr, const float* xi, float* xm) {
  float c[3];
  lower3_mul(blk + 18, xi, c);
  for (int i = 0; i < 3; ++i) {
    xm[i] = (blk[3 * i] * xl[0] + blk[3 * i + 1] * xl[1] + blk[3 * i + 2] * xl[2]) +
            (blk[9 + 3 * i] * xr[0] + blk[9 + 3 * i + 1] * xr[1] + blk[9 + 3 * i + 2] * xr[2]) + c[i];
  }
}

// Cubic Hermite of n3 on a node of h seconds with the exact end slopes n3' = a3 (n2 - n3).
BS_HD void noise_hermite(const float* xl, const float* xr, float a3, float h, float* c) {
  const float dl = a3 * (xl[1] - xl[2]), dr = a3 * (xr[1] - xr[2]);
  const float delta = (xr[2] - xl[2]) / h;
  c[0] = xl[2];
  c[1] = dl;
  c[2] = (3.0f * delta - 2.0f * dl - dr) / h;
  c[3] = (dl + dr - 2.0f * delta) / (h * h);
}

// Exclusion margin z sigma_br + g |W (x_L, x_R)| of a node (m: sigma_br, g, W packed).
BS_HD float noise_margin(const float* m, float z, const float* xl, const float* xr) {
  const float e[6] = {xl[0], xl[1], xl[2], xr[0], xr[1], xr[2]};
  const float* W = m + 2;
  float norm2 = 0.0f;
  int idx = 0;
  for (int i = 0; i < 6; ++i) {
    float s = 0.0f;
    for (int j = 0; j <= i; ++j) s = s + W[idx++] * e[j];
    norm2 = norm2 + s * s;
  }
  return z * m[0] + m[1] * sqrt_f(norm2);
}

BS_HD int64_t level_length(int level) { return kNoiseCellNs >> level; }

// ---------------------------------------------------------------------------------------------
// Transient diffusion (noise.h:70-160, pixel.h:420-560): a cell whose input-node diffusion is rho D1 has
// Q = rho Q1 + Q2; the kernel factors it and forms its bridges in information form.
// ---------------------------------------------------------------------------------------------
BS_HD void lower3_tmul(const float* L, const float* x, float* y) {
  y[0] = L[0] * x[0] + L[1] * x[1] + L[3] * x[2];
  y[1] = L[2] * x[1] + L[4] * x[2];
  y[2] = L[5] * x[2];
}

// Lower Cholesky factor of a packed symmetric PSD 3x3; a pivot at or below a tiny fraction of the trace is 0 with its
// column.
BS_HD void chol3_f(const float* q, float* c) {
  const float tiny = (fabs_f(q[0]) + fabs_f(q[2]) + fabs_f(q[5])) * static_cast<float>(1e-20);
  float d = q[0];
  c[0] = d > tiny ? sqrt_f(d) : 0.0f;
  c[1] = c[0] > 0.0f ? q[1] / c[0] : 0.0f;
  c[3] = c[0] > 0.0f ? q[3] / c[0] : 0.0f;
  d = q[2] - c[1] * c[1];
  c[2] = d > tiny ? sqrt_f(d) : 0.0f;
  c[4] = c[2] > 0.0f ? (q[4] - c[3] * c[1]) / c[2] : 0.0f;
  d = q[5] - c[3] * c[3] - c[4] * c[4];
  c[5] = d > tiny ? sqrt_f(d) : 0.0f;
}

BS_HD void split_chol(const float* q12, float rho, float* c) {
  float q[6];
  for (int i = 0; i < 6; ++i) q[i] = rho * q12[i] + q12[6 + i];
  chol3_f(q, c);
}

// The midpoint of a node with ratio rho from the half-node's block (Phi_l, Q1_l, Q2_l): precision J = Q^-1 +
// Phi^T Q^-1 Phi, mean J^-1 (Q^-1 Phi x_L + Phi^T Q^-1 x_R), drawn as U^-T (U^-1 b + xi) with U = chol J.
static BS_COLD void bridge_midpoint_split(const float* blk, float rho, const float* xl, const float* xr,
                                          const float* xi, float* xm) {
  const float* phi = blk;
  float c[6];
  split_chol(blk + 6, rho, c);
  float n[6];
  n[0] = 1.0f / c[0];
  n[2] = 1.0f / c[2];
  n[5] = 1.0f / c[5];
  n[1] = -c[1] * n[0] * n[2];
  n[4] = -c[4] * n[2] * n[5];
  n[3] = -(c[3] * n[0] + c[4] * n[1]) * n[5];
  float m[6];
  m[0] = n[0] * phi[0];
  m[1] = n[1] * phi[0] + n[2] * phi[1];
  m[2] = n[2] * phi[2];
  m[3] = n[3] * phi[0] + n[4] * phi[1] + n[5] * phi[3];
  m[4] = n[4] * phi[2] + n[5] * phi[4];
  m[5] = n[5] * phi[5];
  float j[6];
  j[0] = (n[0] * n[0] + n[1] * n[1] + n[3] * n[3]) + (m[0] * m[0] + m[1] * m[1] + m[3] * m[3]);
  j[1] = (n[2] * n[1] + n[4] * n[3]) + (m[2] * m[1] + m[4] * m[3]);
  j[2] = (n[2] * n[2] + n[4] * n[4]) + (m[2] * m[2] + m[4] * m[4]);
  j[3] = n[5] * n[3] + m[5] * m[3];
  j[4] = n[5] * n[4] + m[5] * m[4];
  j[5] = n[5] * n[5] + m[5] * m[5];
  float u[6];
  chol3_f(j, u);
  float a[3], b1[3], b2[3];
  lower3_mul(m, xl, a);
  lower3_tmul(n, a, b1);
  lower3_mul(n, xr, a);
  lower3_tmul(m, a, b2);
  float y[3];
  y[0] = (b1[0] + b2[0]) / u[0];
  y[1] = ((b1[1] + b2[1]) - u[1] * y[0]) / u[2];
  y[2] = ((b1[2] + b2[2]) - u[3] * y[0] - u[4] * y[1]) / u[5];
  for (int i = 0; i < 3; ++i) y[i] = y[i] + xi[i];
  xm[2] = y[2] / u[5];
  xm[1] = (y[1] - u[4] * xm[2]) / u[2];
  xm[0] = (y[0] - u[1] * xm[1] - u[3] * xm[2]) / u[0];
}

// The margin of a node with ratio rho: sigma_br(rho) <= sigma_br(1) sqrt(1 + (rho - 1) f_l) for rho > 1, and the
// mean-mismatch term scaled by sqrt(max(1, rho)).
BS_HD float noise_margin_rho(const float* m, float z, const float* xl, const float* xr, float rho, float f_l) {
  const float e[6] = {xl[0], xl[1], xl[2], xr[0], xr[1], xr[2]};
  const float* W = m + 2;
  float norm2 = 0.0f;
  int idx = 0;
  for (int i = 0; i < 6; ++i) {
    float s = 0.0f;
    for (int jj = 0; jj <= i; ++jj) s = s + W[idx++] * e[jj];
    norm2 = norm2 + s * s;
  }
  const float big = rho > 1.0f ? rho : 1.0f;
  const float s_br = rho > 1.0f ? sqrt_f(1.0f + (rho - 1.0f) * f_l) : 1.0f;
  return z * m[0] * s_br + m[1] * sqrt_f(norm2) * sqrt_f(big);
}

// One input piece's step of J = int over the cell of e^{-2 int_s^te k u} k (I + u) ds (pixel.h:467-489).
BS_HD float diffusion_ramp(float jw, float ikI, float dl, float dkI) {
  const float a = 2.0f * dl;
  const float em = expm1_f(-a);
  float g0, c;
  if (a > static_cast<float>(0.05)) {
    g0 = -em / a;
    c = 1.0f / a - g0 * (1.0f / a + 0.5f);
  } else {
    g0 = 1.0f - a * (0.5f - a * (1.0f / 6.0f));
    c = a * (1.0f / 12.0f - a * (1.0f / 24.0f - a * (1.0f / 80.0f)));
  }
  return jw * (1.0f + em) + (ikI + dl) * g0 + dkI * c;
}

// J over one input piece (pixel.h:494-537): a constant piece in closed form; a ramp in at most 32 sub-pieces, only
// its last 12 units of int k u where longer.
static BS_COLD float diffusion_weight(float jw, float z_a, float z_b, float I_a, float I_b, float ikI, float h,
                                      float k) {
  if (I_a == I_b) {
    const float em = expm1_f(-ikI);
    const float e1 = 1.0f + em, e2 = e1 * e1;
    const float r = z_a * I_a - 1.0f;
    const float d = 1.0f + r * e1;
    const float zr = z_b / z_a;
    const float jp = ((-em) * (2.0f + em) + 3.0f * r * (-em) * e1 + ikI * (r * r) * e2) / (d * d);
    return jw * (e2 / (zr * zr)) + jp;
  }
  float z = z_a, I0 = I_a, hr = h, ik = ikI;
  float dl = log_f(z_b / z_a) + ikI;
  if (dl > 12.0f) {
    const float tail = 12.0f * z_b / k;
    if (tail < h) {
      const float hh = h - tail;
      const float Im = I_a + (I_b - I_a) * (hh / h);
      const float zm = z_step(z_a, I_a, Im, hh, k);
      const float ih = integrated_pole(I_a, Im, hh, k);
      jw = diffusion_ramp(jw, ih, log_f(zm / z_a) + ih, hh * k * (Im - I_a));
      z = zm;
      I0 = Im;
      hr = tail;
      ik = integrated_pole(I0, I_b, hr, k);
      dl = log_f(z_b / z) + ik;
    }
  }
  const float total = ik + dl;
  int n = static_cast<int>(total * 4.0f) + 1;
  n = n < 32 ? n : 32;
  if (n == 1) return diffusion_ramp(jw, ik, dl, hr * k * (I_b - I0));
  const float hs = hr / static_cast<float>(n), dI = (I_b - I0) / static_cast<float>(n), Is = I0;
  for (int i = 0; i < n; ++i) {
    const float I1 = i + 1 == n ? I_b : Is + dI * static_cast<float>(i + 1);
    const float z1 = i + 1 == n ? z_b : z_step(z, I0, I1, hs, k);
    const float ik1 = integrated_pole(I0, I1, hs, k);
    jw = diffusion_ramp(jw, ik1, log_f(z1 / z) + ik1, hs * k * (I1 - I0));
    z = z1;
    I0 = I1;
  }
  return jw;
}

// rho = J / (1 - e^{-2 int k u}) clamped to [1/2, 1e6] and rounded to fp32 (pixel.h:541-547).
BS_HD float diffusion_ratio(float jw, float int_ku) {
  const float den = -expm1_f(-2.0f * int_ku);
  if (!(den > 0.0f) || !finite_f(jw)) return 1.0f;
  const float rho = jw / den;
  return rho < 1e6f ? (rho > 0.5f ? rho : 0.5f) : 1e6f;
}

// The comparand of the reference kernel (pixel.h:312-320).
struct Comparand {
  int64_t t_ref;
  float s3_ref, n3_ref, dr_ref, leak, theta_on, theta_off;
};

// Delta from e0 on sub-step sub with the noise Hermite hc of the node starting at node_t (pixel.h:322-340).
static BS_COLD ExpCubic delta_noise(const SubStep& sub, int64_t e0, const float* hc, int64_t node_t,
                                    const Comparand& c) {
  ExpCubic g = e0 == sub.t_a ? sub.s3 : shifted(sub.s3, static_cast<float>(e0 - sub.t_a) * kNsF);
  float c0 = g.c[0] - c.s3_ref;
  const float d = static_cast<float>(e0 - node_t) * kNsF;
  c0 = c0 + ((hc[0] + d * (hc[1] + d * (hc[2] + d * hc[3]))) - c.n3_ref);
  g.c[1] = g.c[1] + (hc[1] + d * (2.0f * hc[2] + d * (3.0f * hc[3])));
  g.c[2] = g.c[2] + (hc[2] + d * (3.0f * hc[3]));
  g.c[3] = g.c[3] + hc[3];
  g.c[0] = c0 + (c.leak * since_ref(e0, c.t_ref) + c.dr_ref);
  g.c[1] = g.c[1] + c.leak;
  return g;
}

// Can Delta, widened by margin, reach a level on the integers [max(lo, e0), e1) (pixel.h:345-352)?
BS_HD bool may_cross(const ExpCubic& delta, int64_t e0, int64_t e1, int64_t lo, float margin, const Comparand& c) {
  const int64_t k_lo = maxi(lo, e0) - e0, k_hi = e1 - 1 - e0;
  if (k_lo > k_hi) return false;
  const RangeF r = range(delta, static_cast<float>(k_lo) * kNsF, static_cast<float>(k_hi) * kNsF);
  return r.hi + margin >= c.theta_on || r.lo - margin <= -c.theta_off;
}

struct Tri {
  float v[3];
};

// The midpoint of a tree node at `level` (time t_mid) from its endpoints (pixel.h:450-464); a cell with rho != 1
// forms it from the split blocks.
BS_HD void bridge_child(const NoiseTableDev& tab, uint64_t seed, uint32_t camera, uint32_t pixel, NoisePosF pos,
                        float rho, int level, int64_t t_mid, const float* xl, const float* xr, float* xm) {
  float xi[3];
  normals3_f(seed, kPurposeNoise, camera, pixel, static_cast<uint64_t>(t_mid), xi);
  if (rho != 1.0f) {
    float blk[18];
    noise_lookup(tab, pos, NoiseLayoutF{tab.levels, true}.split_level(level), 18, blk);
    bridge_midpoint_split(blk, rho, xl, xr, xi, xm);
    return;
  }
  float blk[24];
  noise_lookup(tab, pos, NoiseLayoutF{tab.levels}.bridge(level), 24, blk);
  bridge_midpoint(blk, xl, xr, xi, xm);
}

// The margin of a level-l node: the table's, or with rho != 1 its bound from the split tables (pixel.h:551-561).
BS_HD float node_margin(const NoiseTableDev& tab, NoisePosF pos, int level, float rho, const float* xl,
                        const float* xr) {
  float m[23];
  noise_lookup(tab, pos, NoiseLayoutF{tab.levels}.margin(level), 23, m);
  if (rho != 1.0f) {
    float f_l;
    noise_lookup(tab, pos, NoiseLayoutF{tab.levels, true}.split_margin(level), 1, &f_l);
    return noise_margin_rho(m, tab.margin_z, xl, xr, rho, f_l);
  }
  return noise_margin(m, tab.margin_z, xl, xr);
}

// n3(t) in the cell from tc0 (nodes nk, nk1, rate ln_a1) by descending the keyed tree (pixel.h:565-594).
static BS_COLD float n3_at(const NoiseTableDev& tab, float a3, uint64_t seed, uint32_t camera, uint32_t pixel,
                           float ln_a1, float rho, Tri nk, Tri nk1, int64_t tc0, int64_t t) {
  if (t == tc0) return nk.v[2];
  if (t == tc0 + kNoiseCellNs) return nk1.v[2];
  const NoisePosF pos = noise_pos(tab, ln_a1);
  float xl[3], xr[3], xm[3];
  for (int i = 0; i < 3; ++i) {
    xl[i] = nk.v[i];
    xr[i] = nk1.v[i];
  }
  int64_t node_t = tc0;
  for (int l = 1; l <= tab.levels; ++l) {
    const int64_t mid = node_t + level_length(l);
    bridge_child(tab, seed, camera, pixel, pos, rho, l, mid, xl, xr, xm);
    if (t == mid) return xm[2];
    if (t < mid) {
      for (int i = 0; i < 3; ++i) xr[i] = xm[i];
    } else {
      for (int i = 0; i < 3; ++i) xl[i] = xm[i];
      node_t = mid;
    }
  }
  float hc[4];
  noise_hermite(xl, xr, a3, static_cast<float>(level_length(tab.levels)) * kNsF, hc);
  const float u = static_cast<float>(t - node_t) * kNsF;
  return hc[0] + u * (hc[1] + u * (hc[2] + u * hc[3]));
}

struct Found {
  bool found, on;
  int64_t t;
  float s3, n3;
  uint32_t leaves;
};

// The time-ordered depth-first walk of the cell [tc0, tc0 + 2^16) for sub-step sub from lo, below a level-0 node
// that may fire (pixel.h:634-725 without the high-pass filter, rho = 1): a non-leaf node is split only where its
// margin-widened hull may reach a level; leaves are searched exactly; the first crossing wins.
static BS_COLD Found walk(const NoiseTableDev& tab, float a3, uint64_t seed, uint32_t camera, uint32_t pixel,
                          float ln_a1, float rho, Tri nk, Tri nk1, int64_t tc0, const SubStep sub, int64_t lo,
                          Comparand c) {
  struct Node {
    int level;
    int64_t t;
    float xl[3], xr[3];
  };
  Found out{false, false, 0, 0.0f, 0.0f, 0};
  const NoisePosF pos = noise_pos(tab, ln_a1);
  Node stack[12];
  int sp = 0;
  Node& root = stack[sp++];
  root.level = 0;
  root.t = tc0;
  for (int i = 0; i < 3; ++i) {
    root.xl[i] = nk.v[i];
    root.xr[i] = nk1.v[i];
  }
  bool top = tab.levels > 0;  // the level-0 node is known not to be excluded
  while (sp > 0) {
    const Node node = stack[--sp];
    const int64_t length = level_length(node.level);
    const int64_t span_lo = maxi(node.t, lo), span_hi = mini(node.t + length, sub.t_b);
    if (span_lo >= span_hi) continue;
    if (node.level < tab.levels) {
      if (!top) {
        float hc[4];
        noise_hermite(node.xl, node.xr, a3, static_cast<float>(length) * kNsF, hc);
        const float margin = node_margin(tab, pos, node.level, rho, node.xl, node.xr);
        const int64_t e0 = maxi(sub.t_a, span_lo), e1 = mini(sub.t_b, span_hi);
        if (e0 >= e1 || !may_cross(delta_noise(sub, e0, hc, node.t, c), e0, e1, lo, margin, c)) continue;
      }
      top = false;
      const int64_t mid = node.t + level_length(node.level + 1);
      float xm[3];
      bridge_child(tab, seed, camera, pixel, pos, rho, node.level + 1, mid, node.xl, node.xr, xm);
      Node& right = stack[sp++];
      right.level = node.level + 1;
      right.t = mid;
      Node& left = stack[sp++];
      left.level = node.level + 1;
      left.t = node.t;
      for (int i = 0; i < 3; ++i) {
        left.xl[i] = node.xl[i];
        left.xr[i] = xm[i];
        right.xl[i] = xm[i];
        right.xr[i] = node.xr[i];
      }
      continue;
    }
    float hc[4];
    noise_hermite(node.xl, node.xr, a3, static_cast<float>(length) * kNsF, hc);
    const int64_t e0 = maxi(sub.t_a, span_lo), e1 = mini(sub.t_b, span_hi);
    if (e0 >= e1) continue;
    ++out.leaves;
    const CascadeHit hit = cascade_search(delta_noise(sub, e0, hc, node.t, c), e0, e1, lo, c.theta_on, c.theta_off);
    if (!hit.found) continue;
    const float u = static_cast<float>(hit.t - node.t) * kNsF;
    out.found = true;
    out.on = hit.on;
    out.t = hit.t;
    out.s3 = sub.s3(static_cast<float>(hit.t - sub.t_a) * kNsF);
    out.n3 = hc[0] + u * (hc[1] + u * (hc[2] + u * hc[3]));
    return out;
  }
  return out;
}

// ---------------------------------------------------------------------------------------------
// Input: a run of samples with the held sample at the model time (pixel.h:1051-1120, one constant group)
// ---------------------------------------------------------------------------------------------
struct RunInput {
  int64_t t_state;
  float held;         // the last sample of the previous call (clamped)
  const int64_t* t;   // n samples, strictly increasing, t[0] >= t_state
  const float* v;     // raw values (clamped on read)
  int32_t n, skip;    // skip = 1 when t[0] == t_state (that sample replaces the held one)
  float irr_max;

  BS_HD int n_aug() const { return 1 + n - skip; }
  BS_HD int64_t time(int i) const { return i == 0 ? t_state : t[i - 1 + skip]; }
  BS_HD float value(int i) const { return i == 0 && skip == 0 ? held : clamp_irr(v[i - 1 + skip], irr_max); }
  BS_HD int segment_at(int64_t tt) const {
    int lo = 0, hi = n_aug() - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) / 2;
      if (time(mid) <= tt) lo = mid;
      else hi = mid - 1;
    }
    return lo;
  }
  BS_HD int segment_of(int seg, int64_t tt) const {
    const int last = n_aug() - 1;
    while (seg < last && time(seg + 1) <= tt) ++seg;
    return seg;
  }
  BS_HD int64_t segment_end(int seg) const { return seg + 1 < n_aug() ? time(seg + 1) : kForever; }
  BS_HD float group_value(int seg, int64_t tt) const {
    if (seg + 1 >= n_aug()) return value(seg);
    const int64_t t0 = time(seg), t1 = time(seg + 1);
    const float f = static_cast<float>(tt - t0) / static_cast<float>(t1 - t0);
    const float v0 = value(seg), v1 = value(seg + 1);
    return v0 + (v1 - v0) * f;
  }
};

// ---------------------------------------------------------------------------------------------
// The processor
// ---------------------------------------------------------------------------------------------
// In: the input view (RunInput, or the fused engine's cell buffer), with the same members.
template <class Sink, class In = RunInput>
struct LatticeProc {
  PixelRegs& s;
  CascadeRegs& q;
  LatticeRegs& L;
  const PixelMapRegs& m;
  const SensorConsts& k;
  const CascadeConsts& cc;
  const NoiseTableDev& tab;
  uint32_t pixel;
  Sink& sink;
  PixelCounters& c;
  CascadeCounters& cn;
  const In& in;
  int seg = 0;
  float hc0[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  float margin0 = 0.0f;
  // The settled rate of the last z.
  float settled_z = -1.0f, settled_ln = 0.0f;

  BS_HD Tri nk() const { return Tri{{L.nk[0], L.nk[1], L.nk[2]}}; }
  BS_HD Tri nk1() const { return Tri{{L.nk1[0], L.nk1[1], L.nk1[2]}}; }
  BS_HD Comparand comparand() const {
    return Comparand{s.t_ref, s.s3_ref, s.n3_ref, s.dr_ref, m.leak, m.theta_on, m.theta_off};
  }

  // A resumed call inside a cell: its level-0 hull as the lattice draw left it (pixel.h:1003-1012).
  BS_HD void resume() {
    if (L.have_k1) level0(noise_pos(tab, L.ln_a1));
  }

  // The piece from t within one segment, up to limit (pixel.h:1189-1232, constant groups).
  BS_HD LinearPiece next_piece(int& sg, int64_t t, int64_t limit) const {
    sg = in.segment_of(sg, t);
    const int64_t tb = mini(limit, in.segment_end(sg));
    return LinearPiece{t, tb, m.dark + m.scale * in.group_value(sg, t), m.dark + m.scale * in.group_value(sg, tb)};
  }

  BS_HD void level0(NoisePosF pos) {
    noise_hermite(L.nk, L.nk1, cc.a3, static_cast<float>(kNoiseCellNs) * kNsF, hc0);
    if (tab.levels > 0) margin0 = node_margin(tab, pos, 0, L.rho, L.nk, L.nk1);
  }

  // The lattice draw of n at the cell's end at the cell's rate, and the level-0 hull (pixel.h:1336-1376); a cell with
  // rho != 1 factors rho Q1 + Q2 (split_lattice_step, pixel.h:420-431).
  BS_HD void draw_lattice(int64_t tc1) {
    float xi[3], step[12];
    normals3_f(k.seed, kPurposeNoise, k.camera, pixel, static_cast<uint64_t>(tc1), xi);
    const NoisePosF pos = noise_pos(tab, L.ln_a1);
    if (L.rho != 1.0f) {
      float q12[12], chol[6];
      noise_lookup(tab, pos, NoiseLayoutF::kStepPhi, 6, step);
      noise_lookup(tab, pos, NoiseLayoutF{tab.levels, true}.split_step(), 12, q12);
      split_chol(q12, L.rho, chol);
      lattice_step(step, chol, L.nk, xi, L.nk1);
    } else {
      noise_lookup(tab, pos, NoiseLayoutF::kStepPhi, 12, step);
      lattice_step(step, step + 6, L.nk, xi, L.nk1);
    }
    level0(pos);
    L.have_k1 = 1;
  }

  // A settled pixel under constant input for the whole cell: a1 = k u = k / z (pixel.h:1320-1333).
  BS_HD void settled_rate(int64_t t, float pre, int64_t tc1) {
    L.rho = 1.0f;  // settled: u = I, the transient diffusion is the frozen one
    if (pre == 0.0f && q.z == settled_z) {
      L.ln_a1 = settled_ln;
      return;
    }
    const float h_cell = static_cast<float>(kNoiseCellNs) * kNsF;
    const float int_ku = pre + cc.k * static_cast<float>(tc1 - t) * kNsF / q.z;
    L.ln_a1 = log_f(int_ku / h_cell);
    if (pre == 0.0f) {
      settled_z = q.z;
      settled_ln = L.ln_a1;
    }
  }

  // The cell's frozen rate from a z-only look-ahead to its end (pixel.h:1272-1316 and settled_rate :1320-1333);
  // pre: int k u before t (init only).
  BS_HD void enter_cell(int64_t t, float pre) {
    L.cell = t >> kNoiseCellLog2;
    const int64_t tc1 = (L.cell + 1) * kNoiseCellNs;
    int sg = seg;
    LinearPiece pc = next_piece(sg, t, tc1);
    const CascadeState3 st{q.z, q.s2, q.s3};
    const float h_cell = static_cast<float>(kNoiseCellNs) * kNsF;
    if (pc.t_b == tc1 && pc.I_a == pc.I_b && cascade_settled(cc, st, q.x1, pc.I_a)) {
      settled_rate(t, pre, tc1);
    } else {
      float z = q.z, int_kI = 0.0f;
      // Transient diffusion: J over the cell; before t0 (init) the pixel is settled, which contributes 1 - e^{-2 pre}.
      float jw = 0.0f;
      if (tab.transient && pre > 0.0f) jw = diffusion_weight(jw, 1.0f, 1.0f, 1.0f, 1.0f, pre, 0.0f, 0.0f);
      while (true) {
        const float h = static_cast<float>(pc.t_b - pc.t_a) * kNsF;
        const float z_a = z;
        if (!(pc.I_a == pc.I_b && fabs_f(z * pc.I_a - 1.0f) <= cc.eps_drop)) z = z_step(z, pc.I_a, pc.I_b, h, cc.k);
        const float ikI = integrated_pole(pc.I_a, pc.I_b, h, cc.k);
        int_kI = int_kI + ikI;
        if (tab.transient) jw = diffusion_weight(jw, z_a, z, pc.I_a, pc.I_b, ikI, h, cc.k);
        if (pc.t_b >= tc1) break;
        pc = next_piece(sg, pc.t_b, tc1);
      }
      const float int_ku = pre + log_f(z / q.z) + int_kI;
      L.ln_a1 = log_f(maxr(int_ku / h_cell, static_cast<float>(1e-30)));
      L.rho = tab.transient ? diffusion_ratio(jw, int_ku) : 1.0f;
    }
    draw_lattice(tc1);
  }

  BS_HD void next_cell() {
    for (int i = 0; i < 3; ++i) L.nk[i] = L.nk1[i];
    L.have_k1 = 0;
    ++L.cell;
  }

  BS_HD float n3_here(int64_t t) const {
    return n3_at(tab, cc.a3, k.seed, k.camera, pixel, L.ln_a1, L.rho, nk(), nk1(), L.cell * kNoiseCellNs, t);
  }

  BS_HD void set_reference(int64_t t, float s3, float n3, float offset) {
    s.t_ref = t;
    s.s3_ref = s3;
    s.n3_ref = n3;
    s.dr_ref = offset;
  }

  // The event and the reset (pixel.h:1534-1588) with the noise's share.
  BS_COLD void fire(int64_t t, bool on, float s3, float n3) {
    const float ds = s3 - s.s3_ref;
    const float dn = n3 - s.n3_ref;
    const float l = m.leak * since_ref(t, s.t_ref);
    const float dl = l + s.dr_ref;
    const float D = ds + dn + dl;
    const bool first = (s.flags & kFlagFirstAfterInit) != 0u;
    const uint8_t label = first ? first_label(on, ds, dn, l, k.label_cut) : split_label(ds, dl, D, k.label_cut);
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
      set_reference(t, s3, n3, D - (on ? m.theta_on : -m.theta_off));
      s.t_search = t + 1 + k.refractory_ns;
    } else if (k.refractory_ns == 0) {
      set_reference(t, s3, n3, -k.eps_ci);
      s.t_search = t + 1;
    } else {
      s.blind_until = t + k.refractory_ns;
      s.t_search = s.blind_until + 1;
    }
  }

  // The sub-step against the cell's tree (pixel.h:1601-1650 comparator_tree with handle_blind).
  BS_HD void comparator(const SubStep& sub) {
    const int64_t tc0 = L.cell * kNoiseCellNs;
    while (true) {
      if (s.blind_until != kNotBlind) {
        if (s.blind_until >= sub.t_b) return;
        const int64_t t = s.blind_until;
        const float n3 = n3_here(t);
        set_reference(t, sub.s3(static_cast<float>(t - sub.t_a) * kNsF), n3, -k.eps_ci);
        s.blind_until = kNotBlind;
      }
      const int64_t lo = maxi(s.t_search, sub.t_a);
      if (lo >= sub.t_b) return;
      const Comparand cm = comparand();
      if (tab.levels > 0 && !may_cross(delta_noise(sub, lo, hc0, tc0, cm), lo, sub.t_b, lo, margin0, cm)) {
        s.t_search = maxi(s.t_search, sub.t_b);
        return;
      }
      const Found f = walk(tab, cc.a3, k.seed, k.camera, pixel, L.ln_a1, L.rho, nk(), nk1(), tc0, sub, lo, cm);
      c.leaves += f.leaves;
      if (!f.found) {
        s.t_search = maxi(s.t_search, sub.t_b);
        return;
      }
      fire(f.t, f.on, f.s3, f.n3);
    }
  }

  // [t0, t1) inside one cell: pieces, sub-steps, the comparator (pixel.h:1458-1474).
  BS_HD void run_segment(int64_t t0, int64_t t1) {
    int64_t t = t0;
    while (t < t1) {
      const LinearPiece pc = next_piece(seg, t, t1);
      ++c.pieces;
      int64_t ta = pc.t_a, h_hint = 0;
      while (ta < pc.t_b) {
        SubStep sub;
        ta = cascade_substep(cc, q, s.flags, s.i_scale, pc, ta, h_hint, sub, cn);
        comparator(sub);
      }
      t = pc.t_b;
    }
  }

  // [t_from, t_to) of a call (pixel.h:913-945 advance_slice with noise, the general path): cell by cell. A call may
  // run as consecutive ranges cut at cell boundaries: the same bits.
  BS_HD void advance_range(int64_t t_from, int64_t t_to) {
    seg = in.segment_at(t_from);
    int64_t t = t_from;
    while (t < t_to) {
      if (!L.have_k1) enter_cell(t, 0.0f);
      const int64_t boundary = (L.cell + 1) * kNoiseCellNs;
      const int64_t seg_end = mini(t_to, boundary);
      run_segment(t, seg_end);
      if (seg_end == boundary) next_cell();
      t = seg_end;
    }
  }

  // The call from the model time to t_end; the last sample is then held.
  BS_HD void advance(int64_t t_end) {
    advance_range(in.t_state, t_end);
    if (in.n > 0) s.held = in.value(in.n_aug() - 1);
  }

  // init with noise (pixel.h:819-845): the stationary noise at the cell's first node, the part of the cell before t0
  // as the steady state extended backwards, the reference at t0 on s3 and n3(t0).
  BS_HD void init(int64_t t0, float phi0) {
    L.cell = t0 >> kNoiseCellLog2;
    const int64_t tk = L.cell * kNoiseCellNs;
    float xi[3], chol[6];
    normals3_f(k.seed, kPurposeNoiseInit, k.camera, pixel, static_cast<uint64_t>(tk), xi);
    noise_lookup(tab, noise_pos(tab, log_f(cc.k * s.i_scale)), NoiseLayoutF::kPinfChol, 6, chol);
    lower3_mul(chol, xi, L.nk);
    L.have_k1 = 0;
    L.rho = 1.0f;
    float n3_0;
    if (t0 != tk) {
      seg = in.segment_at(t0);
      enter_cell(t0, cc.k * s.i_scale * static_cast<float>(t0 - tk) * kNsF);
      n3_0 = n3_here(t0);
    } else {
      n3_0 = L.nk[2];
    }
    set_reference(t0, q.s3, n3_0, phi0);
  }
};

}  // namespace bs
