// Host construction of the cascade's noise-lattice tables (src/sensor/noise_tables.cpp:10-411):
// per node of ln a1 on [ln 1e-2, ln 1e9] at 64 nodes per decade, the lattice step Phi(h0) and chol Q(h0), chol of
// the stationary covariance, per tree level l = 1..L the midpoint bridge (A_m, K, chol Sigma_m) of a node of
// h0 / 2^(l-1), and per level l = 0..L-1 the exclusion margin (sigma_br, g, W = chol(C_ee)^-1 packed).
//
// The linearized noise n = (n1, n2, n3) obeys dn = A n dt + G dW, A = [[-a1, 0, 0], [a2, -a2, 0], [0, a3, -a3]],
// G G^T = diag(2 k q a1, 2 sigma_o^2 a2, 0). Phi and Q come from a 16-term Taylor series on a step scaled to
// ||A delta|| <= 1/64, then doubled back (Q(2h) = Phi Q Phi^T + Q, Phi(2h) = Phi^2): every term is non-negative.
// All arithmetic is long double in the reference's order of operations (the table is bitwise the reference's: the
// kernels read its float copy), with the host's long-double exp and sqrt.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <vector>

#include "bs_math.cuh"

namespace bs {

constexpr int kNoiseCellLog2 = 16;
constexpr int64_t kNoiseCellNs = int64_t{1} << kNoiseCellLog2;
constexpr double kNoiseLnA1Min = -4.605170185988091;  // ln 1e-2
constexpr double kNoiseLnA1Max = 20.72326583694641;   // ln 1e9
constexpr int kNoiseNodesPerDecade = 64;

// Per-node layout (floats): step Phi 6 (packed lower: 00, 10, 11, 20, 21, 22), step chol 6, P_inf chol 6; then per
// level l = 1..L the bridge A (9, row-major), K (9), chol Sigma (6); then per level l = 0..L-1 the margin sigma_br,
// g and W (21, packed lower row-major). With the split blocks (transient diffusion): Q1_0 and Q2_0 of the lattice
// step (12, symmetric packed as the lower triangle); per level l = 1..L Phi_l (6), Q1_l (6), Q2_l (6); per level
// l = 0..L-1 the input node's largest share f_l of the bridge residual (1).
struct NoiseLayoutF {
  int levels;
  bool split = false;
  static constexpr int kStepPhi = 0, kStepChol = 6, kPinfChol = 12;
  BS_HD int stride() const { return 18 + 47 * levels + (split ? 12 + 19 * levels : 0); }
  BS_HD int bridge(int l) const { return 18 + 24 * (l - 1); }
  BS_HD int margin(int l) const { return 18 + 24 * levels + 23 * l; }
  BS_HD int split_step() const { return 18 + 47 * levels; }
  BS_HD int split_level(int l) const { return 18 + 47 * levels + 12 + 18 * (l - 1); }
  BS_HD int split_margin(int l) const { return 18 + 47 * levels + 12 + 18 * levels + l; }
};

struct NoiseModelH {
  double kq, a2, a3, sigma_o;
  int levels;
  bool split = false;  // also the blocks of transient diffusion
};

namespace noise_host {

using LD = long double;

struct M3 {
  LD m[3][3] = {};
};

inline M3 mul(const M3& a, const M3& b) {
  M3 r;
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) {
      LD s = 0;
      for (int k = 0; k < 3; ++k) s += a.m[i][k] * b.m[k][j];
      r.m[i][j] = s;
    }
  }
  return r;
}
inline M3 tr(const M3& a) {
  M3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r.m[i][j] = a.m[j][i];
  return r;
}
inline M3 add(const M3& a, const M3& b) {
  M3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r.m[i][j] = a.m[i][j] + b.m[i][j];
  return r;
}
inline M3 scale(const M3& a, LD s) {
  M3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r.m[i][j] = a.m[i][j] * s;
  return r;
}
inline M3 identity() {
  M3 r;
  for (int i = 0; i < 3; ++i) r.m[i][i] = 1;
  return r;
}

struct Sys {
  M3 A, GG;
};

// The noise sources of a system: both, the input node's only (D1) or the output node's only (D2); Q1 + Q2 = Q.
enum class Sources { kBoth, kInput, kOutput };

inline Sys system_of(const NoiseModelH& m, LD a1, Sources src = Sources::kBoth) {
  Sys s;
  s.A.m[0][0] = -a1;
  s.A.m[1][0] = m.a2;
  s.A.m[1][1] = -m.a2;
  s.A.m[2][1] = m.a3;
  s.A.m[2][2] = -m.a3;
  if (src != Sources::kOutput) s.GG.m[0][0] = 2 * static_cast<LD>(m.kq) * a1;
  if (src != Sources::kInput) s.GG.m[1][1] = 2 * static_cast<LD>(m.sigma_o) * m.sigma_o * m.a2;
  return s;
}

// Phi(h) and Q(h) by the scaled Taylor series and doubling.
inline void transition(const Sys& sys, LD h, M3& phi, M3& q) {
  LD norm = 0;
  for (int i = 0; i < 3; ++i) {
    LD row = 0;
    for (int j = 0; j < 3; ++j) row += std::fabs(sys.A.m[i][j]);
    norm = std::max(norm, row);
  }
  int halvings = 0;
  LD delta = h;
  while (norm * delta > LD(1) / 64 && halvings < 200) {
    delta /= 2;
    ++halvings;
  }
  const M3 Ad = scale(sys.A, delta);
  M3 term = identity();
  phi = term;
  for (int n = 1; n <= 16; ++n) {
    term = scale(mul(term, Ad), LD(1) / n);
    phi = add(phi, term);
  }
  M3 Mn = sys.GG;
  LD coef = delta;
  q = scale(Mn, coef);
  const M3 At = tr(sys.A);
  for (int n = 1; n <= 16; ++n) {
    Mn = add(mul(sys.A, Mn), mul(Mn, At));
    coef = coef * delta / (n + 1);
    q = add(q, scale(Mn, coef));
  }
  for (int k = 0; k < halvings; ++k) {
    q = add(mul(mul(phi, q), tr(phi)), q);
    phi = mul(phi, phi);
  }
}

// The stationary covariance: the lower bidiagonal Lyapunov equation solved row by row.
inline M3 stationary(const NoiseModelH& m, LD a1) {
  const LD a2 = m.a2, a3 = m.a3;
  M3 p;
  p.m[0][0] = m.kq;
  p.m[1][0] = a2 * p.m[0][0] / (a1 + a2);
  p.m[1][1] = p.m[1][0] + static_cast<LD>(m.sigma_o) * m.sigma_o;
  p.m[2][0] = a3 * p.m[1][0] / (a1 + a3);
  p.m[2][1] = (a3 * p.m[1][1] + a2 * p.m[2][0]) / (a2 + a3);
  p.m[2][2] = p.m[2][1];
  p.m[0][1] = p.m[1][0];
  p.m[0][2] = p.m[2][0];
  p.m[1][2] = p.m[2][1];
  return p;
}

// Cholesky of a symmetric PSD N x N; pivots at or below a tiny fraction of the trace become 0 with their column.
template <int N>
void cholesky(const LD (&a)[N][N], LD (&l)[N][N]) {
  LD trace = 0;
  for (int i = 0; i < N; ++i) trace += std::fabs(a[i][i]);
  const LD tiny = trace * static_cast<LD>(1e-36) + static_cast<LD>(1e-300);
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j) l[i][j] = 0;
  for (int j = 0; j < N; ++j) {
    LD d = a[j][j];
    for (int k = 0; k < j; ++k) d -= l[j][k] * l[j][k];
    d = d > tiny ? d : 0;
    l[j][j] = std::sqrt(d);
    for (int i = j + 1; i < N; ++i) {
      LD s = a[i][j];
      for (int k = 0; k < j; ++k) s -= l[i][k] * l[j][k];
      l[i][j] = l[j][j] > 0 ? s / l[j][j] : 0;
    }
  }
}

// x = (L L^T)^-1 b.
template <int N>
void chol_solve(const LD (&l)[N][N], const LD (&b)[N], LD (&x)[N]) {
  LD y[N];
  for (int i = 0; i < N; ++i) {
    LD s = b[i];
    for (int k = 0; k < i; ++k) s -= l[i][k] * y[k];
    y[i] = l[i][i] > 0 ? s / l[i][i] : 0;
  }
  for (int i = N - 1; i >= 0; --i) {
    LD s = y[i];
    for (int k = i + 1; k < N; ++k) s -= l[k][i] * x[k];
    x[i] = l[i][i] > 0 ? s / l[i][i] : 0;
  }
}

inline void pack_lower3(const M3& m, double* out) {
  out[0] = static_cast<double>(m.m[0][0]);
  out[1] = static_cast<double>(m.m[1][0]);
  out[2] = static_cast<double>(m.m[1][1]);
  out[3] = static_cast<double>(m.m[2][0]);
  out[4] = static_cast<double>(m.m[2][1]);
  out[5] = static_cast<double>(m.m[2][2]);
}

inline M3 sym_chol(const M3& a) {
  LD in[3][3], l[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) in[i][j] = 0.5L * (a.m[i][j] + a.m[j][i]);
  cholesky<3>(in, l);
  M3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r.m[i][j] = l[i][j];
  return r;
}

inline M3 spd_inverse(const M3& a) {
  LD in[3][3], l[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) in[i][j] = 0.5L * (a.m[i][j] + a.m[j][i]);
  cholesky<3>(in, l);
  M3 r;
  for (int j = 0; j < 3; ++j) {
    LD e[3] = {0, 0, 0}, x[3];
    e[j] = 1;
    chol_solve<3>(l, e, x);
    for (int i = 0; i < 3; ++i) r.m[i][j] = x[i];
  }
  return r;
}

// Exclusion margin of a node of length h: the largest bridge residual std of n3 and the largest endpoint-dependent
// mean mismatch g of its cubic Hermite over the node's 19 interior points i / 20, and W = chol(C_ee)^-1.
inline void margin_block(const NoiseModelH& m, const Sys& sys, LD a1, LD h, double* out) {
  const M3 P = stationary(m, a1);
  constexpr int kPoints = 20;
  M3 step, unused;
  transition(sys, h / kPoints, step, unused);
  M3 pw[kPoints + 1];
  pw[0] = identity();
  for (int i = 1; i <= kPoints; ++i) pw[i] = mul(pw[i - 1], step);
  const M3& phi_h = pw[kPoints];
  LD C[6][6];
  const M3 PphiT = mul(P, tr(phi_h)), phiP = mul(phi_h, P);
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) {
      C[i][j] = P.m[i][j];
      C[i][j + 3] = PphiT.m[i][j];
      C[i + 3][j] = phiP.m[i][j];
      C[i + 3][j + 3] = P.m[i][j];
    }
  }
  LD L6[6][6];
  cholesky<6>(C, L6);
  LD sigma_br = 0, g = 0;
  const LD a3 = m.a3;
  for (int iu = 1; iu < kPoints; ++iu) {
    const LD u = static_cast<LD>(iu) / kPoints;
    const M3 cL = mul(pw[iu], P), cR = mul(P, tr(pw[kPoints - iu]));
    LD c[6], w[6];
    for (int j = 0; j < 3; ++j) {
      c[j] = cL.m[2][j];
      c[j + 3] = cR.m[2][j];
    }
    chol_solve<6>(L6, c, w);
    LD var = P.m[2][2];
    for (int j = 0; j < 6; ++j) var -= c[j] * w[j];
    const LD H00 = 2 * u * u * u - 3 * u * u + 1, H10 = u * u * u - 2 * u * u + u;
    const LD H01 = -2 * u * u * u + 3 * u * u, H11 = u * u * u - u * u;
    const LD wh[6] = {0, H10 * h * a3, H00 - H10 * h * a3, 0, H11 * h * a3, H01 - H11 * h * a3};
    LD dw[6], g2 = 0;
    for (int j = 0; j < 6; ++j) dw[j] = w[j] - wh[j];
    for (int i = 0; i < 6; ++i)
      for (int j = 0; j < 6; ++j) g2 += dw[i] * C[i][j] * dw[j];
    sigma_br = std::max(sigma_br, std::sqrt(std::max(var, LD(0))));
    g = std::max(g, std::sqrt(std::max(g2, LD(0))));
  }
  out[0] = static_cast<double>(sigma_br);
  out[1] = static_cast<double>(g);
  LD W[6][6] = {};
  for (int j = 0; j < 6; ++j) {
    W[j][j] = L6[j][j] > 0 ? 1 / L6[j][j] : 0;
    for (int i = j + 1; i < 6; ++i) {
      LD s = 0;
      for (int k = j; k < i; ++k) s -= L6[i][k] * W[k][j];
      W[i][j] = L6[i][i] > 0 ? s / L6[i][i] : 0;
    }
  }
  int idx = 2;
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j <= i; ++j) out[idx++] = static_cast<double>(W[i][j]);
}

// The input node's largest share f = max_t V1 / (V1 + V2) of the bridge residual of n3 on a node of length h, with the
// predictor of margin_block held fixed (noise_tables.cpp:271-325).
inline LD margin_share(const NoiseModelH& m, const Sys& sys, LD a1, LD h) {
  NoiseModelH m1 = m, m2 = m;
  m1.sigma_o = 0;
  m2.kq = 0;
  const M3 P = stationary(m, a1), P1 = stationary(m1, a1), P2 = stationary(m2, a1);
  constexpr int kPoints = 20;
  M3 step, unused;
  transition(sys, h / kPoints, step, unused);
  M3 pw[kPoints + 1];
  pw[0] = identity();
  for (int i = 1; i <= kPoints; ++i) pw[i] = mul(pw[i - 1], step);
  const M3& phi_h = pw[kPoints];
  const auto cee = [&](const M3& Pk, LD (&C)[6][6]) {
    const M3 PphiT = mul(Pk, tr(phi_h)), phiP = mul(phi_h, Pk);
    for (int i = 0; i < 3; ++i) {
      for (int j = 0; j < 3; ++j) {
        C[i][j] = Pk.m[i][j];
        C[i][j + 3] = PphiT.m[i][j];
        C[i + 3][j] = phiP.m[i][j];
        C[i + 3][j + 3] = Pk.m[i][j];
      }
    }
  };
  LD C[6][6], C1[6][6], C2[6][6], L6[6][6];
  cee(P, C);
  cee(P1, C1);
  cee(P2, C2);
  cholesky<6>(C, L6);
  LD f = 0;
  for (int iu = 1; iu < kPoints; ++iu) {
    const auto c_of = [&](const M3& Pk, LD (&c)[6]) {
      const M3 cL = mul(pw[iu], Pk), cR = mul(Pk, tr(pw[kPoints - iu]));
      for (int j = 0; j < 3; ++j) {
        c[j] = cL.m[2][j];
        c[j + 3] = cR.m[2][j];
      }
    };
    LD c[6], c1[6], c2[6], w[6];
    c_of(P, c);
    c_of(P1, c1);
    c_of(P2, c2);
    chol_solve<6>(L6, c, w);
    const auto resid = [&](const M3& Pk, const LD (&ck)[6], const LD (&Ck)[6][6]) {
      LD v = Pk.m[2][2];
      for (int i = 0; i < 6; ++i) {
        v -= 2 * w[i] * ck[i];
        for (int j = 0; j < 6; ++j) v += w[i] * Ck[i][j] * w[j];
      }
      return std::max(v, LD(0));
    };
    const LD v1 = resid(P1, c1, C1), v2 = resid(P2, c2, C2);
    if (v1 + v2 > 0) f = std::max(f, v1 / (v1 + v2));
  }
  return f;
}

}  // namespace noise_host

struct NoiseTablesH {
  int n_nodes = 0, stride = 0, levels = 0;
  double inv_dln = 0;
  std::vector<float> data;  // n_nodes x stride
};

// The tables of one model (noise_tables.cpp:347-408).
inline NoiseTablesH build_noise_tables(const NoiseModelH& model) {
  using namespace noise_host;
  if (model.levels < 0 || model.levels > 10) throw std::invalid_argument("noise tables: levels must lie in [0, 10]");
  NoiseTablesH t;
  t.levels = model.levels;
  const double dln = log_d(10.0) / kNoiseNodesPerDecade;
  t.inv_dln = 1.0 / dln;
  t.n_nodes = static_cast<int>(std::lround((kNoiseLnA1Max - kNoiseLnA1Min) * t.inv_dln)) + 1;
  const NoiseLayoutF lay{model.levels, model.split};
  t.stride = lay.stride();
  std::vector<double> d64(static_cast<size_t>(t.n_nodes) * t.stride, 0.0);
  const LD h0 = static_cast<LD>(kNoiseCellNs) * 1e-9L;
  for (int node = 0; node < t.n_nodes; ++node) {
    const LD a1 = std::exp(static_cast<LD>(kNoiseLnA1Min) + static_cast<LD>(node) * static_cast<LD>(dln));
    double* row = d64.data() + static_cast<size_t>(node) * t.stride;
    const Sys sys = system_of(model, a1);
    std::vector<M3> phis(model.levels + 1), qs(model.levels + 1);
    for (int l = 0; l <= model.levels; ++l) transition(sys, h0 / static_cast<LD>(int64_t{1} << l), phis[l], qs[l]);
    pack_lower3(phis[0], row + NoiseLayoutF::kStepPhi);
    pack_lower3(sym_chol(qs[0]), row + NoiseLayoutF::kStepChol);
    pack_lower3(sym_chol(stationary(model, a1)), row + NoiseLayoutF::kPinfChol);
    for (int l = 1; l <= model.levels; ++l) {
      // The midpoint of a level-(l-1) node given both ends; the parent's covariance is the doubling step.
      const M3& ph = phis[l];
      const M3& qh = qs[l];
      const M3 parent = add(mul(mul(ph, qh), tr(ph)), qh);
      const M3 K = mul(mul(qh, tr(ph)), spd_inverse(parent));
      const M3 Am = add(ph, scale(mul(mul(K, ph), ph), -1));
      const M3 sig = add(qh, scale(mul(mul(K, ph), qh), -1));
      double* b = row + lay.bridge(l);
      for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) {
          b[3 * i + j] = static_cast<double>(Am.m[i][j]);
          b[9 + 3 * i + j] = static_cast<double>(K.m[i][j]);
        }
      }
      pack_lower3(sym_chol(sig), b + 18);
    }
    for (int l = 0; l < model.levels; ++l) {
      margin_block(model, sys, a1, h0 / static_cast<LD>(int64_t{1} << l), row + lay.margin(l));
    }
    if (model.split) {
      const Sys s_in = system_of(model, a1, Sources::kInput), s_out = system_of(model, a1, Sources::kOutput);
      for (int l = 0; l <= model.levels; ++l) {
        M3 phi, q1, q2;
        const LD h = h0 / static_cast<LD>(int64_t{1} << l);
        transition(s_in, h, phi, q1);
        transition(s_out, h, phi, q2);
        double* b = row + (l == 0 ? lay.split_step() : lay.split_level(l));
        if (l > 0) {
          pack_lower3(phis[l], b);
          b += 6;
        }
        pack_lower3(q1, b);
        pack_lower3(q2, b + 6);
      }
      for (int l = 0; l < model.levels; ++l) {
        row[lay.split_margin(l)] =
            static_cast<double>(margin_share(model, sys, a1, h0 / static_cast<LD>(int64_t{1} << l)));
      }
    }
  }
  t.data.resize(d64.size());
  for (size_t i = 0; i < d64.size(); ++i) t.data[i] = static_cast<float>(d64[i]);
  return t;
}

}  // namespace bs
