// The stationary initial state of the cascade with its noise lattice (accuracy.initial_state = stationary;
// src/sensor/sensor_model.cpp:492-700), run on the host after the phase-law init:
//   1. the probe: of the pixels ordered by (ln of the mean photocurrent, index), one per stratum of equal count (the
//      smallest Philox(seed, 0x0012, camera, pixel, t0) word 0 in its stratum) runs its own history: init at
//      t0 - T_b with the phase law and the frame held, advanced to t0 by the pixel kernel (events dropped), with 64
//      snapshots of its comparator over the last 2/3 of T_b; then its reference is re-based at t0 (F034);
//   2. the transfer: every other pixel takes the comparator of its nearest probe in (theta_on, theta_off, ln I,
//      modulated share) at a keyed snapshot (word 1), moved to keep the distance to the probe's nearer level in units
//      of the noise sigma_v(I) (the ratio clamped to [1/2, 2]); a snapshot that would put Delta(t0) on or past a level
//      is skipped for the next one, cyclically; if none fits, the pixel keeps the phase law.
// The histories run this build's lattice processor compiled for the host (the reference also runs them on the host),
// one thread per probe at a time; the features and the transfer are fp64 as in the reference.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <thread>
#include <vector>

#include "lattice.cuh"

namespace bs {

constexpr uint32_t kPurposeStationaryProbe = 0x0012;
constexpr int kSnapshots = 64;

// One pixel's state as the kernels keep it.
struct HostPixel {
  PixelRegs s;
  CascadeRegs q;
  LatticeRegs L;
};

struct StationaryInputs {
  const PixelMapRegs* maps;                                // the kernel's fp32 maps
  const double *theta_on, *theta_off, *leak;               // the fp64 maps
  const float* phi0;
  const float* frame;                                      // the init frame (raw irradiance, one group)
  SensorConsts k;
  CascadeConsts cc;
  NoiseTableDev tab;                                       // host copy of the tables
  NoiseModelH nm;                                          // kq, a2, a3, sigma_o
  double k_param;                                          // SensorParams::k (A^-1 s^-1)
  double leak_rate_at_t;                                   // leak_rate_hz x its Arrhenius factor
  int64_t burnin_ns;                                       // stationary_burnin_ns (0: from the leak rate)
  int32_t probe_pixels;                                    // stationary_probe_pixels
};

// The history length T_b (sensor_model.cpp:482-490, no high-pass filter): 1.5 / R_L clamped to [60 s, 600 s], whole
// noise cells.
inline int64_t probe_history_ns(double leak_rate_at_t, int64_t burnin_ns) {
  int64_t t = burnin_ns;
  if (t == 0) {
    const double r = leak_rate_at_t;
    const double s = r > 0 ? std::min(std::max(1.5 / r, 60.0), 600.0) : 600.0;
    t = static_cast<int64_t>(s * 1e9);
  }
  return std::max<int64_t>(t / kNoiseCellNs, 1) * kNoiseCellNs;
}

struct ProbeFeature {
  double on, off, ln_i, share, sigma;
};

// The transfer's features of a pixel in units of their tolerance (levels 0.01, ln I 0.1, share 0.1) and sigma_v(I)
// (sensor_model.cpp:116-131; constant groups: the modulated share is 0).
inline ProbeFeature probe_feature(const StationaryInputs& in, uint32_t p, const HostPixel& x) {
  const double I = x.s.i_scale;
  const noise_host::M3 P = noise_host::stationary(in.nm, static_cast<noise_host::LD>(in.k_param * I * 1e-15));
  const double cov22 = static_cast<double>(P.m[2][2]);
  return {in.theta_on[p] / 0.01, in.theta_off[p] / 0.01, log_d(I) / 0.1, 0.0 / I / 0.1, std::sqrt(cov22)};
}

struct NullHostSink {
  void push(const RawEvent&) {}
};

struct ProbeSnap {
  int64_t blind_until, t_search;
  double c;
};

// Replaces the phase-law states px (of the pixels 0..n-1, ids = indices) with the stationary start at t0.
inline void stationary_start(std::vector<HostPixel>& px, const StationaryInputs& in, int64_t t0) {
  const size_t n = px.size();
  std::vector<ProbeFeature> f(n);
  for (size_t p = 0; p < n; ++p) f[p] = probe_feature(in, static_cast<uint32_t>(p), px[p]);
  std::vector<uint32_t> eligible(n);
  for (size_t p = 0; p < n; ++p) eligible[p] = static_cast<uint32_t>(p);
  if (eligible.empty()) return;
  std::sort(eligible.begin(), eligible.end(),
            [&](uint32_t a, uint32_t b) { return f[a].ln_i != f[b].ln_i ? f[a].ln_i < f[b].ln_i : a < b; });
  const size_t m = eligible.size();
  const size_t P = std::min(m, static_cast<size_t>(std::max(in.probe_pixels, 0)));
  if (P == 0) return;
  const auto key = [&](uint32_t p, int i) {
    return draw(in.k.seed, kPurposeStationaryProbe, in.k.camera, p, static_cast<uint64_t>(t0)).v[i];
  };
  std::vector<uint32_t> probe(P);
  for (size_t s = 0; s < P; ++s) {
    uint32_t best = eligible[s * m / P], best_key = UINT32_MAX;
    for (size_t i = s * m / P; i < (s + 1) * m / P; ++i) {
      const uint32_t kk = key(eligible[i], 0);
      if (kk < best_key) best = eligible[i], best_key = kk;
    }
    probe[s] = best;
  }
  // The histories: snapshot j at t0 - (63 - j) dt, dt whole cells over the last 2/3 of T_b (the last at t0).
  const int64_t T_b = probe_history_ns(in.leak_rate_at_t, in.burnin_ns);
  const int64_t dt = std::max<int64_t>(T_b * 2 / 3 / (kSnapshots - 1) / kNoiseCellNs, 1) * kNoiseCellNs;
  const int64_t t_p = t0 - std::max<int64_t>(T_b, (kSnapshots - 1) * dt);
  std::vector<HostPixel> hist(P);
  std::vector<ProbeSnap> snap(P * kSnapshots);
  const auto run_probe = [&](size_t i) {
    const uint32_t qid = probe[i];
    const PixelMapRegs& mq = in.maps[qid];
    HostPixel& x = hist[i];
    NullHostSink sink;
    PixelCounters c;
    CascadeCounters cn;
    const float v = clamp_irr(in.frame[qid], in.k.irr_max);
    pixel_init(x.s, mq, in.k, qid, t_p, v, in.phi0[qid]);
    cascade_init(x.q, x.s);
    {
      const RunInput none{t_p, v, nullptr, nullptr, 0, 0, in.k.irr_max};
      LatticeProc<NullHostSink> proc{x.s, x.q, x.L, mq, in.k, in.cc, in.tab, qid, sink, c, cn, none};
      proc.init(t_p, in.phi0[qid]);
    }
    int64_t t = t_p;
    for (int j = 0; j < kSnapshots; ++j) {
      const int64_t t_j = t0 - static_cast<int64_t>(kSnapshots - 1 - j) * dt;
      const RunInput none{t, x.s.held, nullptr, nullptr, 0, 0, in.k.irr_max};
      LatticeProc<NullHostSink> proc{x.s, x.q, x.L, mq, in.k, in.cc, in.tab, qid, sink, c, cn, none};
      proc.resume();
      proc.advance(t_j);
      t = t_j;
      const PixelRegs& s = x.s;
      snap[i * kSnapshots + j] = {s.blind_until == kNotBlind ? kNotBlind : s.blind_until - t_j, s.t_search - t_j,
                                  -static_cast<double>(s.s3_ref) - static_cast<double>(s.n3_ref) +
                                      in.leak[qid] * static_cast<double>(t_j - s.t_ref) * 1e-9 +
                                      static_cast<double>(s.dr_ref)};
    }
    // Re-based at t0 as init's states are (rebase_history, pixel.h:852-865).
    const RunInput none{t0, x.s.held, nullptr, nullptr, 0, 0, in.k.irr_max};
    LatticeProc<NullHostSink> proc{x.s, x.q, x.L, mq, in.k, in.cc, in.tab, qid, sink, c, cn, none};
    x.s.flags = kFlagFirstAfterInit;
    if (x.s.blind_until == kNotBlind) {
      const float n3 = proc.n3_here(t0);
      const float dl = mq.leak * since_ref(t0, x.s.t_ref) + x.s.dr_ref;
      const float delta = (x.q.s3 - x.s.s3_ref) + (n3 - x.s.n3_ref) + dl;
      proc.set_reference(t0, x.q.s3, n3, delta);
    }
  };
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const size_t workers = std::min<size_t>(P, hw);
  std::vector<std::thread> pool;
  for (size_t w = 0; w < workers; ++w) {
    pool.emplace_back([&, w] {
      for (size_t i = w; i < P; i += workers) run_probe(i);
    });
  }
  for (std::thread& th : pool) th.join();
  // The transfer.
  std::vector<int32_t> probe_of(n, -1);
  for (size_t i = 0; i < P; ++i) probe_of[probe[i]] = static_cast<int32_t>(i);
  std::vector<ProbeFeature> pf(P);
  for (size_t i = 0; i < P; ++i) pf[i] = f[probe[i]];
  for (size_t p = 0; p < n; ++p) {
    HostPixel& x = px[p];
    if (probe_of[p] >= 0) {
      x = hist[static_cast<size_t>(probe_of[p])];
      continue;
    }
    const ProbeFeature& a = f[p];
    size_t j = 0;
    double best = INFINITY;
    for (size_t i = 0; i < P; ++i) {
      const ProbeFeature& o = pf[i];
      const double dd = (a.on - o.on) * (a.on - o.on) + (a.off - o.off) * (a.off - o.off) +
                        (a.ln_i - o.ln_i) * (a.ln_i - o.ln_i) + (a.share - o.share) * (a.share - o.share);
      if (dd < best) best = dd, j = i;
    }
    const double r = std::min(std::max(a.sigma / pf[j].sigma, 0.5), 2.0);
    const double n3_0 = x.s.n3_ref, s3_0 = x.q.s3;
    const int first = static_cast<int>((static_cast<uint64_t>(key(static_cast<uint32_t>(p), 1)) * kSnapshots) >> 32);
    const uint32_t qj = probe[j];
    for (int kk = 0; kk < kSnapshots; ++kk) {
      const ProbeSnap& q = snap[j * kSnapshots + (first + kk) % kSnapshots];
      if (q.blind_until != kNotBlind) {  // in the refractory: the release sets the reference
        x.s.t_search = std::max(t0 + q.t_search, t0 + 1);
        x.s.blind_until = t0 + q.blind_until;
        break;
      }
      const double u_on = in.theta_on[qj] - q.c, u_off = in.theta_off[qj] + q.c;
      const double c = u_on <= u_off ? in.theta_on[p] - u_on * r : -in.theta_off[p] + u_off * r;
      const double delta = c + n3_0 + s3_0;
      if (!(delta < in.theta_on[p] && delta > -in.theta_off[p])) continue;
      x.s.t_search = std::max(t0 + q.t_search, t0 + 1);
      x.s.dr_ref = static_cast<float>(delta);
      x.s.blind_until = kNotBlind;
      break;
    }
  }
}

}  // namespace bs
