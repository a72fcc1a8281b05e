// Host build of the device's cascade processors (ballasim_b200/csrc/cascade.cuh, lattice.cuh) and noise tables
// (noise_build.h), for CPU parity tests against the reference's fp32 kernel: the same per-pixel loops over CSR runs
// as advance_runs_cascade_kernel and advance_runs_lattice_kernel, with g++ and -ffp-contract=off in place of nvcc
// and --fmad=false.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "cascade.cuh"
#include "lattice.cuh"
#include "noise_build.h"
#include "stationary.h"

using namespace bs;

namespace {

struct VecSink {
  std::vector<RawEvent>* out;
  void push(const RawEvent& e) { out->push_back(e); }
};

struct Host {
  uint32_t n;
  std::vector<PixelMapRegs> maps;
  std::vector<float> phi0;
  std::vector<PixelRegs> st;
  std::vector<CascadeRegs> cq;
  SensorConsts k{};
  CascadeConsts cc{};
  int64_t t_state = 0;
  std::vector<RawEvent> events;
  uint64_t substeps = 0, attempts = 0, leaves = 0;
};

}  // namespace

extern "C" {

// consts: k, a2, a3, tau_o, tau_sf, eps_accept, eps_drop, eps_pl_base, eps_ci, label_cut, irr_max.
void* hc_create(uint32_t n, const float* on, const float* off, const float* leak, const float* dark,
                const float* phi0, float scale, const float* consts, int ideal_reset, int64_t refractory_ns) {
  auto* h = new Host;
  h->n = n;
  h->maps.resize(n);
  h->phi0.assign(phi0, phi0 + n);
  for (uint32_t p = 0; p < n; ++p) {
    h->maps[p] = PixelMapRegs{on[p], off[p], leak[p], dark[p], scale, 0.0, 0.0};
  }
  h->cc = CascadeConsts{consts[0], consts[1], consts[2], consts[3], consts[4], consts[5], consts[6], consts[7]};
  h->k.eps_ci = consts[8];
  h->k.label_cut = consts[9];
  h->k.irr_max = consts[10];
  h->k.ideal_reset = ideal_reset;
  h->k.refractory_ns = refractory_ns;
  h->k.noise = 0;
  h->st.resize(n);
  h->cq.resize(n);
  return h;
}

void hc_destroy(void* hp) { delete static_cast<Host*>(hp); }

void hc_init(void* hp, int64_t t0, const float* irr0) {
  Host& h = *static_cast<Host*>(hp);
  for (uint32_t p = 0; p < h.n; ++p) {
    const float v = clamp_irr(irr0[p], h.k.irr_max);
    pixel_init(h.st[p], h.maps[p], h.k, p, t0, v, h.phi0[p]);
    cascade_init(h.cq[p], h.st[p]);
  }
  h.t_state = t0;
}

// One call: rows (ids[i], row_start[i], row_count[i]) of (t, irr) samples, then every pixel to t_end.
void hc_advance(void* hp, const uint32_t* ids, size_t n_ids, const int64_t* t, const float* irr,
                const int64_t* row_start, const int32_t* row_count, int64_t t_end) {
  Host& h = *static_cast<Host*>(hp);
  std::vector<int32_t> row_of(h.n, -1);
  for (size_t i = 0; i < n_ids; ++i) row_of[ids[i]] = static_cast<int32_t>(i);
  VecSink sink{&h.events};
  for (uint32_t p = 0; p < h.n; ++p) {
    PixelRegs& s = h.st[p];
    PixelCounters c;
    CascadeCounters cn;
    CascadeProc<VecSink> proc{s, h.cq[p], h.maps[p], h.k, h.cc, p, sink, c, cn};
    int64_t prev_t = h.t_state;
    float prev_v = s.held;
    const int32_t row = row_of[p];
    int32_t cnt = 0;
    if (row >= 0) {
      cnt = row_count[row];
      for (int32_t i = 0; i < cnt; ++i) {
        const int64_t ti = t[row_start[row] + i];
        const float vi = clamp_irr(irr[row_start[row] + i], h.k.irr_max);
        if (i == 0 && ti == h.t_state) {
          prev_v = vi;
          continue;
        }
        proc.segment(Segment{prev_t, ti, prev_v, vi}, prev_t, ti);
        prev_t = ti;
        prev_v = vi;
      }
    }
    proc.segment(Segment{prev_t, kForever, prev_v, prev_v}, prev_t, t_end);
    if (row >= 0 && cnt > 0) s.held = prev_v;
    h.substeps += cn.substeps;
    h.attempts += cn.attempts;
    h.leaves += c.leaves;
  }
  h.t_state = t_end;
}

size_t hc_event_count(void* hp) { return static_cast<Host*>(hp)->events.size(); }

void hc_take(void* hp, RawEvent* out) {
  Host& h = *static_cast<Host*>(hp);
  if (!h.events.empty()) std::memcpy(out, h.events.data(), h.events.size() * sizeof(RawEvent));
  h.events.clear();
}

// The cascade state of every pixel: z, x1, s2, s3, tv (5 floats per pixel).
void hc_state(void* hp, float* out) {
  Host& h = *static_cast<Host*>(hp);
  for (uint32_t p = 0; p < h.n; ++p) {
    const CascadeRegs& q = h.cq[p];
    const float v[5] = {q.z, q.x1, q.s2, q.s3, q.tv};
    std::memcpy(out + 5 * p, v, sizeof v);
  }
}

void hc_stats(void* hp, uint64_t* out) {
  Host& h = *static_cast<Host*>(hp);
  out[0] = h.substeps;
  out[1] = h.attempts;
  out[2] = h.leaves;
}

// The special functions alone, for bitwise checks against the reference's: which 0 expm1, 1..5 resid_exp(j = which
// - 1), 6 erfcx, 7 dawson, 8 z_step (x: z0, I0, I1, h, k per entry, 5 floats).
void hc_special(int which, const float* x, size_t n, float* out) {
  for (size_t i = 0; i < n; ++i) {
    if (which == 0) out[i] = expm1_f(x[i]);
    else if (which <= 5) out[i] = resid_exp_f(which - 1, x[i]);
    else if (which == 6) out[i] = erfcx_f(x[i]);
    else if (which == 7) out[i] = dawson_f(x[i]);
    else out[i] = z_step(x[5 * i], x[5 * i + 1], x[5 * i + 2], x[5 * i + 3], x[5 * i + 4]);
  }
}

// This build's noise tables (noise_build.h): copies up to cap floats; returns n_nodes * stride.
int64_t hc_noise_table(double kq, double a2, double a3, double sigma_o, int levels, int split, float* out,
                       size_t cap) {
  const NoiseTablesH t = build_noise_tables(NoiseModelH{kq, a2, a3, sigma_o, levels, split != 0});
  std::memcpy(out, t.data.data(), std::min(cap, t.data.size()) * sizeof(float));
  return static_cast<int64_t>(t.data.size());
}

// ---- the cascade with its noise lattice (lattice.cuh) ----
namespace {
struct HostLattice {
  Host base;
  NoiseTablesH tables;
  NoiseTableDev view{};
  std::vector<LatticeRegs> lat;
};
}  // namespace

// lat: kq, sigma_o, margin_z, a2 = 1 / tau_o, a3 = 1 / tau_sf, transient (0 or 1) (fp64); levels; seed; camera.
void* hl_create(uint32_t n, const float* on, const float* off, const float* leak, const float* dark, const float* phi0,
                float scale, const float* consts, int ideal_reset, int64_t refractory_ns, const double* lat, int levels,
                uint64_t seed, uint32_t camera) {
  auto* h = new HostLattice;
  Host* b = static_cast<Host*>(hc_create(n, on, off, leak, dark, phi0, scale, consts, ideal_reset, refractory_ns));
  h->base = std::move(*b);
  delete b;
  h->base.k.seed = seed;
  h->base.k.camera = camera;
  h->tables = build_noise_tables(NoiseModelH{lat[0], lat[3], lat[4], lat[1], levels, lat[5] != 0.0});
  h->view = NoiseTableDev{h->tables.data.data(), h->tables.n_nodes, h->tables.stride, levels,
                          static_cast<float>(kNoiseLnA1Min), static_cast<float>(h->tables.inv_dln),
                          static_cast<float>(lat[2]), lat[5] != 0.0 ? 1 : 0};
  h->lat.resize(n);
  return h;
}

void hl_destroy(void* hp) { delete static_cast<HostLattice*>(hp); }

void hl_init(void* hp, int64_t t0, const float* irr0) {
  HostLattice& h = *static_cast<HostLattice*>(hp);
  Host& b = h.base;
  VecSink sink{&b.events};
  for (uint32_t p = 0; p < b.n; ++p) {
    const float v = clamp_irr(irr0[p], b.k.irr_max);
    pixel_init(b.st[p], b.maps[p], b.k, p, t0, v, b.phi0[p]);
    cascade_init(b.cq[p], b.st[p]);
    PixelCounters c;
    CascadeCounters cn;
    const RunInput in{t0, v, nullptr, nullptr, 0, 0, b.k.irr_max};
    LatticeProc<VecSink> proc{b.st[p], b.cq[p], h.lat[p], b.maps[p], b.k, b.cc, h.view, p, sink, c, cn, in};
    proc.init(t0, b.phi0[p]);
  }
  b.t_state = t0;
}

// The stationary start after hl_init (stationary.h): maps64 = theta_on, theta_off, leak (fp64, n each); st = kq, a2,
// a3, sigma_o, k (A^-1 s^-1), the leak rate at the temperature; burnin_ns; probe_pixels.
void hl_stationary(void* hp, int64_t t0, const float* frame, const double* maps64, const double* st, int64_t burnin_ns,
                   int32_t probe_pixels) {
  HostLattice& h = *static_cast<HostLattice*>(hp);
  Host& b = h.base;
  std::vector<HostPixel> px(b.n);
  for (uint32_t p = 0; p < b.n; ++p) px[p] = HostPixel{b.st[p], b.cq[p], h.lat[p]};
  StationaryInputs in{b.maps.data(), maps64, maps64 + b.n, maps64 + 2 * b.n, b.phi0.data(), frame, b.k, b.cc, h.view,
                      NoiseModelH{st[0], st[1], st[2], st[3], h.view.levels, h.view.transient != 0}, st[4], st[5],
                      burnin_ns, probe_pixels};
  stationary_start(px, in, t0);
  for (uint32_t p = 0; p < b.n; ++p) {
    b.st[p] = px[p].s;
    b.cq[p] = px[p].q;
    h.lat[p] = px[p].L;
  }
}

void hl_advance(void* hp, const uint32_t* ids, size_t n_ids, const int64_t* t, const float* irr,
                const int64_t* row_start, const int32_t* row_count, int64_t t_end) {
  HostLattice& h = *static_cast<HostLattice*>(hp);
  Host& b = h.base;
  std::vector<int32_t> row_of(b.n, -1);
  for (size_t i = 0; i < n_ids; ++i) row_of[ids[i]] = static_cast<int32_t>(i);
  VecSink sink{&b.events};
  for (uint32_t p = 0; p < b.n; ++p) {
    const int32_t row = row_of[p];
    const int32_t cnt = row >= 0 ? row_count[row] : 0;
    const int64_t* tp = row >= 0 ? t + row_start[row] : nullptr;
    const float* vp = row >= 0 ? irr + row_start[row] : nullptr;
    const int32_t skip = cnt > 0 && tp[0] == b.t_state ? 1 : 0;
    const RunInput in{b.t_state, b.st[p].held, tp, vp, cnt, skip, b.k.irr_max};
    PixelCounters c;
    CascadeCounters cn;
    LatticeProc<VecSink> proc{b.st[p], b.cq[p], h.lat[p], b.maps[p], b.k, b.cc, h.view, p, sink, c, cn, in};
    proc.resume();
    proc.advance(t_end);
    b.substeps += cn.substeps;
    b.leaves += c.leaves;
  }
  b.t_state = t_end;
}

size_t hl_event_count(void* hp) { return static_cast<HostLattice*>(hp)->base.events.size(); }
void hl_take(void* hp, RawEvent* out) { hc_take(&static_cast<HostLattice*>(hp)->base, out); }

}  // extern "C"
