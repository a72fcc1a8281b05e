// sample_window with a renderer behind a C callback: the reference's host window engine (WindowEngine<Space::kHost>,
// src/engine/window_impl.h:462-714) driving its RenderHook (src/engine/window.h:69-84) with 24-byte SampleRequest
// rows (src/backend/api.h:25-34). Breadth-first over the listed pixels, as the reference schedules it:
//  - the lattice: every pixel's 2^level + 1 slots, slot 0 the carried sample (never rendered), the others in one
//    render call, pixel-major in the listed order and by time within a pixel (BuildRequests, sampling.h:416-434);
//  - round 0's flags of each lattice interval (i - 1, i) from the triples (i - 1, i, i + 1) and (i - 2, i - 1, i)
//    and the signature flip (Round0Flags, sampling.h:471-523);
//  - up to max_refine_levels refinement rounds: one render call for the midpoints of the round's intervals in
//    interval order, then each half flagged by its signature flip or the triple (lo, mid, hi) (HalfFlags,
//    sampling.h:612-678), kept where it can still be split (min_split = 2 min_dt_ns);
//  - the runs: each pixel's samples by time (PixelRuns, sampling.h:764-839); the carried sample becomes the
//    pixel's last lattice slot (t_w + 2^23).
// Each round's eta_L midpoint tests go to the device in one launch (bs_midpoint_eta); rules without the midpoint
// test make no device call. The statistics are the reference's WindowStats counters.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/ballasim_b200.h"

namespace bs {
void set_last_error(const char* msg);  // model.cu: the message bs_last_error() returns
}

namespace {

constexpr int kWindowLog2 = 23;

struct Cancelled : std::runtime_error {
  using std::runtime_error::runtime_error;
};

}  // namespace

struct bs_window {
  int32_t groups = 1;
  std::vector<float> m_min, m_max;
  // the last window's runs and statistics
  std::vector<int64_t> offsets, t;
  std::vector<float> irr;
  uint64_t flagged_signature = 0, flagged_midpoint = 0, refine_cap_hits = 0, render_calls = 0;
  std::vector<uint64_t> samples_by_round;

  // Round scratch: every sample's time offset, owner, irradiance rows and signature, in render order.
  std::vector<uint32_t> dt, owner;
  std::vector<float> rows;
  std::vector<uint64_t> sig;
  std::vector<bs_sample_request> req;
  std::vector<uint32_t> out_index;
  std::vector<float> ea, em, eb, eta;
  std::vector<uint8_t> ex;

  void check_cancel(const volatile int32_t* cancel, const char* where) const {
    if (cancel != nullptr && *cancel != 0) throw Cancelled(std::string(where) + ": cancelled");
  }

  // The triples (a[i], m[i], b[i]) of sample rows: exceeds[i] = eta_L > tol (all false without the midpoint test).
  void exceeds(const bs_window_rules& r, const std::vector<uint32_t>& a, const std::vector<uint32_t>& m,
               const std::vector<uint32_t>& b, std::vector<uint8_t>& out) {
    const size_t n = a.size();
    out.assign(n, 0);
    if (!r.midpoint || n == 0) return;
    const size_t G = static_cast<size_t>(groups);
    ea.resize(n * G);
    em.resize(n * G);
    eb.resize(n * G);
    eta.resize(n);
    for (size_t i = 0; i < n; ++i) {
      std::memcpy(&ea[i * G], &rows[a[i] * G], G * sizeof(float));
      std::memcpy(&em[i * G], &rows[m[i] * G], G * sizeof(float));
      std::memcpy(&eb[i * G], &rows[b[i] * G], G * sizeof(float));
    }
    const bs_status st = bs_midpoint_eta(r.tol, r.dark, groups, m_min.data(), m_max.data(), ea.data(), em.data(),
                                         eb.data(), n, eta.data(), out.data());
    if (st != BS_OK) throw std::runtime_error(bs_last_error());
  }

  // One render call for samples [g0, g1) of the scratch arrays, in that order (out_index = the sample's row).
  void render(int64_t t_w, const uint32_t* ids, const bs_window_rules& r, int shift, uint32_t g0, uint32_t g1,
              bs_render_fn fn, void* user) {
    const size_t n = g1 - g0;
    if (n == 0) return;
    req.resize(n);
    out_index.resize(n);
    for (size_t i = 0; i < n; ++i) {
      const uint32_t g = g0 + static_cast<uint32_t>(i);
      const uint32_t d = dt[g];
      req[i] = bs_sample_request{r.cam, 0, ids[owner[g]], 0, r.subsamples, static_cast<int32_t>(d), d >> shift};
      out_index[i] = g;
    }
    ++render_calls;
    const int32_t rc = fn(user, req.data(), n, out_index.data(), rows.data(), sig.data(), r.subsamples);
    if (rc != 0) throw std::invalid_argument("render: the render callback failed (status " + std::to_string(rc) + ")");
  }

  void run(int64_t t_w, const uint32_t* ids, const uint8_t* lv, size_t n, float* ci, uint64_t* cs,
           const bs_window_rules& r, bs_render_fn fn, void* user) {
    if (r.min_dt_ns < 1 || r.min_dt_ns > (int64_t{1} << kWindowLog2) || (r.min_dt_ns & (r.min_dt_ns - 1)) != 0) {
      throw std::invalid_argument("min_dt_ns must be a power of two in [1, 2^23]");
    }
    if (r.max_refine_levels < 0) throw std::invalid_argument("max_refine_levels must be >= 0");
    int shift = 0;
    while ((int64_t{1} << shift) < r.min_dt_ns) ++shift;
    const int max_level = kWindowLog2 - shift;
    for (size_t a = 0; a < n; ++a) {
      if (lv[a] > max_level) throw std::invalid_argument("levels must lie in [0, 23 - log2(min_dt_ns)]");
    }
    const uint32_t min_split = static_cast<uint32_t>(2 * r.min_dt_ns);
    const size_t G = static_cast<size_t>(groups);
    flagged_signature = flagged_midpoint = refine_cap_hits = render_calls = 0;
    samples_by_round.assign(1, 0);
    offsets.assign(n + 1, 0);
    t.clear();
    irr.clear();
    if (n == 0) return;
    check_cancel(r.cancel, "window: batch");
    // The lattice: pixel a's slots [off0[a], off0[a + 1]), slot 0 the carried sample.
    std::vector<uint64_t> off0(n + 1, 0);
    for (size_t a = 0; a < n; ++a) off0[a + 1] = off0[a] + (uint64_t{1} << lv[a]) + 1;
    const uint64_t s0 = off0[n];
    if (s0 > 0xFFFFFFFFull) throw std::invalid_argument("window: too many samples");
    dt.resize(s0);
    owner.resize(s0);
    rows.assign(s0 * G, 0.0f);
    sig.assign(s0, 0);
    for (size_t a = 0; a < n; ++a) {
      const uint32_t step = uint32_t{1} << (kWindowLog2 - lv[a]);
      for (uint64_t g = off0[a]; g < off0[a + 1]; ++g) {
        dt[g] = static_cast<uint32_t>(g - off0[a]) * step;
        owner[g] = static_cast<uint32_t>(a);
      }
      std::memcpy(&rows[off0[a] * G], ci + a * G, G * sizeof(float));
      sig[off0[a]] = cs[a];
    }
    // One render call for every slot past each pixel's first, in slot order; the carried rows stay as they are.
    {
      std::vector<uint32_t> lat;
      lat.reserve(s0 - n);
      for (uint32_t g = 0; g < s0; ++g) {
        if (g != off0[owner[g]]) lat.push_back(g);
      }
      req.resize(lat.size());
      out_index.resize(lat.size());
      for (size_t i = 0; i < lat.size(); ++i) {
        const uint32_t g = lat[i];
        req[i] = bs_sample_request{r.cam, 0, ids[owner[g]], 0, r.subsamples, static_cast<int32_t>(dt[g]),
                                   dt[g] >> shift};
        out_index[i] = g;
      }
      if (!lat.empty()) {
        ++render_calls;
        const int32_t rc = fn(user, req.data(), lat.size(), out_index.data(), rows.data(), sig.data(), r.subsamples);
        if (rc != 0) {
          throw std::invalid_argument("render: the render callback failed (status " + std::to_string(rc) + ")");
        }
      }
      samples_by_round[0] = lat.size();
    }
    // Round 0: interval (i - 1, i) of every slot i past a pixel's first; node k tests the triple (k - 1, k, k + 1).
    std::vector<uint32_t> ia, im, ib;
    std::vector<uint8_t> node_ex;
    std::vector<uint8_t> node(s0, 0);
    for (uint32_t k = 0; k < s0; ++k) {
      const uint64_t j = k - off0[owner[k]];
      if (j >= 1 && k + 1 < off0[owner[k] + 1]) {
        ia.push_back(k - 1);
        im.push_back(k);
        ib.push_back(k + 1);
      }
    }
    exceeds(r, ia, im, ib, node_ex);
    for (size_t q = 0; q < im.size(); ++q) node[im[q]] = node_ex[q];
    std::vector<uint32_t> lo, hi;
    uint64_t words[3] = {0, 0, 0};
    for (uint32_t i = 0; i < s0; ++i) {
      const uint32_t a = owner[i];
      const uint64_t j = i - off0[a], cnt = off0[a + 1] - off0[a];
      if (j == 0) continue;
      const bool flip = r.refine_signature && sig[i] != sig[i - 1];
      const bool mid = (j + 1 < cnt && node[i]) || (j >= 2 && node[i - 1]);
      const bool want = flip || mid;
      const bool split = want && dt[i] - dt[i - 1] >= min_split;
      words[0] += flip;
      words[1] += mid && !flip;
      words[2] += want && !split;
      if (split) {
        lo.push_back(i - 1);
        hi.push_back(i);
      }
    }
    uint32_t samples = static_cast<uint32_t>(s0);
    std::vector<uint8_t> bad;
    for (int k = 0;; ++k) {
      flagged_signature += words[0];
      flagged_midpoint += words[1];
      if (k == r.max_refine_levels) {
        refine_cap_hits += words[2] + lo.size();
        break;
      }
      refine_cap_hits += words[2];
      if (lo.empty()) break;
      check_cancel(r.cancel, "window: refinement round");
      const uint32_t m = static_cast<uint32_t>(lo.size());
      if (static_cast<uint64_t>(samples) + m > 0xFFFFFFFFull) throw std::invalid_argument("window: too many samples");
      dt.resize(samples + m);
      owner.resize(samples + m);
      rows.resize((static_cast<size_t>(samples) + m) * G, 0.0f);
      sig.resize(samples + m, 0);
      std::vector<uint32_t> g(m);
      for (uint32_t q = 0; q < m; ++q) {
        g[q] = samples + q;
        dt[g[q]] = (dt[lo[q]] + dt[hi[q]]) >> 1;
        owner[g[q]] = owner[hi[q]];
      }
      render(t_w, ids, r, shift, samples, samples + m, fn, user);
      samples += m;
      exceeds(r, lo, g, hi, bad);
      std::vector<uint32_t> nlo, nhi;
      words[0] = words[1] = words[2] = 0;
      for (uint32_t q = 0; q < m; ++q) {
        const bool s1 = r.refine_signature && sig[lo[q]] != sig[g[q]];
        const bool s2 = r.refine_signature && sig[g[q]] != sig[hi[q]];
        const bool f1 = s1 || bad[q], f2 = s2 || bad[q];
        const bool p1 = f1 && dt[g[q]] - dt[lo[q]] >= min_split;
        const bool p2 = f2 && dt[hi[q]] - dt[g[q]] >= min_split;
        words[0] += static_cast<uint64_t>(s1) + s2;
        words[1] += static_cast<uint64_t>(bad[q] && !s1) + (bad[q] && !s2);
        words[2] += static_cast<uint64_t>(f1 && !p1) + (f2 && !p2);
        if (p1) {
          nlo.push_back(lo[q]);
          nhi.push_back(g[q]);
        }
        if (p2) {
          nlo.push_back(g[q]);
          nhi.push_back(hi[q]);
        }
      }
      lo.swap(nlo);
      hi.swap(nhi);
      samples_by_round.push_back(m);
    }
    // The runs: each pixel's samples by time; the carried sample becomes its last lattice slot.
    std::vector<uint32_t> order(samples);
    std::iota(order.begin(), order.end(), 0u);
    std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) {
      return owner[x] != owner[y] ? owner[x] < owner[y] : dt[x] < dt[y];
    });
    t.resize(samples);
    irr.resize(static_cast<size_t>(samples) * G);
    for (uint32_t q = 0; q < samples; ++q) {
      t[q] = t_w + dt[order[q]];
      std::memcpy(&irr[static_cast<size_t>(q) * G], &rows[static_cast<size_t>(order[q]) * G], G * sizeof(float));
      ++offsets[owner[order[q]] + 1];
    }
    for (size_t a = 0; a < n; ++a) offsets[a + 1] += offsets[a];
    for (size_t a = 0; a < n; ++a) {
      const uint64_t last = off0[a + 1] - 1;
      std::memcpy(ci + a * G, &rows[last * G], G * sizeof(float));
      cs[a] = sig[last];
    }
  }
};

extern "C" {

bs_status bs_window_create(int32_t groups, const float* m_min, const float* m_max, bs_window** out) {
  try {
    if (!out) throw std::invalid_argument("null argument: out");
    if (groups < 1 || groups > 8) throw std::invalid_argument("window: need 1 to 8 light groups");
    auto* w = new bs_window;
    w->groups = groups;
    w->m_min.assign(groups, 1.0f);
    w->m_max.assign(groups, 1.0f);
    if (m_min) std::copy(m_min, m_min + groups, w->m_min.begin());
    if (m_max) std::copy(m_max, m_max + groups, w->m_max.begin());
    *out = w;
    return BS_OK;
  } catch (const std::invalid_argument& e) {
    bs::set_last_error(e.what());
    return BS_EINVAL;
  } catch (const std::exception& e) {
    bs::set_last_error(e.what());
    return BS_ELOGIC;
  }
}

bs_status bs_window_destroy(bs_window* w) {
  delete w;
  return BS_OK;
}

bs_status bs_window_run(bs_window* w, int64_t t_w, const uint32_t* pixel_ids, const uint8_t* levels, size_t n,
                        float* carried_irr, uint64_t* carried_sig, const bs_window_rules* rules, bs_render_fn render,
                        void* user, size_t* n_samples) {
  try {
    if (!w || !rules || !render) throw std::invalid_argument("null argument");
    if (n > 0 && (!pixel_ids || !levels || !carried_irr || !carried_sig)) throw std::invalid_argument("null argument");
    if ((t_w & ((int64_t{1} << kWindowLog2) - 1)) != 0) throw std::invalid_argument("window: t_w must be a multiple of 2^23");
    w->run(t_w, pixel_ids, levels, n, carried_irr, carried_sig, *rules, render, user);
    if (n_samples) *n_samples = w->t.size();
    return BS_OK;
  } catch (const Cancelled& e) {
    bs::set_last_error(e.what());
    return BS_ECANCELLED;
  } catch (const std::invalid_argument& e) {
    bs::set_last_error(e.what());
    return BS_EINVAL;
  } catch (const std::bad_alloc&) {
    bs::set_last_error("window: out of host memory");
    return BS_ENOMEM;
  } catch (const std::exception& e) {
    bs::set_last_error(e.what());
    return BS_ECUDA;
  }
}

bs_status bs_window_runs(const bs_window* w, int64_t* offsets, int64_t* t_ns, float* irr) {
  if (!w) {
    bs::set_last_error("null argument");
    return BS_EINVAL;
  }
  if (offsets) std::copy(w->offsets.begin(), w->offsets.end(), offsets);
  if (t_ns) std::copy(w->t.begin(), w->t.end(), t_ns);
  if (irr) std::copy(w->irr.begin(), w->irr.end(), irr);
  return BS_OK;
}

bs_status bs_window_stats(const bs_window* w, uint64_t counters[4], uint64_t* samples_by_round, size_t cap,
                          size_t* rounds) {
  if (!w) {
    bs::set_last_error("null argument");
    return BS_EINVAL;
  }
  if (counters) {
    counters[0] = w->flagged_signature;
    counters[1] = w->flagged_midpoint;
    counters[2] = w->refine_cap_hits;
    counters[3] = w->render_calls;
  }
  if (samples_by_round) {
    std::copy(w->samples_by_round.begin(), w->samples_by_round.begin() + std::min(cap, w->samples_by_round.size()),
              samples_by_round);
  }
  if (rounds) *rounds = w->samples_by_round.size();
  return BS_OK;
}

}  // extern "C"
