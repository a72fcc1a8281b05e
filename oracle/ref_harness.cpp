// A C-ABI harness around the reference's own CPU implementation of the path, compiled from its
// sources in place by oracle/build.py (build_ref) into oracle/_ref/libballa_ref.so. TEST INFRASTRUCTURE
// ONLY: it pins the oracle port (oracle/port) and is the CPU baseline of bench.py's reference arm.
//
// It drives balla::sensor::SensorModel (src/sensor/sensor_model.h:98-320) on the fp32 precision
// (the bitwise contract, src/sensor/sensor_cuda.h:1-3) and balla::engine::WindowEngine<kHost>
// (src/engine/window.h:132-175) with a render hook that evaluates the project's analytic fields
// through the oracle port's field evaluator (the same inputs for both sides).
#include <chrono>
#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "engine/window.h"
#include "export/errors.h"
#include "export/raw_writer.h"
#include "sensor/output_order.h"
#include "sensor/params.h"
#include "sensor/readout.h"
#include "sensor/sensor_model.h"
#include "sensor/stage1.h"
#include "sensor/noise_tables.h"
#include "core/pmath/special.h"

extern "C" {
#include "port/oracle.h"
}

using namespace balla;

namespace {

thread_local std::string g_error;

int fail(const std::exception& e) {
  g_error = e.what();
  return -1;
}

// Parameter overrides by field name (a subset of src/sensor/params.h's rows).
void set_field(sensor::SensorParams& p, const std::string& key, double v) {
  if (key == "theta_on") p.theta_on = v;
  else if (key == "theta_off") p.theta_off = v;
  else if (key == "sigma_theta_on") p.sigma_theta_on = v;
  else if (key == "sigma_theta_off") p.sigma_theta_off = v;
  else if (key == "theta_onoff_corr") p.theta_onoff_corr = v;
  else if (key == "theta_floor") p.theta_floor = v;
  else if (key == "reset_mode") p.reset_mode = static_cast<sensor::ResetMode>(static_cast<int32_t>(v));
  else if (key == "refractory_s") p.refractory_s = v;
  else if (key == "eps_ci") p.eps_ci = v;
  else if (key == "initial_phase") p.initial_phase = static_cast<sensor::InitialPhase>(static_cast<int32_t>(v));
  else if (key == "leak_rate_hz") p.leak_rate_hz = v;
  else if (key == "leak_sigma_log10") p.leak_sigma_log10 = v;
  else if (key == "dark_current_fA") p.dark_current_fA = v;
  else if (key == "dark_sigma_ln") p.dark_sigma_ln = v;
  else if (key == "illuminance_scale") p.illuminance_scale = v;
  else if (key == "label_share_cut") p.label_share_cut = v;
  else if (key == "readout_quantum_s") p.readout_quantum_s = v;
  else if (key == "readout_delay_s") p.readout_delay_s = v;
  else if (key == "temperature_K") p.temperature_K = v;
  else if (key == "photoreceptor") {
    p.photoreceptor = v == 0.0 ? sensor::Photoreceptor::kCascade : sensor::Photoreceptor::kInstantaneous;
  } else if (key == "noise") p.noise = v != 0.0;
  else if (key == "k") p.k = v;
  else if (key == "tau_o") p.tau_o = v;
  else if (key == "tau_sf") p.tau_sf = v;
  else if (key == "eps_L") p.eps_L = v;
  else if (key == "sigma_o") p.sigma_o = v;
  else if (key == "noise_leaf_level") p.noise_leaf_level = static_cast<int32_t>(v);
  else if (key == "noise_margin_z") p.noise_margin_z = v;
  else if (key == "noise_diffusion") {
    p.noise_diffusion = v == 0.0 ? sensor::NoiseDiffusion::kFrozen : sensor::NoiseDiffusion::kTransient;
  } else if (key == "initial_state") {
    p.initial_state = v == 0.0 ? sensor::InitialState::kPhase : sensor::InitialState::kStationary;
  } else if (key == "stationary_burnin_ns") p.stationary_burnin_ns = static_cast<int64_t>(v);
  else if (key == "stationary_probe_pixels") p.stationary_probe_pixels = static_cast<int32_t>(v);
  else if (key == "leak_ea_eV") p.leak_ea_eV = v;
  else if (key == "dark_ea_eV") p.dark_ea_eV = v;
  else if (key == "reference_temperature_K") p.reference_temperature_K = v;
  else if (key == "clock_offset_ns") p.clock_offset_ns = static_cast<int64_t>(v);
  else if (key == "clock_drift_ppm") p.clock_drift_ppm = v;
  else if (key == "hot_fraction") p.hot_fraction = v;
  else if (key == "veiling_glare") p.veiling_glare = v;
  else throw std::invalid_argument("ref harness: unknown field " + key);
}

struct RefModel {
  std::unique_ptr<sensor::SensorModel> model;
  std::vector<sensor::RawEvent> events;
};

class FieldHook final : public engine::RenderHook {
 public:
  FieldHook(const orc_field* f, int64_t t_w) : f_(f), t_w_(t_w) {}
  void render(render::SampleRequest* req, size_t n, const uint32_t* out_index, float* irr, uint64_t* sig, uint32_t*,
              uint32_t) override {
    for (size_t i = 0; i < n; ++i) {
      const uint32_t px = req[i].pixel;
      irr[out_index[i]] = orc_field_eval(f_, px % f_->width, px / f_->width, t_w_ + req[i].t_off_ns);
      sig[out_index[i]] = 0;
    }
    calls_ += n;
  }
  size_t calls_ = 0;

 private:
  const orc_field* f_;
  int64_t t_w_;
};

engine::SampleConfig make_config(float tol, float dark, int midpoint, int refine_signature, int max_refine_levels,
                                 int64_t min_dt_ns) {
  // sample_window's rules (src/engine/bindings/engine_module.cpp:311-355) with the default economy rules.
  engine::SampleConfig cfg;
  cfg.rules.refine_signature = refine_signature != 0;
  cfg.rules.max_refine_levels = max_refine_levels;
  cfg.rules.min_split = static_cast<uint32_t>(2 * min_dt_ns);
  cfg.rules.shift = 0;
  while ((int64_t{1} << cfg.rules.shift) < min_dt_ns) ++cfg.rules.shift;
  cfg.rules.midpoint = midpoint != 0;
  engine::economy_rules(cfg.rules, std::nullopt, std::nullopt, 0.0, 0.0, std::nullopt);
  if (cfg.rules.midpoint) cfg.rules.mid = engine::midpoint_params(tol, dark, {{1.0, 1.0}});
  cfg.groups = 1;
  return cfg;
}

}  // namespace

extern "C" {

const char* ref_last_error() { return g_error.c_str(); }

// preset: a family name; keys/values: n_over overrides (SensorParams field names); fp64 != 0: the reference's fp64
// CPU kernel (its default precision, Precision::kFp64, src/sensor/sensor_model.h:30), else fp32.
void* ref_model_create_prec(const char* preset, const char* const* keys, const double* values, int n_over,
                            uint32_t width, uint32_t height, uint64_t seed, uint32_t camera, int num_threads,
                            int fp64) {
  try {
    sensor::SensorParams p = sensor::preset(preset);
    for (int i = 0; i < n_over; ++i) set_field(p, keys[i], values[i]);
    p.validate();
    auto* m = new RefModel;
    m->model = std::make_unique<sensor::SensorModel>(
        p, width, height, seed, std::vector<sensor::Waveform>{sensor::make_constant_waveform()}, camera, num_threads,
        fp64 ? sensor::Precision::kFp64 : sensor::Precision::kFp32, sensor::Device::kCpu);
    return m;
  } catch (const std::exception& e) {
    fail(e);
    return nullptr;
  }
}

void* ref_model_create(const char* preset, const char* const* keys, const double* values, int n_over, uint32_t width,
                       uint32_t height, uint64_t seed, uint32_t camera, int num_threads) {
  return ref_model_create_prec(preset, keys, values, n_over, width, height, seed, camera, num_threads, 0);
}

void ref_model_destroy(void* h) { delete static_cast<RefModel*>(h); }

// The reference's parameter fingerprint (fingerprint, src/sensor/params.cpp:246) of a preset with overrides and one
// constant light group; 0 with the message in ref_last_error on a refused parameter set.
uint64_t ref_fingerprint(const char* preset, const char* const* keys, const double* values, int n_over) {
  try {
    sensor::SensorParams p = sensor::preset(preset);
    for (int i = 0; i < n_over; ++i) set_field(p, keys[i], values[i]);
    return sensor::fingerprint(p, std::vector<sensor::Waveform>{sensor::make_constant_waveform()});
  } catch (const std::exception& e) {
    fail(e);
    return 0;
  }
}

// SensorModel::state_bytes / save_state / load_state (src/sensor/sensor_model.cpp:1198-1262).
size_t ref_model_state_bytes(void* h) { return static_cast<RefModel*>(h)->model->state_bytes(); }
int ref_model_save_state(void* h, uint8_t* out, size_t n) {
  try {
    const std::vector<uint8_t> b = static_cast<RefModel*>(h)->model->save_state();
    if (b.size() != n) throw std::invalid_argument("ref harness: state buffer size");
    std::memcpy(out, b.data(), n);
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}
int ref_model_load_state(void* h, const uint8_t* data, size_t n) {
  try {
    static_cast<RefModel*>(h)->model->load_state(data, n);
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

int ref_model_init(void* h, int64_t t0, const float* irr0) {
  try {
    static_cast<RefModel*>(h)->model->init(t0, irr0);
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// Appends the raw events (unsorted) of one advance; ref_model_take_events returns them sorted by (t_cross, pixel).
int ref_model_advance_runs(void* h, const uint32_t* ids, size_t n, const int64_t* t, const float* irr, size_t ns,
                           const int64_t* row_start, const int32_t* row_count, int64_t t_end) {
  try {
    auto* m = static_cast<RefModel*>(h);
    std::vector<sensor::RawEvent> ev = m->model->advance_runs_raw(ids, n, t, irr, ns, row_start, row_count, t_end);
    m->events.insert(m->events.end(), ev.begin(), ev.end());
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

size_t ref_model_event_count(void* h) { return static_cast<RefModel*>(h)->events.size(); }

// Event columns sorted by (t_cross, pixel); clears the list.
void ref_model_take_events(void* h, uint32_t* pixel, uint8_t* p, uint8_t* label, uint16_t* flags, int64_t* t,
                           float* ds, float* dn, float* dl, float* l_first) {
  auto* m = static_cast<RefModel*>(h);
  std::sort(m->events.begin(), m->events.end(), [](const sensor::RawEvent& a, const sensor::RawEvent& b) {
    return a.t_cross != b.t_cross ? a.t_cross < b.t_cross : a.pixel < b.pixel;
  });
  for (size_t i = 0; i < m->events.size(); ++i) {
    const sensor::RawEvent& e = m->events[i];
    pixel[i] = e.pixel;
    p[i] = e.polarity;
    label[i] = e.label;
    flags[i] = e.flags;
    t[i] = e.t_cross;
    ds[i] = e.ds;
    dn[i] = e.dn;
    dl[i] = e.dl;
    l_first[i] = e.l_first;
  }
  m->events.clear();
}

void ref_model_maps(void* h, double* on, double* off, double* leak, double* dark, double* phi0) {
  const auto& px = static_cast<RefModel*>(h)->model->maps().pixels;
  for (size_t i = 0; i < px.size(); ++i) {
    on[i] = px[i].theta_on;
    off[i] = px[i].theta_off;
    leak[i] = px[i].leak;
    dark[i] = px[i].dark_fA;
    phi0[i] = px[i].phi0;
  }
}

int64_t ref_model_time(void* h) { return static_cast<RefModel*>(h)->model->time_ns(); }
float ref_model_irr_max(void* h) { return static_cast<RefModel*>(h)->model->irr_max(); }

// SensorModel::set_photometry; gain NULL (n 0): 1 everywhere.
int ref_model_set_photometry(void* h, double scale, const float* gain, size_t n) {
  try {
    static_cast<RefModel*>(h)->model->set_photometry(scale, gain ? std::vector<float>(gain, gain + n)
                                                                 : std::vector<float>{});
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}
int ref_model_threads(void* h) { return static_cast<RefModel*>(h)->model->num_threads(); }

// The window's samples by WindowEngine<kHost>::run (src/engine/window_impl.h:715-867). Returns the sample count
// (offsets n + 1, t and irr filled up to cap) or -(count) when cap is too small; carried_* updated in place.
int64_t ref_sample_window(const orc_field* f, float tol, float dark, int midpoint, int refine_signature,
                          int max_refine_levels, int64_t min_dt_ns, int64_t t_w, const uint32_t* pixel,
                          const uint8_t* level, size_t n, float* carried_irr, uint64_t* carried_sig, int64_t* offsets,
                          int64_t* t_out, float* irr_out, size_t cap) {
  try {
    const engine::SampleConfig cfg = make_config(tol, dark, midpoint, refine_signature, max_refine_levels, min_dt_ns);
    engine::WindowEngine<engine::Space::kHost> eng;
    FieldHook hook(f, t_w);
    engine::WindowEngine<engine::Space::kHost>::Input in{};
    in.t_w = t_w;
    in.pixel = pixel;
    in.level = level;
    in.n = n;
    in.carried_irr = carried_irr;
    in.carried_sig = carried_sig;
    eng.run(in, cfg, hook, std::numeric_limits<size_t>::max(), nullptr);
    const size_t s = eng.samples();
    std::memcpy(offsets, eng.offsets(), (n + 1) * sizeof(int64_t));
    if (s > cap) return -static_cast<int64_t>(s);
    std::memcpy(t_out, eng.t(), s * sizeof(int64_t));
    std::memcpy(irr_out, eng.irr(), s * sizeof(float));
    return static_cast<int64_t>(s);
  } catch (const std::exception& e) {
    fail(e);
    return INT64_MIN;
  }
}

// A C callback as the renderer (the role engine_module.cpp:227-262 gives a Python callable): pixel ids and absolute
// times in request order, irradiance (n, groups) and signatures (n,) back; a non-zero return fails the window.
typedef int (*ref_render_fn)(void* user, const uint32_t* pixel, const int64_t* t, size_t n, float* irr, uint64_t* sig);

class CallbackHook final : public engine::RenderHook {
 public:
  CallbackHook(ref_render_fn fn, void* user, int64_t t_w, int groups) : fn_(fn), user_(user), t_w_(t_w), g_(groups) {}
  void render(render::SampleRequest* req, size_t n, const uint32_t* out_index, float* irr, uint64_t* sig, uint32_t*,
              uint32_t) override {
    std::vector<uint32_t> px(n);
    std::vector<int64_t> t(n);
    std::vector<float> e(n * static_cast<size_t>(g_));
    std::vector<uint64_t> s(n);
    for (size_t i = 0; i < n; ++i) {
      px[i] = req[i].pixel;
      t[i] = t_w_ + req[i].t_off_ns;
    }
    if (fn_(user_, px.data(), t.data(), n, e.data(), s.data()) != 0) throw std::runtime_error("render callback failed");
    for (size_t i = 0; i < n; ++i) {
      std::memcpy(irr + static_cast<size_t>(out_index[i]) * g_, e.data() + i * g_, g_ * sizeof(float));
      sig[out_index[i]] = s[i];
    }
    ++calls_;
  }
  size_t calls_ = 0;

 private:
  ref_render_fn fn_;
  void* user_;
  int64_t t_w_;
  int g_;
};

// sample_window with a renderer callback (engine_module.cpp:265-355 on WindowEngine<kHost>), groups light groups and
// the midpoint test's waveform ranges m_min / m_max (midpoint 0: none). As ref_sample_window (irr_out (S, groups));
// stats: flagged_signature, flagged_midpoint, refine_cap_hits, render calls, rounds, then samples_by_round (at most
// 32 rounds written).
int64_t ref_sample_window_cb(int groups, float tol, float dark, const double* m_min, const double* m_max, int midpoint,
                             int refine_signature, int max_refine_levels, int64_t min_dt_ns, int64_t t_w,
                             const uint32_t* pixel, const uint8_t* level, size_t n, float* carried_irr,
                             uint64_t* carried_sig, ref_render_fn fn, void* user, int64_t* offsets, int64_t* t_out,
                             float* irr_out, size_t cap, uint64_t* stats) {
  try {
    engine::SampleConfig cfg = make_config(tol, dark, 0, refine_signature, max_refine_levels, min_dt_ns);
    cfg.groups = groups;
    if (midpoint != 0) {
      std::vector<std::pair<double, double>> ranges;
      for (int g = 0; g < groups; ++g) ranges.emplace_back(m_min[g], m_max[g]);
      cfg.rules.midpoint = true;
      cfg.rules.mid = engine::midpoint_params(tol, dark, ranges);
    }
    engine::WindowEngine<engine::Space::kHost> eng;
    CallbackHook hook(fn, user, t_w, groups);
    engine::WindowEngine<engine::Space::kHost>::Input in{};
    in.t_w = t_w;
    in.pixel = pixel;
    in.level = level;
    in.n = n;
    in.carried_irr = carried_irr;
    in.carried_sig = carried_sig;
    const engine::WindowStats st = eng.run(in, cfg, hook, std::numeric_limits<size_t>::max(), nullptr);
    stats[0] = st.flagged_signature;
    stats[1] = st.flagged_midpoint;
    stats[2] = st.refine_cap_hits;
    stats[3] = hook.calls_;
    stats[4] = st.samples_by_round.size();
    for (size_t k = 0; k < st.samples_by_round.size() && k < 32; ++k) stats[5 + k] = st.samples_by_round[k];
    const size_t s = eng.samples();
    std::memcpy(offsets, eng.offsets(), (n + 1) * sizeof(int64_t));
    if (s > cap) return -static_cast<int64_t>(s);
    std::memcpy(t_out, eng.t(), s * sizeof(int64_t));
    std::memcpy(irr_out, eng.irr(), s * static_cast<size_t>(groups) * sizeof(float));
    return static_cast<int64_t>(s);
  } catch (const std::exception& e) {
    fail(e);
    return INT64_MIN;
  }
}

// The reference's event files: RawWriter (format 0 evt2, 1 evt21, 2 evt3; th_change: EVT 2.0's on-change TIME_HIGH)
// or DatWriter (format 3), fed batches [bounds[k], bounds[k + 1]) of the columns; status[k] = 1 for a refused batch
// (message: the last refusal). info: bytes, count, t_first, t_last; sha: 65 chars. Returns 0, or -1 when the
// writer could not be made or closed (ref_last_error).
int ref_event_file(const char* path, int format, int th_change, int32_t width, int32_t height, int64_t origin_us,
                   int64_t epoch_ns, int32_t rem_min, int32_t rem_max, const char* version, const uint16_t* x,
                   const uint16_t* y, const uint8_t* p, const int64_t* t, const int64_t* bounds, int n_batches,
                   int32_t* status, char* message, size_t message_cap, int64_t* info, char* sha) {
  try {
    exporter::RawOptions o;
    o.evt2_time_high = th_change ? exporter::Evt2TimeHigh::kOnChange : exporter::Evt2TimeHigh::kOpenEb;
    o.t_ns_rem_min = rem_min;
    o.t_ns_rem_max = rem_max;
    o.version = version;
    const exporter::TimeMap m{origin_us, epoch_ns};
    std::unique_ptr<exporter::RawWriter> raw;
    std::unique_ptr<exporter::DatWriter> dat;
    if (format == 3) {
      dat = std::make_unique<exporter::DatWriter>(path, width, height, m, o);
    } else {
      const exporter::RawFormat f = format == 0   ? exporter::RawFormat::kEvt2
                                    : format == 1 ? exporter::RawFormat::kEvt21
                                                  : exporter::RawFormat::kEvt3;
      raw = std::make_unique<exporter::RawWriter>(path, f, width, height, m, o);
    }
    for (int k = 0; k < n_batches; ++k) {
      const size_t a = static_cast<size_t>(bounds[k]), b = static_cast<size_t>(bounds[k + 1]);
      const exporter::Events e{x + a, y + a, p + a, t + a, b - a};
      status[k] = 0;
      try {
        if (dat) {
          dat->append(e);
        } else {
          raw->append(e);
        }
      } catch (const exporter::Refused& r) {
        status[k] = 1;
        std::snprintf(message, message_cap, "%s", r.what());
      }
    }
    const exporter::FileInfo fi = dat ? dat->close() : raw->close();
    info[0] = static_cast<int64_t>(fi.bytes);
    info[1] = fi.streams.at(0).count;
    info[2] = fi.streams.at(0).t_first;
    info[3] = fi.streams.at(0).t_last;
    std::snprintf(sha, 65, "%s", fi.sha256.c_str());
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// fixed_rate_window with a renderer callback (engine_module.cpp:356-365): the fixed-rate grid of period_ns, no
// refinement. As ref_sample_window_cb otherwise (stats: samples_by_round at stats[5]).
int64_t ref_fixed_rate_window_cb(int groups, int64_t period_ns, int64_t t_w, const uint32_t* pixel, size_t n,
                                 float* carried_irr, uint64_t* carried_sig, ref_render_fn fn, void* user,
                                 int64_t* offsets, int64_t* t_out, float* irr_out, size_t cap, uint64_t* stats) {
  try {
    engine::SampleConfig cfg;
    cfg.rules.fixed = true;
    cfg.rules.period_ns = period_ns;
    cfg.rules.m = engine::fixed_rate_samples(t_w, period_ns);
    cfg.groups = groups;
    engine::WindowEngine<engine::Space::kHost> eng;
    CallbackHook hook(fn, user, t_w, groups);
    engine::WindowEngine<engine::Space::kHost>::Input in{};
    in.t_w = t_w;
    in.pixel = pixel;
    in.level = nullptr;
    in.n = n;
    in.carried_irr = carried_irr;
    in.carried_sig = carried_sig;
    const engine::WindowStats st = eng.run(in, cfg, hook, std::numeric_limits<size_t>::max(), nullptr);
    stats[0] = st.flagged_signature;
    stats[1] = st.flagged_midpoint;
    stats[2] = st.refine_cap_hits;
    stats[3] = hook.calls_;
    stats[4] = st.samples_by_round.size();
    for (size_t k = 0; k < st.samples_by_round.size() && k < 32; ++k) stats[5 + k] = st.samples_by_round[k];
    const size_t s = eng.samples();
    std::memcpy(offsets, eng.offsets(), (n + 1) * sizeof(int64_t));
    if (s > cap) return -static_cast<int64_t>(s);
    std::memcpy(t_out, eng.t(), s * sizeof(int64_t));
    std::memcpy(irr_out, eng.irr(), s * static_cast<size_t>(groups) * sizeof(float));
    return static_cast<int64_t>(s);
  } catch (const std::exception& e) {
    fail(e);
    return INT64_MIN;
  }
}

// The whole chain of one sensor on an analytic field, the reference's own code end to end: init at t0 from the
// field, then per window WindowEngine<kHost> (serial by design, src/engine/par.h:1-8) and SensorModel::advance_runs
// on the model's thread pool. Levels: the field's rule per pixel and window. Returns the event count, or -1.
// out_stats: [pixel-samples, sampler seconds, sensor seconds, windows].
int64_t ref_simulate(void* h, const orc_field* f, float tol, float dark, int max_refine_levels, int64_t min_dt_ns,
                     int32_t l_min, int32_t l_max, int64_t t0, int32_t windows, double* out_stats) {
  try {
    auto* m = static_cast<RefModel*>(h);
    const uint32_t W = m->model->width(), H = m->model->height();
    const size_t np = static_cast<size_t>(W) * H;
    std::vector<float> frame(np);
    for (size_t p = 0; p < np; ++p) frame[p] = orc_field_eval(f, p % W, p / W, t0);
    m->model->init(t0, frame.data());
    std::vector<uint32_t> ids(np);
    for (size_t p = 0; p < np; ++p) ids[p] = static_cast<uint32_t>(p);
    std::vector<uint8_t> lv(np);
    std::vector<float> carried = frame;
    std::vector<uint64_t> sig(np, 0);
    std::vector<int32_t> counts(np);
    const engine::SampleConfig cfg = make_config(tol, dark, 1, 1, max_refine_levels, min_dt_ns);
    engine::WindowEngine<engine::Space::kHost> eng;
    double samples = 0, t_sample = 0, t_sense = 0;
    int64_t events = 0;
    using clk = std::chrono::steady_clock;
    for (int32_t w = 0; w < windows; ++w) {
      const int64_t t_w = t0 + static_cast<int64_t>(w) * time::kWindowNs;
      const auto a = clk::now();
      for (size_t p = 0; p < np; ++p) {
        lv[p] = static_cast<uint8_t>(orc_field_level(f, p % W, p / W, t_w, l_min, l_max));
      }
      FieldHook hook(f, t_w);
      engine::WindowEngine<engine::Space::kHost>::Input in{};
      in.t_w = t_w;
      in.pixel = ids.data();
      in.level = lv.data();
      in.n = np;
      in.carried_irr = carried.data();
      in.carried_sig = sig.data();
      eng.run(in, cfg, hook, std::numeric_limits<size_t>::max(), nullptr);
      const auto b = clk::now();
      const int64_t* off = eng.offsets();
      for (size_t p = 0; p < np; ++p) counts[p] = static_cast<int32_t>(off[p + 1] - off[p]);
      std::vector<sensor::RawEvent> ev = m->model->advance_runs_raw(ids.data(), np, eng.t(), eng.irr(), eng.samples(),
                                                                    off, counts.data(), t_w + time::kWindowNs);
      const auto c = clk::now();
      samples += static_cast<double>(eng.samples());
      events += static_cast<int64_t>(ev.size());
      m->events.insert(m->events.end(), ev.begin(), ev.end());
      t_sample += std::chrono::duration<double>(b - a).count();
      t_sense += std::chrono::duration<double>(c - b).count();
    }
    if (out_stats != nullptr) {
      out_stats[0] = samples;
      out_stats[1] = t_sample;
      out_stats[2] = t_sense;
      out_stats[3] = windows;
    }
    return events;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// The reference's output order (sensor/output_order.h output_order) of n event columns, and its readout
// (sensor/readout.h reported_time) and output cut, for the output stage's parity.
void ref_output_order(const int64_t* t_cross, const uint16_t* x, const uint16_t* y, const int64_t* t_reported,
                      size_t n, uint32_t height, uint32_t* perm) {
  std::vector<uint32_t> p;
  balla::sensor::output_order({t_cross, n}, {x, n}, {y, n}, {t_reported, n}, balla::sensor::order_y_bits(height), p);
  std::memcpy(perm, p.data(), n * sizeof(uint32_t));
}
int64_t ref_reported_time(int64_t quantum, int64_t delay, int64_t phase, int64_t offset, double drift, int64_t t) {
  return balla::sensor::reported_time(balla::sensor::Readout{quantum, delay, phase, offset, drift}, t);
}
int64_t ref_output_cut(int64_t quantum, int64_t delay, int64_t phase, int64_t offset, double drift, int64_t t_end) {
  return balla::sensor::output_cut(balla::sensor::Readout{quantum, delay, phase, offset, drift}, t_end);
}
uint8_t ref_label_s1(uint8_t c3) { return balla::sensor::label_s1(c3); }
// The reference's fp32 special functions (core/pmath) and stage-1 solve (sensor/stage1.h z_step): which 0 expm1,
// 1..5 resid_exp(j = which - 1), 6 erfcx, 7 dawson, 8 z_step (x: z0, I0, I1, h, k per entry).
void ref_special(int which, const float* x, size_t n, float* out) {
  for (size_t i = 0; i < n; ++i) {
    if (which == 0) out[i] = balla::pmath::expm1(x[i]);
    else if (which <= 5) out[i] = balla::pmath::resid_exp(which - 1, x[i]);
    else if (which == 6) out[i] = balla::pmath::erfcx(x[i]);
    else if (which == 7) out[i] = balla::pmath::dawson(x[i]);
    else out[i] = balla::sensor::z_step(x[5 * i], x[5 * i + 1], x[5 * i + 2], x[5 * i + 3], x[5 * i + 4]);
  }
}
// The reference's fp32 noise-lattice tables (sensor/noise_tables.h NoiseTables, frozen diffusion): copies up to cap
// floats; returns n_nodes * stride (stride = 18 + 47 levels, + 12 + 19 levels with the split blocks).
int64_t ref_noise_table(double kq, double a2, double a3, double sigma_o, int levels, int split, float* out,
                        size_t cap) {
  try {
    balla::sensor::NoiseModel nm{};
    nm.split = split != 0;
    nm.kq = kq;
    nm.a2 = a2;
    nm.a3 = a3;
    nm.sigma_o = sigma_o;
    nm.levels = levels;
    nm.margin_z = 6.0;
    balla::sensor::NoiseTables t(nm);
    const std::vector<float>& d = t.data32();
    std::memcpy(out, d.data(), std::min(cap, d.size()) * sizeof(float));
    return static_cast<int64_t>(d.size());
  } catch (const std::exception& e) {
    return fail(e);
  }
}
int64_t ref_readout_phase(uint64_t seed, uint32_t camera, int64_t quantum) {
  return balla::sensor::readout_phase_ns(seed, camera, quantum);
}

}  // extern "C"
