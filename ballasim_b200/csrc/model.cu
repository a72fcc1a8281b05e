// Host side of the C ABI (include/ballasim_b200.h): the sensor model, the window sampler and the fused engine as
// C++ objects owning device memory, behind extern "C" entry points with status codes.
//
// SensorModel (src/sensor/sensor_model.h:98-320) on this path: parameter checks, the frozen maps drawn on the host
// in fp64 (src/sensor/maps.cpp:26-156, with the deterministic log / sincos of bs_math.cuh so that they are the
// reference's bits), the per-pixel state double-buffered on the device, and one synchronization per call to read
// its counters. Events are sorted by (t_cross, pixel) and read out (src/sensor/readout.h:22-27) on download.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/ballasim_b200.h"
#include "device.h"
#include "stationary.h"

namespace bs {
namespace {

thread_local std::string g_error;

struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct BudgetError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    if (e == cudaErrorMemoryAllocation) {
      cudaGetLastError();
      throw BudgetError(std::string(what) + ": out of device memory");
    }
    throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
  }
}
#define CK(x) ck((x), #x)

template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t cap = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  T* ensure(size_t n) {
    if (n <= cap && p) return p;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    const size_t want = n == 0 ? 1 : n;
    CK(cudaMalloc(&p, want * sizeof(T)));
    cap = want;
    return p;
  }
};

template <class T>
struct PinBuf {
  T* p = nullptr;
  size_t cap = 0;
  PinBuf() = default;
  PinBuf(const PinBuf&) = delete;
  PinBuf& operator=(const PinBuf&) = delete;
  ~PinBuf() {
    if (p) cudaFreeHost(p);
  }
  T* ensure(size_t n) {
    if (n <= cap && p) return p;
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    const size_t want = n == 0 ? 1 : n;
    CK(cudaMallocHost(&p, want * sizeof(T)));
    cap = want;
    return p;
  }
};

bool device_ok() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return false;
  }
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, 0) != cudaSuccess) return false;
  return prop.major == 10;
}

void require_device() {
  if (!device_ok()) throw CudaError("no CUDA device of compute capability 10.x (B200) is visible");
}

// ---------------------------------------------------------------------------------------------
// maps (src/sensor/maps.cpp:26-156), fp64
// ---------------------------------------------------------------------------------------------
struct HostMaps {
  std::vector<double> theta_on, theta_off, leak, dark, phi0, ba_rate;
};

void normals4(uint64_t seed, uint32_t camera, uint32_t pixel, uint64_t block, double* out) {
  const U4 r = draw(seed, kPurposeSensorMap, camera, pixel, block);
  const double u0 = open_uniform_d(r.v[0]), u1 = open_uniform_d(r.v[1]);
  const double u2 = open_uniform_d(r.v[2]), u3 = open_uniform_d(r.v[3]);
  const double two_pi = 0x1.921fb54442d18p+2;
  const double r0 = std::sqrt(-2.0 * log_d(u0)), r1 = std::sqrt(-2.0 * log_d(u2));
  double s0, c0, s1, c1;
  sincos_d(two_pi * u1, &s0, &c0);
  sincos_d(two_pi * u3, &s1, &c1);
  out[0] = r0 * c0;
  out[1] = r0 * s0;
  out[2] = r1 * c1;
  out[3] = r1 * s1;
}

double arrhenius(double ea, double t, double t0) { return exp_d(-ea / 8.617333262e-5 * (1.0 / t - 1.0 / t0)); }
double dmax(double a, double b) { return a < b ? b : a; }

HostMaps draw_maps(const bs_params& p, uint64_t seed, uint32_t camera, uint32_t n) {
  HostMaps m;
  m.theta_on.resize(n);
  m.theta_off.resize(n);
  m.leak.resize(n);
  m.dark.resize(n);
  m.phi0.resize(n);
  m.ba_rate.assign(n, 0.0);
  const double leak_temp = arrhenius(p.leak_ea_eV, p.temperature_K, p.reference_temperature_K);
  const double dark_temp = arrhenius(p.dark_ea_eV, p.temperature_K, p.reference_temperature_K);
  const double rho = p.theta_onoff_corr, rho_c = std::sqrt(1.0 - rho * rho);
  const double ln10 = log_d(10.0);
  const bool ba = p.noise_ba_median_hz > 0.0;
  for (uint32_t px = 0; px < n; ++px) {
    double xi[4];
    normals4(seed, camera, px, 0, xi);
    const U4 u = draw(seed, kPurposeSensorMap, camera, px, 1);
    const double u_phase = open_uniform_d(u.v[0]);
    const double xi_off = rho == 0.0 ? xi[1] : rho * xi[0] + rho_c * xi[1];
    const double on = dmax(p.theta_floor, p.theta_on + p.sigma_theta_on * xi[0]);
    const double off = dmax(p.theta_floor, p.theta_off + p.sigma_theta_off * xi_off);
    const double leak_rate = p.leak_rate_hz * exp_d(p.leak_sigma_log10 * xi[2] * ln10) * leak_temp;
    m.dark[px] = p.dark_current_fA * exp_d(p.dark_sigma_ln * xi[3]) * dark_temp;
    m.theta_on[px] = on;
    m.theta_off[px] = off;
    m.leak[px] = on * leak_rate;
    m.phi0[px] = p.initial_phase == 0 ? u_phase * on : p.initial_phase == 1 ? -off + u_phase * (on + off) : 0.0;
    if (ba) {
      // The pixel's background-activity rate (this build's noise): log-normal, median noise_ba_median_hz, spread
      // noise_ba_sigma_ln, from its own Box-Muller normal of stream 0x0082.
      const U4 w = draw(seed, kPurposeBackgroundMap, camera, px, 0);
      double s, c;
      sincos_d(0x1.921fb54442d18p+2 * open_uniform_d(w.v[1]), &s, &c);
      const double z = std::sqrt(-2.0 * log_d(open_uniform_d(w.v[0]))) * c;
      m.ba_rate[px] = p.noise_ba_median_hz * exp_d(p.noise_ba_sigma_ln * z);
    }
  }
  return m;
}

uint64_t fnv1a(const void* data, size_t n, uint64_t h = 0xcbf29ce484222325ull) {
  const auto* b = static_cast<const unsigned char*>(data);
  for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 0x100000001b3ull;
  return h;
}

// ---------------------------------------------------------------------------------------------
// device state
// ---------------------------------------------------------------------------------------------
struct StateBufs {
  DevBuf<int64_t> i64;   // 5 x n: t_ref, t_search, blind_until, t_shot, t_ba; with the lattice 1 x n more: cell
  DevBuf<float> f32;     // 5 x n: s3_ref, n3_ref, dr_ref, i_scale, held; with the cascade 5 x n more: z, x1, s2, s3,
                         // tv; with the lattice 8 x n more: nk 0..2, nk1 0..2, ln_a1, rho
  DevBuf<uint32_t> u32;  // 3 x n: flags, n_shot, n_ba; with the lattice 1 x n more: have_k1
  static size_t i64_words(int mode) { return mode == 2 ? 6 : 5; }
  static size_t f32_words(int mode) { return mode == 2 ? 18 : mode == 1 ? 10 : 5; }
  static size_t u32_words(int mode) { return mode == 2 ? 4 : 3; }
  // mode 0: the instantaneous response, 1: the cascade, 2: the cascade with its noise lattice.
  StateSoA soa(size_t n, int mode) {
    const bool cascade = mode != 0;
    i64.ensure(i64_words(mode) * n);
    f32.ensure(f32_words(mode) * n);
    u32.ensure(u32_words(mode) * n);
    StateSoA s;
    s.t_ref = i64.p;
    s.t_search = i64.p + n;
    s.blind_until = i64.p + 2 * n;
    s.t_shot = i64.p + 3 * n;
    s.t_ba = i64.p + 4 * n;
    s.s3_ref = f32.p;
    s.n3_ref = f32.p + n;
    s.dr_ref = f32.p + 2 * n;
    s.i_scale = f32.p + 3 * n;
    s.held = f32.p + 4 * n;
    s.flags = u32.p;
    s.n_shot = u32.p + n;
    s.n_ba = u32.p + 2 * n;
    float* c = cascade ? f32.p + 5 * n : nullptr;
    s.z = c;
    s.x1 = c ? c + n : nullptr;
    s.s2 = c ? c + 2 * n : nullptr;
    s.s3 = c ? c + 3 * n : nullptr;
    s.tv = c ? c + 4 * n : nullptr;
    s.lat = mode == 2 ? f32.p + 10 * n : nullptr;
    s.cell = mode == 2 ? i64.p + 5 * n : nullptr;
    s.have_k1 = mode == 2 ? u32.p + 3 * n : nullptr;
    return s;
  }
};

// The first member of every device object: refuses before any CUDA call when no B200 is visible.
struct DeviceGate {
  DeviceGate() { require_device(); }
};

struct Timer {
  cudaEvent_t a = nullptr, b = nullptr;
  Timer() {
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
  }
  ~Timer() {
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  }
};

}  // namespace

// ---------------------------------------------------------------------------------------------
// the sensor model
// ---------------------------------------------------------------------------------------------
struct Model {
  DeviceGate gate;
  bs_params p{};
  uint32_t width = 0, height = 0, n = 0, camera = 0;
  uint64_t seed = 0;
  HostMaps maps;
  SensorConsts k{};
  CascadeConsts cc{};
  DevBuf<float> tables;   // the noise lattice's (noise_build.h), on the device
  NoiseTableDev tab{};    // data null without the lattice
  std::vector<float> tables_host;  // and on the host (the stationary start's histories)
  cudaStream_t own = nullptr;
  DevBuf<float> mapf;    // 6 x n
  DevBuf<double> mapd;   // 2 x n
  MapSoA map{};
  std::vector<float> gain;  // set_photometry's per-pixel gains (empty: 1 everywhere)
  double gain_max = 1.0;    // the largest of them (1 without a gain map)
  StateBufs st[2];
  StateSoA soa[2]{};
  int cur = 0;
  DevBuf<int32_t> row_of;
  DevBuf<uint32_t> listed;  // the row-major CSR kernel's bitmap of listed pixels
  DevBuf<SensorConsts> k_dev;  // a device copy of k (the row-major kernel's out-of-line calls read it)
  DevBuf<unsigned long long> counters;
  PinBuf<unsigned long long> counters_h;
  DevBuf<RawEvent> events;
  size_t event_cap = 0;
  size_t last_events = 0;      // events of the last device call (on the device)
  std::vector<RawEvent> kept;  // host-kept events (advance_runs, engine runs)
  // staging for host runs
  DevBuf<uint32_t> s_pixel;
  DevBuf<int64_t> s_start, s_t;
  DevBuf<int32_t> s_count;
  DevBuf<float> s_irr, s_frame;
  int64_t t_state = 0;
  bool initialized = false;
  bool fresh = false;  // no call has advanced the model since init (every pixel's search armed at t0 + 1)
  // 0: the row-major kernel split in two (instantaneous response); 1: the row-major kernel in one launch; else the
  // per-pixel kernel's block.
  int block = 0;
  DevBuf<unsigned char> row_rest;  // the split row-major kernel's posted rows (room for every pixel) and their count
  DevBuf<unsigned int> row_rest_count;
  int32_t long_row = 32;  // the row-major kernel: runs longer than this are walked by the whole warp
  uint64_t stat_pieces = 0, stat_leaves = 0, stat_clamps = 0, stat_samples = 0, stat_noise = 0, stat_launches = 0,
           stat_reruns = 0;
  double launch_ms_total = 0, launch_ms_max = 0;
  int64_t readout_phase = 0;
  Timer timer;
  mutable Timer take_timer;           // the last download's device part: sort + column split
  mutable Timer take_timer_copy;      // and its device-to-host copy
  mutable double take_ms[4] = {0, 0, 0, 0};  // sort + split, copy out, host column copies, whole call (ms)

  cudaStream_t stream_of(void* s) const { return s ? static_cast<cudaStream_t>(s) : own; }

  Model(const bs_params& prm, uint32_t w, uint32_t h, uint64_t sd, uint32_t cam, int32_t groups)
      : p(prm), width(w), height(h), camera(cam), seed(sd) {
    validate(groups);
    require_device();
    n = w * h;
    maps = draw_maps(p, seed, camera, n);
    CK(cudaStreamCreateWithFlags(&own, cudaStreamNonBlocking));
    // make_constants (src/sensor/sensor_model.cpp:394-433), fp32; the clamp at the largest gain.
    k.irr_max = static_cast<float>(1e9 / (p.illuminance_scale * gain_max));
    k.eps_ci = static_cast<float>(p.eps_ci);
    k.label_cut = static_cast<float>(p.label_share_cut);
    k.ideal_reset = p.reset_mode == 1;
    k.refractory_ns = std::llround(p.refractory_s * 1e9);
    k.noise = (p.noise_shot_rate_hz > 0.0 || p.noise_ba_median_hz > 0.0) ? 1 : 0;
    k.shot_rate_hz = p.noise_shot_rate_hz;
    k.seed = seed;
    k.camera = camera;
    k.cascade = p.photoreceptor == 0 ? 1 : 0;
    if (k.cascade) {
      // cascade_constants<float> (src/sensor/sensor_model.cpp:376-389) and eps_pl_base (:397).
      const double eps_h = p.eps_L / 8.0;
      cc.k = static_cast<float>(p.k * 1e-15);
      cc.a2 = static_cast<float>(1.0 / p.tau_o);
      cc.a3 = static_cast<float>(1.0 / p.tau_sf);
      cc.tau_o = static_cast<float>(p.tau_o);
      cc.tau_sf = static_cast<float>(p.tau_sf);
      cc.eps_accept = static_cast<float>(eps_h / 1.5);
      cc.eps_drop = static_cast<float>(std::max(eps_h / 1024.0, 32.0 * 0x1p-23));
      cc.eps_pl_base = static_cast<float>(p.eps_L / 8.0);
      if (p.noise != 0) {
        // The noise model of the lattice (src/sensor/sensor_model.cpp:260-268): k q with q the elementary charge.
        const NoiseTablesH t = build_noise_tables(NoiseModelH{p.k * 1.602176634e-19, 1.0 / p.tau_o, 1.0 / p.tau_sf,
                                                              p.sigma_o, p.noise_leaf_level, p.noise_diffusion == 1});
        tables.ensure(t.data.size());
        CK(cudaMemcpy(tables.p, t.data.data(), t.data.size() * sizeof(float), cudaMemcpyHostToDevice));
        tables_host = t.data;
        tab = NoiseTableDev{tables.p, t.n_nodes, t.stride, t.levels, static_cast<float>(kNoiseLnA1Min),
                            static_cast<float>(t.inv_dln), static_cast<float>(p.noise_margin_z),
                            p.noise_diffusion == 1 ? 1 : 0};
      }
    }
    upload_maps();
    soa[0] = st[0].soa(n, mode());
    soa[1] = st[1].soa(n, mode());
    row_of.ensure(n);
    listed.ensure((n + 31) / 32);
    counters.ensure(kCntWords);
    counters_h.ensure(kCntWords);
    ensure_events(1 << 16);
    const int64_t q = std::llround(p.readout_quantum_s * 1e9);
    readout_phase = q > 0 ? static_cast<int64_t>(draw(seed, kPurposeReadoutPhase, camera, 0, 0).v[0] %
                                                 static_cast<uint64_t>(q))
                          : 0;
  }
  ~Model() {
    if (own) cudaStreamDestroy(own);
  }

  void validate(int32_t groups) const {
    if (p.photoreceptor != 0 && p.photoreceptor != 1) {
      throw std::invalid_argument("SensorParams: photoreceptor must be 'cascade' or 'instantaneous'");
    }
    if (p.photoreceptor == 0) {
      if (p.noise != 0 && p.noise_diffusion != 0 && p.noise_diffusion != 1) {
        throw std::invalid_argument("SensorParams: noise_diffusion must be 'frozen' or 'transient'");
      }
      if (p.noise != 0 && (p.noise_leaf_level < 0 || p.noise_leaf_level > 10)) {
        throw std::invalid_argument("SensorParams: noise_leaf_level must lie in [0, 10]");
      }
      if (p.noise != 0 && !(p.sigma_o >= 0.0)) throw std::invalid_argument("SensorParams: sigma_o must be >= 0");
      if (p.initial_state == 1 && (p.stationary_probe_pixels < 1 || p.stationary_burnin_ns < 0)) {
        throw std::invalid_argument(
            "SensorParams: stationary_probe_pixels must be >= 1 and stationary_burnin_ns >= 0");
      }
      if (p.noise_shot_rate_hz > 0.0 || p.noise_ba_median_hz > 0.0) {
        throw std::invalid_argument("SensorModel: shot and background-activity noise run with the instantaneous "
                                    "response only");
      }
      if (!(p.k > 0.0) || !(p.tau_o > 0.0) || !(p.tau_sf > 0.0) || !(p.eps_L > 0.0)) {
        throw std::invalid_argument("SensorParams: k, tau_o, tau_sf and eps_L must be > 0");
      }
      if (!(std::max(p.tau_o, p.tau_sf) >= 1.1 * std::min(p.tau_o, p.tau_sf))) {
        throw std::invalid_argument(
            "SensorParams: tau_sf and tau_o must differ by at least 10 % (the larger >= 1.1 x the smaller)");
      }
    }
    if (groups != 1) throw std::invalid_argument("SensorModel: this build runs one constant light group");
    if (width == 0 || height == 0 || width > 65535 || height > 65535) {
      throw std::invalid_argument("SensorModel: width and height must lie in [1, 65535]");
    }
    if (static_cast<uint64_t>(width) * height > 0xFFFFFFFFull) throw std::invalid_argument("SensorModel: too many pixels");
    if (camera > 255) throw std::invalid_argument("SensorModel: camera index must be < 256 (purpose.h layout)");
    if (p.hot_fraction != 0.0) throw std::invalid_argument("SensorModel: this build has no hot pixels (hot_fraction 0)");
    if (!(p.illuminance_scale > 0.0)) throw std::invalid_argument("SensorParams: illuminance_scale must be > 0");
    if (!(p.theta_on > p.theta_floor) || !(p.theta_off > p.theta_floor)) {
      throw std::invalid_argument("SensorParams: theta_on and theta_off must exceed theta_floor");
    }
    if (!(std::fabs(p.eps_ci) < 0.5 * p.theta_floor)) {
      throw std::invalid_argument("SensorParams: |eps_ci| must be < theta_floor / 2");
    }
    if (!(p.dark_current_fA > 0.0)) throw std::invalid_argument("SensorParams: dark_current_fA must be > 0");
    if (!(p.refractory_s >= 0.0 && p.refractory_s < 10.0)) {
      throw std::invalid_argument("SensorParams: refractory_s must lie in [0, 10)");
    }
  }

  // A pixel's photocurrent per renderer unit, fp32 scale x gain (src/sensor/pixel.h:775).
  float pixel_scale(uint32_t i) const {
    return static_cast<float>(p.illuminance_scale) * (gain.empty() ? 1.0f : gain[i]);
  }

  // SensorModel::set_photometry (src/sensor/sensor_model.cpp:350-373): the scale and the gain map (g null: 1
  // everywhere); the clamp follows the largest gain, and the states take it at the next init.
  void set_photometry(double scale, const float* g, size_t n_gain) {
    if (g && n_gain != n) {
      throw std::invalid_argument("SensorModel.set_photometry: one gain per pixel of the frame (or none)");
    }
    if (!(scale > 0.0) || !std::isfinite(scale)) {
      throw std::invalid_argument("SensorParams: illuminance_scale must be > 0");
    }
    double g_max = g ? 0.0 : 1.0;
    for (size_t i = 0; g && i < n_gain; ++i) {
      if (!(g[i] > 0.0f) || !std::isfinite(g[i])) {
        throw std::invalid_argument("SensorModel.set_photometry: gains must be finite and > 0");
      }
      g_max = std::max(g_max, static_cast<double>(g[i]));
    }
    p.illuminance_scale = scale;
    gain.assign(g, g ? g + n_gain : g);
    gain_max = g_max;
    k.irr_max = static_cast<float>(1e9 / (p.illuminance_scale * gain_max));
    upload_maps();
  }

  void upload_maps() {
    std::vector<float> f(6 * static_cast<size_t>(n));
    std::vector<double> d(2 * static_cast<size_t>(n));
    for (uint32_t i = 0; i < n; ++i) {
      f[i] = static_cast<float>(maps.theta_on[i]);
      f[n + i] = static_cast<float>(maps.theta_off[i]);
      f[2 * static_cast<size_t>(n) + i] = static_cast<float>(maps.leak[i]);
      f[3 * static_cast<size_t>(n) + i] = static_cast<float>(maps.dark[i]);
      f[4 * static_cast<size_t>(n) + i] = pixel_scale(i);
      f[5 * static_cast<size_t>(n) + i] = static_cast<float>(maps.phi0[i]);
      d[i] = maps.ba_rate[i];
      // shot noise: lambda_max = r sqrt(100 fA / I_dk) over the pixel's fp32 dark current
      d[n + i] = p.noise_shot_rate_hz > 0.0 ? p.noise_shot_rate_hz * std::sqrt(100.0 / static_cast<double>(f[3 * static_cast<size_t>(n) + i])) : 0.0;
    }
    mapf.ensure(f.size());
    mapd.ensure(d.size());
    CK(cudaMemcpy(mapf.p, f.data(), f.size() * sizeof(float), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(mapd.p, d.data(), d.size() * sizeof(double), cudaMemcpyHostToDevice));
    map.theta_on = mapf.p;
    map.theta_off = mapf.p + n;
    map.leak = mapf.p + 2 * static_cast<size_t>(n);
    map.dark = mapf.p + 3 * static_cast<size_t>(n);
    map.scale = mapf.p + 4 * static_cast<size_t>(n);
    map.phi0 = mapf.p + 5 * static_cast<size_t>(n);
    map.ba_rate = mapd.p;
    map.shot_max = mapd.p + n;
  }

  void ensure_events(size_t cap) {
    if (cap <= event_cap) return;
    events.ensure(cap);
    event_cap = cap;
  }

  void read_counters(cudaStream_t s) {
    CK(cudaMemcpyAsync(counters_h.p, counters.p, kCntWords * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
  }

  void init_device(int64_t t0, const float* irr0_dev, cudaStream_t s, const float* host_copy) {
    CK(cudaMemsetAsync(counters.p, 0, kCntWords * sizeof(unsigned long long), s));
    launch_init_counted(k, cc, tab, map, soa[cur], n, t0, irr0_dev, counters.p, s);
    CK(cudaGetLastError());
    read_counters(s);
    if (counters_h.p[kCntErrors] & kErrNonFinite) {
      size_t at = 0;
      if (host_copy) {
        while (at < n && std::isfinite(host_copy[at])) ++at;
      }
      initialized = false;
      throw std::invalid_argument("SensorModel.init: non-finite irradiance at pixel " + std::to_string(at));
    }
    stat_clamps += counters_h.p[kCntClamps];
    if (mode() == 2 && p.initial_state == 1) stationary(t0, irr0_dev, host_copy, s);
    t_state = t0;
    initialized = true;
    fresh = true;
    last_events = 0;
    kept.clear();
    n_held = n_ready = 0;  // a new run: nothing held by the output stage
  }

  // The stationary start of the lattice (stationary.h) on the host, from the phase-law states init just wrote.
  void stationary(int64_t t0, const float* irr0_dev, const float* host_copy, cudaStream_t s) {
    CK(cudaStreamSynchronize(s));
    std::vector<float> frame(n);
    if (host_copy) {
      std::copy(host_copy, host_copy + n, frame.begin());
    } else {
      CK(cudaMemcpy(frame.data(), irr0_dev, n * sizeof(float), cudaMemcpyDeviceToHost));
    }
    StateBufs& b = st[cur];
    const size_t ni = i64_words() * n, nf = f32_words() * n, nu = u32_words() * n;
    std::vector<int64_t> i64(ni);
    std::vector<float> f32(nf);
    std::vector<uint32_t> u32(nu);
    CK(cudaMemcpy(i64.data(), b.i64.p, ni * sizeof(int64_t), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(f32.data(), b.f32.p, nf * sizeof(float), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(u32.data(), b.u32.p, nu * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    // The planes of StateBufs::soa (mode 2).
    std::vector<HostPixel> px(n);
    std::vector<PixelMapRegs> regs(n);
    std::vector<float> phi0(n);
    for (size_t i = 0; i < n; ++i) {
      HostPixel& x = px[i];
      x.s.t_ref = i64[i];
      x.s.t_search = i64[n + i];
      x.s.blind_until = i64[2 * n + i];
      x.s.t_shot = i64[3 * n + i];
      x.s.t_ba = i64[4 * n + i];
      x.L.cell = i64[5 * n + i];
      x.s.s3_ref = f32[i];
      x.s.n3_ref = f32[n + i];
      x.s.dr_ref = f32[2 * n + i];
      x.s.i_scale = f32[3 * n + i];
      x.s.held = f32[4 * n + i];
      x.q = CascadeRegs{f32[5 * n + i], f32[6 * n + i], f32[7 * n + i], f32[8 * n + i], f32[9 * n + i]};
      for (int j = 0; j < 3; ++j) {
        x.L.nk[j] = f32[(10 + j) * n + i];
        x.L.nk1[j] = f32[(13 + j) * n + i];
      }
      x.L.ln_a1 = f32[16 * n + i];
      x.L.rho = f32[17 * n + i];
      x.s.flags = u32[i];
      x.s.n_shot = u32[n + i];
      x.s.n_ba = u32[2 * n + i];
      x.L.have_k1 = u32[3 * n + i];
      regs[i] = PixelMapRegs{static_cast<float>(maps.theta_on[i]), static_cast<float>(maps.theta_off[i]),
                             static_cast<float>(maps.leak[i]), static_cast<float>(maps.dark[i]),
                             pixel_scale(static_cast<uint32_t>(i)), 0.0, 0.0};
      phi0[i] = static_cast<float>(maps.phi0[i]);
    }
    NoiseTableDev host_tab = tab;
    host_tab.data = tables_host.data();
    const double leak_at_t = p.leak_rate_hz * arrhenius(p.leak_ea_eV, p.temperature_K, p.reference_temperature_K);
    const StationaryInputs in{regs.data(), maps.theta_on.data(), maps.theta_off.data(), maps.leak.data(),
                              phi0.data(), frame.data(), k, cc, host_tab,
                              NoiseModelH{p.k * 1.602176634e-19, 1.0 / p.tau_o, 1.0 / p.tau_sf, p.sigma_o,
                                          p.noise_leaf_level, p.noise_diffusion == 1},
                              p.k, leak_at_t, p.stationary_burnin_ns, p.stationary_probe_pixels};
    stationary_start(px, in, t0);
    for (size_t i = 0; i < n; ++i) {
      const HostPixel& x = px[i];
      i64[i] = x.s.t_ref;
      i64[n + i] = x.s.t_search;
      i64[2 * n + i] = x.s.blind_until;
      i64[5 * n + i] = x.L.cell;
      f32[i] = x.s.s3_ref;
      f32[n + i] = x.s.n3_ref;
      f32[2 * n + i] = x.s.dr_ref;
      f32[3 * n + i] = x.s.i_scale;
      f32[4 * n + i] = x.s.held;
      const float qv[5] = {x.q.z, x.q.x1, x.q.s2, x.q.s3, x.q.tv};
      for (int j = 0; j < 5; ++j) f32[(5 + j) * n + i] = qv[j];
      for (int j = 0; j < 3; ++j) {
        f32[(10 + j) * n + i] = x.L.nk[j];
        f32[(13 + j) * n + i] = x.L.nk1[j];
      }
      f32[16 * n + i] = x.L.ln_a1;
      f32[17 * n + i] = x.L.rho;
      u32[i] = x.s.flags;
      u32[3 * n + i] = x.L.have_k1;
    }
    CK(cudaMemcpy(b.i64.p, i64.data(), ni * sizeof(int64_t), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(b.f32.p, f32.data(), nf * sizeof(float), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(b.u32.p, u32.data(), nu * sizeof(uint32_t), cudaMemcpyHostToDevice));
  }

  void init_host(int64_t t0, const float* irr0) {
    if (!irr0) throw std::invalid_argument("init: irradiance0 must have shape (height * width, groups)");
    s_frame.ensure(n);
    CK(cudaMemcpyAsync(s_frame.p, irr0, n * sizeof(float), cudaMemcpyHostToDevice, own));
    init_device(t0, s_frame.p, own, irr0);
  }

  void check_ready(int64_t t_end) const {
    if (!initialized) {
      throw std::logic_error("SensorModel.advance: call init() or load_state() first (a call that failed part-way "
                             "leaves the model uninitialized)");
    }
    if (t_end < t_state) throw std::invalid_argument("SensorModel.advance: t_end_ns is before the model time");
  }

  static const char* error_text(unsigned long long e) {
    if (e & kErrPixelRange) return "SensorModel.advance: pixel id out of range";
    if (e & kErrDuplicate) return "SensorModel.advance: duplicate pixel id";
    if (e & kErrRunRange) return "SensorModel.advance: sample run out of range";
    if (e & kErrOrder) {
      return "SensorModel.advance: sample times must be strictly increasing and start at or after the model time";
    }
    if (e & kErrAfterEnd) return "SensorModel.advance: sample after t_end_ns";
    if (e & kErrNonFinite) return "SensorModel.advance: non-finite irradiance";
    if (e & kErrSearchBound) return "engine: a crossing search ran past its bound";
    if (e & kErrRestList) return "engine: the split engine's list of posted pixels overflowed";
    return "SensorModel.advance: refused input";
  }

  // One device call over runs in device memory; the state is committed only when it succeeds.
  void advance_device(const bs_device_runs& r, int64_t t_end, cudaStream_t s) {
    check_ready(t_end);
    if (r.n > n) throw std::invalid_argument("SensorModel.advance: more runs than pixels");
    for (int attempt = 0;; ++attempt) {
      CK(cudaMemsetAsync(counters.p, 0, kCntWords * sizeof(unsigned long long), s));
      const EventBuf evb{events.p, static_cast<unsigned long long>(event_cap)};
      if (!k.cascade && (block == 0 || block == 1)) {
        // The instantaneous response: row-major over the runs, long runs walked by the whole warp; split (block 0):
        // a row stopped at its first segment that is not clean is finished by a second kernel, one thread per row.
        CK(cudaMemsetAsync(listed.p, 0, ((n + 31) / 32) * sizeof(uint32_t), s));
        k_dev.ensure(1);
        CK(cudaMemcpyAsync(k_dev.p, &k, sizeof(SensorConsts), cudaMemcpyHostToDevice, s));
        void* rest = nullptr;
        int rest_blocks = 0;
        if (block == 0) {
          rest = row_rest.ensure(static_cast<size_t>(n) * row_rest_bytes());
          row_rest_count.ensure(1);
          CK(cudaMemsetAsync(row_rest_count.p, 0, sizeof(unsigned int), s));
          int dev = 0, sms = 0;
          CK(cudaGetDevice(&dev));
          CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
          rest_blocks = sms * std::max(1, rows_rest_blocks_per_sm());
        }
        CK(cudaEventRecord(timer.a, s));
        launch_advance_rows(k, map, soa[cur], soa[1 - cur], n, r.pixel, static_cast<uint32_t>(r.n), r.row_start,
                            r.row_count, r.t, r.irr, r.n_samples, t_state, t_end, long_row, listed.p, evb, counters.p,
                            k_dev.p, rest, row_rest_count.p, rest_blocks, fresh, s);
      } else {
        CK(cudaMemsetAsync(row_of.p, 0xFF, n * sizeof(int32_t), s));
        launch_scatter_rows(r.pixel, static_cast<uint32_t>(r.n), row_of.p, n, counters.p, s);
        CK(cudaEventRecord(timer.a, s));
        launch_advance_runs(k, cc, tab, map, soa[cur], soa[1 - cur], n, nullptr, r.n ? row_of.p : nullptr,
                            r.row_start, r.row_count, r.t, r.irr, r.n_samples, t_state, t_end, evb, counters.p, block,
                            s);
      }
      CK(cudaGetLastError());
      CK(cudaEventRecord(timer.b, s));
      read_counters(s);
      float ms = 0;
      cudaEventElapsedTime(&ms, timer.a, timer.b);
      ++stat_launches;
      launch_ms_total += ms;
      launch_ms_max = std::max(launch_ms_max, static_cast<double>(ms));
      const unsigned long long* c = counters_h.p;
      if (c[kCntErrors] != 0) throw std::invalid_argument(error_text(c[kCntErrors]));
      if (c[kCntEvents] > event_cap) {
        ++stat_reruns;
        ensure_events(static_cast<size_t>(c[kCntEvents] + c[kCntEvents] / 4 + 1024));
        continue;
      }
      stat_pieces += c[kCntPieces];
      stat_leaves += c[kCntLeaves];
      stat_clamps += c[kCntClamps];
      stat_samples += c[kCntSamples];
      stat_noise += c[kCntNoise];
      last_events = static_cast<size_t>(c[kCntEvents]);
      cur = 1 - cur;
      t_state = t_end;
      fresh = false;
      return;
    }
  }

  void advance_host(const uint32_t* ids, size_t nr, const int64_t* t, const float* irr, size_t ns,
                    const int64_t* row_start, const int32_t* row_count, int64_t t_end) {
    check_ready(t_end);
    if (nr > 0 && (!ids || !row_start || !row_count)) throw std::invalid_argument("advance: null run arrays");
    if (ns > 0 && (!t || !irr)) throw std::invalid_argument("advance: null sample arrays");
    s_pixel.ensure(nr);
    s_start.ensure(nr);
    s_count.ensure(nr);
    s_t.ensure(ns);
    s_irr.ensure(ns);
    if (nr) {
      CK(cudaMemcpyAsync(s_pixel.p, ids, nr * sizeof(uint32_t), cudaMemcpyHostToDevice, own));
      CK(cudaMemcpyAsync(s_start.p, row_start, nr * sizeof(int64_t), cudaMemcpyHostToDevice, own));
      CK(cudaMemcpyAsync(s_count.p, row_count, nr * sizeof(int32_t), cudaMemcpyHostToDevice, own));
    }
    if (ns) {
      CK(cudaMemcpyAsync(s_t.p, t, ns * sizeof(int64_t), cudaMemcpyHostToDevice, own));
      CK(cudaMemcpyAsync(s_irr.p, irr, ns * sizeof(float), cudaMemcpyHostToDevice, own));
    }
    bs_device_runs r{s_pixel.p, s_start.p, s_count.p, nr, s_t.p, s_irr.p, ns};
    advance_device(r, t_end, own);
    kept = download(events.p, last_events, own);
  }

  // The events of a call, sorted by (t_cross, pixel) on the device (finish_events' order) and copied into pinned
  // host memory; the pointer stays valid until the next download.
  const RawEvent* download_pinned(const RawEvent* dev, size_t count, cudaStream_t s) const {
    staged.ensure(count);
    if (count) {
      if (count > 0x7fffffffull) throw std::invalid_argument("too many events in one call");
      const uint32_t n = static_cast<uint32_t>(count);
      sorted.ensure(count);
      sort_scratch.ensure(sort_events_scratch_bytes(n));
      CK(sort_events(dev, n, sorted.p, sort_scratch.p, s));
      CK(cudaMemcpyAsync(staged.p, sorted.p, count * sizeof(RawEvent), cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
    }
    return staged.p;
  }
  std::vector<RawEvent> download(const RawEvent* dev, size_t count, cudaStream_t s) const {
    const RawEvent* p = download_pinned(dev, count, s);
    return std::vector<RawEvent>(p, p + count);
  }
  mutable DevBuf<RawEvent> sorted;
  mutable DevBuf<unsigned char> sort_scratch;
  mutable PinBuf<RawEvent> staged;
  mutable DevBuf<unsigned char> col_dev;
  mutable PinBuf<unsigned char> col_pin;

  // A download's columns: the caller's array, the element size and the column's offset in the pinned buffer.
  struct Col {
    void* dst;
    size_t elem;
    size_t at;
  };
  mutable Col pend_cols[12] = {};
  mutable size_t pend_count = 0;
  mutable std::chrono::steady_clock::time_point pend_w0;

  // The events of a device buffer, sorted on the device, split there into the requested columns (256-byte aligned,
  // side by side), copied out in one transfer through pinned memory, then each column into the caller's array.
  void download_columns(const RawEvent* dev, size_t count, bs_event_columns* o, cudaStream_t s) const {
    if (!download_enqueue(dev, count, o, s)) return;
    CK(cudaStreamSynchronize(s));
    download_finish();
  }

  // The download's device part queued on stream s (the sort, the column split, the copy out, with the timing events;
  // take_timer_copy.b marks the copy's end); false when there is nothing to copy.
  bool download_enqueue(const RawEvent* dev, size_t count, const bs_event_columns* o, cudaStream_t s) const {
    pend_w0 = std::chrono::steady_clock::now();
    pend_count = 0;
    for (double& v : take_ms) v = 0.0;
    if (count == 0) return false;
    if (count > 0x7fffffffull) throw std::invalid_argument("too many events in one call");
    const uint32_t n = static_cast<uint32_t>(count);
    sorted.ensure(count);
    sort_scratch.ensure(sort_events_scratch_bytes(n));
    CK(cudaEventRecord(take_timer.a, s));
    CK(sort_events(dev, n, sorted.p, sort_scratch.p, s));
    Col cols[12] = {{o->pixel, 4, 0},      {o->x, 2, 0},     {o->y, 2, 0},  {o->p, 1, 0},
                    {o->t_cross_ns, 8, 0}, {o->t_reported_ns, 8, 0},        {o->label, 1, 0},
                    {o->flags, 2, 0},      {o->ds, 4, 0},    {o->dn, 4, 0}, {o->dl, 4, 0},
                    {o->l_first, 4, 0}};
    size_t total = 0;
    for (Col& c : cols) {
      if (!c.dst) continue;
      c.at = total;
      total += (c.elem * count + 255) & ~size_t{255};
    }
    if (total == 0) return false;
    col_dev.ensure(total);
    col_pin.ensure(total);
    unsigned char* base = col_dev.p;
    const auto at = [&](int i) { return cols[i].dst ? static_cast<void*>(base + cols[i].at) : nullptr; };
    const EventColumnsDev d{static_cast<uint32_t*>(at(0)), static_cast<uint16_t*>(at(1)),
                            static_cast<uint16_t*>(at(2)), static_cast<uint8_t*>(at(3)),
                            static_cast<int64_t*>(at(4)), static_cast<int64_t*>(at(5)),
                            static_cast<uint8_t*>(at(6)), static_cast<uint16_t*>(at(7)),
                            static_cast<float*>(at(8)),   static_cast<float*>(at(9)),
                            static_cast<float*>(at(10)),  static_cast<float*>(at(11))};
    CK(event_columns(sorted.p, n, width, readout(), d, s));
    CK(cudaEventRecord(take_timer.b, s));
    CK(cudaMemcpyAsync(col_pin.p, col_dev.p, total, cudaMemcpyDeviceToHost, s));
    CK(cudaEventRecord(take_timer_copy.b, s));
    std::copy(cols, cols + 12, pend_cols);
    pend_count = count;
    return true;
  }

  // The download's host part, once its copy out has completed: the columns into the caller's arrays, up to 8
  // threads, each over an equal share of all the columns' bytes (a share can span columns; the caller's fresh pages
  // are first touched here, so the shares fault in parallel).
  void download_finish() const {
    const size_t count = pend_count;
    if (count == 0) return;
    const auto w1 = std::chrono::steady_clock::now();
    float ms_split = 0.0f, ms_copy = 0.0f;
    cudaEventElapsedTime(&ms_split, take_timer.a, take_timer.b);
    cudaEventElapsedTime(&ms_copy, take_timer.b, take_timer_copy.b);
    take_ms[0] = ms_split;
    take_ms[1] = ms_copy;
    size_t bytes = 0;
    for (const Col& c : pend_cols) {
      if (c.dst) bytes += c.elem * count;
    }
    const auto copy_range = [&](size_t lo, size_t hi) {
      size_t base_at = 0;
      for (const Col& c : pend_cols) {
        if (!c.dst) continue;
        const size_t len = c.elem * count, a = std::max(lo, base_at), b = std::min(hi, base_at + len);
        if (a < b) {
          std::memcpy(static_cast<unsigned char*>(c.dst) + (a - base_at), col_pin.p + c.at + (a - base_at), b - a);
        }
        base_at += len;
      }
    };
    const size_t hw = std::max<size_t>(1, std::thread::hardware_concurrency());
    const size_t k = bytes < (size_t{4} << 20) ? 1 : std::min<size_t>({8, hw, bytes >> 20});
    if (k == 1) {
      copy_range(0, bytes);
    } else {
      std::vector<std::thread> th;
      for (size_t i = 0; i < k; ++i) th.emplace_back(copy_range, bytes * i / k, bytes * (i + 1) / k);
      for (std::thread& t : th) t.join();
    }
    const auto w2 = std::chrono::steady_clock::now();
    take_ms[2] = std::chrono::duration<double, std::milli>(w2 - w1).count();
    take_ms[3] = std::chrono::duration<double, std::milli>(w2 - pend_w0).count();
    pend_count = 0;
  }

  // ---- the output stage: events in output order, released at the model time's cut, the rest held ----
  DevBuf<OutRecord> out_held, out_all, out_sorted;
  DevBuf<unsigned char> out_scratch;
  DevBuf<unsigned long long> out_ready;
  PinBuf<OutRecord> out_pin;
  PinBuf<unsigned long long> out_ready_h;
  size_t n_held = 0, n_ready = 0;

  ReadoutDev readout() const {
    return ReadoutDev{std::llround(p.readout_quantum_s * 1e9), std::llround(p.readout_delay_s * 1e9), readout_phase,
                      p.clock_offset_ns, p.clock_drift_ppm};
  }
  int y_bits() const {
    int b = 1;
    while ((uint64_t{1} << b) < height) ++b;
    return b;
  }

  // Moves the last call's events (not yet taken) and the held ones through the output stage; returns how many are
  // released (output_take copies them out).
  size_t output_prepare() {
    const size_t n_raw = last_events;
    const size_t total = n_held + n_raw;
    if (total > 0x7fffffffull) throw std::invalid_argument("too many events for the output stage");
    const uint32_t n = static_cast<uint32_t>(total);
    out_all.ensure(total);
    out_sorted.ensure(total);
    out_scratch.ensure(output_scratch_bytes(n));
    out_ready.ensure(1);
    out_ready_h.ensure(1);
    const int64_t limit = output_cut(readout(), t_state);
    CK(output_stage(out_held.p, static_cast<uint32_t>(n_held), events.p, static_cast<uint32_t>(n_raw), width,
                    y_bits(), readout(), limit, out_all.p, out_sorted.p, out_scratch.p, out_ready.p, own));
    CK(cudaMemcpyAsync(out_ready_h.p, out_ready.p, sizeof(unsigned long long), cudaMemcpyDeviceToHost, own));
    CK(cudaStreamSynchronize(own));
    n_ready = static_cast<size_t>(out_ready_h.p[0]);
    out_pin.ensure(n_ready);
    if (n_ready) {
      CK(cudaMemcpyAsync(out_pin.p, out_sorted.p, n_ready * sizeof(OutRecord), cudaMemcpyDeviceToHost, own));
    }
    const size_t keep = total - n_ready;
    out_held.ensure(keep);
    if (keep) {
      CK(cudaMemcpyAsync(out_held.p, out_sorted.p + n_ready, keep * sizeof(OutRecord), cudaMemcpyDeviceToDevice,
                         own));
    }
    CK(cudaStreamSynchronize(own));
    n_held = keep;
    last_events = 0;  // the call's events now belong to the output stage
    kept.clear();
    return n_ready;
  }

  void output_take(bs_output_columns* o) {
    for (size_t i = 0; i < n_ready; ++i) {
      const OutRecord& r = out_pin.p[i];
      if (o->t_reported_ns) o->t_reported_ns[i] = r.t_reported;
      if (o->t_cross_ns) o->t_cross_ns[i] = r.t_cross;
      if (o->x) o->x[i] = r.x;
      if (o->y) o->y[i] = r.y;
      if (o->flags) o->flags[i] = r.flags;
      if (o->p) o->p[i] = r.p;
      if (o->label) o->label[i] = r.label;
    }
    n_ready = 0;
  }

  int64_t reported(int64_t t) const { return reported_time(readout(), t); }

  void columns(const std::vector<RawEvent>& ev, bs_event_columns* o) const { columns(ev.data(), ev.size(), o); }
  void columns(const RawEvent* ev, size_t n, bs_event_columns* o) const {
    for (size_t i = 0; i < n; ++i) {
      const RawEvent& e = ev[i];
      if (o->pixel) o->pixel[i] = e.pixel;
      if (o->x) o->x[i] = static_cast<uint16_t>(e.pixel % width);
      if (o->y) o->y[i] = static_cast<uint16_t>(e.pixel / width);
      if (o->p) o->p[i] = e.polarity;
      if (o->t_cross_ns) o->t_cross_ns[i] = e.t_cross;
      if (o->t_reported_ns) o->t_reported_ns[i] = reported(e.t_cross);
      if (o->label) o->label[i] = e.label;
      if (o->flags) o->flags[i] = e.flags;
      if (o->ds) o->ds[i] = e.ds;
      if (o->dn) o->dn[i] = e.dn;
      if (o->dl) o->dl[i] = e.dl;
      if (o->l_first) o->l_first[i] = e.l_first;
    }
  }

  // save / load in the reference's saved-state format (SensorModel::save_state / load_state,
  // src/sensor/sensor_model.cpp:1198-1262): a StateHeader, then one 200-byte PixelState (src/sensor/pixel.h:105-121,
  // fp64 fields) per pixel in pixel order. This model's fp32 state converts to and from the fp64 fields exactly, as
  // the reference's fp32 kernel's load / store do (pixel.h:976-1041); the lattice's rho is stored as rho_m1 = rho - 1
  // under transient diffusion and 0 under frozen (exact: rho is a float ratio). Fields a photoreceptor does not use
  // are written 0 and not read. With this project's shot and background-activity noise on, one NoiseRecord per pixel
  // follows (the two candidate chains' next times and counts; the reference has no such noise).
  struct StateHeader {
    uint32_t magic, version;
    uint32_t width, height;
    uint32_t groups, camera;
    uint64_t seed;
    uint64_t fingerprint;
    int64_t t_state;
    uint32_t initialized;
    uint32_t state_size;
  };
  struct PixelStateRec {
    double z, x1, s2, s3, i_scale, tv, nk[3], nk1[3], ln_a1;
    int64_t cell, t_ref;
    double s3_ref, n3_ref, dr_ref;
    int64_t blind_until, t_search;
    float held[8];
    uint16_t flags;
    uint8_t have_k1, reserved;
    float rho_m1;
  };
  struct NoiseRecord {
    int64_t t_shot, t_ba;
    uint32_t n_shot, n_ba;
    uint32_t pad[2];
  };
  static_assert(sizeof(StateHeader) == 56, "StateHeader layout is the reference's");
  static_assert(sizeof(PixelStateRec) == 200, "PixelState layout is the reference's");
  static_assert(sizeof(NoiseRecord) == 32, "NoiseRecord is 32 bytes");
  static constexpr uint32_t kStateMagic = 0x534e5342;  // "BSNS" (sensor_model.cpp:28)
  static constexpr uint32_t kStateVersion = 6, kStateVersionNoHpf = 5;
  int mode() const { return k.cascade == 0 ? 0 : (p.noise != 0 ? 2 : 1); }
  size_t i64_words() const { return StateBufs::i64_words(mode()); }
  size_t f32_words() const { return StateBufs::f32_words(mode()); }
  size_t u32_words() const { return StateBufs::u32_words(mode()); }
  bool noise_section() const { return k.noise != 0; }
  size_t state_bytes() const {
    return sizeof(StateHeader) + static_cast<size_t>(n) * sizeof(PixelStateRec) +
           (noise_section() ? static_cast<size_t>(n) * sizeof(NoiseRecord) : 0);
  }
  // state_fingerprint (sensor_model.cpp:53-66): the parameters' fingerprint, continued over the gains when some gain
  // is not 1.
  uint64_t fingerprint() const {
    if (std::all_of(gain.begin(), gain.end(), [](float v) { return v == 1.0f; })) return p.fingerprint;
    return fnv1a(gain.data(), gain.size() * sizeof(float), p.fingerprint);
  }

  void save(uint8_t* out, size_t bytes) const {
    if (bytes != state_bytes()) throw std::invalid_argument("SensorModel.save_state: buffer size does not match");
    StateHeader h{kStateMagic, kStateVersion, width, height, 1u, camera, seed, fingerprint(), t_state,
                  initialized ? 1u : 0u, static_cast<uint32_t>(sizeof(PixelStateRec))};
    std::memcpy(out, &h, sizeof(h));
    const StateBufs& b = st[cur];
    const size_t ni = i64_words() * n, nf = f32_words() * n, nu = u32_words() * n;
    std::vector<int64_t> i64(ni);
    std::vector<float> f32(nf);
    std::vector<uint32_t> u32(nu);
    CK(cudaMemcpy(i64.data(), b.i64.p, ni * sizeof(int64_t), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(f32.data(), b.f32.p, nf * sizeof(float), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(u32.data(), b.u32.p, nu * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    const int md = mode();
    const bool transient = md == 2 && p.noise_diffusion == 1;
    uint8_t* q = out + sizeof(h);
    for (size_t i = 0; i < n; ++i) {
      PixelStateRec r{};
      r.t_ref = i64[i];
      r.t_search = i64[n + i];
      r.blind_until = i64[2 * n + i];
      r.s3_ref = f32[i];
      r.n3_ref = f32[n + i];
      r.dr_ref = f32[2 * n + i];
      r.i_scale = f32[3 * n + i];
      r.held[0] = f32[4 * n + i];
      r.flags = static_cast<uint16_t>(u32[i]);
      if (md >= 1) {
        r.z = f32[5 * n + i];
        r.x1 = f32[6 * n + i];
        r.s2 = f32[7 * n + i];
        r.s3 = f32[8 * n + i];
        r.tv = f32[9 * n + i];
      }
      if (md == 2) {
        for (int j = 0; j < 3; ++j) {
          r.nk[j] = f32[(10 + j) * n + i];
          r.nk1[j] = f32[(13 + j) * n + i];
        }
        r.ln_a1 = f32[16 * n + i];
        r.rho_m1 = transient ? f32[17 * n + i] - 1.0f : 0.0f;
        r.cell = i64[5 * n + i];
        r.have_k1 = u32[3 * n + i] != 0u ? 1 : 0;
      }
      std::memcpy(q + i * sizeof(PixelStateRec), &r, sizeof(r));
    }
    if (noise_section()) {
      uint8_t* z = q + n * sizeof(PixelStateRec);
      for (size_t i = 0; i < n; ++i) {
        const NoiseRecord r{i64[3 * n + i], i64[4 * n + i], u32[n + i], u32[2 * n + i], {0u, 0u}};
        std::memcpy(z + i * sizeof(NoiseRecord), &r, sizeof(r));
      }
    }
  }

  void load(const uint8_t* data, size_t bytes) {
    if (bytes != state_bytes()) throw std::invalid_argument("SensorModel.load_state: size does not match this model");
    StateHeader h;
    std::memcpy(&h, data, sizeof(h));
    if (h.magic != kStateMagic || (h.version != kStateVersion && h.version != kStateVersionNoHpf) ||
        h.state_size != sizeof(PixelStateRec)) {
      throw std::invalid_argument("SensorModel.load_state: not a sensor state of this version");
    }
    if (h.width != width || h.height != height || h.groups != 1u || h.camera != camera || h.seed != seed ||
        h.fingerprint != fingerprint()) {
      throw std::invalid_argument("SensorModel.load_state: state was saved by a model with other parameters");
    }
    initialized = false;  // until the upload completes
    const size_t ni = i64_words() * n, nf = f32_words() * n, nu = u32_words() * n;
    std::vector<int64_t> i64(ni, 0);
    std::vector<float> f32(nf, 0.0f);
    std::vector<uint32_t> u32(nu, 0u);
    const int md = mode();
    const uint8_t* q = data + sizeof(h);
    for (size_t i = 0; i < n; ++i) {
      PixelStateRec r;
      std::memcpy(&r, q + i * sizeof(PixelStateRec), sizeof(r));
      i64[i] = r.t_ref;
      i64[n + i] = r.t_search;
      i64[2 * n + i] = r.blind_until;
      i64[3 * n + i] = kForever;  // the noise chains (the noise section below, when on)
      i64[4 * n + i] = kForever;
      f32[i] = static_cast<float>(r.s3_ref);
      f32[n + i] = static_cast<float>(r.n3_ref);
      f32[2 * n + i] = static_cast<float>(r.dr_ref);
      f32[3 * n + i] = static_cast<float>(r.i_scale);
      f32[4 * n + i] = r.held[0];
      u32[i] = r.flags;
      if (md >= 1) {
        f32[5 * n + i] = static_cast<float>(r.z);
        f32[6 * n + i] = static_cast<float>(r.x1);
        f32[7 * n + i] = static_cast<float>(r.s2);
        f32[8 * n + i] = static_cast<float>(r.s3);
        f32[9 * n + i] = static_cast<float>(r.tv);
      }
      if (md == 2) {
        for (int j = 0; j < 3; ++j) {
          f32[(10 + j) * n + i] = static_cast<float>(r.nk[j]);
          f32[(13 + j) * n + i] = static_cast<float>(r.nk1[j]);
        }
        f32[16 * n + i] = static_cast<float>(r.ln_a1);
        f32[17 * n + i] = 1.0f + r.rho_m1;
        i64[5 * n + i] = r.cell;
        u32[3 * n + i] = r.have_k1 != 0 ? 1u : 0u;
      }
    }
    if (noise_section()) {
      const uint8_t* z = q + n * sizeof(PixelStateRec);
      for (size_t i = 0; i < n; ++i) {
        NoiseRecord r;
        std::memcpy(&r, z + i * sizeof(NoiseRecord), sizeof(r));
        i64[3 * n + i] = r.t_shot;
        i64[4 * n + i] = r.t_ba;
        u32[n + i] = r.n_shot;
        u32[2 * n + i] = r.n_ba;
      }
    }
    StateBufs& b = st[cur];
    CK(cudaMemcpy(b.i64.p, i64.data(), ni * sizeof(int64_t), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(b.f32.p, f32.data(), nf * sizeof(float), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(b.u32.p, u32.data(), nu * sizeof(uint32_t), cudaMemcpyHostToDevice));
    t_state = h.t_state;
    initialized = h.initialized != 0;
    fresh = false;
    last_events = 0;
    kept.clear();
  }
};

// ---------------------------------------------------------------------------------------------
// the sampler
// ---------------------------------------------------------------------------------------------
struct FieldHolder {
  FieldDev f{};
  DevBuf<float> blobs;
  void set(const bs_field& h) {
    if (h.kind != kFieldTanhEdge && h.kind != kFieldBlobs) throw std::invalid_argument("field: unknown kind");
    if (h.width == 0 || h.height == 0) throw std::invalid_argument("field: empty frame");
    if (h.kind == kFieldBlobs && h.n_blobs > 0 && !h.blobs) throw std::invalid_argument("field: null blob table");
    f.kind = h.kind;
    f.width = h.width;
    f.height = h.height;
    f.base = h.base;
    f.amp = h.amp;
    f.nx = h.nx;
    f.ny = h.ny;
    f.c = h.c;
    f.speed = h.speed;
    f.width_px = h.width_px;
    f.n_blobs = h.kind == kFieldBlobs ? h.n_blobs : 0;
    f.blobs = nullptr;
    if (f.n_blobs > 0) {
      blobs.ensure(static_cast<size_t>(f.n_blobs) * kBlobWords);
      CK(cudaMemcpy(blobs.p, h.blobs, static_cast<size_t>(f.n_blobs) * kBlobWords * sizeof(float),
                    cudaMemcpyHostToDevice));
      f.blobs = blobs.p;
    }
  }
};

SamplerRules make_rules(const bs_sample_rules& r) {
  if (r.min_dt_ns < 1 || r.min_dt_ns > kWindowNs || (r.min_dt_ns & (r.min_dt_ns - 1)) != 0) {
    throw std::invalid_argument("min_dt_ns must be a power of two in [1, 2^23]");
  }
  if (r.max_refine_levels < 0) throw std::invalid_argument("max_refine_levels must be >= 0");
  int shift = 0;
  while ((int64_t{1} << shift) < r.min_dt_ns) ++shift;
  SamplerRules s{};
  s.tol = r.tol;
  s.dark = r.dark;
  s.midpoint = r.midpoint;
  s.refine_signature = r.refine_signature;
  // A depth-first walk stops where halves fall under min_split anyway; deeper caps change nothing.
  s.max_refine_levels = std::min(r.max_refine_levels, 23);
  s.min_split = static_cast<uint32_t>(2 * r.min_dt_ns);
  s.l_min = r.l_min;
  s.l_max = std::min(r.l_max, kWindowLog2 - shift);
  return s;
}

struct Sampler {
  DeviceGate gate;
  FieldHolder field;
  cudaStream_t own = nullptr;
  DevBuf<uint32_t> pixel, counts;
  DevBuf<uint8_t> level;
  DevBuf<float> carried_in, carried_out, irr;
  DevBuf<uint64_t> sig_in, sig_out;
  DevBuf<int64_t> offsets, scratch, t;
  size_t n = 0, samples = 0;
  explicit Sampler(const bs_field& f) {
    require_device();
    field.set(f);
    CK(cudaStreamCreateWithFlags(&own, cudaStreamNonBlocking));
  }
  ~Sampler() {
    if (own) cudaStreamDestroy(own);
  }

  void window(int64_t t_w, const uint32_t* ids, const uint8_t* lv, size_t np, float* c_irr, uint64_t* c_sig,
              const bs_sample_rules& rr) {
    const SamplerRules r = make_rules(rr);
    int shift = 0;
    while ((int64_t{1} << shift) < rr.min_dt_ns) ++shift;
    const int max_level = kWindowLog2 - shift;
    for (size_t i = 0; i < np; ++i) {
      if (lv[i] > max_level) throw std::invalid_argument("levels must lie in [0, 23 - log2(min_dt_ns)]");
      if (ids[i] >= field.f.width * field.f.height) throw std::invalid_argument("pixel id outside the field");
    }
    if (np > 0xFFFFFFFFull) throw std::invalid_argument("too many pixels");
    n = np;
    dev_ids = nullptr;
    pixel.ensure(np);
    level.ensure(np);
    carried_in.ensure(np);
    carried_out.ensure(np);
    sig_in.ensure(np);
    sig_out.ensure(np);
    counts.ensure(np);
    offsets.ensure(np + 1);
    scratch.ensure(scan_scratch_words(static_cast<uint32_t>(np)));
    cudaStream_t s = own;
    if (np) {
      CK(cudaMemcpyAsync(pixel.p, ids, np * 4, cudaMemcpyHostToDevice, s));
      CK(cudaMemcpyAsync(level.p, lv, np, cudaMemcpyHostToDevice, s));
      CK(cudaMemcpyAsync(carried_in.p, c_irr, np * 4, cudaMemcpyHostToDevice, s));
      CK(cudaMemcpyAsync(sig_in.p, c_sig, np * 8, cudaMemcpyHostToDevice, s));
    }
    launch_sample_window(field.f, r, t_w, pixel.p, level.p, static_cast<uint32_t>(np), carried_in.p, sig_in.p,
                         counts.p, nullptr, nullptr, nullptr, nullptr, nullptr, 0, s);
    launch_scan(counts.p, static_cast<uint32_t>(np), offsets.p, scratch.p, s);
    CK(cudaGetLastError());
    int64_t total = 0;
    CK(cudaMemcpyAsync(&total, offsets.p + np, 8, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    samples = static_cast<size_t>(total);
    t.ensure(samples);
    irr.ensure(samples);
    launch_sample_window(field.f, r, t_w, pixel.p, level.p, static_cast<uint32_t>(np), carried_in.p, sig_in.p,
                         counts.p, offsets.p, t.p, irr.p, carried_out.p, sig_out.p, 1, s);
    CK(cudaGetLastError());
    if (np) {
      CK(cudaMemcpyAsync(c_irr, carried_out.p, np * 4, cudaMemcpyDeviceToHost, s));
      CK(cudaMemcpyAsync(c_sig, sig_out.p, np * 8, cudaMemcpyDeviceToHost, s));
    }
    CK(cudaStreamSynchronize(s));
  }

  // The same window with every input and the carried samples in device memory (WindowEngine<Space::kDevice>::run,
  // src/engine/window.h:133-174): the ids and levels are read in place and checked on the device, the carried
  // samples are read from c_in / s_in and the window's last samples written to c_out / s_out (the caller's device
  // arrays; they may not alias). The runs stay in this sampler's memory (bs_sampler_device_runs). Two
  // synchronizations of `s` read the check and the sample count; the write pass is left queued on `s`.
  void window_device(int64_t t_w, const uint32_t* ids, const uint8_t* lv, size_t np, const float* c_in,
                     const uint64_t* s_in, float* c_out, uint64_t* s_out, const bs_sample_rules& rr, cudaStream_t s) {
    const SamplerRules r = make_rules(rr);
    int shift = 0;
    while ((int64_t{1} << shift) < rr.min_dt_ns) ++shift;
    if (np > 0xFFFFFFFFull) throw std::invalid_argument("too many pixels");
    const uint32_t nn = static_cast<uint32_t>(np);
    counts.ensure(np);
    offsets.ensure(np + 1);
    scratch.ensure(scan_scratch_words(nn));
    info.ensure(2);
    // One walk: the samples staged in a scratch list (room for the last window's total and a quarter, at least
    // 8 a pixel; a pixel that does not fit is walked again when its row is written). The walk checks each pixel's
    // id and level first (a lattice level sets the walk's length); the flags come back with the total, and nothing
    // the caller passed is written unless both are clear.
    const size_t cap = std::min<size_t>(std::max<size_t>(np * 8, stage_want), 0xFFFFFFF0ull);
    stage_dt.ensure(cap);
    stage_v.ensure(cap);
    stage_at.ensure(np);
    stage_c.ensure(np);
    stage_s.ensure(np);
    stage_used.ensure(4);  // [0] the list's use, [2..3] the flags
    unsigned long long* flags = reinterpret_cast<unsigned long long*>(stage_used.p + 2);
    CK(cudaMemsetAsync(stage_used.p, 0, 4 * sizeof(unsigned int), s));
    launch_sample_window_staged(field.f, r, t_w, ids, lv, nn, c_in, s_in, counts.p, nullptr, nullptr, nullptr, c_out,
                                s_out, stage_dt.p, stage_v.p, stage_at.p, stage_used.p, static_cast<uint32_t>(cap),
                                stage_c.p, stage_s.p, field.f.width * field.f.height, kWindowLog2 - shift, flags, 0, s);
    launch_scan(counts.p, nn, offsets.p, scratch.p, s);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(info.p, flags, 8, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(info.p + 1, offsets.p + np, 8, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (info.p[0] & 1ull) throw std::invalid_argument("levels must lie in [0, 23 - log2(min_dt_ns)]");
    if (info.p[0] & 2ull) throw std::invalid_argument("pixel id outside the field");
    n = np;
    dev_ids = ids;
    samples = static_cast<size_t>(info.p[1]);
    stage_want = samples + samples / 4;
    t.ensure(samples);
    irr.ensure(samples);
    launch_sample_window_staged(field.f, r, t_w, ids, lv, nn, c_in, s_in, counts.p, offsets.p, t.p, irr.p, c_out,
                                s_out, stage_dt.p, stage_v.p, stage_at.p, stage_used.p, static_cast<uint32_t>(cap),
                                stage_c.p, stage_s.p, field.f.width * field.f.height, kWindowLog2 - shift, flags, 1, s);
    CK(cudaGetLastError());
  }
  DevBuf<uint32_t> stage_dt;  // the one-walk path's scratch list of staged samples, and each pixel's start in it
  DevBuf<float> stage_v;
  DevBuf<uint32_t> stage_at;
  DevBuf<unsigned int> stage_used;
  DevBuf<float> stage_c;  // each pixel's carried sample and signature until the rows are placed
  DevBuf<uint64_t> stage_s;
  size_t stage_want = 0;
  PinBuf<unsigned long long> info;
  const uint32_t* dev_ids = nullptr;  // the last device window's ids (the caller's array), null after a host window
};

// ---------------------------------------------------------------------------------------------
// the learned step proposal: the MLP and its training pairs
// ---------------------------------------------------------------------------------------------
struct LearnedBufs {
  DevBuf<float> hx, pv;
  DevBuf<uint64_t> gaps;
  DevBuf<uint8_t> valid;
  LearnedSoA soa(size_t n) {
    return LearnedSoA{hx.ensure(8 * n), gaps.ensure(n), pv.ensure(n), valid.ensure(n)};
  }
};

struct Mlp {
  DeviceGate gate;
  DevBuf<float> params, m, v, partial, losses;
  DevBuf<uint16_t> ops;
  DevBuf<double> partial_loss, grad, loss;
  DevBuf<int64_t> step;
  DevBuf<unsigned int> done;  // [0]: Adam's block counter; [1]: the training kernel's error word
  cudaStream_t own = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint64_t graph_key[8] = {};
  static constexpr int64_t kLossCap = int64_t{1} << 22;  // steps whose loss is kept

  // He-uniform weights (U(-a, a), a = sqrt(6 / fan_in)) from Philox, zero biases, Adam state zero.
  explicit Mlp(uint64_t seed) {
    CK(cudaStreamCreateWithFlags(&own, cudaStreamNonBlocking));
    std::vector<float> h(kMlpParams, 0.0f);
    for (int p = 0; p < kMlpParams; ++p) {
      float a = 0.0f;
      if (p < kOffB1) a = std::sqrt(6.0f / kMlpIn);
      else if (p >= kOffW2 && p < kOffB2) a = std::sqrt(6.0f / kMlpHid);
      else if (p >= kOffW3 && p < kOffB3) a = std::sqrt(6.0f / kMlpHid);
      if (a == 0.0f) continue;
      const U4 u = draw(seed, kPurposeInit, 0u, static_cast<uint32_t>(p), 0);
      const float r = (static_cast<float>(u.v[0] >> 8) + 0.5f) * 0x1p-24f;
      h[p] = (2.0f * r - 1.0f) * a;
    }
    params.ensure(kMlpParams);
    m.ensure(kMlpParams);
    v.ensure(kMlpParams);
    ops.ensure(kOpWords);
    step.ensure(1);
    done.ensure(2);
    grad.ensure(kMlpParams);
    loss.ensure(1);
    losses.ensure(kLossCap);
    set(h.data());
  }
  ~Mlp() {
    release_graph();
    if (own) cudaStreamDestroy(own);
  }
  void release_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
  }

  void set(const float* h) {
    for (int p = 0; p < kMlpParams; ++p) {
      if (!std::isfinite(h[p])) throw std::invalid_argument("mlp: non-finite parameter " + std::to_string(p));
    }
    CK(cudaMemcpyAsync(params.p, h, kMlpParams * sizeof(float), cudaMemcpyHostToDevice, own));
    CK(cudaMemsetAsync(m.p, 0, kMlpParams * sizeof(float), own));
    CK(cudaMemsetAsync(v.p, 0, kMlpParams * sizeof(float), own));
    CK(cudaMemsetAsync(ops.p, 0, kOpWords * sizeof(uint16_t), own));
    CK(cudaMemsetAsync(step.p, 0, sizeof(int64_t), own));
    CK(cudaMemsetAsync(done.p, 0, 2 * sizeof(unsigned int), own));
    launch_operands(params.p, ops.p, own);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(own));
  }
  void get(float* h) const {
    CK(cudaMemcpy(h, params.p, kMlpParams * sizeof(float), cudaMemcpyDeviceToHost));
  }
  int64_t steps() const {
    int64_t s = 0;
    CK(cudaMemcpy(&s, step.p, sizeof(int64_t), cudaMemcpyDeviceToHost));
    return s;
  }

  void forward(const uint16_t* x, size_t n, float* y, cudaStream_t s) {
    if (n && (!x || !y)) throw std::invalid_argument("mlp.forward: null device array");
    launch_mlp_forward(ops.p, params.p, x, n, y, s);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s));
  }

  void gradient(const uint16_t* x, const float* y, size_t n, double* g_host, double* loss_host, cudaStream_t s) {
    if (n == 0 || n > 0xFFFFFFFFull) throw std::invalid_argument("mlp.gradient: n must be in [1, 2^32)");
    if (!x || !y) throw std::invalid_argument("mlp.gradient: null device array");
    const int ctas = train_grid(static_cast<uint32_t>(n));
    partial.ensure(static_cast<size_t>(ctas) * kMlpParamsPad);
    partial_loss.ensure(ctas);
    TrainArgs a{x, y, n, static_cast<uint32_t>(n), 0, 0, step.p, ops.p, params.p, partial.p, partial_loss.p,
                1.0f / static_cast<float>(n), 0.5f, done.p + 1};
    launch_train_partials(a, s);
    launch_reduce_partials(partial.p, partial_loss.p, ctas, a.inv_rows, grad.p, loss.p, s);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(g_host, grad.p, kMlpParams * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(loss_host, loss.p, sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    check_chains();
  }

  // The training kernel's error word: a tensor-core chain whose completion it did not see in time.
  void check_chains() {
    unsigned int e = 0;
    CK(cudaMemcpy(&e, done.p + 1, sizeof(e), cudaMemcpyDeviceToHost));
    if (e != 0) {
      CK(cudaMemset(done.p + 1, 0, sizeof(e)));
      throw CudaError("mlp: a tensor-core chain of the training step did not complete within its wait bound");
    }
  }

  // `steps` Adam steps on batches of `batch` rows drawn with replacement from the n pairs. The steps run from a
  // CUDA graph of 32 steps (two launches each), replayed; the loss of every step is kept on the device.
  void train(const uint16_t* x, const float* y, size_t n, int32_t steps, int32_t batch, float lr, float tau,
             uint64_t seed, float* losses_host, cudaStream_t s) {
    if (!(tau > 0.0f && tau < 1.0f)) throw std::invalid_argument("mlp.train: tau must lie in (0, 1)");
    if (n == 0) throw std::invalid_argument("mlp.train: no pairs");
    if (!x || !y) throw std::invalid_argument("mlp.train: null device array");
    if (steps < 0 || batch < 1 || batch > (1 << 24)) throw std::invalid_argument("mlp.train: bad steps or batch");
    if (!(lr > 0.0f) || !std::isfinite(lr)) throw std::invalid_argument("mlp.train: lr must be positive");
    const int ctas = train_grid(static_cast<uint32_t>(batch));
    partial.ensure(static_cast<size_t>(ctas) * kMlpParamsPad);
    partial_loss.ensure(ctas);
    const int64_t s0 = steps_from_device(s);
    const TrainArgs a{x, y, n, static_cast<uint32_t>(batch), 1, seed, step.p, ops.p, params.p, partial.p,
                      partial_loss.p, 1.0f / static_cast<float>(batch), tau, done.p + 1};
    auto one = [&](cudaStream_t st) {
      launch_train_partials(a, st);
      launch_adam(params.p, m.p, v.p, ops.p, partial.p, partial_loss.p, ctas, lr, a.inv_rows, step.p, losses.p,
                  static_cast<int64_t>(losses.cap), done.p, st);
    };
    constexpr int kGraphSteps = 32;
    int32_t left = steps;
    if (left > 0) {  // the first step runs eagerly (it also configures the kernel's shared-memory size)
      one(s);
      CK(cudaGetLastError());
      --left;
    }
    if (left >= kGraphSteps) {
      // The graph holds its launches' arguments and buffer addresses: rebuild it when any of them changes.
      const uint64_t key[8] = {reinterpret_cast<uint64_t>(x), reinterpret_cast<uint64_t>(y), n,
                               (static_cast<uint64_t>(batch) << 32) ^ f2u(lr), seed ^ (uint64_t{f2u(tau)} << 32),
                               reinterpret_cast<uint64_t>(partial.p), reinterpret_cast<uint64_t>(partial_loss.p),
                               static_cast<uint64_t>(ctas)};
      if (!exec || std::memcmp(key, graph_key, sizeof(key)) != 0) {
        release_graph();
        CK(cudaStreamBeginCapture(own, cudaStreamCaptureModeThreadLocal));
        for (int k = 0; k < kGraphSteps; ++k) one(own);
        CK(cudaStreamEndCapture(own, &graph));
        CK(cudaGraphInstantiate(&exec, graph, 0));
        std::memcpy(graph_key, key, sizeof(key));
      }
      // The graph runs on the library's own stream, ordered after the caller's work.
      cudaEvent_t ev;
      CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
      CK(cudaEventRecord(ev, s));
      CK(cudaStreamWaitEvent(own, ev, 0));
      while (left >= kGraphSteps) {
        CK(cudaGraphLaunch(exec, own));
        left -= kGraphSteps;
      }
      CK(cudaEventRecord(ev, own));
      CK(cudaStreamWaitEvent(s, ev, 0));
      CK(cudaEventDestroy(ev));
    }
    for (; left > 0; --left) one(s);
    CK(cudaGetLastError());
    if (losses_host && steps > 0) {
      const int64_t kept = std::max<int64_t>(0, std::min<int64_t>(steps, kLossCap - s0));
      for (int32_t i = static_cast<int32_t>(kept); i < steps; ++i) losses_host[i] = NAN;
      if (kept > 0) {
        CK(cudaMemcpyAsync(losses_host, losses.p + s0, static_cast<size_t>(kept) * sizeof(float),
                           cudaMemcpyDeviceToHost, s));
      }
    }
    CK(cudaStreamSynchronize(s));
    check_chains();
  }

  int64_t steps_from_device(cudaStream_t s) {
    int64_t v0 = 0;
    CK(cudaMemcpyAsync(&v0, step.p, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return v0;
  }
};

// Training pairs from the plain sampler over windows [0, windows) of a field (every pixel listed, levels by the
// field's rule, runs on the device), walked by launch_walk_pairs.
void trace_pairs(const bs_field& fh, const bs_sample_rules& rr, int64_t t0, int32_t windows, uint32_t stride,
                 float eps, uint64_t seed, uint16_t* x, float* y, uint64_t* key, size_t cap, size_t* n_out,
                 size_t* total, cudaStream_t s) {
  if (windows < 0) throw std::invalid_argument("trace_pairs: windows must be >= 0");
  if (stride < 1) throw std::invalid_argument("trace_pairs: stride must be >= 1");
  if (!(eps > 0.0f)) throw std::invalid_argument("trace_pairs: eps must be positive");
  if (cap > 0 && (!x || !y)) throw std::invalid_argument("trace_pairs: null device array");
  if ((t0 & (kWindowNs - 1)) != 0) throw std::invalid_argument("trace_pairs: t0 must be a window start");
  FieldHolder field;
  field.set(fh);
  const SamplerRules r = make_rules(rr);
  int sh = 0;
  while ((int64_t{1} << sh) < rr.min_dt_ns) ++sh;
  const uint32_t np = field.f.width * field.f.height;
  std::vector<uint32_t> iota(np);
  for (uint32_t i = 0; i < np; ++i) iota[i] = i;
  DevBuf<uint32_t> ids, counts;
  DevBuf<uint8_t> level;
  DevBuf<float> carried[2], irr;
  DevBuf<uint64_t> sig[2];
  DevBuf<int64_t> offsets, scratch, t;
  DevBuf<unsigned long long> count;
  LearnedBufs walk;
  ids.ensure(np);
  counts.ensure(np);
  level.ensure(np);
  carried[0].ensure(np);
  carried[1].ensure(np);
  sig[0].ensure(np);
  sig[1].ensure(np);
  offsets.ensure(np + 1);
  scratch.ensure(scan_scratch_words(np));
  count.ensure(1);
  const LearnedSoA st = walk.soa(np);
  CK(cudaMemcpyAsync(ids.p, iota.data(), np * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
  CK(cudaMemsetAsync(sig[0].p, 0, np * sizeof(uint64_t), s));
  CK(cudaMemsetAsync(count.p, 0, sizeof(unsigned long long), s));
  launch_field_frame(field.f, t0, np, carried[0].p, s);
  int cur = 0;
  for (int32_t w = 0; w < windows; ++w) {
    const int64_t t_w = t0 + static_cast<int64_t>(w) * kWindowNs;
    launch_levels(field.f, t_w, r.l_min, r.l_max, np, level.p, s);
    launch_sample_window(field.f, r, t_w, ids.p, level.p, np, carried[cur].p, sig[cur].p, counts.p, nullptr,
                         nullptr, nullptr, nullptr, nullptr, 0, s);
    launch_scan(counts.p, np, offsets.p, scratch.p, s);
    CK(cudaGetLastError());
    int64_t n_samples = 0;
    CK(cudaMemcpyAsync(&n_samples, offsets.p + np, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    t.ensure(static_cast<size_t>(n_samples));
    irr.ensure(static_cast<size_t>(n_samples));
    launch_sample_window(field.f, r, t_w, ids.p, level.p, np, carried[cur].p, sig[cur].p, counts.p, offsets.p, t.p,
                         irr.p, carried[1 - cur].p, sig[1 - cur].p, 1, s);
    WalkArgs a{offsets.p, t.p, irr.p, level.p, np, stride, t_w, w, w == 0 ? 1 : 0, sh, eps, seed, st,
               x, y, key, count.p, static_cast<unsigned long long>(cap)};
    launch_walk_pairs(a, s);
    CK(cudaGetLastError());
    cur = 1 - cur;
  }
  unsigned long long produced = 0;
  CK(cudaMemcpyAsync(&produced, count.p, sizeof(produced), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  *total = static_cast<size_t>(produced);
  *n_out = std::min(static_cast<size_t>(produced), cap);
}

// ---------------------------------------------------------------------------------------------
// the fused engine
// ---------------------------------------------------------------------------------------------
struct Engine {
  DeviceGate gate;
  std::vector<Model*> models;
  std::vector<std::unique_ptr<FieldHolder>> fields;
  SamplerRules rules{};
  std::vector<std::unique_ptr<DevBuf<float>>> carried;  // 2 per sensor
  std::vector<int> carried_cur;
  DevBuf<EngineSensor> sensors_dev;
  DevBuf<unsigned int> tile_counter;
  std::vector<EngineSensor> host;
  uint32_t total_tiles = 0;
  int warps_per_block = 4, blocks_per_sm = 0, stage = 0, tile_lw = 3;
  double last_ms = 0;
  Timer timer;
  mutable Timer take_timer;           // the last download's device part: sort + column split
  mutable Timer take_timer_copy;      // and its device-to-host copy
  mutable double take_ms[4] = {0, 0, 0, 0};  // sort + split, copy out, host column copies, whole call (ms)
  cudaStream_t own = nullptr;
  cudaEvent_t order = nullptr;
  // The step as a CUDA graph (rebuilt when its launch shape, window count or proposal changes), fed from pinned
  // descriptors and model time.
  bool use_graph = true;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint64_t graph_key[8] = {};
  PinBuf<EngineSensor> host_pin;
  PinBuf<int64_t> t0_pin;
  DevBuf<int64_t> t0_dev;
  PinBuf<unsigned long long> rec_n_pin;
  // The learned step proposal (null: the plain sampler), its walk state (2 per sensor) and the record buffers.
  const Mlp* mlp = nullptr;
  float margin = 0.25f;
  std::vector<std::unique_ptr<LearnedBufs>> lbufs;
  std::vector<int> lcur;
  DevBuf<RecRow> rec[2];
  DevBuf<unsigned long long> rec_count;
  size_t rec_cap = 0;
  unsigned long long rec_n[2] = {0, 0};
  // The split engine (stage kStageSplit): two scratch states and carried frames per sensor that the windows between
  // a call's first and last pass the state through, the per-window descriptors, the posted-pixel list (room for every
  // pixel), and per window a tile counter and a list count.
  std::vector<std::unique_ptr<StateBufs>> split_state;
  std::vector<std::unique_ptr<DevBuf<float>>> split_carried;
  DevBuf<EngineSensor> split_desc;
  PinBuf<EngineSensor> split_desc_pin;
  DevBuf<unsigned char> rest;
  DevBuf<unsigned int> split_counts;
  unsigned int rest_capacity = 0;

  static int32_t models_cascade(bs_model* m) { return m ? reinterpret_cast<Model*>(m)->mode() : 0; }
  // 0 the instantaneous response, 1 the cascade, 2 the cascade with its noise lattice (every sensor alike).
  int cascade() const { return models.empty() ? 0 : models[0]->mode(); }

  Engine(bs_model* const* ms, const bs_field* fs, int32_t cnt, const bs_sample_rules& r) {
    require_device();
    if (cnt < 1) throw std::invalid_argument("engine: at least one sensor");
    if (cnt > 65535) throw std::invalid_argument("engine: at most 65535 sensors");
    rules = make_rules(r);
    uint32_t tile0 = 0;
    for (int32_t i = 0; i < cnt; ++i) {
      Model* m = reinterpret_cast<Model*>(ms[i]);
      if (!m) throw std::invalid_argument("engine: null model");
      if (fs[i].width != m->width || fs[i].height != m->height) {
        throw std::invalid_argument("engine: each field must have its model's frame size");
      }
      if (m->mode() != models_cascade(ms[0])) {
        throw std::invalid_argument("engine: the sensors of one engine run the same photoreceptor and noise model");
      }
      if (m->mode() == 2 && r.min_dt_ns < 4096) {
        throw std::invalid_argument("engine: the noise lattice needs min_dt_ns >= 4096 (at most 16 samples a cell)");
      }
      models.push_back(m);
      auto f = std::make_unique<FieldHolder>();
      f->set(fs[i]);
      fields.push_back(std::move(f));
      for (int b = 0; b < 2; ++b) {
        carried.push_back(std::make_unique<DevBuf<float>>());
        carried.back()->ensure(m->n);
      }
      carried_cur.push_back(0);
      EngineSensor e{};
      e.width = m->width;
      e.height = m->height;
      e.tiles_x = (m->width + 7) / 8;
      e.tiles_y = (m->height + 3) / 4;
      e.tile0 = tile0;
      tile0 += e.tiles_x * e.tiles_y;
      host.push_back(e);
    }
    total_tiles = tile0;
    retile();
    sensors_dev.ensure(host.size());
    tile_counter.ensure(1);
    t0_dev.ensure(1);
    CK(cudaStreamCreateWithFlags(&own, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&order, cudaEventDisableTiming));
  }
  ~Engine() {
    release_graph();
    if (order) cudaEventDestroy(order);
    if (own) cudaStreamDestroy(own);
  }

  void start(int64_t t0, cudaStream_t s, const float* const* host_frames = nullptr) {
    for (size_t i = 0; i < models.size(); ++i) {
      Model* m = models[i];
      float* frame = carried[2 * i + carried_cur[i]]->p;
      if (host_frames != nullptr) {
        if (!host_frames[i]) throw std::invalid_argument("engine: null frame");
        CK(cudaMemcpyAsync(frame, host_frames[i], m->n * sizeof(float), cudaMemcpyHostToDevice, s));
      } else {
        launch_field_frame(fields[i]->f, t0, m->n, frame, s);
        CK(cudaGetLastError());
      }
      m->init_device(t0, frame, s, host_frames ? host_frames[i] : nullptr);
    }
    if (mlp) reset_walks(s);
  }

  // The learned walk state of every pixel restarts from the current carried frame (a flat virtual history).
  void reset_walks(cudaStream_t s) {
    while (lbufs.size() < 2 * models.size()) lbufs.push_back(std::make_unique<LearnedBufs>());
    lcur.assign(models.size(), 0);
    for (size_t i = 0; i < models.size(); ++i) {
      const uint32_t n = models[i]->n;
      launch_learned_reset(lbufs[2 * i]->soa(n), n, carried[2 * i + carried_cur[i]]->p, s);
      lbufs[2 * i + 1]->soa(n);
    }
    CK(cudaGetLastError());
  }

  void set_proposal(const Mlp* p, float mg) {
    if (p && !std::isfinite(mg)) throw std::invalid_argument("engine: margin must be finite");
    if (p && cascade()) throw std::invalid_argument("engine: the learned proposal runs with the instantaneous response");
    mlp = p;
    margin = mg;
    if (p) {
      reset_walks(own);
      CK(cudaStreamSynchronize(own));
    }
  }

  void set_record(size_t cap) {
    rec_cap = cap;
    rec_n[0] = rec_n[1] = 0;
    if (cap) {
      rec[0].ensure(cap);
      rec[1].ensure(cap);
    }
    rec_count.ensure(2);
  }

  // Copies up to cap rows of record `which` (0 samples, 1 proposed steps) of the last run; n gets the rows recorded
  // (more than the record's capacity means the record is incomplete).
  void take_record(int which, size_t cap, int64_t* t, uint32_t* pixel, float* v, size_t* n) {
    if (which != 0 && which != 1) throw std::invalid_argument("engine: record 0 (samples) or 1 (steps)");
    const size_t have = static_cast<size_t>(std::min<unsigned long long>(rec_n[which], rec_cap));
    const size_t k = std::min(have, cap);
    std::vector<RecRow> rows(k);
    if (k) CK(cudaMemcpy(rows.data(), rec[which].p, k * sizeof(RecRow), cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < k; ++i) {
      if (t) t[i] = rows[i].t;
      if (pixel) pixel[i] = rows[i].pixel;
      if (v) v[i] = rows[i].v;
    }
    *n = static_cast<size_t>(rec_n[which]);
  }

  // The launch shape: tile width 2^tile_lw (tiles of 2^tile_lw x 2^(5 - tile_lw) px, one warp each), warps per
  // block, blocks per SM (0: as many as fit) and the plain engine's staging depth.
  void retile() {
    uint32_t tile0 = 0;
    const uint32_t tw = 1u << tile_lw, th = 32u >> tile_lw;
    for (EngineSensor& e : host) {
      e.tiles_x = (e.width + tw - 1) / tw;
      e.tiles_y = (e.height + th - 1) / th;
      e.tile0 = tile0;
      tile0 += e.tiles_x * e.tiles_y;
    }
    total_tiles = tile0;
  }

  int block_warps() const { return mlp ? 4 : warps_per_block; }
  static int sm_count() {
    int dev = 0, sms = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    return sms;
  }
  int grid_blocks() const {
    int dev = 0, sms = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int wpb = block_warps();
    const int per_sm = blocks_per_sm > 0 ? blocks_per_sm
                                         : std::max(1, mlp ? learned_engine_max_blocks_per_sm(wpb)
                                                           : engine_max_blocks_per_sm(wpb, stage, cascade()));
    return static_cast<int>(
        std::min<uint64_t>(static_cast<uint64_t>(sms) * per_sm, (total_tiles + wpb - 1) / wpb));
  }

  // Fills the pinned launch descriptors from the models' current buffers.
  void describe(int64_t t0) {
    host_pin.ensure(host.size());
    for (size_t i = 0; i < models.size(); ++i) {
      Model* m = models[i];
      EngineSensor& e = host[i];
      e.field = fields[i]->f;
      e.consts = m->k;
      e.cc = m->cc;
      e.tab = m->tab;
      e.in = m->soa[m->cur];
      e.out = m->soa[1 - m->cur];
      e.map = m->map;
      e.carried_in = carried[2 * i + carried_cur[i]]->p;
      e.carried_out = carried[2 * i + 1 - carried_cur[i]]->p;
      e.ev = EventBuf{m->events.p, static_cast<unsigned long long>(m->event_cap)};
      e.counters = m->counters.p;
      if (mlp) {
        e.lin = lbufs[2 * i + lcur[i]]->soa(m->n);
        e.lout = lbufs[2 * i + 1 - lcur[i]]->soa(m->n);
      }
      host_pin.p[i] = e;
    }
    t0_pin.p[0] = t0;
  }

  // The split engine's descriptors, window-major: window w reads what w - 1 wrote (the call's input state for the
  // first window), and writes a scratch state (the call's output state for the last one).
  void describe_split(int32_t windows) {
    const size_t ns = models.size();
    if (split_state.size() < 2 * ns) {
      split_state.clear();
      split_carried.clear();
      for (size_t i = 0; i < 2 * ns; ++i) {
        split_state.push_back(std::make_unique<StateBufs>());
        split_carried.push_back(std::make_unique<DevBuf<float>>());
      }
    }
    unsigned int pixels = 0;
    for (Model* m : models) pixels += m->n;
    if (rest_capacity < pixels) {
      rest.ensure(static_cast<size_t>(pixels) * rest_record_bytes());
      rest_capacity = pixels;
    }
    const size_t nw = static_cast<size_t>(std::max(windows, 1));
    split_desc_pin.ensure(nw * ns);
    split_desc.ensure(nw * ns);
    split_counts.ensure(2 * nw);
    for (size_t i = 0; i < ns; ++i) {
      Model* m = models[i];
      const StateSoA tmp[2] = {split_state[2 * i]->soa(m->n, m->mode()), split_state[2 * i + 1]->soa(m->n, m->mode())};
      float* tmp_c[2] = {split_carried[2 * i]->ensure(m->n), split_carried[2 * i + 1]->ensure(m->n)};
      for (size_t w = 0; w < nw; ++w) {
        EngineSensor e = host_pin.p[i];
        if (w > 0) {
          e.in = tmp[(w - 1) % 2];
          e.carried_in = tmp_c[(w - 1) % 2];
        }
        if (w + 1 < nw) {
          e.out = tmp[w % 2];
          e.carried_out = tmp_c[w % 2];
        }
        split_desc_pin.p[w * ns + i] = e;
      }
    }
  }

  // One step's device work, in stream order (what the CUDA graph holds): counters cleared, descriptors and the
  // model time uploaded from pinned memory, the persistent kernel between two timing events, counters read back.
  void enqueue(int32_t windows, int blocks, cudaStream_t st, bool capturing) {
    const unsigned rec_flags = capturing ? cudaEventRecordExternal : cudaEventRecordDefault;
    for (Model* m : models) CK(cudaMemsetAsync(m->counters.p, 0, kCntWords * sizeof(unsigned long long), st));
    if (rec_cap) CK(cudaMemsetAsync(rec_count.p, 0, 2 * sizeof(unsigned long long), st));
    CK(cudaMemcpyAsync(sensors_dev.p, host_pin.p, host.size() * sizeof(EngineSensor), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(t0_dev.p, t0_pin.p, sizeof(int64_t), cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(tile_counter.p, 0, sizeof(unsigned int), st));
    // Inside a captured graph, external records become event-record nodes (the timing of every replay).
    CK(cudaEventRecordWithFlags(timer.a, st, rec_flags));
    if (windows > 0 && total_tiles > 0) {
      if (mlp) {
        int sh = 0;
        while ((2u << sh) < rules.min_split) ++sh;
        const LearnedLaunch l{mlp->ops.p, mlp->params.p, margin, sh,
                              RecBuf{rec[0].p, rec_count.p, rec_cap}, RecBuf{rec[1].p, rec_count.p + 1, rec_cap}};
        launch_learned_engine(sensors_dev.p, static_cast<int>(host.size()), total_tiles, t0_dev.p, 0, windows,
                              rules, l, tile_counter.p, blocks, block_warps(), tile_lw, st);
      } else if (stage == kStageSplit) {
        const size_t ns = host.size();
        CK(cudaMemcpyAsync(split_desc.p, split_desc_pin.p, static_cast<size_t>(windows) * ns * sizeof(EngineSensor),
                           cudaMemcpyHostToDevice, st));
        CK(cudaMemsetAsync(split_counts.p, 0, 2 * static_cast<size_t>(windows) * sizeof(unsigned int), st));
        const int rest_blocks = sm_count() * std::max(1, engine_rest_blocks_per_sm());
        for (int32_t w = 0; w < windows; ++w) {
          launch_engine_split(split_desc.p + static_cast<size_t>(w) * ns, static_cast<int>(ns), total_tiles, t0_dev.p,
                              w, rules, split_counts.p + 2 * w, rest.p, split_counts.p + 2 * w + 1, rest_capacity,
                              blocks, warps_per_block, tile_lw, rest_blocks, st);
        }
      } else {
        launch_engine(sensors_dev.p, static_cast<int>(host.size()), total_tiles, t0_dev.p, 0, windows, rules,
                      tile_counter.p, blocks, warps_per_block, stage, tile_lw, cascade(), st);
      }
    }
    CK(cudaGetLastError());
    CK(cudaEventRecordWithFlags(timer.b, st, rec_flags));
    for (Model* m : models) {
      CK(cudaMemcpyAsync(m->counters_h.p, m->counters.p, kCntWords * sizeof(unsigned long long),
                         cudaMemcpyDeviceToHost, st));
    }
    if (rec_cap) CK(cudaMemcpyAsync(rec_n_pin.p, rec_count.p, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
  }

  void release_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
  }

  // Runs the step once (re-running it with larger event buffers while they overflow); with commit the models move
  // to the step's end, without it (a trial) they keep their state.
  void step(int32_t windows, cudaStream_t s, bool commit, uint64_t* samples_out, uint64_t* events_out) {
    if (windows < 0) throw std::invalid_argument("engine: windows must be >= 0");
    const int64_t t0 = models[0]->t_state;
    for (Model* m : models) {
      if (!m->initialized) throw std::logic_error("engine: call start() first");
      if (m->t_state != t0) throw std::logic_error("engine: the sensors' model times differ");
      if ((t0 & (kWindowNs - 1)) != 0) throw std::invalid_argument("engine: the model time must be a window start");
    }
    if (mlp && lcur.size() != models.size()) throw std::logic_error("engine: call start() after set_proposal()");
    const int blocks = grid_blocks();
    t0_pin.ensure(1);
    rec_n_pin.ensure(2);
    for (;;) {
      describe(t0);
      if (stage == kStageSplit) describe_split(windows);
      if (use_graph && rec_cap == 0) {
        const uint64_t key[8] = {static_cast<uint64_t>(windows), static_cast<uint64_t>(blocks),
                                 static_cast<uint64_t>(block_warps()), static_cast<uint64_t>(stage),
                                 static_cast<uint64_t>(tile_lw), reinterpret_cast<uint64_t>(mlp),
                                 (static_cast<uint64_t>(f2u(margin)) << 32) | total_tiles, 1};
        if (!exec || std::memcmp(key, graph_key, sizeof(key)) != 0) {
          release_graph();
          CK(cudaStreamBeginCapture(own, cudaStreamCaptureModeThreadLocal));
          try {
            enqueue(windows, blocks, own, true);
          } catch (...) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(own, &g);
            if (g) cudaGraphDestroy(g);
            throw;
          }
          CK(cudaStreamEndCapture(own, &graph));
          CK(cudaGraphInstantiate(&exec, graph, 0));
          std::memcpy(graph_key, key, sizeof(key));
        }
        CK(cudaEventRecord(order, s));
        CK(cudaStreamWaitEvent(own, order, 0));
        CK(cudaGraphLaunch(exec, own));
        CK(cudaEventRecord(order, own));
        CK(cudaStreamWaitEvent(s, order, 0));
        CK(cudaStreamSynchronize(own));
      } else {
        enqueue(windows, blocks, s, false);
        CK(cudaStreamSynchronize(s));
      }
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, timer.a, timer.b));
      last_ms = ms;
      bool rerun = false;
      for (Model* m : models) {
        const unsigned long long ev = m->counters_h.p[kCntEvents];
        if (ev > m->event_cap) {
          m->ensure_events(static_cast<size_t>(ev + ev / 4 + 1024));
          ++m->stat_reruns;
          rerun = true;
        }
      }
      if (rerun) continue;
      for (Model* m : models) {
        const unsigned long long e = m->counters_h.p[kCntErrors];
        if (e != 0) throw std::runtime_error(std::string("engine: ") + Model::error_text(e));
      }
      if (rec_cap) {
        rec_n[0] = rec_n_pin.p[0];
        rec_n[1] = rec_n_pin.p[1];
      }
      uint64_t samples = 0, events = 0;
      for (size_t i = 0; i < models.size(); ++i) {
        const unsigned long long* c = models[i]->counters_h.p;
        samples += c[kCntSamples];
        events += c[kCntEvents];
      }
      if (samples_out) *samples_out = samples;
      if (events_out) *events_out = events;
      if (!commit) return;
      for (size_t i = 0; i < models.size(); ++i) {
        Model* m = models[i];
        const unsigned long long* c = m->counters_h.p;
        m->stat_pieces += c[kCntPieces];
        m->stat_leaves += c[kCntLeaves];
        m->stat_samples += c[kCntSamples];
        m->stat_noise += c[kCntNoise];
        ++m->stat_launches;
        m->launch_ms_total += ms;
        m->launch_ms_max = std::max(m->launch_ms_max, static_cast<double>(ms));
        m->last_events = static_cast<size_t>(c[kCntEvents]);
        m->kept.clear();
        m->cur = 1 - m->cur;
        m->t_state = t0 + static_cast<int64_t>(windows) * kWindowNs;
        m->fresh = false;
        carried_cur[i] = 1 - carried_cur[i];
        if (mlp) lcur[i] = 1 - lcur[i];
      }
      return;
    }
  }

  void run(int32_t windows, cudaStream_t s, uint64_t* samples_out, uint64_t* events_out) {
    step(windows, s, true, samples_out, events_out);
  }

  // Every sensor's events as bs_model_take_events gives them, into outs[i] for sensor i: the sensors' device parts
  // (sort, column split, copy out) are queued on their own streams first, then each sensor's host copies run as soon
  // as its copy out has completed, while the device works on the sensors after it.
  void take_events(bs_event_columns* outs) {
    std::vector<char> queued(models.size(), 0);
    for (size_t i = 0; i < models.size(); ++i) {
      Model* m = models[i];
      if (m->kept.empty() && m->last_events > 0) {
        queued[i] = m->download_enqueue(m->events.p, m->last_events, &outs[i], m->own) ? 1 : 0;
      }
    }
    for (size_t i = 0; i < models.size(); ++i) {
      Model* m = models[i];
      if (queued[i]) {
        CK(cudaEventSynchronize(m->take_timer_copy.b));
        m->download_finish();
      } else if (!m->kept.empty()) {
        m->columns(m->kept, &outs[i]);
      }
      m->kept.clear();
      m->last_events = 0;
    }
  }

  void set_launch(int32_t warps, int32_t per_sm, int32_t stg, int32_t lw) {
    if (warps < 0 || warps > 4) throw std::invalid_argument("engine: warps per block must lie in [1, 4]");
    if (per_sm < 0 || per_sm > 32) throw std::invalid_argument("engine: blocks_per_sm in [0, 32]");
    if (stg != 0 && stg != kStageSplit && stg != 16 && stg != 32 && stg != 64) {
      throw std::invalid_argument(
          "engine: stage 0, 1 (the split engine), 16, 32 or 64 (32 deep with the warp-cooperative search)");
    }
    if (stg == kStageSplit && (cascade() != 0 || mlp)) {
      throw std::invalid_argument("engine: the split engine (stage 1) is the instantaneous response's");
    }
    if (stg == 64 && (cascade() != 0 || mlp)) {
      throw std::invalid_argument("engine: the warp-cooperative search (stage 64) is the instantaneous response's");
    }
    if (stg != 0 && cascade() == 1) throw std::invalid_argument("engine: the cascade runs unstaged (stage 0)");
    if (stg != 0 && stg != 32 && cascade() == 2) {
      throw std::invalid_argument("engine: the noise lattice runs unstaged (stage 0) or staged 32 deep (stage 32)");
    }
    if (lw != 0 && (lw < 2 || lw > 5)) throw std::invalid_argument("engine: tile width 4, 8, 16 or 32");
    warps_per_block = warps ? warps : 4;
    blocks_per_sm = per_sm;
    stage = stg;
    tile_lw = lw ? lw : 3;
    retile();
  }

  // Times each candidate launch shape on trial steps of `windows` windows from the current state (the models keep
  // their state) and keeps the fastest. Candidates: tile width 4, 8, 16 px (height 8, 4, 2) x warps per block 2, 4 x
  // staging depth 0, 16, 64 (32 deep with the warp-cooperative search; the learned engine: tile widths only; the
  // cascade: stage 0; the lattice: 0 or 32). Returns the candidates tried (ms of the second of
  // two trial steps each); rows are {tile_lw, warps, stage, ms}.
  std::vector<std::array<double, 4>> autotune(int32_t windows, cudaStream_t s) {
    if (windows < 1) throw std::invalid_argument("engine.autotune: windows >= 1");
    std::vector<std::array<double, 4>> rows;
    const int keep[4] = {tile_lw, warps_per_block, stage, blocks_per_sm};
    double best = 1e300;
    int bl = keep[0], bw = keep[1], bs = keep[2];
    for (int lw : {2, 3, 4}) {
      for (int w : {2, 4}) {
        for (int st : {0, kStageSplit, 16, 64}) {
          if ((mlp && (w != 4 || st != 0)) || (cascade() == 1 && st != 0)) continue;
          if (cascade() == 2 && (st == 64 || st == kStageSplit)) continue;
          if (cascade() == 2 && st != 0) st = 32;
          set_launch(w, 0, st, lw);
          step(windows, s, false, nullptr, nullptr);
          step(windows, s, false, nullptr, nullptr);
          rows.push_back({static_cast<double>(lw), static_cast<double>(w), static_cast<double>(st), last_ms});
          if (last_ms < best) {
            best = last_ms;
            bl = lw;
            bw = w;
            bs = st;
          }
        }
      }
    }
    set_launch(bw, keep[3], bs, bl);
    return rows;
  }
};

}  // namespace bs

// ---------------------------------------------------------------------------------------------
// extern "C"
// ---------------------------------------------------------------------------------------------
using bs::g_error;

template <class F>
static bs_status guarded(F&& f) {
  try {
    f();
    return BS_OK;
  } catch (const std::invalid_argument& e) {
    g_error = e.what();
    return BS_EINVAL;
  } catch (const bs::BudgetError& e) {
    g_error = e.what();
    return BS_ENOMEM;
  } catch (const bs::CudaError& e) {
    g_error = e.what();
    return BS_ECUDA;
  } catch (const std::logic_error& e) {
    g_error = e.what();
    return BS_ELOGIC;
  } catch (const std::bad_alloc&) {
    g_error = "out of host memory";
    return BS_ENOMEM;
  } catch (const std::exception& e) {
    g_error = e.what();
    return BS_ECUDA;
  }
}

namespace bs {
// For entry points in other translation units: the message bs_last_error() returns on this thread.
void set_last_error(const char* msg) { g_error = msg; }
}  // namespace bs

#define NEED(p)                                                      \
  do {                                                               \
    if (!(p)) throw std::invalid_argument("null argument: " #p);     \
  } while (0)

struct bs_model : bs::Model {
  using bs::Model::Model;
};
struct bs_sampler : bs::Sampler {
  using bs::Sampler::Sampler;
};
struct bs_engine : bs::Engine {
  using bs::Engine::Engine;
};
struct bs_mlp : bs::Mlp {
  using bs::Mlp::Mlp;
};

extern "C" {

const char* bs_last_error(void) { return g_error.c_str(); }
const char* bs_version(void) { return "ballasim_b200 0.1 (sm_100a)"; }
int32_t bs_cuda_available(void) { return bs::device_ok() ? 1 : 0; }

bs_status bs_model_create(const bs_params* params, uint32_t width, uint32_t height, uint64_t seed, uint32_t camera,
                          int32_t groups, bs_model** out) {
  return guarded([&] {
    NEED(params);
    NEED(out);
    *out = nullptr;
    *out = new bs_model(*params, width, height, seed, camera, groups);
  });
}
bs_status bs_model_destroy(bs_model* m) {
  return guarded([&] { delete m; });
}
bs_status bs_model_init(bs_model* m, int64_t t0_ns, const float* irr0) {
  return guarded([&] {
    NEED(m);
    m->init_host(t0_ns, irr0);
  });
}
bs_status bs_model_init_device(bs_model* m, int64_t t0_ns, const float* irr0_dev, void* stream) {
  return guarded([&] {
    NEED(m);
    NEED(irr0_dev);
    m->init_device(t0_ns, irr0_dev, m->stream_of(stream), nullptr);
  });
}
bs_status bs_model_advance_runs(bs_model* m, const uint32_t* pixel_ids, size_t n, const int64_t* t, const float* irr,
                                size_t n_samples, const int64_t* row_start, const int32_t* row_count,
                                int64_t t_end_ns, size_t* n_events) {
  return guarded([&] {
    NEED(m);
    m->advance_host(pixel_ids, n, t, irr, n_samples, row_start, row_count, t_end_ns);
    if (n_events) *n_events = m->kept.size();
  });
}
bs_status bs_model_advance_device(bs_model* m, const bs_device_runs* runs, int64_t t_end_ns, void* stream,
                                  bs_device_events* out) {
  return guarded([&] {
    NEED(m);
    NEED(runs);
    m->advance_device(*runs, t_end_ns, m->stream_of(stream));
    m->kept.clear();
    if (out) {
      out->data = m->events.p;
      out->count = m->last_events;
    }
  });
}
bs_status bs_model_download_events(bs_model* m, const bs_device_events* ev, bs_event_columns* out) {
  return guarded([&] {
    NEED(m);
    NEED(ev);
    NEED(out);
    m->download_columns(static_cast<const bs::RawEvent*>(ev->data), ev->count, out, m->own);
  });
}
bs_status bs_model_take_timing(const bs_model* m, double out[4]) {
  return guarded([&] {
    NEED(m);
    NEED(out);
    for (int i = 0; i < 4; ++i) out[i] = m->take_ms[i];
  });
}
bs_status bs_model_event_count(const bs_model* m, size_t* n) {
  return guarded([&] {
    NEED(m);
    NEED(n);
    *n = m->kept.empty() ? m->last_events : m->kept.size();
  });
}
bs_status bs_model_take_events(bs_model* m, bs_event_columns* out) {
  return guarded([&] {
    NEED(m);
    NEED(out);
    if (m->kept.empty() && m->last_events > 0) {
      m->download_columns(m->events.p, m->last_events, out, m->own);
    } else {
      m->columns(m->kept, out);
    }
    m->kept.clear();
    m->last_events = 0;
  });
}
bs_status bs_model_output_prepare(bs_model* m, size_t* n_ready) {
  return guarded([&] {
    NEED(m);
    NEED(n_ready);
    if (!m->initialized) throw std::logic_error("output: call init() first");
    *n_ready = m->output_prepare();
  });
}
bs_status bs_model_output_take(bs_model* m, bs_output_columns* out) {
  return guarded([&] {
    NEED(m);
    NEED(out);
    m->output_take(out);
  });
}
bs_status bs_model_output_held(const bs_model* m, size_t* n_held) {
  return guarded([&] {
    NEED(m);
    NEED(n_held);
    *n_held = m->n_held;
  });
}
bs_status bs_model_maps(const bs_model* m, double* on, double* off, double* leak, double* dark, double* phi0) {
  return guarded([&] {
    NEED(m);
    const size_t n = m->n;
    if (on) std::copy_n(m->maps.theta_on.data(), n, on);
    if (off) std::copy_n(m->maps.theta_off.data(), n, off);
    if (leak) std::copy_n(m->maps.leak.data(), n, leak);
    if (dark) std::copy_n(m->maps.dark.data(), n, dark);
    if (phi0) std::copy_n(m->maps.phi0.data(), n, phi0);
  });
}
bs_status bs_model_set_photometry(bs_model* m, double illuminance_scale, const float* gain, size_t n_gain) {
  return guarded([&] {
    NEED(m);
    if (!gain && n_gain != 0) throw std::invalid_argument("SensorModel.set_photometry: gain is NULL");
    m->set_photometry(illuminance_scale, gain, n_gain);
  });
}
bs_status bs_model_gain_map(const bs_model* m, float* out) {
  return guarded([&] {
    NEED(m);
    NEED(out);
    if (m->gain.empty()) {
      std::fill_n(out, m->n, 1.0f);
    } else {
      std::copy_n(m->gain.data(), m->n, out);
    }
  });
}
bs_status bs_model_noise_maps(const bs_model* m, double* ba_rate_hz, double* shot_max_hz) {
  return guarded([&] {
    NEED(m);
    const size_t n = m->n;
    if (ba_rate_hz) std::copy_n(m->maps.ba_rate.data(), n, ba_rate_hz);
    if (shot_max_hz) bs::CK(cudaMemcpy(shot_max_hz, m->map.shot_max, n * sizeof(double), cudaMemcpyDeviceToHost));
  });
}
bs_status bs_model_stats(const bs_model* m, uint64_t out[9]) {
  return guarded([&] {
    NEED(m);
    NEED(out);
    out[0] = m->stat_pieces;
    out[1] = m->stat_leaves;
    out[2] = m->stat_clamps;
    out[3] = m->stat_samples;
    out[4] = m->stat_noise;
    out[5] = m->stat_launches;
    out[6] = m->stat_reruns;
    out[7] = static_cast<uint64_t>(m->launch_ms_total * 1000.0);
    out[8] = static_cast<uint64_t>(m->launch_ms_max * 1000.0);
  });
}
bs_status bs_model_reset_stats(bs_model* m) {
  return guarded([&] {
    NEED(m);
    m->stat_pieces = m->stat_leaves = m->stat_clamps = m->stat_samples = m->stat_noise = 0;
    m->stat_launches = m->stat_reruns = 0;
    m->launch_ms_total = m->launch_ms_max = 0;
  });
}
bs_status bs_model_info(const bs_model* m, int64_t* time_ns, float* irr_max, int32_t* initialized) {
  return guarded([&] {
    NEED(m);
    if (time_ns) *time_ns = m->t_state;
    if (irr_max) *irr_max = m->k.irr_max;
    if (initialized) *initialized = m->initialized ? 1 : 0;
  });
}
bs_status bs_model_state_bytes(const bs_model* m, size_t* n) {
  return guarded([&] {
    NEED(m);
    NEED(n);
    *n = m->state_bytes();
  });
}
bs_status bs_model_save_state(const bs_model* m, uint8_t* out, size_t n) {
  return guarded([&] {
    NEED(m);
    NEED(out);
    m->save(out, n);
  });
}
bs_status bs_model_load_state(bs_model* m, const uint8_t* data, size_t n) {
  return guarded([&] {
    NEED(m);
    NEED(data);
    m->load(data, n);
  });
}
bs_status bs_model_set_long_run(bs_model* m, int32_t samples) {
  return guarded([&] {
    NEED(m);
    if (samples < -1) throw std::invalid_argument("long run: -1 (none), 0 (the default) or a sample count");
    m->long_row = samples == 0 ? 32 : (samples < 0 ? std::numeric_limits<int32_t>::max() : samples);
  });
}
bs_status bs_model_set_block(bs_model* m, int32_t threads) {
  return guarded([&] {
    NEED(m);
    if (threads != 0 && threads != 1 && (threads < 32 || threads > 128 || threads % 32 != 0)) {
      throw std::invalid_argument("threads per block must be 32, 64, 96 or 128 (0, 1: the row-major kernel)");
    }
    m->block = threads;
  });
}

bs_status bs_sampler_create(const bs_field* field, bs_sampler** out) {
  return guarded([&] {
    NEED(field);
    NEED(out);
    *out = nullptr;
    *out = new bs_sampler(*field);
  });
}
bs_status bs_sampler_destroy(bs_sampler* s) {
  return guarded([&] { delete s; });
}
bs_status bs_sample_window(bs_sampler* s, int64_t t_w, const uint32_t* pixel_ids, const uint8_t* levels, size_t n,
                           float* carried_irr, uint64_t* carried_sig, const bs_sample_rules* rules,
                           size_t* n_samples) {
  return guarded([&] {
    NEED(s);
    NEED(rules);
    if (n) {
      NEED(pixel_ids);
      NEED(levels);
      NEED(carried_irr);
      NEED(carried_sig);
    }
    s->window(t_w, pixel_ids, levels, n, carried_irr, carried_sig, *rules);
    if (n_samples) *n_samples = s->samples;
  });
}
bs_status bs_sample_window_device(bs_sampler* s, int64_t t_w, const uint32_t* pixel_ids, const uint8_t* levels,
                                  size_t n, const float* carried_irr, const uint64_t* carried_sig,
                                  float* carried_irr_out, uint64_t* carried_sig_out, const bs_sample_rules* rules,
                                  void* stream, size_t* n_samples) {
  return guarded([&] {
    NEED(s);
    NEED(rules);
    if (n) {
      NEED(pixel_ids);
      NEED(levels);
      NEED(carried_irr);
      NEED(carried_sig);
      NEED(carried_irr_out);
      NEED(carried_sig_out);
    }
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : s->own;
    s->window_device(t_w, pixel_ids, levels, n, carried_irr, carried_sig, carried_irr_out, carried_sig_out, *rules,
                     st);
    if (n_samples) *n_samples = s->samples;
  });
}
bs_status bs_field_levels_device(bs_sampler* s, int64_t t_w, int32_t l_min, int32_t l_max, uint8_t* out,
                                 void* stream) {
  return guarded([&] {
    NEED(s);
    NEED(out);
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : s->own;
    bs::launch_levels(s->field.f, t_w, l_min, l_max, s->field.f.width * s->field.f.height, out, st);
    bs::CK(cudaGetLastError());
  });
}
bs_status bs_field_frame_device(bs_sampler* s, int64_t t_ns, float* out, void* stream) {
  return guarded([&] {
    NEED(s);
    NEED(out);
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : s->own;
    bs::launch_field_frame(s->field.f, t_ns, s->field.f.width * s->field.f.height, out, st);
    bs::CK(cudaGetLastError());
  });
}
bs_status bs_sampler_download(bs_sampler* s, int64_t* offsets, int64_t* t_ns, float* irr) {
  return guarded([&] {
    NEED(s);
    if (offsets) bs::CK(cudaMemcpy(offsets, s->offsets.p, (s->n + 1) * 8, cudaMemcpyDeviceToHost));
    if (t_ns && s->samples) bs::CK(cudaMemcpy(t_ns, s->t.p, s->samples * 8, cudaMemcpyDeviceToHost));
    if (irr && s->samples) bs::CK(cudaMemcpy(irr, s->irr.p, s->samples * 4, cudaMemcpyDeviceToHost));
  });
}
bs_status bs_sampler_device_runs(bs_sampler* s, bs_device_runs* out) {
  return guarded([&] {
    NEED(s);
    NEED(out);
    out->pixel = s->dev_ids ? s->dev_ids : s->pixel.p;
    out->row_start = s->offsets.p;
    out->row_count = reinterpret_cast<const int32_t*>(s->counts.p);
    out->n = s->n;
    out->t = s->t.p;
    out->irr = s->irr.p;
    out->n_samples = s->samples;
  });
}
bs_status bs_field_levels(bs_sampler* s, int64_t t_w, int32_t l_min, int32_t l_max, uint8_t* out) {
  return guarded([&] {
    NEED(s);
    NEED(out);
    const uint32_t n = s->field.f.width * s->field.f.height;
    bs::DevBuf<uint8_t> lv;
    lv.ensure(n);
    bs::launch_levels(s->field.f, t_w, l_min, l_max, n, lv.p, s->own);
    bs::CK(cudaGetLastError());
    bs::CK(cudaMemcpyAsync(out, lv.p, n, cudaMemcpyDeviceToHost, s->own));
    bs::CK(cudaStreamSynchronize(s->own));
  });
}
bs_status bs_field_frame(bs_sampler* s, int64_t t_ns, float* out) {
  return guarded([&] {
    NEED(s);
    NEED(out);
    const uint32_t n = s->field.f.width * s->field.f.height;
    bs::DevBuf<float> fr;
    fr.ensure(n);
    bs::launch_field_frame(s->field.f, t_ns, n, fr.p, s->own);
    bs::CK(cudaGetLastError());
    bs::CK(cudaMemcpyAsync(out, fr.p, n * 4, cudaMemcpyDeviceToHost, s->own));
    bs::CK(cudaStreamSynchronize(s->own));
  });
}
bs_status bs_midpoint_eta(float tol, float dark, int32_t groups, const float* m_min, const float* m_max,
                          const float* ea, const float* em, const float* eb, size_t n, float* eta, uint8_t* exceeds) {
  return guarded([&] {
    if (groups < 1 || groups > 8) throw std::invalid_argument("midpoint test: need 1 to 8 light groups");
    NEED(m_min);
    NEED(m_max);
    if (n == 0) return;
    NEED(ea);
    NEED(em);
    NEED(eb);
    NEED(eta);
    NEED(exceeds);
    bs::require_device();
    const size_t w = n * static_cast<size_t>(groups);
    bs::DevBuf<float> a, m, b, e;
    bs::DevBuf<uint8_t> x;
    a.ensure(w);
    m.ensure(w);
    b.ensure(w);
    e.ensure(n);
    x.ensure(n);
    bs::CK(cudaMemcpy(a.p, ea, w * 4, cudaMemcpyHostToDevice));
    bs::CK(cudaMemcpy(m.p, em, w * 4, cudaMemcpyHostToDevice));
    bs::CK(cudaMemcpy(b.p, eb, w * 4, cudaMemcpyHostToDevice));
    bs::launch_midpoint_eta(tol, dark, groups, m_min, m_max, a.p, m.p, b.p, static_cast<uint32_t>(n), e.p, x.p,
                            nullptr);
    bs::CK(cudaGetLastError());
    bs::CK(cudaMemcpy(eta, e.p, n * 4, cudaMemcpyDeviceToHost));
    bs::CK(cudaMemcpy(exceeds, x.p, n, cudaMemcpyDeviceToHost));
  });
}
bs_status bs_level_cap(const int64_t* levels, size_t n, int64_t budget, int32_t l_min, int32_t* cap) {
  return guarded([&] {
    NEED(cap);
    if (l_min < 0 || l_min > bs::kWindowLog2) throw std::invalid_argument("l_min must lie in [0, 23]");
    std::vector<int64_t> counts;
    for (size_t i = 0; i < n; ++i) {
      if (levels[i] < 0 || levels[i] > bs::kWindowLog2) {
        throw std::invalid_argument("level_cap: levels must lie in [0, 23]");
      }
      if (static_cast<size_t>(levels[i]) >= counts.size()) counts.resize(static_cast<size_t>(levels[i]) + 1, 0);
      ++counts[static_cast<size_t>(levels[i])];
    }
    while (!counts.empty() && counts.back() == 0) counts.pop_back();
    const auto total = [&](int64_t c) {
      int64_t sum = 0;
      for (size_t l = 0; l < counts.size(); ++l) sum += counts[l] * ((int64_t{1} << std::min<int64_t>(l, c)) + 1);
      return sum;
    };
    const int64_t top = static_cast<int64_t>(counts.size()) - 1;
    *cap = -1;
    if (counts.empty() || total(top) <= budget) return;
    for (int64_t c = top - 1; c >= l_min; --c) {
      if (total(c) <= budget) {
        *cap = static_cast<int32_t>(c);
        return;
      }
    }
    throw std::invalid_argument("accuracy.max_samples_per_window = " + std::to_string(budget) +
                                " cannot hold one window of " + std::to_string(n) + " active pixels at level " +
                                std::to_string(l_min) + " (" + std::to_string(total(l_min)) + " samples); raise it");
  });
}

bs_status bs_engine_create(bs_model* const* models, const bs_field* fields, int32_t n, const bs_sample_rules* rules,
                           bs_engine** out) {
  return guarded([&] {
    NEED(models);
    NEED(fields);
    NEED(rules);
    NEED(out);
    *out = nullptr;
    *out = new bs_engine(models, fields, n, *rules);
  });
}
bs_status bs_engine_destroy(bs_engine* e) {
  return guarded([&] { delete e; });
}
bs_status bs_engine_start(bs_engine* e, int64_t t0_ns, void* stream) {
  return guarded([&] {
    NEED(e);
    e->start(t0_ns, stream ? static_cast<cudaStream_t>(stream) : e->own);
  });
}
bs_status bs_engine_start_frames(bs_engine* e, int64_t t0_ns, const float* const* frames, void* stream) {
  return guarded([&] {
    NEED(e);
    NEED(frames);
    e->start(t0_ns, stream ? static_cast<cudaStream_t>(stream) : e->own, frames);
  });
}
bs_status bs_engine_run(bs_engine* e, int32_t windows, void* stream, uint64_t* pixel_samples, uint64_t* events) {
  return guarded([&] {
    NEED(e);
    e->run(windows, stream ? static_cast<cudaStream_t>(stream) : e->own, pixel_samples, events);
  });
}
bs_status bs_engine_take_events(bs_engine* e, bs_event_columns* out) {
  return guarded([&] {
    NEED(e);
    NEED(out);
    e->take_events(out);
  });
}
bs_status bs_engine_set_launch(bs_engine* e, int32_t warps_per_block, int32_t blocks_per_sm, int32_t stage,
                               int32_t tile_width) {
  return guarded([&] {
    NEED(e);
    int lw = 0;
    if (tile_width != 0) {
      while ((1 << lw) < tile_width) ++lw;
      if ((1 << lw) != tile_width) throw std::invalid_argument("tile width must be 4, 8, 16 or 32");
    }
    e->set_launch(warps_per_block, blocks_per_sm, stage, lw);
  });
}
bs_status bs_engine_get_launch(const bs_engine* e, int32_t out[4]) {
  return guarded([&] {
    NEED(e);
    NEED(out);
    out[0] = e->warps_per_block;
    out[1] = e->blocks_per_sm;
    out[2] = e->stage;
    out[3] = 1 << e->tile_lw;
  });
}
bs_status bs_engine_set_graph(bs_engine* e, int32_t on) {
  return guarded([&] {
    NEED(e);
    e->use_graph = on != 0;
    if (!e->use_graph) e->release_graph();
  });
}
bs_status bs_engine_autotune(bs_engine* e, int32_t windows, void* stream, double* rows, size_t cap, size_t* n) {
  return guarded([&] {
    NEED(e);
    NEED(n);
    const auto r = e->autotune(windows, static_cast<cudaStream_t>(stream));
    *n = r.size();
    for (size_t i = 0; i < r.size() && i < cap && rows; ++i) {
      rows[4 * i + 0] = static_cast<double>(1 << static_cast<int>(r[i][0]));
      rows[4 * i + 1] = r[i][1];
      rows[4 * i + 2] = r[i][2];
      rows[4 * i + 3] = r[i][3];
    }
  });
}
bs_status bs_engine_last_ms(const bs_engine* e, double* ms) {
  return guarded([&] {
    NEED(e);
    NEED(ms);
    *ms = e->last_ms;
  });
}

bs_status bs_mlp_create(uint64_t seed, bs_mlp** out) {
  return guarded([&] {
    NEED(out);
    *out = nullptr;
    *out = new bs_mlp(seed);
  });
}
bs_status bs_mlp_destroy(bs_mlp* m) {
  return guarded([&] { delete m; });
}
bs_status bs_mlp_get_params(const bs_mlp* m, float* params) {
  return guarded([&] {
    NEED(m);
    NEED(params);
    m->get(params);
  });
}
bs_status bs_mlp_set_params(bs_mlp* m, const float* params) {
  return guarded([&] {
    NEED(m);
    NEED(params);
    m->set(params);
  });
}
bs_status bs_mlp_steps(const bs_mlp* m, int64_t* steps) {
  return guarded([&] {
    NEED(m);
    NEED(steps);
    *steps = m->steps();
  });
}
bs_status bs_mlp_forward(bs_mlp* m, const uint16_t* x, size_t n, float* y, void* stream) {
  return guarded([&] {
    NEED(m);
    m->forward(x, n, y, stream ? static_cast<cudaStream_t>(stream) : m->own);
  });
}
bs_status bs_mlp_gradient(bs_mlp* m, const uint16_t* x, const float* y, size_t n, double* grad, double* loss,
                          void* stream) {
  return guarded([&] {
    NEED(m);
    NEED(grad);
    NEED(loss);
    m->gradient(x, y, n, grad, loss, stream ? static_cast<cudaStream_t>(stream) : m->own);
  });
}
bs_status bs_mlp_train(bs_mlp* m, const uint16_t* x, const float* y, size_t n, int32_t steps, int32_t batch, float lr,
                       float tau, uint64_t seed, float* losses, void* stream) {
  return guarded([&] {
    NEED(m);
    m->train(x, y, n, steps, batch, lr, tau, seed, losses, stream ? static_cast<cudaStream_t>(stream) : m->own);
  });
}
bs_status bs_trace_pairs(const bs_field* field, const bs_sample_rules* rules, int64_t t0_ns, int32_t windows,
                         uint32_t stride, float eps, uint64_t seed, uint16_t* x, float* y, uint64_t* keys, size_t cap,
                         size_t* n_out, size_t* total, void* stream) {
  return guarded([&] {
    NEED(field);
    NEED(rules);
    NEED(n_out);
    NEED(total);
    bs::require_device();
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    bs::trace_pairs(*field, *rules, t0_ns, windows, stride, eps, seed, x, y, keys, cap, n_out, total, s);
  });
}
bs_status bs_engine_set_proposal(bs_engine* e, const bs_mlp* mlp, float margin) {
  return guarded([&] {
    NEED(e);
    e->set_proposal(mlp, margin);
  });
}
bs_status bs_engine_set_record(bs_engine* e, size_t capacity) {
  return guarded([&] {
    NEED(e);
    e->set_record(capacity);
  });
}
bs_status bs_engine_take_record(bs_engine* e, int32_t which, size_t cap, int64_t* t, uint32_t* pixel, float* v,
                                size_t* n) {
  return guarded([&] {
    NEED(e);
    NEED(n);
    e->take_record(which, cap, t, pixel, v, n);
  });
}

}  // extern "C"
