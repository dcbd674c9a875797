// engine.cu -- the C ABI of include/optflow_cuda.h: engine state, device buffers, and the order of the
// kernels of one pair (coarse POC -> dense start -> fine stage -> confidence -> finish).
//
// Everything between the upload of the inputs and the download of the outputs runs on one CUDA stream
// with no host synchronisation: conditional steps of the reference (the energy-threshold reset, the
// trusted pre-warp's "any low / not all trusted" cases) are decided on the device from counters that the
// kernels read, so a whole pair can be captured and replayed as a CUDA graph.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>

#include "fft.cuh"
#include "synth_field.cuh"
#include "kernels.cuh"
#include "net.cuh"
#include "../../include/optflow_cuda_testing.h"
#include "../../include/optflow_cuda_synth.h"
#include "../../include/optflow_cuda_net.h"

namespace ofc {
thread_local uint64_t* g_launch_counter = nullptr;
thread_local Profiler* g_profiler = nullptr;

// Events around the launches of the kernels whose name contains `filter`; resolved into per-kernel totals
// when read (ofc_profile_read) or when the pool runs low.
struct Profiler {
  std::string filter;
  // while a pair is captured as a graph, the event pairs go to the graph's list (recorded at every replay)
  std::vector<std::tuple<std::string, cudaEvent_t, cudaEvent_t>>* capture = nullptr;
  struct Pending {
    std::string name;
    cudaEvent_t a, b;
  };
  std::vector<Pending> pending;
  std::vector<cudaEvent_t> pool;
  std::map<std::string, std::pair<uint64_t, double>> totals;
  std::mutex mu;
  cudaEvent_t take() {
    if (pool.empty()) {
      cudaEvent_t e;
      OFC_CUDA(cudaEventCreate(&e));
      return e;
    }
    cudaEvent_t e = pool.back();
    pool.pop_back();
    return e;
  }
  void resolve() {
    for (auto& p : pending) {
      OFC_CUDA(cudaEventSynchronize(p.b));
      float ms = 0;
      OFC_CUDA(cudaEventElapsedTime(&ms, p.a, p.b));
      auto& t = totals[p.name];
      t.first += 1;
      t.second += ms;
      pool.push_back(p.a);
      pool.push_back(p.b);
    }
    pending.clear();
  }
  ~Profiler() {
    for (auto& p : pending) { cudaEventDestroy(p.a); cudaEventDestroy(p.b); }
    for (auto e : pool) cudaEventDestroy(e);
  }
};

void raise_smem_limit(const void* fn, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, size_t> limit;
  int dev = 0;
  OFC_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  size_t& cur = limit[{fn, dev}];
  if (bytes <= cur) return;
  OFC_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  cur = bytes;
}

void prof_before(const char* name, cudaStream_t st, void** token) {
  Profiler* p = g_profiler;
  std::string n(name);
  if (!n.empty() && n.front() == '(') n = n.substr(1, n.size() - 2);
  if (!p->filter.empty() && n.find(p->filter) == std::string::npos) return;
  std::lock_guard<std::mutex> lk(p->mu);
  if (p->capture) {
    cudaEvent_t a, b;
    OFC_CUDA(cudaEventCreate(&a));
    OFC_CUDA(cudaEventCreate(&b));
    // External: a record node in the graph (a plain record inside a capture only orders streams)
    OFC_CUDA(cudaEventRecordWithFlags(a, st, cudaEventRecordExternal));
    p->capture->emplace_back(n, a, b);
    *token = (void*)(uintptr_t)(1 + 2 * (p->capture->size() - 1));  // odd: an index into the capture list
    return;
  }
  if (p->pending.size() > 4096) p->resolve();
  Profiler::Pending q{n, p->take(), p->take()};
  OFC_CUDA(cudaEventRecord(q.a, st));
  p->pending.push_back(q);
  *token = &p->pending.back();
}

void prof_after(void* token, cudaStream_t st) {
  uintptr_t t = (uintptr_t)token;
  if (t & 1) {
    OFC_CUDA(cudaEventRecordWithFlags(std::get<2>((*g_profiler->capture)[(t - 1) / 2]), st, cudaEventRecordExternal));
    return;
  }
  OFC_CUDA(cudaEventRecord(((Profiler::Pending*)token)->b, st));
}
}

using namespace ofc;

namespace {

// ---------------------------------------------------------------- config helpers (config.py:247-272)
double smax_of(const ofc_config& c) {
  double m = 0;
  for (int i = 0; i < c.n_scales; i++) m = std::max(m, c.scales[i]);
  return m;
}
double auto_guard(const ofc_config& c) { return 3.0 * c.lam * smax_of(c) / (2 * PI * c.bandwidth); }
double guard_px(const ofc_config& c) { return c.edge_guard >= 0 ? c.edge_guard : auto_guard(c); }
double min_area_px(const ofc_config& c) {
  if (c.edge_guard_min_area >= 0) return c.edge_guard_min_area;
  double l = c.lam * smax_of(c);
  return 2.0 * l * l;
}

std::string validate(const ofc_config& c) {  // Config.validate, config.py:166-245 (pair-path keys)
  auto finite = [](double v) { return std::isfinite(v); };
  if (c.n_scales < 1) return "scales must not be empty";
  if (c.n_scales > OFC_MAX_SCALES) return "the CUDA engine holds at most 16 scales";
  if (c.poc_win < 16 || (c.poc_win & (c.poc_win - 1))) return "poc_win must be a power of two >= 16";
  if (c.grid_step < 1 || c.strain_win < 5 || c.strain_win % 2 == 0) return "grid_step >= 1 and strain_win odd >= 5 required";
  if (c.dc_cut <= 0) return "dc_cut must be positive";
  if (c.phase_tol <= 0) return "phase_tol must be positive";
  if (c.shape_order != 1 && c.shape_order != 2) return "shape_order must be 1 or 2";
  double smin = c.scales[0];
  for (int i = 0; i < c.n_scales; i++) smin = std::min(smin, c.scales[i]);
  if (c.lam * smin < 3 || c.sigma_w <= 0 || c.sigma_s <= 0)
    return "shortest wavelength lam*min(scales) must be >= 3 px; sigmas must be positive";
  const double* fl[] = {&c.max_disp, &c.poc_peak_min, &c.median_thresh, &c.lam, &c.bandwidth, &c.dc_cut, &c.sigma_w,
                        &c.sigma_s, &c.conf_min, &c.edge_guard, &c.edge_guard_min_area, &c.phase_tol};
  const char* nm[] = {"max_disp", "poc_peak_min", "median_thresh", "lam", "bandwidth", "dc_cut", "sigma_w",
                      "sigma_s", "conf_min", "edge_guard", "edge_guard_min_area", "phase_tol"};
  for (int i = 0; i < 12; i++)
    if (!finite(*fl[i])) return std::string(nm[i]) + " must be a finite number";
  for (int i = 0; i < c.n_scales; i++)
    if (!finite(c.scales[i])) return "scales must be finite numbers";
  if (c.bandwidth <= 0 || c.max_disp <= 0 || c.median_thresh <= 0) return "bandwidth, max_disp and median_thresh must be positive";
  if (c.n_orient < 1 || c.outer_iters < 1 || c.inner_iters < 1) return "n_orient, outer_iters and inner_iters must be >= 1";
  if (!(c.conf_min >= 0 && c.conf_min <= 1) || !(c.poc_peak_min >= 0 && c.poc_peak_min <= 1))
    return "conf_min and poc_peak_min must lie in [0, 1]";
  if (c.prewarp_freeze_at < 0) return "prewarp_freeze_at must be >= 0";
  if (c.n_orient * c.n_scales > 64 || c.sigma_w > 256 || c.sigma_s > 256 || c.strain_win > 255 || c.poc_win > 1024)
    return "at most 64 filters (n_orient * len(scales)); sigma_w, sigma_s <= 256, strain_win <= 255 and poc_win <= 1024 required";
  if (c.grid_step > 4096 || guard_px(c) > 256)
    return "grid_step <= 4096 and an edge guard (edge_guard, or the automatic one from lam, scales and bandwidth) <= 256 px required";
  return "";
}

// ---------------------------------------------------------------- POC geometry (poc.py:61-64,168-195)
int pow2_floor(long n) {
  if (n < 1) return 0;
  int b = 0;
  while ((n >> (b + 1)) > 0) b++;
  return 1 << b;
}
bool level_window(int h, int w, int win, int& wy, int& wx) {
  int lim_h = pow2_floor(2 * h / 3), lim_w = pow2_floor(2 * w / 3);
  if (win <= lim_h && win <= lim_w) { wy = wx = win; return true; }
  if (h <= w) {
    wy = std::min(win, lim_h);
    wx = std::min(lim_w, std::max(win, win * win / std::max(wy, 1)));
  } else {
    wx = std::min(win, lim_w);
    wy = std::min(lim_h, std::max(win, win * win / std::max(wx, 1)));
  }
  return std::min(wy, wx) >= 16;
}
int n_levels(double max_disp, int win, int h, int w) {
  int L = (int)std::max(0.0, std::ceil(std::log2(std::max(max_disp, 1e-9) / (win / 4.0))));
  int wy, wx;
  while (L > 0 && !level_window(h >> L, w >> L, win, wy, wx)) L--;
  return L;
}
std::vector<int> arange(int a, int b, int step) {
  std::vector<int> v;
  for (int i = a; i < b; i += step) v.push_back(i);
  return v;
}

std::vector<double> gauss_kernel(double sigma) {  // interp.py:79-83
  int r = (int)(4.0 * sigma + 0.5);
  std::vector<double> k(2 * r + 1);
  double s = 0;
  for (int i = -r; i <= r; i++) {
    double t = i / sigma;
    k[i + r] = std::exp(-0.5 * t * t);
  }
  for (double v : k) s += v;
  for (double& v : k) v /= s;
  return k;
}

// ---------------------------------------------------------------- device buffers
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};

// page-locked host memory (the staging buffers of streamed frames and results)
struct HostBuf {
  void* p = nullptr;
  size_t bytes = 0;
  ~HostBuf() {
    if (p) cudaFreeHost(p);
  }
};

// the learned coarse proposal of an engine (ofc_set_coarse_net): the network's parameters on the device, the
// per-tile fallback test, and its counters
struct Proposal {
  float* params = nullptr;  // float32 parameters (the biases are read from here)
  uint16_t* w16 = nullptr;  // their bfloat16 copy, the tensor-core GEMMs' weights
  int tile = 256;           // fallback tiles of tile x tile pixels
  double max_low = 0.25;    // a tile fails when more than this share of its judged pixels has conf < conf_min
  std::atomic<uint64_t> pairs{0}, tiles{0}, failed{0}, fallbacks{0};
  ~Proposal() {
    if (params) cudaFree(params);
    if (w16) cudaFree(w16);
  }
};

struct Lane {
  cudaStream_t stream = nullptr;
  std::shared_ptr<Proposal> proposal;  // null: the POC coarse stage
  std::mutex busy;
  std::unordered_map<std::string, std::unique_ptr<DevBuf>> pool;
  std::map<int, std::pair<FftPlan, std::unique_ptr<DevBuf>>> plans;
  cudaEvent_t ev[4] = {};
  // a second compute stream for work that overlaps the main one inside a pair (the reference pack beside the
  // coarse stage) and its fork / join events
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  cudaEvent_t masked = nullptr;  // the pair's masked field and valid mask are written (recorded inside its finish stage)
  // the copy stream of batched calls and its ordering events (created on first use)
  cudaStream_t copy = nullptr;
  cudaEvent_t bev[8] = {};
  cudaEvent_t sev[2] = {};  // timing events of a sequence frame's finish (the pair's ev[] time its legs)
  void ensure_copy_stream() {
    if (copy) return;
    OFC_CUDA(cudaStreamCreateWithFlags(&copy, cudaStreamNonBlocking));
    for (auto& e : bev) OFC_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    for (auto& e : sev) OFC_CUDA(cudaEventCreate(&e));
  }

  template <class T>
  T* get(const std::string& name, size_t count) {
    size_t bytes = std::max<size_t>(count * sizeof(T), 256);
    auto& b = pool[name];
    if (!b) b.reset(new DevBuf());
    if (b->bytes < bytes) {
      if (b->p) {
        // captured graphs hold the old address: drop them (after the work in flight) before the buffer goes
        OFC_CUDA(cudaStreamSynchronize(stream));
        graphs.clear();
        OFC_CUDA(cudaFree(b->p));
      }
      b->p = nullptr;
      b->bytes = 0;
      OFC_CUDA(cudaMalloc(&b->p, bytes));
      b->bytes = bytes;
    }
    return (T*)b->p;
  }
  std::unordered_map<std::string, std::unique_ptr<HostBuf>> hpool;
  template <class T>
  T* pinned(const std::string& name, size_t count) {
    size_t bytes = std::max<size_t>(count * sizeof(T), 256);
    auto& b = hpool[name];
    if (!b) b.reset(new HostBuf());
    if (b->bytes < bytes) {
      if (b->p) {
        OFC_CUDA(cudaStreamSynchronize(stream));
        if (copy) OFC_CUDA(cudaStreamSynchronize(copy));
        OFC_CUDA(cudaFreeHost(b->p));
      }
      b->p = nullptr;
      b->bytes = 0;
      OFC_CUDA(cudaHostAlloc(&b->p, bytes, cudaHostAllocDefault));
      b->bytes = bytes;
    }
    return (T*)b->p;
  }
  template <class T>
  T* upload(const std::string& name, const T* host, size_t count) {
    T* d = get<T>(name, count);
    OFC_CUDA(cudaMemcpyAsync(d, host, count * sizeof(T), cudaMemcpyHostToDevice, stream));
    return d;
  }
  // constant tables uploaded once per key (sizes and configuration in the key): the per-pair sequence then
  // issues no host-to-device copy, so it can be captured as a CUDA graph
  std::unordered_map<std::string, std::unique_ptr<DevBuf>> consts;
  template <class T>
  const T* cached(const std::string& key, const T* host, size_t count) {
    auto& b = consts[key];
    if (!b) {
      b.reset(new DevBuf());
      OFC_CUDA(cudaMalloc(&b->p, std::max<size_t>(count * sizeof(T), 256)));
      b->bytes = count * sizeof(T);
      OFC_CUDA(cudaMemcpy(b->p, host, count * sizeof(T), cudaMemcpyHostToDevice));
    }
    return (const T*)b->p;
  }
  bool has_const(const std::string& key) const { return consts.count(key) != 0; }

  // captured pair sequences, per (size, configuration, inputs present); events: the profile-mode event pairs
  // recorded inside the graph (kernel name, start, end)
  struct Graph {
    cudaGraphExec_t exec[4] = {nullptr, nullptr, nullptr, nullptr};
    uint64_t launches[4] = {0, 0, 0, 0};  // kernels per stage graph (the launch counter's share of a replay)
    bool eager = false;                // the capture failed: this key runs eagerly
    std::vector<std::tuple<std::string, cudaEvent_t, cudaEvent_t>> events;
    ~Graph() {
      for (auto g : exec)
        if (g) cudaGraphExecDestroy(g);
      for (auto& e : events) {
        cudaEventDestroy(std::get<1>(e));
        cudaEventDestroy(std::get<2>(e));
      }
    }
  };
  std::unordered_map<std::string, std::unique_ptr<Graph>> graphs;

  const FftPlan& plan(int L) {
    auto it = plans.find(L);
    if (it != plans.end()) return it->second.first;
    FftPlan pl = fft_make_plan(L);
    // twiddles of the stages' length, then (Bluestein) the chirp and the filter
    std::vector<float2> tw = fft_twiddles(fft_work_len(pl));
    const size_t ntw = tw.size();
    if (pl.M) {
      std::vector<float2> bt = fft_bluestein_tables(L, pl.M);
      tw.insert(tw.end(), bt.begin(), bt.end());
    }
    std::unique_ptr<DevBuf> b(new DevBuf());
    size_t b32 = tw.size() * sizeof(float2);
    OFC_CUDA(cudaMalloc(&b->p, b32));
    b->bytes = b32;
    OFC_CUDA(cudaMemcpy(b->p, tw.data(), b32, cudaMemcpyHostToDevice));
    pl.tw = (const float2*)b->p;
    if (pl.M) {
      pl.chirp = pl.tw + ntw;
      pl.filt = pl.chirp + L;
    }
    auto& slot = plans[L];
    slot.first = pl;
    slot.second = std::move(b);
    return slot.first;
  }
  // the worker lanes of a batched call (ofc_track_pairs), created on first use and owned by this lane
  std::vector<std::unique_ptr<Lane>> aux;
  void release() {
    for (auto& a : aux) a->release();
    graphs.clear();
    consts.clear();
    pool.clear();
    hpool.clear();
    plans.clear();
  }
};

// a lane's streams and events (ofc_create), and their end (ofc_destroy): work in flight is waited for first
void lane_init(Lane& l) {
  OFC_CUDA(cudaStreamCreateWithFlags(&l.stream, cudaStreamNonBlocking));
  OFC_CUDA(cudaStreamCreateWithFlags(&l.side, cudaStreamNonBlocking));
  OFC_CUDA(cudaEventCreateWithFlags(&l.fork, cudaEventDisableTiming));
  OFC_CUDA(cudaEventCreateWithFlags(&l.join, cudaEventDisableTiming));
  OFC_CUDA(cudaEventCreateWithFlags(&l.masked, cudaEventDisableTiming));
  for (auto& ev : l.ev) OFC_CUDA(cudaEventCreate(&ev));
}

void lane_sync(Lane& l) {
  for (auto& a : l.aux) lane_sync(*a);
  cudaStreamSynchronize(l.stream);
  cudaStreamSynchronize(l.side);
  if (l.copy) cudaStreamSynchronize(l.copy);
}

void lane_destroy(Lane& l) {
  for (auto& a : l.aux) lane_destroy(*a);
  l.aux.clear();
  cudaStreamSynchronize(l.stream);
  if (l.copy) cudaStreamSynchronize(l.copy);
  cudaStreamSynchronize(l.side);
  l.release();
  for (auto& ev : l.ev) cudaEventDestroy(ev);
  cudaEventDestroy(l.fork);
  cudaEventDestroy(l.join);
  cudaEventDestroy(l.masked);
  cudaStreamDestroy(l.side);
  if (l.copy) {
    for (auto& ev : l.bev) cudaEventDestroy(ev);
    for (auto& ev : l.sev) cudaEventDestroy(ev);
    cudaStreamDestroy(l.copy);
  }
  cudaStreamDestroy(l.stream);
}

// a key of the configuration fields the pair path reads
std::string cfg_key(const ofc_config& c) {
  char buf[512];
  int n = std::snprintf(buf, sizeof buf, "%d,%d,%.17g,%.17g,%.17g,%.17g,%d,%d,%.17g,%.17g,%.17g,%d,%.17g,%d,%d,%.17g,%.17g,%.17g,%.17g,%d,%d",
                        c.grid_step, c.poc_win, c.max_disp, c.poc_peak_min, c.median_thresh, c.lam, c.n_scales,
                        c.n_orient, c.bandwidth, c.dc_cut, c.sigma_w, c.shape_order, c.sigma_s, c.outer_iters,
                        c.inner_iters, c.conf_min, c.edge_guard, c.edge_guard_min_area, c.phase_tol, c.strain_win,
                        c.prewarp_freeze_at);
  std::string k(buf, n > 0 ? (size_t)n : 0);
  for (int i = 0; i < c.n_scales; i++) {
    std::snprintf(buf, sizeof buf, ",%.17g", c.scales[i]);
    k += buf;
  }
  return k;
}

}  // namespace

struct ofc_engine {
  int device = 0;
  int nlanes = 1;
  uint64_t launches = 0;
  std::vector<std::unique_ptr<Lane>> lanes;
  std::unique_ptr<ofc::Profiler> prof;
};

namespace {

void set_err(char* err, size_t len, const std::string& m) {
  if (err && len) {
    size_t n = std::min(len - 1, m.size());
    std::memcpy(err, m.data(), n);
    err[n] = 0;
  }
}

// Runs f on a free lane of the engine (GpuEngine refuses instead of blocking, engine.rs:660-676).
template <class F>
int guarded(ofc_engine* e, char* err, size_t errlen, F&& f) {
  if (!e) { set_err(err, errlen, "null engine"); return OFC_ERR_ARG; }
  Lane* lane = nullptr;
  std::unique_lock<std::mutex> lk;
  for (auto& l : e->lanes) {
    std::unique_lock<std::mutex> t(l->busy, std::try_to_lock);
    if (t.owns_lock()) { lk = std::move(t); lane = l.get(); break; }
  }
  if (!lane) {
    set_err(err, errlen, "the CUDA engine is busy: more concurrent calls than its " + std::to_string(e->nlanes) + " lane(s)");
    return OFC_ERR_BUSY;
  }
  g_launch_counter = &e->launches;
  g_profiler = e->prof.get();
  try {
    OFC_CUDA(cudaSetDevice(e->device));
    f(*lane);
    g_launch_counter = nullptr;
    g_profiler = nullptr;
    return OFC_OK;
  } catch (const Error& x) {
    g_launch_counter = nullptr;
    g_profiler = nullptr;
    set_err(err, errlen, x.what());
    return x.status;
  } catch (const std::exception& x) {
    g_launch_counter = nullptr;
    g_profiler = nullptr;
    set_err(err, errlen, x.what());
    return OFC_ERR_DEVICE;
  }
}

// ---------------------------------------------------------------- the fine stage on one window
struct FineOut {
  double* ux;  // W*H each (ux and uy contiguous: uy = ux + W*H)
  double* uy;
  double* energy;
  double* resid;
  EnergyStats* stats;  // median of the final energy
};

// the Gabor tables of a padded size on the device (float64 and float32 copies)
GaborTables upload_gabor(Lane& L, int ph, int pw, const ofc_config& c) {
  const std::string key = "gabor:" + std::to_string(ph) + "x" + std::to_string(pw) + ":" + cfg_key(c);
  const double* d64;
  const float* d32;
  if (L.has_const(key)) {
    d64 = L.cached<double>(key, nullptr, 0);
    d32 = L.cached<float>(key + ":f32", nullptr, 0);
  } else {
    std::vector<double> gt = gabor_tables_host(ph, pw, c);
    std::vector<float> g32(gt.begin(), gt.end());
    d64 = L.cached(key, gt.data(), gt.size());
    d32 = L.cached(key + ":f32", g32.data(), g32.size());
  }
  GaborTables g;
  gabor_bind(g, d64, d32, ph, pw, c.n_scales * c.n_orient);
  return g;
}

// window taps: Gaussian (sigma) and, for the moments, k(t) t^p for p = 0..4
const double* gauss_taps(Lane& L, double sigma, int& r) {
  std::vector<double> k = gauss_kernel(sigma);
  r = (int)k.size() / 2;
  char key[64];
  std::snprintf(key, sizeof key, "gauss:%.17g", sigma);
  return L.cached(key, k.data(), k.size());
}
// the window taps k(t) t^p, p = 0..4, on the device (5 x (2r + 1)) and, for the default radius, as the kernel
// parameter tp (t = 0..r)
const double* moment_taps(Lane& L, double sigma, int& r, MomTaps& tp) {
  std::vector<double> kw = gauss_kernel(sigma);
  r = (int)kw.size() / 2;
  const int K = 2 * r + 1;
  std::vector<double> mt((size_t)5 * K);
  for (int p = 0; p < 5; p++)
    for (int t = -r; t <= r; t++) mt[(size_t)p * K + t + r] = kw[t + r] * std::pow((double)t, p);
  tp = MomTaps{};
  if (r == MOM_R)
    for (int p = 0; p < 5; p++)
      for (int t = 0; t <= r; t++) tp.k[p][t] = mt[(size_t)p * K + t + r];
  char key[64];
  std::snprintf(key, sizeof key, "moments:%.17g", sigma);
  return L.cached(key, mt.data(), mt.size());
}

// reference_phase (phaseflow.py:100-111) of i1: float32 transforms, as the reference's Rust port computes them
// (gabor.rs:230-270, rustfft f32), with (r.re, r.im, gx, gy) and amp formed per pixel in float64 and stored
// float32 per filter. Filters are processed in groups to bound the scratch (3 planes of ph x pw per filter).
void reference_pack(Lane& L, const float* i1, int W, int H, const GaborTables& g, float4* ref4, float* amp,
                    cudaStream_t st) {
  const int ph = H + 2 * PAD, pw = W + 2 * PAD;
  const size_t Np = (size_t)ph * pw;
  const int G = std::min(g.F, 4);
  const FftPlan& plw = L.plan(pw);
  const FftPlan& plh = L.plan(ph);
  float2* T32 = L.get<float2>("fft_T", Np);
  float2* U32 = L.get<float2>("ref_U32", Np * 3 * G);
  launch_fft_rows_fwd_real(i1, W, H, plw, ph, T32, st);
  launch_fft_cols_fwd(T32, plh, pw, st);
  for (int k0 = 0; k0 < g.F; k0 += G) {
    int k1 = std::min(g.F, k0 + G);
    launch_fft_cols_ref_f32(T32, plh, pw, g, k0, k1, U32, st);
    launch_fft_rows_inv_ref_f32(U32, plw, ph, k0, k1, W, H, ref4, amp, st);
  }
}

// The parts of refine_dev that depend on the images only: the reference pack of i1 and the spline of i2, on
// stream st (the pair path runs them on the lane's side stream beside the coarse stage).
void fine_prep(Lane& L, const float* i1, int W, int H, const float* i2, int w2, int h2, const ofc_config& c,
               cudaStream_t st) {
  const size_t N = (size_t)W * H;
  const int ph = H + 2 * PAD, pw = W + 2 * PAD;
  const int F = c.n_scales * c.n_orient;
  GaborTables g = upload_gabor(L, ph, pw, c);
  float4* ref4 = L.get<float4>("ref4", N * F);
  float* amp = L.get<float>("ref_amp", N * F);
  reference_pack(L, i1, W, H, g, ref4, amp, st);
  float* c2 = L.get<float>("spline2", (size_t)w2 * h2);
  double* tmp2 = L.get<double>("spline2_tmp", (size_t)w2 * h2 * 2);
  launch_bspline_f32(i2, c2, tmp2, w2, h2, st);
}

// refine_raw (phaseflow.rs:1514-1613 / phaseflow.py:427-507) on the device. u2: 2 planes (ux | uy) holding
// the start and receiving the result. prepared: fine_prep already ran for these images (ordered before this call).
FineOut refine_dev(Lane& L, const float* i1, int W, int H, const float* i2, int w2, int h2, long shx, long shy,
                   double* u2, const ofc_config& c, bool prepared) {
  cudaStream_t st = L.stream;
  const size_t N = (size_t)W * H;
  const int ph = H + 2 * PAD, pw = W + 2 * PAD;
  const size_t Np = (size_t)ph * pw;
  const int F = c.n_scales * c.n_orient;
  const FftPlan& plw = L.plan(pw);
  const FftPlan& plh = L.plan(ph);
  GaborTables g = upload_gabor(L, ph, pw, c);
  // taps: smoothing Gaussian (sigma_s) and window moments k(t) t^p, p = 0..4 (sigma_w)
  int rs = 0, rw = 0;
  const double* d_ks = gauss_taps(L, c.sigma_s, rs);
  MomTaps mtp;
  const double* d_mt = moment_taps(L, c.sigma_w, rw, mtp);

  // reference pack (phaseflow.py:431, reference_phase)
  float2* T = L.get<float2>("fft_T", Np);
  float2* U = L.get<float2>("fft_U", Np * F);
  float4* ref4 = L.get<float4>("ref4", N * F);
  float* amp = L.get<float>("ref_amp", N * F);
  // spline of image 2 (kept for all iterations)
  float* c2 = L.get<float>("spline2", (size_t)w2 * h2);
  if (!prepared) fine_prep(L, i1, W, H, i2, w2, h2, c, st);

  double* u2b = L.get<double>("u2b", 2 * N);
  double* s2 = L.get<double>("s2", 2 * N);
  double* cs2 = L.get<double>("cs2", 2 * N);
  double* pre2 = L.get<double>("pre2", 2 * N);
  double* tmpb = L.get<double>("blur_tmp", 2 * N);
  double* energy = L.get<double>("energy", N);
  double* resid = L.get<double>("resid", N);
  double* slope = L.get<double>("slope", 4 * N);
  double* sums = L.get<double>("sums", 7 * N);
  double* yplanes = L.get<double>("yplanes", (size_t)moment_yplanes(c.shape_order) * N);
  float* warped = L.get<float>("warped", N);
  float2* R = L.get<float2>("resp", resp_values(F, Np));
  EnergyStats* stats = L.get<EnergyStats>("stats", 1);
  unsigned long long* hist = L.get<unsigned long long>("hist", median_scratch(N));
  uint8_t* low = L.get<uint8_t>("low", N);
  uint8_t* frozen = L.get<uint8_t>("frozen", N);
  uint8_t* okm = L.get<uint8_t>("okmask", N);
  int* vdist = L.get<int>("vdist", N);
  int* cold2 = L.get<int>("col_d2", N);
  int* colrow = L.get<int>("col_row", N);
  PrewarpCounts* counts = L.get<PrewarpCounts>("pw_counts", 2);
  OFC_CUDA(cudaMemsetAsync(hist, 0, 4096 * sizeof(unsigned long long), st));
  launch_fill_f64(resid, PI, N, st);
  launch_fill_f64(energy, 1.0, N, st);
  OFC_CUDA(cudaMemsetAsync(slope, 0, 4 * N * sizeof(double), st));

  const double R_trust = auto_guard(c);
  const int Kf = c.prewarp_freeze_at;
  double* ucur = u2;
  double* unext = u2b;
  bool primed = false;  // the first median starts the select state itself; each reset primes the next one's
  for (int it = 0; it < c.outer_iters; it++) {
    const double* blur_in = ucur;
    if (it > 0) {
      uint8_t* lowp = low;
      if (Kf >= 1 && it > Kf) {
        lowp = frozen;  // the low pixels of iteration K (prewarp.rs:79-116)
        OFC_CUDA(cudaMemcpyAsync(&counts[0].low, &counts[1].low, sizeof(int), cudaMemcpyDeviceToDevice, st));
      } else {
        OFC_CUDA(cudaMemsetAsync(&counts[0].low, 0, sizeof(int), st));
        launch_confidence(energy, resid, ucur, ucur + N, W, H, stats, c.phase_tol, c.conf_min, false, 0.0, nullptr,
                          nullptr, low, &counts[0].low, st);
        if (Kf >= 1 && it == Kf) {
          OFC_CUDA(cudaMemcpyAsync(frozen, low, N, cudaMemcpyDeviceToDevice, st));
          OFC_CUDA(cudaMemcpyAsync(&counts[1].low, &counts[0].low, sizeof(int), cudaMemcpyDeviceToDevice, st));
        }
      }
      launch_prewarp_fill(lowp, ucur, ucur + N, slope, W, H, R_trust, &counts[0], okm, vdist, cold2, colrow, pre2,
                          pre2 + N, st);
      blur_in = pre2;
    }
    launch_corr_y(blur_in, tmpb, 2, W, H, d_ks, rs, st);
    launch_corr_x(tmpb, s2, 2, W, H, d_ks, rs, st);
    // the spline of the smoothed field needs only s2: it runs on the side stream beside the warp and the response
    // transforms (which leave HBM mostly idle), joined before the inner iterations read it
    OFC_CUDA(cudaEventRecord(L.fork, st));
    OFC_CUDA(cudaStreamWaitEvent(L.side, L.fork, 0));
    launch_bspline_f64_pair(s2, (double2*)cs2, tmpb, W, H, L.side);
    OFC_CUDA(cudaEventRecord(L.join, L.side));
    launch_warp(c2, w2, h2, s2, s2 + N, shx, shy, W, H, warped, st);
    launch_fft_rows_fwd_real(warped, W, H, plw, ph, T, st);
    launch_fft_cols_filters(T, plh, pw, g, U, st);
    launch_fft_rows_inv_resp(U, plw, ph, F, R, st);
    OFC_CUDA(cudaStreamWaitEvent(st, L.join, 0));
    for (int in = 0; in < c.inner_iters; in++) {
      launch_accumulate(ref4, R, F, ph, pw, ucur, ucur + N, s2, s2 + N, (const double2*)cs2, W, H, sums, st);
      launch_moments_solve(sums, ucur, ucur + N, W, H, c.shape_order, d_mt, rw, mtp, yplanes, unext, unext + N, energy,
                           resid, slope, st);
      const bool last_inner = in == c.inner_iters - 1;
      launch_energy_median(energy, N, stats, last_inner, hist, st, primed);
      launch_reset(energy, ucur, ucur + N, (int)N, stats, unext, unext + N, resid, slope, st, true);
      primed = true;
      std::swap(ucur, unext);
    }
  }
  if (ucur != u2) OFC_CUDA(cudaMemcpyAsync(u2, ucur, 2 * N * sizeof(double), cudaMemcpyDeviceToDevice, st));
  return FineOut{u2, u2 + N, energy, resid, stats};
}

// ---------------------------------------------------------------- the coarse stage
struct CoarseOut {
  int nx, ny;
  const int* xs;  // device
  const int* ys;
  double* ux;
  double* uy;
  double* peak;
  std::vector<int> hxs, hys;
  // per pyramid level (level 0 first): the integer peaks of the raw POC grid (2 ints per point) and its shape
  std::vector<int*> ipk;
  std::vector<int> lnx, lny;
};

// coarse_flow (poc.py:216-239); a, b: float32 images W x H on the device; init: 2 planes or null
CoarseOut coarse_dev(Lane& L, const float* a, const float* b, int W, int H, const double* init, const ofc_config& c) {
  cudaStream_t st = L.stream;
  if (c.poc_win > 64) throw Error(OFC_ERR_ARG, "the CUDA engine's POC windows are at most 64 x 64 (poc_win <= 64)");
  const size_t N = (size_t)W * H;
  int Lv = n_levels(c.max_disp, c.poc_win, H, W);
  int r1 = 0;
  const double* d_k1 = gauss_taps(L, 1.0, r1);
  // pyramid (float64): level 0 is the input itself
  std::vector<double*> pa(Lv + 1), pb(Lv + 1);
  std::vector<int> pws(Lv + 1), phs(Lv + 1);
  pa[0] = L.get<double>("pyr_a0", N);
  pb[0] = L.get<double>("pyr_b0", N);
  launch_f32_to_f64(a, pa[0], N, st);
  launch_f32_to_f64(b, pb[0], N, st);
  pws[0] = W;
  phs[0] = H;
  double* tmp = L.get<double>("pyr_tmp", N);
  for (int l = 1; l <= Lv; l++) {
    int w = (pws[l - 1] + 1) / 2, h = (phs[l - 1] + 1) / 2;
    pa[l] = L.get<double>("pyr_a" + std::to_string(l), (size_t)w * h);
    pb[l] = L.get<double>("pyr_b" + std::to_string(l), (size_t)w * h);
    launch_downsample(pa[l - 1], pws[l - 1], phs[l - 1], pa[l], tmp, d_k1, r1, st);
    launch_downsample(pb[l - 1], pws[l - 1], phs[l - 1], pb[l], tmp, d_k1, r1, st);
    pws[l] = w;
    phs[l] = h;
  }
  std::vector<int> xs0 = arange(c.poc_win / 2, W - c.poc_win / 2 + 1, c.grid_step);
  std::vector<int> ys0 = arange(c.poc_win / 2, H - c.poc_win / 2 + 1, c.grid_step);
  CoarseOut prev{};
  bool have = false;
  std::vector<int*> ipk(Lv + 1);
  std::vector<int> lnx(Lv + 1), lny(Lv + 1);
  for (int lev = Lv; lev >= 0; lev--) {
    int w = pws[lev], h = phs[lev];
    int wy = c.poc_win, wx = c.poc_win;
    std::vector<int> gx = xs0, gy = ys0;
    if (lev != 0) {
      level_window(h, w, c.poc_win, wy, wx);
      gx = arange(wx / 2, w - wx / 2 + 1, c.grid_step);
      gy = arange(wy / 2, h - wy / 2 + 1, c.grid_step);
    }
    if (gx.empty() || gy.empty()) throw Error(OFC_ERR_ARG, "image too small for the POC grid");
    int nx = (int)gx.size(), ny = (int)gy.size();
    std::string sfx = std::to_string(lev);
    const std::string gk = "pocgrid:" + std::to_string(W) + "x" + std::to_string(H) + ":" + sfx + ":" +
                           std::to_string(c.poc_win) + ":" + std::to_string(c.grid_step);
    const int* dxs = L.cached(gk + ":x", gx.data(), gx.size());
    const int* dys = L.cached(gk + ":y", gy.data(), gy.size());
    std::vector<unsigned char> pc(poc_const_bytes());
    poc_const_host(wy, wx, pc.data());
    const void* dconst = L.cached("pocconst:" + std::to_string(wy) + "x" + std::to_string(wx), pc.data(), pc.size());
    double* iu = nullptr;
    double* iv = nullptr;
    if (have) {
      iu = L.get<double>("poc_iu" + sfx, (size_t)nx * ny);
      iv = L.get<double>("poc_iv" + sfx, (size_t)nx * ny);
      launch_grid_sample(prev.ux, prev.uy, prev.xs, prev.ys, prev.nx, prev.ny, dxs, dys, nx, ny, 0.5, 2.0, iu, iv, st);
    } else if (init) {
      iu = L.get<double>("poc_iu" + sfx, (size_t)nx * ny);
      iv = L.get<double>("poc_iv" + sfx, (size_t)nx * ny);
      launch_init_from_dense(init, init + N, W, dxs, dys, nx, ny, 1 << lev, iu, iv, st);
    }
    double* gu = L.get<double>("poc_u" + sfx, (size_t)nx * ny);
    double* gv = L.get<double>("poc_v" + sfx, (size_t)nx * ny);
    double* gp = L.get<double>("poc_p" + sfx, (size_t)nx * ny);
    PocLevel lv{w, h, nx, ny, wy, wx};
    ipk[lev] = L.get<int>("poc_ipk" + sfx, (size_t)2 * nx * ny);
    lnx[lev] = nx;
    lny[lev] = ny;
    launch_poc_grid(pa[lev], pb[lev], lv, dxs, dys, iu, iv, dconst, gu, gv, gp, ipk[lev], st);
    uint8_t* scr = L.get<uint8_t>("poc_flags", (size_t)3 * nx * ny);
    launch_poc_clean(gu, gv, gp, nx, ny, c.poc_peak_min, c.median_thresh, iu, iv, scr, st);
    prev = CoarseOut{nx, ny, dxs, dys, gu, gv, gp, gx, gy, {}, {}, {}};
    have = true;
  }
  prev.ipk = ipk;
  prev.lnx = lnx;
  prev.lny = lny;
  return prev;
}

// dense start of track_pair (track.py:131-137) into u2 (2 planes)
void dense_start(Lane& L, const CoarseOut& g, int W, int H, const double* init, double* u2) {
  cudaStream_t st = L.stream;
  const size_t N = (size_t)W * H;
  if (!init) {
    launch_grid_sample(g.ux, g.uy, g.xs, g.ys, g.nx, g.ny, nullptr, nullptr, W, H, 1.0, 1.0, u2, u2 + N, st);
    return;
  }
  double* cu = L.get<double>("corr_u", (size_t)g.nx * g.ny);
  double* cv = L.get<double>("corr_v", (size_t)g.nx * g.ny);
  launch_grid_minus_dense(g.ux, g.uy, init, init + N, W, g.xs, g.ys, g.nx, g.ny, cu, cv, st);
  launch_grid_sample(cu, cv, g.xs, g.ys, g.nx, g.ny, nullptr, nullptr, W, H, 1.0, 1.0, u2, u2 + N, st);
  launch_add(u2, init, 2 * N, st);
}

// _finish (track.py:56-108): low (u8), roi (u8 or null), ux/uy (raw, f64) -> outputs
// fine_planes: o.conf, o.raw_ux and o.raw_uy were written already (the pair path writes them at the end of the fine
// stage, so that a host download of them overlaps this stage)
void finish_dev(Lane& L, const uint8_t* low, const uint8_t* roi, const double* ux, const double* uy,
                const double* conf64, int W, int H, const ofc_config& c, const ofc_pair_out& o, bool fine_planes) {
  cudaStream_t st = L.stream;
  const size_t N = (size_t)W * H;
  double guard = guard_px(c);
  uint8_t* big = L.get<uint8_t>("fin_big", N);
  uint8_t* src = L.get<uint8_t>("fin_src", N);
  uint8_t* bad = L.get<uint8_t>("fin_bad", N);
  int* parent = L.get<int>("fin_parent", N);
  int* size = L.get<int>("fin_size", N);
  int* vdist = L.get<int>("vdist", N);
  double* mx = L.get<double>("fin_mx", 2 * N);
  double* my = mx + N;
  if (guard > 0) launch_large_components(low, W, H, min_area_px(c), parent, size, big, st);
  launch_finish_mask(low, roi, big, W, H, guard, ux, uy, src, bad, vdist, mx, my, st);
  // the masked field and the valid mask first; then the event L.masked (a host download of those planes may start
  // there, during the strain)
  if (fine_planes) {
    launch_pair_outputs(mx, my, ux, uy, conf64, (int)N, o.ux, o.uy, nullptr, o.valid, nullptr, nullptr, st);
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    OFC_CUDA(cudaStreamIsCapturing(st, &cap));
    if (cap == cudaStreamCaptureStatusActive) OFC_CUDA(cudaEventRecordWithFlags(L.masked, st, cudaEventRecordExternal));
    else OFC_CUDA(cudaEventRecord(L.masked, st));
  } else {
    launch_pair_outputs(mx, my, ux, uy, conf64, (int)N, o.ux, o.uy, o.conf, o.valid, o.raw_ux, o.raw_uy, st);
  }
  double* yp = L.get<double>("strain_y", 11 * N);
  launch_strain(mx, my, W, H, c.strain_win, yp, nullptr, nullptr, nullptr, nullptr, o.exx, o.eyy, o.exy, o.gmax, o.vol,
                st);
}

// the whole pair on device buffers; d_out fields are device pointers
// One pair on the lane's own buffers, in three stages: 0 = coarse POC + dense start, 1 = fine stage + confidence,
// 2 = guard + strain + outputs. Inputs: in_i1, in_i2 (float W*H), in_roi (bytes, when has_roi), in_u, in_v (float,
// when has_init); outputs: out_pair (10 planes) and out_valid.
void pair_stage(Lane& L, int stage, int W, int H, bool has_roi, bool has_init, const ofc_config& c) {
  cudaStream_t st = L.stream;
  const size_t N = (size_t)W * H;
  const float* i1 = L.get<float>("in_i1", N);
  const float* i2 = L.get<float>("in_i2", N);
  double* u2 = L.get<double>("u2", 2 * N);
  double* conf64 = L.get<double>("conf64", N);
  uint8_t* low = L.get<uint8_t>("low_final", N);
  if (stage == 0) {
    // the reference pack of i1 and the spline of i2 on the side stream, beside the coarse stage (joined below)
    OFC_CUDA(cudaEventRecord(L.fork, st));
    OFC_CUDA(cudaStreamWaitEvent(L.side, L.fork, 0));
    fine_prep(L, i1, W, H, i2, W, H, c, L.side);
    OFC_CUDA(cudaEventRecord(L.join, L.side));
    double* init = nullptr;
    if (has_init) {
      init = L.get<double>("init2", 2 * N);
      launch_f32_to_f64(L.get<float>("in_u", N), init, N, st);
      launch_f32_to_f64(L.get<float>("in_v", N), init + N, N, st);
    }
    CoarseOut g = coarse_dev(L, i1, i2, W, H, init, c);
    dense_start(L, g, W, H, init, u2);
    OFC_CUDA(cudaStreamWaitEvent(st, L.join, 0));
  } else if (stage == 1) {
    FineOut f = refine_dev(L, i1, W, H, i2, W, H, 0, 0, u2, c, true);
    double B = guard_px(c) > 0 ? 4.0 * c.sigma_w : 0.0;
    // the output planes that depend on the fine stage only: conf, raw_ux, raw_uy (device_pair_out's layout)
    float* op = L.get<float>("out_pair", 10 * N);
    launch_confidence(f.energy, f.resid, f.ux, f.uy, W, H, f.stats, c.phase_tol, c.conf_min, true, B, op + 2 * N,
                      conf64, low, nullptr, st);
    launch_f64_to_f32(u2, op + 8 * N, N, st);
    launch_f64_to_f32(u2 + N, op + 9 * N, N, st);
  } else if (stage == 3) {
    // the learned proposal in place of stage 0's POC: the network on the pair (padded to a multiple of 8 by edge
    // replication), its 1/8-resolution flow interpolated to the dense start (kept in u2_learned for a fallback)
    OFC_CUDA(cudaEventRecord(L.fork, st));
    OFC_CUDA(cudaStreamWaitEvent(L.side, L.fork, 0));
    fine_prep(L, i1, W, H, i2, W, H, c, L.side);
    OFC_CUDA(cudaEventRecord(L.join, L.side));
    const Proposal& P = *L.proposal;
    const int W8 = (W + 7) / 8 * 8, H8 = (H + 7) / 8 * 8;
    const float* a = i1;
    const float* b = i2;
    if (W8 != W || H8 != H) {
      float* pa = L.get<float>("net_pad1", (size_t)W8 * H8);
      float* pb = L.get<float>("net_pad2", (size_t)W8 * H8);
      launch_pad8(i1, W, H, W8, H8, pa, st);
      launch_pad8(i2, W, H, W8, H8, pb, st);
      a = pa;
      b = pb;
    }
    float* flow = L.get<float>("net_flow", (size_t)(W8 / 8) * (H8 / 8) * 2);
    net::Workspace ws{[&L](const std::string& n, size_t bytes) { return (void*)L.get<uint8_t>(n, bytes); }, st};
    net::forward(ws, P.params, P.w16, a, b, 1, H8, W8, flow);
    launch_cells_to_dense(flow, W8 / 8, H8 / 8, W, H, u2, L.get<double>("u2_learned", 2 * N), st);
    OFC_CUDA(cudaStreamWaitEvent(st, L.join, 0));
  } else if (stage == 4) {
    // the fallback's start: POC + dense start inside the failed tiles, the network's start elsewhere (the reference
    // pack of i1 and the spline of i2 from stage 3 stay valid)
    const Proposal& P = *L.proposal;
    const int nt = ((W + P.tile - 1) / P.tile) * ((H + P.tile - 1) / P.tile);
    CoarseOut g = coarse_dev(L, i1, i2, W, H, nullptr, c);
    dense_start(L, g, W, H, nullptr, u2);
    launch_blend_tiles(L.get<uint8_t>("tile_flags", nt), L.get<double>("u2_learned", 2 * N), W, H, P.tile, u2, st);
  } else if (stage == 5) {
    // the per-tile check of the refined result; the failed-tile count to page-locked memory for the host
    const Proposal& P = *L.proposal;
    const int nt = ((W + P.tile - 1) / P.tile) * ((H + P.tile - 1) / P.tile);
    const uint8_t* roi = has_roi ? L.get<uint8_t>("in_roi", N) : nullptr;
    int* nfail = L.get<int>("tile_nfail", 1);
    // judged pixels: inside the ROI, beyond the border rule's band plus the network's reach (4 sigma_w + 40 px)
    const int B = (int)std::ceil(4.0 * c.sigma_w) + 8 * net::CORR_R;
    launch_tile_check(conf64, roi, W, H, P.tile, B, c.conf_min, P.max_low, L.get<uint8_t>("tile_flags", nt), nfail,
                      st);
    OFC_CUDA(cudaMemcpyAsync(L.pinned<int>("tile_nfail_h", 1), nfail, sizeof(int), cudaMemcpyDeviceToHost, st));
  } else {
    ofc_pair_out o{};
    float* p = L.get<float>("out_pair", 10 * N);
    float** f[10] = {&o.ux, &o.uy, &o.conf, &o.exx, &o.eyy, &o.exy, &o.gmax, &o.vol, &o.raw_ux, &o.raw_uy};
    for (int i = 0; i < 10; i++) *f[i] = p + i * N;
    o.valid = L.get<uint8_t>("out_valid", N);
    const uint8_t* roi = has_roi ? L.get<uint8_t>("in_roi", N) : nullptr;
    finish_dev(L, low, roi, u2, u2 + N, conf64, W, H, c, o, true);
  }
}

// Runs the stages `stages[0..n)` (pair_stage ids) on L.stream. The first call for a key (size, configuration, inputs
// present, profile filter, stage list) runs them eagerly, which allocates every buffer and uploads every constant,
// and then captures each stage as a CUDA graph; later calls replay the graphs. timing: record the stage events
// L.ev[0..n) at the start of each stage and L.ev[3] at the end.
void run_stage_list(Lane& L, const std::string& key, const int* stages, int n, int W, int H, bool has_roi,
                    bool has_init, const ofc_config& c, bool timing) {
  cudaStream_t st = L.stream;
  Profiler* prof = g_profiler;
  auto it = L.graphs.find(key);
  if (it == L.graphs.end() || it->second->eager) {
    for (int sgi = 0; sgi < n; sgi++) {
      if (timing) OFC_CUDA(cudaEventRecord(L.ev[sgi], st));
      pair_stage(L, stages[sgi], W, H, has_roi, has_init, c);
    }
    if (timing) OFC_CUDA(cudaEventRecord(L.ev[3], st));
  }
  if (it == L.graphs.end()) {
    std::unique_ptr<Lane::Graph> g(new Lane::Graph());
    bool ok = true;
    for (int sgi = 0; sgi < n && ok; sgi++) {
      cudaGraph_t graph = nullptr;
      const uint64_t before = g_launch_counter ? *g_launch_counter : 0;
      OFC_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
      if (prof) prof->capture = &g->events;
      try {
        pair_stage(L, stages[sgi], W, H, has_roi, has_init, c);
      } catch (...) {
        if (prof) prof->capture = nullptr;
        cudaStreamEndCapture(st, &graph);
        if (graph) cudaGraphDestroy(graph);
        throw;
      }
      if (prof) prof->capture = nullptr;
      if (g_launch_counter) {
        g->launches[sgi] = *g_launch_counter - before;  // captured, not launched
        *g_launch_counter = before;
      }
      OFC_CUDA(cudaStreamEndCapture(st, &graph));
      cudaError_t e = cudaGraphInstantiate(&g->exec[sgi], graph, 0);
      cudaGraphDestroy(graph);
      if (e != cudaSuccess) {
        ok = false;
        (void)cudaGetLastError();
      }
    }
    if (!ok) {
      std::unique_ptr<Lane::Graph> bad(new Lane::Graph());
      bad->eager = true;
      g = std::move(bad);
    }
    L.graphs[key] = std::move(g);
  } else if (!it->second->eager) {
    Lane::Graph& g = *it->second;
    for (int sgi = 0; sgi < n; sgi++) {
      if (timing) OFC_CUDA(cudaEventRecord(L.ev[sgi], st));
      OFC_CUDA(cudaGraphLaunch(g.exec[sgi], st));
      if (g_launch_counter) *g_launch_counter += g.launches[sgi];
    }
    if (timing) OFC_CUDA(cudaEventRecord(L.ev[3], st));
    if (prof && !g.events.empty()) {
      // the replay's kernel times: the graph records its event pairs anew at every launch
      OFC_CUDA(cudaStreamSynchronize(st));
      std::lock_guard<std::mutex> lk(prof->mu);
      for (auto& ev : g.events) {
        float ms = 0;
        OFC_CUDA(cudaEventElapsedTime(&ms, std::get<1>(ev), std::get<2>(ev)));
        auto& t = prof->totals[std::get<0>(ev)];
        t.first += 1;
        t.second += ms;
      }
    }
  }
}

std::string pair_key(int W, int H, bool has_roi, bool has_init, const ofc_config& c, const std::string& tail) {
  Profiler* prof = g_profiler;
  return std::to_string(W) + "x" + std::to_string(H) + ":" + cfg_key(c) + ":" + (has_roi ? "r" : "-") +
         (has_init ? "i" : "-") + ":" + tail + ":" + (prof ? "P" + prof->filter : "");
}

// A pair with the learned coarse proposal: the network's start (stage 3), the fine stage (1) and the per-tile check
// (5); when a tile fails, the POC start inside the failed tiles (4) and the fine stage again (1); then the finish (2).
// The host reads the failed-tile count between the two parts. Stage events as run_pair's: the coarse start, the
// fine start, the finish start (after a fallback) and the end.
void run_pair_learned(Lane& L, int W, int H, bool has_roi, const ofc_config& c, bool timing) {
  Proposal& P = *L.proposal;
  cudaStream_t st = L.stream;
  const std::string tail = "learned" + std::to_string(P.tile) + "/" + std::to_string(P.max_low);
  static const int first[3] = {3, 1, 5}, fallback[2] = {4, 1}, finish[1] = {2};
  if (timing) OFC_CUDA(cudaEventRecord(L.ev[0], st));
  run_stage_list(L, pair_key(W, H, has_roi, false, c, tail + "a"), first, 1, W, H, has_roi, false, c, false);
  if (timing) OFC_CUDA(cudaEventRecord(L.ev[1], st));
  run_stage_list(L, pair_key(W, H, has_roi, false, c, tail + "b"), first + 1, 2, W, H, has_roi, false, c, false);
  OFC_CUDA(cudaStreamSynchronize(st));
  const int nfail = *L.pinned<int>("tile_nfail_h", 1);
  const int nt = ((W + P.tile - 1) / P.tile) * ((H + P.tile - 1) / P.tile);
  P.pairs++;
  P.tiles += nt;
  P.failed += nfail;
  if (nfail > 0) {
    P.fallbacks++;
    run_stage_list(L, pair_key(W, H, has_roi, false, c, tail + "f"), fallback, 2, W, H, has_roi, false, c, false);
  }
  if (timing) OFC_CUDA(cudaEventRecord(L.ev[2], st));
  run_stage_list(L, pair_key(W, H, has_roi, false, c, tail + "e"), finish, 1, W, H, has_roi, false, c, false);
  if (timing) OFC_CUDA(cudaEventRecord(L.ev[3], st));
}

// The pair's three stages (nstages 3), or a sequence leg's first two (nstages 2: coarse and fine, whose conf, raw_ux
// and raw_uy planes of "out_pair" are its result). A lane with a learned proposal runs pairs without a start field
// through run_pair_learned; sequence legs and pairs with a start keep the POC coarse stage.
void run_pair(Lane& L, int W, int H, bool has_roi, bool has_init, const ofc_config& c, bool timing, int nstages) {
  if (L.proposal && !has_init && nstages == 3) {
    run_pair_learned(L, W, H, has_roi, c, timing);
    return;
  }
  static const int stages[3] = {0, 1, 2};
  run_stage_list(L, pair_key(W, H, has_roi, has_init, c, std::to_string(nstages)), stages, nstages, W, H, has_roi,
                 has_init, c, timing);
}

// seconds per stage of the last run_pair that recorded its stage events (waits for its end)
void pair_timing(Lane& L, double* timing) {
  OFC_CUDA(cudaEventSynchronize(L.ev[3]));
  float ms[3];
  for (int i = 0; i < 3; i++) OFC_CUDA(cudaEventElapsedTime(&ms[i], L.ev[i], L.ev[i + 1]));
  for (int i = 0; i < 3; i++) timing[i] = ms[i] * 1e-3;
}

void check_sizes(size_t w, size_t h) {
  if (w < 1 || h < 1) throw Error(OFC_ERR_ARG, "empty image");
  if (w > 32768 || h > 32768 || w * h > (size_t)1 << 30) throw Error(OFC_ERR_WINDOW, "image too large for the CUDA engine");
}

void check_fine_window(size_t w, size_t h, const ofc_config& c) {
  check_sizes(w, h);
  int pw = (int)w + 2 * PAD, ph = (int)h + 2 * PAD;
  if (fft_work_length(pw) == 0 || fft_work_length(ph) == 0)
    throw Error(OFC_ERR_WINDOW, "window " + std::to_string(w) + "x" + std::to_string(h) +
                                    ": no FFT plan for the padded size " + std::to_string(pw) + "x" +
                                    std::to_string(ph));
  if (!fft_fits(ph, pw))
    throw Error(OFC_ERR_WINDOW, "window " + std::to_string(w) + "x" + std::to_string(h) +
                                    " exceeds the shared-memory FFT passes of the CUDA engine");
}

// ---------------------------------------------------------------- temporal averaging front-end (tavg)
// rust/crates/optflow-cli/src/tavg.rs (the CLI's implementation; python/optflow_ref/tavg.py is its specification,
// whose scipy map_coordinates warp differs from the CLI's B-spline warp only near the image border).

// least squares v = c0 + c1 x + c2 y through the selected points in centred coordinates, by Gaussian elimination
// with partial pivoting (the last of equal pivots) on the 3 x 3 normal equations (tavg.rs:34-79); false on a pivot
// below 1e-12
static bool tavg_lstsq(const std::vector<double>& xs, const std::vector<double>& ys, const std::vector<double>& v,
                       const std::vector<char>& sel, double out[3]) {
  double n = 0, mx = 0, my = 0;
  for (size_t i = 0; i < xs.size(); i++)
    if (sel[i]) { n += 1; mx += xs[i]; my += ys[i]; }
  mx /= n;
  my /= n;
  double a[3][4] = {};
  for (size_t i = 0; i < xs.size(); i++) {
    if (!sel[i]) continue;
    const double row[3] = {1.0, xs[i] - mx, ys[i] - my};
    for (int r = 0; r < 3; r++) {
      for (int c = 0; c < 3; c++) a[r][c] += row[r] * row[c];
      a[r][3] += row[r] * v[i];
    }
  }
  for (int c = 0; c < 3; c++) {
    int p = c;
    for (int i = c + 1; i < 3; i++)
      if (std::fabs(a[i][c]) >= std::fabs(a[p][c])) p = i;
    if (std::fabs(a[p][c]) < 1e-12) return false;
    for (int k = 0; k < 4; k++) std::swap(a[c][k], a[p][k]);
    for (int i = c + 1; i < 3; i++) {
      const double f = a[i][c] / a[c][c];
      for (int k = c; k < 4; k++) a[i][k] -= f * a[c][k];
    }
  }
  double x[3];
  for (int i = 2; i >= 0; i--) {
    double t = a[i][3];
    for (int j = i + 1; j < 3; j++) t -= a[i][j] * x[j];
    x[i] = t / a[i][i];
  }
  out[0] = x[0] - x[1] * mx - x[2] * my;
  out[1] = x[1];
  out[2] = x[2];
  return true;
}

// robust affine through scattered displacements (tavg.rs:81-114): four fits, each keeping the points whose
// residual is at most max(3 x 1.4826 MAD, 0.05 px) of the previous one; false below 6 points or on a failed solve
static bool tavg_fit_affine(const std::vector<double>& xs, const std::vector<double>& ys, const std::vector<double>& ux,
                            const std::vector<double>& uy, double cx[3], double cy[3]) {
  const size_t n = xs.size();
  std::vector<char> sel(n, 1);
  std::vector<double> r(n);
  for (int pass = 0; pass < 4; pass++) {
    size_t cnt = 0;
    for (char s2 : sel) cnt += s2 ? 1 : 0;
    if (cnt < 6) return false;
    if (!tavg_lstsq(xs, ys, ux, sel, cx) || !tavg_lstsq(xs, ys, uy, sel, cy)) return false;
    std::vector<double> rs;
    for (size_t i = 0; i < n; i++) {
      r[i] = std::hypot(cx[0] + cx[1] * xs[i] + cx[2] * ys[i] - ux[i], cy[0] + cy[1] * xs[i] + cy[2] * ys[i] - uy[i]);
      if (sel[i]) rs.push_back(r[i]);
    }
    std::sort(rs.begin(), rs.end());
    const size_t m = rs.size();
    const double med = m % 2 ? rs[m / 2] : 0.5 * (rs[m / 2 - 1] + rs[m / 2]);
    const double lim = std::max(3.0 * 1.4826 * med, 0.05);
    for (size_t i = 0; i < n; i++) sel[i] = r[i] <= lim ? 1 : 0;
  }
  return true;
}

// the affine field c0 + c1 x + c2 y per axis, rounded to float32 (the CLI's Image<f32> field, tavg.rs:152-157)
__global__ void k_affine_field(double ax, double bx, double cx, double ay, double by, double cy, int W, int H,
                               double* __restrict__ ux, double* __restrict__ uy) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= W) return;
  const size_t p = (size_t)y * W + x;
  ux[p] = (double)(float)(ax + bx * (double)x + cx * (double)y);
  uy[p] = (double)(float)(ay + by * (double)x + cy * (double)y);
}

// align_to (tavg.rs:116-161) on device images c, o (W x H f32) into out: false when no motion could be estimated
// (no output written). model 0: the robust affine fit to the POC grid points with a peak and (hmask, host, nullable)
// inside the mask; 1: the coarse flow interpolated bilinearly. out = o(x + u(x)) by the cubic B-spline of o.
static bool tavg_align_dev(Lane& L, const float* c, const float* o, int W, int H, const uint8_t* hmask, int model,
                           const ofc_config& cfg, float* out) {
  cudaStream_t st = L.stream;
  const size_t N = (size_t)W * H;
  CoarseOut g = coarse_dev(L, c, o, W, H, nullptr, cfg);
  double* u2 = L.get<double>("tavg_u2", 2 * N);
  if (model == 1) {
    launch_grid_sample(g.ux, g.uy, g.xs, g.ys, g.nx, g.ny, nullptr, nullptr, W, H, 1.0, 1.0, u2, u2 + N, st);
    float* f = L.get<float>("tavg_f32", 2 * N);  // the field as float32 (tavg.rs:127-133)
    launch_f64_to_f32(u2, f, 2 * N, st);
    launch_f32_to_f64(f, u2, 2 * N, st);
  } else {
    const size_t ng = (size_t)g.nx * g.ny;
    std::vector<double> gu(ng), gv(ng), gp(ng);
    OFC_CUDA(cudaMemcpyAsync(gu.data(), g.ux, ng * 8, cudaMemcpyDeviceToHost, st));
    OFC_CUDA(cudaMemcpyAsync(gv.data(), g.uy, ng * 8, cudaMemcpyDeviceToHost, st));
    OFC_CUDA(cudaMemcpyAsync(gp.data(), g.peak, ng * 8, cudaMemcpyDeviceToHost, st));
    OFC_CUDA(cudaStreamSynchronize(st));
    std::vector<double> xs, ys, vx, vy;
    for (int iy = 0; iy < g.ny; iy++)
      for (int ix = 0; ix < g.nx; ix++) {
        const size_t j = (size_t)iy * g.nx + ix;
        const int x = g.hxs[ix], y = g.hys[iy];
        if (!((float)gp[j] > 0.0f)) continue;
        if (hmask && !hmask[(size_t)y * W + x]) continue;
        xs.push_back(x);
        ys.push_back(y);
        vx.push_back((double)(float)gu[j]);  // the grid is float32 (poc.rs Grid)
        vy.push_back((double)(float)gv[j]);
      }
    if (xs.size() < 6) return false;
    double cx[3], cy[3];
    if (!tavg_fit_affine(xs, ys, vx, vy, cx, cy)) return false;
    OFC_LAUNCH(k_affine_field, dim3(div_up(W, 128), H), 128, 0, st, cx[0], cx[1], cx[2], cy[0], cy[1], cy[2], W, H, u2,
               u2 + N);
  }
  float* c2 = L.get<float>("tavg_spline", N);
  double* tmp = L.get<double>("tavg_spline_tmp", 2 * N);
  launch_bspline_f32(o, c2, tmp, W, H, st);
  launch_warp(c2, W, H, u2, u2 + N, 0, 0, W, H, out, st);
  return true;
}

// the mean of the frames of a window in float64: the sum of the others (in order) added to the centre, over their
// count (tavg.rs:195-206)
__global__ void k_tavg_add(const float* __restrict__ f, size_t n, double* __restrict__ acc, int first) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    acc[i] = first ? (double)f[i] : acc[i] + (double)f[i];
}
__global__ void k_tavg_mean(const float* __restrict__ c, const double* __restrict__ acc, size_t n, double cnt,
                            float* __restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = (float)(((double)c[i] + acc[i]) / cnt);
}

// average_window_with on device frames (tavg.rs:163-210; tavg.py:61-74): the mean of frames[0..n) (each W x H)
// around frames[centre] into out; align 0 plain, 1 affine (hmask the fit's ROI, host, nullable), 2 dense; a
// neighbour whose alignment fails is left out, or with keep_unaligned enters unaligned. Returns the frames used.
int window_mean_dev(Lane& L, const float* const* frames, size_t n, size_t centre, int W, int H, int align,
                    const uint8_t* hmask, bool keep_unaligned, const ofc_config& c, float* out) {
  cudaStream_t st = L.stream;
  const size_t N = (size_t)W * H;
  float* dal = L.get<float>("tavg_out", N);
  double* acc = L.get<double>("tavg_acc", N);
  const unsigned blocks = std::min(div_up(N, 256), 8192u);
  const float* dc = frames[centre];
  int used = 0;
  for (size_t i = 0; i < n; i++) {
    if (i == centre) continue;
    const float* add = frames[i];
    if (align) {
      if (tavg_align_dev(L, dc, frames[i], W, H, align == 1 ? hmask : nullptr, align - 1, c, dal)) add = dal;
      else if (!keep_unaligned) continue;
    }
    OFC_LAUNCH(k_tavg_add, blocks, 256, 0, st, add, N, acc, used == 0 ? 1 : 0);
    used++;
  }
  if (used == 0) OFC_CUDA(cudaMemcpyAsync(out, dc, N * 4, cudaMemcpyDeviceToDevice, st));
  else OFC_LAUNCH(k_tavg_mean, blocks, 256, 0, st, dc, acc, N, (double)(used + 1), out);
  return used + 1;
}

// ---------------------------------------------------------------- sequence chain (track_sequence)
// rust/crates/optflow-core/src/track.rs:863-1245 (python/optflow_ref/track.py:231-315)

// bilinear sample in float64 with the reference's rules (track.rs:866-896): NaN outside [0, w-1] x [0, h-1], for a
// non-finite coordinate, and where a NaN of the image enters the cell
__device__ __forceinline__ double bilinear64(const float* __restrict__ a, int w, int h, double x, double y) {
  if (!(isfinite(x) && isfinite(y)) || x < 0.0 || y < 0.0 || x > (double)(w - 1) || y > (double)(h - 1)) return nan("");
  int x0 = 0, x1 = 0, y0 = 0, y1 = 0;
  double tx = 0.0, ty = 0.0;
  if (w > 1) { x0 = min((int)floor(x), w - 2); x1 = x0 + 1; tx = x - x0; }
  if (h > 1) { y0 = min((int)floor(y), h - 2); y1 = y0 + 1; ty = y - y0; }
  auto at = [&](int yy, int xx) { return (double)a[(size_t)yy * w + xx]; };
  return (1.0 - ty) * ((1.0 - tx) * at(y0, x0) + tx * at(y0, x1)) + ty * ((1.0 - tx) * at(y1, x0) + tx * at(y1, x1));
}

// compose (track.rs:904-930): c = a + b(X + a), float64, stored float32
__global__ void k_compose(const float* __restrict__ ax, const float* __restrict__ ay, const float* __restrict__ bx,
                          const float* __restrict__ by, int W, int H, float* __restrict__ cx, float* __restrict__ cy) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= W) return;
  const size_t i = (size_t)y * W + x;
  const double u = ax[i], v = ay[i], px = x + u, py = y + v;
  cx[i] = (float)(u + bilinear64(bx, W, H, px, py));
  cy[i] = (float)(v + bilinear64(by, W, H, px, py));
}

// link_conf (track.rs:935-955): min(c0r, conf(X + u0r)), a NaN sample counting as 0; out may be c0r
__global__ void k_link_conf(const double* c0r, const float* __restrict__ conf, const float* __restrict__ ux,
                            const float* __restrict__ uy, int W, int H, double* out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= W) return;
  const size_t i = (size_t)y * W + x;
  const double c = bilinear64(conf, W, H, x + (double)ux[i], y + (double)uy[i]);
  out[i] = fmin(c0r[i], isfinite(c) ? c : 0.0);
}

// mean_conf (track.rs:957-1023): the reportable image of the leg (the border rule on its raw field), then per pixel
// the sampled confidence where it counts; the rows summed in order by one thread each, the rows folded in order
__global__ void k_reportable(const float* __restrict__ rx, const float* __restrict__ ry, int W, int H, double B,
                             float* __restrict__ rep) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= W) return;
  const size_t i = (size_t)y * W + x;
  const double tx = x + (double)rx[i], ty = y + (double)ry[i];
  const double own = (double)min(min(x, y), min(W - 1 - x, H - 1 - y));
  rep[i] = (own >= B && tx >= B && ty >= B && (W - 1) - tx >= B && (H - 1) - ty >= B) ? 1.f : 0.f;
}
// one block of MC_T threads per row: each thread sums the pixels x = tid, tid + MC_T, ..., then a fixed-order tree
// (warp shuffles, then the warps in order) gives the row's sum and count, the same on every run
constexpr int MC_T = 128;
__global__ void __launch_bounds__(MC_T) k_mean_conf_rows(const float* __restrict__ conf, const float* __restrict__ rep,
                                                         const float* __restrict__ ux, const float* __restrict__ uy,
                                                         const uint8_t* __restrict__ mask, int W, int H,
                                                         double* __restrict__ rsum, long long* __restrict__ rcnt) {
  __shared__ double wsum[MC_T / 32];
  __shared__ long long wcnt[MC_T / 32];
  const int y = blockIdx.x;
  double sum = 0.0;
  long long n = 0;
  for (int x = threadIdx.x; x < W; x += MC_T) {
    const size_t i = (size_t)y * W + x;
    const double px = x + (double)ux[i], py = y + (double)uy[i];
    const double c = bilinear64(conf, W, H, px, py);
    if (isfinite(c) && bilinear64(rep, W, H, px, py) > 0.5 && (!mask || mask[i])) {
      sum += c;
      n++;
    }
  }
  for (int o = 16; o; o >>= 1) {
    sum += __shfl_down_sync(0xffffffffu, sum, o);
    n += __shfl_down_sync(0xffffffffu, n, o);
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) {
    wsum[wid] = sum;
    wcnt[wid] = n;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    long long c = 0;
    for (int k = 0; k < MC_T / 32; k++) {
      s += wsum[k];
      c += wcnt[k];
    }
    rsum[y] = s;
    rcnt[y] = c;
  }
}
__global__ void k_mean_conf_fold(const double* __restrict__ rsum, const long long* __restrict__ rcnt, int H,
                                 double* out) {
  double s = 0.0;
  long long n = 0;
  for (int y = 0; y < H; y++) {
    s += rsum[y];
    n += rcnt[y];
  }
  *out = n == 0 ? 0.0 : s / (double)n;
}

// ---------------------------------------------------------------- hybrid sequence mode
// python/optflow_ref/track.py:331-503 (rust/crates/optflow-core/src/track/hybrid.rs)

// pixel classes of one hybrid frame, one uint16 per pixel (the boolean planes of track.py:441-487)
enum : uint16_t {
  HY_GOOD = 1,     // direct-good (after the re-acquisition: good | re)
  HY_CANDRE = 2,   // re-acquisition candidate: direct_ok, unanchored, in the ROI, the reference older than k - 1
  HY_NEED = 4,     // needs the adjacent leg: not good, in the ROI, u_{k-1} finite, n_fb + 1 <= fb_max
  HY_HASFB = 8,    // a fallback value exists (need and adjacent confidence >= conf_min)
  HY_AGREE = 16,   // |u_direct - u_fallback| <= fb_tol
  HY_RENOFB = 32,  // candidate without a fallback value (after the spatial gate when it ran)
  HY_RE = 64,      // re-acquired
  HY_FBCAND = 128, // fallback candidate
  HY_FBOK = 256    // fallback candidate that passed the spatial gate
};

__device__ __forceinline__ double conf_at64(const float* __restrict__ conf, int W, int H, double px, double py) {
  const double c = bilinear64(conf, W, H, px, py);
  return isfinite(c) ? c : 0.0;
}

// the reference moves to k - 1 (track.py:433-437): c0K = the old leg's confidence at X + u0K where the pixel was
// direct-good at k - 1, else 0 (unanchored); anch = good_prev
__global__ void k_hyb_move(const float* __restrict__ pconf, const float* __restrict__ u0x,
                           const float* __restrict__ u0y, const uint8_t* __restrict__ good_prev, int W, int H,
                           double* __restrict__ c0r, uint8_t* __restrict__ anch) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= W) return;
  const size_t i = (size_t)y * W + x;
  const bool g = good_prev[i] != 0;
  c0r[i] = g ? conf_at64(pconf, W, H, x + (double)u0x[i], y + (double)u0y[i]) : 0.0;
  anch[i] = g ? 1 : 0;
}

// the direct leg on the frame-0 grid (track.py:441-451): c = compose(u0K, leg), leg_c = conf_at(leg, u0K), link,
// and the classes good, cand_re, need; any[0] = some pixel needs the adjacent leg
__global__ void k_hyb_classify(const float* __restrict__ rx, const float* __restrict__ ry,
                               const float* __restrict__ conf, const float* __restrict__ u0x,
                               const float* __restrict__ u0y, const double* __restrict__ c0r,
                               const uint8_t* __restrict__ anch, const float* __restrict__ upx,
                               const float* __restrict__ upy, const int* __restrict__ nfb,
                               const uint8_t* __restrict__ roi, int W, int H, double conf_min, int fb_max,
                               int reacq_ok, float* __restrict__ cx, float* __restrict__ cy,
                               double* __restrict__ legc, double* __restrict__ link, uint16_t* __restrict__ fl,
                               int* any) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= W) return;
  const size_t i = (size_t)y * W + x;
  const double u = u0x[i], v = u0y[i], px = x + u, py = y + v;
  const float vx = (float)(u + bilinear64(rx, W, H, px, py)), vy = (float)(v + bilinear64(ry, W, H, px, py));
  const double lc = conf_at64(conf, W, H, px, py);
  const bool an = anch[i] != 0, in = !roi || roi[i];
  const double lk = an ? fmin(c0r[i], lc) : lc;
  const bool dok = isfinite(vx) && isfinite(vy) && lk >= conf_min;
  const bool good = dok && an;
  const bool cre = dok && !an && in && reacq_ok;
  const bool need = !good && in && isfinite(upx[i]) && isfinite(upy[i]) && nfb[i] < fb_max;
  cx[i] = vx;
  cy[i] = vy;
  legc[i] = lc;
  link[i] = lk;
  fl[i] = (good ? HY_GOOD : 0) | (cre ? HY_CANDRE : 0) | (need ? HY_NEED : 0);
  if (need) *any = 1;
}

// the adjacent leg carried from u_{k-1} (track.py:453-464): a = compose(u_{k-1}, adj), u_{k-1} where that leaves the
// image, ca = conf_at(adj, u_{k-1}); without the leg (rx null) a = u_{k-1}, ca = 0
__global__ void k_hyb_adjacent(const float* __restrict__ rx, const float* __restrict__ ry,
                               const float* __restrict__ conf, const float* __restrict__ upx,
                               const float* __restrict__ upy, int W, int H, float* __restrict__ ax,
                               float* __restrict__ ay, double* __restrict__ ca) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= W) return;
  const size_t i = (size_t)y * W + x;
  if (!rx) {
    ax[i] = upx[i];
    ay[i] = upy[i];
    ca[i] = 0.0;
    return;
  }
  const double u = upx[i], v = upy[i], px = x + u, py = y + v;
  const float vx = (float)(u + bilinear64(rx, W, H, px, py)), vy = (float)(v + bilinear64(ry, W, H, px, py));
  const bool ok = isfinite(vx) && isfinite(vy);
  ax[i] = ok ? vx : upx[i];
  ay[i] = ok ? vy : upy[i];
  ca[i] = conf_at64(conf, W, H, px, py);
}

// has_fb, agree, re_nofb (track.py:465-470); support = good & roi for the gate of re_nofb; any[1] = some ROI pixel
// is a candidate without a fallback value
__global__ void k_hyb_pre(uint16_t* __restrict__ fl, const float* __restrict__ cx, const float* __restrict__ cy,
                          const float* __restrict__ ax, const float* __restrict__ ay, const double* __restrict__ ca,
                          const uint8_t* __restrict__ roi, size_t N, double conf_min, double fb_tol,
                          uint8_t* __restrict__ support, int* any) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
    uint16_t f = fl[i];
    const bool in = !roi || roi[i];
    const bool hasfb = (f & HY_NEED) && ca[i] >= conf_min;
    const bool agree = hypot((double)cx[i] - (double)ax[i], (double)cy[i] - (double)ay[i]) <= fb_tol;
    const bool renofb = (f & HY_CANDRE) && !hasfb;
    f |= (hasfb ? HY_HASFB : 0) | (agree ? HY_AGREE : 0) | (renofb ? HY_RENOFB : 0);
    fl[i] = f;
    support[i] = ((f & HY_GOOD) && in) ? 1 : 0;
    if (renofb && in) any[1] = 1;
  }
}

// re-acquisition and the counters (track.py:476-481): re = (cand_re & has_fb & agree) | re_nofb (gated by gate0
// when given), c0K = leg_c and anchored where re, good |= re, n_fb = 0 where good else min(n_fb + 1, fb_max + 1),
// fb_cand; support = good & roi for the fallback gate; any[2] = some ROI pixel is a fallback candidate
__global__ void k_hyb_re(uint16_t* __restrict__ fl, const uint8_t* __restrict__ gate0,
                         const double* __restrict__ legc, double* __restrict__ c0r, uint8_t* __restrict__ anch,
                         int* __restrict__ nfb, const double* __restrict__ ca, const uint8_t* __restrict__ roi,
                         size_t N, int fb_max, double conf_min, uint8_t* __restrict__ support, int* any) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
    uint16_t f = fl[i];
    const bool in = !roi || roi[i];
    const bool renofb = (f & HY_RENOFB) && (!gate0 || gate0[i]);
    const bool re = ((f & HY_CANDRE) && (f & HY_HASFB) && (f & HY_AGREE)) || renofb;
    bool good = (f & HY_GOOD) != 0;
    if (re) {
      c0r[i] = legc[i];
      anch[i] = 1;
      good = true;
    }
    const int nf = good ? 0 : (int)min((long long)nfb[i] + 1, (long long)fb_max + 1);
    nfb[i] = nf;
    const bool fbc = !good && (f & HY_NEED) && nf <= fb_max && ca[i] >= conf_min;
    f = (uint16_t)((f & ~(HY_GOOD | HY_RENOFB)) | (good ? HY_GOOD : 0) | (renofb ? HY_RENOFB : 0) |
                   (re ? HY_RE : 0) | (fbc ? HY_FBCAND : 0));
    fl[i] = f;
    support[i] = (good && in) ? 1 : 0;
    if (fbc && in) any[2] = 1;
  }
}

// the frame's output (track.py:486-501): u = c where good else a (u_{k} of the next frame, and its float64 copy
// for the finish), conf = link or ca (1 - n_fb / (fb_max + 1))^+, low = !(good | fb_ok), good_prev = good;
// cnt[0..2] += fb_ok, fb_cand & !fb_ok, re over the ROI; cnt[3] = max n_fb over the image
__global__ void k_hyb_out(uint16_t* __restrict__ fl, const uint8_t* __restrict__ gate, const float* __restrict__ cx,
                          const float* __restrict__ cy, const float* __restrict__ ax, const float* __restrict__ ay,
                          const double* __restrict__ link, const double* __restrict__ ca, const int* __restrict__ nfb,
                          const uint8_t* __restrict__ roi, size_t N, int fb_max, float* __restrict__ ux,
                          float* __restrict__ uy, double* __restrict__ u64x, double* __restrict__ u64y,
                          double* __restrict__ conf, uint8_t* __restrict__ low, uint8_t* __restrict__ good_prev,
                          unsigned long long* cnt) {
  unsigned long long c0 = 0, c1 = 0, c2 = 0, mx = 0;
  const double cap = (double)fb_max + 1.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
    uint16_t f = fl[i];
    const bool in = !roi || roi[i];
    const bool good = (f & HY_GOOD) != 0;
    const bool fbok = (f & HY_FBCAND) && (!gate || gate[i]);
    const float vx = good ? cx[i] : ax[i], vy = good ? cy[i] : ay[i];
    ux[i] = vx;
    uy[i] = vy;
    u64x[i] = vx;
    u64y[i] = vy;
    const int nf = nfb[i];
    conf[i] = good ? link[i] : ca[i] * fmax(0.0, 1.0 - (double)nf / cap);
    low[i] = (good || fbok) ? 0 : 1;
    good_prev[i] = good ? 1 : 0;
    fl[i] = (uint16_t)(f | (fbok ? HY_FBOK : 0));
    c0 += (fbok && in);
    c1 += ((f & HY_FBCAND) && !fbok && in);
    c2 += ((f & HY_RE) && in);
    mx = max(mx, (unsigned long long)nf);
  }
  for (int o = 16; o > 0; o >>= 1) {
    c0 += __shfl_down_sync(0xffffffffu, c0, o);
    c1 += __shfl_down_sync(0xffffffffu, c1, o);
    c2 += __shfl_down_sync(0xffffffffu, c2, o);
    mx = max(mx, __shfl_down_sync(0xffffffffu, mx, o));
  }
  if ((threadIdx.x & 31) == 0) {
    if (c0) atomicAdd(&cnt[0], c0);
    if (c1) atomicAdd(&cnt[1], c1);
    if (c2) atomicAdd(&cnt[2], c2);
    atomicMax(&cnt[3], mx);
  }
}

// _local_affine_agreement (track.py:331-382): window sums of the 12 moments of the selected pixels, rows first
// (zero outside the image), then the columns and the 3 x 3 ridge solve per pixel. Moments, in order: 1, x, y, xx,
// xy, yy, u, xu, yu, v, xv, yv, each a product of the pixel's own float64 values (the reference's box(w * xx * comp)).
constexpr int LAA_M = 12;

template <typename T>
__global__ void k_laa_rows(const uint8_t* __restrict__ sel, const T* __restrict__ ux, const T* __restrict__ uy, int W,
                           int H, int r, double* __restrict__ rows) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= W) return;
  const size_t row = (size_t)y * W, N = (size_t)W * H;
  double s[LAA_M];
#pragma unroll
  for (int m = 0; m < LAA_M; m++) s[m] = 0.0;
  const double yd = y;
  const int q0 = max(0, x - r), q1 = min(W - 1, x + r);
  for (int q = q0; q <= q1; q++) {
    if (!sel[row + q]) continue;
    const double xd = q, u = (double)ux[row + q], v = (double)uy[row + q];
    s[0] += 1.0;
    s[1] += xd;
    s[2] += yd;
    s[3] += xd * xd;
    s[4] += xd * yd;
    s[5] += yd * yd;
    s[6] += u;
    s[7] += xd * u;
    s[8] += yd * u;
    s[9] += v;
    s[10] += xd * v;
    s[11] += yd * v;
  }
#pragma unroll
  for (int m = 0; m < LAA_M; m++) rows[m * N + row + x] = s[m];
}

// m c = b for two right-hand sides by Gaussian elimination with partial pivoting (the first of equal pivots, as
// LAPACK's getrf); false for a zero or non-finite pivot (hybrid.rs:112-144)
__device__ bool solve3x2(double a[3][5], double out[3][2]) {
  for (int c = 0; c < 3; c++) {
    int p = c;
    for (int i = c + 1; i < 3; i++)
      if (fabs(a[i][c]) > fabs(a[p][c])) p = i;
    if (a[p][c] == 0.0 || !isfinite(a[p][c])) return false;
    if (p != c)
      for (int j = 0; j < 5; j++) {
        const double t = a[c][j];
        a[c][j] = a[p][j];
        a[p][j] = t;
      }
    for (int i = c + 1; i < 3; i++) {
      const double f = a[i][c] / a[c][c];
      for (int j = c; j < 5; j++) a[i][j] -= f * a[c][j];
    }
  }
  for (int k = 0; k < 2; k++)
    for (int i = 2; i >= 0; i--) {
      double s = a[i][3 + k];
      for (int j = i + 1; j < 3; j++) s -= a[i][j] * out[j][k];
      out[i][k] = s / a[i][i];
    }
  return true;
}

// the column sums and the fit at every pixel; pass 0 writes the robust selection of the next pass (support pixels
// within 3 tol of their own model), pass 1 the test ok = n + 0.5 >= min_support, n >= 3, |(tx, ty) - a| <= tol
template <typename T>
__global__ void k_laa_solve(const double* __restrict__ rows, int W, int H, int r, double ridge, int pass,
                            const uint8_t* __restrict__ support, const T* __restrict__ ux, const T* __restrict__ uy,
                            const T* __restrict__ tx, const T* __restrict__ ty, double tol, double min_support,
                            uint8_t* __restrict__ out, int* __restrict__ nout) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= W) return;
  const size_t N = (size_t)W * H, i = (size_t)y * W + x;
  double S[LAA_M];
#pragma unroll
  for (int m = 0; m < LAA_M; m++) S[m] = 0.0;
  const int q0 = max(0, y - r), q1 = min(H - 1, y + r);
  for (int q = q0; q <= q1; q++) {
    const size_t j = (size_t)q * W + x;
#pragma unroll
    for (int m = 0; m < LAA_M; m++) S[m] += rows[m * N + j];
  }
  const double xd = x, yd = y, s1 = S[0];
  const bool okfit = s1 >= 3.0;
  double a0 = nan(""), a1 = nan("");
  if (okfit) {
    const double sxc = S[1] - xd * s1, syc = S[2] - yd * s1;
    const double sxxc = S[3] - 2.0 * xd * S[1] + xd * xd * s1;
    const double sxyc = S[4] - xd * S[2] - yd * S[1] + xd * yd * s1;
    const double syyc = S[5] - 2.0 * yd * S[2] + yd * yd * s1;
    double a[3][5] = {{s1, sxc, syc, S[6], S[9]},
                      {sxc, sxxc + ridge * s1, sxyc, S[7] - xd * S[6], S[10] - xd * S[9]},
                      {syc, sxyc, syyc + ridge * s1, S[8] - yd * S[6], S[11] - yd * S[9]}};
    double c[3][2];
    if (solve3x2(a, c)) {
      a0 = c[0][0];
      a1 = c[0][1];
    }
  }
  if (pass == 0) {
    out[i] = (support[i] && hypot((double)ux[i] - a0, (double)uy[i] - a1) <= 3.0 * tol) ? 1 : 0;
  } else {
    out[i] = (s1 + 0.5 >= min_support && okfit && hypot((double)tx[i] - a0, (double)ty[i] - a1) <= tol) ? 1 : 0;
    if (nout) nout[i] = (int)rint(s1);
  }
}

// ---------------------------------------------------------------- frame front-end (to_gray + downscale)
// io.rs:44-52 (luminance, lut8), io.rs:258-281 (downscale), video.rs:290-300 (rgb_to_gray); every product and sum
// rounded on its own (no contraction), as the CLI evaluates them

__device__ __forceinline__ double luminance64(double r, double g, double b) {
  return __dadd_rn(__dadd_rn(__dmul_rn(0.299, r), __dmul_rn(0.587, g)), __dmul_rn(0.114, b));
}

template <int PIX>
__device__ __forceinline__ double grey_at(const uint8_t* __restrict__ px, size_t i, const double* __restrict__ lut8) {
  if (PIX == OFC_PIX_F32) return (double)reinterpret_cast<const float*>(px)[i];
  if (PIX == OFC_PIX_GRAY8) return lut8[px[i]];
  if (PIX == OFC_PIX_GRAY16) return __ddiv_rn((double)reinterpret_cast<const uint16_t*>(px)[i], 65535.0);
  if (PIX == OFC_PIX_RGB24) return luminance64(lut8[px[3 * i]], lut8[px[3 * i + 1]], lut8[px[3 * i + 2]]);
  if (PIX == OFC_PIX_RGBA32) return luminance64(lut8[px[4 * i]], lut8[px[4 * i + 1]], lut8[px[4 * i + 2]]);
  const uint16_t* q = reinterpret_cast<const uint16_t*>(px) + 3 * i;  // OFC_PIX_RGB48
  return luminance64(__ddiv_rn((double)q[0], 65535.0), __ddiv_rn((double)q[1], 65535.0),
                     __ddiv_rn((double)q[2], 65535.0));
}

// one output pixel per thread: the scale x scale block's rows summed left to right, the row sums in order,
// / scale^2, rounded to float32 (scale 1: the grey level itself)
template <int PIX>
__global__ void k_to_gray(const uint8_t* __restrict__ px, int w_in, int scale, int W, int H,
                          const double* __restrict__ lut8, float* __restrict__ out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= W) return;
  double sum = 0.0;
  for (int dy = 0; dy < scale; dy++) {
    const size_t row = (size_t)(y * scale + dy) * w_in + (size_t)x * scale;
    double rs = 0.0;
    for (int dx = 0; dx < scale; dx++) rs = __dadd_rn(rs, grey_at<PIX>(px, row + dx, lut8));
    sum = __dadd_rn(sum, rs);
  }
  out[(size_t)y * W + x] = (float)__ddiv_rn(sum, (double)scale * (double)scale);
}

// low = conf < conf_min (track.py:66) for ofc_finish
__global__ void k_threshold_low(const double* c64, double cm, uint8_t* low, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    low[i] = c64[i] < cm ? 1 : 0;
}
void ofc_threshold_low(const double* c64, double cm, uint8_t* low, size_t n, cudaStream_t st) {
  OFC_LAUNCH(k_threshold_low, std::min<size_t>(div_up(n, 256), 4096), 256, 0, st, c64, cm, low, n);
}

void cfg_check(const ofc_config* c) {
  if (!c) throw Error(OFC_ERR_ARG, "null config");
  std::string m = validate(*c);
  if (!m.empty()) throw Error(OFC_ERR_ARG, m);
}

// Config.validate for the hybrid keys (config.py:195-200), the reference's messages
void hybrid_check(const ofc_hybrid* hy) {
  if (!hy) throw Error(OFC_ERR_ARG, "null hybrid keys");
  if (hy->fb_max < 0) throw Error(OFC_ERR_ARG, "fb_max must be >= 0");
  if (!std::isfinite(hy->fb_radius) || !std::isfinite(hy->fb_tol) || hy->fb_tol <= 0 || hy->fb_radius == 0)
    throw Error(OFC_ERR_ARG, "fb_radius must be finite and nonzero (negative: 4 sigma_w), fb_tol finite and positive");
  if (hy->fb_min_support < 0) throw Error(OFC_ERR_ARG, "fb_min_support must be >= 0 and tavg in [0, 64]");
}

// bytes per pixel of an OFC_PIX_* format; 0 for an unknown one
size_t pixel_bytes(int32_t pixel) {
  switch (pixel) {
    case OFC_PIX_F32: return 4;
    case OFC_PIX_GRAY8: return 1;
    case OFC_PIX_GRAY16: return 2;
    case OFC_PIX_RGB24: return 3;
    case OFC_PIX_RGBA32: return 4;
    case OFC_PIX_RGB48: return 6;
    default: return 0;
  }
}

// to_gray + downscale of a device image of w_in x (H * scale) or more rows into the W x H float32 plane out
void to_gray_dev(Lane& L, const uint8_t* px, int32_t pixel, int w_in, int scale, int W, int H, float* out) {
  const double* lut8 = nullptr;
  if (L.has_const("lut8")) {
    lut8 = L.cached<double>("lut8", nullptr, 256);
  } else {
    double lut[256];
    for (int v = 0; v < 256; v++) lut[v] = v / 255.0;  // lut8 (io.rs:50-52)
    lut8 = L.cached("lut8", lut, 256);
  }
  const dim3 g(div_up(W, 128), H);
  cudaStream_t st = L.stream;
  switch (pixel) {
    case OFC_PIX_F32: OFC_LAUNCH(k_to_gray<OFC_PIX_F32>, g, 128, 0, st, px, w_in, scale, W, H, lut8, out); break;
    case OFC_PIX_GRAY8: OFC_LAUNCH(k_to_gray<OFC_PIX_GRAY8>, g, 128, 0, st, px, w_in, scale, W, H, lut8, out); break;
    case OFC_PIX_GRAY16: OFC_LAUNCH(k_to_gray<OFC_PIX_GRAY16>, g, 128, 0, st, px, w_in, scale, W, H, lut8, out); break;
    case OFC_PIX_RGB24: OFC_LAUNCH(k_to_gray<OFC_PIX_RGB24>, g, 128, 0, st, px, w_in, scale, W, H, lut8, out); break;
    case OFC_PIX_RGBA32: OFC_LAUNCH(k_to_gray<OFC_PIX_RGBA32>, g, 128, 0, st, px, w_in, scale, W, H, lut8, out); break;
    case OFC_PIX_RGB48: OFC_LAUNCH(k_to_gray<OFC_PIX_RGB48>, g, 128, 0, st, px, w_in, scale, W, H, lut8, out); break;
    default: throw Error(OFC_ERR_ARG, "unknown pixel format " + std::to_string(pixel));
  }
}

// the checks of a frame format: a known pixel, scale >= 1 (io.rs:260), a tracked size of at least one pixel
void check_format(int32_t pixel, size_t w, size_t h, int32_t scale) {
  if (pixel_bytes(pixel) == 0) throw Error(OFC_ERR_ARG, "unknown pixel format " + std::to_string(pixel));
  if (scale < 1) throw Error(OFC_ERR_ARG, "scale must be >= 1, got " + std::to_string(scale));
  check_sizes(w, h);
  check_sizes(w / scale, h / scale);
}

// _local_affine_agreement on device planes (track.py:331-382): two passes of row sums and column sums + solve; the
// half-size r = max(1, round(radius)) (ties to even), the ridge 1e-3 r^2 on B
template <typename T>
void laa_dev(Lane& L, int W, int H, const uint8_t* support, const T* ux, const T* uy, const T* tx, const T* ty,
             double radius, long long min_support, double tol, uint8_t* ok, int* nout) {
  cudaStream_t st = L.stream;
  const size_t N = (size_t)W * H;
  const double rd = std::max(1.0, std::nearbyint(radius));
  const double ridge = 1e-3 * rd * rd;
  const int r = (int)std::min(rd, (double)std::max(W, H));  // a wider window clips to the same sums
  double* rows = L.get<double>("laa_rows", LAA_M * N);
  uint8_t* sel = L.get<uint8_t>("laa_sel", N);
  const dim3 g(div_up(W, 128), H);
  const double ms = (double)min_support;
  OFC_LAUNCH(k_laa_rows<T>, g, 128, 0, st, support, ux, uy, W, H, r, rows);
  OFC_LAUNCH(k_laa_solve<T>, g, 128, 0, st, rows, W, H, r, ridge, 0, support, ux, uy, tx, ty, tol, ms, sel, nullptr);
  OFC_LAUNCH(k_laa_rows<T>, g, 128, 0, st, sel, ux, uy, W, H, r, rows);
  OFC_LAUNCH(k_laa_solve<T>, g, 128, 0, st, rows, W, H, r, ridge, 1, sel, ux, uy, tx, ty, tol, ms, ok, nout);
}

}  // namespace

// synth.cu
namespace ofc {
void synth_render_dev(const SynthBlob* blobs, const int* cell_start, int ncx, int ncy, double cell, int w, int h,
                      int ss, const ofc_field* field, double* out, cudaStream_t st);
}

namespace {
// per blob the reference's subsample rectangle (synth.py:174-179: floor/ceil of (mapped centre -+ (5.2 r + 2) + 0.5)
// * ss, clipped to the image); blobs with an empty rectangle are dropped, the rest binned by the cell of the mapped
// centre (cells 1 px wider than the largest half size, the grid starting one cell before the image) and rendered
// on the device
void launch_synth_render(Lane& L, const double* bx, const double* by, const double* br, const double* ba, size_t n,
                         int w, int h, int ss, const ofc_field* field, double* out) {
  double rmax = 0;
  for (size_t i = 0; i < n; i++) rmax = std::max(rmax, br[i]);
  const double cell = std::ceil(5.2 * rmax + 2.0) + 2.0;
  const long W = (long)w * ss, H = (long)h * ss;
  const int ncx = (int)std::ceil((w + 2 * cell) / cell) + 1, ncy = (int)std::ceil((h + 2 * cell) / cell) + 1;
  std::vector<SynthBlob> kept;
  std::vector<int> cid;
  for (size_t k = 0; k < n; k++) {
    double px = bx[k], py = by[k];
    if (field) field_fwd(*field, bx[k], by[k], px, py);
    double rad = 5.2 * br[k] + 2.0;
    long j0 = std::max((long)std::floor((px - rad + 0.5) * ss), 0L);
    long j1 = std::min((long)std::ceil((px + rad + 0.5) * ss), W);
    long i0 = std::max((long)std::floor((py - rad + 0.5) * ss), 0L);
    long i1 = std::min((long)std::ceil((py + rad + 0.5) * ss), H);
    if (j0 >= j1 || i0 >= i1) continue;
    int cx = std::min(std::max((int)std::floor((px + cell) / cell), 0), ncx - 1);
    int cy = std::min(std::max((int)std::floor((py + cell) / cell), 0), ncy - 1);
    kept.push_back({bx[k], by[k], br[k], ba[k], (int)i0, (int)i1, (int)j0, (int)j1});
    cid.push_back(cy * ncx + cx);
  }
  std::vector<int> cnt((size_t)ncx * ncy + 1, 0);
  for (int c : cid) cnt[c + 1]++;
  for (size_t c = 1; c < cnt.size(); c++) cnt[c] += cnt[c - 1];
  std::vector<SynthBlob> sorted(kept.size());
  std::vector<int> fill(cnt.begin(), cnt.end() - 1);
  for (size_t i = 0; i < kept.size(); i++) sorted[fill[cid[i]]++] = kept[i];
  SynthBlob* db = L.upload("syn_blobs", sorted.data(), std::max<size_t>(sorted.size(), 1));
  int* dc = L.upload("syn_cells", cnt.data(), cnt.size());
  double* dout = L.get<double>("syn_out", (size_t)w * h);
  ofc_field* df = nullptr;
  if (field) {
    // the device copy of the field points at a device copy of its grid coefficients
    ofc_field dev = *field;
    if (field->grid && field->gnx > 0 && field->gny > 0)
      dev.grid = L.upload("syn_grid", field->grid, (size_t)2 * field->gnx * field->gny);
    else
      dev.grid = nullptr;
    df = L.upload("syn_field", &dev, 1);
  }
  synth_render_dev(db, dc, ncx, ncy, cell, w, h, ss, df, dout, L.stream);
  OFC_CUDA(cudaMemcpyAsync(out, dout, (size_t)w * h * sizeof(double), cudaMemcpyDeviceToHost, L.stream));
  OFC_CUDA(cudaStreamSynchronize(L.stream));
}
}  // namespace

// ================================================================= C ABI
extern "C" {

int ofc_abi_version(void) { return OFC_ABI_VERSION; }

void ofc_config_default(ofc_config* c) {
  std::memset(c, 0, sizeof(*c));
  c->grid_step = 16;
  c->poc_win = 64;
  c->max_disp = 32.0;
  c->poc_peak_min = 0.1;
  c->median_thresh = 2.0;
  c->lam = 8.0;
  c->n_scales = 3;
  c->scales[0] = 0.6;
  c->scales[1] = 1.0;
  c->scales[2] = 1.6;
  c->n_orient = 4;
  c->bandwidth = 0.5;
  c->dc_cut = 2.0;
  c->sigma_w = 4.0;
  c->shape_order = 1;
  c->sigma_s = 4.0;
  c->outer_iters = 8;
  c->inner_iters = 2;
  c->conf_min = 0.2;
  c->edge_guard = -1.0;
  c->edge_guard_min_area = -1.0;
  c->phase_tol = 0.4;
  c->strain_win = 15;
  c->prewarp_freeze_at = 0;
}

int ofc_config_validate(const ofc_config* c, char* err, size_t errlen) {
  if (!c) { set_err(err, errlen, "null config"); return OFC_ERR_ARG; }
  std::string m = validate(*c);
  if (m.empty()) return OFC_OK;
  set_err(err, errlen, m);
  return OFC_ERR_ARG;
}

double ofc_edge_guard_px(const ofc_config* c) { return guard_px(*c); }
double ofc_auto_edge_guard_px(const ofc_config* c) { return auto_guard(*c); }
double ofc_edge_guard_min_area_px(const ofc_config* c) { return min_area_px(*c); }

ofc_engine* ofc_create(int device, int lanes, char* err, size_t errlen) {
  try {
    if (lanes < 1 || lanes > 2) throw Error(OFC_ERR_ARG, "lanes must be 1 or 2");
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0)
      throw Error(OFC_ERR_DEVICE, std::string("no CUDA device: ") + (e != cudaSuccess ? cudaGetErrorString(e) : "0 devices"));
    if (device < 0 || device >= n) throw Error(OFC_ERR_DEVICE, "CUDA device " + std::to_string(device) + " does not exist");
    OFC_CUDA(cudaSetDevice(device));
    cudaDeviceProp prop;
    OFC_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10) throw Error(OFC_ERR_DEVICE, std::string("the engine is built for sm_100a; device is ") + prop.name);
    std::unique_ptr<ofc_engine> eng(new ofc_engine());
    eng->device = device;
    eng->nlanes = lanes;
    for (int i = 0; i < lanes; i++) {
      std::unique_ptr<Lane> l(new Lane());
      lane_init(*l);
      eng->lanes.push_back(std::move(l));
    }
    return eng.release();
  } catch (const Error& x) {
    set_err(err, errlen, x.what());
    return nullptr;
  }
}

void ofc_destroy(ofc_engine* e) {
  if (!e) return;
  cudaSetDevice(e->device);
  for (auto& l : e->lanes) {
    std::lock_guard<std::mutex> lk(l->busy);
    lane_destroy(*l);
  }
  delete e;
}

int ofc_lanes(const ofc_engine* e) { return e ? e->nlanes : 0; }

uint64_t ofc_kernel_launches(const ofc_engine* e) { return e ? e->launches : 0; }

int ofc_check_window(ofc_engine* e, size_t w, size_t h, const ofc_config* c, char* err, size_t errlen) {
  return guarded(e, err, errlen, [&](Lane&) {
    cfg_check(c);
    check_fine_window(w, h, *c);
    // device memory of the fine stage of one window (bytes per padded / window pixel, see the buffers of refine_dev)
    size_t N = w * h, Np = (w + 2 * PAD) * (h + 2 * PAD);
    int F = c->n_scales * c->n_orient;
    size_t need = Np * 8 * (1 + 3 * F + F) + N * (20 * F + 8 * 60 + 4 * 8);
    size_t fre = 0, tot = 0;
    OFC_CUDA(cudaMemGetInfo(&fre, &tot));
    if (need > tot * 9 / 10)
      throw Error(OFC_ERR_WINDOW, "window " + std::to_string(w) + "x" + std::to_string(h) + " needs " +
                                      std::to_string(need >> 20) + " MiB of device memory");
  });
}

void ofc_release_caches(ofc_engine* e) {
  if (!e) return;
  cudaSetDevice(e->device);
  for (auto& l : e->lanes) {
    std::lock_guard<std::mutex> lk(l->busy);
    lane_sync(*l);
    l->release();
  }
}

int ofc_refine_raw(ofc_engine* e, const float* i1, size_t w, size_t h, const float* i2, size_t w2, size_t h2,
                   int64_t shift_x, int64_t shift_y, const float* ux, const float* uy, const ofc_config* c,
                   double* out_ux, double* out_uy, double* out_energy, double* out_resid, char* err, size_t errlen) {
  return guarded(e, err, errlen, [&](Lane& L) {
    cfg_check(c);
    check_fine_window(w, h, *c);
    check_sizes(w2, h2);
    if (!i1 || !i2 || !ux || !uy) throw Error(OFC_ERR_ARG, "null input");
    const size_t N = w * h;
    cudaStream_t st = L.stream;
    float* d1 = L.upload("in_i1", i1, N);
    float* d2 = L.upload("in_i2", i2, w2 * h2);
    float* du = L.upload("in_u", ux, N);
    float* dv = L.upload("in_v", uy, N);
    double* u2 = L.get<double>("u2", 2 * N);
    launch_f32_to_f64(du, u2, N, st);
    launch_f32_to_f64(dv, u2 + N, N, st);
    FineOut f = refine_dev(L, d1, (int)w, (int)h, d2, (int)w2, (int)h2, (long)shift_x, (long)shift_y, u2, *c, false);
    if (out_ux) OFC_CUDA(cudaMemcpyAsync(out_ux, f.ux, N * 8, cudaMemcpyDeviceToHost, st));
    if (out_uy) OFC_CUDA(cudaMemcpyAsync(out_uy, f.uy, N * 8, cudaMemcpyDeviceToHost, st));
    if (out_energy) OFC_CUDA(cudaMemcpyAsync(out_energy, f.energy, N * 8, cudaMemcpyDeviceToHost, st));
    if (out_resid) OFC_CUDA(cudaMemcpyAsync(out_resid, f.resid, N * 8, cudaMemcpyDeviceToHost, st));
    OFC_CUDA(cudaStreamSynchronize(st));
  });
}

int ofc_refine_batch(ofc_engine* e, const ofc_window* wins, size_t n, const ofc_config* c, char* err, size_t errlen) {
  return guarded(e, err, errlen, [&](Lane& L) {
    cfg_check(c);
    if (n == 0) return;
    if (!wins) throw Error(OFC_ERR_ARG, "null window list");
    size_t maxN = 0, max2 = 0;
    for (size_t k = 0; k < n; k++) {
      const ofc_window& w = wins[k];
      try {
        check_fine_window(w.w, w.h, *c);
        check_sizes(w.w2, w.h2);
        if (!w.i1 || !w.i2 || !w.ux || !w.uy) throw Error(OFC_ERR_ARG, "null input");
      } catch (const Error& x) {
        throw Error(x.status, "window " + std::to_string(k) + ": " + x.what());
      }
      maxN = std::max(maxN, w.w * w.h);
      max2 = std::max(max2, w.w2 * w.h2);
    }
    L.ensure_copy_stream();
    cudaStream_t st = L.stream, cs = L.copy;
    cudaEvent_t* in_ready = L.bev;       // inputs of set s uploaded
    cudaEvent_t* in_free = L.bev + 2;    // the refine that read set s is done
    cudaEvent_t* out_ready = L.bev + 4;  // outputs staged in staging set s
    cudaEvent_t* out_done = L.bev + 6;   // staging set s downloaded
    // two input sets and two output staging sets, sized for the largest window before any work is queued
    float *in1[2], *in2[2], *inu[2], *inv[2];
    double* stage[2];
    for (int s2 = 0; s2 < 2; s2++) {
      const std::string t = std::to_string(s2);
      in1[s2] = L.get<float>("batch_i1_" + t, maxN);
      in2[s2] = L.get<float>("batch_i2_" + t, max2);
      inu[s2] = L.get<float>("batch_u_" + t, maxN);
      inv[s2] = L.get<float>("batch_v_" + t, maxN);
      stage[s2] = L.get<double>("batch_out_" + t, 4 * maxN);
    }
    double* u2 = L.get<double>("u2", 2 * maxN);
    auto upload = [&](size_t k, int s2) {
      const ofc_window& w = wins[k];
      const size_t N = w.w * w.h;
      OFC_CUDA(cudaMemcpyAsync(in1[s2], w.i1, N * 4, cudaMemcpyHostToDevice, cs));
      OFC_CUDA(cudaMemcpyAsync(in2[s2], w.i2, w.w2 * w.h2 * 4, cudaMemcpyHostToDevice, cs));
      OFC_CUDA(cudaMemcpyAsync(inu[s2], w.ux, N * 4, cudaMemcpyHostToDevice, cs));
      OFC_CUDA(cudaMemcpyAsync(inv[s2], w.uy, N * 4, cudaMemcpyHostToDevice, cs));
      OFC_CUDA(cudaEventRecord(in_ready[s2], cs));
    };
    auto download = [&](size_t k) {
      const int s2 = (int)(k & 1);
      const ofc_window& w = wins[k];
      const size_t N = w.w * w.h;
      OFC_CUDA(cudaStreamWaitEvent(cs, out_ready[s2], 0));
      double* outs[4] = {w.out_ux, w.out_uy, w.out_energy, w.out_resid};
      for (int q = 0; q < 4; q++)
        if (outs[q]) OFC_CUDA(cudaMemcpyAsync(outs[q], stage[s2] + q * N, N * 8, cudaMemcpyDeviceToHost, cs));
      OFC_CUDA(cudaEventRecord(out_done[s2], cs));
    };
    // copy stream: upload k + 1 while k computes, download k - 1 after k is queued (so that a pageable download,
    // which holds the host until it is done, leaves the compute stream with work). On an error both streams are
    // drained before the call returns, so no copy into the caller's buffers outlives it.
    struct Drain {
      cudaStream_t a, b;
      ~Drain() {
        cudaStreamSynchronize(a);
        cudaStreamSynchronize(b);
      }
    } drain{cs, st};
    upload(0, 0);
    for (size_t k = 0; k < n; k++) {
      const int s2 = (int)(k & 1);
      const ofc_window& w = wins[k];
      const size_t N = w.w * w.h;
      OFC_CUDA(cudaStreamWaitEvent(st, in_ready[s2], 0));
      launch_f32_to_f64(inu[s2], u2, N, st);
      launch_f32_to_f64(inv[s2], u2 + N, N, st);
      FineOut f = refine_dev(L, in1[s2], (int)w.w, (int)w.h, in2[s2], (int)w.w2, (int)w.h2, (long)w.shift_x,
                             (long)w.shift_y, u2, *c, false);
      OFC_CUDA(cudaEventRecord(in_free[s2], st));
      if (k >= 2) OFC_CUDA(cudaStreamWaitEvent(st, out_done[s2], 0));  // staging set s2 held window k - 2
      const double* res[4] = {f.ux, f.uy, f.energy, f.resid};
      for (int q = 0; q < 4; q++)
        OFC_CUDA(cudaMemcpyAsync(stage[s2] + q * N, res[q], N * 8, cudaMemcpyDeviceToDevice, st));
      OFC_CUDA(cudaEventRecord(out_ready[s2], st));
      if (k + 1 < n) {
        if (k >= 1) OFC_CUDA(cudaStreamWaitEvent(cs, in_free[s2 ^ 1], 0));  // window k - 1 read set s2 ^ 1
        upload(k + 1, s2 ^ 1);
      }
      if (k >= 1) download(k - 1);
    }
    download(n - 1);
    OFC_CUDA(cudaStreamSynchronize(cs));
    OFC_CUDA(cudaStreamSynchronize(st));
  });
}

int ofc_refine(ofc_engine* e, const float* i1, const float* i2, size_t w, size_t h, const float* ux, const float* uy,
               const ofc_config* c, float* out_ux, float* out_uy, float* out_conf, float* out_resid, uint8_t* out_low,
               char* err, size_t errlen) {
  return guarded(e, err, errlen, [&](Lane& L) {
    cfg_check(c);
    check_fine_window(w, h, *c);
    if (!i1 || !i2 || !ux || !uy) throw Error(OFC_ERR_ARG, "null input");
    const size_t N = w * h;
    cudaStream_t st = L.stream;
    float* d1 = L.upload("in_i1", i1, N);
    float* d2 = L.upload("in_i2", i2, N);
    float* du = L.upload("in_u", ux, N);
    float* dv = L.upload("in_v", uy, N);
    double* u2 = L.get<double>("u2", 2 * N);
    launch_f32_to_f64(du, u2, N, st);
    launch_f32_to_f64(dv, u2 + N, N, st);
    FineOut f = refine_dev(L, d1, (int)w, (int)h, d2, (int)w, (int)h, 0, 0, u2, *c, false);
    float* conf = L.get<float>("out_conf", N);
    uint8_t* low = L.get<uint8_t>("low_final", N);
    double B = guard_px(*c) > 0 ? 4.0 * c->sigma_w : 0.0;
    launch_confidence(f.energy, f.resid, f.ux, f.uy, (int)w, (int)h, f.stats, c->phase_tol, c->conf_min, true, B, conf,
                      nullptr, low, nullptr, st);
    float* o32 = L.get<float>("out_f32", 3 * N);
    launch_f64_to_f32(f.ux, o32, N, st);
    launch_f64_to_f32(f.uy, o32 + N, N, st);
    launch_f64_to_f32(f.resid, o32 + 2 * N, N, st);
    if (out_ux) OFC_CUDA(cudaMemcpyAsync(out_ux, o32, N * 4, cudaMemcpyDeviceToHost, st));
    if (out_uy) OFC_CUDA(cudaMemcpyAsync(out_uy, o32 + N, N * 4, cudaMemcpyDeviceToHost, st));
    if (out_resid) OFC_CUDA(cudaMemcpyAsync(out_resid, o32 + 2 * N, N * 4, cudaMemcpyDeviceToHost, st));
    if (out_conf) OFC_CUDA(cudaMemcpyAsync(out_conf, conf, N * 4, cudaMemcpyDeviceToHost, st));
    if (out_low) OFC_CUDA(cudaMemcpyAsync(out_low, low, N, cudaMemcpyDeviceToHost, st));
    OFC_CUDA(cudaStreamSynchronize(st));
  });
}

int ofc_grid_shape(size_t w, size_t h, const ofc_config* c, size_t* nx, size_t* ny) {
  if (!c || !nx || !ny) return OFC_ERR_ARG;
  std::vector<int> xs = arange(c->poc_win / 2, (int)w - c->poc_win / 2 + 1, c->grid_step);
  std::vector<int> ys = arange(c->poc_win / 2, (int)h - c->poc_win / 2 + 1, c->grid_step);
  *nx = xs.size();
  *ny = ys.size();
  return (xs.empty() || ys.empty()) ? OFC_ERR_ARG : OFC_OK;
}

int ofc_coarse_flow(ofc_engine* e, const float* a, const float* b, size_t w, size_t h, const float* init_ux,
                    const float* init_uy, const ofc_config* c, int32_t* xs, int32_t* ys, float* gux, float* guy,
                    float* gpeak, char* err, size_t errlen) {
  return guarded(e, err, errlen, [&](Lane& L) {
    cfg_check(c);
    check_sizes(w, h);
    if (!a || !b) throw Error(OFC_ERR_ARG, "null input");
    if ((init_ux == nullptr) != (init_uy == nullptr)) throw Error(OFC_ERR_ARG, "init_ux and init_uy must both be given");
    const size_t N = w * h;
    cudaStream_t st = L.stream;
    float* da = L.upload("in_i1", a, N);
    float* db = L.upload("in_i2", b, N);
    double* init = nullptr;
    if (init_ux) {
      float* du = L.upload("in_u", init_ux, N);
      float* dv = L.upload("in_v", init_uy, N);
      init = L.get<double>("init2", 2 * N);
      launch_f32_to_f64(du, init, N, st);
      launch_f32_to_f64(dv, init + N, N, st);
    }
    CoarseOut g = coarse_dev(L, da, db, (int)w, (int)h, init, *c);
    size_t n = (size_t)g.nx * g.ny;
    float* o = L.get<float>("out_f32", 3 * n);
    launch_f64_to_f32(g.ux, o, n, st);
    launch_f64_to_f32(g.uy, o + n, n, st);
    launch_f64_to_f32(g.peak, o + 2 * n, n, st);
    if (gux) OFC_CUDA(cudaMemcpyAsync(gux, o, n * 4, cudaMemcpyDeviceToHost, st));
    if (guy) OFC_CUDA(cudaMemcpyAsync(guy, o + n, n * 4, cudaMemcpyDeviceToHost, st));
    if (gpeak) OFC_CUDA(cudaMemcpyAsync(gpeak, o + 2 * n, n * 4, cudaMemcpyDeviceToHost, st));
    OFC_CUDA(cudaStreamSynchronize(st));
    if (xs) std::copy(g.hxs.begin(), g.hxs.end(), xs);
    if (ys) std::copy(g.hys.begin(), g.hys.end(), ys);
  });
}

int ofc_strain(ofc_engine* e, const float* ux, const float* uy, size_t w, size_t h, int32_t win, float* dudx,
               float* dudy, float* dvdx, float* dvdy, float* exx, float* eyy, float* exy, float* gmax, float* vol,
               char* err, size_t errlen) {
  return guarded(e, err, errlen, [&](Lane& L) {
    check_sizes(w, h);
    if (win < 1 || win > 255) throw Error(OFC_ERR_ARG, "strain window must lie in [1, 255]");
    const size_t N = w * h;
    cudaStream_t st = L.stream;
    float* du = L.upload("in_u", ux, N);
    float* dv = L.upload("in_v", uy, N);
    double* m2 = L.get<double>("fin_mx", 2 * N);
    launch_f32_to_f64(du, m2, N, st);
    launch_f32_to_f64(dv, m2 + N, N, st);
    double* yp = L.get<double>("strain_y", 11 * N);
    float* o = L.get<float>("out_f32", 9 * N);
    launch_strain(m2, m2 + N, (int)w, (int)h, win, yp, o, o + N, o + 2 * N, o + 3 * N, o + 4 * N, o + 5 * N, o + 6 * N,
                  o + 7 * N, o + 8 * N, st);
    float* outs[9] = {dudx, dudy, dvdx, dvdy, exx, eyy, exy, gmax, vol};
    for (int i = 0; i < 9; i++)
      if (outs[i]) OFC_CUDA(cudaMemcpyAsync(outs[i], o + i * N, N * 4, cudaMemcpyDeviceToHost, st));
    OFC_CUDA(cudaStreamSynchronize(st));
  });
}

// the host planes of a staged frame into the caller's (each pointer nullable) and the timing
static void copy_pair_out(const ofc_pair_out& s, ofc_pair_out* d, size_t N) {
  float* const* src[10] = {&s.ux, &s.uy, &s.conf, &s.exx, &s.eyy, &s.exy, &s.gmax, &s.vol, &s.raw_ux, &s.raw_uy};
  float** dst[10] = {&d->ux, &d->uy, &d->conf, &d->exx, &d->eyy, &d->exy, &d->gmax, &d->vol, &d->raw_ux, &d->raw_uy};
  for (int i = 0; i < 10; i++)
    if (*dst[i]) std::memcpy(*dst[i], *src[i], N * 4);
  if (d->valid) std::memcpy(d->valid, s.valid, N);
  for (int i = 0; i < 3; i++) d->timing[i] = s.timing[i];
}

static void download_pair(Lane& L, const ofc_pair_out& d, ofc_pair_out* h, size_t N) {
  cudaStream_t st = L.stream;
  float* const* dsrc[10] = {&d.ux, &d.uy, &d.conf, &d.exx, &d.eyy, &d.exy, &d.gmax, &d.vol, &d.raw_ux, &d.raw_uy};
  float** hdst[10] = {&h->ux, &h->uy, &h->conf, &h->exx, &h->eyy, &h->exy, &h->gmax, &h->vol, &h->raw_ux, &h->raw_uy};
  for (int i = 0; i < 10; i++)
    if (*hdst[i]) OFC_CUDA(cudaMemcpyAsync(*hdst[i], *dsrc[i], N * 4, cudaMemcpyDeviceToHost, st));
  if (h->valid) OFC_CUDA(cudaMemcpyAsync(h->valid, d.valid, N, cudaMemcpyDeviceToHost, st));
}

static ofc_pair_out device_pair_out(Lane& L, size_t N) {
  ofc_pair_out d{};
  float* p = L.get<float>("out_pair", 10 * N);
  float** f[10] = {&d.ux, &d.uy, &d.conf, &d.exx, &d.eyy, &d.exy, &d.gmax, &d.vol, &d.raw_ux, &d.raw_uy};
  for (int i = 0; i < 10; i++) *f[i] = p + i * N;
  d.valid = L.get<uint8_t>("out_valid", N);
  return d;
}

int ofc_finish(ofc_engine* e, const float* ux, const float* uy, const float* conf, const uint8_t* roi, size_t w,
               size_t h, const ofc_config* c, ofc_pair_out* out, char* err, size_t errlen) {
  return guarded(e, err, errlen, [&](Lane& L) {
    cfg_check(c);
    check_sizes(w, h);
    if (!ux || !uy || !conf || !out) throw Error(OFC_ERR_ARG, "null argument");
    const size_t N = w * h;
    cudaStream_t st = L.stream;
    float* du = L.upload("in_u", ux, N);
    float* dv = L.upload("in_v", uy, N);
    float* dc = L.upload("in_conf", conf, N);
    const uint8_t* droi = roi ? L.upload("in_roi", roi, N) : nullptr;
    double* u2 = L.get<double>("u2", 2 * N);
    double* c64 = L.get<double>("conf64", N);
    launch_f32_to_f64(du, u2, N, st);
    launch_f32_to_f64(dv, u2 + N, N, st);
    launch_f32_to_f64(dc, c64, N, st);
    // low = conf < conf_min on the given confidence (track.py:66)
    uint8_t* low = L.get<uint8_t>("low_final", N);
    ofc_threshold_low(c64, c->conf_min, low, N, st);
    ofc_pair_out d = device_pair_out(L, N);
    finish_dev(L, low, droi, u2, u2 + N, c64, (int)w, (int)h, *c, d, false);
    download_pair(L, d, out, N);
    OFC_CUDA(cudaStreamSynchronize(st));
    std::memset(out->timing, 0, sizeof(out->timing));
  });
}

int ofc_track_pairs(ofc_engine* e, const ofc_pair_in* pairs, size_t n, const ofc_config* c, ofc_pair_out* outs,
                    char* err, size_t errlen) {
  return guarded(e, err, errlen, [&](Lane& L) {
    cfg_check(c);
    if (n == 0) return;
    if (!pairs || !outs) throw Error(OFC_ERR_ARG, "null argument");
    for (size_t i = 0; i < n; i++) {
      const ofc_pair_in& p = pairs[i];
      const std::string at = "pair " + std::to_string(i) + ": ";
      if (!p.i1 || !p.i2) throw Error(OFC_ERR_ARG, at + "null image");
      if ((p.init_ux == nullptr) != (p.init_uy == nullptr))
        throw Error(OFC_ERR_ARG, at + "init_ux and init_uy must both be given");
      try {
        check_fine_window(p.w, p.h, *c);
      } catch (const Error& x) {
        throw Error(x.status, at + x.what());
      }
      if ((int)std::min(p.w, p.h) < c->poc_win)
        throw Error(OFC_ERR_ARG, at + "image smaller than poc_win (" + std::to_string(c->poc_win) + ")");
    }
    // the largest padded windows first, so that a worker's buffers are sized once
    std::vector<size_t> order(n);
    for (size_t i = 0; i < n; i++) order[i] = i;
    auto padded = [&](size_t i) { return (pairs[i].w + 2 * PAD) * (pairs[i].h + 2 * PAD); };
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return padded(a) > padded(b); });
    // worker lanes: 8 (config 3's 64 uneven pairs: 4 lanes 79, 8 lanes 92, 16 lanes 95 M pixel-pairs/s, 8 lanes holding
    // 31 GB of device memory), or OFC_PAIR_WORKERS (1 to 16) from the environment
    int workers = 8;
    if (const char* ev = std::getenv("OFC_PAIR_WORKERS")) workers = std::min(std::max(std::atoi(ev), 1), 16);
    const int K = (int)std::min<size_t>(n, (size_t)workers);
    while ((int)L.aux.size() < K) {
      std::unique_ptr<Lane> a(new Lane());
      lane_init(*a);
      L.aux.push_back(std::move(a));
    }
    for (auto& a : L.aux) a->proposal = L.proposal;
    // one pair on worker lane j: inputs up, the pair, its planes down through page-locked staging into the caller's
    // buffers
    auto one_pair = [&](int j, size_t i) {
      Lane& A = *L.aux[j];
      const ofc_pair_in& p = pairs[i];
      const size_t N = p.w * p.h;
      A.upload("in_i1", p.i1, N);
      A.upload("in_i2", p.i2, N);
      if (p.roi) A.upload("in_roi", p.roi, N);
      if (p.init_ux) {
        A.upload("in_u", p.init_ux, N);
        A.upload("in_v", p.init_uy, N);
      }
      run_pair(A, (int)p.w, (int)p.h, p.roi != nullptr, p.init_ux != nullptr, *c, true, 3);
      const ofc_pair_out d = device_pair_out(A, N);
      float* hout = A.pinned<float>("batch_hout", 10 * N);
      uint8_t* hvalid = A.pinned<uint8_t>("batch_hvalid", N);
      OFC_CUDA(cudaMemcpyAsync(hout, d.ux, 10 * N * 4, cudaMemcpyDeviceToHost, A.stream));
      OFC_CUDA(cudaMemcpyAsync(hvalid, d.valid, N, cudaMemcpyDeviceToHost, A.stream));
      OFC_CUDA(cudaStreamSynchronize(A.stream));
      ofc_pair_out o{};
      float** f[10] = {&o.ux, &o.uy, &o.conf, &o.exx, &o.eyy, &o.exy, &o.gmax, &o.vol, &o.raw_ux, &o.raw_uy};
      for (int q = 0; q < 10; q++) *f[q] = hout + q * N;
      o.valid = hvalid;
      pair_timing(A, o.timing);
      copy_pair_out(o, &outs[i], N);
    };
    // A host thread per worker lane, lane j taking pairs j, j + K, j + 2K, ... of the size order (the assignment of
    // the one-thread form, so a lane meets the same sizes, and replays the same graphs, on every call with the same
    // pairs): the uploads from the caller's memory and the copies back into it run side by side instead of in turn
    // between the lanes' pairs. Profile mode (one list of event pairs, filled while a graph is captured) keeps one
    // host thread.
    if (K > 1 && !g_profiler) {
      std::atomic<bool> stop{false};
      std::mutex emu;
      int est = OFC_OK;
      std::string emsg;
      std::vector<uint64_t> launched(K, 0);
      const int dev = e->device;
      auto work = [&](int j) {
        g_launch_counter = &launched[j];
        g_profiler = nullptr;
        try {
          OFC_CUDA(cudaSetDevice(dev));
          for (size_t q = (size_t)j; q < n && !stop.load(); q += (size_t)K) one_pair(j, order[q]);
        } catch (const Error& x) {
          std::lock_guard<std::mutex> lk(emu);
          if (est == OFC_OK) {
            est = x.status;
            emsg = x.what();
          }
          stop = true;
        } catch (const std::exception& x) {
          std::lock_guard<std::mutex> lk(emu);
          if (est == OFC_OK) {
            est = OFC_ERR_DEVICE;
            emsg = x.what();
          }
          stop = true;
        }
        g_launch_counter = nullptr;
      };
      std::vector<std::thread> threads;
      for (int j = 0; j < K; j++) threads.emplace_back(work, j);
      for (auto& t : threads) t.join();
      if (g_launch_counter)
        for (uint64_t v : launched) *g_launch_counter += v;
      if (est != OFC_OK) throw Error(est, emsg);
      return;
    }
    std::vector<long long> busy(K, -1);
    // a worker's finished pair: its planes from page-locked staging into the caller's buffers
    auto drain = [&](int j) {
      if (busy[j] < 0) return;
      Lane& A = *L.aux[j];
      const size_t i = (size_t)busy[j], N = pairs[i].w * pairs[i].h;
      busy[j] = -1;
      OFC_CUDA(cudaStreamSynchronize(A.stream));
      float* hout = A.pinned<float>("batch_hout", 10 * N);
      ofc_pair_out o{};
      float** f[10] = {&o.ux, &o.uy, &o.conf, &o.exx, &o.eyy, &o.exy, &o.gmax, &o.vol, &o.raw_ux, &o.raw_uy};
      for (int q = 0; q < 10; q++) *f[q] = hout + q * N;
      o.valid = A.pinned<uint8_t>("batch_hvalid", N);
      pair_timing(A, o.timing);
      copy_pair_out(o, &outs[i], N);
    };
    for (size_t q = 0; q < n; q++) {
      const size_t i = order[q];
      const int j = (int)(q % K);
      drain(j);
      Lane& A = *L.aux[j];
      const ofc_pair_in& p = pairs[i];
      const size_t N = p.w * p.h;
      A.upload("in_i1", p.i1, N);
      A.upload("in_i2", p.i2, N);
      if (p.roi) A.upload("in_roi", p.roi, N);
      if (p.init_ux) {
        A.upload("in_u", p.init_ux, N);
        A.upload("in_v", p.init_uy, N);
      }
      run_pair(A, (int)p.w, (int)p.h, p.roi != nullptr, p.init_ux != nullptr, *c, true, 3);
      const ofc_pair_out d = device_pair_out(A, N);
      float* hout = A.pinned<float>("batch_hout", 10 * N);
      uint8_t* hvalid = A.pinned<uint8_t>("batch_hvalid", N);
      OFC_CUDA(cudaMemcpyAsync(hout, d.ux, 10 * N * 4, cudaMemcpyDeviceToHost, A.stream));
      OFC_CUDA(cudaMemcpyAsync(hvalid, d.valid, N, cudaMemcpyDeviceToHost, A.stream));
      busy[j] = (long long)i;
    }
    for (int j = 0; j < K; j++) drain(j);
  });
}

int ofc_track_pair(ofc_engine* e, const float* i1, const float* i2, size_t w, size_t h, const uint8_t* roi,
                   const float* init_ux, const float* init_uy, const ofc_config* c, ofc_pair_out* out, char* err,
                   size_t errlen) {
  return guarded(e, err, errlen, [&](Lane& L) {
    cfg_check(c);
    check_fine_window(w, h, *c);
    if (!i1 || !i2 || !out) throw Error(OFC_ERR_ARG, "null argument");
    if ((init_ux == nullptr) != (init_uy == nullptr)) throw Error(OFC_ERR_ARG, "init_ux and init_uy must both be given");
    if ((int)std::min(w, h) < c->poc_win)
      throw Error(OFC_ERR_ARG, "image smaller than poc_win (" + std::to_string(c->poc_win) + ")");
    const size_t N = w * h;
    L.upload("in_i1", i1, N);
    L.upload("in_i2", i2, N);
    if (roi) L.upload("in_roi", roi, N);
    if (init_ux) {
      L.upload("in_u", init_ux, N);
      L.upload("in_v", init_uy, N);
    }
    run_pair(L, (int)w, (int)h, roi != nullptr, init_ux != nullptr, *c, true, 3);
    // conf, raw_ux and raw_uy are final when the fine stage ends (event ev[2]), ux, uy and valid when the finish
    // stage has masked the field (event L.masked): their downloads run on the copy stream during the rest of the
    // pair; the strain planes follow on the lane's stream
    const ofc_pair_out d = device_pair_out(L, N);
    L.ensure_copy_stream();
    struct Drain {
      cudaStream_t a, b;
      ~Drain() {
        cudaStreamSynchronize(a);
        cudaStreamSynchronize(b);
      }
    } drain{L.copy, L.stream};
    OFC_CUDA(cudaStreamWaitEvent(L.copy, L.ev[2], 0));
    ofc_pair_out early{}, masked{}, late = *out;
    early.conf = out->conf;
    early.raw_ux = out->raw_ux;
    early.raw_uy = out->raw_uy;
    masked.ux = out->ux;
    masked.uy = out->uy;
    masked.valid = out->valid;
    late.conf = late.raw_ux = late.raw_uy = late.ux = late.uy = nullptr;
    late.valid = nullptr;
    cudaStream_t keep = L.stream;
    L.stream = L.copy;
    download_pair(L, d, &early, N);
    OFC_CUDA(cudaStreamWaitEvent(L.copy, L.masked, 0));  // ux, uy, valid during the strain
    download_pair(L, d, &masked, N);
    L.stream = keep;
    download_pair(L, d, &late, N);
    OFC_CUDA(cudaStreamSynchronize(L.copy));
    OFC_CUDA(cudaStreamSynchronize(L.stream));
    double timing[3];
    pair_timing(L, timing);
    for (int i = 0; i < 3; i++) out->timing[i] = timing[i];
  });
}

}  // extern "C"

namespace {

// ---------------------------------------------------------------- sequences: one driver for chain and hybrid
// track.py:260-315 (chain) and 385-503 (hybrid); rust/crates/optflow-core/src/track.rs:1030-1245, track/hybrid.rs.
// Frames come from `frame` (the caller's arrays, or a source filling page-locked slots one frame ahead while the
// GPU works), go through ofc_to_gray's conversion when they are not float32 grey at full size, and each frame's
// results go to `emit` from page-locked staging while the GPU tracks the next frame.
struct SeqIO {
  int W = 0, H = 0;           // the tracked grid
  const uint8_t* roi = nullptr;  // host, W x H, nullable
  const ofc_config* c = nullptr;
  bool hybrid = false;
  ofc_hybrid hy{};
  int32_t pixel = OFC_PIX_F32;
  int w_in = 0, h_in = 0, scale = 1;
  // frame k's bytes: a host pointer (pageable or `slot`), or nullptr when the sequence has no frame k
  std::function<const void*(int64_t k, void* slot)> frame;
  // when set, frame k of the sequence is made on the device into dst (the stream's window means) instead of coming
  // from `frame`; false: the sequence has no frame k
  std::function<bool(int64_t k, float* dst)> produce;
  std::function<double(int64_t k)> ruc;  // ref_update_conf at frame k
  std::function<void(int64_t k, const ofc_pair_out& out, const int32_t* fb, const ofc_hybrid_frame& info)> emit;
  ofc_leg_fn leg = nullptr;
  void* leg_user = nullptr;
};

int64_t run_sequence(Lane& L, const SeqIO& io) {
  const ofc_config& c = *io.c;
  const int W = io.W, H = io.H;
  const size_t N = (size_t)W * H;
  cudaStream_t st = L.stream;
  L.ensure_copy_stream();
  const dim3 g2(div_up(W, 128), H);
  const unsigned gN = std::min<unsigned>(div_up(N, 256), 148 * 8);
  const double cm = c.conf_min, radius = io.hy.fb_radius > 0 ? io.hy.fb_radius : 4.0 * c.sigma_w;
  const bool gate_on = io.hybrid && io.hy.fb_min_support > 0;
  size_t n_roi = N;
  if (io.roi) {
    n_roi = 0;
    for (size_t i = 0; i < N; i++) n_roi += io.roi[i] != 0;
  }
  // the run's state (track.py:423-431)
  float* ref = L.get<float>("seq_ref", N);
  float* prev = L.get<float>("seq_prev", N);
  float* fk = L.get<float>("seq_fk", N);
  float* u0r = L.get<float>("seq_u0r", 2 * N);
  float* u0n = L.get<float>("seq_u0n", 2 * N);
  double* c0r = L.get<double>("seq_c0r", N);
  float* praw = L.get<float>("seq_praw", 2 * N);  // the last final direct leg: its raw field and conf
  float* pconf = L.get<float>("seq_pconf", N);
  float* cxy = L.get<float>("hy_cxy", 2 * N);
  double* conf64 = L.get<double>("hy_conf", N);
  double* u64 = L.get<double>("hy_u64", 2 * N);
  float* rep = L.get<float>("seq_rep", N);
  double* rsum = L.get<double>("seq_rsum", (size_t)H);
  long long* rcnt = L.get<long long>("seq_rcnt", (size_t)H);
  double* dmean = L.get<double>("seq_mean", 1);
  uint8_t* low = L.get<uint8_t>("seq_low", N);
  uint8_t *anch = nullptr, *goodp = nullptr, *support = nullptr, *gate0 = nullptr, *gate = nullptr;
  int *nfb = nullptr, *dany = nullptr;
  float *uprev = nullptr, *padj = nullptr, *axy = nullptr;
  double *legc = nullptr, *link = nullptr, *ca = nullptr;
  uint16_t* fl = nullptr;
  unsigned long long* dcnt = nullptr;
  if (io.hybrid) {
    anch = L.get<uint8_t>("hy_anch", N);
    goodp = L.get<uint8_t>("hy_goodp", N);
    nfb = L.get<int>("hy_nfb", N);
    uprev = L.get<float>("hy_uprev", 2 * N);
    padj = L.get<float>("hy_padj", 2 * N);
    axy = L.get<float>("hy_axy", 2 * N);
    legc = L.get<double>("hy_legc", N);
    link = L.get<double>("hy_link", N);
    ca = L.get<double>("hy_ca", N);
    fl = L.get<uint16_t>("hy_flags", N);
    support = L.get<uint8_t>("hy_support", N);
    gate0 = L.get<uint8_t>("hy_gate0", N);
    gate = L.get<uint8_t>("hy_gate", N);
    dany = L.get<int>("hy_any", 4);
    dcnt = L.get<unsigned long long>("hy_cnt", 4);
  }
  const uint8_t* droi = io.roi ? L.upload("seq_roi", io.roi, N) : nullptr;
  float* in1 = L.get<float>("in_i1", N);
  float* in2 = L.get<float>("in_i2", N);
  float* inu = L.get<float>("in_u", N);
  float* inv = L.get<float>("in_v", N);
  const ofc_pair_out d = device_pair_out(L, N);  // a leg's conf, raw_ux, raw_uy; the frame's outputs
  const double B = guard_px(c) > 0 ? 4.0 * c.sigma_w : 0.0;
  // frame input: two page-locked slots (a source fills one while the other's upload may be in flight), the raw
  // frame on the device when it needs the conversion
  const bool direct = io.pixel == OFC_PIX_F32 && io.scale == 1;
  const size_t in_bytes = pixel_bytes(io.pixel) * (size_t)io.w_in * io.h_in;
  void* slot[2] = {L.pinned<uint8_t>("seq_slot0", in_bytes), L.pinned<uint8_t>("seq_slot1", in_bytes)};
  cudaEvent_t slot_free[2] = {L.bev[2], L.bev[3]};
  bool slot_used[2] = {false, false};
  uint8_t* rawin = direct ? nullptr : L.get<uint8_t>("seq_rawin", in_bytes);
  auto load = [&](const void* p, int s, float* dst) {
    if (direct) {
      OFC_CUDA(cudaMemcpyAsync(dst, p, N * 4, cudaMemcpyHostToDevice, st));
    } else {
      OFC_CUDA(cudaMemcpyAsync(rawin, p, in_bytes, cudaMemcpyHostToDevice, st));
      to_gray_dev(L, rawin, io.pixel, io.w_in, io.scale, W, H, dst);
    }
    if (p == slot[s]) {
      OFC_CUDA(cudaEventRecord(slot_free[s], st));
      slot_used[s] = true;
    }
  };
  auto fetch = [&](int64_t k) -> const void* {
    const int s = (int)(k & 1);
    if (slot_used[s]) OFC_CUDA(cudaEventSynchronize(slot_free[s]));
    slot_used[s] = false;
    return io.frame(k, slot[s]);
  };
  // result output: the frame's planes copied on the device into staging (the next frame's legs overwrite them),
  // then to page-locked memory on the copy stream; emitted during the next frame's first leg
  float* dstage = L.get<float>("seq_stage", 10 * N);
  uint8_t* dstage_v = L.get<uint8_t>("seq_stage_v", N);
  int* dstage_fb = io.hybrid ? L.get<int>("seq_stage_fb", N) : nullptr;
  float* hout = L.pinned<float>("seq_hout", 10 * N);
  uint8_t* hvalid = L.pinned<uint8_t>("seq_hvalid", N);
  int32_t* hfb = io.hybrid ? L.pinned<int32_t>("seq_hfb", N) : nullptr;
  cudaEvent_t staged = L.bev[0], copied = L.bev[1];
  bool copy_issued = false;
  struct Pending {
    bool active = false;
    int64_t k = 0;
    double coarse = 0, fine = 0;
    ofc_hybrid_frame info{};
  } pending;
  const void* next = nullptr;
  bool fetched = false;
  int64_t k = 1, emitted = 0;
  auto flush = [&]() {
    if (!pending.active) return;
    OFC_CUDA(cudaEventSynchronize(copied));
    float ms = 0;
    OFC_CUDA(cudaEventElapsedTime(&ms, L.sev[0], L.sev[1]));
    ofc_pair_out o{};
    float** f[10] = {&o.ux, &o.uy, &o.conf, &o.exx, &o.eyy, &o.exy, &o.gmax, &o.vol, &o.raw_ux, &o.raw_uy};
    for (int i = 0; i < 10; i++) *f[i] = hout + i * N;
    o.valid = hvalid;
    o.timing[0] = pending.coarse;
    o.timing[1] = pending.fine;
    o.timing[2] = ms * 1e-3;
    pending.active = false;
    io.emit(pending.k, o, hfb, pending.info);
    emitted++;
  };
  // while the GPU runs a frame's first leg: deliver the previous frame's results, fetch the next frame
  // produced frames: the next frame's window is made into fk_next while this frame's first leg runs (its reads from
  // the source overlap the leg; its kernels follow the leg's on the stream)
  float* fk_next = io.produce ? L.get<float>("seq_fk_next", N) : nullptr;
  bool have_next = false;
  auto service = [&]() {
    flush();
    if (!fetched) {
      if (io.produce) have_next = io.produce(k + 1, fk_next);
      else next = fetch(k + 1);
      fetched = true;
    }
  };
  // one leg frames[ia] -> frames[ib] (track.py:200-206) into d's conf / raw planes: the engine's coarse and fine
  // stages with the dense start `init` (2 planes, nullable), or the caller's leg source; returns coarse, fine (s)
  std::vector<float> hbuf;
  auto leg = [&](const float* a, int64_t ia, const float* b, int64_t ib, const float* init,
                 bool first) -> std::pair<double, double> {
    if (io.leg) {
      if (first) service();
      hbuf.resize(5 * N);
      float* hi = hbuf.data();
      float* ho = hi + 2 * N;
      if (init) OFC_CUDA(cudaMemcpyAsync(hi, init, 2 * N * 4, cudaMemcpyDeviceToHost, st));
      OFC_CUDA(cudaStreamSynchronize(st));
      if (io.leg(io.leg_user, (int32_t)ia, (int32_t)ib, init ? hi : nullptr, init ? hi + N : nullptr, ho, ho + N,
                 ho + 2 * N) != 0)
        throw Error(OFC_ERR_ARG, "the leg source failed on the leg " + std::to_string(ia) + " -> " + std::to_string(ib));
      OFC_CUDA(cudaMemcpyAsync(d.raw_ux, ho, N * 4, cudaMemcpyHostToDevice, st));
      OFC_CUDA(cudaMemcpyAsync(d.raw_uy, ho + N, N * 4, cudaMemcpyHostToDevice, st));
      OFC_CUDA(cudaMemcpyAsync(d.conf, ho + 2 * N, N * 4, cudaMemcpyHostToDevice, st));
      OFC_CUDA(cudaStreamSynchronize(st));
      return {0.0, 0.0};
    }
    OFC_CUDA(cudaMemcpyAsync(in1, a, N * 4, cudaMemcpyDeviceToDevice, st));
    OFC_CUDA(cudaMemcpyAsync(in2, b, N * 4, cudaMemcpyDeviceToDevice, st));
    if (init) {
      OFC_CUDA(cudaMemcpyAsync(inu, init, N * 4, cudaMemcpyDeviceToDevice, st));
      OFC_CUDA(cudaMemcpyAsync(inv, init + N, N * 4, cudaMemcpyDeviceToDevice, st));
    }
    run_pair(L, W, H, false, init != nullptr, c, true, 2);
    if (first) service();
    float ms0 = 0, ms1 = 0;
    OFC_CUDA(cudaEventSynchronize(L.ev[3]));
    OFC_CUDA(cudaEventElapsedTime(&ms0, L.ev[0], L.ev[1]));
    OFC_CUDA(cudaEventElapsedTime(&ms1, L.ev[1], L.ev[3]));
    return {ms0 * 1e-3, ms1 * 1e-3};
  };
  auto leg_mean = [&]() {
    OFC_LAUNCH(k_reportable, g2, 128, 0, st, d.raw_ux, d.raw_uy, W, H, B, rep);
    OFC_LAUNCH(k_mean_conf_rows, H, MC_T, 0, st, d.conf, rep, u0r, u0r + N, droi, W, H, rsum, rcnt);
    OFC_LAUNCH(k_mean_conf_fold, 1, 1, 0, st, rsum, rcnt, H, dmean);
    double m = 0;
    OFC_CUDA(cudaMemcpyAsync(&m, dmean, 8, cudaMemcpyDeviceToHost, st));
    OFC_CUDA(cudaStreamSynchronize(st));
    return m;
  };
  int any[4];
  auto read_any = [&]() {
    OFC_CUDA(cudaMemcpyAsync(any, dany, sizeof(any), cudaMemcpyDeviceToHost, st));
    OFC_CUDA(cudaStreamSynchronize(st));
  };

  if (io.produce) {
    if (!io.produce(0, ref)) throw Error(OFC_ERR_ARG, "no frames");
  } else {
    const void* f0 = fetch(0);
    if (!f0) throw Error(OFC_ERR_ARG, "no frames");
    load(f0, 0, ref);
  }
  OFC_CUDA(cudaMemcpyAsync(prev, ref, N * 4, cudaMemcpyDeviceToDevice, st));
  OFC_CUDA(cudaMemsetAsync(u0r, 0, 2 * N * 4, st));
  launch_fill_f64(c0r, 1.0, N, st);
  if (io.hybrid) {
    OFC_CUDA(cudaMemsetAsync(anch, 1, N, st));
    OFC_CUDA(cudaMemsetAsync(goodp, 1, N, st));
    OFC_CUDA(cudaMemsetAsync(nfb, 0, N * 4, st));
    OFC_CUDA(cudaMemsetAsync(uprev, 0, 2 * N * 4, st));
  }
  bool have_prev = false, have_padj = false;
  int64_t ref_idx = 0;
  // hybrid: the adjacent leg k - 1 -> k runs on a worker lane beside the direct leg when the previous frame needed
  // one (its inputs are known before the direct leg: prev, fk and the previous adjacent field as the start); it is
  // used only where the reference's rule asks for it (track.py:452-457), so the results are those of the legs run
  // one after the other
  Lane* A = nullptr;
  if (io.hybrid && !io.leg) {
    if (L.aux.empty()) {
      std::unique_ptr<Lane> a(new Lane());
      lane_init(*a);
      L.aux.push_back(std::move(a));
    }
    A = L.aux[0].get();
  }
  cudaEvent_t spec_ready = L.bev[4], spec_taken = L.bev[5], spec_done = L.bev[6];
  if (io.produce) have_next = io.produce(1, fk);
  else next = fetch(1);
  while (io.produce ? have_next : next != nullptr) {
    if (!io.produce) load(next, (int)(k & 1), fk);
    fetched = false;
    next = nullptr;
    const double ruc = io.ruc(k);
    bool spec = false;
    if (A && ref_idx != k - 1 && have_padj) {
      spec = true;
      OFC_CUDA(cudaEventRecord(spec_ready, st));
      OFC_CUDA(cudaStreamWaitEvent(A->stream, spec_ready, 0));
      OFC_CUDA(cudaMemcpyAsync(A->get<float>("in_i1", N), prev, N * 4, cudaMemcpyDeviceToDevice, A->stream));
      OFC_CUDA(cudaMemcpyAsync(A->get<float>("in_i2", N), fk, N * 4, cudaMemcpyDeviceToDevice, A->stream));
      OFC_CUDA(cudaMemcpyAsync(A->get<float>("in_u", N), padj, N * 4, cudaMemcpyDeviceToDevice, A->stream));
      OFC_CUDA(cudaMemcpyAsync(A->get<float>("in_v", N), padj + N, N * 4, cudaMemcpyDeviceToDevice, A->stream));
      OFC_CUDA(cudaEventRecord(spec_taken, A->stream));
      run_pair(*A, W, H, false, true, c, true, 2);
      OFC_CUDA(cudaEventRecord(spec_done, A->stream));
    }
    std::pair<double, double> t = leg(ref, ref_idx, fk, k, have_prev ? praw : nullptr, true);
    double cmean = leg_mean();
    if (cmean < ruc && ref_idx != k - 1) {
      if (io.hybrid) {
        // c0K replaced, anchors = good_prev, u0K = u_{k-1} (track.py:433-440)
        OFC_LAUNCH(k_hyb_move, g2, 128, 0, st, pconf, u0r, u0r + N, goodp, W, H, c0r, anch);
        OFC_CUDA(cudaMemcpyAsync(u0r, uprev, 2 * N * 4, cudaMemcpyDeviceToDevice, st));
      } else {
        // the previous leg extends the link of frame 0 (track.rs:1135-1155)
        OFC_LAUNCH(k_link_conf, g2, 128, 0, st, c0r, pconf, u0r, u0r + N, W, H, c0r);
        OFC_LAUNCH(k_compose, g2, 128, 0, st, u0r, u0r + N, praw, praw + N, W, H, u0n, u0n + N);
        OFC_CUDA(cudaMemcpyAsync(u0r, u0n, 2 * N * 4, cudaMemcpyDeviceToDevice, st));
      }
      OFC_CUDA(cudaMemcpyAsync(ref, prev, N * 4, cudaMemcpyDeviceToDevice, st));
      ref_idx = k - 1;
      t = leg(ref, ref_idx, fk, k, nullptr, false);
      cmean = leg_mean();
    }
    OFC_CUDA(cudaMemcpyAsync(praw, d.raw_ux, N * 4, cudaMemcpyDeviceToDevice, st));
    OFC_CUDA(cudaMemcpyAsync(praw + N, d.raw_uy, N * 4, cudaMemcpyDeviceToDevice, st));
    OFC_CUDA(cudaMemcpyAsync(pconf, d.conf, N * 4, cudaMemcpyDeviceToDevice, st));
    ofc_hybrid_frame info{};
    info.reference = (int32_t)ref_idx;
    info.mean_conf = cmean;
    if (!io.hybrid) {
      // frame 0 -> k and its link confidence (track.rs:1157-1200)
      OFC_LAUNCH(k_compose, g2, 128, 0, st, u0r, u0r + N, praw, praw + N, W, H, cxy, cxy + N);
      OFC_LAUNCH(k_link_conf, g2, 128, 0, st, c0r, pconf, u0r, u0r + N, W, H, conf64);
      launch_f32_to_f64(cxy, u64, 2 * N, st);
      ofc_threshold_low(conf64, cm, low, N, st);
    } else {
      OFC_CUDA(cudaMemsetAsync(dany, 0, 4 * sizeof(int), st));
      OFC_CUDA(cudaMemsetAsync(dcnt, 0, 4 * sizeof(unsigned long long), st));
      OFC_LAUNCH(k_hyb_classify, g2, 128, 0, st, praw, praw + N, pconf, u0r, u0r + N, c0r, anch, uprev, uprev + N,
                 nfb, droi, W, H, cm, io.hy.fb_max, ref_idx + 1 < k ? 1 : 0, cxy, cxy + N, legc, link, fl, dany);
      read_any();
      const float *arx = nullptr, *ary = nullptr, *acf = nullptr;
      if (spec) OFC_CUDA(cudaStreamWaitEvent(st, spec_taken, 0));  // padj and prev may change from here on
      if (any[0]) {
        if (ref_idx == k - 1) {  // the direct leg is the adjacent leg
          arx = praw;
          ary = praw + N;
          acf = pconf;
        } else if (spec) {  // the worker lane's leg (the same inputs as the leg below)
          OFC_CUDA(cudaStreamWaitEvent(st, spec_done, 0));
          const ofc_pair_out da = device_pair_out(*A, N);
          float ms0 = 0, ms1 = 0;  // the two stages of the worker's leg (run_pair records ev[0], ev[1], ev[3])
          OFC_CUDA(cudaEventSynchronize(A->ev[3]));
          OFC_CUDA(cudaEventElapsedTime(&ms0, A->ev[0], A->ev[1]));
          OFC_CUDA(cudaEventElapsedTime(&ms1, A->ev[1], A->ev[3]));
          t.first += ms0 * 1e-3;
          t.second += ms1 * 1e-3;
          arx = da.raw_ux;
          ary = da.raw_uy;
          acf = da.conf;
        } else {
          const std::pair<double, double> ta = leg(prev, k - 1, fk, k, have_padj ? padj : nullptr, false);
          t.first += ta.first;
          t.second += ta.second;
          arx = d.raw_ux;
          ary = d.raw_uy;
          acf = d.conf;
        }
      }
      OFC_LAUNCH(k_hyb_adjacent, g2, 128, 0, st, arx, ary, acf, uprev, uprev + N, W, H, axy, axy + N, ca);
      if (any[0]) {
        OFC_CUDA(cudaMemcpyAsync(padj, arx, N * 4, cudaMemcpyDeviceToDevice, st));
        OFC_CUDA(cudaMemcpyAsync(padj + N, ary, N * 4, cudaMemcpyDeviceToDevice, st));
      }
      have_padj = any[0] != 0;
      OFC_LAUNCH(k_hyb_pre, gN, 256, 0, st, fl, cxy, cxy + N, axy, axy + N, ca, droi, N, cm, io.hy.fb_tol, support,
                 dany);
      read_any();
      const uint8_t* g0 = nullptr;
      if (gate_on && any[1]) {
        laa_dev<float>(L, W, H, support, cxy, cxy + N, cxy, cxy + N, radius, io.hy.fb_min_support, io.hy.fb_tol,
                       gate0, nullptr);
        g0 = gate0;
      }
      OFC_LAUNCH(k_hyb_re, gN, 256, 0, st, fl, g0, legc, c0r, anch, nfb, ca, droi, N, io.hy.fb_max, cm, support,
                 dany);
      read_any();
      const uint8_t* g1 = nullptr;
      if (gate_on && any[2]) {
        laa_dev<float>(L, W, H, support, cxy, cxy + N, axy, axy + N, radius, io.hy.fb_min_support, io.hy.fb_tol,
                       gate, nullptr);
        g1 = gate;
      }
      OFC_LAUNCH(k_hyb_out, gN, 256, 0, st, fl, g1, cxy, cxy + N, axy, axy + N, link, ca, nfb, droi, N, io.hy.fb_max,
                 uprev, uprev + N, u64, u64 + N, conf64, low, goodp, dcnt);
      unsigned long long cnt[4];
      OFC_CUDA(cudaMemcpyAsync(cnt, dcnt, sizeof(cnt), cudaMemcpyDeviceToHost, st));
      OFC_CUDA(cudaStreamSynchronize(st));
      info.n_fb_max = (int32_t)cnt[3];
      info.fallback_frac = (double)cnt[0] / (double)n_roi;
      info.fb_gate_rejected = (double)cnt[1] / (double)n_roi;
      info.reacquired = (double)cnt[2] / (double)n_roi;
    }
    if (!fetched) service();  // a scripted run whose legs all came from the caller
    OFC_CUDA(cudaEventRecord(L.sev[0], st));
    finish_dev(L, low, droi, u64, u64 + N, conf64, W, H, c, d, false);
    OFC_CUDA(cudaEventRecord(L.sev[1], st));
    // stage the results (after the previous frame's copy has left the staging), copy them out on the copy stream
    if (copy_issued) OFC_CUDA(cudaStreamWaitEvent(st, copied, 0));
    OFC_CUDA(cudaMemcpyAsync(dstage, d.ux, 10 * N * 4, cudaMemcpyDeviceToDevice, st));
    OFC_CUDA(cudaMemcpyAsync(dstage_v, d.valid, N, cudaMemcpyDeviceToDevice, st));
    if (io.hybrid) OFC_CUDA(cudaMemcpyAsync(dstage_fb, nfb, N * 4, cudaMemcpyDeviceToDevice, st));
    OFC_CUDA(cudaEventRecord(staged, st));
    OFC_CUDA(cudaStreamWaitEvent(L.copy, staged, 0));
    OFC_CUDA(cudaMemcpyAsync(hout, dstage, 10 * N * 4, cudaMemcpyDeviceToHost, L.copy));
    OFC_CUDA(cudaMemcpyAsync(hvalid, dstage_v, N, cudaMemcpyDeviceToHost, L.copy));
    if (io.hybrid) OFC_CUDA(cudaMemcpyAsync(hfb, dstage_fb, N * 4, cudaMemcpyDeviceToHost, L.copy));
    OFC_CUDA(cudaEventRecord(copied, L.copy));
    copy_issued = true;
    pending.active = true;
    pending.k = k;
    pending.coarse = t.first;
    pending.fine = t.second;
    pending.info = info;
    OFC_CUDA(cudaMemcpyAsync(prev, fk, N * 4, cudaMemcpyDeviceToDevice, st));
    have_prev = true;
    k++;
    if (io.produce) std::swap(fk, fk_next);
  }
  flush();
  OFC_CUDA(cudaStreamSynchronize(st));
  return emitted;
}

// the checks shared by the sequence entry points (track.py:274-279)
void sequence_checks(const ofc_config* c, size_t w, size_t h, const uint8_t* roi) {
  cfg_check(c);
  check_sizes(w, h);
  if (roi) {
    bool any = false;
    for (size_t i = 0, N = w * h; i < N && !any; i++) any = roi[i] != 0;
    if (!any) throw Error(OFC_ERR_ARG, "ROI mask is empty");
  }
}

void size_checks(size_t w, size_t h, const ofc_config* c, bool legs) {
  if ((int)std::min(w, h) < c->poc_win)
    throw Error(OFC_ERR_ARG, "image smaller than poc_win (" + std::to_string(c->poc_win) + ")");
  if (!legs) check_fine_window(w, h, *c);
}

}  // namespace

extern "C" {

int ofc_track_sequence(ofc_engine* e, const float* const* frames, size_t n, size_t w, size_t h, const uint8_t* roi,
                       const ofc_config* c, double ref_update_conf, ofc_pair_out* outs, int32_t* reference,
                       double* mean_conf, char* err, size_t errlen) {
  return guarded(e, err, errlen, [&](Lane& L) {
    sequence_checks(c, w, h, roi);
    if (!frames || n == 0) throw Error(OFC_ERR_ARG, "no frames");
    for (size_t k = 0; k < n; k++)
      if (!frames[k]) throw Error(OFC_ERR_ARG, "null frame " + std::to_string(k));
    if (n > 1 && !outs) throw Error(OFC_ERR_ARG, "null outputs");
    if (!std::isfinite(ref_update_conf)) throw Error(OFC_ERR_ARG, "ref_update_conf must be a finite number");
    if (n == 1) return;
    size_checks(w, h, c, false);
    const size_t N = w * h;
    SeqIO io;
    io.W = (int)w;
    io.H = (int)h;
    io.roi = roi;
    io.c = c;
    io.w_in = (int)w;
    io.h_in = (int)h;
    io.frame = [&](int64_t k, void*) -> const void* { return k < (int64_t)n ? frames[k] : nullptr; };
    io.ruc = [&](int64_t) { return ref_update_conf; };
    io.emit = [&](int64_t k, const ofc_pair_out& o, const int32_t*, const ofc_hybrid_frame& info) {
      copy_pair_out(o, &outs[k - 1], N);
      if (reference) reference[k - 1] = info.reference;
      if (mean_conf) mean_conf[k - 1] = info.mean_conf;
    };
    run_sequence(L, io);
  });
}

int ofc_track_sequence_hybrid(ofc_engine* e, const float* const* frames, size_t n, size_t w, size_t h,
                              const uint8_t* roi, const ofc_config* c, const double* ruc, const ofc_hybrid* hy,
                              ofc_pair_out* outs, int32_t* fb, ofc_hybrid_frame* info, ofc_leg_fn legfn,
                              void* leg_user, char* err, size_t errlen) {
  return guarded(e, err, errlen, [&](Lane& L) {
    sequence_checks(c, w, h, roi);
    hybrid_check(hy);
    if (!frames || n == 0) throw Error(OFC_ERR_ARG, "no frames");
    for (size_t k = 0; k < n; k++)
      if (!frames[k]) throw Error(OFC_ERR_ARG, "null frame " + std::to_string(k));
    if (n > 1 && !outs) throw Error(OFC_ERR_ARG, "null outputs");
    if (n > 1 && !ruc) throw Error(OFC_ERR_ARG, "null ref_update_conf");
    for (size_t k = 0; k + 1 < n; k++)
      if (!std::isfinite(ruc[k])) throw Error(OFC_ERR_ARG, "ref_update_conf must be a finite number");
    if (n == 1) return;
    size_checks(w, h, c, legfn != nullptr);
    const size_t N = w * h;
    SeqIO io;
    io.W = (int)w;
    io.H = (int)h;
    io.roi = roi;
    io.c = c;
    io.hybrid = true;
    io.hy = *hy;
    io.w_in = (int)w;
    io.h_in = (int)h;
    io.leg = legfn;
    io.leg_user = leg_user;
    io.frame = [&](int64_t k, void*) -> const void* { return k < (int64_t)n ? frames[k] : nullptr; };
    io.ruc = [&](int64_t k) { return ruc[k - 1]; };
    io.emit = [&](int64_t k, const ofc_pair_out& o, const int32_t* f, const ofc_hybrid_frame& fi) {
      copy_pair_out(o, &outs[k - 1], N);
      if (fb) std::memcpy(fb + (k - 1) * N, f, N * 4);
      if (info) info[k - 1] = fi;
    };
    run_sequence(L, io);
  });
}

int ofc_track_stream(ofc_engine* e, const ofc_stream* s, const uint8_t* roi, const ofc_config* c, int64_t* n_out,
                     char* err, size_t errlen) {
  if (n_out) *n_out = 0;
  return guarded(e, err, errlen, [&](Lane& L) {
    if (!s) throw Error(OFC_ERR_ARG, "null stream");
    if (!s->source || !s->sink) throw Error(OFC_ERR_ARG, "the stream needs a source and a sink");
    check_format(s->pixel, s->w_in, s->h_in, s->scale);
    const size_t w = s->w_in / s->scale, h = s->h_in / s->scale;
    sequence_checks(c, w, h, roi);
    if (s->hybrid) hybrid_check(&s->hy);
    if (!std::isfinite(s->ref_update_conf)) throw Error(OFC_ERR_ARG, "ref_update_conf must be a finite number");
    size_checks(w, h, c, false);
    SeqIO io;
    io.W = (int)w;
    io.H = (int)h;
    io.roi = roi;
    io.c = c;
    io.hybrid = s->hybrid != 0;
    io.hy = s->hy;
    io.pixel = s->pixel;
    io.w_in = (int)s->w_in;
    io.h_in = (int)s->h_in;
    io.scale = s->scale;
    if (s->step < 1) throw Error(OFC_ERR_ARG, "step must be >= 1, got " + std::to_string(s->step));
    if (s->start < 0) throw Error(OFC_ERR_ARG, "start must be >= 0, got " + std::to_string(s->start));
    if (s->tavg < 0) throw Error(OFC_ERR_ARG, "tavg must be >= 0, got " + std::to_string(s->tavg));
    const int64_t start = s->start, step = s->step, stop = s->stop;
    auto raw = [&](int64_t i, void* slot) -> bool {  // raw frame i of the source into slot; false at its end
      const int r = s->source(s->source_user, i, slot);
      if (r == 1) return false;
      if (r != 0) throw Error(OFC_ERR_ARG, "the frame source failed on frame " + std::to_string(i));
      return true;
    };
    io.frame = [&](int64_t k, void* slot) -> const void* {
      const int64_t i = start + k * step;
      if (stop >= 0 && i >= stop) return nullptr;
      return raw(i, slot) ? slot : nullptr;
    };
    // tavg (io.py:126-153): the downscaled raw frames stay on the device in a ring, from which each sampled frame's
    // window mean is made (window_mean_dev) when the frames after it have been read
    const int m = s->tavg;
    const int W = (int)w, H = (int)h;
    const size_t N = w * h, in_bytes = pixel_bytes(s->pixel) * s->w_in * s->h_in;
    std::map<int64_t, float*> ring;
    std::vector<float*> spare;
    int nring = 0;
    int64_t raw_next = 0, last = -1;
    bool ended = false, slot_busy = false;
    uint8_t* traw = nullptr;
    void* tslot = nullptr;
    if (m > 0) {
      traw = L.get<uint8_t>("stream_tavg_raw", in_bytes);
      tslot = L.pinned<uint8_t>("stream_tavg_slot", in_bytes);
      L.ensure_copy_stream();
      io.produce = [&](int64_t k, float* dst) -> bool {
        cudaStream_t st = L.stream;
        const int64_t sidx = start + k * step;
        if (stop >= 0 && sidx >= stop) return false;
        const int64_t lo = std::max<int64_t>(0, sidx - m);
        for (auto it = ring.begin(); it != ring.end();) {  // frames below the window go back to the spares
          if (it->first < lo) {
            spare.push_back(it->second);
            it = ring.erase(it);
          } else {
            ++it;
          }
        }
        raw_next = std::max(raw_next, lo);
        while (!ended && raw_next <= sidx + m && (stop < 0 || raw_next < stop + m)) {
          if (slot_busy) OFC_CUDA(cudaEventSynchronize(L.bev[7]));  // the slot's last upload has left it
          if (!raw(raw_next, tslot)) {
            ended = true;
            break;
          }
          float* d = nullptr;
          if (!spare.empty()) {
            d = spare.back();
            spare.pop_back();
          } else {
            d = L.get<float>("stream_tavg_ring" + std::to_string(nring++), N);
          }
          OFC_CUDA(cudaMemcpyAsync(traw, tslot, in_bytes, cudaMemcpyHostToDevice, st));
          OFC_CUDA(cudaEventRecord(L.bev[7], st));
          slot_busy = true;
          to_gray_dev(L, traw, s->pixel, (int)s->w_in, s->scale, W, H, d);
          ring[raw_next] = d;
          last = raw_next;
          raw_next++;
        }
        if (!ring.count(sidx)) return false;  // the source ended before the sampled frame
        const int64_t hi = std::min(sidx + m, last);
        std::vector<const float*> fr;
        for (int64_t i = lo; i <= hi; i++) fr.push_back(ring.at(i));
        const size_t centre = (size_t)(sidx - lo);
        if (!s->tavg_align && sidx - lo != hi - sidx && std::min(W, H) >= c->poc_win)
          window_mean_dev(L, fr.data(), fr.size(), centre, W, H, 2, nullptr, true, *c, dst);
        else
          window_mean_dev(L, fr.data(), fr.size(), centre, W, H, s->tavg_align ? 1 : 0,
                          s->tavg_align ? s->tavg_mask : nullptr, false, *c, dst);
        return true;
      };
    }
    io.ruc = [&](int64_t) { return s->ref_update_conf; };
    io.emit = [&](int64_t k, const ofc_pair_out& o, const int32_t* f, const ofc_hybrid_frame& fi) {
      if (s->sink(s->sink_user, k, &o, f, &fi) != 0)
        throw Error(OFC_ERR_ARG, "the result sink stopped the run at frame " + std::to_string(k));
      if (n_out) *n_out = k;
    };
    run_sequence(L, io);
  });
}

int ofc_to_gray(ofc_engine* e, const void* px, int32_t pixel, size_t w, size_t h, int32_t scale, float* out,
                char* err, size_t errlen) {
  return guarded(e, err, errlen, [&](Lane& L) {
    if (!px || !out) throw Error(OFC_ERR_ARG, "null argument");
    check_format(pixel, w, h, scale);
    const size_t bytes = pixel_bytes(pixel) * w * h, W = w / scale, H = h / scale;
    const uint8_t* d = L.upload("gray_in", (const uint8_t*)px, bytes);
    float* o = L.get<float>("gray_out", W * H);
    to_gray_dev(L, d, pixel, (int)w, scale, (int)W, (int)H, o);
    OFC_CUDA(cudaMemcpyAsync(out, o, W * H * 4, cudaMemcpyDeviceToHost, L.stream));
    OFC_CUDA(cudaStreamSynchronize(L.stream));
  });
}

int ofc_local_affine_agreement(ofc_engine* e, size_t w, size_t h, const double* ux, const double* uy,
                               const uint8_t* support, const double* tx, const double* ty, double radius,
                               int64_t min_support, double tol, uint8_t* ok, int32_t* n, char* err, size_t errlen) {
  return guarded(e, err, errlen, [&](Lane& L) {
    check_sizes(w, h);
    if (!ux || !uy || !support || !tx || !ty || !ok) throw Error(OFC_ERR_ARG, "null argument");
    if (!std::isfinite(radius) || !std::isfinite(tol)) throw Error(OFC_ERR_ARG, "radius and tol must be finite");
    const size_t N = w * h;
    const double* dux = L.upload("laa_ux", ux, N);
    const double* duy = L.upload("laa_uy", uy, N);
    const double* dtx = L.upload("laa_tx", tx, N);
    const double* dty = L.upload("laa_ty", ty, N);
    const uint8_t* dsup = L.upload("laa_support", support, N);
    uint8_t* dok = L.get<uint8_t>("laa_ok", N);
    int* dn = L.get<int>("laa_n", N);
    laa_dev<double>(L, (int)w, (int)h, dsup, dux, duy, dtx, dty, radius, (long long)min_support, tol, dok, dn);
    OFC_CUDA(cudaMemcpyAsync(ok, dok, N, cudaMemcpyDeviceToHost, L.stream));
    if (n) OFC_CUDA(cudaMemcpyAsync(n, dn, N * 4, cudaMemcpyDeviceToHost, L.stream));
    OFC_CUDA(cudaStreamSynchronize(L.stream));
  });
}

int ofc_align_to(ofc_engine* e, const float* centre, const float* other, size_t w, size_t h, const uint8_t* mask,
                 int model, const ofc_config* c, float* out, int* aligned, char* err, size_t errlen) {
  return guarded(e, err, errlen, [&](Lane& L) {
    cfg_check(c);
    check_sizes(w, h);
    if (!centre || !other || !out || !aligned) throw Error(OFC_ERR_ARG, "null argument");
    if (model != 0 && model != 1) throw Error(OFC_ERR_ARG, "tavg model must be 0 (affine) or 1 (dense)");
    if ((int)std::min(w, h) < c->poc_win)
      throw Error(OFC_ERR_ARG, "image smaller than poc_win (" + std::to_string(c->poc_win) + ")");
    const size_t N = w * h;
    const float* dc = L.upload("tavg_c", centre, N);
    const float* d_o = L.upload("tavg_o", other, N);
    float* d_out = L.get<float>("tavg_out", N);
    const bool ok = tavg_align_dev(L, dc, d_o, (int)w, (int)h, model == 0 ? mask : nullptr, model, *c, d_out);
    if (ok) OFC_CUDA(cudaMemcpyAsync(out, d_out, N * 4, cudaMemcpyDeviceToHost, L.stream));
    OFC_CUDA(cudaStreamSynchronize(L.stream));
    *aligned = ok ? 1 : 0;
  });
}

int ofc_average_window(ofc_engine* e, const float* const* frames, size_t n, size_t centre, size_t w, size_t h,
                       int align, const uint8_t* mask, int keep_unaligned, const ofc_config* c, float* out,
                       int* used_count, char* err, size_t errlen) {
  return guarded(e, err, errlen, [&](Lane& L) {
    cfg_check(c);
    check_sizes(w, h);
    if (!frames || !out || n == 0) throw Error(OFC_ERR_ARG, "no frames");
    if (centre >= n) throw Error(OFC_ERR_ARG, "centre index beyond the frames");
    for (size_t i = 0; i < n; i++)
      if (!frames[i]) throw Error(OFC_ERR_ARG, "null frame " + std::to_string(i));
    if (align < 0 || align > 2) throw Error(OFC_ERR_ARG, "align must be 0 (none), 1 (affine) or 2 (dense)");
    if (align && (int)std::min(w, h) < c->poc_win)
      throw Error(OFC_ERR_ARG, "image smaller than poc_win (" + std::to_string(c->poc_win) + ")");
    const size_t N = w * h;
    cudaStream_t st = L.stream;
    float* dwin = L.get<float>("tavg_win", n * N);
    std::vector<const float*> dframes(n);
    for (size_t i = 0; i < n; i++) {
      OFC_CUDA(cudaMemcpyAsync(dwin + i * N, frames[i], N * 4, cudaMemcpyHostToDevice, st));
      dframes[i] = dwin + i * N;
    }
    float* dout = L.get<float>("tavg_mean", N);
    const int used = window_mean_dev(L, dframes.data(), n, centre, (int)w, (int)h, align, mask, keep_unaligned != 0,
                                     *c, dout);
    OFC_CUDA(cudaMemcpyAsync(out, dout, N * 4, cudaMemcpyDeviceToHost, st));
    OFC_CUDA(cudaStreamSynchronize(st));
    if (used_count) *used_count = used;
  });
}

int ofc_track_pair_device(ofc_engine* e, const float* d_i1, const float* d_i2, size_t w, size_t h, const uint8_t* d_roi,
                          const float* d_init_ux, const float* d_init_uy, const ofc_config* c, ofc_pair_out* d_out,
                          void* stream, char* err, size_t errlen) {
  return guarded(e, err, errlen, [&](Lane& L) {
    cfg_check(c);
    check_fine_window(w, h, *c);
    if (!d_i1 || !d_i2 || !d_out) throw Error(OFC_ERR_ARG, "null argument");
    if ((d_init_ux == nullptr) != (d_init_uy == nullptr))
      throw Error(OFC_ERR_ARG, "init_ux and init_uy must both be given");
    if ((int)std::min(w, h) < c->poc_win)
      throw Error(OFC_ERR_ARG, "image smaller than poc_win (" + std::to_string(c->poc_win) + ")");
    const size_t N = w * h;
    cudaStream_t keep = L.stream;
    if (stream) L.stream = (cudaStream_t)stream;
    try {
      // the caller's buffers are copied into the lane's (the captured graphs read and write fixed addresses)
      cudaStream_t st = L.stream;
      OFC_CUDA(cudaMemcpyAsync(L.get<float>("in_i1", N), d_i1, N * 4, cudaMemcpyDeviceToDevice, st));
      OFC_CUDA(cudaMemcpyAsync(L.get<float>("in_i2", N), d_i2, N * 4, cudaMemcpyDeviceToDevice, st));
      if (d_roi) OFC_CUDA(cudaMemcpyAsync(L.get<uint8_t>("in_roi", N), d_roi, N, cudaMemcpyDeviceToDevice, st));
      if (d_init_ux) {
        OFC_CUDA(cudaMemcpyAsync(L.get<float>("in_u", N), d_init_ux, N * 4, cudaMemcpyDeviceToDevice, st));
        OFC_CUDA(cudaMemcpyAsync(L.get<float>("in_v", N), d_init_uy, N * 4, cudaMemcpyDeviceToDevice, st));
      }
      run_pair(L, (int)w, (int)h, d_roi != nullptr, d_init_ux != nullptr, *c, false, 3);
      const ofc_pair_out d = device_pair_out(L, N);
      float* const* dsrc[10] = {&d.ux, &d.uy, &d.conf, &d.exx, &d.eyy, &d.exy, &d.gmax, &d.vol, &d.raw_ux, &d.raw_uy};
      float* const* udst[10] = {&d_out->ux,  &d_out->uy,  &d_out->conf, &d_out->exx,    &d_out->eyy,
                                &d_out->exy, &d_out->gmax, &d_out->vol, &d_out->raw_ux, &d_out->raw_uy};
      for (int i = 0; i < 10; i++)
        if (*udst[i]) OFC_CUDA(cudaMemcpyAsync(*udst[i], *dsrc[i], N * 4, cudaMemcpyDeviceToDevice, st));
      if (d_out->valid) OFC_CUDA(cudaMemcpyAsync(d_out->valid, d.valid, N, cudaMemcpyDeviceToDevice, st));
    } catch (...) {
      L.stream = keep;
      throw;
    }
    L.stream = keep;
    std::memset(d_out->timing, 0, sizeof(d_out->timing));
  });
}

}  // extern "C"


// ================================================================= single-stage entry points (testing header)
extern "C" {

int ofc_test_fft_lines(ofc_engine* e, float* data, size_t lines, size_t L, int inverse, char* err, size_t errlen) {
  return guarded(e, err, errlen, [&](Lane& Ln) {
    if (fft_work_length((int)L) == 0) throw Error(OFC_ERR_ARG, "unsupported FFT length");
    const FftPlan& pl = Ln.plan((int)L);
    float2* d = Ln.upload("t_fft", (const float2*)data, lines * L);
    launch_fft_lines(d, (int)lines, pl, inverse != 0, Ln.stream);
    OFC_CUDA(cudaMemcpyAsync(data, d, lines * L * sizeof(float2), cudaMemcpyDeviceToHost, Ln.stream));
    OFC_CUDA(cudaStreamSynchronize(Ln.stream));
  });
}


int ofc_test_reference_phase(ofc_engine* e, const float* i1, size_t w, size_t h, const ofc_config* c, float* r_re,
                             float* r_im, float* gx, float* gy, float* amp, char* err, size_t errlen) {
  return guarded(e, err, errlen, [&](Lane& L) {
    cfg_check(c);
    check_fine_window(w, h, *c);
    const int W = (int)w, H = (int)h, ph = H + 2 * PAD, pw = W + 2 * PAD, F = c->n_scales * c->n_orient;
    const size_t N = w * h;
    GaborTables g = upload_gabor(L, ph, pw, *c);
    float* d1 = L.upload("in_i1", i1, N);
    float4* ref4 = L.get<float4>("ref4", N * F);
    float* a = L.get<float>("ref_amp", N * F);
    reference_pack(L, d1, W, H, g, ref4, a, L.stream);
    std::vector<float4> h4(N * F);
    OFC_CUDA(cudaMemcpyAsync(h4.data(), ref4, N * F * sizeof(float4), cudaMemcpyDeviceToHost, L.stream));
    if (amp) OFC_CUDA(cudaMemcpyAsync(amp, a, N * F * sizeof(float), cudaMemcpyDeviceToHost, L.stream));
    OFC_CUDA(cudaStreamSynchronize(L.stream));
    for (size_t i = 0; i < N * F; i++) {
      if (r_re) r_re[i] = h4[i].x;
      if (r_im) r_im[i] = h4[i].y;
      if (gx) gx[i] = h4[i].z;
      if (gy) gy[i] = h4[i].w;
    }
  });
}

int ofc_test_responses(ofc_engine* e, const float* img, size_t w, size_t h, const ofc_config* c, float* resp, char* err,
                       size_t errlen) {
  return guarded(e, err, errlen, [&](Lane& L) {
    cfg_check(c);
    check_fine_window(w, h, *c);
    const int W = (int)w, H = (int)h, ph = H + 2 * PAD, pw = W + 2 * PAD, F = c->n_scales * c->n_orient;
    const size_t N = w * h, Np = (size_t)ph * pw;
    GaborTables g = upload_gabor(L, ph, pw, *c);
    float* d1 = L.upload("in_i1", img, N);
    float2* T = L.get<float2>("fft_T", Np);
    float2* U = L.get<float2>("fft_U", Np * F);
    float2* R = L.get<float2>("resp", resp_values(F, Np));
    launch_fft_rows_fwd_real(d1, W, H, L.plan(pw), ph, T, L.stream);
    launch_fft_cols_filters(T, L.plan(ph), pw, g, U, L.stream);
    launch_fft_rows_inv_resp(U, L.plan(pw), ph, F, R, L.stream);
    // the pair layout back to F planes of ph x pw
    std::vector<float2> h(resp_values(F, Np));
    OFC_CUDA(cudaMemcpyAsync(h.data(), R, h.size() * sizeof(float2), cudaMemcpyDeviceToHost, L.stream));
    OFC_CUDA(cudaStreamSynchronize(L.stream));
    float2* out = reinterpret_cast<float2*>(resp);
    for (int k = 0; k < F; k++)
      for (size_t i = 0; i < Np; i++) out[(size_t)k * Np + i] = h[((size_t)(k / 2) * Np + i) * 2 + (k & 1)];
  });
}

int ofc_test_local_solve(ofc_engine* e, const double* sums, const double* ux, const double* uy, size_t w, size_t h,
                         const ofc_config* c, double* oux, double* ouy, double* energy, double* resid, double* slope,
                         char* err, size_t errlen) {
  return guarded(e, err, errlen, [&](Lane& L) {
    cfg_check(c);
    const int W = (int)w, H = (int)h;
    const size_t N = w * h;
    int rw = 0;
    MomTaps mtp;
    const double* d_mt = moment_taps(L, c->sigma_w, rw, mtp);
    double* ds = L.upload("sums", sums, 7 * N);
    double* u2 = L.get<double>("u2", 2 * N);
    OFC_CUDA(cudaMemcpyAsync(u2, ux, N * 8, cudaMemcpyHostToDevice, L.stream));
    OFC_CUDA(cudaMemcpyAsync(u2 + N, uy, N * 8, cudaMemcpyHostToDevice, L.stream));
    double* o2 = L.get<double>("u2b", 2 * N);
    double* en = L.get<double>("energy", N);
    double* rs = L.get<double>("resid", N);
    double* sl = L.get<double>("slope", 4 * N);
    double* yp = L.get<double>("yplanes", (size_t)moment_yplanes(c->shape_order) * N);
    EnergyStats* stats = L.get<EnergyStats>("stats", 1);
    unsigned long long* hist = L.get<unsigned long long>("hist", median_scratch(N));
    OFC_CUDA(cudaMemsetAsync(hist, 0, 4096 * sizeof(unsigned long long), L.stream));
    launch_moments_solve(ds, u2, u2 + N, W, H, c->shape_order, d_mt, rw, mtp, yp, o2, o2 + N, en, rs, sl, L.stream);
    launch_energy_median(en, N, stats, false, hist, L.stream);
    launch_reset(en, u2, u2 + N, (int)N, stats, o2, o2 + N, rs, sl, L.stream);
    OFC_CUDA(cudaMemcpyAsync(oux, o2, N * 8, cudaMemcpyDeviceToHost, L.stream));
    OFC_CUDA(cudaMemcpyAsync(ouy, o2 + N, N * 8, cudaMemcpyDeviceToHost, L.stream));
    OFC_CUDA(cudaMemcpyAsync(energy, en, N * 8, cudaMemcpyDeviceToHost, L.stream));
    OFC_CUDA(cudaMemcpyAsync(resid, rs, N * 8, cudaMemcpyDeviceToHost, L.stream));
    if (slope) OFC_CUDA(cudaMemcpyAsync(slope, sl, 4 * N * 8, cudaMemcpyDeviceToHost, L.stream));
    OFC_CUDA(cudaStreamSynchronize(L.stream));
  });
}

int ofc_test_median(ofc_engine* e, const double* v, size_t n, double* median, char* err, size_t errlen) {
  return guarded(e, err, errlen, [&](Lane& L) {
    if (n == 0) throw Error(OFC_ERR_ARG, "empty");
    double* d = L.upload("t_med", v, n);
    EnergyStats* stats = L.get<EnergyStats>("stats", 1);
    unsigned long long* hist = L.get<unsigned long long>("hist", median_scratch(n));
    OFC_CUDA(cudaMemsetAsync(hist, 0, 4096 * sizeof(unsigned long long), L.stream));
    launch_energy_median(d, n, stats, true, hist, L.stream);
    EnergyStats hs;
    OFC_CUDA(cudaMemcpyAsync(&hs, stats, sizeof(hs), cudaMemcpyDeviceToHost, L.stream));
    OFC_CUDA(cudaStreamSynchronize(L.stream));
    *median = hs.median;
  });
}

int ofc_test_large_components(ofc_engine* e, const uint8_t* b, size_t w, size_t h, double min_area, uint8_t* out,
                              char* err, size_t errlen) {
  return guarded(e, err, errlen, [&](Lane& L) {
    const size_t N = w * h;
    uint8_t* d = L.upload("t_cc", b, N);
    uint8_t* o = L.get<uint8_t>("fin_big", N);
    int* parent = L.get<int>("fin_parent", N);
    int* size = L.get<int>("fin_size", N);
    launch_large_components(d, (int)w, (int)h, min_area, parent, size, o, L.stream);
    OFC_CUDA(cudaMemcpyAsync(out, o, N, cudaMemcpyDeviceToHost, L.stream));
    OFC_CUDA(cudaStreamSynchronize(L.stream));
  });
}

int ofc_test_poc_peaks(ofc_engine* e, const float* a, const float* b, size_t w, size_t h, const ofc_config* c,
                       int level, int32_t* ipk, size_t cap, int32_t* nx, int32_t* ny, char* err, size_t errlen) {
  return guarded(e, err, errlen, [&](Lane& L) {
    cfg_check(c);
    check_sizes(w, h);
    if (!a || !b || !ipk || !nx || !ny) throw Error(OFC_ERR_ARG, "null argument");
    const size_t N = w * h;
    float* da = L.upload("in_i1", a, N);
    float* db = L.upload("in_i2", b, N);
    CoarseOut g = coarse_dev(L, da, db, (int)w, (int)h, nullptr, *c);
    if (level < 0 || level >= (int)g.ipk.size())
      throw Error(OFC_ERR_ARG, "pyramid level " + std::to_string(level) + " does not exist");
    const size_t n = (size_t)g.lnx[level] * g.lny[level];
    if (2 * n > cap) throw Error(OFC_ERR_ARG, "ipk holds fewer than 2 * nx * ny values");
    OFC_CUDA(cudaMemcpyAsync(ipk, g.ipk[level], 2 * n * sizeof(int), cudaMemcpyDeviceToHost, L.stream));
    OFC_CUDA(cudaStreamSynchronize(L.stream));
    *nx = g.lnx[level];
    *ny = g.lny[level];
  });
}

}  // extern "C"
namespace {
__global__ void k_test_atan2(const float* __restrict__ y, const float* __restrict__ x, size_t n, float* mine,
                             float* cuda) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    mine[i] = atan2_phase(y[i], x[i]);
    cuda[i] = atan2f(y[i], x[i]);
  }
}
}  // namespace
extern "C" {

int ofc_test_atan2(ofc_engine* e, const float* y, const float* x, size_t n, float* mine, float* cuda, char* err,
                   size_t errlen) {
  return guarded(e, err, errlen, [&](Lane& L) {
    if (n == 0) return;
    if (!y || !x || !mine || !cuda) throw Error(OFC_ERR_ARG, "null argument");
    const float* dy = L.upload("t_at_y", y, n);
    const float* dx = L.upload("t_at_x", x, n);
    float* dm = L.get<float>("t_at_m", n);
    float* dc = L.get<float>("t_at_c", n);
    OFC_LAUNCH(k_test_atan2, 296, 256, 0, L.stream, dy, dx, n, dm, dc);
    OFC_CUDA(cudaMemcpyAsync(mine, dm, n * 4, cudaMemcpyDeviceToHost, L.stream));
    OFC_CUDA(cudaMemcpyAsync(cuda, dc, n * 4, cudaMemcpyDeviceToHost, L.stream));
    OFC_CUDA(cudaStreamSynchronize(L.stream));
  });
}

int ofc_test_warp(ofc_engine* e, const float* c2, size_t w2, size_t h2, const double* sx, const double* sy, long shx,
                  long shy, size_t w, size_t h, int mode, float* out, uint32_t* timeouts, char* err, size_t errlen) {
  return guarded(e, err, errlen, [&](Lane& L) {
    check_sizes(w2, h2);
    check_sizes(w, h);
    if (!c2 || !sx || !sy || !out) throw Error(OFC_ERR_ARG, "null argument");
    const size_t N = w * h;
    float* dc = L.upload("t_warp_c2", c2, w2 * h2);
    double* dsx = L.upload("t_warp_sx", sx, N);
    double* dsy = L.upload("t_warp_sy", sy, N);
    float* o = L.get<float>("t_warp_out", N);
    unsigned* tmo = L.get<unsigned>("t_warp_timeouts", 1);
    OFC_CUDA(cudaMemsetAsync(tmo, 0, sizeof(unsigned), L.stream));
    launch_warp_mode(mode, dc, (int)w2, (int)h2, dsx, dsy, shx, shy, (int)w, (int)h, o, tmo, L.stream);
    OFC_CUDA(cudaMemcpyAsync(out, o, N * sizeof(float), cudaMemcpyDeviceToHost, L.stream));
    unsigned th = 0;
    OFC_CUDA(cudaMemcpyAsync(&th, tmo, sizeof(unsigned), cudaMemcpyDeviceToHost, L.stream));
    OFC_CUDA(cudaStreamSynchronize(L.stream));
    if (timeouts) *timeouts = th;
  });
}

int ofc_test_prewarp_fill(ofc_engine* e, const uint8_t* low, const double* ux, const double* uy, const double* slope,
                          size_t w, size_t h, double radius, double* oux, double* ouy, char* err, size_t errlen) {
  return guarded(e, err, errlen, [&](Lane& L) {
    const size_t N = w * h;
    const int W = (int)w, H = (int)h;
    uint8_t* dl = L.upload("t_low", low, N);
    double* u2 = L.get<double>("u2", 2 * N);
    OFC_CUDA(cudaMemcpyAsync(u2, ux, N * 8, cudaMemcpyHostToDevice, L.stream));
    OFC_CUDA(cudaMemcpyAsync(u2 + N, uy, N * 8, cudaMemcpyHostToDevice, L.stream));
    double* sl = L.upload("slope", slope, 4 * N);
    PrewarpCounts* counts = L.get<PrewarpCounts>("pw_counts", 2);
    int nlow = 0;
    for (size_t i = 0; i < N; i++) nlow += low[i] ? 1 : 0;
    OFC_CUDA(cudaMemcpyAsync(&counts[0].low, &nlow, sizeof(int), cudaMemcpyHostToDevice, L.stream));
    uint8_t* okm = L.get<uint8_t>("okmask", N);
    int* vdist = L.get<int>("vdist", N);
    int* cold2 = L.get<int>("col_d2", N);
    int* colrow = L.get<int>("col_row", N);
    double* pre2 = L.get<double>("pre2", 2 * N);
    launch_prewarp_fill(dl, u2, u2 + N, sl, W, H, radius, &counts[0], okm, vdist, cold2, colrow, pre2, pre2 + N,
                        L.stream);
    OFC_CUDA(cudaMemcpyAsync(oux, pre2, N * 8, cudaMemcpyDeviceToHost, L.stream));
    OFC_CUDA(cudaMemcpyAsync(ouy, pre2 + N, N * 8, cudaMemcpyDeviceToHost, L.stream));
    OFC_CUDA(cudaStreamSynchronize(L.stream));
  });
}

// refine's first inner-iteration sums from the start field (ux, uy) with the accumulate in `mode` (0: the gather
// kernel, 1: the TMA-staged kernel); *timeouts: its stage waits that gave up
static int first_sums(ofc_engine* e, const float* i1, const float* i2, size_t w, size_t h, const double* ux,
                      const double* uy, const ofc_config* c, int mode, double* sums, uint32_t* timeouts, char* err,
                      size_t errlen) {
  return guarded(e, err, errlen, [&](Lane& L) {
    cfg_check(c);
    check_fine_window(w, h, *c);
    const int W = (int)w, H = (int)h, ph = H + 2 * PAD, pw = W + 2 * PAD, F = c->n_scales * c->n_orient;
    const size_t N = w * h, Np = (size_t)ph * pw;
    cudaStream_t st = L.stream;
    GaborTables g = upload_gabor(L, ph, pw, *c);
    float* d1 = L.upload("in_i1", i1, N);
    float* d2 = L.upload("in_i2", i2, N);
    double* u2 = L.get<double>("u2", 2 * N);
    OFC_CUDA(cudaMemcpyAsync(u2, ux, N * 8, cudaMemcpyHostToDevice, st));
    OFC_CUDA(cudaMemcpyAsync(u2 + N, uy, N * 8, cudaMemcpyHostToDevice, st));
    float2* T = L.get<float2>("fft_T", Np);
    float2* U = L.get<float2>("fft_U", Np * F);
    float4* ref4 = L.get<float4>("ref4", N * F);
    float* amp = L.get<float>("ref_amp", N * F);
    reference_pack(L, d1, W, H, g, ref4, amp, L.stream);
    float* c2 = L.get<float>("spline2", N);
    double* tmp2 = L.get<double>("spline2_tmp", 2 * N);
    launch_bspline_f32(d2, c2, tmp2, W, H, st);
    std::vector<double> ks = gauss_kernel(c->sigma_s);
    double* d_ks = L.upload("taps_s", ks.data(), ks.size());
    double* s2 = L.get<double>("s2", 2 * N);
    double* cs2 = L.get<double>("cs2", 2 * N);
    double* tmpb = L.get<double>("blur_tmp", 2 * N);
    launch_corr_y(u2, tmpb, 2, W, H, d_ks, (int)ks.size() / 2, st);
    launch_corr_x(tmpb, s2, 2, W, H, d_ks, (int)ks.size() / 2, st);
    float* warped = L.get<float>("warped", N);
    launch_warp(c2, W, H, s2, s2 + N, 0, 0, W, H, warped, st);
    float2* R = L.get<float2>("resp", resp_values(F, Np));
    launch_fft_rows_fwd_real(warped, W, H, L.plan(pw), ph, T, st);
    launch_fft_cols_filters(T, L.plan(ph), pw, g, U, st);
    launch_fft_rows_inv_resp(U, L.plan(pw), ph, F, R, st);
    launch_bspline_f64_pair(s2, (double2*)cs2, tmpb, W, H, st);
    double* ds = L.get<double>("sums", 7 * N);
    unsigned* tmo = L.get<unsigned>("t_acc_timeouts", 1);
    OFC_CUDA(cudaMemsetAsync(tmo, 0, sizeof(unsigned), st));
    launch_accumulate_mode(mode, ref4, R, F, ph, pw, u2, u2 + N, s2, s2 + N, (const double2*)cs2, W, H, ds, tmo, st);
    OFC_CUDA(cudaMemcpyAsync(sums, ds, 7 * N * 8, cudaMemcpyDeviceToHost, st));
    unsigned th = 0;
    OFC_CUDA(cudaMemcpyAsync(&th, tmo, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    OFC_CUDA(cudaStreamSynchronize(st));
    if (timeouts) *timeouts = th;
  });
}

int ofc_test_first_sums(ofc_engine* e, const float* i1, const float* i2, size_t w, size_t h, const double* ux,
                        const double* uy, const ofc_config* c, double* sums, char* err, size_t errlen) {
  return first_sums(e, i1, i2, w, h, ux, uy, c, 0, sums, nullptr, err, errlen);
}

int ofc_test_accumulate(ofc_engine* e, const float* i1, const float* i2, size_t w, size_t h, const double* ux,
                        const double* uy, const ofc_config* c, int mode, double* sums, uint32_t* timeouts, char* err,
                        size_t errlen) {
  return first_sums(e, i1, i2, w, h, ux, uy, c, mode, sums, timeouts, err, errlen);
}

int ofc_set_profile(ofc_engine* e, const char* filter) {
  if (!e) return OFC_ERR_ARG;
  try {
    cudaSetDevice(e->device);
    for (auto& l : e->lanes) OFC_CUDA(cudaStreamSynchronize(l->stream));
    if (!filter) {
      if (e->prof) e->prof->resolve();
      e->prof.reset();
      return OFC_OK;
    }
    if (!e->prof) e->prof.reset(new ofc::Profiler());
    e->prof->filter = filter;
    return OFC_OK;
  } catch (const Error& x) {
    return x.status;
  }
}

int ofc_profile_read(ofc_engine* e, char* names, size_t stride, uint64_t* counts, double* ms, size_t cap) {
  if (!e || !e->prof) return -1;
  try {
    cudaSetDevice(e->device);
    std::lock_guard<std::mutex> lk(e->prof->mu);
    e->prof->resolve();
    size_t i = 0;
    for (auto& kv : e->prof->totals) {
      if (i >= cap) break;
      if (names && stride) {
        size_t n = std::min(stride - 1, kv.first.size());
        std::memcpy(names + i * stride, kv.first.data(), n);
        names[i * stride + n] = 0;
      }
      if (counts) counts[i] = kv.second.first;
      if (ms) ms[i] = kv.second.second;
      i++;
    }
    e->prof->totals.clear();
    return (int)i;
  } catch (const Error&) {
    return -1;
  }
}

int ofc_synth_render(ofc_engine* e, const double* bx, const double* by, const double* br, const double* ba, size_t n,
                     size_t w, size_t h, int ss, const ofc_field* field, double* out, char* err, size_t errlen) {
  return guarded(e, err, errlen, [&](Lane& L) {
    check_sizes(w, h);
    if (ss < 1 || ss > 16) throw Error(OFC_ERR_ARG, "ss must lie in [1, 16]");
    launch_synth_render(L, bx, by, br, ba, n, (int)w, (int)h, ss, field, out);
  });
}

// ---------------------------------------------------------------- learned coarse proposal
static void drop_graphs(Lane& l) {
  for (auto& a : l.aux) drop_graphs(*a);
  l.graphs.clear();
}

int ofc_set_coarse_net(ofc_engine* e, const float* params, size_t n, int tile, double max_low_share, char* err,
                       size_t errlen) {
  if (!e) {
    set_err(err, errlen, "null engine");
    return OFC_ERR_ARG;
  }
  // every lane: its graphs hold the old proposal's buffers
  std::vector<std::unique_lock<std::mutex>> locks;
  for (auto& l : e->lanes) {
    std::unique_lock<std::mutex> t(l->busy, std::try_to_lock);
    if (!t.owns_lock()) {
      set_err(err, errlen, "the CUDA engine is busy: the proposal changes only between calls");
      return OFC_ERR_BUSY;
    }
    locks.push_back(std::move(t));
  }
  try {
    OFC_CUDA(cudaSetDevice(e->device));
    std::shared_ptr<Proposal> P;
    if (params) {
      const size_t cnt = net::param_count();
      if (n != cnt) throw Error(OFC_ERR_ARG, "the coarse network takes " + std::to_string(cnt) + " parameters");
      if (tile < 32) throw Error(OFC_ERR_ARG, "fallback tiles must be at least 32 px");
      if (!(max_low_share >= 0.0 && max_low_share <= 1.0)) throw Error(OFC_ERR_ARG, "max_low_share must lie in [0, 1]");
      P = std::make_shared<Proposal>();
      P->tile = tile;
      P->max_low = max_low_share;
      OFC_CUDA(cudaMalloc(&P->params, cnt * sizeof(float)));
      OFC_CUDA(cudaMalloc(&P->w16, cnt * sizeof(uint16_t)));
      OFC_CUDA(cudaMemcpy(P->params, params, cnt * sizeof(float), cudaMemcpyHostToDevice));
      net::Workspace ws{[](const std::string&, size_t) -> void* { return nullptr; }, e->lanes[0]->stream};
      net::to_bf16(ws, P->params, P->w16);
      OFC_CUDA(cudaStreamSynchronize(e->lanes[0]->stream));
    }
    for (auto& l : e->lanes) {
      lane_sync(*l);
      drop_graphs(*l);
      l->proposal = P;
      for (auto& a : l->aux) a->proposal = P;
    }
    return OFC_OK;
  } catch (const Error& x) {
    set_err(err, errlen, x.what());
    return x.status;
  }
}

int ofc_coarse_net_stats(ofc_engine* e, uint64_t* out) {
  if (!e || !out) return OFC_ERR_ARG;
  out[0] = out[1] = out[2] = out[3] = 0;
  const Proposal* P = e->lanes.empty() ? nullptr : e->lanes[0]->proposal.get();
  if (!P) return OFC_OK;
  out[0] = P->pairs;
  out[1] = P->tiles;
  out[2] = P->failed;
  out[3] = P->fallbacks;
  return OFC_OK;
}

// ---------------------------------------------------------------- FFT plan table (autotuner)
int ofc_fft_tune(ofc_engine* e, const int32_t* lengths, size_t n, int lines, int32_t* best, float* ms, char* err,
                 size_t errlen) {
  return guarded(e, err, errlen, [&](Lane& Ln) {
    if (!lengths || !best || lines < 1) throw Error(OFC_ERR_ARG, "null argument or no lines");
    cudaEvent_t e0, e1;
    OFC_CUDA(cudaEventCreate(&e0));
    OFC_CUDA(cudaEventCreate(&e1));
    for (size_t i = 0; i < n; i++) {
      const int L = lengths[i];
      best[i] = 0;
      float bt = INFINITY;
      for (int v = 0; v < FFT_PLAN_VARIANTS; v++) {
        float t = INFINITY;
        const int work = fft_work_length(L);
        if (work > 0 && !(L == FFT_FIXED_L && work == L)) {
          FftPlan pl;
          bool ok = true;
          try {
            pl = fft_make_plan(L, v);
          } catch (const Error&) {
            ok = false;
          }
          if (ok) {
            std::vector<float2> tw = fft_twiddles(fft_work_len(pl));
            const size_t ntw = tw.size();
            if (pl.M) {
              std::vector<float2> bt2 = fft_bluestein_tables(L, pl.M);
              tw.insert(tw.end(), bt2.begin(), bt2.end());
            }
            float2* dtw = Ln.upload("tune_tw", tw.data(), tw.size());
            pl.tw = dtw;
            if (pl.M) {
              pl.chirp = pl.tw + ntw;
              pl.filt = pl.chirp + L;
            }
            float2* d = Ln.get<float2>("tune_lines", (size_t)lines * L);
            OFC_CUDA(cudaMemsetAsync(d, 0, (size_t)lines * L * sizeof(float2), Ln.stream));
            launch_fft_lines(d, lines, pl, false, Ln.stream);
            std::vector<float> rep;
            for (int r = 0; r < 5; r++) {
              OFC_CUDA(cudaEventRecord(e0, Ln.stream));
              launch_fft_lines(d, lines, pl, false, Ln.stream);
              OFC_CUDA(cudaEventRecord(e1, Ln.stream));
              OFC_CUDA(cudaEventSynchronize(e1));
              float m = 0;
              OFC_CUDA(cudaEventElapsedTime(&m, e0, e1));
              rep.push_back(m);
            }
            std::sort(rep.begin(), rep.end());
            t = rep[rep.size() / 2];
          }
        }
        if (ms) ms[i * FFT_PLAN_VARIANTS + v] = t;
        if (t < bt) {
          bt = t;
          best[i] = v;
        }
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  });
}

int ofc_fft_set_plans(const int32_t* lengths, const int32_t* variants, size_t n) {
  if (n && (!lengths || !variants)) return OFC_ERR_ARG;
  for (size_t i = 0; i < n; i++)
    if (variants[i] < 0 || variants[i] >= FFT_PLAN_VARIANTS) return OFC_ERR_ARG;
  for (size_t i = 0; i < n; i++) fft_set_plan_variant(lengths[i], variants[i]);
  return OFC_OK;
}

int ofc_fft_plan_variants(void) { return FFT_PLAN_VARIANTS; }

}  // extern "C"
