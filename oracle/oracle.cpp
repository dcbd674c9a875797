// oracle.cpp -- CPU restatement, in float64, of optflow-soil's pair path (coarse POC -> dense
// start -> local-phase refinement -> guard + strain).
//
// THIS IS TEST INFRASTRUCTURE. It is the checker of the CUDA engine and the CPU baseline that the
// benchmark times beside it; nothing in the product links, loads or calls it. It restates the
// reference's Python specification (python/optflow_ref/*.py, which the reference's Rust port must
// match to 1e-3 px, rust/README.md:3-5), with every function citing the file:line it follows.
// Its parity is pinned by tests/test_oracle.py against golden vectors written by the reference
// itself (tests/golden/make_golden.py) and against the reference's own fixtures.
//
// Arithmetic is IEEE float64 throughout, like numpy's. The FFT is this file's own mixed-radix
// Stockham transform (numpy's pocketfft is not available to C); its results agree with numpy's to
// rounding. Linear systems are solved by Cholesky (the Rust port's choice, phaseflow.rs:379-455,
// strain.rs:64-112) where numpy uses LU: the same solution to rounding for the SPD systems here.
// Threads: OpenMP over rows/lines; results do not depend on the thread count.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <climits>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>
#include <chrono>
#include <omp.h>

#include "../include/optflow_cuda.h"
#include "../include/optflow_cuda_synth.h"

namespace {

using cd = std::complex<double>;
using std::vector;
const double PI = 3.14159265358979323846;
const double INF = std::numeric_limits<double>::infinity();
const double NaN = std::numeric_limits<double>::quiet_NaN();
const int PAD = 32;               // phaseflow.py:47
const double APERTURE_TOL = 1e-3; // phaseflow.py:50
// round the Gabor responses and the reference pack to float32 storage, as the Rust port stores them
// (phaseflow.rs:988-1173: Complex32 responses, f32 RefPack); off by default (float64 like the Python)
bool g_f32_storage = false;

template <class T>
struct Img {
  int w = 0, h = 0;
  vector<T> d;
  Img() {}
  Img(int w_, int h_, T v = T()) : w(w_), h(h_), d((size_t)w_ * h_, v) {}
  T& operator()(int x, int y) { return d[(size_t)y * w + x]; }
  const T& operator()(int x, int y) const { return d[(size_t)y * w + x]; }
  size_t n() const { return d.size(); }
};
using ImgD = Img<double>;
using ImgC = Img<cd>;
using ImgB = Img<uint8_t>;

// ------------------------------------------------------------------ config (config.py:247-272)
double auto_edge_guard_px(const ofc_config& c) {
  double m = 0;
  for (int i = 0; i < c.n_scales; i++) m = std::max(m, c.scales[i]);
  return 3.0 * c.lam * m / (2 * PI * c.bandwidth);
}
double edge_guard_px(const ofc_config& c) { return c.edge_guard >= 0 ? c.edge_guard : auto_edge_guard_px(c); }
double edge_guard_min_area_px(const ofc_config& c) {
  if (c.edge_guard_min_area >= 0) return c.edge_guard_min_area;
  double m = 0;
  for (int i = 0; i < c.n_scales; i++) m = std::max(m, c.scales[i]);
  return 2.0 * (c.lam * m) * (c.lam * m);
}

// ------------------------------------------------------------------ FFT
// numpy.fft conventions: forward sum x[t] exp(-2 pi i k t / n), inverse with +i and 1/n.
// Mixed-radix Stockham (decimation in frequency): stage of radix p on the remaining length `len`
// with stride s: y[r + s(pq + k)] = w_len^{kq} sum_j x[r + s(q + mj)] w_p^{jk}, m = len / p.
struct Fft1 {
  int n = 0;
  vector<int> fac;
  vector<cd> W;  // W[t] = exp(-2 pi i t / n)
  explicit Fft1(int n_) : n(n_) {
    int m = n;
    while (m % 4 == 0) { fac.push_back(4); m /= 4; }
    while (m % 2 == 0) { fac.push_back(2); m /= 2; }
    for (int p = 3; (long)p * p <= m; p += 2)
      while (m % p == 0) { fac.push_back(p); m /= p; }
    if (m > 1) fac.push_back(m);
    W.resize(n);
    for (int t = 0; t < n; t++) {
      // angle reduced to [0, pi/4]-symmetric evaluation is unnecessary at float64: sin/cos of
      // 2 pi t / n with t < n is accurate to an ulp
      double a = -2.0 * PI * (double)t / (double)n;
      W[t] = cd(std::cos(a), std::sin(a));
    }
  }
  // in place; tmp must hold n values
  void run(cd* x, cd* tmp, bool inverse) const {
    if (n == 1) return;
    cd* a = x;
    cd* b = tmp;
    int s = 1, len = n;
    vector<cd> in(64), dft;
    for (int p : fac) {
      int m = len / p;
      if ((int)in.size() < p) in.resize(p);
      // p-point DFT matrix of this radix
      dft.assign((size_t)p * p, cd());
      for (int j = 0; j < p; j++)
        for (int k = 0; k < p; k++) {
          cd v = W[(size_t)((long)j * k % p) * (n / p)];
          dft[(size_t)j * p + k] = inverse ? std::conj(v) : v;
        }
      for (int q = 0; q < m; q++) {
        for (int k = 0; k < p; k++) {
          cd tw = W[(size_t)((long)k * q * s % n)];
          if (inverse) tw = std::conj(tw);
          for (int r = 0; r < s; r++) {
            cd acc = 0;
            for (int j = 0; j < p; j++) acc += a[r + (size_t)s * (q + (size_t)m * j)] * dft[(size_t)j * p + k];
            b[r + (size_t)s * ((size_t)p * q + k)] = acc * tw;
          }
        }
      }
      std::swap(a, b);
      s *= p;
      len = m;
    }
    if (a != x) std::copy(a, a + n, x);
    if (inverse) {
      double sc = 1.0 / n;
      for (int i = 0; i < n; i++) x[i] *= sc;
    }
  }
};

// 2-D transform of an h x w row-major array (numpy fft2 / ifft2: axis 1 then axis 0; the order
// of the separable passes changes only rounding).
void fft2(ImgC& a, bool inverse) {
  Fft1 fr(a.w), fc(a.h);
#pragma omp parallel
  {
    vector<cd> tmp(std::max(a.w, a.h)), col(a.h);
#pragma omp for schedule(static)
    for (int y = 0; y < a.h; y++) fr.run(&a.d[(size_t)y * a.w], tmp.data(), inverse);
#pragma omp for schedule(static)
    for (int x = 0; x < a.w; x++) {
      for (int y = 0; y < a.h; y++) col[y] = a(x, y);
      fc.run(col.data(), tmp.data(), inverse);
      for (int y = 0; y < a.h; y++) a(x, y) = col[y];
    }
  }
}

// np.fft.fftfreq(n) * 2 * pi (numpy multiplies the integers by 1/n)
vector<double> fftfreq2pi(int n) {
  vector<double> f(n);
  double val = 1.0 / n;
  int N = (n - 1) / 2 + 1;
  for (int i = 0; i < n; i++) {
    double k = i < N ? i : i - n;
    f[i] = k * val * 2 * PI;
  }
  return f;
}

// ------------------------------------------------------------------ interp (interp.py)
const double Z = std::sqrt(3.0) - 2.0;
const int HORIZON = (int)std::ceil(std::log(1e-12) / std::log(std::fabs(std::sqrt(3.0) - 2.0)));  // 21

// _prefilter_axis0 along one line with stride (interp.py:13-27)
template <class T>
void prefilter_line(T* c, size_t n, size_t stride) {
  if (n == 1) return;
  const double z = Z;
  for (size_t i = 0; i < n; i++) c[i * stride] *= 6.0;
  size_t hz = std::min<size_t>(n, HORIZON);
  T s = T(0);
  for (size_t k = 0; k < hz; k++) s += std::pow(z, (double)k) * c[k * stride];
  c[0] = s;
  for (size_t i = 1; i < n; i++) c[i * stride] += z * c[(i - 1) * stride];
  c[(n - 1) * stride] = (z / (z * z - 1.0)) * (c[(n - 1) * stride] + z * c[(n - 2) * stride]);
  for (size_t i = n - 1; i-- > 0;) c[i * stride] = z * (c[(i + 1) * stride] - c[i * stride]);
}

// bspline_coeffs (interp.py:30-35): axis 0 (columns, along y), then axis 1 (rows)
template <class T>
void bspline_inplace(Img<T>& c) {
#pragma omp parallel for schedule(static)
  for (int x = 0; x < c.w; x++) prefilter_line(&c.d[x], c.h, c.w);
#pragma omp parallel for schedule(static)
  for (int y = 0; y < c.h; y++) prefilter_line(&c.d[(size_t)y * c.w], c.w, 1);
}

inline long mirror(long i, long n) {  // interp.py:38-43
  if (n == 1) return 0;
  long p = 2 * (n - 1);
  i = std::labs(i) % p;
  return i >= n ? p - i : i;
}

inline void weights(double t, double w[4]) {  // interp.py:46-49
  double t2 = t * t, t3 = t2 * t;
  w[0] = (1 - t) * (1 - t) * (1 - t) / 6;
  w[1] = (3 * t3 - 6 * t2 + 4) / 6;
  w[2] = (-3 * t3 + 3 * t2 + 3 * t + 1) / 6;
  w[3] = t3 / 6;
}

// sample (interp.py:52-69): clamp, 4x4 taps with mirrored indices
template <class T>
T sample(const Img<T>& c, double x, double y) {
  if (std::isnan(x) || std::isnan(y)) return T(NaN);
  x = std::min(std::max(x, 0.0), c.w - 1.0);
  y = std::min(std::max(y, 0.0), c.h - 1.0);
  double fx = std::floor(x), fy = std::floor(y);
  long x0 = (long)fx, y0 = (long)fy;
  double wx[4], wy[4];
  weights(x - fx, wx);
  weights(y - fy, wy);
  long xi[4];
  for (int k = 0; k < 4; k++) xi[k] = mirror(x0 + k - 1, c.w);
  T out = T(0);
  for (int j = 0; j < 4; j++) {
    long yi = mirror(y0 + j - 1, c.h);
    const T* row = &c.d[(size_t)yi * c.w];
    T acc = wx[0] * row[xi[0]];
    for (int k = 1; k < 4; k++) acc = acc + wx[k] * row[xi[k]];
    out += wy[j] * acc;
  }
  return out;
}

vector<double> gauss_kernel(double sigma) {  // interp.py:79-83
  int r = (int)(4.0 * sigma + 0.5);
  vector<double> k(2 * r + 1);
  double s = 0;
  for (int i = -r; i <= r; i++) {
    double t = i / sigma;
    k[i + r] = std::exp(-0.5 * t * t);
  }
  for (double v : k) s += v;
  for (double& v : k) v /= s;
  return k;
}

// scipy.ndimage.correlate1d along one axis; mode "nearest" (edge replicated) or "constant" (0)
void correlate1d(const ImgD& in, ImgD& out, const vector<double>& k, int axis, bool nearest) {
  int r = (int)k.size() / 2;
  out = ImgD(in.w, in.h);
  int W = in.w, H = in.h;
#pragma omp parallel for schedule(static)
  for (int y = 0; y < H; y++)
    for (int x = 0; x < W; x++) {
      double s = 0;
      for (int j = -r; j <= r; j++) {
        int xx = x, yy = y;
        if (axis == 0) yy += j; else xx += j;
        double v;
        if (nearest) {
          xx = std::min(std::max(xx, 0), W - 1);
          yy = std::min(std::max(yy, 0), H - 1);
          v = in(xx, yy);
        } else {
          v = (xx < 0 || yy < 0 || xx >= W || yy >= H) ? 0.0 : in(xx, yy);
        }
        s += k[j + r] * v;
      }
      out(x, y) = s;
    }
}

ImgD gauss_blur(const ImgD& a, double sigma) {  // interp.py:86-92
  vector<double> k = gauss_kernel(sigma);
  ImgD t, o;
  correlate1d(a, t, k, 0, true);
  correlate1d(t, o, k, 1, true);
  return o;
}

// ------------------------------------------------------------------ EDT (scipy semantics)
// 1-D lower envelope of parabolas (Felzenszwalb-Huttenlocher); infinite entries are skipped. On a
// tie the parabola with the smaller position wins: with the pass along y first this gives scipy
// 1.18's feature transform rule, the nearest source with the smallest (d^2, column, row)
// (rust/crates/optflow-core/src/edt.rs:167-183 documents and pins the same rule).
struct Env {
  vector<double> f, z;
  vector<int> v;
  void resize(int n) { f.assign(n, INF); z.assign(n + 1, 0); v.assign(n, 0); }
  bool build() {
    int n = (int)f.size(), k = 0;
    bool any = false;
    for (int q = 0; q < n; q++) {
      if (std::isinf(f[q])) continue;
      if (!any) { any = true; v[0] = q; z[0] = -INF; z[1] = INF; continue; }
      double qf = q;
      for (;;) {
        int p = v[k];
        double pf = p;
        double s = ((f[q] + qf * qf) - (f[p] + pf * pf)) / (2.0 * (qf - pf));
        if (s <= z[k]) { k--; }
        else { k++; v[k] = q; z[k] = s; z[k + 1] = INF; break; }
      }
    }
    return any;
  }
  // out[q] = min_p (q-p)^2 + f[p], src[q] = argmin (ties: smaller p)
  void read(double* out, int* src) const {
    int n = (int)f.size(), k = 0;
    for (int q = 0; q < n; q++) {
      while (z[k + 1] < (double)q) k++;
      double d = (double)q - v[k];
      out[q] = d * d + f[v[k]];
      if (src) src[q] = v[k];
    }
  }
};

// squared distance from every pixel to the nearest pixel with `zero[p]` set
// (scipy distance_transform_edt of an input that is nonzero where zero[p] is false)
ImgD sqdist_to(const ImgB& zero) {
  int W = zero.w, H = zero.h;
  ImgD cold(W, H, INF), out(W, H, INF);
#pragma omp parallel
  {
    Env e;
    vector<double> tmp(std::max(W, H));
#pragma omp for schedule(static)
    for (int x = 0; x < W; x++) {
      e.resize(H);
      for (int y = 0; y < H; y++) e.f[y] = zero(x, y) ? 0.0 : INF;
      if (e.build()) { e.read(tmp.data(), nullptr); for (int y = 0; y < H; y++) cold(x, y) = tmp[y]; }
    }
#pragma omp for schedule(static)
    for (int y = 0; y < H; y++) {
      e.resize(W);
      for (int x = 0; x < W; x++) e.f[x] = cold(x, y);
      if (e.build()) { e.read(tmp.data(), nullptr); for (int x = 0; x < W; x++) out(x, y) = tmp[x]; }
    }
  }
  return out;
}

// feature transform: index (y * W + x) of the nearest source pixel (scipy
// distance_transform_edt(~src, return_indices=True)); src must have a pixel set
vector<int64_t> nearest_source(const ImgB& src) {
  int W = src.w, H = src.h;
  ImgD cold(W, H, INF);
  Img<int> crow(W, H, 0);
  vector<int64_t> out((size_t)W * H, 0);
#pragma omp parallel
  {
    Env e;
    vector<double> tmp(std::max(W, H));
    vector<int> idx(std::max(W, H));
#pragma omp for schedule(static)
    for (int x = 0; x < W; x++) {
      e.resize(H);
      for (int y = 0; y < H; y++) e.f[y] = src(x, y) ? 0.0 : INF;
      if (e.build()) {
        e.read(tmp.data(), idx.data());
        for (int y = 0; y < H; y++) { cold(x, y) = tmp[y]; crow(x, y) = idx[y]; }
      }
    }
#pragma omp for schedule(static)
    for (int y = 0; y < H; y++) {
      e.resize(W);
      for (int x = 0; x < W; x++) e.f[x] = cold(x, y);
      e.build();
      e.read(tmp.data(), idx.data());
      for (int x = 0; x < W; x++) {
        int c = idx[x];
        out[(size_t)y * W + x] = (int64_t)crow(c, y) * W + c;
      }
    }
  }
  return out;
}

// pixels of 4-connected components of `b` with at least min_area pixels (track.py:45-53)
ImgB large_components(const ImgB& b, double min_area) {
  int W = b.w, H = b.h;
  ImgB out(W, H, 0), seen(W, H, 0);
  vector<int64_t> comp;
  for (int64_t s = 0; s < (int64_t)W * H; s++) {
    if (!b.d[s] || seen.d[s]) continue;
    seen.d[s] = 1;
    comp.clear();
    comp.push_back(s);
    for (size_t i = 0; i < comp.size(); i++) {
      int64_t p = comp[i];
      int x = (int)(p % W), y = (int)(p / W);
      auto visit = [&](int64_t q) { if (b.d[q] && !seen.d[q]) { seen.d[q] = 1; comp.push_back(q); } };
      if (x > 0) visit(p - 1);
      if (x + 1 < W) visit(p + 1);
      if (y > 0) visit(p - W);
      if (y + 1 < H) visit(p + W);
    }
    if ((double)comp.size() >= min_area)
      for (int64_t p : comp) out.d[p] = 1;
  }
  return out;
}

double median(vector<double> v) {  // np.median (even count: mean of the two middle values)
  size_t n = v.size();
  if (n == 0) return NaN;
  for (double x : v) if (std::isnan(x)) return NaN;
  size_t m = n / 2;
  std::nth_element(v.begin(), v.begin() + m, v.end());
  double hi = v[m];
  if (n % 2) return hi;
  double lo = *std::max_element(v.begin(), v.begin() + m);
  return (lo + hi) / 2.0;
}

// ------------------------------------------------------------------ phaseflow (phaseflow.py)
struct Bank {  // gabor_bank (phaseflow.py:73-89)
  int h, w;
  vector<double> fx, fy;
  vector<ImgD> G;
};

Bank gabor_bank(int h, int w, const ofc_config& c) {
  Bank b;
  b.h = h; b.w = w;
  b.fy = fftfreq2pi(h);
  b.fx = fftfreq2pi(w);
  double smax = 0;
  for (int i = 0; i < c.n_scales; i++) smax = std::max(smax, c.scales[i]);
  double s_hp = c.dc_cut * c.lam * smax / (2 * PI);
  ImgD hp(w, h);
  for (int y = 0; y < h; y++)
    for (int x = 0; x < w; x++) {
      double r2 = b.fx[x] * b.fx[x] + b.fy[y] * b.fy[y];
      hp(x, y) = 1.0 - std::exp(-r2 * (s_hp * s_hp) / 2);
    }
  for (int si = 0; si < c.n_scales; si++) {
    double w0 = 2 * PI / (c.lam * c.scales[si]);
    double s = c.bandwidth * w0;
    for (int k = 0; k < c.n_orient; k++) {
      double th = PI * k / c.n_orient;
      double cx = w0 * std::cos(th), cy = w0 * std::sin(th);
      ImgD g(w, h);
      for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
          double dx = b.fx[x] - cx, dy = b.fy[y] - cy;
          g(x, y) = hp(x, y) * std::exp(-(dx * dx + dy * dy) / (2 * s * s));
        }
      b.G.push_back(std::move(g));
    }
  }
  return b;
}

// reflect pad by PAD (np.pad mode "reflect" = the mirror of interp.py:38)
ImgC pad_reflect(const ImgD& a) {
  ImgC p(a.w + 2 * PAD, a.h + 2 * PAD);
#pragma omp parallel for schedule(static)
  for (int y = 0; y < p.h; y++)
    for (int x = 0; x < p.w; x++) p(x, y) = a((int)mirror(x - PAD, a.w), (int)mirror(y - PAD, a.h));
  return p;
}

struct RefK {  // reference_phase (phaseflow.py:100-111), per filter
  ImgC r;
  ImgD gx, gy, amp;
};

vector<RefK> reference_phase(const ImgD& I1, const Bank& b) {
  ImgC F = pad_reflect(I1);
  fft2(F, false);
  int W = I1.w, H = I1.h;
  vector<RefK> out(b.G.size());
  for (size_t k = 0; k < b.G.size(); k++) {
    ImgC P(F.w, F.h), Px(F.w, F.h), Py(F.w, F.h);
    for (int y = 0; y < F.h; y++)
      for (int x = 0; x < F.w; x++) {
        cd p = F(x, y) * b.G[k](x, y);
        P(x, y) = p;
        Px(x, y) = (p * cd(0, 1)) * b.fx[x];
        Py(x, y) = (p * cd(0, 1)) * b.fy[y];
      }
    fft2(P, true);
    fft2(Px, true);
    fft2(Py, true);
    RefK& o = out[k];
    o.r = ImgC(W, H); o.gx = ImgD(W, H); o.gy = ImgD(W, H); o.amp = ImgD(W, H);
    for (int y = 0; y < H; y++)
      for (int x = 0; x < W; x++) {
        cd r = P(x + PAD, y + PAD), rx = Px(x + PAD, y + PAD), ry = Py(x + PAD, y + PAD);
        double a2 = std::norm(r) + 1e-12;
        o.r(x, y) = r;
        o.gx(x, y) = std::imag(std::conj(r) * rx) / a2;
        o.gy(x, y) = std::imag(std::conj(r) * ry) / a2;
        o.amp(x, y) = std::sqrt(a2);
        if (g_f32_storage) {
          o.r(x, y) = cd((float)r.real(), (float)r.imag());
          o.gx(x, y) = (float)o.gx(x, y);
          o.gy(x, y) = (float)o.gy(x, y);
          o.amp(x, y) = (float)o.amp(x, y);
        }
      }
  }
  return out;
}

// window_moment (phaseflow.py:114-120): Gaussian window times offset powers, edges replicated
ImgD window_moment(const ImgD& a, double sigma, int px, int py) {
  vector<double> k = gauss_kernel(sigma);
  int r = (int)k.size() / 2;
  vector<double> ky(k.size()), kx(k.size());
  for (int i = -r; i <= r; i++) {
    ky[i + r] = k[i + r] * std::pow((double)i, py);
    kx[i + r] = k[i + r] * std::pow((double)i, px);
  }
  ImgD t, o;
  correlate1d(a, t, ky, 0, true);
  correlate1d(t, o, kx, 1, true);
  return o;
}

struct Unk { int c, px, py; };
vector<Unk> shape_unknowns(int order) {  // phaseflow.py:123-129
  vector<std::pair<int, int>> pw = {{0, 0}, {1, 0}, {0, 1}};
  if (order == 2) pw = {{0, 0}, {1, 0}, {0, 1}, {2, 0}, {1, 1}, {0, 2}};
  vector<Unk> u = {{0, pw[0].first, pw[0].second}, {1, pw[0].first, pw[0].second}};
  for (size_t i = 1; i < pw.size(); i++)
    for (int c = 0; c < 2; c++) u.push_back({c, pw[i].first, pw[i].second});
  return u;
}

// Cholesky solve of an SPD n x n system (lower triangle read); false on a non-positive pivot or
// a non-finite solution (phaseflow.rs:394-455)
bool cholesky_solve(vector<double>& M, vector<double>& b, int n) {
  for (int j = 0; j < n; j++) {
    double d = M[j * n + j];
    for (int k = 0; k < j; k++) d -= M[j * n + k] * M[j * n + k];
    if (!(std::isfinite(d) && d > 0)) return false;
    double l = std::sqrt(d);
    M[j * n + j] = l;
    for (int i = j + 1; i < n; i++) {
      double s = M[i * n + j];
      for (int k = 0; k < j; k++) s -= M[i * n + k] * M[j * n + k];
      M[i * n + j] = s / l;
    }
  }
  for (int i = 0; i < n; i++) {
    double s = b[i];
    for (int k = 0; k < i; k++) s -= M[i * n + k] * b[k];
    b[i] = s / M[i * n + i];
  }
  for (int i = n - 1; i >= 0; i--) {
    double s = b[i];
    for (int k = i + 1; k < n; k++) s -= M[k * n + i] * b[k];
    b[i] = s / M[i * n + i];
  }
  for (int i = 0; i < n; i++) if (!std::isfinite(b[i])) return false;
  return true;
}

struct Solved { ImgD ux, uy, energy, resid; vector<double> slope; };

// local_solve / _solve (phaseflow.py:132-188)
Solved local_solve(const ImgD sums[7], const ImgD& ux, const ImgD& uy, double sigma, int order) {
  int W = ux.w, H = ux.h;
  size_t N = ux.n();
  vector<Unk> unk = shape_unknowns(order);
  int n = (int)unk.size();
  // moments of the products (key 0: gxx, 1: gxy, 2: gyy) and rhs (3: gxc, 4: gyc) by powers
  auto key_of = [](int ci, int cj) { int a = std::min(ci, cj), b = std::max(ci, cj); return a == 0 ? (b == 0 ? 0 : 1) : 2; };
  std::vector<std::vector<ImgD>> cache(5, std::vector<ImgD>(25));
  std::vector<std::vector<char>> have(5, std::vector<char>(25, 0));
  auto mom = [&](int key, int px, int py) -> const ImgD& {
    int slot = px * 5 + py;
    if (!have[key][slot]) { cache[key][slot] = window_moment(sums[key], sigma, px, py); have[key][slot] = 1; }
    return cache[key][slot];
  };
  vector<const ImgD*> Mp((size_t)n * n), bp(n);
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++)
      Mp[(size_t)i * n + j] = &mom(key_of(unk[i].c, unk[j].c), unk[i].px + unk[j].px, unk[i].py + unk[j].py);
  for (int i = 0; i < n; i++) bp[i] = &mom(3 + unk[i].c, unk[i].px, unk[i].py);
  ImgD mgcc = window_moment(sums[5], sigma, 0, 0), mgw = window_moment(sums[6], sigma, 0, 0);
  Solved s;
  s.ux = ImgD(W, H); s.uy = ImgD(W, H); s.energy = ImgD(W, H); s.resid = ImgD(W, H);
  s.slope.assign(N * 4, 0.0);
  vector<double> en(N);
  for (size_t p = 0; p < N; p++) en[p] = (*Mp[0]).d[p] + (*Mp[(size_t)n + 1]).d[p];
  double med = median(en);
  double thr = 1e-9 * med + 1e-30;
#pragma omp parallel
  {
    vector<double> M((size_t)n * n), b(n), b0(n);
#pragma omp for schedule(static)
    for (long pl = 0; pl < (long)N; pl++) {
      size_t p = (size_t)pl;
      double m00 = Mp[0]->d[p], m11 = Mp[(size_t)n + 1]->d[p], m01 = Mp[1]->d[p];
      double e = m00 + m11;
      double det2 = m00 * m11 - m01 * m01;
      s.energy.d[p] = e;
      bool ok = e > thr && det2 > APERTURE_TOL * e * e;
      if (ok) {
        double tr = 0;
        for (int i = 0; i < n; i++) tr += Mp[(size_t)i * n + i]->d[p];
        double ridge = 1e-12 * tr / n;
        for (int i = 0; i < n; i++)
          for (int j = 0; j < n; j++) M[(size_t)i * n + j] = Mp[(size_t)i * n + j]->d[p] + (i == j ? ridge : 0.0);
        for (int i = 0; i < n; i++) b[i] = b0[i] = bp[i]->d[p];
        ok = cholesky_solve(M, b, n);
      }
      if (ok) {
        double fit = 0;
        for (int i = 0; i < n; i++) fit += b[i] * b0[i];
        double r = mgcc.d[p] - fit;
        s.resid.d[p] = std::sqrt(std::max(r, 0.0) / (mgw.d[p] + 1e-30));
        s.ux.d[p] = b[0];
        s.uy.d[p] = b[1];
        for (int i = 0; i < 4; i++) s.slope[p * 4 + i] = b[2 + i];
      } else {
        s.resid.d[p] = PI;
        s.ux.d[p] = ux.d[p];
        s.uy.d[p] = uy.d[p];
      }
    }
  }
  return s;
}

// _confidence (phaseflow.py:320-323), before the border rule
ImgD confidence_raw(const ImgD& energy, const ImgD& resid, const ofc_config& c) {
  double scale = 0.25 * median(energy.d) + 1e-30;
  ImgD out(energy.w, energy.h);
  for (size_t p = 0; p < out.n(); p++) {
    double tex = std::min(1.0, energy.d[p] / scale);
    if (std::isnan(energy.d[p] / scale)) tex = NaN;
    double q = resid.d[p] / c.phase_tol;
    out.d[p] = tex * std::exp(-(q * q));
  }
  return out;
}

// prewarp (phaseflow.py:326-355), with the Rust port's freeze of the low pixels
// (rust/crates/optflow-core/src/prewarp.rs:79-116)
void prewarp(const ImgD& ux0, const ImgD& uy0, const vector<double>& slope, const ImgB& low,
             const ofc_config& c, ImgD& sx, ImgD& sy) {
  int W = ux0.w, H = ux0.h;
  ImgD ux = ux0, uy = uy0;
  bool any_low = false;
  for (uint8_t v : low.d) any_low |= v != 0;
  if (any_low) {
    ImgD d2 = sqdist_to(low);
    double R = auto_edge_guard_px(c);
    ImgB ok(W, H, 0);
    bool any_ok = false, all_ok = true;
    for (size_t p = 0; p < ok.n(); p++) {
      ok.d[p] = std::sqrt(d2.d[p]) > R;
      any_ok |= ok.d[p] != 0;
      all_ok &= ok.d[p] != 0;
    }
    if (any_ok && !all_ok) {
      vector<int64_t> idx = nearest_source(ok);
#pragma omp parallel for schedule(static)
      for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++) {
          size_t p = (size_t)y * W + x;
          if (ok.d[p]) continue;
          int64_t q = idx[p];
          int ix = (int)(q % W), iy = (int)(q / W);
          double dx = (double)x - ix, dy = (double)y - iy;
          const double* g = &slope[(size_t)q * 4];
          ux.d[p] = ux0.d[q] + g[0] * dx + g[2] * dy;
          uy.d[p] = uy0.d[q] + g[1] * dx + g[3] * dy;
        }
    }
  }
  sx = gauss_blur(ux, c.sigma_s);
  sy = gauss_blur(uy, c.sigma_s);
}

// the seven per-pixel sums of one inner iteration (phaseflow.py:468-483)
void accumulate(const vector<RefK>& ref, const vector<ImgC>& resp, const ImgD& sx, const ImgD& sy, const ImgD& csx,
                const ImgD& csy, const ImgD& ux, const ImgD& uy, ImgD sums[7]) {
  int W = ux.w, H = ux.h, F = (int)ref.size();
  for (int i = 0; i < 7; i++) sums[i] = ImgD(W, H, 0.0);
#pragma omp parallel for schedule(static)
  for (int y = 0; y < H; y++)
    for (int x = 0; x < W; x++) {
      size_t p = (size_t)y * W + x;
      double u = ux.d[p], v = uy.d[p];
      double tx = x + u, ty = y + v;
      double px = tx - sx.d[p], py = ty - sy.d[p];
      for (int s = 0; s < 2; s++) {
        double nx = tx - sample(csx, px, py), ny = ty - sample(csy, px, py);
        px = nx; py = ny;
      }
      double a[7] = {0, 0, 0, 0, 0, 0, 0};
      for (int k = 0; k < F; k++) {
        cd r1 = ref[k].r.d[p];
        cd r2 = sample(resp[k], px + PAD, py + PAD);
        double dphi = std::arg(r1 * std::conj(r2));
        double wk = ref[k].amp.d[p] * std::abs(r2);
        double gx = ref[k].gx.d[p], gy = ref[k].gy.d[p];
        double cc = dphi + gx * u + gy * v;
        a[0] += wk * gx * gx; a[1] += wk * gx * gy; a[2] += wk * gy * gy;
        a[3] += wk * gx * cc; a[4] += wk * gy * cc; a[5] += wk * cc * cc;
        a[6] += wk;
      }
      for (int i = 0; i < 7; i++) sums[i].d[p] = a[i];
    }
}

struct RawFlow { ImgD ux, uy, energy, resid; };

// refine (phaseflow.py:427-511) without the crack options, up to the confidence
RawFlow refine_raw(const ImgD& I1, const ImgD& I2, const ImgD& ux_in, const ImgD& uy_in, const ofc_config& c) {
  int W = I1.w, H = I1.h;
  Bank bank = gabor_bank(H + 2 * PAD, W + 2 * PAD, c);
  vector<RefK> ref = reference_phase(I1, bank);
  ImgD c2 = I2;
  bspline_inplace(c2);
  ImgD ux = ux_in, uy = uy_in;
  ImgD resid(W, H, PI), energy(W, H, 1.0);
  vector<double> slope;
  ImgB frozen;
  bool have_frozen = false;
  int F = (int)bank.G.size();
  for (int it = 0; it < c.outer_iters; it++) {
    ImgD sx, sy;
    if (it == 0) {
      sx = gauss_blur(ux, c.sigma_s);
      sy = gauss_blur(uy, c.sigma_s);
    } else {
      ImgB low;
      int K = c.prewarp_freeze_at;
      if (K >= 1 && it > K && have_frozen) {
        low = frozen;
      } else {
        ImgD conf = confidence_raw(energy, resid, c);
        low = ImgB(W, H, 0);
        for (size_t p = 0; p < low.n(); p++) low.d[p] = conf.d[p] < c.conf_min;
        if (K >= 1 && it == K) { frozen = low; have_frozen = true; }
      }
      prewarp(ux, uy, slope, low, c, sx, sy);
    }
    // warp(I2, sx, sy) (interp.py:72-76), reflect pad, forward transform
    ImgD warped(W, H);
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; y++)
      for (int x = 0; x < W; x++) warped(x, y) = sample(c2, x + sx(x, y), y + sy(x, y));
    ImgC F2 = pad_reflect(warped);
    fft2(F2, false);
    vector<ImgC> resp(F);
    for (int k = 0; k < F; k++) {
      ImgC R(F2.w, F2.h);
      for (size_t p = 0; p < R.n(); p++) R.d[p] = F2.d[p] * bank.G[k].d[p];
      fft2(R, true);
      bspline_inplace(R);
      if (g_f32_storage)
        for (cd& v : R.d) v = cd((float)v.real(), (float)v.imag());
      resp[k] = std::move(R);
    }
    ImgD csx = sx, csy = sy;
    bspline_inplace(csx);
    bspline_inplace(csy);
    for (int inner = 0; inner < c.inner_iters; inner++) {
      ImgD sums[7];
      accumulate(ref, resp, sx, sy, csx, csy, ux, uy, sums);
      Solved s = local_solve(sums, ux, uy, c.sigma_w, c.shape_order);
      ux = std::move(s.ux); uy = std::move(s.uy);
      energy = std::move(s.energy); resid = std::move(s.resid);
      slope = std::move(s.slope);
    }
  }
  return RawFlow{ux, uy, energy, resid};
}

double border_width(const ofc_config& c) { return edge_guard_px(c) > 0 ? 4.0 * c.sigma_w : 0.0; }

// the confidence of refine with the border rule (phaseflow.py:297-317,508-510); low = conf < conf_min
void refine_conf(const RawFlow& rf, const ofc_config& c, ImgD& conf) {
  int W = rf.ux.w, H = rf.ux.h;
  conf = confidence_raw(rf.energy, rf.resid, c);
  double B = border_width(c);
  for (int y = 0; y < H; y++)
    for (int x = 0; x < W; x++) {
      double tx = x + rf.ux(x, y), ty = y + rf.uy(x, y);
      double own = std::min(std::min((double)x, (double)y), std::min((double)(W - 1 - x), (double)(H - 1 - y)));
      double mt = std::min(std::min(tx, ty), std::min((W - 1) - tx, (H - 1) - ty));
      bool rep = own >= B && tx >= B && ty >= B && (W - 1) - tx >= B && (H - 1) - ty >= B;
      (void)mt;
      double v = conf(x, y);
      conf(x, y) = rep ? std::min(std::max(v, 0.0), 1.0) : 0.0;
      if (rep && std::isnan(v)) conf(x, y) = NaN;
    }
}

// ------------------------------------------------------------------ POC (poc.py)
struct Grid {
  vector<int> xs, ys;
  ImgD ux, uy, peak;
  // the integer peak of the last correlation surface evaluated at each point: window offset (round(d)) plus the
  // unclamped argmax of the shifted surface minus the half window (poc.py:50 np.argmax); INT_MIN if none was
  vector<int> ipx, ipy;
};

double parabola(double m, double c, double p) {  // poc.py:34-36
  double den = m - 2.0 * c + p;
  return den == 0 ? 0.0 : 0.5 * (m - p) / den;
}

double mean_of(const vector<double>& v) {  // numpy pairwise sum is rounding-level different
  long double s = 0;
  for (double x : v) s += x;
  return (double)(s / v.size());
}

struct PocTables {
  int h, w;
  vector<double> wnd, lp;
  double lpm;
  Fft1 fr, fc;
  PocTables(int h_, int w_) : h(h_), w(w_), fr(w_), fc(h_) {  // poc.py:18-31
    auto hann = [](int n) { vector<double> v(n); for (int i = 0; i < n; i++) v[i] = 0.5 - 0.5 * std::cos(2 * PI * i / n); return v; };
    vector<double> hy = hann(h), hx = hann(w);
    wnd.resize((size_t)h * w);
    lp.resize((size_t)h * w);
    double cnt = 0;
    for (int y = 0; y < h; y++)
      for (int x = 0; x < w; x++) {
        wnd[(size_t)y * w + x] = hy[y] * hx[x];
        int ky = y <= (h - 1) / 2 ? y : y - h, kx = x <= (w - 1) / 2 ? x : x - w;
        double fy = std::fabs(ky * (1.0 / h)), fx = std::fabs(kx * (1.0 / w));
        double m = (fy <= 0.25 && fx <= 0.25) ? 1.0 : 0.0;
        lp[(size_t)y * w + x] = m;
        cnt += m;
      }
    lpm = cnt / ((double)h * w);
  }
  void fft2(vector<cd>& a, bool inv) const {
    vector<cd> tmp(std::max(h, w)), col(h);
    for (int y = 0; y < h; y++) fr.run(&a[(size_t)y * w], tmp.data(), inv);
    for (int x = 0; x < w; x++) {
      for (int y = 0; y < h; y++) col[y] = a[(size_t)y * w + x];
      fc.run(col.data(), tmp.data(), inv);
      for (int y = 0; y < h; y++) a[(size_t)y * w + x] = col[y];
    }
  }
};

// poc_shift (poc.py:39-54): a, b are h x w windows (row-major)
void poc_shift(const PocTables& T, const vector<double>& a, const vector<double>& b, double& dx, double& dy, double& pk,
               size_t* argmax = nullptr) {
  int h = T.h, w = T.w;
  size_t n = (size_t)h * w;
  double ma = mean_of(a), mb = mean_of(b);
  vector<cd> A(n), B(n);
  for (size_t i = 0; i < n; i++) { A[i] = (a[i] - ma) * T.wnd[i]; B[i] = (b[i] - mb) * T.wnd[i]; }
  T.fft2(A, false);
  T.fft2(B, false);
  vector<cd> C(n);
  for (size_t i = 0; i < n; i++) {
    cd c = B[i] * std::conj(A[i]);
    c /= (std::abs(c) + 1e-12);
    C[i] = c * T.lp[i];
  }
  T.fft2(C, true);
  vector<double> r(n);
  for (int y = 0; y < h; y++)
    for (int x = 0; x < w; x++) {
      int sy = ((y - h / 2) % h + h) % h, sxx = ((x - w / 2) % w + w) % w;  // fftshift
      r[(size_t)y * w + x] = std::real(C[(size_t)sy * w + sxx]) / T.lpm;
    }
  size_t best = 0;  // np.argmax: first maximum, a NaN wins
  for (size_t i = 0; i < n; i++) {
    if (std::isnan(r[i])) { best = i; break; }
    if (r[i] > r[best]) best = i;
  }
  if (argmax) *argmax = best;
  int iy = (int)(best / w), ix = (int)(best % w);
  iy = std::min(std::max(iy, 1), h - 2);
  ix = std::min(std::max(ix, 1), w - 2);
  double sx = parabola(r[(size_t)iy * w + ix - 1], r[(size_t)iy * w + ix], r[(size_t)iy * w + ix + 1]);
  double sy = parabola(r[(size_t)(iy - 1) * w + ix], r[(size_t)iy * w + ix], r[(size_t)(iy + 1) * w + ix]);
  dx = ix - w / 2 + sx;
  dy = iy - h / 2 + sy;
  pk = r[(size_t)iy * w + ix];
}

vector<int> arange(int a, int b, int step) { vector<int> v; for (int i = a; i < b; i += step) v.push_back(i); return v; }

void grid_points(int h, int w, int step, int wy, int wx, vector<int>& xs, vector<int>& ys) {  // poc.py:61-64
  xs = arange(wx / 2, w - wx / 2 + 1, step);
  ys = arange(wy / 2, h - wy / 2 + 1, step);
}

// poc_grid (poc.py:67-92)
Grid poc_grid(const ImgD& I1, const ImgD& I2, const vector<int>& xs, const vector<int>& ys, int wy, int wx,
              const ImgD* ix, const ImgD* iy, int iters = 3) {
  int H = I1.h, W = I1.w;
  int hy = wy / 2, hx = wx / 2;
  int ny = (int)ys.size(), nx = (int)xs.size();
  Grid g;
  g.xs = xs; g.ys = ys;
  g.ux = ImgD(nx, ny); g.uy = ImgD(nx, ny); g.peak = ImgD(nx, ny);
  g.ipx.assign((size_t)nx * ny, INT_MIN);
  g.ipy.assign((size_t)nx * ny, INT_MIN);
  PocTables T(wy, wx);
#pragma omp parallel for schedule(dynamic, 4)
  for (int i = 0; i < ny; i++) {
    vector<double> a((size_t)wy * wx), b((size_t)wy * wx);
    for (int j = 0; j < nx; j++) {
      int y = ys[i], x = xs[j];
      double dx = ix ? (*ix)(j, i) : 0.0, dy = iy ? (*iy)(j, i) : 0.0;
      for (int r = 0; r < wy; r++)
        for (int q = 0; q < wx; q++) a[(size_t)r * wx + q] = I1(x - hx + q, y - hy + r);
      double pk = 0.0;
      for (int t = 0; t < iters; t++) {
        long ox = (long)std::nearbyint(dx), oy = (long)std::nearbyint(dy);  // Python round: half to even
        long y0 = y - hy + oy, x0 = x - hx + ox;
        if (y0 < 0 || x0 < 0 || y0 + wy > H || x0 + wx > W) { pk = 0.0; break; }
        for (int r = 0; r < wy; r++)
          for (int q = 0; q < wx; q++) b[(size_t)r * wx + q] = I2((int)(x0 + q), (int)(y0 + r));
        double sx, sy;
        size_t am = 0;
        poc_shift(T, a, b, sx, sy, pk, &am);
        g.ipx[(size_t)i * nx + j] = (int)(ox + (long)(am % wx) - wx / 2);
        g.ipy[(size_t)i * nx + j] = (int)(oy + (long)(am / wx) - wy / 2);
        dx = ox + sx;
        dy = oy + sy;
        if (std::fabs(sx) < 0.5 && std::fabs(sy) < 0.5) break;
      }
      g.ux(j, i) = dx; g.uy(j, i) = dy; g.peak(j, i) = pk;
    }
  }
  return g;
}

// clean (poc.py:95-140)
Grid clean(const Grid& g, double peak_min, double thresh, const ImgD* fbx, const ImgD* fby, int max_pass = 100) {
  ImgD ux = g.ux, uy = g.uy;
  int ny = ux.h, nx = ux.w;
  ImgB valid(nx, ny, 0);
  for (size_t p = 0; p < valid.n(); p++) valid.d[p] = g.peak.d[p] >= peak_min;
  const int offs[8][2] = {{-1, -1}, {-1, 0}, {-1, 1}, {0, -1}, {0, 1}, {1, -1}, {1, 0}, {1, 1}};
  auto neighbours = [&](int i, int j, const ImgB& ok, vector<std::pair<int, int>>& nb) {
    nb.clear();
    for (auto& o : offs) {
      int a = i + o[0], b = j + o[1];
      if (a >= 0 && a < ny && b >= 0 && b < nx && ok(b, a)) nb.push_back({a, b});
    }
  };
  ImgB out = valid;
  vector<std::pair<int, int>> nb;
  vector<double> vals;
  for (int i = 0; i < ny; i++)
    for (int j = 0; j < nx; j++) {
      if (!valid(j, i)) continue;
      neighbours(i, j, valid, nb);
      if (nb.size() < 3) continue;
      for (int comp = 0; comp < 2; comp++) {
        const ImgD& cmp = comp == 0 ? ux : uy;
        vals.clear();
        for (auto& p : nb) vals.push_back(cmp(p.second, p.first));
        double med = median(vals);
        vector<double> dev;
        for (double v : vals) dev.push_back(std::fabs(v - med));
        double res = median(dev);
        if (std::fabs(cmp(j, i) - med) / (res + 0.1) > thresh) out(j, i) = 0;
      }
    }
  bool any = false;
  for (uint8_t v : out.d) any |= v != 0;
  Grid r;
  r.xs = g.xs; r.ys = g.ys;
  if (!any) {
    r.ux = fbx ? *fbx : ImgD(nx, ny, 0.0);
    r.uy = fby ? *fby : ImgD(nx, ny, 0.0);
    r.peak = ImgD(nx, ny, 0.0);
    for (size_t p = 0; p < r.peak.n(); p++) r.peak.d[p] = g.peak.d[p] * 0;
    return r;
  }
  for (int pass = 0; pass < max_pass; pass++) {
    bool all = true;
    for (uint8_t v : out.d) all &= v != 0;
    if (all) break;
    ImgB nw = out;
    for (int i = 0; i < ny; i++)
      for (int j = 0; j < nx; j++) {
        if (out(j, i)) continue;
        neighbours(i, j, out, nb);
        if (nb.empty()) continue;
        vals.clear();
        for (auto& p : nb) vals.push_back(ux(p.second, p.first));
        ux(j, i) = median(vals);
        vals.clear();
        for (auto& p : nb) vals.push_back(uy(p.second, p.first));
        uy(j, i) = median(vals);
        nw(j, i) = 1;
      }
    out = nw;
  }
  r.ux = ux; r.uy = uy;
  r.peak = ImgD(nx, ny, 0.0);
  for (size_t p = 0; p < r.peak.n(); p++) r.peak.d[p] = valid.d[p] ? g.peak.d[p] : 0.0;
  return r;
}

// grid_sample (poc.py:143-161): bilinear, clamped to the grid
void grid_frac(double q, const vector<int>& nodes, double& t, long& i0) {
  if (nodes.size() == 1) { t = 0; i0 = 0; return; }
  double f = (q - nodes[0]) / (double)(nodes[1] - nodes[0]);
  f = std::min(std::max(f, 0.0), (double)(nodes.size() - 1));
  i0 = std::min((long)std::floor(f), (long)nodes.size() - 2);
  t = f - i0;
}
double grid_bil(const ImgD& a, double tx, long x0, double ty, long y0) {
  long x1 = std::min(x0 + 1, (long)a.w - 1), y1 = std::min(y0 + 1, (long)a.h - 1);
  return (1 - ty) * ((1 - tx) * a(x0, y0) + tx * a(x1, y0)) + ty * ((1 - tx) * a(x0, y1) + tx * a(x1, y1));
}

ImgD downsample(const ImgD& img) {  // poc.py:164-165
  ImgD b = gauss_blur(img, 1.0);
  ImgD o((b.w + 1) / 2, (b.h + 1) / 2);
  for (int y = 0; y < o.h; y++)
    for (int x = 0; x < o.w; x++) o(x, y) = b(2 * x, 2 * y);
  return o;
}

int pow2_floor(long n) { if (n < 1) return 0; int b = 0; while ((n >> (b + 1)) > 0) b++; return 1 << b; }

bool level_window(int h, int w, int win, int& wy, int& wx) {  // poc.py:172-187
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

int n_levels(double max_disp, int win, int h, int w) {  // poc.py:190-195
  int L = (int)std::max(0.0, std::ceil(std::log2(std::max(max_disp, 1e-9) / (win / 4.0))));
  int wy, wx;
  while (L > 0 && !level_window(h >> L, w >> L, win, wy, wx)) L--;
  return L;
}

// coarse_flow (poc.py:216-239)
// raw (optional): the uncleaned POC grid of every level, level 0 first
Grid coarse_flow(const ImgD& I1, const ImgD& I2, const ofc_config& c, const ImgD* idx, const ImgD* idy,
                 vector<Grid>* raw_levels = nullptr) {
  int H = I1.h, W = I1.w;
  vector<int> xs, ys;
  grid_points(H, W, c.grid_step, c.poc_win, c.poc_win, xs, ys);
  int L = n_levels(c.max_disp, c.poc_win, H, W);
  vector<std::pair<ImgD, ImgD>> pyr;
  pyr.push_back({I1, I2});
  for (int l = 0; l < L; l++) pyr.push_back({downsample(pyr.back().first), downsample(pyr.back().second)});
  if (raw_levels) raw_levels->assign(L + 1, Grid());
  Grid g;
  bool have = false;
  for (int lev = L; lev >= 0; lev--) {
    const ImgD& a = pyr[lev].first;
    const ImgD& b = pyr[lev].second;
    int wy = c.poc_win, wx = c.poc_win;
    vector<int> gx = xs, gy = ys;
    if (lev != 0) {
      level_window(a.h, a.w, c.poc_win, wy, wx);
      grid_points(a.h, a.w, c.grid_step, wy, wx, gx, gy);
    }
    int nx = (int)gx.size(), ny = (int)gy.size();
    ImgD ix, iy;
    bool has_init = false;
    if (have) {
      ix = ImgD(nx, ny); iy = ImgD(nx, ny);
      for (int i = 0; i < ny; i++)
        for (int j = 0; j < nx; j++) {
          double tx, ty; long x0, y0;
          grid_frac(gx[j] / 2.0, g.xs, tx, x0);
          grid_frac(gy[i] / 2.0, g.ys, ty, y0);
          ix(j, i) = 2.0 * grid_bil(g.ux, tx, x0, ty, y0);
          iy(j, i) = 2.0 * grid_bil(g.uy, tx, x0, ty, y0);
        }
      has_init = true;
    } else if (idx) {
      int sc = 1 << lev;
      ix = ImgD(nx, ny); iy = ImgD(nx, ny);
      for (int i = 0; i < ny; i++)
        for (int j = 0; j < nx; j++) {
          ix(j, i) = (*idx)(gx[j] * sc, gy[i] * sc) / sc;
          iy(j, i) = (*idy)(gx[j] * sc, gy[i] * sc) / sc;
        }
      has_init = true;
    }
    Grid raw = poc_grid(a, b, gx, gy, wy, wx, has_init ? &ix : nullptr, has_init ? &iy : nullptr);
    if (raw_levels) (*raw_levels)[lev] = raw;
    g = clean(raw, c.poc_peak_min, c.median_thresh, has_init ? &ix : nullptr, has_init ? &iy : nullptr);
    have = true;
  }
  return g;
}

// dense start of track_pair (track.py:131-137)
void dense_start(const Grid& g, int W, int H, const ImgD* idx, const ImgD* idy, ImgD& gx, ImgD& gy) {
  gx = ImgD(W, H); gy = ImgD(W, H);
  ImgD cx, cy;
  if (idx) {
    cx = g.ux; cy = g.uy;
    for (size_t i = 0; i < g.ys.size(); i++)
      for (size_t j = 0; j < g.xs.size(); j++) {
        cx((int)j, (int)i) = g.ux((int)j, (int)i) - (*idx)(g.xs[j], g.ys[i]);
        cy((int)j, (int)i) = g.uy((int)j, (int)i) - (*idy)(g.xs[j], g.ys[i]);
      }
  }
#pragma omp parallel for schedule(static)
  for (int y = 0; y < H; y++)
    for (int x = 0; x < W; x++) {
      double tx, ty; long x0, y0;
      grid_frac(x, g.xs, tx, x0);
      grid_frac(y, g.ys, ty, y0);
      if (idx) {
        gx(x, y) = (*idx)(x, y) + grid_bil(cx, tx, x0, ty, y0);
        gy(x, y) = (*idy)(x, y) + grid_bil(cy, tx, x0, ty, y0);
      } else {
        gx(x, y) = grid_bil(g.ux, tx, x0, ty, y0);
        gy(x, y) = grid_bil(g.uy, tx, x0, ty, y0);
      }
    }
}

// ------------------------------------------------------------------ strain (strain.py)
const int BASIS[6][2] = {{0, 0}, {1, 0}, {0, 1}, {2, 0}, {1, 1}, {0, 2}};

void displacement_gradient(const ImgD& ux, const ImgD& uy, int win, ImgD& dudx, ImgD& dudy, ImgD& dvdx, ImgD& dvdy,
                           double min_frac = 0.5) {  // strain.py:61-97
  int W = ux.w, H = ux.h;
  int h = win / 2;
  ImgD m(W, H), u0(W, H), v0(W, H);
  for (size_t p = 0; p < m.n(); p++) {
    bool ok = std::isfinite(ux.d[p]) && std::isfinite(uy.d[p]);
    m.d[p] = ok ? 1.0 : 0.0;
    u0.d[p] = ok ? ux.d[p] : 0.0;
    v0.d[p] = ok ? uy.d[p] : 0.0;
  }
  auto moment = [&](const ImgD& a, int px, int py) {  // strain.py:10-14
    vector<double> ky(2 * h + 1), kx(2 * h + 1);
    for (int t = -h; t <= h; t++) { ky[t + h] = std::pow((double)t, py); kx[t + h] = std::pow((double)t, px); }
    ImgD t1, o;
    correlate1d(a, t1, ky, 0, false);
    correlate1d(t1, o, kx, 1, false);
    return o;
  };
  ImgD Mm[5][5];
  bool have[5][5] = {};
  for (int i = 0; i < 6; i++)
    for (int j = 0; j < 6; j++) {
      int px = BASIS[i][0] + BASIS[j][0], py = BASIS[i][1] + BASIS[j][1];
      if (!have[px][py]) { Mm[px][py] = moment(m, px, py); have[px][py] = true; }
    }
  ImgD ru[6], rv[6];
  for (int i = 0; i < 6; i++) { ru[i] = moment(u0, BASIS[i][0], BASIS[i][1]); rv[i] = moment(v0, BASIS[i][0], BASIS[i][1]); }
  dudx = ImgD(W, H); dudy = ImgD(W, H); dvdx = ImgD(W, H); dvdy = ImgD(W, H);
  double need = min_frac * win * win;
#pragma omp parallel
  {
    vector<double> M(36), M2(36), b(6), b2(6);
#pragma omp for schedule(static)
    for (long pl = 0; pl < (long)m.n(); pl++) {
      size_t p = (size_t)pl;
      double count = Mm[0][0].d[p];
      bool ok = count >= need;
      double r[4] = {NaN, NaN, NaN, NaN};
      if (ok) {
        for (int i = 0; i < 6; i++)
          for (int j = 0; j < 6; j++) M[i * 6 + j] = Mm[BASIS[i][0] + BASIS[j][0]][BASIS[i][1] + BASIS[j][1]].d[p];
        M2 = M;
        for (int i = 0; i < 6; i++) { b[i] = ru[i].d[p]; b2[i] = rv[i].d[p]; }
        bool a1 = cholesky_solve(M, b, 6);
        bool a2 = cholesky_solve(M2, b2, 6);
        if (a1 && a2) { r[0] = b[1]; r[1] = b[2]; r[2] = b2[1]; r[3] = b2[2]; }
      }
      dudx.d[p] = r[0]; dudy.d[p] = r[1]; dvdx.d[p] = r[2]; dvdy.d[p] = r[3];
    }
  }
}

struct Strain { ImgD exx, eyy, exy, gmax, vol; };
Strain strain_fields(const ImgD& a, const ImgD& b, const ImgD& c, const ImgD& d) {  // strain.py:100-112
  Strain s;
  int W = a.w, H = a.h;
  s.exx = ImgD(W, H); s.eyy = ImgD(W, H); s.exy = ImgD(W, H); s.gmax = ImgD(W, H); s.vol = ImgD(W, H);
  for (size_t p = 0; p < a.n(); p++) {
    double dudx = a.d[p], dudy = b.d[p], dvdx = c.d[p], dvdy = d.d[p];
    double exx = dudx + 0.5 * (dudx * dudx + dvdx * dvdx);
    double eyy = dvdy + 0.5 * (dudy * dudy + dvdy * dvdy);
    double exy = 0.5 * (dudy + dvdx) + 0.5 * (dudx * dudy + dvdx * dvdy);
    double q = (exx - eyy) / 2;
    s.exx.d[p] = exx; s.eyy.d[p] = eyy; s.exy.d[p] = exy;
    s.gmax.d[p] = 2.0 * std::sqrt(q * q + exy * exy);
    s.vol.d[p] = (1 + dudx) * (1 + dvdy) - dudy * dvdx - 1.0;
  }
  return s;
}

// _finish (track.py:56-108) without the crack options
void finish(const ImgD& ux, const ImgD& uy, const ImgD& conf, const ImgB* mask, const ofc_config& c,
            ImgD& mx, ImgD& my, Strain& st) {
  int W = ux.w, H = ux.h;
  ImgB low(W, H), bad(W, H);
  for (size_t p = 0; p < low.n(); p++) {
    low.d[p] = conf.d[p] < c.conf_min;
    bad.d[p] = low.d[p] || (mask && !mask->d[p]);
  }
  double guard = edge_guard_px(c);
  if (guard > 0) {
    ImgB src = large_components(low, edge_guard_min_area_px(c));
    bool any = false;
    for (size_t p = 0; p < src.n(); p++) {
      if (mask && !mask->d[p]) src.d[p] = 1;
      any |= src.d[p] != 0;
    }
    if (any) {
      ImgD d2 = sqdist_to(src);
      for (size_t p = 0; p < src.n(); p++) if (std::sqrt(d2.d[p]) <= guard) bad.d[p] = 1;
    }
    for (int y = 0; y < H; y++)
      for (int x = 0; x < W; x++) {
        int bd = std::min(std::min(x, y), std::min(W - 1 - x, H - 1 - y));
        if (bd < guard) bad(x, y) = 1;
      }
  }
  mx = ImgD(W, H); my = ImgD(W, H);
  for (size_t p = 0; p < mx.n(); p++) {
    mx.d[p] = bad.d[p] ? NaN : ux.d[p];
    my.d[p] = bad.d[p] ? NaN : uy.d[p];
  }
  ImgD a, b, cc, d;
  displacement_gradient(mx, my, c.strain_win, a, b, cc, d);
  st = strain_fields(a, b, cc, d);
}

// ------------------------------------------------------------------ synthetic speckle (synth.py:20-190)
// The field of include/optflow_cuda_synth.h: x = c + A (X - c) + t + amp sin(2 pi X_x / wavelength) (sx, sy), plus the
// optional grid (cubic B-spline of coefficients), footing settlement and shear-band displacements of X.
void field_extra_u(const ofc_field& f, double X, double Y, double& ux, double& uy) {
  ux = uy = 0.0;
  if (f.grid && f.gnx > 0 && f.gny > 0) {
    auto basis = [](double t, double* w) {  // uniform cubic B-spline weights of taps i-1..i+2
      w[0] = (1 - t) * (1 - t) * (1 - t) / 6;
      w[1] = (3 * t * t * t - 6 * t * t + 4) / 6;
      w[2] = (-3 * t * t * t + 3 * t * t + 3 * t + 1) / 6;
      w[3] = t * t * t / 6;
    };
    double gx = (X - f.gx0) / f.gh, gy = (Y - f.gy0) / f.gh, wx[4], wy[4];
    long ix = (long)std::floor(gx), iy = (long)std::floor(gy);
    basis(gx - ix, wx);
    basis(gy - iy, wy);
    for (int a = 0; a < 4; a++)
      for (int b = 0; b < 4; b++) {
        long r = std::min(std::max(iy - 1 + a, 0L), (long)f.gny - 1), c = std::min(std::max(ix - 1 + b, 0L), (long)f.gnx - 1);
        ux += wy[a] * wx[b] * f.grid[r * f.gnx + c];
        uy += wy[a] * wx[b] * f.grid[(size_t)f.gnx * f.gny + r * f.gnx + c];
      }
  }
  if (f.fs != 0.0) {
    double px = std::min(std::max(X, f.fx0), f.fx1);
    uy += f.fs * std::exp(-std::hypot(X - px, Y - f.fy) / f.fdecay);
  }
  for (int k = 0; k < f.n_bands; k++) {
    const ofc_band& b = f.bands[k];
    double s = -b.ty * (X - b.ex) + b.tx * (Y - b.ey), a = b.tx * (X - b.ex) + b.ty * (Y - b.ey);
    double tp = b.length > 0 ? 0.25 * (1 + std::tanh(a / b.width)) * (1 + std::tanh((b.length - a) / b.width)) : 1.0;
    double v = 0.5 * b.delta * (std::tanh(s / b.width) + b.bias) * tp;
    ux += v * b.tx;
    uy += v * b.ty;
  }
}

bool field_has_extra(const ofc_field& f) { return f.grid || f.fs != 0.0 || f.n_bands > 0; }

void field_fwd(const ofc_field& f, double X, double Y, double& x, double& y) {  // synth.py:42-46
  double dx = X - f.cx, dy = Y - f.cy;
  x = f.cx + f.a00 * dx + f.a01 * dy + f.tx;
  y = f.cy + f.a10 * dx + f.a11 * dy + f.ty;
  if (f.amp != 0.0) {
    double s = f.amp * std::sin(2 * PI * X / f.wavelength);
    x = x + s * f.sx;
    y = y + s * f.sy;
  }
  if (field_has_extra(f)) {
    double ux, uy;
    field_extra_u(f, X, Y, ux, uy);
    x += ux;
    y += uy;
  }
}

// the affine inverse (synth.py:48-51), then Newton steps until the step is below 1e-13: the sinusoid's Jacobian in
// closed form, the optional terms' by central differences (step 1e-5 px)
void field_inv(const ofc_field& f, double x, double y, double& X, double& Y) {
  double det = f.a00 * f.a11 - f.a01 * f.a10;
  double b00 = f.a11 / det, b01 = -f.a01 / det, b10 = -f.a10 / det, b11 = f.a00 / det;
  double dx = x - f.cx - f.tx, dy = y - f.cy - f.ty;
  X = f.cx + b00 * dx + b01 * dy;
  Y = f.cy + b10 * dx + b11 * dy;
  const bool extra = field_has_extra(f);
  if (f.amp == 0.0 && !extra) return;
  for (int it = 0; it < 30; it++) {
    double fx, fy;
    field_fwd(f, X, Y, fx, fy);
    fx -= x;
    fy -= y;
    double j00 = f.a00, j01 = f.a01, j10 = f.a10, j11 = f.a11;
    if (f.amp != 0.0) {
      double ds = f.amp * (2 * PI / f.wavelength) * std::cos(2 * PI * X / f.wavelength);
      j00 += ds * f.sx;
      j10 += ds * f.sy;
    }
    if (extra) {
      const double e = 1e-5;
      double ax, ay, bx, by, cx, cy, ex, ey;
      field_extra_u(f, X + e, Y, ax, ay);
      field_extra_u(f, X - e, Y, bx, by);
      field_extra_u(f, X, Y + e, cx, cy);
      field_extra_u(f, X, Y - e, ex, ey);
      j00 += (ax - bx) / (2 * e);
      j10 += (ay - by) / (2 * e);
      j01 += (cx - ex) / (2 * e);
      j11 += (cy - ey) / (2 * e);
    }
    double d = j00 * j11 - j01 * j10;
    double sx = (j11 * fx - j01 * fy) / d, sy = (-j10 * fx + j00 * fy) / d;
    X -= sx;
    Y -= sy;
    if (std::fabs(sx) + std::fabs(sy) < 1e-13) break;
  }
}

// synth.render (synth.py:150-190) without a gap: every blob k, in index order, adds a_k exp(-d^2 / (2 r_k^2)) to
// the ss x ss subsamples of the rectangle of half size 5.2 r_k + 2 around its mapped centre, d measured between
// the subsample's inverse-mapped position and the blob's reference centre; a pixel is 0.5 + 0.25 tanh(mean).
// Rows of pixels run in parallel; each row adds its blobs in index order, so the sums are the reference's.
void render(const double* bx, const double* by, const double* br, const double* ba, size_t n, int w, int h, int ss,
            const ofc_field* f, double* out) {
  const long W = (long)w * ss, H = (long)h * ss;
  vector<long> i0(n), i1(n), j0(n), j1(n);
  vector<vector<int>> rows(h);
  for (size_t k = 0; k < n; k++) {
    double px = bx[k], py = by[k];
    if (f) field_fwd(*f, bx[k], by[k], px, py);
    double rad = 5.2 * br[k] + 2.0;
    j0[k] = std::max((long)std::floor((px - rad + 0.5) * ss), 0L);
    j1[k] = std::min((long)std::ceil((px + rad + 0.5) * ss), W);
    i0[k] = std::max((long)std::floor((py - rad + 0.5) * ss), 0L);
    i1[k] = std::min((long)std::ceil((py + rad + 0.5) * ss), H);
    if (j0[k] >= j1[k] || i0[k] >= i1[k]) continue;
    for (long y = i0[k] / ss; y <= (i1[k] - 1) / ss; y++) rows[y].push_back((int)k);
  }
  vector<double> off(ss);
  for (int s = 0; s < ss; s++) off[s] = (s + 0.5) / ss - 0.5;
#pragma omp parallel
  {
    vector<double> X(ss * W), Y(ss * W), acc(ss * W);
#pragma omp for schedule(dynamic, 4)
    for (int y = 0; y < h; y++) {
      for (int si = 0; si < ss; si++)
        for (long j = 0; j < W; j++) {
          double xs = (double)(j / ss) + off[j % ss], ys = (double)y + off[si];
          size_t q = (size_t)si * W + j;
          if (f) field_inv(*f, xs, ys, X[q], Y[q]);
          else { X[q] = xs; Y[q] = ys; }
          acc[q] = 0.0;
        }
      for (int k : rows[y]) {
        long a0 = std::max(i0[k], (long)y * ss), a1 = std::min(i1[k], (long)(y + 1) * ss);
        double r2 = 2 * (br[k] * br[k]);
        for (long i = a0; i < a1; i++)
          for (long j = j0[k]; j < j1[k]; j++) {
            size_t q = (size_t)(i - (long)y * ss) * W + j;
            double dx = X[q] - bx[k], dy = Y[q] - by[k];
            acc[q] += ba[k] * std::exp(-(dx * dx + dy * dy) / r2);
          }
      }
      for (int x = 0; x < w; x++) {
        double s = 0;
        for (int si = 0; si < ss; si++)
          for (int sj = 0; sj < ss; sj++) s += acc[(size_t)si * W + (size_t)x * ss + sj];
        out[(size_t)y * w + x] = 0.5 + 0.25 * std::tanh(s / (ss * ss));
      }
    }
  }
}

// ------------------------------------------------------------------ glue
ImgD from_ptr(const double* p, int w, int h) { ImgD a(w, h); std::memcpy(a.d.data(), p, sizeof(double) * a.n()); return a; }
void to_ptr(const ImgD& a, double* p) { if (p) std::memcpy(p, a.d.data(), sizeof(double) * a.n()); }

}  // namespace

// ------------------------------------------------------------------ C API (test infrastructure)
extern "C" {

void oro_render(const double* bx, const double* by, const double* br, const double* ba, size_t n, int w, int h, int ss,
                const ofc_field* f, double* out) {
  render(bx, by, br, ba, n, w, h, ss, f, out);
}

// the integer POC peaks (Grid::ipx, ipy) of pyramid level `level` of coarse_flow; returns the level's nx * ny, or
// -1 when the level does not exist (cap: the room in ipk, 2 ints per grid point)
int oro_coarse_peaks(const double* a, const double* b, int w, int h, const double* iux, const double* iuy,
                     const ofc_config* c, int level, int* ipk, size_t cap, int* nx, int* ny) {
  ImgD A = from_ptr(a, w, h), B = from_ptr(b, w, h), ix, iy;
  if (iux) { ix = from_ptr(iux, w, h); iy = from_ptr(iuy, w, h); }
  vector<Grid> raw;
  coarse_flow(A, B, *c, iux ? &ix : nullptr, iux ? &iy : nullptr, &raw);
  if (level < 0 || level >= (int)raw.size()) return -1;
  const Grid& g = raw[level];
  *nx = (int)g.xs.size();
  *ny = (int)g.ys.size();
  size_t n = g.ipx.size();
  if (2 * n > cap) return -1;
  for (size_t i = 0; i < n; i++) { ipk[2 * i] = g.ipx[i]; ipk[2 * i + 1] = g.ipy[i]; }
  return (int)n;
}

void oro_set_f32_storage(int on) { g_f32_storage = on != 0; }

int oro_threads(int n) { if (n > 0) omp_set_num_threads(n); return omp_get_max_threads(); }

// numpy fft2 / ifft2 of an h x w complex array stored as interleaved (re, im) doubles
void oro_fft2(double* data, int w, int h, int inverse) {
  ImgC a(w, h);
  for (size_t i = 0; i < a.n(); i++) a.d[i] = cd(data[2 * i], data[2 * i + 1]);
  fft2(a, inverse != 0);
  for (size_t i = 0; i < a.n(); i++) { data[2 * i] = a.d[i].real(); data[2 * i + 1] = a.d[i].imag(); }
}

void oro_bspline_coeffs(const double* in, double* out, int w, int h) {
  ImgD a = from_ptr(in, w, h);
  bspline_inplace(a);
  to_ptr(a, out);
}

void oro_sample(const double* coeffs, int w, int h, const double* x, const double* y, size_t n, double* out) {
  ImgD c = from_ptr(coeffs, w, h);
  for (size_t i = 0; i < n; i++) out[i] = sample(c, x[i], y[i]);
}

void oro_gauss_blur(const double* in, double* out, int w, int h, double sigma) {
  to_ptr(gauss_blur(from_ptr(in, w, h), sigma), out);
}

// scipy distance_transform_edt(input) (distances) and, when idx is given, the feature transform
// indices of distance_transform_edt(input, return_indices=True) (flat y * w + x)
void oro_edt(const uint8_t* input, int w, int h, double* dist, int64_t* idx) {
  ImgB z(w, h);
  for (size_t p = 0; p < z.n(); p++) z.d[p] = input[p] == 0;
  if (dist) {
    ImgD d2 = sqdist_to(z);
    for (size_t p = 0; p < z.n(); p++) dist[p] = std::sqrt(d2.d[p]);
  }
  if (idx) {
    vector<int64_t> v = nearest_source(z);
    std::memcpy(idx, v.data(), sizeof(int64_t) * v.size());
  }
}

void oro_large_components(const uint8_t* b, int w, int h, double min_area, uint8_t* out) {
  ImgB a(w, h);
  std::memcpy(a.d.data(), b, a.n());
  ImgB o = large_components(a, min_area);
  std::memcpy(out, o.d.data(), o.n());
}

// reference_phase: per filter k, planes r_re, r_im, gx, gy, amp (each F x h x w)
int oro_reference_phase(const double* i1, int w, int h, const ofc_config* c, double* r_re, double* r_im, double* gx,
                        double* gy, double* amp) {
  ImgD I1 = from_ptr(i1, w, h);
  Bank b = gabor_bank(h + 2 * PAD, w + 2 * PAD, *c);
  vector<RefK> ref = reference_phase(I1, b);
  size_t N = (size_t)w * h;
  for (size_t k = 0; k < ref.size(); k++)
    for (size_t p = 0; p < N; p++) {
      r_re[k * N + p] = ref[k].r.d[p].real();
      r_im[k * N + p] = ref[k].r.d[p].imag();
      gx[k * N + p] = ref[k].gx.d[p];
      gy[k * N + p] = ref[k].gy.d[p];
      amp[k * N + p] = ref[k].amp.d[p];
    }
  return (int)ref.size();
}

// local_solve (phaseflow.py:177-188) on given per-pixel sums (7 planes: gxx gxy gyy gxc gyc gcc gw)
void oro_local_solve(const double* sums, const double* ux, const double* uy, int w, int h, double sigma, int order,
                     double* oux, double* ouy, double* energy, double* resid, double* slope) {
  ImgD s[7];
  size_t N = (size_t)w * h;
  for (int i = 0; i < 7; i++) s[i] = from_ptr(sums + i * N, w, h);
  Solved r = local_solve(s, from_ptr(ux, w, h), from_ptr(uy, w, h), sigma, order);
  to_ptr(r.ux, oux); to_ptr(r.uy, ouy); to_ptr(r.energy, energy); to_ptr(r.resid, resid);
  if (slope) std::memcpy(slope, r.slope.data(), sizeof(double) * N * 4);
}

// refine (phaseflow.py:427-511): returns ux, uy, conf (border rule applied), resid, energy
void oro_refine(const double* i1, const double* i2, int w, int h, const double* ux0, const double* uy0,
                const ofc_config* c, double* ux, double* uy, double* conf, double* resid, double* energy) {
  RawFlow rf = refine_raw(from_ptr(i1, w, h), from_ptr(i2, w, h), from_ptr(ux0, w, h), from_ptr(uy0, w, h), *c);
  ImgD cf;
  refine_conf(rf, *c, cf);
  to_ptr(rf.ux, ux); to_ptr(rf.uy, uy); to_ptr(cf, conf); to_ptr(rf.resid, resid); to_ptr(rf.energy, energy);
}

// the sums of the first inner iteration of refine from (ux, uy): pre-warp s = blur(u), warp, responses,
// accumulate (7 planes of w*h)
void oro_first_sums(const double* i1, const double* i2, int w, int h, const double* ux0, const double* uy0,
                    const ofc_config* c, double* sums_out) {
  ImgD I1 = from_ptr(i1, w, h), I2 = from_ptr(i2, w, h), ux = from_ptr(ux0, w, h), uy = from_ptr(uy0, w, h);
  Bank bank = gabor_bank(h + 2 * PAD, w + 2 * PAD, *c);
  vector<RefK> ref = reference_phase(I1, bank);
  ImgD c2 = I2;
  bspline_inplace(c2);
  ImgD sx = gauss_blur(ux, c->sigma_s), sy = gauss_blur(uy, c->sigma_s);
  ImgD warped(w, h);
  for (int y = 0; y < h; y++)
    for (int x = 0; x < w; x++) warped(x, y) = sample(c2, x + sx(x, y), y + sy(x, y));
  ImgC F2 = pad_reflect(warped);
  fft2(F2, false);
  vector<ImgC> resp(bank.G.size());
  for (size_t k = 0; k < bank.G.size(); k++) {
    ImgC R(F2.w, F2.h);
    for (size_t p = 0; p < R.n(); p++) R.d[p] = F2.d[p] * bank.G[k].d[p];
    fft2(R, true);
    bspline_inplace(R);
    if (g_f32_storage)
      for (cd& v : R.d) v = cd((float)v.real(), (float)v.imag());
    resp[k] = std::move(R);
  }
  ImgD csx = sx, csy = sy;
  bspline_inplace(csx);
  bspline_inplace(csy);
  ImgD sums[7];
  accumulate(ref, resp, sx, sy, csx, csy, ux, uy, sums);
  size_t N = (size_t)w * h;
  for (int i = 0; i < 7; i++) std::memcpy(sums_out + i * N, sums[i].d.data(), N * sizeof(double));
}

void oro_poc_shift(const double* a, const double* b, int w, int h, double* out3) {
  PocTables T(h, w);
  vector<double> va(a, a + (size_t)w * h), vb(b, b + (size_t)w * h);
  poc_shift(T, va, vb, out3[0], out3[1], out3[2]);
}

int oro_n_levels(double max_disp, int win, int h, int w) { return n_levels(max_disp, win, h, w); }
int oro_level_window(int h, int w, int win, int* wy, int* wx) { return level_window(h, w, win, *wy, *wx) ? 1 : 0; }

void oro_grid_shape(int w, int h, const ofc_config* c, int* nx, int* ny) {
  vector<int> xs, ys;
  grid_points(h, w, c->grid_step, c->poc_win, c->poc_win, xs, ys);
  *nx = (int)xs.size();
  *ny = (int)ys.size();
}

// poc_grid + clean at one level with a given window and optional init (ny x nx)
void oro_poc_grid(const double* a, const double* b, int w, int h, const int* xs, int nx, const int* ys, int ny, int wy,
                  int wx, const double* iux, const double* iuy, double* ux, double* uy, double* peak) {
  ImgD A = from_ptr(a, w, h), B = from_ptr(b, w, h);
  ImgD ix, iy;
  if (iux) { ix = from_ptr(iux, nx, ny); iy = from_ptr(iuy, nx, ny); }
  Grid g = poc_grid(A, B, vector<int>(xs, xs + nx), vector<int>(ys, ys + ny), wy, wx, iux ? &ix : nullptr, iux ? &iy : nullptr);
  to_ptr(g.ux, ux); to_ptr(g.uy, uy); to_ptr(g.peak, peak);
}

void oro_coarse_flow(const double* a, const double* b, int w, int h, const double* iux, const double* iuy,
                     const ofc_config* c, int* xs, int* ys, double* ux, double* uy, double* peak) {
  ImgD A = from_ptr(a, w, h), B = from_ptr(b, w, h);
  ImgD ix, iy;
  if (iux) { ix = from_ptr(iux, w, h); iy = from_ptr(iuy, w, h); }
  Grid g = coarse_flow(A, B, *c, iux ? &ix : nullptr, iux ? &iy : nullptr);
  for (size_t i = 0; i < g.xs.size(); i++) xs[i] = g.xs[i];
  for (size_t i = 0; i < g.ys.size(); i++) ys[i] = g.ys[i];
  to_ptr(g.ux, ux); to_ptr(g.uy, uy); to_ptr(g.peak, peak);
}

void oro_displacement_gradient(const double* ux, const double* uy, int w, int h, int win, double* dudx, double* dudy,
                               double* dvdx, double* dvdy) {
  ImgD a, b, c, d;
  displacement_gradient(from_ptr(ux, w, h), from_ptr(uy, w, h), win, a, b, c, d);
  to_ptr(a, dudx); to_ptr(b, dudy); to_ptr(c, dvdx); to_ptr(d, dvdy);
}

// _finish: mx, my (NaN-masked) and the strain maps exx eyy exy gmax vol
void oro_finish(const double* ux, const double* uy, const double* conf, const uint8_t* roi, int w, int h,
                const ofc_config* c, double* mx, double* my, double* exx, double* eyy, double* exy, double* gmax,
                double* vol) {
  ImgB mask;
  if (roi) { mask = ImgB(w, h); std::memcpy(mask.d.data(), roi, mask.n()); }
  ImgD MX, MY;
  Strain st;
  finish(from_ptr(ux, w, h), from_ptr(uy, w, h), from_ptr(conf, w, h), roi ? &mask : nullptr, *c, MX, MY, st);
  to_ptr(MX, mx); to_ptr(MY, my);
  to_ptr(st.exx, exx); to_ptr(st.eyy, eyy); to_ptr(st.exy, exy); to_ptr(st.gmax, gmax); to_ptr(st.vol, vol);
}

// track_pair (track.py:115-146): out planes ux uy conf exx eyy exy gmax vol raw_ux raw_uy (11 x h x w
// doubles, NaN-masked where invalid) and timing[3] = coarse, fine, strain seconds
void oro_track_pair(const double* i1, const double* i2, int w, int h, const uint8_t* roi, const double* iux,
                    const double* iuy, const ofc_config* c, double* out, double* timing) {
  using clk = std::chrono::steady_clock;
  auto t0 = clk::now();
  ImgD I1 = from_ptr(i1, w, h), I2 = from_ptr(i2, w, h);
  ImgD ix, iy;
  if (iux) { ix = from_ptr(iux, w, h); iy = from_ptr(iuy, w, h); }
  Grid g = coarse_flow(I1, I2, *c, iux ? &ix : nullptr, iux ? &iy : nullptr);
  ImgD gx, gy;
  dense_start(g, w, h, iux ? &ix : nullptr, iux ? &iy : nullptr, gx, gy);
  auto t1 = clk::now();
  RawFlow rf = refine_raw(I1, I2, gx, gy, *c);
  ImgD conf;
  refine_conf(rf, *c, conf);
  auto t2 = clk::now();
  ImgB mask;
  if (roi) { mask = ImgB(w, h); std::memcpy(mask.d.data(), roi, mask.n()); }
  ImgD mx, my;
  Strain st;
  finish(rf.ux, rf.uy, conf, roi ? &mask : nullptr, *c, mx, my, st);
  auto t3 = clk::now();
  size_t N = (size_t)w * h;
  const ImgD* planes[10] = {&mx, &my, &conf, &st.exx, &st.eyy, &st.exy, &st.gmax, &st.vol, &rf.ux, &rf.uy};
  for (int i = 0; i < 10; i++) std::memcpy(out + i * N, planes[i]->d.data(), sizeof(double) * N);
  if (timing) {
    timing[0] = std::chrono::duration<double>(t1 - t0).count();
    timing[1] = std::chrono::duration<double>(t2 - t1).count();
    timing[2] = std::chrono::duration<double>(t3 - t2).count();
  }
}

}  // extern "C"
