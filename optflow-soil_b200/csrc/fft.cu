// fft.cu -- FP32 mixed-radix FFTs in shared memory with the fused Gabor multiply and B-spline prefilter.
//
// One thread block transforms C interleaved lines held in shared memory (element i of line l at
// buf[i * C + l]), ping-ponging between two buffers of L * C values: each Stockham stage reads a butterfly's
// inputs from one and writes its outputs to the other. Radices 2, 4 and 8 have register butterflies, 3, 5, 7,
// 11 and 13 the symmetric odd form, other primes (up to 31) a direct DFT. Twiddles come from a table rounded
// from float64.
//
// The pass structure of one "responses" evaluation (per outer iteration of the fine stage):
//   rows:    reflect pad + real->complex + forward row FFT                      (read 4 B/px, write 8 B/px)
//   columns: forward column FFT in place (read 8, write 8); then per (column pair, filter k): x G_k and the
//            B-spline prefilter's periodic factor 1 / ((4 + 2 cos wx)(4 + 2 cos wy)) (separable tables), inverse
//            column FFT, the prefilter's edge terms along y                        (read 8F, write 8F)
//   rows:    inverse row FFT, the prefilter's edge terms along x, scale 36 / (ph pw)  (read 8F, write 8F)
// The prefilter is separable and linear, so its factors and edge terms along one axis commute with the
// transforms along the other, and the result is bspline_coeffs(ifft2(F2 * G)) of phaseflow.py:456 up to rounding.
#include "fft.cuh"

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <type_traits>

#include <cuda_pipeline.h>

namespace ofc {

// ------------------------------------------------------------------------------------------ host
bool fft_supported(int L) {
  if (L < 1) return false;
  int m = L;
  for (int p : {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31})
    while (m % p == 0) m /= p;
  return m == 1;
}

static int stage_count(int m) {
  int n = 0;
  while (m % 8 == 0) { n++; m /= 8; }
  while (m % 4 == 0) { n++; m /= 4; }
  while (m % 2 == 0) { n++; m /= 2; }
  for (int p : {3, 5, 7, 11, 13, 17, 19, 23, 29, 31})
    while (m % p == 0) { n++; m /= p; }
  return n;
}

// The cost of a Bluestein inner length M: M times its Stockham stages of the radices with a butterfly of their own (8,
// 4, 2 and the odd primes up to 19), a stage of radix 11 or 13 counted 1.2 and of 17 or 19 1.5 (their butterflies take
// more registers); infinite for other factors. The transforms are bound by their stage barriers, not by arithmetic:
// 604 = 4 151 (the padded height of 540-row frames) takes M = 1216 = 8 8 19 (3 stages) instead of the smallest
// 2^a 3^b 5^c 7^d, 1215 = 3^5 5 (6 stages).
static double bluestein_cost(int M) {
  double c = 0;
  int m = M;
  while (m % 8 == 0) { c += 1; m /= 8; }
  while (m % 4 == 0) { c += 1; m /= 4; }
  while (m % 2 == 0) { c += 1; m /= 2; }
  for (int p : {3, 5, 7, 11, 13, 17, 19}) {
    const double w = p <= 7 ? 1.0 : (p <= 13 ? 1.2 : 1.5);
    while (m % p == 0) { c += w; m /= p; }
  }
  return m == 1 ? c * M : 1e30;
}

int fft_work_length(int L) {
  if (L < 1) return 0;
  if (fft_supported(L)) return stage_count(L) <= FFT_MAXST ? L : 0;
  // Bluestein: among the lengths M in [2L - 1, 1.25 (2L - 1)] the one of least stage cost (the smallest on ties),
  // never above the smallest 2^a 3^b 5^c 7^d where that one fits the passes' shared memory and a larger one might not
  // (about 6800: four line buffers of the row pass, two two-column buffers of the column pass)
  const int lo = 2 * L - 1;
  int smooth = 0;
  for (int M = lo; M <= 8 * L && !smooth; M++) {
    int m = M;
    for (int p : {2, 3, 5, 7})
      while (m % p == 0) m /= p;
    if (m == 1) smooth = M;
  }
  constexpr int FIT = 6800;
  const int hi = (smooth && smooth <= FIT) ? std::min(lo + lo / 4, std::max(smooth, FIT)) : lo + lo / 4;
  int best = 0;
  double bc = 1e29;  // below the cost of a length with an unsupported factor
  for (int M = lo; M <= hi; M++) {
    const double c = bluestein_cost(M);
    if (c < bc) {
      bc = c;
      best = M;
    }
  }
  return best && stage_count(best) <= FFT_MAXST ? best : 0;
}

std::vector<float2> fft_bluestein_tables(int L, int M) {
  // chirp w[n] = exp(-i pi n^2 / L): the phase from n^2 mod 2L in integers, then float64
  std::vector<double> wr(L), wi(L);
  for (int n = 0; n < L; n++) {
    const long long q = ((long long)n * n) % (2LL * L);
    const double a = -PI * (double)q / (double)L;
    wr[n] = std::cos(a);
    wi[n] = std::sin(a);
  }
  // b = conj(w) wrapped to length M; filt = DFT_M(b) / M in float64 (a direct sum with an integer-indexed table)
  std::vector<double> br(M, 0.0), bi(M, 0.0), cr(M), ci(M);
  for (int n = 0; n < L; n++) {
    br[n] = wr[n];
    bi[n] = -wi[n];
    if (n) {
      br[M - n] = wr[n];
      bi[M - n] = -wi[n];
    }
  }
  for (int t = 0; t < M; t++) {
    const double a = -2.0 * PI * (double)t / (double)M;
    cr[t] = std::cos(a);
    ci[t] = std::sin(a);
  }
  std::vector<float2> out((size_t)L + M);
  for (int n = 0; n < L; n++) out[n] = make_float2((float)wr[n], (float)wi[n]);
  for (int k = 0; k < M; k++) {
    double sr = 0.0, si = 0.0;
    long long idx = 0;
    for (int n = 0; n < M; n++) {
      if (br[n] != 0.0 || bi[n] != 0.0) {
        sr += br[n] * cr[idx] - bi[n] * ci[idx];
        si += br[n] * ci[idx] + bi[n] * cr[idx];
      }
      idx += k;
      if (idx >= M) idx -= M;
    }
    out[(size_t)L + k] = make_float2((float)(sr / M), (float)(si / M));
  }
  return out;
}

namespace {
std::mutex g_plan_mu;
std::map<int, int> g_plan_table;  // padded length -> factor order (fft_set_plan_variant)
}  // namespace

void fft_set_plan_variant(int L, int variant) {
  std::lock_guard<std::mutex> lk(g_plan_mu);
  if (variant <= 0) g_plan_table.erase(L);
  else g_plan_table[L] = variant;
}

int fft_plan_variant(int L) {
  std::lock_guard<std::mutex> lk(g_plan_mu);
  auto it = g_plan_table.find(L);
  return it == g_plan_table.end() ? 0 : it->second;
}

// The factor orders a plan of length n can take (the transform is the same; the stages, their strides and the
// rounding differ): 0 radix 8 first, then 4, 2 and the odd radices ascending; 1 the odd radices first; 2 the power of
// two in radix-4 stages (a radix 2 last when the power is odd); 3 the order of 0 reversed.
static std::vector<int> factor_order(int n, int variant) {
  std::vector<int> two, odd;
  int m = n, e = 0;
  while (m % 2 == 0) { m /= 2; e++; }
  for (int p : {3, 5, 7, 11, 13, 17, 19, 23, 29, 31})
    while (m % p == 0) { odd.push_back(p); m /= p; }
  if (m != 1) return {};
  if (variant == 2) {
    for (; e >= 2; e -= 2) two.push_back(4);
    if (e) two.push_back(2);
  } else {
    for (; e >= 3; e -= 3) two.push_back(8);
    if (e == 2) two.push_back(4);
    if (e == 1) two.push_back(2);
  }
  std::vector<int> f;
  if (variant == 1) {
    f = odd;
    f.insert(f.end(), two.begin(), two.end());
  } else {
    f = two;
    f.insert(f.end(), odd.begin(), odd.end());
  }
  if (variant == 3) std::reverse(f.begin(), f.end());
  return f;
}

FftPlan fft_make_plan(int L) { return fft_make_plan(L, fft_plan_variant(L)); }

FftPlan fft_make_plan(int L, int variant) {
  const int work = fft_work_length(L);
  if (work == 0) throw Error(OFC_ERR_WINDOW, "no FFT plan for length " + std::to_string(L));
  if (variant < 0 || variant >= FFT_PLAN_VARIANTS) throw Error(OFC_ERR_ARG, "no FFT plan variant " + std::to_string(variant));
  FftPlan pl;
  pl.L = L;
  pl.M = work == L ? 0 : work;
  std::vector<int> f = factor_order(work, variant);
  if (f.empty() || (int)f.size() > FFT_MAXST)
    throw Error(OFC_ERR_WINDOW, "FFT length " + std::to_string(L) + " needs too many stages");
  int s = 1;
  pl.nst = (int)f.size();
  for (int i = 0; i < pl.nst; i++) {
    pl.p[i] = f[i];
    pl.s[i] = s;
    // ceil(2^32 / s): q = umulhi(bi, magic) = floor(bi / s) for every bi < L * 4 here
    pl.magic[i] = s == 1 ? 0u : (unsigned)((((unsigned long long)1 << 32) + s - 1) / s);
    s *= f[i];
  }
  return pl;
}

std::vector<float2> fft_twiddles(int L) {
  std::vector<float2> t(L);
  for (int i = 0; i < L; i++) {
    double a = -2.0 * PI * (double)i / (double)L;
    t[i] = make_float2((float)std::cos(a), (float)std::sin(a));
  }
  return t;
}

int fft_threads(int L, int C) {
  int need = (L * C + FFT_E - 1) / FFT_E;
  int unit = 32;
  while (unit % C) unit += 32;  // multiple of 32 and of C
  int cap = (FFT_TMAX / unit) * unit;
  int T = ((need + unit - 1) / unit) * unit;
  return std::max(unit, std::min(T, cap));
}

size_t gabor_yt2_offset(int ph, int pw, int F) {
  const size_t base = (size_t)4 * (pw + ph) + (size_t)F * (pw + ph);
  return (base + 1) & ~(size_t)1;
}

std::vector<double> gabor_tables_host(int ph, int pw, const ofc_config& c) {
  int F = c.n_scales * c.n_orient;
  std::vector<double> t((size_t)4 * (pw + ph) + (size_t)F * (pw + ph));
  double* fx = t.data();
  double* fy = fx + pw;
  double* hx = fy + ph;
  double* hy = hx + pw;
  double* omx = hy + ph;
  double* omy = omx + pw;
  double* ex = omy + ph;
  double* ey = ex + (size_t)F * pw;
  auto freq = [](int n, double* f) {  // np.fft.fftfreq(n) * 2 * pi
    double val = 1.0 / n;
    int N = (n - 1) / 2 + 1;
    for (int i = 0; i < n; i++) f[i] = (double)(i < N ? i : i - n) * val * 2 * PI;
  };
  freq(pw, fx);
  freq(ph, fy);
  double smax = 0;
  for (int i = 0; i < c.n_scales; i++) smax = std::max(smax, c.scales[i]);
  double s_hp = c.dc_cut * c.lam * smax / (2 * PI);
  for (int x = 0; x < pw; x++) {
    double e = -(fx[x] * fx[x]) * (s_hp * s_hp) / 2;
    hx[x] = std::exp(e);
    omx[x] = -std::expm1(e);
  }
  for (int y = 0; y < ph; y++) {
    double e = -(fy[y] * fy[y]) * (s_hp * s_hp) / 2;
    hy[y] = std::exp(e);
    omy[y] = -std::expm1(e);
  }
  int k = 0;
  for (int si = 0; si < c.n_scales; si++) {
    double w0 = 2 * PI / (c.lam * c.scales[si]);
    double s = c.bandwidth * w0;
    for (int o = 0; o < c.n_orient; o++, k++) {
      double th = PI * o / c.n_orient;
      double cx = w0 * std::cos(th), cy = w0 * std::sin(th);
      for (int x = 0; x < pw; x++) { double d = fx[x] - cx; ex[(size_t)k * pw + x] = std::exp(-(d * d) / (2 * s * s)); }
      for (int y = 0; y < ph; y++) { double d = fy[y] - cy; ey[(size_t)k * ph + y] = std::exp(-(d * d) / (2 * s * s)); }
    }
  }
  // the B-spline prefilter on the periodic grid, per axis: 1 / (4 + 2 cos w)
  double* bx = ey + (size_t)F * ph;
  double* by = bx + pw;
  for (int x = 0; x < pw; x++) bx[x] = 1.0 / (4.0 + 2.0 * std::cos(2 * PI * (double)x / pw));
  for (int y = 0; y < ph; y++) by[y] = 1.0 / (4.0 + 2.0 * std::cos(2 * PI * (double)y / ph));
  // per filter and row: (omy[y], ey_k[y] by[y]), from an even offset (a float2 table in the float32 image)
  std::vector<double> yt((size_t)2 * F * ph);
  for (int k2 = 0; k2 < F; k2++)
    for (int y = 0; y < ph; y++) {
      yt[2 * ((size_t)k2 * ph + y)] = omy[y];
      yt[2 * ((size_t)k2 * ph + y) + 1] = ey[(size_t)k2 * ph + y] * by[y];
    }
  const size_t o = gabor_yt2_offset(ph, pw, F);
  t.resize(o + yt.size(), 0.0);
  std::copy(yt.begin(), yt.end(), t.begin() + o);
  return t;
}

void gabor_bind(GaborTables& g, const double* d64, const float* d32, int ph, int pw, int F) {
  g.F = F;
  g.ph = ph;
  g.pw = pw;
  g.fx = d64;
  g.fy = g.fx + pw;
  g.hx = g.fy + ph;
  g.hy = g.hx + pw;
  g.omx = g.hy + ph;
  g.omy = g.omx + pw;
  g.ex = g.omy + ph;
  g.ey = g.ex + (size_t)F * pw;
  g.hxf = d32 + pw + ph;
  g.omxf = g.hxf + pw + ph;
  g.omyf = g.omxf + pw;
  g.exf = g.omyf + ph;
  g.eyf = g.exf + (size_t)F * pw;
  g.bxf = g.eyf + (size_t)F * ph;
  g.byf = g.bxf + pw;
  g.yt2 = (const float2*)(d32 + gabor_yt2_offset(ph, pw, F));
}

// ------------------------------------------------------------------------------------------ device
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 conjf2(float2 a) { return make_float2(a.x, -a.y); }
// multiply by -i (forward) or +i (inverse)
__device__ __forceinline__ float2 rot(float2 a, bool inv) { return inv ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x); }
template <class C2> __device__ __forceinline__ C2 mkc(double re, double im);
template <> __device__ __forceinline__ float2 mkc<float2>(double re, double im) { return make_float2((float)re, (float)im); }

// cos and sin of 2 pi m / P at compile time (Taylor series after reduction to [-pi/8, pi/8] by octant; exact to
// float64 rounding for the small P here), for the constant coefficients of the odd-radix butterflies
constexpr double ct_poly_sin(double x) {
  double t = x, s = x;
  for (int n = 1; n < 14; n++) {
    t *= -x * x / ((2 * n) * (2 * n + 1));
    s += t;
  }
  return s;
}
constexpr double ct_poly_cos(double x) {
  double t = 1, s = 1;
  for (int n = 1; n < 14; n++) {
    t *= -x * x / ((2 * n - 1) * (2 * n));
    s += t;
  }
  return s;
}
// angle 2 pi m / P = q (pi / 4) + r with |r| <= pi / 8
constexpr void ct_sincos(int m, int P, double& c, double& sn) {
  double a = 2 * PI * (double)m / (double)P;
  int q = (int)(a / (PI / 4) + 0.5);
  double r = a - q * (PI / 4);
  double cr = ct_poly_cos(r), sr = ct_poly_sin(r);
  constexpr double h = 0.70710678118654752440;  // cos(pi / 4)
  double cq[8] = {1, h, 0, -h, -1, -h, 0, h}, sq[8] = {0, h, 1, h, 0, -h, -1, -h};
  c = cq[q & 7] * cr - sq[q & 7] * sr;
  sn = sq[q & 7] * cr + cq[q & 7] * sr;
}
template <int P>
struct OddCoef {  // cs[k][j] = cos(2 pi j k / P), sn[k][j] = -sin(2 pi j k / P) (the forward kernel exp(-2 pi i jk / P))
  float cs[P][P] = {}, sn[P][P] = {};
  constexpr OddCoef() {
    for (int k = 0; k < P; k++)
      for (int j = 0; j < P; j++) {
        double c = 0, s = 0;
        ct_sincos((j * k) % P, P, c, s);
        cs[k][j] = (float)c;
        sn[k][j] = (float)(-s);
      }
  }
};

// Odd-radix butterfly with the symmetric form: for j = 1..(P-1)/2, a_j = v_j + v_{P-j}, b_j = v_j - v_{P-j};
// o_0 = v_0 + sum a_j; o_k = v_0 + sum_j a_j cos_jk + i sum_j b_j sin_jk, o_{P-k} = the same with -i, where
// w^{jk} = cos_jk + i sin_jk (w = exp(-2 pi i / P), conjugated for the inverse) are compile-time constants.
template <int P, class C2, class Load, class Emit>
__device__ __forceinline__ void odd_butterfly(Load in, bool inv, Emit emit) {
  constexpr int Hh = (P - 1) / 2;
  constexpr OddCoef<P> K{};
  C2 v0 = in(0);
  C2 av[Hh], bv[Hh];
#pragma unroll
  for (int j = 1; j <= Hh; j++) {
    C2 x = in(j), y = in(P - j);
    av[j - 1] = cadd(x, y);
    bv[j - 1] = csub(x, y);
  }
  C2 s0 = v0;
#pragma unroll
  for (int j = 0; j < Hh; j++) s0 = cadd(s0, av[j]);
  emit(0, s0);
  const float sg = inv ? -1.f : 1.f;
#pragma unroll
  for (int k = 1; k <= Hh; k++) {
    C2 t = v0, u = mkc<C2>(0.0, 0.0);
#pragma unroll
    for (int j = 1; j <= Hh; j++) {
      const float cs = K.cs[k][j], sn = K.sn[k][j];
      t.x = fmaf(av[j - 1].x, cs, t.x);
      t.y = fmaf(av[j - 1].y, cs, t.y);
      u.x = fmaf(bv[j - 1].x, sn, u.x);
      u.y = fmaf(bv[j - 1].y, sn, u.y);
    }
    u.x *= sg;
    u.y *= sg;
    // i u = (-u.y, u.x)
    emit(k, mkc<C2>(t.x - u.y, t.y + u.x));
    emit(P - k, mkc<C2>(t.x + u.y, t.y - u.x));
  }
}

// Shared-memory layouts of the transform buffers: element i at i + (i >> sh), sh = FFT_PAD (one pad slot
// per 16 values) or 31 (no padding; i < 2^31). A stage whose outputs lie s * C apart with s * C < 32 writes
// padded, which spreads its stores over the banks; the other buffers, and always the final one, are
// unpadded. Buffer capacity: fft_buf_len(L, C) values.
constexpr int FFT_PAD = 4;
__host__ __device__ constexpr int fft_buf_len(int L, int C) { return L * C + ((L * C) >> FFT_PAD) + 1; }

// The butterfly of radix P (P = 0: a direct DFT of runtime radix RP) on inputs in(j), j < P, with outputs
// through emit(k, value) (which applies the inter-stage twiddle); tw_m(m) = w_P^m for the direct DFT.
template <int P, class C2, class In, class Emit, class TwM>
__device__ __forceinline__ void butterfly(In in, Emit emit, TwM tw_m, int RP, bool inv) {
  if constexpr (P == 2) {
    C2 a0 = in(0), a1 = in(1);
    emit(0, cadd(a0, a1));
    emit(1, csub(a0, a1));
  } else if constexpr (P == 4) {
    C2 a0 = in(0), a1 = in(1), a2 = in(2), a3 = in(3);
    C2 t0 = cadd(a0, a2), t1 = csub(a0, a2);
    C2 t2 = cadd(a1, a3), t3 = rot(csub(a1, a3), inv);
    emit(0, cadd(t0, t2));
    emit(2, csub(t0, t2));
    emit(1, cadd(t1, t3));
    emit(3, csub(t1, t3));
  } else if constexpr (P == 8) {
    C2 v[8];
#pragma unroll
    for (int j = 0; j < 8; j++) v[j] = in(j);
    C2 e[4], d[4];
    {
      C2 t0 = cadd(v[0], v[4]), t1 = csub(v[0], v[4]);
      C2 t2 = cadd(v[2], v[6]), t3 = rot(csub(v[2], v[6]), inv);
      e[0] = cadd(t0, t2); e[2] = csub(t0, t2); e[1] = cadd(t1, t3); e[3] = csub(t1, t3);
    }
    {
      C2 t0 = cadd(v[1], v[5]), t1 = csub(v[1], v[5]);
      C2 t2 = cadd(v[3], v[7]), t3 = rot(csub(v[3], v[7]), inv);
      d[0] = cadd(t0, t2); d[2] = csub(t0, t2); d[1] = cadd(t1, t3); d[3] = csub(t1, t3);
    }
    // w8^k, k = 1..3: (h, -h), (0, -1), (-h, -h) forward; conjugates inverse (h = cos(pi / 4))
    constexpr float h = 0.70710678118654752440f;
    const float sg = inv ? 1.f : -1.f;
    C2 t1 = mkc<C2>(h * (d[1].x - sg * d[1].y), h * (d[1].y + sg * d[1].x));
    C2 t2 = mkc<C2>(-sg * d[2].y, sg * d[2].x);
    C2 t3 = mkc<C2>(h * (-d[3].x - sg * d[3].y), h * (-d[3].y + sg * d[3].x));
    emit(0, cadd(e[0], d[0]));
    emit(4, csub(e[0], d[0]));
    emit(1, cadd(e[1], t1));
    emit(5, csub(e[1], t1));
    emit(2, cadd(e[2], t2));
    emit(6, csub(e[2], t2));
    emit(3, cadd(e[3], t3));
    emit(7, csub(e[3], t3));
  } else if constexpr (P == 3 || P == 5 || P == 7 || P == 11 || P == 13 || P == 17 || P == 19) {
    odd_butterfly<P, C2>(in, inv, emit);
  } else {
    for (int k = 0; k < RP; k++) {
      C2 acc = in(0);
      int jk = 0;
      for (int j = 1; j < RP; j++) {
        jk += k;
        if (jk >= RP) jk -= RP;
        C2 av = in(j);
        C2 w = tw_m(jk);
        acc.x = fma(av.x, w.x, fma(-av.y, w.y, acc.x));
        acc.y = fma(av.x, w.y, fma(av.y, w.x, acc.y));
      }
      emit(k, acc);
    }
  }
}

// One Stockham stage of radix P from buffer A (layout shift ish) to buffer B (layout shift osh); C interleaved
// lines of length L, C = 1 << lc. q, r of a butterfly come from multiplications by precomputed reciprocals
// (magic = ceil(2^32 / s), exact for the sizes here). Radices 2, 4, 8 have hand-written butterflies, 3, 5, 7,
// 11 and 13 the symmetric odd form, and any other radix (P = 0 here) a direct DFT with its inputs read from
// shared memory. Each radix is its own non-inlined function, so that the registers of one radix's butterfly do
// not add to another's. Butterfly b reads elements b + j istep (b = bi C + l with bi = q s + r).
template <int P, class C2>
__device__ __noinline__ void stage_loop(const C2* __restrict__ A, C2* __restrict__ B, int lc, int L, int Pr, int s,
                                        unsigned magic, const C2* __restrict__ tw, bool inv, int ish, int osh) {
  const int RP = P ? P : Pr;
  const int C = 1 << lc;
  const int m = L / (RP * s);
  const int nb = (L / RP) << lc;
  const int LP = L / RP;
  const int istep = s * m * C, ostep = s * C;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    const int l = b & (C - 1), bi = b >> lc;
    const int q = s == 1 ? bi : (int)__umulhi((unsigned)bi, magic), r = bi - q * s;
    const int ob = (r + s * RP * q) * C + l;
    auto in = [&](int j) {
      const int i = b + j * istep;
      return A[i + (i >> ish)];
    };
    auto emit = [&](int k, C2 val) {
      if (k > 0 && q > 0) {
        C2 w = __ldg(tw + (size_t)k * q * s);  // k q s < L
        val = cmul(val, inv ? conjf2(w) : w);
      }
      const int o = ob + k * ostep;
      B[o + (o >> osh)] = val;
    };
    auto tw_m = [&](int mm) {  // w_P^mm
      C2 w = __ldg(tw + (size_t)mm * LP);
      return inv ? conjf2(w) : w;
    };
    butterfly<P, C2>(in, emit, tw_m, RP, inv);
  }
}

// The same stage with every size known at compile time (radix P, stride S, length L, lines C, layout shifts):
// the quotients, strides and padded offsets fold into constants.
template <int P, int S, int L, int C, int ISH, int OSH, class C2>
__device__ __noinline__ void stage_fixed(const C2* __restrict__ A, C2* __restrict__ B, const C2* __restrict__ tw,
                                         bool inv) {
  constexpr int PB =
      (P == 2 || P == 3 || P == 4 || P == 5 || P == 7 || P == 8 || P == 11 || P == 13 || P == 17 || P == 19) ? P : 0;
  constexpr int M = L / (P * S), NB = (L / P) * C, ISTEP = S * M * C, OSTEP = S * C, LP = L / P;
  for (int b = threadIdx.x; b < NB; b += blockDim.x) {
    const int l = b % C, bi = b / C;
    const int q = bi / S, r = bi - q * S;
    const int ob = (r + S * P * q) * C + l;
    auto in = [&](int j) {
      const int i = b + j * ISTEP;
      if constexpr (ISH < 31) return A[i + (i >> ISH)];
      else return A[i];
    };
    auto emit = [&](int k, C2 val) {
      if (k > 0 && q > 0) {
        C2 w = __ldg(tw + k * S * q);  // k q S < L
        val = cmul(val, inv ? conjf2(w) : w);
      }
      const int o = ob + k * OSTEP;
      if constexpr (OSH < 31) B[o + (o >> OSH)] = val;
      else B[o] = val;
    };
    auto tw_m = [&](int mm) {  // w_P^mm
      C2 w = __ldg(tw + mm * LP);
      return inv ? conjf2(w) : w;
    };
    butterfly<PB, C2>(in, emit, tw_m, P, inv);
  }
}

// compile-time plan: the factorisation of fft_make_plan (8s, 4s, 2s, then odd primes up to 31)
struct CPlan {
  int nst = 0;
  int p[FFT_MAXST] = {}, s[FFT_MAXST] = {};
};
constexpr CPlan cplan(int L) {
  CPlan c{};
  int m = L, f[FFT_MAXST] = {}, n = 0;
  while (m % 8 == 0) { f[n++] = 8; m /= 8; }
  while (m % 4 == 0) { f[n++] = 4; m /= 4; }
  while (m % 2 == 0) { f[n++] = 2; m /= 2; }
  const int primes[10] = {3, 5, 7, 11, 13, 17, 19, 23, 29, 31};
  for (int i = 0; i < 10; i++)
    while (m % primes[i] == 0) { f[n++] = primes[i]; m /= primes[i]; }
  int st = 1;
  for (int i = 0; i < n; i++) {
    c.p[i] = f[i];
    c.s[i] = st;
    st *= f[i];
  }
  c.nst = n;
  return c;
}

template <int L, int C, int ST, class C2>
__device__ __forceinline__ C2* fft_run_fixed(C2* a, C2* b, const C2* tw, bool inv) {
  constexpr CPlan P = cplan(L);
  if constexpr (ST == P.nst) {
    return a;
  } else {
    constexpr int OSH = (ST + 1 < P.nst && P.s[ST] * C < 32) ? FFT_PAD : 31;
    constexpr int ISH = ST == 0 ? 31 : (P.s[ST - 1] * C < 32 ? FFT_PAD : 31);
    stage_fixed<P.p[ST], P.s[ST], L, C, ISH, OSH, C2>(a, b, tw, inv);
    __syncthreads();
    return fft_run_fixed<L, C, ST + 1, C2>(b, a, tw, inv);
  }
}

// The first stage of a fixed-length inverse column transform of a column pair with the responses' factor folded into
// its loads: element i is raw[i] G, G = (hx + omx omy) ex ey bx by with (omy, ey by) the row table's entry of row
// i / 2 and hx, omx, exb = ex bx the factors of the thread's column, which stays fixed (blockDim and the stage's input
// stride are even). The products are rounded as the separate multiply pass rounded them (no contraction into the
// butterfly's additions), so the transform sees the same values without that pass's shared-memory round trip and
// barrier.
template <int P, int S, int L, int C, int OSH, class C2>
__device__ __noinline__ void stage_fixed_mul(const C2* __restrict__ raw, C2* __restrict__ B, const C2* __restrict__ tw,
                                             bool inv, const float2* __restrict__ yt, float hx, float omx, float exb) {
  static_assert(C == 2 && S == 1, "the first stage of a column pair");
  constexpr int PB =
      (P == 2 || P == 3 || P == 4 || P == 5 || P == 7 || P == 8 || P == 11 || P == 13 || P == 17 || P == 19) ? P : 0;
  constexpr int M = L / (P * S), NB = (L / P) * C, ISTEP = S * M * C, OSTEP = S * C, LP = L / P;
  static_assert(ISTEP % 2 == 0, "an element's column is the thread's");
  for (int b = threadIdx.x; b < NB; b += blockDim.x) {
    const int l = b % C, bi = b / C;
    const int q = bi / S, r = bi - q * S;
    const int ob = (r + S * P * q) * C + l;
    auto in = [&](int j) {
      const int i = b + j * ISTEP;
      const float2 t = __ldg(yt + (i >> 1));
      const C2 sv = raw[i];
      const float G = fmaf(hx, t.x, omx) * exb * t.y;
      return mkc<C2>(__fmul_rn(sv.x, G), __fmul_rn(sv.y, G));
    };
    auto emit = [&](int k, C2 val) {
      if (k > 0 && q > 0) {
        C2 w = __ldg(tw + k * S * q);  // k q S < L
        val = cmul(val, inv ? conjf2(w) : w);
      }
      const int o = ob + k * OSTEP;
      if constexpr (OSH < 31) B[o + (o >> OSH)] = val;
      else B[o] = val;
    };
    auto tw_m = [&](int mm) {  // w_P^mm
      C2 w = __ldg(tw + mm * LP);
      return inv ? conjf2(w) : w;
    };
    butterfly<PB, C2>(in, emit, tw_m, P, inv);
  }
}

// the fixed-length transform of a column pair whose first stage reads the staged pair `raw` through the factor
// (stage_fixed_mul into a), then the remaining stages between a and b; returns the buffer holding the result
template <int L, int C, class C2>
__device__ __forceinline__ C2* fft_run_fixed_mul(const C2* raw, C2* a, C2* b, const C2* tw, bool inv,
                                                 const float2* yt, float hx, float omx, float exb) {
  constexpr CPlan P = cplan(L);
  static_assert(P.nst >= 2, "at least two stages");
  constexpr int OSH = (1 < P.nst && P.s[0] * C < 32) ? FFT_PAD : 31;
  stage_fixed_mul<P.p[0], P.s[0], L, C, OSH, C2>(raw, a, tw, inv, yt, hx, omx, exb);
  __syncthreads();
  return fft_run_fixed<L, C, 1, C2>(a, b, tw, inv);
}

template <class C2>
__device__ __forceinline__ void fft_stage(const C2* __restrict__ A, C2* __restrict__ B, int lc, int L, int P, int s,
                                          unsigned magic, const C2* __restrict__ tw, bool inv, int ish, int osh) {
  switch (P) {
    case 2: stage_loop<2, C2>(A, B, lc, L, P, s, magic, tw, inv, ish, osh); break;
    case 3: stage_loop<3, C2>(A, B, lc, L, P, s, magic, tw, inv, ish, osh); break;
    case 4: stage_loop<4, C2>(A, B, lc, L, P, s, magic, tw, inv, ish, osh); break;
    case 5: stage_loop<5, C2>(A, B, lc, L, P, s, magic, tw, inv, ish, osh); break;
    case 7: stage_loop<7, C2>(A, B, lc, L, P, s, magic, tw, inv, ish, osh); break;
    case 8: stage_loop<8, C2>(A, B, lc, L, P, s, magic, tw, inv, ish, osh); break;
    case 11: stage_loop<11, C2>(A, B, lc, L, P, s, magic, tw, inv, ish, osh); break;
    case 13: stage_loop<13, C2>(A, B, lc, L, P, s, magic, tw, inv, ish, osh); break;
    case 17: stage_loop<17, C2>(A, B, lc, L, P, s, magic, tw, inv, ish, osh); break;
    case 19: stage_loop<19, C2>(A, B, lc, L, P, s, magic, tw, inv, ish, osh); break;
    default: stage_loop<0, C2>(A, B, lc, L, P, s, magic, tw, inv, ish, osh); break;
  }
  __syncthreads();
}

// runs the plan on buf (tmp: scratch of the same capacity, fft_buf_len(fft_work_len(pl), C)); buf holds the input
// unpadded and the returned buffer the result unpadded. FIXL > 0: the length is FIXL and the plan is fixed at
// compile time; FIXL = 0: a runtime plan transformed directly; FIXL = -1: a runtime Bluestein plan (kernels are
// instantiated per FIXL, so that each carries only its own path's code and registers).
// the plan's stages on their length SL (L, or Bluestein's M): a holds the input unpadded, the returned buffer the
// result unpadded
template <int C, class C2>
__device__ C2* fft_stages(C2* a, C2* b, const FftPlan& pl, int SL, bool inv) {
  constexpr int lc = C == 4 ? 2 : (C == 2 ? 1 : 0);
  const C2* tw = (const C2*)pl.tw;
  int ish = 31;
  for (int st = 0; st < pl.nst; st++) {
    const int osh = (st + 1 < pl.nst && pl.s[st] * C < 32) ? FFT_PAD : 31;
    fft_stage<C2>(a, b, lc, SL, pl.p[st], pl.s[st], pl.magic[st], tw, inv, ish, osh);
    ish = osh;
    C2* t = a;
    a = b;
    b = t;
  }
  return a;
}

// Bluestein (the plan's M > 0): X_k = w_k sum_n (x_n w_n) conj(w_{k - n}), w_n = exp(-i pi n^2 / L), the convolution
// cyclic over M >= 2L - 1 by two length-M transforms; the inverse transform as conj(forward(conj(x))). buf and tmp
// hold fft_buf_len(M, C) values each. FM > 0: the inner length is FM, its two transforms on the plan fixed at compile
// time (L still read at run time).
template <int C, class C2, int FM = 0>
__device__ __forceinline__ C2* fft_bluestein(C2* buf, C2* tmp, const FftPlan& pl, bool inv) {
  constexpr int lc = C == 4 ? 2 : (C == 2 ? 1 : 0);
  const int L = pl.L, M = FM > 0 ? FM : pl.M;
  auto inner = [&](C2* a, C2* b, bool iv) {
    if constexpr (FM > 0) return fft_run_fixed<FM, C, 0, C2>(a, b, (const C2*)pl.tw, iv);
    else return fft_stages<C, C2>(a, b, pl, M, iv);
  };
  const float2* w = pl.chirp;
  const float2* f = pl.filt;
  for (int idx = threadIdx.x; idx < M * C; idx += blockDim.x) {
    const int i = idx >> lc;
    float2 v = make_float2(0.f, 0.f);
    if (i < L) {
      v = buf[idx];
      if (inv) v.y = -v.y;
      v = cmul(v, __ldg(w + i));
    }
    buf[idx] = v;
  }
  __syncthreads();
  C2* r = inner(buf, tmp, false);
  for (int idx = threadIdx.x; idx < M * C; idx += blockDim.x) r[idx] = cmul(r[idx], __ldg(f + (idx >> lc)));
  __syncthreads();
  C2* q = inner(r, r == buf ? tmp : buf, true);
  for (int idx = threadIdx.x; idx < L * C; idx += blockDim.x) {
    float2 v = cmul(q[idx], __ldg(w + (idx >> lc)));
    if (inv) v.y = -v.y;
    q[idx] = v;
  }
  __syncthreads();
  return q;
}

template <int FIXL, int C, class C2>
__device__ C2* fft_run(C2* buf, C2* tmp, const FftPlan& pl, bool inv) {
  static_assert(C == 1 || C == 2 || C == 4, "C: a power of two up to 4");
  static_assert(std::is_same<C2, float2>::value, "float32 transforms");
  if constexpr (FIXL > 0) {
    return fft_run_fixed<FIXL, C, 0, C2>(buf, tmp, (const C2*)pl.tw, inv);
  } else if constexpr (FIXL == -1) {  // the kernels' instantiation for Bluestein plans (pl.M > 0)
    return fft_bluestein<C, C2>(buf, tmp, pl, inv);
  } else if constexpr (FIXL < -1) {  // Bluestein with the inner length -FIXL fixed at compile time
    return fft_bluestein<C, C2, -FIXL>(buf, tmp, pl, inv);
  } else {
    return fft_stages<C, C2>(buf, tmp, pl, pl.L, inv);
  }
}

// z^e, 0 <= e < 64, of the B-spline pole z = sqrt(3) - 2 (interp.py:9): the product of its binary powers z^(2^b),
// formed in float64 at compile time and rounded once
constexpr double BZ1 = -0.26794919243112270, BZ2 = BZ1 * BZ1, BZ4 = BZ2 * BZ2, BZ8 = BZ4 * BZ4, BZ16 = BZ8 * BZ8,
                 BZ32 = BZ16 * BZ16;
__device__ __forceinline__ float zpow(int e) {
  float r = (e & 1) ? (float)BZ1 : 1.f;
  r *= (e & 2) ? (float)BZ2 : 1.f;
  r *= (e & 4) ? (float)BZ4 : 1.f;
  r *= (e & 8) ? (float)BZ8 : 1.f;
  r *= (e & 16) ? (float)BZ16 : 1.f;
  r *= (e & 32) ? (float)BZ32 : 1.f;
  return r;
}

// Cubic B-spline prefilter (interp.py:13-27, without the factor 6, which the caller folds into its scale) of C
// interleaved complex lines of length n in buf, given the lines already divided by 4 + 2 cos w on the periodic
// grid (the response multiply folds that factor into the filter). Per axis the recursion's transfer function is
// -z / (1 - 2 z cos w + z^2) = 1 / (4 + 2 cos w), so the periodic division is the recursion on the periodic
// extension; the reference's recursion on the line (causal start sum_{k < 21} z^k x[k], anticausal start
// z / (z^2 - 1) (y[n-1] + z y[n-2])) differs from it by two closed-form edge terms:
//   c[i] = c_per[i] - D0 z^(i+1) / (1 - z^2) + E z^(n-1-i),
//   D0 = y[0] - y_per[0] = sum_{k < 21} z^k x[k] - sum_{k >= 0} z^k x[-k],  E = c[n-1] - c_per[n-1],
// with x recovered locally as x[i] = c_per[i-1] + 4 c_per[i] + c_per[i+1] (circular) and the sums cut at
// z^32 < 1e-18 (lines here are at least 65 long, so the terms of the two ends never meet). scratch: 2 C float4.
template <int C>
__device__ void bspline_edge_consts(float2* buf, int n, float4* scratch) {
  const float z = (float)BZ1;
  const float g = (float)(BZ1 / (BZ2 - 1.0));
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  auto c = [&](int i, int l) { return buf[(i < 0 ? i + n : (i >= n ? i - n : i)) * C + l]; };
  auto xr = [&](int i, int l) {
    const float2 a = c(i - 1, l), b = c(i, l), d = c(i + 1, l);
    return make_float2(fmaf(4.f, b.x, a.x + d.x), fmaf(4.f, b.y, a.y + d.y));
  };
  for (int l = wid; l < C; l += (int)(blockDim.x >> 5)) {  // a warp per line: its two edge constants, lane k
    const int k = lane;                                       // taking the terms of z^k
    const float zk = zpow(k);
    const int hz = min(n, HORIZON);
    float2 d0 = make_float2(0.f, 0.f);
    if (k < hz) {
      const float2 v = xr(k, l);
      d0 = make_float2(zk * v.x, zk * v.y);
    }
    const float2 w = xr(k == 0 ? 0 : n - k, l);
    d0.x = fmaf(-zk, w.x, d0.x);
    d0.y = fmaf(-zk, w.y, d0.y);
    const float2 ya = xr(n - 1 - k, l), yb = xr(n - 2 - k, l);
    float ax = zk * ya.x, ay = zk * ya.y, bx = zk * yb.x, by = zk * yb.y;
    for (int o = 16; o; o >>= 1) {
      d0.x += __shfl_xor_sync(0xffffffffu, d0.x, o);
      d0.y += __shfl_xor_sync(0xffffffffu, d0.y, o);
      ax += __shfl_xor_sync(0xffffffffu, ax, o);
      ay += __shfl_xor_sync(0xffffffffu, ay, o);
      bx += __shfl_xor_sync(0xffffffffu, bx, o);
      by += __shfl_xor_sync(0xffffffffu, by, o);
    }
    if (lane == 0) {
      const float2 cl = c(n - 1, l);
      scratch[l] = make_float4(d0.x, d0.y, g * fmaf(z, bx, ax) - cl.x, g * fmaf(z, by, ay) - cl.y);
    }
  }
  __syncthreads();
}

// value v of row j of a line of length n with the edge terms of its constants k added (the first and last 32 rows)
__device__ __forceinline__ float2 bspline_edge_fix(float2 v, int j, int n, float4 k) {
  const float q = (float)(1.0 / (1.0 - BZ2));
  if (j < 32) {
    const float zp = zpow(j + 1);  // z^(i+1), i = j
    v.x = fmaf(-k.x * q, zp, v.x);
    v.y = fmaf(-k.y * q, zp, v.y);
  } else if (j >= n - 32) {
    const float zp = zpow(n - 1 - j);
    v.x = fmaf(k.z, zp, v.x);
    v.y = fmaf(k.w, zp, v.y);
  }
  return v;
}

// the edge constants (bspline_edge_consts) and their terms applied in place
template <int C>
__device__ void bspline_edges(float2* buf, int n, float4* scratch) {
  bspline_edge_consts<C>(buf, n, scratch);
  for (int t = threadIdx.x; t < 64 * C; t += blockDim.x) {
    const int l = t % C, j = t / C;  // j < 32: the start of the line; j >= 32: its end
    const int i = j < 32 ? j : n - 64 + j;
    buf[i * C + l] = bspline_edge_fix(buf[i * C + l], i, n, scratch[l]);
  }
  __syncthreads();
}

// reflect (mirror without repeating the edge, interp.py:38-43) of an index at most one period outside [0, n)
__device__ __forceinline__ int reflect_near(int i, int n) {
  int m = i < 0 ? -i : i;
  if (m >= n) m = 2 * (n - 1) - m;
  if (m < 0 || m >= n) m = (int)mirror_idx(i, n);  // far outside (n tiny): the general rule
  return m;
}

// ---------------------------------------------------------------- kernels
// Every kernel stages its lines in buffers of fft_buf_len(L, C) values (the transforms' padded layouts); the
// prefilter's carries live in the buffer the transform left idle. The kernels are instantiated for FIXL = 0 (any
// supported length, the plan read at run time), FIXL = -1 (Bluestein) and FIXL = each length of fft_fixed_length (the
// padded lengths of 256-, 512-, 768-, 960-, 1024-, 1536- and 2048-wide images: 320, 576, 832, 1024, 1088, 1600,
// 2112 = 8 8 3 11; the plan fixed at compile time), and FIXL = -FFT_FIXED_M (Bluestein with that inner length fixed);
// the launchers pick by the plan.

// buffer stride of the kernels that stage several lines: fft_buf_len rounded up to an even count (16-byte aligned)
__host__ __device__ constexpr int fft_buf_stride(int L, int C) { return (fft_buf_len(L, C) + 1) & ~1; }

template <int FIXL>
__global__ void __launch_bounds__(FFT_TMAX, 2) k_fft_rows_fwd_real(const float* __restrict__ img, int W, int H,
                                                                  FftPlan plw, int ph, float2* __restrict__ out) {
  extern __shared__ __align__(16) unsigned char smraw[];
  float2* sm = (float2*)smraw;
  const int pw = FIXL > 0 ? FIXL : plw.L;
  float2* t = sm + fft_buf_len(FIXL > 0 ? FIXL : fft_work_len(plw), 1);
  const int yp = blockIdx.x;
  const int ys = reflect_near(yp - PAD, H);
  const float* row = img + (size_t)ys * W;
  for (int x = threadIdx.x; x < pw; x += blockDim.x) sm[x] = make_float2(__ldg(row + reflect_near(x - PAD, W)), 0.f);
  __syncthreads();
  float2* r = fft_run<FIXL, 1>(sm, t, plw, false);
  float2* o = out + (size_t)yp * pw;
  for (int x = threadIdx.x; x < pw; x += blockDim.x) o[x] = r[x];
}

// The column pass of the responses in two kernels, so that a block holds only two buffers of C columns
// (several blocks per SM instead of one): k_fft_cols_fwd writes the column spectrum S (ph x pw, row-major,
// small enough to stay in L2), then the inverse pass (k_fft_cols_pair, or k_fft_cols_inv_filter where the column
// pair does not fit beside the two buffers) multiplies S by the factors of each plane, inverts along y and stores.
constexpr int COLS_TMAX = 320;  // threads per block of the split column pass

template <int C, int FIXL>
__global__ void __launch_bounds__(COLS_TMAX, 3) k_fft_cols_fwd(const float2* Tin, FftPlan plh, int pw, float2* S) {
  constexpr int LC = C == 4 ? 2 : (C == 2 ? 1 : 0);
  extern __shared__ __align__(16) unsigned char smraw[];
  float2* A = (float2*)smraw;
  const int ph = FIXL > 0 ? FIXL : plh.L, n = ph * C;
  float2* B = A + fft_buf_stride(FIXL > 0 ? FIXL : fft_work_len(plh), C);  // 16-byte aligned: the result may be either buffer
  const int x0 = blockIdx.x * C;
  // C = 2 with an even row pitch: each row of the pair is 16 bytes on a 16-byte boundary, copied asynchronously
  const bool rows16 = C == 2 && pw % 2 == 0;
  if (rows16) {
    for (int y = threadIdx.x; y < ph; y += blockDim.x) __pipeline_memcpy_async(A + 2 * y, Tin + (size_t)y * pw + x0, 16);
    __pipeline_commit();
    __pipeline_wait_prior(0);
  } else {
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      int y = i >> LC, x = x0 + (i & (C - 1));
      A[i] = x < pw ? Tin[(size_t)y * pw + x] : make_float2(0.f, 0.f);
    }
  }
  __syncthreads();
  float2* r = fft_run<FIXL, C>(A, B, plh, false);
  if (rows16) {
    for (int y = threadIdx.x; y < ph; y += blockDim.x) *(float4*)(S + (size_t)y * pw + x0) = *(const float4*)(r + 2 * y);
  } else {
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      int y = i >> LC, x = x0 + (i & (C - 1));
      if (x < pw) S[(size_t)y * pw + x] = r[i];
    }
  }
}

// The inverse column pass with the spectrum of a column pair staged once per block: the block copies its two
// columns of S (ph x 2) into shared memory, then for each of its planes multiplies them by the plane's factor into
// A, inverts along y (A, B) and stores the pair. REFPACK = false: the responses of the filters
// [RESP_G blockIdx.y, RESP_G (blockIdx.y + 1)) (x G_k and the B-spline prefilter's periodic factors, inverse,
// the prefilter's edge terms along y) into plane k of U. REFPACK = true: variant v = blockIdx.y of the reference
// pack (S G, S G i fx, S G i fy; factors in float64) of the filters [k0, k1) into plane 3 (k - k0) + v of U.
// A thread's column is fixed (blockDim is even), so the x factors are read once.
constexpr int RESP_G = 4;

// A[i] = raw[i] f(i, t_i) for the n values of a column pair, t_i the row table entry of element i (row i / 2). With
// the length fixed (FIXL, blockDim = NT) the table loads of UN elements are issued together before their
// multiplies, so that their latencies overlap.
template <int FIXL, int NT, int UN, class T, class Fn>
__device__ __forceinline__ void cols_multiply(int n, const T* __restrict__ tab, Fn f) {
  if constexpr (FIXL > 0) {
    constexpr int NI = (2 * FIXL + NT - 1) / NT;
#pragma unroll
    for (int m0 = 0; m0 < NI; m0 += UN) {
      T tv[UN];
#pragma unroll
      for (int u = 0; u < UN; u++) {
        const int i = threadIdx.x + NT * (m0 + u);
        if (m0 + u < NI && i < 2 * FIXL) tv[u] = __ldg(tab + (i >> 1));
      }
#pragma unroll
      for (int u = 0; u < UN; u++) {
        const int i = threadIdx.x + NT * (m0 + u);
        if (m0 + u < NI && i < 2 * FIXL) f(i, tv[u]);
      }
    }
  } else {
    for (int i = threadIdx.x; i < n; i += blockDim.x) f(i, __ldg(tab + (i >> 1)));
  }
}

// threads of the fixed-length column-pair kernel: the responses COLS_TMAX; the reference pack, whose float64 factors
// take more time per element, one per radix-8 butterfly of the two columns (2 x 2112 / 8)
constexpr int PAIR_T_REF = 544;
template <bool REFPACK>
constexpr int pair_threads(int fixl) { return fixl > 0 && REFPACK ? PAIR_T_REF : COLS_TMAX; }
template <bool REFPACK, int FIXL>
__global__ void __launch_bounds__(pair_threads<REFPACK>(FIXL), 2) k_fft_cols_pair(const float2* __restrict__ S, FftPlan plh, int pw,
                                                                GaborTables g, int k0, int k1, float2* __restrict__ U) {
  constexpr int C = 2;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int ph = FIXL > 0 ? FIXL : plh.L, n = ph * C, tid = threadIdx.x, nt = blockDim.x;
  float2* raw = (float2*)smraw;
  float2* A = raw + n;
  float2* B = A + fft_buf_stride(FIXL > 0 ? FIXL : fft_work_len(plh), C);
  const int x0 = blockIdx.x * C;
  const bool rows16 = x0 + 1 < pw && pw % 2 == 0;  // each row of the pair is 16 bytes on a 16-byte boundary
  if (rows16) {
    for (int y = tid; y < ph; y += nt) __pipeline_memcpy_async(raw + 2 * y, S + (size_t)y * pw + x0, 16);
    __pipeline_commit();
    __pipeline_wait_prior(0);
  } else {
    for (int i = tid; i < n; i += nt) {
      const int y = i >> 1, x = x0 + (i & 1);
      raw[i] = x < pw ? S[(size_t)y * pw + x] : make_float2(0.f, 0.f);
    }
  }
  __syncthreads();
  const int x = min(x0 + (tid & 1), pw - 1);
  auto store = [&](const float2* r, int plane) {
    float2* dst = U + (size_t)plane * ph * pw + x0;
    if (rows16) {
      for (int y = tid; y < ph; y += nt) *(float4*)(dst + (size_t)y * pw) = *(const float4*)(r + 2 * y);
    } else {
      for (int i = tid; i < n; i += nt)
        if (x0 + (i & 1) < pw) dst[(size_t)(i >> 1) * pw + (i & 1)] = r[i];
    }
  };
  // the same with the prefilter's edge terms along y (constants kc of the two columns) added as the rows are stored
  auto store_edges = [&](const float2* r, const float4* kc, int plane) {
    float2* dst = U + (size_t)plane * ph * pw + x0;
    if (rows16) {
      for (int y = tid; y < ph; y += nt) {
        const float4 v = *(const float4*)(r + 2 * y);
        const float2 a = bspline_edge_fix(make_float2(v.x, v.y), y, ph, kc[0]);
        const float2 b = bspline_edge_fix(make_float2(v.z, v.w), y, ph, kc[1]);
        *(float4*)(dst + (size_t)y * pw) = make_float4(a.x, a.y, b.x, b.y);
      }
    } else {
      for (int i = tid; i < n; i += nt)
        if (x0 + (i & 1) < pw) dst[(size_t)(i >> 1) * pw + (i & 1)] = bspline_edge_fix(r[i], i >> 1, ph, kc[i & 1]);
    }
  };
  if (!REFPACK) {
    const float hx = __ldg(g.hxf + x), omx = __ldg(g.omxf + x), bx = __ldg(g.bxf + x);
    const int kend = min(g.F, (int)(blockIdx.y + 1) * RESP_G);
    for (int k = blockIdx.y * RESP_G; k < kend; k++) {
      // G = (hx + omx omy) ex ey (bx by): the x factors of the thread's column, (omy, ey by) from the row table
      const float exb = __ldg(g.exf + (size_t)k * pw + x) * bx;
      float2* r;
      if constexpr (FIXL > 0) {
        r = fft_run_fixed_mul<FIXL, C, float2>(raw, A, B, (const float2*)plh.tw, true, g.yt2 + (size_t)k * ph, hx,
                                               omx, exb);
      } else {
        cols_multiply<FIXL, COLS_TMAX, 14>(n, g.yt2 + (size_t)k * ph, [&](int i, float2 t) {
          const float2 sv = raw[i];
          const float G = fmaf(hx, t.x, omx) * exb * t.y;
          A[i] = make_float2(sv.x * G, sv.y * G);
        });
        __syncthreads();
        r = fft_run<FIXL, C>(A, B, plh, true);
      }
      float2* idle = r == A ? B : A;
      bspline_edge_consts<C>(r, ph, (float4*)idle);  // the prefilter's edge terms along y, added by the store
      store_edges(r, (const float4*)idle, k);
      __syncthreads();
    }
  } else {
    const int v = blockIdx.y;
    const double hx = g.hx[x], omx = g.omx[x], fx = g.fx[x];
    for (int k = k0; k < k1; k++) {
      const double ex = g.ex[(size_t)k * pw + x];
      const double* eyk = g.ey + (size_t)k * ph;
      // the row factors omy[y], ey_k[y] (and fy[y]) per element
      auto mul = [&](int i, double omy, double eyv, double fyv) {
        const float2 sv = raw[i];
        const double G = fma(hx, omy, omx) * ex * eyv;
        double re = sv.x * G, im = sv.y * G;
        if (v == 1) { const double t = re; re = -im * fx; im = t * fx; }          // x i fx
        else if (v == 2) { const double t = re; re = -im * fyv; im = t * fyv; }  // x i fy
        A[i] = make_float2((float)re, (float)im);
      };
      if constexpr (FIXL > 0) {
        // the three row factors of UN elements loaded together before their multiplies, so that their latencies
        // overlap (blockDim = PAIR_T_REF)
        constexpr int NT = PAIR_T_REF, NI = (2 * FIXL + NT - 1) / NT, UN = 4;
#pragma unroll
        for (int m0 = 0; m0 < NI; m0 += UN) {
          double oy[UN], ey[UN], fy[UN];
#pragma unroll
          for (int u = 0; u < UN; u++) {
            const int i = threadIdx.x + NT * (m0 + u);
            oy[u] = ey[u] = fy[u] = 0.0;
            if (m0 + u < NI && i < 2 * FIXL) {
              const int y = i >> 1;
              oy[u] = __ldg(g.omy + y);
              ey[u] = __ldg(eyk + y);
              if (v == 2) fy[u] = __ldg(g.fy + y);
            }
          }
#pragma unroll
          for (int u = 0; u < UN; u++) {
            const int i = threadIdx.x + NT * (m0 + u);
            if (m0 + u < NI && i < 2 * FIXL) mul(i, oy[u], ey[u], fy[u]);
          }
        }
      } else {
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
          const int y = i >> 1;
          mul(i, __ldg(g.omy + y), __ldg(eyk + y), v == 2 ? __ldg(g.fy + y) : 0.0);
        }
      }
      __syncthreads();
      float2* r = fft_run<FIXL, C>(A, B, plh, true);
      store(r, 3 * (k - k0) + v);
      __syncthreads();
    }
  }
}

// The same inverse column pass with one block per (C columns, plane) and no staged spectrum: the form for padded
// heights whose column pair does not fit in shared memory beside the two transform buffers.
template <int C, bool REFPACK, int FIXL>
__global__ void __launch_bounds__(COLS_TMAX, 3) k_fft_cols_inv_filter(const float2* __restrict__ S, FftPlan plh, int pw,
                                                                      GaborTables g, int k0, float2* __restrict__ U) {
  constexpr int LC = C == 4 ? 2 : (C == 2 ? 1 : 0);
  extern __shared__ __align__(16) unsigned char smraw[];
  float2* A = (float2*)smraw;
  const int ph = plh.L, n = ph * C;
  float2* B = A + fft_buf_len(fft_work_len(plh), C);
  const int x0 = blockIdx.x * C;
  const int k = REFPACK ? k0 + blockIdx.y / 3 : blockIdx.y, var = REFPACK ? blockIdx.y % 3 : 0;
  const float* exkf = g.exf + (size_t)k * pw;
  const float* eykf = g.eyf + (size_t)k * ph;
  const double* exk = g.ex + (size_t)k * pw;
  const double* eyk = g.ey + (size_t)k * ph;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    int y = i >> LC, xr = x0 + (i & (C - 1)), x = min(xr, pw - 1);
    float2 sv = xr < pw ? S[(size_t)y * pw + x] : make_float2(0.f, 0.f);
    if (!REFPACK) {
      // the Gabor factor and the B-spline prefilter on the periodic grid along both axes
      float G = fmaf(__ldg(g.hxf + x), __ldg(g.omyf + y), __ldg(g.omxf + x)) * (__ldg(exkf + x) * __ldg(eykf + y)) *
                (__ldg(g.bxf + x) * __ldg(g.byf + y));
      A[i] = make_float2(sv.x * G, sv.y * G);
    } else {
      double G = fma(g.hx[x], g.omy[y], g.omx[x]) * exk[x] * eyk[y];
      double re = sv.x * G, im = sv.y * G;
      if (var == 1) { double f = g.fx[x]; double t = re; re = -im * f; im = t * f; }        // x i fx
      else if (var == 2) { double f = g.fy[y]; double t = re; re = -im * f; im = t * f; }   // x i fy
      A[i] = make_float2((float)re, (float)im);
    }
  }
  __syncthreads();
  float2* r = fft_run<FIXL, C>(A, B, plh, true);
  if (!REFPACK) {
    float2* idle = r == A ? B : A;
    bspline_edges<C>(r, ph, (float4*)(((uintptr_t)idle + 15) & ~(uintptr_t)15));  // the prefilter's edge terms along y
  }
  float2* dst = U + (size_t)blockIdx.y * ph * pw;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    int y = i >> LC, x = x0 + (i & (C - 1));
    if (x < pw) dst[(size_t)y * pw + x] = r[i];
  }
}

// Inverse row transforms of the filtered spectra into the responses R, persistent: a block walks the node rows
// blockIdx.x, + gridDim.x, ...; per node row it transforms the row's two lines one after the other, each followed by
// the prefilter's edge terms along x, and stores both at once with the scale 36 / (ph pw).
// R holds the filters in pairs, node-major: pair j = filters 2j and 2j + 1 (the second a copy of filter F - 1 when F
// is odd), filter 2j + c at node (y, x) at R[((j ph + y) pw + x) 2 + c], so that one 16-byte load takes a tap of both
// filters of a pair, and node row (j, y) is one run of pw 16-byte stores.
// Four line buffers: the first line's result waits in one while the second line is transformed in two others, and the
// fourth receives the next row's first line (cp.async) meanwhile; the next row's second line is copied while its
// first line is transformed. (Both lines in one interleaved transform waits longer at the Stockham barriers of its
// 512-thread blocks: 0.377 ms per launch at 2112; one line per block with 8-byte stores 16 bytes apart: 0.36 ms.)
template <int FIXL>
__global__ void __launch_bounds__(FIXL > 0 ? 288 : FFT_TMAX, FIXL > 0 ? 3 : 2)
    k_fft_rows_inv_resp(const float2* __restrict__ U, FftPlan plw, int ph, int F, int nrows, float scale,
                        float2* __restrict__ R) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int L = FIXL > 0 ? FIXL : plw.L, nb = fft_buf_stride(FIXL > 0 ? FIXL : fft_work_len(plw), 1);
  float2* b0 = (float2*)smraw;
  float2 *x0 = b0, *x1 = b0 + nb, *fa = b0 + 2 * nb, *fb = b0 + 3 * nb;
  // copies line c of node row `row` into dst as one group of asynchronous copies (an empty group past the end)
  auto fetch = [&](int row, int c, float2* dst) {
    if (row < nrows) {
      const int j = row / ph, y = row - j * ph;
      const float2* src = U + ((size_t)min(2 * j + c, F - 1) * ph + y) * L;
      if (L % 2 == 0) {  // 16-byte chunks: the line starts on a 16-byte boundary
        for (int i = threadIdx.x; i < L / 2; i += blockDim.x) __pipeline_memcpy_async(dst + 2 * i, src + 2 * i, 16);
      } else {
        for (int i = threadIdx.x; i < L; i += blockDim.x) __pipeline_memcpy_async(dst + i, src + i, 8);
      }
    }
    __pipeline_commit();
  };
  int row = blockIdx.x;
  fetch(row, 0, x0);
  fetch(row, 1, x1);
  for (; row < nrows; row += gridDim.x) {
    const int nxt = row + gridDim.x;
    __pipeline_wait_prior(1);  // line 0 has landed (line 1 may be in flight)
    __syncthreads();
    float2* r0 = fft_run<FIXL, 1>(x0, fa, plw, true);
    float2* s0 = r0 == x0 ? fa : x0;
    bspline_edge_consts<1>(r0, L, (float4*)s0);  // the edge terms along x, added by the store
    const float4 k0 = *(const float4*)s0;        // s0 is line 1's transform buffer next
    fetch(nxt, 0, fb);         // the next row's line 0 during line 1's transform
    __pipeline_wait_prior(1);  // line 1 has landed
    __syncthreads();
    float2* r1 = fft_run<FIXL, 1>(x1, s0, plw, true);
    float2* s1 = r1 == x1 ? s0 : x1;
    bspline_edge_consts<1>(r1, L, (float4*)s1);
    const float4 k1 = *(const float4*)s1;
    float4* o = (float4*)R + (size_t)row * L;
    for (int x = threadIdx.x; x < L; x += blockDim.x) {
      const float2 a = bspline_edge_fix(r0[x], x, L, k0), b = bspline_edge_fix(r1[x], x, L, k1);
      o[x] = make_float4(a.x * scale, a.y * scale, b.x * scale, b.y * scale);
    }
    __syncthreads();
    // free now: r0, r1 and s1; the next row's line 0 is in fb
    fetch(nxt, 1, s1);
    x0 = fb;
    x1 = s1;
    fa = r0;
    fb = r1;
  }
  __pipeline_wait_prior(0);
}

template <int FIXL>
__global__ void __launch_bounds__(FFT_TMAX, 2) k_fft_rows_inv_ref(const float2* __restrict__ U, FftPlan plw, int ph, int W,
                                                               int H, int k0, float4* __restrict__ ref4,
                                                               float* __restrict__ amp) {
  extern __shared__ __align__(16) unsigned char smraw[];
  float2* sm = (float2*)smraw;
  const int pw = FIXL > 0 ? FIXL : plw.L, nb = fft_buf_stride(FIXL > 0 ? FIXL : fft_work_len(plw), 1);
  float2* t = sm + 3 * nb;
  const int y = blockIdx.x, kk = blockIdx.y, k = k0 + kk;  // y: row of the W x H crop
  const size_t plane = (size_t)ph * pw;
  // the three rows in three groups of asynchronous copies: rows 1 and 2 land while row 0 is transformed
  for (int v = 0; v < 3; v++) {
    const float2* src = U + (size_t)(3 * kk + v) * plane + (size_t)(y + PAD) * pw;
    if (pw % 2 == 0) {  // 16-byte chunks: the row starts on a 16-byte boundary
      for (int i = threadIdx.x; i < pw / 2; i += blockDim.x) __pipeline_memcpy_async(sm + v * nb + 2 * i, src + 2 * i, 16);
    } else {
      for (int i = threadIdx.x; i < pw; i += blockDim.x) __pipeline_memcpy_async(sm + v * nb + i, src + i, 8);
    }
    __pipeline_commit();
  }
  float2* rr[3];
  for (int v = 0; v < 3; v++) {
    if (v == 0) __pipeline_wait_prior(2);
    else if (v == 1) __pipeline_wait_prior(1);
    else __pipeline_wait_prior(0);
    __syncthreads();
    float2* res = fft_run<FIXL, 1>(sm + v * nb, t, plw, true);
    if (res != sm + v * nb) {
      for (int x = threadIdx.x; x < pw; x += blockDim.x) sm[v * nb + x] = res[x];
      __syncthreads();
    }
    rr[v] = sm + v * nb;
  }
  const double sc = 1.0 / ((double)ph * (double)pw);
  for (int x = threadIdx.x; x < W; x += blockDim.x) {
    int xp = x + PAD;
    float2 a = rr[0][xp], b = rr[1][xp], c = rr[2][xp];
    double rre = a.x * sc, rim = a.y * sc;
    double xre = b.x * sc, xim = b.y * sc, yre = c.x * sc, yim = c.y * sc;
    double a2 = rre * rre + rim * rim + 1e-12;
    // Im(conj(r) rx) / a2 (phaseflow.py:109-110), one reciprocal for both (stored as float32)
    const double ia2 = 1.0 / a2;
    double gx = (rre * xim - rim * xre) * ia2;
    double gy = (rre * yim - rim * yre) * ia2;
    size_t o = (size_t)k * W * H + (size_t)y * W + x;
    ref4[o] = make_float4((float)rre, (float)rim, (float)gx, (float)gy);
    amp[o] = (float)sqrt(a2);
  }
}

template <int FIXL>
__global__ void __launch_bounds__(FFT_TMAX, 2) k_fft_lines(float2* data, FftPlan pl, int inv) {
  extern __shared__ float2 sm[];
  const int L = FIXL > 0 ? FIXL : pl.L;
  float2* row = data + (size_t)blockIdx.x * L;
  for (int x = threadIdx.x; x < L; x += blockDim.x) sm[x] = row[x];
  __syncthreads();
  float2* r = fft_run<FIXL, 1>(sm, sm + fft_buf_len(FIXL > 0 ? FIXL : fft_work_len(pl), 1), pl, inv != 0);
  for (int x = threadIdx.x; x < L; x += blockDim.x) row[x] = r[x];
}

// ---------------------------------------------------------------- launchers
constexpr size_t SMEM_MAX = 227 * 1024;

static void set_smem(const void* fn, size_t bytes) {
  raise_smem_limit(fn, bytes);
}

static size_t fbytes(int L, int C) { return (size_t)fft_buf_len(L, C) * sizeof(float2); }

// shared memory of a transform with the prefilter's edge terms: two buffers, the idle one holding C float4
// from its first 16-byte boundary
static size_t smem_prefilter(int L, int C, int T) {
  (void)T;
  return std::max<size_t>(2 * fbytes(L, C), fbytes(L, C) + 16 + (size_t)C * sizeof(float4));
}
// k_fft_cols_pair: the column pair (2 L values) and two buffers of the work length (L, or Bluestein's M) at the even
// stride
static size_t smem_cols_pair(int L, int WL) {
  return ((size_t)2 * L + 2 * (size_t)fft_buf_stride(WL, 2)) * sizeof(float2);
}
// k_fft_rows_inv_resp: four line buffers at the even stride
static size_t smem_rows_resp(int L) { return 4 * (size_t)fft_buf_stride(L, 1) * sizeof(float2); }

// calls f with std::integral_constant<int, FIXL> for the kernels' instantiation of a plan: a length with a plan fixed
// at compile time, a Bluestein plan whose inner length -FIXL has one (FIXL < -1), the runtime direct plan (0) or the
// runtime Bluestein plan (-1)
template <class Fn>
static void by_plan(const FftPlan& pl, Fn f) {
  using std::integral_constant;
  if (!pl.M) {
    switch (pl.L) {
      case 320: f(integral_constant<int, 320>{}); return;
      case 576: f(integral_constant<int, 576>{}); return;
      case 832: f(integral_constant<int, 832>{}); return;
      case 1024: f(integral_constant<int, 1024>{}); return;
      case 1088: f(integral_constant<int, 1088>{}); return;
      case 1600: f(integral_constant<int, 1600>{}); return;
      case FFT_FIXED_L: f(integral_constant<int, FFT_FIXED_L>{}); return;
      default: break;
    }
  }
  // the Bluestein inner length of 604 = 4 151 (the padded height of 540-row frames: the CLI's 1080p video at scale 2)
  if (pl.M == FFT_FIXED_M) {
    f(integral_constant<int, -FFT_FIXED_M>{});
    return;
  }
  if (pl.M) f(integral_constant<int, -1>{});
  else f(integral_constant<int, 0>{});
}

bool fft_fixed_length(int L) {
  return L == 320 || L == 576 || L == 832 || L == 1024 || L == 1088 || L == 1600 || L == FFT_FIXED_L;
}

// blocks of a persistent launch: as many as are resident at once, at most one per unit of work
static int persistent_blocks(const void* fn, int threads, size_t smem, int work) {
  int dev = 0, sms = 0, per = 0;
  OFC_CUDA(cudaGetDevice(&dev));
  OFC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  OFC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, threads, smem));
  return std::max(1, std::min(work, std::max(per, 1) * sms));
}

bool fft_fits(int ph, int pw) {
  try {
    const int wh = fft_work_length(ph), ww = fft_work_length(pw);
    if (wh == 0 || ww == 0) return false;
    int Tc = std::min(fft_threads(wh, 2), COLS_TMAX);
    if (smem_prefilter(wh, 2, Tc) > SMEM_MAX || 2 * (size_t)fft_buf_stride(wh, 2) * sizeof(float2) > SMEM_MAX) return false;
    return 4 * (size_t)fft_buf_stride(ww, 1) * sizeof(float2) <= SMEM_MAX && smem_rows_resp(ww) <= SMEM_MAX;
  } catch (const Error&) {
    return false;
  }
}

void launch_fft_rows_fwd_real(const float* img, int W, int H, const FftPlan& plw, int ph, float2* out, cudaStream_t st) {
  int T = fft_threads(fft_work_len(plw), 1);
  size_t sm = 2 * fbytes(fft_work_len(plw), 1);
  by_plan(plw, [&](auto fl) {
    constexpr int FL = decltype(fl)::value;
    set_smem((const void*)k_fft_rows_fwd_real<FL>, sm);
    OFC_LAUNCH(k_fft_rows_fwd_real<FL>, ph, T, sm, st, img, W, H, plw, ph, out);
  });
}

static void cols_fwd(float2* T, const FftPlan& plh, int pw, cudaStream_t st) {
  constexpr int C = 2;
  const int wh = fft_work_len(plh);
  int nt = std::min(fft_threads(wh, C), COLS_TMAX);
  size_t sm_f = 2 * (size_t)fft_buf_stride(wh, C) * sizeof(float2);
  // in place: a block reads its C columns whole before it writes their spectrum back
  by_plan(plh, [&](auto fl) {
    constexpr int FL = decltype(fl)::value;
    set_smem((const void*)k_fft_cols_fwd<C, FL>, sm_f);
    OFC_LAUNCH((k_fft_cols_fwd<C, FL>), div_up(pw, C), nt, sm_f, st, T, plh, pw, T);
  });
}

// the inverse column pass of the responses (REFPACK false, planes = filters) or of the reference pack's filters
// [k0, k1) (planes = 3 (k1 - k0))
template <bool REFPACK>
static void cols_inverse(const float2* S, const FftPlan& plh, int pw, const GaborTables& g, int k0, int k1, float2* U,
                         cudaStream_t st) {
  constexpr int C = 2;
  const int ph = plh.L, wh = fft_work_len(plh);
  int nt = std::min(fft_threads(wh, C), COLS_TMAX);
  const size_t sm_p = smem_cols_pair(ph, wh);
  if (sm_p <= SMEM_MAX) {
    if (fft_fixed_length(ph)) nt = pair_threads<REFPACK>(ph);  // the block size the fixed-length kernel assumes
    dim3 grid(div_up(pw, C), REFPACK ? 3 : div_up(g.F, RESP_G));
    by_plan(plh, [&](auto fl) {
      constexpr int FL = decltype(fl)::value;
      set_smem((const void*)k_fft_cols_pair<REFPACK, FL>, sm_p);
      if constexpr (REFPACK) OFC_LAUNCH((k_fft_cols_pair<true, FL>), grid, nt, sm_p, st, S, plh, pw, g, k0, k1, U);
      else OFC_LAUNCH((k_fft_cols_pair<false, FL>), grid, nt, sm_p, st, S, plh, pw, g, k0, k1, U);
    });
    return;
  }
  size_t sm_i = REFPACK ? 2 * fbytes(wh, C) : smem_prefilter(wh, C, nt);
  if (sm_i > SMEM_MAX) throw Error(OFC_ERR_WINDOW, "padded height " + std::to_string(ph) + " too large for the column pass");
  dim3 grid(div_up(pw, C), REFPACK ? 3 * (k1 - k0) : g.F);
  auto launch = [&](auto fl) {
    constexpr int FL = decltype(fl)::value;
    set_smem((const void*)k_fft_cols_inv_filter<C, REFPACK, FL>, sm_i);
    OFC_LAUNCH((k_fft_cols_inv_filter<C, REFPACK, FL>), grid, nt, sm_i, st, S, plh, pw, g, k0, U);
  };
  if (plh.M) launch(std::integral_constant<int, -1>{});
  else launch(std::integral_constant<int, 0>{});
}

void launch_fft_cols_filters(float2* T, const FftPlan& plh, int pw, const GaborTables& g, float2* U, cudaStream_t st) {
  cols_fwd(T, plh, pw, st);
  cols_inverse<false>(T, plh, pw, g, 0, g.F, U, st);
}

void launch_fft_rows_inv_resp(const float2* U, const FftPlan& plw, int ph, int F, float2* R, cudaStream_t st) {
  const int T = fft_threads(fft_work_len(plw), 1);
  const size_t sm = smem_rows_resp(fft_work_len(plw));
  const float scale = (float)(36.0 / ((double)ph * (double)plw.L));
  const int nrows = ((F + 1) / 2) * ph;
  by_plan(plw, [&](auto fl) {
    constexpr int FL = decltype(fl)::value;
    const void* fn = (const void*)k_fft_rows_inv_resp<FL>;
    set_smem(fn, sm);
    OFC_LAUNCH(k_fft_rows_inv_resp<FL>, persistent_blocks(fn, T, sm, nrows), T, sm, st, U, plw, ph, F, nrows, scale,
               R);
  });
}

void launch_fft_cols_fwd(float2* T, const FftPlan& plh, int pw, cudaStream_t st) { cols_fwd(T, plh, pw, st); }

void launch_fft_cols_ref_f32(const float2* S, const FftPlan& plh, int pw, const GaborTables& g, int k0, int k1,
                             float2* U, cudaStream_t st) {
  cols_inverse<true>(S, plh, pw, g, k0, k1, U, st);
}

void launch_fft_rows_inv_ref_f32(const float2* U, const FftPlan& plw, int ph, int k0, int k1, int W, int H,
                                 float4* ref4, float* amp, cudaStream_t st) {
  int T = fft_threads(fft_work_len(plw), 1);
  size_t sm = 4 * (size_t)fft_buf_stride(fft_work_len(plw), 1) * sizeof(float2);
  dim3 grid(H, k1 - k0);
  by_plan(plw, [&](auto fl) {
    constexpr int FL = decltype(fl)::value;
    set_smem((const void*)k_fft_rows_inv_ref<FL>, sm);
    OFC_LAUNCH(k_fft_rows_inv_ref<FL>, grid, T, sm, st, U, plw, ph, W, H, k0, ref4, amp);
  });
}

void launch_fft_lines(float2* data, int lines, const FftPlan& pl, bool inverse, cudaStream_t st) {
  int T = fft_threads(fft_work_len(pl), 1);
  size_t sm = 2 * fbytes(fft_work_len(pl), 1);
  by_plan(pl, [&](auto fl) {
    constexpr int FL = decltype(fl)::value;
    set_smem((const void*)k_fft_lines<FL>, sm);
    OFC_LAUNCH(k_fft_lines<FL>, lines, T, sm, st, data, pl, inverse ? 1 : 0);
  });
}

}  // namespace ofc
