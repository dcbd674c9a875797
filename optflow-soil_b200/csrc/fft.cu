// fft.cu -- FP32 mixed-radix FFTs in shared memory with the fused Gabor multiply and B-spline prefilter.
//
// One thread block transforms C interleaved lines held in shared memory (element i of line l at
// buf[i * C + l]), ping-ponging between two buffers of L * C values: each Stockham stage reads a butterfly's
// inputs from one and writes its outputs to the other. Radices 2, 3, 4, 5 and 8 have register butterflies;
// other primes (up to 31) a direct DFT. Twiddles come from a table rounded from float64.
//
// The pass structure of one "responses" evaluation (per outer iteration of the fine stage):
//   rows:    reflect pad + real->complex + forward row FFT                      (read 4 B/px, write 8 B/px)
//   columns: forward column FFT, then per filter k: x G_k (separable, float64 tables), inverse column FFT,
//            causal + anticausal B-spline prefilter along y                       (read 8, write 8F)
//   rows:    inverse row FFT, prefilter along x, scale 36 / (ph pw)               (read 8F, write 8F)
// The prefilter along y commutes with the inverse FFT along x (operators on different axes), so the
// result is bspline_coeffs(ifft2(F2 * G)) of phaseflow.py:456 up to rounding.
#include "fft.cuh"

#include <cmath>

namespace ofc {

// ------------------------------------------------------------------------------------------ host
bool fft_supported(int L) {
  if (L < 1) return false;
  int m = L;
  for (int p : {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31})
    while (m % p == 0) m /= p;
  return m == 1;
}

FftPlan fft_make_plan(int L) {
  if (!fft_supported(L))
    throw Error(OFC_ERR_WINDOW, "FFT length " + std::to_string(L) + " has a prime factor above 31");
  FftPlan pl;
  pl.L = L;
  int m = L;
  std::vector<int> f;
  while (m % 8 == 0) { f.push_back(8); m /= 8; }
  while (m % 4 == 0) { f.push_back(4); m /= 4; }
  while (m % 2 == 0) { f.push_back(2); m /= 2; }
  for (int p : {3, 5, 7, 11, 13, 17, 19, 23, 29, 31})
    while (m % p == 0) { f.push_back(p); m /= p; }
  if ((int)f.size() > FFT_MAXST) throw Error(OFC_ERR_WINDOW, "FFT length " + std::to_string(L) + " needs too many stages");
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

std::vector<double2> fft_twiddles_f64(int L) {
  std::vector<double2> t(L);
  for (int i = 0; i < L; i++) {
    double a = -2.0 * PI * (double)i / (double)L;
    t[i] = make_double2(std::cos(a), std::sin(a));
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

std::vector<double> gabor_tables_host(int ph, int pw, const ofc_config& c) {
  int F = c.n_scales * c.n_orient;
  std::vector<double> t((size_t)3 * (pw + ph) + (size_t)F * (pw + ph));
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
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 conjf2(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 rot(double2 a, bool inv) { return inv ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x); }
template <class C2> __device__ __forceinline__ C2 mkc(double re, double im);
template <> __device__ __forceinline__ float2 mkc<float2>(double re, double im) { return make_float2((float)re, (float)im); }
template <> __device__ __forceinline__ double2 mkc<double2>(double re, double im) { return make_double2(re, im); }

// Odd-radix butterfly with the symmetric form: for j = 1..(P-1)/2, a_j = v_j + v_{P-j}, b_j = v_j - v_{P-j};
// o_0 = v_0 + sum a_j; o_k = v_0 + sum_j a_j cos_jk + i sum_j b_j sin_jk, o_{P-k} = the same with -i, where
// w^{jk} = cos_jk + i sin_jk (w = exp(-2 pi i / P), conjugated for the inverse) is read from the twiddle table.
template <int P, class C2, class Emit>
__device__ __forceinline__ void odd_butterfly(const C2* in, size_t istep, const C2* __restrict__ tw, int LP, bool inv,
                                              Emit emit) {
  constexpr int Hh = (P - 1) / 2;
  C2 v0 = in[0];
  C2 av[Hh], bv[Hh];
#pragma unroll
  for (int j = 1; j <= Hh; j++) {
    C2 x = in[j * istep], y = in[(P - j) * istep];
    av[j - 1] = cadd(x, y);
    bv[j - 1] = csub(x, y);
  }
  C2 s0 = v0;
#pragma unroll
  for (int j = 0; j < Hh; j++) s0 = cadd(s0, av[j]);
  emit(0, s0);
#pragma unroll
  for (int k = 1; k <= Hh; k++) {
    C2 t = v0, u = mkc<C2>(0.0, 0.0);
#pragma unroll
    for (int j = 1; j <= Hh; j++) {
      C2 w = __ldg(tw + (size_t)((j * k) % P) * LP);
      auto cs = w.x;
      auto sn = inv ? -w.y : w.y;
      t.x = fma(av[j - 1].x, cs, t.x);
      t.y = fma(av[j - 1].y, cs, t.y);
      u.x = fma(bv[j - 1].x, sn, u.x);
      u.y = fma(bv[j - 1].y, sn, u.y);
    }
    // i u = (-u.y, u.x)
    emit(k, mkc<C2>(t.x - u.y, t.y + u.x));
    emit(P - k, mkc<C2>(t.x + u.y, t.y - u.x));
  }
}

// One Stockham stage of radix P from buffer A to buffer B (C interleaved lines of length L, C = 1 << lc). q, r
// of a butterfly come from multiplications by precomputed reciprocals (magic = ceil(2^32 / s), exact for the
// sizes here). Radices 2, 4, 8 have hand-written butterflies, 3, 5, 7, 11 and 13 the symmetric odd form, and any
// other radix (P = 0 here) a direct DFT with its inputs read from shared memory. Each radix is its own
// non-inlined function, so that the registers of one radix's butterfly do not add to another's.
template <int P, class C2>
__device__ __noinline__ void stage_loop(const C2* __restrict__ A, C2* __restrict__ B, int lc, int L, int Pr, int s,
                                        unsigned magic, const C2* __restrict__ tw, bool inv) {
  const int RP = P ? P : Pr;
  const int C = 1 << lc;
  const int m = L / (RP * s);
  const int nb = (L / RP) << lc;
  const int LP = L / RP;
  const size_t istep = (size_t)s * m * C, ostep = (size_t)s * C;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    const int l = b & (C - 1), bi = b >> lc;
    const int q = s == 1 ? bi : (int)__umulhi((unsigned)bi, magic), r = bi - q * s;
    const C2* in = A + (size_t)(r + s * q) * C + l;
    C2* out = B + (size_t)(r + s * RP * q) * C + l;
    auto emit = [&](int k, C2 val) {
      if (k > 0 && q > 0) {
        C2 w = __ldg(tw + (size_t)k * q * s);  // k q s < L
        val = cmul(val, inv ? conjf2(w) : w);
      }
      out[k * ostep] = val;
    };
    auto tw_m = [&](int mm) {  // w_P^mm
      C2 w = __ldg(tw + (size_t)mm * LP);
      return inv ? conjf2(w) : w;
    };
    if constexpr (P == 2) {
      C2 a0 = in[0], a1 = in[istep];
      emit(0, cadd(a0, a1));
      emit(1, csub(a0, a1));
    } else if constexpr (P == 4) {
      C2 a0 = in[0], a1 = in[istep], a2 = in[2 * istep], a3 = in[3 * istep];
      C2 t0 = cadd(a0, a2), t1 = csub(a0, a2);
      C2 t2 = cadd(a1, a3), t3 = rot(csub(a1, a3), inv);
      emit(0, cadd(t0, t2));
      emit(2, csub(t0, t2));
      emit(1, cadd(t1, t3));
      emit(3, csub(t1, t3));
    } else if constexpr (P == 8) {
      C2 v[8];
#pragma unroll
      for (int j = 0; j < 8; j++) v[j] = in[j * istep];
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
#pragma unroll
      for (int k = 0; k < 4; k++) {
        C2 t = k == 0 ? d[0] : cmul(d[k], tw_m(k));
        emit(k, cadd(e[k], t));
        emit(k + 4, csub(e[k], t));
      }
    } else if constexpr (P == 3 || P == 5 || P == 7 || P == 11 || P == 13) {
      odd_butterfly<P>(in, istep, tw, LP, inv, emit);
    } else {
      for (int k = 0; k < RP; k++) {
        C2 acc = in[0];
        int jk = 0;
        for (int j = 1; j < RP; j++) {
          jk += k;
          if (jk >= RP) jk -= RP;
          C2 av = in[j * istep];
          C2 w = tw_m(jk);
          acc.x = fma(av.x, w.x, fma(-av.y, w.y, acc.x));
          acc.y = fma(av.x, w.y, fma(av.y, w.x, acc.y));
        }
        emit(k, acc);
      }
    }
  }
}

template <class C2>
__device__ __forceinline__ void fft_stage(const C2* __restrict__ A, C2* __restrict__ B, int lc, int L, int P, int s,
                                          unsigned magic, const C2* __restrict__ tw, bool inv) {
  switch (P) {
    case 2: stage_loop<2, C2>(A, B, lc, L, P, s, magic, tw, inv); break;
    case 3: stage_loop<3, C2>(A, B, lc, L, P, s, magic, tw, inv); break;
    case 4: stage_loop<4, C2>(A, B, lc, L, P, s, magic, tw, inv); break;
    case 5: stage_loop<5, C2>(A, B, lc, L, P, s, magic, tw, inv); break;
    case 7: stage_loop<7, C2>(A, B, lc, L, P, s, magic, tw, inv); break;
    case 8: stage_loop<8, C2>(A, B, lc, L, P, s, magic, tw, inv); break;
    case 11: stage_loop<11, C2>(A, B, lc, L, P, s, magic, tw, inv); break;
    case 13: stage_loop<13, C2>(A, B, lc, L, P, s, magic, tw, inv); break;
    default: stage_loop<0, C2>(A, B, lc, L, P, s, magic, tw, inv); break;
  }
  __syncthreads();
}

// runs the plan on buf (tmp: scratch of the same size); returns the buffer that holds the result
template <class C2>
__device__ C2* fft_run(C2* buf, C2* tmp, int C, const FftPlan& pl, bool inv) {
  C2* a = buf;
  C2* b = tmp;
  const C2* tw;
  if constexpr (sizeof(C2) == sizeof(double2)) tw = (const C2*)pl.twd;
  else tw = (const C2*)pl.tw;
  const int lc = C == 4 ? 2 : (C == 2 ? 1 : 0);
  for (int st = 0; st < pl.nst; st++) {
    fft_stage<C2>(a, b, lc, pl.L, pl.p[st], pl.s[st], pl.magic[st], tw, inv);
    C2* t = a;
    a = b;
    b = t;
  }
  return a;
}

// Cubic B-spline prefilter (interp.py:13-27, without the factor 6, which the caller folds into its
// scale) of C interleaved complex lines of length n in buf, in float64 arithmetic. The line is cut into
// T / C segments; each recursive pass computes every segment's entry value from a warm-up of IIR_WARM
// samples (z^29 < 3e-17, below float64 rounding), then runs its segment. carry: 2 * T double2 of scratch.
__device__ void prefilter_smem(float2* buf, int C, int n, double2* carry, double2* edge) {
  if (n == 1) return;
  const double z = bspline_z();
  const int tid = threadIdx.x, T = blockDim.x;
  const int S = T / C;  // segments per line
  const int l = tid % C, sg = tid / C;
  const int len = (n + S - 1) / S;
  const int s0 = sg * len, e0 = min(n, s0 + len);
  const bool live = sg < S && s0 < e0;
  auto X = [&](int i) { float2 v = buf[(size_t)i * C + l]; return make_double2(v.x, v.y); };
  // ---- causal: y[0] = sum_{k < min(n, 21)} z^k x[k]; y[i] = x[i] + z y[i-1]
  if (live) {
    if (sg == 0) {
      int hz = min(n, HORIZON);
      double2 a = make_double2(0, 0);
      double zk = 1.0;
      for (int k = 0; k < hz; k++) {
        double2 v = X(k);
        a.x += zk * v.x;
        a.y += zk * v.y;
        zk *= z;
      }
      edge[l] = a;  // y[0]
    }
    // y[e0 - 1]
    int start = e0 - 1 - IIR_WARM_F32;
    double2 y;
    if (start <= 0) {
      int hz = min(n, HORIZON);
      y = make_double2(0, 0);
      double zk = 1.0;
      for (int k = 0; k < hz; k++) {
        double2 v = X(k);
        y.x += zk * v.x;
        y.y += zk * v.y;
        zk *= z;
      }
      for (int i = 1; i < e0; i++) {
        double2 v = X(i);
        y.x = v.x + z * y.x;
        y.y = v.y + z * y.y;
      }
    } else {
      y = make_double2(0, 0);
      for (int i = start; i < e0; i++) {
        double2 v = X(i);
        y.x = v.x + z * y.x;
        y.y = v.y + z * y.y;
      }
    }
    carry[tid] = y;
  }
  __syncthreads();
  if (live) {
    double2 y;
    int i0;
    if (sg == 0) {
      y = edge[l];
      buf[l] = make_float2((float)y.x, (float)y.y);
      i0 = 1;
    } else {
      y = carry[tid - C];
      i0 = s0;
    }
    for (int i = i0; i < e0; i++) {
      double2 v = X(i);
      y.x = v.x + z * y.x;
      y.y = v.y + z * y.y;
      buf[(size_t)i * C + l] = make_float2((float)y.x, (float)y.y);
    }
  }
  __syncthreads();
  // ---- anticausal: c[n-1] = z / (z^2 - 1) (y[n-1] + z y[n-2]); c[i] = z (c[i+1] - y[i])
  const double g = z / (z * z - 1.0);
  if (live) {
    double2 c;
    int stop = s0 + IIR_WARM_F32;
    if (e0 == n) {
      double2 a = X(n - 1), b = X(n - 2);
      edge[C + l] = make_double2(g * (a.x + z * b.x), g * (a.y + z * b.y));
    }
    if (stop >= n - 1) {
      double2 a = X(n - 1), b = X(n - 2);
      c = make_double2(g * (a.x + z * b.x), g * (a.y + z * b.y));
      for (int i = n - 2; i >= s0; i--) {
        double2 v = X(i);
        c.x = z * (c.x - v.x);
        c.y = z * (c.y - v.y);
      }
    } else {
      c = make_double2(0, 0);
      for (int i = stop; i >= s0; i--) {
        double2 v = X(i);
        c.x = z * (c.x - v.x);
        c.y = z * (c.y - v.y);
      }
    }
    carry[T + tid] = c;  // c[s0]
  }
  __syncthreads();
  if (live) {
    double2 c;
    int i0;
    if (e0 == n) {
      c = edge[C + l];
      buf[(size_t)(n - 1) * C + l] = make_float2((float)c.x, (float)c.y);
      i0 = n - 2;
    } else {
      c = carry[T + tid + C];  // c[e0] of the next segment
      i0 = e0 - 1;
    }
    for (int i = i0; i >= s0; i--) {
      double2 v = X(i);
      c.x = z * (c.x - v.x);
      c.y = z * (c.y - v.y);
      buf[(size_t)i * C + l] = make_float2((float)c.x, (float)c.y);
    }
  }
  __syncthreads();
}

// ---------------------------------------------------------------- kernels
template <class C2>
__global__ void __launch_bounds__(FFT_TMAX) k_fft_rows_fwd_real(const float* __restrict__ img, int W, int H, FftPlan plw,
                                                                int ph, C2* __restrict__ out) {
  extern __shared__ __align__(16) unsigned char smraw[];
  C2* sm = (C2*)smraw;
  const int pw = plw.L;
  C2* t = sm + pw;
  const int yp = blockIdx.x;
  const int ys = (int)mirror_idx(yp - PAD, H);
  const float* row = img + (size_t)ys * W;
  for (int x = threadIdx.x; x < pw; x += blockDim.x) sm[x] = mkc<C2>(__ldg(row + mirror_idx(x - PAD, W)), 0.0);
  __syncthreads();
  C2* r = fft_run(sm, t, 1, plw, false);
  C2* o = out + (size_t)yp * pw;
  for (int x = threadIdx.x; x < pw; x += blockDim.x) o[x] = r[x];
}

// Tin: ph x pw row-transformed; per block C adjacent columns. Shared memory: S (spectrum), W1, W2 (ping-pong),
// prefilter carries.
template <class C2>
__global__ void __launch_bounds__(FFT_TMAX) k_fft_cols_filters(const C2* __restrict__ Tin, FftPlan plh, int pw,
                                                               GaborTables g, int C, int refpack, int k0,
                                                               int k1, C2* __restrict__ U) {
  extern __shared__ __align__(16) unsigned char smraw[];
  C2* sm = (C2*)smraw;
  const int ph = plh.L;
  const size_t LC = (size_t)ph * C;
  C2* S = sm;
  C2* W1 = sm + LC;
  C2* W2 = sm + 2 * LC;
  double2* carry = (double2*)(((uintptr_t)(sm + 3 * LC) + 15) & ~(uintptr_t)15);  // 16-byte aligned
  double2* edge = carry + 2 * blockDim.x;
  const int x0 = blockIdx.x * C;
  for (int i = threadIdx.x; i < ph * C; i += blockDim.x) {
    int y = i / C, l = i - y * C, x = x0 + l;
    S[i] = x < pw ? Tin[(size_t)y * pw + x] : mkc<C2>(0.0, 0.0);
  }
  __syncthreads();
  C2* spec = fft_run(S, W1, C, plh, false);
  if (spec != S) {
    for (int i = threadIdx.x; i < ph * C; i += blockDim.x) S[i] = spec[i];
    __syncthreads();
  }
  const size_t plane = (size_t)ph * pw;
  const int nvar = refpack ? 3 : 1;
  for (int k = k0; k < k1; k++) {
    const double* exk = g.ex + (size_t)k * pw;
    const double* eyk = g.ey + (size_t)k * ph;
    const float* exkf = g.exf + (size_t)k * pw;
    const float* eykf = g.eyf + (size_t)k * ph;
    for (int v = 0; v < nvar; v++) {
      for (int i = threadIdx.x; i < ph * C; i += blockDim.x) {
        int y = i / C, l = i - y * C, x = min(x0 + l, pw - 1);
        C2 sv = S[i];
        if constexpr (sizeof(C2) == sizeof(float2)) {
          float G = fmaf(g.hxf[x], g.omyf[y], g.omxf[x]) * (exkf[x] * eykf[y]);
          W1[i] = mkc<C2>(sv.x * G, sv.y * G);
        } else {
          double G = fma(g.hx[x], g.omy[y], g.omx[x]) * exk[x] * eyk[y];
          double re = sv.x * G, im = sv.y * G;
          if (v == 1) { double f = g.fx[x]; double t = re; re = -im * f; im = t * f; }        // x i fx
          else if (v == 2) { double f = g.fy[y]; double t = re; re = -im * f; im = t * f; }   // x i fy
          W1[i] = mkc<C2>(re, im);
        }
      }
      __syncthreads();
      C2* res = fft_run(W1, W2, C, plh, true);
      if constexpr (sizeof(C2) == sizeof(float2)) {
        if (!refpack) prefilter_smem((float2*)res, C, ph, carry, edge);
      }
      C2* dst = U + (size_t)((k - k0) * nvar + v) * plane;
      for (int i = threadIdx.x; i < ph * C; i += blockDim.x) {
        int y = i / C, l = i - y * C, x = x0 + l;
        if (x < pw) dst[(size_t)y * pw + x] = res[i];
      }
      __syncthreads();
    }
  }
}

__global__ void __launch_bounds__(FFT_TMAX, 2) k_fft_rows_inv_resp(const float2* __restrict__ U, FftPlan plw, int ph,
                                                                float scale, float2* __restrict__ R) {
  extern __shared__ float2 sm[];
  const int pw = plw.L;
  float2* t = sm + pw;
  double2* carry = (double2*)(sm + 2 * pw);
  double2* edge = carry + 2 * blockDim.x;
  const int y = blockIdx.x, k = blockIdx.y;
  const size_t off = (size_t)k * ph * pw + (size_t)y * pw;
  for (int x = threadIdx.x; x < pw; x += blockDim.x) sm[x] = U[off + x];
  __syncthreads();
  float2* r = fft_run(sm, t, 1, plw, true);
  prefilter_smem(r, 1, pw, carry, edge);
  for (int x = threadIdx.x; x < pw; x += blockDim.x) {
    float2 v = r[x];
    R[off + x] = make_float2(v.x * scale, v.y * scale);
  }
}

template <class C2>
__global__ void __launch_bounds__(FFT_TMAX) k_fft_rows_inv_ref(const C2* __restrict__ U, FftPlan plw, int ph, int W,
                                                               int H, int k0, float4* __restrict__ ref4,
                                                               float* __restrict__ amp) {
  extern __shared__ __align__(16) unsigned char smraw[];
  C2* sm = (C2*)smraw;
  const int pw = plw.L;
  C2* t = sm + 3 * pw;
  const int y = blockIdx.x, kk = blockIdx.y, k = k0 + kk;  // y: row of the W x H crop
  const size_t plane = (size_t)ph * pw;
  for (int i = threadIdx.x; i < pw * 3; i += blockDim.x) {
    int v = i / pw, x = i - v * pw;
    sm[i] = U[(size_t)(3 * kk + v) * plane + (size_t)(y + PAD) * pw + x];
  }
  __syncthreads();
  C2* rr[3];
  for (int v = 0; v < 3; v++) {
    C2* res = fft_run(sm + v * pw, t, 1, plw, true);
    if (res != sm + v * pw) {
      for (int x = threadIdx.x; x < pw; x += blockDim.x) sm[v * pw + x] = res[x];
      __syncthreads();
    }
    rr[v] = sm + v * pw;
  }
  const double sc = 1.0 / ((double)ph * (double)pw);
  for (int x = threadIdx.x; x < W; x += blockDim.x) {
    int xp = x + PAD;
    C2 a = rr[0][xp], b = rr[1][xp], c = rr[2][xp];
    double rre = a.x * sc, rim = a.y * sc;
    double xre = b.x * sc, xim = b.y * sc, yre = c.x * sc, yim = c.y * sc;
    double a2 = rre * rre + rim * rim + 1e-12;
    // Im(conj(r) rx) / a2 (phaseflow.py:109-110)
    double gx = (rre * xim - rim * xre) / a2;
    double gy = (rre * yim - rim * yre) / a2;
    size_t o = (size_t)k * W * H + (size_t)y * W + x;
    ref4[o] = make_float4((float)rre, (float)rim, (float)gx, (float)gy);
    amp[o] = (float)sqrt(a2);
  }
}

__global__ void __launch_bounds__(FFT_TMAX, 2) k_fft_lines(float2* data, FftPlan pl, int inv) {
  extern __shared__ float2 sm[];
  float2* row = data + (size_t)blockIdx.x * pl.L;
  for (int x = threadIdx.x; x < pl.L; x += blockDim.x) sm[x] = row[x];
  __syncthreads();
  float2* r = fft_run(sm, sm + pl.L, 1, pl, inv != 0);
  for (int x = threadIdx.x; x < pl.L; x += blockDim.x) row[x] = r[x];
}

// ---------------------------------------------------------------- launchers
constexpr size_t SMEM_MAX = 227 * 1024;

static void set_smem(const void* fn, size_t bytes) {
  OFC_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}

// columns per block of the column pass: C adjacent columns make 32-byte row segments; elem: bytes per value
static int cols_C(int ph, size_t elem, bool carries, int& T, size_t& sm) {
  for (int C : {int(32 / elem), int(16 / elem), 1}) {
    if (C < 1) continue;
    T = fft_threads(ph, C);
    sm = (size_t)3 * ph * C * elem + 16 + (carries ? (size_t)(2 * T + 2 * C) * sizeof(double2) : 0);
    if (sm <= SMEM_MAX) return C;
  }
  throw Error(OFC_ERR_WINDOW, "padded height " + std::to_string(ph) + " too large for the column pass");
}

bool fft_fits(int ph, int pw) {
  try {
    int T;
    size_t sm;
    cols_C(ph, sizeof(float2), true, T, sm);
    cols_C(ph, sizeof(double2), false, T, sm);
    return 4 * (size_t)pw * sizeof(double2) <= SMEM_MAX;
  } catch (const Error&) {
    return false;
  }
}

void launch_fft_rows_fwd_real(const float* img, int W, int H, const FftPlan& plw, int ph, float2* out, cudaStream_t st) {
  int T = fft_threads(plw.L, 1);
  size_t sm = (size_t)2 * plw.L * sizeof(float2);
  set_smem((const void*)k_fft_rows_fwd_real<float2>, sm);
  OFC_LAUNCH(k_fft_rows_fwd_real<float2>, ph, T, sm, st, img, W, H, plw, ph, out);
}

void launch_fft_rows_fwd_real_f64(const float* img, int W, int H, const FftPlan& plw, int ph, double2* out,
                                  cudaStream_t st) {
  int T = fft_threads(plw.L, 1);
  size_t sm = (size_t)2 * plw.L * sizeof(double2);
  set_smem((const void*)k_fft_rows_fwd_real<double2>, sm);
  OFC_LAUNCH(k_fft_rows_fwd_real<double2>, ph, T, sm, st, img, W, H, plw, ph, out);
}

void launch_fft_cols_filters(const float2* Tin, const FftPlan& plh, int pw, const GaborTables& g, float2* U,
                             cudaStream_t st) {
  int T;
  size_t sm;
  int C = cols_C(plh.L, sizeof(float2), true, T, sm);
  set_smem((const void*)k_fft_cols_filters<float2>, sm);
  OFC_LAUNCH(k_fft_cols_filters<float2>, div_up(pw, C), T, sm, st, Tin, plh, pw, g, C, 0, 0, g.F, U);
}

void launch_fft_cols_ref_f64(const double2* Tin, const FftPlan& plh, int pw, const GaborTables& g, int k0, int k1,
                             double2* U, cudaStream_t st) {
  int T;
  size_t sm;
  int C = cols_C(plh.L, sizeof(double2), false, T, sm);
  set_smem((const void*)k_fft_cols_filters<double2>, sm);
  OFC_LAUNCH(k_fft_cols_filters<double2>, div_up(pw, C), T, sm, st, Tin, plh, pw, g, C, 1, k0, k1, U);
}

void launch_fft_rows_inv_resp(const float2* U, const FftPlan& plw, int ph, int F, float2* R, cudaStream_t st) {
  int T = fft_threads(plw.L, 1);
  size_t sm = (size_t)2 * plw.L * sizeof(float2) + (size_t)(2 * T + 2) * sizeof(double2);
  set_smem((const void*)k_fft_rows_inv_resp, sm);
  float scale = (float)(36.0 / ((double)ph * (double)plw.L));
  dim3 grid(ph, F);
  OFC_LAUNCH(k_fft_rows_inv_resp, grid, T, sm, st, U, plw, ph, scale, R);
}

void launch_fft_rows_inv_ref_f64(const double2* U, const FftPlan& plw, int ph, int k0, int k1, int W, int H,
                                 float4* ref4, float* amp, cudaStream_t st) {
  int T = fft_threads(plw.L, 1);
  size_t sm = (size_t)4 * plw.L * sizeof(double2);
  set_smem((const void*)k_fft_rows_inv_ref<double2>, sm);
  dim3 grid(H, k1 - k0);
  OFC_LAUNCH(k_fft_rows_inv_ref<double2>, grid, T, sm, st, U, plw, ph, W, H, k0, ref4, amp);
}

void launch_fft_lines(float2* data, int lines, const FftPlan& pl, bool inverse, cudaStream_t st) {
  int T = fft_threads(pl.L, 1);
  size_t sm = (size_t)2 * pl.L * sizeof(float2);
  set_smem((const void*)k_fft_lines, sm);
  OFC_LAUNCH(k_fft_lines, lines, T, sm, st, data, pl, inverse ? 1 : 0);
}

}  // namespace ofc
