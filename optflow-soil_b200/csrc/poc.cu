// poc.cu -- the coarse stage in float64 (python/optflow_ref/poc.py; rust/crates/optflow-core/src/poc.rs:43-767):
// windowed band-limited phase-only correlation on a grid, one thread block per grid point, with the
// re-centring iterations, the outlier clean-up and the bilinear grid sampling.
#include <cfloat>

#include "kernels.cuh"

namespace ofc {

constexpr int POC_MAXN = 4096;  // window pixels held in shared memory (64 x 64)
constexpr int POC_T = 256;

// ---------------------------------------------------------------- downsample (poc.py:164-165)
__global__ void k_corr_x_decimate(const double* __restrict__ tmp, int W, int H, const double* __restrict__ taps, int r,
                                  double* __restrict__ out) {
  int Wo = (W + 1) / 2;
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  int y = blockIdx.y;
  if (x >= Wo) return;
  const double* row = tmp + (size_t)(2 * y) * W;
  double s = 0;
  for (int j = -r; j <= r; j++) s += taps[j + r] * row[min(max(2 * x + j, 0), W - 1)];
  out[(size_t)y * Wo + x] = s;
}

void launch_downsample(const double* in, int W, int H, double* out, double* tmp, const double* taps, int r,
                       cudaStream_t st) {
  launch_corr_y(in, tmp, 1, W, H, taps, r, st);
  dim3 g(div_up((W + 1) / 2, 128), (H + 1) / 2);
  OFC_LAUNCH(k_corr_x_decimate, g, 128, 0, st, tmp, W, H, taps, r, out);
}

// ---------------------------------------------------------------- float64 power-of-two FFT in smem
__device__ __forceinline__ double2 dmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// one radix-2 Stockham stage over `nlines` lines of length n (element i of line l at l * ls + i * es);
// tw64: W_64^t = exp(-2 pi i t / 64), t < 64 (n divides 64)
__device__ void fft2_stage_d(double2* Z, int n, int nlines, int es, int ls, int s, const double2* tw64, bool inv) {
  const int m = n / (2 * s);
  const int nb = (n / 2) * nlines;
  constexpr int MB = POC_MAXN / 2 / POC_T;  // 8 butterflies per thread at most
  double2 v0[MB], v1[MB];
#pragma unroll
  for (int i = 0; i < MB; i++) {
    int b = threadIdx.x + i * POC_T;
    if (b < nb) {
      int l = b % nlines, bi = b / nlines;
      int q = bi / s, r = bi - q * s;
      v0[i] = Z[l * ls + (r + s * q) * es];
      v1[i] = Z[l * ls + (r + s * (q + m)) * es];
    }
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < MB; i++) {
    int b = threadIdx.x + i * POC_T;
    if (b < nb) {
      int l = b % nlines, bi = b / nlines;
      int q = bi / s, r = bi - q * s;
      double2 o0 = make_double2(v0[i].x + v1[i].x, v0[i].y + v1[i].y);
      double2 o1 = make_double2(v0[i].x - v1[i].x, v0[i].y - v1[i].y);
      if (q > 0) {
        double2 w = tw64[(q * s) * (64 / n)];
        if (inv) w.y = -w.y;
        o1 = dmul(o1, w);
      }
      Z[l * ls + (r + s * 2 * q) * es] = o0;
      Z[l * ls + (r + s * (2 * q + 1)) * es] = o1;
    }
  }
  __syncthreads();
}

__device__ void fft2d_d(double2* Z, int h, int w, const double2* tw64, bool inv) {
  for (int s = 1; s < w; s *= 2) fft2_stage_d(Z, w, h, 1, w, s, tw64, inv);   // rows
  for (int s = 1; s < h; s *= 2) fft2_stage_d(Z, h, w, w, 1, s, tw64, inv);   // columns
}

__device__ double block_sum_d(double v, double* red) {
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffff, v, o);
  int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double t = 0;
  if (threadIdx.x == 0) {
    for (int i = 0; i < POC_T / 32; i++) t += red[i];
    red[POC_T / 32] = t;
  }
  __syncthreads();
  return red[POC_T / 32];
}

struct PocConst {
  double2 tw64[64];
  double hy[64], hx[64];
};

// poc_shift (poc.py:39-54) of the window B at (x0, y0) of image b against the stored spectrum of A
// (on the low-pass support only, alp); returns dx, dy, peak in res[0..2]
__device__ void poc_shift_dev(const double* __restrict__ b, int W, int x0, int y0, int wy, int wx, const PocConst& pc,
                              const double2* alp, int nly, int nlx, double lpm, double2* Z, double* red, double* res) {
  const int n = wy * wx;
  double s = 0;
  for (int i = threadIdx.x; i < n; i += POC_T) {
    int r = i / wx, q = i - r * wx;
    double v = b[(size_t)(y0 + r) * W + x0 + q];
    Z[i] = make_double2(v, 0);
    s += v;
  }
  double mean = block_sum_d(s, red) / n;
  for (int i = threadIdx.x; i < n; i += POC_T) {
    int r = i / wx, q = i - r * wx;
    Z[i] = make_double2((Z[i].x - mean) * (pc.hy[r * (64 / wy)] * pc.hx[q * (64 / wx)]), 0);
  }
  __syncthreads();
  fft2d_d(Z, wy, wx, pc.tw64, false);
  // C = B conj(A) / (|.| + 1e-12) on the low-pass support, zero elsewhere
  const int qy = wy / 4, qx = wx / 4;
  for (int i = threadIdx.x; i < n; i += POC_T) {
    int ky = i / wx, kx = i - ky * wx;
    int iy = ky <= qy ? ky : (ky >= wy - qy ? ky - (wy - 2 * qy - 1) : -1);
    int ix = kx <= qx ? kx : (kx >= wx - qx ? kx - (wx - 2 * qx - 1) : -1);
    double2 c = make_double2(0, 0);
    if (iy >= 0 && ix >= 0) {
      double2 B = Z[i], A = alp[iy * nlx + ix];
      c = make_double2(B.x * A.x + B.y * A.y, B.y * A.x - B.x * A.y);
      double mag = hypot(c.x, c.y) + 1e-12;
      c.x /= mag;
      c.y /= mag;
    }
    Z[i] = c;
  }
  __syncthreads();
  fft2d_d(Z, wy, wx, pc.tw64, true);
  // r = fftshift(real(ifft2)) / lpm; first maximum in row-major order, a NaN wins
  const double sc = 1.0 / ((double)n) / lpm;
  double best = -DBL_MAX;
  int bi = 0x7fffffff;
  bool bnan = false;
  for (int i = threadIdx.x; i < n; i += POC_T) {
    int y = i / wx, x = i - y * wx;
    int sy = (y - wy / 2 + wy) % wy, sx = (x - wx / 2 + wx) % wx;
    double v = Z[sy * wx + sx].x * sc;
    bool vn = v != v;
    bool take = bnan ? (vn && i < bi) : (vn || v > best || (v == best && i < bi));
    if (take) { best = v; bi = i; bnan = vn; }
  }
  for (int o = 16; o; o >>= 1) {
    double ov = __shfl_xor_sync(0xffffffff, best, o);
    int oi = __shfl_xor_sync(0xffffffff, bi, o);
    bool on = __shfl_xor_sync(0xffffffff, (int)bnan, o) != 0;
    bool take = bnan ? (on && oi < bi) : (on || ov > best || (ov == best && oi < bi));
    if (take) { best = ov; bi = oi; bnan = on; }
  }
  __shared__ double sv[POC_T / 32];
  __shared__ int si[POC_T / 32];
  __shared__ int sn[POC_T / 32];
  int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) { sv[wid] = best; si[wid] = bi; sn[wid] = bnan; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < POC_T / 32; k++) {
      bool on = sn[k] != 0;
      bool take = bnan ? (on && si[k] < bi) : (on || sv[k] > best || (sv[k] == best && si[k] < bi));
      if (take) { best = sv[k]; bi = si[k]; bnan = on; }
    }
    int iy = bi / wx, ix = bi - iy * wx;
    iy = min(max(iy, 1), wy - 2);
    ix = min(max(ix, 1), wx - 2);
    auto R = [&](int y, int x) {
      int sy = (y - wy / 2 + wy) % wy, sx = (x - wx / 2 + wx) % wx;
      return Z[sy * wx + sx].x * sc;
    };
    auto parabola = [](double m, double c, double p) {  // poc.py:34-36
      double den = m - 2.0 * c + p;
      return den == 0 ? 0.0 : 0.5 * (m - p) / den;
    };
    double c = R(iy, ix);
    double sxp = parabola(R(iy, ix - 1), c, R(iy, ix + 1));
    double syp = parabola(R(iy - 1, ix), c, R(iy + 1, ix));
    res[0] = ix - wx / 2 + sxp;
    res[1] = iy - wy / 2 + syp;
    res[2] = c;
  }
  __syncthreads();
}

__global__ void __launch_bounds__(POC_T) k_poc_grid(const double* __restrict__ a, const double* __restrict__ b, int W,
                                                     int H, int wy, int wx, const int* __restrict__ xs,
                                                     const int* __restrict__ ys, int nx, const double* iux,
                                                     const double* iuy, const PocConst* __restrict__ pcg, double lpm,
                                                     double* oux, double* ouy, double* opeak) {
  extern __shared__ double2 dsm[];
  double2* Z = dsm;
  const int nly = 2 * (wy / 4) + 1, nlx = 2 * (wx / 4) + 1;
  double2* alp = Z + wy * wx;
  __shared__ PocConst pc;
  __shared__ double red[POC_T / 32 + 1];
  __shared__ double res[3];
  for (int i = threadIdx.x; i < (int)(sizeof(PocConst) / sizeof(double)); i += POC_T)
    ((double*)&pc)[i] = ((const double*)pcg)[i];
  const int gi = blockIdx.x;
  const int j = gi % nx, i = gi / nx;
  const int x = xs[j], y = ys[i];
  const int hy = wy / 2, hx = wx / 2;
  const int n = wy * wx;
  __syncthreads();
  // spectrum of A (poc.py:44), kept on the low-pass support
  double s = 0;
  for (int t = threadIdx.x; t < n; t += POC_T) {
    int r = t / wx, q = t - r * wx;
    double v = a[(size_t)(y - hy + r) * W + (x - hx + q)];
    Z[t] = make_double2(v, 0);
    s += v;
  }
  double mean = block_sum_d(s, red) / n;
  for (int t = threadIdx.x; t < n; t += POC_T) {
    int r = t / wx, q = t - r * wx;
    Z[t] = make_double2((Z[t].x - mean) * (pc.hy[r * (64 / wy)] * pc.hx[q * (64 / wx)]), 0);
  }
  __syncthreads();
  fft2d_d(Z, wy, wx, pc.tw64, false);
  const int qy = wy / 4, qx = wx / 4;
  for (int t = threadIdx.x; t < nly * nlx; t += POC_T) {
    int iy = t / nlx, ix = t - iy * nlx;
    int ky = iy <= qy ? iy : iy + (wy - 2 * qy - 1);
    int kx = ix <= qx ? ix : ix + (wx - 2 * qx - 1);
    alp[t] = Z[ky * wx + kx];
  }
  __syncthreads();
  double dx = iux ? iux[gi] : 0.0, dy = iuy ? iuy[gi] : 0.0;
  double pk = 0.0;
  for (int it = 0; it < 3; it++) {
    double ox = rint(dx), oy = rint(dy);  // Python round(): half to even
    long y0 = y - hy + (long)oy, x0 = x - hx + (long)ox;
    if (y0 < 0 || x0 < 0 || y0 + wy > H || x0 + wx > W) { pk = 0.0; break; }
    poc_shift_dev(b, W, (int)x0, (int)y0, wy, wx, pc, alp, nly, nlx, lpm, Z, red, res);
    double sx = res[0], sy = res[1];
    pk = res[2];
    dx = ox + sx;
    dy = oy + sy;
    if (fabs(sx) < 0.5 && fabs(sy) < 0.5) break;
  }
  if (threadIdx.x == 0) {
    oux[gi] = dx;
    ouy[gi] = dy;
    opeak[gi] = pk;
  }
}

void launch_poc_grid(const double* a, const double* b, const PocLevel& lv, const int* xs, const int* ys,
                     const double* iux, const double* iuy, double* ux, double* uy, double* peak, cudaStream_t st) {
  if (lv.wy * lv.wx > POC_MAXN || lv.wy > 64 || lv.wx > 64)
    throw Error(OFC_ERR_ARG, "the CUDA engine's POC windows are at most 64 x 64 (poc_win <= 64)");
  // constants: twiddles of length 64, Hann windows of the level's window, rounded from float64
  PocConst hc;
  for (int t = 0; t < 64; t++) {
    double ang = -2.0 * PI * t / 64.0;
    hc.tw64[t] = make_double2(std::cos(ang), std::sin(ang));
  }
  for (int t = 0; t < 64; t++) {
    hc.hy[t] = 0.0;
    hc.hx[t] = 0.0;
  }
  // hann(n)[k] = 0.5 - 0.5 cos(2 pi k / n), stored at k * (64 / n)
  for (int k = 0; k < lv.wy; k++) hc.hy[k * (64 / lv.wy)] = 0.5 - 0.5 * std::cos(2 * PI * k / lv.wy);
  for (int k = 0; k < lv.wx; k++) hc.hx[k * (64 / lv.wx)] = 0.5 - 0.5 * std::cos(2 * PI * k / lv.wx);
  PocConst* dc = nullptr;
  OFC_CUDA(cudaMallocAsync((void**)&dc, sizeof(PocConst), st));
  OFC_CUDA(cudaMemcpyAsync(dc, &hc, sizeof(PocConst), cudaMemcpyHostToDevice, st));
  // lp.mean(): the share of frequencies with |f| <= 0.25 on both axes
  double lpm = (double)(2 * (lv.wy / 4) + 1) * (double)(2 * (lv.wx / 4) + 1) / ((double)lv.wy * lv.wx);
  size_t smem = (size_t)(lv.wy * lv.wx + (2 * (lv.wy / 4) + 1) * (2 * (lv.wx / 4) + 1)) * sizeof(double2);
  OFC_CUDA(cudaFuncSetAttribute((const void*)k_poc_grid, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  OFC_LAUNCH(k_poc_grid, lv.nx * lv.ny, POC_T, smem, st, a, b, lv.W, lv.H, lv.wy, lv.wx, xs, ys, lv.nx, iux, iuy, dc,
             lpm, ux, uy, peak);
  OFC_CUDA(cudaFreeAsync(dc, st));
}

// ---------------------------------------------------------------- clean (poc.py:95-140)
__device__ void sort_small(double* v, int n) {
  for (int i = 1; i < n; i++) {
    double t = v[i];
    int j = i - 1;
    while (j >= 0 && v[j] > t) { v[j + 1] = v[j]; j--; }
    v[j + 1] = t;
  }
}
__device__ double median_small(double* v, int n) {  // np.median of n <= 8 values (no NaN)
  sort_small(v, n);
  return n % 2 ? v[n / 2] : (v[n / 2 - 1] + v[n / 2]) / 2.0;
}

__global__ void k_poc_clean(double* ux, double* uy, double* peak, int nx, int ny, double peak_min, double thresh,
                            const double* fbx, const double* fby, uint8_t* flags) {
  const int n = nx * ny;
  uint8_t* valid = flags;
  uint8_t* out = flags + n;
  uint8_t* nw = flags + 2 * n;
  __shared__ int any, all;
  const int di[8] = {-1, -1, -1, 0, 0, 1, 1, 1}, dj[8] = {-1, 0, 1, -1, 1, -1, 0, 1};
  for (int p = threadIdx.x; p < n; p += blockDim.x) valid[p] = peak[p] >= peak_min;
  __syncthreads();
  for (int p = threadIdx.x; p < n; p += blockDim.x) {
    int i = p / nx, j = p - i * nx;
    uint8_t o = valid[p];
    if (o) {
      double vx[8], vy[8];
      int c = 0;
      for (int k = 0; k < 8; k++) {
        int a = i + di[k], b = j + dj[k];
        if (a >= 0 && a < ny && b >= 0 && b < nx && valid[a * nx + b]) {
          vx[c] = ux[a * nx + b];
          vy[c] = uy[a * nx + b];
          c++;
        }
      }
      if (c >= 3) {
        for (int comp = 0; comp < 2; comp++) {
          double* vals = comp == 0 ? vx : vy;
          double self = comp == 0 ? ux[p] : uy[p];
          double med = median_small(vals, c);
          double dev[8];
          for (int k = 0; k < c; k++) dev[k] = fabs(vals[k] - med);
          double res = median_small(dev, c);
          if (fabs(self - med) / (res + 0.1) > thresh) o = 0;
        }
      }
    }
    out[p] = o;
  }
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  for (int p = threadIdx.x; p < n; p += blockDim.x)
    if (out[p]) any = 1;
  __syncthreads();
  if (!any) {
    for (int p = threadIdx.x; p < n; p += blockDim.x) {
      ux[p] = fbx ? fbx[p] : 0.0;
      uy[p] = fby ? fby[p] : 0.0;
      peak[p] = peak[p] * 0;
    }
    return;
  }
  for (int pass = 0; pass < 100; pass++) {
    if (threadIdx.x == 0) all = 1;
    __syncthreads();
    for (int p = threadIdx.x; p < n; p += blockDim.x)
      if (!out[p]) all = 0;
    __syncthreads();
    if (all) break;
    for (int p = threadIdx.x; p < n; p += blockDim.x) {
      nw[p] = out[p];
      if (out[p]) continue;
      int i = p / nx, j = p - i * nx;
      double vx[8], vy[8];
      int c = 0;
      for (int k = 0; k < 8; k++) {
        int a = i + di[k], b = j + dj[k];
        if (a >= 0 && a < ny && b >= 0 && b < nx && out[a * nx + b]) {
          vx[c] = ux[a * nx + b];
          vy[c] = uy[a * nx + b];
          c++;
        }
      }
      if (c) {
        ux[p] = median_small(vx, c);
        uy[p] = median_small(vy, c);
        nw[p] = 1;
      }
    }
    __syncthreads();
    for (int p = threadIdx.x; p < n; p += blockDim.x) out[p] = nw[p];
    __syncthreads();
  }
  for (int p = threadIdx.x; p < n; p += blockDim.x)
    if (!valid[p]) peak[p] = 0.0;
}

void launch_poc_clean(double* ux, double* uy, double* peak, int nx, int ny, double peak_min, double thresh,
                      const double* fbx, const double* fby, uint8_t* scratch, cudaStream_t st) {
  OFC_LAUNCH(k_poc_clean, 1, 1024, 0, st, ux, uy, peak, nx, ny, peak_min, thresh, fbx, fby, scratch);
}

// ---------------------------------------------------------------- grid sampling (poc.py:143-161)
__device__ __forceinline__ void grid_frac(double q, const int* nodes, int n, double& t, int& i0) {
  if (n == 1) { t = 0; i0 = 0; return; }
  double f = (q - nodes[0]) / (double)(nodes[1] - nodes[0]);
  f = fmin(fmax(f, 0.0), (double)(n - 1));
  i0 = min((int)floor(f), n - 2);
  t = f - i0;
}

__global__ void k_grid_sample(const double* __restrict__ gux, const double* __restrict__ guy, const int* gxs,
                              const int* gys, int gnx, int gny, const int* txs, const int* tys, int tnx, int tny,
                              double scale, double mult, double* oux, double* ouy) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  int i = blockIdx.y;
  if (j >= tnx) return;
  double X = txs ? (double)txs[j] : (double)j;
  double Y = tys ? (double)tys[i] : (double)i;
  double tx, ty;
  int x0, y0;
  grid_frac(X * scale, gxs, gnx, tx, x0);
  grid_frac(Y * scale, gys, gny, ty, y0);
  int x1 = min(x0 + 1, gnx - 1), y1 = min(y0 + 1, gny - 1);
  auto bil = [&](const double* a) {
    return (1 - ty) * ((1 - tx) * a[y0 * gnx + x0] + tx * a[y0 * gnx + x1]) +
           ty * ((1 - tx) * a[y1 * gnx + x0] + tx * a[y1 * gnx + x1]);
  };
  size_t o = (size_t)i * tnx + j;
  oux[o] = mult * bil(gux);
  ouy[o] = mult * bil(guy);
}

void launch_grid_sample(const double* gux, const double* guy, const int* gxs, const int* gys, int gnx, int gny,
                        const int* txs, const int* tys, int tnx, int tny, double scale, double mult, double* oux,
                        double* ouy, cudaStream_t st) {
  dim3 g(div_up(tnx, 128), tny);
  OFC_LAUNCH(k_grid_sample, g, 128, 0, st, gux, guy, gxs, gys, gnx, gny, txs, tys, tnx, tny, scale, mult, oux, ouy);
}

__global__ void k_init_from_dense(const double* dux, const double* duy, int W, const int* xs, const int* ys, int nx,
                                  int ny, int sc, double* iux, double* iuy) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  int i = blockIdx.y;
  if (j >= nx) return;
  size_t q = (size_t)ys[i] * sc * W + (size_t)xs[j] * sc;
  iux[i * nx + j] = dux[q] / sc;
  iuy[i * nx + j] = duy[q] / sc;
}

void launch_init_from_dense(const double* dux, const double* duy, int W, const int* xs, const int* ys, int nx, int ny,
                            int sc, double* iux, double* iuy, cudaStream_t st) {
  dim3 g(div_up(nx, 128), ny);
  OFC_LAUNCH(k_init_from_dense, g, 128, 0, st, dux, duy, W, xs, ys, nx, ny, sc, iux, iuy);
}

__global__ void k_grid_minus_dense(const double* gux, const double* guy, const double* dux, const double* duy, int W,
                                   const int* xs, const int* ys, int nx, int ny, double* cux, double* cuy) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  int i = blockIdx.y;
  if (j >= nx) return;
  size_t q = (size_t)ys[i] * W + xs[j];
  cux[i * nx + j] = gux[i * nx + j] - dux[q];
  cuy[i * nx + j] = guy[i * nx + j] - duy[q];
}

void launch_grid_minus_dense(const double* gux, const double* guy, const double* dux, const double* duy, int W,
                             const int* xs, const int* ys, int nx, int ny, double* cux, double* cuy, cudaStream_t st) {
  dim3 g(div_up(nx, 128), ny);
  OFC_LAUNCH(k_grid_minus_dense, g, 128, 0, st, gux, guy, dux, duy, W, xs, ys, nx, ny, cux, cuy);
}

__global__ void k_add(double* a, const double* b, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) a[i] += b[i];
}
void launch_add(double* a, const double* b, size_t n, cudaStream_t st) {
  OFC_LAUNCH(k_add, std::min<size_t>(div_up(n, 256), 4096), 256, 0, st, a, b, n);
}

}  // namespace ofc
