// poc.cu -- the coarse stage in float64 (python/optflow_ref/poc.py; rust/crates/optflow-core/src/poc.rs:43-767):
// windowed band-limited phase-only correlation on a grid, one thread block per grid point, with the
// re-centring iterations, the outlier clean-up and the bilinear grid sampling.
#include <cfloat>
#include <climits>
#include <cstring>

#include "kernels.cuh"

namespace ofc {

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

// ---------------------------------------------------------------- float64 FFTs inside one warp
// A line of n = 16, 32 or 64 complex values lives in a warp: n = 64 as (v0, v1) = (x[l], x[l + 32]) in lane l;
// n = 32 as v0 = x[l]; n = 16 as v0 = x[l & 15] (lanes 16..31 hold a second line). Radix-2 butterflies
// across lanes use shuffles; twiddles W_64^t come from a shared table (W_{2h}^j = W_64^{j 32 / h}).
// dif: natural order in, bit-reversed out; dit: bit-reversed in, natural out.
__device__ __forceinline__ double2 dmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 shfl_xor_d2(double2 v, int m) {
  return make_double2(__shfl_xor_sync(0xffffffff, v.x, m), __shfl_xor_sync(0xffffffff, v.y, m));
}
__device__ __forceinline__ double2 twid(const double2* tw64, int t, bool inv) {
  double2 w = tw64[t];
  return inv ? make_double2(w.x, -w.y) : w;
}

__device__ __forceinline__ void warp_dif(double2& v0, double2& v1, int n, bool inv, const double2* tw64) {
  const int l = threadIdx.x & 31;
  int top = n / 2;
  if (n == 64) {
    double2 a = make_double2(v0.x + v1.x, v0.y + v1.y);
    double2 b = dmul(make_double2(v0.x - v1.x, v0.y - v1.y), twid(tw64, l, inv));
    v0 = a;
    v1 = b;
    top = 16;
  }
  for (int h = top; h >= 1; h >>= 1) {
    const bool up = (l & h) != 0;
    const double2 w = twid(tw64, (l & (h - 1)) * (32 / h), inv);
    double2 p0 = shfl_xor_d2(v0, h);
    v0 = up ? dmul(make_double2(p0.x - v0.x, p0.y - v0.y), w) : make_double2(v0.x + p0.x, v0.y + p0.y);
    if (n == 64) {
      double2 p1 = shfl_xor_d2(v1, h);
      v1 = up ? dmul(make_double2(p1.x - v1.x, p1.y - v1.y), w) : make_double2(v1.x + p1.x, v1.y + p1.y);
    }
  }
}

__device__ __forceinline__ void warp_dit(double2& v0, double2& v1, int n, bool inv, const double2* tw64) {
  const int l = threadIdx.x & 31;
  const int top = n == 64 ? 16 : n / 2;
  for (int h = 1; h <= top; h <<= 1) {
    const bool up = (l & h) != 0;
    const double2 w = twid(tw64, (l & (h - 1)) * (32 / h), inv);
    double2 t0 = up ? dmul(v0, w) : v0;
    double2 p0 = shfl_xor_d2(t0, h);
    v0 = up ? make_double2(p0.x - t0.x, p0.y - t0.y) : make_double2(t0.x + p0.x, t0.y + p0.y);
    if (n == 64) {
      double2 t1 = up ? dmul(v1, w) : v1;
      double2 p1 = shfl_xor_d2(t1, h);
      v1 = up ? make_double2(p1.x - t1.x, p1.y - t1.y) : make_double2(t1.x + p1.x, t1.y + p1.y);
    }
  }
  if (n == 64) {
    double2 t = dmul(v1, twid(tw64, l, inv));
    double2 a = make_double2(v0.x + t.x, v0.y + t.y), b = make_double2(v0.x - t.x, v0.y - t.y);
    v0 = a;
    v1 = b;
  }
}

// The twiddles a lane of the 64-point transforms uses, held in registers (a shared table read by the lanes of a
// warp at the strides (l & (h - 1)) 32 / h falls on few banks): w[0] = W_64^l for the outer radix-2 step, then
// w[s] = W_64^((l & (h - 1)) 32 / h) for the steps h = 16, 8, 4, 2, 1 (s = 1..5).
struct Tw64 {
  double2 w[6];
};
__device__ __forceinline__ Tw64 lane_tw64(const double2* tw64) {
  const int l = threadIdx.x & 31;
  Tw64 t;
  t.w[0] = tw64[l];
  int s = 1;
#pragma unroll
  for (int h = 16; h >= 1; h >>= 1, s++) t.w[s] = tw64[(l & (h - 1)) * (32 / h)];
  return t;
}
__device__ __forceinline__ double2 cjif(double2 w, bool inv) { return inv ? make_double2(w.x, -w.y) : w; }

// warp_dif / warp_dit for n = 64 with the lane's twiddles in registers (the same arithmetic)
__device__ __forceinline__ void warp_dif64(double2& v0, double2& v1, bool inv, const Tw64& T) {
  const int l = threadIdx.x & 31;
  {
    double2 a = make_double2(v0.x + v1.x, v0.y + v1.y);
    double2 b = dmul(make_double2(v0.x - v1.x, v0.y - v1.y), cjif(T.w[0], inv));
    v0 = a;
    v1 = b;
  }
  int s = 1;
#pragma unroll
  for (int h = 16; h >= 1; h >>= 1, s++) {
    const bool up = (l & h) != 0;
    const double2 w = cjif(T.w[s], inv);
    double2 p0 = shfl_xor_d2(v0, h);
    v0 = up ? dmul(make_double2(p0.x - v0.x, p0.y - v0.y), w) : make_double2(v0.x + p0.x, v0.y + p0.y);
    double2 p1 = shfl_xor_d2(v1, h);
    v1 = up ? dmul(make_double2(p1.x - v1.x, p1.y - v1.y), w) : make_double2(v1.x + p1.x, v1.y + p1.y);
  }
}
__device__ __forceinline__ void warp_dit64(double2& v0, double2& v1, bool inv, const Tw64& T) {
  const int l = threadIdx.x & 31;
  int s = 5;
#pragma unroll
  for (int h = 1; h <= 16; h <<= 1, s--) {
    const bool up = (l & h) != 0;
    const double2 w = cjif(T.w[s], inv);
    double2 t0 = up ? dmul(v0, w) : v0;
    double2 p0 = shfl_xor_d2(t0, h);
    v0 = up ? make_double2(p0.x - t0.x, p0.y - t0.y) : make_double2(t0.x + p0.x, t0.y + p0.y);
    double2 t1 = up ? dmul(v1, w) : v1;
    double2 p1 = shfl_xor_d2(t1, h);
    v1 = up ? make_double2(p1.x - t1.x, p1.y - t1.y) : make_double2(t1.x + p1.x, t1.y + p1.y);
  }
  double2 t = dmul(v1, cjif(T.w[0], inv));
  double2 a = make_double2(v0.x + t.x, v0.y + t.y), b = make_double2(v0.x - t.x, v0.y - t.y);
  v0 = a;
  v1 = b;
}

__device__ __forceinline__ int brev(int i, int bits) { return (int)(__brev((unsigned)i) >> (32 - bits)); }
__device__ __forceinline__ int ilog2(int n) { return 31 - __clz(n); }

// position -> natural index for the element held in register r of lane l of a length-n line
__device__ __forceinline__ int pos_of(int r, int n) {
  const int l = threadIdx.x & 31;
  return n == 64 ? r * 32 + l : (n == 32 ? l : (l & 15));
}

__device__ double block_sum_d(double v, double* red) {
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffff, v, o);
  int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double t = 0;
  for (int i = 0; i < POC_T / 32; i++) t += red[i];
  return t;
}

struct PocConst {
  double2 tw64[64];
  double hy[64], hx[64];
};

// lines of a window handled by warp `wid` in a pass over `nlines` lines of length n: n = 16 packs two lines
// per warp
__device__ __forceinline__ int lines_per_warp(int n) { return n == 16 ? 2 : 1; }

// Row transforms of a real window (values win(y, x), window mean removed, Hann weighted) into Z (natural
// order, Z[y * (wx + 1) + kx]: rows padded by one entry, so that a warp reading a column, one row per lane,
// spreads over the banks instead of hitting one).
template <class Get>
__device__ void rows_forward(Get get, double mean, int wy, int wx, const PocConst& pc, double2* Z) {
  const int wid = threadIdx.x >> 5, l = threadIdx.x & 31;
  const int lpw = lines_per_warp(wx), bits = ilog2(wx);
  for (int y0 = wid * lpw; y0 < wy; y0 += (POC_T / 32) * lpw) {
    int y = y0 + (lpw == 2 ? (l >> 4) : 0);
    double2 v0 = make_double2(0, 0), v1 = make_double2(0, 0);
    if (y < wy) {
      int x = pos_of(0, wx);
      v0 = make_double2((get(y, x) - mean) * (pc.hy[y * (64 / wy)] * pc.hx[x * (64 / wx)]), 0);
      if (wx == 64) v1 = make_double2((get(y, x + 32) - mean) * (pc.hy[y * (64 / wy)] * pc.hx[x + 32]), 0);
    }
    warp_dif(v0, v1, wx, false, pc.tw64);
    if (y < wy) {
      Z[y * (wx + 1) + brev(pos_of(0, wx), bits)] = v0;
      if (wx == 64) Z[y * (wx + 1) + brev(pos_of(1, wx), bits)] = v1;
    }
  }
}

// poc_shift (poc.py:39-54) of window B = b[y0 : y0 + wy, x0 : x0 + wx] against A's spectrum on the low-pass
// support (alp, natural order); res = (dx, dy, peak)
__device__ void poc_shift_dev(const double* __restrict__ b, int W, int x0, int y0, int wy, int wx, const PocConst& pc,
                              const double2* alp, int nlx, double lpm, double2* Z, double* red, double* res) {
  const int wid = threadIdx.x >> 5, l = threadIdx.x & 31;
  const int n = wy * wx;
  const int qy = wy / 4, qx = wx / 4;
  double s = 0;
  for (int i = threadIdx.x; i < n; i += POC_T) s += b[(size_t)(y0 + i / wx) * W + x0 + (i % wx)];
  const double mean = block_sum_d(s, red) / n;
  rows_forward([&](int y, int x) { return b[(size_t)(y0 + y) * W + x0 + x]; }, mean, wy, wx, pc, Z);
  __syncthreads();
  // columns on the low-pass support: forward (dif) -> C = B conj(A) / (|.| + 1e-12) on the support, 0 off it ->
  // inverse (dit); the result goes back to the column of Z in natural order
  {
    const int lpw = lines_per_warp(wy), bits = ilog2(wy);
    const int nlx2 = 2 * qx + 1;
    for (int c0 = wid * lpw; c0 < nlx2; c0 += (POC_T / 32) * lpw) {
      int ci = c0 + (lpw == 2 ? (l >> 4) : 0);
      bool live = ci < nlx2;
      int kx = ci <= qx ? ci : ci + (wx - 2 * qx - 1);
      double2 v0 = make_double2(0, 0), v1 = make_double2(0, 0);
      if (live) {
        v0 = Z[pos_of(0, wy) * (wx + 1) + kx];
        if (wy == 64) v1 = Z[pos_of(1, wy) * (wx + 1) + kx];
      }
      warp_dif(v0, v1, wy, false, pc.tw64);
      for (int r = 0; r < (wy == 64 ? 2 : 1); r++) {
        double2& v = r == 0 ? v0 : v1;
        int ky = brev(pos_of(r, wy), bits);
        int iy = ky <= qy ? ky : (ky >= wy - qy ? ky - (wy - 2 * qy - 1) : -1);
        double2 cc = make_double2(0, 0);
        if (live && iy >= 0) {
          double2 A = alp[iy * nlx + ci];
          cc = make_double2(v.x * A.x + v.y * A.y, v.y * A.x - v.x * A.y);
          double mag = hypot(cc.x, cc.y) + 1e-12;
          cc.x /= mag;
          cc.y /= mag;
        }
        v = cc;
      }
      warp_dit(v0, v1, wy, true, pc.tw64);
      if (live) {
        Z[pos_of(0, wy) * (wx + 1) + kx] = v0;
        if (wy == 64) Z[pos_of(1, wy) * (wx + 1) + kx] = v1;
      }
    }
  }
  __syncthreads();
  // inverse rows (only the low-pass columns are non-zero); r = fftshift(real) / lpm; the surface is kept in
  // natural order in the first half of each row of Z (each warp overwrites only rows it has read)
  const double sc = 1.0 / ((double)n) / lpm;
  double* surf = (double*)Z;
  double best = -DBL_MAX;
  int bi = 0x7fffffff;
  bool bnan = false;
  {
    const int lpw = lines_per_warp(wx), bits = ilog2(wx);
    for (int y0r = wid * lpw; y0r < wy; y0r += (POC_T / 32) * lpw) {
      int y = y0r + (lpw == 2 ? (l >> 4) : 0);
      bool live = y < wy;
      double2 v0 = make_double2(0, 0), v1 = make_double2(0, 0);
      int x0i = pos_of(0, wx), x1i = x0i + 32;
      auto lp = [&](int x) { return x <= qx || x >= wx - qx; };
      if (live && lp(x0i)) v0 = Z[y * (wx + 1) + x0i];
      if (live && wx == 64 && lp(x1i)) v1 = Z[y * (wx + 1) + x1i];
      __syncwarp();
      warp_dif(v0, v1, wx, true, pc.tw64);
      for (int r = 0; r < (wx == 64 ? 2 : 1); r++) {
        double v = (r == 0 ? v0.x : v1.x) * sc;
        int x = brev(pos_of(r, wx), bits);
        if (live) {
          surf[y * 2 * (wx + 1) + x] = v;
          int sy = (y + wy / 2) % wy, sxx = (x + wx / 2) % wx;
          int idx = sy * wx + sxx;
          bool vn = v != v;
          bool take = bnan ? (vn && idx < bi) : (vn || v > best || (v == best && idx < bi));
          if (take) { best = v; bi = idx; bnan = vn; }
        }
      }
    }
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
  if (l == 0) { sv[wid] = best; si[wid] = bi; sn[wid] = bnan; }
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
    auto R = [&](int ys, int xs) {  // the shifted surface at (ys, xs)
      int y = (ys - wy / 2 + wy) % wy, x = (xs - wx / 2 + wx) % wx;
      return surf[y * 2 * (wx + 1) + x];
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
    res[3] = (double)bi;  // the unclamped argmax of the shifted surface
  }
  __syncthreads();
}

// ipk (nullable): per grid point the integer peak of the last surface evaluated, round(d) + argmax - half window
// (x, y), INT_MIN where the first window already left the image
__global__ void __launch_bounds__(POC_T, 2) k_poc_grid(const double* __restrict__ a, const double* __restrict__ b,
                                                        int W, int H, int wy, int wx, const int* __restrict__ xs,
                                                        const int* __restrict__ ys, int nx, const double* iux,
                                                        const double* iuy, const PocConst* __restrict__ pcg,
                                                        double lpm, double* oux, double* ouy, double* opeak,
                                                        int* ipk) {
  extern __shared__ double2 dsm[];
  double2* Z = dsm;
  const int qy = wy / 4, qx = wx / 4;
  const int nlx = 2 * qx + 1;
  double2* alp = Z + wy * (wx + 1);
  __shared__ PocConst pc;
  __shared__ double red[POC_T / 32];
  __shared__ double res[4];
  for (int i = threadIdx.x; i < (int)(sizeof(PocConst) / sizeof(double)); i += POC_T)
    ((double*)&pc)[i] = ((const double*)pcg)[i];
  const int gi = blockIdx.x;
  const int j = gi % nx, i = gi / nx;
  const int x = xs[j], y = ys[i];
  const int hy = wy / 2, hx = wx / 2;
  const int n = wy * wx;
  const int wid = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  // spectrum of A (poc.py:44) on the low-pass support, natural order: alp[iy * nlx + ix]
  const double* aw = a + (size_t)(y - hy) * W + (x - hx);
  double s = 0;
  for (int t = threadIdx.x; t < n; t += POC_T) s += aw[(size_t)(t / wx) * W + (t % wx)];
  const double mean = block_sum_d(s, red) / n;
  rows_forward([&](int yy, int xx) { return aw[(size_t)yy * W + xx]; }, mean, wy, wx, pc, Z);
  __syncthreads();
  {
    const int lpw = lines_per_warp(wy), bits = ilog2(wy);
    for (int c0 = wid * lpw; c0 < nlx; c0 += (POC_T / 32) * lpw) {
      int ci = c0 + (lpw == 2 ? (l >> 4) : 0);
      bool live = ci < nlx;
      int kx = ci <= qx ? ci : ci + (wx - 2 * qx - 1);
      double2 v0 = make_double2(0, 0), v1 = make_double2(0, 0);
      if (live) {
        v0 = Z[pos_of(0, wy) * (wx + 1) + kx];
        if (wy == 64) v1 = Z[pos_of(1, wy) * (wx + 1) + kx];
      }
      warp_dif(v0, v1, wy, false, pc.tw64);
      for (int r = 0; r < (wy == 64 ? 2 : 1); r++) {
        int ky = brev(pos_of(r, wy), bits);
        int iy = ky <= qy ? ky : (ky >= wy - qy ? ky - (wy - 2 * qy - 1) : -1);
        if (live && iy >= 0) alp[iy * nlx + ci] = r == 0 ? v0 : v1;
      }
    }
  }
  __syncthreads();
  double dx = iux ? iux[gi] : 0.0, dy = iuy ? iuy[gi] : 0.0;
  double pk = 0.0;
  int px = INT_MIN, py = INT_MIN;
  for (int it = 0; it < 3; it++) {
    double ox = rint(dx), oy = rint(dy);  // Python round(): half to even
    long y0 = y - hy + (long)oy, x0 = x - hx + (long)ox;
    if (y0 < 0 || x0 < 0 || y0 + wy > H || x0 + wx > W) { pk = 0.0; break; }
    poc_shift_dev(b, W, (int)x0, (int)y0, wy, wx, pc, alp, nlx, lpm, Z, red, res);
    double sx = res[0], sy = res[1];
    pk = res[2];
    const int am = (int)res[3];
    px = (int)ox + am % wx - hx;
    py = (int)oy + am / wx - hy;
    dx = ox + sx;
    dy = oy + sy;
    if (fabs(sx) < 0.5 && fabs(sy) < 0.5) break;
  }
  if (threadIdx.x == 0) {
    oux[gi] = dx;
    ouy[gi] = dy;
    opeak[gi] = pk;
    if (ipk) {
      ipk[2 * gi] = px;
      ipk[2 * gi + 1] = py;
    }
  }
}

// ---------------------------------------------------------------- 64 x 64 windows: real transforms, half spectrum
// The windows are real, so (1) the forward row transforms run two rows per complex transform, z = a1 + i a2,
// unpacked as A1[k] = (Z[k] + conj Z[-k]) / 2, A2[k] = (Z[k] - conj Z[-k]) / (2 i); (2) only the columns
// kx = 0..16 of the low-pass support are transformed along y: the columns 48..63 are their conjugate mirror
// (the cross-power spectrum of real windows is Hermitian, C(-k) = conj C(k)); (3) after the inverse column
// transforms every row is Hermitian in kx, so its inverse is real and two rows share one complex inverse,
// r1 + i r2 = ifft(D1 + i D2). Per re-centring 98 line transforms instead of 194. Hz[y * ZS + kx]: the half
// spectrum (kx = 0..16; row stride 17 entries = 4 banks, so a warp reading a column spreads over the banks).
constexpr int ZS = 17;

__device__ __forceinline__ double2 shfl_d2(double2 v, int src) {
  return make_double2(__shfl_sync(0xffffffff, v.x, src), __shfl_sync(0xffffffff, v.y, src));
}
__device__ __forceinline__ int brev5(int i) { return (int)(__brev((unsigned)i) >> 27); }

// forward rows of a real 64 x 64 window (get(y, x) minus mean, Hann weighted) into the half spectrum Hz
template <class Get>
__device__ void rows_forward64(Get get, double mean, const PocConst& pc, const Tw64& tw, double2* Hz) {
  const int wid = threadIdx.x >> 5, l = threadIdx.x & 31;
  // lane l holds Z[k0] (register 0) and Z[k0 + 1] (register 1), k0 = 2 brev5(l) (the bit-reversed output);
  // Z[-k0] lies in register 0 of lane pl0, Z[-(k0 + 1)] in register 1 of lane 31 - l
  const int k0 = 2 * brev5(l), pl0 = brev5((32 - brev5(l)) & 31);
  for (int j = wid; j < 32; j += POC_T / 32) {
    const int y1 = 2 * j, y2 = 2 * j + 1;
    double2 v0 = make_double2((get(y1, l) - mean) * (pc.hy[y1] * pc.hx[l]), (get(y2, l) - mean) * (pc.hy[y2] * pc.hx[l]));
    double2 v1 = make_double2((get(y1, l + 32) - mean) * (pc.hy[y1] * pc.hx[l + 32]),
                              (get(y2, l + 32) - mean) * (pc.hy[y2] * pc.hx[l + 32]));
    warp_dif64(v0, v1, false, tw);
    const double2 p0 = shfl_d2(v0, pl0), p1 = shfl_d2(v1, 31 - l);
    auto unpack = [&](double2 z, double2 q, int k) {
      if (k <= 16) {
        Hz[y1 * ZS + k] = make_double2(0.5 * (z.x + q.x), 0.5 * (z.y - q.y));
        Hz[y2 * ZS + k] = make_double2(0.5 * (z.y + q.y), -0.5 * (z.x - q.x));
      }
    };
    unpack(v0, p0, k0);
    unpack(v1, p1, k0 + 1);
  }
}

// row index of the low-pass support for a transformed row ky (ky <= 16 or ky >= 48), or -1
__device__ __forceinline__ int lp_row64(int ky) { return ky <= 16 ? ky : (ky >= 48 ? ky - 31 : -1); }

// poc_shift (poc.py:39-54) of window B = b[y0 : y0 + 64, x0 : x0 + 64] against A's half spectrum on the low-pass
// support (alp[iy * 17 + kx], iy = 0..32); res = (dx, dy, peak)
__device__ void poc_shift64(const double* __restrict__ b, int W, int x0, int y0, const PocConst& pc, const Tw64& tw,
                            const double2* alp, double lpm, double2* Hz, double* surf, double* red, double* res) {
  const int wid = threadIdx.x >> 5, l = threadIdx.x & 31;
  double s = 0;
  for (int i = threadIdx.x; i < 4096; i += POC_T) s += b[(size_t)(y0 + (i >> 6)) * W + x0 + (i & 63)];
  const double mean = block_sum_d(s, red) / 4096.0;
  const double* bw = b + (size_t)y0 * W + x0;
  rows_forward64([&](int y, int x) { return bw[(size_t)y * W + x]; }, mean, pc, tw, Hz);
  __syncthreads();
  // columns kx = 0..16: forward (dif) -> C = B conj(A) / (|.| + 1e-12) on the low-pass rows, 0 elsewhere ->
  // inverse (dit) back to natural order
  for (int ci = wid; ci < ZS; ci += POC_T / 32) {
    double2 v0 = Hz[l * ZS + ci], v1 = Hz[(l + 32) * ZS + ci];
    warp_dif64(v0, v1, false, tw);
    for (int r = 0; r < 2; r++) {
      double2& v = r == 0 ? v0 : v1;
      const int iy = lp_row64(brev(32 * r + l, 6));
      double2 cc = make_double2(0, 0);
      if (iy >= 0) {
        const double2 A = alp[iy * ZS + ci];
        cc = make_double2(v.x * A.x + v.y * A.y, v.y * A.x - v.x * A.y);
        const double mag = hypot(cc.x, cc.y) + 1e-12;
        cc.x /= mag;
        cc.y /= mag;
      }
      v = cc;
    }
    warp_dit64(v0, v1, true, tw);
    Hz[l * ZS + ci] = v0;
    Hz[(l + 32) * ZS + ci] = v1;
  }
  __syncthreads();
  // inverse rows, two per transform: E = D1 + i D2 with D[kx] = Hz[kx] (kx <= 16), conj Hz[64 - kx] (kx >= 48);
  // the real surface r = fftshift(ifft2(C)) / lpm in natural order, and the first maximum (NaN wins)
  const double sc = 1.0 / 4096.0 / lpm;
  double best = -DBL_MAX;
  int bi = 0x7fffffff;
  bool bnan = false;
  for (int j = wid; j < 32; j += POC_T / 32) {
    const int y1 = 2 * j, y2 = 2 * j + 1;
    double2 v0 = make_double2(0, 0), v1 = make_double2(0, 0);
    if (l <= 16) {
      const double2 d1 = Hz[y1 * ZS + l], d2 = Hz[y2 * ZS + l];
      v0 = make_double2(d1.x - d2.y, d1.y + d2.x);
    }
    if (l >= 16) {
      const int m = 32 - l;  // kx = 32 + l, 64 - kx = 32 - l
      const double2 d1 = Hz[y1 * ZS + m], d2 = Hz[y2 * ZS + m];  // conj d1 + i conj d2
      v1 = make_double2(d1.x + d2.y, -d1.y + d2.x);
    }
    warp_dif64(v0, v1, true, tw);
    for (int r = 0; r < 2; r++) {
      const double2 v = r == 0 ? v0 : v1;
      const int x = brev(32 * r + l, 6);
      const int sxx = (x + 32) & 63;
      for (int h = 0; h < 2; h++) {
        const int y = h == 0 ? y1 : y2;
        const double val = (h == 0 ? v.x : v.y) * sc;
        surf[y * 64 + 32 * r + l] = val;  // stored in the transform's (bit-reversed) column order
        const int idx = ((y + 32) & 63) * 64 + sxx;
        const bool vn = val != val;
        const bool take = bnan ? (vn && idx < bi) : (vn || val > best || (val == best && idx < bi));
        if (take) { best = val; bi = idx; bnan = vn; }
      }
    }
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
  if (l == 0) { sv[wid] = best; si[wid] = bi; sn[wid] = bnan; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < POC_T / 32; k++) {
      bool on = sn[k] != 0;
      bool take = bnan ? (on && si[k] < bi) : (on || sv[k] > best || (sv[k] == best && si[k] < bi));
      if (take) { best = sv[k]; bi = si[k]; bnan = on; }
    }
    int iy = bi >> 6, ix = bi & 63;
    iy = min(max(iy, 1), 62);
    ix = min(max(ix, 1), 62);
    // the shifted surface; column x of the unshifted surface sits at position brev6(x) of its row
    auto R = [&](int ys, int xs) { return surf[((ys + 32) & 63) * 64 + brev((xs + 32) & 63, 6)]; };
    auto parabola = [](double m, double c, double p) {  // poc.py:34-36
      double den = m - 2.0 * c + p;
      return den == 0 ? 0.0 : 0.5 * (m - p) / den;
    };
    double c = R(iy, ix);
    double sxp = parabola(R(iy, ix - 1), c, R(iy, ix + 1));
    double syp = parabola(R(iy - 1, ix), c, R(iy + 1, ix));
    res[0] = ix - 32 + sxp;
    res[1] = iy - 32 + syp;
    res[2] = c;
    res[3] = (double)bi;  // the unclamped argmax of the shifted surface
  }
  __syncthreads();
}

__global__ void __launch_bounds__(POC_T, 3) k_poc_grid64(const double* __restrict__ a, const double* __restrict__ b,
                                                          int W, int H, const int* __restrict__ xs,
                                                          const int* __restrict__ ys, int nx, const double* iux,
                                                          const double* iuy, const PocConst* __restrict__ pcg,
                                                          double lpm, double* oux, double* ouy, double* opeak,
                                                          int* ipk) {
  extern __shared__ double2 dsm[];
  double2* Hz = dsm;                    // 64 x 17
  double2* alp = Hz + 64 * ZS;          // 33 x 17
  double* surf = (double*)(alp + 33 * ZS);  // 64 x 64
  __shared__ PocConst pc;
  __shared__ double red[POC_T / 32];
  __shared__ double res[4];
  for (int i = threadIdx.x; i < (int)(sizeof(PocConst) / sizeof(double)); i += POC_T)
    ((double*)&pc)[i] = ((const double*)pcg)[i];
  const int gi = blockIdx.x;
  const int j = gi % nx, i = gi / nx;
  const int x = xs[j], y = ys[i];
  const int wid = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  // half spectrum of A (poc.py:44) on the low-pass support: alp[iy * 17 + kx]
  const double* aw = a + (size_t)(y - 32) * W + (x - 32);
  const Tw64 tw = lane_tw64(pc.tw64);
  double s = 0;
  for (int t = threadIdx.x; t < 4096; t += POC_T) s += aw[(size_t)(t >> 6) * W + (t & 63)];
  const double mean = block_sum_d(s, red) / 4096.0;
  rows_forward64([&](int yy, int xx) { return aw[(size_t)yy * W + xx]; }, mean, pc, tw, Hz);
  __syncthreads();
  for (int ci = wid; ci < ZS; ci += POC_T / 32) {
    double2 v0 = Hz[l * ZS + ci], v1 = Hz[(l + 32) * ZS + ci];
    warp_dif64(v0, v1, false, tw);
    for (int r = 0; r < 2; r++) {
      const int iy = lp_row64(brev(32 * r + l, 6));
      if (iy >= 0) alp[iy * ZS + ci] = r == 0 ? v0 : v1;
    }
  }
  __syncthreads();
  double dx = iux ? iux[gi] : 0.0, dy = iuy ? iuy[gi] : 0.0;
  double pk = 0.0;
  int px = INT_MIN, py = INT_MIN;
  for (int it = 0; it < 3; it++) {
    double ox = rint(dx), oy = rint(dy);  // Python round(): half to even
    long y0 = y - 32 + (long)oy, x0 = x - 32 + (long)ox;
    if (y0 < 0 || x0 < 0 || y0 + 64 > H || x0 + 64 > W) { pk = 0.0; break; }
    poc_shift64(b, W, (int)x0, (int)y0, pc, tw, alp, lpm, Hz, surf, red, res);
    double sx = res[0], sy = res[1];
    pk = res[2];
    const int am = (int)res[3];
    px = (int)ox + (am & 63) - 32;
    py = (int)oy + (am >> 6) - 32;
    dx = ox + sx;
    dy = oy + sy;
    if (fabs(sx) < 0.5 && fabs(sy) < 0.5) break;
  }
  if (threadIdx.x == 0) {
    oux[gi] = dx;
    ouy[gi] = dy;
    opeak[gi] = pk;
    if (ipk) {
      ipk[2 * gi] = px;
      ipk[2 * gi + 1] = py;
    }
  }
}

size_t poc_const_bytes() { return sizeof(PocConst); }

// constants of a window: twiddles of length 64 and the Hann windows, rounded from float64 (poc.py:18-31)
void poc_const_host(int wy, int wx, void* out) {
  PocConst hc;
  for (int t = 0; t < 64; t++) {
    double ang = -2.0 * PI * t / 64.0;
    hc.tw64[t] = make_double2(std::cos(ang), std::sin(ang));
    hc.hy[t] = 0.0;
    hc.hx[t] = 0.0;
  }
  // hann(n)[k] = 0.5 - 0.5 cos(2 pi k / n), stored at k * (64 / n)
  for (int k = 0; k < wy; k++) hc.hy[k * (64 / wy)] = 0.5 - 0.5 * std::cos(2 * PI * k / wy);
  for (int k = 0; k < wx; k++) hc.hx[k * (64 / wx)] = 0.5 - 0.5 * std::cos(2 * PI * k / wx);
  std::memcpy(out, &hc, sizeof(hc));
}

void launch_poc_grid(const double* a, const double* b, const PocLevel& lv, const int* xs, const int* ys,
                     const double* iux, const double* iuy, const void* dconst, double* ux, double* uy, double* peak,
                     int* ipk, cudaStream_t st) {
  auto ok_len = [](int n) { return n == 16 || n == 32 || n == 64; };
  if (!ok_len(lv.wy) || !ok_len(lv.wx))
    throw Error(OFC_ERR_ARG, "the CUDA engine's POC windows are 16, 32 or 64 px a side (poc_win <= 64)");
  // lp.mean(): the share of frequencies with |f| <= 0.25 on both axes
  double lpm = (double)(2 * (lv.wy / 4) + 1) * (double)(2 * (lv.wx / 4) + 1) / ((double)lv.wy * lv.wx);
  if (lv.wy == 64 && lv.wx == 64) {
    const size_t sm64 = (size_t)(64 * ZS + 33 * ZS) * sizeof(double2) + 64 * 64 * sizeof(double);
    raise_smem_limit((const void*)k_poc_grid64, sm64);
    OFC_LAUNCH(k_poc_grid64, lv.nx * lv.ny, POC_T, sm64, st, a, b, lv.W, lv.H, xs, ys, lv.nx, iux, iuy,
               (const PocConst*)dconst, lpm, ux, uy, peak, ipk);
    return;
  }
  size_t smem = (size_t)(lv.wy * (lv.wx + 1) + (2 * (lv.wy / 4) + 1) * (2 * (lv.wx / 4) + 1)) * sizeof(double2);
  raise_smem_limit((const void*)k_poc_grid, smem);
  OFC_LAUNCH(k_poc_grid, lv.nx * lv.ny, POC_T, smem, st, a, b, lv.W, lv.H, lv.wy, lv.wx, xs, ys, lv.nx, iux, iuy,
             (const PocConst*)dconst, lpm, ux, uy, peak, ipk);
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

// valid = peak >= peak_min; out = valid and not a normalised-median outlier among its valid 8-neighbours
// (poc.py:101-121); one thread per grid point
__global__ void k_poc_outliers(const double* __restrict__ ux, const double* __restrict__ uy,
                               const double* __restrict__ peak, int nx, int ny, double peak_min, double thresh,
                               uint8_t* __restrict__ out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nx * ny) return;
  const int di[8] = {-1, -1, -1, 0, 0, 1, 1, 1}, dj[8] = {-1, 0, 1, -1, 1, -1, 0, 1};
  const int i = p / nx, j = p - i * nx;
  uint8_t o = peak[p] >= peak_min;
  if (o) {
    double vx[8], vy[8];
    int c = 0;
    for (int k = 0; k < 8; k++) {
      int a = i + di[k], b = j + dj[k];
      if (a >= 0 && a < ny && b >= 0 && b < nx && peak[a * nx + b] >= peak_min) {
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

// the rest of clean (poc.py:122-140) in one thread block: no point left -> the fallback; else fill passes from
// the 8-neighbour medians until every point is set; invalid peaks -> 0
__global__ void k_poc_fill(double* ux, double* uy, double* peak, int nx, int ny, double peak_min, const double* fbx,
                           const double* fby, uint8_t* flags) {
  const int n = nx * ny;
  uint8_t* out = flags + n;
  uint8_t* nw = flags + 2 * n;
  __shared__ int any, all;
  const int di[8] = {-1, -1, -1, 0, 0, 1, 1, 1}, dj[8] = {-1, 0, 1, -1, 1, -1, 0, 1};
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
    if (!(peak[p] >= peak_min)) peak[p] = 0.0;
}

void launch_poc_clean(double* ux, double* uy, double* peak, int nx, int ny, double peak_min, double thresh,
                      const double* fbx, const double* fby, uint8_t* scratch, cudaStream_t st) {
  const int n = nx * ny;
  OFC_LAUNCH(k_poc_outliers, div_up(n, 128), 128, 0, st, ux, uy, peak, nx, ny, peak_min, thresh, scratch + n);
  OFC_LAUNCH(k_poc_fill, 1, 1024, 0, st, ux, uy, peak, nx, ny, peak_min, fbx, fby, scratch);
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
