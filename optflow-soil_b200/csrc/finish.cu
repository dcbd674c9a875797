// finish.cu -- validity guard and strain of one tracked pair (python/optflow_ref/track.py:56-108,
// strain.py:61-112; rust/crates/optflow-core/src/track.rs:224-274,330-420, strain.rs:64-287).
#include <cfloat>

#include "kernels.cuh"

namespace ofc {

// ---------------------------------------------------------------- 4-connected components (union-find)
// find with path splitting: parent pointers only ever move to ancestors (smaller indices), so the plain stores
// of the splitting keep every pointer an ancestor while other threads link roots by atomicCAS. Every access is
// volatile: the compiler must neither keep a pointer in a register across another thread's update nor forward
// this thread's own store to a later load.
__device__ __forceinline__ int uf_find(int* parent, int x) {
  volatile int* vp = parent;
  int p = vp[x];
  while (p != x) {
    int gp = vp[p];
    if (gp != p) vp[x] = gp;
    x = p;
    p = gp;
  }
  return x;
}

__device__ void uf_union(int* parent, int a, int b) {
  // roots link to the smaller index, so a parent is never larger than its child and find terminates
  while (true) {
    a = uf_find(parent, a);
    b = uf_find(parent, b);
    if (a == b) return;
    if (a < b) { int t = a; a = b; b = t; }
    int old = atomicCAS(parent + a, a, b);
    if (old == a) return;
  }
}

__global__ void k_ccl_init(const uint8_t* __restrict__ b, int n, int* parent, int* size) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    parent[p] = b[p] ? p : -1;
    size[p] = 0;
  }
}

// rows strided by gridDim.y: a grid's y extent stops at 65,535, below the height of a tall image
__global__ void k_ccl_merge(const uint8_t* __restrict__ b, int W, int H, int* parent) {
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= W) return;
  for (int y = blockIdx.y; y < H; y += gridDim.y) {
    int p = y * W + x;
    if (!b[p]) continue;
    if (x + 1 < W && b[p + 1]) uf_union(parent, p, p + 1);
    if (y + 1 < H && b[p + W]) uf_union(parent, p, p + W);
  }
}

// after the merge: every pixel points to its root. The walk only reads (a splitting write could put an
// intermediate ancestor over another thread's root store), and every store is a root.
__global__ void k_ccl_flatten(const uint8_t* __restrict__ b, int n, int* parent) {
  volatile int* vp = parent;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    if (!b[p]) continue;
    int x = p, q = vp[x];
    while (q != x) {
      x = q;
      q = vp[x];
    }
    vp[p] = x;
  }
}

__global__ void k_ccl_count(const uint8_t* __restrict__ b, int n, const int* __restrict__ parent, int* size) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    if (!b[p]) continue;
    atomicAdd(size + parent[p], 1);
  }
}

__global__ void k_ccl_mark(const uint8_t* __restrict__ b, int n, const int* __restrict__ parent,
                           const int* __restrict__ size, double min_area, uint8_t* out) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    uint8_t v = 0;
    if (b[p]) v = (double)size[parent[p]] >= min_area;
    out[p] = v;
  }
}

void launch_large_components(const uint8_t* b, int W, int H, double min_area, int* parent, int* size, uint8_t* out,
                             cudaStream_t st) {
  int n = W * H;
  unsigned g = std::min(div_up(n, 256), 8192u);
  OFC_LAUNCH(k_ccl_init, g, 256, 0, st, b, n, parent, size);
  OFC_LAUNCH(k_ccl_merge, dim3(div_up(W, 128), std::min(H, 65535)), 128, 0, st, b, W, H, parent);
  OFC_LAUNCH(k_ccl_flatten, g, 256, 0, st, b, n, parent);
  OFC_LAUNCH(k_ccl_count, g, 256, 0, st, b, n, parent, size);
  OFC_LAUNCH(k_ccl_mark, g, 256, 0, st, b, n, parent, size, min_area, out);
}

// ---------------------------------------------------------------- finish mask
__global__ void k_finish_src(const uint8_t* __restrict__ low, const uint8_t* __restrict__ roi,
                             const uint8_t* __restrict__ big, int n, uint8_t* src, uint8_t* bad) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    bool out = roi && !roi[p];
    src[p] = (big && big[p]) || out;
    bad[p] = low[p] || out;
  }
}

__global__ void k_finish_apply(const uint8_t* __restrict__ bad, int W, int H, double guard,
                               const double* __restrict__ ux, const double* __restrict__ uy, double* mx, double* my) {
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  int y = blockIdx.y;
  if (x >= W) return;
  size_t p = (size_t)y * W + x;
  bool b = bad[p];
  if (guard > 0) {
    int bd = min(min(x, y), min(W - 1 - x, H - 1 - y));
    if ((double)bd < guard) b = true;
  }
  mx[p] = b ? nan("") : ux[p];
  my[p] = b ? nan("") : uy[p];
}

void launch_finish_mask(const uint8_t* low, const uint8_t* roi, const uint8_t* big, int W, int H, double guard,
                        const double* ux, const double* uy, uint8_t* src, uint8_t* bad, int* vdist, double* mx,
                        double* my, cudaStream_t st) {
  int n = W * H;
  unsigned g = std::min(div_up(n, 256), 8192u);
  OFC_LAUNCH(k_finish_src, g, 256, 0, st, low, roi, guard > 0 ? big : nullptr, n, src, bad);
  if (guard > 0) launch_within(src, W, H, guard, 0, bad, vdist, st);
  OFC_LAUNCH(k_finish_apply, dim3(div_up(W, 128), H), 128, 0, st, bad, W, H, guard, ux, uy, mx, my);
}

// ---------------------------------------------------------------- strain
// y pass: planes 0..4 = sum_t t^py m(y+t) (py = 0..4), 5..7 = u0 (py 0..2), 8..10 = v0 (py 0..2); zero outside
__global__ void k_strain_y(const double* __restrict__ mx, const double* __restrict__ my, int W, int H, int h,
                           double* __restrict__ yp) {
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  int y = blockIdx.y;
  if (x >= W) return;
  const size_t N = (size_t)W * H;
  double a[11];
#pragma unroll
  for (int i = 0; i < 11; i++) a[i] = 0;
  for (int t = -h; t <= h; t++) {
    int yy = y + t;
    if (yy < 0 || yy >= H) continue;
    size_t q = (size_t)yy * W + x;
    double u = mx[q], v = my[q];
    bool ok = isfinite(u) && isfinite(v);
    double m = ok ? 1.0 : 0.0, u0 = ok ? u : 0.0, v0 = ok ? v : 0.0;
    double tp = 1;
#pragma unroll
    for (int p = 0; p < 5; p++) {
      a[p] += tp * m;
      if (p < 3) {
        a[5 + p] += tp * u0;
        a[8 + p] += tp * v0;
      }
      tp *= t;
    }
  }
  size_t o = (size_t)y * W + x;
#pragma unroll
  for (int i = 0; i < 11; i++) yp[i * N + o] = a[i];
}

__global__ void k_strain_x(const double* __restrict__ yp, int W, int H, int h, int win, float* dudx, float* dudy,
                           float* dvdx, float* dvdy, float* exx_o, float* eyy_o, float* exy_o, float* gmax_o,
                           float* vol_o) {
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  int y = blockIdx.y;
  if (x >= W) return;
  const size_t N = (size_t)W * H;
  // Mm[px][py] for px + py <= 4 (15 values), ru[i], rv[i] over the basis
  double mm[5][5];
  double ru[3][3], rv[3][3];  // [px][py], px + py <= 2
#pragma unroll
  for (int i = 0; i < 5; i++)
#pragma unroll
    for (int j = 0; j < 5; j++) mm[i][j] = 0;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) ru[i][j] = rv[i][j] = 0;
  const double* row = yp + (size_t)y * W;
  for (int t = -h; t <= h; t++) {
    int xx = x + t;
    if (xx < 0 || xx >= W) continue;
    double m[5], u[3], v[3];
#pragma unroll
    for (int p = 0; p < 5; p++) m[p] = row[p * N + xx];
#pragma unroll
    for (int p = 0; p < 3; p++) { u[p] = row[(5 + p) * N + xx]; v[p] = row[(8 + p) * N + xx]; }
    double tp[5];
    tp[0] = 1;
#pragma unroll
    for (int p = 1; p < 5; p++) tp[p] = tp[p - 1] * t;
#pragma unroll
    for (int px = 0; px < 5; px++)
#pragma unroll
      for (int py = 0; py + px < 5; py++) mm[px][py] += tp[px] * m[py];
#pragma unroll
    for (int px = 0; px < 3; px++)
#pragma unroll
      for (int py = 0; py + px < 3; py++) {
        ru[px][py] += tp[px] * u[py];
        rv[px][py] += tp[px] * v[py];
      }
  }
  const int B[6][2] = {{0, 0}, {1, 0}, {0, 1}, {2, 0}, {1, 1}, {0, 2}};  // strain.py:7
  double r[4];
  const double nanv = nan("");
  r[0] = r[1] = r[2] = r[3] = nanv;
  if (mm[0][0] >= 0.5 * win * win) {
    double L[36], bu[6], bv[6], il[6];
    bool ok = true;
#pragma unroll
    for (int i = 0; i < 6; i++) {
#pragma unroll
      for (int j = 0; j < 6; j++) L[i * 6 + j] = mm[B[i][0] + B[j][0]][B[i][1] + B[j][1]];
      bu[i] = ru[B[i][0]][B[i][1]];
      bv[i] = rv[B[i][0]][B[i][1]];
    }
    // Cholesky with two right-hand sides (the same arithmetic as the fine stage's solve)
#pragma unroll
    for (int j = 0; j < 6; j++) {
      double d = L[j * 6 + j];
#pragma unroll
      for (int k = 0; k < 6; k++)  // constant trip counts with guards keep L in registers
        if (k < j) d -= L[j * 6 + k] * L[j * 6 + k];
      if (!(d > 0.0 && d <= DBL_MAX)) ok = false;
      double l = sqrt(d);
      il[j] = 1.0 / l;  // one division per pivot; the rest multiply by it
      L[j * 6 + j] = l;
#pragma unroll
      for (int i = 0; i < 6; i++) {
        if (i <= j) continue;
        double s = L[i * 6 + j];
#pragma unroll
        for (int k = 0; k < 6; k++)
          if (k < j) s -= L[i * 6 + k] * L[j * 6 + k];
        L[i * 6 + j] = s * il[j];
      }
    }
    if (ok) {
#pragma unroll
      for (int i = 0; i < 6; i++) {
        double su = bu[i], sv = bv[i];
#pragma unroll
        for (int k = 0; k < 6; k++)
          if (k < i) { su -= L[i * 6 + k] * bu[k]; sv -= L[i * 6 + k] * bv[k]; }
        bu[i] = su * il[i];
        bv[i] = sv * il[i];
      }
#pragma unroll
      for (int i = 5; i >= 0; i--) {
        double su = bu[i], sv = bv[i];
#pragma unroll
        for (int k = 0; k < 6; k++)
          if (k > i) { su -= L[k * 6 + i] * bu[k]; sv -= L[k * 6 + i] * bv[k]; }
        bu[i] = su * il[i];
        bv[i] = sv * il[i];
      }
      bool fin = true;
#pragma unroll
      for (int i = 0; i < 6; i++) fin &= isfinite(bu[i]) && isfinite(bv[i]);
      if (fin) { r[0] = bu[1]; r[1] = bu[2]; r[2] = bv[1]; r[3] = bv[2]; }
    }
  }
  size_t o = (size_t)y * W + x;
  if (dudx) dudx[o] = (float)r[0];
  if (dudy) dudy[o] = (float)r[1];
  if (dvdx) dvdx[o] = (float)r[2];
  if (dvdy) dvdy[o] = (float)r[3];
  // strain_fields (strain.py:100-112)
  double ux_x = r[0], ux_y = r[1], uy_x = r[2], uy_y = r[3];
  double exx = ux_x + 0.5 * (ux_x * ux_x + uy_x * uy_x);
  double eyy = uy_y + 0.5 * (ux_y * ux_y + uy_y * uy_y);
  double exy = 0.5 * (ux_y + uy_x) + 0.5 * (ux_x * ux_y + uy_x * uy_y);
  double q = (exx - eyy) / 2;
  if (exx_o) exx_o[o] = (float)exx;
  if (eyy_o) eyy_o[o] = (float)eyy;
  if (exy_o) exy_o[o] = (float)exy;
  if (gmax_o) gmax_o[o] = (float)(2.0 * sqrt(q * q + exy * exy));
  if (vol_o) vol_o[o] = (float)((1 + ux_x) * (1 + uy_y) - ux_y * uy_x - 1.0);
}

void launch_strain(const double* mx, const double* my, int W, int H, int win, double* yplanes, float* dudx, float* dudy,
                   float* dvdx, float* dvdy, float* exx, float* eyy, float* exy, float* gmax, float* vol,
                   cudaStream_t st) {
  int h = win / 2;
  dim3 g(div_up(W, 128), H);
  OFC_LAUNCH(k_strain_y, g, 128, 0, st, mx, my, W, H, h, yplanes);
  OFC_LAUNCH(k_strain_x, g, 128, 0, st, yplanes, W, H, h, win, dudx, dudy, dvdx, dvdy, exx, eyy, exy, gmax, vol);
}

__global__ void k_pair_outputs(const double* __restrict__ mx, const double* __restrict__ my,
                               const double* __restrict__ rux, const double* __restrict__ ruy,
                               const double* __restrict__ conf64, int n, float* ux, float* uy, float* conf,
                               uint8_t* valid, float* raw_ux, float* raw_uy) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    double a = mx[p];
    if (ux) ux[p] = (float)a;
    if (uy) uy[p] = (float)my[p];
    if (conf) conf[p] = (float)conf64[p];
    if (valid) valid[p] = isfinite(a) ? 1 : 0;
    if (raw_ux) raw_ux[p] = (float)rux[p];
    if (raw_uy) raw_uy[p] = (float)ruy[p];
  }
}

void launch_pair_outputs(const double* mx, const double* my, const double* rux, const double* ruy, const double* conf64,
                         int n, float* ux, float* uy, float* conf, uint8_t* valid, float* raw_ux, float* raw_uy,
                         cudaStream_t st) {
  OFC_LAUNCH(k_pair_outputs, std::min(div_up(n, 256), 8192u), 256, 0, st, mx, my, rux, ruy, conf64, n, ux, uy, conf,
             valid, raw_ux, raw_uy);
}

}  // namespace ofc
