// synth.cu -- speckle rendering on the GPU (python/optflow_ref/synth.py:20-190 restated): Gaussian blobs
// evaluated at the inverse-mapped coordinates of ss x ss subsamples per pixel, 0.5 + 0.25 tanh(mean).
#include "common.cuh"
#include "../../include/optflow_cuda_synth.h"

namespace ofc {

// x = c + A (X - c) + t + amp sin(k X_x) (sx, sy): X from x by Newton iterations from the affine inverse
__device__ void field_inverse(const ofc_field& f, double x, double y, double& X, double& Y) {
  double det = f.a00 * f.a11 - f.a01 * f.a10;
  double dx = x - f.cx - f.tx, dy = y - f.cy - f.ty;
  X = f.cx + (f.a11 * dx - f.a01 * dy) / det;
  Y = f.cy + (-f.a10 * dx + f.a00 * dy) / det;
  if (f.amp == 0.0) return;
  const double k = 2 * PI / f.wavelength;
  for (int it = 0; it < 30; it++) {
    double s = f.amp * sin(k * X), ds = f.amp * k * cos(k * X);
    double fx = f.cx + f.a00 * (X - f.cx) + f.a01 * (Y - f.cy) + f.tx + s * f.sx - x;
    double fy = f.cy + f.a10 * (X - f.cx) + f.a11 * (Y - f.cy) + f.ty + s * f.sy - y;
    double j00 = f.a00 + ds * f.sx, j01 = f.a01, j10 = f.a10 + ds * f.sy, j11 = f.a11;
    double d = j00 * j11 - j01 * j10;
    double ddx = (j11 * fx - j01 * fy) / d, ddy = (-j10 * fx + j00 * fy) / d;
    X -= ddx;
    Y -= ddy;
    if (fabs(ddx) + fabs(ddy) < 1e-13) break;
  }
}

__global__ void k_synth_render(const double* __restrict__ bx, const double* __restrict__ by,
                               const double* __restrict__ br, const double* __restrict__ ba,
                               const int* __restrict__ cell_start, int ncx, int ncy, double x0, double y0, double cell,
                               int w, int h, int ss, const ofc_field* field, float* out) {
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  int y = blockIdx.y;
  if (x >= w) return;
  double acc = 0;
  for (int sy = 0; sy < ss; sy++)
    for (int sx = 0; sx < ss; sx++) {
      double px = x + (sx + 0.5) / ss - 0.5, py = y + (sy + 0.5) / ss - 0.5;
      double X = px, Y = py;
      if (field) field_inverse(*field, px, py, X, Y);
      int cx = (int)floor((X - x0) / cell), cy = (int)floor((Y - y0) / cell);
      double a = 0;
      for (int j = max(cy - 1, 0); j <= min(cy + 1, ncy - 1); j++)
        for (int i = max(cx - 1, 0); i <= min(cx + 1, ncx - 1); i++) {
          int c = j * ncx + i;
          for (int b = cell_start[c]; b < cell_start[c + 1]; b++) {
            double ddx = X - bx[b], ddy = Y - by[b], r = br[b];
            double d2 = ddx * ddx + ddy * ddy;
            double rad = 5.2 * r + 2.0;
            if (d2 > rad * rad) continue;
            a += ba[b] * (double)__expf((float)(-d2 / (2 * r * r)));
          }
        }
      acc += a;
    }
  out[(size_t)y * w + x] = (float)(0.5 + 0.25 * tanh(acc / (ss * ss)));
}

void synth_render_dev(const double* bx, const double* by, const double* br, const double* ba, const int* cell_start,
                      int ncx, int ncy, double x0, double y0, double cell, int w, int h, int ss, const ofc_field* field,
                      float* out, cudaStream_t st) {
  dim3 g(div_up(w, 128), h);
  OFC_LAUNCH(k_synth_render, g, 128, 0, st, bx, by, br, ba, cell_start, ncx, ncy, x0, y0, cell, w, h, ss, field, out);
}

}  // namespace ofc
