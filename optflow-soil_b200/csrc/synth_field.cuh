// synth_field.cuh -- the displacement model of the synthetic speckle renderer (include/optflow_cuda_synth.h
// ofc_field): forward map x(X) and its Jacobian, on the host (the blobs' mapped centres) and on the device (the
// Newton inverse of every subsample). The affine + sinusoid part restates synth.Affine (python/optflow_ref/
// synth.py:33-51) with a sinusoid along X_x; the optional grid, settlement and band terms are this engine's own
// test fields (a Gaussian-process sample on a B-spline grid, a footing settling into sand, finite shear bands).
#pragma once
#include <cmath>

#include "../../include/optflow_cuda_synth.h"

namespace ofc {

#ifdef __CUDACC__
#define OFC_HD __host__ __device__
#else
#define OFC_HD
#endif

constexpr double SYN_PI = 3.14159265358979323846;

// cubic B-spline weights and their derivatives at fraction t of the interval [i, i + 1): taps i - 1 .. i + 2
OFC_HD inline void bspline_w(double t, double w[4], double d[4]) {
  const double s = 1.0 - t, t2 = t * t;
  w[0] = s * s * s / 6.0;
  w[1] = (3.0 * t2 * t - 6.0 * t2 + 4.0) / 6.0;
  w[2] = (-3.0 * t2 * t + 3.0 * t2 + 3.0 * t + 1.0) / 6.0;
  w[3] = t2 * t / 6.0;
  d[0] = -0.5 * s * s;
  d[1] = 1.5 * t2 - 2.0 * t;
  d[2] = -1.5 * t2 + t + 0.5;
  d[3] = 0.5 * t2;
}

// the optional terms (grid, settlement, bands): displacement (ux, uy) at X and its Jacobian j = du/dX
OFC_HD inline void field_extra(const ofc_field& f, double X, double Y, double& ux, double& uy, double j[4]) {
  ux = uy = 0.0;
  j[0] = j[1] = j[2] = j[3] = 0.0;
  if (f.grid && f.gnx > 0 && f.gny > 0) {
    const double gx = (X - f.gx0) / f.gh, gy = (Y - f.gy0) / f.gh;
    const double fx = floor(gx), fy = floor(gy);
    double wx[4], dx[4], wy[4], dy[4];
    bspline_w(gx - fx, wx, dx);
    bspline_w(gy - fy, wy, dy);
    const long ix = (long)fx, iy = (long)fy;
    const size_t plane = (size_t)f.gnx * f.gny;
    for (int a = 0; a < 4; a++) {
      long r = iy - 1 + a;
      r = r < 0 ? 0 : (r >= f.gny ? f.gny - 1 : r);
      double sx = 0, sy = 0, sdx = 0, sdy = 0;
      for (int b = 0; b < 4; b++) {
        long c = ix - 1 + b;
        c = c < 0 ? 0 : (c >= f.gnx ? f.gnx - 1 : c);
        const double vx = f.grid[(size_t)r * f.gnx + c], vy = f.grid[plane + (size_t)r * f.gnx + c];
        sx += wx[b] * vx;
        sy += wx[b] * vy;
        sdx += dx[b] * vx;
        sdy += dx[b] * vy;
      }
      ux += wy[a] * sx;
      uy += wy[a] * sy;
      j[0] += wy[a] * sdx / f.gh;
      j[1] += dy[a] * sx / f.gh;
      j[2] += wy[a] * sdy / f.gh;
      j[3] += dy[a] * sy / f.gh;
    }
  }
  if (f.fs != 0.0) {
    const double px = X < f.fx0 ? f.fx0 : (X > f.fx1 ? f.fx1 : X);
    const double ddx = X - px, ddy = Y - f.fy;
    const double d = sqrt(ddx * ddx + ddy * ddy);
    const double e = f.fs * exp(-d / f.fdecay);
    uy += e;
    if (d > 0) {
      j[2] += -e / f.fdecay * ddx / d;
      j[3] += -e / f.fdecay * ddy / d;
    }
  }
  for (int k = 0; k < f.n_bands && k < OFC_MAX_BANDS; k++) {
    const ofc_band& b = f.bands[k];
    const double rx = X - b.ex, ry = Y - b.ey;
    const double s = -b.ty * rx + b.tx * ry, a = b.tx * rx + b.ty * ry;
    const double th = tanh(s / b.width);
    double tp = 1.0, dtp = 0.0;
    if (b.length > 0) {
      const double t1 = tanh(a / b.width), t2 = tanh((b.length - a) / b.width);
      tp = 0.25 * (1.0 + t1) * (1.0 + t2);
      dtp = 0.25 / b.width * ((1.0 - t1 * t1) * (1.0 + t2) - (1.0 + t1) * (1.0 - t2 * t2));
    }
    const double g = 0.5 * b.delta * (th + b.bias);
    const double v = g * tp;
    ux += v * b.tx;
    uy += v * b.ty;
    // dv/dX = 0.5 delta (1 - th^2) / width * tp * n + g * dtp * t, n = (-ty, tx)
    const double cs = 0.5 * b.delta * (1.0 - th * th) / b.width * tp;
    const double gX = cs * -b.ty + g * dtp * b.tx, gY = cs * b.tx + g * dtp * b.ty;
    j[0] += b.tx * gX;
    j[1] += b.tx * gY;
    j[2] += b.ty * gX;
    j[3] += b.ty * gY;
  }
}

OFC_HD inline bool field_has_extra(const ofc_field& f) { return f.grid || f.fs != 0.0 || f.n_bands > 0; }

// x(X)
OFC_HD inline void field_fwd(const ofc_field& f, double X, double Y, double& x, double& y) {
  double dx = X - f.cx, dy = Y - f.cy;
  x = f.cx + f.a00 * dx + f.a01 * dy + f.tx;
  y = f.cy + f.a10 * dx + f.a11 * dy + f.ty;
  if (f.amp != 0.0) {
    double s = f.amp * sin(2 * SYN_PI * X / f.wavelength);
    x = x + s * f.sx;
    y = y + s * f.sy;
  }
  if (field_has_extra(f)) {
    double ux, uy, j[4];
    field_extra(f, X, Y, ux, uy, j);
    x += ux;
    y += uy;
  }
}

// X with x(X) = (x, y): the affine inverse, then Newton steps until the step is below 1e-13 (30 at most)
OFC_HD inline void field_inverse(const ofc_field& f, double x, double y, double& X, double& Y) {
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
      double ds = f.amp * (2 * SYN_PI / f.wavelength) * cos(2 * SYN_PI * X / f.wavelength);
      j00 += ds * f.sx;
      j10 += ds * f.sy;
    }
    if (extra) {
      double ux, uy, j[4];
      field_extra(f, X, Y, ux, uy, j);
      j00 += j[0];
      j01 += j[1];
      j10 += j[2];
      j11 += j[3];
    }
    double d = j00 * j11 - j01 * j10;
    double sx = (j11 * fx - j01 * fy) / d, sy = (-j10 * fx + j00 * fy) / d;
    X -= sx;
    Y -= sy;
    if (fabs(sx) + fabs(sy) < 1e-13) break;
  }
}

}  // namespace ofc
