// common.cuh -- shared device helpers of the optflow B200 engine (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/optflow_cuda.h"

namespace ofc {

constexpr double PI = 3.14159265358979323846;
constexpr int PAD = 32;                 // reflect padding of the Gabor responses (phaseflow.py:47)
constexpr double APERTURE_TOL = 1e-3;   // phaseflow.py:50
constexpr int HORIZON = 21;             // ceil(log(1e-12) / log|sqrt(3) - 2|) (interp.py:10)
constexpr int IIR_WARM = 28;            // samples of warm-up of a segmented recursive filter: z^29 < 3e-17

// An error that leaves the call with a status and a message (EngineError of the reference).
struct Error : std::runtime_error {
  int status;
  Error(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

#define OFC_CUDA(call)                                                                          \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess)                                                                      \
      throw ::ofc::Error(OFC_ERR_DEVICE, std::string("CUDA error ") + cudaGetErrorString(e_) + \
                                             " at " + __FILE__ + ":" + std::to_string(__LINE__)); \
  } while (0)

// kernel launch with error check, the engine's launch counter and, in profile mode, CUDA events around the
// launches whose kernel name matches the profile filter (the reference's per-kernel GPU timing,
// OPTFLOW_GPU_KERNELS, rust/README.md:157-159)
struct Profiler;
extern thread_local uint64_t* g_launch_counter;
extern thread_local Profiler* g_profiler;
void prof_before(const char* name, cudaStream_t st, void** token);
void prof_after(void* token, cudaStream_t st);
#define OFC_LAUNCH(kernel, grid, block, smem, stream, ...)                         \
  do {                                                                             \
    void* ofc_tok_ = nullptr;                                                      \
    if (::ofc::g_profiler) ::ofc::prof_before(#kernel, (stream), &ofc_tok_);       \
    kernel<<<(grid), (block), (smem), (stream)>>>(__VA_ARGS__);                    \
    OFC_CUDA(cudaGetLastError());                                                  \
    if (ofc_tok_) ::ofc::prof_after(ofc_tok_, (stream));                           \
    if (::ofc::g_launch_counter) ++*::ofc::g_launch_counter;                       \
  } while (0)

inline unsigned div_up(size_t a, size_t b) { return (unsigned)((a + b - 1) / b); }

// raises kernel fn's dynamic shared-memory limit on the current device to at least `bytes` and never lowers it:
// the limit belongs to the kernel, not to a launch, so host threads that launch it with different sizes at once
// (the pair driver's lanes) must not shrink it under each other's launches
void raise_smem_limit(const void* fn, size_t bytes);

// atan2(y, x) in float32 for finite or NaN arguments, from the mathematics: with a = min(|x|, |y|) / max(|x|, |y|)
// in [0, 1], atan(a) = a P(a^2), P the 8-term fit of atan(a) / a made by atan_fit.py (a minimax fit of the relative
// error by iteratively reweighted least squares; 1.6e-7 rad at most in a float32 Horner); then pi/2 - r where
// |y| > |x|, pi - r where x is negative (its sign bit: -0 included) and the sign of y (+-0 as atan2 gives them).
// At most 5e-7 rad (about 2 ulp of pi) from the exact angle of the float32 arguments with the quotient's rounding and
// the reflections; NaN in gives NaN; atan2(+-0, +0) = +-0 and atan2(+-0, -0) = +-pi.
__device__ __forceinline__ float atan2_phase(float y, float x) {
  if (y != y || x != x) return y + x;
  const float ax = fabsf(x), ay = fabsf(y);
  const float mx = fmaxf(ax, ay), mn = fminf(ax, ay);
  float a;
  if (mx > 1e-30f && mx < 1e30f) a = __fdividef(mn, mx);  // the reciprocal's range: a fast quotient
  else a = mx > 0.f ? mn / mx : 0.f;
  const float t = a * a;
  float p = -4.693272372e-03f;
  p = fmaf(p, t, 2.425239656e-02f);
  p = fmaf(p, t, -5.948639446e-02f);
  p = fmaf(p, t, 9.914293821e-02f);
  p = fmaf(p, t, -1.401948170e-01f);
  p = fmaf(p, t, 1.996972415e-01f);
  p = fmaf(p, t, -3.333199078e-01f);
  p = fmaf(p, t, 9.999999010e-01f);
  float r = p * a;
  if (ay > ax) r = 1.57079632679489662f - r;
  if (signbit(x)) r = 3.14159265358979324f - r;
  return copysignf(r, y);
}

// ---------------------------------------------------------------- cubic B-spline (interp.py)
__host__ __device__ inline long mirror_idx(long i, long n) {  // interp.py:38-43
  if (n == 1) return 0;
  long p = 2 * (n - 1);
  i = i < 0 ? -i : i;
  i %= p;
  return i >= n ? p - i : i;
}

// the reference's quotients by 6 as products with the nearest double to 1/6: a float64 division is a sequence of a
// dozen dependent instructions on the GPU, and the product is within an ulp of the quotient
__host__ __device__ inline void bspline_weights(double t, double w[4]) {  // interp.py:46-49
  const double s = 1.0 / 6.0;
  double t2 = t * t, t3 = t2 * t;
  double u = 1 - t;
  w[0] = u * u * u * s;
  w[1] = (3 * t3 - 6 * t2 + 4) * s;
  w[2] = (-3 * t3 + 3 * t2 + 3 * t + 1) * s;
  w[3] = t3 * s;
}

// taps of sample(): clamp to [0, n-1], floor, weights, mirrored indices (interp.py:52-69)
struct Taps {
  int xi[4], yi[4];
  double wx[4], wy[4];
  bool cx;  // xi[k] = xi[0] + k (no reflection in x): a row's four taps are adjacent
};

// mirror_idx for an index at most one reflection outside [0, n) (the taps of a clamped position lie in
// [-1, n + 1]): two compares instead of a division; the general rule where one reflection is not enough (n < 3)
__device__ __forceinline__ int mirror_near(int i, int n) {
  int m = i < 0 ? -i : i;
  if (m >= n) m = 2 * (n - 1) - m;
  if (m < 0 || m >= n) m = (int)mirror_idx(i, n);
  return m;
}

__device__ inline bool make_taps(double x, double y, int w, int h, Taps& t) {
  if (!(x == x) || !(y == y)) return false;
  x = fmin(fmax(x, 0.0), (double)(w - 1));
  y = fmin(fmax(y, 0.0), (double)(h - 1));
  double fx = floor(x), fy = floor(y);
  int x0 = (int)fx, y0 = (int)fy;
  bspline_weights(x - fx, t.wx);
  bspline_weights(y - fy, t.wy);
  // taps inside the plane (the usual case) need no mirroring: the same indices without the reflection tests
  const bool ix = x0 >= 1 && x0 + 2 <= w - 1, iy = y0 >= 1 && y0 + 2 <= h - 1;
  t.cx = ix;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    t.xi[k] = ix ? x0 + k - 1 : mirror_near(x0 + k - 1, w);
    t.yi[k] = iy ? y0 + k - 1 : mirror_near(y0 + k - 1, h);
  }
  return true;
}

template <class T>
__device__ inline double sample_real(const T* c, int w, const Taps& t) {
  double out = 0;
  if (t.cx) {  // adjacent taps: one address per row, the same operations in the same order
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const T* row = c + (size_t)t.yi[j] * w + t.xi[0];
      double acc = t.wx[0] * (double)row[0];
#pragma unroll
      for (int k = 1; k < 4; k++) acc += t.wx[k] * (double)row[k];
      out += t.wy[j] * acc;
    }
    return out;
  }
#pragma unroll
  for (int j = 0; j < 4; j++) {
    const T* row = c + (size_t)t.yi[j] * w;
    double acc = t.wx[0] * (double)row[t.xi[0]];
#pragma unroll
    for (int k = 1; k < 4; k++) acc += t.wx[k] * (double)row[t.xi[k]];
    out += t.wy[j] * acc;
  }
  return out;
}

// two real splines sampled at the same taps (one set of 32-bit offsets for both)
template <class T>
__device__ __forceinline__ void sample2_real(const T* __restrict__ c1, const T* __restrict__ c2, int w, const Taps& t,
                                             double& o1, double& o2) {
  int o[16];
#pragma unroll
  for (int j = 0; j < 4; j++)
#pragma unroll
    for (int k = 0; k < 4; k++) o[j * 4 + k] = t.yi[j] * w + t.xi[k];
  o1 = 0;
  o2 = 0;
#pragma unroll
  for (int j = 0; j < 4; j++) {
    double a1 = t.wx[0] * (double)c1[o[j * 4]], a2 = t.wx[0] * (double)c2[o[j * 4]];
#pragma unroll
    for (int k = 1; k < 4; k++) {
      a1 += t.wx[k] * (double)c1[o[j * 4 + k]];
      a2 += t.wx[k] * (double)c2[o[j * 4 + k]];
    }
    o1 += t.wy[j] * a1;
    o2 += t.wy[j] * a2;
  }
}

// two real splines stored interleaved (double2 per pixel), sampled at the same taps
__device__ __forceinline__ double2 sample_pair(const double2* __restrict__ c, int w, const Taps& t) {
  double o1 = 0, o2 = 0;
  if (t.cx) {  // adjacent taps: one address per row, the four loads at fixed offsets from it
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const double2* row = c + (size_t)t.yi[j] * w + t.xi[0];
      const double2 c0 = __ldg(row);
      double a1 = t.wx[0] * c0.x, a2 = t.wx[0] * c0.y;
#pragma unroll
      for (int k = 1; k < 4; k++) {
        const double2 v = __ldg(row + k);
        a1 += t.wx[k] * v.x;
        a2 += t.wx[k] * v.y;
      }
      o1 += t.wy[j] * a1;
      o2 += t.wy[j] * a2;
    }
    return make_double2(o1, o2);
  }
#pragma unroll
  for (int j = 0; j < 4; j++) {
    const double2* row = c + (size_t)t.yi[j] * w;
    const double2 c0 = __ldg(row + t.xi[0]);
    double a1 = t.wx[0] * c0.x, a2 = t.wx[0] * c0.y;
#pragma unroll
    for (int k = 1; k < 4; k++) {
      const double2 v = __ldg(row + t.xi[k]);
      a1 += t.wx[k] * v.x;
      a2 += t.wx[k] * v.y;
    }
    o1 += t.wy[j] * a1;
    o2 += t.wy[j] * a2;
  }
  return make_double2(o1, o2);
}

// complex spline stored as float2; float accumulation of the 16 taps with f64-derived weights
__device__ inline float2 sample_c32(const float2* __restrict__ c, int w, const Taps& t) {
  float re = 0.f, im = 0.f;
#pragma unroll
  for (int j = 0; j < 4; j++) {
    const float2* row = c + (size_t)t.yi[j] * w;
    float are = 0.f, aim = 0.f;
#pragma unroll
    for (int k = 0; k < 4; k++) {
      float2 v = __ldg(row + t.xi[k]);
      float wk = (float)t.wx[k];
      are = fmaf(wk, v.x, are);
      aim = fmaf(wk, v.y, aim);
    }
    float wj = (float)t.wy[j];
    re = fmaf(wj, are, re);
    im = fmaf(wj, aim, im);
  }
  return make_float2(re, im);
}

// scalar bspline prefilter pole
__host__ __device__ inline double bspline_z() { return sqrt(3.0) - 2.0; }  // interp.py:9

// one blob of the synthetic speckle renderer (synth.cu): reference centre, radius, amplitude and the subsample
// rectangle [i0, i1) x [j0, j1) it adds to
struct SynthBlob {
  double cx, cy, r, a;
  int i0, i1, j0, j1;
};

}  // namespace ofc
