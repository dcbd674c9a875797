// fine.cu -- the per-pixel kernels of the fine stage (python/optflow_ref/phaseflow.py:427-511,
// rust/crates/optflow-core/src/phaseflow.rs:1514-1613): smoothing, splines, warp, accumulate, window moments
// and the local solve, the energy median, the confidence and the trusted pre-warp.
#include <cfloat>

#include "kernels.cuh"

#include <cuda_pipeline.h>

namespace ofc {

// ---------------------------------------------------------------- separable correlation ("nearest")
template <class Tin>
__global__ void k_corr_y(const Tin* __restrict__ in, double* __restrict__ out, int W, int H,
                         const double* __restrict__ taps, int r) {
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  int y = blockIdx.y;
  int pl = blockIdx.z;
  if (x >= W) return;
  const Tin* a = in + (size_t)pl * W * H;
  double s = 0;
  for (int j = -r; j <= r; j++) {
    int yy = min(max(y + j, 0), H - 1);
    s += taps[j + r] * (double)a[(size_t)yy * W + x];
  }
  out[(size_t)pl * W * H + (size_t)y * W + x] = s;
}

__global__ void k_corr_x(const double* __restrict__ in, double* __restrict__ out, int W, int H,
                         const double* __restrict__ taps, int r) {
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  int y = blockIdx.y;
  int pl = blockIdx.z;
  if (x >= W) return;
  const double* a = in + (size_t)pl * W * H + (size_t)y * W;
  double s = 0;
  for (int j = -r; j <= r; j++) {
    int xx = min(max(x + j, 0), W - 1);
    s += taps[j + r] * a[xx];
  }
  out[(size_t)pl * W * H + (size_t)y * W + x] = s;
}

// The same correlations for the default smoothing window (r = 16, sigma_s = 4). y: a thread owns CY_RY
// consecutive rows of a column and loads their 2r + CY_RY input rows once (instead of 2r + 1 loads per output,
// most of them L2 traffic); x: a block stages a row segment and its halo in shared memory and a thread forms
// CX_RX consecutive outputs from one register window (odd CX_RX: the warp's reads fall on distinct banks).
// Symmetric taps are paired (k(t) = k(-t)). Eight rows per thread in y (40 loads for 8 outputs, 80 registers, six
// blocks per SM) took 0.040 ms per pass of the two field planes at 2048^2 against 0.052 ms with four.
constexpr int CORR_R = 16, CY_RY = 8, CX_RX = 3;

__global__ void __launch_bounds__(128, 6) k_corr_y_rb(const double* __restrict__ in, double* __restrict__ out, int W,
                                                     int H, const double* __restrict__ taps) {
  constexpr int R = CORR_R, RY = CY_RY, NV = RY + 2 * R;
  __shared__ double tk[R + 1];
  if (threadIdx.x <= R) tk[threadIdx.x] = taps[R + threadIdx.x];
  __syncthreads();
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y0 = blockIdx.y * RY;
  if (x >= W) return;
  const double* a = in + (size_t)blockIdx.z * W * H + x;
  double v[NV];
#pragma unroll
  for (int i = 0; i < NV; i++) v[i] = a[(size_t)min(max(y0 - R + i, 0), H - 1) * W];
  double acc[RY];
#pragma unroll
  for (int j = 0; j < RY; j++) acc[j] = tk[0] * v[j + R];
#pragma unroll
  for (int t = 1; t <= R; t++) {
    const double k = tk[t];
#pragma unroll
    for (int j = 0; j < RY; j++) acc[j] = fma(k, v[j + R + t] + v[j + R - t], acc[j]);
  }
  double* o = out + (size_t)blockIdx.z * W * H + x;
#pragma unroll
  for (int j = 0; j < RY; j++)
    if (y0 + j < H) o[(size_t)(y0 + j) * W] = acc[j];
}

__global__ void __launch_bounds__(128) k_corr_x_rb(const double* __restrict__ in, double* __restrict__ out, int W, int H,
                                                  const double* __restrict__ taps) {
  constexpr int R = CORR_R, RX = CX_RX, NT = 128, SEG = NT * RX, WIN = SEG + 2 * R, NV = RX + 2 * R;
  __shared__ double tk[R + 1];
  __shared__ double wb[WIN];
  __shared__ double ob[SEG];
  const int tid = threadIdx.x, x0 = blockIdx.x * SEG;
  const double* row = in + (size_t)blockIdx.z * W * H + (size_t)blockIdx.y * W;
  if (tid <= R) tk[tid] = taps[R + tid];
  for (int i = tid; i < WIN; i += NT) wb[i] = row[min(max(x0 - R + i, 0), W - 1)];
  __syncthreads();
  double v[NV];
#pragma unroll
  for (int i = 0; i < NV; i++) v[i] = wb[tid * RX + i];
  double acc[RX];
#pragma unroll
  for (int j = 0; j < RX; j++) acc[j] = tk[0] * v[j + R];
#pragma unroll
  for (int t = 1; t <= R; t++) {
    const double k = tk[t];
#pragma unroll
    for (int j = 0; j < RX; j++) acc[j] = fma(k, v[j + R + t] + v[j + R - t], acc[j]);
  }
#pragma unroll
  for (int j = 0; j < RX; j++) ob[tid * RX + j] = acc[j];
  __syncthreads();
  double* o = out + (size_t)blockIdx.z * W * H + (size_t)blockIdx.y * W;
  for (int i = tid; i < SEG; i += NT)
    if (x0 + i < W) o[x0 + i] = ob[i];
}

void launch_corr_y(const double* in, double* out, int n_planes, int W, int H, const double* taps, int r, cudaStream_t st) {
  if (r == CORR_R) {
    dim3 g(div_up(W, 128), div_up(H, CY_RY), n_planes);
    OFC_LAUNCH(k_corr_y_rb, g, 128, 0, st, in, out, W, H, taps);
    return;
  }
  dim3 g(div_up(W, 128), H, n_planes);
  OFC_LAUNCH(k_corr_y<double>, g, 128, 0, st, in, out, W, H, taps, r);
}
void launch_corr_x(const double* in, double* out, int n_planes, int W, int H, const double* taps, int r, cudaStream_t st) {
  if (r == CORR_R) {
    dim3 g(div_up(W, 128 * CX_RX), H, n_planes);
    OFC_LAUNCH(k_corr_x_rb, g, 128, 0, st, in, out, W, H, taps);
    return;
  }
  dim3 g(div_up(W, 128), H, n_planes);
  OFC_LAUNCH(k_corr_x, g, 128, 0, st, in, out, W, H, taps, r);
}
void launch_corr_y_f32in(const float* in, double* out, int W, int H, const double* taps, int r, cudaStream_t st) {
  dim3 g(div_up(W, 128), H, 1);
  OFC_LAUNCH(k_corr_y<float>, g, 128, 0, st, in, out, W, H, taps, r);
}

// ---------------------------------------------------------------- B-spline prefilter in global memory
// Segmented recursive filter along one axis (interp.py:13-27): a line of length n with element stride
// `es`, lines `ls` apart. Each thread filters one segment of one line, entering it after a warm-up of
// IIR_WARM samples (exact when the warm-up reaches the line's start/end). Causal: in -> y (times 6);
// anticausal: y -> out.
constexpr int SEG = 32;

template <class Tin>
__global__ void k_iir_causal(const Tin* __restrict__ in, double* __restrict__ y, int n, int nlines, long es, long ls,
                             long plane) {
  int line = blockIdx.x * blockDim.x + threadIdx.x;
  if (line >= nlines) return;
  const int s0 = blockIdx.y * SEG;
  if (s0 >= n) return;
  const int e0 = min(n, s0 + SEG);
  const Tin* a = in + (size_t)blockIdx.z * plane + (size_t)line * ls;
  double* o = y + (size_t)blockIdx.z * plane + (size_t)line * ls;
  if (n == 1) { o[0] = (double)a[0]; return; }
  const double z = bspline_z();
  double acc;
  int i0;
  if (s0 - IIR_WARM <= 0) {
    int hz = min(n, HORIZON);
    acc = 0;
    double zk = 1;
    for (int k = 0; k < hz; k++) { acc += zk * (6.0 * (double)a[(size_t)k * es]); zk *= z; }
    if (s0 == 0) o[0] = acc;
    for (int i = 1; i < s0; i++) acc = 6.0 * (double)a[(size_t)i * es] + z * acc;
    i0 = s0 == 0 ? 1 : s0;
  } else {
    acc = 0;
    for (int i = s0 - IIR_WARM; i < s0; i++) acc = 6.0 * (double)a[(size_t)i * es] + z * acc;
    i0 = s0;
  }
  for (int i = i0; i < e0; i++) {
    acc = 6.0 * (double)a[(size_t)i * es] + z * acc;
    o[(size_t)i * es] = acc;
  }
}

template <class Tout>
__global__ void k_iir_anticausal(const double* __restrict__ y, Tout* __restrict__ out, int n, int nlines, long es,
                                 long ls, long plane) {
  int line = blockIdx.x * blockDim.x + threadIdx.x;
  if (line >= nlines) return;
  const int s0 = blockIdx.y * SEG;
  if (s0 >= n) return;
  const int e0 = min(n, s0 + SEG);
  const double* a = y + (size_t)blockIdx.z * plane + (size_t)line * ls;
  Tout* o = out + (size_t)blockIdx.z * plane + (size_t)line * ls;
  if (n == 1) { o[0] = (Tout)a[0]; return; }
  const double z = bspline_z();
  const double g = z / (z * z - 1.0);
  double c;
  if (e0 + IIR_WARM >= n - 1) {
    c = g * (a[(size_t)(n - 1) * es] + z * a[(size_t)(n - 2) * es]);
    if (e0 == n) o[(size_t)(n - 1) * es] = (Tout)c;
    for (int i = n - 2; i >= e0; i--) c = z * (c - a[(size_t)i * es]);
    if (e0 == n) {
      for (int i = n - 2; i >= s0; i--) { c = z * (c - a[(size_t)i * es]); o[(size_t)i * es] = (Tout)c; }
      return;
    }
  } else {
    c = 0;
    for (int i = e0 + IIR_WARM; i >= e0; i--) c = z * (c - a[(size_t)i * es]);
  }
  // c = c[e0]
  for (int i = e0 - 1; i >= s0; i--) { c = z * (c - a[(size_t)i * es]); o[(size_t)i * es] = (Tout)c; }
}

// Both recursions along x (rows) in one pass through a shared-memory tile: a block of XR_ROWS threads owns
// XR_ROWS rows and the column segment [s0, s0 + XR_SEG); it loads columns [s0 - IIR_WARM, e0 + IIR_WARM]
// (clamped to the row) with coalesced row reads, each thread runs the causal recursion over its tile row (warm-up
// from the tile's start, or the exact start at column 0) and then the anticausal one down to s0 (warm-up from the
// tile's end, or the exact start at the row's end), and the block stores the segment with coalesced row writes.
// One thread per row makes the recursion sequential in a row; an odd row stride keeps the threads' column
// accesses on distinct banks.
constexpr int XR_ROWS = 64, XR_SEG = 64, XR_TW = XR_SEG + 2 * IIR_WARM + 1;  // 121 doubles per tile row (odd)

// ILV: the planes (two) are written interleaved, out[2 p + plane]
template <class Tout, bool ILV>
__global__ void __launch_bounds__(XR_ROWS) k_iir_x(const double* __restrict__ in, Tout* __restrict__ out, int n, int nrows,
                                                  long plane) {
  extern __shared__ double tile[];  // XR_ROWS x XR_TW
  const int r0 = blockIdx.y * XR_ROWS, s0 = blockIdx.x * XR_SEG;
  const int e0 = min(n, s0 + XR_SEG), c0 = max(0, s0 - IIR_WARM), c1 = min(n, e0 + IIR_WARM + 1), cw = c1 - c0;
  const double* a = in + (size_t)blockIdx.z * plane;
  Tout* o = out + (size_t)blockIdx.z * plane;
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  // asynchronous copies: the whole tile is in flight at once (a load-then-store loop waits a DRAM latency per row)
  for (int rr = wid; rr < XR_ROWS; rr += nw) {
    if (r0 + rr >= nrows) break;
    const double* src = a + (size_t)(r0 + rr) * n + c0;
    for (int c = lane; c < cw; c += 32) __pipeline_memcpy_async(&tile[rr * XR_TW + c], src + c, sizeof(double));
  }
  __pipeline_commit();
  __pipeline_wait_prior(0);
  __syncthreads();
  const int row = threadIdx.x;
  if (r0 + row < nrows) {
    double* t = tile + row * XR_TW;  // t[i - c0] = value at column i
    if (n == 1) {
      // a single column: the coefficient is the value (as the separate passes give)
    } else {
      const double z = bspline_z();
      double acc;
      int i0;
      if (c0 == 0) {  // exact start: y[0] = sum_{k < min(n, 21)} z^k 6 x[k]
        const int hz = min(n, HORIZON);
        acc = 0;
        double zk = 1;
        for (int k = 0; k < hz; k++) {
          acc += zk * (6.0 * t[k]);
          zk *= z;
        }
        t[0] = acc;
        i0 = 1;
      } else {
        acc = 0;
        i0 = 0;
      }
#pragma unroll 4
      for (int i = i0; i < cw; i++) {
        acc = 6.0 * t[i] + z * acc;
        t[i] = acc;
      }
      const double g = z / (z * z - 1.0);
      double c;
      int i1;
      if (c1 == n) {  // exact start: c[n-1] = z / (z^2 - 1) (y[n-1] + z y[n-2])
        c = g * (t[cw - 1] + z * t[cw - 2]);
        t[cw - 1] = c;
        i1 = cw - 2;
      } else {
        c = 0;
        i1 = cw - 1;
      }
#pragma unroll 4
      for (int i = i1; i >= s0 - c0; i--) {
        c = z * (c - t[i]);
        t[i] = c;
      }
    }
  }
  __syncthreads();
  for (int rr = wid; rr < XR_ROWS; rr += nw) {
    if (r0 + rr >= nrows) break;
    const double* t = tile + rr * XR_TW + (s0 - c0);
    if (ILV) {
      Tout* dst = out + ((size_t)(r0 + rr) * n + s0) * 2 + blockIdx.z;
      for (int c = lane; c < e0 - s0; c += 32) dst[2 * c] = (Tout)t[c];
    } else {
      Tout* dst = o + (size_t)(r0 + rr) * n + s0;
      for (int c = lane; c < e0 - s0; c += 32) dst[c] = (Tout)t[c];
    }
  }
}

// y pass: in -> tmp (causal) -> tmp2 (anticausal); x pass: tmp2 -> out (ILV: two planes interleaved). tmp may alias
// out (it is dead once the x pass starts); tmp2 must not, since the x pass's tiles overlap.
template <class Tin, class Tout, bool ILV = false>
static void bspline_axes(const Tin* in, Tout* out, double* tmp, double* tmp2, int n_planes, int W, int H, cudaStream_t st) {
  long plane = (long)W * H;
  // along y: lines = columns (stride 1 apart), element stride W
  dim3 gy(div_up(W, 128), div_up(H, SEG), n_planes);
  OFC_LAUNCH((k_iir_causal<Tin>), gy, 128, 0, st, in, tmp, H, W, (long)W, 1L, plane);
  OFC_LAUNCH((k_iir_anticausal<double>), gy, 128, 0, st, tmp, tmp2, H, W, (long)W, 1L, plane);
  // along x: both recursions in one pass through shared-memory tiles
  const size_t sm = (size_t)XR_ROWS * XR_TW * sizeof(double);
  raise_smem_limit((const void*)k_iir_x<Tout, ILV>, sm);
  dim3 gx(div_up(W, XR_SEG), div_up(H, XR_ROWS), n_planes);
  OFC_LAUNCH((k_iir_x<Tout, ILV>), gx, XR_ROWS, sm, st, tmp2, out, W, H, plane);
}

void launch_bspline_f64(const double* in, double* out, double* tmp, int n_planes, int W, int H, cudaStream_t st) {
  // out doubles as the causal scratch of the y pass; tmp holds the y pass's result for the x pass
  bspline_axes<double, double>(in, out, (double*)out, tmp, n_planes, W, H, st);
}

void launch_bspline_f64_pair(const double* in, double2* out, double* tmp, int W, int H, cudaStream_t st) {
  // out (2 W H doubles) doubles as the causal scratch of the y pass; tmp holds the y pass's result
  bspline_axes<double, double, true>(in, (double*)out, (double*)out, tmp, 2, W, H, st);
}

void launch_bspline_f32(const float* in, float* out, double* tmp, int W, int H, cudaStream_t st) {
  // tmp holds 2 planes
  bspline_axes<float, float>(in, out, tmp, tmp + (size_t)W * H, 1, W, H, st);
}

// ---------------------------------------------------------------- warp
__global__ void __launch_bounds__(128, 8) k_warp(const float* __restrict__ c2, int w2, int h2, const double* __restrict__ sx,
                       const double* __restrict__ sy, long shx, long shy, int W, int H, float* __restrict__ out) {
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= W) return;
  for (int y = blockIdx.y; y < H; y += gridDim.y) {  // rows beyond the grid's 65535 in steps of gridDim.y
    size_t p = (size_t)y * W + x;
    Taps t;
    double v;
    if (make_taps(((double)x + (double)shx) + sx[p], ((double)y + (double)shy) + sy[p], w2, h2, t))
      v = sample_real(c2, w2, t);
    else
      v = nan("");
    out[p] = (float)v;
  }
}

// the warp as a plain gather: the form for coefficient planes whose row pitch is not a multiple of 16 bytes (no
// tensor map), and the reference the TMA-staged warp (warp_tma.cu) is checked against
void launch_warp_gather(const float* c2, int w2, int h2, const double* sx, const double* sy, long shx, long shy, int W,
                        int H, float* out, cudaStream_t st) {
  dim3 g(div_up(W, 128), (unsigned)std::min(H, 65535));
  OFC_LAUNCH(k_warp, g, 128, 0, st, c2, w2, h2, sx, sy, shx, shy, W, H, out);
}

// ---------------------------------------------------------------- accumulate
// One pixel per thread. The fixed point X' + s(X') = X + u(X) and the positions are float64; the responses are
// sampled with float32 weights and accumulation (they are stored as complex float32), and the phase difference
// angle(r1 conj(r2)) is taken in float32 by atan2_phase (the inputs carry float32 precision; the angle is within
// 5e-7 rad of theirs, at about half the instructions of atan2f); c = dphi + gx u + gy v and the seven sums are float64, since u reaches tens of pixels and the residual
// sum gcc - theta . b cancels. The kernel is latency-bound, so: the F reference-pack values of the pixel are
// copied to shared memory asynchronously at the start (in flight during the fixed point); |r1| |r2| is one square
// root of |r1|^2 |r2|^2, with |r1|^2 formed from the pack; the 16 tap offsets are computed once and reused by every
// filter; the field spline is stored interleaved (one 16-byte load per tap for both components); the responses are
// stored in filter pairs, node-major, so one 16-byte load per tap serves two filters (96 tap loads per pixel at F = 12
// instead of 192).
constexpr int ACC_BX = 32, ACC_BY = 8, ACC_T = ACC_BX * ACC_BY;
#ifndef ACC_MINB
#define ACC_MINB 4
#endif
__global__ void __launch_bounds__(ACC_T, ACC_MINB) k_accumulate(const float4* __restrict__ ref4, const float2* __restrict__ R,
                                                      int F, int ph, int pw, const double* __restrict__ ux,
                                                      const double* __restrict__ uy, const double* __restrict__ sx,
                                                      const double* __restrict__ sy, const double2* __restrict__ cs,
                                                      int W, int H, double* __restrict__ sums) {
  extern __shared__ float4 pk[];  // F x ACC_T
  // a block covers ACC_BX x ACC_BY pixels: its warps' response taps share rows in L1
  const int x = blockIdx.x * ACC_BX + threadIdx.x, y = blockIdx.y * ACC_BY + threadIdx.y;
  const int tid = threadIdx.y * ACC_BX + threadIdx.x;
  if (x >= W || y >= H) return;
  const size_t N = (size_t)W * H;
  const size_t p = (size_t)y * W + x;
  for (int k = 0; k < F; k++) __pipeline_memcpy_async(&pk[k * ACC_T + tid], ref4 + (size_t)k * N + p, 16);
  __pipeline_commit();
  const double u = ux[p], v = uy[p];
  const double tx = x + u, ty = y + v;
  double px = tx - sx[p], py = ty - sy[p];
  // X' + s(X') = X + u(X): two fixed-point steps on the spline of s (phaseflow.py:469-472)
  for (int it = 0; it < 2; it++) {
    Taps t;
    double nx, ny;
    if (make_taps(px, py, W, H, t)) {
      const double2 sv = sample_pair(cs, W, t);
      nx = tx - sv.x;
      ny = ty - sv.y;
    } else {
      nx = ny = nan("");
    }
    px = nx;
    py = ny;
  }
  double a0 = 0, a1 = 0, a2 = 0, a3 = 0, a4 = 0, a5 = 0, a6 = 0;
  Taps t;
  const bool ok = make_taps(px + PAD, py + PAD, pw, ph, t);
  float fwx[4], fwy[4];
#pragma unroll
  for (int k = 0; k < 4; k++) {
    fwx[k] = (float)t.wx[k];
    fwy[k] = (float)t.wy[k];
  }
  const size_t plane = (size_t)ph * pw;
  const float fnan = __int_as_float(0x7fc00000);
  // filter k's contribution from its complex response sample b at X' (r2 of phaseflow.py:476-483)
  auto add = [&](int k, float br, float bi) {
    const float4 r1 = pk[k * ACC_T + tid];
    // |r1|^2 as the reference pack's amplitude squared (phaseflow.py:111), from the stored float32 response
    const float q1 = fmaf(r1.x, r1.x, fmaf(r1.y, r1.y, 1e-12f));
    // r1 conj(r2)
    const float re = fmaf(r1.x, br, r1.y * bi);
    const float im = fmaf(r1.y, br, -r1.x * bi);
    const double dphi = (double)atan2_phase(im, re);
    const double wk = (double)sqrtf(q1 * fmaf(br, br, bi * bi));  // |r1| |r2|
    const double gx = r1.z, gy = r1.w;
    const double c = dphi + gx * u + gy * v;
    const double wgx = wk * gx, wgy = wk * gy;
    a0 = fma(wgx, gx, a0);
    a1 = fma(wgx, gy, a1);
    a2 = fma(wgy, gy, a2);
    a3 = fma(wgx, c, a3);
    a4 = fma(wgy, c, a4);
    a5 = fma(wk * c, c, a5);
    a6 += wk;
  };
  // the responses in filter pairs, node-major: one 16-byte load per tap gives both filters of a pair. A pair's
  // sample from its plane Rj, tap (jj, q) at Rj + off(jj, q); the next pair's tap rows go into L1 meanwhile
  const float4* R4 = reinterpret_cast<const float4*>(R);
  const int npairs = (F + 1) >> 1;
  auto pair_sample = [&](const float4* Rj, bool next, auto off, float& b0r, float& b0i, float& b1r, float& b1i) {
    if (next) {
#pragma unroll
      for (int jj = 0; jj < 4; jj++) asm volatile("prefetch.global.L1 [%0];" ::"l"(Rj + plane + off(jj, 0)));
    }
    b0r = b0i = b1r = b1i = 0.f;
#pragma unroll
    for (int jj = 0; jj < 4; jj++) {
      float a0r = 0.f, a0i = 0.f, a1r = 0.f, a1i = 0.f;
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const float4 cv = __ldg(Rj + off(jj, q));
        a0r = fmaf(fwx[q], cv.x, a0r);
        a0i = fmaf(fwx[q], cv.y, a0i);
        a1r = fmaf(fwx[q], cv.z, a1r);
        a1i = fmaf(fwx[q], cv.w, a1i);
      }
      b0r = fmaf(fwy[jj], a0r, b0r);
      b0i = fmaf(fwy[jj], a0i, b0i);
      b1r = fmaf(fwy[jj], a1r, b1r);
      b1i = fmaf(fwy[jj], a1i, b1i);
    }
  };
  __pipeline_wait_prior(0);
  if (ok && t.cx && t.yi[1] == t.yi[0] + 1 && t.yi[2] == t.yi[0] + 2 && t.yi[3] == t.yi[0] + 3) {
    // no reflection in either direction (all but the positions within a node of the padded plane's edge): the 4 x 4
    // taps are a block, one address per row and the four loads at fixed offsets from it
    const float4* Rj = R4 + ((size_t)t.yi[0] * pw + t.xi[0]);
    for (int j = 0; j < npairs; j++, Rj += plane) {
      float b0r, b0i, b1r, b1i;
      pair_sample(Rj, j + 1 < npairs, [&](int jj, int q) { return jj * pw + q; }, b0r, b0i, b1r, b1i);
      add(2 * j, b0r, b0i);
      if (2 * j + 1 < F) add(2 * j + 1, b1r, b1i);
    }
  } else {
    int ro[4], xo[4];  // tap (j, q) at ro[j] + xo[q] in a filter's plane
#pragma unroll
    for (int k = 0; k < 4; k++) {
      ro[k] = ok ? t.yi[k] * pw : 0;
      xo[k] = ok ? t.xi[k] : 0;
    }
    for (int j = 0; j < npairs; j++) {
      float b0r = fnan, b0i = fnan, b1r = fnan, b1i = fnan;
      if (ok)
        pair_sample(R4 + (size_t)j * plane, j + 1 < npairs, [&](int jj, int q) { return ro[jj] + xo[q]; }, b0r, b0i,
                    b1r, b1i);
      add(2 * j, b0r, b0i);
      if (2 * j + 1 < F) add(2 * j + 1, b1r, b1i);
    }
  }
  sums[p] = a0;
  sums[N + p] = a1;
  sums[2 * N + p] = a2;
  sums[3 * N + p] = a3;
  sums[4 * N + p] = a4;
  sums[5 * N + p] = a5;
  sums[6 * N + p] = a6;
}

// the accumulate as a gather from the response planes: the form for planes without tensor maps, and the reference
// the TMA-staged kernel (accumulate_tma.cu) is checked against
void launch_accumulate_gather(const float4* ref4, const float2* R, int F, int ph, int pw, const double* ux,
                              const double* uy, const double* sx, const double* sy, const double2* cs, int W, int H,
                              double* sums, cudaStream_t st) {
  dim3 g(div_up(W, ACC_BX), div_up(H, ACC_BY));
  const size_t sm = (size_t)F * ACC_T * sizeof(float4);
  if (sm > 227 * 1024) throw Error(OFC_ERR_WINDOW, "too many Gabor filters (" + std::to_string(F) + ") for the CUDA engine");
  raise_smem_limit((const void*)k_accumulate, sm);
  OFC_LAUNCH(k_accumulate, g, dim3(ACC_BX, ACC_BY), sm, st, ref4, R, F, ph, pw, ux, uy, sx, sy, cs, W, H, sums);
}

// ---------------------------------------------------------------- window moments + solve
// The moments a shape function of order 1 or 2 needs (phaseflow.py:123-161), resolved at compile time:
// sources 0..6 = gxx gxy gyy gxc gyc gcc gw; a moment is (source, px, py); the y pass makes (source, py).
struct MomTable {
  int n = 0, ny = 0, nm = 0;
  int ysrc[32] = {}, ypow[32] = {};
  int mjob[64] = {}, mpx[64] = {};
  int Midx[144] = {}, bidx[12] = {};
  int gcc = 0, gw = 0;
};

__host__ __device__ constexpr MomTable build_table(int order) {
  MomTable T{};
  int uc[12] = {}, ux_[12] = {}, uy_[12] = {};
  int pw1[6][2] = {{0, 0}, {1, 0}, {0, 1}, {2, 0}, {1, 1}, {0, 2}};
  int npw = order == 1 ? 3 : 6;
  int n = 0;
  uc[n] = 0; ux_[n] = 0; uy_[n] = 0; n++;
  uc[n] = 1; ux_[n] = 0; uy_[n] = 0; n++;
  for (int i = 1; i < npw; i++)
    for (int c = 0; c < 2; c++) { uc[n] = c; ux_[n] = pw1[i][0]; uy_[n] = pw1[i][1]; n++; }
  T.n = n;
  // moment list
  int msrc[64] = {}, mx[64] = {}, my[64] = {};
  int nm = 0;
  auto find_or_add = [&](int s, int px, int py) {
    for (int i = 0; i < nm; i++)
      if (msrc[i] == s && mx[i] == px && my[i] == py) return i;
    msrc[nm] = s; mx[nm] = px; my[nm] = py;
    return nm++;
  };
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) {
      int a = uc[i] < uc[j] ? uc[i] : uc[j], b = uc[i] < uc[j] ? uc[j] : uc[i];
      int key = a == 0 ? (b == 0 ? 0 : 1) : 2;
      T.Midx[i * n + j] = find_or_add(key, ux_[i] + ux_[j], uy_[i] + uy_[j]);
    }
  for (int i = 0; i < n; i++) T.bidx[i] = find_or_add(3 + uc[i], ux_[i], uy_[i]);
  T.gcc = find_or_add(5, 0, 0);
  T.gw = find_or_add(6, 0, 0);
  T.nm = nm;
  int ny = 0;
  for (int m = 0; m < nm; m++) {
    int j = -1;
    for (int q = 0; q < ny; q++)
      if (T.ysrc[q] == msrc[m] && T.ypow[q] == my[m]) j = q;
    if (j < 0) { T.ysrc[ny] = msrc[m]; T.ypow[ny] = my[m]; j = ny++; }
    T.mjob[m] = j;
    T.mpx[m] = mx[m];
  }
  T.ny = ny;
  return T;
}

int moment_yplanes(int order) { return build_table(order).ny; }

// The window taps k(t) t^p are symmetric in t for even p and antisymmetric for odd p, so each pass pairs
// the samples at +t and -t: sum_t k(t) t^p a(q + t) = [p == 0] k(0) a(q) + sum_{t >= 1} k(t) t^p (a(q + t) +- a(q - t)),
// which halves the float64 multiply-adds (the passes are float64-throughput bound).
template <int ORDER>
__global__ void __launch_bounds__(128) k_moments_y(const double* __restrict__ sums, int W, int H,
                                                   const double* __restrict__ mtaps, int r,
                                                   double* __restrict__ yplanes) {
  constexpr MomTable T = build_table(ORDER);
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  int y = blockIdx.y;
  if (x >= W) return;
  const size_t N = (size_t)W * H;
  const int K = 2 * r + 1;
  double acc[T.ny];
#pragma unroll
  for (int j = 0; j < T.ny; j++) acc[j] = 0;
#pragma unroll
  for (int j = 0; j < T.ny; j++)
    acc[j] = T.ypow[j] == 0 ? mtaps[r] * sums[(size_t)T.ysrc[j] * N + (size_t)y * W + x] : 0.0;
  for (int t = 1; t <= r; t++) {
    const size_t op = (size_t)min(y + t, H - 1) * W + x, om = (size_t)max(y - t, 0) * W + x;
#pragma unroll
    for (int src = 0; src < 7; src++) {
      bool used = false;
#pragma unroll
      for (int j = 0; j < T.ny; j++) used |= T.ysrc[j] == src;
      if (!used) continue;
      const double ap = sums[(size_t)src * N + op], am = sums[(size_t)src * N + om];
      const double sp = ap + am, dm = ap - am;
#pragma unroll
      for (int j = 0; j < T.ny; j++)
        if (T.ysrc[j] == src) acc[j] = fma(mtaps[T.ypow[j] * K + r + t], (T.ypow[j] & 1) ? dm : sp, acc[j]);
    }
  }
  size_t p = (size_t)y * W + x;
#pragma unroll
  for (int j = 0; j < T.ny; j++) yplanes[j * N + p] = acc[j];
}

// Every inner loop below runs over a constant trip count with a guard (k < j rather than a bound of j): a bound
// that depends on the outer index can leave the inner loop rolled, and the matrix then lives in local memory.
// One division per pivot: the factor's column and both substitutions multiply by the pivot's reciprocal.
template <int N>
__device__ __forceinline__ bool cholesky_solve_dev(double (&M)[N * N], double (&b)[N]) {
  bool okp = true;
  double il[N];
#pragma unroll
  for (int j = 0; j < N; j++) {
    double d = M[j * N + j];
#pragma unroll
    for (int k = 0; k < N; k++)
      if (k < j) d -= M[j * N + k] * M[j * N + k];
    okp &= d > 0.0 && d <= DBL_MAX;  // a failed pivot goes on with meaningless values and reports false
    // the substitutions below read the pivots only as 1 / l: one reciprocal square root instead of a square root and
    // a division (each a sequence of dependent float64 instructions)
    il[j] = rsqrt(d);
#pragma unroll
    for (int i = 0; i < N; i++) {
      if (i <= j) continue;
      double s = M[i * N + j];
#pragma unroll
      for (int k = 0; k < N; k++)
        if (k < j) s -= M[i * N + k] * M[j * N + k];
      M[i * N + j] = s * il[j];
    }
  }
#pragma unroll
  for (int i = 0; i < N; i++) {
    double s = b[i];
#pragma unroll
    for (int k = 0; k < N; k++)
      if (k < i) s -= M[i * N + k] * b[k];
    b[i] = s * il[i];
  }
#pragma unroll
  for (int i = N - 1; i >= 0; i--) {
    double s = b[i];
#pragma unroll
    for (int k = 0; k < N; k++)
      if (k > i) s -= M[k * N + i] * b[k];
    b[i] = s * il[i];
  }
  bool fin = okp;
#pragma unroll
  for (int i = 0; i < N; i++) fin &= isfinite(b[i]);
  return fin;
}

template <int ORDER>
__global__ void __launch_bounds__(128) k_moments_x_solve(const double* __restrict__ yplanes,
                                                         const double* __restrict__ uxin,
                                                         const double* __restrict__ uyin, int W, int H,
                                                         const double* __restrict__ mtaps, int r,
                                                         double* __restrict__ oux, double* __restrict__ ouy,
                                                         double* __restrict__ energy, double* __restrict__ resid,
                                                         double* __restrict__ slope) {
  constexpr MomTable T = build_table(ORDER);
  constexpr int n = ORDER == 1 ? 6 : 12;
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  int y = blockIdx.y;
  if (x >= W) return;
  const size_t N = (size_t)W * H;
  const int K = 2 * r + 1;
  // one pass over the tap pairs t = 1..r with every moment's accumulator live (independent chains)
  double m[T.nm];
  const double* row = yplanes + (size_t)y * W;
#pragma unroll
  for (int i = 0; i < T.nm; i++) m[i] = T.mpx[i] == 0 ? mtaps[r] * row[(size_t)T.mjob[i] * N + x] : 0.0;
  for (int t = 1; t <= r; t++) {
    const int xp = min(x + t, W - 1), xm = max(x - t, 0);
#pragma unroll
    for (int j = 0; j < T.ny; j++) {
      const double ap = row[(size_t)j * N + xp], am = row[(size_t)j * N + xm];
      const double sp = ap + am, dm = ap - am;
#pragma unroll
      for (int i = 0; i < T.nm; i++)
        if (T.mjob[i] == j) m[i] = fma(mtaps[T.mpx[i] * K + r + t], (T.mpx[i] & 1) ? dm : sp, m[i]);
    }
  }
  const size_t p = (size_t)y * W + x;
  double M[n * n], b[n], b0[n];
#pragma unroll
  for (int i = 0; i < n * n; i++) M[i] = m[T.Midx[i]];
#pragma unroll
  for (int i = 0; i < n; i++) b0[i] = b[i] = m[T.bidx[i]];
  const double m00 = M[0], m11 = M[n + 1], m01 = M[1];
  const double e = m00 + m11;
  const double det2 = m00 * m11 - m01 * m01;
  energy[p] = e;
  bool ok = det2 > APERTURE_TOL * e * e;
  if (ok) {
    double tr = 0;
#pragma unroll
    for (int i = 0; i < n; i++) tr += M[i * n + i];
    double ridge = (1e-12 / n) * tr;
#pragma unroll
    for (int i = 0; i < n; i++) M[i * n + i] += ridge;
    ok = cholesky_solve_dev<n>(M, b);
  }
  if (ok) {
    double fit = 0;
#pragma unroll
    for (int i = 0; i < n; i++) fit += b[i] * b0[i];
    double rr = m[T.gcc] - fit;
    resid[p] = sqrt(fmax(rr, 0.0) / (m[T.gw] + 1e-30));
    oux[p] = b[0];
    ouy[p] = b[1];
#pragma unroll
    for (int i = 0; i < 4; i++) slope[i * N + p] = b[2 + i];
  } else {
    resid[p] = PI;
    oux[p] = uxin[p];
    ouy[p] = uyin[p];
#pragma unroll
    for (int i = 0; i < 4; i++) slope[i * N + p] = 0.0;
  }
}

// ---- register-blocked window moments for the default window (r = MOM_R = 16, 33 taps)
// y pass: a thread owns RY consecutive rows of one column; it loads the RY + 2r rows of a source plane once
// (instead of 2r + 1 loads per output row, most of them L2 traffic) and forms every y-plane of that source,
// with the tap loop outermost so that the RY x (powers) accumulators advance side by side (independent
// float64 chains: the pass is bound by float64 latency otherwise).
constexpr int MOM_RY = 4;

template <int ORDER>
__global__ void __launch_bounds__(128, 4) k_moments_y_rb(const double* __restrict__ sums, int W, int H, MomTaps tp,
                                                         double* __restrict__ yplanes) {
  constexpr MomTable T = build_table(ORDER);
  constexpr int R = MOM_R, RY = MOM_RY, NV = RY + 2 * R;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y0 = blockIdx.y * RY;
  if (x >= W) return;
  const size_t N = (size_t)W * H;
#pragma unroll
  for (int src = 0; src < 7; src++) {
    bool used = false;
    bool pw[5] = {false, false, false, false, false};
#pragma unroll
    for (int j = 0; j < T.ny; j++)
      if (T.ysrc[j] == src) {
        used = true;
        pw[T.ypow[j]] = true;
      }
    if (!used) continue;
    const double* plane = sums + (size_t)src * N + x;
    double v[NV];
#pragma unroll
    for (int i = 0; i < NV; i++) v[i] = plane[(size_t)min(max(y0 - R + i, 0), H - 1) * W];
    double acc[RY][5];
#pragma unroll
    for (int j = 0; j < RY; j++)
#pragma unroll
      for (int p = 0; p < 5; p++) acc[j][p] = p == 0 ? tp.k[0][0] * v[j + R] : 0.0;
#pragma unroll
    for (int t = 1; t <= R; t++)
#pragma unroll
      for (int j = 0; j < RY; j++) {
        const double sp = v[j + R + t] + v[j + R - t], dm = v[j + R + t] - v[j + R - t];
#pragma unroll
        for (int p = 0; p < 5; p++)
          if (pw[p]) acc[j][p] = fma(tp.k[p][t], (p & 1) ? dm : sp, acc[j][p]);
      }
#pragma unroll
    for (int j = 0; j < RY; j++) {
      if (y0 + j >= H) break;
      const size_t o = (size_t)(y0 + j) * W + x;
#pragma unroll
      for (int q = 0; q < T.ny; q++)
        if (T.ysrc[q] == src) yplanes[(size_t)q * N + o] = acc[j][T.ypow[q]];
    }
  }
}

// x pass + solve: a block owns a row segment of SEG = GT RX pixels and has two groups of GT threads. The groups
// take the y-planes in pairs, group g plane Q + g of each pair: a group stages its plane's segment and 2r halo in
// shared memory (double-buffered per group, its next plane's loads in flight meanwhile); a thread takes the RX + 2r
// values around its RX consecutive pixels into registers (an odd RX keeps the warp's reads on distinct banks) and
// writes their moments into a shared tile of nm x SEG (tap loop outermost, RX x powers accumulators side by side).
// Then every thread of the block solves the pixels tid, tid + 2 GT, ... from the tile. Two groups give twice the warps
// per SM of one group of GT threads at the same tile (the tile, 8 nm bytes per pixel, bounds the blocks per SM), and
// each moment is formed by the same operations in the same order either way. Order 1 runs 4 blocks per SM (110
// registers); order 2 runs 2 (its 12 x 12 solve in registers takes 218).
template <int ORDER>
struct MomX {
  static constexpr int RX = ORDER == 1 ? 3 : 1;
  static constexpr int GT = 64, NT = 2 * GT, SEG = GT * RX, WIN = SEG + 2 * MOM_R;
  static constexpr size_t smem() { return (size_t)(4 * WIN + build_table(ORDER).nm * SEG) * sizeof(double); }
};

// the NPF values of a row segment (with its halo) that thread lt of a group stages: i = lt + GT j
template <int ORDER>
struct MomPf {
  static constexpr int NPF = (MomX<ORDER>::WIN + MomX<ORDER>::GT - 1) / MomX<ORDER>::GT;
  double v[NPF];
};

template <int ORDER>
__device__ __forceinline__ void mom_x_fetch(const double* __restrict__ row, int x0, int W, int lt, MomPf<ORDER>& pf) {
  constexpr int R = MOM_R, GT = MomX<ORDER>::GT, WIN = MomX<ORDER>::WIN;
#pragma unroll
  for (int j = 0; j < MomPf<ORDER>::NPF; j++) {
    const int i = lt + GT * j;
    if (i < WIN) pf.v[j] = row[min(max(x0 - R + i, 0), W - 1)];
  }
}

template <int ORDER>
__device__ __forceinline__ void mom_x_stage(double* wb, int lt, const MomPf<ORDER>& pf) {
  constexpr int GT = MomX<ORDER>::GT, WIN = MomX<ORDER>::WIN;
#pragma unroll
  for (int j = 0; j < MomPf<ORDER>::NPF; j++) {
    const int i = lt + GT * j;
    if (i < WIN) wb[i] = pf.v[j];
  }
}

// Per y-plane of an order: the number of x powers it feeds (always a prefix 0 .. npow - 1 of the powers) and the
// moment-tile row of each, so that one plane body per power count serves every plane
struct PlaneRows {
  int npow[32] = {};
  int mi[32][5] = {};
};
__host__ __device__ constexpr PlaneRows build_plane_rows(int order) {
  PlaneRows r{};
  const MomTable T = build_table(order);
  for (int q = 0; q < T.ny; q++) {
    for (int p = 0; p < 5; p++) r.mi[q][p] = -1;
    int np = 0;
    for (int m = 0; m < T.nm; m++)
      if (T.mjob[m] == q) {
        r.mi[q][T.mpx[m]] = m;
        if (T.mpx[m] + 1 > np) np = T.mpx[m] + 1;
      }
    r.npow[q] = np;
  }
  return r;
}
__host__ __device__ constexpr bool plane_rows_are_prefixes(int order) {
  const PlaneRows r = build_plane_rows(order);
  const MomTable T = build_table(order);
  for (int q = 0; q < T.ny; q++)
    for (int p = 0; p < r.npow[q]; p++)
      if (r.mi[q][p] < 0) return false;
  return true;
}
static_assert(plane_rows_are_prefixes(1) && plane_rows_are_prefixes(2), "a y-plane feeds a gap in the powers");
__host__ __device__ constexpr int max_plane_powers(int order) {
  const PlaneRows r = build_plane_rows(order);
  int mx = 0;
  for (int q = 0; q < build_table(order).ny; q++) mx = r.npow[q] > mx ? r.npow[q] : mx;
  return mx;
}
static_assert(max_plane_powers(1) == 3 && max_plane_powers(2) == 5, "the bodies' power counts");
__constant__ PlaneRows c_plane_rows[2] = {build_plane_rows(1), build_plane_rows(2)};

// one plane's x moments of powers 0 .. NP - 1 for a thread's RX pixels, from the segment in `wb`, into the tile rows mi
template <int ORDER, int NP>
__device__ __forceinline__ void mom_x_plane_np(const double* wb, double* mom, const int* mi, int lt, const MomTaps& tp) {
  constexpr int R = MOM_R, RX = MomX<ORDER>::RX, SEG = MomX<ORDER>::SEG, NV = RX + 2 * R;
  double v[NV];
#pragma unroll
  for (int i = 0; i < NV; i++) v[i] = wb[lt * RX + i];
  double acc[RX][NP];
#pragma unroll
  for (int i = 0; i < RX; i++)
#pragma unroll
    for (int p = 0; p < NP; p++) acc[i][p] = p == 0 ? tp.k[0][0] * v[i + R] : 0.0;
#pragma unroll
  for (int t = 1; t <= R; t++)
#pragma unroll
    for (int i = 0; i < RX; i++) {
      const double sp = v[i + R + t] + v[i + R - t], dm = v[i + R + t] - v[i + R - t];
#pragma unroll
      for (int p = 0; p < NP; p++) acc[i][p] = fma(tp.k[p][t], (p & 1) ? dm : sp, acc[i][p]);
    }
#pragma unroll
  for (int p = 0; p < NP; p++)
#pragma unroll
    for (int i = 0; i < RX; i++) mom[mi[p] * SEG + lt * RX + i] = acc[i][p];
}

template <int ORDER>
__global__ void __launch_bounds__(MomX<ORDER>::NT, ORDER == 1 ? 4 : 2) k_moments_x_solve_rb(const double* __restrict__ yplanes,
                                                               const double* __restrict__ uxin,
                                                               const double* __restrict__ uyin, int W, int H,
                                                               MomTaps tp, double* __restrict__ oux,
                                                               double* __restrict__ ouy, double* __restrict__ energy,
                                                               double* __restrict__ resid, double* __restrict__ slope) {
  constexpr MomTable T = build_table(ORDER);
  constexpr int n = ORDER == 1 ? 6 : 12;
  constexpr int GT = MomX<ORDER>::GT, NT = MomX<ORDER>::NT, SEG = MomX<ORDER>::SEG, WIN = MomX<ORDER>::WIN;
  extern __shared__ double smd[];
  double* mom = smd + 4 * WIN;
  const int tid = threadIdx.x, g = tid / GT, lt = tid - g * GT, y = blockIdx.y, x0 = blockIdx.x * SEG;
  const size_t N = (size_t)W * H;
  MomPf<ORDER> pf;
  if (g < T.ny) {  // group g's first plane into its buffer 0
    mom_x_fetch<ORDER>(yplanes + (size_t)g * N + (size_t)y * W, x0, W, lt, pf);
    mom_x_stage<ORDER>(smd + 2 * WIN * g, lt, pf);
  }
  __syncthreads();
  // the plane pairs (K, K + 1): group g takes plane K + g from its buffer (K / 2) & 1, one body per power count
  const PlaneRows& PR = c_plane_rows[ORDER - 1];
  double* gb = smd + 2 * WIN * g;  // the group's two buffers
#pragma unroll 1
  for (int K = 0; K < T.ny; K += 2) {
    const int Q = K + g;
    const double* wb = gb + ((K / 2) & 1) * WIN;
    double* wnext = gb + (((K / 2) + 1) & 1) * WIN;
    if (Q + 2 < T.ny) mom_x_fetch<ORDER>(yplanes + (size_t)(Q + 2) * N + (size_t)y * W, x0, W, lt, pf);
    if (Q < T.ny) {
      int mi[5];
#pragma unroll
      for (int p = 0; p < 5; p++) mi[p] = PR.mi[Q][p];
      const int np = PR.npow[Q];  // order 1: at most 3 (powers 0 .. 2); order 2: at most 5
      if (np == 1) mom_x_plane_np<ORDER, 1>(wb, mom, mi, lt, tp);
      else if (np == 2) mom_x_plane_np<ORDER, 2>(wb, mom, mi, lt, tp);
      else if (ORDER == 1 || np == 3) mom_x_plane_np<ORDER, 3>(wb, mom, mi, lt, tp);
      else if constexpr (ORDER > 1) {
        if (np == 4) mom_x_plane_np<ORDER, 4>(wb, mom, mi, lt, tp);
        else mom_x_plane_np<ORDER, 5>(wb, mom, mi, lt, tp);
      }
    }
    if (Q + 2 < T.ny) mom_x_stage<ORDER>(wnext, lt, pf);
    __syncthreads();
  }
#pragma unroll 1
  for (int s = tid; s < SEG; s += NT) {
    const int x = x0 + s;
    if (x >= W) continue;
    double m[T.nm];
#pragma unroll
    for (int k = 0; k < T.nm; k++) m[k] = mom[k * SEG + s];
    const size_t p = (size_t)y * W + x;
    double M[n * n], b[n], b0[n];
#pragma unroll
    for (int k = 0; k < n * n; k++) M[k] = m[T.Midx[k]];
#pragma unroll
    for (int k = 0; k < n; k++) b0[k] = b[k] = m[T.bidx[k]];
    const double m00 = M[0], m11 = M[n + 1], m01 = M[1];
    const double e = m00 + m11;
    const double det2 = m00 * m11 - m01 * m01;
    energy[p] = e;
    bool ok = det2 > APERTURE_TOL * e * e;
    if (ok) {
      double tr = 0;
#pragma unroll
      for (int k = 0; k < n; k++) tr += M[k * n + k];
      double ridge = (1e-12 / n) * tr;
#pragma unroll
      for (int k = 0; k < n; k++) M[k * n + k] += ridge;
      ok = cholesky_solve_dev<n>(M, b);
    }
    if (ok) {
      double fit = 0;
#pragma unroll
      for (int k = 0; k < n; k++) fit += b[k] * b0[k];
      double rr = m[T.gcc] - fit;
      resid[p] = sqrt(fmax(rr, 0.0) / (m[T.gw] + 1e-30));
      oux[p] = b[0];
      ouy[p] = b[1];
#pragma unroll
      for (int k = 0; k < 4; k++) slope[k * N + p] = b[2 + k];
    } else {
      resid[p] = PI;
      oux[p] = uxin[p];
      ouy[p] = uyin[p];
#pragma unroll
      for (int k = 0; k < 4; k++) slope[k * N + p] = 0.0;
    }
  }
}

template <int ORDER>
static void launch_moments_rb(const double* sums, const double* ux, const double* uy, int W, int H, const MomTaps& tp,
                              double* yplanes, double* oux, double* ouy, double* energy, double* resid, double* slope,
                              cudaStream_t st) {
  dim3 gy(div_up(W, 128), div_up(H, MOM_RY));
  OFC_LAUNCH(k_moments_y_rb<ORDER>, gy, 128, 0, st, sums, W, H, tp, yplanes);
  const size_t sm = MomX<ORDER>::smem();
  raise_smem_limit((const void*)k_moments_x_solve_rb<ORDER>, sm);
  dim3 gx(div_up(W, MomX<ORDER>::SEG), H);
  OFC_LAUNCH(k_moments_x_solve_rb<ORDER>, gx, MomX<ORDER>::NT, sm, st, yplanes, ux, uy, W, H, tp, oux, ouy, energy, resid,
             slope);
}

void launch_moments_solve(const double* sums, const double* ux, const double* uy, int W, int H, int order,
                          const double* mtaps, int r, const MomTaps& tp, double* yplanes, double* oux, double* ouy,
                          double* energy, double* resid, double* slope, cudaStream_t st) {
  if (r == MOM_R) {
    if (order == 1) launch_moments_rb<1>(sums, ux, uy, W, H, tp, yplanes, oux, ouy, energy, resid, slope, st);
    else launch_moments_rb<2>(sums, ux, uy, W, H, tp, yplanes, oux, ouy, energy, resid, slope, st);
    return;
  }
  dim3 g(div_up(W, 128), H);
  if (order == 1) {
    OFC_LAUNCH(k_moments_y<1>, g, 128, 0, st, sums, W, H, mtaps, r, yplanes);
    OFC_LAUNCH(k_moments_x_solve<1>, g, 128, 0, st, yplanes, ux, uy, W, H, mtaps, r, oux, ouy, energy, resid, slope);
  } else {
    OFC_LAUNCH(k_moments_y<2>, g, 128, 0, st, sums, W, H, mtaps, r, yplanes);
    OFC_LAUNCH(k_moments_x_solve<2>, g, 128, 0, st, yplanes, ux, uy, W, H, mtaps, r, oux, ouy, energy, resid, slope);
  }
}

// ---------------------------------------------------------------- energy statistics and median
__device__ __forceinline__ unsigned long long okey(double v) {  // order-preserving key of a double
  unsigned long long u = (unsigned long long)__double_as_longlong(v);
  return (u >> 63) ? ~u : (u | 0x8000000000000000ULL);
}
__device__ __forceinline__ double okey_inv(unsigned long long k) {
  unsigned long long u = (k >> 63) ? (k & 0x7FFFFFFFFFFFFFFFULL) : ~k;
  return __longlong_as_double((long long)u);
}

__device__ double atomic_min_d(double* a, double v) {
  unsigned long long* p = (unsigned long long*)a;
  unsigned long long old = *p, assumed;
  while (v < __longlong_as_double(old)) {
    assumed = old;
    old = atomicCAS(p, assumed, __double_as_longlong(v));
    if (old == assumed) break;
  }
  return __longlong_as_double(old);
}
__device__ double atomic_max_d(double* a, double v) {
  unsigned long long* p = (unsigned long long*)a;
  unsigned long long old = *p, assumed;
  while (v > __longlong_as_double(old)) {
    assumed = old;
    old = atomicCAS(p, assumed, __double_as_longlong(v));
    if (old == assumed) break;
  }
  return __longlong_as_double(old);
}

// ---- median of the energy (np.median, phaseflow.py:149-151): an exact radix select over order-preserving keys.
// 1. k_stats_hist0: min / max / NaN (the reset rule, phaseflow.rs:846-854) and the histogram of the top 12 key bits
//    in one scan; the last block decides whether the median is needed and picks the first digit.
// 2. k_radix_hist pass 1: the next 12 bits among the elements of that bucket.
// 3. k_radix_compact: the elements of the 24-bit bucket into a candidate list (room for all n), and the largest
//    key below the bucket.
// 4. k_radix_final (one block): the remaining 40 bits over the candidates, the largest key below the median's, and
//    the median (the mean of the two middle values for even n).
// Four or five launches per median whatever the data (k_stats_init first, unless the last k_reset primed the state);
// a bucket of many equal energies (heavy ties) only makes the one-block final select longer.
constexpr int RBITS = 12, RBINS = 1 << RBITS;
constexpr int RH_T = 512;

// the select state a median starts from (median, need_median and skip_reset, which the median's readers use, are
// left alone)
__device__ __forceinline__ void stats_prime(EnergyStats* s, size_t n) {
  s->lo = DBL_MAX;
  s->hi = -DBL_MAX;
  s->nan = 0;
  s->prefix = 0;
  s->rank = (long long)(n / 2);
  s->less = 0;
  s->ticket = 0;
  s->lo_val = 0;
  s->ncand = 0;
  s->below_max = 0;
}

__global__ void k_stats_init(EnergyStats* s, size_t n) { stats_prime(s, n); }

__device__ __forceinline__ void digit_of(int pass, int& shift, int& bits) {
  int hi = 64 - RBITS * pass;
  bits = hi >= RBITS ? RBITS : hi;
  shift = hi - bits;
}

// run by every thread of the last block of a histogram pass: scans the RBINS counts of hist, finds the bin that
// holds rank, extends the prefix by it, and clears hist and the ticket for the next pass
__device__ void radix_pick(unsigned long long* hist, EnergyStats* s, int shift, long long* wsum) {
  constexpr int per = RBINS / RH_T;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  long long c[per];
  long long loc = 0;
#pragma unroll
  for (int j = 0; j < per; j++) {
    c[j] = (long long)__ldcg(hist + tid * per + j);
    loc += c[j];
  }
  long long inc = loc;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    long long v = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += v;
  }
  if (lane == 31) wsum[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    long long w = lane < RH_T / 32 ? wsum[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      long long v = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += v;
    }
    if (lane < RH_T / 32) wsum[lane] = w;
  }
  __syncthreads();
  const long long excl = inc - loc + (wid ? wsum[wid - 1] : 0);
  const long long rank = s->rank;
  if (excl <= rank && rank < excl + loc) {  // exactly one thread
    long long acc = excl;
    int bin = tid * per;
#pragma unroll
    for (int j = 0; j < per; j++) {
      if (acc + c[j] > rank) {
        bin = tid * per + j;
        break;
      }
      acc += c[j];
    }
    s->prefix |= ((unsigned long long)bin) << shift;
    s->rank = rank - acc;
    s->less += acc;
  }
#pragma unroll
  for (int j = 0; j < per; j++) hist[tid * per + j] = 0;
  if (tid == 0) s->ticket = 0;
}

// adds the block histogram h to hist; returns true in every thread of the block that finished last
__device__ bool radix_flush(const unsigned int* h, unsigned long long* hist, EnergyStats* s, bool* last) {
  for (int i = threadIdx.x; i < RBINS; i += blockDim.x)
    if (h[i]) atomicAdd(&hist[i], (unsigned long long)h[i]);
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) *last = atomicAdd(&s->ticket, 1u) == gridDim.x - 1;
  __syncthreads();
  if (*last) __threadfence();
  return *last;
}

__global__ void __launch_bounds__(RH_T) k_stats_hist0(const double* __restrict__ e, size_t n, EnergyStats* s, int force,
                                                     unsigned long long* hist) {
  __shared__ unsigned int h[RBINS];
  __shared__ long long wsum[RH_T / 32];
  __shared__ double rlo[RH_T / 32], rhi[RH_T / 32];
  __shared__ int rnan[RH_T / 32];
  __shared__ bool last;
  for (int i = threadIdx.x; i < RBINS; i += blockDim.x) h[i] = 0;
  __syncthreads();
  double lo = DBL_MAX, hi = -DBL_MAX;
  int anynan = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double v = e[i];
    if (v != v) anynan = 1;
    else { lo = fmin(lo, v); hi = fmax(hi, v); }
    atomicAdd(&h[okey(v) >> (64 - RBITS)], 1u);
  }
  for (int o = 16; o; o >>= 1) {
    lo = fmin(lo, __shfl_xor_sync(0xffffffff, lo, o));
    hi = fmax(hi, __shfl_xor_sync(0xffffffff, hi, o));
    anynan |= __shfl_xor_sync(0xffffffff, anynan, o);
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) { rlo[wid] = lo; rhi[wid] = hi; rnan[wid] = anynan; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < RH_T / 32; w++) { lo = fmin(lo, rlo[w]); hi = fmax(hi, rhi[w]); anynan |= rnan[w]; }
    atomic_min_d(&s->lo, lo);
    atomic_max_d(&s->hi, hi);
    if (anynan) atomicOr(&s->nan, 1);
  }
  if (!radix_flush(h, hist, s, &last)) return;
  // the reset needs the median unless every energy is above 1e-9 max + 1e-30 (phaseflow.rs:846-854)
  const int snan = __ldcg(&s->nan);
  const double slo = __ldcg(&s->lo), shi = __ldcg(&s->hi);
  const bool skip = !snan && shi <= DBL_MAX / 2 && slo > 1e-9 * shi + 1e-30;
  const bool need = force || !skip;
  __syncthreads();
  if (threadIdx.x == 0) {
    s->skip_reset = skip ? 1 : 0;
    s->need_median = need ? 1 : 0;
    s->median = snan ? nan("") : 0.0;
  }
  if (need && !snan) {
    radix_pick(hist, s, 64 - RBITS, wsum);
  } else {
    for (int i = threadIdx.x; i < RBINS; i += blockDim.x) hist[i] = 0;
    if (threadIdx.x == 0) s->ticket = 0;
  }
}

// One pass over the elements that match the prefix: a block histogram of the digit, added to hist; the last block
// picks.
__global__ void __launch_bounds__(RH_T) k_radix_hist(const double* __restrict__ e, size_t n, EnergyStats* s, int pass,
                                                    unsigned long long* hist) {
  if (!s->need_median || s->nan) return;
  __shared__ unsigned int h[RBINS];
  __shared__ long long wsum[RH_T / 32];
  __shared__ bool last;
  for (int i = threadIdx.x; i < RBINS; i += blockDim.x) h[i] = 0;
  __syncthreads();
  int shift, bits;
  digit_of(pass, shift, bits);
  const unsigned long long prefix = s->prefix;
  const int hib = 64 - RBITS * pass;  // bits already fixed above `hib`
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    unsigned long long k = okey(e[i]);
    bool match = hib == 64 ? true : ((k >> hib) == (prefix >> hib));
    if (match) atomicAdd(&h[(k >> shift) & ((1ULL << bits) - 1)], 1u);
  }
  __syncthreads();
  if (!radix_flush(h, hist, s, &last)) return;
  radix_pick(hist, s, shift, wsum);
}

constexpr int CBITS = 64 - 2 * RBITS;  // key bits below the bucket of the first two passes

__global__ void k_radix_compact(const double* __restrict__ e, size_t n, EnergyStats* s, unsigned long long* cand) {
  if (!s->need_median || s->nan) return;
  const unsigned long long pre = s->prefix >> CBITS;
  unsigned long long below = 0;
  const int lane = threadIdx.x & 31;
  for (size_t i0 = blockIdx.x * (size_t)blockDim.x; i0 < n; i0 += (size_t)gridDim.x * blockDim.x) {
    const size_t i = i0 + threadIdx.x;
    unsigned long long k = 0;
    bool in = false;
    if (i < n) {
      k = okey(e[i]);
      const unsigned long long kk = k >> CBITS;
      in = kk == pre;
      if (kk < pre && k > below) below = k;
    }
    const unsigned m = __ballot_sync(0xffffffffu, in);
    if (m) {  // one atomic per warp: the warp's matches take consecutive slots
      unsigned base = 0;
      if (lane == __ffs(m) - 1) base = atomicAdd(&s->ncand, (unsigned)__popc(m));
      base = __shfl_sync(0xffffffffu, base, __ffs(m) - 1);
      const unsigned slot = base + __popc(m & ((1u << lane) - 1));
      if (in) cand[slot] = k;  // slots < n: at most n elements match
    }
  }
  for (int o = 16; o; o >>= 1) {
    const unsigned long long v = __shfl_xor_sync(0xffffffffu, below, o);
    below = v > below ? v : below;
  }
  if (lane == 0 && below) atomicMax(&s->below_max, below);
}

// the remaining CBITS bits of the median's key over the candidates (10-bit digits), and the largest key below it
// after the passes: prefix = key of the element of rank n/2; for even n the one of rank n/2 - 1 is the same value
// when `less` (elements below it) < n/2, else the largest element below it (lo_val)
__device__ void median_finish(EnergyStats* s, size_t n) {
  const double hi = okey_inv(s->prefix);
  if (n % 2) {
    s->median = hi;
    return;
  }
  double lo = hi;
  if (s->less >= (long long)(n / 2)) {
    unsigned long long k = *(unsigned long long*)&s->lo_val;
    lo = okey_inv(k);
  }
  s->median = (lo + hi) / 2.0;
}

// the last bits of the select over the candidates, then the median itself (thread 0)
__global__ void __launch_bounds__(1024) k_radix_final(EnergyStats* s, const unsigned long long* __restrict__ cand,
                                                      size_t n) {
  if (!s->need_median) return;
  if (s->nan) {
    if (threadIdx.x == 0) s->median = nan("");
    return;
  }
  const unsigned nc = s->ncand;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  __shared__ unsigned int h[1024];
  __shared__ unsigned int wtot[32];
  __shared__ unsigned long long sh_prefix, wmax[32];
  __shared__ long long sh_rank, sh_less;
  unsigned long long prefix = s->prefix;
  long long rank = s->rank, less = s->less;
  for (int shift = CBITS - 10; shift >= 0; shift -= 10) {
    h[tid] = 0;
    __syncthreads();
    for (unsigned i = tid; i < nc; i += 1024) {
      const unsigned long long k = cand[i];
      if ((k >> (shift + 10)) == (prefix >> (shift + 10))) atomicAdd(&h[(k >> shift) & 1023], 1u);
    }
    __syncthreads();
    const unsigned c = h[tid];
    unsigned inc = c;
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned v = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += v;
    }
    if (lane == 31) wtot[wid] = inc;
    __syncthreads();
    if (wid == 0) {
      unsigned w = wtot[lane];
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned v = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += v;
      }
      wtot[lane] = w;
    }
    __syncthreads();
    const long long excl = (long long)(inc - c) + (wid ? wtot[wid - 1] : 0);
    if (excl <= rank && rank < excl + (long long)c) {  // exactly one thread
      sh_prefix = prefix | ((unsigned long long)tid << shift);
      sh_rank = rank - excl;
      sh_less = less + excl;
    }
    __syncthreads();
    prefix = sh_prefix;
    rank = sh_rank;
    less = sh_less;
  }
  unsigned long long best = 0;
  for (unsigned i = tid; i < nc; i += 1024) {
    const unsigned long long k = cand[i];
    if (k < prefix && k > best) best = k;
  }
  for (int o = 16; o; o >>= 1) {
    const unsigned long long v = __shfl_xor_sync(0xffffffffu, best, o);
    best = v > best ? v : best;
  }
  if (lane == 0) wmax[wid] = best;
  __syncthreads();
  if (tid == 0) {
    best = s->below_max;
    for (int w = 0; w < 32; w++) best = wmax[w] > best ? wmax[w] : best;
    s->prefix = prefix;
    s->rank = rank;
    s->less = less;
    *(unsigned long long*)&s->lo_val = best;
    median_finish(s, n);
  }
}

void launch_energy_median(const double* energy, size_t n, EnergyStats* stats, bool force_median,
                          unsigned long long* scratch, cudaStream_t st, bool primed) {
  unsigned long long* hist = scratch;
  unsigned long long* cand = scratch + RBINS;
  if (!primed) OFC_LAUNCH(k_stats_init, 1, 1, 0, st, stats, n);
  OFC_LAUNCH(k_stats_hist0, 296, RH_T, 0, st, energy, n, stats, force_median ? 1 : 0, hist);
  OFC_LAUNCH(k_radix_hist, 296, RH_T, 0, st, energy, n, stats, 1, hist);
  OFC_LAUNCH(k_radix_compact, 296, 256, 0, st, energy, n, stats, cand);
  OFC_LAUNCH(k_radix_final, 1, 1024, 0, st, stats, cand, n);
}

__global__ void k_reset(const double* __restrict__ energy, const double* __restrict__ uxin,
                        const double* __restrict__ uyin, int n, EnergyStats* s, double* ux, double* uy,
                        double* resid, double* slope, int prime) {
  // the next median's start state, in place of its own k_stats_init launch (this kernel is the last reader of the
  // select state's result, and it reads only median and skip_reset)
  if (prime && blockIdx.x == 0 && threadIdx.x == 0) stats_prime(s, (size_t)n);
  if (s->skip_reset) return;
  const double thr = 1e-9 * s->median + 1e-30;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    if (!(energy[p] > thr)) {
      ux[p] = uxin[p];
      uy[p] = uyin[p];
      resid[p] = PI;
      for (int i = 0; i < 4; i++) slope[(size_t)i * n + p] = 0.0;
    }
  }
}

void launch_reset(const double* energy, const double* ux_in, const double* uy_in, int n, EnergyStats* stats,
                  double* ux, double* uy, double* resid, double* slope, cudaStream_t st, bool prime_next) {
  OFC_LAUNCH(k_reset, div_up(n, 256), 256, 0, st, energy, ux_in, uy_in, n, stats, ux, uy, resid, slope,
             prime_next ? 1 : 0);
}

// ---------------------------------------------------------------- confidence
__global__ void k_confidence(const double* __restrict__ energy, const double* __restrict__ resid,
                             const double* __restrict__ ux, const double* __restrict__ uy, int W, int H,
                             const EnergyStats* s, double tol, double conf_min, int border, double B,
                             float* conf_out, double* conf64, uint8_t* low, int* count_low) {
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  int y = blockIdx.y;
  if (x >= W) return;
  size_t p = (size_t)y * W + x;
  double scale = 0.25 * s->median + 1e-30;
  double ratio = energy[p] / scale;
  double tex = ratio != ratio ? ratio : fmin(1.0, ratio);
  double q = resid[p] / tol;
  double c = tex * exp(-(q * q));
  if (border) {
    double tx = x + ux[p], ty = y + uy[p];
    double own = (double)min(min(x, y), min(W - 1 - x, H - 1 - y));
    bool rep = own >= B && tx >= B && ty >= B && (W - 1) - tx >= B && (H - 1) - ty >= B;
    c = rep ? (c != c ? c : fmin(fmax(c, 0.0), 1.0)) : 0.0;
  }
  bool lw = c < conf_min;
  if (conf_out) conf_out[p] = (float)c;
  if (conf64) conf64[p] = c;
  if (low) low[p] = lw ? 1 : 0;
  if (count_low) {
    unsigned m = __ballot_sync(__activemask(), lw);
    if ((threadIdx.x & 31) == __ffs(__activemask()) - 1 && m) atomicAdd(count_low, __popc(m));
  }
}

void launch_confidence(const double* energy, const double* resid, const double* ux, const double* uy, int W, int H,
                       const EnergyStats* stats, double phase_tol, double conf_min, bool border, double B,
                       float* conf_out, double* conf64, uint8_t* low, int* count_low, cudaStream_t st) {
  dim3 g(div_up(W, 128), H);
  OFC_LAUNCH(k_confidence, g, 128, 0, st, energy, resid, ux, uy, W, H, stats, phase_tol, conf_min, border ? 1 : 0, B,
             conf_out, conf64, low, count_low);
}

// ---------------------------------------------------------------- bounded distance tests
// vertical distance (rows) to the nearest src pixel of the column within `cap`, else cap + 1
__global__ void k_vdist(const uint8_t* __restrict__ src, int W, int H, int cap, int* __restrict__ vd,
                        const int* gate) {
  if (gate && *gate == 0) return;
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  int y = blockIdx.y;
  if (x >= W) return;
  int best = cap + 1;
  for (int d = 0; d <= cap && d < best; d++) {
    if ((y - d >= 0 && src[(size_t)(y - d) * W + x]) || (y + d < H && src[(size_t)(y + d) * W + x])) best = d;
  }
  vd[(size_t)y * W + x] = best;
}

// squared distance from vd within cap; mode 0: out |= (d <= limit); mode 1: out = (d > limit); counts ok
__global__ void k_within(const int* __restrict__ vd, int W, int H, int cap, double limit, int mode, uint8_t* out,
                         const int* gate, int* count) {
  if (gate && *gate == 0) return;
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  int y = blockIdx.y;
  if (x >= W) return;
  long best = -1;
  const int* row = vd + (size_t)y * W;
  for (int dx = -cap; dx <= cap; dx++) {
    int xx = x + dx;
    if (xx < 0 || xx >= W) continue;
    int v = row[xx];
    if (v > cap) continue;
    long d2 = (long)dx * dx + (long)v * v;
    if (best < 0 || d2 < best) best = d2;
  }
  bool inside = best >= 0 && sqrt((double)best) <= limit;
  size_t p = (size_t)y * W + x;
  if (mode == 0) {
    if (inside) out[p] = 1;
  } else {
    bool okp = !inside;
    out[p] = okp ? 1 : 0;
    if (count) {
      unsigned m = __ballot_sync(__activemask(), okp);
      if ((threadIdx.x & 31) == __ffs(__activemask()) - 1 && m) atomicAdd(count, __popc(m));
    }
  }
}

// The same test in one pass through a shared-memory tile of WT_X x WT_Y pixels with a halo of cap (<= WT_CAPMAX)
// on every side: the vertical distances of the tile's columns come from two running scans per column (the last
// src row at or above, the next at or below), then each pixel takes the smallest dx^2 + v^2 over |dx| <= cap.
// Results equal k_vdist + k_within's; count (mode 1) is summed per block.
constexpr int WT_X = 128, WT_Y = 32, WT_CAPMAX = 32, WT_T = 256;

template <int CAPT>
__global__ void __launch_bounds__(WT_T) k_within_tile(const uint8_t* __restrict__ src, int W, int H, int cap_rt,
                                                      double limit, int mode, uint8_t* out, const int* gate,
                                                      int* count) {
  if (gate && *gate == 0) return;
  const int cap = CAPT ? CAPT : cap_rt;
  __shared__ uint8_t s[(WT_Y + 2 * WT_CAPMAX) * (WT_X + 2 * WT_CAPMAX)];
  __shared__ uint8_t vd[WT_Y * (WT_X + 2 * WT_CAPMAX)];
  __shared__ int wsum[WT_T / 32];
  const int TW = WT_X + 2 * cap, TH = WT_Y + 2 * cap, tid = threadIdx.x;
  const int bx = blockIdx.x * WT_X, by = blockIdx.y * WT_Y;
  // the tile, 8 loads in flight per thread
  for (int i0 = 0; i0 < TW * TH; i0 += 8 * WT_T) {
    uint8_t v[8];
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int i = i0 + u * WT_T + tid;
      const int ty = i / TW, tx = i - ty * TW, gx = bx - cap + tx, gy = by - cap + ty;
      v[u] = (i < TW * TH && gx >= 0 && gx < W && gy >= 0 && gy < H) ? __ldg(src + (size_t)gy * W + gx) : 0;
    }
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int i = i0 + u * WT_T + tid;
      if (i < TW * TH) s[i] = v[u];
    }
  }
  __syncthreads();
  for (int tx = tid; tx < TW; tx += WT_T) {
    int last = -(1 << 20);
    for (int ty = 0; ty < cap + WT_Y; ty++) {
      if (s[ty * TW + tx]) last = ty;
      if (ty >= cap) vd[(ty - cap) * TW + tx] = (uint8_t)min(ty - last, cap + 1);
    }
    int next = 1 << 20;
    for (int ty = TH - 1; ty >= cap; ty--) {
      if (s[ty * TW + tx]) next = ty;
      if (ty < cap + WT_Y) {
        uint8_t& v = vd[(ty - cap) * TW + tx];
        v = (uint8_t)min((int)v, min(next - ty, cap + 1));
      }
    }
  }
  __syncthreads();
  int cnt = 0;
  for (int i = tid; i < WT_X * WT_Y; i += WT_T) {  // the same trip count for every thread
    const int r = i / WT_X, c = i - r * WT_X, gx = bx + c, gy = by + r;
    const uint8_t* row = vd + r * TW + c + cap;
    int best = 1 << 30;  // no vertical distance within cap: d2 stays above every limit^2 with limit < cap
#pragma unroll
    for (int dx = -cap; dx <= cap; dx++) {
      const int v = row[dx];
      const int d2 = v > cap ? (1 << 30) : dx * dx + v * v;
      best = min(best, d2);
    }
    const bool inside = best < (1 << 30) && sqrt((double)best) <= limit;
    if (gx < W && gy < H) {
      const size_t p = (size_t)gy * W + gx;
      if (mode == 0) {
        if (inside) out[p] = 1;
      } else {
        out[p] = inside ? 0 : 1;
        cnt += inside ? 0 : 1;
      }
    }
  }
  if (count) {
    cnt = __reduce_add_sync(0xffffffffu, cnt);
    if ((tid & 31) == 0) wsum[tid >> 5] = cnt;
    __syncthreads();
    if (tid == 0) {
      int t = 0;
      for (int w = 0; w < WT_T / 32; w++) t += wsum[w];
      if (t) atomicAdd(count, t);
    }
  }
}

// out |= (distance to src <= limit) (mode 0), or out = (distance > limit) with the count of such pixels (mode 1),
// gated on *gate != 0 when gate is given
static void within(const uint8_t* src, int W, int H, double limit, int mode, uint8_t* out, int* vdist, const int* gate,
                   int* count, cudaStream_t st) {
  const int cap = (int)floor(limit) + 1;
  if (cap <= WT_CAPMAX) {
    dim3 g(div_up(W, WT_X), div_up(H, WT_Y));
    if (cap == 13)  // the default radii (12.22 px)
      OFC_LAUNCH(k_within_tile<13>, g, WT_T, 0, st, src, W, H, cap, limit, mode, out, gate, count);
    else
      OFC_LAUNCH(k_within_tile<0>, g, WT_T, 0, st, src, W, H, cap, limit, mode, out, gate, count);
    return;
  }
  dim3 g(div_up(W, 128), H);
  OFC_LAUNCH(k_vdist, g, 128, 0, st, src, W, H, cap, vdist, gate);
  OFC_LAUNCH(k_within, g, 128, 0, st, vdist, W, H, cap, limit, mode, out, gate, count);
}

void launch_within(const uint8_t* src, int W, int H, double limit, int mode, uint8_t* out, int* vdist, cudaStream_t st) {
  within(src, W, H, limit, mode, out, vdist, nullptr, nullptr, st);
}

// ---------------------------------------------------------------- trusted pre-warp
// Nearest ok pixel of each pixel's column (ties to the smaller row): col_d2 = dy^2 (or -1 without one), col_row.
// Two levels: k_col_segments records, per column and segment of CSEG rows, the first and last ok row; each pixel
// then scans its own segment and, beyond it, the segments' summaries (at most H / CSEG of them).
constexpr int CSEG = 64;

__global__ void k_col_segments(const uint8_t* __restrict__ ok, int W, int H, const PrewarpCounts* c,
                               int* __restrict__ seg_first, int* __restrict__ seg_last) {
  if (!(c->low > 0 && c->ok > 0 && c->ok < W * H)) return;
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  int sg = blockIdx.y;
  if (x >= W) return;
  int y0 = sg * CSEG, y1 = min(H, y0 + CSEG);
  int first = -1, last = -1;
  for (int y = y0; y < y1; y++)
    if (ok[(size_t)y * W + x]) {
      if (first < 0) first = y;
      last = y;
    }
  seg_first[(size_t)sg * W + x] = first;
  seg_last[(size_t)sg * W + x] = last;
}

__global__ void k_col_nearest(const uint8_t* __restrict__ ok, int W, int H, const PrewarpCounts* c,
                              const int* __restrict__ seg_first, const int* __restrict__ seg_last,
                              int* __restrict__ col_d2, int* __restrict__ col_row) {
  if (!(c->low > 0 && c->ok > 0 && c->ok < W * H)) return;
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  int y = blockIdx.y;
  if (x >= W) return;
  const size_t p = (size_t)y * W + x;
  const int sg = y / CSEG, y0 = sg * CSEG, y1 = min(H, y0 + CSEG);
  int up = -1, dn = -1;
  for (int yy = y; yy >= y0; yy--)
    if (ok[(size_t)yy * W + x]) { up = yy; break; }
  if (up < 0)
    for (int s2 = sg - 1; s2 >= 0; s2--) {
      int l = seg_last[(size_t)s2 * W + x];
      if (l >= 0) { up = l; break; }
    }
  for (int yy = y; yy < y1; yy++)
    if (ok[(size_t)yy * W + x]) { dn = yy; break; }
  if (dn < 0) {
    const int nseg = (H + CSEG - 1) / CSEG;
    for (int s2 = sg + 1; s2 < nseg; s2++) {
      int f = seg_first[(size_t)s2 * W + x];
      if (f >= 0) { dn = f; break; }
    }
  }
  int r = up;
  long d = up >= 0 ? (long)(y - up) : -1;
  if (dn >= 0 && (r < 0 || (long)(dn - y) < d)) { r = dn; d = dn - y; }
  col_row[p] = r;
  col_d2[p] = r < 0 ? -1 : (int)(d * d);
}

// for every pixel that is not ok: the nearest ok pixel (smallest (d^2, column, row)), then the first-order
// extrapolation u(N) + grad u(N) (X - N) (phaseflow.py:346-354); ok pixels keep u
__global__ void k_extrapolate(const uint8_t* __restrict__ ok, const int* __restrict__ col_d2,
                              const int* __restrict__ col_row, const double* __restrict__ ux,
                              const double* __restrict__ uy, const double* __restrict__ slope, int W, int H,
                              const PrewarpCounts* c, double* ux_pre, double* uy_pre) {
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  int y = blockIdx.y;
  if (x >= W) return;
  size_t p = (size_t)y * W + x;
  const bool apply = c->low > 0 && c->ok > 0 && c->ok < W * H;
  if (!apply || ok[p]) {
    ux_pre[p] = ux[p];
    uy_pre[p] = uy[p];
    return;
  }
  const int* cd = col_d2 + (size_t)y * W;
  const int* cr = col_row + (size_t)y * W;
  long best = -1;
  int bc = -1;
  for (long D = 0; D < W; D++) {
    if (best >= 0 && D * D > best) break;
    long xl = x - D, xr = x + D;
    if (xl >= 0 && cd[xl] >= 0) {
      long d2 = D * D + cd[xl];
      if (best < 0 || d2 < best || (d2 == best && xl < bc)) { best = d2; bc = (int)xl; }
    }
    if (D > 0 && xr < W && cd[xr] >= 0) {
      long d2 = D * D + cd[xr];
      if (best < 0 || d2 < best || (d2 == best && xr < bc)) { best = d2; bc = (int)xr; }
    }
  }
  int br = cr[bc];
  size_t q = (size_t)br * W + bc;
  size_t N = (size_t)W * H;
  double dx = (double)x - bc, dy = (double)y - br;
  ux_pre[p] = ux[q] + slope[q] * dx + slope[2 * N + q] * dy;
  uy_pre[p] = uy[q] + slope[N + q] * dx + slope[3 * N + q] * dy;
}

__global__ void k_zero_counts(PrewarpCounts* c) { c->ok = 0; }

void launch_prewarp_fill(const uint8_t* low, const double* ux, const double* uy, const double* slope, int W, int H,
                         double R, PrewarpCounts* counts, uint8_t* ok, int* vdist, int* col_d2, int* col_row,
                         double* ux_pre, double* uy_pre, cudaStream_t st) {
  dim3 g(div_up(W, 128), H);
  OFC_LAUNCH(k_zero_counts, 1, 1, 0, st, counts);
  // ok = distance to the nearest low pixel > R (gated on any low pixel)
  within(low, W, H, R, 1, ok, vdist, (const int*)&counts->low, &counts->ok, st);
  int* seg = vdist;  // the vertical distances are spent: 2 * ceil(H / CSEG) * W ints of segment summaries
  const int nseg = (H + CSEG - 1) / CSEG;
  OFC_LAUNCH(k_col_segments, dim3(div_up(W, 128), nseg), 128, 0, st, ok, W, H, counts, seg, seg + (size_t)nseg * W);
  OFC_LAUNCH(k_col_nearest, g, 128, 0, st, ok, W, H, counts, seg, seg + (size_t)nseg * W, col_d2, col_row);
  OFC_LAUNCH(k_extrapolate, g, 128, 0, st, ok, col_d2, col_row, ux, uy, slope, W, H, counts, ux_pre, uy_pre);
}

// ---------------------------------------------------------------- conversions
__global__ void k_d2f(const double* in, float* out, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = (float)in[i];
}
__global__ void k_f2d(const float* in, double* out, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = (double)in[i];
}
__global__ void k_fill(double* p, double v, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) p[i] = v;
}
void launch_f64_to_f32(const double* in, float* out, size_t n, cudaStream_t st) {
  OFC_LAUNCH(k_d2f, std::min<size_t>(div_up(n, 256), 4096), 256, 0, st, in, out, n);
}
void launch_f32_to_f64(const float* in, double* out, size_t n, cudaStream_t st) {
  OFC_LAUNCH(k_f2d, std::min<size_t>(div_up(n, 256), 4096), 256, 0, st, in, out, n);
}
void launch_fill_f64(double* p, double v, size_t n, cudaStream_t st) {
  OFC_LAUNCH(k_fill, std::min<size_t>(div_up(n, 256), 4096), 256, 0, st, p, v, n);
}

}  // namespace ofc
