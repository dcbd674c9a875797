// net.cu -- the learned coarse proposal (net.cuh): forward, backward and Adam on the GPU. The convolutions are
// im2col + tensor-core GEMMs (gemm_sm100.cu: bfloat16 operands, float32 accumulation); everything else (input
// normalisation, the correlation volume, soft-argmax, bias + ReLU, the loss, col2im, the optimiser) is in the
// kernels below, float32 throughout.
#include <cuda_bf16.h>

#include <cmath>
#include <string>
#include <vector>

#include "common.cuh"
#include "gemm_sm100.cuh"
#include "net.cuh"

namespace ofc {
namespace net {

size_t param_offset(int layer) {
  size_t o = 0;
  for (int l = 0; l < layer; l++) o += (size_t)SPECS[l].cout * kpad(SPECS[l].cin) + SPECS[l].cout;
  return o;
}
size_t param_count() { return param_offset(NCONV); }

namespace {

constexpr int PCH = 4096;  // pixel rows per weight-gradient GEMM batch (the pixel sum is split over the batch)
constexpr float CHARB_EPS2 = 0.01f;
constexpr size_t GEMM_WS = 1 << 20;

__device__ __forceinline__ float bf(uint16_t v) { return __uint_as_float((uint32_t)v << 16); }
__device__ __forceinline__ uint16_t to_bf(float v) {
  __nv_bfloat16 b = __float2bfloat16_rn(v);
  return *reinterpret_cast<uint16_t*>(&b);
}

// ---------------------------------------------------------------- input
__global__ void k_net_stats(const float* __restrict__ i1, const float* __restrict__ i2, int nb, size_t n,
                            double* stats) {
  const int img = blockIdx.y;
  const float* src = img < nb ? i1 + (size_t)img * n : i2 + (size_t)(img - nb) * n;
  double s = 0, q = 0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    double v = src[i];
    s += v;
    q += v * v;
  }
  for (int o = 16; o; o >>= 1) {
    s += __shfl_xor_sync(0xffffffff, s, o);
    q += __shfl_xor_sync(0xffffffff, q, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(stats + 2 * img, s);
    atomicAdd(stats + 2 * img + 1, q);
  }
}

// (image - mean) / (std + 1e-6) as bfloat16, one channel; images 0 .. nb - 1 from i1, then nb .. 2 nb - 1 from i2
__global__ void k_net_input(const float* __restrict__ i1, const float* __restrict__ i2, int nb, int h, int w,
                            const double* __restrict__ stats, uint16_t* out) {
  const int img = blockIdx.y;
  const size_t n = (size_t)h * w;
  const float* src = img < nb ? i1 + (size_t)img * n : i2 + (size_t)(img - nb) * n;
  const double mean = stats[2 * img] / n;
  const double var = fmax(stats[2 * img + 1] / n - mean * mean, 0.0);
  const float inv = (float)(1.0 / (sqrt(var) + 1e-6));
  const float m = (float)mean;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[(size_t)img * n + i] = to_bf((src[i] - m) * inv);
}

// ---------------------------------------------------------------- im2col / col2im (3 x 3, padding = dilation)
// col[m][k], m = (n, oy, ox), k = (ky 3 + kx) cin + c; rows m >= M and columns k >= 9 cin are zero
__global__ void k_im2col(const uint16_t* __restrict__ in, int Hi, int Wi, int cin, int Ho, int Wo, int stride,
                         int dil, int kp, size_t M, size_t Mpad, uint16_t* __restrict__ col) {
  const int groups = kp / 8;
  const size_t total = Mpad * groups;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const size_t m = t / groups;
    const int g = (int)(t - m * groups);
    uint16_t v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (m < M) {
      const int ox = (int)(m % Wo);
      const size_t r = m / Wo;
      const int oy = (int)(r % Ho);
      const size_t n = r / Ho;
      if ((cin & 7) == 0) {
        const int k0 = g * 8;
        if (k0 < 9 * cin) {
          const int tap = k0 / cin, c = k0 - tap * cin;
          const int iy = oy * stride - dil + (tap / 3) * dil, ix = ox * stride - dil + (tap % 3) * dil;
          if (iy >= 0 && iy < Hi && ix >= 0 && ix < Wi)
            *reinterpret_cast<uint4*>(v) =
                *reinterpret_cast<const uint4*>(in + (((n * Hi + iy) * Wi + ix) * cin + c));
        }
      } else {
        for (int j = 0; j < 8; j++) {
          const int k = g * 8 + j;
          if (k >= 9 * cin) break;
          const int tap = k / cin, c = k - tap * cin;
          const int iy = oy * stride - dil + (tap / 3) * dil, ix = ox * stride - dil + (tap % 3) * dil;
          if (iy >= 0 && iy < Hi && ix >= 0 && ix < Wi) v[j] = in[((n * Hi + iy) * Wi + ix) * cin + c];
        }
      }
    }
    *reinterpret_cast<uint4*>(col + m * kp + g * 8) = *reinterpret_cast<uint4*>(v);
  }
}

// dX[n][iy][ix][c] = sum of dcol over the (output, tap) pairs that read input (iy, ix)
__global__ void k_col2im(const float* __restrict__ dcol, int Hi, int Wi, int cin, int Ho, int Wo, int stride, int dil,
                         int kp, size_t nimg, float* __restrict__ dx) {
  const size_t total = nimg * Hi * Wi * cin;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(t % cin);
    size_t r = t / cin;
    const int ix = (int)(r % Wi);
    r /= Wi;
    const int iy = (int)(r % Hi);
    const size_t n = r / Hi;
    float s = 0.f;
    for (int ky = 0; ky < 3; ky++) {
      const int ty = iy + dil - ky * dil;
      if (ty < 0 || ty % stride) continue;
      const int oy = ty / stride;
      if (oy >= Ho) continue;
      for (int kx = 0; kx < 3; kx++) {
        const int tx = ix + dil - kx * dil;
        if (tx < 0 || tx % stride) continue;
        const int ox = tx / stride;
        if (ox >= Wo) continue;
        s += dcol[((n * Ho + oy) * Wo + ox) * kp + (ky * 3 + kx) * cin + c];
      }
    }
    dx[t] = s;
  }
}

// ---------------------------------------------------------------- bias + activation
__global__ void k_bias_act(const float* __restrict__ y, const float* __restrict__ bias, int cout, size_t M, int relu,
                           uint16_t* __restrict__ out16, float* __restrict__ out32) {
  const size_t total = M * cout;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    float v = y[t] + bias[t % cout];
    if (relu) v = fmaxf(v, 0.f);
    if (out16) out16[t] = to_bf(v);
    if (out32) out32[t] = v;
  }
}

// dY (bfloat16, rows >= M zero) = dout masked by the ReLU of the layer's output (act16 > 0), and the bias gradient
// (column sums of the masked dout) accumulated into db; blockDim = (256 / cout) * cout
__global__ void k_act_grad(const float* __restrict__ dout, const uint16_t* __restrict__ act16, int cout, size_t M,
                           size_t Mpad, int relu, uint16_t* __restrict__ dy16, float* __restrict__ db) {
  __shared__ float part[256];
  const int lanes = blockDim.x / cout;  // threads per column
  const int c = threadIdx.x % cout, lane = threadIdx.x / cout;
  float s = 0.f;
  const size_t rows_per_block = 64 * (size_t)lanes;
  const size_t r0 = (size_t)blockIdx.x * rows_per_block;
  for (size_t m = r0 + lane; m < r0 + rows_per_block && m < Mpad; m += lanes) {
    float g = 0.f;
    if (m < M) {
      g = dout[m * cout + c];
      if (relu && !(bf(act16[m * cout + c]) > 0.f)) g = 0.f;
    }
    s += g;
    dy16[m * cout + c] = to_bf(g);
  }
  part[threadIdx.x] = s;
  __syncthreads();
  if (lane == 0) {
    float t = 0.f;
    for (int l = 0; l < lanes; l++) t += part[l * cout + c];
    atomicAdd(db + c, t);
  }
}

// sum of the weight-gradient GEMM's partial products over the pixel batches
__global__ void k_sum_partials(const float* __restrict__ part, int L, size_t n, float* __restrict__ out) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int l = 0; l < L; l++) s += part[(size_t)l * n + i];
    out[i] = s;
  }
}

// ---------------------------------------------------------------- correlation volume
// f: 2 nb images of h x w x 32 (the first nb from image 1); out: nb x h x w x 160 bfloat16 (121 correlations,
// f1, 7 zeros) and corr32: nb x h x w x 121 float
__global__ void k_corr_fwd(const uint16_t* __restrict__ f, int nb, int h, int w, uint16_t* __restrict__ out,
                           float* __restrict__ corr32) {
  const size_t np = (size_t)nb * h * w;
  const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  const int x = (int)(p % w);
  const int y = (int)((p / w) % h);
  const size_t n = p / ((size_t)w * h);
  float a[FEAT];
  const uint16_t* f1 = f + p * FEAT;
#pragma unroll
  for (int c = 0; c < FEAT; c++) a[c] = bf(f1[c]);
  const uint16_t* f2 = f + np * FEAT + n * h * w * FEAT;
  uint16_t* o = out + p * DEC_IN;
  for (int k = 0; k < CORR_N; k++) {
    const int dy = k / CORR_D - CORR_R, dx = k % CORR_D - CORR_R;
    const int qy = y + dy, qx = x + dx;
    float s = 0.f;
    if (qy >= 0 && qy < h && qx >= 0 && qx < w) {
      const uint4* q = reinterpret_cast<const uint4*>(f2 + ((size_t)qy * w + qx) * FEAT);
#pragma unroll
      for (int v = 0; v < FEAT / 8; v++) {
        uint4 u = q[v];
        const uint16_t* e = reinterpret_cast<const uint16_t*>(&u);
#pragma unroll
        for (int j = 0; j < 8; j++) s = fmaf(a[v * 8 + j], bf(e[j]), s);
      }
      s *= 1.0f / FEAT;
    }
    corr32[p * CORR_N + k] = s;
    o[k] = to_bf(s);
  }
#pragma unroll
  for (int c = 0; c < FEAT; c++) o[CORR_N + c] = f1[c];
  for (int c = CORR_N + FEAT; c < DEC_IN; c++) o[c] = 0;
}

// g = the gradient of the correlations (ddec channels 0..120 + dsa) and of the f1 copy (ddec 121..152):
// df (2 nb x h x w x 32): df1(p) = sum_d g(p, d) f2(p + d) / 32 + copy(p); df2(q) = sum_d g(q - d, d) f1(q - d) / 32
__global__ void k_corr_bwd(const uint16_t* __restrict__ f, const float* __restrict__ ddec,
                           const float* __restrict__ dsa, int nb, int h, int w, float* __restrict__ df) {
  const size_t np = (size_t)nb * h * w;
  const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  const int x = (int)(p % w);
  const int y = (int)((p / w) % h);
  const size_t n = p / ((size_t)w * h);
  const uint16_t* F1 = f;
  const uint16_t* F2 = f + np * FEAT;
  float g1[FEAT], g2[FEAT];
#pragma unroll
  for (int c = 0; c < FEAT; c++) {
    g1[c] = ddec[p * DEC_IN + CORR_N + c];
    g2[c] = 0.f;
  }
  for (int k = 0; k < CORR_N; k++) {
    const int dy = k / CORR_D - CORR_R, dx = k % CORR_D - CORR_R;
    // image 1 at p against image 2 at p + d
    int qy = y + dy, qx = x + dx;
    if (qy >= 0 && qy < h && qx >= 0 && qx < w) {
      const float g = (ddec[p * DEC_IN + k] + dsa[p * CORR_N + k]) * (1.0f / FEAT);
      const uint16_t* q = F2 + ((n * h + qy) * w + qx) * FEAT;
#pragma unroll
      for (int c = 0; c < FEAT; c++) g1[c] = fmaf(g, bf(q[c]), g1[c]);
    }
    // image 2 at p is read by image 1 at p - d
    qy = y - dy;
    qx = x - dx;
    if (qy >= 0 && qy < h && qx >= 0 && qx < w) {
      const size_t pq = (n * h + qy) * w + qx;
      const float g = (ddec[pq * DEC_IN + k] + dsa[pq * CORR_N + k]) * (1.0f / FEAT);
      const uint16_t* q = F1 + pq * FEAT;
#pragma unroll
      for (int c = 0; c < FEAT; c++) g2[c] = fmaf(g, bf(q[c]), g2[c]);
    }
  }
#pragma unroll
  for (int c = 0; c < FEAT; c++) {
    df[p * FEAT + c] = g1[c];
    df[(np + p) * FEAT + c] = g2[c];
  }
}

// ---------------------------------------------------------------- soft-argmax prior, flow, loss
__global__ void k_softargmax(const float* __restrict__ corr32, const float* __restrict__ y4, size_t np,
                             float* __restrict__ flow) {
  const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  const float* c = corr32 + p * CORR_N;
  float mx = -INFINITY;
  for (int k = 0; k < CORR_N; k++) mx = fmaxf(mx, c[k]);
  float z = 0.f, sx = 0.f, sy = 0.f;
  for (int k = 0; k < CORR_N; k++) {
    const float e = __expf(c[k] - mx);
    z += e;
    sx += e * (float)(k % CORR_D - CORR_R);
    sy += e * (float)(k / CORR_D - CORR_R);
  }
  flow[2 * p] = SCALE * sx / z + y4[p * 16];
  flow[2 * p + 1] = SCALE * sy / z + y4[p * 16 + 1];
}

__global__ void k_softargmax_bwd(const float* __restrict__ corr32, const float* __restrict__ dflow, size_t np,
                                 float* __restrict__ dsa) {
  const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  const float* c = corr32 + p * CORR_N;
  float mx = -INFINITY;
  for (int k = 0; k < CORR_N; k++) mx = fmaxf(mx, c[k]);
  float z = 0.f;
  for (int k = 0; k < CORR_N; k++) z += __expf(c[k] - mx);
  const float gx = dflow[2 * p] * SCALE, gy = dflow[2 * p + 1] * SCALE;
  float mean = 0.f;
  for (int k = 0; k < CORR_N; k++)
    mean += __expf(c[k] - mx) / z * (gx * (float)(k % CORR_D - CORR_R) + gy * (float)(k / CORR_D - CORR_R));
  for (int k = 0; k < CORR_N; k++) {
    const float e = gx * (float)(k % CORR_D - CORR_R) + gy * (float)(k / CORR_D - CORR_R);
    dsa[p * CORR_N + k] = __expf(c[k] - mx) / z * (e - mean);
  }
}

// loss = inv_count * sum over the masked cells of sqrt(|flow - target|^2 + eps^2); dflow = its gradient; dy4
// (np x 16): dflow in the first two channels
__global__ void k_loss(const float* __restrict__ flow, const float* __restrict__ target, const uint8_t* __restrict__ mask,
                       size_t np, float inv_count, double* loss, float* __restrict__ dflow, float* __restrict__ dy4) {
  const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  double l = 0;
  if (p < np) {
    float gx = 0.f, gy = 0.f;
    if (mask[p]) {
      const float dx = flow[2 * p] - target[2 * p], dy = flow[2 * p + 1] - target[2 * p + 1];
      const float r = sqrtf(dx * dx + dy * dy + CHARB_EPS2);
      l = r * inv_count;
      gx = dx / r * inv_count;
      gy = dy / r * inv_count;
    }
    dflow[2 * p] = gx;
    dflow[2 * p + 1] = gy;
    for (int c = 0; c < 16; c++) dy4[p * 16 + c] = c == 0 ? gx : (c == 1 ? gy : 0.f);
  }
  for (int o = 16; o; o >>= 1) l += __shfl_xor_sync(0xffffffff, l, o);
  if ((threadIdx.x & 31) == 0 && l != 0) atomicAdd(loss, l);
}

// ---------------------------------------------------------------- optimiser
__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       size_t n, float lr, float b1, float b2, float eps, float c1, float c2) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi, vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

__global__ void k_to_bf16(const float* __restrict__ p, size_t n, uint16_t* __restrict__ o) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    o[i] = to_bf(p[i]);
}

unsigned grid_for(size_t n, int t = 256) { return (unsigned)std::min<size_t>((n + t - 1) / t, 148 * 16); }

template <class T>
T* get(const Workspace& ws, const std::string& name, size_t n) {
  return static_cast<T*>(ws.alloc(name, std::max<size_t>(n, 1) * sizeof(T)));
}

struct LayerGeom {
  int nimg, Hi, Wi, Ho, Wo;
  size_t M, Mpad;
};

// forward (and backward when grads != null)
void run(const Workspace& ws, const float* params, const uint16_t* w16, const float* i1, const float* i2, int nb,
         int h, int w, const float* target, const uint8_t* mask, float* flow, float* grads, double* loss) {
  if (h % SCALE || w % SCALE || h < 16 || w < 16) throw Error(OFC_ERR_ARG, "network input sides must be multiples of 8");
  cudaStream_t st = ws.st;
  const int nimg = 2 * nb;
  const int h8 = h / SCALE, w8 = w / SCALE;
  LayerGeom G[NCONV];
  for (int l = 0; l < NCONV; l++) {
    const int n = l < 4 ? nimg : nb;
    int Hi, Wi;
    if (l == 0) { Hi = h; Wi = w; }
    else if (l == 4) { Hi = h8; Wi = w8; }
    else { Hi = G[l - 1].Ho; Wi = G[l - 1].Wo; }
    const int s = SPECS[l].stride;
    G[l] = {n, Hi, Wi, Hi / s, Wi / s, 0, 0};
    G[l].M = (size_t)n * G[l].Ho * G[l].Wo;
    G[l].Mpad = (G[l].M + PCH - 1) / PCH * PCH;
  }
  // input
  double* stats = get<double>(ws, "net_stats", 2 * nimg);
  OFC_CUDA(cudaMemsetAsync(stats, 0, 2 * nimg * sizeof(double), st));
  const size_t npx = (size_t)h * w;
  OFC_LAUNCH(k_net_stats, dim3(64, nimg), 256, 0, st, i1, i2, nb, npx, stats);
  uint16_t* x0 = get<uint16_t>(ws, "net_x0", nimg * npx);
  OFC_LAUNCH(k_net_input, dim3(64, nimg), 256, 0, st, i1, i2, nb, h, w, stats, x0);
  void* gws = ws.alloc("net_gemm_ws", GEMM_WS);
  uint16_t* act[NCONV] = {};
  uint16_t* col[NCONV] = {};
  uint16_t* dec_in = get<uint16_t>(ws, "net_decin", (size_t)nb * h8 * w8 * DEC_IN);
  float* corr32 = get<float>(ws, "net_corr32", (size_t)nb * h8 * w8 * CORR_N);
  float* y4 = nullptr;
  for (int l = 0; l < NCONV; l++) {
    const ConvSpec& S = SPECS[l];
    const LayerGeom& g = G[l];
    const int kp = kpad(S.cin);
    const uint16_t* in = l == 0 ? x0 : (l == 4 ? dec_in : act[l - 1]);
    col[l] = get<uint16_t>(ws, "net_col" + std::to_string(l), g.Mpad * kp);
    OFC_LAUNCH(k_im2col, grid_for(g.Mpad * kp / 8), 256, 0, st, in, g.Hi, g.Wi, S.cin, g.Ho, g.Wo, S.stride, S.dil, kp,
               g.M, g.Mpad, col[l]);
    const float* bias = params + param_offset(l) + (size_t)S.cout * kp;
    if (l == NCONV - 1) {
      // the last layer's float32 output: the flow's residual channels
      float* y32 = get<float>(ws, "net_y" + std::to_string(l), g.Mpad * S.cout);
      GemmArgs a{(int)g.M, S.cout, kp, 1, col[l], kp, 0, w16 + param_offset(l), kp, 0, y32, S.cout, 0, 0.f,
                 "k_gemm_sm100_fprop"};
      gemm_bf16(GemmKind::ForwardTN, a, gws, GEMM_WS, st);
      y4 = get<float>(ws, "net_y4", g.M * S.cout);
      OFC_LAUNCH(k_bias_act, grid_for(g.M * S.cout), 256, 0, st, y32, bias, S.cout, g.M, 0, (uint16_t*)nullptr, y4);
    } else {
      // bias, ReLU and the bfloat16 store in the GEMM's epilogue
      act[l] = get<uint16_t>(ws, "net_act" + std::to_string(l), g.M * S.cout);
      FusedArgs a{(int)g.M, S.cout, kp, col[l], kp, w16 + param_offset(l), kp, act[l], S.cout, bias,
                  "k_gemm_sm100_fprop_fused"};
      gemm_bf16_fused(S.relu != 0, a, gws, GEMM_WS, st);
    }
    if (l == 3) {
      const size_t np = (size_t)nb * h8 * w8;
      OFC_LAUNCH(k_corr_fwd, div_up(np, 128), 128, 0, st, act[3], nb, h8, w8, dec_in, corr32);
    }
  }
  const size_t ncell = (size_t)nb * h8 * w8;
  OFC_LAUNCH(k_softargmax, div_up(ncell, 128), 128, 0, st, corr32, y4, ncell, flow);
  if (!grads) return;

  // ---- backward
  float* dflow = get<float>(ws, "net_dflow", ncell * 2);
  float* dout = get<float>(ws, "net_dy4", ncell * 16);
  OFC_CUDA(cudaMemsetAsync(loss, 0, sizeof(double), st));
  OFC_LAUNCH(k_loss, div_up(ncell, 128), 128, 0, st, flow, target, mask, ncell, 1.0f / (float)ncell, loss, dflow, dout);
  OFC_CUDA(cudaMemsetAsync(grads, 0, param_count() * sizeof(float), st));
  float* dsa = get<float>(ws, "net_dsa", ncell * CORR_N);
  OFC_LAUNCH(k_softargmax_bwd, div_up(ncell, 128), 128, 0, st, corr32, dflow, ncell, dsa);
  for (int l = NCONV - 1; l >= 0; l--) {
    const ConvSpec& S = SPECS[l];
    const LayerGeom& g = G[l];
    const int kp = kpad(S.cin);
    float* dW = grads + param_offset(l);
    float* db = dW + (size_t)S.cout * kp;
    uint16_t* dy16 = get<uint16_t>(ws, "net_dy16_" + std::to_string(l), g.Mpad * S.cout);
    const int lanes = 256 / S.cout;
    const unsigned nblk = div_up(g.Mpad, 64 * (size_t)lanes);
    const bool last = l == NCONV - 1;
    OFC_LAUNCH(k_act_grad, nblk, lanes * S.cout, 0, st, dout, last ? (const uint16_t*)nullptr : act[l], S.cout, g.M,
               g.Mpad, last ? 0 : S.relu, dy16, db);
    // weight gradient: per pixel batch dY^T col, then the batches summed
    const int L = (int)(g.Mpad / PCH);
    float* part = get<float>(ws, "net_wpart" + std::to_string(l), (size_t)L * S.cout * kp);
    GemmArgs a{S.cout, kp, PCH, L, dy16, S.cout, (int64_t)PCH * S.cout, col[l], kp, (int64_t)PCH * kp, part, kp,
               (int64_t)S.cout * kp, 0.f, "k_gemm_sm100_wgrad"};
    gemm_bf16(GemmKind::WgradNT, a, gws, GEMM_WS, st);
    OFC_LAUNCH(k_sum_partials, grid_for((size_t)S.cout * kp), 256, 0, st, part, L, (size_t)S.cout * kp, dW);
    if (l == 0) break;
    // input gradient: dcol = dY W, then col2im
    float* dcol = get<float>(ws, "net_dcol" + std::to_string(l), g.Mpad * kp);
    GemmArgs d{(int)g.M, kp, S.cout, 1, dy16, S.cout, 0, w16 + param_offset(l), kp, 0, dcol, kp, 0, 0.f,
               "k_gemm_sm100_dgrad"};
    gemm_bf16(GemmKind::DgradNN, d, gws, GEMM_WS, st);
    const size_t nin = (size_t)g.nimg * g.Hi * g.Wi * S.cin;
    float* dx = get<float>(ws, "net_dx" + std::to_string(l), nin);
    OFC_LAUNCH(k_col2im, grid_for(nin), 256, 0, st, dcol, g.Hi, g.Wi, S.cin, g.Ho, g.Wo, S.stride, S.dil, kp,
               (size_t)g.nimg, dx);
    if (l == 4) {
      // decoder input -> correlation volume and f1 copy -> encoder features of both images
      float* df = get<float>(ws, "net_df", (size_t)nimg * h8 * w8 * FEAT);
      OFC_LAUNCH(k_corr_bwd, div_up(ncell, 128), 128, 0, st, act[3], dx, dsa, nb, h8, w8, df);
      dout = df;
    } else {
      dout = dx;
    }
  }
}

}  // namespace

void forward(const Workspace& ws, const float* params, const uint16_t* weights16, const float* i1, const float* i2,
             int nb, int h, int w, float* flow) {
  run(ws, params, weights16, i1, i2, nb, h, w, nullptr, nullptr, flow, nullptr, nullptr);
}

void forward_backward(const Workspace& ws, const float* params, const uint16_t* weights16, const float* i1,
                      const float* i2, int nb, int h, int w, const float* target, const uint8_t* mask, float* flow,
                      float* grads, double* loss) {
  run(ws, params, weights16, i1, i2, nb, h, w, target, mask, flow, grads, loss);
}

void adam(const Workspace& ws, float* params, const float* grads, float* m, float* v, uint16_t* weights16, float lr,
          float beta1, float beta2, float eps, int step) {
  const size_t n = param_count();
  const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
  OFC_LAUNCH(k_adam, grid_for(n), 256, 0, ws.st, params, grads, m, v, n, lr, beta1, beta2, eps, c1, c2);
  OFC_LAUNCH(k_to_bf16, grid_for(n), 256, 0, ws.st, params, n, weights16);
}

void to_bf16(const Workspace& ws, const float* params, uint16_t* weights16) {
  const size_t n = param_count();
  OFC_LAUNCH(k_to_bf16, grid_for(n), 256, 0, ws.st, params, n, weights16);
}

}  // namespace net
}  // namespace ofc
