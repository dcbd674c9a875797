// proposal.cu -- the learned coarse proposal inside the pair path: the network's inputs (the pair, padded to a
// multiple of 8 by edge replication), the dense start from its 1/8-resolution flow (bilinear between the cell
// centres 8 i + 3.5), the per-tile check of the refined result, and the start field of a fallback (the POC start
// inside the failed tiles, the network's elsewhere).
#include "kernels.cuh"

namespace ofc {

__global__ void k_pad8(const float* __restrict__ in, int W, int H, int W8, int H8, float* __restrict__ out) {
  const size_t n = (size_t)W8 * H8;
  for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
    const int x = (int)(p % W8), y = (int)(p / W8);
    out[p] = in[(size_t)min(y, H - 1) * W + min(x, W - 1)];
  }
}

void launch_pad8(const float* in, int W, int H, int W8, int H8, float* out, cudaStream_t st) {
  OFC_LAUNCH(k_pad8, std::min(div_up((size_t)W8 * H8, 256), 148u * 16), 256, 0, st, in, W, H, W8, H8, out);
}

// u2 (2 planes, float64) = the cell flow (w8 x h8 x 2 floats at the centres 8 i + 3.5) bilinearly interpolated at
// every pixel, clamped to the outermost cells; copy (nullable) receives the same planes
__global__ void k_cells_to_dense(const float* __restrict__ flow, int w8, int h8, int W, int H, double* __restrict__ u2,
                                 double* __restrict__ copy) {
  const size_t N = (size_t)W * H;
  for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (size_t)gridDim.x * blockDim.x) {
    const int x = (int)(p % W), y = (int)(p / W);
    const double gx = fmin(fmax((x - 3.5) / 8.0, 0.0), (double)(w8 - 1));
    const double gy = fmin(fmax((y - 3.5) / 8.0, 0.0), (double)(h8 - 1));
    const int x0 = min((int)gx, max(w8 - 2, 0)), y0 = min((int)gy, max(h8 - 2, 0));
    const int x1 = min(x0 + 1, w8 - 1), y1 = min(y0 + 1, h8 - 1);
    const double tx = gx - x0, ty = gy - y0;
    for (int c = 0; c < 2; c++) {
      const double a = flow[((size_t)y0 * w8 + x0) * 2 + c], b = flow[((size_t)y0 * w8 + x1) * 2 + c];
      const double d = flow[((size_t)y1 * w8 + x0) * 2 + c], e = flow[((size_t)y1 * w8 + x1) * 2 + c];
      const double v = (1 - ty) * ((1 - tx) * a + tx * b) + ty * ((1 - tx) * d + tx * e);
      u2[c * N + p] = v;
      if (copy) copy[c * N + p] = v;
    }
  }
}

void launch_cells_to_dense(const float* flow, int w8, int h8, int W, int H, double* u2, double* copy, cudaStream_t st) {
  OFC_LAUNCH(k_cells_to_dense, std::min(div_up((size_t)W * H, 256), 148u * 16), 256, 0, st, flow, w8, h8, W, H, u2,
             copy);
}

// per tile of T x T pixels: the share of low-confidence pixels (conf < conf_min) among the pixels it judges (inside
// the ROI when there is one, at least B px from the image border); flags[t] = share > max_low (a tile that judges no
// pixel passes); nfail counts the failed tiles. One block of 256 threads per tile.
__global__ void k_tile_check(const double* __restrict__ conf, const uint8_t* __restrict__ roi, int W, int H, int T,
                             int B, double conf_min, double max_low, uint8_t* __restrict__ flags, int* nfail) {
  const int ntx = (W + T - 1) / T;
  const int tx = blockIdx.x % ntx, ty = blockIdx.x / ntx;
  const int x0 = tx * T, y0 = ty * T, x1 = min(x0 + T, W), y1 = min(y0 + T, H);
  int judged = 0, low = 0;
  for (int i = threadIdx.x; i < (x1 - x0) * (y1 - y0); i += blockDim.x) {
    const int x = x0 + i % (x1 - x0), y = y0 + i / (x1 - x0);
    if (x < B || y < B || x >= W - B || y >= H - B) continue;
    const size_t p = (size_t)y * W + x;
    if (roi && !roi[p]) continue;
    judged++;
    low += conf[p] < conf_min;
  }
  __shared__ int sj[32], sl[32];
  for (int o = 16; o; o >>= 1) {
    judged += __shfl_xor_sync(0xffffffff, judged, o);
    low += __shfl_xor_sync(0xffffffff, low, o);
  }
  if ((threadIdx.x & 31) == 0) {
    sj[threadIdx.x >> 5] = judged;
    sl[threadIdx.x >> 5] = low;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int j = 0, l = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); k++) {
      j += sj[k];
      l += sl[k];
    }
    const bool fail = j > 0 && (double)l > max_low * (double)j;
    flags[blockIdx.x] = fail;
    if (fail) atomicAdd(nfail, 1);
  }
}

void launch_tile_check(const double* conf, const uint8_t* roi, int W, int H, int T, int B, double conf_min,
                       double max_low, uint8_t* flags, int* nfail, cudaStream_t st) {
  const int nt = ((W + T - 1) / T) * ((H + T - 1) / T);
  OFC_CUDA(cudaMemsetAsync(nfail, 0, sizeof(int), st));
  OFC_LAUNCH(k_tile_check, nt, 256, 0, st, conf, roi, W, H, T, B, conf_min, max_low, flags, nfail);
}

// the fallback's start: the POC start (u2 on entry) inside the failed tiles, the network's start elsewhere
__global__ void k_blend_tiles(const uint8_t* __restrict__ flags, const double* __restrict__ learned, int W, int H,
                              int T, double* __restrict__ u2) {
  const size_t N = (size_t)W * H;
  const int ntx = (W + T - 1) / T;
  for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (size_t)gridDim.x * blockDim.x) {
    const int x = (int)(p % W), y = (int)(p / W);
    if (!flags[(y / T) * ntx + x / T]) {
      u2[p] = learned[p];
      u2[N + p] = learned[N + p];
    }
  }
}

void launch_blend_tiles(const uint8_t* flags, const double* learned, int W, int H, int T, double* u2, cudaStream_t st) {
  OFC_LAUNCH(k_blend_tiles, std::min(div_up((size_t)W * H, 256), 148u * 16), 256, 0, st, flags, learned, W, H, T, u2);
}

}  // namespace ofc
