// warp_tma.cu -- the warp of image 2 by the smoothed field (warp_shifted, rust/crates/optflow-core/src/phaseflow.rs:
// 1420-1439; the tavg alignment's remap, rust/crates/optflow-cli/src/tavg.rs:116-210) with each output tile's source
// region staged in shared memory by one TMA tile load.
//
// A block owns a tile of 32 x 16 output pixels. Its threads form the sample positions (x + shift + s(x), float64),
// the block takes the smallest and largest tap coordinates, and one thread loads the 64 x 40 box of B-spline
// coefficients that covers them with cp.async.bulk.tensor (a 2-D tensor map of the coefficient plane; the box's x
// origin rounded down to a multiple of 4 floats, the 16-byte rule of tiled TMA copies), completed on an mbarrier.
// Every pixel whose 4 x 4 taps lie inside the image (no mirroring) samples the box; pixels whose taps mirror at the
// border, and every pixel of a tile whose taps span more than the box, sample the plane in global memory as the
// gather kernel does. Both paths run the same sampler on the same taps, so the output equals the gather kernel's bit
// for bit. Waits on the mbarrier are bounded: a thread that gives up counts a timeout and samples global memory, and
// the issuing thread waits again (bounded) before the block leaves, so no copy lands in a freed buffer.
#include <climits>

#include "kernels.cuh"
#include "tma.cuh"

namespace ofc {
namespace {

constexpr int WT_X = 32, WT_Y = 16, WT_THREADS = 128;
constexpr int BOX_W = 64, BOX_H = 40;
// the tap origin floor(clamp(p, 0, n - 1)) of make_taps
__device__ __forceinline__ int tap_floor(double p, int n) { return (int)floor(fmin(fmax(p, 0.0), (double)(n - 1))); }

__global__ void __launch_bounds__(WT_THREADS, 6) k_warp_tma(const __grid_constant__ CUtensorMap tmap,
                                                            const float* __restrict__ c2, int w2, int h2,
                                                            const double* __restrict__ sx,
                                                            const double* __restrict__ sy, long shx, long shy, int W,
                                                            int H, float* __restrict__ out, unsigned* timeouts) {
  __shared__ alignas(128) float box[BOX_H * BOX_W];
  __shared__ alignas(8) unsigned long long mbar;
  __shared__ int smin_x, smax_x, smin_y, smax_y, s_bx0, s_by0, s_use;
  const int tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;
  const int x = blockIdx.x * WT_X + tx;
  if (tid == 0) {
    smin_x = smin_y = INT_MAX;
    smax_x = smax_y = INT_MIN;
  }
  __syncthreads();
  double px[WT_Y / 4], py[WT_Y / 4];
  int lo_x = INT_MAX, hi_x = INT_MIN, lo_y = INT_MAX, hi_y = INT_MIN;
#pragma unroll
  for (int k = 0; k < WT_Y / 4; k++) {
    const int y = blockIdx.y * WT_Y + ty + 4 * k;
    px[k] = py[k] = nan("");
    if (x < W && y < H) {
      const size_t p = (size_t)y * W + x;
      px[k] = ((double)x + (double)shx) + sx[p];
      py[k] = ((double)y + (double)shy) + sy[p];
      if (px[k] == px[k] && py[k] == py[k]) {
        const int ix = tap_floor(px[k], w2), iy = tap_floor(py[k], h2);
        lo_x = min(lo_x, ix);
        hi_x = max(hi_x, ix);
        lo_y = min(lo_y, iy);
        hi_y = max(hi_y, iy);
      }
    }
  }
  // the warp's extremes by warp reductions, then one shared atomic per warp and quantity
  lo_x = __reduce_min_sync(0xffffffffu, lo_x);
  hi_x = __reduce_max_sync(0xffffffffu, hi_x);
  lo_y = __reduce_min_sync(0xffffffffu, lo_y);
  hi_y = __reduce_max_sync(0xffffffffu, hi_y);
  if (tx == 0 && lo_x <= hi_x) {
    atomicMin(&smin_x, lo_x);
    atomicMax(&smax_x, hi_x);
    atomicMin(&smin_y, lo_y);
    atomicMax(&smax_y, hi_y);
  }
  __syncthreads();
  const uint32_t mbar_addr = smem_addr(&mbar);
  if (tid == 0) {
    const int bx0 = ((smin_x - 1) >> 2) << 2;  // a multiple of 4 floats (16 bytes), rounded towards -inf
    const int by0 = smin_y - 1;
    const int use = smin_x <= smax_x && smax_x + 2 - bx0 < BOX_W && smax_y + 2 - by0 < BOX_H;
    s_bx0 = bx0;
    s_by0 = by0;
    s_use = use;
    if (use) {
      mbar_init(mbar_addr, 1);
      mbar_fence_init();
      mbar_expect(mbar_addr, (unsigned)(BOX_W * BOX_H * sizeof(float)));
      tma_load_2d(smem_addr(box), &tmap, bx0, by0, mbar_addr);
    }
  }
  __syncthreads();
  const bool use = s_use != 0;
  bool ready = false;
  if (use) {
    ready = mbar_wait(mbar_addr, 0);
    if (!ready) atomicAdd(timeouts, 1u);
  }
  const int bx0 = s_bx0, by0 = s_by0;
#pragma unroll
  for (int k = 0; k < WT_Y / 4; k++) {
    const int y = blockIdx.y * WT_Y + ty + 4 * k;
    if (x >= W || y >= H) continue;
    Taps t;
    double v;
    if (make_taps(px[k], py[k], w2, h2, t)) {
      const int ix = t.xi[1], iy = t.yi[1];
      const bool direct = t.xi[0] == ix - 1 && t.xi[3] == ix + 2 && t.yi[0] == iy - 1 && t.yi[3] == iy + 2 &&
                          ix - 1 >= 0 && ix + 2 <= w2 - 1 && iy - 1 >= 0 && iy + 2 <= h2 - 1;
      if (ready && direct) {
#pragma unroll
        for (int q = 0; q < 4; q++) {
          t.xi[q] -= bx0;
          t.yi[q] -= by0;
        }
        v = sample_real(box, BOX_W, t);
      } else {
        v = sample_real(c2, w2, t);
      }
    } else {
      v = nan("");
    }
    out[(size_t)y * W + x] = (float)v;
  }
  if (use && tid == 0 && !ready) mbar_wait(mbar_addr, 0);  // a copy still in flight lands before the block leaves
}

// a tensor map of the w2 x h2 float32 plane c2 with 64 x 40 boxes; false when the plane cannot have one (row pitch
// not a multiple of 16 bytes, base not 16-byte aligned, a plane smaller than the box, or no driver entry point)
bool make_tmap(const float* c2, int w2, int h2, CUtensorMap* m) {
  if (w2 % 4 != 0 || w2 < BOX_W || h2 < BOX_H) return false;
  const uint64_t dims[2] = {(uint64_t)w2, (uint64_t)h2};
  const uint64_t strides[1] = {(uint64_t)w2 * sizeof(float)};
  const uint32_t box[2] = {BOX_W, BOX_H};
  return tma_map_f32(m, c2, 2, dims, strides, box);
}

__device__ unsigned g_warp_timeouts;  // timed-out tile waits of launches that pass no counter of their own

}  // namespace

// mode 0: the gather kernel; otherwise the TMA-staged kernel where the plane allows a tensor map (the gather kernel
// where it does not). timeouts counts tiles whose box wait gave up (a device counter; nullptr: a library-wide one).
void launch_warp_mode(int mode, const float* c2, int w2, int h2, const double* sx, const double* sy, long shx,
                      long shy, int W, int H, float* out, unsigned* timeouts, cudaStream_t st) {
  CUtensorMap m;
  if (mode == 0 || div_up(H, WT_Y) > 65535u || !make_tmap(c2, w2, h2, &m)) {
    launch_warp_gather(c2, w2, h2, sx, sy, shx, shy, W, H, out, st);
    return;
  }
  if (!timeouts) {
    void* p = nullptr;
    OFC_CUDA(cudaGetSymbolAddress(&p, g_warp_timeouts));
    timeouts = (unsigned*)p;
  }
  dim3 g(div_up(W, WT_X), div_up(H, WT_Y));
  OFC_LAUNCH(k_warp_tma, g, WT_THREADS, 0, st, m, c2, w2, h2, sx, sy, shx, shy, W, H, out, timeouts);
}

// The engine's warp is the gather kernel: its taps hit L1 (76 % of sectors), it is bound by issue and the latency of
// its dependent float64 arithmetic, and the staged form's block reductions and barrier cost more than the box saves
// (2048^2: 93 against 113 us per launch).
void launch_warp(const float* c2, int w2, int h2, const double* sx, const double* sy, long shx, long shy, int W, int H,
                 float* out, cudaStream_t st) {
  launch_warp_mode(0, c2, w2, h2, sx, sy, shx, shy, W, H, out, nullptr, st);
}

}  // namespace ofc
