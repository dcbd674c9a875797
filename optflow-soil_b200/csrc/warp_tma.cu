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
#include <cuda.h>

#include <climits>
#include <mutex>

#include "kernels.cuh"

namespace ofc {
namespace {

constexpr int WT_X = 32, WT_Y = 16, WT_THREADS = 128;
constexpr int BOX_W = 64, BOX_H = 40;
constexpr unsigned WAIT_LIMIT = 1u << 22;

__device__ __forceinline__ bool mbar_try_wait(uint32_t addr, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(addr), "r"(parity)
      : "memory");
  return ok != 0;
}

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
  const uint32_t mbar_addr = (uint32_t)__cvta_generic_to_shared(&mbar);
  if (tid == 0) {
    const int bx0 = ((smin_x - 1) >> 2) << 2;  // a multiple of 4 floats (16 bytes), rounded towards -inf
    const int by0 = smin_y - 1;
    const int use = smin_x <= smax_x && smax_x + 2 - bx0 < BOX_W && smax_y + 2 - by0 < BOX_H;
    s_bx0 = bx0;
    s_by0 = by0;
    s_use = use;
    if (use) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar_addr), "r"(1) : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar_addr),
                   "r"((unsigned)(BOX_W * BOX_H * sizeof(float)))
                   : "memory");
      const uint32_t dst = (uint32_t)__cvta_generic_to_shared(box);
      asm volatile(
          "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
              "r"(dst),
          "l"(reinterpret_cast<uint64_t>(&tmap)), "r"(bx0), "r"(by0), "r"(mbar_addr)
          : "memory");
    }
  }
  __syncthreads();
  const bool use = s_use != 0;
  bool ready = false;
  if (use) {
    for (unsigned it = 0; it < WAIT_LIMIT && !ready; it++) ready = mbar_try_wait(mbar_addr, 0);
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
  if (use && tid == 0 && !ready) {
    // the copy may still be in flight: wait for it (bounded) before the block's shared memory is released
    bool done = false;
    for (unsigned it = 0; it < WAIT_LIMIT && !done; it++) done = mbar_try_wait(mbar_addr, 0);
  }
}

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_fn() {
  static std::once_flag once;
  static EncodeTiled fn = nullptr;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiled>(p);
    (void)cudaGetLastError();
  });
  return fn;
}

// a tensor map of the w2 x h2 float32 plane c2 with 64 x 40 boxes; false when the plane cannot have one (row pitch
// not a multiple of 16 bytes, base not 16-byte aligned, a plane smaller than the box, or no driver entry point)
bool make_tmap(const float* c2, int w2, int h2, CUtensorMap* m) {
  if (w2 % 4 != 0 || ((uintptr_t)c2 & 15) != 0 || w2 < BOX_W || h2 < BOX_H) return false;
  EncodeTiled enc = encode_fn();
  if (!enc) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)w2, (cuuint64_t)h2};
  const cuuint64_t strides[1] = {(cuuint64_t)w2 * sizeof(float)};
  const cuuint32_t boxd[2] = {BOX_W, BOX_H};
  const cuuint32_t estr[2] = {1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(c2), dims, strides, boxd, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
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
