// accumulate_tma.cu -- the seven per-pixel sums of an inner iteration (phaseflow.py:459-483,
// rust/crates/optflow-core/src/phaseflow.rs:1217-1401) with the response taps and the reference pack staged in
// shared memory by TMA tile copies.
//
// A block owns 32 x 8 pixels. Per filter pair j (the responses are stored in filter pairs, node-major: one 16-byte
// node holds both filters' complex values) a stage holds
//   - the response box: 48 x 16 nodes of pair j's plane around the block's tap positions (12 KB), and
//   - the reference pack tile: (re, im, gx, gy) of filters 2j and 2j + 1 at the block's 256 pixels (8 KB).
// Two stages alternate: while the block samples pair j from one, the copies of pair j + 1 land in the other, and pair
// j + 2's are issued into the first once every thread has read it. The pack copies of pairs 0 and 1 are issued at
// the start, so they land during the fixed point; the response boxes follow once the fixed point has placed the
// block's taps (the box origin is the smallest tap node less one, its x in whole 16-byte nodes).
// Pixels whose 4 x 4 taps mirror at the padded plane's border, and every pixel of a block whose taps span more than
// the box, read the responses from global memory at the gather kernel's (fine.cu) tap indices; every pixel sums the same
// values in the same order on either path, so the sums equal the gather kernel's bit for bit. A pair's arithmetic
// runs before the barrier that releases its stage; the next pair's copies are in flight meanwhile.
// Waits are bounded: a thread whose wait gives up counts a timeout, the block stops issuing copies and takes the
// global-memory path for the rest, and thread 0 waits (bounded) for copies still in flight before the block leaves.
#include <climits>

#include "kernels.cuh"
#include "tma.cuh"

namespace ofc {
namespace {

constexpr int AT_BX = 32, AT_BY = 8, AT_T = AT_BX * AT_BY;  // pixels of a block
constexpr int RB_X = 48, RB_Y = 16;                          // response box, nodes
constexpr unsigned RBOX_BYTES = RB_X * RB_Y * 16, PBOX_BYTES = 2 * AT_T * 16;
constexpr unsigned STAGE_BYTES = RBOX_BYTES + PBOX_BYTES;

struct alignas(128) Stage {
  float4 resp[RB_Y * RB_X];  // node (ry, rx) of the box: (re, im) of filter 2j, (re, im) of filter 2j + 1
  float4 pack[2][AT_T];      // (re, im, gx, gy) of filters 2j, 2j + 1 at pixel (ty, tx)
};

// the 4 x 4 taps of both filters of a pair from 16-byte nodes base[jj rs + q]
__device__ __forceinline__ void sample_pair_nodes(const float4* __restrict__ base, int rs, const float* fwx,
                                                  const float* fwy, float& b0r, float& b0i, float& b1r, float& b1i) {
  b0r = b0i = b1r = b1i = 0.f;
#pragma unroll
  for (int jj = 0; jj < 4; jj++) {
    float a0r = 0.f, a0i = 0.f, a1r = 0.f, a1i = 0.f;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const float4 cv = base[jj * rs + q];
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
}

// the same from a pair's plane Rj in global memory for the taps (ix - 1 .. ix + 2) x (iy - 1 .. iy + 2) of make_taps,
// each index mirrored into the plane (the identity inside it)
__device__ __forceinline__ void sample_pair_plane(const float4* __restrict__ Rj, int ix, int iy, int pw, int ph,
                                                  const float* fwx, const float* fwy, float& b0r, float& b0i, float& b1r,
                                                  float& b1i) {
  b0r = b0i = b1r = b1i = 0.f;
#pragma unroll
  for (int jj = 0; jj < 4; jj++) {
    const float4* row = Rj + (size_t)mirror_near(iy - 1 + jj, ph) * pw;
    float a0r = 0.f, a0i = 0.f, a1r = 0.f, a1i = 0.f;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const float4 cv = __ldg(row + mirror_near(ix - 1 + q, pw));
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
}

#ifndef ACC_TMA_MINB
#define ACC_TMA_MINB 4
#endif
__global__ void __launch_bounds__(AT_T, ACC_TMA_MINB)
    k_accumulate_tma(const __grid_constant__ CUtensorMap rmap, const __grid_constant__ CUtensorMap pmap,
                     const float4* __restrict__ ref4, const float2* __restrict__ R, int F, int ph, int pw,
                     const double* __restrict__ ux, const double* __restrict__ uy, const double* __restrict__ sx,
                     const double* __restrict__ sy, const double2* __restrict__ cs, int W, int H,
                     double* __restrict__ sums, unsigned* timeouts) {
  __shared__ Stage stg[2];
  __shared__ alignas(8) unsigned long long bar[2];
  __shared__ int s_min_x, s_max_x, s_min_y, s_max_y, s_fail;
  __shared__ int s_pend[2], s_seen[2];  // thread 0's books: copies issued, completions observed per stage
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * AT_BX + tx;
  const int x0 = blockIdx.x * AT_BX, y0 = blockIdx.y * AT_BY;
  const int x = x0 + tx, y = y0 + ty;
  const bool inside = x < W && y < H;
  const int npairs = (F + 1) >> 1;
  const uint32_t bar0 = smem_addr(&bar[0]), bar1 = smem_addr(&bar[1]);
  if (tid == 0) {
    s_pend[0] = s_pend[1] = s_seen[0] = s_seen[1] = 0;
    s_min_x = s_min_y = INT_MAX;
    s_max_x = s_max_y = INT_MIN;
    s_fail = 0;
    mbar_init(bar0, 1);
    mbar_init(bar1, 1);
    mbar_fence_init();
    // the pack tiles of pairs 0 and 1: their coordinates do not depend on the fixed point
    for (int j = 0; j < min(npairs, 2); j++) {
      const uint32_t bb = j ? bar1 : bar0;
      mbar_expect(bb, STAGE_BYTES);
      tma_load_3d(smem_addr(stg[j].pack), &pmap, 4 * x0, y0, 2 * j, bb);
      s_pend[j]++;
    }
  }
  const size_t N = (size_t)W * H;
  const size_t p = inside ? (size_t)y * W + x : 0;
  double u = 0, v = 0, px = 0, py = 0;
  if (inside) {
    u = ux[p];
    v = uy[p];
    const double tpx = x + u, tpy = y + v;
    px = tpx - sx[p];
    py = tpy - sy[p];
    // X' + s(X') = X + u(X): two fixed-point steps on the spline of s (phaseflow.py:469-472)
    for (int it = 0; it < 2; it++) {
      Taps t;
      double nx, ny;
      if (make_taps(px, py, W, H, t)) {
        const double2 sv = sample_pair(cs, W, t);
        nx = tpx - sv.x;
        ny = tpy - sv.y;
      } else {
        nx = ny = nan("");
      }
      px = nx;
      py = ny;
    }
  }
  float fwx[4], fwy[4];
  int ix = 0, iy = 0;
  bool ok = false;
  {
    Taps t{};
    ok = inside && make_taps(px + PAD, py + PAD, pw, ph, t);
#pragma unroll
    for (int k = 0; k < 4; k++) {
      fwx[k] = (float)t.wx[k];
      fwy[k] = (float)t.wy[k];
    }
    ix = t.xi[1];
    iy = t.yi[1];
  }
  // taps (ix - 1 .. ix + 2) x (iy - 1 .. iy + 2) inside the padded plane: no mirrored index
  const bool direct = ok && ix >= 1 && ix + 2 <= pw - 1 && iy >= 1 && iy + 2 <= ph - 1;
  {
    int lo_x = direct ? ix : INT_MAX, hi_x = direct ? ix : INT_MIN;
    int lo_y = direct ? iy : INT_MAX, hi_y = direct ? iy : INT_MIN;
    lo_x = __reduce_min_sync(0xffffffffu, lo_x);
    hi_x = __reduce_max_sync(0xffffffffu, hi_x);
    lo_y = __reduce_min_sync(0xffffffffu, lo_y);
    hi_y = __reduce_max_sync(0xffffffffu, hi_y);
    if (tx == 0 && lo_x <= hi_x) {
      atomicMin(&s_min_x, lo_x);
      atomicMax(&s_max_x, hi_x);
      atomicMin(&s_min_y, lo_y);
      atomicMax(&s_max_y, hi_y);
    }
  }
  __syncthreads();
  // the box: nodes [bx0, bx0 + RB_X) x [by0, by0 + RB_Y) of each pair's plane
  const int bx0 = s_min_x - 1, by0 = s_min_y - 1;
  const bool use = s_min_x <= s_max_x && s_max_x + 2 - bx0 < RB_X && s_max_y + 2 - by0 < RB_Y;
  if (tid == 0) {
    // the response boxes of pairs 0 and 1 (where the box does not hold the block's taps, a box at the plane's origin
    // completes the stage's byte count and is not read)
    for (int j = 0; j < min(npairs, 2); j++)
      tma_load_3d(smem_addr(stg[j].resp), &rmap, use ? 4 * bx0 : 0, use ? by0 : 0, j, j ? bar1 : bar0);
  }
  const int sb = (iy - 1 - by0) * RB_X + (ix - 1 - bx0);  // the first tap in the box (direct pixels)
  const size_t plane = (size_t)ph * pw;
  const float4* R4 = reinterpret_cast<const float4*>(R);
  const float fnan = __int_as_float(0x7fc00000);
  double a0 = 0, a1 = 0, a2 = 0, a3 = 0, a4 = 0, a5 = 0, a6 = 0;
  // filter k's contribution from its complex response sample b at X' (r2 of phaseflow.py:476-483)
  auto add = [&](const float4 r1, float br, float bi) {
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
  bool fail = false;  // block-uniform: a wait gave up, no copies are issued any more
  for (int j = 0; j < npairs; j++) {
    const int s = j & 1;
    const uint32_t bb = s ? bar1 : bar0;
    bool rdy = false;
    if (!fail) {
      rdy = mbar_wait(bb, (j >> 1) & 1);
      if (rdy) {
        if (tid == 0) {
          s_pend[s]--;
          s_seen[s]++;
        }
      } else {
        s_fail = 1;
        atomicAdd(timeouts, 1u);
      }
    }
    const bool two = 2 * j + 1 < F;
    float b0r = fnan, b0i = fnan, b1r = fnan, b1i = fnan;
    if (rdy && use && direct) sample_pair_nodes(stg[s].resp + sb, RB_X, fwx, fwy, b0r, b0i, b1r, b1i);
    else if (ok) sample_pair_plane(R4 + (size_t)j * plane, ix, iy, pw, ph, fwx, fwy, b0r, b0i, b1r, b1i);
    if (inside) {
      add(rdy ? stg[s].pack[0][tid] : __ldg(ref4 + (size_t)(2 * j) * N + p), b0r, b0i);
      if (two) add(rdy ? stg[s].pack[1][tid] : __ldg(ref4 + (size_t)(2 * j + 1) * N + p), b1r, b1i);
    }
    __syncthreads();  // every thread is done with stage s
    fail = fail || s_fail != 0;
    if (tid == 0 && !fail && j + 2 < npairs) {
      mbar_expect(bb, STAGE_BYTES);
      tma_load_3d(smem_addr(stg[s].pack), &pmap, 4 * x0, y0, 2 * (j + 2), bb);
      tma_load_3d(smem_addr(stg[s].resp), &rmap, use ? 4 * bx0 : 0, use ? by0 : 0, j + 2, bb);
      s_pend[s]++;
    }
  }
  if (tid == 0) {
    // copies still in flight after a wait gave up land before the block's shared memory is released
    for (int s = 0; s < 2; s++)
      while (s_pend[s] > 0 && mbar_wait(s ? bar1 : bar0, s_seen[s] & 1)) {
        s_pend[s]--;
        s_seen[s]++;
      }
  }
  if (!inside) return;
  sums[p] = a0;
  sums[N + p] = a1;
  sums[2 * N + p] = a2;
  sums[3 * N + p] = a3;
  sums[4 * N + p] = a4;
  sums[5 * N + p] = a5;
  sums[6 * N + p] = a6;
}

__device__ unsigned g_acc_timeouts;  // timed-out stage waits of launches that pass no counter of their own

}  // namespace

// mode 0: the gather kernel (fine.cu); otherwise the TMA-staged kernel where the planes allow tensor maps (the gather
// kernel where they do not). timeouts counts stage waits that gave up (a device counter; nullptr: a library-wide one).
void launch_accumulate_mode(int mode, const float4* ref4, const float2* R, int F, int ph, int pw, const double* ux,
                            const double* uy, const double* sx, const double* sy, const double2* cs, int W, int H,
                            double* sums, unsigned* timeouts, cudaStream_t st) {
  CUtensorMap rm, pm;
  const int npairs = (F + 1) / 2;
  bool tma = mode != 0 && W >= AT_BX && H >= AT_BY && F >= 2 && pw >= RB_X && ph >= RB_Y &&
             div_up(H, AT_BY) <= 65535u;
  if (tma) {
    const uint64_t rd[3] = {4ull * pw, (uint64_t)ph, (uint64_t)npairs};
    const uint64_t rs[2] = {16ull * pw, 16ull * pw * ph};
    const uint32_t rb[3] = {4 * RB_X, RB_Y, 1};
    const uint64_t pd[3] = {4ull * W, (uint64_t)H, (uint64_t)F};
    const uint64_t ps[2] = {16ull * W, 16ull * W * H};
    const uint32_t pb[3] = {4 * AT_BX, AT_BY, 2};
    tma = tma_map_f32(&rm, R, 3, rd, rs, rb) && tma_map_f32(&pm, ref4, 3, pd, ps, pb);
  }
  if (!tma) {
    launch_accumulate_gather(ref4, R, F, ph, pw, ux, uy, sx, sy, cs, W, H, sums, st);
    return;
  }
  if (!timeouts) {
    void* q = nullptr;
    OFC_CUDA(cudaGetSymbolAddress(&q, g_acc_timeouts));
    timeouts = (unsigned*)q;
  }
  dim3 g(div_up(W, AT_BX), div_up(H, AT_BY));
  OFC_LAUNCH(k_accumulate_tma, g, dim3(AT_BX, AT_BY), 0, st, rm, pm, ref4, R, F, ph, pw, ux, uy, sx, sy, cs, W, H, sums,
             timeouts);
}

// The engine's accumulate is the gather kernel. The staged form reads its taps from shared memory (long-scoreboard
// stalls per issued instruction 5.4 -> 2.1) but executes more instructions (497 M against 467 M per 2048^2 launch:
// the stage waits, the barrier, the box bookkeeping), and both forms are bound by issue and the latency of each
// pixel's dependent chain (fixed point, taps, atan2f, float64 sums), not by the tap reads: 0.681 against 0.667 ms.
void launch_accumulate(const float4* ref4, const float2* R, int F, int ph, int pw, const double* ux, const double* uy,
                       const double* sx, const double* sy, const double2* cs, int W, int H, double* sums,
                       cudaStream_t st) {
  launch_accumulate_mode(0, ref4, R, F, ph, pw, ux, uy, sx, sy, cs, W, H, sums, nullptr, st);
}

}  // namespace ofc
