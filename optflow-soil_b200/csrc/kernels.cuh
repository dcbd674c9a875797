// kernels.cuh -- launchers of the non-FFT kernels of the engine (fine.cu, select.cu, poc.cu, finish.cu).
#pragma once
#include "common.cuh"

namespace ofc {

// ---------------------------------------------------------------- fine.cu
// separable correlation with edge replication ("nearest", scipy correlate1d) of n_planes planes at once
// (planes are contiguous W*H blocks); taps: 2r+1 doubles on the device
void launch_corr_y(const double* in, double* out, int n_planes, int W, int H, const double* taps, int r, cudaStream_t st);
void launch_corr_x(const double* in, double* out, int n_planes, int W, int H, const double* taps, int r, cudaStream_t st);
void launch_corr_y_f32in(const float* in, double* out, int W, int H, const double* taps, int r, cudaStream_t st);

// cubic B-spline coefficients (interp.py:30-35) of n_planes real planes: along y, then along x;
// in -> out (float64 or float32 storage), tmp: W*H*n_planes float64 scratch
void launch_bspline_f64(const double* in, double* out, double* tmp, int n_planes, int W, int H, cudaStream_t st);
void launch_bspline_f32(const float* in, float* out, double* tmp, int W, int H, cudaStream_t st);
// the same for the two planes of in, written interleaved (out: W H double2); tmp: 2 W H doubles
void launch_bspline_f64_pair(const double* in, double2* out, double* tmp, int W, int H, cudaStream_t st);

// warp (interp.py:72-76 with the window shift of phaseflow.rs:1420-1439): out(x, y) = spline2 at
// (x + shx + sx, y + shy + sy); spline2 is w2 x h2, out W x H
void launch_warp(const float* c2, int w2, int h2, const double* sx, const double* sy, long shx, long shy, int W, int H,
                 float* out, cudaStream_t st);
// the gather form of the warp (fine.cu); launch_warp (warp_tma.cu) stages each output tile's source region with a TMA
// tile load and falls back to this where the coefficient plane has no tensor map
void launch_warp_gather(const float* c2, int w2, int h2, const double* sx, const double* sy, long shx, long shy, int W,
                        int H, float* out, cudaStream_t st);
// the TMA-staged warp alone (mode 1) or the gather (mode 0), with the count of its timed-out tile waits
void launch_warp_mode(int mode, const float* c2, int w2, int h2, const double* sx, const double* sy, long shx,
                      long shy, int W, int H, float* out, unsigned* timeouts, cudaStream_t st);

// the seven per-pixel sums of an inner iteration (phaseflow.py:468-483); ref4: F planes W x H of the reference
// pack (r.re, r.im, gx, gy); R: the responses in filter pairs, node-major (launch_fft_rows_inv_resp); sums: 7 planes
// W x H
void launch_accumulate(const float4* ref4, const float2* R, int F, int ph, int pw, const double* ux, const double* uy,
                       const double* sx, const double* sy, const double2* cs, int W, int H, double* sums,
                       cudaStream_t st);
// the gather form (fine.cu) and the TMA-staged form (accumulate_tma.cu; mode 0: the gather form; timeouts: a device
// counter of stage waits that gave up, nullptr for a library-wide one); launch_accumulate takes the gather form
void launch_accumulate_gather(const float4* ref4, const float2* R, int F, int ph, int pw, const double* ux,
                              const double* uy, const double* sx, const double* sy, const double2* cs, int W, int H,
                              double* sums, cudaStream_t st);
void launch_accumulate_mode(int mode, const float4* ref4, const float2* R, int F, int ph, int pw, const double* ux,
                            const double* uy, const double* sx, const double* sy, const double2* cs, int W, int H,
                            double* sums, unsigned* timeouts, cudaStream_t st);

// Gaussian window moments + the per-pixel shape-function solve (phaseflow.py:114-161): mtaps: the
// window taps k(t) t^p for p = 0..4 (5 x (2r+1) doubles, device); tp: the same taps for t = 0..r as a kernel
// parameter (used by the register-blocked kernels of the default window, r = MOM_R); yplanes: scratch of ny planes
constexpr int MOM_R = 16;
struct MomTaps {
  double k[5][MOM_R + 1];  // k[p][t] = k(t) t^p
};
int moment_yplanes(int order);
void launch_moments_solve(const double* sums, const double* ux, const double* uy, int W, int H, int order,
                          const double* mtaps, int r, const MomTaps& tp, double* yplanes, double* oux, double* ouy,
                          double* energy, double* resid, double* slope, cudaStream_t st);

// min / max / NaN of the energy and whether its median is needed (stats: device struct, see fine.cu)
struct EnergyStats {
  double lo, hi;
  int nan;
  int need_median;  // set by the reduction: the reset needs it, or the caller forces it
  int skip_reset;   // every energy is above 1e-9 max + 1e-30: no pixel is reset
  double median;
  // radix-select state
  unsigned long long prefix;
  long long rank;
  long long less;
  double lo_val;
  unsigned int ticket;  // blocks of the current histogram pass that are done (the last one picks)
  unsigned int ncand;   // elements in the bucket of the first two digits (candidates of the final select)
  unsigned long long below_max;  // the largest key below that bucket
};
// unsigned long long of the median's scratch for n energies: the histogram, then up to n candidates
inline size_t median_scratch(size_t n) { return 4096 + n; }
// stats->lo/hi/nan/skip_reset of energy, and its median into stats->median (np.median) when the reset needs it
// or force_median; scratch: median_scratch(n) unsigned long long whose first 4096 are zero (they are left zero)
// primed: stats already hold a median's start state (a launch_reset with prime_next since the last median)
void launch_energy_median(const double* energy, size_t n, EnergyStats* stats, bool force_median,
                          unsigned long long* scratch, cudaStream_t st, bool primed = false);
// reset below 1e-9 median + 1e-30 (phaseflow.py:149-151,158-161); prime_next: also put the next median's start state
// into stats (its median and skip_reset stay as they are)
void launch_reset(const double* energy, const double* ux_in, const double* uy_in, int n, EnergyStats* stats,
                  double* ux, double* uy, double* resid, double* slope, cudaStream_t st, bool prime_next = false);

// confidence before the border rule (phaseflow.py:320-323) and low = conf < conf_min; with border = true
// also the border rule (phaseflow.py:297-317,508-510): conf_out (f32), low (u8), conf64 (nullable)
void launch_confidence(const double* energy, const double* resid, const double* ux, const double* uy, int W, int H,
                       const EnergyStats* stats, double phase_tol, double conf_min, bool border, double B,
                       float* conf_out, double* conf64, uint8_t* low, int* count_low, cudaStream_t st);

// trusted pre-warp (phaseflow.py:326-355): from low (u8) and the counters; writes ux_pre/uy_pre
struct PrewarpCounts {
  int low;
  int ok;
};
void launch_prewarp_fill(const uint8_t* low, const double* ux, const double* uy, const double* slope, int W, int H,
                         double R, PrewarpCounts* counts, uint8_t* ok, int* vdist, int* col_d2, int* col_row,
                         double* ux_pre, double* uy_pre, cudaStream_t st);

// bounded distance test: flag[p] |= (distance from p to the nearest src pixel <= limit) (mode 0) or
// out[p] = (distance > limit) (mode 1); vdist: W*H ints of scratch
void launch_within(const uint8_t* src, int W, int H, double limit, int mode, uint8_t* out, int* vdist, cudaStream_t st);

void launch_f64_to_f32(const double* in, float* out, size_t n, cudaStream_t st);
void launch_f32_to_f64(const float* in, double* out, size_t n, cudaStream_t st);
void launch_fill_f64(double* p, double v, size_t n, cudaStream_t st);

// ---------------------------------------------------------------- poc.cu
struct PocLevel {
  int W, H;       // level image size
  int nx, ny;     // grid
  int wy, wx;     // window
};
// downsample (poc.py:164-165) of a float64 (or float32 for level 0) image
void launch_downsample(const double* in, int W, int H, double* out, double* tmp, const double* taps, int r,
                       cudaStream_t st);
// poc_grid (poc.py:67-92): one thread block per grid point; init (nullable) ny x nx; dconst: the window's
// constants on the device (poc_const_host, poc_const_bytes() bytes)
size_t poc_const_bytes();
void poc_const_host(int wy, int wx, void* out);
void launch_poc_grid(const double* a, const double* b, const PocLevel& lv, const int* xs, const int* ys,
                     const double* iux, const double* iuy, const void* dconst, double* ux, double* uy, double* peak,
                     int* ipk, cudaStream_t st);
// clean (poc.py:95-140) in one thread block; fallback = init (nullable)
void launch_poc_clean(double* ux, double* uy, double* peak, int nx, int ny, double peak_min, double thresh,
                      const double* fbx, const double* fby, uint8_t* scratch, cudaStream_t st);
// grid_sample (poc.py:143-161) of grid g (gnx x gny at nodes gxs, gys) at points (scale*X, scale*Y) of a
// target grid (txs, tys: tnx x tny) times mult; or, with txs == nullptr, at every pixel of a tnx x tny image
void launch_grid_sample(const double* gux, const double* guy, const int* gxs, const int* gys, int gnx, int gny,
                        const int* txs, const int* tys, int tnx, int tny, double scale, double mult, double* oux,
                        double* ouy, cudaStream_t st);
// the init of the coarsest level from a dense guess: init_dense[Y sc, X sc] / sc
void launch_init_from_dense(const double* dux, const double* duy, int W, const int* xs, const int* ys, int nx, int ny,
                            int sc, double* iux, double* iuy, cudaStream_t st);
// dense start with a guess (track.py:133-137): corr = g - init at the grid points
void launch_grid_minus_dense(const double* gux, const double* guy, const double* dux, const double* duy, int W,
                             const int* xs, const int* ys, int nx, int ny, double* cux, double* cuy, cudaStream_t st);
void launch_add(double* a, const double* b, size_t n, cudaStream_t st);

// ---------------------------------------------------------------- finish.cu
// pixels of 4-connected components of b with at least min_area pixels (track.py:45-53)
void launch_large_components(const uint8_t* b, int W, int H, double min_area, int* parent, int* size, uint8_t* out,
                             cudaStream_t st);
// finish masks: bad = low | ~roi | guard | border; mx/my = NaN where bad (track.py:66-98)
void launch_finish_mask(const uint8_t* low, const uint8_t* roi, const uint8_t* big, int W, int H, double guard,
                        const double* ux, const double* uy, uint8_t* src, uint8_t* bad, int* vdist, double* mx,
                        double* my, cudaStream_t st);
// displacement_gradient + strain_fields (strain.py:61-112): outputs nullable f32 planes
void launch_strain(const double* mx, const double* my, int W, int H, int win, double* yplanes, float* dudx,
                   float* dudy, float* dvdx, float* dvdy, float* exx, float* eyy, float* exy, float* gmax, float* vol,
                   cudaStream_t st);
void launch_pair_outputs(const double* mx, const double* my, const double* rux, const double* ruy,
                         const double* conf64, int n, float* ux, float* uy, float* conf, uint8_t* valid, float* raw_ux,
                         float* raw_uy, cudaStream_t st);

// ---------------------------------------------------------------- learned coarse proposal (proposal.cu)
void launch_pad8(const float* in, int W, int H, int W8, int H8, float* out, cudaStream_t st);
void launch_cells_to_dense(const float* flow, int w8, int h8, int W, int H, double* u2, double* copy, cudaStream_t st);
void launch_tile_check(const double* conf, const uint8_t* roi, int W, int H, int T, int B, double conf_min,
                       double max_low, uint8_t* flags, int* nfail, cudaStream_t st);
void launch_blend_tiles(const uint8_t* flags, const double* learned, int W, int H, int T, double* u2, cudaStream_t st);

}  // namespace ofc
