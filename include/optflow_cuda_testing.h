/*
 * optflow_cuda_testing.h -- entry points into single stages of the CUDA engine, for the parity tests that
 * pin each kernel against the reference's intermediate arrays. Same conventions as optflow_cuda.h (host
 * buffers, int status, error text). None of these has a counterpart in the reference's engine interface;
 * each cites the reference function whose output it reproduces.
 */
#ifndef OPTFLOW_CUDA_TESTING_H
#define OPTFLOW_CUDA_TESTING_H

#include "optflow_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

/* `lines` complex lines of length L (interleaved re, im float32), transformed in place: numpy fft
 * (forward) or the unscaled inverse sum (inverse != 0), i.e. L * numpy ifft. */
OFC_API int ofc_test_fft_lines(ofc_engine* eng, float* data, size_t lines, size_t L, int inverse, char* err,
                               size_t errlen);

/* phaseflow.reference_phase (python/optflow_ref/phaseflow.py:100-111): per filter k (F = n_scales *
 * n_orient planes of w*h floats each) r.re, r.im, gx, gy, amp. */
OFC_API int ofc_test_reference_phase(ofc_engine* eng, const float* i1, size_t w, size_t h, const ofc_config* cfg,
                                     float* r_re, float* r_im, float* gx, float* gy, float* amp, char* err,
                                     size_t errlen);

/* bspline_coeffs(ifft2(fft2(pad(img)) * G_k)) of phaseflow.py:455-456 for every filter k: F planes of
 * (h + 64) x (w + 64) complex values (interleaved float32). */
OFC_API int ofc_test_responses(ofc_engine* eng, const float* img, size_t w, size_t h, const ofc_config* cfg,
                               float* resp, char* err, size_t errlen);

/* local_solve (phaseflow.py:177-188) on given per-pixel sums (7 planes of w*h doubles: gxx gxy gyy gxc
 * gyc gcc gw): ux, uy, energy, resid (doubles), slope (4 planes). */
OFC_API int ofc_test_local_solve(ofc_engine* eng, const double* sums, const double* ux, const double* uy, size_t w,
                                 size_t h, const ofc_config* cfg, double* oux, double* ouy, double* energy,
                                 double* resid, double* slope, char* err, size_t errlen);

/* np.median of n doubles. */
OFC_API int ofc_test_median(ofc_engine* eng, const double* v, size_t n, double* median, char* err, size_t errlen);

/* track._large_components (python/optflow_ref/track.py:45-53) of a w x h mask. */
OFC_API int ofc_test_large_components(ofc_engine* eng, const uint8_t* b, size_t w, size_t h, double min_area,
                                      uint8_t* out, char* err, size_t errlen);

/* The integer peaks of the raw POC grid of pyramid level `level` (0 = full size) of coarse_flow
 * (python/optflow_ref/poc.py:67-92, 216-239): per grid point (x, y) = the window offset round(d) plus the argmax
 * of the last shifted correlation surface evaluated there (poc.py:50) minus the half window; INT_MIN where the
 * first window already left the image. ipk holds cap ints (2 per grid point); nx, ny receive the level's grid. */
OFC_API int ofc_test_poc_peaks(ofc_engine* eng, const float* a, const float* b, size_t w, size_t h,
                               const ofc_config* cfg, int level, int32_t* ipk, size_t cap, int32_t* nx, int32_t* ny,
                               char* err, size_t errlen);

/* The trusted pre-warp fill of phaseflow.prewarp (phaseflow.py:344-354) before the blur: ux, uy (doubles),
 * slope (4 planes), low mask -> filled ux, uy. */
OFC_API int ofc_test_prewarp_fill(ofc_engine* eng, const uint8_t* low, const double* ux, const double* uy,
                                  const double* slope, size_t w, size_t h, double radius, double* oux, double* ouy,
                                  char* err, size_t errlen);

/* The seven per-pixel sums (gxx gxy gyy gxc gyc gcc gw, 7 planes of w*h doubles) of refine's first inner
 * iteration from the start field (ux, uy): pre-warp = Gaussian blur of u, warp of i2, responses, accumulate
 * (python/optflow_ref/phaseflow.py:451-483). */
OFC_API int ofc_test_first_sums(ofc_engine* eng, const float* i1, const float* i2, size_t w, size_t h, const double* ux,
                                const double* uy, const ofc_config* cfg, double* sums, char* err, size_t errlen);

/* ofc_test_first_sums with the accumulate kernel chosen: mode 0 the gather kernel, mode 1 the TMA-staged kernel
 * (the gather kernel where the planes have no tensor maps); *timeouts receives its stage waits that gave up (0 on a
 * healthy run). */
OFC_API int ofc_test_accumulate(ofc_engine* eng, const float* i1, const float* i2, size_t w, size_t h, const double* ux,
                                const double* uy, const ofc_config* cfg, int mode, double* sums, uint32_t* timeouts,
                                char* err, size_t errlen);

/* The float32 atan2 of the accumulate's phase differences (the phase of r1 conj(r2), phaseflow.py:476-483, np.angle)
 * beside CUDA's atan2f on the same n arguments: mine[i] = atan2_phase(y[i], x[i]), cuda[i] = atan2f(y[i], x[i]). */
OFC_API int ofc_test_atan2(ofc_engine* eng, const float* y, const float* x, size_t n, float* mine, float* cuda,
                           char* err, size_t errlen);

/* The warp of the pre-warp and of the temporal-averaging alignment (warp_shifted, rust/crates/optflow-core/src/
 * phaseflow.rs:1420-1439): out(x, y) = the cubic B-spline of the w2 x h2 coefficient plane c2 sampled at
 * (x + shx + sx(x, y), y + shy + sy(x, y)) for the W x H fields sx, sy (doubles); NaN where a position is NaN.
 * mode 0 runs the plain gather kernel, mode 1 the TMA-staged kernel (the gather kernel where the plane has no tensor
 * map); *timeouts receives the tiles of mode 1 whose shared-memory wait gave up (0 on a healthy run). */
OFC_API int ofc_test_warp(ofc_engine* eng, const float* c2, size_t w2, size_t h2, const double* sx, const double* sy,
                          long shx, long shy, size_t w, size_t h, int mode, float* out, uint32_t* timeouts, char* err,
                          size_t errlen);

#ifdef __cplusplus
}
#endif
#endif /* OPTFLOW_CUDA_TESTING_H */
