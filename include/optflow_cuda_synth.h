/*
 * optflow_cuda_synth.h -- synthetic speckle images with exactly known displacement fields, rendered on the
 * GPU. A CUDA restatement of the reference's generator (python/optflow_ref/synth.py:20-190: Gaussian blobs
 * evaluated analytically at inverse-mapped coordinates, ss x ss supersampling, 0.5 + 0.25 tanh(mean)), used
 * to make the benchmark's 2048^2 pairs; it has no counterpart in the reference's engine interface.
 */
#ifndef OPTFLOW_CUDA_SYNTH_H
#define OPTFLOW_CUDA_SYNTH_H

#include "optflow_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

/* The deformation x = c + A (X - c) + t + amp * sin(2 pi X_x / wavelength) * (sx, sy) (amp = 0: affine,
 * synth.Affine / uniform_strain). */
typedef struct ofc_field {
    double a00, a01, a10, a11; /* A */
    double cx, cy;             /* centre c */
    double tx, ty;             /* translation t */
    double amp, wavelength;    /* sinusoid along X_x */
    double sx, sy;             /* its direction */
} ofc_field;

/* Render a w x h float64 image of n blobs (centres bx, by, radii br, amplitudes ba, as synth.make_pattern draws
 * them) deformed by `field` (NULL: the reference image) with ss x ss subsamples per pixel: synth.render
 * (synth.py:150-190), the same blob rectangles and float64 arithmetic, so its images equal the reference
 * generator's to rounding. */
OFC_API int ofc_synth_render(ofc_engine* eng, const double* bx, const double* by, const double* br, const double* ba,
                             size_t n, size_t w, size_t h, int ss, const ofc_field* field, double* out, char* err,
                             size_t errlen);

/* Per-kernel device time of this engine's launches since the last call (profile mode): up to `cap` entries
 * of kernel name (NUL-terminated, names_stride bytes each), launch count and total milliseconds. Returns the
 * number of entries, or -1 on error. ofc_set_profile(eng, filter): time the launches of kernels whose name
 * contains `filter` ("" = all, NULL = off) with CUDA events on the launching stream. */
OFC_API int ofc_set_profile(ofc_engine* eng, const char* filter);
OFC_API int ofc_profile_read(ofc_engine* eng, char* names, size_t names_stride, uint64_t* counts, double* ms,
                             size_t cap);

#ifdef __cplusplus
}
#endif
#endif /* OPTFLOW_CUDA_SYNTH_H */
