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

/* A straight shear band (synth.ShearBand, python/optflow_ref/synth.py:88-110, generalised): with
 * s = n . (X - e) across it (n = (-ty, tx)) and a = t . (X - e) along it, the material moves by
 * 0.5 delta (tanh(s / width) + bias) taper(a) (tx, ty); taper = 1 for length = 0 (an infinite band; bias 0 is
 * synth.ShearBand), else 0.25 (1 + tanh(a / width)) (1 + tanh((length - a) / width)) (a band of that length
 * starting at e). bias = 1 moves only the side s > 0. */
typedef struct ofc_band {
    double ex, ey;   /* a point of the centre line (the start, for a finite band) */
    double tx, ty;   /* unit vector along the band: the direction of slip */
    double delta;    /* slip */
    double width;    /* tanh width across the band and at its ends */
    double length;   /* 0: infinite */
    double bias;
} ofc_band;

#define OFC_MAX_BANDS 4

/* The deformation of the reference point X: x = c + A (X - c) + t + amp * sin(2 pi X_x / wavelength) * (sx, sy)
 * (amp = 0: affine, synth.Affine / uniform_strain), plus three optional displacement terms, each a function of X:
 *  - grid: the cubic B-spline whose coefficients sit at (gx0 + i gh, gy0 + j gh), i < gnx, j < gny (indices
 *    clamped outside), `grid` holding the x plane then the y plane (2 gnx gny doubles, row-major, host memory);
 *    a smooth random field (a Gaussian-process sample) is given this way;
 *  - a footing settlement: u_y += fs exp(-d / fdecay), d = the distance from X to the segment (fx0, fy)-(fx1, fy);
 *  - n_bands shear bands.
 * The renderer inverts x(X) by Newton steps from the affine inverse. Zero-initialise the struct: every optional
 * term is off at zero. */
typedef struct ofc_field {
    double a00, a01, a10, a11; /* A */
    double cx, cy;             /* centre c */
    double tx, ty;             /* translation t */
    double amp, wavelength;    /* sinusoid along X_x */
    double sx, sy;             /* its direction */
    const double* grid;        /* NULL: no grid term */
    int gnx, gny;
    double gx0, gy0, gh;
    double fs, fdecay, fx0, fx1, fy; /* fs = 0: no settlement */
    int n_bands;
    ofc_band bands[OFC_MAX_BANDS];
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
