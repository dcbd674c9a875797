/*
 * optflow_cuda.h -- C ABI of the B200 (sm_100a) engine for optflow-soil's dense local-phase
 * flow + DIC pair path.
 *
 * The ABI is what a thin FFI crate (`optflow-cuda`, cargo feature `cuda`) binds to implement
 * the reference's `FineEngine` trait and the two stages the trait does not cover yet (coarse POC
 * and the finish). Every entry point is plain C: host pointers and sizes in, host pointers out,
 * an int status (0 = ok, else an error whose text is written to `err`, at most `errlen` bytes,
 * NUL-terminated). No call ever falls back to CPU code: a missing or failing device is an error,
 * like `EngineError` -> `TrackError::Engine` -> exit status 2 in the reference
 * (rust/crates/optflow-cli/src/run.rs:115-135).
 *
 * Images are row-major, `w` columns by `h` rows, pixel (x, y) at index y * w + x, values as the
 * reference's `Image<f32>` (luminance in [0, 1]). Displacements are in pixels.
 */
#ifndef OPTFLOW_CUDA_H
#define OPTFLOW_CUDA_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define OFC_API __attribute__((visibility("default")))
#else
#define OFC_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define OFC_ABI_VERSION 1
#define OFC_MAX_SCALES 16

/* Status codes. */
#define OFC_OK 0
#define OFC_ERR_ARG 1     /* invalid argument or configuration (Config::validate's messages) */
#define OFC_ERR_DEVICE 2  /* CUDA error, no device, out of device memory */
#define OFC_ERR_BUSY 3    /* more concurrent calls than lanes (GpuEngine refuses, never blocks) */
#define OFC_ERR_WINDOW 4  /* window larger than the engine accepts (check_window) */

/*
 * Every `Config` field the pair path reads, with the reference's meaning and defaults
 * (python/optflow_ref/config.py:22-120; rust/crates/optflow-core/src/config.rs:487-600).
 * Fill with ofc_config_default() and override; the engine validates it like Config::validate
 * (config.py:166-245) for the keys it holds.
 */
typedef struct ofc_config {
    /* coarse stage (POC grid) */
    int32_t grid_step;          /* 16 */
    int32_t poc_win;            /* 64, power of two >= 16 */
    double max_disp;            /* 32 px: sets the pyramid depth */
    double poc_peak_min;        /* 0.1 */
    double median_thresh;       /* 2.0 */
    /* fine stage (local phase of the Gabor bank) */
    double lam;                 /* 8 */
    int32_t n_scales;           /* 3 */
    double scales[OFC_MAX_SCALES]; /* 0.6, 1.0, 1.6 */
    int32_t n_orient;           /* 4 */
    double bandwidth;           /* 0.5 */
    double dc_cut;              /* 2.0 */
    double sigma_w;             /* 4 */
    int32_t shape_order;        /* 1 (affine, 6 unknowns) or 2 (quadratic, 12) */
    double sigma_s;             /* 4 */
    int32_t outer_iters;        /* 8 */
    int32_t inner_iters;        /* 2 */
    /* validity and strain */
    double conf_min;            /* 0.2 */
    double edge_guard;          /* -1 = automatic */
    double edge_guard_min_area; /* -1 = automatic */
    double phase_tol;           /* 0.4 rad */
    int32_t strain_win;         /* 15 */
    int32_t prewarp_freeze_at;  /* 0 = off (Rust-only key, rust/crates/optflow-core/src/prewarp.rs:79-116) */
} ofc_config;

/* Outputs of one tracked pair (track::Result, python/optflow_ref/track.py:15-31; the CLI's
 * `.npy` set, rust/crates/optflow-cli/src/io.rs:573-625). Every pointer holds w*h elements and may
 * be NULL when the caller does not want that output. */
typedef struct ofc_pair_out {
    float* ux;      /* NaN where invalid */
    float* uy;
    float* conf;    /* confidence before masking */
    float* exx;     /* Green-Lagrange strain */
    float* eyy;
    float* exy;
    float* gmax;
    float* vol;
    uint8_t* valid; /* 1 where ux is finite */
    float* raw_ux;  /* unmasked field (the init of a sequence's next frame) */
    float* raw_uy;
    double timing[3]; /* seconds: coarse, fine, strain (device time, CUDA events) */
} ofc_pair_out;

typedef struct ofc_engine ofc_engine;

/* ABI version of the loaded library (OFC_ABI_VERSION). */
OFC_API int ofc_abi_version(void);

/* Config::default() (config.py:24-120). */
OFC_API void ofc_config_default(ofc_config* cfg);

/* Config::validate() for the keys above (config.py:166-245); message text as the reference's. */
OFC_API int ofc_config_validate(const ofc_config* cfg, char* err, size_t errlen);

/* The resolved guard distances of the config (Config::edge_guard_px, auto_edge_guard_px,
 * edge_guard_min_area_px; config.py:257-272). */
OFC_API double ofc_edge_guard_px(const ofc_config* cfg);
OFC_API double ofc_auto_edge_guard_px(const ofc_config* cfg);
OFC_API double ofc_edge_guard_min_area_px(const ofc_config* cfg);

/* GpuEngine::new / with_lanes (rust/crates/optflow-gpu/src/engine.rs:94,103): an engine on CUDA
 * device `device` that accepts up to `lanes` (1 or 2) concurrent calls. NULL on error. */
OFC_API ofc_engine* ofc_create(int device, int lanes, char* err, size_t errlen);
OFC_API void ofc_destroy(ofc_engine* eng);

/* FineEngine::lanes (engine.rs:63-70). */
OFC_API int ofc_lanes(const ofc_engine* eng);

/* FineEngine::check_window (engine.rs:42-46): refuse a window the engine cannot hold. */
OFC_API int ofc_check_window(ofc_engine* eng, size_t w, size_t h, const ofc_config* cfg, char* err, size_t errlen);

/* FineEngine::release_caches (engine.rs:114-117): free plans and pooled device buffers. */
OFC_API void ofc_release_caches(ofc_engine* eng);

/*
 * FineEngine::refine_raw (rust/crates/optflow-core/src/engine.rs:32-40; contract of
 * phaseflow.rs:1441-1459): the outer/inner iterations of the fine stage on one window.
 * i1, ux, uy: w x h; i2: w2 x h2, pixel (x, y) of i1 sits at (x + shift_x, y + shift_y) in i2
 * before it is displaced (positions outside i2 clamp to its border). Outputs: RawFlow planes
 * (phaseflow.rs:1408-1414), w*h doubles each.
 */
OFC_API int ofc_refine_raw(ofc_engine* eng, const float* i1, size_t w, size_t h,
                   const float* i2, size_t w2, size_t h2, int64_t shift_x, int64_t shift_y,
                   const float* ux, const float* uy, const ofc_config* cfg,
                   double* out_ux, double* out_uy, double* out_energy, double* out_resid,
                   char* err, size_t errlen);

/*
 * The refine_raw calls of a tiling driver's windows (the tile loop of rust/crates/optflow-core/src/tile.rs:420-472
 * calls FineEngine::refine_prepared once per tile; the batch replaces that loop): window k has the arguments of
 * ofc_refine_raw. The results equal n calls of ofc_refine_raw, bit for bit. Window k + 1's inputs upload and
 * window k - 1's outputs download on a second stream while window k computes; with pinned host buffers
 * (cudaHostAlloc or cudaHostRegister) the copies overlap the compute. Any output pointer may be NULL. All
 * windows are checked before any work; the error text names the failing window.
 */
typedef struct ofc_window {
  const float* i1;     /* w x h */
  size_t w, h;
  const float* i2;     /* w2 x h2 */
  size_t w2, h2;
  int64_t shift_x, shift_y;
  const float* ux;     /* w x h */
  const float* uy;
  double* out_ux;      /* w x h each */
  double* out_uy;
  double* out_energy;
  double* out_resid;
} ofc_window;
OFC_API int ofc_refine_batch(ofc_engine* eng, const ofc_window* wins, size_t n, const ofc_config* cfg,
                     char* err, size_t errlen);

/*
 * track::track_sequence, chain mode (rust/crates/optflow-core/src/track.rs:1030-1245; python/optflow_ref/track.py:
 * 260-315): frames[0..n) (each w x h) against a moving reference. Frame k is tracked directly against the current
 * reference (coarse + fine, the previous leg's raw field as the dense start); the reference moves to frame k - 1
 * when the leg's mean confidence over the reportable ROI pixels falls below ref_update_conf (the previous leg then
 * extends the frame-0 link: its displacement is composed and its confidence min-accumulated). outs[k - 1] gets
 * frame k's result on the frame-0 grid (composed raw field, link confidence, guard and strain of the finish; timing
 * coarse / fine of the leg, strain of the finish); reference[k - 1] and mean_conf[k - 1] (nullable) the reference
 * index and the mean confidence. roi (nullable): the frame-0 ROI of the finish and of the mean. The hybrid mode is
 * ofc_track_sequence_hybrid; a frame source instead of arrays is ofc_track_stream.
 */
OFC_API int ofc_track_sequence(ofc_engine* eng, const float* const* frames, size_t n, size_t w, size_t h,
                       const uint8_t* roi, const ofc_config* cfg, double ref_update_conf, ofc_pair_out* outs,
                       int32_t* reference, double* mean_conf, char* err, size_t errlen);

/* The hybrid keys of Config (config.py:69-78; rust/crates/optflow-core/src/config.rs): fb_max >= 0 frames a pixel
 * may be carried by the adjacent leg, fb_radius (px, > 0; <= 0 means 4 sigma_w: Config.fb_radius_px), fb_min_support
 * >= 0 direct-good pixels the gate's window must hold (0 switches the gate off), fb_tol > 0 px. */
typedef struct ofc_hybrid {
    int32_t fb_max;         /* 10 */
    double fb_radius;       /* -1 */
    int32_t fb_min_support; /* 20 */
    double fb_tol;          /* 0.5 */
} ofc_hybrid;

/* Per-frame record of a hybrid run (Result.timing of track.py:498-501): the reference index, the direct leg's mean
 * confidence, the largest fallback counter, and the shares of ROI pixels valid by fallback, rejected by the
 * spatial gate, and re-acquired. */
typedef struct ofc_hybrid_frame {
    int32_t reference;
    int32_t n_fb_max;
    double mean_conf;
    double fallback_frac;
    double fb_gate_rejected;
    double reacquired;
} ofc_hybrid_frame;

/* A leg source that replaces the engine's own pair tracking (the reference's tests script legs the same way by
 * replacing track_pair, python/tests/test_hybrid.py:38-52): called on the host for the leg frames[i] -> frames[j]
 * with the dense start (init_ux/init_uy, w x h, NULL when the leg has none); writes the leg's raw field and its
 * confidence (w x h each) and returns 0, or non-zero to stop the run with OFC_ERR_ARG. */
typedef int (*ofc_leg_fn)(void* user, int32_t i, int32_t j, const float* init_ux, const float* init_uy,
                          float* raw_ux, float* raw_uy, float* conf);

/*
 * track::track_sequence with seq_mode "hybrid" (python/optflow_ref/track.py:385-503; rust/crates/optflow-core/src/
 * track/hybrid.rs:252-566): the chain's direct leg per pixel where its link confidence reaches conf_min, else the
 * adjacent leg k - 1 -> k carries the pixel for at most fb_max frames, valid only where it agrees with the local
 * affine model of the direct-good pixels (ofc_local_affine_agreement; fb_min_support > 0); pixels in fallback when
 * the reference moves are unanchored until a leg from an older reference agrees with them. ref_update_conf[k - 1]
 * is the threshold at frame k (the reference reads cfg.ref_update_conf anew at every frame). outs[k - 1] as in
 * ofc_track_sequence (conf: the link confidence, or the decayed adjacent one of a fallback pixel); fb (nullable,
 * (n - 1) x w x h) the fallback counters; info (nullable, n - 1). leg (nullable): a scripted leg source.
 */
OFC_API int ofc_track_sequence_hybrid(ofc_engine* eng, const float* const* frames, size_t n, size_t w, size_t h,
                              const uint8_t* roi, const ofc_config* cfg, const double* ref_update_conf,
                              const ofc_hybrid* hy, ofc_pair_out* outs, int32_t* fb, ofc_hybrid_frame* info,
                              ofc_leg_fn leg, void* leg_user, char* err, size_t errlen);

/* Pixel formats of frames handed to the engine (rows packed, channels interleaved): the grey levels of
 * io.py:15-29 (to_gray) and io.rs:150-256 (gray_from), the rgb24 frames ffmpeg delivers for a video
 * (video.rs:290-300, rgb_to_gray). */
#define OFC_PIX_F32 0    /* grey float32, taken as it is */
#define OFC_PIX_GRAY8 1  /* v / 255 */
#define OFC_PIX_GRAY16 2 /* v / 65535 */
#define OFC_PIX_RGB24 3  /* 0.299 R + 0.587 G + 0.114 B of v / 255, left to right */
#define OFC_PIX_RGBA32 4 /* the same, alpha ignored */
#define OFC_PIX_RGB48 5  /* the same of v / 65535 */

/*
 * to_gray + downscale + into_f32 (io.rs:44-52,258-281; io.py:15-51): the grey levels of a w x h image of `pixel`,
 * box-averaged over scale x scale blocks (scale >= 1, the remainder cropped; the block's rows summed left to right,
 * the row sums in order, / scale^2), in float64, rounded to float32. out: (w / scale) x (h / scale) values.
 */
OFC_API int ofc_to_gray(ofc_engine* eng, const void* px, int32_t pixel, size_t w, size_t h, int32_t scale,
                float* out, char* err, size_t errlen);

/* A frame source: writes frame k (w_in x h_in pixels of the stream's pixel format) to dst, page-locked memory
 * of the engine, and returns 0; 1 when the sequence has no frame k; any other value stops the run with
 * OFC_ERR_ARG. It is called for frame k + 1 while the GPU tracks frame k. */
typedef int (*ofc_source_fn)(void* user, int64_t k, void* dst);
/* A result sink: frame k's outputs (host views into page-locked memory, valid during the call; fb NULL in chain
 * mode; info's hybrid shares 0 in chain mode), called while the GPU tracks frame k + 1. Non-zero stops the run
 * with OFC_ERR_ARG. */
typedef int (*ofc_sink_fn)(void* user, int64_t k, const ofc_pair_out* out, const int32_t* fb,
                           const ofc_hybrid_frame* info);

typedef struct ofc_stream {
    int32_t pixel;          /* OFC_PIX_* of the source's frames */
    size_t w_in, h_in;      /* their size; the tracked frames are (w_in / scale) x (h_in / scale) */
    int32_t scale;          /* box downscale factor >= 1 (the CLI's --scale) */
    int32_t hybrid;         /* 0: seq_mode "chain", 1: "hybrid" */
    ofc_hybrid hy;          /* the hybrid keys (hybrid only) */
    double ref_update_conf;
    ofc_source_fn source;
    void* source_user;
    ofc_sink_fn sink;
    void* sink_user;
    /* the sampled frames (io.py:100-123, iter_frames): the raw frames start, start + step, ... < stop (stop < 0: to
     * the source's end) are the sequence's frames 0, 1, 2, ...; the source's k is the raw frame index. step >= 1. */
    int64_t start, step, stop;
    /* tavg > 0 (io.py:126-153): each sampled frame s is the mean of the downscaled raw frames s - tavg .. s + tavg,
     * clipped to the source, kept on the device; with tavg_align every window is aligned to s with the affine model
     * (tavg_mask, nullable: the fit's ROI on the tracked grid), else a window that the source's start or end makes
     * one-sided is aligned with the dense model (a frame that fails enters unaligned). */
    int32_t tavg;
    int32_t tavg_align;
    const uint8_t* tavg_mask;
} ofc_stream;

/*
 * track::track_sequence over a frame source (the CLI's `optflow seq`, run.rs / track.rs:1276-1287): frames are
 * pulled one ahead into page-locked buffers while the GPU works, converted to grey and downscaled on the GPU
 * (ofc_to_gray), tracked in chain or hybrid mode (ofc_track_sequence, ofc_track_sequence_hybrid), and each
 * frame's results go to the sink while the next frame is tracked (device staging, then a copy stream). roi
 * (nullable): on the tracked grid. *n_out (nullable): the frames delivered to the sink.
 */
OFC_API int ofc_track_stream(ofc_engine* eng, const ofc_stream* s, const uint8_t* roi, const ofc_config* cfg,
                     int64_t* n_out, char* err, size_t errlen);

/*
 * _local_affine_agreement (python/optflow_ref/track.py:331-382; rust/crates/optflow-core/src/track/hybrid.rs:
 * 146-250): per pixel an affine model u(q) = a + B (q - p), ridge 1e-3 r^2 on B, fitted to (ux, uy) of the support
 * pixels in the window of half-size r = max(1, round(radius)), in two passes (the second drops support pixels
 * whose residual against their own first-pass model exceeds 3 tol). ok = the last pass held >= min_support pixels,
 * at least 3, and |(tx, ty) - a| <= tol; n (nullable) = the number of them. All planes w x h.
 */
OFC_API int ofc_local_affine_agreement(ofc_engine* eng, size_t w, size_t h, const double* ux, const double* uy,
                               const uint8_t* support, const double* tx, const double* ty, double radius,
                               int64_t min_support, double tol, uint8_t* ok, int32_t* n, char* err, size_t errlen);

/*
 * tavg::align_to (rust/crates/optflow-cli/src/tavg.rs:116-161; python/optflow_ref/tavg.py:30-58): `other`
 * resampled onto the pixel grid of `centre` (both w x h) by the motion of the coarse POC flow centre -> other:
 * model 0, the robust affine fit (tavg.rs:81-114) to the grid points with a peak and, when mask (w x h, nullable)
 * is given, inside it; model 1 ("dense"), the coarse flow interpolated bilinearly. out = other(x + u(x)) by
 * the cubic B-spline of `other` (interp::warp). *aligned = 0 (out untouched) when no motion could be estimated
 * (fewer than 6 grid points, or a degenerate fit).
 */
OFC_API int ofc_align_to(ofc_engine* eng, const float* centre, const float* other, size_t w, size_t h,
                 const uint8_t* mask, int model, const ofc_config* cfg, float* out, int* aligned,
                 char* err, size_t errlen);

/*
 * tavg::average_window_with (rust/crates/optflow-cli/src/tavg.rs:163-210; python/optflow_ref/tavg.py:61-74):
 * the mean of frames[0..n) (each w x h) around frames[centre], summed in float64 (the others in order, then the
 * centre). align 0: plain mean; 1: every other frame aligned to the centre first (affine model, mask as in
 * ofc_align_to); 2: the same with the dense model. A frame whose alignment fails is left out, or with
 * keep_unaligned enters unaligned. *used (nullable): the frames in the mean, the centre included.
 */
OFC_API int ofc_average_window(ofc_engine* eng, const float* const* frames, size_t n, size_t centre, size_t w,
                       size_t h, int align, const uint8_t* mask, int keep_unaligned, const ofc_config* cfg,
                       float* out, int* used, char* err, size_t errlen);

/*
 * phaseflow::refine / refine_low (python/optflow_ref/phaseflow.py:427-511;
 * rust/crates/optflow-core/src/phaseflow.rs:1684-1757): refine_raw on the whole image plus the
 * confidence with its border rule. out_low (nullable) = the f64 confidence < conf_min.
 */
OFC_API int ofc_refine(ofc_engine* eng, const float* i1, const float* i2, size_t w, size_t h,
               const float* ux, const float* uy, const ofc_config* cfg,
               float* out_ux, float* out_uy, float* out_conf, float* out_resid, uint8_t* out_low,
               char* err, size_t errlen);

/* Grid of the coarse stage for a w x h image (poc.grid_points, python/optflow_ref/poc.py:61-64). */
OFC_API int ofc_grid_shape(size_t w, size_t h, const ofc_config* cfg, size_t* nx, size_t* ny);

/*
 * poc::coarse_flow (python/optflow_ref/poc.py:216-239; rust/crates/optflow-core/src/poc.rs:694-767):
 * grid displacement at full resolution. init_ux/init_uy (nullable, w x h): a dense guess.
 * Outputs: xs (nx), ys (ny), gux/guy/gpeak (ny x nx).
 */
OFC_API int ofc_coarse_flow(ofc_engine* eng, const float* a, const float* b, size_t w, size_t h,
                    const float* init_ux, const float* init_uy, const ofc_config* cfg,
                    int32_t* xs, int32_t* ys, float* gux, float* guy, float* gpeak,
                    char* err, size_t errlen);

/*
 * strain::displacement_gradient + strain_fields (python/optflow_ref/strain.py:61-112;
 * rust/crates/optflow-core/src/strain.rs:121-287): NaN-aware quadratic least-squares fit over
 * win x win windows. Any output pointer may be NULL.
 */
OFC_API int ofc_strain(ofc_engine* eng, const float* ux, const float* uy, size_t w, size_t h, int32_t win,
               float* dudx, float* dudy, float* dvdx, float* dvdy,
               float* exx, float* eyy, float* exy, float* gmax, float* vol,
               char* err, size_t errlen);

/*
 * track::_finish (python/optflow_ref/track.py:56-108; rust/crates/optflow-core/src/track.rs:224-274,
 * 330-420): low = conf < conf_min, guard band around large low components and the ROI exterior,
 * border strip, NaN mask, strain. conf is the f64 confidence rounded to f32; roi nullable.
 * out->raw_* and out->conf are copies of the inputs.
 */
OFC_API int ofc_finish(ofc_engine* eng, const float* ux, const float* uy, const float* conf, const uint8_t* roi,
               size_t w, size_t h, const ofc_config* cfg, ofc_pair_out* out, char* err, size_t errlen);

/* One pair of a batch (the arguments of ofc_track_pair). */
typedef struct ofc_pair_in {
    const float* i1;
    const float* i2;
    size_t w, h;
    const uint8_t* roi;    /* nullable */
    const float* init_ux;  /* nullable; both or neither */
    const float* init_uy;
} ofc_pair_in;

/*
 * Many independent pairs of any sizes (the CLI's pair runs, or the pairs of a sequence step) in one call: each
 * result equals ofc_track_pair's bit for bit. The pairs run on up to eight worker lanes (the environment variable
 * OFC_PAIR_WORKERS sets 1 to 16) of their own streams and buffers, the largest windows first, each lane fed by a
 * host thread of its own (its uploads, launches and copies back run beside the other lanes'; in profile mode one
 * host thread feeds them in turn), so small pairs overlap instead of leaving the GPU idle between their launches.
 * outs[i] gets pairs[i]'s results; the call returns when every pair is done.
 */
OFC_API int ofc_track_pairs(ofc_engine* eng, const ofc_pair_in* pairs, size_t n, const ofc_config* cfg,
                    ofc_pair_out* outs, char* err, size_t errlen);

/*
 * track::track_pair (python/optflow_ref/track.py:115-146; rust/crates/optflow-core/src/track.rs:
 * 567-623,765): coarse POC -> dense start -> fine stage -> finish, one pair, host buffers.
 * roi (nullable): w*h bytes, nonzero = inside. init_ux/init_uy (nullable): a dense guess.
 */
OFC_API int ofc_track_pair(ofc_engine* eng, const float* i1, const float* i2, size_t w, size_t h,
                   const uint8_t* roi, const float* init_ux, const float* init_uy,
                   const ofc_config* cfg, ofc_pair_out* out, char* err, size_t errlen);

/*
 * ofc_track_pair on device-resident buffers: every pointer (inputs and the out fields) is device
 * memory of the engine's device; the work is queued on `stream` (a cudaStream_t, NULL = the
 * engine's own stream) and the call returns once it is queued, with out->timing left zero.
 * Inputs must stay untouched until the stream reaches the end of the work. The inputs are copied
 * into the engine's own buffers and the outputs out of them on `stream`; the pair itself runs as
 * three CUDA graphs, captured on the first call for a (size, configuration, ROI and init present)
 * after one eager run, and replayed by later calls, so `stream` must not be under capture itself.
 * ofc_track_pair runs the same graphs on the engine's stream.
 */
OFC_API int ofc_track_pair_device(ofc_engine* eng, const float* d_i1, const float* d_i2, size_t w, size_t h,
                          const uint8_t* d_roi, const float* d_init_ux, const float* d_init_uy,
                          const ofc_config* cfg, ofc_pair_out* d_out, void* stream,
                          char* err, size_t errlen);

/*
 * The large-component mask of the guard (track._large_components, python/optflow_ref/track.py:45-53) for callers
 * that cannot allocate device memory (no counterpart in the reference: it exists for hosts whose device memory
 * is owned by someone else, such as a runtime whose pool allocator owns every device allocation, or an embedded
 * host that may not grow device memory after start-up). No engine: d_mask (w*h bytes, nonzero = set) and d_out (w*h bytes) are the caller's
 * device buffers on the current device, and the work is queued on `stream` (a cudaStream_t, NULL = the legacy
 * default stream); the result is valid once the stream has reached the end of it. The call allocates nothing:
 * its union-find scratch is a fixed device array of 2 * OFC_NOALLOC_MAX_PIXELS ints (8 MiB) that every device
 * loading this library holds until exit, so w * h must not exceed OFC_NOALLOC_MAX_PIXELS (error OFC_ERR_WINDOW).
 * The first call on a device looks the array's device address up and should come before any stream capture.
 * Every call shares the one array: calls whose work overlaps on the GPU (two streams, or two host threads) race
 * and give wrong masks; keep them ordered on one stream.
 */
#define OFC_NOALLOC_MAX_PIXELS (1u << 20)
OFC_API int ofc_large_components_noalloc(const uint8_t* d_mask, size_t w, size_t h, double min_area, uint8_t* d_out,
                                         void* stream, char* err, size_t errlen);

/* Number of this library's kernels launched by this engine since it was created (the kernels
 * are all hand-written; no library kernel runs on the path). */
OFC_API uint64_t ofc_kernel_launches(const ofc_engine* eng);

/* FFT plan autotuner (no counterpart in the reference, whose Metal engine orders a length's factors by a fixed rule,
 * rust/crates/optflow-gpu/src/fft.rs:190 factorise). A padded length's runtime plan can take one of
 * ofc_fft_plan_variants() factor orders; the transform is the same, its speed and float32 rounding differ.
 * ofc_fft_tune times every order of each length on `lines` lines on the engine's device (CUDA events, median of
 * five) and returns the fastest order per length (best) and the times (ms: n x variants, INFINITY where an order
 * does not exist). ofc_fft_set_plans installs a plan table for the process: plans that engines build afterwards take
 * the table's order (a plan already built keeps its own), so results are reproducible for a given table. 2112 (the
 * padded length of 2048-wide images) runs on a compile-time plan and is not tuned. */
OFC_API int ofc_fft_plan_variants(void);
OFC_API int ofc_fft_tune(ofc_engine* eng, const int32_t* lengths, size_t n, int lines, int32_t* best, float* ms,
                         char* err, size_t errlen);
OFC_API int ofc_fft_set_plans(const int32_t* lengths, const int32_t* variants, size_t n);

#ifdef __cplusplus
}
#endif
#endif /* OPTFLOW_CUDA_H */
