"""ctypes mirror of include/optflow_cuda.h and the loader of the CUDA engine library.

The library is built in-tree (``optflow-soil_b200/lib/liboptflow_cuda.so``, see ``build.py``).
There is no fallback: if it is missing or fails to load, every call raises.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(HERE)
LIB_DIR = os.path.join(PKG_ROOT, "lib")
LIB_PATH = os.path.join(LIB_DIR, "liboptflow_cuda.so")

OFC_ABI_VERSION = 1
OFC_MAX_SCALES = 16

c_float_p = ctypes.POINTER(ctypes.c_float)
c_double_p = ctypes.POINTER(ctypes.c_double)
c_u8_p = ctypes.POINTER(ctypes.c_uint8)
c_i32_p = ctypes.POINTER(ctypes.c_int32)


class OfcConfig(ctypes.Structure):
    """struct ofc_config (include/optflow_cuda.h)."""
    _fields_ = [
        ("grid_step", ctypes.c_int32),
        ("poc_win", ctypes.c_int32),
        ("max_disp", ctypes.c_double),
        ("poc_peak_min", ctypes.c_double),
        ("median_thresh", ctypes.c_double),
        ("lam", ctypes.c_double),
        ("n_scales", ctypes.c_int32),
        ("scales", ctypes.c_double * OFC_MAX_SCALES),
        ("n_orient", ctypes.c_int32),
        ("bandwidth", ctypes.c_double),
        ("dc_cut", ctypes.c_double),
        ("sigma_w", ctypes.c_double),
        ("shape_order", ctypes.c_int32),
        ("sigma_s", ctypes.c_double),
        ("outer_iters", ctypes.c_int32),
        ("inner_iters", ctypes.c_int32),
        ("conf_min", ctypes.c_double),
        ("edge_guard", ctypes.c_double),
        ("edge_guard_min_area", ctypes.c_double),
        ("phase_tol", ctypes.c_double),
        ("strain_win", ctypes.c_int32),
        ("prewarp_freeze_at", ctypes.c_int32),
    ]


class OfcPairOut(ctypes.Structure):
    """struct ofc_pair_out (include/optflow_cuda.h)."""
    _fields_ = [
        ("ux", c_float_p),
        ("uy", c_float_p),
        ("conf", c_float_p),
        ("exx", c_float_p),
        ("eyy", c_float_p),
        ("exy", c_float_p),
        ("gmax", c_float_p),
        ("vol", c_float_p),
        ("valid", c_u8_p),
        ("raw_ux", c_float_p),
        ("raw_uy", c_float_p),
        ("timing", ctypes.c_double * 3),
    ]


class OfcWindow(ctypes.Structure):
    """ofc_window of include/optflow_cuda.h: the arguments of one refine_raw call of a batch."""
    _fields_ = [
        ("i1", c_float_p),
        ("w", ctypes.c_size_t),
        ("h", ctypes.c_size_t),
        ("i2", c_float_p),
        ("w2", ctypes.c_size_t),
        ("h2", ctypes.c_size_t),
        ("shift_x", ctypes.c_int64),
        ("shift_y", ctypes.c_int64),
        ("ux", c_float_p),
        ("uy", c_float_p),
        ("out_ux", c_double_p),
        ("out_uy", c_double_p),
        ("out_energy", c_double_p),
        ("out_resid", c_double_p),
    ]


class OfcPairIn(ctypes.Structure):
    """ofc_pair_in of include/optflow_cuda.h: one pair of a batch."""
    _fields_ = [
        ("i1", c_float_p),
        ("i2", c_float_p),
        ("w", ctypes.c_size_t),
        ("h", ctypes.c_size_t),
        ("roi", c_u8_p),
        ("init_ux", c_float_p),
        ("init_uy", c_float_p),
    ]


class OfcHybrid(ctypes.Structure):
    """ofc_hybrid of include/optflow_cuda.h: the hybrid keys of Config."""
    _fields_ = [
        ("fb_max", ctypes.c_int32),
        ("fb_radius", ctypes.c_double),
        ("fb_min_support", ctypes.c_int32),
        ("fb_tol", ctypes.c_double),
    ]


class OfcHybridFrame(ctypes.Structure):
    """ofc_hybrid_frame of include/optflow_cuda.h: the per-frame record of a hybrid run."""
    _fields_ = [
        ("reference", ctypes.c_int32),
        ("n_fb_max", ctypes.c_int32),
        ("mean_conf", ctypes.c_double),
        ("fallback_frac", ctypes.c_double),
        ("fb_gate_rejected", ctypes.c_double),
        ("reacquired", ctypes.c_double),
    ]


# ofc_leg_fn: (user, i, j, init_ux, init_uy, raw_ux, raw_uy, conf) -> 0 on success
LEG_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, c_float_p, c_float_p,
                          c_float_p, c_float_p, c_float_p)

OFC_PIX = {"f32": 0, "gray8": 1, "gray16": 2, "rgb24": 3, "rgba32": 4, "rgb48": 5}

# ofc_source_fn: (user, k, dst) -> 0 frame written, 1 no frame k, else error
SOURCE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p)
# ofc_sink_fn: (user, k, out, fb, info) -> 0 to go on
SINK_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, c_i32_p,
                           ctypes.POINTER(OfcHybridFrame))


class OfcStream(ctypes.Structure):
    """ofc_stream of include/optflow_cuda.h: a frame source, its format and a result sink."""
    _fields_ = [
        ("pixel", ctypes.c_int32),
        ("w_in", ctypes.c_size_t),
        ("h_in", ctypes.c_size_t),
        ("scale", ctypes.c_int32),
        ("hybrid", ctypes.c_int32),
        ("hy", OfcHybrid),
        ("ref_update_conf", ctypes.c_double),
        ("source", SOURCE_FN),
        ("source_user", ctypes.c_void_p),
        ("sink", SINK_FN),
        ("sink_user", ctypes.c_void_p),
        ("start", ctypes.c_int64),
        ("step", ctypes.c_int64),
        ("stop", ctypes.c_int64),
        ("tavg", ctypes.c_int32),
        ("tavg_align", ctypes.c_int32),
        ("tavg_mask", c_u8_p),
    ]


PAIR_FIELDS = ("ux", "uy", "conf", "exx", "eyy", "exy", "gmax", "vol", "valid", "raw_ux", "raw_uy")

# every symbol the header declares, with its ctypes signature (restype, argtypes)
_P = ctypes.c_void_p
_S = ctypes.c_size_t
_E = ctypes.c_char_p
SIGNATURES = {
    "ofc_abi_version": (ctypes.c_int, []),
    "ofc_config_default": (None, [ctypes.POINTER(OfcConfig)]),
    "ofc_config_validate": (ctypes.c_int, [ctypes.POINTER(OfcConfig), _E, _S]),
    "ofc_edge_guard_px": (ctypes.c_double, [ctypes.POINTER(OfcConfig)]),
    "ofc_auto_edge_guard_px": (ctypes.c_double, [ctypes.POINTER(OfcConfig)]),
    "ofc_edge_guard_min_area_px": (ctypes.c_double, [ctypes.POINTER(OfcConfig)]),
    "ofc_create": (_P, [ctypes.c_int, ctypes.c_int, _E, _S]),
    "ofc_destroy": (None, [_P]),
    "ofc_lanes": (ctypes.c_int, [_P]),
    "ofc_check_window": (ctypes.c_int, [_P, _S, _S, ctypes.POINTER(OfcConfig), _E, _S]),
    "ofc_release_caches": (None, [_P]),
    "ofc_refine_raw": (ctypes.c_int, [_P, c_float_p, _S, _S, c_float_p, _S, _S, ctypes.c_int64, ctypes.c_int64,
                                      c_float_p, c_float_p, ctypes.POINTER(OfcConfig),
                                      c_double_p, c_double_p, c_double_p, c_double_p, _E, _S]),
    "ofc_refine_batch": (ctypes.c_int, [_P, ctypes.c_void_p, _S, ctypes.POINTER(OfcConfig), _E, _S]),
    "ofc_track_sequence": (ctypes.c_int, [_P, ctypes.POINTER(c_float_p), _S, _S, _S, c_u8_p, ctypes.POINTER(OfcConfig),
                                          ctypes.c_double, ctypes.POINTER(OfcPairOut), c_i32_p, c_double_p, _E, _S]),
    "ofc_track_sequence_hybrid": (ctypes.c_int, [_P, ctypes.POINTER(c_float_p), _S, _S, _S, c_u8_p,
                                                 ctypes.POINTER(OfcConfig), c_double_p, ctypes.POINTER(OfcHybrid),
                                                 ctypes.POINTER(OfcPairOut), c_i32_p, ctypes.POINTER(OfcHybridFrame),
                                                 LEG_FN, _P, _E, _S]),
    "ofc_local_affine_agreement": (ctypes.c_int, [_P, _S, _S, c_double_p, c_double_p, c_u8_p, c_double_p, c_double_p,
                                                  ctypes.c_double, ctypes.c_int64, ctypes.c_double, c_u8_p, c_i32_p,
                                                  _E, _S]),
    "ofc_to_gray": (ctypes.c_int, [_P, ctypes.c_void_p, ctypes.c_int32, _S, _S, ctypes.c_int32, c_float_p, _E, _S]),
    "ofc_track_stream": (ctypes.c_int, [_P, ctypes.POINTER(OfcStream), c_u8_p, ctypes.POINTER(OfcConfig),
                                        ctypes.POINTER(ctypes.c_int64), _E, _S]),
    "ofc_align_to": (ctypes.c_int, [_P, c_float_p, c_float_p, _S, _S, c_u8_p, ctypes.c_int, ctypes.POINTER(OfcConfig),
                                    c_float_p, ctypes.POINTER(ctypes.c_int), _E, _S]),
    "ofc_average_window": (ctypes.c_int, [_P, ctypes.POINTER(c_float_p), _S, _S, _S, _S, ctypes.c_int, c_u8_p,
                                          ctypes.c_int, ctypes.POINTER(OfcConfig), c_float_p,
                                          ctypes.POINTER(ctypes.c_int), _E, _S]),
    "ofc_refine": (ctypes.c_int, [_P, c_float_p, c_float_p, _S, _S, c_float_p, c_float_p, ctypes.POINTER(OfcConfig),
                                  c_float_p, c_float_p, c_float_p, c_float_p, c_u8_p, _E, _S]),
    "ofc_grid_shape": (ctypes.c_int, [_S, _S, ctypes.POINTER(OfcConfig), ctypes.POINTER(_S), ctypes.POINTER(_S)]),
    "ofc_coarse_flow": (ctypes.c_int, [_P, c_float_p, c_float_p, _S, _S, c_float_p, c_float_p,
                                       ctypes.POINTER(OfcConfig), c_i32_p, c_i32_p, c_float_p, c_float_p, c_float_p,
                                       _E, _S]),
    "ofc_strain": (ctypes.c_int, [_P, c_float_p, c_float_p, _S, _S, ctypes.c_int32] + [c_float_p] * 9 + [_E, _S]),
    "ofc_finish": (ctypes.c_int, [_P, c_float_p, c_float_p, c_float_p, c_u8_p, _S, _S, ctypes.POINTER(OfcConfig),
                                  ctypes.POINTER(OfcPairOut), _E, _S]),
    "ofc_track_pairs": (ctypes.c_int, [_P, ctypes.POINTER(OfcPairIn), _S, ctypes.POINTER(OfcConfig),
                                       ctypes.POINTER(OfcPairOut), _E, _S]),
    "ofc_track_pair": (ctypes.c_int, [_P, c_float_p, c_float_p, _S, _S, c_u8_p, c_float_p, c_float_p,
                                      ctypes.POINTER(OfcConfig), ctypes.POINTER(OfcPairOut), _E, _S]),
    "ofc_track_pair_device": (ctypes.c_int, [_P, _P, _P, _S, _S, _P, _P, _P, ctypes.POINTER(OfcConfig),
                                             ctypes.POINTER(OfcPairOut), _P, _E, _S]),
    "ofc_kernel_launches": (ctypes.c_uint64, [_P]),
    "ofc_large_components_noalloc": (ctypes.c_int, [_P, _S, _S, ctypes.c_double, _P, _P, _E, _S]),
}


# include/optflow_cuda_testing.h
TEST_SIGNATURES = {
    "ofc_test_fft_lines": (ctypes.c_int, [_P, c_float_p, _S, _S, ctypes.c_int, _E, _S]),
    "ofc_test_reference_phase": (ctypes.c_int, [_P, c_float_p, _S, _S, ctypes.POINTER(OfcConfig)] + [c_float_p] * 5
                                 + [_E, _S]),
    "ofc_test_responses": (ctypes.c_int, [_P, c_float_p, _S, _S, ctypes.POINTER(OfcConfig), c_float_p, _E, _S]),
    "ofc_test_local_solve": (ctypes.c_int, [_P, c_double_p, c_double_p, c_double_p, _S, _S, ctypes.POINTER(OfcConfig)]
                             + [c_double_p] * 5 + [_E, _S]),
    "ofc_test_median": (ctypes.c_int, [_P, c_double_p, _S, c_double_p, _E, _S]),
    "ofc_test_large_components": (ctypes.c_int, [_P, c_u8_p, _S, _S, ctypes.c_double, c_u8_p, _E, _S]),
    "ofc_test_first_sums": (ctypes.c_int, [_P, c_float_p, c_float_p, _S, _S, c_double_p, c_double_p,
                                           ctypes.POINTER(OfcConfig), c_double_p, _E, _S]),
    "ofc_test_prewarp_fill": (ctypes.c_int, [_P, c_u8_p, c_double_p, c_double_p, c_double_p, _S, _S, ctypes.c_double,
                                             c_double_p, c_double_p, _E, _S]),
    "ofc_test_poc_peaks": (ctypes.c_int, [_P, c_float_p, c_float_p, _S, _S, ctypes.POINTER(OfcConfig), ctypes.c_int,
                                          c_i32_p, _S, c_i32_p, c_i32_p, _E, _S]),
    "ofc_test_accumulate": (ctypes.c_int, [_P, c_float_p, c_float_p, _S, _S, c_double_p, c_double_p,
                                           ctypes.POINTER(OfcConfig), ctypes.c_int, c_double_p,
                                           ctypes.POINTER(ctypes.c_uint32), _E, _S]),
    "ofc_test_atan2": (ctypes.c_int, [_P, c_float_p, c_float_p, _S, c_float_p, c_float_p, _E, _S]),
    "ofc_test_warp": (ctypes.c_int, [_P, c_float_p, _S, _S, c_double_p, c_double_p, ctypes.c_long, ctypes.c_long, _S,
                                     _S, ctypes.c_int, c_float_p, ctypes.POINTER(ctypes.c_uint32), _E, _S]),
}


class OfcBand(ctypes.Structure):
    """struct ofc_band (include/optflow_cuda_synth.h)."""
    _fields_ = [(n, ctypes.c_double) for n in ("ex", "ey", "tx", "ty", "delta", "width", "length", "bias")]


class OfcField(ctypes.Structure):
    """struct ofc_field (include/optflow_cuda_synth.h)."""
    _fields_ = ([(n, ctypes.c_double) for n in ("a00", "a01", "a10", "a11", "cx", "cy", "tx", "ty", "amp",
                                                 "wavelength", "sx", "sy")]
                + [("grid", c_double_p), ("gnx", ctypes.c_int), ("gny", ctypes.c_int)]
                + [(n, ctypes.c_double) for n in ("gx0", "gy0", "gh", "fs", "fdecay", "fx0", "fx1", "fy")]
                + [("n_bands", ctypes.c_int), ("bands", OfcBand * 4)])


# include/optflow_cuda_synth.h
SYNTH_SIGNATURES = {
    "ofc_synth_render": (ctypes.c_int, [_P, c_double_p, c_double_p, c_double_p, c_double_p, _S, _S, _S, ctypes.c_int,
                                        ctypes.POINTER(OfcField), c_double_p, _E, _S]),
    "ofc_set_profile": (ctypes.c_int, [_P, ctypes.c_char_p]),
    "ofc_profile_read": (ctypes.c_int, [_P, ctypes.c_char_p, _S, ctypes.POINTER(ctypes.c_uint64), c_double_p, _S]),
}


class EngineError(RuntimeError):
    """An error reported by the CUDA engine (the reference's EngineError, engine.rs:21-24)."""

    def __init__(self, status, message):
        super().__init__(message)
        self.status = status


_LIB = None


# include/optflow_cuda_net.h
NET_SIGNATURES = {
    "ofc_net_param_count": (ctypes.c_size_t, []),
    "ofc_net_create": (_P, [ctypes.c_int, _E, _S]),
    "ofc_net_destroy": (None, [_P]),
    "ofc_net_set_params": (ctypes.c_int, [_P, c_float_p, _S, _E, _S]),
    "ofc_net_get_params": (ctypes.c_int, [_P, c_float_p, _S, _E, _S]),
    "ofc_net_forward": (ctypes.c_int, [_P, _P, _P, ctypes.c_int, ctypes.c_int, ctypes.c_int, _P, _P, _E, _S]),
    "ofc_net_gradients": (ctypes.c_int, [_P, _P, _P, ctypes.c_int, ctypes.c_int, ctypes.c_int, _P, _P, _P, _P,
                                         c_double_p, _P, _E, _S]),
    "ofc_net_adam": (ctypes.c_int, [_P, _P, ctypes.c_float, _P, _E, _S]),
    "ofc_set_coarse_net": (ctypes.c_int, [_P, c_float_p, _S, ctypes.c_int, ctypes.c_double, _E, _S]),
    "ofc_coarse_net_stats": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_uint64)]),
}

# include/optflow_cuda.h: the FFT plan table
PLAN_SIGNATURES = {
    "ofc_fft_plan_variants": (ctypes.c_int, []),
    "ofc_fft_tune": (ctypes.c_int, [_P, c_i32_p, _S, ctypes.c_int, c_i32_p, c_float_p, _E, _S]),
    "ofc_fft_set_plans": (ctypes.c_int, [c_i32_p, c_i32_p, _S]),
}


def load(path=None):
    """Load the engine library once and bind every declared symbol. Raises if it is missing."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = path or os.environ.get("OPTFLOW_CUDA_LIB", LIB_PATH)
    if not os.path.exists(p):
        raise EngineError(2, f"CUDA engine library not built: {p} (run __graft_entry__.build() or "
                             f"python optflow-soil_b200/build.py)")
    lib = ctypes.CDLL(p)
    for name, (res, args) in {**SIGNATURES, **TEST_SIGNATURES, **SYNTH_SIGNATURES, **NET_SIGNATURES,
                                **PLAN_SIGNATURES}.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.ofc_abi_version() != OFC_ABI_VERSION:
        raise EngineError(2, f"ABI version mismatch: library {lib.ofc_abi_version()}, expected {OFC_ABI_VERSION}")
    if path is None:
        _LIB = lib
    return lib
