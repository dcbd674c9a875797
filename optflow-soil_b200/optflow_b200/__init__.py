"""optflow_b200 -- B200 (sm_100a) engine for optflow-soil's dense local-phase flow + DIC pair path.

The host side mirrors the reference's Python API (python/optflow_ref/track.py, phaseflow.py, poc.py,
strain.py) over the C ABI of include/optflow_cuda.h; every computation runs in the CUDA library.
"""
from ._abi import EngineError, load  # noqa: F401
from .config import Config  # noqa: F401
from .api import (Engine, Flow, Grid, Result, coarse_flow, displacement_gradient, finish, refine,  # noqa: F401
                  refine_raw, refine_batch, strain_fields, track_pair, track_pairs, track_pair_device,
                  track_sequence, track_sequence_hybrid, local_affine_agreement)
from .stream import iter_frames, pixel_format, save_result, to_gray, track_stream  # noqa: F401,E402
