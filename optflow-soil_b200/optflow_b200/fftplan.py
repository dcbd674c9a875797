"""The FFT plan table (include/optflow_cuda.h ofc_fft_tune / ofc_fft_set_plans): the factor order of each padded
length's runtime plan, chosen once by timing and kept in fft_plans.json beside this module, so that every engine of
every process builds the same plans (and so gives the same results) for a given table.

    python -m optflow_b200.fftplan tune [L ...]     time every order on the GPU and rewrite fft_plans.json

Engines install the table when the first one is created (``install``); a process may install another table before
its engines build their plans.
"""
import ctypes
import json
import os
import sys

import numpy as np

from . import _abi

TABLE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "fft_plans.json")
# the padded lengths (side + 64) of the sizes the benchmarks and the CLI's tiling meet: sides 256 .. 1536 of the
# batched pairs, 540 and 960 of 1920 x 1080 video at scale 2, the CLI's 1088 px tile windows
DEFAULT_LENGTHS = [320, 576, 604, 832, 1024, 1088, 1152, 1600]
_installed = False


def install(path=TABLE, force=False):
    """Install the plan table of `path` for this process (once, unless force)."""
    global _installed
    if _installed and not force:
        return
    _installed = True
    if not os.path.exists(path):
        return
    with open(path) as fh:
        table = json.load(fh)["plans"]
    lengths = np.array([int(k) for k in table], np.int32)
    variants = np.array([int(v) for v in table.values()], np.int32)
    st = _abi.load().ofc_fft_set_plans(lengths.ctypes.data_as(_abi.c_i32_p), variants.ctypes.data_as(_abi.c_i32_p),
                                       lengths.size)
    if st != 0:
        raise _abi.EngineError(st, f"invalid FFT plan table {path}")


def tune(lengths=None, engine=None, lines=4096):
    """{length: (fastest order, [ms per order])} timed on the engine's device."""
    from .api import default_engine
    eng = engine or default_engine()
    L = np.array(lengths or DEFAULT_LENGTHS, np.int32)
    nv = eng.lib.ofc_fft_plan_variants()
    best = np.zeros(L.size, np.int32)
    ms = np.zeros(L.size * nv, np.float32)
    eng._call("ofc_fft_tune", L.ctypes.data_as(_abi.c_i32_p), L.size, int(lines), best.ctypes.data_as(_abi.c_i32_p),
              ms.ctypes.data_as(_abi.c_float_p))
    return {int(l): (int(b), [float(x) for x in ms[i * nv:(i + 1) * nv]]) for i, (l, b) in enumerate(zip(L, best))}


def main(argv=None):
    argv = list(sys.argv[1:] if argv is None else argv)
    if not argv or argv[0] != "tune":
        print(__doc__)
        return
    res = tune([int(a) for a in argv[1:]] or None)
    out = {"plans": {str(l): b for l, (b, _) in res.items()},
           "timings_ms": {str(l): t for l, (_, t) in res.items()},
           "note": "factor order per padded length (0 radix-8 first, 1 odd radices first, 2 radix-4, 3 reversed), "
                   "fastest of 4096 forward lines each, CUDA events, median of five"}
    with open(TABLE, "w") as fh:
        json.dump(out, fh, indent=1)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
