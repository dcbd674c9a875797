"""Writes tests/golden/ref_fixtures.npz: the reference's own committed parity fixtures that the oracle is pinned to.

The arrays come unchanged from the reference checkout's ``rust/crates/optflow-core/tests/fixtures/*.npy`` (made by
its ``python/bench/make_parity_fixtures.py``) and its ``meta.json`` (stored as one JSON string under ``meta.json``).
Only the groups that tests/test_oracle.py reads are packed: interp, gabor, poc, refine, strain, edt and pair.

Run in a checkout that has the reference:
    python tests/golden/collect_ref_fixtures.py <reference checkout>     (or set OPTFLOW_REFERENCE)
"""
import glob
import json
import os
import sys

import numpy as np

GROUPS = ("interp_", "gabor_", "poc_", "refine_", "strain_", "edt_", "pair_")


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("OPTFLOW_REFERENCE")
    if not ref:
        sys.exit("usage: collect_ref_fixtures.py <reference checkout> (or set OPTFLOW_REFERENCE)")
    fx = os.path.join(ref, "rust", "crates", "optflow-core", "tests", "fixtures")
    arrays = {}
    for path in sorted(glob.glob(os.path.join(fx, "*.npy"))):
        name = os.path.basename(path)[:-4]
        if name.startswith(GROUPS):
            arrays[name] = np.load(path)
    with open(os.path.join(fx, "meta.json")) as fh:
        arrays["meta.json"] = np.array(json.dumps(json.load(fh)))
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_fixtures.npz")
    np.savez_compressed(out, **arrays)
    print(f"{out}: {len(arrays)} arrays")


if __name__ == "__main__":
    main()
