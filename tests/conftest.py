"""Shared test setup: import paths, the gpu marker, golden-vector loading."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "optflow-soil_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")
# the reference's committed parity fixtures, packed by tests/golden/collect_ref_fixtures.py
_REF_FIXTURES = None


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def golden(name):
    with np.load(os.path.join(GOLDEN, name + ".npz")) as z:
        return {k: z[k] for k in z.files}


def ref_fixture(name):
    global _REF_FIXTURES
    if _REF_FIXTURES is None:
        with np.load(os.path.join(GOLDEN, "ref_fixtures.npz")) as z:
            _REF_FIXTURES = {k: z[k] for k in z.files}
    return _REF_FIXTURES[name]


def ref_meta():
    import json
    return json.loads(str(ref_fixture("meta.json")))


def rms(a, b, mask=None):
    d = np.asarray(a, np.float64) - np.asarray(b, np.float64)
    if mask is not None:
        d = d[mask]
    d = d[np.isfinite(d)]
    return float(np.sqrt(np.mean(d * d))) if d.size else 0.0


@pytest.fixture(scope="session")
def oracle():
    import oracle as o
    o.lib()
    return o
