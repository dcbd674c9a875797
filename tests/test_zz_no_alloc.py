"""ofc_large_components_noalloc: the guard's large-component mask for callers that cannot allocate device
memory (a runtime whose pool allocator owns every device allocation, or an embedded host that may not grow device
memory after start-up). It must give exactly what the allocating entry point gives, on consecutive calls that
share its fixed scratch array, and refuse images larger than that array. This file sorts last so that a run that
stops at the first failure has already run every other test; it also passes alone in a fresh process."""
import ctypes

import numpy as np
import pytest

from optflow_b200 import _abi

pytestmark = pytest.mark.gpu


def _noalloc(lib, mask, min_area, stream):
    import torch
    d_mask = torch.from_numpy(np.ascontiguousarray(mask, dtype=np.uint8)).cuda()
    d_out = torch.full_like(d_mask, 7)  # stale values that the call must overwrite
    h, w = mask.shape
    err = ctypes.create_string_buffer(512)
    st = lib.ofc_large_components_noalloc(d_mask.data_ptr(), w, h, ctypes.c_double(min_area), d_out.data_ptr(),
                                          ctypes.c_void_p(stream.cuda_stream), err, 512)
    assert st == 0, err.value.decode()
    stream.synchronize()
    return d_out.cpu().numpy().astype(bool)


def test_noalloc_matches_the_allocating_entry_point_on_consecutive_calls():
    import torch
    from optflow_b200 import testing
    lib = _abi.load()
    stream = torch.cuda.Stream()
    rng = np.random.default_rng(41)
    cases = [((300, 400), 0.55, 327.68), ((512, 512), 0.45, 50.0), ((97, 1000), 0.6, 5.0)]
    for (h, w), p, area in cases:
        mask = rng.random((h, w)) < p
        want = testing.large_components(mask, area)
        for _ in range(2):  # two calls in a row on the shared scratch
            got = _noalloc(lib, mask, area, stream)
            np.testing.assert_array_equal(got, want)


def test_noalloc_tall_and_wide_images_at_the_size_limit():
    """Images taller than a grid's 65,535-row y extent, and a single row, still give the exact mask."""
    import oracle
    import torch
    from optflow_b200 import testing
    lib = _abi.load()
    stream = torch.cuda.Stream()
    rng = np.random.default_rng(43)
    for (h, w), p in [((65536, 16), 0.5), ((100000, 8), 0.6), ((1, 1 << 20), 0.7)]:
        mask = rng.random((h, w)) < p
        want = oracle.large_components(mask, 40.0)
        np.testing.assert_array_equal(testing.large_components(mask, 40.0), want)
        for _ in range(2):
            np.testing.assert_array_equal(_noalloc(lib, mask, 40.0, stream), want)


def test_noalloc_refuses_images_beyond_its_scratch():
    import torch
    lib = _abi.load()
    side = 1025  # 1025^2 > OFC_NOALLOC_MAX_PIXELS = 2^20
    d = torch.zeros((side, side), dtype=torch.uint8, device="cuda")
    err = ctypes.create_string_buffer(512)
    st = lib.ofc_large_components_noalloc(d.data_ptr(), side, side, ctypes.c_double(1.0), d.data_ptr(), None, err,
                                          512)
    assert st == 4 and "exceed" in err.value.decode()
