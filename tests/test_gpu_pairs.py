"""Many pairs in one call (ofc_track_pairs): every result equals the single-pair call's (ofc_track_pair, pinned to the
reference in test_gpu_parity.py) bit for bit, for pairs of uneven sizes with and without an ROI and a start field,
in any order; errors name the failing pair."""
import numpy as np
import pytest
from test_gpu_parity import _synthetic_pair

from optflow_b200 import Config, track_pair, track_pairs

pytestmark = pytest.mark.gpu

PLANES = ("ux", "uy", "conf", "raw_ux", "raw_uy", "valid")
STRAIN = ("Exx", "Eyy", "Exy", "gmax", "vol")


def _items():
    a, b = _synthetic_pair(256, 3)
    c, d = _synthetic_pair(192, 4, t=(-1.2, 0.7))
    roi = np.zeros((160, 224), bool)
    roi[20:-20, 24:-24] = True
    init = (np.full((128, 160), 2.0, np.float32), np.full((128, 160), -1.0, np.float32))
    return [
        (a[:128, :160], b[:128, :160], None, init),  # small, with a start field
        (a, b),                                       # the largest, first in the work order
        (c[:160, :], d[:160, :]),                     # 192 x 160
        (a[:160, :224], b[:160, :224], roi),          # 224 x 160 with an ROI
        (c, d),
        (a[64:, :96 + 64], b[64:, :96 + 64]),         # 160 x 192
    ]


def test_track_pairs_equals_track_pair():
    items = _items()
    cfg = Config()
    got = track_pairs(items, cfg)
    assert len(got) == len(items)
    for i, (it, r) in enumerate(zip(items, got)):
        want = track_pair(it[0], it[1], cfg, mask=it[2] if len(it) > 2 else None, init=it[3] if len(it) > 3 else None)
        for q in PLANES:
            np.testing.assert_array_equal(getattr(r, q), getattr(want, q), err_msg=f"pair {i}: {q}")
        for q in STRAIN:
            np.testing.assert_array_equal(r.strain[q], want.strain[q], err_msg=f"pair {i}: {q}")
        assert np.isfinite(r.ux).mean() > 0.2, i
    # a second call reuses the workers' buffers and graphs
    again = track_pairs(items[::-1], cfg)
    for r, w in zip(again, got[::-1]):
        np.testing.assert_array_equal(r.ux, w.ux)


def test_track_pairs_errors():
    items = _items()
    assert track_pairs([], Config()) == []
    with pytest.raises(ValueError, match="pair 1: image smaller than poc_win"):
        track_pairs([items[0], (items[0][0][:40, :40], items[0][1][:40, :40])], Config())
    with pytest.raises(ValueError, match="ROI mask shape"):
        track_pairs([(items[0][0], items[0][1], np.ones((3, 3), bool))], Config())
