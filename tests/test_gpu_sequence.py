"""track_sequence in chain mode on the GPU (ofc_track_sequence) against the reference's own track_sequence
(tests/golden/seq.npz, written by tests/golden/make_golden_seq.py): the per-frame results with the pair bars of
test_gpu_parity.compare_pair, the reference index of every frame exactly, the leg's mean confidence within 1e-3.
Two runs: the reference stays at frame 0, and ref_update_conf = 0.995 moves it to k - 1 at frames 2 and 3."""
import numpy as np
import pytest
from conftest import golden
from test_gpu_parity import compare_pair

from optflow_b200 import Config, track_pair, track_sequence

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("tag,ruc", [("a", 0.5), ("b", 0.995)])
def test_track_sequence_golden(tag, ruc):
    g = golden("seq")
    fr, roi = list(g["frames"]), g["roi"].astype(bool)
    seen = 0
    for k, r in track_sequence(fr, Config(ref_update_conf=ruc), mask=roi):
        want = {q: g[f"{tag}{k}_{q}"] for q in ("ux", "uy", "conf", "raw_ux", "raw_uy", "Exx", "Eyy", "Exy", "gmax",
                                                  "vol")}
        compare_pair(r, want, f"seq {tag} frame {k}")
        assert r.timing["reference"] == int(g[f"{tag}{k}_ref"]), (tag, k)
        assert abs(r.timing["mean_conf"] - float(g[f"{tag}{k}_mean"])) < 1e-3, (tag, k)
        seen += 1
    assert seen == len(fr) - 1


def test_track_sequence_first_leg_is_the_pair():
    """With the reference at frame 0 and no start field, frame 1's raw field and confidence are track_pair's (the
    composition with a zero field samples the leg at the pixels themselves); the masks differ at most where the
    confidence rounded to float32 (the leg's stored confidence, as in the reference) crosses conf_min."""
    g = golden("seq")
    fr, roi = list(g["frames"]), g["roi"].astype(bool)
    k, r = next(track_sequence(fr[:2], Config(), mask=roi))
    p = track_pair(fr[0], fr[1], Config(), mask=roi)
    assert k == 1
    for q in ("conf", "raw_ux", "raw_uy"):
        np.testing.assert_array_equal(getattr(r, q), getattr(p, q), err_msg=q)
    both = np.isfinite(r.ux) & np.isfinite(p.ux)
    np.testing.assert_array_equal(r.ux[both], p.ux[both])
    assert (np.isfinite(r.ux) != np.isfinite(p.ux)).mean() < 1e-3


def test_track_sequence_arguments():
    g = golden("seq")
    fr = list(g["frames"])
    with pytest.raises(ValueError, match="no frames"):
        next(track_sequence([], Config()))
    with pytest.raises(ValueError, match="ROI mask is empty"):
        next(track_sequence(fr, Config(), mask=np.zeros(fr[0].shape, bool)))
    with pytest.raises(ValueError, match="frame 2"):
        next(track_sequence(fr[:2] + [fr[2][:64]], Config()))
    assert list(track_sequence(fr[:1], Config())) == []
