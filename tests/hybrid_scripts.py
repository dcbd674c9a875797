"""Scripted legs for the hybrid sequence tests, shared by tests/golden/make_golden_hybrid.py (which runs the
reference's own track_sequence on them with its track_pair replaced, as python/tests/test_hybrid.py:38-52 does) and
tests/test_gpu_hybrid.py (which hands them to the engine as its leg source).

Frames are constants (frame k holds the value k) of 96 x 96 px; a leg i -> j has the displacement disp(i, j) and the
confidence conf(i, j), each a scalar or a 96 x 96 plane. The scenarios follow the cases of the reference's
python/tests/test_hybrid.py: a blind direct leg on a 20 x 20 patch, adjacent legs that see a static overlay or fall
0.3 px short there, reference moves forced for one frame (ref_update_conf 2.0), and the gate's radius and support.
"""
import numpy as np

H = W = 96
PATCH = (slice(30, 50), slice(30, 50))
BASE = dict(edge_guard=0.0, strain_win=5)


def frames(n):
    return [np.full((H, W), float(k)) for k in range(n)]


def _plane(v):
    return np.broadcast_to(np.asarray(v, dtype=np.float64), (H, W)).copy()


def patch_conf(low, blind):
    """0.9 everywhere, `low` on the patch for the legs blind(i, j) selects."""
    def conf(i, j):
        c = np.full((H, W), 0.9)
        if blind(i, j):
            c[PATCH] = low
        return c
    return conf


def _shift(i, j):
    return float(j - i)


def _overlay_disp(i, j):
    """Adjacent legs from frame 2 on see a static overlay on the patch (displacement 0)."""
    d = np.full((H, W), float(j - i))
    if j - i == 1 and j >= 2:
        d[PATCH] = 0.0
    return d


def _overlay_conf(i, j):
    c = np.full((H, W), 0.9)
    if i == 0 and j >= 2:
        c[PATCH] = 0.0
    elif j - i == 1:
        c[PATCH] = 0.99
    return c


def _short_disp(i, j):
    d = np.full((H, W), float(j - i))
    if i > 0 and j - i == 1:
        d[PATCH] -= 0.3
    return d


def _off_disp(i, j):
    d = np.full((H, W), float(j - i))
    if i == 3 and j >= 5:
        d[PATCH] += 1.0
    return d


def _nofb_conf(i, j):
    c = np.full((H, W), 0.9)
    if (i == 0 and j >= 3) or (i, j) in ((3, 4), (4, 5)):
        c[PATCH] = 0.0
    return c


def _toggle(n, k_on, k_off):
    """ref_update_conf per frame k = 1..n-1: 2.0 (the reference moves) for the frames after k_on up to k_off."""
    return [2.0 if k_on < k <= k_off else 0.0 for k in range(1, n)]


# name: (frames, Config keys, ref_update_conf per frame, disp(i, j), conf(i, j))
SCENARIOS = {
    "expiry": (7, dict(fb_max=3), None, _shift, patch_conf(0.0, lambda i, j: i == 0 and j >= 2)),
    "blind_adjacent": (4, {}, None, _shift, patch_conf(0.1, lambda i, j: j >= 2)),
    "low_frame": (6, {}, None, _shift, patch_conf(0.0, lambda i, j: j == 3)),
    "bridge": (6, {}, None, _shift, patch_conf(0.0, lambda i, j: i == 0 and j == 3)),
    "overlay_gate": (5, {}, None, _overlay_disp, _overlay_conf),
    "overlay_v2": (5, dict(fb_min_support=0), None, _overlay_disp, _overlay_conf),
    "short_tol": (3, {}, None, _short_disp, patch_conf(0.0, lambda i, j: i == 0 and j >= 2)),
    "short_tight": (3, dict(fb_tol=0.2), None, _short_disp, patch_conf(0.0, lambda i, j: i == 0 and j >= 2)),
    "radius3": (3, dict(fb_radius=3.0), None, _shift, patch_conf(0.0, lambda i, j: i == 0 and j >= 2)),
    "unanchored": (9, dict(fb_max=5), [0.0, 0.0, 0.0] + [2.0] * 5, _shift,
                   patch_conf(0.0, lambda i, j: i == 0 and j >= 3)),
    "recover_move": (9, dict(fb_max=6), _toggle(9, 3, 4), _shift, patch_conf(0.0, lambda i, j: i == 0 and j >= 3)),
    "no_recover": (9, dict(fb_max=4), _toggle(9, 3, 4), _off_disp, patch_conf(0.0, lambda i, j: i == 0 and j >= 3)),
    "no_recover_v2": (9, dict(fb_max=4, fb_min_support=0), _toggle(9, 3, 4), _off_disp,
                      patch_conf(0.0, lambda i, j: i == 0 and j >= 3)),
    "nofb_recover": (8, dict(fb_max=6), _toggle(8, 3, 4), _shift, _nofb_conf),
}


def config_keys(name):
    """The Config keywords of a scenario (its reference never moves unless its ref_update_conf list says so)."""
    return dict(BASE, seq_mode="hybrid", ref_update_conf=0.0, **SCENARIOS[name][1])


def ruc_list(name):
    n, _, ruc, _, _ = SCENARIOS[name]
    return [0.0] * (n - 1) if ruc is None else list(ruc)


def leg(name, i, j):
    """(raw_ux, raw_uy, conf) of the leg i -> j of a scenario, float64 planes."""
    _, _, _, disp, conf = SCENARIOS[name]
    ux = _plane(disp(i, j))
    return ux, 0.0 * ux, _plane(conf(i, j))
