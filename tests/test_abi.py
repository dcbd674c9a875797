"""The C ABI without a GPU: the library loads, exports every symbol its headers declare, holds the
reference's config defaults and validation messages, and refuses to run (no CPU fallback) without a device."""
import ctypes
import os
import re

import numpy as np

import pytest
import torch
from conftest import ROOT

from optflow_b200 import _abi
from optflow_b200.config import Config


def declared_symbols():
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if h.endswith(".h"):
            text = open(os.path.join(ROOT, "include", h)).read()
            names += re.findall(r"OFC_API\s+[\w\s\*]+?\b(ofc_\w+)\s*\(", text)
    return names


@pytest.fixture(scope="module")
def lib():
    return _abi.load()


def test_every_declared_symbol_is_exported(lib):
    names = declared_symbols()
    assert len(names) >= 20
    bound = (set(_abi.SIGNATURES) | set(_abi.TEST_SIGNATURES) | set(_abi.SYNTH_SIGNATURES) | set(_abi.NET_SIGNATURES)
             | set(_abi.PLAN_SIGNATURES))
    assert set(names) == bound, set(names) ^ bound
    for n in names:
        assert getattr(lib, n) is not None


def test_abi_version_and_struct_layout(lib):
    assert lib.ofc_abi_version() == _abi.OFC_ABI_VERSION
    c = _abi.OfcConfig()
    lib.ofc_config_default(ctypes.byref(c))
    d = Config()
    assert c.grid_step == d.grid_step and c.poc_win == d.poc_win and c.strain_win == d.strain_win
    assert c.n_scales == 3 and list(c.scales[:3]) == list(d.scales)
    assert (c.lam, c.bandwidth, c.dc_cut, c.sigma_w, c.sigma_s) == (d.lam, d.bandwidth, d.dc_cut, d.sigma_w, d.sigma_s)
    assert (c.outer_iters, c.inner_iters, c.shape_order) == (d.outer_iters, d.inner_iters, d.shape_order)
    assert (c.conf_min, c.edge_guard, c.phase_tol) == (d.conf_min, d.edge_guard, d.phase_tol)
    # the struct the package builds equals the library's default
    p = d.to_ofc()
    assert bytes(p) == bytes(c)


def test_guard_distances(lib):
    c = Config().to_ofc()
    assert abs(lib.ofc_edge_guard_px(ctypes.byref(c)) - Config().edge_guard_px()) < 1e-12
    assert abs(lib.ofc_auto_edge_guard_px(ctypes.byref(c)) - 12.2231) < 1e-3
    assert abs(lib.ofc_edge_guard_min_area_px(ctypes.byref(c)) - 327.68) < 1e-9


@pytest.mark.parametrize("kw,msg", [
    (dict(poc_win=48), "poc_win must be a power of two >= 16"),
    (dict(strain_win=14), "grid_step >= 1 and strain_win odd >= 5 required"),
    (dict(shape_order=3), "shape_order must be 1 or 2"),
    (dict(phase_tol=0.0), "phase_tol must be positive"),
    (dict(conf_min=1.5), "conf_min and poc_peak_min must lie in [0, 1]"),
    (dict(lam=2.0), "shortest wavelength lam*min(scales) must be >= 3 px; sigmas must be positive"),
    (dict(sigma_w=float("nan")), "sigma_w must be a finite number"),
    (dict(outer_iters=0), "n_orient, outer_iters and inner_iters must be >= 1"),
])
def test_validation_messages(lib, kw, msg):
    cfg = Config(**kw)
    with pytest.raises(ValueError) as e:
        cfg.validate()
    assert str(e.value) == msg
    c = cfg.to_ofc()
    err = ctypes.create_string_buffer(512)
    assert lib.ofc_config_validate(ctypes.byref(c), err, 512) == 1
    assert err.value.decode() == msg


@pytest.mark.skipif(torch.cuda.is_available(), reason="needs a machine without a GPU")
def test_no_device_is_an_error_not_a_fallback():
    from optflow_b200 import EngineError, Engine
    with pytest.raises(EngineError) as e:
        Engine(0)
    assert "CUDA" in str(e.value) or "device" in str(e.value)


def test_config_json_round_trip():
    c = Config(lam=7.0, scales=(0.5, 1.0), edge_guard=3.0)
    d = Config.from_json(c.to_json())
    assert d == c
    with pytest.raises(ValueError, match="unknown config keys"):
        Config.from_json('{"nope": 1}')


@pytest.mark.parametrize("kw,msg", [
    (dict(fb_max=-1), "fb_max must be >= 0"),
    (dict(fb_tol=0.0), "fb_radius must be finite and nonzero (negative: 4 sigma_w), fb_tol finite and positive"),
    (dict(fb_radius=0.0), "fb_radius must be finite and nonzero (negative: 4 sigma_w), fb_tol finite and positive"),
    (dict(fb_min_support=-1), "fb_min_support must be >= 0 and tavg in [0, 64]"),
    (dict(seq_mode="x"), "seq_mode must be 'chain' or 'hybrid', got 'x'"),
])
def test_hybrid_key_validation(kw, msg):
    """The hybrid keys' rules and messages of config.py:195-200."""
    with pytest.raises(ValueError) as e:
        Config(**kw).validate()
    assert str(e.value) == msg
    assert Config().fb_radius_px() == 16.0 and Config(fb_radius=12.0).fb_radius_px() == 12.0


def test_pixel_formats_and_save_result(tmp_path):
    """The frame formats the stream takes, and save_result's file set (io.py:203-233): float32 planes, valid as
    uint8 from ux, fb as int32 for hybrid results, timing.json."""
    import json

    from optflow_b200 import Result
    from optflow_b200.stream import pixel_format, save_result
    z = lambda *s, t=np.uint8: np.zeros(s, t)
    assert [pixel_format(a) for a in (z(4, 5), z(4, 5, 3), z(4, 5, 4), z(4, 5, t=np.uint16), z(4, 5, 3, t=np.uint16),
                                      z(4, 5, t=np.float64))] == ["gray8", "rgb24", "rgba32", "gray16", "rgb48", "f32"]
    for bad in (z(4, 5, 2), z(4, 5, t=np.int32), z(4, 5, 4, t=np.uint16)):
        with pytest.raises(ValueError, match="unsupported"):
            pixel_format(bad)
    rng = np.random.default_rng(2)
    p = lambda: rng.random((6, 7))
    ux = p()
    ux[0, 0] = np.nan
    st = {k: p() for k in ("Exx", "Eyy", "Exy", "gmax", "vol")}
    r = Result(ux, p(), p(), st, p(), p(), {"coarse": 0.1, "reference": 2}, None, np.arange(42).reshape(6, 7))
    save_result(str(tmp_path / "f1"), r, raw=True)
    names = sorted(f.name for f in (tmp_path / "f1").iterdir())
    assert names == sorted(["ux.npy", "uy.npy", "conf.npy", "Exx.npy", "Eyy.npy", "Exy.npy", "gmax.npy", "vol.npy",
                            "raw_ux.npy", "raw_uy.npy", "valid.npy", "fb.npy", "timing.json"])
    back = np.load(tmp_path / "f1" / "ux.npy")
    assert back.dtype == np.dtype("<f4") and np.array_equal(back, ux.astype(np.float32), equal_nan=True)
    assert np.load(tmp_path / "f1" / "valid.npy").tolist() == np.isfinite(ux).astype(np.uint8).tolist()
    assert np.load(tmp_path / "f1" / "fb.npy").dtype == np.dtype("<i4")
    assert json.load(open(tmp_path / "f1" / "timing.json")) == {"coarse": 0.1, "reference": 2}
