"""The C ABI without a GPU: the library loads, exports every symbol its headers declare, holds the
reference's config defaults and validation messages, and refuses to run (no CPU fallback) without a device."""
import ctypes
import os
import re

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
    bound = set(_abi.SIGNATURES) | set(_abi.TEST_SIGNATURES) | set(_abi.SYNTH_SIGNATURES)
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
