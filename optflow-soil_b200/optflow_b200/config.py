"""Processing parameters of the pair path, with the reference's names, defaults and error messages.

Mirrors ``Config`` of python/optflow_ref/config.py:22-120 (and rust/crates/optflow-core/src/config.rs:487)
for every key the dense flow + strain path reads. The sequence, temporal-averaging and crack keys of the
reference are accepted with their defaults so that a reference config JSON loads unchanged; the engine
ignores them (they are not on the pair path) except that a non-default crack option is refused
(those run on the CPU only in the reference, rust/crates/optflow-core/src/engine.rs:82-112).
"""
import json
import math
from dataclasses import asdict, dataclass, fields

from ._abi import OFC_MAX_SCALES, OfcConfig


def _finite(v):
    return isinstance(v, (int, float)) and not isinstance(v, bool) and math.isfinite(v)


@dataclass
class Config:
    grid_step: int = 16
    poc_win: int = 64
    max_disp: float = 32.0
    poc_peak_min: float = 0.1
    median_thresh: float = 2.0
    lam: float = 8.0
    scales: tuple = (0.6, 1.0, 1.6)
    n_orient: int = 4
    bandwidth: float = 0.5
    dc_cut: float = 2.0
    sigma_w: float = 4.0
    shape_order: int = 1
    sigma_s: float = 4.0
    outer_iters: int = 8
    inner_iters: int = 2
    conf_min: float = 0.2
    edge_guard: float = -1.0
    edge_guard_min_area: float = -1.0
    phase_tol: float = 0.4
    strain_win: int = 15
    ref_update_conf: float = 0.5
    seq_mode: str = "chain"
    fb_max: int = 10
    fb_radius: float = -1.0
    fb_min_support: int = 20
    fb_tol: float = 0.5
    tavg: int = 0
    tavg_align: bool = False
    tavg_model: str = "affine"
    prewarp_freeze_at: int = 0
    crack_split: bool = False
    crack_out: bool = False
    crack_sides: bool = False
    crack_model: str = "off"

    # -- the reference's derived quantities (config.py:247-272)
    def auto_edge_guard_px(self) -> float:
        return 3.0 * self.lam * max(self.scales) / (2 * math.pi * self.bandwidth)

    def edge_guard_px(self) -> float:
        return float(self.edge_guard) if self.edge_guard >= 0 else self.auto_edge_guard_px()

    def edge_guard_min_area_px(self) -> float:
        if self.edge_guard_min_area >= 0:
            return float(self.edge_guard_min_area)
        return 2.0 * (self.lam * max(self.scales)) ** 2

    def fb_radius_px(self) -> float:
        """Config.fb_radius_px (config.py:253-255): the hybrid gate's window half-size."""
        return float(self.fb_radius) if self.fb_radius > 0 else 4.0 * self.sigma_w

    def n_filters(self) -> int:
        return self.n_orient * len(self.scales)

    def validate(self) -> None:
        """Config.validate (config.py:166-245) for the keys of the pair path; same messages."""
        if self.seq_mode not in ("chain", "hybrid"):
            raise ValueError(f"seq_mode must be 'chain' or 'hybrid', got {self.seq_mode!r}")
        if not self.scales:
            raise ValueError("scales must not be empty")
        if self.poc_win < 16 or self.poc_win & (self.poc_win - 1):
            raise ValueError("poc_win must be a power of two >= 16")
        if self.grid_step < 1 or self.strain_win < 5 or self.strain_win % 2 == 0:
            raise ValueError("grid_step >= 1 and strain_win odd >= 5 required")
        if self.dc_cut <= 0:
            raise ValueError("dc_cut must be positive")
        if self.phase_tol <= 0:
            raise ValueError("phase_tol must be positive")
        if self.shape_order not in (1, 2):
            raise ValueError("shape_order must be 1 or 2")
        if self.lam * min(self.scales) < 3 or self.sigma_w <= 0 or self.sigma_s <= 0:
            raise ValueError("shortest wavelength lam*min(scales) must be >= 3 px; sigmas must be positive")
        for name in ("max_disp", "poc_peak_min", "median_thresh", "lam", "bandwidth", "dc_cut", "sigma_w",
                     "sigma_s", "conf_min", "edge_guard", "edge_guard_min_area", "phase_tol", "ref_update_conf"):
            if not _finite(getattr(self, name)):
                raise ValueError(f"{name} must be a finite number")
        if not all(_finite(x) for x in self.scales):
            raise ValueError("scales must be finite numbers")
        if self.bandwidth <= 0 or self.max_disp <= 0 or self.median_thresh <= 0:
            raise ValueError("bandwidth, max_disp and median_thresh must be positive")
        if self.n_orient < 1 or self.outer_iters < 1 or self.inner_iters < 1:
            raise ValueError("n_orient, outer_iters and inner_iters must be >= 1")
        if not 0 <= self.conf_min <= 1 or not 0 <= self.poc_peak_min <= 1:
            raise ValueError("conf_min and poc_peak_min must lie in [0, 1]")
        if self.fb_max < 0:
            raise ValueError("fb_max must be >= 0")
        if not _finite(self.fb_radius) or not _finite(self.fb_tol) or self.fb_tol <= 0 or self.fb_radius == 0:
            raise ValueError("fb_radius must be finite and nonzero (negative: 4 sigma_w), fb_tol finite and positive")
        if self.fb_min_support < 0 or self.tavg < 0 or self.tavg > 64:
            raise ValueError("fb_min_support must be >= 0 and tavg in [0, 64]")
        if self.prewarp_freeze_at < 0:
            raise ValueError("prewarp_freeze_at must be >= 0")
        if (self.n_orient * len(self.scales) > 64 or self.sigma_w > 256 or self.sigma_s > 256
                or self.strain_win > 255 or self.poc_win > 1024):
            raise ValueError("at most 64 filters (n_orient * len(scales)); sigma_w, sigma_s <= 256, "
                             "strain_win <= 255 and poc_win <= 1024 required")
        if self.grid_step > 4096 or self.edge_guard_px() > 256:
            raise ValueError("grid_step <= 4096 and an edge guard (edge_guard, or the automatic one from lam, "
                             "scales and bandwidth) <= 256 px required")
        if len(self.scales) > OFC_MAX_SCALES:
            raise ValueError(f"the CUDA engine holds at most {OFC_MAX_SCALES} scales")
        if self.crack_split or self.crack_out or self.crack_sides or self.crack_model != "off":
            raise ValueError("the crack options run on the CPU only (use --device cpu)")

    def to_ofc(self) -> OfcConfig:
        """The POD struct the C ABI reads."""
        c = OfcConfig()
        for f in OfcConfig._fields_:
            name = f[0]
            if name == "scales":
                for i, s in enumerate(self.scales):
                    c.scales[i] = float(s)
            elif name == "n_scales":
                c.n_scales = len(self.scales)
            else:
                setattr(c, name, getattr(self, name))
        return c

    def to_json(self) -> str:
        return json.dumps(asdict(self), indent=2)

    @classmethod
    def from_json(cls, text: str) -> "Config":
        data = json.loads(text)
        if not isinstance(data, dict):
            raise ValueError("config must be a JSON object")
        known = {f.name for f in fields(cls)}
        unknown = set(data) - known
        if unknown:
            raise ValueError(f"unknown config keys: {sorted(unknown)}")
        if "scales" in data:
            data["scales"] = tuple(float(x) for x in data["scales"])
        cfg = cls(**data)
        cfg.validate()
        return cfg
