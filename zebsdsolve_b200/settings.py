"""Every option of the pipeline with its default: the drop-in keyword set of zebsdsolve's
`src/settings.zig` (Settings, settings.zig:34-402).

Front ends set options with a JSON object or keyword arguments; keys are these names, enums their
names as strings, absent keys keep their value.  An unknown key is an error, and a value the
pipeline cannot run with is rejected with the settings left as they were (settings.zig:403-461).
The speed-only options (`batch`, `tile_mb`, `refine_pixels`, `wg_fft`, `wg_refine`) are accepted
and validated as the reference does; on this engine they size device batches and tiles.  Results
do not depend on them.  `tile_mb` (the spectra one pass may hold) defaults to the reference's
largest valid value, 8192, rather than its 256: a B200 holds 180 GB, and tiles of a few thousand
patterns keep the tensor-core and slab kernels' grids full.
"""
import json
import math

ENUMS = {
    "stored_patterns": ("processed", "unprocessed"),
    "full_resolution": ("none", "scores", "refine"),
    "static_background": ("none", "average", "file"),
    "dynamic_background": ("none", "subtract", "divide"),
    "pc_vote": ("ballots", "mean"),
    "plane_kind": ("affine", "projective"),
    "plane_frame": ("nominal", "follow"),
    "plane_weights": ("equal", "information"),
    "plane_method": ("joint", "points"),
    "plane_interp": ("bilinear", "bicubic", "keys6"),
    "phase_by": ("nmi", "ncc"),
    "ipf_colors": ("classic", "hue", "perfect", "perfect_rotation"),
    "method": ("spherical", "dictionary", "pca"),
    "sweep_method": ("same", "spherical", "dictionary", "pca"),
}

# (name, default) in settings.zig's order
DEFAULTS = dict([
    ("map_rows", 0), ("map_cols", 0), ("pattern_height", 0), ("pattern_width", 0), ("stored_patterns", "processed"),
    ("scan_x_sign", -1), ("scan_y_sign", -1), ("roi_x", 0), ("roi_y", 0), ("roi_w", 0), ("roi_h", 0),
    ("toy_seed", 1), ("toy_rows", 48), ("toy_cols", 64), ("toy_grains", 24), ("toy_spread_deg", 0.0),
    ("toy_blank", 0.0), ("toy_height", 60), ("toy_width", 60), ("toy_contrast", 1.0), ("toy_background_sigma", 0.0),
    ("toy_counts", 20.0), ("toy_noise_seed", 0),
    ("detector_width_mm", 24.0),
    ("binning", 1.0), ("full_resolution", "none"),
    ("nlpar", False), ("nlpar_radius", 3), ("nlpar_iterations", 1), ("nlpar_lambda", 0.7),
    ("static_background", "average"), ("static_patterns", 1024), ("dynamic_background", "subtract"),
    ("dynamic_sigma", 0.15), ("clahe", False), ("clahe_grid", 4), ("clahe_bins", 64), ("clahe_clip", 40.0),
    ("bandpass", False), ("bp_fine", 1.0), ("bp_coarse", 8.0), ("mask", True), ("mask_radius", 1.0),
    ("pixel_angle_deg", 0.0), ("master_smooth", 0.3),
    ("bandwidth", 64),
    ("fit_bandwidth", 64), ("fit_grid", 5), ("pc_steps", 9), ("pc_span", 0.1), ("pc_steps_z", 5), ("pc_span_z", 0.06),
    ("pc_vote", "ballots"), ("pc_top_k", 12), ("pc_gate", 0.85), ("pc_kde_sigma", 0.015), ("pc_inlier_radius", 0.04),
    ("pc_nms", 0), ("pc_z_min", 0.1), ("pc_levels", 3), ("pc_shrink", 0.35),
    ("plane_kind", "affine"), ("plane_frame", "nominal"), ("plane_weights", "information"), ("plane_method", "points"),
    ("plane_stride", 2), ("plane_patterns_max", 4096), ("plane_trust", 0.05), ("plane_outlier", 4.0),
    ("plane_iters", 60), ("plane_interp", "bicubic"), ("plane_master_px", 0.0), ("plane_master_auto", True),
    ("sim_voltage_kv", 20.0), ("sim_tilt_deg", 70.0), ("sim_bin_kev", 1.0), ("sim_dmin_nm", 0.05), ("sim_halfw", 500),
    ("sim_c_strong", 20.0), ("sim_c_weak", 40.0), ("sim_c_cutoff", 200.0), ("sim_dbdiff_cutoff", 1.0), ("sim_rank", 3),
    ("sim_correct", True), ("sim_stop", 0.01),
    ("refine", True), ("refine_iters", 8), ("refine_step", 2.0),
    ("phase_by", "nmi"), ("nmi_bins", 16),
    ("ipf_colors", "perfect"),
    ("method", "spherical"), ("dict_grid", 30), ("batch", 256),
    ("tile_mb", 8192), ("refine_pixels", 64), ("wg_fft", 64), ("wg_refine", 64),
    ("sweeps", 1), ("sweep_bandwidth", 32), ("sweep_dict_grid", 20), ("sweep_method", "same"),
    ("pca_components", 256), ("pca_epochs", 2),
    ("accept_nmi", 0.0), ("accept_z", 15.0), ("accept_step_deg", 0.2),
    # this engine's own: which arithmetic the Wigner-d contraction runs in ("f32": the plain FP32
    # form on the CUDA cores; "bf16": BF16 tensor cores with FP32 accumulation, operands split
    # hi + lo for the orders l <= 16; "bf16x3": split for every order, near FP32 throughout)
    ("precision", "f32"),
])
ENUMS["precision"] = ("f32", "bf16", "bf16x3")

# the largest order l whose products keep the lo parts, per precision (None: plain FP32)
SPLIT_L = {"f32": None, "bf16": 16, "bf16x3": 1 << 20}


class SettingsError(ValueError):
    """An unknown key (UnknownSetting), a bad enum name (InvalidEnumTag) or an out-of-range value
    (BadSetting); the settings are unchanged."""


def _coerce(name, value, default):
    if name in ENUMS:
        if not isinstance(value, str) or value not in ENUMS[name]:
            raise SettingsError(f"InvalidEnumTag: {name}={value!r}")
        return value
    if isinstance(default, bool):
        if not isinstance(value, bool):
            raise SettingsError(f"InvalidType: {name} wants a boolean")
        return value
    if isinstance(default, int):
        if isinstance(value, bool) or not isinstance(value, (int, float)) or float(value) != int(value):
            raise SettingsError(f"InvalidType: {name} wants an integer")
        v = int(value)
        if v < 0 and name not in ("scan_x_sign", "scan_y_sign"):
            raise SettingsError(f"Overflow: {name}={v}")
        return v
    if isinstance(value, bool) or not isinstance(value, (int, float)):
        raise SettingsError(f"InvalidType: {name} wants a number")
    return float(value)


def _pow2(v):
    return v > 0 and (v & (v - 1)) == 0


def check(s):
    """settings.zig:427-461 — raise SettingsError(BadSetting) for a value the pipeline cannot run with."""
    bad = []

    def need(cond, what):
        if not cond:
            bad.append(what)

    need(1 <= s["binning"] <= 64, "binning")
    need(8 <= s["bandwidth"] <= 256 and 8 <= s["fit_bandwidth"] <= 256, "bandwidth")
    need(1 <= s["clahe_grid"] <= 16 and 2 <= s["clahe_bins"] <= 256 and s["clahe_clip"] > 0, "clahe")
    need(1 <= s["fit_grid"] <= 31, "fit_grid")
    need(s["detector_width_mm"] > 0, "detector_width_mm")
    need(s["plane_stride"] >= 1 and s["plane_iters"] >= 1 and s["plane_trust"] > 0 and s["plane_outlier"] >= 0, "plane")
    need(s["plane_master_px"] >= 0, "plane_master_px")
    need(1 <= s["pc_steps"] <= 65 and 1 <= s["pc_steps_z"] <= 65, "pc_steps")
    need(1 <= s["pc_levels"] <= 8, "pc_levels")
    need(s["pc_z_min"] >= 0, "pc_z_min")
    need(1 <= s["toy_rows"] <= 4096 and 1 <= s["toy_cols"] <= 4096 and s["toy_grains"] >= 1, "toy map")
    need(8 <= s["toy_height"] <= 1024 and 8 <= s["toy_width"] <= 1024, "toy pattern")
    need(s["toy_spread_deg"] >= 0 and 0 <= s["toy_blank"] <= 1 and 0 < s["toy_contrast"] <= 1 and s["toy_background_sigma"] >= 0, "toy detector")
    need(0 <= s["toy_counts"] <= 1e6, "toy_counts")
    need(1 <= s["pc_top_k"] <= 256 and 0 <= s["pc_gate"] <= 1 and 0 < s["pc_kde_sigma"] <= 1 and s["pc_inlier_radius"] > 0 and s["pc_nms"] <= 9, "pc vote")
    need(2 <= s["nmi_bins"] <= 32, "nmi_bins")
    need(1 <= s["batch"] <= 4096, "batch")
    for k in ("wg_fft", "wg_refine"):
        need(16 <= s[k] <= 256 and _pow2(s[k]), k)
    need(8 <= s["tile_mb"] <= 8192 and 8 <= s["refine_pixels"] <= 65536, "tile_mb/refine_pixels")
    need(2 <= s["dict_grid"] <= 200, "dict_grid")
    need(1 <= s["sweeps"] <= 6, "sweeps")
    need(4 <= s["pca_components"] <= 1024 and 1 <= s["pca_epochs"] <= 16, "pca")
    need(8 <= s["sweep_bandwidth"] <= 256 and 2 <= s["sweep_dict_grid"] <= 200, "sweep")
    need(s["static_patterns"] >= 1, "static_patterns")
    need(s["nlpar_radius"] >= 1 and s["nlpar_iterations"] >= 1 and s["nlpar_radius"] * s["nlpar_iterations"] <= 8 and s["nlpar_lambda"] > 0, "nlpar")
    need(abs(s["scan_x_sign"]) == 1 and abs(s["scan_y_sign"]) == 1, "scan signs")
    need(s["mask_radius"] > 0 and s["dynamic_sigma"] > 0 and s["bp_fine"] >= 0 and s["bp_coarse"] > s["bp_fine"], "filters")
    need(s["pixel_angle_deg"] >= 0 and s["master_smooth"] >= 0 and s["accept_step_deg"] > 0 and 0 <= s["accept_nmi"] <= 1, "scores")
    need(s["sim_voltage_kv"] > 0 and s["sim_bin_kev"] > 0 and s["sim_dmin_nm"] > 0 and 0 <= s["sim_tilt_deg"] <= 90, "sim")
    need(8 <= s["sim_halfw"] <= 2000 and 1 <= s["sim_rank"] <= 16, "sim size")
    need(s["sim_c_strong"] > 0 and s["sim_c_weak"] >= 0 and s["sim_c_cutoff"] >= s["sim_c_strong"] and s["sim_dbdiff_cutoff"] >= 0 and s["sim_stop"] >= 0, "sim beams")
    for v in s.values():
        if isinstance(v, float) and not math.isfinite(v):
            bad.append("non-finite value")
    if bad:
        raise SettingsError("BadSetting: " + ", ".join(bad))


class Settings:
    """The current options; `apply` is atomic (settings.zig:403-424)."""

    def __init__(self):
        self._v = dict(DEFAULTS)

    def __getitem__(self, k):
        return self._v[k]

    def __getattr__(self, k):
        try:
            return self.__dict__["_v"][k]
        except KeyError:
            raise AttributeError(k) from None

    def as_dict(self):
        return dict(self._v)

    def apply(self, overrides):
        if isinstance(overrides, (str, bytes)):
            try:
                overrides = json.loads(overrides)
            except json.JSONDecodeError as e:
                raise SettingsError(f"SyntaxError: {e}") from None
        if not isinstance(overrides, dict):
            raise SettingsError("ExpectedObject")
        nxt = dict(self._v)
        for k, v in overrides.items():
            if k not in DEFAULTS:
                raise SettingsError(f"UnknownSetting: {k}")
            nxt[k] = _coerce(k, v, DEFAULTS[k])
        check(nxt)
        self._v = nxt

    def to_json(self):
        return json.dumps({k: v for k, v in self._v.items()})

    def sweep(self, i):
        """settings.zig:465-482 — (bandwidth, dict_grid, method) of sweep i."""
        s = self._v
        if s["sweeps"] <= 1 or i + 1 >= s["sweeps"]:
            return s["bandwidth"], s["dict_grid"], s["method"]
        method = s["method"] if s["sweep_method"] == "same" else s["sweep_method"]
        f = i / (s["sweeps"] - 1)

        def between(a, b, t):
            return int(_round_half_away(a * (b / a) ** t))

        return between(s["sweep_bandwidth"], s["bandwidth"], f), between(s["sweep_dict_grid"], s["dict_grid"], f), method


def _round_half_away(x):
    return math.floor(x + 0.5) if x >= 0 else -math.floor(-x + 0.5)
