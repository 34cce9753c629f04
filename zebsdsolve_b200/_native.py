"""ctypes bindings to libzebsdsolve_b200.so, the C ABI of include/zebsdsolve_b200.h.

The library is built in place (python -m zebsdsolve_b200.build). There is no fallback: when it
is missing, or no CUDA device is present, loading raises NativeError.
"""
import ctypes
import os
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_NAME = "libzebsdsolve_b200.so"

c_int, c_uint, c_float, c_double, c_size_t, c_void_p, c_char_p, c_longlong = (
    ctypes.c_int, ctypes.c_uint, ctypes.c_float, ctypes.c_double, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_char_p,
    ctypes.c_longlong)


class NativeError(RuntimeError):
    """A library call failed (the message is the library's) or the library cannot be used."""


class Frame(ctypes.Structure):
    _fields_ = [("h", ctypes.c_int32), ("w", ctypes.c_int32), ("c0", c_float * 3), ("c1", c_float * 3),
                ("c2", c_float * 3), ("mask", c_float * 3)]


class SphereTables(ctypes.Structure):
    _fields_ = [("L", ctypes.c_int32), ("n_theta", ctypes.c_int32), ("n_phi", ctypes.c_int32),
                ("n_pairs", ctypes.c_int32), ("ring", c_void_p), ("phi_cs", c_void_p), ("wplm", c_void_p),
                ("tw", c_void_p)]


class So3Dims(ctypes.Structure):
    _fields_ = [("L", ctypes.c_int32), ("n", ctypes.c_int32), ("nb", ctypes.c_int32), ("nc", ctypes.c_int32),
                ("fold", ctypes.c_int32), ("mu_max", ctypes.c_int32), ("n_pairs", ctypes.c_int32)]


class RefineOpts(ctypes.Structure):
    _fields_ = [("iters", ctypes.c_int32), ("max_step", c_float), ("scale0", c_float), ("scale_min", c_float),
                ("scale_max", c_float), ("nmi_bins", ctypes.c_int32), ("stamp", c_float)]


P = c_void_p
_SIGS = {
    "zeb_error": ([ctypes.c_char_p, c_size_t], c_size_t),
    "zeb_version": ([], c_char_p),
    "zeb_gauss_legendre": ([c_int, P, P, P], c_int),
    "zeb_legendre_table": ([c_int, c_int, P, P, P], c_int),
    "zeb_wigner_half_pi": ([c_int, P, P], c_int),
    "zeb_prep": ([P, c_int, c_int, c_int, c_int, P, c_int, c_float, P, c_int, P, P], c_int),
    "zeb_prep_scratch_bytes": ([c_int, c_int, c_int, c_float], c_size_t),
    "zeb_prep_ex": ([P, c_int, c_int, c_int, c_int, P, c_int, c_float, P, c_int, P, P, P], c_int),
    "zeb_prep_reduced": ([P, c_int, c_int, c_int, c_int, ctypes.c_double, P, c_int, c_float, P, c_int, P, P, P], c_int),
    "zeb_master_blur_pass": ([P, P, c_int, c_float, c_float, c_int, P], c_int),
    "zeb_master_gradient": ([P, P, c_int, P], c_int),
    "zeb_master_pairs": ([P, P, c_int, P, P, P], c_int),
    "zeb_master_sample_grid": ([P, c_int, P, c_int, c_int, P, P], c_int),
    "zeb_sphere_scratch_bytes": ([ctypes.POINTER(SphereTables), c_int], c_size_t),
    "zeb_sphere_coefficients": ([P, P, c_int, ctypes.POINTER(Frame), ctypes.POINTER(SphereTables), c_uint, P, P, P, P],
                                c_int),
    "zeb_sphere_coefficients_spans": ([P, P, c_int, ctypes.POINTER(Frame), ctypes.POINTER(SphereTables), P, c_uint, P, P,
                                       P, P], c_int),
    "zeb_sphere_spans": ([ctypes.POINTER(Frame), ctypes.POINTER(SphereTables), P, c_int, c_int, P, P], c_int),
    "zeb_correlation_table": ([ctypes.POINTER(So3Dims), P, P, P, P], c_int),
    "zeb_spectrum_f32": ([P, c_int, ctypes.POINTER(So3Dims), P, P, P], c_int),
    "zeb_spectrum_bytes": ([ctypes.POINTER(So3Dims), c_int], c_size_t),
    "zeb_spectrum_bf16": ([P, c_int, ctypes.POINTER(So3Dims), c_int, P, P, P, P, P], c_int),
    "zeb_tc_pack_master": ([ctypes.POINTER(So3Dims), c_int, P, P, P], c_int),
    "zeb_tc_master_bytes": ([ctypes.POINTER(So3Dims), c_int], c_size_t),
    "zeb_tc_patterns_bytes": ([ctypes.POINTER(So3Dims), c_int, c_int], c_size_t),
    "zeb_peaks_scratch_bytes": ([ctypes.POINTER(So3Dims), c_int], c_size_t),
    "zeb_correlate_peaks": ([P, c_int, ctypes.POINTER(So3Dims), P, P, c_int, P, P, P], c_int),
    "zeb_spectrum_h_bytes": ([ctypes.POINTER(So3Dims), c_int], c_size_t),
    "zeb_set_test_stall": ([c_longlong], c_int),
    "zeb_master_quads": ([P, c_int, P, P], c_int),
    "zeb_panel_split_bytes": ([c_int, c_int], c_size_t),
    "zeb_pack_panel_split": ([P, c_int, c_int, c_int, c_int, P, P], c_int),
    "zeb_project_bf16": ([P, c_int, P, c_int, c_int, P, P, P], c_int),
    "zeb_project_f32": ([P, c_int, P, c_int, c_int, P, P], c_int),
    "zeb_refine_list_h": ([P, P, P, c_int, c_int, ctypes.POINTER(Frame), P, c_int, P, P, c_int,
                           ctypes.POINTER(RefineOpts), P, P], c_int),
    "zeb_spectrum_bf16_h": ([P, c_int, ctypes.POINTER(So3Dims), c_int, P, P, P, c_float, P, P], c_int),
    "zeb_correlate_peaks_h": ([P, c_int, ctypes.POINTER(So3Dims), c_float, P, P, P, P, P], c_int),
    "zeb_correlate_peaks_static": ([P, c_int, ctypes.POINTER(So3Dims), P, P, c_int, P, P], c_int),
    "zeb_correlate_volume": ([P, c_int, ctypes.POINTER(So3Dims), P, P, P], c_int),
    "zeb_rden_build": ([P, P, P, c_int, c_longlong, P, P], c_int),
    "zeb_refine": ([P, P, P, c_int, c_int, ctypes.POINTER(Frame), P, P, c_int, ctypes.POINTER(RefineOpts), P, P], c_int),
    "zeb_chance": ([P, P, c_int, c_int, ctypes.POINTER(Frame), P, c_int, c_int, P, P], c_int),
    "zeb_records_fz": ([P, c_int, P, c_int, P, P], c_int),
    "zeb_records_fz_bunge": ([P, c_int, P, c_int, P, P, P], c_int),
    "zeb_det6": ([c_int, P, P, c_int, ctypes.POINTER(Frame), P, P, c_int, P, P, P, P], c_int),
    "zeb_det6_list": ([c_int, P, P, c_int, ctypes.POINTER(Frame), P, c_int, P, P, c_int, P, P, P, P], c_int),
    "zeb_solve6": ([P, P, c_int, P, P, P], c_int),
    "zeb_mask_pixels": ([ctypes.POINTER(Frame)], c_int),
    "zeb_pc_splat": ([c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_void_p], c_int),
    "zeb_clahe_scratch_bytes": ([c_int, c_int, c_int], c_size_t),
    "zeb_nlpar_scratch_bytes": ([c_int, c_int, c_int, c_int], c_size_t),
    "zeb_nlpar": ([c_void_p, c_int, c_void_p, c_void_p, c_int, c_int, c_float, c_void_p, c_void_p, c_void_p, c_void_p,
                   c_void_p], c_int),
    "zeb_clahe": ([c_void_p, c_int, c_int, c_int, c_int, c_int, c_float, c_void_p, c_void_p], c_int),
    "zeb_combine": ([c_void_p, c_void_p, c_void_p, c_longlong, c_int, c_void_p], c_int),
    "zeb_master_symmetrize": ([c_void_p, c_void_p, c_int, c_void_p, c_int, c_void_p], c_int),
    "zeb_sums6_list": ([c_void_p, c_void_p, c_int, ctypes.POINTER(Frame), c_void_p, c_int, c_void_p, c_void_p, c_int,
                        c_int, c_void_p, c_void_p, c_void_p, c_void_p], c_int),
    "zeb_mask_list": ([ctypes.POINTER(Frame), P, P], c_int),
    "zeb_refine_list": ([P, P, P, c_int, c_int, ctypes.POINTER(Frame), P, c_int, P, P, c_int, ctypes.POINTER(RefineOpts),
                         P, P], c_int),
    "zeb_panel_bytes": ([c_int, c_int], c_size_t),
    "zeb_pack_panel": ([P, c_int, c_int, c_int, P, P], c_int),
    "zeb_dict_sims": ([ctypes.POINTER(Frame), P, c_int, P, P, c_int, P, P], c_int),
    "zeb_match_slices": ([c_int, c_int, c_int, c_int], c_int),
    "zeb_match_bf16": ([P, c_int, P, c_int, c_int, c_int, P, P, P, P], c_int),
    "zeb_match_f32": ([P, c_int, P, c_int, c_int, c_int, P, P, P], c_int),
    "zeb_match_best": ([P, c_int, P, c_int, c_int, P, c_int, P, P, P], c_int),
    "zeb_project": ([P, c_int, P, c_int, ctypes.POINTER(Frame), P, P], c_int),
}

_lib = None
ZEB_PEAKS_STATIC_SLABS = 1 << 19  # include/zebsdsolve_b200.h

# kernels each entry point launches (for the launch counts the benchmark reports)
KERNELS = {"zeb_nlpar": 5, "zeb_pc_splat": 0, "zeb_sums6_list": 1, "zeb_clahe": 4, "zeb_combine": 1, "zeb_master_symmetrize": 1, "zeb_prep": 1, "zeb_prep_ex": 1, "zeb_prep_reduced": 1, "zeb_sphere_coefficients": 3, "zeb_sphere_coefficients_spans": 3, "zeb_sphere_spans": 1, "zeb_spectrum_f32": 1,
           "zeb_spectrum_bf16": 2, "zeb_tc_pack_master": 0, "zeb_correlate_peaks": 2, "zeb_correlate_peaks_static": 2, "zeb_spectrum_bf16_h": 2, "zeb_correlate_peaks_h": 2, "zeb_master_quads": 1, "zeb_refine_list_h": 1, "zeb_pack_panel_split": 1, "zeb_project_bf16": 1, "zeb_project_f32": 1, "zeb_correlate_volume": 1, "zeb_rden_build": 1,
           "zeb_refine": 1, "zeb_chance": 1, "zeb_project": 1, "zeb_records_fz": 1, "zeb_records_fz_bunge": 1, "zeb_det6": 1, "zeb_det6_list": 1, "zeb_solve6": 1, "zeb_pack_panel": 1, "zeb_mask_list": 1, "zeb_refine_list": 1, "zeb_dict_sims": 1, "zeb_match_bf16": 1, "zeb_match_f32": 1, "zeb_match_best": 1, "zeb_master_blur_pass": 1, "zeb_master_gradient": 1, "zeb_master_pairs": 1,
           "zeb_master_sample_grid": 1, "zeb_gauss_legendre": 1, "zeb_legendre_table": 1, "zeb_wigner_half_pi": 1,
           "zeb_correlation_table": 1}
launches = {"count": 0}


def lib_path():
    return Path(os.environ.get("ZEBSDSOLVE_B200_LIB", HERE / LIB_NAME))


def load():
    """The library with every signature bound (cached)."""
    global _lib
    if _lib is not None:
        return _lib
    p = lib_path()
    if not p.exists():
        raise NativeError(f"{p} not found: build it with `python -m zebsdsolve_b200.build`")
    lib = ctypes.CDLL(str(p))
    for name, (args, res) in _SIGS.items():
        fn = getattr(lib, name)
        fn.argtypes, fn.restype = args, res
    _lib = lib
    return lib


def symbols():
    """Names this module binds (every entry point of include/zebsdsolve_b200.h)."""
    return list(_SIGS)


def last_error(lib=None):
    lib = lib or load()
    buf = ctypes.create_string_buffer(1024)
    n = lib.zeb_error(buf, 1024)
    return buf.value.decode(errors="replace") if n else ""


# Solver.profile: while on, every entry point that launches kernels is bracketed by two CUDA events
# on the current stream (the one the entry points are given); profile_report sums them by name
profiling = {"on": False, "pairs": [], "totals": {}}


def profile_flush(wait=True):
    """Fold the recorded event pairs into the per-entry-point totals (name → [calls, ms]); with
    wait, after the device has finished them, else only the pairs already complete."""
    import torch

    if wait and profiling["pairs"]:
        torch.cuda.synchronize()
    keep = []
    for name, e0, e1 in profiling["pairs"]:
        if wait or e1.query():
            t = profiling["totals"].setdefault(name, [0, 0.0])
            t[0] += 1
            t[1] += e0.elapsed_time(e1)
        else:
            keep.append((name, e0, e1))
    profiling["pairs"] = keep


def call(name, *args):
    """Call an entry point; a negative return raises NativeError with the library's message."""
    lib = load()
    timed = profiling["on"] and KERNELS.get(name, 0) > 0
    if timed:
        import torch

        e0 = torch.cuda.Event(enable_timing=True)
        e0.record()
    rc = getattr(lib, name)(*args)
    if timed:
        e1 = torch.cuda.Event(enable_timing=True)
        e1.record()
        profiling["pairs"].append((name, e0, e1))
        if len(profiling["pairs"]) > 4096:
            profile_flush(wait=False)
    launches["count"] += KERNELS.get(name, 0)
    if isinstance(rc, int) and rc < 0:
        raise NativeError(f"{name}: {last_error(lib) or rc}")
    return rc
