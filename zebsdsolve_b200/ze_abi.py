"""The reference's own C ABI (the `ze_*` calls of zebsdsolve 0.2.8: src/exports.zig and
src/native_api.zig, bound by python/zebsdsolve/_native.py), carried out over this package's engine.

libzebsdsolve.so (csrc/ze_abi.c) exports every `ze_*` symbol with the reference's argument types
and struct layouts; each call takes the interpreter lock and lands in `call(name, *args)` here
with its arguments as plain integers (addresses, sizes, indices) and floats. The reference's own
Python package therefore runs unmodified over this library:

    ZEBSDSOLVE_LIB=<package>/libzebsdsolve.so ZEBSDSOLVE_WGPU=<anything> python -c "import zebsdsolve"

Conventions as exports.zig:1-8: a call returns 0 (or a count, size or index) on success and a
negative code on failure, `ze_error` then saying why (and clearing it); calls that fill a buffer
return the size they need and copy only when the capacity given suffices. The engine handle is an
opaque non-null pointer. The calls of the parts this engine does not build (master simulation and
crystals, toy scans, colour maps, the .h5oina export, orientation conventions other than the
engine's own, WGSL) fail with a message that says so.
"""
import ctypes
import json
import traceback

import numpy as np

METHODS = ("spherical", "dictionary", "pca")
PLANE_MODELS = ("centre", "line", "affine", "projective")
# scan.zig:27 Format, in order (ScanInfo.format; 100: patterns from memory)
FORMATS = ("kikuchipy h5ebsd", "Bruker h5ebsd", "EDAX h5ebsd", "Oxford h5oina", "EDAX up1/up2", "Oxford ebsp",
           "NORDIF", "EMsoft patterns")
FORMAT_ALIASES = {"edax_up": "EDAX up1/up2", "oxford_ebsp": "Oxford ebsp", "nordif": "NORDIF"}
# convention.zig:54-59, 102-109: the engine's own frame (kikuchipy's), the only one here

U32, I32, U64, F64 = ctypes.c_uint32, ctypes.c_int32, ctypes.c_uint64, ctypes.c_double


# ── the reference's extern structs, field for field (engine.zig:55-107, geometry.zig:28-50,
#    pcfit.zig Result, planefit.zig PlaneResult and PlanePoint, simulate.zig Summary) ──

class ScanInfo(ctypes.Structure):
    _fields_ = [("rows", U32), ("cols", U32), ("pat_h", U32), ("pat_w", U32), ("pixel", U32),
                ("has_background", U32), ("has_pc", U32), ("format", U32), ("voltage_kv", F64),
                ("bytes", F64), ("has_px", U32), ("pattern_kinds", U32)]


class PhaseInfo(ctypes.Structure):
    _fields_ = [("side", U32), ("point_group", U32), ("space_group", U32), ("laue", U32), ("n_fold", U32),
                ("mirror", U32), ("inversion", U32), ("pad", U32), ("voltage_kv", F64), ("name", ctypes.c_char * 64)]


class Geometry(ctypes.Structure):
    _fields_ = [("pc", F64 * 3), ("sample_tilt_deg", F64), ("detector_tilt_deg", F64), ("rot", F64 * 3),
                ("px_um", F64), ("step_x_um", F64), ("step_y_um", F64), ("plane_kind", U32), ("pad", U32),
                ("plane", F64 * 12)]


class PcResult(ctypes.Structure):
    _fields_ = [("pc", F64 * 3), ("start", F64 * 3), ("score", F64), ("start_score", F64), ("n_patterns", U32),
                ("n_candidates", U32), ("levels", U32), ("at_border", U32)]


class PlaneResult(ctypes.Structure):
    _fields_ = [("plane", F64 * 12), ("pc", F64 * 3), ("start_pc", F64 * 3), ("rot", F64 * 3),
                ("said_rot", F64 * 3), ("said_rot_se", F64 * 3), ("step", F64 * 2), ("step_se", F64 * 2),
                ("skew", F64), ("skew_se", F64), ("pc_se", F64 * 3), ("rmsd", F64 * 3), ("ncc", F64),
                ("start_ncc", F64), ("kind", U32), ("frame", U32), ("n_patterns", U32), ("n_used", U32),
                ("iterations", U32), ("blocks", U32), ("model", U32), ("compared", U32), ("cv", F64 * 4),
                ("cv_se", F64 * 4), ("method", U32), ("pad", U32)]


class PlanePoint(ctypes.Structure):
    _fields_ = [("cell", U64), ("pc", F64 * 3), ("fit", F64 * 3), ("ncc", F64), ("used", U32), ("pad", U32)]


class SimSummary(ctypes.Structure):
    _fields_ = [(k, U32) for k in ("n_k", "n_sites", "n_g", "n_bins", "n_bins_run", "max_beams", "failed", "stopped",
                                   "halfw", "rank", "max_weak", "overflow")] + [("last_change", F64)]


class IndexStatus(ctypes.Structure):
    _fields_ = [("sweep", U32), ("sweeps", U32), ("bandwidth", U32), ("dict_grid", U32), ("done", U64),
                ("total", U64), ("region", U64), ("accepted", U64), ("method", U32), ("pad", U32)]


# ── memory the caller owns ──

_CT = {np.float32: ctypes.c_float, np.float64: ctypes.c_double, np.uint32: ctypes.c_uint32,
       np.int32: ctypes.c_int32, np.uint64: ctypes.c_uint64, np.int64: ctypes.c_int64, np.uint16: ctypes.c_uint16,
       np.uint8: ctypes.c_uint8}


def _view(addr, n, dtype):
    """A writable numpy view of n values of dtype at the caller's address."""
    if n == 0:
        return np.zeros(0, dtype)
    if not addr:
        raise ValueError("null buffer")
    return np.ctypeslib.as_array((_CT[dtype] * int(n)).from_address(addr))


def _text(addr, n):
    return ctypes.string_at(addr, n).decode() if n else ""


def _put(addr, cap, data):
    """Copy the bytes that fit into buf[0:cap]; returns their count."""
    k = min(int(cap), len(data))
    if k and addr:
        ctypes.memmove(addr, data, k)
    return k


class NotBuilt(Exception):
    pass


class _Handle:
    def __init__(self, solver):
        self.s = solver
        self.err = ""
        self.pending = b""  # events serialized but not yet taken (ze_events)


_handles = {}
_next = [1]
_create_err = [""]


def _api(what, fail=-1):
    """The call's body on the engine of handle h; an exception becomes `fail` and ze_error's message."""

    def wrap(fn):
        def run(h, *a):
            x = _handles.get(int(h))
            if x is None:
                return fail
            try:
                return fn(x, *a)
            except NotBuilt as ex:
                x.err = f"{what}: {ex}"
            except Exception as ex:  # noqa: BLE001 - the ABI's error channel
                msg = str(ex) or type(ex).__name__
                x.err = msg if msg.startswith(what + ":") else f"{what}: {msg}"
            return fail

        run.__name__ = fn.__name__
        return run

    return wrap


def _not_built(what, why, fail=-1):
    @_api(what, fail)
    def fn(x, *a):
        raise NotBuilt(why)

    return fn


# ── creation (native_api.zig:18-50) ──

def ze_create(lib_path):
    """The adapter library's path the reference opens wgpu-native from is not used: the engine runs
    on the current CUDA device."""
    from . import Solver

    _create_err[0] = ""
    try:
        s = Solver()
    except Exception as ex:  # noqa: BLE001
        _create_err[0] = f"engine init failed: {ex}"
        return 0
    h = _next[0] * 16
    _next[0] += 1
    _handles[h] = _Handle(s)
    return h


def ze_create_error(buf, cap):
    b = _create_err[0].encode()
    return _put(buf, cap, b)


def ze_destroy(h):
    x = _handles.pop(int(h), None)
    if x is not None:
        x.s.close()


# ── plumbing (exports.zig:30-66) ──

def ze_adapter(h, buf, cap):
    import torch

    x = _handles.get(int(h))
    if x is None:
        return 0
    name = torch.cuda.get_device_name(x.s._e.dev).encode()
    return _put(buf, cap, name)


def ze_error(h, buf, cap):
    x = _handles.get(int(h))
    if x is None:
        return 0
    b = x.err.encode()
    x.err = ""
    return _put(buf, cap, b)


@_api("configure")
def ze_configure(x, js, n):
    settings = json.loads(_text(js, n) or "{}")
    if not isinstance(settings, dict):
        raise ValueError("settings are a JSON object")
    x.s.configure(**settings)
    return 0


@_api("settings", 0)
def ze_settings(x, buf, cap):
    b = json.dumps(x.s.settings).encode()
    _put(buf, cap, b)
    return len(b)


@_api("events", 0)
def ze_events(x, buf, cap):
    x.pending += b"".join(json.dumps(e).encode() + b"\n" for e in x.s.events())
    # whole lines only; a line longer than the whole buffer is dropped (0 means no lines are left)
    while x.pending:
        cut = x.pending.rfind(b"\n", 0, int(cap)) + 1
        if cut:
            n = _put(buf, cap, x.pending[:cut])
            x.pending = x.pending[cut:]
            return n
        x.pending = x.pending[x.pending.find(b"\n") + 1:]
    return 0


def ze_cancel(h):
    x = _handles.get(int(h))
    if x is not None:
        x.s.cancel()


# ── scan (exports.zig:70-122, 433-466) ──

@_api("open_scan")
def ze_open_scan(x, paths, n):
    names = [p for p in _text(paths, n).split("\n") if p][:8]
    x.s.open(*names)
    return 0


@_api("set_patterns")
def ze_set_patterns(x, data, n, pixel, rows, cols, h, w):
    if pixel > 2:
        raise ValueError("UnsupportedPixelType")
    dt = (np.uint8, np.uint16, np.float32)[pixel]
    count = rows * cols * h * w
    if count * np.dtype(dt).itemsize != n:
        raise ValueError(f"BadLength: {n} bytes for {rows} x {cols} patterns of {h} x {w}")
    # the engine keeps its own copy: the caller's buffer may go once this returns
    a = _view(data, count, dt).reshape(rows, cols, h, w).copy()
    x.s.set_patterns(a)
    return 0


@_api("synthesize")
def ze_synthesize(x, quats, phase, grain, n):
    """exports.zig:97-102 — a toy scan from the phases loaded, in place of any scan open
    (Solver.synthesize): its orientations (4 f32 a cell), phases and grains (i32) into the
    caller's buffers, n = toy_rows × toy_cols cells (BadLength otherwise)."""
    st = x.s._e.set
    if n != st["toy_rows"] * st["toy_cols"]:
        raise RuntimeError("BadLength")
    got = x.s.synthesize()
    _view(quats, 4 * n, np.float32)[:] = got["quaternions"].reshape(-1)
    _view(phase, n, np.int32)[:] = got["phase"].reshape(-1)
    _view(grain, n, np.int32)[:] = got["grain"].reshape(-1)
    return 0


def ze_close_scan(h):
    x = _handles.get(int(h))
    if x is None:
        return
    e = x.s._e
    e.patterns, e.res, e.scan_source, e.pixel = None, None, None, None
    e._pinned, e._resident = None, None


def _scan(x):
    e = x.s._e
    if e.patterns is None:
        return None
    return x.s.scan


def ze_scan_info(h, out):
    x = _handles.get(int(h))
    s = ScanInfo.from_address(out)
    ctypes.memset(out, 0, ctypes.sizeof(ScanInfo))
    if x is None:
        return
    try:
        sc = _scan(x)
    except Exception:  # noqa: BLE001 - no scan: all zero
        sc = None
    if sc is None:
        return
    e = x.s._e
    s.rows, s.cols = sc["rows"], sc["cols"]
    s.pat_h, s.pat_w = sc["pattern_shape"]
    s.pixel = int(e.pixel)
    s.has_background, s.has_pc, s.has_px = int(sc["has_background"]), int(sc["has_pc"]), int(sc["has_px"])
    v = sc.get("voltage_kv")
    s.voltage_kv = float(v) if v is not None and np.isfinite(v) else 0.0
    src = getattr(e, "scan_source", None)
    if src:
        fmt = FORMAT_ALIASES.get(src.get("format"), src.get("format"))
        s.format = FORMATS.index(fmt) if fmt in FORMATS else 0
        kinds = src.get("pattern_kinds") or []
        s.pattern_kinds = (1 if "processed" in kinds else 0) | (2 if "unprocessed" in kinds else 0) | \
            (4 if e.set["stored_patterns"] == "unprocessed" and "unprocessed" in kinds else 0)
        try:
            import os

            s.bytes = float(os.path.getsize(src["paths"][0]))
        except Exception:  # noqa: BLE001
            s.bytes = float(e.patterns.nbytes)
    else:
        s.format = 100
        s.bytes = float(e.patterns.nbytes)


def ze_scan_format(h, buf, cap):
    x = _handles.get(int(h))
    if x is None or x.s._e.patterns is None:
        return 0
    src = getattr(x.s._e, "scan_source", None)
    name = "memory" if not src else FORMAT_ALIASES.get(src.get("format"), src.get("format"))
    return _put(buf, cap, name.encode())


def _stored_overview_of(x):
    src = getattr(x.s._e, "scan_source", None) if x.s._e.patterns is not None else None
    return (src or {}).get("overview") or (0, None)


def ze_scan_overview_kind(h):
    """exports.zig:451-454 — the stored quality map's kind: 0 none, 1 band contrast, 2 image
    quality, 3 Radon quality, 4 pattern quality."""
    x = _handles.get(int(h))
    return int(_stored_overview_of(x)[0]) if x is not None else 0


@_api("scan_overview")
def ze_scan_overview(x, out, cap):
    """exports.zig:456-465 — the stored quality map's size (rows × cols; 0 for none), and with a
    buffer its values as float32; BufferTooSmall when cap is short."""
    kind, read = _stored_overview_of(x)
    if not kind:
        return 0
    sc = x.s.scan
    n = sc["rows"] * sc["cols"]
    if out:
        if cap < n:
            raise RuntimeError("BufferTooSmall")
        _view(out, n, np.float32)[:] = read()
    return n


@_api("stored_orientations")
def ze_stored_orientations(x, euler, phase, n):
    """exports.zig:819-834 — the maker's stored orientations: Bunge angles (3 f64 a cell) and a
    phase label a cell (−1: not indexed), n cells; 1, or 0 when the file stores none."""
    src = getattr(x.s._e, "scan_source", None) if x.s._e.patterns is not None else None
    read = (src or {}).get("stored")
    got = read() if read is not None else None
    if got is None:
        return 0
    if got["phase"].size != n:
        raise RuntimeError("BadLength")
    _view(euler, 3 * n, np.float64)[:] = got["euler"].reshape(-1)
    _view(phase, n, np.int32)[:] = got["phase"]
    return 1


# ── geometry (exports.zig:124-158) ──

def _geo_out(g, out):
    o = Geometry.from_address(out)
    o.pc[:] = [float(v) for v in g.pc]
    o.sample_tilt_deg, o.detector_tilt_deg = float(g.sample_tilt_deg), float(g.detector_tilt_deg)
    o.rot[:] = [float(v) for v in g.rot]
    o.px_um, o.step_x_um, o.step_y_um = float(g.px_um), float(g.step_x_um), float(g.step_y_um)
    o.plane_kind, o.pad = int(g.plane_kind), 0
    o.plane[:] = [float(v) for v in np.asarray(g.plane, np.float64).reshape(12)]


def _geo_fields(addr):
    g = Geometry.from_address(addr)
    return {"pc": list(g.pc), "sample_tilt_deg": g.sample_tilt_deg, "detector_tilt_deg": g.detector_tilt_deg,
            "rot": list(g.rot), "px_um": g.px_um, "step_x_um": g.step_x_um, "step_y_um": g.step_y_um,
            "plane_kind": int(g.plane_kind), "plane": list(g.plane)}


def ze_get_geometry(h, out):
    x = _handles.get(int(h))
    if x is not None:
        _geo_out(x.s._e.geo, out)


def ze_set_geometry(h, addr):
    """The whole struct comes back; what the caller changed is what differs from the geometry in
    use, and only that is given (exports.zig:141-155)."""
    x = _handles.get(int(h))
    if x is None:
        return
    try:
        x.s.set_geometry(**_geo_fields(addr))
    except Exception as ex:  # noqa: BLE001 - a void call: kept for ze_error
        x.err = f"set_geometry: {ex}"


# ── phases (exports.zig:160-398) ──

@_api("add_phase")
def ze_add_phase(x, path, n):
    return int(x.s.add_phase(_text(path, n)))


def ze_clear_phases(h):
    x = _handles.get(int(h))
    if x is not None:
        x.s.clear_phases()


def ze_phase_count(h):
    x = _handles.get(int(h))
    return 0 if x is None else len(x.s._e.phases)


@_api("phase_info")
def ze_phase_info(x, i, out):
    from .rotations import LAUE_NUMBERS

    e = x.s._e
    if i >= len(e.phases):
        raise IndexError("NoSuchPhase")
    m = e.phases[i].master
    o = PhaseInfo.from_address(out)
    ctypes.memset(out, 0, ctypes.sizeof(PhaseInfo))
    o.side, o.point_group, o.space_group = int(m.side), int(m.point_group), int(m.space_group)
    o.laue = int(LAUE_NUMBERS.get(m.laue, 0))
    o.voltage_kv = float(m.voltage_kv) if m.voltage_kv is not None and np.isfinite(m.voltage_kv) else 0.0
    # the selection rules as the band last prepared found them
    for b in e.bands.values():
        pb = b.get("phases", {}).get(i) if isinstance(b, dict) else None
        if pb is not None:
            r = pb[1].rules
            o.n_fold, o.mirror, o.inversion = int(r.n_fold), int(r.mirror), int(r.inversion)
    o.name = str(m.name).encode()[:63]
    return 0


@_api("master_image")
def ze_master_image(x, phase, out, n):
    m = x.s.master(int(phase)).reshape(-1)
    if n < m.size:
        raise ValueError(f"BufferTooSmall: {m.size} values, {n} given")
    _view(out, m.size, np.float32)[:] = m
    return 0


ze_sim_read_cif = _not_built("sim_read_cif", "master simulation (crystals, CIF) is not part of this engine")
ze_sim_set_crystal = _not_built("sim_set_crystal", "master simulation (crystals) is not part of this engine")
ze_sim_edit_crystal = _not_built("sim_edit_crystal", "master simulation (crystals) is not part of this engine")
ze_sim_crystal = _not_built("sim_crystal", "master simulation (crystals) is not part of this engine")
ze_sim_run = _not_built("sim_run", "master simulation is not part of this engine")
ze_sim_sheets = _not_built("sim_sheets", "master simulation is not part of this engine")
ze_sim_add_phase = _not_built("sim_add_phase", "master simulation is not part of this engine")
ze_sim_npz = _not_built("sim_npz", "master simulation is not part of this engine")
ze_sim_energy = _not_built("sim_energy", "master simulation is not part of this engine")
ze_cell_info = _not_built("cell_info", "the crystal's cell picture is not part of this engine")
ze_cell_view = _not_built("cell_view", "the crystal's cell picture is not part of this engine")
ze_sphere_view = _not_built("sphere_view", "the master's globe pictures are not part of this engine")


# ── patterns (exports.zig:401-476) ──

@_api("pattern_shape")
def ze_pattern_shape(x, full, out):
    h, w = x.s.shape(bool(full))
    _view(out, 2, np.uint32)[:] = (h, w)
    return 0


@_api("pattern")
def ze_pattern(x, cell, processed, full, out, n):
    if processed > 3:
        raise ValueError("UnknownKind")
    p = np.asarray(x.s._e.pattern(int(cell), int(processed), bool(full)), np.float32).reshape(-1)
    if n != p.size:
        raise ValueError(f"BadLength: {p.size} values, {n} given")
    _view(out, p.size, np.float32)[:] = p
    return 0


@_api("nlpar_view", 0)
def ze_nlpar_view(x, out, shares, cap):
    v = x.s.nlpar_view()
    if v is None:
        return 0
    _view(out, 3, np.float32)[:] = (v["noise"], v["left"], v["own"])
    sh = np.asarray(v["shares"], np.float32).reshape(-1)
    side = int(round(np.sqrt(sh.size)))
    if shares and cap >= sh.size:
        _view(shares, sh.size, np.float32)[:] = sh
    return side


@_api("lattice")
def ze_lattice(x, want, out, cap):
    cells = np.asarray(x.s.lattice(int(want)), np.uint64)
    if cap >= cells.size and cells.size:
        _view(out, cells.size, np.uint64)[:] = cells
    return int(cells.size)


def ze_pixel_angle(h):
    x = _handles.get(int(h))
    if x is None or x.s._e.patterns is None:
        return 0.0
    try:
        return float(x.s.pixel_angle)
    except Exception:  # noqa: BLE001 - 0 without a scan
        return 0.0


@_api("pattern_stats")
def ze_pattern_stats(x, cells, n, out, cap):
    if cap < 2 * n:
        raise ValueError("BufferTooSmall")
    c = _view(cells, n, np.uint64).astype(np.int64)
    mean, std = x.s.pattern_stats(c)
    o = _view(out, 2 * n, np.float32)
    o[0::2], o[1::2] = mean, std
    return 0


@_api("simulate")
def ze_simulate(x, phase, cells, quats, n, full, out, cap):
    e = x.s._e
    c = _view(cells, n, np.uint64).astype(np.int64)
    q = _view(quats, 4 * n, np.float32).reshape(n, 4).copy()
    binning = e.set["binning"]
    swap = bool(full) and binning != 1
    if swap:
        e.set.apply({"binning": 1.0})
    try:
        sims = np.asarray(e.simulate(int(phase), c, q), np.float32).reshape(-1)
    finally:
        if swap:
            e.set.apply({"binning": binning})
    if cap != sims.size:
        raise ValueError(f"BadLength: {sims.size} values, {cap} given")
    _view(out, sims.size, np.float32)[:] = sims
    return 0


# ── the pattern-centre vote and the plane fit (exports.zig:478-591) ──

@_api("fit_pc")
def ze_fit_pc(x, out):
    r = x.s.fit_pc()
    o = PcResult.from_address(out)
    o.pc[:], o.start[:] = r["pc"], r["start"]
    o.score, o.start_score = float(r["score"]), float(r["start_score"])
    o.n_patterns, o.n_candidates = int(r["n_patterns"]), int(r["n_candidates"])
    o.levels, o.at_border = int(r["levels"]), int(bool(r["at_border"]))
    return 0


def _axes_out(axes, cap, lv):
    x_, y_, z_ = lv["axes"]
    a = np.concatenate([np.asarray(x_, np.float64), np.asarray(y_, np.float64), np.asarray(z_, np.float64)])
    if axes and cap >= a.size:
        _view(axes, a.size, np.float64)[:] = a
    return a.size


def _shape_out(shape, lv):
    x_, y_, z_ = lv["axes"]
    _view(shape, 3, np.uint32)[:] = (len(z_), len(y_), len(x_))


@_api("pc_scores")
def ze_pc_scores(x, shape, axes, axes_cap, scores, cap):
    hist = x.s._e.pc_history
    if not hist:
        _view(shape, 3, np.uint32)[:] = 0
        return 0
    lv = hist[-1]
    _shape_out(shape, lv)
    sc = np.asarray(lv["scores"], np.float32).reshape(-1)
    x_, y_, z_ = lv["axes"]
    if axes_cap >= len(x_) + len(y_) + len(z_) and cap >= sc.size:
        _axes_out(axes, axes_cap, lv)
        _view(scores, sc.size, np.float32)[:] = sc
    return int(sc.size)


def ze_pc_level_count(h):
    x = _handles.get(int(h))
    return 0 if x is None else len(x.s._e.pc_history)


@_api("pc_level")
def ze_pc_level(x, i, shape, info, axes, axes_cap, scores, cap, pat_best, pat_ncc, pat_cap):
    hist = x.s._e.pc_history
    if i >= len(hist):
        return -1
    lv = hist[i]
    _shape_out(shape, lv)
    _view(info, 2, np.uint32)[:] = (int(lv["best"]), int(bool(lv["walked"])))
    sc = np.asarray(lv["scores"], np.float32).reshape(-1)
    best = np.asarray(lv["pat_best"], np.uint32).reshape(-1)
    ncc = np.asarray(lv["pat_ncc"], np.float32).reshape(-1)
    x_, y_, z_ = lv["axes"]
    if axes_cap >= len(x_) + len(y_) + len(z_) and cap >= sc.size and pat_cap >= best.size:
        _axes_out(axes, axes_cap, lv)
        _view(scores, sc.size, np.float32)[:] = sc
        _view(pat_best, best.size, np.uint32)[:] = best
        _view(pat_ncc, ncc.size, np.float32)[:] = ncc
    return int(sc.size)


@_api("pc_level_scores")
def ze_pc_level_scores(x, i, out, cap):
    hist = x.s._e.pc_history
    if i >= len(hist):
        return -1
    s = np.asarray(hist[i]["pat_scores"], np.float32).reshape(-1)
    if out and cap >= s.size:
        _view(out, s.size, np.float32)[:] = s
    return int(s.size)


@_api("pc_level_ballots")
def ze_pc_level_ballots(x, i, out, cap, info):
    hist = x.s._e.pc_history
    if i >= len(hist):
        return -1
    lv = hist[i]
    pk = [float(v) for v in lv["peak"]]
    _view(info, 5, np.float64)[:] = (*pk[:3], float(lv["ballots"]), float(lv["inliers"]))
    d = lv["density"]
    if d is None:
        return 0
    d = np.asarray(d, np.float32).reshape(-1)
    if out and cap >= d.size:
        _view(out, d.size, np.float32)[:] = d
    return int(d.size)


def _plane_out(x, r, out):
    """The plane fit's result (our Solver's dict of it) as planefit.zig's PlaneResult."""
    e = x.s._e
    o = PlaneResult.from_address(out)
    ctypes.memset(out, 0, ctypes.sizeof(PlaneResult))
    o.plane[:] = [float(v) for v in np.asarray(r["plane"], np.float64).reshape(12)]
    o.pc[:], o.start_pc[:], o.rot[:] = r["pc"], r["start_pc"], r["rot"]
    sd = r["said"]
    o.said_rot[:], o.said_rot_se[:] = sd["rot"], sd["rot_se"]
    o.step[:], o.step_se[:] = sd["step"], sd["step_se"]
    o.skew, o.skew_se = float(sd["skew"]), float(sd["skew_se"])
    o.pc_se[:], o.rmsd[:] = r["pc_se"], r["rmsd"]
    o.ncc, o.start_ncc = float(r["ncc"]), float(r["start_ncc"])
    o.kind = ("none", "affine", "projective").index(r["kind"])
    o.frame = int(r["frame"] == "follow")
    o.n_patterns, o.n_used, o.iterations = int(r["n_patterns"]), int(r["n_used"]), int(r["iterations"])
    o.blocks = int(sd["blocks"])
    o.model = PLANE_MODELS.index(r["model"]) if r["model"] in PLANE_MODELS else 0
    o.method = 1 if r["method"] == "points" else 0
    o.compared = int(bool(r["models"]))
    for k, m in enumerate(PLANE_MODELS):
        if m in r["models"]:
            o.cv[k], o.cv_se[k] = float(r["models"][m]["cv"]), float(r["models"][m]["cv_se"])
    del e


@_api("fit_auto")
def ze_fit_auto(x, out):
    _plane_out(x, x.s.fit_geometry(), out)
    return 0


@_api("fit_plane")
def ze_fit_plane(x, out):
    _plane_out(x, x.s.fit_plane(), out)
    return 0


@_api("plane_points", 0)
def ze_plane_points(x, out, cap):
    p = x.s._e.plane_points
    if p is None:
        return 0
    n = len(p["cells"])
    if out and cap >= n:
        arr = (PlanePoint * n).from_address(out)
        for k in range(n):
            a = arr[k]
            a.cell = int(p["cells"][k])
            a.pc[:] = [float(v) for v in p["pc"][k]]
            a.fit[:] = [float(v) for v in p["fit"][k]]
            a.ncc, a.used, a.pad = float(p["ncc"][k]), int(bool(p["used"][k])), 0
    return n


@_api("fit_patterns")
def ze_fit_patterns(x, cells, phases, quats, ncc, cap):
    c, ph, q, s = x.s.fit_patterns()
    n = len(c)
    if cap >= n and n:
        _view(cells, n, np.uint64)[:] = c
        _view(phases, n, np.int32)[:] = ph
        _view(quats, 4 * n, np.float32)[:] = np.asarray(q, np.float32).reshape(-1)
        _view(ncc, n, np.float32)[:] = s
    return n


# ── indexing (exports.zig:594-723) ──

@_api("index_begin")
def ze_index_begin(x):
    x.s.index_begin()
    return 0


@_api("index_step")
def ze_index_step(x):
    """The next part of the sweep (up to Engine.STEP_RUN_CELLS cells) as one pipelined run on the
    device: the cells and records of the reference's steps of a few batches, with fewer waits."""
    return int(x.s._call("index", x.s._e.index_step_run))


@_api("tune")
def ze_tune_begin(x):
    """The engine times its own trials on the device (Solver.tune): the whole tune runs here, and
    the caller's trial and report protocol (exports.zig:613-626) finds it finished."""
    x.s.tune()
    return 0


@_api("tune")
def ze_tune_trial(x):
    return 0


def ze_tune_report(h, seconds):
    return 0


@_api("chance")
def ze_chance(x, phase, out):
    med, spread = x.s.chance(int(phase))
    _view(out, 2, np.float32)[:] = (med, spread)
    return 0


def ze_index_status(h, out):
    o = IndexStatus.from_address(out)
    ctypes.memset(out, 0, ctypes.sizeof(IndexStatus))
    x = _handles.get(int(h))
    if x is None:
        return
    st = x.s.index_status
    o.sweep, o.sweeps, o.bandwidth, o.dict_grid = st["sweep"], st["sweeps"], st["bandwidth"], st["dict_grid"]
    o.done, o.total, o.region, o.accepted = st["done"], st["total"], st["region"], st["accepted"]
    o.method = METHODS.index(st["method"])


def ze_sweep(h, i, out):
    x = _handles.get(int(h))
    if x is None:
        return
    bw, dg, method = x.s._e.set.sweep(int(i))
    _view(out, 3, np.uint32)[:] = (int(bw), int(dg), METHODS.index(method))


def _index_cells(x, cells, n, out, cap, method, bandwidth, grid):
    e = x.s._e
    n_ph = len(e.phases)
    if cap != n_ph * n * 8:
        raise ValueError("BadLength")
    c = _view(cells, n, np.uint64).astype(np.int64)
    r = x.s._call("index_cells", e.index_cells, c, bandwidth, method, grid)
    _view(out, cap, np.float32)[:] = np.asarray(r, np.float32).reshape(-1)
    return 0


@_api("index_cells")
def ze_index_cells(x, cells, n, out, cap):
    return _index_cells(x, cells, n, out, cap, x.s._e.set["method"], None, None)


@_api("index_cells")
def ze_index_cells_by(x, cells, n, method, bandwidth, grid, out, cap):
    if method > 2 or bandwidth < 8 or bandwidth > 256 or grid < 2 or grid > 200:
        raise ValueError("BadSetting")
    return _index_cells(x, cells, n, out, cap, METHODS[method], int(bandwidth), int(grid))


@_api("cell_under")
def ze_cell_under(x, cell, geo, bandwidth, full, recs, n_recs, sim, cap):
    n_ph = len(x.s._e.phases)
    if n_ph == 0 or n_recs != n_ph * 8:
        raise ValueError("BadLength")
    if bandwidth < 8 or bandwidth > 256:
        raise ValueError("BadSetting")
    p, r, s = x.s._cell_under(int(cell), int(bandwidth), bool(full), _geo_fields(geo))
    s = np.asarray(s, np.float32).reshape(-1)
    if cap != s.size:
        raise ValueError(f"BadLength: {s.size} values, {cap} given")
    _view(recs, n_recs, np.float32)[:] = np.asarray(r, np.float32).reshape(-1)
    _view(sim, s.size, np.float32)[:] = s
    return int(p)


@_api("results")
def ze_results(x, kind, out, cap):
    e = x.s._e
    res = e.res
    if res is None:
        raise ValueError("NoScan")
    n = len(res["ncc"])
    if kind == 4:
        if cap < 12 * n:
            raise ValueError("BufferTooSmall")
        b = np.asarray(res["euler"], np.float32).reshape(n, 3).copy()
        b[res["phase"] < 0] = 0
        ctypes.memmove(out, b.ctypes.data, 12 * n)
        return 3 * n
    src = {0: ("quat", np.float32), 1: ("ncc", np.float32), 2: ("nmi", np.float32), 3: ("phase", np.int32),
           5: ("z", np.float32), 6: ("sweep", np.int32)}.get(int(kind))
    if src is None:
        raise ValueError("UnknownKind")
    data = np.ascontiguousarray(res[src[0]], src[1])
    if cap < data.nbytes:
        raise ValueError("BufferTooSmall")
    ctypes.memmove(out, data.ctypes.data, data.nbytes)
    return data.nbytes // 4


@_api("map")
def ze_map(x, kind, out, n):
    """exports.zig:726-729 — a result map as RGBA8 (4 bytes a cell): the score, phase and sweep maps
    (kinds 3-7); the IPF kinds 0-2 fail with NotImplemented. BadLength unless n is 4 × the cells."""
    from .output import result_map

    res = x.s._e.res
    if res is None:
        raise RuntimeError("NoScan")
    if n != 4 * len(res["ncc"]):
        raise RuntimeError("BadLength")
    _view(out, n, np.uint8)[:] = result_map(int(kind), res).reshape(-1)
    return 0
ze_ipf_key = _not_built("ipf_key", "IPF colour keys are not part of this engine")


@_api("export")
def ze_export(x, kind, buf, cap):
    if kind > 1:
        raise ValueError("UnknownKind")
    data = x.s.export_text(("ang", "ctf")[kind]).encode()
    if buf and cap >= len(data):
        ctypes.memmove(buf, data, len(data))
    return len(data)


ze_export_h5oina = _not_built("export_h5oina", "the .h5oina export is not part of this engine")
@_api("identify_frame")
def ze_identify_frame(x, euler, phase, n, buf, cap):
    """exports.zig:785-817 — the convention of a maker's orientations (Bunge radians, 3 f64 a cell,
    and a label a cell, negative: not indexed; with a null `euler` the scan file's own), found
    against the results, as JSON: the frame, how well it holds, the misorientation left, the
    labels matched and whether the exports took it. BufferTooSmall when cap is short."""
    if euler:
        if not phase:
            raise RuntimeError("MissingPhases")
        got = x.s.identify_frame(_view(euler, 3 * n, np.float64).copy(), _view(phase, n, np.int32).copy())
    else:
        got = x.s.identify_frame()
    keys = ("frame", "cells", "within", "median_deg", "runner_up_deg", "installed", "misorientation_cells",
            "misorientation", "misorientation_rows", "misorientation_cols", "matched")
    b = json.dumps({k: got[k] for k in keys}, separators=(",", ":")).encode()
    if cap < len(b):
        raise RuntimeError("BufferTooSmall")
    _put(buf, cap, b)
    return len(b)


def _frame_of(x):
    from .convention import Frame

    return (getattr(x.s._e, "convention", None) if x is not None else None) or Frame()


def ze_frame(h, buf, cap):
    """exports.zig:836-845 — the convention the exports write in, as JSON (axes, active, crystal
    and a line naming it); its length, copied as far as cap allows."""
    b = json.dumps(_frame_of(_handles.get(int(h))).as_dict(), separators=(",", ":")).encode()
    _put(buf, cap, b)
    return len(b)


@_api("set_frame")
def ze_set_frame(x, js, n):
    """exports.zig:847-859 — set the exports' convention from JSON as ze_frame gives it (axes,
    active, crystal; other keys ignored), or the engine's own when empty; InvalidFrame unless it
    is one of the conventions."""
    from .convention import Frame

    x.s._e.convention = None if n == 0 else Frame.from_dict(json.loads(_text(js, n)))
    return 0


def _ops(x, phase):
    e = x.s._e
    if x is not None and phase < len(e.phases):
        return e.phases[phase].master.rotations()
    return np.array([[1.0, 0.0, 0.0, 0.0]])


def ze_reduce(h, phase, q, euler):
    from .rotations import to_bunge, to_fz

    x = _handles.get(int(h))
    if x is None:
        return
    qv = _view(q, 4, np.float32)
    r = to_fz(qv.astype(np.float64).reshape(1, 4), _ops(x, int(phase)))
    qv[:] = np.asarray(r, np.float64).reshape(4)
    _view(euler, 3, np.float64)[:] = np.asarray(to_bunge(np.asarray(r, np.float64).reshape(1, 4))).reshape(3)


def ze_disorientation(h, phase, a, b):
    from .rotations import disorientation

    x = _handles.get(int(h))
    if x is None:
        return 0.0
    qa = _view(a, 4, np.float32).astype(np.float64).reshape(1, 4)
    qb = _view(b, 4, np.float32).astype(np.float64).reshape(1, 4)
    return float(np.asarray(disorientation(qa, qb, _ops(x, int(phase)))).reshape(-1)[0])


# ── tests and profiling (exports.zig:883-931) ──

def ze_compile_wgsl(h, code, code_len, entry, entry_len, msg, cap):
    """No WGSL is compiled here (the kernels are CUDA): the message says so (its length, ≥ 1)."""
    return max(_put(msg, cap, b"WGSL is not compiled by this engine: its kernels are CUDA for sm_100a"), 1)


def ze_shader(index, name, name_cap, buf, cap):
    """No WGSL modules: 0, past the last."""
    return 0


def ze_gpu_counts(h, out):
    x = _handles.get(int(h))
    o = _view(out, 4, np.uint32)
    if x is None:
        o[:] = 0
        return
    c = x.s.gpu_counts()
    o[:] = (c["dispatches"], c["submits"], c["reads"], c["waits"])


def ze_profile(h, on):
    x = _handles.get(int(h))
    return 0 if x is None else int(bool(x.s.profile(bool(on))))


def ze_profile_report(h, buf, cap):
    x = _handles.get(int(h))
    if x is None:
        return 0
    return _put(buf, cap, x.s.profile_report().encode())


# ── the dispatcher libzebsdsolve.so calls ──

NAMES = tuple(k for k in list(globals()) if k.startswith("ze_") and callable(globals()[k]))
_TABLE = {k: globals()[k] for k in NAMES}


def call(name, *args):
    """One ze_* call from the C library. Never raises: a failure inside a call's own error
    handling is printed and gives -1 (0 for the calls that return a size or count)."""
    try:
        return _TABLE[name](*args)
    except Exception:  # noqa: BLE001
        traceback.print_exc()
        return -1
