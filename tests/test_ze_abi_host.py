"""The reference's C ABI (libzebsdsolve.so) on the CPU, through the library itself: a stand-in engine
behind a handle (no GPU), driven by ctypes with the reference's argument types, so that what
crosses the boundary is checked: the structs filled field by field, the calls that return the
size they need and copy only when the capacity suffices, the event lines handed out in whole
lines, the patterns copied (the caller's buffer may go), the results of every kind, and failures
as negative codes with ze_error's message, which one read clears."""
import ctypes
import json

import numpy as np
import pytest

from zebsdsolve_b200 import build, ze_abi as Z
from zebsdsolve_b200.engine import Geometry
from zebsdsolve_b200.settings import Settings

P, SZ, U32, U64, I32, I64, F64 = (ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint32, ctypes.c_uint64,
                                  ctypes.c_int32, ctypes.c_int64, ctypes.c_double)


class _Master:
    def __init__(self):
        self.side, self.point_group, self.space_group, self.laue = 201, 32, 225, "o"
        self.voltage_kv, self.name = 20.0, "Ni_master_20kV"

    def rotations(self):
        return np.array([[1.0, 0, 0, 0], [0, 0, 0, 1.0]])  # the identity and 180° about z


class _Phase:
    def __init__(self):
        self.master = _Master()


class _Engine:
    def __init__(self):
        self.set = Settings()
        self.geo = Geometry()
        self.phases = [_Phase()]
        self.bands = {}
        self.patterns = None
        self.pixel = None
        self.scan_source = None
        self.res = None
        self.pc_history = []
        self.plane_points = None
        self.steps = 0

    def index_step_run(self):
        self.steps += 1
        return max(0, 3 - self.steps)

    def index_cells(self, cells, bandwidth, method, grid):
        r = np.zeros((len(self.phases), len(cells), 8), np.float32)
        r[..., 0] = 1.0
        r[..., 4] = cells / 10.0
        return r


class _Solver:
    """What ze_abi reaches of the package's Solver, without a device."""

    def __init__(self):
        self._e = _Engine()
        self._events = []
        self.given = []

    def _call(self, what, fn, *a, **k):
        return fn(*a, **k)

    def configure(self, **kw):
        self._e.set.apply(kw)
        self._events.append({"kind": "log", "text": f"configured {sorted(kw)}"})

    @property
    def settings(self):
        return self._e.set.as_dict()

    def events(self):
        out, self._events = self._events, []
        return out

    def set_patterns(self, a):
        self._e.patterns = a
        self._e.pixel = {np.dtype(np.uint8): 0, np.dtype(np.uint16): 1, np.dtype(np.float32): 2}[a.dtype]
        n = a.shape[0] * a.shape[1]
        self._e.res = {"quat": np.tile(np.array([1, 0, 0, 0], np.float32), (n, 1)),
                       "ncc": np.arange(n, dtype=np.float32) / n, "nmi": np.full(n, 0.5, np.float32),
                       "phase": np.where(np.arange(n) % 2 == 0, 0, -1).astype(np.int32),
                       "z": np.full(n, 3.0, np.float32), "sweep": np.zeros(n, np.int32),
                       "euler": np.full((n, 3), 0.25, np.float32)}

    @property
    def scan(self):
        r, c, h, w = self._e.patterns.shape
        return {"rows": r, "cols": c, "pattern_shape": (h, w), "has_background": False, "has_pc": False,
                "has_px": False, "voltage_kv": float("nan")}

    def set_geometry(self, **fields):
        self.given.append(fields)
        self._e.geo.given(fields, Geometry())

    def lattice(self, want):
        return np.arange(0, 2 * int(want), 2, dtype=np.uint64)

    def index_begin(self):
        self._e.steps = 0

    @property
    def index_status(self):
        return {"sweep": 0, "sweeps": 1, "bandwidth": 64, "dict_grid": 30, "done": 7, "total": 12, "region": 12,
                "accepted": 5, "method": "spherical"}

    def fit_patterns(self):
        return (np.array([3, 5], np.uint64), np.array([0, 0], np.int32),
                np.array([[1, 0, 0, 0], [0, 1, 0, 0]], np.float32), np.array([0.5, 0.6], np.float32))


@pytest.fixture(scope="module")
def lib():
    lib = ctypes.CDLL(str(build.build_abi()))
    for name, args, res in (
            ("ze_error", [P, ctypes.c_char_p, SZ], SZ), ("ze_configure", [P, ctypes.c_char_p, SZ], I32),
            ("ze_settings", [P, ctypes.c_char_p, SZ], SZ), ("ze_events", [P, ctypes.c_char_p, SZ], SZ),
            ("ze_set_patterns", [P, P, SZ, U32, U32, U32, U32, U32], I32),
            ("ze_scan_info", [P, ctypes.POINTER(Z.ScanInfo)], None), ("ze_scan_format", [P, ctypes.c_char_p, SZ], SZ),
            ("ze_get_geometry", [P, ctypes.POINTER(Z.Geometry)], None),
            ("ze_set_geometry", [P, ctypes.POINTER(Z.Geometry)], None),
            ("ze_phase_count", [P], U32), ("ze_phase_info", [P, U32, ctypes.POINTER(Z.PhaseInfo)], I32),
            ("ze_lattice", [P, U32, P, SZ], I64), ("ze_index_begin", [P], I32), ("ze_index_step", [P], I64),
            ("ze_index_status", [P, ctypes.POINTER(Z.IndexStatus)], None), ("ze_sweep", [P, U32, P], None),
            ("ze_index_cells", [P, P, SZ, P, SZ], I32), ("ze_results", [P, U32, P, SZ], I64),
            ("ze_fit_patterns", [P, P, P, P, P, SZ], I32), ("ze_reduce", [P, U32, P, P], None),
            ("ze_disorientation", [P, U32, P, P], F64), ("ze_sim_run", [P, P], I32),
            ("ze_set_frame", [P, ctypes.c_char_p, SZ], I32), ("ze_compile_wgsl", [P, P, SZ, P, SZ, ctypes.c_char_p, SZ], I32)):
        fn = getattr(lib, name)
        fn.argtypes, fn.restype = args, res
    return lib


@pytest.fixture()
def eng():
    h = 0x7F00
    Z._handles[h] = Z._Handle(_Solver())
    yield h, Z._handles[h].s
    Z._handles.pop(h, None)


def _err(lib, h):
    buf = ctypes.create_string_buffer(1024)
    n = lib.ze_error(h, buf, 1024)
    return buf.raw[:n].decode()


def test_settings_events_and_the_error_channel(lib, eng):
    h, s = eng
    j = b'{"bandwidth": 32, "sweeps": 2}'
    assert lib.ze_configure(h, j, len(j)) == 0 and _err(lib, h) == ""
    # the size it needs, then the copy
    need = lib.ze_settings(h, None, 0)
    buf = ctypes.create_string_buffer(need)
    assert lib.ze_settings(h, buf, need) == need
    got = json.loads(buf.raw[:need])
    assert got["bandwidth"] == 32 and got["sweeps"] == 2
    # events in whole lines: a buffer that holds one line at a time hands them out one by one, and a
    # line longer than the whole buffer is dropped without ending the others
    s._events += [{"kind": "log", "text": "a" * 20}, {"kind": "log", "text": "x" * 200},
                  {"kind": "log", "text": "b" * 20}]

    def drain(cap):
        small = ctypes.create_string_buffer(cap)
        texts = []
        while True:
            n = lib.ze_events(h, small, cap)
            if n == 0:
                return texts
            texts += [json.loads(x)["text"] for x in small.raw[:n].decode().splitlines()]

    assert drain(80) == ["configured ['bandwidth', 'sweeps']", "a" * 20, "b" * 20]
    # a refused setting: a negative code, the message once
    bad = b'{"bandwidth": "wide"}'
    assert lib.ze_configure(h, bad, len(bad)) < 0
    msg = _err(lib, h)
    assert msg.startswith("configure") and _err(lib, h) == ""
    # a part this engine does not build
    assert lib.ze_sim_run(h, None) < 0 and "not part of this engine" in _err(lib, h)
    j = b'{"axes": [2, 1, 3], "active": false, "crystal": "x_a_z_cstar"}'  # left-handed: no convention
    assert lib.ze_set_frame(h, j, len(j)) < 0 and "InvalidFrame" in _err(lib, h)
    j = b'{"axes": [2, 1, -3], "active": false, "crystal": "x_a_z_cstar"}'
    assert lib.ze_set_frame(h, j, len(j)) == 0 and s._e.convention.axes == (2, 1, -3)
    own = b'{"axes": [1, 2, 3], "active": false, "crystal": "x_a_z_cstar"}'
    assert lib.ze_set_frame(h, own, len(own)) == 0
    msg = ctypes.create_string_buffer(256)
    assert lib.ze_compile_wgsl(h, None, 0, None, 0, msg, 256) > 0 and b"CUDA" in msg.value
    # an unknown handle touches nothing
    assert lib.ze_configure(0x10, b"{}", 2) < 0


def test_patterns_scan_and_results(lib, eng):
    h, s = eng
    pats = np.arange(3 * 4 * 6 * 5, dtype=np.uint16).reshape(3, 4, 6, 5)
    buf = pats.copy()
    assert lib.ze_set_patterns(h, buf.ctypes.data, buf.nbytes, 1, 3, 4, 6, 5) == 0
    buf[:] = 0  # the engine has its own copy
    assert np.array_equal(s._e.patterns, pats)
    assert lib.ze_set_patterns(h, buf.ctypes.data, buf.nbytes - 2, 1, 3, 4, 6, 5) < 0
    assert "BadLength" in _err(lib, h)
    si = Z.ScanInfo()
    lib.ze_scan_info(h, ctypes.byref(si))
    assert (si.rows, si.cols, si.pat_h, si.pat_w, si.pixel, si.format, si.bytes) == (3, 4, 6, 5, 1, 100, pats.nbytes)
    fb = ctypes.create_string_buffer(32)
    k = lib.ze_scan_format(h, fb, 32)
    assert fb.raw[:k] == b"memory"
    n = 12
    res = s._e.res
    for kind, key, dt, width in ((0, "quat", np.float32, 4), (1, "ncc", np.float32, 1), (2, "nmi", np.float32, 1),
                                 (3, "phase", np.int32, 1), (5, "z", np.float32, 1), (6, "sweep", np.int32, 1)):
        out = np.empty(n * width, dt)
        assert lib.ze_results(h, kind, out.ctypes.data, out.nbytes) == n * width
        assert np.array_equal(out.reshape(res[key].shape), res[key]), key
    eu = np.empty(n * 3, np.float32)
    assert lib.ze_results(h, 4, eu.ctypes.data, eu.nbytes) == 3 * n
    want = res["euler"].copy()
    want[res["phase"] < 0] = 0  # cells not indexed: zero angles, as the reference writes them
    assert np.array_equal(eu.reshape(n, 3), want)
    small = np.empty(3, np.float32)
    assert lib.ze_results(h, 1, small.ctypes.data, small.nbytes) < 0 and "BufferTooSmall" in _err(lib, h)
    assert lib.ze_results(h, 9, small.ctypes.data, small.nbytes) < 0 and "UnknownKind" in _err(lib, h)
    # index_cells: one record per phase per cell, the length checked
    cells = np.array([2, 7], np.uint64)
    rec = np.empty(2 * 8, np.float32)
    assert lib.ze_index_cells(h, cells.ctypes.data, 2, rec.ctypes.data, rec.size) == 0
    assert np.allclose(rec.reshape(1, 2, 8)[0, :, 4], [0.2, 0.7])
    assert lib.ze_index_cells(h, cells.ctypes.data, 2, rec.ctypes.data, rec.size - 1) < 0


def test_geometry_round_trip_gives_only_what_changed(lib, eng):
    h, s = eng
    g = Z.Geometry()
    lib.ze_get_geometry(h, ctypes.byref(g))
    assert list(g.pc) == [0.5, 0.5, 0.5] and g.sample_tilt_deg == 70.0
    g.pc[:] = (0.48, 0.31, 0.6)
    g.detector_tilt_deg = 4.0
    lib.ze_set_geometry(h, ctypes.byref(g))
    assert _err(lib, h) == ""
    g2 = Z.Geometry()
    lib.ze_get_geometry(h, ctypes.byref(g2))
    assert list(g2.pc) == [0.48, 0.31, 0.6] and g2.detector_tilt_deg == 4.0 and g2.sample_tilt_deg == 70.0


def test_phases_indexing_and_fits(lib, eng):
    h, s = eng
    assert lib.ze_phase_count(h) == 1
    pi = Z.PhaseInfo()
    assert lib.ze_phase_info(h, 0, ctypes.byref(pi)) == 0
    assert (pi.side, pi.point_group, pi.space_group, pi.laue, pi.name) == (201, 32, 225, 11, b"Ni_master_20kV")
    assert lib.ze_phase_info(h, 3, ctypes.byref(pi)) < 0 and "NoSuchPhase" in _err(lib, h)
    # the lattice: the count first, then the cells
    n = lib.ze_lattice(h, 5, None, 0)
    out = np.empty(n, np.uint64)
    assert n == 5 and lib.ze_lattice(h, 5, out.ctypes.data, n) == 5 and list(out) == [0, 2, 4, 6, 8]
    # steps until none is left, and where they stand
    assert lib.ze_index_begin(h) == 0
    left = [lib.ze_index_step(h) for _ in range(3)]
    assert left == [2, 1, 0]
    st = Z.IndexStatus()
    lib.ze_index_status(h, ctypes.byref(st))
    assert (st.done, st.total, st.region, st.accepted, st.bandwidth, st.method) == (7, 12, 12, 5, 64, 0)
    sw = np.empty(3, np.uint32)
    lib.ze_sweep(h, 0, sw.ctypes.data)
    assert list(sw) == [64, 30, 0]
    # the last fit's patterns: the count, then the arrays
    k = lib.ze_fit_patterns(h, None, None, None, None, 0)
    cells, ph, q, ncc = np.empty(k, np.uint64), np.empty(k, np.int32), np.empty(4 * k, np.float32), np.empty(k, np.float32)
    assert k == 2 and lib.ze_fit_patterns(h, cells.ctypes.data, ph.ctypes.data, q.ctypes.data, ncc.ctypes.data, k) == 2
    assert list(cells) == [3, 5] and np.allclose(ncc, [0.5, 0.6])
    # an orientation reduced by the phase's rotations, and a disorientation under them
    qz = np.array([0.0, 0.0, 0.0, 1.0], np.float32)  # 180° about z: the identity under this phase
    eu = np.empty(3, np.float64)
    lib.ze_reduce(h, 0, qz.ctypes.data, eu.ctypes.data)
    assert np.allclose(np.abs(qz), [1, 0, 0, 0]) and np.allclose(eu, 0, atol=1e-12)
    a = np.array([1, 0, 0, 0], np.float32)
    b = np.array([0, 0, 0, 1], np.float32)
    assert lib.ze_disorientation(h, 0, a.ctypes.data, b.ctypes.data) == pytest.approx(0.0, abs=1e-6)
    assert lib.ze_disorientation(h, 7, a.ctypes.data, b.ctypes.data) == pytest.approx(np.pi, abs=1e-6)


class _FitSolver(_Solver):
    """The stand-in with a pattern-centre search, a plane fit, an NLPAR view and an export."""

    def __init__(self):
        super().__init__()
        ax = (np.array([0.4, 0.5, 0.6]), np.array([0.2, 0.3]), np.array([0.55]))
        self._e.pc_history = [{"axes": ax, "scores": np.arange(6, dtype=np.float32), "best": 4, "walked": True,
                               "pat_best": np.array([1, 4, 5], np.uint32), "pat_ncc": np.array([0.3, 0.4, 0.5], np.float32),
                               "pat_scores": np.arange(18, dtype=np.float32), "density": np.ones(6, np.float32),
                               "peak": (1.5, 0.5, 0.0), "ballots": 3, "inliers": 2}]
        self._e.plane_points = {"cells": np.array([3, 9], np.uint64), "pc": np.array([[0.5, 0.3, 0.6], [0.51, 0.31, 0.61]]),
                                "fit": np.array([[0.5, 0.3, 0.6], [0.5, 0.3, 0.6]]), "ncc": np.array([0.7, 0.8]),
                                "used": np.array([True, False])}

    def fit_pc(self):
        return {"pc": [0.5, 0.3, 0.6], "start": [0.5, 0.5, 0.5], "score": 0.8, "start_score": 0.6, "n_patterns": 25,
                "n_candidates": 125, "levels": 3, "at_border": False}

    def fit_plane(self):
        return {"plane": np.arange(12, dtype=np.float64).reshape(4, 3), "kind": "affine", "frame": "follow",
                "model": "line", "method": "points", "models": {"centre": {"cv": 0.2, "cv_se": 0.01}},
                "pc": [0.5, 0.3, 0.6], "pc_se": [1e-3, 2e-3, 3e-3], "start_pc": [0.5, 0.5, 0.5], "rot": [0.0, 0.01, 0.0],
                "n_patterns": 40, "n_used": 38, "rmsd": [1e-3, 1e-3, 2e-3], "ncc": 0.8, "start_ncc": 0.7, "iterations": 6,
                "said": {"rot": [0.0, 0.02, 0.0], "rot_se": [1e-3] * 3, "step": [1.0, 1.01], "step_se": [1e-3, 1e-3],
                         "skew": 0.001, "skew_se": 1e-4, "blocks": 5}}

    def nlpar_view(self):
        return {"noise": 2.0, "left": 0.4, "own": 0.3, "shares": np.arange(9, dtype=np.float32).reshape(3, 3)}

    def pattern_stats(self, cells):
        c = np.asarray(cells, np.float32)
        return c + 0.5, c * 2

    def master(self, phase):
        return np.arange(2 * 201 * 201, dtype=np.float32).reshape(2, 201, 201)

    def export_text(self, kind):
        return f"# {kind} header\n1 2 3\n"


@pytest.fixture()
def fit_eng():
    h = 0x7F10
    Z._handles[h] = Z._Handle(_FitSolver())
    yield h, Z._handles[h].s
    Z._handles.pop(h, None)


def _fn(lib, name, args, res):
    fn = getattr(lib, name)
    fn.argtypes, fn.restype = args, res
    return fn


def test_fits_grids_and_exports(lib, fit_eng):
    h, s = fit_eng
    pr = Z.PcResult()
    assert _fn(lib, "ze_fit_pc", [P, ctypes.POINTER(Z.PcResult)], I32)(h, ctypes.byref(pr)) == 0
    assert list(pr.pc) == [0.5, 0.3, 0.6] and (pr.n_patterns, pr.n_candidates, pr.levels, pr.at_border) == (25, 125, 3, 0)
    # the last grid: its shape and size first, then its values
    shape = np.empty(3, np.uint32)
    scores_fn = _fn(lib, "ze_pc_scores", [P, P, P, SZ, P, SZ], I32)
    assert scores_fn(h, shape.ctypes.data, None, 0, None, 0) == 6 and list(shape) == [1, 2, 3]
    axes, sc = np.empty(6), np.empty(6, np.float32)
    assert scores_fn(h, shape.ctypes.data, axes.ctypes.data, 6, sc.ctypes.data, 6) == 6
    assert np.allclose(axes, [0.4, 0.5, 0.6, 0.2, 0.3, 0.55]) and np.array_equal(sc, np.arange(6))
    assert _fn(lib, "ze_pc_level_count", [P], U32)(h) == 1
    info = np.empty(2, np.uint32)
    best, ncc = np.empty(3, np.uint32), np.empty(3, np.float32)
    level = _fn(lib, "ze_pc_level", [P, U32, P, P, P, SZ, P, SZ, P, P, SZ], I32)
    assert level(h, 0, shape.ctypes.data, info.ctypes.data, axes.ctypes.data, 6, sc.ctypes.data, 6, best.ctypes.data,
                 ncc.ctypes.data, 3) == 6
    assert list(info) == [4, 1] and list(best) == [1, 4, 5] and np.allclose(ncc, [0.3, 0.4, 0.5])
    assert level(h, 1, shape.ctypes.data, info.ctypes.data, None, 0, None, 0, None, None, 0) == -1
    per = np.empty(18, np.float32)
    assert _fn(lib, "ze_pc_level_scores", [P, U32, P, SZ], I32)(h, 0, per.ctypes.data, 18) == 18
    dinfo, den = np.empty(5), np.empty(6, np.float32)
    assert _fn(lib, "ze_pc_level_ballots", [P, U32, P, SZ, P], I32)(h, 0, den.ctypes.data, 6, dinfo.ctypes.data) == 6
    assert list(dinfo) == [1.5, 0.5, 0.0, 3.0, 2.0] and np.array_equal(den, np.ones(6))
    # the plane fit into planefit.zig's struct; its points
    r = Z.PlaneResult()
    assert _fn(lib, "ze_fit_plane", [P, ctypes.POINTER(Z.PlaneResult)], I32)(h, ctypes.byref(r)) == 0
    assert list(r.plane) == list(range(12)) and (r.kind, r.frame, r.model, r.method, r.compared) == (1, 1, 1, 1, 1)
    assert (r.n_patterns, r.n_used, r.iterations, r.blocks) == (40, 38, 6, 5) and r.cv[0] == 0.2 and r.cv[1] == 0.0
    assert list(r.step) == [1.0, 1.01] and r.skew == 0.001 and list(r.pc_se) == [1e-3, 2e-3, 3e-3]
    pts_fn = _fn(lib, "ze_plane_points", [P, P, SZ], SZ)
    n = pts_fn(h, None, 0)
    pts = (Z.PlanePoint * n)()
    assert n == 2 and pts_fn(h, ctypes.cast(pts, P), n) == 2
    assert (pts[0].cell, pts[1].cell, pts[0].used, pts[1].used) == (3, 9, 1, 0) and list(pts[1].pc) == [0.51, 0.31, 0.61]
    # NLPAR's view: its side first, then the shares
    out3 = np.empty(3, np.float32)
    view = _fn(lib, "ze_nlpar_view", [P, P, P, SZ], U32)
    assert view(h, out3.ctypes.data, None, 0) == 3 and np.allclose(out3, [2.0, 0.4, 0.3])
    shares = np.empty(9, np.float32)
    assert view(h, out3.ctypes.data, shares.ctypes.data, 9) == 3 and np.array_equal(shares, np.arange(9))
    # statistics of given cells, two values a cell; a buffer too small is refused
    cells = np.array([2, 5], np.uint64)
    st = np.empty(4, np.float32)
    stats = _fn(lib, "ze_pattern_stats", [P, P, SZ, P, SZ], I32)
    assert stats(h, cells.ctypes.data, 2, st.ctypes.data, 4) == 0 and list(st) == [2.5, 4.0, 5.5, 10.0]
    assert stats(h, cells.ctypes.data, 2, st.ctypes.data, 3) < 0 and "BufferTooSmall" in _err(lib, h)
    # the master image; the export's size, then its text
    img = np.empty(2 * 201 * 201, np.float32)
    mi = _fn(lib, "ze_master_image", [P, U32, P, SZ], I32)
    assert mi(h, 0, img.ctypes.data, img.size) == 0 and img[-1] == img.size - 1
    assert mi(h, 0, img.ctypes.data, 10) < 0 and "BufferTooSmall" in _err(lib, h)
    ex = _fn(lib, "ze_export", [P, U32, P, SZ], I64)
    size = ex(h, 1, None, 0)
    text = ctypes.create_string_buffer(size)
    assert ex(h, 1, text, size) == size and text.raw[:size] == b"# ctf header\n1 2 3\n"
    assert ex(h, 5, None, 0) < 0 and "UnknownKind" in _err(lib, h)
    # the search given by the caller is checked before it runs
    rec = np.empty(16, np.float32)
    by = _fn(lib, "ze_index_cells_by", [P, P, SZ, U32, U32, U32, P, SZ], I32)
    assert by(h, cells.ctypes.data, 2, 0, 4, 30, rec.ctypes.data, 16) < 0 and "BadSetting" in _err(lib, h)
    assert by(h, cells.ctypes.data, 2, 0, 32, 30, rec.ctypes.data, 16) == 0
