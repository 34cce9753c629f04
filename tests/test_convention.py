"""Orientation conventions (convention.zig), on the CPU: the crystal axes on hexagonal, cubic and
monoclinic cells; a convention's two directions undoing each other; `identify` finding a planted
convention among all 192 and measuring the misorientation left and its change over the map;
the exports written in a convention; and the Solver's and the reference's C ABI's frame calls
(ze_frame, ze_set_frame, ze_identify_frame) over an engine without a device."""
import ctypes
import json
import math

import numpy as np
import pytest

from zebsdsolve_b200 import build, convention as C, output as O, rotations as R, ze_abi as Z

HEX = (3.232, 3.232, 5.148, 90.0, 90.0, 120.0)


def _hex_rotations():
    z = [R.exp_map([0, 0, k * math.pi / 3]) for k in range(6)]
    return np.array(z + [R.qmul(q, R.exp_map([math.pi, 0, 0])) for q in z])


def test_crystal_axes_on_cells():
    t = C.crystal_rotation("x_astar_z_c", HEX)
    v = R.qapply(R.qconj(t), np.array([1.0, 0, 0]))
    assert v[0] == pytest.approx(math.sqrt(3) / 2, abs=1e-12) and v[1] == pytest.approx(0.5, abs=1e-12)
    y = C.crystal_rotation("y_b_z_cstar", HEX)  # b ⊥ a*, c* ∥ c on a hexagonal cell: the same axes
    assert C._apart([[1.0, 0, 0, 0]], t[None], y[None])[0] < 1e-7
    for c in C.CRYSTAL_AXES:  # on a cube every description is the masters' own
        assert C._apart([[1.0, 0, 0, 0]], C.crystal_rotation(c, (3.52, 3.52, 3.52, 90, 90, 90))[None],
                        np.array([[1.0, 0, 0, 0]]))[0] < 1e-7
    mono = C.crystal_rotation("x_astar_z_c", (5.1, 5.2, 5.3, 90, 99.2, 90))  # a* is a turned β − 90° about b
    assert 2 * math.acos(min(1.0, abs(mono[0]))) == pytest.approx(math.radians(9.2), abs=1e-9)
    assert C.crystal_rotation("x_astar_z_c", None) is None and C.crystal_rotation("x_a_z_cstar", None) is not None


def test_a_frame_undoes_itself_and_describes_itself():
    f = C.Frame((2, -1, 3), True, "x_astar_z_c")
    assert f.valid() and not C.Frame((2, 1, 3)).valid() and not C.Frame((1, 1, 3)).valid()
    c = f.crystal_of((3.2, 3.2, 5.1, 90, 90, 120))
    q = R.qstd(R.exp_map(np.random.default_rng(0).normal(size=(50, 3))))
    back = f.from_frame(f.to_frame(q, c), c)
    assert np.allclose(np.abs(np.sum(back * q, 1)), 1, atol=1e-12)
    assert f.describe() == "X +y Y -x Z +z, active, X||a* Z||c" and C.Frame().describe() == "X +x Y +y Z +z, passive, X||a Z||c*"
    assert C.Frame.from_dict(f.as_dict()) == f
    with pytest.raises(C.ConventionError, match="InvalidFrame"):
        C.Frame.from_dict({"axes": [2, 1, 3]})
    with pytest.raises(C.ConventionError, match="InvalidFrame"):
        C.Frame.from_dict({"crystal": "sideways"})


def _planted(active, n=600, cols=30, seed=7):
    """A reference in a planted convention: the engine's orientations seen with sample axes turned
    by m0 at the map's middle, changing by dm from the first row to the last, a symmetric
    equivalent, 0.003 rad of noise, and every tenth cell wrong."""
    rng = np.random.default_rng(seed)
    sym = _hex_rotations()
    planted = C.Frame((2, -1, 3), active, "x_astar_z_c")
    c = planted.crystal_of(HEX)
    m0, dm = np.array([0.02, -0.01, 0.005]), np.array([0.0, 0.03, 0.0])
    q = R.qstd(R.exp_map(3 * (rng.random((n, 3)) - 0.5)))
    u = (np.arange(n) // cols) / (n // cols - 1) - 0.5
    m = R.exp_map(m0 + u[:, None] * dm)
    seen = R.qmul(q, R.qconj(m))
    g = sym[rng.integers(0, len(sym), n)]
    noise = R.exp_map(0.003 * rng.normal(size=(n, 3)))
    w = planted.to_frame(R.qmul(noise, R.qmul(g, seen)), c)
    wrong = np.arange(n) % 10 == 0
    w[wrong] = R.exp_map(rng.random((wrong.sum(), 3)))
    return q.astype(np.float32), R.to_bunge(w), planted, m0, dm, sym


@pytest.mark.parametrize("active", [False, True])
def test_identify_finds_a_planted_convention(active):
    q, eu, planted, m0, dm, sym = _planted(active)
    n = len(q)
    frame, out = C.identify(q, np.zeros(n, np.int32), 30, eu, np.full(n, 3), [(sym, HEX)])
    assert frame == planted and out["matched"] == [3] and out["cells"] == n
    assert np.allclose(out["misorientation"], m0, atol=1e-3)
    assert np.allclose(out["misorientation_rows"], dm, atol=2e-3) and np.allclose(out["misorientation_cols"], 0, atol=2e-3)
    assert out["median_deg"] < 3 and out["runner_up_deg"] > 10 and 0.85 < out["within"] <= 0.91


def test_identify_refusals_and_labels():
    q, eu, planted, m0, dm, sym = _planted(False, n=60)
    with pytest.raises(C.ConventionError, match="TooFewCommonCells"):
        C.identify(q, np.full(60, -1), 30, eu, np.zeros(60), [(sym, HEX)])
    with pytest.raises(C.ConventionError, match="BadLength"):
        C.identify(q, np.zeros(60), 30, eu[:59], np.zeros(60), [(sym, HEX)])
    with pytest.raises(C.ConventionError, match="NoPhases"):
        C.identify(q, np.zeros(60), 30, eu, np.zeros(60), [])
    # the reference's most frequent label where the engine found the phase; ties to the smaller
    assert C.match_labels([0, 0, 0, 1, 1, -1], [5, 5, 2, 7, 4, 9], 2)[:3] == [5, 4, -1]


def test_exports_write_in_the_frame():
    q, eu, planted, m0, dm, sym = _planted(True, n=12, cols=4)
    res = {"quat": q, "ncc": np.full(12, 0.5, np.float32), "nmi": np.full(12, 0.4, np.float32),
           "phase": np.where(np.arange(12) == 5, -1, 0).astype(np.int32)}
    phases = [{"name": "Ti", "laue": "d6", "lattice": HEX, "space_group": 194}]

    class G:
        pc, step_x_um, step_y_um, sample_tilt_deg = (0.5, 0.5, 0.6), 1.0, 1.0, 70.0
    text = O.export_text("ang", res, phases, G, 3, 4, 60, 60, frame=planted)
    assert f"# FRAME: {planted.describe()}" in text
    rows = np.loadtxt(text.splitlines(), comments="#")
    back = planted.from_frame(C.from_bunge(rows[:, :3]), planted.crystal_of(HEX))
    ok = res["phase"] >= 0
    assert np.allclose(np.abs(np.sum(back[ok] * R.qstd(q[ok].astype(np.float64)), 1)), 1, atol=1e-8)
    assert np.allclose(rows[~ok, :3], 12.56637)
    ctf = O.export_text("ctf", res, phases, G, 3, 4, 60, 60, frame=planted)
    assert f"zebsdsolve; frame {planted.describe()}" in ctf
    with pytest.raises(O.ExportError, match="MissingPhaseLattice"):
        O.export_text("ang", res, [dict(phases[0], lattice=None)], G, 3, 4, 60, 60, frame=planted)


class _Master:
    def __init__(self, rots, lattice):
        self._r, self.lattice, self.name, self.laue, self.space_group = rots, lattice, "Ti", "d6", 194

    def rotations(self):
        return self._r


class _Phase:
    def __init__(self, m):
        self.master = m


def _solver():
    import zebsdsolve_b200 as ze
    from zebsdsolve_b200 import engine as E
    from zebsdsolve_b200.settings import Settings

    s = ze.Solver.__new__(ze.Solver)
    e = E.Engine.__new__(E.Engine)
    e.set, e.geo, e._resident, e.patterns, e.events = Settings(), E.Geometry(), None, None, []
    s._e = e
    return s


def test_solver_and_c_abi_frame_calls():
    q, eu, planted, m0, dm, sym = _planted(True)
    s = _solver()
    s.set_patterns(np.zeros((20, 30, 6, 5), np.uint8))
    s._e.phases = [_Phase(_Master(sym, HEX))]
    s._e.res["quat"][:] = q
    s._e.res["phase"][:] = 0
    lib = ctypes.CDLL(str(build.build_abi()))
    P, SZ = ctypes.c_void_p, ctypes.c_size_t
    lib.ze_frame.argtypes, lib.ze_frame.restype = [P, ctypes.c_char_p, SZ], SZ
    lib.ze_set_frame.argtypes, lib.ze_set_frame.restype = [P, ctypes.c_char_p, SZ], ctypes.c_int32
    lib.ze_identify_frame.argtypes = [P, P, P, ctypes.c_uint64, ctypes.c_char_p, SZ]
    lib.ze_identify_frame.restype = ctypes.c_int64
    lib.ze_error.argtypes, lib.ze_error.restype = [P, ctypes.c_char_p, SZ], SZ
    h = 0x7F30
    Z._handles[h] = Z._Handle(s)
    try:
        buf = ctypes.create_string_buffer(8192)
        k = lib.ze_frame(h, buf, 8192)
        assert json.loads(buf.raw[:k]) == C.Frame().as_dict() == s.frame
        # no stored orientations from memory
        assert lib.ze_identify_frame(h, None, None, 0, buf, 8192) < 0
        k = lib.ze_error(h, buf, 8192)
        assert b"NoStoredOrientations" in buf.raw[:k]
        ph = np.full(len(q), 3, np.int32)
        assert lib.ze_identify_frame(h, eu.ctypes.data, ph.ctypes.data, len(q), buf, 10) < 0  # too small
        k = lib.ze_identify_frame(h, eu.ctypes.data, ph.ctypes.data, len(q), buf, 8192)
        got = json.loads(buf.raw[:k])
        assert got["installed"] and got["frame"] == planted.as_dict() and got["matched"] == [3]
        assert np.allclose(got["misorientation"], m0, atol=1e-3)
        assert s.frame == planted.as_dict()  # installed: the exports write in it
        assert any("frame of the stored orientations" in ev.get("text", "") for ev in s._e.events)
        j = json.dumps({"axes": [2, 1, 3]}).encode()
        assert lib.ze_set_frame(h, j, len(j)) < 0
        k = lib.ze_error(h, buf, 8192)
        assert b"InvalidFrame" in buf.raw[:k]
        assert lib.ze_set_frame(h, b"", 0) == 0 and s.frame == C.Frame().as_dict()
        j = json.dumps({"axes": [-1, -2, 3], "active": False, "crystal": "y_b_z_cstar", "text": "x"}).encode()
        assert lib.ze_set_frame(h, j, len(j)) == 0 and s.frame["axes"] == [-1, -2, 3]
        s.set_patterns(np.zeros((20, 30, 6, 5), np.uint8))  # a new scan: the engine's own again
        assert s.frame == C.Frame().as_dict()
        # (the convention is kept apart from the engine's detector frame, a method of its own)
        assert callable(s._e.frame) and s._e.frame.__func__ is type(s._e).frame
    finally:
        Z._handles.pop(h, None)
