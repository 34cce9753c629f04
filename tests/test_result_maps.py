"""The result maps (output.zig:15-84), on the CPU: the score maps (NCC, NMI, z) as gray between
the indexed cells' extremes, the phase and sweep maps in the reference's palette, cells not
indexed transparent black, checked against a cell-by-cell restatement; then through the
Solver and the reference's C ABI (ze_map) behind a stand-in engine, its length and kind checks."""
import ctypes
import math

import numpy as np
import pytest

from zebsdsolve_b200 import build, output as O, ze_abi as Z
from test_ze_abi_host import _Solver


def _cellwise(kind, res):
    """output.zig:15-84 one cell at a time (Python floats in float32 steps)."""
    n = len(res["ncc"])
    key = {3: "ncc", 4: "nmi", 6: "z"}.get(kind)
    lo, hi = math.inf, -math.inf
    if key:
        for i in range(n):
            v = float(res[key][i])
            if res["phase"][i] >= 0 and not math.isnan(v):
                lo, hi = min(lo, v), max(hi, v)
        if not hi > lo:
            hi = lo + 1
    out = np.zeros((n, 4), np.uint8)
    for i in range(n):
        ph = int(res["phase"][i])
        if ph < 0:
            continue
        if key:
            t = np.float32((np.float32(res[key][i]) - np.float32(lo)) / (np.float32(hi) - np.float32(lo)))
            t = 1.0 if math.isnan(t) else min(max(float(t), 0.0), 1.0)
            g = int(math.floor(255 * t + 0.5))
            out[i, :3] = g
        elif kind == 5:
            out[i, :3] = O.PALETTE[ph % 8]
        else:
            sw = int(res["sweep"][i])
            out[i, :3] = (0x3a, 0x3a, 0x3e) if sw < 0 else O.PALETTE[sw % 8]
        out[i, 3] = 255
    return out


def _res(n=40, seed=0):
    rng = np.random.default_rng(seed)
    return {"ncc": rng.random(n).astype(np.float32), "nmi": rng.normal(0.3, 0.1, n).astype(np.float32),
            "z": rng.normal(20, 8, n).astype(np.float32), "phase": rng.integers(-1, 11, n).astype(np.int32),
            "sweep": rng.integers(-1, 12, n).astype(np.int32), "quat": np.zeros((n, 4), np.float32)}


@pytest.mark.parametrize("kind", [3, 4, 5, 6, 7])
def test_maps_against_the_cell_by_cell_restatement(kind):
    for seed in range(3):
        res = _res(seed=seed)
        got = O.result_map(kind, res)
        assert np.array_equal(got, _cellwise(kind, res)), (kind, seed)
        assert (got[res["phase"] < 0] == 0).all() and (got[res["phase"] >= 0, 3] == 255).all()
    # one indexed value: a single level; the extremes map to black and white
    res = _res(8)
    res["phase"][:] = -1
    res["phase"][3] = 0
    if kind in (3, 4, 6):
        assert (O.result_map(kind, res)[3, :3] == 0).all()
        res["phase"][:] = 0
        g = O.result_map(kind, res)[:, 0]
        v = res[{3: "ncc", 4: "nmi", 6: "z"}[kind]]
        assert g[np.argmin(v)] == 0 and g[np.argmax(v)] == 255


def test_map_kinds_and_palette():
    res = _res()
    with pytest.raises(ValueError, match="UnknownKind"):
        O.result_map(8, res)
    with pytest.raises(NotImplementedError, match="IPF"):
        O.result_map(2, res)
    res["phase"][:4], res["sweep"][:4] = [0, 1, 8, 9], [-1, 0, 3, 11]
    assert O.result_map(5, res)[:4, :3].tolist() == [O.PALETTE[k].tolist() for k in (0, 1, 0, 1)]
    assert O.result_map(7, res)[:4, :3].tolist() == [[0x3a, 0x3a, 0x3e]] + [O.PALETTE[k].tolist() for k in (0, 3, 3)]


def test_solver_and_c_abi_maps():
    lib = ctypes.CDLL(str(build.build_abi()))
    P, SZ = ctypes.c_void_p, ctypes.c_size_t
    lib.ze_map.argtypes, lib.ze_map.restype = [P, ctypes.c_uint32, P, SZ], ctypes.c_int32
    lib.ze_error.argtypes, lib.ze_error.restype = [P, ctypes.c_char_p, SZ], SZ
    h = 0x7F20
    Z._handles[h] = Z._Handle(_Solver())
    try:
        s = Z._handles[h].s
        s.set_patterns(np.zeros((3, 4, 6, 5), np.uint16))
        res = s._e.res
        for kind in (3, 4, 5, 6, 7):
            out = np.zeros(4 * 12, np.uint8)
            assert lib.ze_map(h, kind, out.ctypes.data, out.size) == 0
            assert np.array_equal(out.reshape(12, 4), O.result_map(kind, res))
        out = np.zeros(4 * 12, np.uint8)
        buf = ctypes.create_string_buffer(256)
        for kind, size, why in ((3, 47, b"BadLength"), (9, 48, b"UnknownKind"), (0, 48, b"NotImplemented")):
            assert lib.ze_map(h, kind, out.ctypes.data, size) < 0
            k = lib.ze_error(h, buf, 256)
            assert why in buf.raw[:k], (kind, buf.raw[:k])
    finally:
        Z._handles.pop(h, None)


def test_solver_map():
    import zebsdsolve_b200 as ze
    from zebsdsolve_b200 import engine as E
    from zebsdsolve_b200.settings import Settings

    s = ze.Solver.__new__(ze.Solver)
    e = E.Engine.__new__(E.Engine)
    e.set, e.geo, e._resident, e.patterns = Settings(), E.Geometry(), None, None
    s._e = e
    s.set_patterns(np.zeros((3, 4, 6, 5), np.uint8))
    e.res.update({k: v[:12] for k, v in _res(12).items() if k != "quat"})
    m = s.map("nmi")
    assert m.shape == (3, 4, 4) and np.array_equal(m.reshape(12, 4), O.result_map(4, e.res))
    with pytest.raises(ze.Error, match="UnknownKind"):
        s.map("bogus")
    with pytest.raises(ze.Error, match="IPF"):
        s.map("ipf_z")
