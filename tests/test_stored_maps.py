"""The scan readers' stored maps, on the CPU: the acquisition's quality map (band contrast, image
quality, Radon quality, pattern quality) found under the makers' names in the reference's order
and shapes (scan.zig:294-332; its tests/test_stored_overview.py cases: kikuchipy "band_contrast"
(6,), Oxford "Band Contrast" (2, 3), EDAX "IQ" (6, 1), Bruker "RadonQuality" (1, 6), EMsoft "IQ"
(6,), a wrong-shaped first name skipped for the next), an EDAX .up's image quality from its .ang,
and the maker's stored orientations (scan.zig:220-291, ang.zig:227-264); then both through the
reference's C ABI (ze_scan_overview_kind, ze_scan_overview, ze_stored_orientations) behind a
stand-in engine."""
import ctypes
import math
import struct

import numpy as np
import pytest

from h5_writer import D, Writer
from zebsdsolve_b200 import build, scan as SC, ze_abi as Z
from test_ze_abi_host import _Solver

ROWS, COLS, H, W = 2, 3, 6, 5


def _pats(n, dtype=np.uint8):
    return (np.arange(n * H * W) % 200).astype(dtype).reshape(n, H, W)


def _h5ebsd(path, vendor, extra):
    """A minimal h5ebsd file of ROWS × COLS patterns in a maker's layout, with `extra` datasets
    beside the patterns."""
    n = ROWS * COLS
    names = {"kikuchipy": ("patterns", "n_rows", "n_columns"), "bruker": ("RawPatterns", "NROWS", "NCOLS"),
             "edax": ("Pattern", "nRows", "nColumns"), "oxford": ("Processed Patterns", "Y Cells", "X Cells")}[vendor]
    data = {names[0]: D(_pats(n)), **extra}
    head = {names[1]: D(np.array([ROWS], np.int32)), names[2]: D(np.array([COLS], np.int32))}
    Writer(0, 1).write(path, {"Scan 1": {"EBSD": {"Data": data, "Header": head}}})
    return path


Q = np.arange(ROWS * COLS, dtype=np.float32) * 10 + 5


@pytest.mark.parametrize("vendor,name,shape,kind", [
    ("kikuchipy", "band_contrast", (6,), 1), ("oxford", "Band Contrast", (2, 3), 1), ("edax", "IQ", (6, 1), 2),
    ("bruker", "RadonQuality", (1, 6), 3), ("kikuchipy", "Pattern Quality", (6,), 4)])
def test_stored_overview_names_and_shapes(tmp_path, vendor, name, shape, kind):
    sc = SC.open_scan([_h5ebsd(tmp_path / "s.h5", vendor, {name: D(Q.reshape(shape))})])
    k, read = sc.info["overview"]
    assert k == kind and np.array_equal(read(), Q) and read().dtype == np.float32


def test_stored_overview_order_types_and_refusals(tmp_path):
    # a first name in the wrong shape is skipped for the next; a raster transposed is not a raster
    extra = {"Band Contrast": D(Q.reshape(3, 2)), "IQ": D(Q.astype(np.uint16))}
    k, read = SC.open_scan([_h5ebsd(tmp_path / "a.h5", "oxford", extra)]).info["overview"]
    assert k == 2 and np.array_equal(read(), Q)
    # the order, not the file's: band contrast before image quality
    extra = {"IQ": D(Q), "BandContrast": D(Q[::-1].astype(np.int64))}
    k, read = SC.open_scan([_h5ebsd(tmp_path / "b.h5", "edax", extra)]).info["overview"]
    assert k == 1 and np.array_equal(read(), Q[::-1])
    # float64 past float32's range and non-finite values read as NaN
    v = Q.astype(np.float64)
    v[1], v[4] = 1e300, np.inf
    k, read = SC.open_scan([_h5ebsd(tmp_path / "c.h5", "kikuchipy", {"iq": D(v)})]).info["overview"]
    got = read()
    assert k == 2 and np.isnan(got[[1, 4]]).all() and np.array_equal(np.delete(got, [1, 4]), np.delete(Q, [1, 4]))
    # wrong count, strings, a group of that name: none
    extra = {"IQ": D(Q[:5]), "Image Quality": D(np.array([b"abc"] * 6)), "RadonQuality": {"x": D(Q)}}
    assert SC.open_scan([_h5ebsd(tmp_path / "d.h5", "edax", extra)]).info["overview"] == (0, None)
    assert SC.open_scan([_h5ebsd(tmp_path / "e.h5", "edax", {})]).info["overview"] == (0, None)


def test_emsoft_overview(tmp_path):
    n = ROWS * COLS
    Writer(0, 1).write(tmp_path / "em.h5", {"EMData": {"EBSD": {"EBSDPatterns": D(_pats(n, np.float32)), "IQ": D(Q)}}})
    sc = SC.open_scan([tmp_path / "em.h5"], rows=ROWS, cols=COLS)
    k, read = sc.info["overview"]
    assert k == 2 and np.array_equal(read(), Q) and sc.info["stored"] is None


def test_stored_orientations_by_maker(tmp_path):
    n = ROWS * COLS
    rng = np.random.default_rng(1)
    e = rng.uniform(0, 2 * np.pi, (n, 3))
    e[4] = 4 * np.pi  # the makers' not-indexed marker
    ph = np.array([1, 0, 2, 1, 1, 2], np.int32)
    # Oxford: one (n, 3) "Euler", its phase 0 not indexed
    sc = SC.open_scan([_h5ebsd(tmp_path / "o.h5", "oxford", {"Euler": D(e.astype(np.float32)), "Phase": D(ph)})])
    got = sc.info["stored"]()
    assert np.allclose(got["euler"], e.astype(np.float32)) and got["euler"].dtype == np.float64
    assert list(got["phase"]) == [1, -1, 2, 1, -1, 2]
    # Bruker: columns in degrees
    cols = {"phi1": D(np.degrees(e[:, 0])), "PHI": D(np.degrees(e[:, 1])), "phi2": D(np.degrees(e[:, 2])),
            "Phase": D(ph.astype(np.uint8))}
    got = SC.open_scan([_h5ebsd(tmp_path / "b.h5", "bruker", cols)]).info["stored"]()
    ok = np.arange(n) != 4
    assert np.allclose(got["euler"][ok], e[ok]) and list(got["phase"]) == [1, -1, 2, 1, -1, 2]
    # EDAX: either spelling, its phase 0 a phase; no Phase: 0 everywhere
    cols = {"Phi1": D(e[:, 0]), "PHI": D(e[:, 1]), "phi2": D(e[:, 2])}
    got = SC.open_scan([_h5ebsd(tmp_path / "e.h5", "edax", cols)]).info["stored"]()
    assert np.array_equal(got["euler"], e) and list(got["phase"]) == [0, 0, 0, 0, -1, 0]
    # a missing angle, a short column, or a maker without any: none
    del cols["phi2"]
    assert SC.open_scan([_h5ebsd(tmp_path / "f.h5", "edax", cols)]).info["stored"]() is None
    cols["phi2"] = D(e[:5, 2])
    assert SC.open_scan([_h5ebsd(tmp_path / "g.h5", "edax", cols)]).info["stored"]() is None
    assert SC.open_scan([_h5ebsd(tmp_path / "k.h5", "kikuchipy", {})]).info["stored"]() is None


def _up_and_ang(tmp_path, records, dx=0.5, dy=0.5, version=3):
    n = ROWS * COLS
    with open(tmp_path / "s.up2", "wb") as fh:
        head = struct.pack("<IIII", version, W, H, 42 if version >= 3 else 16)
        if version >= 3:
            head += struct.pack("<BIIBdd", 0, COLS, ROWS, 0, dx, dy)
        fh.write(head + _pats(n, np.uint16).astype("<u2").tobytes())
    lines = ["# GRID: SqrGrid", f"# XSTEP: {dx}", f"# YSTEP: {dy}", f"# NCOLS_ODD: {COLS}", f"# NCOLS_EVEN: {COLS}",
             f"# NROWS: {ROWS}", "# SOFTWARE: EDAX OIM"] + records
    with open(tmp_path / "s.ang", "w") as fh:
        fh.write("\n".join(lines) + "\n")
    return [tmp_path / "s.up2", tmp_path / "s.ang"]


def _records(e, iq, ph, dx=0.5, dy=0.5, jitter=0.0):
    return [f"{e[k, 0]:.6f} {e[k, 1]:.6f} {e[k, 2]:.6f} {k % COLS * dx + (jitter if k == 4 else 0):.5f} {k // COLS * dy:.5f} "
            f"{iq[k]} 0.5 {ph[k]} 0 1.0" for k in range(len(iq))]


def test_up_takes_the_ang_quality_and_orientations(tmp_path):
    n = ROWS * COLS
    e = np.tile([[0.5, 1.0, 1.5]], (n, 1)) + np.arange(n)[:, None] * 0.1
    e[2] = 12.56637  # 4π: not indexed
    iq = ["100.5", "200", "nan", "1e60", "5", "6"]
    ph = ["1", "0", "1", "-1", "x", "2"]
    sc = SC.open_scan(_up_and_ang(tmp_path, _records(e, iq, ph)))
    k, read = sc.info["overview"]
    got = read()
    assert k == 2 and got[0] == 100.5 and got[1] == 200 and np.isnan(got[2]) and np.isnan(got[3]) and got[5] == 6
    st = sc.info["stored"]()
    assert np.allclose(st["euler"], np.round(e, 6)) and list(st["phase"]) == [1, 0, -1, -1, -1, 2]
    # the records' coordinates step through the map row-major by the steps
    with pytest.raises(SC.ScanError, match="ANGCoordinatesNotRowMajor"):
        SC.open_scan(_up_and_ang(tmp_path, _records(e, iq, ph, jitter=0.01)))
    with pytest.raises(SC.ScanError, match="UPANGStepMismatch"):  # the .up's own steps differ
        SC.open_scan(_up_and_ang(tmp_path, _records(e, iq, ph, dx=0.6), dx=0.5)[:1] +
                     [_rewrite_steps(tmp_path / "s.ang", 0.6)])
    # too few or too many records, a short record, a header after the records
    with pytest.raises(SC.ScanError, match="ANGPatternCountMismatch"):
        SC.open_scan(_up_and_ang(tmp_path, _records(e, iq, ph)[:5]))
    with pytest.raises(SC.ScanError, match="ANGPatternCountMismatch"):
        SC.open_scan(_up_and_ang(tmp_path, _records(e, iq, ph) + _records(e, iq, ph)[:1]))
    with pytest.raises(SC.ScanError, match="InvalidANGRecord"):
        SC.open_scan(_up_and_ang(tmp_path, _records(e, iq, ph)[:5] + ["0 0 0 1.0 0.5 7"]))
    with pytest.raises(SC.ScanError, match="InvalidANGRecord"):
        SC.open_scan(_up_and_ang(tmp_path, _records(e, iq, ph)[:3] + ["# NOTE"] + _records(e, iq, ph)[3:]))
    # an .up without its .ang stores neither
    sc = SC.open_scan(_up_and_ang(tmp_path, _records(e, iq, ph))[:1])
    assert sc.info["overview"] == (0, None) and sc.info["stored"] is None


def _rewrite_steps(path, dx):
    """The .ang's header and records at x step dx (the .up beside it keeps its own)."""
    text = open(path).read().replace("# XSTEP: 0.5", f"# XSTEP: {dx}")
    open(path, "w").write(text)
    return path


def test_the_c_abi_hands_out_both(tmp_path):
    lib = ctypes.CDLL(str(build.build_abi()))
    P, SZ = ctypes.c_void_p, ctypes.c_size_t
    lib.ze_scan_overview_kind.argtypes, lib.ze_scan_overview_kind.restype = [P], ctypes.c_uint32
    lib.ze_scan_overview.argtypes, lib.ze_scan_overview.restype = [P, P, SZ], ctypes.c_int64
    lib.ze_stored_orientations.argtypes, lib.ze_stored_orientations.restype = [P, P, P, ctypes.c_uint64], ctypes.c_int32
    lib.ze_error.argtypes, lib.ze_error.restype = [P, ctypes.c_char_p, SZ], SZ
    h = 0x7F10
    Z._handles[h] = Z._Handle(_Solver())
    try:
        s = Z._handles[h].s
        s.set_patterns(np.zeros((ROWS, COLS, H, W), np.uint16))  # from memory: none stored
        assert lib.ze_scan_overview_kind(h) == 0 and lib.ze_scan_overview(h, None, 0) == 0
        assert lib.ze_stored_orientations(h, None, None, 6) == 0
        n = ROWS * COLS
        e = np.tile([[0.5, 1.0, 1.5]], (n, 1))
        sc = SC.open_scan(_up_and_ang(tmp_path, _records(e, [str(v) for v in Q], ["1"] * n)))
        s._e.scan_source = {"format": sc.format, "overview": sc.info["overview"], "stored": sc.info["stored"]}
        assert lib.ze_scan_overview_kind(h) == 2
        assert lib.ze_scan_overview(h, None, 0) == n  # the size, nothing read
        out = np.zeros(n, np.float32)
        assert lib.ze_scan_overview(h, out.ctypes.data, n) == n and np.array_equal(out, Q)
        assert lib.ze_scan_overview(h, out.ctypes.data, n - 1) < 0
        buf = ctypes.create_string_buffer(256)
        k = lib.ze_error(h, buf, 256)
        assert b"BufferTooSmall" in buf.raw[:k]
        eu, ph = np.zeros(3 * n), np.zeros(n, np.int32)
        assert lib.ze_stored_orientations(h, eu.ctypes.data, ph.ctypes.data, n) == 1
        assert np.allclose(eu.reshape(n, 3), e) and (ph == 1).all()
        assert lib.ze_stored_orientations(h, eu.ctypes.data, ph.ctypes.data, n - 1) < 0
    finally:
        Z._handles.pop(h, None)


def test_the_solver_hands_out_both(tmp_path):
    """Solver.open keeps the readers' stored maps; Solver.stored_overview/stored_orientations give
    them shaped as the map (an engine without a device: the host side of open alone)."""
    import zebsdsolve_b200 as ze
    from zebsdsolve_b200 import engine as E
    from zebsdsolve_b200.settings import Settings

    s = ze.Solver.__new__(ze.Solver)
    e = E.Engine.__new__(E.Engine)
    e.set, e.geo, e._resident, e.patterns = Settings(), E.Geometry(), None, None
    s._e = e
    ph = np.array([1, 0, 2, 1, 1, 2], np.int32)
    s.open(_h5ebsd(tmp_path / "o.h5", "oxford", {"Band Contrast": D(Q.reshape(2, 3)), "Phase": D(ph),
                                                  "Euler": D(np.full((6, 3), 0.5, np.float32))}))
    ov, st = s.stored_overview(), s.stored_orientations()
    assert ov["kind"] == 1 and ov["label"] == "Band contrast" and np.array_equal(ov["values"], Q.reshape(2, 3))
    assert st["euler"].shape == (2, 3, 3) and np.allclose(st["euler"], 0.5)
    assert np.array_equal(st["phase"], np.where(ph == 0, -1, ph).reshape(2, 3))
    s.set_patterns(np.zeros((2, 3, H, W), np.uint8))  # patterns from memory: none stored
    assert s.stored_overview() is None and s.stored_orientations() is None


@pytest.mark.parametrize("line,why", [
    ("# GRID: SqrGrid", "DuplicateANGMetadata"), ("# NROWS: 2", "DuplicateANGMetadata"),
    ("# XSTEP: 0.5", "DuplicateANGMetadata"), ("# COLUMN_HEADERS: phi1, PHI, phi2", "UnsupportedANGColumns"),
    ("# XUNITS: nm", "UnsupportedANGUnits"), ("# Indexed by ACOM", "UnsupportedANGConvention"),
    ("# TEM data", "UnsupportedANGConvention"), ("# x-star: abc", "InvalidANGPatternCentre")])
def test_ang_header_refusals(tmp_path, line, why):
    """ang.zig:170-214: the header lines the reference refuses."""
    n = ROWS * COLS
    paths = _up_and_ang(tmp_path, [line] + _records(np.zeros((n, 3)), ["1"] * n, ["0"] * n))
    with pytest.raises(SC.ScanError, match=why):
        SC.open_scan(paths)


def test_ang_header_dimensions_steps_and_units(tmp_path):
    n = ROWS * COLS
    recs = _records(np.zeros((n, 3)), ["1"] * n, ["0"] * n)
    for unit in ("# SCAN_UNIT: um", "# XUNITS: [microns]", "# YUNITS: µm"):
        SC.open_scan(_up_and_ang(tmp_path, [unit] + recs))  # micrometres, however written
    text = open(_up_and_ang(tmp_path, recs)[1]).read()
    for a, b, why in (("# NROWS: 2", "# NROWS: two", "InvalidANGDimensions"),
                      ("# NROWS: 2", "# NROWS: 0", "InvalidANGDimensions"),
                      ("# XSTEP: 0.5", "# XSTEP: -0.5", "InvalidANGStep"),
                      ("# YSTEP: 0.5", "# YSTEP: inf", "InvalidANGStep")):
        open(tmp_path / "s.ang", "w").write(text.replace(a, b))
        with pytest.raises(SC.ScanError, match=why):
            SC.open_scan([tmp_path / "s.up2", tmp_path / "s.ang"])
