"""The HDF5 reader (the reference's src/io/hdf5.zig) and the HDF5 scan layouts (src/scan.zig:536-838).

Pinned by files written by the HDF5 library itself: kikuchipy's nickel scan (h5py: superblock 0,
symbol-table groups, a chunked pattern dataset under a version 1 B-tree with a partial last chunk,
contiguous header arrays, fixed-length strings), read as the reference's own test reads it
(tests/test_api.py:666-671: 55 × 75 patterns of 60 × 60, its pattern centre (0.42326, 0.21363,
0.50207), a 70° tilt, a background); and a MATLAB 7.3 file that SciPy ships (a 512-byte user
block before the superblock, an attribute). The layouts neither holds are written by
tests/h5_writer.py, field by field from the format specification: version 2 superblocks and
object headers, compact links, continuation blocks, multi-level chunk trees, the version 4
single-chunk and implicit indexes, the four filters, fill values, enumerations, variable-length
strings; LZF against hand-assembled streams.
"""
import math
import os
import struct

import numpy as np
import pytest

from conftest import testdata
from h5_writer import D, Writer
from zebsdsolve_b200 import hdf5 as H
from zebsdsolve_b200 import scan as SC


def test_lzf_hand_assembled_streams():
    # a literal run of 3, then 6 bytes from 3 back (overlapping its own output)
    assert H.lzf_decompress(b"\x02abc\x80\x02", 9) == b"abcabcabc"
    # one literal, then a long match (7 + 11 + 2 = 20 bytes) from 1 back
    assert H.lzf_decompress(b"\x00x\xe0\x0b\x00", 21) == b"x" * 21
    with pytest.raises(H.H5Error):
        H.lzf_decompress(b"\x80\x05", 4)  # a reference before the start


def test_matlab_file_with_a_user_block():
    scipy_io = pytest.importorskip("scipy.io.matlab")
    path = os.path.join(os.path.dirname(scipy_io.__file__), "tests", "data", "testhdf5_7.4_GLNX86.mat")
    if not os.path.isfile(path):
        pytest.skip("SciPy's MATLAB test files are not installed")
    f = H.File(path)
    assert f.base == 512
    a = f.find("testdouble")
    v = f.read(f.dataset(a)).reshape(-1)
    np.testing.assert_allclose(v, np.arange(9) * math.pi / 4, rtol=0, atol=1e-15)
    assert f.attributes(a) == {"MATLAB_class": "double"}


def _nickel():
    p = testdata("nickel", "patterns_v2.h5")
    if p is None:
        pytest.skip("the reference's test data is not here (tests/golden/copy_testdata.sh)")
    return p


def test_nickel_scan_opens_as_the_reference_reads_it():
    sc = SC.open_scan([_nickel()])
    i = sc.info
    assert sc.format == "kikuchipy h5ebsd" and (i["rows"], i["cols"], i["pat_h"], i["pat_w"]) == (55, 75, 60, 60)
    assert sc.patterns.shape == (4125, 60, 60) and sc.patterns.dtype == np.uint8
    np.testing.assert_allclose(i["pc"], (0.42326, 0.21363, 0.50207), atol=1e-4)
    assert i["sample_tilt_deg"] == 70 and i["detector_tilt_deg"] == 0 and i["step_x_um"] == 1.5 == i["step_y_um"]
    assert i["px_um"] == 70 * 8 and i["voltage_kv"] == 20
    assert i["background"].shape == (60, 60) and 0 < i["background"].min() < i["background"].max() <= 255


def test_nickel_chunks_stitch_in_order():
    """The patterns are stored 277 to a chunk (the last one partial): a neighbour across a chunk's
    edge is as alike as one inside a chunk, which a chunk read out of place would not be."""
    p = SC.open_scan([_nickel()]).patterns.astype(np.float64).reshape(4125, -1)
    p -= p.mean(1, keepdims=True)
    p /= np.linalg.norm(p, axis=1, keepdims=True)
    r = (p[1:] * p[:-1]).sum(1)  # r[k]: pattern k + 1 against pattern k
    edges = np.arange(277, 4125, 277) - 1
    inner = np.setdiff1d(np.arange(len(r)), edges)
    assert np.median(r[edges]) > 0.8 * np.median(r[inner])
    assert p.shape[0] == 4125 and np.isfinite(p).all()


def _roundtrip(tmp_path, superblock, header, user_block=0):
    rng = np.random.default_rng(5)
    big = rng.integers(0, 60000, (13, 7, 9)).astype(np.uint16)
    tree = {
        "plain": D(rng.normal(size=(4, 5)).astype(np.float32), big=True, attrs={"unit": "um", "scale": 2.5}),
        "small": D(np.arange(6, dtype=np.int16).reshape(2, 3), layout="compact"),
        "tree": D(big, layout="chunked", chunk=(4, 3, 5), filters=["shuffle", "deflate", "fletcher32"], fanout=3),
        "holes": D(big, layout="chunked", chunk=(4, 7, 9), unwritten={(1, 0, 0), (3, 0, 0)}, fill=7),
        "lzf": D(big[:5], layout="chunked", chunk=(2, 7, 9), filters=["lzf"]),
        "single": D(big[:3], layout="chunked", chunk=(3, 7, 9), index="single", filters=["deflate"]),
        "implicit": D(big[:6], layout="chunked", chunk=(2, 7, 9), index="implicit"),
        "flags": D(np.array([1, 0, 1], np.uint8), enum=True),
        "name": D(np.array([b"nickel  "])),
        "notes": D(["first", "a longer second one"], vlen=True),
        "Group A": {"x": D(np.array([3.0])), "y": D(np.array([4], np.int64)), "z": D(np.array([5], np.uint32)),
                    "w": D(np.array([6.0], np.float32)), "deeper": {"v": D(np.array([8], np.int8))}},
    }
    path = tmp_path / f"t{superblock}{header}.h5"
    Writer(superblock, header, user_block).write(path, tree)
    f = H.File(path)
    assert sorted(f.list(f.root)) == sorted(tree)
    rd = lambda name: f.read(f.dataset(f.find(name)))  # noqa: E731
    np.testing.assert_array_equal(rd("plain"), tree["plain"].data)
    assert f.attributes(f.find("plain")) == {"unit": "um", "scale": 2.5}
    np.testing.assert_array_equal(rd("small"), tree["small"].data)
    np.testing.assert_array_equal(rd("tree"), big)
    holes = big.copy()
    holes[4:8] = 7
    holes[12:] = 7
    np.testing.assert_array_equal(rd("holes"), holes)
    np.testing.assert_array_equal(rd("lzf"), big[:5])
    np.testing.assert_array_equal(rd("single"), big[:3])
    np.testing.assert_array_equal(rd("implicit"), big[:6])
    np.testing.assert_array_equal(rd("flags"), [1, 0, 1])
    assert f.string(f.find("name")) == "nickel"
    assert f._strings(f.dataset(f.find("notes")), rd("notes")) == ["first", "a longer second one"]
    assert f.string(f.find("notes")) == "first"
    g = f.find("Group A")
    assert f.is_group(g) and not f.is_group(f.find("plain"))
    assert [f.number(f.child(g, k)) for k in "xyzw"] == [3.0, 4.0, 5.0, 6.0]
    assert f.number(f.find("Group A/deeper/v")) == 8.0 and f.find("Group A/none") is None
    ds = f.dataset(f.find("tree"))
    assert ds.layout == "chunked" and ds.index == "btree" and [x[0] for x in ds.filters] == [2, 1, 3]


@pytest.mark.parametrize("superblock,header,user_block", [(0, 1, 0), (0, 1, 512), (2, 2, 0), (2, 1, 1024)])
def test_written_layouts_read_back(tmp_path, superblock, header, user_block):
    _roundtrip(tmp_path, superblock, header, user_block)


def test_refusals_name_what_is_not_covered(tmp_path):
    f = H.File.__new__(H.File)
    f.so, f.sl = 8, 8
    lay = bytes([4, 2, 0, 2, 4]) + struct.pack("<II", 8, 1)
    for kind, what in ((3, "fixed-array"), (4, "extensible-array"), (5, "version 2 B-tree")):
        with pytest.raises(H.H5Unsupported, match=what):
            f._layout(H.Dataset(), lay + bytes([kind]) + bytes(32))
    with pytest.raises(H.H5Unsupported, match="compression filter 307"):
        f._filters(bytes([2, 1]) + struct.pack("<HHHH", 307, 6, 0, 0) + b"bzip2\0")
    with pytest.raises(H.H5Unsupported, match="superblock version"):
        (tmp_path / "v9.h5").write_bytes(b"\x89HDF\r\n\x1a\n" + bytes([9]) + bytes(100))
        H.File(tmp_path / "v9.h5")
    (tmp_path / "none.h5").write_bytes(bytes(600))
    with pytest.raises(H.H5Error, match="no superblock"):
        H.File(tmp_path / "none.h5")
    # a group in dense storage: a link info message with a fractal heap
    w = Writer(2, 2)
    dense = w.header([(0x02, bytes([0, 0]) + struct.pack("<Q", 4096) + b"\xff" * 8)])
    root = w.header([(0x02, bytes([0, 0]) + b"\xff" * 16), (0x06, bytes([1, 0x10, 0, 1]) + b"g" + struct.pack("<Q", dense))])
    path = tmp_path / "dense.h5"
    w.group = lambda tree: root
    w.write(path, {})
    h = H.File(path)
    with pytest.raises(H.H5Unsupported, match="dense group"):
        h.list(h.find("g"))
    with pytest.raises(SC.ScanError, match="UnsupportedHdf5: dense group"):
        SC.open_scan([path], scan_name="g")


# ── the vendors' layouts ──

def _pats(n, h, w, dt=np.uint16, seed=0):
    return np.random.default_rng(seed).integers(1, 4000, (n, h, w)).astype(dt)


def test_kikuchipy_layout_four_axes(tmp_path):
    rows, cols = 3, 4
    pats = _pats(rows * cols, 6, 8, np.uint8).reshape(rows, cols, 6, 8)
    head = {"n_rows": D(np.array([rows])), "n_columns": D(np.array([cols])), "step_x": D(np.array([0.5])),
            "step_y": D(np.array([0.75])), "sample_tilt": D(np.array([69.5])), "elevation_angle": D(np.array([10.0])),
            "pcx": D(np.full((rows, cols), 0.45)), "pcy": D(np.linspace(0.2, 0.3, rows * cols).reshape(rows, cols)),
            "pcz": D(np.full((rows, cols), 0.6)), "detector_pixel_size": D(np.array([1])),
            "static_background": D(np.full((6, 8), 9, np.uint16))}
    tree = {"other": {"x": D(np.array([1]))},
            "Scan 7": {"EBSD": {"Data": {"patterns": D(pats, layout="chunked", chunk=(1, 2, 6, 8), filters=["deflate"])},
                                "Header": head}, "SEM": {"Header": {"beam_energy": D(np.array([15.0]))}}}}
    Writer(2, 2).write(tmp_path / "k.h5", tree)
    sc = SC.open_scan([tmp_path / "k.h5"])
    i = sc.info
    assert sc.format == "kikuchipy h5ebsd" and (i["rows"], i["cols"]) == (rows, cols)
    np.testing.assert_array_equal(sc.map(), pats)
    assert i["pc"] == pytest.approx((0.45, 0.25, 0.6)) and math.isnan(i["px_um"])  # (1: the size unknown)
    assert (i["step_x_um"], i["step_y_um"], i["sample_tilt_deg"], i["detector_tilt_deg"], i["voltage_kv"]) == \
        (0.5, 0.75, 69.5, 10.0, 15.0)
    assert (i["background"] == 9).all()
    with pytest.raises(SC.ScanError, match="NoScanInFile"):
        SC.open_scan([tmp_path / "k.h5"], scan_name="other")


def test_bruker_layout_clipped_pcy(tmp_path):
    pats = _pats(6, 5, 8)
    data = {"RawPatterns": D(pats), "PCX": D(np.full(6, 0.5)), "PCY": D(np.full(6, 0.2)), "DD": D(np.full(6, 0.7))}
    head = {"NROWS": D(np.array([2], np.int32)), "NCOLS": D(np.array([3], np.int32)), "XSTEP": D(np.array([1.0])),
            "YSTEP": D(np.array([1.0])), "Sample Tilt": D(np.array([70.0])), "CameraTilt": D(np.array([5.0])),
            "DetectorFullHeightMicrons": D(np.array([24000.0])), "UnClippedPatternHeight": D(np.array([8.0])),
            "KV": D(np.array([20.0])), "StaticBackground": D(np.ones((5, 8), np.float32))}
    Writer(0, 1).write(tmp_path / "b.h5", {"Scan": {"EBSD": {"Data": data, "Header": head}}})
    sc = SC.open_scan([tmp_path / "b.h5"])
    i = sc.info
    assert sc.format == "Bruker h5ebsd" and (i["rows"], i["cols"]) == (2, 3)
    # PCY of the unclipped height (8 px) read on the stored one (5 px)
    assert i["pc"] == pytest.approx((0.5, 0.2 * 8 / 5, 0.7)) and "UnClippedPatternHeight" in i["pc_note"]
    assert i["px_um"] == 3000.0 and i["sample_tilt_deg"] == 70.0 and i["detector_tilt_deg"] == 5.0
    np.testing.assert_array_equal(sc.patterns, pats)


def test_edax_layout_calibration(tmp_path):
    pats = _pats(4, 6, 9)
    head = {"nRows": D(np.array([2])), "nColumns": D(np.array([2])), "Step X": D(np.array([2.0])),
            "Step Y": D(np.array([2.0])), "Sample Tilt": D(np.array([70.0])), "Camera Elevation Angle": D(np.array([4.0])),
            "Camera Diameter": D(np.array([27.0])),
            "Pattern Center Calibration": {"x-star": D(np.array([0.48])), "y-star": D(np.array([0.7])),
                                           "z-star": D(np.array([0.6]))}}
    Writer(2, 1).write(tmp_path / "e.h5", {"S1": {"EBSD": {"Data": {"Pattern": D(pats)}, "Header": head}}})
    i = SC.open_scan([tmp_path / "e.h5"]).info
    # y from the bottom; z a fraction of the smaller side (the height, 6 of 9)
    assert i["pc"] == pytest.approx((0.48, 0.3, 0.6)) and i["px_um"] == pytest.approx(3000.0)
    assert i["background"] is None and i["detector_tilt_deg"] == 4.0


def _oxford(tmp_path, euler=(0.0, math.pi / 2, 0.0), turn=math.pi, both=True):
    rows, cols, h, w = 3, 4, 6, 9
    r, c = np.meshgrid(np.arange(rows), np.arange(cols), indexing="ij")
    data = {"Processed Patterns": D(_pats(rows * cols, h, w, np.uint8)),
            "Pattern Center X": D((0.5 + 0.01 * c).reshape(-1).astype(np.float32)),
            "Pattern Center Y": D((0.3 + 0.02 * r).reshape(-1).astype(np.float32)),
            "Detector Distance": D(np.full(rows * cols, 0.4, np.float32))}
    if both:
        data["Unprocessed Patterns"] = D(_pats(rows * cols, h, w, np.int16, seed=1))
    head = {"Y Cells": D(np.array([rows], np.int32)), "X Cells": D(np.array([cols], np.int32)),
            "X Step": D(np.array([0.5], np.float32)), "Y Step": D(np.array([0.5], np.float32)),
            "Tilt Angle": D(np.array([math.radians(70)], np.float32)), "Tilt Axis": D(np.array([0.0])),
            "Scanning Rotation Angle": D(np.array([turn])), "Detector Orientation Euler": D(np.array(euler)),
            "Beam Voltage": D(np.array([20.0])), "Processed Static Background": D(np.full((h, w), 3, np.uint8)),
            "Unprocessed Static Background": D(np.full((h, w), 5, np.uint16))}
    Writer(0, 1).write(tmp_path / "o.h5oina", {"1": {"EBSD": {"Data": data, "Header": head}}})
    return tmp_path / "o.h5oina", data


def test_oxford_layout(tmp_path):
    path, data = _oxford(tmp_path)
    sc = SC.open_scan([path])
    i = sc.info
    ratio = 9 / 6
    assert sc.format == "Oxford h5oina" and i["pattern_kinds"] == ["processed", "unprocessed"] and not i["unprocessed"]
    np.testing.assert_array_equal(sc.patterns, data["Processed Patterns"].data)
    # y from the bottom, y and z fractions of the width; the mean over the map
    assert i["pc"] == pytest.approx((0.515, 1 - 0.32 * ratio, 0.4 * ratio), abs=1e-6)
    assert i["pc_per_col"] == pytest.approx((0.01, 0.0, 0.0), abs=1e-6)
    assert i["pc_per_row"] == pytest.approx((0.0, -0.02 * ratio, 0.0), abs=1e-6)
    assert i["sample_tilt_deg"] == pytest.approx(70.0, abs=1e-4) and i["scan_turn"] == 1
    assert i["detector_rot"] == pytest.approx((0, 0, 0), abs=1e-12) and (i["background"] == 3).all()
    u = SC.open_scan([path], unprocessed=True)
    assert u.info["unprocessed"] and u.patterns.dtype == np.float32 and (u.info["background"] == 5).all()
    np.testing.assert_array_equal(u.patterns, data["Unprocessed Patterns"].data.astype(np.float32))
    # unturned: the beam the other way; a detector turned 2° about its normal
    path, _ = _oxford(tmp_path, euler=(math.radians(2), math.pi / 2, 0.0), turn=0.0, both=False)
    i = SC.open_scan([path]).info
    assert i["scan_turn"] == -1 and "pattern_kinds" in i and i["pattern_kinds"] == ["processed"]
    rot = np.array(i["detector_rot"])
    assert abs(np.linalg.norm(rot) - math.radians(2)) < 1e-9
    path, _ = _oxford(tmp_path, euler=(math.radians(40), math.pi / 2, 0.0), both=False)
    assert SC.open_scan([path]).info["detector_rot"] is None  # more than 15° off: not read


def test_emsoft_layout(tmp_path):
    pats = _pats(6, 10, 12).astype(np.float32)
    tree = {"EMData": {"EBSD": {"EBSDPatterns": D(pats)}},
            "NMLparameters": {"EBSDNameList": {"xpc": D(np.array([2.4])), "ypc": D(np.array([-1.0])),
                                               "L": D(np.array([15000.0])), "delta": D(np.array([50.0])),
                                               "numsx": D(np.array([24])), "numsy": D(np.array([20])),
                                               "thetac": D(np.array([10.0])), "energymax": D(np.array([20.0]))},
                              "MCCLNameList": {"sig": D(np.array([70.0]))}}}
    Writer(2, 2).write(tmp_path / "em.h5", tree)
    sc = SC.open_scan([tmp_path / "em.h5"], rows=2, cols=3)
    i = sc.info
    assert sc.format == "EMsoft patterns" and (i["rows"], i["cols"]) == (2, 3)
    assert i["pc"] == pytest.approx((0.5 - 2.4 / 24, 0.5 + 1.0 / 20, 15000 / (20 * 50)))
    assert i["px_um"] == pytest.approx(50 * 20 / 10) and i["detector_tilt_deg"] == 10 and i["sample_tilt_deg"] == 70
    np.testing.assert_array_equal(sc.patterns, pats)
