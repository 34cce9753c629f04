"""Scan files and exports on the host (zebsdsolve_b200.scan, zebsdsolve_b200.output): EDAX .up1 /
.up2 (versions 1 and 3, with and without the scan's .ang), Oxford .ebsp (records stored out of
scan order, the map's shape from the beam positions), NORDIF Pattern.dat with Setting.txt, the
refusals (HDF5, bad headers, shapes that do not fit); the .ang and .ctf exports (the reference's
src/output.zig layout), read back: the stored orientations, the pattern centre through the .ang
reader's EDAX convention, the markers of cells not indexed."""
import math
import struct

import numpy as np
import pytest

from zebsdsolve_b200 import output, rotations as R, scan as SC
from zebsdsolve_b200.master import lattice_of


def _pats(n, h, w, dt, seed=0):
    rng = np.random.default_rng(seed)
    hi = 255 if dt == np.uint8 else 4000
    return rng.integers(0, hi, (n, h, w)).astype(dt)


def _write_up(path, pats, version, nx=0, ny=0, dx=1.5, dy=2.5, extra_bytes=0):
    n, h, w = pats.shape
    if version == 1:
        head = struct.pack("<IIII", 1, w, h, 16)
    else:
        off = 42 + extra_bytes
        head = struct.pack("<IIII", version, w, h, off) + struct.pack("<BIIBdd", 0, nx, ny, 0, dx, dy) + bytes(extra_bytes)
    with open(path, "wb") as fh:
        fh.write(head)
        fh.write(pats.astype(pats.dtype.newbyteorder("<")).tobytes())


def _ang_header(path, rows, cols, dx, dy, pc=None, software="EDAX OIM"):
    lines = []
    if pc is not None:
        lines += [f"# x-star {pc[0]}", f"# y-star {pc[1]}", f"# z-star {pc[2]}"]
    lines += ["# GRID: SqrGrid", f"# XSTEP: {dx}", f"# YSTEP: {dy}", f"# NCOLS_ODD: {cols}", f"# NCOLS_EVEN: {cols}",
              f"# NROWS: {rows}"]
    if software:
        lines.append(f"# SOFTWARE: {software}")
    lines += [f"  0.1 0.2 0.3 {k % cols * dx:.5f} {k // cols * dy:.5f} 1.0 0.5 0 0 0.0" for k in range(rows * cols)]
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")


def test_up1_version1_and_up2_version3(tmp_path):
    p8 = _pats(12, 6, 8, np.uint8)
    _write_up(tmp_path / "a.up1", p8, 1)
    s = SC.open_scan([tmp_path / "a.up1"], rows=3, cols=4)
    assert s.format == "edax_up" and np.array_equal(s.map(), p8.reshape(3, 4, 6, 8))
    assert (s.info["rows"], s.info["cols"], s.info["pat_h"], s.info["pat_w"]) == (3, 4, 6, 8)
    assert SC.open_scan([tmp_path / "a.up1"]).info["cols"] == 12  # no shape given: one row
    p16 = _pats(15, 5, 7, np.uint16, 1)
    _write_up(tmp_path / "b.up2", p16, 3, nx=5, ny=3, dx=1.5, dy=2.5)
    s = SC.open_scan([tmp_path / "b.up2"])
    assert np.array_equal(s.map(), p16.reshape(3, 5, 5, 7)) and s.patterns.dtype == np.dtype("<u2")
    assert (s.info["rows"], s.info["cols"], s.info["step_x_um"], s.info["step_y_um"]) == (3, 5, 1.5, 2.5)


def test_up2_with_its_ang(tmp_path):
    p = _pats(6, 60, 80, np.uint16, 2)
    _write_up(tmp_path / "s.up2", p, 3, nx=3, ny=2, dx=0.5, dy=0.5)
    _ang_header(tmp_path / "s.ang", 2, 3, 0.5, 0.5, pc=(0.41, 0.62, 0.55))
    s = SC.open_scan([tmp_path / "s.up2", tmp_path / "s.ang"])
    # EDAX: x, y in fractions of width and height, y from the bottom, z of the smaller side
    assert np.allclose(s.info["pc"], [0.41, 1 - 0.62, 0.55 * 60 / 60]) and "EDAX" in s.info["pc_note"]
    _ang_header(tmp_path / "w.ang", 2, 3, 0.5, 0.5, pc=(0.41, 0.62, 0.55), software="EMSphInx")
    s = SC.open_scan([tmp_path / "s.up2", tmp_path / "w.ang"])
    assert np.allclose(s.info["pc"], [0.41, 1 - 0.62 * 80 / 60, 0.55 * 80 / 60])
    _ang_header(tmp_path / "u.ang", 2, 3, 0.5, 0.5, pc=(0.41, 0.62, 0.55), software=None)
    s = SC.open_scan([tmp_path / "s.up2", tmp_path / "u.ang"])  # unknown writer, rectangular: not applied
    assert s.info["pc"] is None and "not applied" in s.info["pc_note"]
    _ang_header(tmp_path / "bad.ang", 2, 3, 0.7, 0.5)
    with pytest.raises(SC.ScanError, match="UPANGStepMismatch"):
        SC.open_scan([tmp_path / "s.up2", tmp_path / "bad.ang"])
    with pytest.raises(SC.ScanError, match="DuplicateANGSidecar"):
        SC.open_scan([tmp_path / "s.up2", tmp_path / "s.ang", tmp_path / "w.ang"])


def _write_ebsp(path, pats, version, order, positions=None):
    n, h, w = pats.shape
    nbytes = h * w * pats.dtype.itemsize
    table = 0 if version == 0 else (9 if version > 3 else 8)
    rec_head = 16 if version < 5 else 24
    foot = 18 if version >= 2 else 0
    rec = rec_head + nbytes + foot
    base = table + 8 * n
    offsets = np.zeros(n, np.int64)
    body = bytearray()
    for k, i in enumerate(order):  # records in acquisition order
        offsets[i] = base + k * rec
        head = (bytes(8) if version >= 5 else b"") + struct.pack("<iiii", 0, h, w, nbytes)
        body += head + pats[i].tobytes()
        if foot:
            x, y = positions[i]
            body += struct.pack("<Bd", 1, x) + struct.pack("<Bd", 1, y)
    with open(path, "wb") as fh:
        if version:
            fh.write(struct.pack("<q", -version) + bytes(table - 8))
        fh.write(offsets.tobytes())
        fh.write(bytes(body))


@pytest.mark.parametrize("version", [0, 4, 5])
def test_ebsp_records_out_of_order(tmp_path, version):
    rows, cols, n = 3, 4, 12
    p = _pats(n, 5, 6, np.uint16, 3)
    order = np.random.default_rng(4).permutation(n)
    pos = [(c * 2.0, r * 2.0) for r in range(rows) for c in range(cols)]
    _write_ebsp(tmp_path / "a.ebsp", p, version, order, pos)
    s = SC.open_scan([tmp_path / "a.ebsp"], rows=0 if version else rows, cols=0 if version else cols)
    assert np.array_equal(s.map(), p.reshape(rows, cols, 5, 6))
    if version >= 2:  # the map's shape and step from the beam positions
        assert (s.info["rows"], s.info["cols"], s.info["step_x_um"]) == (rows, cols, 2.0)


def test_nordif_with_setting(tmp_path):
    p = _pats(6, 4, 5, np.uint8, 5)
    (tmp_path / "Pattern.dat").write_bytes(p.tobytes())
    (tmp_path / "Setting.txt").write_text("[Microscope]\nAccelerating voltage\t20\t\nTilt angle\t69.5\t\n"
                                          "[Acquisition settings]\nResolution\t5x4\t\n[Area]\nNumber of samples\t2x3\t\n"
                                          "Step size\t1.25\t\n[Detector angles]\nElevation\t2.5\t\n")
    s = SC.open_scan([tmp_path / "Pattern.dat", tmp_path / "Setting.txt"])
    assert np.array_equal(s.map(), p.reshape(2, 3, 4, 5))
    i = s.info
    assert (i["rows"], i["cols"], i["pat_w"], i["pat_h"], i["step_x_um"], i["voltage_kv"], i["sample_tilt_deg"],
            i["detector_tilt_deg"]) == (2, 3, 5, 4, 1.25, 20.0, 69.5, 2.5)


def test_refusals(tmp_path):
    (tmp_path / "x.h5").write_bytes(b"\x89HDF\r\n\x1a\n" + bytes(100))
    with pytest.raises(SC.ScanError, match="UnsupportedHdf5: offset size"):
        SC.open_scan([tmp_path / "x.h5"])
    with pytest.raises(SC.ScanError, match="UnknownScanFormat"):
        SC.open_scan([tmp_path / "x.xyz"])
    (tmp_path / "bad.up1").write_bytes(struct.pack("<IIII", 2, 8, 8, 16) + bytes(64))
    with pytest.raises(SC.ScanError, match="BadScanFile"):
        SC.open_scan([tmp_path / "bad.up1"])
    _write_up(tmp_path / "c.up1", _pats(5, 4, 4, np.uint8), 1)
    with pytest.raises(SC.ScanError, match="ScanShapeMismatch"):
        SC.open_scan([tmp_path / "c.up1"], rows=2, cols=3)
    (tmp_path / "Pattern.dat").write_bytes(bytes(10))
    with pytest.raises(SC.ScanError, match="ScanShapeUnknown"):
        SC.open_scan([tmp_path / "Pattern.dat"])


class _Geo:
    pc = np.array([0.47, 0.31, 0.58])
    step_x_um, step_y_um, sample_tilt_deg = 1.5, 2.0, 70.0


def _results(rows, cols, seed=1):
    rng = np.random.default_rng(seed)
    n = rows * cols
    q = R.qstd(rng.normal(size=(n, 4)))
    phase = rng.integers(0, 2, n)
    phase[[1, 5]] = -1
    return {"quat": q.astype(np.float32), "ncc": rng.uniform(0, 1, n).astype(np.float32),
            "nmi": rng.uniform(0, 1, n).astype(np.float32), "phase": phase.astype(np.int32)}


PHASES = [{"name": "Ni", "laue": "o", "lattice": [3.52, 3.52, 3.52, 90, 90, 90], "space_group": 225},
          {"name": "GaN", "laue": "d6", "lattice": [3.19, 3.19, 5.19, 90, 90, 120], "space_group": 186}]


def test_ang_export_reads_back(tmp_path):
    rows, cols = 3, 4
    res = _results(rows, cols)
    text = output.export_text("ang", res, PHASES, _Geo, rows, cols, 60, 80)
    path = tmp_path / "r.ang"
    path.write_text(text)
    data = np.loadtxt(path, comments="#", ndmin=2)
    assert data.shape == (12, 10)
    ok = res["phase"] >= 0
    p1, P, p2 = data[:, 0], data[:, 1], data[:, 2]
    sig, dlt = 0.5 * (p1 + p2), 0.5 * (p1 - p2)
    q_back = np.stack([np.cos(P / 2) * np.cos(sig), -np.sin(P / 2) * np.cos(dlt), -np.sin(P / 2) * np.sin(dlt),
                       -np.cos(P / 2) * np.sin(sig)], -1)
    d = R.qmul(R.qconj(R.qstd(res["quat"].astype(np.float64))), R.qstd(q_back))
    dis = np.degrees(2 * np.arcsin(np.clip(np.linalg.norm(d[:, 1:], axis=1), 0, 1)))  # well-conditioned near 0
    assert dis[ok].max() < 1e-3 and np.allclose(data[~ok, 0], 12.56637) and (data[~ok, 6] == -1).all()
    assert np.array_equal(data[ok, 7], res["phase"][ok] + 1)
    assert np.allclose(data[:, 3], np.tile(np.arange(cols) * 1.5, rows)) and np.allclose(data[:, 4], np.repeat(np.arange(rows) * 2.0, cols))
    assert "# Symmetry              43" in text and "# Symmetry              62" in text
    # the header's pattern centre read back through the .ang reader (EDAX convention named)
    hdr = SC.read_ang_header(path, 80, 60)
    assert np.allclose(hdr["pc"], _Geo.pc, atol=1e-6) and (hdr["rows"], hdr["cols"]) == (rows, cols)


def test_ctf_export(tmp_path):
    rows, cols = 2, 3
    res = _results(rows, cols, 2)
    text = output.export_text("ctf", res, PHASES, _Geo, rows, cols, 60, 60, voltage_kv=20.0)
    lines = text.splitlines()
    assert lines[0] == "Channel Text File" and "XCells\t3" in lines and "YCells\t2" in lines and "KV\t20.0" in lines[11]
    assert lines[13].split("\t")[2:5] == ["Ni", "11", "225"] and lines[14].split("\t")[2:5] == ["GaN", "9", "186"]
    rows_ = [l.split("\t") for l in lines[16:]]
    assert len(rows_) == 6
    for k, r in enumerate(rows_):
        if res["phase"][k] < 0:
            assert r[0] == "0" and r[4] == "3"
        else:
            e = np.radians([float(v) for v in r[5:8]])
            assert np.allclose(e, R.to_bunge(res["quat"][k:k + 1].astype(np.float64))[0], atol=1e-5)
            assert int(r[9]) == int(math.floor(255 * res["ncc"][k] + 0.5))
    with pytest.raises(output.ExportError, match="MissingPhaseLattice"):
        output.export_text("ang", res, [dict(PHASES[0], lattice=None)], _Geo, rows, cols, 60, 60)


def test_master_cell():
    cell = {"a_angstrom": 3.52, "b_angstrom": 3.52, "c_angstrom": 3.52, "alpha_deg": 90, "beta_deg": 90, "gamma_deg": 90}
    assert lattice_of({"cell": cell}) == [3.52, 3.52, 3.52, 90.0, 90.0, 90.0]
    assert lattice_of({}) is None and lattice_of({"cell": dict(cell, a_angstrom=-1)}) is None
