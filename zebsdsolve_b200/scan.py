"""Scan files (the reference's src/scan.zig, src/ang.zig): EDAX .up1 / .up2 (with their scan's
.ang for the map's shape, the steps and the pattern centre), Oxford .ebsp (uncompressed), NORDIF
Pattern.dat (with Setting.txt), and the HDF5 layouts — h5ebsd as kikuchipy, Bruker (Esprit) and
EDAX (OIM) write it, Oxford's .h5oina and EMsoft's EMEBSD output — through this package's own
HDF5 reader. Patterns are mapped from the file where they lie in it contiguously (read into
memory otherwise); numbered row-major over the map, top row first, as stored.
"""
import math
import os
import re

import numpy as np

from . import hdf5 as H5
from . import rotations as R


class ScanError(ValueError):
    pass


def _ext(path):
    return os.path.splitext(str(path))[1].lower().lstrip(".")


def _valid_step(x):
    return math.isfinite(x) and x > 0


def _same_step(a, b):
    return abs(a - b) <= max(max(a, b) * 1e-6, min(5e-6, min(a, b) * 0.01))


class Scan:
    """An opened scan: `patterns` [n, h, w] (np.memmap of the file, the stored pixel type) and
    `info` (rows, cols, pat_h, pat_w, step_x_um, step_y_um, pc, pc_note, voltage_kv,
    sample_tilt_deg, detector_tilt_deg, px_um, background (float32 [h, w]), detector_rot (a
    rotation vector); NaN / None where the file says nothing). `info["overview"]` is the file's
    stored quality map, (kind, a function giving its rows × cols values as float32) or (0, None);
    `info["stored"]` a function giving the maker's own orientations ({"euler": (n, 3) float64
    radians, "phase": (n,) int32, −1 where not indexed} or None), or None."""

    def __init__(self, fmt, patterns, info):
        self.format, self.patterns, self.info = fmt, patterns, info

    def map(self):
        """The first rows × cols patterns as (rows, cols, h, w)."""
        i = self.info
        return self.patterns[: i["rows"] * i["cols"]].reshape(i["rows"], i["cols"], i["pat_h"], i["pat_w"])


def _blank_info():
    nan = float("nan")
    return {"rows": 0, "cols": 0, "pat_h": 0, "pat_w": 0, "step_x_um": nan, "step_y_um": nan, "pc": None,
            "pc_note": "", "voltage_kv": nan, "sample_tilt_deg": nan, "detector_tilt_deg": nan, "px_um": nan,
            "background": None, "detector_rot": None, "overview": (0, None), "stored": None}


def open_scan(paths, rows=0, cols=0, pat_h=0, pat_w=0, unprocessed=False, scan_name=""):
    """scan.zig Scan.open — by the first path's extension; rows/cols (and for NORDIF pat_h, pat_w)
    say what the file does not. HDF5: `scan_name` picks the scan group (else the first with
    EBSD/Data and EBSD/Header); `unprocessed` reads an Oxford file's unprocessed patterns where
    it stores both kinds."""
    paths = [str(p) for p in paths]
    if not paths:
        raise ScanError("NoScanFile")
    ext = _ext(paths[0])
    if ext in ("up1", "up2"):
        return _open_up(paths, ext == "up2", rows, cols)
    if ext == "ebsp":
        return _open_ebsp(paths[0], rows, cols)
    if ext == "dat":
        return _open_nordif(paths, rows, cols, pat_h, pat_w)
    if ext in ("h5", "hdf5", "h5ebsd", "h5oina"):
        return _open_h5(paths[0], rows, cols, unprocessed, scan_name)
    raise ScanError(f"UnknownScanFormat: {os.path.basename(paths[0])}")


def _shape(info, n, rows, cols):
    if rows and cols:
        info["rows"], info["cols"] = rows, cols
    if info["rows"] == 0:
        info["rows"], info["cols"] = 1, n
    if info["rows"] * info["cols"] > n:
        raise ScanError("ScanShapeMismatch")


def _open_up(paths, is16, rows, cols):
    """scan.zig:842-923 — EDAX .up1 (8-bit) / .up2 (16-bit): a 16-byte header (version, width,
    height, data offset), from version 3 the map's shape, hex flag and steps; an .ang beside it
    gives the shape, the steps, the pattern centre, and from its records the image-quality map and
    the maker's orientations."""
    side = [p for p in paths[1:] if _ext(p) == "ang"]
    if len(side) > 1:
        raise ScanError("DuplicateANGSidecar")
    size = os.path.getsize(paths[0])
    if size < 16:
        raise ScanError("BadScanFile")
    head = np.fromfile(paths[0], np.uint8, count=min(size, 64))
    version, w, h, off = (int(v) for v in head[:16].view("<u4"))
    if (version != 1 and version < 3) or w == 0 or h == 0 or off < 16 or off > size:
        raise ScanError("BadScanFile")
    dt = np.dtype("<u2") if is16 else np.dtype("u1")
    pb = w * h * dt.itemsize
    if (size - off) % pb:
        raise ScanError("UPIncompletePattern")
    n = (size - off) // pb
    if n == 0:
        raise ScanError("ScanShapeMismatch")
    info = _blank_info()
    info.update(pat_w=w, pat_h=h)
    nx = ny = hexg = extra = 0
    dx = dy = float("nan")
    if version >= 3:
        if off < 42:
            raise ScanError("BadScanFile")
        extra = int(head[16])
        nx, ny = (int(v) for v in head[17:25].view("<u4"))
        hexg = int(head[25])
        dx, dy = (float(v) for v in head[26:42].view("<f8"))
        if hexg == 0 and nx * ny == n:
            info.update(cols=nx, rows=ny, step_x_um=dx, step_y_um=dy)
    if side:
        if hexg:
            raise ScanError("UnsupportedUPHexGrid")
        if version >= 3:
            if nx == 0 or ny == 0 or nx * ny != n:
                raise ScanError("AmbiguousUPExtraPatterns" if extra else "UPPatternCountMismatch")
            if not (_valid_step(dx) and _valid_step(dy)):
                raise ScanError("InvalidUPStep")
        ang = read_ang_header(side[0], w, h)
        if ang["rows"] * ang["cols"] != n:
            raise ScanError("ANGPatternCountMismatch")
        rec = read_ang_records(side[0], ang["rows"], ang["cols"], (ang["step_x_um"], ang["step_y_um"]),
                               (dx, dy) if version >= 3 else None)
        if version >= 3 and (nx != ang["cols"] or ny != ang["rows"]):
            raise ScanError("ScanShapeMismatch")
        if version >= 3 and not (_same_step(dx, ang["step_x_um"]) and _same_step(dy, ang["step_y_um"])):
            raise ScanError("UPANGStepMismatch")
        if (rows and rows != ang["rows"]) or (cols and cols != ang["cols"]):
            raise ScanError("ScanShapeMismatch")
        info.update(rows=ang["rows"], cols=ang["cols"], step_x_um=ang["step_x_um"], step_y_um=ang["step_y_um"],
                    pc=ang["pc"], pc_note=ang["pc_note"], overview=(2, lambda: rec["iq"]),
                    stored=lambda: {"euler": rec["euler"], "phase": rec["phase"]})
    else:
        _shape(info, n, rows, cols)
    pats = np.memmap(paths[0], dt, "r", offset=off, shape=(n, h, w))
    return Scan("edax_up", pats, info)


_MICRO = ("um", "µm", "μm", "micron", "microns", "micrometer", "micrometers", "micrometre", "micrometres")


def read_ang_header(path, width, height):
    """ang.zig:87-270 (the header): the map's shape and steps and the pattern centre in the
    Bruker convention — EDAX's (x and y in fractions of width and height, y from the bottom, z of
    the smaller side) or, when EMSphInx or zebsdsolve 0.2.1 and before wrote it, width-scaled."""
    raw = [None, None, None]
    rows = odd = even = 0
    dx = dy = 0.0
    width_producer = edax_producer = software_seen = header_start = numeric_version = False
    square = False
    with open(path, "r", errors="replace") as fh:
        for line in fh:
            line = line.strip(" \t\r\n")
            if not line:
                continue
            if not line.startswith("#"):
                break
            content = line[1:].strip(" \t")
            # ang.zig:177-187: an ACOM (TEM) file's angles follow another convention
            words = re.findall(r"[A-Za-z0-9_]+", content)
            if "ACOM" in words or any(a == "TEM" and b == "data" for a, b in zip(words, words[1:])):
                raise ScanError("UnsupportedANGConvention")
            m = re.match(r"[: \t]*([^: \t]+)(.*)", content)
            if m is None:
                continue
            key, value = m.group(1), m.group(2).strip(": \t")
            k = {"x-star": 0, "y-star": 1, "z-star": 2}.get(key)
            if k is not None:
                if raw[k] is not None:
                    raise ScanError("DuplicateANGPatternCentre")
                try:
                    raw[k] = float(value)
                except ValueError:
                    raise ScanError("InvalidANGPatternCentre") from None
                if not math.isfinite(raw[k]):
                    raise ScanError("InvalidANGPatternCentre")
            elif key == "SOFTWARE":
                software_seen = True
                words = value.split()
                prod = words[0] if words else ""
                if prod in ("EDAX", "OIM"):
                    edax_producer = True
                if prod == "EMSphInx":
                    width_producer = True
                if prod == "zebsdsolve":
                    if "EDAX" in value:
                        edax_producer = True
                    else:
                        width_producer = True
            elif key == "HEADER" and value == "Start":
                header_start = True
            elif key == "VERSION":
                numeric_version = value.isdigit() and int(value) < 1 << 32
            # ang.zig:190-214: each grid line once, whole numbers and positive steps, micrometres
            if key == "GRID":
                if square:
                    raise ScanError("DuplicateANGMetadata")
                if value != "SqrGrid":
                    raise ScanError("UnsupportedANGGrid")
                square = True
            elif key in ("NROWS", "NCOLS_ODD", "NCOLS_EVEN"):
                if {"NROWS": rows, "NCOLS_ODD": odd, "NCOLS_EVEN": even}[key]:
                    raise ScanError("DuplicateANGMetadata")
                if not (value.isdigit() and 0 < int(value) < 1 << 32):
                    raise ScanError("InvalidANGDimensions")
                if key == "NROWS":
                    rows = int(value)
                elif key == "NCOLS_ODD":
                    odd = int(value)
                else:
                    even = int(value)
            elif key in ("XSTEP", "YSTEP"):
                if (dx if key == "XSTEP" else dy) != 0:
                    raise ScanError("DuplicateANGMetadata")
                try:
                    v = float(value)
                except ValueError:
                    raise ScanError("InvalidANGStep") from None
                if not (math.isfinite(v) and v > 0):
                    raise ScanError("InvalidANGStep")
                dx, dy = (v, dy) if key == "XSTEP" else (dx, v)
            elif key in ("COLUMN_HEADERS", "COLUMN_UNITS"):
                raise ScanError("UnsupportedANGColumns")
            elif key in ("SCAN_UNIT", "SCANUNIT", "XUNITS", "YUNITS"):
                if value.strip(" \t[]()") not in _MICRO:
                    raise ScanError("UnsupportedANGUnits")
    if not square or rows == 0 or odd == 0 or even == 0:
        raise ScanError("ANGGridMetadataRequired")
    if odd != even:
        raise ScanError("UnsupportedANGGrid")
    if not (dx > 0 and dy > 0):
        raise ScanError("InvalidANGStep")
    out = {"rows": rows, "cols": odd, "step_x_um": dx, "step_y_um": dy, "pc": None, "pc_note": ""}
    present = sum(v is not None for v in raw)
    if present == 0 or (present == 3 and raw == [0.0, 0.0, 0.0]):
        return out
    if present != 3:
        raise ScanError("IncompleteANGPatternCentre")
    if raw[2] <= 0 or width == 0 or height == 0:
        raise ScanError("InvalidANGPatternCentre")
    if width_producer and edax_producer and width != height:
        out["pc_note"] = "ANG pattern centre not applied: conflicting writers named"
        return out
    width_scaled = width_producer and not edax_producer
    edax = edax_producer or (not width_producer and not software_seen and header_start and numeric_version)
    if not width_scaled and not edax and width != height:
        out["pc_note"] = "ANG pattern centre not applied: its convention is unknown for a rectangular pattern"
        return out
    w, h = float(width), float(height)
    if width_scaled:
        pc = [raw[0], 1 - raw[1] * w / h, raw[2] * w / h]
        note = "ANG pattern centre: width-scaled (EMSphInx, zebsdsolve 0.2.1 and before)"
    else:
        pc = [raw[0], 1 - raw[1], raw[2] * min(w, h) / h]
        note = "ANG pattern centre: EDAX convention" if edax else "ANG pattern centre: square pattern, the conventions agree"
    if not all(math.isfinite(v) for v in pc) or not pc[2] > 0:
        raise ScanError("InvalidANGPatternCentre")
    out["pc"], out["pc_note"] = pc, note
    return out


def _coordinates_not_row_major(actual, origin, travel, step):
    """ang.zig:74-85 per record, over all records at once: 0 where a record's coordinate is at its
    place in row-major order (origin + travel), within the looser of 1e-6 of the step and
    min(5e-6, 1 % of the step) — else within min(1e-5, 1 % of the step) plus 2^-24 of the
    magnitudes involved (positions a maker computed in float32 and printed to five decimals);
    1 where it is not; 2 where that allowance reaches an eighth of the step (the file's
    precision cannot tell the cells apart)."""
    expected = origin + travel
    with np.errstate(invalid="ignore", over="ignore"):
        residual = np.abs((actual - origin) - travel)
        strict = max(step * 1e-6, min(5e-6, step * 0.01))
        budget = min(1e-5, step * 0.01) + 2.0 ** -24 * (abs(origin) + np.abs(expected) + 2 * np.abs(travel))
        code = np.where(residual <= strict, 0,
                        np.where(~np.isfinite(budget) | (budget >= step / 8), 2, np.where(residual > budget, 1, 0)))
    code[~(np.isfinite(actual) & np.isfinite(expected))] = 1
    return code


def read_ang_records(path, rows, cols, steps, up_steps=None):
    """ang.zig:216-268 (the records): per map cell, in row-major order, the legacy columns phi1 Phi
    phi2 x y IQ CI phase. Returns {"iq": float32 (n,) (NaN where not finite), "euler": float64
    (n, 3) Bunge angles as written, "phase": int32 (n,) — the label, −1 where it is negative, not an
    integer, or the angles are not finite or past 2π (ANG's not-indexed 4π)}. The x and y columns
    must step through the grid row-major by the header's `steps` (x, y), and by the .up file's own
    (`up_steps`) where it states them."""
    n = rows * cols
    vals = np.full((n, 6), np.nan)
    label = np.full(n, -1, np.int64)
    count = 0
    with open(path, "r", errors="replace") as fh:
        for line in fh:
            line = line.strip(" \t\r\n")
            if not line:
                continue
            if line[0] == "#":
                if count:
                    raise ScanError("InvalidANGRecord")
                continue
            if count >= n:
                raise ScanError("ANGPatternCountMismatch")
            words = line.split()
            if len(words) < 8:
                raise ScanError("InvalidANGRecord")
            try:
                vals[count] = [float(w) for w in words[:6]]
            except ValueError:
                raise ScanError("InvalidANGRecord") from None
            try:
                v = int(words[7])
                label[count] = v if -(1 << 31) <= v < 1 << 31 else -1
            except ValueError:
                pass
            count += 1
    if count != n or count == 0:
        raise ScanError("ANGPatternCountMismatch")
    k = np.arange(n)
    col, row = (k % cols).astype(np.float64), (k // cols).astype(np.float64)
    checks = []
    for st, err in ((steps, None), (up_steps, "UPANGStepMismatch")):
        if st is None:
            continue
        cx = _coordinates_not_row_major(vals[:, 3], vals[0, 3], col * st[0], st[0])
        cy = _coordinates_not_row_major(vals[:, 4], vals[0, 4], row * st[1], st[1])
        checks.append((cx, err))
        checks.append((cy, err))
    # the first record that fails a check, and its first failing check, give the error
    bad = np.zeros(n, bool)
    for c, _ in checks:
        bad |= c != 0
    if bad.any():
        i = int(np.argmax(bad))
        for c, err in checks:
            if c[i]:
                raise ScanError(err or ("ANGCoordinatePrecisionInsufficient" if c[i] == 2 else "ANGCoordinatesNotRowMajor"))
    euler = vals[:, :3].copy()
    phase = np.where(label >= 0, label, -1).astype(np.int32)
    return {"iq": _f32_or_nan(vals[:, 5]), "euler": euler, "phase": _marked_unindexed(euler, phase)}


def _open_ebsp(path, rows, cols):
    """scan.zig:927-1011 — Oxford .ebsp (uncompressed): a version word (negated from version 1),
    a table of each pattern's record offset in scan order, records of a header (compressed flag,
    height, width, bytes) and the pixels, from version 2 a footer with the beam's position (the
    map's shape from the first, second and last)."""
    size = os.path.getsize(path)
    if size < 24:
        raise ScanError("BadScanFile")
    data = np.memmap(path, np.uint8, "r")

    def i64(at):
        return int(data[at:at + 8].view("<i8")[0])

    def i32(at):
        return int(data[at:at + 4].view("<i4")[0])

    def f64(at):
        return float(data[at:at + 8].view("<f8")[0])

    first8 = i64(0)
    version = -first8 if first8 < 0 else 0
    hdr = 16 if version < 5 else 24
    table = 0 if version == 0 else (9 if version > 3 else 8)
    bound, seen = None, 0
    while bound is None or seen < bound:
        at = table + seen * 8
        if at + 8 > size:
            break
        o = i64(at)
        if o > 0:
            if o <= table:
                raise ScanError("BadScanFile")
            b = (o - table) // 8
            bound = b if bound is None else min(bound, b)
        seen += 1
    if not bound:
        raise ScanError("BadScanFile")
    n = bound
    offs = np.frombuffer(bytes(data[table:table + n * 8]), "<i8")
    first_record = table + n * 8
    ph = first_record + (8 if version >= 5 else 0)
    compressed, h, w, nbytes = i32(ph), i32(ph + 4), i32(ph + 8), i32(ph + 12)
    if compressed != 0:
        raise ScanError("CompressedEbspUnsupported")
    if h <= 0 or w <= 0:
        raise ScanError("BadScanFile")
    px = h * w
    if nbytes == px:
        dt = np.dtype("u1")
    elif nbytes == 2 * px:
        dt = np.dtype("<u2")
    else:
        raise ScanError("BadScanFile")
    starts = np.where(offs <= 0, 0, offs + hdr).astype(np.int64)
    info = _blank_info()
    info.update(pat_h=h, pat_w=w)
    if version >= 2 and n > 1 and starts[0] and starts[1] and starts[n - 1]:
        foot0 = int(starts[0]) + nbytes
        if data[foot0] != 0 and data[foot0 + 9] != 0 and int(starts[n - 1]) + nbytes + 18 <= size:
            x0, y0 = f64(foot0 + 1), f64(foot0 + 10)
            x1 = f64(int(starts[1]) + nbytes + 1)
            xl, yl = f64(int(starts[n - 1]) + nbytes + 1), f64(int(starts[n - 1]) + nbytes + 10)
            step = abs(x1 - x0)
            if step > 0 and math.isfinite(xl) and math.isfinite(yl):
                fx = math.floor(abs(xl - x0) / step + 0.5) + 1
                fy = math.floor(abs(yl - y0) / step + 0.5) + 1
                if fx * fy == n:
                    info.update(cols=fx, rows=fy, step_x_um=step, step_y_um=step)
    _shape(info, n, rows, cols)
    pats = np.zeros((n, h, w), dt)
    for i, s0 in enumerate(starts):
        if s0:
            pats[i] = np.frombuffer(bytes(data[s0:s0 + nbytes]), dt).reshape(h, w)
    return Scan("oxford_ebsp", pats, info)


def _open_nordif(paths, rows, cols, pat_h, pat_w):
    """scan.zig:1015-1063 — NORDIF Pattern.dat (8-bit patterns, nothing else) with Setting.txt
    (Acquisition settings: Resolution w x h; Area: Number of samples rows x cols, Step size;
    Microscope: Accelerating voltage, Tilt angle; Detector angles: Elevation)."""
    info = _blank_info()
    setting = paths[1] if len(paths) > 1 else os.path.join(os.path.dirname(paths[0]), "Setting.txt")

    def pair(v):
        if "x" not in v:
            return None
        a, b = v.split("x", 1)
        try:
            return int(a.strip()), int(b.strip())
        except ValueError:
            return None

    if os.path.isfile(setting):
        section = ""
        with open(setting, "r", errors="replace") as fh:
            for line in fh.read(1 << 20).splitlines():
                if line.startswith("["):
                    section = line.strip("[]\t ")
                    continue
                col = line.split("\t")
                if len(col) < 2:
                    continue
                key, val = col[0], col[1].strip(" ")
                try:
                    if section == "Acquisition settings" and key == "Resolution" and pair(val):
                        info["pat_w"], info["pat_h"] = pair(val)
                    elif section == "Area" and key == "Number of samples" and pair(val):
                        info["rows"], info["cols"] = pair(val)
                    elif section == "Area" and key == "Step size":
                        info["step_x_um"] = info["step_y_um"] = float(val)
                    elif section == "Microscope" and key == "Accelerating voltage":
                        info["voltage_kv"] = float(val)
                    elif section == "Microscope" and key == "Tilt angle":
                        info["sample_tilt_deg"] = float(val)
                    elif section == "Detector angles" and key == "Elevation":
                        info["detector_tilt_deg"] = float(val)
                except ValueError:
                    pass
    if rows and cols:
        info["rows"], info["cols"] = rows, cols
    if pat_h and pat_w:
        info["pat_h"], info["pat_w"] = pat_h, pat_w
    if info["rows"] == 0 or info["pat_h"] == 0:
        raise ScanError("ScanShapeUnknown")
    n = info["rows"] * info["cols"]
    if n * info["pat_h"] * info["pat_w"] > os.path.getsize(paths[0]):
        raise ScanError("ScanShapeMismatch")
    pats = np.memmap(paths[0], np.uint8, "r", shape=(n, info["pat_h"], info["pat_w"]))
    return Scan("nordif", pats, info)


# ── HDF5 ──

# scan.zig:583-586 — what each writer names the same things: format, pattern datasets (Data),
# header fields (Header), static background; Oxford's unprocessed patterns beside the processed
_H5_VENDORS = (
    ("kikuchipy h5ebsd", ("patterns",), "n_rows", "n_columns", "step_x", "step_y", "sample_tilt",
     "elevation_angle", "static_background", "", ""),
    ("Bruker h5ebsd", ("RawPatterns",), "NROWS", "NCOLS", "XSTEP", "YSTEP", "SampleTilt", "CameraTilt",
     "StaticBackground", "", ""),
    ("EDAX h5ebsd", ("Pattern",), "nRows", "nColumns", "Step X", "Step Y", "Sample Tilt", "Camera Elevation Angle",
     "", "", ""),
    ("Oxford h5oina", ("Processed Patterns",), "Y Cells", "X Cells", "X Step", "Y Step", "Tilt Angle", "",
     "Processed Static Background", "Unprocessed Patterns", "Unprocessed Static Background"),
)


def _h5_get(h, group, name):
    """A header number, NaN where absent or not a number."""
    if not name:
        return float("nan")
    try:
        a = h.child(group, name)
        return float("nan") if a is None else h.number(a)
    except H5.H5Error:
        return float("nan")


def _h5_values(h, group, name, limit=1 << 24):
    try:
        a = h.child(group, name)
        if a is None:
            return None
        v = h.numbers(a)
        return v[:limit] if v.size else None
    except H5.H5Error:
        return None


# scan.zig:294-332: the makers' names for a stored quality map, in the order they are tried, each
# with its kind (1 band contrast, 2 image quality, 3 Radon quality, 4 pattern quality)
OVERVIEW_NAMES = (("Band Contrast", 1), ("band_contrast", 1), ("BandContrast", 1), ("Image Quality", 2),
                  ("IQ", 2), ("image_quality", 2), ("iq", 2), ("ImageQuality", 2), ("RadonQuality", 3),
                  ("Radon Quality", 3), ("Pattern Quality", 4), ("PatternQuality", 4))
OVERVIEW_LABELS = {1: "Band contrast", 2: "Image quality", 3: "Radon quality", 4: "Pattern quality"}


def _f32_or_nan(v):
    """Values as float32, NaN where not finite or past float32's range (scan.zig:217, ang.zig:259)."""
    v = np.asarray(v, np.float64)
    with np.errstate(invalid="ignore"):
        ok = np.isfinite(v) & (np.abs(v) <= float(np.finfo(np.float32).max))
    return np.where(ok, v, np.nan).astype(np.float32)


def _h5_first(h, group, name, count):
    """The first `count` values of a numeric dataset as float64, or None where it is absent, not
    numeric or shorter (hdf5.zig:1043-1055 reads min(stored, asked) values)."""
    try:
        a = h.child(group, name)
        v = h.numbers(a) if a is not None else None
    except H5.H5Error:
        return None
    return v[:count] if v is not None and v.size >= count and count else None


def _h5_overview(h, group, rows, cols):
    """scan.zig:294-332 — the stored quality map: the first of OVERVIEW_NAMES under the data group
    whose dataset holds one number per map cell, as a vector (n, (n, 1) or (1, n)) or as the raster
    (rows, cols), in an integer of 1, 2, 4 or 8 bytes or a float of 4 or 8. Returns (kind, a reader
    of its n values as float32, scan.zig:205-217), or (0, None). The values are read when asked."""
    n = rows * cols
    for name, kind in OVERVIEW_NAMES:
        try:
            a = h.child(group, name)
            ds = h.dataset(a) if a is not None else None
        except H5.H5Error:
            continue
        if ds is None or ds.shape is None or n == 0:
            continue
        if tuple(int(d) for d in ds.shape) not in ((n,), (n, 1), (1, n), (rows, cols)):
            continue
        k, size = ds.dtype.kind, ds.dtype.size
        if not ((k in "ui" and size in (1, 2, 4, 8)) or (k == "f" and size in (4, 8))):
            continue

        def read(a=a):
            try:
                v = h.numbers(a)
            except H5.H5Error:
                v = None
            if v is None or v.size != n:
                raise ScanError("InvalidStoredOverview")
            return _f32_or_nan(v)
        return kind, read
    return 0, None


# scan.zig:236-243: where each maker keeps its own orientations — one (n, 3) dataset or a column per
# angle (the names each may go by) —, whether in degrees, and whether its phase 0 marks a cell not
# indexed
_STORED_ORIENTATIONS = {
    "Oxford h5oina": ("Euler", None, False, True),
    "Bruker h5ebsd": ("", (("phi1",), ("PHI",), ("phi2",)), True, True),
    "EDAX h5ebsd": ("", (("phi1", "Phi1"), ("Phi", "PHI"), ("phi2", "Phi2")), False, False),
}


def _marked_unindexed(euler, phase):
    """Cells whose angles are not finite or past 2π (+0.01; 4π is the makers' not-indexed marker)
    get phase −1 (scan.zig:283-289, ang.zig:261-264)."""
    with np.errstate(invalid="ignore"):
        ok = np.all(np.isfinite(euler) & (np.abs(euler) <= 2 * np.pi + 0.01), axis=1)
    phase[~ok] = -1
    return phase


def _h5_stored(h, data, fmt, n):
    """scan.zig:224-291 — the orientations an HDF5 file stores from its maker's indexing: Bunge
    angles in radians (Bruker's degrees converted) and the "Phase" label per cell (0 where absent;
    Oxford's and Bruker's 0, and any cell whose angles are past 2π, as −1), or None."""
    if fmt not in _STORED_ORIENTATIONS or n == 0:
        return None
    one, three, degrees, zero_unindexed = _STORED_ORIENTATIONS[fmt]
    if one:
        e = _h5_first(h, data, one, 3 * n)
        if e is None:
            return None
        euler = e.reshape(n, 3).copy()
    else:
        angles = []
        for names in three:
            col = next((v for v in (_h5_first(h, data, nm, n) for nm in names) if v is not None), None)
            if col is None:
                return None
            angles.append(col)
        euler = np.stack(angles, 1)
    if degrees:
        euler = np.radians(euler)
    phase = np.zeros(n, np.int32)
    p = _h5_first(h, data, "Phase", n)
    if p is not None:
        with np.errstate(invalid="ignore"):
            ok = np.isfinite(p) & (np.abs(p) < 1 << 30)
        phase = np.where(ok, np.trunc(np.where(ok, p, 0)), -1).astype(np.int32)
    if zero_unindexed:
        phase[phase == 0] = -1
    return {"euler": np.ascontiguousarray(euler, np.float64), "phase": _marked_unindexed(euler, phase)}


def _h5_mean(h, group, name):
    """scan.zig:653-668 — the mean of a per-pattern array."""
    v = _h5_values(h, group, name)
    return float("nan") if v is None else float(v.sum() / max(v.size, 1))


def _h5_drift(h, group, name, rows, cols):
    """scan.zig:637-651 — how a per-pattern array changes from one column to the next and from one
    row to the next, on average (the last column less the first over the columns between, and
    likewise down the rows)."""
    nan = (float("nan"), float("nan"))
    if rows < 2 or cols < 2:
        return nan
    v = _h5_values(h, group, name)
    if v is None or v.size != rows * cols:
        return nan
    m = v.reshape(rows, cols)
    return (float((m[:, -1] - m[:, 0]).sum()) / (rows * (cols - 1)),
            float((m[-1, :] - m[0, :]).sum()) / (cols * (rows - 1)))


def _bunge_matrix(e):
    """The active rotation Rz(φ1) Rx(Φ) Rz(φ2) of Bunge angles, row-major."""
    c1, s1, c, s, c2, s2 = math.cos(e[0]), math.sin(e[0]), math.cos(e[1]), math.sin(e[1]), math.cos(e[2]), math.sin(e[2])
    return np.array([[c1 * c2 - s1 * c * s2, -c1 * s2 - s1 * c * c2, s1 * s],
                     [s1 * c2 + c1 * c * s2, -s1 * s2 + c1 * c * c2, -c1 * s],
                     [s * s2, s * c2, c]])


# Oxford's nominal detector orientation (0, 90°, 0): Bunge angles of the detector's axes (x along
# the pattern's columns, y up it, z its normal toward the sample) in the sample's (scan.zig:94-97)
_OXFORD_NOMINAL = (0.0, math.pi / 2, 0.0)


def oxford_detector_rot(e):
    """scan.zig:121-127 — Oxford's stored detector orientation as the geometry's rotation vector
    (detector axes), None where not finite or more than 15° from the nominal one."""
    if not all(math.isfinite(float(v)) for v in e):
        return None
    b = _bunge_matrix(_OXFORD_NOMINAL).T @ _bunge_matrix(e)
    v = np.asarray(R.log_map(R.from_matrix(b)), np.float64)
    if float(np.linalg.norm(v)) > math.radians(15.0):
        return None
    return [float(-v[1]), float(v[0]), float(v[2])]


def _h5_pixels(ds):
    """scan.zig:613-624 — u8 and u16 as stored, f32 as stored, signed 16-bit (Oxford's unprocessed
    patterns) widened to f32."""
    k, n = ds.dtype.kind, ds.dtype.size
    if (k == "u" and n in (1, 2)) or (k == "f" and n == 4) or (k == "i" and n == 2):
        return
    raise ScanError("UnsupportedPixelType")


def _h5_patterns(h, ds):
    arr = h.read(ds)
    if ds.dtype.kind == "i":
        return arr.astype(np.float32)
    if ds.dtype.big:
        return arr.astype(arr.dtype.newbyteorder("="))
    return arr


def _open_h5(path, rows, cols, unprocessed, scan_name):
    """scan.zig:536-791 — an h5ebsd-like file: the scan group (the named one, else the first group
    holding EBSD/Data and EBSD/Header), the patterns, and the header's geometry as each writer
    states it; else EMsoft's EMData/EBSD/EBSDPatterns."""
    try:
        h = H5.File(path)
    except H5.H5Unsupported as e:
        raise ScanError(f"UnsupportedHdf5: {e}") from None
    except H5.H5Error as e:
        raise ScanError(f"BadScanFile: {e}") from None
    try:
        return _open_h5_in(h, rows, cols, unprocessed, scan_name)
    except H5.H5Unsupported as e:
        raise ScanError(f"UnsupportedHdf5: {e}") from None
    except H5.H5Error as e:
        raise ScanError(f"BadScanFile: {e}") from None


def _open_h5_in(h, rows, cols, unprocessed, scan_name):
    scan = None
    for nm in h.list(h.root):
        if scan_name and nm != scan_name:
            continue
        a = h.child(h.root, nm)
        if a is None or not h.is_group(a):
            continue
        e = h.child(a, "EBSD")
        if e is not None and h.child(e, "Data") is not None and h.child(e, "Header") is not None:
            scan = a
            break
    if scan is None:
        a = h.find("EMData/EBSD/EBSDPatterns")
        if a is not None:
            return _open_emsoft(h, a, rows, cols)
        raise ScanError("NoScanInFile")
    ebsd = h.child(scan, "EBSD")
    data, header = h.child(ebsd, "Data"), h.child(ebsd, "Header")
    info = _blank_info()
    vendor = None
    for v in _H5_VENDORS:
        if h.child(header, v[2]) is None:
            continue
        processed = next((a for a in (h.child(data, pn) for pn in v[1]) if a is not None), None)
        raw = h.child(data, v[9]) if v[9] else None
        if processed is None and raw is None:
            continue
        vendor = v
        if v[9]:
            info["pattern_kinds"] = [k for k, a in (("processed", processed), ("unprocessed", raw)) if a is not None]
        info["unprocessed"] = raw is not None and (processed is None or unprocessed)
        pat_addr = raw if info["unprocessed"] else processed
        break
    if vendor is None:
        raise ScanError("NoPatternsInFile")
    fmt, _, k_rows, k_cols, k_sx, k_sy, k_tilt, k_det, k_bg, _, k_ubg = vendor
    ds = h.dataset(pat_addr)
    if ds.shape is None or len(ds.shape) not in (3, 4):
        raise ScanError("NoPatternsInFile")
    _h5_pixels(ds)
    info["pat_h"], info["pat_w"] = int(ds.shape[-2]), int(ds.shape[-1])
    n_stored = ds.shape[0] * ds.shape[1] if len(ds.shape) == 4 else ds.shape[0]
    r, c = _h5_get(h, header, k_rows), _h5_get(h, header, k_cols)
    info["rows"] = int(r) if r > 0 else 0
    info["cols"] = int(c) if c > 0 else 0
    if rows and cols:
        info["rows"], info["cols"] = rows, cols
    if info["rows"] * info["cols"] != n_stored:
        if len(ds.shape) == 4:
            info["rows"], info["cols"] = int(ds.shape[0]), int(ds.shape[1])
        elif info["rows"] == 0 or info["cols"] == 0:
            info["rows"], info["cols"] = 1, int(n_stored)
        else:
            raise ScanError("ScanIsNotAFullGrid")
    info["overview"] = _h5_overview(h, data, info["rows"], info["cols"])
    info["stored"] = lambda: _h5_stored(h, data, fmt, info["rows"] * info["cols"])
    info["step_x_um"], info["step_y_um"] = _h5_get(h, header, k_sx), _h5_get(h, header, k_sy)
    info["sample_tilt_deg"] = _h5_get(h, header, k_tilt)
    if math.isnan(info["sample_tilt_deg"]) and fmt == "Bruker h5ebsd":
        info["sample_tilt_deg"] = _h5_get(h, header, "Sample Tilt")
    info["detector_tilt_deg"] = _h5_get(h, header, k_det)
    ratio = info["pat_w"] / info["pat_h"]
    pc = None
    if fmt == "kikuchipy h5ebsd":
        pc = [_h5_mean(h, header, k) for k in ("pcx", "pcy", "pcz")]
        px, binning = _h5_get(h, header, "detector_pixel_size"), _h5_get(h, header, "binning")
        if px > 1:  # kikuchipy writes 1 when the size is unknown
            info["px_um"] = px * (binning if binning > 0 else 1)
        sem = h.child(scan, "SEM")
        sh = h.child(sem, "Header") if sem is not None else None
        if sh is not None:
            info["voltage_kv"] = _h5_get(h, sh, "beam_energy")
    elif fmt == "Bruker h5ebsd":
        pc = [_h5_mean(h, data, k) for k in ("PCX", "PCY", "DD")]
        full, unclipped = _h5_get(h, header, "DetectorFullHeightMicrons"), _h5_get(h, header, "UnClippedPatternHeight")
        if full > 0 and unclipped > 0:
            info["px_um"] = full / unclipped
        # a clipped pattern's PCY is a fraction of the height before clipping, from the top; DD
        # of the stored height (scan.zig:707-716)
        if unclipped > info["pat_h"] and not math.isnan(pc[1]):
            pc[1] *= unclipped / info["pat_h"]
            info["pc_note"] = ("Bruker's PCY read as a fraction of the pattern's height before clipping "
                               "(UnClippedPatternHeight), DD of its stored height")
        info["voltage_kv"] = _h5_get(h, header, "KV")
    elif fmt == "EDAX h5ebsd":
        dia = _h5_get(h, header, "Camera Diameter")  # the pattern spans the camera (millimetres)
        if dia > 0 and info["pat_w"] > 0:
            info["px_um"] = 1000.0 * dia / info["pat_w"]
        cal = h.child(header, "Pattern Center Calibration")
        if cal is not None:
            x, y, z = (_h5_get(h, cal, k) for k in ("x-star", "y-star", "z-star"))
            # y from the bottom, x and y fractions of the width and height, z of the smaller of
            # the two; all zero means not calibrated
            if x != 0 or y != 0 or z != 0:
                pc = [x, 1 - y, z * min(ratio, 1)]
    else:  # Oxford: y from the bottom, y and z fractions of the width; the tilt in radians
        x, y, z = (_h5_mean(h, data, k) for k in ("Pattern Center X", "Pattern Center Y", "Detector Distance"))
        pc = [x, 1 - y * ratio, z * ratio]
        dx, dy, dz = (_h5_drift(h, data, k, info["rows"], info["cols"])
                      for k in ("Pattern Center X", "Pattern Center Y", "Detector Distance"))
        info["pc_per_col"] = [dx[0], -dy[0] * ratio, dz[0] * ratio]
        info["pc_per_row"] = [dx[1], -dy[1] * ratio, dz[1] * ratio]
        turn = _h5_get(h, header, "Scanning Rotation Angle")
        info["scan_turn"] = 1
        if math.isfinite(turn):
            w = turn % (2 * math.pi)
            if abs(w - math.pi) <= 1e-4:
                info["turn_note"] = "a half turn: the beam as the scan signs say"
            elif min(w, 2 * math.pi - w) <= 1e-4:
                info["scan_turn"] = -1
                info["turn_note"] = "none: the beam the other way from what the scan signs say"
            else:
                info["turn_note"] = "neither none nor a half turn, which is not read: the beam as the scan signs say"
        info["sample_tilt_deg"] = math.degrees(info["sample_tilt_deg"])
        info["tilt_axis_deg"] = math.degrees(_h5_get(h, header, "Tilt Axis"))
        eu = _h5_values(h, header, "Detector Orientation Euler")
        if eu is not None and eu.size == 3:
            info["detector_rot"] = oxford_detector_rot(eu)
        info["voltage_kv"] = _h5_get(h, header, "Beam Voltage")
    if pc is not None and not any(math.isnan(v) for v in pc):
        info["pc"] = tuple(float(v) for v in pc)
    bg_name = k_ubg if info.get("unprocessed") else k_bg
    a = h.child(header, bg_name) if bg_name else None
    if a is not None:
        try:
            bds = h.dataset(a)
            whole = bds.elements == info["pat_h"] * info["pat_w"]
            if k_ubg:  # (an Oxford acquisition's: only this detector's pixels, a row at a time)
                whole = bds.shape == (info["pat_h"], info["pat_w"])
            if whole and bds.dtype.kind in "uif":
                info["background"] = np.asarray(h.read(bds), np.float32).reshape(info["pat_h"], info["pat_w"])
        except H5.H5Error:
            pass
    pats = _h5_patterns(h, ds).reshape(n_stored, info["pat_h"], info["pat_w"])
    return Scan(fmt, pats, info)


def _open_emsoft(h, pat_addr, rows, cols):
    """scan.zig:793-838 — EMsoft's EMEBSD output: patterns (n, h, w) and the simulation's detector
    parameters (EBSDNameList: xpc, ypc pixel offsets of the pattern centre from the detector's
    middle, L and the pixel size delta in micrometres, at the unbinned size numsx × numsy)."""
    ds = h.dataset(pat_addr)
    if ds.shape is None or len(ds.shape) != 3:
        raise ScanError("NoPatternsInFile")
    k, sz = ds.dtype.kind, ds.dtype.size
    if not ((k == "u" and sz in (1, 2)) or (k == "f" and sz == 4)):
        raise ScanError("UnsupportedPixelType")
    info = _blank_info()
    n = int(ds.shape[0])
    info["pat_h"], info["pat_w"] = int(ds.shape[1]), int(ds.shape[2])
    info["rows"], info["cols"] = 1, n
    if rows and cols and rows * cols == n:
        info["rows"], info["cols"] = rows, cols
    # EMsoft's per-pattern scalars sit beside EBSDPatterns
    info["overview"] = _h5_overview(h, h.find("EMData/EBSD"), info["rows"], info["cols"])
    nml = h.find("NMLparameters/EBSDNameList")
    if nml is not None:
        xpc, ypc, L, delta, numsx, numsy = (_h5_get(h, nml, k) for k in ("xpc", "ypc", "L", "delta", "numsx", "numsy"))
        if delta > 0 and numsx > 0 and numsy > 0 and not math.isnan(xpc + ypc + L):
            info["pc"] = (0.5 - xpc / numsx, 0.5 - ypc / numsy, L / (numsy * delta))
            info["px_um"] = delta * numsy / info["pat_h"]
        info["detector_tilt_deg"] = _h5_get(h, nml, "thetac")
        info["voltage_kv"] = _h5_get(h, nml, "energymax")
        mc = h.find("NMLparameters/MCCLNameList")
        if mc is not None:
            info["sample_tilt_deg"] = _h5_get(h, mc, "sig")
    return Scan("EMsoft patterns", _h5_patterns(h, ds), info)
