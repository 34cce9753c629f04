"""Scan files (the reference's src/scan.zig, src/ang.zig): the pattern files that need no HDF5
reader — EDAX .up1 / .up2 (with their scan's .ang for the map's shape, the steps and the pattern
centre), Oxford .ebsp (uncompressed) and NORDIF Pattern.dat (with Setting.txt). The patterns are
mapped from the file, not read into memory; numbered row-major over the map, top row first, as
stored. HDF5 scan files (h5ebsd of kikuchipy, Bruker, EDAX; Oxford .h5oina; EMsoft) are refused:
this engine has no HDF5 reader.
"""
import math
import os

import numpy as np


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
    sample_tilt_deg, detector_tilt_deg; NaN / None where the file says nothing)."""

    def __init__(self, fmt, patterns, info):
        self.format, self.patterns, self.info = fmt, patterns, info

    def map(self):
        """The first rows × cols patterns as (rows, cols, h, w)."""
        i = self.info
        return self.patterns[: i["rows"] * i["cols"]].reshape(i["rows"], i["cols"], i["pat_h"], i["pat_w"])


def _blank_info():
    nan = float("nan")
    return {"rows": 0, "cols": 0, "pat_h": 0, "pat_w": 0, "step_x_um": nan, "step_y_um": nan, "pc": None,
            "pc_note": "", "voltage_kv": nan, "sample_tilt_deg": nan, "detector_tilt_deg": nan}


def open_scan(paths, rows=0, cols=0, pat_h=0, pat_w=0):
    """scan.zig Scan.open — by the first path's extension; rows/cols (and for NORDIF pat_h, pat_w)
    say what the file does not."""
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
        raise ScanError(f"UnsupportedFormat: {os.path.basename(paths[0])} is an HDF5 file; this engine reads "
                        ".up1, .up2, .ebsp and NORDIF .dat scans (pass HDF5 patterns as an array)")
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
    gives the shape, the steps and the pattern centre."""
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
        if version >= 3 and (nx != ang["cols"] or ny != ang["rows"]):
            raise ScanError("ScanShapeMismatch")
        if version >= 3 and not (_same_step(dx, ang["step_x_um"]) and _same_step(dy, ang["step_y_um"])):
            raise ScanError("UPANGStepMismatch")
        if (rows and rows != ang["rows"]) or (cols and cols != ang["cols"]):
            raise ScanError("ScanShapeMismatch")
        info.update(rows=ang["rows"], cols=ang["cols"], step_x_um=ang["step_x_um"], step_y_um=ang["step_y_um"],
                    pc=ang["pc"], pc_note=ang["pc_note"])
    else:
        _shape(info, n, rows, cols)
    pats = np.memmap(paths[0], dt, "r", offset=off, shape=(n, h, w))
    return Scan("edax_up", pats, info)


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
            line = line.strip()
            if not line:
                continue
            if not line.startswith("#"):
                break
            content = line[1:].strip()
            parts = content.replace(":", " ").split(None, 1)
            if not parts:
                continue
            key, value = parts[0], (parts[1].strip(": \t") if len(parts) > 1 else "")
            k = {"x-star": 0, "y-star": 1, "z-star": 2}.get(key)
            if k is not None:
                if raw[k] is not None:
                    raise ScanError("DuplicateANGPatternCentre")
                try:
                    raw[k] = float(value.split()[0])
                except (ValueError, IndexError):
                    raise ScanError("InvalidANGPatternCentre") from None
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
                numeric_version = value.isdigit()
            elif key == "GRID":
                if value != "SqrGrid":
                    raise ScanError("UnsupportedANGGrid")
                square = True
            elif key == "NROWS":
                rows = int(value)
            elif key == "NCOLS_ODD":
                odd = int(value)
            elif key == "NCOLS_EVEN":
                even = int(value)
            elif key == "XSTEP":
                dx = float(value)
            elif key == "YSTEP":
                dy = float(value)
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
