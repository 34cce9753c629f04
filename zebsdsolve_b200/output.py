"""The results as the text files other EBSD software reads (the reference's src/output.zig
exportText): EDAX/TSL .ang and HKL .ctf, the orientations as Bunge angles of the stored
quaternions (each in its phase's fundamental zone) in the engine's own frame (sample x on the
surface toward the detector, z out of it; each master's crystal axes X ∥ a, Z ∥ c*). Cells not
indexed carry the formats' own markers.
"""
import math

import numpy as np

from . import rotations as R

VERSION = "0.2.8"
# output.zig:124-138 — the TSL symmetry code of each Laue class, and the class's number (sym.zig)
TSL = {"c1": 1, "c2": 2, "d2": 22, "c4": 4, "d4": 42, "c3": 3, "d3": 32, "c6": 6, "d6": 62, "t": 23, "o": 43}
LAUE_NUMBER = {"c1": 1, "c2": 2, "d2": 3, "c4": 4, "d4": 5, "c3": 6, "d3": 7, "c6": 8, "d6": 9, "t": 10, "o": 11}


class ExportError(ValueError):
    pass


def export_text(kind, res, phases, geo, rows, cols, pat_h, pat_w, voltage_kv=float("nan"), frame=None):
    """output.zig:148-216 — kind "ang" or "ctf". res: quat [n, 4], ncc, nmi, phase [n] (−1: not
    indexed); phases: dicts of name, laue (the Laue class's key), lattice (a, b, c, α, β, γ) and
    space_group; geo: pc (Bruker), step_x_um, step_y_um, sample_tilt_deg; frame: the convention
    the orientations are written in (convention.Frame; None: the engine's own), named in the
    header."""
    from .convention import Frame

    frame = frame or Frame()
    crystal = []
    for p in phases:
        c = frame.crystal_of(p.get("lattice")) if p.get("lattice") is not None else None
        if c is None:
            raise ExportError("MissingPhaseLattice: a phase's master names no cell (a, b, c, α, β, γ)")
        crystal.append(c)
    q = np.asarray(res["quat"], np.float64).reshape(-1, 4)
    phase = np.asarray(res["phase"]).reshape(-1)
    if frame.is_engine():
        bunge = R.to_bunge(q)
    else:
        c = np.array(crystal + [[1.0, 0.0, 0.0, 0.0]])[np.where((phase >= 0) & (phase < len(crystal)), phase, -1)]
        bunge = R.to_bunge(frame.to_frame(q, c))
    frame_text = frame.describe()
    ncc = np.asarray(res["ncc"], np.float64).reshape(-1)
    nmi = np.asarray(res["nmi"], np.float64).reshape(-1)
    n_ph = len(phases)
    out = []
    if kind == "ang":
        ratio = pat_w / pat_h
        # EDAX measures the pattern centre's y from the bottom, x and y in fractions of the width
        # and height, z of the smaller of the two
        out.append(f"# TEM_PIX_PER_UM          1.000000\n# x-star                 {geo.pc[0]:.6f}\n"
                   f"# y-star                 {1 - geo.pc[1]:.6f}\n# z-star                 {geo.pc[2] / min(ratio, 1):.6f}\n"
                   "# WorkingDistance        0.000000\n#\n")
        for pi, p in enumerate(phases):
            L = p["lattice"]
            out.append(f"# Phase {pi + 1}\n# MaterialName  \t{p['name']}\n# Formula     \t\n# Info \t\t\n"
                       f"# Symmetry              {TSL[p['laue']]}\n"
                       f"# LatticeConstants      {L[0]:.8f} {L[1]:.8f} {L[2]:.8f}  {L[3]:.8f}  {L[4]:.8f}  {L[5]:.8f}\n"
                       "# NumberFamilies        0\n#\n")
        out.append(f"# GRID: SqrGrid\n# XSTEP: {geo.step_x_um:.6f}\n# YSTEP: {geo.step_y_um:.6f}\n# NCOLS_ODD: {cols}\n"
                   f"# NCOLS_EVEN: {cols}\n# NROWS: {rows}\n#\n# SOFTWARE: zebsdsolve {VERSION} (EDAX pattern centre)\n"
                   f"# FRAME: {frame_text}\n# COLUMNS: phi1 PHI phi2 x y IQ(NMI) CI(NCC) Phase SEM Fit\n")
        for r in range(rows):
            for c in range(cols):
                at = r * cols + c
                x, y = c * geo.step_x_um, r * geo.step_y_um
                ph = int(phase[at])
                if ph < 0:
                    out.append(f"  12.56637   12.56637   12.56637 {x:12.5f} {y:12.5f}      0.0  -1.000  0      0  0.000\n")
                    continue
                b = bunge[at]
                pid = 0 if n_ph == 1 else ph + 1  # single-phase files number the phase 0
                out.append(f"{b[0]:10.5f} {b[1]:10.5f} {b[2]:10.5f} {x:12.5f} {y:12.5f} {nmi[at]:8.4f} {ncc[at]:7.4f} "
                           f"{pid:2d} {0:6d} {0.0:6.3f}\n")
    elif kind == "ctf":
        kv = 0.0 if math.isnan(voltage_kv) else voltage_kv
        out.append(f"Channel Text File\nPrj\tzebsdsolve; frame {frame_text}\nAuthor\t\nJobMode\tGrid\nXCells\t{cols}\n"
                   f"YCells\t{rows}\nXStep\t{geo.step_x_um:.6f}\nYStep\t{geo.step_y_um:.6f}\nAcqE1\t0\nAcqE2\t0\nAcqE3\t0\n")
        out.append(f"Euler angles refer to Sample Coordinate system (CS0)!\tMag\t0\tCoverage\t100\tDevice\t0\tKV\t{kv:.1f}"
                   f"\tTiltAngle\t{geo.sample_tilt_deg:.2f}\tTiltAxis\t0\n")
        out.append(f"Phases\t{n_ph}\n")
        for p in phases:
            L = p["lattice"]
            out.append(f"{L[0]:.8f};{L[1]:.8f};{L[2]:.8f}\t{L[3]:.8f};{L[4]:.8f};{L[5]:.8f}\t{p['name']}\t"
                       f"{LAUE_NUMBER[p['laue']]}\t{p['space_group']}\t\t\t\n")
        out.append("Phase\tX\tY\tBands\tError\tEuler1\tEuler2\tEuler3\tMAD\tBC\tBS\n")
        deg = 180.0 / math.pi
        for r in range(rows):
            for c in range(cols):
                at = r * cols + c
                x, y = c * geo.step_x_um, r * geo.step_y_um
                ph = int(phase[at])
                if ph < 0:
                    out.append(f"0\t{x:.4f}\t{y:.4f}\t0\t3\t0.0000\t0.0000\t0.0000\t0.0000\t0\t0\n")
                    continue
                b = bunge[at] * deg
                bc = int(math.floor(255 * min(max(ncc[at], 0.0), 1.0) + 0.5))
                bs = int(math.floor(255 * min(max(nmi[at], 0.0), 1.0) + 0.5))
                out.append(f"{ph + 1}\t{x:.4f}\t{y:.4f}\t0\t0\t{b[0]:.4f}\t{b[1]:.4f}\t{b[2]:.4f}\t0.0000\t{bc}\t{bs}\n")
    else:
        raise ExportError(f"UnknownKind: {kind!r}")
    return "".join(out)


# output.zig:10-13: the colours of phases and sweeps (the label modulo eight), as the reference's maps
# draw them, so that a map made here matches one made there pixel for pixel
PALETTE = np.array([[0x3b, 0x82, 0xf6], [0xf5, 0x9e, 0x0b], [0x10, 0xb9, 0x81], [0xef, 0x44, 0x44],
                    [0x8b, 0x5c, 0xf6], [0x14, 0xb8, 0xa6], [0xec, 0x48, 0x99], [0x84, 0xcc, 0x16]], np.uint8)
NO_SWEEP = np.array([0x3a, 0x3a, 0x3e], np.uint8)
MAPS = {"ipf_x": 0, "ipf_y": 1, "ipf_z": 2, "ncc": 3, "nmi": 4, "phase": 5, "z": 6, "sweep": 7}


def result_map(kind, res):
    """output.zig:15-84 — a result map as RGBA8 (n, 4), cells in map order: kind 3 NCC, 4 NMI and 6
    the NMI's distance above chance as gray between the indexed cells' extremes (one level where
    they are equal; values past them clamped), 5 the phase's colour, 7 the colour of the sweep that
    accepted the cell (dark gray: none did). Cells not indexed are transparent black. Kinds 0-2,
    the inverse pole figure colours, take the colour keys of the crystal classes, which this
    package does not build: they raise."""
    if kind not in range(8):
        raise ValueError("UnknownKind")
    if kind <= 2:
        raise NotImplementedError("NotImplemented: IPF colours (their keys are not part of this engine)")
    phase = np.asarray(res["phase"])
    ok = phase >= 0
    out = np.zeros((phase.size, 4), np.uint8)
    if kind in (3, 4, 6):
        v = np.asarray(res[{3: "ncc", 4: "nmi", 6: "z"}[kind]], np.float32)
        # extremes over the indexed cells, NaN passed over (the minimum and maximum of IEEE 754-2008)
        lo = np.fmin.reduce(v[ok], initial=np.float32(np.inf)).astype(np.float32)
        hi = np.fmax.reduce(v[ok], initial=np.float32(-np.inf)).astype(np.float32)
        if not hi > lo:
            hi = np.float32(lo + np.float32(1))
        with np.errstate(invalid="ignore", divide="ignore", over="ignore"):
            t = np.fmax(np.float32(0), np.fmin((v - lo) / (hi - lo), np.float32(1)))
            gray = np.floor(np.float32(255) * t + np.float32(0.5))  # (t ≥ 0: half away from zero)
        out[:, :3] = np.nan_to_num(gray, nan=0.0).astype(np.uint8)[:, None]
    elif kind == 5:
        out[:, :3] = PALETTE[np.where(ok, phase, 0) % len(PALETTE)]
    else:
        sw = np.asarray(res["sweep"])
        out[:, :3] = np.where((sw < 0)[:, None], NO_SWEEP, PALETTE[np.where(sw < 0, 0, sw) % len(PALETTE)])
    out[:, 3] = 255
    out[~ok] = 0
    return out

