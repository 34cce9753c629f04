"""Reference-frame conventions, and how to find the one a maker's stored orientations are in
(zebsdsolve src/convention.zig).

A convention is three choices: the sample axes (which of the engine's axes, with which sign, each
of the convention's X, Y, Z is: the 24 right-handed ways), passive or active angles, and how the
crystal axes sit on the lattice (X ∥ a, Z ∥ c* — the masters' own; X ∥ a*, Z ∥ c; Y ∥ b, Z ∥ c*;
Y ∥ b*, Z ∥ c). The engine computes in its own (the first of each). `identify` compares a maker's
orientations with the engine's results cell by cell, under each phase's own proper rotations,
over every convention, and measures the misorientation that remains between the two (its value at
the map's middle and its change over the rows and the columns), which no convention removes and
nothing applies. Vectorised over cells with numpy (host work: once per scan).
"""
import math

import numpy as np

from . import rotations as R

CRYSTAL_AXES = ("x_a_z_cstar", "x_astar_z_c", "y_b_z_cstar", "y_bstar_z_c")
CRYSTAL_LABELS = {"x_a_z_cstar": "X||a Z||c*", "x_astar_z_c": "X||a* Z||c", "y_b_z_cstar": "Y||b Z||c*",
                  "y_bstar_z_c": "Y||b* Z||c"}
MAX_PHASES = 16
# convention.zig:315-316: the order the sample axes are tried in (the engine's first: it wins ties)
_PERMS = ((1, 2, 3), (1, 3, 2), (2, 1, 3), (2, 3, 1), (3, 1, 2), (3, 2, 1))
_SIGNS = ((1, 1, 1), (1, -1, -1), (-1, 1, -1), (-1, -1, 1), (-1, -1, -1), (-1, 1, 1), (1, -1, 1), (1, 1, -1))


class ConventionError(ValueError):
    pass


def from_bunge(e):
    """Bunge angles (φ1, Φ, φ2) [..., 3] → quaternions [..., 4] with w ≥ 0 (rot.zig:142-148)."""
    e = np.asarray(e, np.float64)
    sigma, delta = 0.5 * (e[..., 0] + e[..., 2]), 0.5 * (e[..., 0] - e[..., 2])
    c, s = np.cos(0.5 * e[..., 1]), np.sin(0.5 * e[..., 1])
    return R.qstd(np.stack([c * np.cos(sigma), -s * np.cos(delta), -s * np.sin(delta), -c * np.sin(sigma)], -1))


def _axes_matrix(axes):
    m = np.zeros((3, 3))
    for i, a in enumerate(axes):
        k = abs(int(a))
        if not 1 <= k <= 3:
            return np.zeros((3, 3))
        m[i, k - 1] = -1.0 if a < 0 else 1.0
    return m


class Frame:
    """A convention (convention.zig:54-110): `axes` the convention's sample X, Y, Z as the
    engine's axes (1 x, 2 y, 3 z; negative: reversed), `active` (angles taking the crystal's axes
    to the sample's), `crystal` one of CRYSTAL_AXES."""

    def __init__(self, axes=(1, 2, 3), active=False, crystal="x_a_z_cstar"):
        self.axes, self.active, self.crystal = tuple(int(a) for a in axes), bool(active), str(crystal)

    def key(self):
        return self.axes, self.active, self.crystal

    def __eq__(self, other):
        return isinstance(other, Frame) and self.key() == other.key()

    def valid(self):
        ks = [abs(a) for a in self.axes]
        return (len(ks) == 3 and sorted(ks) == [1, 2, 3] and self.crystal in CRYSTAL_AXES
                and np.linalg.det(_axes_matrix(self.axes)) > 0)

    def is_engine(self):
        return self == Frame()

    def sample(self):
        """The rotation taking the engine's coordinates to the convention's sample axes."""
        return R.from_matrix(_axes_matrix(self.axes))

    def crystal_of(self, lattice):
        return crystal_rotation(self.crystal, lattice)

    def to_frame(self, q, c):
        """Orientations in the engine's frame [..., 4] as this convention writes them; `c` the
        phase's `crystal_of` (convention.zig:90-94)."""
        g = R.qmul(R.qmul(c, q), R.qconj(self.sample()))
        return R.qstd(R.qconj(g) if self.active else g)

    def from_frame(self, g0, c):
        """The inverse of `to_frame` (convention.zig:96-100)."""
        g = R.qconj(g0) if self.active else np.asarray(g0, np.float64)
        return R.qstd(R.qmul(R.qmul(R.qconj(c), g), self.sample()))

    def describe(self):
        """One ASCII line, as the exports' headers carry it: "X +y Y -x Z +z, passive, X||a* Z||c"."""
        parts = [f"{'XYZ'[i]} {'-' if a < 0 else '+'}{'xyz'[abs(a) - 1]}" for i, a in enumerate(self.axes)]
        return " ".join(parts) + f", {'active' if self.active else 'passive'}, {CRYSTAL_LABELS[self.crystal]}"

    def as_dict(self):
        return {"axes": list(self.axes), "active": self.active, "crystal": self.crystal, "text": self.describe()}

    @classmethod
    def from_dict(cls, d):
        """A frame from {"axes", "active", "crystal"} (other keys ignored; absent ones the engine's);
        InvalidFrame unless it is one of the conventions (exports.zig:849-859)."""
        try:
            f = cls(d.get("axes", (1, 2, 3)), d.get("active", False), d.get("crystal", "x_a_z_cstar"))
        except (TypeError, ValueError):
            raise ConventionError("InvalidFrame") from None
        if not isinstance(d.get("active", False), bool) or not f.valid():
            raise ConventionError("InvalidFrame")
        return f


def crystal_rotation(axes, lattice):
    """convention.zig:122-162 — the rotation taking a master's Cartesian axes (X ∥ a, Z ∥ c*) to
    the convention's crystal axes on the cell (a, b, c in Å; α, β, γ in degrees); None where the
    description needs a cell and there is no valid one."""
    if axes == "x_a_z_cstar":
        return np.array([1.0, 0.0, 0.0, 0.0])
    if lattice is None:
        return None
    lat = [float(v) for v in lattice]
    if not all(v > 0 and math.isfinite(v) for v in lat):
        return None
    ca, cb, cg = (math.cos(math.radians(v)) for v in lat[3:])
    sg = math.sin(math.radians(lat[5]))
    vol = 1 - ca * ca - cb * cb - cg * cg + 2 * ca * cb * cg
    if not (vol > 0 and sg > 0):
        return None
    a = np.array([lat[0], 0.0, 0.0])
    b = np.array([lat[1] * cg, lat[1] * sg, 0.0])
    c = np.array([lat[2] * cb, lat[2] * (ca - cb * cg) / sg, lat[2] * math.sqrt(vol) / sg])

    def unit(v):
        return v / np.linalg.norm(v)
    if axes == "x_astar_z_c":
        x, z = unit(np.cross(b, c)), unit(c)
        y = np.cross(z, x)
    elif axes == "y_b_z_cstar":
        y, z = unit(b), unit(np.cross(a, b))
        x = np.cross(y, z)
    else:
        y, z = unit(np.cross(c, a)), unit(c)
        x = np.cross(y, z)
    return R.from_matrix(np.array([x, y, z]))


def _best_w(rotations, d):
    """|scalar part of g · d| for each rotation g of a phase [..., k], d [..., 4]."""
    g = np.asarray(rotations, np.float64)
    return np.abs(d @ (g * np.array([1.0, -1.0, -1.0, -1.0])).T)


def _apart(rotations, a, b):
    """convention.zig:201-211 — the smallest angle between a and the g · b (radians)."""
    w = _best_w(rotations, R.qmul(a, R.qconj(b))).max(-1)
    return 2 * np.arccos(np.minimum(w, 1.0))


def _median(x):
    """The upper median (convention.zig:215-219); π for none."""
    return float(np.sort(x)[len(x) // 2]) if len(x) else math.pi


def match_labels(phase, ref_phase, n_phases):
    """convention.zig:224-252 — each engine phase's label in the reference: the one it gives most
    often where the engine found that phase (−1: none; ties to the smaller label)."""
    matched = [-1] * MAX_PHASES
    p, r = np.asarray(phase, np.int64), np.asarray(ref_phase, np.int64)
    ok = (p >= 0) & (p < n_phases) & (p < MAX_PHASES) & (r >= 0)
    for k in np.unique(p[ok]):
        labels, counts = np.unique(r[ok & (p == k)], return_counts=True)
        matched[int(k)] = int(labels[np.argmax(counts)])  # (sorted labels: the first of the most is the smallest)
    return matched


def _thin(phase_sorted, most):
    """convention.zig:410-424 — indices of up to `most` of each phase's pairs, evenly spread."""
    out = []
    i, n = 0, len(phase_sorted)
    while i < n:
        j = i
        while j < n and phase_sorted[j] == phase_sorted[i]:
            j += 1
        out.extend(range(i, j, max(1, (j - i + most - 1) // most)))
        i = j
    return np.array(out, np.int64)


def _score(frame, q, g, ph, rotations, crot):
    """convention.zig:426-446 — each phase's median angle under `frame` over its pairs (phases with
    five pairs or more), averaged over the phases; π for none."""
    total, count = 0.0, 0
    for p in np.unique(ph):
        at = ph == p
        if at.sum() >= 5:
            total += _median(_apart(rotations[p], q[at], frame.from_frame(g[at], crot[p])))
            count += 1
    return total / count if count else math.pi


def identify(q, phase, cols, ref_euler, ref_phase, phases):
    """convention.zig:254-404 — the convention of a reference's orientations against the engine's
    results. q: [n, 4] the engine's orientations; phase: [n] (−1 not indexed); cols: the map's
    width; ref_euler: [n, 3] Bunge radians; ref_phase: [n] labels (negative: not indexed); phases:
    [(rotations [k, 4], lattice or None)]. Returns (Frame, a dict of cells, within, median_deg,
    runner_up_deg, matched, misorientation, misorientation_rows, misorientation_cols,
    misorientation_cells)."""
    q = np.asarray(q, np.float64).reshape(-1, 4)
    phase = np.asarray(phase, np.int64).reshape(-1)
    n = len(phase)
    ref_euler = np.asarray(ref_euler, np.float64).reshape(-1)
    ref_phase = np.asarray(ref_phase, np.int64).reshape(-1)
    if len(q) != n or ref_euler.size != 3 * n or ref_phase.size != n:
        raise ConventionError("BadLength")
    if not phases or len(phases) > MAX_PHASES:
        raise ConventionError("NoPhases")
    matched = match_labels(phase, ref_phase, len(phases))
    e = ref_euler.reshape(n, 3)
    lab = np.array(matched + [-1])[np.clip(phase, 0, MAX_PHASES)]
    keep = ((phase >= 0) & (phase < len(phases)) & (ref_phase >= 0) & (ref_phase == lab)
            & np.all(np.isfinite(e), 1))
    cells = np.flatnonzero(keep)
    if len(cells) < 8:
        raise ConventionError("TooFewCommonCells")
    # grouped by phase (stably: in cell order within a phase), each phase scored by itself
    cells = cells[np.argsort(phase[cells], kind="stable")]
    ph, qq, gg = phase[cells], R.qstd(q[cells]), from_bunge(e[cells])
    fit = _thin(ph, 2000)
    probe = fit[_thin(ph[fit], 300)]
    rotations = [np.asarray(r, np.float64) for r, _ in phases]
    # the crystal descriptions that differ for some phase in play (the rest give the same results)
    crystals = []
    for cand in CRYSTAL_AXES:
        distinct = not crystals
        for seen in crystals:
            differs = False
            for rots, lat in phases:
                a, b = crystal_rotation(cand, lat), crystal_rotation(seen, lat)
                if a is not None and b is not None and _apart(rots, a[None], b[None])[0] > 1e-6:
                    differs = True
            distinct = differs
            if not distinct:
                break
        if distinct:
            crystals.append(cand)
    ident = np.array([1.0, 0.0, 0.0, 0.0])
    crot = {k: [crystal_rotation(c, lat) if crystal_rotation(c, lat) is not None else ident
                for _, lat in phases] for k, c in enumerate(crystals)}
    best, best_med, second = Frame(), math.inf, math.inf
    for active in (False, True):
        for k, c in enumerate(crystals):
            for pm in _PERMS:
                for sg in _SIGNS:
                    cand = Frame(tuple(a * s for a, s in zip(pm, sg)), active, c)
                    if not cand.valid():
                        continue
                    med = _score(cand, qq[probe], gg[probe], ph[probe], rotations, crot[k])
                    if med < best_med - 1e-9:
                        if best_med < second and best.key() != cand.key():
                            second = best_med
                        best_med, best = med, cand
                    elif med < second:
                        second = med
    kb = crystals.index(best.crystal)
    cb = np.array([crot[kb][p] for p in ph])
    r = best.from_frame(gg, cb)
    every = np.concatenate([_apart(rotations[p], qq[ph == p], r[ph == p]) for p in np.unique(ph)])
    out = {"cells": int(len(cells)), "within": float(np.mean(every < math.radians(2.0))),
           "median_deg": math.degrees(_median(every)), "runner_up_deg": math.degrees(second),
           "matched": matched[:len(phases)]}
    # the misorientation left: on each cell within a few degrees, the rotation m of the engine's
    # sample axes with reference = c · gk · q · (a · m)*, gk the closest symmetric equivalent; then
    # the plane m = m0 + u · m_rows + w · m_cols, u and w the cell's row and column from −½ to ½
    near = math.radians(max(5.0, 3 * out["median_deg"]))
    a = R.from_matrix(_axes_matrix(best.axes))
    rows = (n + cols - 1) // cols if cols > 0 else 0
    ata, atb, used = np.zeros((3, 3)), np.zeros((3, 3)), 0
    for p in np.unique(ph):
        at = ph == p
        d = R.qmul(qq[at], R.qconj(r[at]))
        w = _best_w(rotations[p], d)
        kbest = np.argmax(w, 1)
        top = w[np.arange(len(w)), kbest]
        ok = 2 * np.arccos(np.minimum(top, 1.0)) <= near
        if not ok.any():
            continue
        gk = rotations[p][kbest[ok]]
        passive = R.qconj(gg[at][ok]) if best.active else gg[at][ok]
        c = cb[at][ok]
        t = R.qmul(R.qmul(R.qmul(R.qconj(passive), c), R.qmul(gk, qq[at][ok])), R.qconj(a))
        m = R.log_map(R.qstd(R.qmul(R.qmul(R.qconj(a), t), a)))
        cell = cells[at][ok]
        u = (cell // cols) / (rows - 1) - 0.5 if rows > 1 else np.zeros(len(cell))
        v = (cell % cols) / (cols - 1) - 0.5 if cols > 1 else np.zeros(len(cell))
        x = np.stack([np.ones(len(cell)), u, v], 1)
        ata += x.T @ x
        atb += (x.T @ m).T  # atb[k][i] = Σ x_i m_k
        used += int(ok.sum())
    mis = np.zeros((3, 3))
    if used >= 8:
        # cells all in one row or one column say nothing of a change that way: held at zero
        for i in (1, 2):
            if ata[i, i] - ata[0, i] * ata[0, i] / ata[0, 0] < 1e-6 * ata[0, 0]:
                ata[i, :], ata[:, i], ata[i, i] = 0, 0, 1
                atb[:, i] = 0
        mis = (np.linalg.inv(ata) @ atb.T).T  # mis[k] = (m0, m_rows, m_cols) of component k
    out.update(misorientation=[float(v) for v in mis[:, 0]], misorientation_rows=[float(v) for v in mis[:, 1]],
               misorientation_cols=[float(v) for v in mis[:, 2]], misorientation_cells=used)
    return best, out
