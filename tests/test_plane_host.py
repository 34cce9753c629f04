"""The plane of source points' arithmetic: the oracle (oracle/plane.py) pinned by the reference's
own known-answer tests (src/plane.zig:366-455, restated here on both the oracle and the product),
and the product (zebsdsolve_b200.plane, vectorized) against the oracle on weighted points of every
model. Tolerances: FP64 sums in another order, 1e-10 relative."""
import math

import numpy as np
import pytest

import oracle.geometry as og
import oracle.plane as opl
from zebsdsolve_b200 import plane as pl
from zebsdsolve_b200.engine import Geometry


def _grid(truth, aspect, at):
    rows, cols, y = [], [], []
    for i in range(7):
        for j in range(7):
            row, col = float(i * 6 + 1), float(j * 9 + 2)
            pc = at(truth, row, col)
            rows.append(row)
            cols.append(col)
            y.append([pc[0] * aspect, pc[1], pc[2]])
    return rows, cols, y


def _both(rows, cols, y, w=None, used=None):
    """The same points for the oracle (dicts) and the product (Points)."""
    n = len(rows)
    w = np.tile(np.eye(3), (n, 1, 1)) if w is None else np.asarray(w)
    used = np.ones(n, bool) if used is None else np.asarray(used)
    o = [opl.point(rows[k], cols[k], y[k], w[k].reshape(9), used[k]) for k in range(n)]
    return o, pl.Points(rows, cols, y, w, used)


def test_each_model_is_found_again_from_its_own_points():
    """plane.zig:366-392"""
    L = [0, 0, 0.43, 0, -3.6e-4, 0.22, 0, 1.3e-4, 0.5, 0, 0, 1]
    for lib, frame in ((opl, lambda: opl.frame_of(40, 60, 1.25)), (pl, lambda: pl.Frame(40, 60, 1.25))):
        fr = frame()
        rows, cols, y = _grid(L, 1.25, opl.at)
        o, p = _both(rows, cols, y)
        pts = o if lib is opl else p
        for m in ("line", "affine"):
            P = lib.fit_model(m, pts, fr)
            assert np.abs(np.asarray(P) - L).max() < 1e-11
        C = lib.fit_model("centre", pts, fr)
        mean = np.mean([opl.at(L, r, c) for r, c in zip(rows, cols)], 0)
        for k in range(3):
            assert abs(C[3 * k + 2] - mean[k]) < 1e-11
        for i in (0, 1, 3, 4, 6, 7):
            assert C[i] == 0


def test_a_plane_is_found_again_affine_and_projective():
    """plane.zig:394-413"""
    A = [-4.0e-4, 1.0e-5, 0.43, 2.0e-5, -3.6e-4, 0.22, -1.0e-5, 1.3e-4, 0.5, 0, 0, 1]
    Pp = list(A)
    Pp[9], Pp[10] = 2.0e-5, -3.0e-5
    for kind, truth in (("affine", A), ("projective", Pp)):
        rows, cols, y = _grid(truth, 1.25, opl.at)
        o, p = _both(rows, cols, y)
        for P in (opl.fit(kind, o, opl.frame_of(40, 60, 1.25)), pl.fit(kind, p, pl.Frame(40, 60, 1.25))):
            assert np.abs(np.asarray(P) - truth).max() < 1e-11, kind


def test_a_projective_plane_through_points_that_hardly_move():
    """plane.zig:415-437"""
    y0 = [0.4233, 0.2136, 0.5021]
    seed = 7
    for noise in (0.0, 1e-4):
        rows, cols, y = [], [], []
        for i in range(3):
            for j in range(3):
                v = list(y0)
                for k in range(3):
                    seed = (seed * 6364136223846793005 + 1442695040888963407) % (1 << 64)
                    v[k] += noise * ((seed >> 11) / 9007199254740992.0 - 0.5)
                rows.append(20.0 + i)
                cols.append(32.0 + j)
                y.append(v)
        o, p = _both(rows, cols, y)
        for theta in (opl.fit_theta("projective", o, opl.frame_of(55, 75, 1)),
                      pl.fit_theta("projective", p, pl.Frame(55, 75, 1))):
            if noise == 0:
                assert theta[9] == 0 and theta[10] == 0
            assert abs(theta[9]) + abs(theta[10]) < 0.01
            for k in range(3):
                assert abs(theta[3 * k + 2] - y0[k]) < 0.003


def test_the_plane_of_the_models_own_scan_says_its_geometry():
    """plane.zig:439-455"""
    kw = dict(pc=(0.42, 0.21, 0.5), px_um=560.0, step_x_um=30.0, step_y_um=40.0)
    g = og.Geometry(rot_vec=(0.02, -0.03, 0.04), **kw)
    gp = Geometry()
    gp.set(rot=(0.02, -0.03, 0.04), **kw)
    rows, cols = 30, 40
    Rm = g.rotation()
    t = g.translation(60, 60)
    fro = opl.frame_of(rows, cols, 1)
    rr, cc, yy = [], [], []
    for k in range(30):
        row, col = float((k * 7) % rows), float((k * 11) % cols)
        s = g.scan_offset(row, col, fro["r0"], fro["c0"], -1, -1, 1)
        pc = og.Geometry.pc_of(Rm, t - s, 60, 60)
        rr.append(row)
        cc.append(col)
        yy.append(pc)
    o, p = _both(rr, cc, yy)
    for w in (opl.said(opl.fit("affine", o, fro), g, rows, cols, 1, 60, -1, -1),
              pl.said(pl.fit("affine", p, pl.Frame(rows, cols, 1)), gp, rows, cols, 1, 60, -1, -1)):
        for i in range(3):
            assert abs(w["pc"][i] - kw["pc"][i]) < 1e-10
            assert abs(w["rot"][i] - (0.02, -0.03, 0.04)[i]) < 1e-9
        assert abs(w["step"][0] - 1) < 1e-9 and abs(w["step"][1] - 1) < 1e-9 and abs(w["skew"]) < 1e-9


@pytest.mark.parametrize("model", ["centre", "line", "affine", "projective"])
def test_product_matches_oracle_on_weighted_points(model):
    rng = np.random.default_rng(11)
    n, rows, cols = 60, 37, 53
    truth = [-4e-4, 2e-5, 0.45, 1e-5, -3e-4, 0.25, -2e-5, 1.5e-4, 0.52, 3e-5 if model == "projective" else 0,
             -2e-5 if model == "projective" else 0, 1]
    rr = rng.integers(0, rows, n).astype(float)
    cc = rng.integers(0, cols, n).astype(float)
    y = np.array([opl.at(truth, r, c) for r, c in zip(rr, cc)]) * np.array([1.3, 1, 1])
    y += rng.normal(0, 2e-4, y.shape)
    B = rng.normal(size=(n, 3, 3))
    w = np.einsum("pki,pkj->pij", B, B) + 0.1 * np.eye(3)
    used = rng.uniform(size=n) > 0.15
    o, p = _both(rr, cc, y, w, used)
    fro, frp = opl.frame_of(rows, cols, 1.3), pl.Frame(rows, cols, 1.3)
    to, tp = opl.fit_theta(model, o, fro), pl.fit_theta(model, p, frp)
    assert np.abs(np.asarray(to) - tp).max() < 1e-10 * max(1.0, np.abs(tp).max())
    Po, Pp = opl.to_plane(model, to, fro), pl.to_plane(model, tp, frp)
    assert np.abs(np.asarray(Po) - Pp).max() < 1e-10
    mo = [opl.misfit(Po, q, 1.3) for q in o]
    assert np.allclose(mo, pl.misfit(Pp, p, 1.3), rtol=1e-9, atol=1e-18)
    for k in range(n):
        yo, Jo = opl.model_at(to, fro, rr[k], cc[k])
        yp, Jp = pl.model_at(tp, frp, rr[k], cc[k])
        assert np.allclose(yo, yp, atol=1e-12) and np.allclose(np.reshape(Jo, (3, 11)), Jp, atol=1e-10)
    g = og.Geometry(pc=(0.45, 0.25, 0.52), px_um=50.0, step_x_um=2.0, step_y_um=3.0)
    gp = Geometry()
    gp.set(pc=(0.45, 0.25, 0.52), px_um=50.0, step_x_um=2.0, step_y_um=3.0)
    so, sp = opl.said(Po, g, rows, cols, 1.3, 60, 1, 1), pl.said(Pp, gp, rows, cols, 1.3, 60, 1, 1)
    for k in ("pc", "rot", "step"):
        assert np.allclose(so[k], sp[k], rtol=1e-9, atol=1e-12), k
    assert math.isclose(so["skew"], sp["skew"], rel_tol=1e-9, abs_tol=1e-12)


def test_too_few_points_and_unbounded_planes_are_refused():
    o, p = _both([0.0, 1.0], [0.0, 1.0], [[0.4, 0.2, 0.5], [0.41, 0.2, 0.5]])
    for m in ("affine", "projective"):
        assert opl.fit_theta(m, o, opl.frame_of(5, 5, 1)) is None and pl.fit_theta(m, p, pl.Frame(5, 5, 1)) is None
    assert not pl.bounded([0] * 9 + [0.5, 0.45]) and pl.bounded([0] * 9 + [0.5, 0.4])
