"""The pattern-centre vote's host arithmetic (zebsdsolve_b200.pcfit) against the oracle's scalar
restatement of pcfit.zig: the fit lattices, the ballots and their densities, and the whole
search (levels, border walks, narrowing) over analytic score surfaces. Bit-equal: the vote is
deterministic host arithmetic in the reference's order."""
import math

import numpy as np
import pytest

import oracle.pcfit as opc
from zebsdsolve_b200 import pcfit
from zebsdsolve_b200.settings import Settings


def _settings(**kw):
    s = Settings()
    s.apply(kw)
    return s


def _region(rows, cols, roi=None):
    x0, y0, w, h = roi or (0, 0, cols, rows)
    return ((y0 + np.arange(h))[:, None] * cols + x0 + np.arange(w)[None, :]).reshape(-1)


@pytest.mark.parametrize("rows,cols,roi", [(8, 12, None), (3, 2, None), (50, 40, (5, 7, 20, 11)), (1, 9, None)])
def test_fit_lattices_match_oracle(rows, cols, roi):
    region = _region(rows, cols, roi)
    for grid in (1, 2, 5, 31):
        assert np.array_equal(pcfit.fit_cells(region, cols, grid), opc.fit_cells(region, cols, grid))
    for stride in (0, 1, 2, 3, 7):
        assert np.array_equal(pcfit.fit_cells_every(region, cols, stride), opc.fit_cells_every(region, cols, stride))
    # the reference's own case: 5 × 5 fit patterns on an 8 × 12 map, each in the middle of its share
    if (rows, cols, roi) == (8, 12, None):
        c = pcfit.fit_cells(region, cols, 5)
        assert len(c) == 25 and c[0] == 0 * 12 + 1 and c[-1] == 7 * 12 + 10


def _scores(rng, n_pat, n, lo, peaky=True):
    n_c = n[0] * n[1] * n[2]
    out = np.zeros((n_pat, n_c), np.float32)
    z, y, x = np.meshgrid(np.arange(n[2]), np.arange(n[1]), np.arange(n[0]), indexing="ij")
    for b in range(n_pat):
        c = rng.uniform(0, 1, 3) * (np.array(n) - 1)
        v = np.exp(-((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) / (2 * 1.5 ** 2)) if peaky else 0
        v = 0.5 * v + 0.2 * rng.uniform(0, 1, v.shape if peaky else x.shape)
        if b % 7 == 3:
            v = -np.abs(v)  # a pattern with nothing above zero casts no ballot
        out[b] = v.reshape(-1).astype(np.float32)
    out[:, :lo] = 0  # unscored slices hold zero
    # ties: equal values keep the lower candidate first
    out[0, lo + 3] = out[0, lo + 5] = out[0].max()
    return out.reshape(-1)


@pytest.mark.parametrize("n,lo_slices,kw", [
    ((9, 9, 5), 0, {}),
    ((9, 9, 5), 2, {}),
    ((5, 7, 3), 0, {"pc_nms": 3, "pc_top_k": 4}),
    ((9, 9, 1), 0, {"pc_gate": 0.5, "pc_top_k": 30, "pc_kde_sigma": 0.05}),
    ((3, 3, 3), 0, {"pc_inlier_radius": 0.001}),
])
def test_ballots_match_oracle(n, lo_slices, kw):
    s = _settings(**kw)
    rng = np.random.default_rng(3)
    n_pat = 25
    lo, hi = lo_slices * n[0] * n[1], n[0] * n[1] * n[2]
    step = [0.0125, 0.0125, 0.015] if n[2] > 1 else [0.0125, 0.0125, 0.0]
    sc = _scores(rng, n_pat, n, lo)
    try:
        want = opc.consensus(s, sc, n_pat, n, step, lo, hi)
    except opc.NoPcSupport:
        with pytest.raises(pcfit.PcError, match="NoPcSupport"):
            pcfit.consensus(s, sc, n_pat, n, step, lo, hi)
        return
    got = pcfit.consensus(s, sc, n_pat, n, step, lo, hi)
    assert got[0] == want[0] and got[1] == want[1] and got[3] == want[3]
    assert np.array_equal(got[2], want[2])  # the density, bit for bit


def _surface(pc_true, n_pat, ridge=0.0, scale=1.0):
    """Each fit pattern's score under candidate pattern centres: a peak at the pattern's own
    view of the true centre, a ridge (shift traded against rotation), a deterministic ripple."""
    own = np.array(pc_true)[None, :] + 0.004 * np.sin(np.arange(n_pat)[:, None] * np.array([1.3, 2.1, 0.7]))

    def score(cands):
        c = np.asarray(cands, np.float64)
        d = c[None, :, :] - own[:, None, :]
        v = np.exp(-(d ** 2).sum(-1) / (2 * (0.03 * scale) ** 2))
        v += ridge * np.exp(-((d[..., 0] - d[..., 1]) ** 2) / (2 * 0.01 ** 2))
        v += 0.01 * np.sin(900 * c[None, :, 0] + 37 * c[None, :, 1] * (1 + np.arange(n_pat)[:, None]) + 11 * c[None, :, 2])
        return (0.6 * v).astype(np.float32)

    return score


def _same(a, b):
    return all(np.array_equal(np.asarray(a[k]), np.asarray(b[k])) for k in a)


@pytest.mark.parametrize("case", ["ballots", "mean", "walk", "zmin", "flat_z", "nms"])
def test_search_matches_oracle(case):
    kw = {"pc_steps": 9, "pc_steps_z": 5, "pc_levels": 3}
    start, truth = (0.50, 0.32, 0.58), (0.515, 0.305, 0.595)
    ridge = 0.3
    if case == "mean":
        kw["pc_vote"] = "mean"
    if case == "walk":  # the truth outside the first grid: it walks before it narrows
        kw.update(pc_span=0.03, pc_span_z=0.02)
        truth = (0.56, 0.28, 0.60)
    if case == "zmin":  # the nearest slices are not scored
        kw.update(pc_z_min=0.55)
    if case == "flat_z":
        kw.update(pc_steps_z=1, pc_steps=7)
    if case == "nms":
        kw.update(pc_nms=3, pc_top_k=6)
    s = _settings(**kw)
    n_pat = 25
    score = _surface(truth, n_pat, ridge)
    want, want_h = opc.search(s, start, n_pat, score)
    got, got_h, best = pcfit.search(s, start, n_pat, score)
    assert got["pc"] == want["pc"] and best == want["best"]
    for k in ("start", "score", "start_score", "n_candidates", "at_border", "levels", "n_patterns"):
        assert got[k] == want[k], k
    assert len(got_h) == len(want_h)
    for g, w in zip(got_h, want_h):
        assert all(np.array_equal(g["axes"][a], np.array(w["axes"][a])) for a in range(3))
        assert np.array_equal(g["scores"], w["scores"]) and np.array_equal(g["pat_scores"], w["pat_scores"])
        assert list(g["pat_best"]) == w["pat_best"] and np.array_equal(g["pat_ncc"], np.float32(w["pat_ncc"]))
        assert g["best"] == w["best"] and g["walked"] == w["walked"] and list(g["peak"]) == list(w["peak"])
        assert g["ballots"] == w["ballots"] and g["inliers"] == w["inliers"]
        assert (g["density"] is None) == (w["density"] is None)
        if g["density"] is not None:
            assert np.array_equal(g["density"], w["density"])
    if case == "walk":
        assert any(h["walked"] for h in got_h) and len(got_h) > 3
    if case in ("ballots", "walk", "nms"):
        assert np.abs(np.array(got["pc"]) - truth).max() < 0.012, got["pc"]
        assert got["score"] > got["start_score"]


def test_search_refusals_match_oracle():
    score = _surface((0.5, 0.3, 0.6), 4)
    s = _settings(pc_z_min=1.0)  # every candidate nearer than the minimum
    with pytest.raises(opc.NoPcCandidates):
        opc.search(s, (0.5, 0.3, 0.6), 4, score)
    with pytest.raises(pcfit.PcError, match="NoPcCandidates"):
        pcfit.search(s, (0.5, 0.3, 0.6), 4, score)
    s = _settings(pc_steps=65, pc_steps_z=65)  # 65³ candidates × 16 patterns > 4 Mi
    with pytest.raises(pcfit.PcError, match="SearchTooLarge"):
        pcfit.search(s, (0.5, 0.3, 0.6), 16, score)
    s = _settings()
    with pytest.raises(pcfit.PcError, match="NoPcSupport"):  # nothing scores above zero
        pcfit.search(s, (0.5, 0.3, 0.6), 4, lambda c: -np.ones((4, len(c)), np.float32))


def test_vertex_and_axis_match_oracle():
    rng = np.random.default_rng(1)
    for _ in range(200):
        lo, mid, hi = rng.normal(size=3)
        assert pcfit.vertex(lo, mid, hi) == opc.vertex(lo, mid, hi)
    for c, sp, n in ((0.5, 0.1, 9), (0.3, 0.06, 5), (0.7, 0.1, 1), (0.5, 0.035, 2)):
        assert list(pcfit.axis(c, sp, n)) == opc.axis(c, sp, n)
    assert math.isclose(pcfit.axis(0.5, 0.1, 9)[4], 0.5)
