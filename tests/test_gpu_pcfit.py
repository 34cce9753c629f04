"""The pattern-centre vote on the GPU: every (fit pattern, candidate) score against the FP64
oracle (the candidate's own window denominators, the largest normalized correlation), tiles of
whole candidates against candidates in parts (the same bits), two phases competing on NMI, and
the whole search on a synthetic scan simulated at a known pattern centre (the reference's
tests/test_api.py:298-372 checks: found within 0.012, the score rises, ballots and density, every
grid kept, the mean vote, a refused search changing nothing)."""
import math
import tempfile

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import oracle.master as om  # noqa: E402
import oracle.pcfit as opc  # noqa: E402
import oracle.spherical as osp  # noqa: E402
import oracle.sym as osym  # noqa: E402

TRUTH = (0.5, 0.3, 0.6)


@pytest.fixture(scope="module")
def small():
    """A 151² master (432, SH ≤ 28) and six noisy patterns on a 1 × 6 map, beam travel on."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import zebsdsolve_b200 as ze
    from zebsdsolve_b200 import synthetic as syn
    from zebsdsolve_b200.master import write_npz

    d = tempfile.mkdtemp()
    paths = []
    for g, seed, side, lmax in (("432", 11, 151, 28), ("622", 12, 151, 28)):
        write_npz(f"{d}/m{g}.npz", syn.master_sheets(seed, side=side, lmax=lmax, group=g), side,
                  syn.group_matrices(g), syn.POINT_GROUP[g])
        paths.append(f"{d}/m{g}.npz")
    s = ze.Solver()
    s.configure(static_background="none", dynamic_background="none", fit_bandwidth=16, fit_grid=2)
    s.add_phase(paths[0])
    n = 6
    s.set_patterns(np.zeros((1, n, 60, 60), np.float32))
    s.set_geometry(pc=TRUTH, sample_tilt_deg=70, detector_tilt_deg=0, px_um=60.0, step_x_um=25.0, step_y_um=25.0)
    rng = np.random.default_rng(5)
    q = syn.uniform_quaternions(rng, n)
    sims = s.simulate(q, cells=np.arange(n))
    pats = sims + 0.3 * sims.std() * rng.normal(size=sims.shape)
    s.set_patterns(pats.astype(np.float32).reshape(1, n, 60, 60))
    return {"s": s, "q": q, "paths": paths}


CANDS = np.array([TRUTH, (0.52, 0.28, 0.62), (0.47, 0.33, 0.57)])


def test_candidate_scores_match_oracle(small):
    from zebsdsolve_b200 import pcfit

    s = small["s"]
    e = s._e
    cells = pcfit.fit_cells(e.region_cells(), 6, 2)
    assert list(cells) == [1, 4]
    sc = pcfit.Scorer(e, cells)
    got = sc(CANDS)  # [pattern][candidate]
    pk = sc.last[0][0]  # [candidate][pattern][8]
    assert got.shape == (2, 3) and np.array_equal(got, pk[..., 4].T)
    L = 16
    tb = osp.Tables(L)
    baked = s.master(0).reshape(-1)
    from zebsdsolve_b200 import synthetic as syn

    m_or = om.Master(151, baked, syn.group_matrices("432"), 30)
    m_or.measure_symmetry()
    hm = om.Harmonics(m_or, baked, L)
    pt = osp.PhaseTables(tb, hm, om.fold_of(hm.rules))
    fr = e.frame()
    frame = (np.array(fr.c0), np.array(fr.c1), np.array(fr.c2))
    pats = sc.pats.cpu().numpy().reshape(len(cells), 60, 60).astype(np.float64)
    ops = m_or.rotations()
    for j, c in enumerate(CANDS):
        t = e.geo.translation(60, 60, pc=c)
        for b in range(len(cells)):
            q, v0, _, _ = opc.candidate_score(tb, pt, hm, pats[b], t, sc.offs[b], frame, np.array(fr.mask), (60, 60))
            assert abs(pk[j, b, 4] - v0) < 2e-4, (j, b, pk[j, b, 4], v0)
            dis = math.degrees(float(osym.disorientation(pk[j, b, :4].astype(np.float64), q, ops)))
            assert dis < 0.05, dis
    # the beam travels: the two patterns sit at different positions under one candidate
    assert np.abs(sc.offs[0] - sc.offs[1]).max() > 0.5


def test_candidates_in_parts_give_the_same_bits(small):
    from zebsdsolve_b200 import pcfit

    e = small["s"]._e
    cells = pcfit.fit_cells(e.region_cells(), 6, 2)
    whole = pcfit.Scorer(e, cells)
    a = whole(CANDS)
    pa = whole.last[0].copy()
    for tile, per in ((1, 1), (4, 2)):  # one item at a time (parts of a candidate); two candidates per tile
        sc = pcfit.Scorer(e, cells)
        sc.tile, sc.cand_per_tile = tile, per
        b = sc(CANDS)
        assert np.array_equal(a, b) and np.array_equal(pa, sc.last[0]), (tile, per)


def test_two_phases_compete_on_nmi(small):
    import zebsdsolve_b200 as ze
    from zebsdsolve_b200 import pcfit

    s0 = small["s"]
    s = ze.Solver()
    s.configure(static_background="none", dynamic_background="none", fit_bandwidth=16, fit_grid=3)
    for p in small["paths"]:
        s.add_phase(p)
    s.set_patterns(s0._e.patterns)
    s.set_geometry(**{k: v for k, v in s0.geometry.items() if k not in ("plane_kind", "plane")})
    e = s._e
    cells = pcfit.fit_cells(e.region_cells(), 6, 3)
    sc = pcfit.Scorer(e, cells)
    got = sc(CANDS)
    pk, choice = sc.last
    assert pk.shape[0] == 2
    # each score is the peak of the phase the records chose; the 432 patterns pick the 432 master
    assert np.array_equal(got.T, np.take_along_axis(pk[..., 4], choice[None], 0)[0])
    assert (choice[0] == 0).all(), choice
    # phase 0's peaks do not depend on phase 1 being there
    one = pcfit.Scorer(small["s"]._e, cells)
    one(CANDS)
    assert np.array_equal(one.last[0][0], pk[0])


@pytest.fixture(scope="module")
def scan():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import zebsdsolve_b200 as ze
    from zebsdsolve_b200 import synthetic as syn
    from zebsdsolve_b200.master import write_npz

    d = tempfile.mkdtemp()
    path = f"{d}/m.npz"
    write_npz(path, syn.master_sheets(3, side=401, lmax=96, group="432", device="cuda"), 401,
              syn.group_matrices("432"), 30)
    s = ze.Solver()
    s.configure(bandwidth=32)  # the vote at its own default bandwidth, 64
    s.add_phase(path)
    rows, cols = 8, 12
    s.set_patterns(np.zeros((rows, cols, 60, 60), np.uint16))
    s.set_geometry(pc=TRUTH, sample_tilt_deg=70, detector_tilt_deg=0)
    rng = np.random.default_rng(21)
    q, _ = syn.grain_map(rng, rows, cols, 6, 0.5)
    sims = s.simulate(q, cells=np.arange(rows * cols))
    pats = syn.counted_patterns(torch.as_tensor(sims, device="cuda"), seed=5).cpu().numpy()
    s.set_patterns(pats.reshape(rows, cols, 60, 60))
    return {"s": s, "q": q, "path": path, "pats": pats.reshape(rows, cols, 60, 60)}


START = (0.515, 0.32, 0.58)


def test_the_vote_finds_the_centre(scan):
    import zebsdsolve_b200 as ze

    s = scan["s"]
    s.set_geometry(pc=START)
    f = s.fit_pc()
    err = np.abs(np.array(f["pc"]) - TRUTH)
    assert err.max() < 0.012 and f["score"] > f["start_score"], (f, err)
    assert f["n_patterns"] == 25 and f["start"] == list(START) and np.allclose(s.geometry["pc"], f["pc"])
    scores, x, y, z = s.pc_scores()
    assert scores.shape == (len(z), len(y), len(x)) and np.isfinite(scores).all()
    levels = s.pc_levels()
    last = levels[-1]
    ix, iy, iz = (int(round(v)) for v in last["peak"])
    # each pattern's ballots: its best candidates down to 0.85 × its best, at most 12
    ps = last["pattern_scores"].reshape(25, -1).astype(np.float64)
    cast = sum(min(12, int(((p >= 0.85 * p.max()) & (p > 0)).sum())) for p in ps)
    assert last["density"].shape == last["scores"].shape and last["ballots"] == cast
    assert 0 < last["inliers"] <= last["ballots"]
    assert np.allclose(last["pattern_scores"].mean(0), last["scores"], atol=1e-5)
    dz, dy, dx = np.unravel_index(int(np.argmax(last["density"])), last["density"].shape)
    assert max(abs(dx - ix), abs(dy - iy), abs(dz - iz)) <= 2
    assert len(levels) >= 3 and np.array_equal(last["scores"], scores) and last["winner"] == (ix, iy, iz)
    assert last["pattern_best"].shape == (25, 3) and np.isfinite(last["pattern_ncc"]).all()
    assert np.ptp(levels[0]["x"]) > np.ptp(last["x"])
    # the fit patterns' poses at the winner are their true orientations
    cells, phs, quats, ncc = s.fit_patterns()
    assert len(cells) == 25 and (phs == 0).all()
    dis = np.degrees(s.disorientation(quats, scan["q"][cells.astype(int)]))
    assert np.median(dis) < 1.0, np.median(dis)

    # the mean of the patterns' scores, the rule the ballots replace
    s.set_geometry(pc=START)
    s.configure(pc_vote="mean")
    fm = s.fit_pc()
    lm = s.pc_levels()[-1]
    assert lm["density"] is None
    assert lm["winner"] == tuple(int(v) for v in np.unravel_index(int(np.argmax(lm["scores"])), lm["scores"].shape)[::-1])
    assert np.abs(np.array(fm["pc"]) - TRUTH).max() < 0.02
    s.configure(pc_vote="ballots")

    # a grid entirely nearer than pc_z_min is refused and changes nothing
    before = (s.geometry, s.pc_scores(), s.pc_levels(), s.fit_patterns())
    for vote in ("mean", "ballots"):
        s.configure(pc_vote=vote, pc_z_min=1)
        with pytest.raises(ze.Error, match="NoPcCandidates"):
            s.fit_pc()
    s.configure(pc_vote="ballots", pc_z_min=0.1)
    assert s.geometry == before[0]
    assert all(np.array_equal(a, b) for a, b in zip(s.pc_scores(), before[1]))
    assert len(s.pc_levels()) == len(before[2])
    for lv, pv in zip(s.pc_levels(), before[2]):
        assert all(np.array_equal(lv[k], pv[k]) for k in ("pattern_scores", "pattern_best", "pattern_ncc"))
    assert all(np.array_equal(a, b) for a, b in zip(s.fit_patterns(), before[3]))


def test_index_with_the_vote_first(scan):
    import zebsdsolve_b200 as ze

    r = ze.index(scan["pats"], [scan["path"]], fit="pc", pc=START, sample_tilt_deg=70, detector_tilt_deg=0,
                 bandwidth=32)
    assert np.abs(np.array(r.geometry["pc"]) - TRUTH).max() < 0.012
    assert r.fit["pc"]["pc"] == r.geometry["pc"]
    f = ze.fit_pattern_center(scan["pats"], [scan["path"]], pc=START, sample_tilt_deg=70, detector_tilt_deg=0)
    assert np.abs(np.array(f["pc"]) - TRUTH).max() < 0.012 and f["scores"].ndim == 3 and len(f["axes"]) == 3
    with pytest.raises(ValueError):
        ze.index(scan["pats"], [scan["path"]], fit="plane")
