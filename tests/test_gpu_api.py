"""The public API's run paths on the GPU: Solver.index (pipelined device passes: uploads on a copy
stream, readbacks landed while the next pass runs) against the reference's step loop
(index_begin / index_step, engine.zig:2426-2465), progress-driven stopping, and sweeps."""
import tempfile

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scan():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from zebsdsolve_b200 import synthetic as syn
    from zebsdsolve_b200.master import write_npz

    sheets = syn.master_sheets(3, side=201, lmax=48, group="432", device="cuda")
    d = tempfile.mkdtemp()
    write_npz(f"{d}/m.npz", sheets, 201, syn.group_matrices("432"), 30)
    return {"path": f"{d}/m.npz"}


def _solver(scan, rows=8, cols=12, **kw):
    import zebsdsolve_b200 as ze
    from zebsdsolve_b200 import synthetic as syn

    s = ze.Solver()
    s.configure(bandwidth=32, **kw)
    s.add_phase(scan["path"])
    s.set_patterns(np.zeros((rows, cols, 60, 60), np.uint16))
    s.set_geometry(pc=(0.5, 0.3, 0.6), sample_tilt_deg=70, detector_tilt_deg=0)
    rng = np.random.default_rng(21)
    q, _ = syn.grain_map(rng, rows, cols, 6, 0.5)
    sims = s.simulate(q, cells=np.arange(rows * cols))
    pats = syn.counted_patterns(torch.as_tensor(sims, device="cuda"), seed=5).cpu().numpy()
    s.set_patterns(pats.reshape(rows, cols, 60, 60))
    return s, q


def test_pipelined_index_equals_the_step_loop(scan):
    s, q = _solver(scan)
    s._e.device_batch = lambda: 40  # three passes, the last one ragged
    r = s.index()
    s2, _ = _solver(scan)
    s2.index_begin()
    while s2.index_step() > 0:
        pass
    r2 = s2.results()
    for k in ("quaternions", "ncc", "nmi", "phase", "z", "sweep"):
        assert np.array_equal(r[k], r2[k]), k
    dis = np.degrees(s.disorientation(r["quaternions"].reshape(-1, 4), q))
    assert np.median(dis) < 0.5


def test_refinement_after_an_indexing_run_starts_from_the_kept_patterns(scan):
    """A whole indexing run keeps its filtered patterns on the device (Engine.keep_prepared); a
    following refine_patterns starts from them without uploading and filtering again, with the
    results of a solver that has no kept patterns, bit for bit; a settings change or a new scan
    drops them."""
    s, q = _solver(scan)
    e = s._e
    e.device_batch = lambda: 40  # three passes, the last one ragged
    cells = np.arange(96)
    fresh, _ = _solver(scan)
    want = fresh.refine_patterns(cells, quaternions=q, gradient="adjoint", rounds=4)
    assert fresh._e._resident is None
    s.index()
    assert e._resident is not None and e._resident["valid"].all()
    got = s.refine_patterns(cells, quaternions=q, gradient="adjoint", rounds=4)
    for k in ("quaternions", "shift", "ncc"):
        assert np.array_equal(got[k], want[k]), k
    # the kept rows are the filtered patterns: a run of cells as a view, scattered cells gathered
    for c in (np.arange(10, 50), np.array([90, 3, 41, 7])):
        kept = e.prepared(c).clone()
        e._resident["key"] = None
        assert torch.equal(kept, e.upload(c)[: kept.numel()])
        e._resident["key"] = e._prep_key()
    s.configure(dynamic_sigma=0.2)
    assert e._resident["key"] != e._prep_key()  # (prepared uploads and filters again)
    s.set_patterns(e.patterns.copy())
    assert e._resident["key"] is None


def test_progress_returning_false_stops_after_a_pass(scan):
    s, _ = _solver(scan)
    s._e.device_batch = lambda: 40
    seen = []

    def progress(st):
        seen.append(st["done"])
        return False

    r = s.index(progress)
    # one call, after the first pass (a short one: its upload is not hidden behind kernels)
    assert len(seen) == 1 and 0 < seen[0] <= 40, seen
    # the pass in flight when the stop came (the next 40) lands too; nothing after it runs
    k = seen[0] + 40
    ph = r["phase"].reshape(-1)
    assert (ph[:k] >= 0).all() and (ph[k:] == -1).all()


def test_two_sweeps_run_to_the_end(scan):
    s, q = _solver(scan, sweeps=2, sweep_bandwidth=16, accept_z=1e9)  # nothing accepted: all go on
    r = s.index()
    st = s.index_status
    assert st["sweep"] == 1 and st["done"] == st["total"] == 96
    assert (r["phase"] >= 0).all()


def test_tune_changes_no_result(scan):
    """tune() times the pipelined path on a sample and keeps the fastest way of cutting up the
    work; the results after it are the results before it, bit for bit."""
    s, q = _solver(scan)
    r1 = s.index()
    seen = []
    out = s.tune(lambda k: seen.append(k))
    assert set(out) == {"before", "after", "summary"} and out["summary"].startswith("tuned on")
    assert seen == list(range(1, len(seen) + 1)) and len(seen) >= 3
    assert 2048 <= out["after"]["device_batch"] <= 65536 and 512 <= out["after"]["tile_mb"] <= 8192
    r2 = s.index()
    for k in ("quaternions", "ncc", "nmi", "phase", "z", "sweep"):
        assert np.array_equal(r1[k], r2[k]), k


def test_a_scan_stepped_through_once_is_not_page_locked_whole(scan):
    """index_step calls index_cells once per ~4096 cells; the scan then counts as indexed once, so
    its uploads stream through the two staging slots and the whole scan is never page-locked.
    A second pass over it (here a Solver.index after the step loop) is what page-locks it."""
    s, _ = _solver(scan)
    e = s._e
    calls = []
    real = e.pinned
    e.pinned = lambda: calls.append(1) or real()
    s.configure(batch=4)  # two steps over the 96 cells: 4 × 16 cells, then the 32 left
    s.index_begin()
    steps = 0
    while s.index_step() > 0:
        steps += 1
    assert steps >= 1 and not calls and e._pinned is None
    s.index()
    assert calls and e._pinned is not None


def test_cell_under_another_centre_leaves_the_geometry(scan):
    """cell_under (__init__.py:198-212): one cell indexed and simulated under another pattern
    centre; the geometry in use is untouched, and under the geometry in use it is index_cells."""
    s, q = _solver(scan)
    before = s.geometry
    u = s.cell_under(7, pc=(0.51, 0.31, 0.61))
    assert s.geometry == before
    assert set(u) == {"phase", "quaternion", "ncc", "nmi", "simulation"}
    assert u["simulation"].shape == (60, 60) and u["phase"] == 0
    same = s.cell_under(7)
    ref = s.index_cells([7], bandwidth=s.settings["fit_bandwidth"])
    assert np.array_equal(same["quaternion"], ref["quaternions"][0, 0])
    assert np.allclose(same["simulation"], s.simulate(same["quaternion"][None], cells=[7])[0])
    # the same cell under the other centre scores differently (its own projection)
    assert abs(u["ncc"] - same["ncc"]) > 1e-6


def test_pattern_stats_profile_and_counts(scan):
    s, _ = _solver(scan)
    mean, std = s.pattern_stats()
    pats = s._e.patterns.reshape(96, -1).astype(np.float64)
    assert mean.shape == (8, 12)
    assert np.allclose(mean.reshape(-1), pats.mean(1), rtol=1e-6) and np.allclose(std.reshape(-1), pats.std(1), rtol=1e-5)
    m2, s2 = s.pattern_stats([3, 50])
    assert np.allclose(m2, mean.reshape(-1)[[3, 50]])
    s.gpu_counts()
    assert s.profile(True) is True
    s.index()
    rep = s.profile_report()
    s.profile(False)
    names = [ln.split()[0] for ln in rep.splitlines()[1:-1]]
    assert "zeb_refine_list" in names and "zeb_sphere_coefficients_spans" in names, rep
    c = s.gpu_counts()
    assert c["dispatches"] > 0 and c["submits"] >= 1 and c["reads"] >= 2 and c["waits"] >= 1, c
    assert s.gpu_counts()["dispatches"] == 0  # since the last call
    # the plain function reads a scan file's patterns (here the test data's h5ebsd, when present)
    from conftest import testdata
    import zebsdsolve_b200 as ze

    path = testdata("nickel", "patterns_v2.h5")
    if path is not None:
        p3 = ze.load_patterns(str(path), cells=[0, 1, 2])
        assert p3.shape == (3, 60, 60) and p3.dtype == np.float32


def test_binned_search_refined_or_scored_at_the_stored_size(scan):
    """settings.full_resolution (engine.zig:996-1003, 2101-2119): the search on patterns binned 2×,
    then the refinement ("refine") or only the scores ("scores") at the stored size: scores change
    (they are the stored size's), orientations are those of the binned run when only the scores
    move, and a refinement at the stored size is at least as good as the binned one."""
    s, q = _solver(scan)
    s.configure(binning=2)
    assert s.pattern_shape == (30, 30) and s.shape(full=True) == (60, 60)
    assert s.pattern(5).shape == (30, 30) and s.pattern(5, full=True).shape == (60, 60)
    full = s.pattern(5, full=True)
    assert abs(float(full.sum())) < 1e-3 and abs(float((full ** 2).sum()) - 1) < 1e-3  # filtered at 60 × 60
    rb = {}
    for mode in ("none", "scores", "refine"):
        s.configure(full_resolution=mode)
        rb[mode] = s.index()
        rb[mode]["dis"] = np.degrees(s.disorientation(rb[mode]["quaternions"].reshape(-1, 4), q))
    assert np.allclose(rb["scores"]["dis"], rb["none"]["dis"], atol=0.05)
    assert abs(float(rb["scores"]["ncc"].mean() - rb["none"]["ncc"].mean())) > 1e-3
    assert rb["refine"]["ncc"].mean() > rb["scores"]["ncc"].mean() - 1e-3
    assert np.median(rb["refine"]["dis"]) <= np.median(rb["none"]["dis"]) + 0.02
    assert (rb["refine"]["phase"] == 0).all()
    # refined at the stored size, the binned search's peaks settle where the unbinned run's do
    s.configure(binning=1, full_resolution="none")
    r1 = s.index()
    apart = np.degrees(s.disorientation(rb["refine"]["quaternions"].reshape(-1, 4), r1["quaternions"].reshape(-1, 4)))
    assert np.median(apart) < 0.02 and (apart < 0.1).mean() > 0.95, np.sort(apart)[-4:]
    assert abs(float(rb["refine"]["ncc"].mean() - r1["ncc"].mean())) < 2e-3


def test_static_background_summed_on_the_device_equals_the_host_sum(scan):
    """The average of the lattice's stored patterns (engine.zig:1344-1424), summed on the device for
    integer pixels: the same float32 image as the host's float64 sum, bit for bit (the sum of
    integers is exact in any order)."""
    import zebsdsolve_b200 as ze
    from zebsdsolve_b200.reduce import reduce_image

    rng = np.random.default_rng(4)
    for dt, top in ((np.uint16, 60000), (np.uint8, 250)):
        pats = rng.integers(0, top, (23, 31, 40, 44)).astype(dt)
        s = ze.Solver()
        s.configure(static_background="average", static_patterns=500)
        s.add_phase(scan["path"])
        s.set_patterns(pats)
        e = s._e
        got = e.static_background().cpu().numpy()
        cells = e.lattice(500)
        acc = pats.reshape(-1, 40, 44)[cells].sum(0, dtype=np.float64)
        want = reduce_image(acc / len(cells), e.factor()).astype(np.float32)
        assert np.array_equal(got, want), dt
