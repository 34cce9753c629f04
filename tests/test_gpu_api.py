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
