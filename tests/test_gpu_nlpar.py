"""Neighbour averaging (NLPAR) on the GPU against the oracle's whole-map restatement
(oracle/nlpar.py), as the reference checks it (tests/test_api.py:473-515): 3 passes of 3 × 3, 2 of
5 × 5 and 1 of 7 × 7 at cells inside and on every edge of the map; the averages before the filters
within 1e-5 of the patterns' spread, after them (unit-normalized) within 2e-5; each average's
shares of its neighbours within 1e-5, NaN where the window leaves the map; a pattern not averaged
has no account; the averages do not depend on how the map is cut into batches; averaging quiets
the patterns (the indexing NCC rises)."""
import tempfile

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import oracle.nlpar as onl  # noqa: E402

ROWS, COLS = 8, 14


@pytest.fixture(scope="module")
def scan():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import zebsdsolve_b200 as ze
    from zebsdsolve_b200 import synthetic as syn
    from zebsdsolve_b200.master import write_npz

    d = tempfile.mkdtemp()
    path = f"{d}/m.npz"
    write_npz(path, syn.master_sheets(4, side=201, lmax=48, group="432", device="cuda"), 201,
              syn.group_matrices("432"), 30)
    s = ze.Solver()
    s.configure(static_background="none", dynamic_background="none", bandwidth=32)
    s.add_phase(path)
    s.set_patterns(np.zeros((ROWS, COLS, 60, 60), np.float32))
    s.set_geometry(pc=(0.5, 0.3, 0.6), sample_tilt_deg=70, detector_tilt_deg=0)
    rng = np.random.default_rng(7)
    grain = np.zeros((ROWS, COLS), int)
    grain[:, 7:] = 1
    grain[:, 3] = 2
    grain[5, 9:13] = 2
    q3 = syn.uniform_quaternions(rng, 3)
    q = q3[grain.ravel()]
    clean = s.simulate(q, cells=np.arange(ROWS * COLS)).reshape(ROWS, COLS, 60, 60)
    noisy = (128 + 50 * clean / clean.std() + 300 * rng.normal(size=clean.shape)).astype(np.float32)
    s.set_patterns(noisy)
    return {"s": s, "noisy": noisy, "q": q, "thin": grain.ravel() == 2}


def _unit(a):
    out = a - a.mean()
    return out / np.sqrt((out ** 2).sum())


@pytest.mark.parametrize("radius,passes,lam", [(1, 3, 0.7), (2, 2, 0.9), (3, 1, 0.7)])
def test_averages_match_oracle(scan, radius, passes, lam):
    s, noisy = scan["s"], scan["noisy"]
    s.configure(mask=False, nlpar=True, nlpar_radius=radius, nlpar_iterations=passes, nlpar_lambda=lam)
    ref, shares = onl.average(noisy, radius, passes, lam)
    spread = float(noisy.std())
    reach = radius * passes
    for cell in (0, COLS - 1, 4 * COLS + 4, 5 * COLS + 10, 3 * COLS + 7, ROWS * COLS - 1):
        r, c = divmod(cell, COLS)
        got = s.pattern(cell, "averaged")
        assert np.abs(got - ref[r, c]).max() / spread < 1e-5, (cell, np.abs(got - ref[r, c]).max() / spread)
        v = s.nlpar_view()
        mine = shares[r, c]
        assert v["shares"].shape == mine.shape
        assert np.abs(np.nan_to_num(v["shares"]) - mine).max() < 1e-5
        assert abs(v["own"] - mine[reach, reach]) < 1e-5 and 0 < v["left"] < 1 and v["noise"] > 0
        edge = min(r, c, ROWS - 1 - r, COLS - 1 - c) < reach
        assert np.isnan(v["shares"]).any() == edge
        processed = s.pattern(cell)
        assert np.abs(processed - _unit(ref[r, c])).max() < 2e-5
        assert s.nlpar_view() is not None
    s.configure(mask=True, nlpar=False)


def test_a_pattern_not_averaged_has_no_account(scan):
    s = scan["s"]
    s.configure(nlpar=False)
    s.pattern(0)
    assert s.nlpar_view() is None
    assert np.array_equal(s.pattern(5, "averaged"), s.pattern(5, False))


def test_averaging_quiets_and_does_not_depend_on_the_batch(scan):
    s, q = scan["s"], scan["q"]
    s.configure(nlpar=False)
    r0 = s.index()
    s.configure(nlpar=True, nlpar_radius=1, nlpar_iterations=3, nlpar_lambda=0.7)
    ra = s.index()
    s._e.device_batch = lambda: 37  # ragged batches: every window built again
    rb = s.index()
    del s._e.device_batch
    apart = np.degrees(s.disorientation(ra["quaternions"].reshape(-1, 4), rb["quaternions"].reshape(-1, 4)))
    assert apart.max() < 0.02 and np.abs(ra["ncc"] - rb["ncc"]).max() < 1e-3, (apart.max(), np.abs(ra["ncc"] - rb["ncc"]).max())
    assert ra["ncc"].mean() > 1.5 * r0["ncc"].mean(), (ra["ncc"].mean(), r0["ncc"].mean())
    d0 = np.degrees(s.disorientation(r0["quaternions"].reshape(-1, 4), q))
    da = np.degrees(s.disorientation(ra["quaternions"].reshape(-1, 4), q))
    assert (da < 1).mean() >= (d0 < 1).mean()
    s.configure(nlpar=False)
