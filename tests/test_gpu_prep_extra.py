"""CLAHE, the band pass and the master's point-group mean on the GPU against the oracle
(oracle/prep.py clahe / run, oracle/detector.py symmetrize): the reference's own CLAHE check
(tests/test_api.py:698-706: three grids, unit-normalized patterns within 2e-4, the mask last),
the band pass with both blurs (direct and box-sum), and a scan indexed with both filters on the
patterns and the master (tests/test_api.py:870-874)."""
import ctypes
import tempfile

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import oracle.detector as od  # noqa: E402
import oracle.prep as op  # noqa: E402


@pytest.fixture(scope="module")
def lib():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from zebsdsolve_b200 import _native

    return _native


def P(t):
    return ctypes.c_void_p(t.data_ptr())


def sp():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _raw(seed, n, h, w):
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:h, 0:w]
    base = 800 + 300 * np.exp(-((yy - 0.4 * h) ** 2 + (xx - 0.6 * w) ** 2) / (0.3 * h * w))
    return (base[None] + 120 * rng.normal(size=(n, h, w))).clip(0, 65535).astype(np.uint16)


def _engine_pats(raw, **settings):
    import zebsdsolve_b200 as ze

    s = ze.Solver()
    s.configure(static_background="none", **settings)
    s.set_patterns(raw[None])
    n, h, w = raw.shape
    e = s._e
    return e.upload(np.arange(n))[: n * h * w].cpu().numpy().reshape(n, h, w), s


def _unit(a, inside=None):
    """Zero mean and unit norm (under a mask), as the engine leaves filtered patterns."""
    m = np.ones(a.shape, bool) if inside is None else inside
    out = np.where(m, a - a[m].mean(), 0).astype(np.float64)
    return out / np.sqrt((out ** 2).sum())


@pytest.mark.parametrize("grid,bins,clip", [(4, 64, 40.0), (7, 32, 2.0), (8, 128, 40.0), (3, 2, 1.0), (1, 256, 40.0)])
@pytest.mark.parametrize("mask", [False, True])
def test_clahe_matches_oracle(lib, grid, bins, clip, mask):
    """zeb_clahe on the engine's own image before CLAHE (static and dynamic backgrounds, not yet
    normalized) equals the oracle's CLAHE of that image bit for bit (float32 throughout, each
    operation rounded as the kernels round); the engine's whole chain is that, normalized under the
    mask (the reference's grids of tests/test_api.py:698-706 and two edge cases)."""
    raw = _raw(grid * bins, 3, 60, 60)
    got, s = _engine_pats(raw, clahe=True, clahe_grid=grid, clahe_bins=bins, clahe_clip=clip, mask=mask,
                          dynamic_background="subtract", dynamic_sigma=0.15)
    n, h, w = raw.shape
    pre = torch.empty(n * h * w, device="cuda")
    m3 = (ctypes.c_float * 3)(*s._e.mask_of(h, w))
    lib.call("zeb_prep_reduced", P(torch.as_tensor(raw, device="cuda")), 1, n, h, w, 1.0, None, 1, 0.15 * 60, m3, 0,
             P(pre), None, sp())
    pre_h = pre.cpu().numpy().reshape(n, h, w)
    scr = torch.empty(lib.load().zeb_clahe_scratch_bytes(n, grid, bins) // 4 + 1, device="cuda")
    lib.call("zeb_clahe", P(pre), n, h, w, grid, bins, clip, P(scr), sp())
    dev = pre.cpu().numpy().reshape(n, h, w)
    inside = op.masked(h, w, s._e.mask_of(h, w))
    for i in range(n):
        ref = op.clahe(pre_h[i], grid, bins, clip)
        assert np.array_equal(dev[i], ref), np.abs(dev[i] - ref).max()
        assert np.abs(got[i] - op.normalize(ref, s._e.mask_of(h, w))).max() < 1e-6
        if mask:
            assert (got[i][~inside] == 0).all()


@pytest.mark.parametrize("fine,coarse,size", [(1.0, 8.0, 60), (0.0, 8.0, 60), (2.0, 15.0, 80)])
def test_bandpass_matches_oracle(lib, fine, coarse, size):
    raw = _raw(int(coarse), 3, size, size)
    got, s = _engine_pats(raw, bandpass=True, bp_fine=fine, bp_coarse=coarse, dynamic_background="none")
    m = s._e.mask_of(size, size)
    for i in range(3):
        ref = op.run(raw[i], dynamic="none", mask=m, bandpass=(fine, coarse))
        assert np.abs(got[i] - ref).max() < 2e-5, np.abs(got[i] - ref).max()


def test_clahe_then_bandpass_matches_oracle(lib):
    raw = _raw(5, 2, 60, 60)
    got, s = _engine_pats(raw, clahe=True, bandpass=True, dynamic_background="subtract")
    m = s._e.mask_of(60, 60)
    for i in range(2):
        ref = op.run(raw[i], dynamic="subtract", dynamic_sigma=0.15 * 60, mask=m, clahe_opts=(4, 64, 40.0),
                     bandpass=(1.0, 8.0))
        assert np.abs(got[i] - ref).max() < 3e-4, np.abs(got[i] - ref).max()


def test_master_symmetrize_matches_oracle(lib):
    from zebsdsolve_b200 import synthetic as syn

    side = 101
    # a master with no symmetry of its own, continuous over the sphere (the two sheets agree on the
    # equator, as every master's do)
    sheets = syn.master_sheets(5, side=side, lmax=20, group="1").reshape(-1)
    ops = syn.group_matrices("432")
    src = torch.as_tensor(sheets, device="cuda")
    dst = torch.empty_like(src)
    o = torch.as_tensor(np.asarray(ops, np.float32).reshape(-1), device="cuda")
    lib.call("zeb_master_symmetrize", P(src), P(dst), side, P(o), len(ops), sp())
    got = dst.cpu().numpy()
    ref = od.symmetrize(sheets.astype(np.float64), side, ops)
    assert np.abs(got - ref).max() < 1e-5, np.abs(got - ref).max()


def test_a_scan_indexes_with_both_filters_on_patterns_and_master(lib):
    """CLAHE and the band pass act on the master too: the scan still indexes to its orientations."""
    import zebsdsolve_b200 as ze
    from zebsdsolve_b200 import synthetic as syn
    from zebsdsolve_b200.master import write_npz

    d = tempfile.mkdtemp()
    write_npz(f"{d}/m.npz", syn.master_sheets(3, side=201, lmax=48, group="432", device="cuda"), 201,
              syn.group_matrices("432"), 30)
    s = ze.Solver()
    s.configure(bandwidth=32)
    s.add_phase(f"{d}/m.npz")
    rows, cols = 6, 8
    s.set_patterns(np.zeros((rows, cols, 60, 60), np.uint16))
    s.set_geometry(pc=(0.5, 0.3, 0.6), sample_tilt_deg=70, detector_tilt_deg=0)
    rng = np.random.default_rng(4)
    q, _ = syn.grain_map(rng, rows, cols, 5, 0.5)
    sims = s.simulate(q, cells=np.arange(rows * cols))
    pats = syn.counted_patterns(torch.as_tensor(sims, device="cuda"), seed=3).cpu().numpy()
    s.set_patterns(pats.reshape(rows, cols, 60, 60))
    r0 = s.index()
    s.configure(clahe=True, bandpass=True)
    key = s._e.bake_key(s._e.phases[0])
    r = s.index()
    assert s._e.phases[0].baked[0] == key and key[2] and key[5] and key[6] >= 1
    dis = np.degrees(s.disorientation(r["quaternions"].reshape(-1, 4), q))
    assert np.median(dis) < 1.0 and (dis < 3).mean() > 0.95, np.median(dis)
    assert (r["phase"] == 0).all()
    s.configure(clahe=False, bandpass=False)
    r1 = s.index()
    assert np.array_equal(r1["quaternions"], r0["quaternions"])  # the plain master is back as it was
