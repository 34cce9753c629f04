"""The plane of source points on the GPU: the plane fit's 43 sums with the master taken bilinear,
bicubic (Catmull–Rom) and by Keys' six-point kernel (zeb_sums6_list) against the FP64 oracle's
restatement of detector.wgsl `sums` / grad_at_cubic / grad_at_keys6; cells indexed where a plane
puts their sources; and the whole fit on a synthetic map whose patterns were simulated with the
beam travelling over the sample (the reference's tests/test_api.py:320-372 checks: the plane fit
refines the centre, the orientations are the true ones where the plane puts the sources, a failed
fit changes nothing)."""
import ctypes
import math
import tempfile

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import oracle.detector as od  # noqa: E402
import oracle.geometry as og  # noqa: E402
import oracle.prep as op  # noqa: E402
import oracle.rot as orot  # noqa: E402


@pytest.fixture(scope="module")
def small():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import zebsdsolve_b200 as ze
    from zebsdsolve_b200 import synthetic as syn
    from zebsdsolve_b200.master import write_npz

    side = 201
    d = tempfile.mkdtemp()
    write_npz(f"{d}/m.npz", syn.master_sheets(7, side=side, lmax=40, group="432"), side, syn.group_matrices("432"), 30)
    s = ze.Solver()
    s.configure(static_background="none", dynamic_background="none", master_smooth=0.0)
    s.add_phase(f"{d}/m.npz")
    h = w = 60
    n = 5
    rng = np.random.default_rng(41)
    s.set_patterns(np.zeros((1, n, h, w), np.float32))
    s.set_geometry(pc=(0.5, 0.3, 0.6), sample_tilt_deg=70, detector_tilt_deg=0, step_x_um=0, step_y_um=0)  # one source
    e = s._e
    e.prepare_masters()
    baked = e.phases[0].baked[1].cpu().numpy().astype(np.float64)
    geo = og.Geometry(pc=(0.5, 0.3, 0.6), sample_tilt_deg=70.0)
    q = syn.uniform_quaternions(rng, n)
    pats = np.stack([od.project(baked, side, geo.frame(), geo.translation(h, w), q[i], h, w) for i in range(n)])
    pats = pats + 0.2 * pats.std() * rng.normal(size=pats.shape)
    s.set_patterns(pats.astype(np.float32).reshape(1, n, h, w))
    return {"s": s, "e": e, "side": side, "baked": baked, "grad": od.gradient_table(baked, side), "geo": geo,
            "pats": pats, "q": q, "h": h, "w": w, "n": n, "rng": rng}


@pytest.mark.parametrize("interp", [0, 1, 2])
def test_plane_sums_match_oracle(small, interp):
    from zebsdsolve_b200 import _native as N

    st = small
    e, n, h, w = st["e"], st["n"], st["h"], st["w"]
    cells = np.arange(n)
    pats = e.upload(cells)[: n * h * w].clone()
    items = torch.as_tensor(np.concatenate([e.positions(cells), np.arange(n, dtype=np.float32)[:, None]], 1),
                            device="cuda")
    fr = e.frame()
    npix = N.load().zeb_mask_pixels(ctypes.byref(fr))
    lst = torch.empty(npix, dtype=torch.int32, device="cuda")
    N.call("zeb_mask_list", ctypes.byref(fr), ctypes.c_void_p(lst.data_ptr()), None)
    rng = np.random.default_rng(interp)
    x = np.concatenate([rng.uniform(-1, 1, (n, 3)), np.zeros((n, 3))], 1).astype(np.float32)
    ax = rng.normal(size=(n, 3))
    q = np.stack([orot.qstd(orot.qmul(orot.so3_exp(0.02 * ax[i]), st["q"][i])) for i in range(n)]).astype(np.float32)
    _, sheets, _, _, gpair = e.phases[0].baked
    out = torch.empty(n * 43, device="cuda")
    xd, qd = torch.as_tensor(x, device="cuda"), torch.as_tensor(q, device="cuda")
    P = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    N.call("zeb_sums6_list", P(pats), P(items), n, ctypes.byref(fr), P(lst), npix, P(sheets), P(gpair), st["side"],
           interp, P(xd), P(qd), P(out), None)
    got = out.cpu().numpy().reshape(n, 43)
    t0 = st["geo"].translation(h, w)
    mask = og.mask_of(h, w)
    for i in range(n):
        pat = op.normalize(st["pats"][i].astype(np.float64), mask)
        ref = od.sums6(st["grad"], st["side"], st["geo"].frame(), t0, q[i].astype(np.float64), x[i, :3].astype(np.float64),
                       pat, mask, interp=interp, sheets=st["baked"])
        scale = np.maximum(np.abs(ref), 1.0)
        assert np.all(np.abs(got[i] - ref) < 2e-4 * scale + 1e-3 * np.abs(ref).max()), (interp, np.abs(got[i] - ref).max())
        a, b = od.local_of(ref), od.local_of(got[i].astype(np.float64))
        assert abs(a[0] - b[0]) < 1e-5
        assert np.abs(a[1] - b[1]).max() < 2e-3 * max(1.0, np.abs(a[1]).max())
    if interp:
        # the smooth surface's gradient is its own: NCC by the oracle at ± a step along each rotation
        i = 0
        pat = op.normalize(st["pats"][i].astype(np.float64), mask)
        for k in range(3):
            dq = np.zeros(3)
            dq[k] = 1e-4

            def f(sign):
                qq = orot.qmul(orot.so3_exp(sign * dq), q[i].astype(np.float64))
                s6 = od.sums6(st["grad"], st["side"], st["geo"].frame(), t0, qq, x[i, :3].astype(np.float64), pat,
                              mask, interp=interp, sheets=st["baked"])
                return od.local_of(s6)[0]

            fd = (f(1) - f(-1)) / 2e-4
            g = od.local_of(got[i].astype(np.float64))[1]
            assert abs(g[3 + k] - fd) < 2e-2 * max(1.0, np.abs(g[3:]).max()), (k, g[3 + k], fd)


@pytest.mark.parametrize("interp", [0, 1])
def test_fit_settle_matches_oracle(small, interp):
    """The plane fit's per-pattern Levenberg–Marquardt over six unknowns (Fit.settle: the device's
    sums, the host's damped steps for all patterns at once) against the oracle's settle of each
    pattern by itself, from orientations 1° off: NCC 2e-4, orientation 0.02°, shift 0.05 px."""
    from zebsdsolve_b200 import _native as N
    from zebsdsolve_b200 import planefit
    from zebsdsolve_b200 import rotations as R

    st = small
    e, n, h, w = st["e"], st["n"], st["h"], st["w"]
    cells = np.arange(n)
    rng = np.random.default_rng(9)
    ax = rng.normal(size=(n, 3))
    ax /= np.linalg.norm(ax, axis=1, keepdims=True)
    q0 = np.stack([orot.qstd(orot.qmul(orot.so3_exp(math.radians(1.0) * ax[i]), st["q"][i])) for i in range(n)])
    f = planefit.Fit.__new__(planefit.Fit)
    f.e, f.n, f.cells = e, n, cells
    f.use, f.n_used, f.phase = np.ones(n, bool), n, np.zeros(n, np.int32)
    f.q, f.shift, f.base = q0.copy(), np.zeros((n, 3)), e.positions64(cells)
    f.fr = e.frame()
    f.pats = e.upload(cells)[: n * h * w].clone()
    npix = N.load().zeb_mask_pixels(ctypes.byref(f.fr))
    f.list = torch.empty(npix, dtype=torch.int32, device="cuda")
    N.call("zeb_mask_list", ctypes.byref(f.fr), ctypes.c_void_p(f.list.data_ptr()), None)
    f.interp, f.masters = interp, None
    trust = 0.05 * h
    f.settle(6, trust, 60)
    G = e.phases[0].master.rotations()
    mask = og.mask_of(h, w)
    t0 = st["geo"].translation(h, w)
    for i in range(n):
        pat = op.normalize(st["pats"][i].astype(np.float64), mask)
        q, shift, ncc, _ = od.settle6(st["grad"], st["side"], st["geo"].frame(), t0, q0[i], pat, mask, trust, 60,
                                      interp=interp, sheets=st["baked"])
        assert abs(f.keep[1][i] - ncc) < 2e-4, (i, f.keep[1][i], ncc)
        assert np.degrees(float(R.disorientation(f.q[i:i + 1], q[None], G)[0])) < 0.02
        assert np.abs(f.shift[i] - shift).max() < 0.05, (f.shift[i], shift)
    dis = np.degrees(R.disorientation(f.q, st["q"], G))
    assert (dis < 0.5).all(), dis


TRUTH = (0.5, 0.3, 0.6)


@pytest.fixture(scope="module")
def scan():
    """An 8 × 12 map of 60 × 60 patterns simulated with the beam travelling 25 µm a step on a
    detector of 60 µm pixels (the patterns' sources move half a pixel a cell), Gaussian noise as
    strong as the signal (the reference test's synthetic scan, tests/test_api.py:57-70)."""
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
    s.configure(bandwidth=32)
    s.add_phase(path)
    rows, cols = 8, 12
    geo = dict(sample_tilt_deg=70, detector_tilt_deg=0, px_um=60.0, step_x_um=25.0, step_y_um=25.0)
    s.set_patterns(np.zeros((rows, cols, 60, 60), np.float32))
    s.set_geometry(pc=TRUTH, **geo)
    rng = np.random.default_rng(23)
    q, _ = syn.grain_map(rng, rows, cols, 6, 0.5)
    sims = s.simulate(q, cells=np.arange(rows * cols))
    pats = (sims + sims.std() * rng.normal(size=sims.shape)).astype(np.float32)
    s.set_patterns(pats.reshape(rows, cols, 60, 60))
    return {"s": s, "q": q, "path": path, "geo": geo, "pats": pats.reshape(rows, cols, 60, 60)}


def test_cells_index_where_the_plane_puts_their_sources(scan):
    """A plane through the sources the scan's steps give puts every cell where the steps do."""
    s = scan["s"]
    e = s._e
    s.set_geometry(pc=TRUTH)
    cells = np.arange(96)
    by_steps = e.positions64(cells)
    rows, cols = 8, 12
    from zebsdsolve_b200 import plane as PL
    from zebsdsolve_b200.planefit import pc_of

    pc = pc_of(e.geo.rotation(), by_steps, 60, 60)
    pts = PL.Points(cells // cols, cells % cols, pc)
    P = PL.fit("affine", pts, PL.Frame(rows, cols, 1.0))
    s.set_geometry(plane_kind="affine", plane=P)
    assert s.geometry["plane_kind"] == "affine"
    assert np.abs(e.positions64(cells) - by_steps).max() < 1e-9
    # a pattern centre set by hand is one for the whole map again
    s.set_geometry(pc=TRUTH)
    assert s.geometry["plane_kind"] == "affine"  # (unchanged: the same pc)
    s.set_geometry(pc=(0.5, 0.3, 0.61))
    assert s.geometry["plane_kind"] == "none"
    s.set_geometry(pc=TRUTH)


@pytest.mark.parametrize("method", ["points", "joint"])
def test_the_plane_fit_refines_the_centre(scan, method):
    import zebsdsolve_b200 as ze

    s = scan["s"]
    start = (0.505, 0.296, 0.604)
    s.set_geometry(pc=start)
    s.configure(plane_stride=1, plane_method=method)
    p = s.fit_plane()
    e = np.abs(np.array(p["pc"]) - TRUTH)
    assert e.max() < 0.002 and p["ncc"] >= p["start_ncc"] and p["start_pc"] == list(start), (p["pc"], e, method)
    assert p["kind"] == "affine" and s.geometry["plane_kind"] == "affine" and 90 <= p["n_patterns"] <= 96
    assert p["plane"].shape == (4, 3) and p["said"]["blocks"] >= 2 and np.isfinite(p["said"]["rot_se"]).all()
    pts = s.plane_points()
    assert len(pts["cells"]) == 96 and pts["pc"].shape == (96, 3) and pts["used"].sum() == p["n_used"] >= 80
    cells, phs, quats, ncc = s.fit_patterns()
    assert len(cells) == 96 and (phs == 0).all()
    # (each pattern fitted with its own source: on noisy 60 × 60 patterns its rotation trades off
    # against the source's shift by tenths of a degree; the map's own indexing below is the check)
    d_own = np.degrees(s.disorientation(quats, scan["q"][cells.astype(int)]))
    assert np.median(d_own) < 1.5, np.median(d_own)
    r = s.index()
    d = np.degrees(s.disorientation(r["quaternions"].reshape(-1, 4), scan["q"]))
    assert np.median(d) < 0.3, np.median(d)
    # a failed fit changes nothing
    before = (s.geometry, s.plane_points(), s.fit_patterns())
    s.configure(accept_z=1e9, plane_stride=40)  # nothing accepted, and too few patterns above chance
    with pytest.raises(ze.Error, match="TooFewFitPatterns"):
        s.fit_plane()
    from zebsdsolve_b200.settings import Settings

    s.configure(accept_z=Settings()["accept_z"], plane_stride=2, plane_method="points")
    assert s.geometry == before[0]
    assert all(np.array_equal(v, before[1][k]) for k, v in s.plane_points().items())
    s.set_geometry(pc=TRUTH)


def test_the_automatic_fit(scan):
    import zebsdsolve_b200 as ze

    s = scan["s"]
    s.set_geometry(pc=(0.515, 0.32, 0.58))  # the geometry as given: the automatic fit starts here
    s.configure(plane_stride=1)
    a = s.fit_geometry()
    e = np.abs(np.array(a["pc"]) - TRUTH)
    assert e.max() < 0.002, (a["pc"], e)
    assert a["model"] in ("centre", "line", "affine") and a["start_pc"] != [0.515, 0.32, 0.58]
    assert set(a["models"]) <= {"centre", "line", "affine"} and len(s.pc_levels()) >= 3
    s.configure(plane_stride=2)
    r = ze.index(scan["pats"], [scan["path"]], fit="geometry", pc=(0.515, 0.32, 0.58), bandwidth=32, plane_stride=1,
                 **scan["geo"])
    assert np.abs(np.array(r.geometry["pc"]) - TRUTH).max() < 0.002 and "geometry" in r.fit
    d = np.degrees(s.disorientation(r.quaternions.reshape(-1, 4), scan["q"]))
    assert np.median(d) < 0.3, np.median(d)
    f = ze.fit_plane(scan["pats"], [scan["path"]], pc=(0.503, 0.298, 0.602), bandwidth=32, plane_stride=1,
                     **scan["geo"])
    assert np.abs(np.array(f["pc"]) - TRUTH).max() < 0.002 and f["points"]["pc"].shape[1] == 3
