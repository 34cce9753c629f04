"""Parity of the CUDA path with the FP64 oracle, stage by stage, through the C ABI (GPU only).

Tolerances are float32 ones: the kernels compute in FP32 (tables in FP64) and the oracle in
FP64 throughout; each assertion states its bound.
"""
import ctypes
import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import oracle.detector as od  # noqa: E402
import oracle.master as om  # noqa: E402
import oracle.prep as op  # noqa: E402
import oracle.sh as osh  # noqa: E402
import oracle.spherical as osp  # noqa: E402
import oracle.sym as osym  # noqa: E402


@pytest.fixture(scope="module")
def lib():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from zebsdsolve_b200 import _native

    return _native


def sp():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def P(t):
    return ctypes.c_void_p(t.data_ptr())


@pytest.fixture(scope="module")
def world(lib):
    """A small synthetic master (432), an engine with it, and a few simulated noisy patterns."""
    import zebsdsolve_b200 as ze
    from zebsdsolve_b200 import synthetic as syn

    sheets = syn.master_sheets(11, side=151, lmax=28, group="432")
    import tempfile
    from zebsdsolve_b200.master import write_npz

    d = tempfile.mkdtemp()
    path = f"{d}/m432.npz"
    write_npz(path, sheets, 151, syn.group_matrices("432"), 30)
    s = ze.Solver()
    s.configure(static_background="none", dynamic_background="none", bandwidth=16)
    s.add_phase(path)
    rng = np.random.default_rng(5)
    n = 6
    s.set_patterns(np.zeros((1, n, 60, 60), np.float32))
    s.set_geometry(pc=(0.5, 0.3, 0.6), sample_tilt_deg=70, detector_tilt_deg=0)
    q = syn.uniform_quaternions(rng, n)
    sims = s.simulate(q, cells=np.arange(n))
    pats = sims + 0.3 * sims.std() * rng.normal(size=sims.shape)
    s.set_patterns(pats.astype(np.float32).reshape(1, n, 60, 60))
    baked = s.master(0).reshape(-1)
    m_or = om.Master(151, baked, syn.group_matrices("432"), 30)
    m_or.measure_symmetry()
    return {"s": s, "q": q, "pats": pats, "baked": baked, "m_or": m_or, "path": path}


def test_fp64_tables_match_oracle(lib):
    from zebsdsolve_b200 import device

    x, w = device.gauss_legendre(64, torch.device("cuda"))
    xo, wo = osh.gauss_legendre(64)
    assert np.abs(x.cpu().numpy() - xo).max() < 1e-14 and np.abs(w.cpu().numpy() - wo).max() < 1e-14
    plm = device.legendre_table(24, x).cpu().numpy()  # [x][pair]
    assert np.abs(plm - osh.legendre_all(24, xo).T).max() < 1e-12
    L = 20
    d = torch.empty(L ** 3, dtype=torch.float64, device="cuda")
    lib.call("zeb_wigner_half_pi", L, P(d), sp())
    assert np.abs(d.cpu().numpy().reshape(L, L, L) - osh.wigner_half_pi(L)).max() < 1e-12


@pytest.mark.parametrize("h,w,sigma,pixel", [(60, 60, 9.0, 1), (96, 96, 14.4, 1), (50, 70, 0.0, 0), (160, 160, 24.0, 2)])
def test_prep_matches_oracle(lib, h, w, sigma, pixel):
    rng = np.random.default_rng(h + w)
    n = 3
    dt = {0: np.uint8, 1: np.uint16, 2: np.float32}[pixel]
    raw = (rng.random((n, h, w)) * (200 if pixel == 0 else 3000)).astype(dt)
    bg = (rng.random((h, w)) * 30).astype(np.float32)
    r = min(h, w) * 0.5
    mask = (0.5 * (h - 1), 0.5 * (w - 1), r * r)
    out = torch.empty(n * h * w, dtype=torch.float32, device="cuda")
    rawd = torch.as_tensor(raw, device="cuda")
    bgd = torch.as_tensor(bg, device="cuda")
    sb = lib.load().zeb_prep_scratch_bytes(n, h, w, sigma)
    scratch = torch.empty(max(sb // 4, 1), dtype=torch.float32, device="cuda")
    m3 = (ctypes.c_float * 3)(*mask)
    lib.call("zeb_prep_ex", P(rawd), pixel, n, h, w, P(bgd), 1 if sigma > 0 else 0, sigma, m3, 1, P(out), P(scratch), sp())
    got = out.cpu().numpy().reshape(n, h, w)
    for i in range(n):
        ref = op.run(raw[i], static=bg, dynamic="subtract" if sigma > 0 else "none", dynamic_sigma=sigma, mask=mask)
        # unit-norm images: values ~ 1/sqrt(h·w); FP32 agreement to 2e-6 absolute
        assert np.abs(got[i] - ref).max() < 2e-6, (h, w, sigma, np.abs(got[i] - ref).max())


@pytest.mark.parametrize("sh,sw,factor,pixel,sigma", [(160, 160, 2.0, 1, 12.0), (90, 96, 3.0, 0, 0.0),
                                                      (150, 150, 2.5, 1, 9.0), (121, 100, 2.0, 2, 7.0)])
def test_prep_reduced_matches_oracle(lib, sh, sw, factor, pixel, sigma):
    """Binning on the device as the patterns are unpacked (reduce.zig) and then the same filters."""
    rng = np.random.default_rng(sh + sw)
    n = 3
    dt = {0: np.uint8, 1: np.uint16, 2: np.float32}[pixel]
    raw = (rng.random((n, sh, sw)) * (200 if pixel == 0 else 3000)).astype(dt)
    h, w = op.reduced_shape(sh, sw, factor)
    bg = (rng.random((h, w)) * 30).astype(np.float32)
    r = min(h, w) * 0.5
    mask = (0.5 * (h - 1), 0.5 * (w - 1), r * r)
    out = torch.empty(n * h * w, dtype=torch.float32, device="cuda")
    rawd = torch.as_tensor(raw, device="cuda")
    bgd = torch.as_tensor(bg, device="cuda")
    sb = lib.load().zeb_prep_scratch_bytes(n, h, w, sigma)
    scratch = torch.empty(max(sb // 4, 1), dtype=torch.float32, device="cuda")
    m3 = (ctypes.c_float * 3)(*mask)
    lib.call("zeb_prep_reduced", P(rawd), pixel, n, sh, sw, ctypes.c_double(factor), P(bgd), 1 if sigma > 0 else 0,
             sigma, m3, 1, P(out), P(scratch), sp())
    got = out.cpu().numpy().reshape(n, h, w)
    for i in range(n):
        red = op.reduce(raw[i], factor)
        assert red.shape == (h, w)
        ref = op.run(red, static=bg, dynamic="subtract" if sigma > 0 else "none", dynamic_sigma=sigma, mask=mask)
        # unit-norm images: FP32 reduction and filters against FP64, to 2e-6 absolute
        assert np.abs(got[i] - ref).max() < 2e-6, (sh, sw, factor, np.abs(got[i] - ref).max())


def test_binned_scan_indexes(world):
    """A 120 × 120 scan binned by 2 indexes like its 60 × 60 patterns: the area means of the
    simulated patterns upsampled by pixel replication are the patterns themselves."""
    import zebsdsolve_b200 as ze

    pats = world["pats"].reshape(-1, 60, 60)
    big = np.repeat(np.repeat(pats, 2, 1), 2, 2).astype(np.float32).reshape(1, -1, 120, 120)
    s = ze.Solver()
    s.configure(static_background="none", dynamic_background="none", bandwidth=16, binning=2)
    s.add_phase(world["path"])
    s.set_patterns(big)
    s.set_geometry(pc=(0.5, 0.3, 0.6), sample_tilt_deg=70, detector_tilt_deg=0)
    assert tuple(s.pattern_shape) == (60, 60)
    r = s.index()
    ref = world["s"].index()
    dis = np.degrees(s.disorientation(r["quaternions"].reshape(-1, 4), ref["quaternions"].reshape(-1, 4)))
    assert dis.max() < 1e-3, dis


def _frame(s):
    e = s._e
    return e.frame()


@pytest.mark.parametrize("L", [16, 64])  # n_phi 64 (the block kernel) and 256 (a warp per ring pair)
def test_sphere_coefficients_match_oracle(world, lib, L):
    from zebsdsolve_b200.device import BandTables

    s = world["s"]
    e = s._e
    bt = BandTables(L, e.dev)
    fr = _frame(s)
    n = world["pats"].shape[0]
    pats = torch.as_tensor(world["pats"].astype(np.float32), device="cuda").reshape(-1)
    t = e.positions(np.arange(n))
    items = torch.as_tensor(np.concatenate([t, np.arange(n, dtype=np.float32)[:, None]], 1), device="cuda")
    alm = torch.empty(n * bt.n_pairs * 2, dtype=torch.float32, device="cuda")
    stats = torch.empty(n * 4, dtype=torch.float32, device="cuda")
    scr = torch.empty(lib.load().zeb_sphere_scratch_bytes(ctypes.byref(bt.st), n) // 4 + 1, device="cuda")
    lib.call("zeb_sphere_coefficients", P(pats), P(items), n, ctypes.byref(fr), ctypes.byref(bt.st), 3, P(alm), P(stats),
             P(scr), sp())
    got = alm.cpu().numpy().reshape(n, -1, 2)
    got = got[..., 0] + 1j * got[..., 1]
    tb = osp.Tables(L)
    frame = (np.array(fr.c0), np.array(fr.c1), np.array(fr.c2))
    for i in range(n):
        ref, st = osp.coefficients(tb, world["pats"][i].astype(np.float64), t[i].astype(np.float64), frame,
                                   np.array(fr.mask))
        # unit-norm coefficients: FP32 sampling and transforms agree to 2e-5
        assert np.abs(got[i] - ref).max() < 2e-5, np.abs(got[i] - ref).max()
        gs = stats.cpu().numpy().reshape(n, 4)[i]
        assert abs(gs[0] - st[0]) < 1e-4 * st[0] and abs(gs[1] - st[1]) < 1e-5 and abs(gs[2] - st[2]) < 1e-4 * st[2]


@pytest.mark.parametrize("L", [32, 64])
def test_sphere_spans_give_the_full_sampling(world, lib, L):
    """Ring spans (zeb_sphere_spans) only drop samples off the detector: coefficients over the spans
    equal the full sampling's (to float rounding of the window sums' order), also for items far
    outside the positions the spans were made for (their rings fall back to whole)."""
    from zebsdsolve_b200.device import BandTables

    s = world["s"]
    e = s._e
    bt = BandTables(L, e.dev)
    fr = _frame(s)
    n = world["pats"].shape[0]
    pats = torch.as_tensor(world["pats"].astype(np.float32), device="cuda").reshape(-1)
    t = e.positions(np.arange(n)).astype(np.float32)
    # the spans are made for the first item's position; items 3.. move by up to 6 pixels
    shift = np.zeros_like(t)
    shift[3:] = np.random.default_rng(4).uniform(-6, 6, size=(n - 3, 3))
    tt = t + shift
    items = torch.as_tensor(np.concatenate([tt, np.arange(n, dtype=np.float32)[:, None]], 1), device="cuda")
    ts = torch.as_tensor(np.array([[*t[0], 0.0]], np.float32), device="cuda")
    spans = torch.empty(bt.n_theta * 2, dtype=torch.int32, device="cuda")
    lib.call("zeb_sphere_spans", ctypes.byref(fr), ctypes.byref(bt.st), P(ts), 1, 2, P(spans), sp())
    sv = spans.cpu().numpy().reshape(-1, 2)
    assert (sv[:, 1] < bt.n_phi).any() and (sv[:, 1] == 0).any()  # the spans do cut work
    out = []
    for sp_arg in (None, P(spans)):
        alm = torch.empty(n * bt.n_pairs * 2, device="cuda")
        stats = torch.empty(n * 4, device="cuda")
        scr = torch.empty(lib.load().zeb_sphere_scratch_bytes(ctypes.byref(bt.st), n) // 4 + 1, device="cuda")
        lib.call("zeb_sphere_coefficients_spans", P(pats), P(items), n, ctypes.byref(fr), ctypes.byref(bt.st), sp_arg, 3,
                 P(alm), P(stats), P(scr), sp())
        out.append((alm.cpu().numpy(), stats.cpu().numpy()))
    assert np.abs(out[0][0] - out[1][0]).max() < 2e-6
    assert np.allclose(out[0][1], out[1][1], rtol=1e-5, atol=1e-6)


def test_master_harmonics_match_oracle(world):
    s = world["s"]
    e = s._e
    L = 16
    b = e.band(L)
    ph = b["phases"][0][1]
    hm = om.Harmonics(world["m_or"], world["baked"], L)
    f = ph.f.cpu().numpy()
    f2 = ph.f2.cpu().numpy()
    assert np.abs(f - hm.f).max() < 1e-9 * max(1.0, np.abs(hm.f).max())
    assert np.abs(f2 - hm.f2).max() < 1e-9 * max(1.0, np.abs(hm.f2).max())
    assert ph.rules.n_fold == hm.rules.n_fold == 4


@pytest.mark.parametrize("L", [16, 32, 64])
def test_correlation_peaks_match_oracle(world, lib, L):
    s = world["s"]
    e = s._e
    b = e.band(L)
    fr = _frame(s)
    e.denominators(b, fr)
    bt = b["tables"]
    ph = b["phases"][0][1]
    n = world["pats"].shape[0]
    pats = torch.as_tensor(world["pats"].astype(np.float32), device="cuda").reshape(-1)
    t = e.positions(np.arange(n))
    items = torch.as_tensor(np.concatenate([t, np.arange(n, dtype=np.float32)[:, None]], 1), device="cuda")
    alm = torch.empty(n * bt.n_pairs * 2, dtype=torch.float32, device="cuda")
    stats = torch.empty(n * 4, dtype=torch.float32, device="cuda")
    scr = torch.empty(lib.load().zeb_sphere_scratch_bytes(ctypes.byref(bt.st), n) // 4 + 1, device="cuda")
    lib.call("zeb_sphere_coefficients", P(pats), P(items), n, ctypes.byref(fr), ctypes.byref(bt.st), 3, P(alm), P(stats),
             P(scr), sp())
    U = torch.empty(lib.load().zeb_spectrum_bytes(ctypes.byref(ph.dims), n) // 4 + 1, device="cuda")
    lib.call("zeb_spectrum_f32", P(alm), n, ctypes.byref(ph.dims), P(ph.Y_f), P(U), sp())
    peaks = torch.empty(n * 8, device="cuda")
    cand = torch.empty(lib.load().zeb_peaks_scratch_bytes(ctypes.byref(ph.dims), n) // 4 + 1, device="cuda")
    lib.call("zeb_correlate_peaks", P(U), n, ctypes.byref(ph.dims), P(bt.tw), P(ph.rden), 1 << 30, P(peaks), P(cand), sp())
    got = peaks.cpu().numpy().reshape(n, 8)
    # one rden per item (rden_div = 1) takes the other slab kernel: the same arithmetic, the same bits
    rep = ph.rden.repeat(n)
    peaks1 = torch.empty(n * 8, device="cuda")
    lib.call("zeb_correlate_peaks", P(U), n, ctypes.byref(ph.dims), P(bt.tw), P(rep), 1, P(peaks1), P(cand), sp())
    assert np.array_equal(peaks1.cpu().numpy().reshape(n, 8), got)
    # the oracle: harmonics of the same baked master, its window denominators, the volume, the peak
    tb = osp.Tables(L)
    hm = om.Harmonics(world["m_or"], world["baked"], L)
    pt = osp.PhaseTables(tb, hm, om.fold_of(hm.rules))
    frame = (np.array(fr.c0), np.array(fr.c1), np.array(fr.c2))
    t0 = e.geo.translation(60, 60)
    walm, wst = osp.coefficients(tb, None, t0, frame, np.array(fr.mask), flags=osp.FLAG_WINDOW, shape=(60, 60))
    rden = osp.window_denominators(tb, pt, walm, wst[0])
    assert np.abs(ph.rden.cpu().numpy().reshape(rden.shape) - rden).max() < 1e-4 * np.abs(rden).max()
    ops = world["m_or"].rotations()
    for i in range(n):
        g, _ = osp.coefficients(tb, world["pats"][i].astype(np.float64), t[i].astype(np.float64), frame, np.array(fr.mask))
        vol = osp.correlation_volume(tb, pt, hm.f, g) * rden
        q, v0, abc, idx = osp.peak(tb, pt, vol)
        assert abs(got[i, 4] - v0) < 2e-4, (got[i, 4], v0)
        dis = math.degrees(float(osym.disorientation(got[i, :4].astype(np.float64), q, ops)))
        assert dis < 0.05, dis


def _spectra(lib, bt, ph, alm, n, status):
    """U of n items in both forms (plain FP32, tensor-core BF16 at the phase's split) through the C ABI."""
    nbytes = lib.load().zeb_spectrum_bytes(ctypes.byref(ph.dims), n)
    U32 = torch.empty(nbytes // 4, device="cuda")
    lib.call("zeb_spectrum_f32", P(alm), n, ctypes.byref(ph.dims), P(ph.Y_f), P(U32), sp())
    U16 = torch.full((nbytes // 4,), float("nan"), device="cuda")
    B = torch.empty(lib.load().zeb_tc_patterns_bytes(ctypes.byref(ph.dims), ph.split, n), dtype=torch.uint8,
                    device="cuda")
    lib.call("zeb_spectrum_bf16", P(alm), n, ctypes.byref(ph.dims), ph.split, P(ph.A), P(B), P(U16), P(status), sp())
    return U32, U16


def _peaks(lib, bt, ph, rden, U, n):
    peaks = torch.empty(n * 8, device="cuda")
    cand = torch.empty(lib.load().zeb_peaks_scratch_bytes(ctypes.byref(ph.dims), n) // 4 + 1, device="cuda")
    lib.call("zeb_correlate_peaks", P(U), n, ctypes.byref(ph.dims), P(bt.tw), P(rden), 1 << 30, P(peaks), P(cand), sp())
    return peaks.cpu().numpy().reshape(n, 8)


def _refined(lib, e, fr, pd, items, seeds, n):
    """Records after 8 refinement iterations from the given peaks (the engine's own settings)."""
    p = e.phases[0]
    recs = torch.empty(n * 8, device="cuda")
    opts = lib.RefineOpts(8, math.radians(2.0), 1.0, 0.02, 1e4, 16, 7.0)
    sd = torch.as_tensor(seeds.astype(np.float32), device="cuda").reshape(-1)
    lib.call("zeb_refine", P(pd), P(items), P(sd), 8, n, ctypes.byref(fr), P(p.baked[3]), P(p.baked[4]), p.master.side,
             ctypes.byref(opts), P(recs), sp())
    return recs.cpu().numpy().reshape(n, 8)


@pytest.mark.parametrize("L,precision", [(32, "bf16x3"), (64, "bf16x3"), (32, "bf16"), (64, "bf16")])
def test_bf16_spectrum_matches_fp32_and_oracle(world, lib, L, precision):
    """The tensor-core spectrum (BF16 operands, FP32 accumulation) against the plain FP32 one and,
    at L = 32, the FP64 oracle.  bf16x3 (every order split hi/lo): U within 5e-5 of its largest
    magnitude, the peak score within 1e-4 and its orientation within 0.05 deg, as the FP32 form.
    bf16 (split for l <= 16, hi*hi above): U within 4e-3, the peak score within 1e-3; a peak may
    land in the other cell of a near tie, so orientations are compared after refinement
    (within 0.1 deg, NCC within 1e-3)."""
    from zebsdsolve_b200 import device

    s = world["s"]
    e = s._e
    b = e.band(L)
    fr = _frame(s)
    e.denominators(b, fr)
    bt = b["tables"]
    ph32 = b["phases"][0][1]
    p = e.phases[0]
    ph = device.PhaseBand(bt, p.baked[1], p.master.side, L, precision)
    assert ph.A is not None and torch.equal(ph.Y_f, ph32.Y_f)
    full = precision == "bf16x3"
    n = world["pats"].shape[0]
    pats = torch.as_tensor(world["pats"].astype(np.float32), device="cuda").reshape(-1)
    t = e.positions(np.arange(n))
    items = torch.as_tensor(np.concatenate([t, np.arange(n, dtype=np.float32)[:, None]], 1), device="cuda")
    alm = torch.empty(n * bt.n_pairs * 2, dtype=torch.float32, device="cuda")
    stats = torch.empty(n * 4, dtype=torch.float32, device="cuda")
    scr = torch.empty(lib.load().zeb_sphere_scratch_bytes(ctypes.byref(bt.st), n) // 4 + 1, device="cuda")
    lib.call("zeb_sphere_coefficients", P(pats), P(items), n, ctypes.byref(fr), ctypes.byref(bt.st), 3, P(alm), P(stats),
             P(scr), sp())
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    U32, U16 = _spectra(lib, bt, ph, alm, n, status)
    assert int(status.item()) == 0
    a32, a16 = U32.cpu().numpy(), U16.cpu().numpy()
    assert np.isfinite(a16).all()
    scale = np.abs(a32).max()
    err = np.abs(a16 - a32).max() / scale
    rms = np.sqrt(np.mean((a16 - a32) ** 2)) / np.sqrt(np.mean(a32 ** 2))
    print(f"L={L} {precision}: U max error {err:.2e} of max, rms {rms:.2e}")
    assert err < (5e-5 if full else 4e-3), err
    assert rms < (5e-5 if full else 3e-3), rms

    g32 = _peaks(lib, bt, ph, ph32.rden, U32, n)
    g16 = _peaks(lib, bt, ph, ph32.rden, U16, n)
    ops = world["m_or"].rotations()

    def dis(q1, q2):
        return math.degrees(float(osym.disorientation(q1.astype(np.float64), q2.astype(np.float64), ops)))

    for i in range(n):
        print(f"  item {i}: score {g16[i, 4]:.6f} vs {g32[i, 4]:.6f}, {dis(g16[i, :4], g32[i, :4]):.4f} deg")
        assert abs(g16[i, 4] - g32[i, 4]) < (1e-4 if full else 1e-3), (g16[i, 4], g32[i, 4])
        if full:
            assert dis(g16[i, :4], g32[i, :4]) < 0.05
    if not full:
        pd = e.preprocess(torch.as_tensor(world["pats"].astype(np.float32), device="cuda"), n)
        r32 = _refined(lib, e, fr, pd, items, g32, n)
        r16 = _refined(lib, e, fr, pd, items, g16, n)
        for i in range(n):
            assert abs(r16[i, 4] - r32[i, 4]) < 1e-3, (r16[i, 4], r32[i, 4])
            assert dis(r16[i, :4], r32[i, :4]) < 0.1, dis(r16[i, :4], r32[i, :4])
    if L == 32:
        tb = osp.Tables(L)
        hm = om.Harmonics(world["m_or"], world["baked"], L)
        pt = osp.PhaseTables(tb, hm, om.fold_of(hm.rules))
        frame = (np.array(fr.c0), np.array(fr.c1), np.array(fr.c2))
        walm, wst = osp.coefficients(tb, None, e.geo.translation(60, 60), frame, np.array(fr.mask),
                                     flags=osp.FLAG_WINDOW, shape=(60, 60))
        rden = osp.window_denominators(tb, pt, walm, wst[0])
        for i in range(n):
            g, _ = osp.coefficients(tb, world["pats"][i].astype(np.float64), t[i].astype(np.float64), frame,
                                    np.array(fr.mask))
            vol = osp.correlation_volume(tb, pt, hm.f, g) * rden
            q, v0, abc, idx = osp.peak(tb, pt, vol)
            assert abs(g16[i, 4] - v0) < (2e-4 if full else 1e-3), (g16[i, 4], v0)
            if full:
                assert dis(g16[i, :4], q) < 0.05

    # several pattern tiles, the last one ragged: 300 items = the 6 coefficient sets repeated
    m = 300
    big = alm[: n * bt.n_pairs * 2].view(n, -1).repeat(m // n, 1).reshape(-1).contiguous()
    V32, V16 = _spectra(lib, bt, ph, big, m, status)
    assert int(status.item()) == 0
    v32 = V32.view(m, -1)
    v16 = V16.view(m, -1)
    assert torch.equal(v16[:n].repeat(m // n, 1), v16), "tiles disagree on equal inputs"
    assert float((v16 - v32).abs().max()) < (5e-5 if full else 4e-3) * float(v32.abs().max())


@pytest.mark.parametrize("kind", ["o", "d6", "c2", "c1"])
def test_records_fz_equals_the_host_reduction(lib, kind):
    """zeb_records_fz against the host's to_fz (FP64, ties within 1e-12 keeping the first): the
    same FP32 values, bit for bit, also for orientations on the zone's boundary."""
    from zebsdsolve_b200 import rotations as R

    rng = np.random.default_rng(12)
    ops = R.group(kind)
    q = rng.normal(size=(4000, 4))
    q[:200] = ops[rng.integers(0, len(ops), 200)]  # symmetry operators themselves: ties
    q[200:400] *= 1.0 + rng.uniform(-1e-3, 1e-3, (200, 1))  # off unit norm
    recs = np.zeros((len(q), 8), np.float32)
    recs[:, :4] = q.astype(np.float32)
    rd = torch.as_tensor(recs, device="cuda")
    od_ = torch.as_tensor(ops, device="cuda")
    fz = torch.empty(len(q) * 4, device="cuda")
    lib.call("zeb_records_fz", P(rd), len(q), P(od_), len(ops), P(fz), sp())
    want = R.to_fz(recs[:, :4].astype(np.float64), ops).astype(np.float32)
    assert np.array_equal(fz.cpu().numpy().reshape(-1, 4), want)


@pytest.mark.parametrize("kind", ["o", "d6"])
def test_records_bunge_equal_the_host_conversion(lib, kind):
    """zeb_records_fz_bunge: the same zone orientations as zeb_records_fz, and their Bunge angles as
    the host's landing converts them (rotations.to_bunge in FP64, rounded to FP32): equal bits but
    where the device's atan2 (within 2 ulp of FP64) and the host's round across an FP32 boundary,
    never more than one FP32 ulp; the poles of the Bunge chart (Φ = 0 or π) included."""
    from zebsdsolve_b200 import rotations as R

    rng = np.random.default_rng(13)
    ops = R.group(kind)
    q = rng.normal(size=(6000, 4))
    q[:100, 1:3] = 0.0  # Φ = 0: x = y = 0
    q[100:200, [0, 3]] = 0.0  # Φ = π: w = z = 0
    q[200:300, 1:3] *= 1e-9  # near the pole
    recs = np.zeros((len(q), 8), np.float32)
    recs[:, :4] = q.astype(np.float32)
    rd = torch.as_tensor(recs, device="cuda")
    od_ = torch.as_tensor(ops, device="cuda")
    fz = torch.empty(len(q) * 4, device="cuda")
    fz2 = torch.empty(len(q) * 4, device="cuda")
    bg = torch.empty(len(q) * 3, device="cuda")
    lib.call("zeb_records_fz", P(rd), len(q), P(od_), len(ops), P(fz), sp())
    lib.call("zeb_records_fz_bunge", P(rd), len(q), P(od_), len(ops), P(fz2), P(bg), sp())
    f = fz.cpu().numpy().reshape(-1, 4)
    assert np.array_equal(f, fz2.cpu().numpy().reshape(-1, 4))
    got = bg.cpu().numpy().reshape(-1, 3)
    want = R.to_bunge(f.astype(np.float64)).astype(np.float32)
    ulp = np.spacing(np.abs(want).astype(np.float32))
    assert np.all(np.abs(got - want) <= ulp), np.abs(got - want).max()
    assert (got == want).mean() >= 0.999


@pytest.mark.parametrize("entry", ["zeb_refine", "zeb_refine_list", "zeb_refine_list_h"])
def test_refine_and_nmi_match_oracle(world, lib, entry):
    """The refinement kernels (pixels compacted per block; the frame's shared pixel list, 128
    threads an item; the same with the BF16 form's FP16 neighbourhood records) against the
    oracle's refinement and NMI, at the same bounds."""
    s = world["s"]
    e = s._e
    e.prepare_masters()
    fr = _frame(s)
    n = world["pats"].shape[0]
    pats = world["pats"].astype(np.float32)
    # normalized patterns as the engine's preprocessing leaves them
    mask = np.array(fr.mask)
    normed = np.stack([op.normalize(p.astype(np.float64), mask) for p in pats]).astype(np.float32)
    t = e.positions(np.arange(n))
    items = torch.as_tensor(np.concatenate([t, np.arange(n, dtype=np.float32)[:, None]], 1), device="cuda")
    rng = np.random.default_rng(9)
    from zebsdsolve_b200 import rotations as R

    start = R.qstd(R.qmul(R.exp_map(rng.normal(0, math.radians(0.8), (n, 3))), world["q"]))
    seeds = torch.as_tensor(np.concatenate([start, np.zeros((n, 4))], 1).astype(np.float32), device="cuda")
    recs = torch.empty(n * 8, device="cuda")
    p = e.phases[0]
    opts = lib.RefineOpts(8, math.radians(2.0), 1.0, 0.02, 1e4, 16, 7.0)
    pd = torch.as_tensor(normed, device="cuda").reshape(-1)
    if entry == "zeb_refine":
        lib.call("zeb_refine", P(pd), P(items), P(seeds), 8, n, ctypes.byref(fr), P(p.baked[3]), P(p.baked[4]),
                 p.master.side, ctypes.byref(opts), P(recs), sp())
    else:
        npix = lib.load().zeb_mask_pixels(ctypes.byref(fr))
        lst = torch.empty(npix, dtype=torch.int32, device="cuda")
        lib.call("zeb_mask_list", ctypes.byref(fr), P(lst), sp())
        rr, cc = np.nonzero(od.in_mask(fr.h, fr.w, mask))  # raster order
        assert np.array_equal(lst.cpu().numpy(), (rr << 16) | cc)
        table = p.baked[4] if entry == "zeb_refine_list" else p.quads[p.baked[0]]
        lib.call(entry, P(pd), P(items), P(seeds), 8, n, ctypes.byref(fr), P(lst), npix, P(p.baked[3]), P(table),
                 p.master.side, ctypes.byref(opts), P(recs), sp())
    got = recs.cpu().numpy().reshape(n, 8)
    grad = od.gradient_table(world["baked"], 151)
    frame = (np.array(fr.c0), np.array(fr.c1), np.array(fr.c2))
    ops = world["m_or"].rotations()
    for i in range(n):
        qb, best, step = od.refine(grad, 151, frame, t[i], start[i], normed[i].astype(np.float64), mask)
        assert abs(got[i, 4] - best) < 2e-4, (got[i, 4], best)
        dis = math.degrees(float(osym.disorientation(got[i, :4].astype(np.float64), qb, ops)))
        assert dis < 0.02, dis
        v = od.nmi(world["baked"], 151, frame, t[i], got[i, :4].astype(np.float64), normed[i].astype(np.float64), mask)
        assert abs(got[i, 5] - v) < 2e-3, (got[i, 5], v)
        assert got[i, 7] == 7.0
        # and the refinement found the truth
        assert math.degrees(float(osym.disorientation(got[i, :4].astype(np.float64), world["q"][i], ops))) < 0.3


def test_chance_decoys_match_oracle(world, lib):
    s = world["s"]
    e = s._e
    e.prepare_masters()
    fr = _frame(s)
    n = world["pats"].shape[0]
    mask = np.array(fr.mask)
    normed = np.stack([op.normalize(p.astype(np.float64), mask) for p in world["pats"]]).astype(np.float32)
    t = e.positions(np.arange(n))
    items = torch.as_tensor(np.concatenate([t, np.arange(n, dtype=np.float32)[:, None]], 1), device="cuda")
    out = torch.empty(3 * n, device="cuda")
    pd = torch.as_tensor(normed, device="cuda").reshape(-1)
    p = e.phases[0]
    lib.call("zeb_chance", P(pd), P(items), n, 3, ctypes.byref(fr), P(p.baked[3]), p.master.side, 16, P(out), sp())
    got = out.cpu().numpy().reshape(3, n)
    frame = (np.array(fr.c0), np.array(fr.c1), np.array(fr.c2))
    for d in range(3):
        qd = od.decoy(np.arange(n), d)
        for i in range(n):
            v = od.nmi(world["baked"], 151, frame, t[i], qd[i], normed[i].astype(np.float64), mask)
            assert abs(got[d, i] - v) < 2e-3


def test_refine_and_chance_on_a_large_detector_match_oracle(world, lib):
    """A 120 × 120 detector (its masked-pixel list exceeds the shared-memory budget, so the kernels
    that evaluate each pixel's ray in place run): refinement, NMI and decoys against the oracle."""
    import zebsdsolve_b200 as ze

    s = ze.Solver()
    s.configure(static_background="none", dynamic_background="none", bandwidth=16)
    s.add_phase(world["path"])
    n = 3
    s.set_patterns(np.zeros((1, n, 120, 120), np.float32))
    s.set_geometry(pc=(0.5, 0.3, 0.6), sample_tilt_deg=70, detector_tilt_deg=0)
    q = world["q"][:n]
    rng = np.random.default_rng(15)
    sims = s.simulate(q, cells=np.arange(n))
    pats = sims + 0.3 * sims.std() * rng.normal(size=sims.shape)
    s.set_patterns(pats.astype(np.float32).reshape(1, n, 120, 120))
    e = s._e
    e.prepare_masters()
    fr = _frame(s)
    assert 120 * 120 * 16 > 200 * 1024
    mask = np.array(fr.mask)
    normed = np.stack([op.normalize(p.astype(np.float64), mask) for p in pats]).astype(np.float32)
    t = e.positions(np.arange(n))
    items = torch.as_tensor(np.concatenate([t, np.arange(n, dtype=np.float32)[:, None]], 1), device="cuda")
    from zebsdsolve_b200 import rotations as R

    start = R.qstd(R.qmul(R.exp_map(rng.normal(0, math.radians(0.8), (n, 3))), q))
    seeds = torch.as_tensor(np.concatenate([start, np.zeros((n, 4))], 1).astype(np.float32), device="cuda")
    recs = torch.empty(n * 8, device="cuda")
    p = e.phases[0]
    opts = lib.RefineOpts(8, math.radians(2.0), 1.0, 0.02, 1e4, 16, 3.0)
    pd = torch.as_tensor(normed, device="cuda").reshape(-1)
    lib.call("zeb_refine", P(pd), P(items), P(seeds), 8, n, ctypes.byref(fr), P(p.baked[3]), P(p.baked[4]), p.master.side,
             ctypes.byref(opts), P(recs), sp())
    got = recs.cpu().numpy().reshape(n, 8)
    out = torch.empty(2 * n, device="cuda")
    lib.call("zeb_chance", P(pd), P(items), n, 2, ctypes.byref(fr), P(p.baked[3]), p.master.side, 16, P(out), sp())
    dec = out.cpu().numpy().reshape(2, n)
    grad = od.gradient_table(world["baked"], 151)
    frame = (np.array(fr.c0), np.array(fr.c1), np.array(fr.c2))
    ops = world["m_or"].rotations()
    for i in range(n):
        qb, best, step = od.refine(grad, 151, frame, t[i], start[i], normed[i].astype(np.float64), mask)
        assert abs(got[i, 4] - best) < 2e-4, (got[i, 4], best)
        assert math.degrees(float(osym.disorientation(got[i, :4].astype(np.float64), qb, ops))) < 0.02
        v = od.nmi(world["baked"], 151, frame, t[i], got[i, :4].astype(np.float64), normed[i].astype(np.float64), mask)
        assert abs(got[i, 5] - v) < 2e-3, (got[i, 5], v)
        for d in range(2):
            vd = od.nmi(world["baked"], 151, frame, t[i], od.decoy(np.arange(n), d)[i], normed[i].astype(np.float64), mask)
            assert abs(dec[d, i] - vd) < 2e-3


@pytest.mark.parametrize("side", [100, 120, 160])
def test_larger_detectors_take_their_own_launch_shapes(world, lib, side):
    """Detectors whose masked-pixel lists leave fewer refinement blocks an SM (100²: 256 threads a
    pattern; 120² and 160²: 512, at 160² with about 160 KB of shared memory, one block an SM) and,
    from 120², whose pattern exceeds the ring kernel's 48 KB of shared memory (sampled from global
    memory): coefficients at L = 64 and the refinement over the shared pixel list against the
    oracle, with the 60 × 60 bounds."""
    import zebsdsolve_b200 as ze
    from zebsdsolve_b200 import rotations as R
    from zebsdsolve_b200.device import BandTables

    s = ze.Solver()
    s.configure(static_background="none", dynamic_background="none", bandwidth=16)
    s.add_phase(world["path"])
    n = 3
    s.set_patterns(np.zeros((1, n, side, side), np.float32))
    s.set_geometry(pc=(0.5, 0.3, 0.6), sample_tilt_deg=70, detector_tilt_deg=0)
    q = world["q"][:n]
    rng = np.random.default_rng(side)
    sims = s.simulate(q, cells=np.arange(n))
    pats = sims + 0.3 * sims.std() * rng.normal(size=sims.shape)
    s.set_patterns(pats.astype(np.float32).reshape(1, n, side, side))
    e = s._e
    e.prepare_masters()
    fr = _frame(s)
    mask = np.array(fr.mask)
    normed = np.stack([op.normalize(p.astype(np.float64), mask) for p in pats]).astype(np.float32)
    t = e.positions(np.arange(n))
    items = torch.as_tensor(np.concatenate([t, np.arange(n, dtype=np.float32)[:, None]], 1), device="cuda")
    pd = torch.as_tensor(normed, device="cuda").reshape(-1)
    frame = (np.array(fr.c0), np.array(fr.c1), np.array(fr.c2))
    # the coefficients at L = 64 (the warp-per-ring-pair kernel)
    bt = BandTables(64, e.dev)
    alm = torch.empty(n * bt.n_pairs * 2, device="cuda")
    stats = torch.empty(n * 4, device="cuda")
    scr = torch.empty(lib.load().zeb_sphere_scratch_bytes(ctypes.byref(bt.st), n) // 4 + 1, device="cuda")
    lib.call("zeb_sphere_coefficients", P(pd), P(items), n, ctypes.byref(fr), ctypes.byref(bt.st), 3, P(alm), P(stats),
             P(scr), sp())
    got = alm.cpu().numpy().reshape(n, -1, 2)
    got = got[..., 0] + 1j * got[..., 1]
    tb = osp.Tables(64)
    for i in range(n):
        ref, _ = osp.coefficients(tb, normed[i].astype(np.float64), t[i].astype(np.float64), frame, mask)
        assert np.abs(got[i] - ref).max() < 2e-5, np.abs(got[i] - ref).max()
    # over the ring spans (each direction sampled once into the shared cache): the same coefficients
    ts = torch.as_tensor(np.concatenate([t[:1], np.zeros((1, 1), np.float32)], 1).astype(np.float32), device="cuda")
    spans = torch.empty(bt.n_theta * 2, dtype=torch.int32, device="cuda")
    lib.call("zeb_sphere_spans", ctypes.byref(fr), ctypes.byref(bt.st), P(ts), 1, 2, P(spans), sp())
    alm2 = torch.empty_like(alm)
    lib.call("zeb_sphere_coefficients_spans", P(pd), P(items), n, ctypes.byref(fr), ctypes.byref(bt.st), P(spans), 3,
             P(alm2), P(stats), P(scr), sp())
    assert float((alm2 - alm).abs().max()) < 2e-6
    # the refinement over the shared pixel list
    lst = e.mask_list(fr)
    assert lst is not None
    start = R.qstd(R.qmul(R.exp_map(rng.normal(0, math.radians(0.8), (n, 3))), q))
    seeds = torch.as_tensor(np.concatenate([start, np.zeros((n, 4))], 1).astype(np.float32), device="cuda")
    recs = torch.empty(n * 8, device="cuda")
    p = e.phases[0]
    opts = lib.RefineOpts(8, math.radians(2.0), 1.0, 0.02, 1e4, 16, 3.0)
    lib.call("zeb_refine_list", P(pd), P(items), P(seeds), 8, n, ctypes.byref(fr), P(lst), lst.numel(), P(p.baked[3]),
             P(p.baked[4]), p.master.side, ctypes.byref(opts), P(recs), sp())
    got = recs.cpu().numpy().reshape(n, 8)
    grad = od.gradient_table(world["baked"], 151)
    ops = world["m_or"].rotations()
    for i in range(n):
        qb, best, step = od.refine(grad, 151, frame, t[i], start[i], normed[i].astype(np.float64), mask)
        assert abs(got[i, 4] - best) < 2e-4, (got[i, 4], best)
        assert math.degrees(float(osym.disorientation(got[i, :4].astype(np.float64), qb, ops))) < 0.02
        v = od.nmi(world["baked"], 151, frame, t[i], got[i, :4].astype(np.float64), normed[i].astype(np.float64), mask)
        assert abs(got[i, 5] - v) < 2e-3, (got[i, 5], v)


@pytest.mark.parametrize("precision", ["f32", "bf16", "bf16x3"])
def test_index_end_to_end_recovers_orientations(lib, precision):
    """The reference's own bar (tests/test_api.py:206-214): 8 × 12 simulated patterns with noise of
    1.0 × their deviation, indexed: median disorientation < 0.15°, max < 1°, in each precision."""
    import tempfile

    import zebsdsolve_b200 as ze
    from zebsdsolve_b200 import synthetic as syn
    from zebsdsolve_b200.master import write_npz

    sheets = syn.master_sheets(2, side=401, lmax=96, group="432", device="cuda")
    d = tempfile.mkdtemp()
    write_npz(f"{d}/m.npz", sheets, 401, syn.group_matrices("432"), 30)
    rng = np.random.default_rng(7)
    s = ze.Solver()
    s.configure(static_background="none", dynamic_background="none", precision=precision)
    s.add_phase(f"{d}/m.npz")
    rows, cols = 8, 12
    s.set_patterns(np.zeros((rows, cols, 60, 60), np.float32))
    s.set_geometry(pc=(0.44, 0.24, 0.53), sample_tilt_deg=70, detector_tilt_deg=0, px_um=70 * 8, step_x_um=20, step_y_um=20)
    q = syn.uniform_quaternions(rng, rows * cols)
    sims = s.simulate(q, cells=np.arange(rows * cols))
    sims = sims + 1.0 * sims.std() * rng.normal(size=sims.shape)
    s.set_patterns(sims.astype(np.float32).reshape(rows, cols, 60, 60))
    r = s.index()
    dis = np.degrees(s.disorientation(r["quaternions"].reshape(-1, 4), q))
    bad = np.flatnonzero(dis > 1.0)
    assert np.median(dis) < 0.15 and dis.max() < 1.0, (np.median(dis), dis.max(), bad.tolist())
    assert (r["phase"] == 0).all()
