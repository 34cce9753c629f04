"""Dictionary indexing on the GPU against the oracle: the simulated entries, the tensor-core top
eight and the FP32 match, Oja's rule, and the methods "dictionary" and "pca" (alone and as the
first of two sweeps) through the public API."""
import ctypes
import tempfile

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import oracle.dictionary as odict  # noqa: E402


def sp():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def P(t):
    return ctypes.c_void_p(t.data_ptr())


@pytest.fixture(scope="module")
def world():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import zebsdsolve_b200 as ze
    from zebsdsolve_b200 import synthetic as syn
    from zebsdsolve_b200.master import write_npz

    sheets = syn.master_sheets(11, side=151, lmax=28, group="432")
    d = tempfile.mkdtemp()
    path = f"{d}/m432.npz"
    write_npz(path, sheets, 151, syn.group_matrices("432"), 30)
    s = ze.Solver()
    s.configure(static_background="none", dynamic_background="none", bandwidth=16)
    s.add_phase(path)
    n = 24
    rng = np.random.default_rng(8)
    s.set_patterns(np.zeros((4, 6, 60, 60), np.float32))
    s.set_geometry(pc=(0.5, 0.3, 0.6), sample_tilt_deg=70, detector_tilt_deg=0)
    q = syn.uniform_quaternions(rng, n)
    sims = s.simulate(q, cells=np.arange(n))
    pats = sims + 0.3 * sims.std() * rng.normal(size=sims.shape)
    s.set_patterns(pats.astype(np.float32).reshape(4, 6, 60, 60))
    e = s._e
    e.prepare_masters()
    return {"s": s, "q": q, "path": path, "e": e}


def _geometry(e):
    fr = e.frame()
    rows, cols, h, w = e.info()
    t = e.geo.translation(h, w).astype(np.float32)
    return fr, t


def test_dictionary_grid_is_the_oracles(world):
    from zebsdsolve_b200 import dictionary as DI

    rots = world["e"].phases[0].master.rotations()
    a = odict.dictionary(6, rots)
    b = DI.cubochoric_grid(6, rots)
    assert a.shape == b.shape and np.array_equal(a, b)


def test_dict_sims_match_oracle(world):
    from zebsdsolve_b200 import dictionary as DI

    e = world["e"]
    p = e.phases[0]
    fr, t = _geometry(e)
    q = DI.cubochoric_grid(4, p.master.rotations())
    qd = torch.as_tensor(q, device="cuda")
    out = torch.empty(len(q), fr.h * fr.w, device="cuda")
    DI.simulate(fr, p.baked[3], p.master.side, t, qd, out)
    frame = (np.array(fr.c0), np.array(fr.c1), np.array(fr.c2))
    ref = odict.sims(p.baked[1].cpu().numpy(), p.master.side, frame, t.astype(np.float64), q, fr.h, fr.w,
                     tuple(fr.mask))
    # unit-norm rows, values ~1/60: FP32 with the fitted arctangent against FP64, to 5e-5
    err = np.abs(out.cpu().numpy() - ref).max()
    assert err < 5e-5, err


def _dictionary_rows(world, grid, noise):
    from zebsdsolve_b200 import dictionary as DI

    e = world["e"]
    p = e.phases[0]
    fr, t = _geometry(e)
    q = DI.cubochoric_grid(grid, p.master.rotations())
    qd = torch.as_tensor(q, device="cuda")
    d = torch.empty(len(q), fr.h * fr.w, device="cuda")
    DI.simulate(fr, p.baked[3], p.master.side, t, qd, d)
    # "patterns": entries rotated a little, with noise, renormalized
    rng = np.random.default_rng(grid)
    pick = rng.choice(len(q), 300)
    x = d[torch.as_tensor(pick, device="cuda")].clone()
    x += noise * torch.randn(x.shape, device="cuda", generator=torch.Generator("cuda").manual_seed(1)) / 60
    x /= torch.linalg.norm(x, dim=1, keepdim=True)
    return x.contiguous(), d, qd


def _bf16(a):
    return a.to(torch.bfloat16).double().cpu().numpy()


def test_tensor_core_top8_matches_a_bf16_reference(world):
    from zebsdsolve_b200 import _native as Nn
    from zebsdsolve_b200 import dictionary as DI

    x, d, qd = _dictionary_rows(world, 10, 2.0)
    n, K = x.shape
    nd = d.shape[0]
    assert nd % 256 and K % 64  # ragged in both
    xp, dp = DI.panel(x), DI.panel(d)
    sl = Nn.load().zeb_match_slices(n, nd, K, 1)
    cv = torch.empty(n * sl * 8, device="cuda")
    ci = torch.empty(n * sl * 8, dtype=torch.int32, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    Nn.call("zeb_match_bf16", P(xp), n, P(dp), nd, K, sl, P(cv), P(ci), P(status), sp())
    assert int(status.item()) == 0
    S = _bf16(x) @ _bf16(d).T  # the BF16 operands' products, accumulated in FP64
    ci_dev = ci
    cv = cv.cpu().numpy().reshape(n, sl, 8)
    ci = ci.cpu().numpy().reshape(n, sl, 8)
    per = -(-((nd + 255) // 256) // sl) * 256
    for p in range(n):
        for k in range(sl):
            lo, hi = k * per, min(nd, (k + 1) * per)
            ref = np.sort(S[p, lo:hi])[::-1][:8]
            got = cv[p, k]
            assert np.all((ci[p, k] >= lo) & (ci[p, k] < hi))
            # FP32 accumulation over 3600 products: the values to 1e-5, each the score of its index
            assert np.abs(got - ref).max() < 1e-5, (p, k, got, ref)
            assert np.abs(S[p, ci[p, k]] - got).max() < 1e-5
    # the FP32 rescoring picks the exact best (FP64 scores of the FP32 rows; near-ties within 1e-6)
    seeds = torch.empty(n * 8, device="cuda")
    Nn.call("zeb_match_best", P(x), n, P(d), nd, K, P(ci_dev), sl * 8, P(qd), P(seeds), sp())
    sd = seeds.cpu().numpy().reshape(n, 8)
    i_ref, v_ref = odict.best(x.cpu().numpy(), d.cpu().numpy())
    got_i = sd[:, 5].astype(int)
    S64 = x.double().cpu().numpy() @ d.double().cpu().numpy().T
    assert np.all(S64[np.arange(n), got_i] >= v_ref - 1e-6)
    assert (got_i == i_ref).mean() > 0.99
    assert np.abs(sd[:, 4] - v_ref).max() < 1e-5
    assert np.allclose(sd[:, :4], qd.cpu().numpy()[got_i])


def test_fp32_match_picks_the_oracles_best(world):
    from zebsdsolve_b200 import _native as Nn

    x, d, qd = _dictionary_rows(world, 9, 3.0)
    n, K = x.shape
    nd = d.shape[0]
    sl = Nn.load().zeb_match_slices(n, nd, K, 0)
    cv = torch.empty(n * sl, device="cuda")
    ci = torch.empty(n * sl, dtype=torch.int32, device="cuda")
    Nn.call("zeb_match_f32", P(x), n, P(d), nd, K, sl, P(cv), P(ci), sp())
    seeds = torch.empty(n * 8, device="cuda")
    Nn.call("zeb_match_best", P(x), n, P(d), nd, K, P(ci), sl, P(qd), P(seeds), sp())
    sd = seeds.cpu().numpy().reshape(n, 8)
    i_ref, v_ref = odict.best(x.cpu().numpy(), d.cpu().numpy())
    S64 = x.double().cpu().numpy() @ d.double().cpu().numpy().T
    got_i = sd[:, 5].astype(int)
    assert np.all(S64[np.arange(n), got_i] >= v_ref - 1e-6)
    assert (got_i == i_ref).mean() > 0.99
    # every slice's best is that slice's best
    cvn, cin = cv.cpu().numpy().reshape(n, sl), ci.cpu().numpy().reshape(n, sl)
    per = -(-((nd + 127) // 128) // sl) * 128
    for k in range(sl):
        lo, hi = k * per, min(nd, (k + 1) * per)
        assert np.all(S64[np.arange(n), cin[:, k]] >= S64[:, lo:hi].max(1) - 1e-6)
        assert np.abs(cvn[:, k] - S64[np.arange(n), cin[:, k]]).max() < 1e-5


def test_oja_components_match_oracle(world):
    from zebsdsolve_b200 import dictionary as DI

    e = world["e"]
    p = e.phases[0]
    fr, t = _geometry(e)
    q = DI.cubochoric_grid(8, p.master.rotations())
    dic = DI.Dictionary(q, e.dev)
    k, epochs = 12, 2
    dic.prepare_pca(fr, p.baked[3], p.master.side, t, k, epochs)
    X = torch.empty(dic.n, fr.h * fr.w, device="cuda")
    DI.simulate(fr, p.baked[3], p.master.side, t, dic.q, X)
    X = X.double().cpu().numpy()
    W0 = torch.randn(k, fr.h * fr.w, generator=torch.Generator().manual_seed(0x7A6562)).double().numpy()
    W_or = odict.learn(W0, X, epochs, dic.chunk(fr.h * fr.w))
    W = dic.W.double().cpu().numpy()
    assert np.abs(W @ W.T - np.eye(k)).max() < 1e-4  # orthonormal rows
    # the same subspace: every principal angle between the two spans near zero
    cos = np.linalg.svd(W @ W_or.T, compute_uv=False)
    assert cos.min() > 0.999, cos
    coef = dic.rows.double().cpu().numpy()
    assert np.abs(coef - X @ W.T).max() < 1e-4


@pytest.mark.parametrize("method,precision", [("dictionary", "f32"), ("dictionary", "bf16"), ("pca", "bf16"),
                                              ("pca", "f32")])
def test_dictionary_methods_recover_orientations(world, method, precision):
    s = world["s"]
    s.configure(method=method, dict_grid=30, precision=precision, pca_components=128)
    try:
        r = s.index()
    finally:
        s.configure(method="spherical", precision="bf16")
    dis = np.degrees(s.disorientation(r["quaternions"].reshape(-1, 4), world["q"]))
    assert np.median(dis) < 0.2 and (dis < 1).mean() > 0.9, (np.median(dis), dis.max())
    if method == "pca":
        # the components are learned once and kept: the second pca run (FP32 match) reuses them
        learned = [ev for ev in s.events() if ev["kind"] == "log" and "components" in ev["text"]]
        assert len(learned) == (1 if precision == "bf16" else 0)


def test_sweeps_mix_methods(world):
    s = world["s"]
    s.configure(sweeps=2, sweep_method="pca", sweep_dict_grid=20, pca_components=64)
    try:
        assert [p[2] for p in s.sweep_plan] == ["pca", "spherical"]
        r = s.index()
    finally:
        s.configure(sweeps=1, sweep_method="same")
    sw = r["sweep"].ravel()
    dis = np.degrees(s.disorientation(r["quaternions"].reshape(-1, 4), world["q"]))
    assert (sw >= 0).all() and np.median(dis) < 0.15 and dis.max() < 1.0, (sw, np.median(dis), dis.max())


@pytest.mark.parametrize("n,k,cols", [(300, 256, 3600), (130, 200, 3500), (1, 512, 6400)])
def test_pca_projection_kernels_match_fp64(n, k, cols):
    """The batch's projection onto the components (pca.zig:159-162): the tcgen05 form from split
    BF16 panels (hi·hi + hi·lo + lo·hi) and the plain FP32 form against FP64, ragged in patterns,
    components and pixels; unit-norm rows, so every coefficient is at most 1 in size."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import ctypes

    from zebsdsolve_b200 import _native as N

    g = torch.Generator(device="cuda").manual_seed(n + k)
    x = torch.randn(n, cols, generator=g, device="cuda")
    x /= x.norm(dim=1, keepdim=True)
    w = torch.randn(k, cols, generator=g, device="cuda")
    w /= w.norm(dim=1, keepdim=True)
    want = (x.double() @ w.double().T).cpu().numpy()
    P = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    sp = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    xs = torch.empty(N.load().zeb_panel_split_bytes(n, cols), dtype=torch.uint8, device="cuda")
    ws = torch.empty(N.load().zeb_panel_split_bytes(k, cols), dtype=torch.uint8, device="cuda")
    N.call("zeb_pack_panel_split", P(x), n, cols, cols, 0, P(xs), sp)
    N.call("zeb_pack_panel_split", P(w), k, cols, cols, 1, P(ws), sp)
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    got = torch.full((n, k), float("nan"), device="cuda")
    N.call("zeb_project_bf16", P(xs), n, P(ws), k, cols, P(got), P(status), sp)
    got32 = torch.full((n, k), float("nan"), device="cuda")
    N.call("zeb_project_f32", P(x), n, P(w), k, cols, P(got32), sp)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    assert np.abs(got.cpu().numpy() - want).max() < 2e-5
    assert np.abs(got32.cpu().numpy() - want).max() < 2e-6
