"""Config 3: the six-unknown refinement (source shift / pattern centre and orientation) on the GPU.

The adjoint kernel (zeb_det6 mode 1, the backward of adjoint.ProjectedNCC) against central finite
differences of the FP64 oracle's forward (steps 1e-4 rad and 1e-5 in pattern centre) and of the
device's own forward; the reference's Gauss–Newton sums (mode 2) against the oracle's
restatement of detector.wgsl `sums`; and the Levenberg–Marquardt settle against the oracle's,
on patterns simulated with jittered pattern centres and perturbed orientations.
"""
import tempfile

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import oracle.detector as od  # noqa: E402
import oracle.geometry as og  # noqa: E402
import oracle.rot as orot  # noqa: E402


@pytest.fixture(scope="module")
def setup():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import zebsdsolve_b200 as ze
    from zebsdsolve_b200 import synthetic as syn
    from zebsdsolve_b200.master import write_npz

    side = 201
    sheets = syn.master_sheets(7, side=side, lmax=40, group="432")
    d = tempfile.mkdtemp()
    write_npz(f"{d}/m.npz", sheets, side, syn.group_matrices("432"), 30)
    s = ze.Solver()
    s.configure(static_background="none", dynamic_background="none", master_smooth=0.0)
    s.add_phase(f"{d}/m.npz")
    h = w = 60
    n = 4
    rng = np.random.default_rng(31)
    pc0 = np.array([0.5, 0.3, 0.6])
    s.set_patterns(np.zeros((1, n, h, w), np.float32))
    s.set_geometry(pc=tuple(pc0), sample_tilt_deg=70, detector_tilt_deg=0, step_x_um=0, step_y_um=0)  # one source for every cell
    e = s._e
    e.prepare_masters()
    baked = e.phases[0].baked[1].cpu().numpy().astype(np.float64)
    grad = od.gradient_table(baked, side)
    geo = og.Geometry(pc=tuple(pc0), sample_tilt_deg=70.0)
    frame = geo.frame()
    mask = og.mask_of(h, w)
    q_true = syn.uniform_quaternions(rng, n)
    pc_true = pc0 + rng.uniform(-0.005, 0.005, (n, 3))
    pats = np.stack([od.project(baked, side, frame, geo.translation_for(pc_true[i], h, w), q_true[i], h, w) for i in range(n)])
    pats = pats + 0.2 * pats.std() * rng.normal(size=pats.shape)
    s.set_patterns(pats.astype(np.float32).reshape(1, n, h, w))
    # starting orientations 1–2° off the truth
    ax = rng.normal(size=(n, 3))
    ax /= np.linalg.norm(ax, axis=1, keepdims=True)
    ang = np.radians(rng.uniform(1.0, 2.0, n))
    q_start = np.stack([orot.qstd(orot.qmul(orot.so3_exp(ax[i] * ang[i]), q_true[i])) for i in range(n)])
    return {"s": s, "e": e, "side": side, "baked": baked, "grad": grad, "frame": frame, "mask": mask, "geo": geo,
            "pats": pats, "q_true": q_true, "pc_true": pc_true, "pc0": pc0, "q_start": q_start, "h": h, "w": w, "n": n}


def _plan(st):
    from zebsdsolve_b200 import adjoint

    e = st["e"]
    cells = np.arange(st["n"])
    pats = e.upload(cells)
    items = e.items_of(cells)
    _, sheets, grad, vpair, gpair = e.phases[0].baked
    return adjoint.Plan(pats, items, e.frame(), vpair, gpair, st["side"]), pats


def _normed(st, i):
    import oracle.prep as op

    return op.normalize(st["pats"][i].astype(np.float64), st["mask"])


def test_reference_sums_match_oracle(setup):
    """zeb_det6 mode 2 (the 43 sums of detector.wgsl `sums`) against the oracle's restatement."""
    st = setup
    plan, _ = _plan(st)
    rng = np.random.default_rng(2)
    x = np.concatenate([rng.uniform(-1, 1, (st["n"], 3)), np.zeros((st["n"], 3))], 1).astype(np.float32)
    q = st["q_start"].astype(np.float32)
    got = plan.run(2, torch.as_tensor(x, device="cuda"), torch.as_tensor(q, device="cuda")).cpu().numpy()
    t0 = st["geo"].translation(st["h"], st["w"])
    for i in range(st["n"]):
        ref = od.sums6(st["grad"], st["side"], st["frame"], t0, q[i].astype(np.float64), x[i, :3].astype(np.float64),
                       _normed(st, i), st["mask"])
        scale = np.maximum(np.abs(ref), 1.0)
        assert np.all(np.abs(got[i] - ref) < 2e-4 * scale + 1e-3 * np.abs(ref).max()), np.abs(got[i] - ref).max()
        a, b = od.local_of(ref), od.local_of(got[i].astype(np.float64))
        assert abs(a[0] - b[0]) < 1e-5
        assert np.abs(a[1] - b[1]).max() < 1e-3 * max(1.0, np.abs(a[1]).max())


def test_adjoint_matches_finite_differences(setup):
    """∂NCC/∂x by the adjoint kernel against central differences of the FP64 oracle's forward
    (1e-4 rad in rotation, 1e-5 in pattern centre; 1 % of the largest component: the bilinear
    surface has a kink at every master pixel edge a step may cross) and of the device's FP32 forward."""
    from zebsdsolve_b200 import adjoint

    st = setup
    plan, _ = _plan(st)
    n = st["n"]
    h, w = st["h"], st["w"]
    J = adjoint.pc_jacobian(st["s"]._e.geo, h, w)  # ∂t/∂pc, pixels per unit of pattern centre
    rng = np.random.default_rng(8)
    x = np.concatenate([rng.uniform(-0.5, 0.5, (n, 3)), rng.normal(0, 0.003, (n, 3))], 1)
    q = st["q_start"]
    xd = torch.as_tensor(x.astype(np.float32), device="cuda")
    qd = torch.as_tensor(q.astype(np.float32), device="cuda")
    adj = plan.run(1, xd, qd).cpu().numpy()
    g = adj[:, :6].astype(np.float64)
    t0 = st["geo"].translation(h, w)

    def f64(i, xi):
        qq = orot.qmul(orot.so3_exp(xi[3:]), q[i])
        s6 = od.sums6(st["grad"], st["side"], st["frame"], t0, qq, xi[:3], _normed(st, i), st["mask"])
        return od.local_of(s6)[0]

    for i in range(n):
        assert abs(adj[i, 6] - f64(i, x[i])) < 2e-5
        # rotation: steps of 1e-4 rad
        for k in range(3):
            e_ = np.zeros(6)
            e_[3 + k] = 1e-4
            fd = (f64(i, x[i] + e_) - f64(i, x[i] - e_)) / 2e-4
            assert abs(g[i, 3 + k] - fd) < 1e-2 * max(1.0, np.abs(g[i, 3:]).max()), (i, k, g[i, 3 + k], fd)
        # pattern centre: steps of 1e-5, through t = t(pc)
        gpc = J.T @ g[i, :3]
        for k in range(3):
            dx = np.zeros(6)
            dx[:3] = J[:, k] * 1e-5
            fd = (f64(i, x[i] + dx) - f64(i, x[i] - dx)) / 2e-5
            assert abs(gpc[k] - fd) < 1e-2 * max(1.0, np.abs(gpc).max()), (i, k, gpc[k], fd)
    # the device's own forward, FP32: the same steps, a float-sized tolerance
    for k in range(3):
        dx = np.zeros((n, 6), np.float32)
        dx[:, 3 + k] = 1e-4
        fp = plan.run(0, xd + torch.as_tensor(dx, device="cuda"), qd).cpu().numpy()
        fm = plan.run(0, xd - torch.as_tensor(dx, device="cuda"), qd).cpu().numpy()
        fd = (fp.astype(np.float64) - fm) / 2e-4
        assert np.all(np.abs(fd - g[:, 3 + k]) < 3e-2 * np.maximum(1.0, np.abs(g[:, 3:]).max(1))), (fd, g[:, 3 + k])


def test_autograd_function_is_the_adjoint(setup):
    """ProjectedNCC through autograd: the backward is the adjoint kernel, and gradients flow
    through the pattern-centre map t = t(pc) to (pcx, pcy, pcz) by the chain rule."""
    from zebsdsolve_b200 import adjoint

    st = setup
    plan, _ = _plan(st)
    n = st["n"]
    J = torch.as_tensor(adjoint.pc_jacobian(st["s"]._e.geo, st["h"], st["w"]), dtype=torch.float32, device="cuda")
    dpc = torch.full((n, 3), 1e-3, device="cuda", requires_grad=True)
    phi = torch.zeros(n, 3, device="cuda", requires_grad=True)
    q = torch.as_tensor(st["q_start"].astype(np.float32), device="cuda")
    x = torch.cat([dpc @ J.T, phi], 1)
    score = adjoint.projected_ncc(x, q, plan)
    score.sum().backward()
    direct = plan.run(1, x.detach().contiguous(), q).cpu()
    assert torch.allclose(phi.grad.cpu(), direct[:, 3:6], rtol=1e-6, atol=1e-7)
    assert torch.allclose(dpc.grad.cpu(), direct[:, :3] @ J.cpu(), rtol=1e-5, atol=1e-6)
    assert torch.allclose(score.detach().cpu(), direct[:, 6], atol=1e-6)


def test_adjoint_and_reference_jacobian_agree(setup):
    """The exact adjoint and the reference's Gauss–Newton gradient (from the gradient table, a
    central difference one master pixel wide, interpolated) differ only by that discretization:
    the same direction, a few percent apart."""
    from zebsdsolve_b200 import adjoint

    st = setup
    plan, _ = _plan(st)
    n = st["n"]
    x = torch.zeros(n, 6, device="cuda")
    q = torch.as_tensor(st["q_start"].astype(np.float32), device="cuda")
    ga = plan.run(1, x, q)[:, :6].double()
    ok, ncc, gr, H = adjoint.local_of(plan.run(2, x, q))
    cos = (ga * gr).sum(1) / (ga.norm(dim=1) * gr.norm(dim=1))
    assert bool(ok.all()) and float(cos.min()) > 0.995, cos
    assert float(((ga - gr).norm(dim=1) / gr.norm(dim=1)).max()) < 0.1


@pytest.mark.parametrize("use_list", [False, True])
def test_one_pass_mode_gives_both_passes(setup, use_list):
    """zeb_det6 mode 3 (the adjoint settle's one pass a round) gives mode 2's 43 sums and, through
    adjoint.adjoint_gradient, mode 1's exact gradient (FP32 summation-order noise: 1e-5 of each
    output's scale; the gradient 1e-4 of its norm)."""
    from zebsdsolve_b200 import adjoint

    st = setup
    e = st["e"]
    plan, _ = _plan(st)
    if use_list:
        plan = adjoint.Plan(plan.pats, plan.items, plan.frame, plan.vpair, plan.gpair, plan.side,
                            e.mask_list(e.frame()))
    rng = np.random.default_rng(3)
    x = torch.as_tensor(np.concatenate([rng.normal(0, 0.5, (st["n"], 3)), rng.normal(0, 0.01, (st["n"], 3))], 1),
                        dtype=torch.float32, device="cuda").contiguous()
    q0 = torch.as_tensor(st["q_start"], dtype=torch.float32, device="cuda").contiguous()
    s3 = plan.run(3, x, q0)
    s2 = plan.run(2, x, q0)
    a, b = s3[:, :43].cpu().numpy(), s2.cpu().numpy()
    scale = np.maximum(np.abs(b).max(0), 1e-6)
    assert np.all(np.abs(a - b) <= 1e-5 * scale + 1e-7), np.abs(a - b).max()
    g1 = plan.run(1, x, q0)[:, :6].double()
    g3 = adjoint.adjoint_gradient(s3)
    err = (g3 - g1).norm(dim=1) / g1.norm(dim=1)
    assert float(err.max()) < 1e-4, err


@pytest.mark.parametrize("gradient", ["reference", "adjoint"])
def test_refine_patterns_settles_like_the_oracle(setup, gradient):
    """The six-unknown Levenberg–Marquardt from orientations 1–2° off and the nominal pattern
    centre, on patterns simulated at centres jittered by ±0.005: with the reference's gradient,
    the oracle's settle matched pattern by pattern (NCC 2e-4, orientation 0.02°, shift 0.05 px);
    with either, the NCC risen and the orientation brought from 1–2° to a few tenths of a degree
    of the truth (rotation and source shift trade off against each other on a 60 × 60 pattern)."""
    st = setup
    s = st["s"]
    n = st["n"]
    from zebsdsolve_b200 import rotations as R

    G = s._e.phases[0].master.rotations()
    r = s.refine_patterns(np.arange(n), quaternions=st["q_start"], trust=0.05, rounds=60, gradient=gradient)
    dis = np.degrees(R.disorientation(r["quaternions"], st["q_true"], G))
    start = np.degrees(R.disorientation(st["q_start"], st["q_true"], G))
    print(gradient, "start", start, "end", dis, "pc error", np.abs(r["pc"] - st["pc_true"]).max(1), "rounds", r["rounds"])
    assert (dis < 0.5).all() and (dis < 0.5 * start).all(), dis
    assert np.abs(r["pc"] - st["pc_true"]).max() < 5e-3
    t0 = st["geo"].translation(st["h"], st["w"])
    for i in range(n):
        q, shift, ncc, it = od.settle6(st["grad"], st["side"], st["frame"], t0, st["q_start"][i], _normed(st, i),
                                       st["mask"], trust=0.05 * st["h"], most=60)
        print(" oracle", i, ncc, r["ncc"][i], shift, r["shift"][i])
        if gradient == "reference":
            assert abs(r["ncc"][i] - ncc) < 2e-4, (r["ncc"][i], ncc)
            assert np.degrees(float(R.disorientation(r["quaternions"][i:i + 1], q[None], G)[0])) < 0.02
            assert np.abs(r["shift"][i] - shift).max() < 0.05, (r["shift"][i], shift)
        else:  # the exact gradient's optimum: the same NCC to the discretization of the reference's
            assert r["ncc"][i] > ncc - 1e-4, (r["ncc"][i], ncc)


@pytest.mark.parametrize("mode", [0, 1, 2, 3])
def test_pixel_list_kernel_equals_the_block_list_kernel(setup, mode):
    """zeb_det6_list (the frame's shared pixel list, 128 threads a pattern) gives zeb_det6's
    outputs in every mode, to FP32 summation-order noise (1e-5 of each output's scale)."""
    from zebsdsolve_b200 import adjoint

    st = setup
    e = st["e"]
    plan, pats = _plan(st)
    lst = e.mask_list(e.frame())
    assert lst is not None
    plan_l = adjoint.Plan(plan.pats, plan.items, plan.frame, plan.vpair, plan.gpair, plan.side, lst)
    rng = np.random.default_rng(mode)
    x = torch.as_tensor(np.concatenate([rng.normal(0, 0.5, (st["n"], 3)), rng.normal(0, 0.01, (st["n"], 3))], 1),
                        dtype=torch.float32, device="cuda").contiguous()
    q0 = torch.as_tensor(st["q_start"], dtype=torch.float32, device="cuda").contiguous()
    a = plan.run(mode, x, q0).cpu().numpy()
    b = plan_l.run(mode, x, q0).cpu().numpy()
    scale = np.maximum(np.abs(a).max(0) if a.ndim > 1 else np.abs(a).max(), 1e-6)
    assert np.all(np.abs(a - b) <= 1e-5 * scale + 1e-7), np.abs(a - b).max()
