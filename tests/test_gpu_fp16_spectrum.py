"""The BF16 form's FP16 spectrum and its tensor-core transform along a, through the C ABI, against
the same GEMM's FP32 spectrum and the CUDA-core transform (zeb_spectrum_bf16 + zeb_correlate_peaks),
which the oracle tests pin (GPU only).

Bounds: U16/s equals the FP32 U to FP16 rounding (2^-11 of the largest |U|, plus the rounding of
the scale's range); the peak scores agree within 5e-4 (both twiddles and U rounded to FP16 on one
side); a peak's cell may move to a neighbour in a near tie, so orientations are compared as a share.
"""
import ctypes
import tempfile

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _sp():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


CASES = [(64, "432", 401, 96, 300), (32, "432", 201, 48, 200), (16, "432", 151, 28, 130), (64, "622", 201, 48, 150)]


@pytest.mark.parametrize("L,group,side,lmax,n", CASES)
def test_fp16_spectrum_and_tensor_core_peaks(L, group, side, lmax, n):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import zebsdsolve_b200 as ze
    from zebsdsolve_b200 import _native as N
    from zebsdsolve_b200 import synthetic as syn
    from zebsdsolve_b200.master import write_npz

    sheets = syn.master_sheets(5, side=side, lmax=lmax, group=group, device="cuda")
    d = tempfile.mkdtemp()
    write_npz(f"{d}/m.npz", sheets, side, syn.group_matrices(group), syn.POINT_GROUP[group])
    s = ze.Solver()
    s.configure(bandwidth=L, precision="bf16")
    s.add_phase(f"{d}/m.npz")
    rng = np.random.default_rng(L + n)
    s.set_patterns(np.zeros((1, n, 60, 60), np.uint16))
    s.set_geometry(pc=(0.5, 0.3, 0.6), sample_tilt_deg=70, detector_tilt_deg=0)
    sims = s._e.simulate_device(0, np.arange(n), syn.uniform_quaternions(rng, n))
    pats16 = syn.counted_patterns(sims, seed=n).cpu().numpy()
    s.set_patterns(pats16.reshape(1, n, 60, 60))
    e = s._e
    b = e.prepare(L)
    bt = b["tables"]
    ph = b["phases"][0][1]
    assert ph.u_scale is not None and ph.split == min(16, L - 1)
    dims = ph.dims
    pats = e.preprocess(torch.as_tensor(pats16, device="cuda"), n, np.arange(n))
    items = e.items_of(np.arange(n))
    fr = e.frame()
    e.denominators(b, fr)
    alm = torch.empty(n * bt.n_pairs * 2, device="cuda")
    stats = torch.empty(n * 4, device="cuda")
    scr = torch.empty(N.load().zeb_sphere_scratch_bytes(ctypes.byref(bt.st), n) // 4 + 1, device="cuda")
    N.call("zeb_sphere_coefficients", _p(pats), _p(items), n, ctypes.byref(fr), ctypes.byref(bt.st), 3, _p(alm),
           _p(stats), _p(scr), _sp())
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    B = torch.empty(N.load().zeb_tc_patterns_bytes(ctypes.byref(dims), ph.split, n), dtype=torch.uint8, device="cuda")
    U = torch.empty(N.load().zeb_spectrum_bytes(ctypes.byref(dims), n) // 4 + 1, device="cuda")
    N.call("zeb_spectrum_bf16", _p(alm), n, ctypes.byref(dims), ph.split, _p(ph.A), _p(B), _p(U), _p(status), _sp())
    U16 = torch.empty(N.load().zeb_spectrum_h_bytes(ctypes.byref(dims), n), dtype=torch.uint8, device="cuda")
    N.call("zeb_spectrum_bf16_h", _p(alm), n, ctypes.byref(dims), ph.split, _p(ph.A), _p(B), _p(U16), ph.u_scale,
           _p(status), _sp())
    torch.cuda.synchronize()
    assert int(status.item()) == 0

    # U16[item tile][j][c][m'][re|im][item % 128] / s against U[item][j][m'][c] (re, im)
    Ln, nb, nc = dims.L, dims.nb, dims.nc
    pt = (n + 127) // 128
    h = U16.view(torch.float16)[: pt * nb * nc * Ln * 2 * 128].view(pt, nb, nc, Ln, 2, 128)
    h = h.permute(1, 2, 3, 4, 0, 5).reshape(nb, nc, Ln, 2, pt * 128)[..., :n].float() / ph.u_scale
    u = U[: n * nb * Ln * nc * 2].view(n, nb, Ln, nc, 2).permute(1, 3, 2, 4, 0)  # → [j][c][m'][ri][item]
    top = float(u.abs().max())
    assert top * ph.u_scale <= 16384 * 1.001  # the scale's bound holds
    err = float((h - u).abs().max())
    assert err <= top * 2.0 ** -11 + 1e-6 * top, (err, top)

    want = torch.empty(n * 8, device="cuda")
    got = torch.full((n * 8,), float("nan"), device="cuda")
    cand = torch.empty(N.load().zeb_peaks_scratch_bytes(ctypes.byref(dims), n) // 4 + 1, device="cuda")
    N.call("zeb_correlate_peaks", _p(U), n, ctypes.byref(dims), _p(bt.tw), _p(ph.rden), 1 << 30, _p(want), _p(cand),
           _sp())
    N.call("zeb_correlate_peaks_h", _p(U16), n, ctypes.byref(dims), ph.u_scale, _p(ph.rden), _p(got), _p(cand),
           _p(status), _sp())
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    w = want.cpu().numpy().reshape(n, 8).astype(np.float64)
    g = got.cpu().numpy().reshape(n, 8).astype(np.float64)
    assert np.isfinite(g).all()
    ds = np.abs(g[:, 4] - w[:, 4])
    assert ds.max() <= 5e-4, np.sort(ds)[-4:]
    # modulo the master's rotations: its symmetric copies in the volume are exact ties, which the
    # two forms' rounding may break either way
    ang = np.degrees(s.disorientation(g[:, :4], w[:, :4]))
    assert (ang <= 0.1).mean() >= 0.9, np.sort(ang)[-8:]


def test_correlate_peaks_h_refuses_what_it_cannot_take():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from zebsdsolve_b200 import _native as N

    d = N.So3Dims(128, 256, 129, 64, 4, 31, 128 * 129 // 2)  # L = 128: beyond the tile of one stage
    x = torch.zeros(1024, device="cuda")
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    with pytest.raises(N.NativeError, match="unsupported dims"):
        N.call("zeb_correlate_peaks_h", _p(x), 4, ctypes.byref(d), 1.0, _p(x), _p(x), _p(x), _p(st), _sp())
