"""zeb_correlate_peaks_static — the peaks entry point that allocates nothing — against the usual
zeb_correlate_peaks, through the C ABI, on two calls in a row.

It serves callers that cannot call cudaMalloc (a host that fixes its device memory at start-up,
a loop that must not let an allocation synchronize the device): its scratch is a static device
array of the library.  This file is collected last so that a run stopping at its first failure
has run every other test; it builds everything it needs itself, so it also passes alone.
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


def test_static_scratch_peaks_match_the_allocating_entry_point():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import zebsdsolve_b200 as ze
    from zebsdsolve_b200 import _native as N
    from zebsdsolve_b200 import synthetic as syn
    from zebsdsolve_b200.master import write_npz

    sheets = syn.master_sheets(21, side=151, lmax=28, group="432")
    d = tempfile.mkdtemp()
    write_npz(f"{d}/m.npz", sheets, 151, syn.group_matrices("432"), 30)
    s = ze.Solver()
    s.configure(static_background="none", dynamic_background="none")
    s.add_phase(f"{d}/m.npz")
    n = 40
    rng = np.random.default_rng(3)
    s.set_patterns(np.zeros((1, n, 60, 60), np.float32))
    s.set_geometry(pc=(0.5, 0.3, 0.6))
    sims = s.simulate(syn.uniform_quaternions(rng, n), cells=np.arange(n))
    s.set_patterns((sims + 0.5 * sims.std() * rng.normal(size=sims.shape)).astype(np.float32).reshape(1, n, 60, 60))
    e = s._e
    L = 32
    b = e.prepare(L)
    bt = b["tables"]
    ph = b["phases"][0][1]
    pats = e.preprocess(torch.as_tensor(e.patterns.reshape(n, 60, 60), device="cuda"), n)
    items = e.items_of(np.arange(n))
    fr = e.frame()
    alm = torch.empty(n * bt.n_pairs * 2, device="cuda")
    stats = torch.empty(n * 4, device="cuda")
    scr = torch.empty(N.load().zeb_sphere_scratch_bytes(ctypes.byref(bt.st), n) // 4 + 1, device="cuda")
    N.call("zeb_sphere_coefficients", _p(pats), _p(items), n, ctypes.byref(fr), ctypes.byref(bt.st), 3, _p(alm),
           _p(stats), _p(scr), _sp())
    U = torch.empty(N.load().zeb_spectrum_bytes(ctypes.byref(ph.dims), n) // 4 + 1, device="cuda")
    N.call("zeb_spectrum_f32", _p(alm), n, ctypes.byref(ph.dims), _p(ph.Y_f), _p(U), _sp())

    want = torch.empty(n * 8, device="cuda")
    cand = torch.empty(N.load().zeb_peaks_scratch_bytes(ctypes.byref(ph.dims), n) // 4 + 1, device="cuda")
    N.call("zeb_correlate_peaks", _p(U), n, ctypes.byref(ph.dims), _p(bt.tw), _p(ph.rden), 1 << 30, _p(want),
           _p(cand), _sp())
    ref = want.cpu().numpy().reshape(n, 8)
    for _ in range(2):
        got = torch.full((n * 8,), float("nan"), device="cuda")
        N.call("zeb_correlate_peaks_static", _p(U), n, ctypes.byref(ph.dims), _p(bt.tw), _p(ph.rden), 1 << 30, _p(got),
               _sp())
        g = got.cpu().numpy().reshape(n, 8)
        # the same kernels on the same inputs: equal to FP32 rounding of the same arithmetic
        assert np.isfinite(g).all()
        assert np.abs(g - ref).max() < 1e-6, np.abs(g - ref).max()

    # a call beyond the static scratch is refused with a message, and launches nothing
    big = N.ZEB_PEAKS_STATIC_SLABS // ph.dims.nb + 1
    with pytest.raises(N.NativeError, match="static scratch"):
        N.call("zeb_correlate_peaks_static", _p(U), big, ctypes.byref(ph.dims), _p(bt.tw), _p(ph.rden), 1 << 30,
               _p(want), _sp())
