"""The other configurations' shapes through the public API on the GPU: bandwidth 128 (config 5's
local sweep) in the plain FP32 and BF16 forms, and a scan of two phases (cubic 432 and
hexagonal 622 masters, config 4) in which every pattern must pick its own phase."""
import tempfile

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def masters():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from zebsdsolve_b200 import synthetic as syn
    from zebsdsolve_b200.master import write_npz

    d = tempfile.mkdtemp()
    out = {}
    for g, seed in (("432", 2), ("622", 3)):
        sheets = syn.master_sheets(seed, side=401, lmax=96, group=g, device="cuda")
        write_npz(f"{d}/m{g}.npz", sheets, 401, syn.group_matrices(g), syn.POINT_GROUP[g])
        out[g] = f"{d}/m{g}.npz"
    return out


def _scan(paths, rows, cols, phase_of, seed, **kw):
    import zebsdsolve_b200 as ze
    from zebsdsolve_b200 import synthetic as syn

    s = ze.Solver()
    s.configure(static_background="none", dynamic_background="none", **kw)
    for p in paths:
        s.add_phase(p)
    n = rows * cols
    s.set_patterns(np.zeros((rows, cols, 60, 60), np.float32))
    s.set_geometry(pc=(0.5, 0.3, 0.6), sample_tilt_deg=70, detector_tilt_deg=0)
    rng = np.random.default_rng(seed)
    q = syn.uniform_quaternions(rng, n)
    pats = np.empty((n, 60, 60), np.float32)
    for ph in np.unique(phase_of):
        sel = np.flatnonzero(phase_of == ph)
        pats[sel] = s.simulate(q[sel], cells=sel, phase=int(ph)).reshape(len(sel), 60, 60)
    pats = pats + 0.5 * pats.std() * rng.normal(size=pats.shape)
    s.set_patterns(pats.astype(np.float32).reshape(rows, cols, 60, 60))
    return s, q


@pytest.mark.parametrize("precision", ["f32", "bf16"])
def test_bandwidth_128_end_to_end(masters, precision):
    s, q = _scan([masters["432"]], 4, 6, np.zeros(24, int), 11, bandwidth=128, precision=precision)
    r = s.index()
    dis = np.degrees(s.disorientation(r["quaternions"].reshape(-1, 4), q))
    assert np.median(dis) < 0.15 and dis.max() < 1.0, (np.median(dis), dis.max())


def test_two_phases_pick_their_phase(masters):
    rng = np.random.default_rng(5)
    phase_of = rng.integers(0, 2, 48)
    s, q = _scan([masters["432"], masters["622"]], 6, 8, phase_of, 13, precision="bf16")
    r = s.index()
    ph = r["phase"].reshape(-1)
    assert (ph == phase_of).mean() >= 0.95, (ph, phase_of)
    for p in (0, 1):
        sel = (ph == p) & (phase_of == p)
        dis = np.degrees(s.disorientation(r["quaternions"].reshape(-1, 4)[sel], q[sel], phase=p))
        assert np.median(dis) < 0.15, (p, np.median(dis))


def test_uneven_scans_of_several_detector_sizes(masters):
    """Config 4's unevenness through one Solver: scans of 40 × 40, 96 × 96 (the wide blur and the
    per-pixel-ray sphere sampling) and 160 × 160 patterns, of different lengths, two phases each,
    indexed one after another at L = 64 in the BF16 form."""
    import zebsdsolve_b200 as ze
    from zebsdsolve_b200 import synthetic as syn

    s = ze.Solver()
    s.configure(static_background="none", dynamic_background="subtract", bandwidth=64, precision="bf16")
    for p in (masters["432"], masters["622"]):
        s.add_phase(p)
    rng = np.random.default_rng(21)
    for side, n in ((40, 30), (96, 20), (160, 12)):
        s.set_patterns(np.zeros((1, n, side, side), np.float32))
        s.set_geometry(pc=(0.5, 0.3, 0.6), sample_tilt_deg=70, detector_tilt_deg=0)
        q = syn.uniform_quaternions(rng, n)
        phase_of = rng.integers(0, 2, n)
        pats = np.empty((n, side, side), np.float32)
        for ph in (0, 1):
            sel = np.flatnonzero(phase_of == ph)
            if len(sel):
                pats[sel] = s.simulate(q[sel], cells=sel, phase=ph).reshape(len(sel), side, side)
        pats = 1000 * (0.6 + 0.1 * pats) + 20 * rng.normal(size=pats.shape)
        s.set_patterns(pats.astype(np.float32).reshape(1, n, side, side))
        r = s.index()
        ph = r["phase"].reshape(-1)
        assert (ph == phase_of).mean() >= 0.9, (side, ph, phase_of)
        ok = ph == phase_of
        dis = np.array([np.degrees(s.disorientation(r["quaternions"].reshape(-1, 4)[i:i + 1], q[i:i + 1],
                                                    phase=int(ph[i])))[0] for i in np.flatnonzero(ok)])
        assert np.median(dis) < 0.2, (side, np.median(dis), dis.max())
