"""Toy scans (engine.zig:2778-2896), on the CPU with the engine's simulation stood in for (a
pattern that is a function of the orientation): the microstructure (each cell in its nearest
grain, one orientation and phase a grain, blank cells), the detector (the simulation from 0 to a
mean of 1 on a flat or humped background of mean 1) and the counting (Poisson at the mean count),
through the Solver and the reference's C ABI (ze_synthesize)."""
import ctypes

import numpy as np
import pytest

import zebsdsolve_b200 as ze
from zebsdsolve_b200 import build, engine as E, rotations as R, ze_abi as Z
from zebsdsolve_b200.settings import Settings


def _solver(n_phases=2):
    s = ze.Solver.__new__(ze.Solver)
    e = E.Engine.__new__(E.Engine)
    e.set, e.geo, e._resident, e.patterns, e.events, e._full = Settings(), E.Geometry(), None, None, [], False
    e.phases = [object()] * n_phases
    calls = []

    def simulate(phase, cells, quats):
        calls.append((phase, np.asarray(cells).copy()))
        assert e._full  # at the stored size
        h, w = e.patterns.shape[2:]
        ramp = np.linspace(0, 1, h * w, dtype=np.float32)
        return (quats[:, :1] * ramp[None, :] + phase).reshape(len(cells), h, w)
    e.simulate = simulate
    s._e = e
    return s, calls


def test_the_microstructure_and_the_detector():
    s, calls = _solver()
    got = s.synthesize(toy_rows=12, toy_cols=16, toy_grains=5, toy_height=8, toy_width=10, toy_counts=0,
                       toy_blank=0.1)
    q, ph, gr = got["quaternions"], got["phase"], got["grain"]
    assert q.shape == (12, 16, 4) and ph.shape == gr.shape == (12, 16) and set(np.unique(gr)) <= set(range(5))
    # one orientation and one phase a grain (no spread); blank cells about a tenth
    for g in np.unique(gr):
        at = gr == g
        assert np.allclose(q[at], q[at][0]) and len(set(ph[at][ph[at] >= 0])) <= 1
    assert 0.02 < np.mean(ph < 0) < 0.25
    assert np.allclose(np.linalg.norm(q, axis=-1), 1, atol=1e-6) and (q[..., 0] >= 0).all()
    # every crystal cell simulated once, under its own phase
    done = np.concatenate([c for _, c in calls])
    assert sorted(done) == sorted(np.flatnonzero(ph.reshape(-1) >= 0))
    for p, c in calls:
        assert (ph.reshape(-1)[c] == p).all()
    # the detector without noise: the crystals' mean 1 and darkest 0; blank cells flat 1
    pats = s._e.patterns.reshape(12 * 16, -1)
    assert s._e.patterns.shape == (12, 16, 8, 10) and s._e.patterns.dtype == np.float32
    crys = ph.reshape(-1) >= 0
    assert pats[crys].mean() == pytest.approx(1.0, abs=1e-5) and pats[crys].min() == pytest.approx(0.0, abs=1e-6)
    assert np.allclose(pats[~crys], 1.0)
    # the same seed, the same scan; a spread turns cells within their grain
    again, _ = _solver()
    g2 = again.synthesize(toy_rows=12, toy_cols=16, toy_grains=5, toy_height=8, toy_width=10, toy_counts=0,
                          toy_blank=0.1)
    assert np.array_equal(g2["quaternions"], q) and np.array_equal(again._e.patterns, s._e.patterns)
    sp, _ = _solver()
    g3 = sp.synthesize(toy_rows=12, toy_cols=16, toy_grains=5, toy_height=8, toy_width=10, toy_spread_deg=1.0)
    ang = np.degrees(2 * np.arccos(np.minimum(1, np.abs(np.sum(g3["quaternions"] * q, -1)))))
    assert np.array_equal(g3["grain"], gr) and 0.05 < np.median(ang) < 3


def test_background_and_counting():
    s, _ = _solver(1)
    s.synthesize(toy_rows=6, toy_cols=8, toy_grains=1, toy_height=20, toy_width=20, toy_counts=0,
                 toy_contrast=0.25, toy_background_sigma=0.3, toy_blank=1.0)
    flat = s._e.patterns.reshape(48, 20, 20)
    # all blank: (1 − contrast) × the hump + contrast × 1; the hump's mean 1, highest in the middle
    assert flat.mean() == pytest.approx(1.0, abs=1e-5) and flat[0, 10, 10] > flat[0, 0, 0]
    s.synthesize(toy_rows=6, toy_cols=8, toy_grains=2, toy_height=20, toy_width=20, toy_counts=50,
                 toy_contrast=1.0, toy_background_sigma=0.0, toy_blank=0.0)
    counted = s._e.patterns
    assert np.array_equal(counted, np.round(counted)) and counted.mean() == pytest.approx(50, rel=0.02)
    s.synthesize(toy_noise_seed=9)
    assert not np.array_equal(s._e.patterns, counted)  # another count of the one microstructure
    assert any("toy scan" in ev.get("text", "") for ev in s._e.events)


def test_the_c_abi_toy_scan():
    s, _ = _solver()
    s.configure(toy_rows=5, toy_cols=7, toy_grains=3, toy_height=8, toy_width=8)
    lib = ctypes.CDLL(str(build.build_abi()))
    P = ctypes.c_void_p
    lib.ze_synthesize.argtypes, lib.ze_synthesize.restype = [P, P, P, P, ctypes.c_size_t], ctypes.c_int32
    lib.ze_error.argtypes, lib.ze_error.restype = [P, ctypes.c_char_p, ctypes.c_size_t], ctypes.c_size_t
    h = 0x7F40
    Z._handles[h] = Z._Handle(s)
    try:
        q, ph, gr = np.zeros(4 * 35, np.float32), np.zeros(35, np.int32), np.zeros(35, np.int32)
        assert lib.ze_synthesize(h, q.ctypes.data, ph.ctypes.data, gr.ctypes.data, 35) == 0
        again, _ = _solver()
        want = again.synthesize(toy_rows=5, toy_cols=7, toy_grains=3, toy_height=8, toy_width=8)
        assert np.array_equal(q.reshape(5, 7, 4), want["quaternions"]) and np.array_equal(gr.reshape(5, 7), want["grain"])
        assert lib.ze_synthesize(h, q.ctypes.data, ph.ctypes.data, gr.ctypes.data, 34) < 0
        buf = ctypes.create_string_buffer(256)
        k = lib.ze_error(h, buf, 256)
        assert b"BadLength" in buf.raw[:k]
    finally:
        Z._handles.pop(h, None)
    none, _ = _solver(0)
    with pytest.raises(ze.Error, match="NoPhases"):
        none.synthesize()
