"""The reference's own C ABI on the GPU: a scan driven through libzebsdsolve.so's ze_* calls (with
the reference's argument types and structs, as python/zebsdsolve/_native.py binds them) gives what
the package's Python API gives on the same patterns, bit for bit: the results of every kind after
the index_begin / index_step loop, index_cells, chance, a pattern, the .ang text, the phase and
scan descriptions, the geometry round trip; failures come back as negative codes with ze_error's
message, which one read clears."""
import ctypes
import json
import tempfile

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

P, SZ, U32, U64, I32, I64, F64 = (ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint32, ctypes.c_uint64,
                                  ctypes.c_int32, ctypes.c_int64, ctypes.c_double)


def _bind():
    from zebsdsolve_b200 import build, ze_abi as Z

    lib = ctypes.CDLL(str(build.build_abi()))
    sigs = {
        "ze_create": ([ctypes.c_char_p], P), "ze_destroy": ([P], None), "ze_error": ([P, ctypes.c_char_p, SZ], SZ),
        "ze_configure": ([P, ctypes.c_char_p, SZ], I32), "ze_settings": ([P, ctypes.c_char_p, SZ], SZ),
        "ze_set_patterns": ([P, P, SZ, U32, U32, U32, U32, U32], I32),
        "ze_set_geometry": ([P, ctypes.POINTER(Z.Geometry)], None),
        "ze_get_geometry": ([P, ctypes.POINTER(Z.Geometry)], None),
        "ze_add_phase": ([P, ctypes.c_char_p, SZ], I32), "ze_phase_count": ([P], U32),
        "ze_phase_info": ([P, U32, ctypes.POINTER(Z.PhaseInfo)], I32),
        "ze_scan_info": ([P, ctypes.POINTER(Z.ScanInfo)], None), "ze_scan_format": ([P, ctypes.c_char_p, SZ], SZ),
        "ze_index_begin": ([P], I32), "ze_index_step": ([P], I64),
        "ze_index_status": ([P, ctypes.POINTER(Z.IndexStatus)], None),
        "ze_results": ([P, U32, P, SZ], I64), "ze_index_cells": ([P, P, SZ, P, SZ], I32),
        "ze_chance": ([P, U32, P], I32), "ze_pattern_shape": ([P, U32, P], I32),
        "ze_pattern": ([P, U64, U32, U32, P, SZ], I32), "ze_export": ([P, U32, P, SZ], I64),
        "ze_reduce": ([P, U32, P, P], None), "ze_events": ([P, ctypes.c_char_p, SZ], SZ),
        "ze_sim_run": ([P, P], I32),
    }
    for name, (args, res) in sigs.items():
        fn = getattr(lib, name)
        fn.argtypes, fn.restype = args, res
    return lib, Z


@pytest.fixture(scope="module")
def world():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import zebsdsolve_b200 as ze
    from zebsdsolve_b200 import synthetic as syn
    from zebsdsolve_b200.master import write_npz

    d = tempfile.mkdtemp()
    paths = []
    keys = ("a_angstrom", "b_angstrom", "c_angstrom", "alpha_deg", "beta_deg", "gamma_deg")
    cells = {"432": ([3.52] * 3 + [90.0] * 3, 225), "622": ([3.19, 3.19, 5.19, 90.0, 90.0, 120.0], 186)}
    for g, seed in (("432", 3), ("622", 4)):
        sheets = syn.master_sheets(seed, side=201, lmax=48, group=g, device="cuda")
        write_npz(f"{d}/m{g}.npz", sheets, 201, syn.group_matrices(g), syn.POINT_GROUP[g],
                  meta={"cell": dict(zip(keys, cells[g][0])), "space_group": cells[g][1]})
        paths.append(f"{d}/m{g}.npz")
    rows, cols = 8, 12
    s = ze.Solver()
    s.configure(bandwidth=32)
    s.add_phase(paths[0])
    s.set_patterns(np.zeros((rows, cols, 60, 60), np.uint16))
    s.set_geometry(pc=(0.5, 0.3, 0.6), sample_tilt_deg=70, detector_tilt_deg=0)
    q, _ = syn.grain_map(np.random.default_rng(21), rows, cols, 6, 0.5)
    sims = s.simulate(q, cells=np.arange(rows * cols))
    pats = syn.counted_patterns(torch.as_tensor(sims, device="cuda"), seed=5).cpu().numpy()
    return {"paths": paths, "pats": np.ascontiguousarray(pats.reshape(rows, cols, 60, 60)), "q": q}


def _err(lib, h):
    buf = ctypes.create_string_buffer(1024)
    n = lib.ze_error(h, buf, 1024)
    return buf.raw[:n].decode()


def test_a_scan_through_the_c_abi_matches_the_python_api(world):
    import zebsdsolve_b200 as ze

    lib, Z = _bind()
    pats = world["pats"]
    rows, cols, h, w = pats.shape
    settings = {"bandwidth": 32, "sweeps": 1}

    # the package's Python API
    s = ze.Solver()
    s.configure(**settings)
    for p in world["paths"]:
        s.add_phase(p)
    s.set_patterns(pats)
    s.set_geometry(pc=(0.5, 0.3, 0.6), sample_tilt_deg=70, detector_tilt_deg=0)
    s.index_begin()
    while s.index_step() > 0:
        pass
    want = s.results()

    # the same through the C ABI
    e = lib.ze_create(b"")
    assert e, "ze_create"
    j = json.dumps(settings).encode()
    assert lib.ze_configure(e, j, len(j)) == 0
    for k, p in enumerate(world["paths"]):
        assert lib.ze_add_phase(e, p.encode(), len(p)) == k
    assert lib.ze_phase_count(e) == 2
    buf = pats.copy()  # the engine copies: the caller's buffer may go once set_patterns returns
    assert lib.ze_set_patterns(e, buf.ctypes.data, buf.nbytes, 1, rows, cols, h, w) == 0
    buf[:] = 0
    g = Z.Geometry()
    lib.ze_get_geometry(e, ctypes.byref(g))
    g.pc[:] = (0.5, 0.3, 0.6)
    g.sample_tilt_deg, g.detector_tilt_deg = 70.0, 0.0
    lib.ze_set_geometry(e, ctypes.byref(g))
    assert _err(lib, e) == ""
    g2 = Z.Geometry()
    lib.ze_get_geometry(e, ctypes.byref(g2))
    assert list(g2.pc) == [0.5, 0.3, 0.6] and g2.px_um == s.geometry["px_um"]

    assert lib.ze_index_begin(e) == 0
    steps = 0
    while True:
        left = lib.ze_index_step(e)
        assert left >= 0, _err(lib, e)
        steps += 1
        if left == 0:
            break
    st = Z.IndexStatus()
    lib.ze_index_status(e, ctypes.byref(st))
    assert (st.region, st.done, st.sweeps, st.bandwidth, st.method) == (rows * cols, rows * cols, 1, 32, 0)

    n = rows * cols
    for kind, key, dt, k in ((0, "quaternions", np.float32, 4), (1, "ncc", np.float32, 1), (2, "nmi", np.float32, 1),
                             (3, "phase", np.int32, 1), (4, "euler", np.float32, 3), (5, "z", np.float32, 1),
                             (6, "sweep", np.int32, 1)):
        a = np.empty(n * k, dt)
        assert lib.ze_results(e, kind, a.ctypes.data, a.nbytes) == n * k, kind
        assert np.array_equal(a.reshape(want[key].shape), want[key]), key
    small = np.empty(4, np.float32)
    assert lib.ze_results(e, 0, small.ctypes.data, small.nbytes) < 0
    assert "BufferTooSmall" in _err(lib, e) and _err(lib, e) == ""

    # index_cells, chance, a pattern, the export
    cells = np.array([5, 17, 40, 95], np.uint64)
    rec = np.empty(2 * len(cells) * 8, np.float32)
    assert lib.ze_index_cells(e, cells.ctypes.data, len(cells), rec.ctypes.data, rec.size) == 0
    r = s.index_cells(cells.astype(np.int64))
    got = rec.reshape(2, len(cells), 8)
    assert np.array_equal(got[..., :4], r["quaternions"]) and np.array_equal(got[..., 4], r["ncc"])
    ch = np.empty(2, np.float32)
    assert lib.ze_chance(e, 1, ch.ctypes.data) == 0
    assert tuple(map(float, ch)) == s.chance(1)
    shp = np.empty(2, np.uint32)
    assert lib.ze_pattern_shape(e, 0, shp.ctypes.data) == 0 and tuple(shp) == (h, w)
    pt = np.empty(h * w, np.float32)
    assert lib.ze_pattern(e, 17, 1, 0, pt.ctypes.data, pt.size) == 0
    assert np.array_equal(pt.reshape(h, w), s.pattern(17))
    size = lib.ze_export(e, 0, None, 0)
    assert size > 0, _err(lib, e)
    text = ctypes.create_string_buffer(size)
    assert lib.ze_export(e, 0, text, size) == size
    assert text.raw[:size].decode() == s.export_text("ang")

    # descriptions and the orientation helpers
    pi = Z.PhaseInfo()
    assert lib.ze_phase_info(e, 1, ctypes.byref(pi)) == 0
    assert (pi.side, pi.point_group, pi.laue) == (201, s.phases[1]["point_group"], 9)
    si = Z.ScanInfo()
    lib.ze_scan_info(e, ctypes.byref(si))
    assert (si.rows, si.cols, si.pat_h, si.pat_w, si.pixel, si.format) == (rows, cols, h, w, 1, 100)
    fb = ctypes.create_string_buffer(64)
    k = lib.ze_scan_format(e, fb, 64)
    assert fb.raw[:k] == b"memory"
    qz = want["quaternions"].reshape(-1, 4)[3].copy()
    eu = np.empty(3, np.float64)
    lib.ze_reduce(e, 0, qz.ctypes.data, eu.ctypes.data)
    q_want, e_want = s.reduce(want["quaternions"].reshape(-1, 4)[3:4], 0)
    assert np.array_equal(qz, q_want[0]) and np.allclose(eu, e_want[0], atol=1e-12)

    # settings as JSON; a refused setting and a part this engine does not build
    sb = ctypes.create_string_buffer(1 << 16)
    k = lib.ze_settings(e, sb, len(sb))
    assert json.loads(sb.raw[:k])["bandwidth"] == 32
    bad = b'{"bandwidth": "wide"}'
    assert lib.ze_configure(e, bad, len(bad)) < 0
    assert _err(lib, e).startswith("configure") and _err(lib, e) == ""
    assert lib.ze_sim_run(e, None) < 0 and "not part of this engine" in _err(lib, e)
    eb = ctypes.create_string_buffer(1 << 16)
    k = lib.ze_events(e, eb, len(eb))
    kinds = {json.loads(x)["kind"] for x in eb.raw[:k].decode().splitlines() if x}
    assert "log" in kinds
    lib.ze_destroy(e)
