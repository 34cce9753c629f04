"""Host-side logic on the CPU: the C-ABI library's exports, the settings keyword set (the
reference's settings.zig tests restated), rotations and symmetry against the oracle, the master
loader, and the synthetic master's symmetry."""
import ctypes
import math
import re
import tempfile
from pathlib import Path

import numpy as np
import pytest

import oracle.master as om
import oracle.sym as osym
from zebsdsolve_b200 import master as M
from zebsdsolve_b200 import rotations as R
from zebsdsolve_b200 import settings as S
from zebsdsolve_b200 import synthetic as syn

ROOT = Path(__file__).resolve().parent.parent


def header_symbols():
    text = (ROOT / "include" / "zebsdsolve_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(zeb_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib_path = ROOT / "zebsdsolve_b200" / "libzebsdsolve_b200.so"
    if not lib_path.exists():
        from zebsdsolve_b200 import build

        build.build()
    lib = ctypes.CDLL(str(lib_path))
    names = header_symbols()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
    from zebsdsolve_b200 import _native

    assert sorted(_native.symbols()) == names
    lib.zeb_version.restype = ctypes.c_char_p
    assert lib.zeb_version() == b"0.2.8"


def test_argument_checks_fail_with_a_message_without_a_gpu():
    # a bad argument is refused before any launch: no device is touched
    from zebsdsolve_b200 import _native

    with pytest.raises(_native.NativeError, match="gauss_legendre"):
        _native.call("zeb_gauss_legendre", 0, None, None, None)


def test_settings_apply_like_the_reference():
    # settings.zig:493-509
    s = S.Settings()
    s.apply('{"bandwidth":88,"clahe":true,"method":"dictionary","static_background":"file","binning":2.5}')
    assert s["bandwidth"] == 88 and s["clahe"] and s["method"] == "dictionary" and s["static_background"] == "file"
    assert s["binning"] == 2.5
    with pytest.raises(S.SettingsError, match="InvalidEnumTag"):
        s.apply({"full_resolution": "all"})
    with pytest.raises(S.SettingsError, match="UnknownSetting"):
        s.apply({"nope": 1})
    with pytest.raises(S.SettingsError, match="BadSetting"):
        s.apply({"bandwidth": 4, "binning": 2})
    assert s["binning"] == 2.5
    assert '"method": "dictionary"' in s.to_json()


def test_sweeps_climb_to_the_final_bandwidth():
    # settings.zig:511-519
    s = S.Settings()
    s.apply({"sweeps": 3, "sweep_bandwidth": 32, "bandwidth": 128, "sweep_dict_grid": 10, "dict_grid": 40})
    assert [s.sweep(i)[0] for i in range(3)] == [32, 64, 128]
    assert s.sweep(1)[1] == 20
    s.apply({"sweeps": 1})
    assert s.sweep(0)[0] == 128
    # test_api.py:282: sweeps=3 from 16 to 64
    s.apply({"sweeps": 3, "sweep_bandwidth": 16, "bandwidth": 64})
    assert [s.sweep(i)[0] for i in range(3)] == [16, 32, 64]


def test_every_reference_setting_has_its_default():
    # every field of settings.zig:34-402 with its default (a sample of each kind)
    d = S.DEFAULTS
    assert d["bandwidth"] == 64 and d["batch"] == 256 and d["refine_iters"] == 8 and d["refine_step"] == 2.0
    assert d["accept_z"] == 15.0 and d["accept_step_deg"] == 0.2 and d["nmi_bins"] == 16
    assert d["static_background"] == "average" and d["dynamic_background"] == "subtract" and d["dynamic_sigma"] == 0.15
    assert d["mask"] is True and d["master_smooth"] == 0.3 and d["wg_fft"] == 64
    # tile_mb: a speed-only option whose default here is the reference's largest valid value
    assert d["tile_mb"] == 8192
    assert len(d) == 107 + 1  # the reference's 107 keys and this engine's `precision`


def test_fz_and_disorientation_match_oracle():
    rng = np.random.default_rng(3)
    q = syn.uniform_quaternions(rng, 50)
    p = syn.uniform_quaternions(rng, 50)
    for kind in ("o", "d6", "t", "c2"):
        ops = R.group(kind)
        assert np.allclose(R.group(kind), osym.operators(kind))
        fz = R.to_fz(q, ops)
        for i in range(50):
            assert np.allclose(fz[i], osym.to_fz(q[i], ops))
        assert np.allclose(R.disorientation(q, p, ops), osym.disorientation(q, p, ops))
    # in the cubic zone: w ≥ cos(62.8°/2) (test_api.py:215)
    assert (R.to_fz(q, R.group("o"))[:, 0] >= math.cos(math.radians(62.81) / 2) - 1e-4).all()


def test_bunge_round_trip():
    rng = np.random.default_rng(4)
    q = syn.uniform_quaternions(rng, 20)
    from oracle import rot as orot

    e = R.to_bunge(q)
    for i in range(20):
        assert np.allclose(e[i], orot.to_bunge(q[i]), atol=1e-9)
        assert abs(abs(np.dot(orot.from_bunge(e[i]), q[i])) - 1) < 1e-12


def test_master_npz_round_trip_and_symmetry():
    sheets = syn.master_sheets(5, side=101, lmax=20, group="432")
    d = tempfile.mkdtemp()
    M.write_npz(f"{d}/m.npz", sheets, 101, syn.group_matrices("432"), 30)
    m = M.load_npz(f"{d}/m.npz")
    assert m.side == 101 and m.name == "m"
    assert np.abs(m.raw - sheets.reshape(-1)).max() < 1e-5
    assert m.setting.rotation == "o" and len(m.rotations()) == 24 and m.laue == "o"
    # the oracle's loader reads the same file to the same sheets and group
    mo = om.load_ebsdsim(f"{d}/m.npz")
    assert np.abs(mo.raw - m.raw).max() < 1e-6
    assert len(mo.rotations()) == 24


def test_hexagonal_master_is_reduced_by_622():
    sheets = syn.master_sheets(6, side=101, lmax=20, group="622")
    d = tempfile.mkdtemp()
    M.write_npz(f"{d}/h.npz", sheets, 101, syn.group_matrices("622"), 24)
    m = M.load_npz(f"{d}/h.npz")
    assert m.setting.rotation == "d6" and len(m.rotations()) == 12


def test_reference_masters_load_when_present():
    # master.zig:811-850 on the reference's own test data (read as plain arrays)
    from conftest import testdata

    ni, gan = testdata("nickel", "Ni_master_20kV.npz"), testdata("gan", "GaN_master_20kV.npz")
    if ni is None or gan is None:
        pytest.skip("the reference's test data is not here (tests/golden/copy_testdata.sh)")
    m = M.load_npz(ni)
    assert m.side == 501 and m.point_group == 32 and m.laue == "o" and len(m.ops) == 48 and len(m.rotations()) == 24
    assert abs(float(m.raw.astype(np.float64).mean())) < 1e-4 and abs(float((m.raw.astype(np.float64) ** 2).mean()) - 1) < 1e-3
    g = M.load_npz(gan)
    assert g.setting.rotation == "c6" and g.setting.laue == "d6" and len(g.rotations()) == 6 and len(g.ops) == 12


def test_atan01_polynomial_error_bound():
    """The detector kernels' atan on [0, 1] (an 8-term odd polynomial in csrc/common.cuh), evaluated
    by Horner in float32 as the kernels do: within 1.5e-7 of atan everywhere on the interval."""
    import re
    from pathlib import Path

    src = (Path(__file__).resolve().parents[1] / "zebsdsolve_b200" / "csrc" / "common.cuh").read_text()
    body = src[src.index("float atan01(float t)"):src.index("return t * p;")]
    cs = [float(x.rstrip("f")) for x in re.findall(r"(-?\d\.\d+e[-+]\d+)f", body)]
    assert len(cs) == 8
    x = np.linspace(0, 1, 1_000_001).astype(np.float32)
    t2 = x * x
    p = np.float32(cs[0])
    for c in cs[1:]:
        p = (p * t2 + np.float32(c)).astype(np.float32)
    err = np.abs((x * p).astype(np.float64) - np.arctan(x.astype(np.float64)))
    assert err.max() < 1.5e-7, err.max()


@pytest.mark.parametrize("factor", [2.0, 3.0, 2.5, 1.75])
def test_host_reduction_matches_oracle(factor):
    """The static background's host reduction equals the oracle's restatement of reduce.zig."""
    import oracle.prep as op
    from zebsdsolve_b200.reduce import reduce_image, reduced_shape

    img = np.random.default_rng(3).random((61, 47)) * 100
    assert reduced_shape(61, 47, factor) == op.reduced_shape(61, 47, factor)
    assert np.abs(reduce_image(img, factor) - op.reduce(img, factor)).max() < 1e-12
