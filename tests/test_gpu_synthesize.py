"""A toy scan (Solver.synthesize: grains, a detector, Poisson counting over the engine's own
simulation) indexed back to the orientations it was made from."""
import tempfile

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def test_a_toy_scan_indexes_to_its_truth():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import zebsdsolve_b200 as ze
    from zebsdsolve_b200 import synthetic as syn
    from zebsdsolve_b200.master import write_npz

    d = tempfile.mkdtemp()
    cell = {"a_angstrom": 3.52, "b_angstrom": 3.52, "c_angstrom": 3.52, "alpha_deg": 90, "beta_deg": 90,
            "gamma_deg": 90}
    write_npz(f"{d}/m.npz", syn.master_sheets(3, side=201, lmax=48, group="432", device="cuda"), 201,
              syn.group_matrices("432"), 30, meta={"cell": cell, "space_group": 225})
    s = ze.Solver()
    s.configure(bandwidth=32)
    s.add_phase(f"{d}/m.npz")
    s.set_geometry(pc=(0.48, 0.31, 0.6), sample_tilt_deg=70, detector_tilt_deg=0)
    got = s.synthesize(toy_rows=8, toy_cols=10, toy_grains=4, toy_counts=200)
    assert (s.scan["rows"], s.scan["cols"], s.scan["pattern_shape"]) == (8, 10, (60, 60))
    assert abs(float(s._e.patterns.mean()) - 200) < 2  # the mean count
    r = s.index()
    dis = np.degrees(s.disorientation(r["quaternions"].reshape(-1, 4), got["quaternions"].reshape(-1, 4)))
    assert np.median(dis) < 1.0
