"""A scan indexed from its files: an EDAX .up2 with its .ang (the map's shape, the steps and the
pattern centre in EDAX's convention) opened through Solver.open and ze.index gives what the same
patterns passed as an array with that geometry give; the results exported as .ang read back as
the stored orientations."""
import struct
import tempfile

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def test_up2_with_ang_indexes_as_the_array_does():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import zebsdsolve_b200 as ze
    from zebsdsolve_b200 import rotations as R
    from zebsdsolve_b200 import synthetic as syn
    from zebsdsolve_b200.master import write_npz

    d = tempfile.mkdtemp()
    cell = {"a_angstrom": 3.52, "b_angstrom": 3.52, "c_angstrom": 3.52, "alpha_deg": 90, "beta_deg": 90, "gamma_deg": 90}
    write_npz(f"{d}/m.npz", syn.master_sheets(3, side=201, lmax=48, group="432", device="cuda"), 201,
              syn.group_matrices("432"), 30, meta={"cell": cell, "space_group": 225})
    rows, cols, pc = 6, 9, (0.48, 0.31, 0.6)
    s = ze.Solver()
    s.configure(bandwidth=32)
    s.add_phase(f"{d}/m.npz")
    s.set_patterns(np.zeros((rows, cols, 60, 60), np.uint16))
    s.set_geometry(pc=pc, sample_tilt_deg=70, detector_tilt_deg=0)
    rng = np.random.default_rng(3)
    q, _ = syn.grain_map(rng, rows, cols, 4, 0.5)
    sims = s.simulate(q, cells=np.arange(rows * cols))
    pats = syn.counted_patterns(torch.as_tensor(sims, device="cuda"), seed=2).cpu().numpy().astype(np.uint16)
    with open(f"{d}/s.up2", "wb") as fh:
        fh.write(struct.pack("<IIII", 3, 60, 60, 42) + struct.pack("<BIIBdd", 0, cols, rows, 0, 1.5, 1.5))
        fh.write(pats.astype("<u2").tobytes())
    lines = [f"# x-star {pc[0]}", f"# y-star {1 - pc[1]}", f"# z-star {pc[2]}", "# GRID: SqrGrid", "# XSTEP: 1.5",
             "# YSTEP: 1.5", f"# NCOLS_ODD: {cols}", f"# NCOLS_EVEN: {cols}", f"# NROWS: {rows}", "# SOFTWARE: OIM"]
    lines += [f"0 0 0 {k % cols * 1.5:.5f} {k // cols * 1.5:.5f} 0 0 0 0 0" for k in range(rows * cols)]
    with open(f"{d}/s.ang", "w") as fh:
        fh.write("\n".join(lines) + "\n")
    s.open(f"{d}/s.up2", f"{d}/s.ang")
    assert s.scan["format"] == "edax_up" and (s.scan["rows"], s.scan["cols"]) == (rows, cols)
    ov, st = s.stored_overview(), s.stored_orientations()  # the .ang's image quality and orientations
    assert ov["kind"] == 2 and ov["label"] == "Image quality" and ov["values"].shape == (rows, cols)
    assert (ov["values"] == 0).all() and st["euler"].shape == (rows, cols, 3) and (st["phase"] == 0).all()
    assert np.allclose(s.geometry["pc"], pc) and s.geometry["step_x_um"] == 1.5
    r_file = s.index()
    r_arr = ze.index(pats.reshape(rows, cols, 60, 60), [f"{d}/m.npz"], pc=pc, sample_tilt_deg=70,
                     detector_tilt_deg=0, step_x_um=1.5, step_y_um=1.5, bandwidth=32)
    assert np.array_equal(r_file["quaternions"], r_arr.quaternions)
    r_api = ze.index([f"{d}/s.up2", f"{d}/s.ang"], [f"{d}/m.npz"], bandwidth=32, sample_tilt_deg=70)
    assert np.array_equal(r_api.quaternions, r_arr.quaternions)
    dis = np.degrees(s.disorientation(r_file["quaternions"].reshape(-1, 4), q))
    assert np.median(dis) < 0.5
    s.export(f"{d}/out.ang")
    data = np.loadtxt(f"{d}/out.ang", comments="#", ndmin=2)
    p1, P, p2 = data[:, 0], data[:, 1], data[:, 2]
    sig, dlt = 0.5 * (p1 + p2), 0.5 * (p1 - p2)
    qa = np.stack([np.cos(P / 2) * np.cos(sig), -np.sin(P / 2) * np.cos(dlt), -np.sin(P / 2) * np.sin(dlt),
                   -np.cos(P / 2) * np.sin(sig)], -1)
    dq = R.qmul(R.qconj(R.qstd(r_file["quaternions"].reshape(-1, 4).astype(np.float64))), R.qstd(qa))
    assert np.degrees(2 * np.arcsin(np.clip(np.linalg.norm(dq[:, 1:], axis=1), 0, 1))).max() < 1e-3
    s.export(f"{d}/out.ctf")
    with pytest.raises(ze.Error, match="not written"):
        s.export(f"{d}/out.h5oina")
