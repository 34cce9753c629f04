"""Failure detection on the GPU without a GPU fault, and the master bake against the oracle.

* The batch stamp (engine.zig:2127-2132): a readback dropped by the host-side injection hook
  (Engine.pending_skip) is caught as DeviceSkippedBatch, and the next batch lands normally.
* The tensor-core kernels' bounded waits: zeb_set_test_stall makes each tcgen05 kernel's MMA
  thread wait on an mbarrier that nothing arrives at; the kernel gives up within the short limit,
  sets its status word, drains what it issued, frees its tensor memory and returns, the host's
  check raises DeviceTimeout, and the context stays usable (the same call then gives the clean
  result). Covered: the spectrum in FP32 (bf16x3) and FP16 (bf16) storage, the tensor-core
  transform along a, and the dictionary match (pca).
* The master bake (engine.zig:1718-1788; mastersph.wgsl:87-138): the device's smoothing on the
  sphere and tangent gradient of a 401² sheet pair against the oracle's sphere_blur and
  gradient_table.
"""
import tempfile

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def solver():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import zebsdsolve_b200 as ze
    from zebsdsolve_b200 import synthetic as syn
    from zebsdsolve_b200.master import write_npz

    sheets = syn.master_sheets(6, side=201, lmax=48, group="432", device="cuda")
    d = tempfile.mkdtemp()
    write_npz(f"{d}/m.npz", sheets, 201, syn.group_matrices("432"), 30)
    s = ze.Solver()
    s.configure(bandwidth=32)
    s.add_phase(f"{d}/m.npz")
    rows, cols = 6, 10
    s.set_patterns(np.zeros((rows, cols, 60, 60), np.uint16))
    s.set_geometry(pc=(0.5, 0.3, 0.6), sample_tilt_deg=70, detector_tilt_deg=0)
    q = syn.uniform_quaternions(np.random.default_rng(12), rows * cols)
    sims = s._e.simulate_device(0, np.arange(rows * cols), q)
    s.set_patterns(syn.counted_patterns(sims, seed=2).cpu().numpy().reshape(rows, cols, 60, 60))
    return s


def test_a_dropped_batch_is_caught_by_its_stamp(solver):
    import zebsdsolve_b200 as ze

    cells = np.arange(24)
    clean = solver.index_cells(cells)
    solver._e.pending_skip = 1
    with pytest.raises(ze.Error, match="DeviceSkippedBatch"):
        solver.index_cells(cells)
    assert solver._e.pending_skip == 0
    again = solver.index_cells(cells)
    assert np.array_equal(again["quaternions"], clean["quaternions"])


@pytest.mark.parametrize("precision,method", [("bf16", "spherical"), ("bf16x3", "spherical"), ("bf16", "pca")])
def test_a_tensor_core_wait_that_runs_out_is_reported(solver, precision, method):
    import zebsdsolve_b200 as ze
    from zebsdsolve_b200 import _native as N

    solver.configure(precision=precision, pca_components=32, dict_grid=8)
    cells = np.arange(40)
    clean = solver.index_cells(cells, method=method)
    N.call("zeb_set_test_stall", 2_000_000)  # 2 ms
    try:
        with pytest.raises(ze.Error, match="DeviceTimeout"):
            solver.index_cells(cells, method=method)
    finally:
        N.call("zeb_set_test_stall", 0)
    # the context is intact and the status word was cleared: the same call gives the clean result
    torch.cuda.synchronize()
    again = solver.index_cells(cells, method=method)
    assert np.array_equal(again["quaternions"], clean["quaternions"])
    assert np.array_equal(again["ncc"], clean["ncc"])
    solver.configure(precision="f32")


def test_master_smoothing_and_gradient_match_the_oracle():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import ctypes

    import oracle.detector as od
    from zebsdsolve_b200 import _native as N
    from zebsdsolve_b200 import synthetic as syn
    from zebsdsolve_b200.device import master_blur

    side = 401
    raw = syn.master_sheets(2, side=side, lmax=96, group="432", device="cuda").reshape(-1)
    sigma = 1.7  # sheet pixels: two passes (σ 1.7 then the rest) of the doubling schedule
    dev = master_blur(torch.as_tensor(raw, device="cuda"), side, sigma)
    got = dev.cpu().numpy().astype(np.float64)
    want = od.sphere_blur(raw, side, sigma)
    assert np.abs(got - want).max() <= 2e-5 * np.abs(want).max(), np.abs(got - want).max()

    grad = torch.empty(got.size * 4, dtype=torch.float32, device="cuda")
    N.call("zeb_master_gradient", ctypes.c_void_p(dev.data_ptr()), ctypes.c_void_p(grad.data_ptr()), side,
           ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    g = grad.cpu().numpy().reshape(-1, 4).astype(np.float64)
    wg = od.gradient_table(got, side)  # the oracle's gradient of the same (device-smoothed) sheets
    assert np.abs(g[:, 3] - wg[:, 3]).max() == 0.0  # the value slot is the sheet itself
    scale = np.abs(wg[:, :3]).max()
    assert np.abs(g[:, :3] - wg[:, :3]).max() <= 1e-4 * scale, np.abs(g[:, :3] - wg[:, :3]).max() / scale
