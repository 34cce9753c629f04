"""The engine's host-side fast paths against their general forms, on the CPU (no device): a run of
consecutive cells' items from its rows' and columns' positions (the beam's travel is separable,
geometry.zig:184-192) equal positions64's, with the same bounding box; a first sweep's pass landed
as slices of the result arrays equals the scattered landing (engine.zig:2392-2419)."""
import numpy as np
import pytest

from zebsdsolve_b200 import engine as E
from zebsdsolve_b200.settings import Settings


def _engine(rows=37, cols=53, px=70.0):
    e = E.Engine.__new__(E.Engine)  # the host logic alone: no device is opened
    e.set = Settings()
    e.geo = E.Geometry()
    e.geo.px_um, e.geo.step_x_um, e.geo.step_y_um = px, 1.7, 2.3
    e.geo.pc = np.array([0.48, 0.31, 0.62])
    e._full = False
    e.patterns = np.zeros((rows, cols, 1, 1), np.uint16)
    e.info = lambda: (rows, cols, 60, 60)
    e.factor = lambda: 1.0
    e.pattern_shape = lambda: (60, 60)
    e.to_device = lambda name, arr: arr
    return e


@pytest.mark.parametrize("signs", [(1, 1), (-1, 1), (1, -1)])
@pytest.mark.parametrize("px", [70.0, 0.0])
def test_items_of_a_run_from_rows_and_columns(signs, px):
    e = _engine(px=px)
    e.set.apply({"scan_x_sign": signs[0], "scan_y_sign": signs[1]})
    runs = [np.arange(37 * 53), np.arange(100, 140), np.arange(50, 60), np.arange(45, 100), np.arange(0, 1),
            np.arange(530, 1700), np.arange(52, 54)]
    for cells in runs:
        got = e.items_of(cells)
        box = e._batch_t
        t = e.positions(cells)
        want = np.concatenate([t, np.arange(len(cells), dtype=np.float32)[:, None]], 1)
        assert np.array_equal(got, want), (len(cells), cells[0])
        assert np.array_equal(box[0], t.min(0)) and np.array_equal(box[1], t.max(0))
        assert box[0].dtype == np.float32
    # scattered cells take the general path
    cells = np.array([7, 3, 900, 41])
    assert np.array_equal(e.items_of(cells)[:, :3], e.positions(cells))


def _landing_engine(n=50):
    e = E.Engine.__new__(E.Engine)
    e.set = Settings()
    e.res = {"quat": np.zeros((n, 4), np.float32), "euler": np.zeros((n, 3), np.float32),
             "ncc": np.zeros(n, np.float32), "nmi": np.zeros(n, np.float32), "z": np.zeros(n, np.float32),
             "phase": np.full(n, -1, np.int32), "sweep": np.full(n, -1, np.int32), "settled": np.zeros(n, bool)}
    e.index_sweep, e.index_accepted, e.index_done = 0, 0, 0
    e.index_cells_list = np.arange(n)
    e.events = []
    e.phases = []
    return e


def test_a_first_sweep_pass_lands_as_slices():
    rng = np.random.default_rng(0)
    recs = rng.random((2, 20, 8)).astype(np.float32)
    recs[..., 6] *= 0.002  # last improving steps around the settle bound
    recs[..., 7] = rng.normal(15, 3, (2, 20))  # z around the acceptance bound
    fz = rng.random((2, 20, 4)).astype(np.float32)
    bg = rng.random((2, 20, 3)).astype(np.float32)
    cells = np.arange(10, 30)
    fast = _landing_engine()
    fast.land(cells, recs, fz, bg)  # every cell new: the slice path
    slow = _landing_engine()
    slow.res["phase"][0] = 0  # (a cell outside the pass, so that nothing else differs)
    slow.land(cells[::-1].copy(), recs[:, ::-1].copy(), fz[:, ::-1].copy(), bg[:, ::-1].copy())  # scattered order
    for k in fast.res:
        assert np.array_equal(fast.res[k][10:30], slow.res[k][10:30]), k
    assert fast.index_accepted == slow.index_accepted and fast.index_done == slow.index_done == 20
