"""The multi-GPU path's host side on CPU: two gloo ranks share a scan's cells (contiguous ranges),
each "indexes" its own with a stand-in for the device work, and rank 0 assembles the whole map;
the slowest rank's time is the job's."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from zebsdsolve_b200 import shard  # noqa: E402


def test_cell_ranges_cover_the_region_once():
    for n in (0, 1, 7, 100, 101):
        for world in (1, 2, 3, 8):
            got = [shard.cell_range(n, r, world) for r in range(world)]
            assert got[0][0] == 0 and got[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(got, got[1:]))
            sizes = [hi - lo for lo, hi in got]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard.cell_range(10, 2, 2)


class _FakeEngine:
    def __init__(self, rows, cols):
        n = rows * cols
        self.rows, self.cols = rows, cols
        self.res = {"quat": np.zeros((n, 4), np.float32), "euler": np.zeros((n, 3), np.float32),
                    "ncc": np.zeros(n, np.float32), "nmi": np.zeros(n, np.float32),
                    "phase": np.full(n, -1, np.int32), "z": np.zeros(n, np.float32),
                    "sweep": np.full(n, -1, np.int32), "settled": np.zeros(n, bool)}

    def region_cells(self):
        # a region of interest: rows 1 … rows − 2 of the map
        return (np.arange(1, self.rows - 1)[:, None] * self.cols + np.arange(self.cols)[None, :]).reshape(-1)


class _FakeSolver:
    def __init__(self, rows, cols):
        self._e = _FakeEngine(rows, cols)

    def results(self):
        return {k: v.copy() for k, v in self._e.res.items()}


def _expected(cells):
    c = np.asarray(cells, np.float32)
    return {"quat": np.stack([c, c + 1, c + 2, c + 3], 1), "euler": np.stack([c, -c, 2 * c], 1),
            "ncc": c / 100, "nmi": c / 200, "phase": (np.asarray(cells) % 2).astype(np.int32), "z": c * 3,
            "sweep": np.zeros(len(cells), np.int32), "settled": np.ones(len(cells), bool)}


def _worker(rank, world, port, out):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        s = _FakeSolver(9, 7)
        seen = []

        def run(cells):
            seen.append(np.asarray(cells))
            return _expected(cells)

        r = shard.index_sharded(s, dist, run=run)
        slowest = shard.max_over_ranks(10.0 + rank, dist)
        if rank == 0:
            region = s._e.region_cells()
            exp = _expected(region)
            ok = all(np.array_equal(r[k][region], exp[k]) for k in exp)
            # cells outside the region are untouched
            outside = np.setdiff1d(np.arange(63), region)
            ok = ok and (r["phase"][outside] == -1).all()
            np.save(out, np.array([ok, slowest, len(seen[0])], dtype=np.float64))
        else:
            assert r is None
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_assemble_the_map(tmp_path):
    import torch.multiprocessing as mp

    out = str(tmp_path / "rank0.npy")
    mp.spawn(_worker, args=(2, _free_port(), out), nprocs=2, join=True)
    ok, slowest, mine = np.load(out)
    assert ok == 1.0
    assert slowest == 11.0  # the max over the ranks
    assert mine == 25  # 7 × 7 region cells split 25 / 24: rank 0 takes 25


# ── the real engine on two ranks (one GPU: each rank's kernels are its own; the ranks meet only
# on the host, in gloo collectives) ──

def _engine_worker(rank, world, port, out, path):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        s = _scan_solver(path)
        r = shard.index_sharded(s, dist)  # the default run(): the engine's sweeps over this rank's cells
        if rank == 0:
            single = _scan_solver(path).index()  # the same scan on one rank
            np.savez(out, **{f"s_{k}": v for k, v in r.items()}, **{f"o_{k}": v for k, v in single.items()})
        else:
            assert r is None
    finally:
        dist.destroy_process_group()


def _scan_solver(path):
    import zebsdsolve_b200 as ze
    from zebsdsolve_b200 import synthetic as syn

    s = ze.Solver()
    s.configure(bandwidth=32, precision="bf16")
    s.add_phase(path)
    rows, cols = 9, 13
    s.set_patterns(np.zeros((rows, cols, 60, 60), np.uint16))
    s.set_geometry(pc=(0.5, 0.3, 0.6), sample_tilt_deg=70, detector_tilt_deg=0)
    q, _ = syn.grain_map(np.random.default_rng(8), rows, cols, 7, 0.5)
    sims = s._e.simulate_device(0, np.arange(rows * cols), q)
    s.set_patterns(syn.counted_patterns(sims, seed=3).cpu().numpy().reshape(rows, cols, 60, 60))
    return s


@pytest.mark.gpu
def test_index_sharded_on_two_ranks_equals_one_rank(tmp_path):
    """shard.index_sharded with its default run() on two ranks: each rank's own chance calibration
    (from the same region lattice), sweeps, acceptance and landing over its contiguous share; rank 0
    assembles the map. Every result field equals a one-rank Solver.index of the same scan."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import tempfile

    import torch.multiprocessing as mp
    from zebsdsolve_b200 import synthetic as syn
    from zebsdsolve_b200.master import write_npz

    d = tempfile.mkdtemp()
    sheets = syn.master_sheets(4, side=201, lmax=48, group="432")
    write_npz(f"{d}/m.npz", sheets, 201, syn.group_matrices("432"), 30)
    out = str(tmp_path / "rank0.npz")
    mp.spawn(_engine_worker, args=(2, _free_port(), out, f"{d}/m.npz"), nprocs=2, join=True)
    z = np.load(out)
    for k in ("quaternions", "euler", "ncc", "nmi", "phase", "z", "sweep"):
        assert np.array_equal(z[f"s_{k}"], z[f"o_{k}"]), k
    assert (z["s_phase"] >= 0).all()


def test_bench_gpus_n_runs_n_ranks():
    """`bench.py --gpus 2` run directly re-executes itself under torch.distributed.run; rank 0 alone
    prints the line (the reference arm: no GPU needed) with n_gpus 2, and the job exits 0."""
    import json
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    p = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "1"], capture_output=True, text=True, timeout=900, env=env)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [json.loads(l) for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1 and lines[0]["n_gpus"] == 2 and lines[0]["impl"] == "reference"
