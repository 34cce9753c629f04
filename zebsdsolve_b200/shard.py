"""One scan over several GPUs: one process per GPU (torch.distributed, NCCL or gloo), each
indexing a contiguous range of the region's cells on its own device. Patterns are independent and
every table is read-only, so nothing is exchanged on the data path; the records of the cells (a
few dozen bytes each) gather to rank 0 in one collective at the end, where the full results are
assembled. The reference runs one engine per device and has no multi-device path; this is the
sharding its per-cell independence allows.

    torchrun --nproc-per-node 8 my_script.py      # in my_script.py:
    dist.init_process_group("nccl"); torch.cuda.set_device(local_rank)
    s = ze.Solver(); ...; s.set_patterns(scan)    # every rank holds the scan (or its own part)
    r = shard.index_sharded(s, dist)              # rank 0: the whole map's results; others: None
"""
import numpy as np

# the per-cell results a rank hands to rank 0 (Engine.res keys)
FIELDS = ("quat", "euler", "ncc", "nmi", "phase", "z", "sweep", "settled")


def cell_range(n, rank, world):
    """The contiguous cells [lo, hi) of rank `rank` among `world`: sizes differ by at most one."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of {world}")
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def gather_cells(local, cells, n_total, dist=None, dst=0):
    """Per-cell arrays of this rank's cells (`local`: name → array whose first axis runs over
    `cells`) assembled on rank `dst` into arrays over all n_total cells; None elsewhere. One
    gather of Python objects (the records are small); without a process group, the local arrays
    are placed and returned."""
    part = (np.asarray(cells, np.int64), {k: np.asarray(v) for k, v in local.items()})
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        parts = [part]
    else:
        rank = dist.get_rank()
        parts = [None] * dist.get_world_size() if rank == dst else None
        dist.gather_object(part, parts, dst=dst)
        if rank != dst:
            return None
    out = {}
    for c, arrs in parts:
        for k, v in arrs.items():
            if k not in out:
                out[k] = np.zeros((n_total,) + v.shape[1:], v.dtype)
            out[k][c] = v
    return out


def max_over_ranks(value, dist=None, device=None):
    """The largest of the ranks' values (a timing: the job ends with its slowest rank)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def index_sharded(solver, dist=None, run=None):
    """Index the solver's region with this rank's share of its cells, then assemble every rank's
    results on rank 0 (returned as Solver.results() would; None on the other ranks). `run(cells)`
    indexes the given cells and returns their per-cell arrays; by default the solver's engine
    runs its sweeps over them (the pipelined path of Solver.index)."""
    e = solver._e
    region = e.region_cells()
    world = dist.get_world_size() if dist is not None and dist.is_initialized() else 1
    rank = dist.get_rank() if world > 1 else 0
    lo, hi = cell_range(len(region), rank, world)
    mine = region[lo:hi]
    if run is None:
        def run(cells):
            e.index_begin()
            e.index_cells_list = np.asarray(cells, np.int64)
            e.index_region = len(cells)
            e.index_run()
            return {k: e.res[k][cells] for k in FIELDS}
    local = run(mine)
    full = gather_cells(local, mine, e.res["quat"].shape[0], dist)
    if full is None:
        return None
    for k, v in full.items():
        e.res[k][region] = v[region]
    return solver.results()
