#!/usr/bin/env python
"""Throughput of the spherical indexing path (patterns/s indexed + refined) on B200.

    python bench.py [--gpus N --steps K --warmup W --precision bf16|bf16x3|f32 --patterns P]
    python bench.py --impl reference ...   # the reference's algorithm on the host cores

Workload (the precision-form configuration at scale): a 316 × 316 scan (99,856 patterns) of
60 × 60 uint16 patterns whose orientations are 200 Voronoi grains with a 0.5° Gaussian spread,
simulated from a seeded 432-symmetrised master (SH degree ≤ 96, 401² Lambert sheets) at pattern
centre (0.5, 0.3, 0.6), sample tilt 70°, with a Gaussian background and Poisson counts; indexed
at L = 64 on the 128³ Euler grid (the reference's defaults: static and dynamic background,
circular mask, 8 refinement iterations).  A step is one pass of the whole path over the whole
scan.  Inputs (720 MB) exceed L2 (126 MB), so no flush is needed between steps.

`value` times the device path with the stored patterns already resident in HBM; `e2e` times the
reference's own C ABI (libzebsdsolve.so: ze_index_begin, the ze_index_step loop, ze_results of
every kind, as the reference's Solver.index issues them) from host memory: uploads, device path,
the records' readback and the host's landing of results; `e2e_python_api` the same through this
package's Python API (Solver.index), whose results the C ABI's must equal.  With --gpus N (N > 1; run directly, the command re-executes itself
under torch.distributed.run, one process per GPU) every rank holds the same scan: `value` has each
rank index all of it (weak scaling, no collective on the data path), `e2e` shards the one scan
over the ranks (shard.index_sharded: contiguous shares, the records gathered to rank 0); both
report the max of the ranks' CUDA-event times.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

ROWS = COLS = 316
H = W = 60
L = 64
GRAINS = 200
SPREAD_DEG = 0.5
PC = (0.5, 0.3, 0.6)
WORKLOAD = ("316x316 scan of 60x60 uint16 patterns, 200 Voronoi grains (0.5 deg spread), 432 master 401^2 "
            "(SH <= 96), bandwidth 64 (128^3 Euler grid), 8 refinement iterations")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=("b200", "reference"))
    ap.add_argument("--precision", default="bf16", choices=("f32", "bf16", "bf16x3"),
                    help="the form timed as `value` and `e2e` (the plain FP32 form is timed beside it)")
    ap.add_argument("--no-fp32-form", action="store_true", help="skip the plain FP32 form's timing")
    ap.add_argument("--patterns", type=int, default=ROWS * COLS, help="scan size (cells), default 316x316")
    ap.add_argument("--batch", type=int, default=16384, help="patterns per device pass in the value measurement")
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-abi", action="store_true", help="skip the end-to-end leg through the reference's C ABI")
    ap.add_argument("--workload", default="index", choices=("index", "adjoint", "uneven", "pcfit", "plane", "large", "nickel",
                                                              "match", "target"),
                    help="index: the scan of 60x60 patterns (the headline); adjoint: six-unknown refinement "
                         "of 120x120 patterns with jittered pattern centres; uneven: many scans of uneven "
                         "lengths and detector sizes, two phases; pcfit: the pattern-centre vote at its default "
                         "settings; plane: the plane of source points (fit_plane, fit_geometry); large: 160x160 "
                         "patterns binned 2x, two sweeps L=64 then L=128, adjoint refinement, and a PCA dictionary; "
                         "nickel: the reference's real scan (kikuchipy's nickel scan, h5ebsd), one pass and two sweeps; "
                         "target: 1M patterns of 60x60 indexed and refined over six unknowns (adjoint), BF16 form "
                         "against the FP32 form")
    ap.add_argument("--large", type=int, default=1000000, help="large and target: patterns of the scan (1 000 000; "
                                                                "large: 51 GB of u16 on the host, target: 7.2 GB)")
    ap.add_argument("--scans", type=int, default=64, help="uneven: number of scans")
    ap.add_argument("--entries", type=int, default=65536, help="match: dictionary entries")
    ap.add_argument("--components", type=int, default=512, help="match: values per row (PCA components)")
    ap.add_argument("--kernel-split", action="store_true",
                    help="nickel: also the device time by kernel (torch.profiler), printed to stderr")
    ap.add_argument("--max-count", type=int, default=200000, help="uneven: the longest scan (log-uniform from 1000)")
    return ap.parse_args()


def scan_shape(n):
    if n == ROWS * COLS:
        return ROWS, COLS
    cols = int(math.ceil(math.sqrt(n)))
    return int(math.ceil(n / cols)), cols


# ── the reference's algorithm on the host (the oracle: parity and the CPU baseline) ──

ORACLE_CELLS = 1024  # the lattice of cells the oracle indexes (>= 1000, spread over the map's grains)


def oracle_scan(raw_sheets, static_bg, L_=L, refine=True, baked=None):
    """The oracle's state for the workload (FP64): the master baked for this detector, its tables
    at L_, the map-centre window's denominators, the static background given."""
    import oracle.geometry as og
    import oracle.pipeline as opl
    from zebsdsolve_b200 import synthetic as syn

    geo = og.Geometry(pc=PC, sample_tilt_deg=70.0)
    return opl.Scan(np.asarray(raw_sheets, np.float64).reshape(-1), 401, syn.group_matrices("432"), geo, H, W, L_,
                    static_bg=static_bg, refine=refine, baked=baked)


def oracle_geometry(px_um=0.0, step_um=1.0):
    """The workload's geometry in the oracle's terms (the pixel size the engine takes by default:
    the detector's 24 mm over 60 pixels; steps of 1 µm)."""
    import oracle.geometry as og

    return og.Geometry(pc=PC, sample_tilt_deg=70.0, px_um=px_um or 1000.0 * 24.0 / W, step_x_um=step_um,
                       step_y_um=step_um)


def oracle_run(scan, raws, ts=None):
    """The oracle over the stored patterns `raws` (at positions `ts`) on the host cores
    (oracle.pipeline.index_many): (records [(q in the fundamental zone, NCC, NMI)], patterns/s,
    cores, seconds)."""
    import oracle.pipeline as opl

    recs, dt, cores = opl.index_many(scan, raws, ts)
    return [(r["q"], r["ncc"], r["nmi"]) for r in recs], len(recs) / dt, cores, dt


def cpu_ref_run(scan, raws, ts=None, threads=None):
    """The C++ FP32 restatement (oracle/cpu_ref) over the stored patterns `raws` (at positions
    `ts`) on `threads` host threads (default: every core this process may use), after a few
    untimed patterns: (records [(q in the fundamental zone, NCC, NMI)], patterns/s, threads,
    seconds)."""
    import oracle.cpu_ref as ocr

    threads = threads or max(1, len(os.sched_getaffinity(0)))
    cr = ocr.CpuRef(scan)
    k = min(len(raws), threads)
    cr.index(raws[:k], None if ts is None else ts[:k], threads)
    t0 = time.perf_counter()
    recs = cr.index(raws, ts, threads)
    dt = time.perf_counter() - t0
    return [(r["q"], r["ncc"], r["nmi"]) for r in recs], len(recs) / dt, threads, dt


def parity_of(oracle_recs, rotations, q, ncc, nmi):
    """Each cell's record against the oracle's: the misorientation (degrees, modulo the group) and
    the NCC and NMI differences."""
    import oracle.sym as osym

    oq = np.array([r[0] for r in oracle_recs], np.float64)
    oncc = np.array([r[1] for r in oracle_recs])
    onmi = np.array([r[2] for r in oracle_recs])
    dis = np.degrees(osym.disorientation(np.asarray(q, np.float64).reshape(-1, 4), oq, rotations))
    dn = np.abs(np.asarray(ncc, np.float64) - oncc)
    dm = np.abs(np.asarray(nmi, np.float64) - onmi)
    return {"n": int(len(dis)), "within_0.1deg": round(float((dis <= 0.1).mean()), 5),
            "median_deg": round(float(np.median(dis)), 5), "p99_deg": round(float(np.percentile(dis, 99)), 5),
            "max_deg": round(float(dis.max()), 5), "ncc_within_1e-3": round(float((dn <= 1e-3).mean()), 5),
            "ncc_abs_max": float(f"{dn.max():.3g}"), "ncc_abs_p99": float(f"{np.percentile(dn, 99):.3g}"),
            "nmi_abs_max": float(f"{dm.max():.3g}")}


def host_workload(rank=0):
    """The workload's lattice cells made on the host, for a run without a GPU (the reference arm):
    the same master and grain map (same seeds), each cell's pattern simulated by the oracle's
    projection of the baked master and given the same noise model (Poisson counts of
    1000·(0.6 + 0.4·m)·B, NumPy's generator), at its own detector position (the engine's default
    pixel size and steps, its default scan signs −1). Returns (raws [cells][H][W] u16, scan, cells,
    positions)."""
    import oracle.detector as od
    import oracle.geometry as og
    import oracle.pipeline as opl
    from zebsdsolve_b200 import synthetic as syn

    rows, cols = ROWS, COLS
    sheets = syn.master_sheets(2, side=401, lmax=96, group="432")
    rng = np.random.default_rng(100 + rank)
    q, _ = syn.grain_map(rng, rows, cols, GRAINS, SPREAD_DEG)
    cells = opl.lattice(rows, cols, ORACLE_CELLS)
    geo = oracle_geometry()
    baked = opl.bake(sheets, 401, opl.pixel_angle(geo, H))
    frame = geo.frame()
    ts = opl.cell_positions(geo, rows, cols, cells, H, W, -1.0, -1.0)
    yy, xx = np.meshgrid(np.arange(H) + 0.5 - H / 2, np.arange(W) + 0.5 - W / 2, indexing="ij")
    B = np.exp(-(xx ** 2 + yy ** 2) / (2 * (0.4 * W) ** 2))
    B *= B.size / B.sum()
    noise = np.random.default_rng(7 + rank)
    raws = np.empty((len(cells), H, W), np.uint16)
    for k, c in enumerate(cells):
        sim = od.project(baked, 401, frame, ts[k], q[c], H, W)
        raws[k] = np.clip(noise.poisson(np.maximum(1000 * (0.6 + 0.4 * sim) * B, 0)), 0, 65535)
    # the lattice is the static background's lattice: its mean is the scan's static background
    scan = oracle_scan(sheets, raws.astype(np.float64).mean(0), baked=baked)
    return raws, scan, cells, ts


def abi_e2e(settings, master, pats, steps, warmup):
    """One scan end to end through the reference's own C ABI (zebsdsolve_b200/libzebsdsolve.so, the
    ze_* calls its Python package binds): ze_set_patterns from a host buffer once, then every step
    what the reference's Solver.index issues: ze_index_begin, ze_index_step until no cell is left,
    and ze_results of every kind into host arrays. Returns (ms per step, {kind: array})."""
    import ctypes

    import torch
    from zebsdsolve_b200 import build, ze_abi as Z

    lib = ctypes.CDLL(str(build.ABI_LIB))
    P, SZ, U32, I32, I64 = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint32, ctypes.c_int32, ctypes.c_int64
    G = ctypes.POINTER(Z.Geometry)
    for name, args, res in (("ze_create", [ctypes.c_char_p], P), ("ze_destroy", [P], None),
                            ("ze_error", [P, ctypes.c_char_p, SZ], SZ), ("ze_configure", [P, ctypes.c_char_p, SZ], I32),
                            ("ze_add_phase", [P, ctypes.c_char_p, SZ], I32),
                            ("ze_set_patterns", [P, P, SZ, U32, U32, U32, U32, U32], I32),
                            ("ze_get_geometry", [P, G], None), ("ze_set_geometry", [P, G], None),
                            ("ze_index_begin", [P], I32), ("ze_index_step", [P], I64),
                            ("ze_results", [P, U32, P, SZ], I64)):
        fn = getattr(lib, name)
        fn.argtypes, fn.restype = args, res
    h = lib.ze_create(b"")
    if not h:
        raise RuntimeError("ze_create failed")

    def ok(rc, what):
        if rc < 0:
            buf = ctypes.create_string_buffer(1024)
            k = lib.ze_error(h, buf, 1024)
            raise RuntimeError(f"{what}: {buf.raw[:k].decode()}")
        return rc

    rows, cols, hh, ww = pats.shape
    j = json.dumps(settings).encode()
    ok(lib.ze_configure(h, j, len(j)), "configure")
    ok(lib.ze_add_phase(h, master.encode(), len(master)), "add_phase")
    ok(lib.ze_set_patterns(h, pats.ctypes.data, pats.nbytes, 1, rows, cols, hh, ww), "set_patterns")
    g = Z.Geometry()
    lib.ze_get_geometry(h, ctypes.byref(g))
    g.pc[:], g.sample_tilt_deg, g.detector_tilt_deg = PC, 70.0, 0.0
    lib.ze_set_geometry(h, ctypes.byref(g))
    n = rows * cols
    outs = {kind: np.empty(n * k, dt) for kind, dt, k in ((0, np.float32, 4), (1, np.float32, 1), (2, np.float32, 1),
                                                          (3, np.int32, 1), (4, np.float32, 3), (5, np.float32, 1),
                                                          (6, np.int32, 1))}

    def run():
        ok(lib.ze_index_begin(h), "index_begin")
        while ok(lib.ze_index_step(h), "index_step") > 0:
            pass
        for kind, o in outs.items():
            ok(lib.ze_results(h, kind, o.ctypes.data, o.nbytes), "results")

    for _ in range(max(2, warmup - 2)):  # as the API leg: the second run makes the page-locked copy
        run()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        run()
    e1.record()
    torch.cuda.synchronize()
    lib.ze_destroy(h)
    return e0.elapsed_time(e1) / steps, outs


def config_of(a, n):
    """The workload as the bench line names it (both arms)."""
    return {"workload": WORKLOAD, "patterns_per_gpu": n, "bandwidth": L, "precision": a.precision,
            "device_batch": min(a.batch, n), "l2": "inputs (720 MB) larger than L2, no flush"}


# ── the device ──

class Clocks:
    """Samples of the SM clock and the throttle reasons during the timed region: read through NVML
    (read-only queries) every 10 ms on a thread, or from nvidia-smi at 200 ms where NVML is not
    available."""

    REASONS = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, index, off=False):
        self.index = index
        self.off = off
        self.proc = None
        self.path = None
        self.thread = None
        self.rows = []  # (sm MHz, max sm MHz, reasons)

    def _nvml_handle(self, nv):
        """The NVML handle of this process's CUDA device: by its UUID (CUDA_VISIBLE_DEVICES may
        renumber the devices), else by index."""
        try:
            import torch

            uuid = str(torch.cuda.get_device_properties(int(self.index)).uuid)
            return nv.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            return nv.nvmlDeviceGetHandleByIndex(int(self.index))

    def _nvml_loop(self, h, nv, stop):
        bits = (nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap)
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        while True:
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                why = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.rows.append((float(sm), float(mx), tuple(n for n, b in zip(self.REASONS, bits) if why & b)))
            except Exception:
                pass
            if stop.wait(0.01):
                return

    def __enter__(self):
        if self.off:
            return self
        try:
            import pynvml as nv

            nv.nvmlInit()
            h = self._nvml_handle(nv)
            self._stop = threading.Event()
            self.thread = threading.Thread(target=self._nvml_loop, args=(h, nv, self._stop), daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.thread = None
        self.path = tempfile.mktemp(suffix=".csv")
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.thread is not None:
            self._stop.set()
            self.thread.join()
        if self.proc is not None:
            self.proc.terminate()
            self.proc.wait()
            try:
                for l in open(self.path).read().strip().splitlines():
                    r = [x.strip() for x in l.split(",")]
                    if len(r) >= 7 and r[0].replace(".", "").isdigit():
                        why = tuple(n for k, n in enumerate(self.REASONS) if "Active" in r[3 + k] and "Not" not in r[3 + k])
                        self.rows.append((float(r[0]), float(r[1]) if r[1].replace(".", "").isdigit() else None, why))
            except Exception:
                pass

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [r[0] for r in self.rows]
        mx = [r[1] for r in self.rows if r[1] is not None]
        reasons = sorted({n for r in self.rows for n in r[2]})
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows), "source": "nvml" if self.proc is None else "nvidia-smi"}


class StageTimer:
    """CUDA events at the stage boundaries of one pass (on the launching stream)."""

    def __init__(self, torch):
        self.torch = torch
        self.events = []

    def mark(self, name):
        e = self.torch.cuda.Event(enable_timing=True)
        e.record()
        self.events.append((name, e))

    def totals(self):
        self.torch.cuda.synchronize()
        out = {}
        for (name, e0), (_, e1) in zip(self.events, self.events[1:]):
            out[name] = out.get(name, 0.0) + e0.elapsed_time(e1)
        return out


def device_main(a):
    import torch

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist_mod

        dist = dist_mod
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    import zebsdsolve_b200 as ze
    from zebsdsolve_b200 import _native
    from zebsdsolve_b200 import synthetic as syn
    from zebsdsolve_b200.master import write_npz

    from zebsdsolve_b200 import shard

    rows, cols = scan_shape(a.patterns)
    n = rows * cols
    sheets = syn.master_sheets(2, side=401, lmax=96, group="432", device="cuda")
    tmp = tempfile.mkdtemp()
    write_npz(f"{tmp}/m432.npz", sheets, 401, syn.group_matrices("432"), 30)
    s = ze.Solver()
    s.configure(bandwidth=L, precision=a.precision)
    s.add_phase(f"{tmp}/m432.npz")
    s.set_patterns(np.zeros((rows, cols, H, W), np.uint16))
    s.set_geometry(pc=PC, sample_tilt_deg=70.0, detector_tilt_deg=0.0)
    e = s._e
    # the same scan on every rank: each indexes all of it for the device-resident value (weak
    # scaling) and its share of it for the end-to-end value (one scan sharded over the ranks)
    rng = np.random.default_rng(100)
    q, grain = syn.grain_map(rng, rows, cols, GRAINS, SPREAD_DEG)
    pats = np.empty((n, H, W), np.uint16)
    for i in range(0, n, 16384):
        sims = e.simulate_device(0, np.arange(i, min(n, i + 16384)), q[i:i + 16384])
        pats[i:i + len(sims)] = syn.counted_patterns(sims, seed=i // 16384).cpu().numpy()
    s.set_patterns(pats.reshape(rows, cols, H, W))
    e.prepare(L)
    torch.cuda.synchronize()

    # value: stored patterns resident in HBM
    raw = torch.as_tensor(pats, device="cuda")
    cells = np.arange(n)
    batch = min(a.batch, n)

    def device_pass(timer=None):
        for b0 in range(0, n, batch):
            c = cells[b0:b0 + batch]
            e.run_device(raw[b0:b0 + len(c)], c, L, timer)

    def max_over_ranks(v):
        from zebsdsolve_b200.shard import max_over_ranks as mor

        return mor(v, dist, "cuda")

    def time_form(precision, clocks=None, nvtx=False):
        """(device-resident ms per step, e2e ms per step, launches, stage ms, results) of one form."""
        s.configure(precision=precision)
        e.prepare(L)
        for _ in range(a.warmup):
            device_pass()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        _native.launches["count"] = 0
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with (clocks if clocks is not None else Clocks(None, off=True)):
            torch.cuda.synchronize()
            if nvtx:
                torch.cuda.nvtx.range_push("timed")  # the range a profiler's launch list is filtered to
            t0.record()
            for _ in range(a.steps):
                device_pass()
            t1.record()
            torch.cuda.synchronize()
            if nvtx:
                torch.cuda.nvtx.range_pop()
        launches = _native.launches["count"]
        e.check_device()  # a tensor-core wait that gave up would have left U incomplete
        ms = max_over_ranks(t0.elapsed_time(t1) / a.steps)
        if dist:
            dist.barrier()
        # stage times of one more pass (CUDA events on the launching stream between the stages)
        timer = StageTimer(torch)
        device_pass(timer)
        stages = timer.totals()
        # e2e: the public API from pinned host memory, every step (uploads, passes, readbacks, landing);
        # two untimed runs: a scan's first run streams through the staging slots, its second makes
        # the page-locked copy of the whole scan that every later run uploads from. With several
        # ranks the one scan is sharded (shard.index_sharded: each rank its contiguous share of the
        # cells, the records gathered to rank 0, which holds the whole map's results)
        def api_run():
            return shard.index_sharded(s, dist) if dist else s.index()

        for _ in range(max(2, a.warmup - 2)):
            api_run()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(a.steps):
            r = api_run()
        e1.record()
        torch.cuda.synchronize()
        ems = max_over_ranks(e0.elapsed_time(e1) / a.steps)
        return ms, ems, launches, stages, r

    clk = Clocks(local)
    ms, ems, launches, stages, r = time_form(a.precision, clk, nvtx=True)
    abi = None
    if world == 1 and not a.no_abi:
        # the same scan through the reference's own C ABI (libzebsdsolve.so), its own engine
        ams, aouts = abi_e2e({"bandwidth": L, "precision": a.precision}, f"{tmp}/m432.npz",
                             pats.reshape(rows, cols, H, W), a.steps, a.warmup)
        same = all(np.array_equal(aouts[k].reshape(r[key].shape), r[key])
                   for k, key in ((0, "quaternions"), (1, "ncc"), (2, "nmi"), (3, "phase"), (4, "euler"), (5, "z"),
                                  (6, "sweep")))
        abi = {"value": round(n / (ams / 1e3), 1), "unit": "patterns/s", "ms_per_step": round(ams, 3),
               "results_equal_python_api": bool(same),
               "note": "the reference's own C ABI (libzebsdsolve.so): ze_set_patterns from host memory once, then "
                       "each step ze_index_begin, the ze_index_step loop and ze_results of all 7 kinds, as the "
                       "reference's Solver.index issues them"}
    u_half = e.bands[L]["phases"][0][1].u_scale is not None  # the timed form keeps U in FP16
    value = n * world / (ms / 1e3)
    e2e = n / (ems / 1e3)  # one scan's patterns over the job's time (all of it on one rank, or sharded)
    fp32 = None
    if not a.no_fp32_form and a.precision != "f32":
        ms32, ems32, _, stages32, r32 = time_form("f32")

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    dis = np.degrees(s.disorientation(r["quaternions"].reshape(-1, 4), q))
    if not a.no_fp32_form and a.precision != "f32":
        dis32 = np.degrees(s.disorientation(r32["quaternions"].reshape(-1, 4), q))
        agree = np.degrees(s.disorientation(r32["quaternions"].reshape(-1, 4), r["quaternions"].reshape(-1, 4)))
        fp32 = {"value": round(n * world / (ms32 / 1e3), 1), "e2e": round(n / (ems32 / 1e3), 1),
                "ms_per_step": round(ms32, 3), "stage_ms_per_step": {k: round(v, 3) for k, v in stages32.items()},
                "median_deg": round(float(np.median(dis32)), 4),
                "forms_within_0.1deg": round(float((agree < 0.1).mean()), 5)}
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    hbm = peaks.get("hbm_gbs", 6650.0)
    ph = e.bands[L]["phases"][0][1]
    d = ph.dims
    # algorithmic HBM bytes of each stage per pattern (its kernels' compulsory reads and writes):
    # U, the spectrum, is complex FP32 (8 bytes a value) in the FP32 form and complex FP16 (4) in
    # the BF16 form
    u_bytes = d.nb * d.L * d.nc * (4 if u_half else 8)
    algo = {"prep": H * W * (2 + 4),                       # u16 in, f32 out
            "sphere": H * W * 4 + d.n_pairs * 8,           # pattern in, coefficients out
            "spectrum": d.n_pairs * 8 + u_bytes,           # coefficients in, U out
            "peaks": u_bytes + 8 * 4,                      # U in, peak out
            "refine": H * W * 4 + 8 * 4}                   # pattern in, record out
    traffic = {}
    tpath = os.path.join(ROOT, "profiles", "traffic.json")  # ncu DRAM bytes per pattern of each stage
    if os.path.exists(tpath):
        traffic = json.load(open(tpath)).get(a.precision, {})
    roof = {}
    for k, ms_k in stages.items():
        if k not in algo or ms_k <= 0:
            continue
        ach = algo[k] * n / (ms_k / 1e3) / 1e9
        t = traffic.get(k)
        roof[k] = {"bound": "hbm", "achieved": round(ach, 1), "peak": hbm, "unit": "GB/s", "frac": round(ach / hbm, 4),
                   "traffic": int(t * batch) if t else None, "ms_per_step": round(ms_k, 3)}
    if "refine" in roof:
        # the refinement is bound by its record gathers from the L2-resident table, not by HBM: one
        # 32-byte FP16 neighbourhood record a masked pixel a pass (refine_iters passes and the
        # last, with the pattern's values from shared memory)
        import ctypes

        fr = e.frame()
        npix = int(_native.load().zeb_mask_pixels(ctypes.byref(fr)))
        passes = int(s.settings["refine_iters"]) + 1
        roof["refine"]["l2_gather"] = {
            "achieved": round(n * passes * npix * 32 / (stages["refine"] / 1e3) / 1e9, 1), "unit": "GB/s",
            "bytes_per_pattern": passes * npix * 32,
            "note": f"{passes} passes x {npix} masked pixels x 32 B records from the L2-resident table"}
    dom = max((k for k in roof), key=lambda k: stages[k])
    line = {
        "metric": "patterns/s indexed+refined on 1 B200, BF16 form vs plain FP32 at <=0.1 deg error",
        "value": round(value, 1), "unit": "patterns/s", "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if a.precision == "f32" else "bf16+f32", "data": "synthetic",
        "config": config_of(a, n),
        "e2e": {"value": round(e2e, 1), "unit": "patterns/s", "h2d_bytes_per_step": int(n * H * W * 2),
                "d2h_bytes_per_step": int(n * (8 + 4) * 4 * len(e.phases)),
                **({"scaling": "strong", "note": f"one {rows}x{cols} scan sharded over {world} ranks "
                                                  "(shard.index_sharded), records gathered to rank 0"}
                   if world > 1 else {})},
        "gpu_launches": int(launches),
        "roofline": dict(roof[dom], kernel=dom, per_launch_patterns=batch),
        "rooflines": roof,
        "accuracy": {"median_deg": round(float(np.median(dis)), 4), "p99_deg": round(float(np.percentile(dis, 99)), 4),
                     "within_0.1deg": round(float((dis < 0.1).mean()), 4)},
        "clocks": clk.summary(),
    }
    if abi is not None:
        # the headline end-to-end figure is the one through the reference's own C ABI; the same
        # scan through this package's Python API (Solver.index) beside it
        line["e2e_python_api"] = {"value": line["e2e"]["value"], "unit": "patterns/s",
                                  "ms_per_step": round(ems, 3)}
        line["e2e"].update(value=abi["value"], ms_per_step=abi["ms_per_step"],
                           results_equal_python_api=abi["results_equal_python_api"], via=abi["note"])
    if fp32 is not None:
        line["fp32_form"] = fp32
        line["vs_fp32_form"] = {"value": round(value / fp32["value"], 3), "e2e": round(e2e / fp32["e2e"], 3)}
    if not a.no_cpu:
        # the oracle (FP64) on a lattice of the workload's own stored patterns, with the GPU path's
        # settings (static background of the same lattice average, dynamic background, mask, the
        # master baked for this detector, 8 refinement iterations): the CPU baseline's timing and
        # each form's parity, cell by cell
        import oracle.pipeline as opl

        ocells = opl.lattice(rows, cols, ORACLE_CELLS)
        scan = oracle_scan(sheets, opl.static_average(pats, rows, cols, 1024))
        g = e.geo
        og_ = oracle_geometry(g.px_um, g.step_x_um)
        ts = opl.cell_positions(og_, rows, cols, ocells, H, W, s.settings["scan_x_sign"], s.settings["scan_y_sign"])
        orecs, v64, cores64, dt64 = oracle_run(scan, pats[ocells], ts)
        # the CPU baseline: the same cells through the C++ FP32 restatement on every host thread
        crecs, vc, cores, dtc = cpu_ref_run(scan, pats[ocells], ts)
        line["cpu_baseline"] = {"value": round(vc, 3), "unit": "patterns/s", "cores": cores, "kind": "port",
                                "sample": f"{len(ocells)} cells on a lattice over the map (their own stored patterns: "
                                          f"filtered, correlated at L={L}, refined, NMI) through the C++ FP32 "
                                          f"restatement of the path (oracle/cpu_ref) on {cores} threads in {dtc:.2f} s"}
        line["oracle_fp64"] = {"value": round(v64, 3), "unit": "patterns/s", "cores": cores64,
                               "sample": f"the same {len(ocells)} cells through the FP64 NumPy oracle in {dt64:.1f} s"}
        forms = {a.precision: r}
        if fp32 is not None:
            forms["f32"] = r32
        line["oracle_parity"] = {"cells": f"{len(ocells)} on a lattice over the {rows}x{cols} map",
                                 "bar": "within 0.1 deg for >= 99.9 % and |dNCC| <= 1e-3"}
        for k, rr in forms.items():
            line["oracle_parity"][k] = parity_of(orecs, scan.rotations, rr["quaternions"].reshape(-1, 4)[ocells],
                                                 rr["ncc"].reshape(-1)[ocells], rr["nmi"].reshape(-1)[ocells])
        line["oracle_parity"]["cpu_ref"] = parity_of(orecs, scan.rotations, np.array([c[0] for c in crecs]),
                                                     np.array([c[1] for c in crecs]), np.array([c[2] for c in crecs]))
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def adjoint_main(a):
    """Six unknowns per pattern (orientation and pattern centre) refined on the detector: a
    316 × 316 scan of 120 × 120 u16 patterns simulated at pattern centres jittered by ±0.005 and
    refined from orientations 1–2° off the truth and the nominal centre, all patterns in one
    Levenberg–Marquardt run (Solver.refine_patterns), with the exact adjoint gradient or the
    reference's. One GPU; value = patterns / wall time of the call (its uploads, filters, every
    round and the results' readback)."""
    import time

    import torch

    import zebsdsolve_b200 as ze
    from zebsdsolve_b200 import adjoint
    from zebsdsolve_b200 import rotations as R
    from zebsdsolve_b200 import synthetic as syn
    from zebsdsolve_b200.master import write_npz

    torch.cuda.set_device(0)
    rows, cols = scan_shape(a.patterns)
    n = rows * cols
    h = w = 120
    sheets = syn.master_sheets(2, side=401, lmax=96, group="432", device="cuda")
    tmp = tempfile.mkdtemp()
    write_npz(f"{tmp}/m432.npz", sheets, 401, syn.group_matrices("432"), 30)
    s = ze.Solver()
    s.add_phase(f"{tmp}/m432.npz")
    s.set_patterns(np.zeros((rows, cols, h, w), np.uint16))
    s.set_geometry(pc=PC, sample_tilt_deg=70.0, detector_tilt_deg=0.0)
    e = s._e
    rng = np.random.default_rng(300)
    q, _ = syn.grain_map(rng, rows, cols, GRAINS, SPREAD_DEG)
    dpc = rng.uniform(-0.005, 0.005, (n, 3))
    J = adjoint.pc_jacobian(e.geo, h, w)
    shifts = dpc @ J.T
    pats = np.empty((n, h, w), np.uint16)
    for i in range(0, n, 8192):
        sl = slice(i, min(n, i + 8192))
        sims = e.simulate_device(0, np.arange(sl.start, sl.stop), q[sl], shifts=shifts[sl])
        pats[sl] = syn.counted_patterns(sims, seed=7 + i // 8192).cpu().numpy()
    s.set_patterns(pats.reshape(rows, cols, h, w))
    ax = rng.normal(size=(n, 3))
    ax /= np.linalg.norm(ax, axis=1, keepdims=True)
    ang = np.radians(rng.uniform(1.0, 2.0, n))
    q0 = R.qstd(R.qmul(R.exp_map(ax * ang[:, None]), q))
    cells = np.arange(n)
    G = e.phases[0].master.rotations()
    out = {}
    for grad in ("adjoint", "reference"):
        for _ in range(max(1, a.warmup)):
            s.refine_patterns(cells[:2048], quaternions=q0[:2048], gradient=grad)
        torch.cuda.synchronize()
        times = []
        for _ in range(max(1, a.steps)):
            t0 = time.perf_counter()
            r = s.refine_patterns(cells, quaternions=q0, gradient=grad)
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t0)
        dis = np.degrees(R.disorientation(r["quaternions"], q, G))
        pcerr = np.abs(r["pc"] - (np.asarray(PC)[None, :] + dpc)).max(1)
        out[grad] = {"value": round(n / float(np.median(times)), 1), "s_per_step": round(float(np.median(times)), 4),
                     "rounds": int(r["rounds"]), "median_deg": round(float(np.median(dis)), 4),
                     "p99_deg": round(float(np.percentile(dis, 99)), 4),
                     "start_median_deg": round(float(np.degrees(np.median(ang))), 3),
                     "median_pc_error": round(float(np.median(pcerr)), 6), "mean_ncc": round(float(r["ncc"].mean()), 5)}
    line = {"metric": "patterns/s, six unknowns refined (orientation + pattern centre), 1 B200",
            "value": out["adjoint"]["value"], "unit": "patterns/s", "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
            "higher_is_better": True, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{rows}x{cols} scan of 120x120 uint16 patterns, pattern centres jittered +-0.005, "
                                   "orientations 1-2 deg off, Levenberg-Marquardt over all patterns at once",
                       "patterns": n},
            "adjoint": out["adjoint"], "reference_gradient": out["reference"]}
    print(json.dumps(line), flush=True)


def uneven_main(a):
    """Many scans of uneven lengths (log-uniform from 1 000 to --max-count patterns) and detector
    sizes (40², 60², 96², 160² u16), each with two phases (432 and 622 masters, grains assigned by
    a fair coin), indexed one after another through one Solver at L = 64 in the BF16 form: the
    whole job's patterns over its wall time, every scan's set-up (pinned copy, chance
    calibration, denominators, masks) included."""
    import time

    import torch

    import zebsdsolve_b200 as ze
    from zebsdsolve_b200 import synthetic as syn
    from zebsdsolve_b200.master import write_npz

    torch.cuda.set_device(0)
    tmp = tempfile.mkdtemp()
    paths = []
    for g, seed in (("432", 2), ("622", 3)):
        sheets = syn.master_sheets(seed, side=401, lmax=96, group=g, device="cuda")
        write_npz(f"{tmp}/m{g}.npz", sheets, 401, syn.group_matrices(g), syn.POINT_GROUP[g])
        paths.append(f"{tmp}/m{g}.npz")
    s = ze.Solver()
    s.configure(bandwidth=L, precision=a.precision)
    for p in paths:
        s.add_phase(p)
    e = s._e
    rng = np.random.default_rng(400)
    counts = np.exp(rng.uniform(np.log(1000), np.log(max(a.max_count, 1001)), a.scans)).astype(int)
    sizes = rng.choice([40, 60, 96, 160], a.scans)

    def make(k):
        """Scan k, simulated on the device (its orientations, phases and patterns)."""
        n, side = int(counts[k]), int(sizes[k])
        cols = int(np.ceil(np.sqrt(n)))
        rows = -(-n // cols)
        n = rows * cols
        g = np.random.default_rng(1000 + k)
        s.set_patterns(np.zeros((rows, cols, side, side), np.uint16))
        s.set_geometry(pc=PC, sample_tilt_deg=70.0, detector_tilt_deg=0.0)
        q, grain = syn.grain_map(g, rows, cols, max(4, n // 500), SPREAD_DEG)
        phase_of = g.integers(0, 2, grain.max() + 1)[grain.reshape(-1)]
        pats = np.empty((n, side, side), np.uint16)
        for ph in (0, 1):
            sel = np.flatnonzero(phase_of == ph)
            for i in range(0, len(sel), 4096):
                c = sel[i:i + 4096]
                sims = e.simulate_device(ph, c, q[c])
                pats[c] = syn.counted_patterns(sims, seed=k * 1000 + i).cpu().numpy()
        return pats.reshape(rows, cols, side, side), q, phase_of

    # warm-up: the first scan indexed once, untimed
    pats, _, _ = make(0)
    s.set_patterns(pats)
    s.index()
    # each scan made, then timed from its patterns on the host to its results (set-up included);
    # one scan is held at a time
    wall, total, right, dis_all, shapes, scan_ms = 0.0, 0, [], [], [], []
    for k in range(a.scans):
        pats, q, phase_of = make(k)
        shapes.append((int(pats.shape[0] * pats.shape[1]), int(pats.shape[2])))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s.set_patterns(pats)
        r = s.index()
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        wall += dt
        scan_ms.append(round(dt * 1e3, 2))
        total += pats.shape[0] * pats.shape[1]
        ph = r["phase"].reshape(-1)
        right.append(ph == phase_of)
        qq = r["quaternions"].reshape(-1, 4)
        for p in (0, 1):
            sel = (ph == p) & (phase_of == p)
            if sel.any():
                dis_all.append(np.degrees(s.disorientation(qq[sel], q[sel], phase=p)))
        del pats
    right = np.concatenate(right)
    dis = np.concatenate(dis_all)
    line = {"metric": "patterns/s over uneven scans (lengths, detector sizes, two phases), 1 B200",
            "value": round(total / wall, 1), "unit": "patterns/s", "n_gpus": 1, "steps": 1, "warmup": 1,
            "higher_is_better": True, "dtype": "bf16+f32", "data": "synthetic",
            "config": {"workload": f"{a.scans} scans, 1000-{a.max_count} patterns (log-uniform), detector sizes "
                                   "40/60/96/160 u16, masters 432 and 622 (401^2, SH <= 96), L = 64",
                       "patterns": total, "scan_patterns": [c for c, _ in shapes],
                       "scan_sizes": [z for _, z in shapes], "scan_ms": scan_ms, "precision": a.precision},
            "wall_s": round(wall, 3),
            "accuracy": {"phase_right": round(float(right.mean()), 4), "median_deg": round(float(np.median(dis)), 4),
                         "within_0.1deg": round(float((dis < 0.1).mean()), 4)}}
    print(json.dumps(line), flush=True)


def reference_main(a):
    """The reference's algorithm on the host cores: its C++ FP32 restatement (oracle/cpu_ref,
    checked against the FP64 oracle; the reference engine itself, Zig + WGSL on wgpu-native, cannot
    run on this box), every host thread taking the next pattern; a step indexes the workload's
    lattice of cells, made on the host (host_workload); W untimed steps, then K timed ones. Under
    torchrun only rank 0 runs."""
    import oracle.cpu_ref as ocr

    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    raws, scan, cells, ts = host_workload()
    cores = max(1, len(os.sched_getaffinity(0)))
    cr = ocr.CpuRef(scan)
    for _ in range(max(a.warmup, 1)):
        cr.index(raws, ts, cores)
    t0 = time.perf_counter()
    for _ in range(a.steps):
        cr.index(raws, ts, cores)
    dt = time.perf_counter() - t0
    done = a.steps * len(raws)
    v = done / dt
    n = ROWS * COLS if a.patterns == ROWS * COLS else a.patterns
    line = {"impl": "reference", "metric": "patterns/s indexed+refined on 1 B200, BF16 form vs plain FP32 at <=0.1 deg error",
            "value": round(v, 3), "unit": "patterns/s", "n_gpus": int(os.environ.get("WORLD_SIZE", a.gpus)),
            "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": round(1e3 * dt / a.steps, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": config_of(a, n),
            "cpu_baseline": {"value": round(v, 3), "unit": "patterns/s", "cores": cores, "kind": "port",
                             "sample": f"a step: the workload's lattice of {len(cells)} cells (made on the host: the "
                                       f"same master and grain map), filtered, correlated at L={L}, refined and "
                                       f"scored through the C++ FP32 restatement of the path (oracle/cpu_ref) on "
                                       f"{cores} threads"},
            "e2e": {"value": round(v, 3), "unit": "patterns/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference engine (Zig + WGSL on wgpu-native) cannot be built or run here; its algorithm is "
                    "timed as a C++ FP32 restatement of the path on the host cores"}
    print(json.dumps(line), flush=True)


def pcfit_cpu_sample(seconds):
    """The oracle's score of one fit pattern under one candidate at L = 64 (its window's
    denominators shared by the 25 fit patterns of a candidate), timed on one host core."""
    import oracle.master as om
    import oracle.spherical as osp
    from zebsdsolve_b200 import synthetic as syn

    side = 201
    sheets = syn.master_sheets(3, side=side, lmax=48, group="432").reshape(-1).astype(np.float64)
    m = om.Master(side, sheets, syn.group_matrices("432"), 30)
    m.measure_symmetry()
    hm = om.Harmonics(m, sheets, L)
    tb = osp.Tables(L)
    pt = osp.PhaseTables(tb, hm, om.fold_of(hm.rules))
    import oracle.geometry as og

    geo = og.Geometry(pc=PC, sample_tilt_deg=70.0)
    frame = geo.frame()
    mask = og.mask_of(H, W)
    rng = np.random.default_rng(1)
    t = geo.translation(H, W)
    t0 = time.perf_counter()
    walm, wst = osp.coefficients(tb, None, t, frame, mask, flags=osp.FLAG_WINDOW, shape=(H, W))
    rden = osp.window_denominators(tb, pt, walm, wst[0])
    t_win = time.perf_counter() - t0
    done, t1 = 0, time.perf_counter()
    while done < 2 or time.perf_counter() - t1 < max(seconds - t_win, 0):
        g, _ = osp.coefficients(tb, rng.normal(size=(H, W)), t, frame, mask)
        osp.peak(tb, pt, osp.correlation_volume(tb, pt, hm.f, g) * rden)
        done += 1
    t_pat = (time.perf_counter() - t1) / done
    return 1.0 / (t_pat + t_win / 25), f"1 candidate window and {done} pattern scores at L=64 through the FP64 oracle"


def pcfit_main(a):
    """The pattern-centre vote at the reference's default settings (25 fit patterns on a 5 x 5
    lattice, 9 x 9 x 5 candidates per grid, 3 levels narrowing by 0.35, ballots, L = 64) on a
    40 x 40 scan of 60 x 60 u16 patterns simulated at a known centre, from a start 0.015-0.02 off:
    (fit patterns x candidates scored) per second of the whole fit, every readback and the host
    vote inside the time."""
    import torch

    import zebsdsolve_b200 as ze
    from zebsdsolve_b200 import synthetic as syn
    from zebsdsolve_b200.master import write_npz

    torch.cuda.set_device(0)
    tmp = tempfile.mkdtemp()
    write_npz(f"{tmp}/m432.npz", syn.master_sheets(2, side=401, lmax=96, group="432", device="cuda"), 401,
              syn.group_matrices("432"), 30)
    rows = cols = 40
    s = ze.Solver()
    s.configure(bandwidth=L, precision=a.precision)
    s.add_phase(f"{tmp}/m432.npz")
    s.set_patterns(np.zeros((rows, cols, H, W), np.uint16))
    s.set_geometry(pc=PC, sample_tilt_deg=70.0, detector_tilt_deg=0.0)
    rng = np.random.default_rng(500)
    q, _ = syn.grain_map(rng, rows, cols, 20, SPREAD_DEG)
    sims = s._e.simulate_device(0, np.arange(rows * cols), q)
    s.set_patterns(syn.counted_patterns(sims, seed=9).cpu().numpy().reshape(rows, cols, H, W))
    start = (PC[0] + 0.015, PC[1] + 0.02, PC[2] - 0.02)
    for _ in range(max(1, a.warmup)):
        s.set_geometry(pc=start)
        s.fit_pc()
    times, fits = [], []
    for _ in range(max(1, a.steps)):
        s.set_geometry(pc=start)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        f = s.fit_pc()
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
        fits.append(f)
    f = fits[-1]
    dt = float(np.median(times))
    from zebsdsolve_b200 import pcfit

    s.set_geometry(pc=start)
    timer = StageTimer(torch)
    pcfit.run(s._e, timer)  # one more fit, untimed, for where its time goes
    stages = {k: round(v, 3) for k, v in timer.totals().items()}
    scored = f["n_candidates"] * f["n_patterns"]
    err = np.abs(np.array(f["pc"]) - PC)
    line = {"metric": "candidate scores/s in the pattern-centre vote (fit patterns x candidate centres), 1 B200",
            "value": round(scored / dt, 1), "unit": "scores/s", "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
            "ms_per_fit": round(1e3 * dt, 2), "higher_is_better": True, "dtype": "bf16+f32", "data": "synthetic",
            "config": {"workload": f"{rows}x{cols} scan of 60x60 uint16 patterns simulated at pc {PC}, 432 master "
                                   f"401^2 (SH <= 96), start {tuple(round(v, 3) for v in start)}, fit_grid 5, "
                                   "9x9x5 candidates, 3 levels, ballots, fit_bandwidth 64", "precision": a.precision},
            "grids": len(s.pc_levels()), "candidates": f["n_candidates"], "fit_patterns": f["n_patterns"],
            "pc": [round(v, 5) for v in f["pc"]], "pc_error": round(float(err.max()), 5),
            "score": round(f["score"], 4), "start_score": round(f["start_score"], 4), "stage_ms_per_fit": stages}
    if not a.no_cpu:
        v, sample = pcfit_cpu_sample(a.cpu_seconds)
        line["cpu_baseline"] = {"value": round(v, 3), "unit": "scores/s", "cores": 1, "kind": "port", "sample": sample}
    print(json.dumps(line), flush=True)


def plane_cpu_sample(seconds, grad, side, frame, t, q, pats, mask):
    """The oracle's settle of one fit pattern over six unknowns (FP64 NumPy), on one host core."""
    import oracle.detector as od

    done, t0 = 0, time.perf_counter()
    while done < 1 or time.perf_counter() - t0 < seconds:
        od.settle6(grad, side, frame, t, q[done % len(q)], pats[done % len(q)], mask, 3.0, 60)
        done += 1
    dt = time.perf_counter() - t0
    return done / dt, f"{done} fit patterns of 60x60 settled over six unknowns by the FP64 oracle"


def plane_main(a):
    """The plane of source points at the reference's default settings (every 2nd cell each way,
    points method, information weights, bicubic master, the master's pixel chosen of five widths)
    on a 100 x 100 map of 60 x 60 patterns simulated with the beam travelling 25 um a step on 60 um
    detector pixels, Gaussian noise as strong as the signal, from a pattern centre 0.005 off: fit
    patterns refined per second of the whole fit (indexing them at fit_bandwidth 64, the
    settles, the plane, its standard errors); then the automatic fit (the vote, then the plane
    with the model the map supports) timed the same way."""
    import torch

    import zebsdsolve_b200 as ze
    from zebsdsolve_b200 import synthetic as syn
    from zebsdsolve_b200.master import write_npz

    torch.cuda.set_device(0)
    tmp = tempfile.mkdtemp()
    write_npz(f"{tmp}/m432.npz", syn.master_sheets(2, side=401, lmax=96, group="432", device="cuda"), 401,
              syn.group_matrices("432"), 30)
    rows = cols = 100
    geo = dict(sample_tilt_deg=70.0, detector_tilt_deg=0.0, px_um=60.0, step_x_um=25.0, step_y_um=25.0)
    s = ze.Solver()
    s.configure(bandwidth=L, precision=a.precision)
    s.add_phase(f"{tmp}/m432.npz")
    s.set_patterns(np.zeros((rows, cols, H, W), np.float32))
    s.set_geometry(pc=PC, **geo)
    rng = np.random.default_rng(600)
    q, _ = syn.grain_map(rng, rows, cols, 40, SPREAD_DEG)
    sims = s._e.simulate_device(0, np.arange(rows * cols), q)
    sims = sims + sims.std() * torch.randn(sims.shape, device=sims.device, generator=torch.Generator("cuda").manual_seed(6))
    s.set_patterns(sims.cpu().numpy().astype(np.float32).reshape(rows, cols, H, W))
    start = (PC[0] + 0.005, PC[1] - 0.004, PC[2] + 0.004)
    out = {}
    for name, call in (("fit_plane", s.fit_plane), ("fit_geometry", s.fit_geometry)):
        times = []
        for i in range(max(1, a.warmup) + max(1, a.steps)):
            s.set_geometry(pc=start)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            r = call()
            torch.cuda.synchronize()
            if i >= max(1, a.warmup):
                times.append(time.perf_counter() - t0)
        dt = float(np.median(times))
        out[name] = {"s_per_fit": round(dt, 4), "fit_patterns": r["n_patterns"], "used": r["n_used"],
                     "rounds": r["iterations"], "model": r["model"], "pc_error": round(float(np.abs(np.array(r["pc"]) - PC).max()), 5),
                     "ncc": round(r["ncc"], 4), "start_ncc": round(r["start_ncc"], 4),
                     "value": round(r["n_patterns"] / dt, 1)}
    line = {"metric": "fit patterns/s in the plane fit (each refined over six unknowns, then the plane), 1 B200",
            "value": out["fit_plane"]["value"], "unit": "patterns/s", "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
            "higher_is_better": True, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{rows}x{cols} map of 60x60 patterns simulated at pc {PC} with the beam travelling "
                                   "(25 um steps, 60 um pixels), Gaussian noise as strong as the signal, start 0.005 "
                                   "off; plane_stride 2, points, information weights, bicubic, master pixel auto"},
            "fit_plane": out["fit_plane"], "fit_geometry": out["fit_geometry"]}
    if not a.no_cpu:
        import oracle.detector as od
        import oracle.geometry as og

        e = s._e
        e.prepare_masters()
        baked = e.phases[0].baked[1].cpu().numpy().astype(np.float64)
        gq = og.Geometry(pc=PC, sample_tilt_deg=70.0)
        mask = og.mask_of(H, W)
        pats = [np.asarray(e.patterns.reshape(-1, H, W)[k], np.float64) for k in range(4)]
        import oracle.prep as op

        pats = [op.normalize(p, mask) for p in pats]
        v, sample = plane_cpu_sample(a.cpu_seconds, od.gradient_table(baked, 401), 401, gq.frame(),
                                     gq.translation(H, W), q[:4], pats, mask)
        line["cpu_baseline"] = {"value": round(v, 3), "unit": "patterns/s", "cores": 1, "kind": "port",
                                "sample": sample}
    print(json.dumps(line), flush=True)


def large_main(a):
    """Config 5's path at --large patterns (1 000 000 by default: 51 GB of stored patterns on the
    host, streamed to the device through two page-locked slots, never locked whole): 160 x 160 u16
    patterns of the 432 master with grains as in the headline workload, binned 2x to 80 x 80;
    indexed in two sweeps (L = 64, then L = 128 for the cells not accepted) in the BF16 form and in
    the plain FP32 form, then every pattern refined over six unknowns with the adjoint gradient;
    beside it the PCA dictionary of 295 389 orientations (dict_grid 96) reduced to 512 components
    and matched on the tensor cores (top 8, rescored in FP32). Each path timed from the patterns
    on the host to its results."""
    import torch

    import zebsdsolve_b200 as ze
    from zebsdsolve_b200 import synthetic as syn
    from zebsdsolve_b200.master import write_npz

    torch.cuda.set_device(0)
    tmp = tempfile.mkdtemp()
    write_npz(f"{tmp}/m432.npz", syn.master_sheets(2, side=401, lmax=96, group="432", device="cuda"), 401,
              syn.group_matrices("432"), 30)
    side = int(math.isqrt(a.large))
    rows = cols = side
    n = rows * cols
    s = ze.Solver()
    s.add_phase(f"{tmp}/m432.npz")
    s.set_patterns(np.zeros((rows, cols, 160, 160), np.uint16))
    s.set_geometry(pc=PC, sample_tilt_deg=70.0, detector_tilt_deg=0.0)
    rng = np.random.default_rng(700)
    q, _ = syn.grain_map(rng, rows, cols, GRAINS, SPREAD_DEG)
    pats = np.empty((n, 160, 160), np.uint16)
    e = s._e
    for i in range(0, n, 4096):
        c = np.arange(i, min(n, i + 4096))
        pats[c] = syn.counted_patterns(e.simulate_device(0, c, q[c]), seed=70 + i // 4096).cpu().numpy()
    s.set_patterns(pats.reshape(rows, cols, 160, 160))
    G = e.phases[0].master.rotations()

    def median_deg(quats):
        return round(float(np.median(np.degrees(s.disorientation(quats.reshape(-1, 4), q)))), 4)

    def timed(fn):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = fn()
        torch.cuda.synchronize()
        return out, time.perf_counter() - t0

    out = {}
    cells = np.arange(n)
    for prec in (a.precision, "f32"):
        s.configure(binning=2, bandwidth=128, sweeps=2, sweep_bandwidth=64, sweep_method="same", precision=prec,
                    method="spherical")
        s.index_cells(cells[:4096], bandwidth=64)  # tables and masters of both bandwidths, untimed
        s.index_cells(cells[:4096], bandwidth=128)
        # one untimed run of each form first (a pass's buffers, the refinement's plan), so that
        # neither form's timing carries the process's first allocations
        s.index()
        s.refine_patterns(cells, gradient="adjoint")
        r, t_index = timed(s.index)
        g, t_ref = timed(lambda: s.refine_patterns(cells, gradient="adjoint"))
        sw = r["sweep"].reshape(-1)
        out[prec] = {"value": round(n / (t_index + t_ref), 1), "index_s": round(t_index, 3), "refine_s": round(t_ref, 3),
                     "accepted_first_sweep": round(float((sw == 0).mean()), 4),
                     "accepted_second_sweep": round(float((sw == 1).mean()), 4),
                     "median_deg_indexed": median_deg(r["quaternions"]), "median_deg_refined": median_deg(g["quaternions"]),
                     "refine_rounds": int(g["rounds"])}
    s.configure(method="pca", dict_grid=96, pca_components=512, sweeps=1, bandwidth=64, precision=a.precision)
    _, t_build = timed(lambda: s.index_cells(cells[:4096]))  # the dictionary simulated and learned
    rp, t_pca = timed(s.index)
    out["pca"] = {"value": round(n / t_pca, 1), "index_s": round(t_pca, 3), "build_s": round(t_build, 3),
                  "median_deg": median_deg(rp["quaternions"]), "dictionary": 295389, "components": 512}
    line = {"metric": "patterns/s, 160x160 binned 2x, sweeps L=64 then L=128 and adjoint refinement, 1 B200",
            "value": out[a.precision]["value"], "unit": "patterns/s", "n_gpus": 1, "steps": 1, "warmup": 1,
            "higher_is_better": True, "dtype": "bf16+f32", "data": "synthetic",
            "config": {"workload": f"{rows}x{cols} scan of 160x160 uint16 patterns (1 000 000 in the configuration), "
                                   f"{GRAINS} Voronoi grains (0.5 deg spread), 432 master 401^2 (SH <= 96), binned 2x "
                                   "to 80x80; PCA dictionary 295 389 orientations, 512 components",
                       "patterns": n, "precision": a.precision},
            a.precision: out[a.precision], "fp32_form": out["f32"],
            "vs_fp32_form": round(out[a.precision]["value"] / out["f32"]["value"], 3), "pca_dictionary": out["pca"]}
    print(json.dumps(line), flush=True)


def target_main(a):
    """Indexing and six-unknown refinement of a --large-pattern scan (1 000 000 by default) of
    60 x 60 u16 patterns (the headline's master and grain map, 7.2 GB on the host): each form
    (BF16 and plain FP32) timed from the patterns on the host to the refined records, Solver.index
    (one pass at L = 64 with its 8-iteration refinement) then Solver.refine_patterns over every
    cell with the adjoint gradient (orientation and pattern centre, Levenberg-Marquardt). Two
    untimed index passes and one refinement first: the second pass makes the page-locked copy of
    the scan that the timed runs of both forms upload from. Accuracy: the median misorientation against the simulated
    orientations after each step, and the two forms against each other."""
    import torch

    import zebsdsolve_b200 as ze
    from zebsdsolve_b200 import synthetic as syn
    from zebsdsolve_b200.master import write_npz

    torch.cuda.set_device(0)
    tmp = tempfile.mkdtemp()
    sheets = syn.master_sheets(2, side=401, lmax=96, group="432", device="cuda")
    write_npz(f"{tmp}/m432.npz", sheets, 401, syn.group_matrices("432"), 30)
    side = int(math.isqrt(a.large))
    rows = cols = side
    n = rows * cols
    s = ze.Solver()
    s.add_phase(f"{tmp}/m432.npz")
    s.set_patterns(np.zeros((rows, cols, H, W), np.uint16))
    s.set_geometry(pc=PC, sample_tilt_deg=70.0, detector_tilt_deg=0.0)
    e = s._e
    rng = np.random.default_rng(100)
    q, _ = syn.grain_map(rng, rows, cols, GRAINS, SPREAD_DEG)
    pats = np.empty((n, H, W), np.uint16)
    for i in range(0, n, 16384):
        c = np.arange(i, min(n, i + 16384))
        pats[c] = syn.counted_patterns(e.simulate_device(0, c, q[c]), seed=i // 16384).cpu().numpy()
    s.set_patterns(pats.reshape(rows, cols, H, W))
    cells = np.arange(n)

    def med(quats):
        return round(float(np.median(np.degrees(s.disorientation(quats.reshape(-1, 4), q)))), 4)

    out, res = {}, {}
    for prec in (a.precision, "f32"):
        s.configure(precision=prec, bandwidth=L, sweeps=1)
        for _ in range(2):
            s.index()
        s.refine_patterns(cells, gradient="adjoint")  # (its buffers and plan made once, untimed)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = s.index()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        g = s.refine_patterns(cells, gradient="adjoint")
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        res[prec] = (r, g)
        out[prec] = {"value": round(n / (t2 - t0), 1), "index_s": round(t1 - t0, 3), "refine_s": round(t2 - t1, 3),
                     "index_value": round(n / (t1 - t0), 1), "median_deg_indexed": med(r["quaternions"]),
                     "median_deg_refined": med(g["quaternions"]), "refine_rounds": int(g["rounds"]),
                     "mean_ncc_refined": round(float(g["ncc"].mean()), 5)}

    def agree(x, y):
        d = np.degrees(s.disorientation(x.reshape(-1, 4), y.reshape(-1, 4)))
        return {"median_deg": round(float(np.median(d)), 5), "within_0.1deg": round(float((d < 0.1).mean()), 5)}

    rb, rf = res[a.precision], res["f32"]
    line = {"metric": "patterns/s indexed + refined over six unknowns (adjoint), 1M 60x60, 1 B200",
            "value": out[a.precision]["value"], "unit": "patterns/s", "n_gpus": 1, "steps": 1, "warmup": 2,
            "higher_is_better": True, "dtype": "bf16+f32", "data": "synthetic",
            "config": {"workload": f"{rows}x{cols} scan of 60x60 uint16 patterns, {GRAINS} Voronoi grains (0.5 deg "
                                   "spread), 432 master 401^2 (SH <= 96), L = 64, then Levenberg-Marquardt over "
                                   "orientation and pattern centre with the adjoint gradient",
                       "patterns": n, "precision": a.precision},
            a.precision: out[a.precision], "fp32_form": out["f32"],
            "vs_fp32_form": round(out[a.precision]["value"] / out["f32"]["value"], 3),
            "forms_agree": {"indexed": agree(rb[0]["quaternions"], rf[0]["quaternions"]),
                            "refined": agree(rb[1]["quaternions"], rf[1]["quaternions"])}}
    print(json.dumps(line), flush=True)


def _testdata(*parts):
    """The reference's test data: under $ZEBSDSOLVE_TESTDATA, else tests/data/ (filled by
    tests/golden/copy_testdata.sh); None where absent."""
    here = os.path.dirname(os.path.abspath(__file__))
    for base in (os.environ.get("ZEBSDSOLVE_TESTDATA"), os.path.join(here, "tests", "data")):
        if base and os.path.isfile(os.path.join(base, *parts)):
            return os.path.join(base, *parts)
    return None


def nickel_main(a):
    """The reference's real scan: kikuchipy's nickel scan (55 x 75 patterns of 60 x 60 u8, h5ebsd)
    read through this package's HDF5 reader and indexed against the nickel master (501^2, m-3m):
    one pass at L = 64, and two sweeps (L = 32, then 64 for the cells not accepted), each timed
    --steps times after --warmup untimed runs, from the patterns on the host to the results on
    the host (Solver.index); the orientations against the ones kikuchipy refined for the scan.
    Beside them the pattern-centre vote and the automatic geometry fit from a start 0.1 off in
    each coordinate, and the plane fit from the file's centre. The reference quotes 22 700 patterns/s (one pass) and 67 000 (two sweeps) on a
    desktop GPU, a median of 0.32 deg and 99.0 % within 3 deg."""
    import torch

    import zebsdsolve_b200 as ze

    scan, ni, qref = (_testdata("nickel", f) for f in ("patterns_v2.h5", "Ni_master_20kV.npz", "reference_quaternions.f32"))
    if scan is None or ni is None or qref is None:
        print(json.dumps({"workload": "nickel", "unavailable": "the reference's test data is not in tests/data "
                          "(tests/golden/copy_testdata.sh) nor under $ZEBSDSOLVE_TESTDATA"}), flush=True)
        return
    torch.cuda.set_device(0)
    q_ref = np.fromfile(qref, "<f4").reshape(-1, 4)
    t0 = time.perf_counter()
    s = ze.Solver()
    s.open(scan)
    t_open = time.perf_counter() - t0
    s.add_phase(ni)
    pc_file = np.array(s.geometry["pc"])
    n = 4125

    def accuracy(r):
        dis = np.degrees(s.disorientation(r["quaternions"].reshape(-1, 4), q_ref))
        return {"median_deg": round(float(np.median(dis)), 4), "within_3deg": round(float((dis < 3).mean()), 4),
                "mean_ncc": round(float(r["ncc"].mean()), 4), "accepted": round(float((r["sweep"] >= 0).mean()), 4),
                "first_sweep": round(float((r["sweep"] == 0).mean()), 4)}

    def timed_index():
        for _ in range(a.warmup):
            s.index()
        times = []
        for _ in range(a.steps):
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            r = s.index()
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t1)
        t = float(np.median(times))
        return {"value": round(n / t, 1), "ms": round(1e3 * t, 2), **accuracy(r)}

    s.configure(sweeps=1, bandwidth=64)
    one = timed_index()
    s.configure(sweeps=2, sweep_bandwidth=32, bandwidth=64)
    two = timed_index()
    # the BF16 form of the spectrum (hi + lo split for l <= 16; the headline's), same settings
    s.configure(sweeps=1, precision="bf16")
    one_bf16 = timed_index()
    s.configure(sweeps=2)
    two_bf16 = timed_index()
    s.configure(sweeps=1, precision="f32", nlpar=True)  # one pass of 7 x 7, lambda 0.7 (the defaults)
    averaged = timed_index()
    s.configure(nlpar=False)
    gan = _testdata("gan", "GaN_master_20kV.npz")
    phases = None
    if gan is not None:
        s.add_phase(gan)
        t1 = time.perf_counter()
        r2 = s.index()
        phases = {"s": round(time.perf_counter() - t1, 4), "nickel": round(float((r2["phase"] == 0).mean()), 4)}
        s.clear_phases()
        s.add_phase(ni)
    fits = {}
    # the vote, and the automatic fit (the vote, then the fit patterns' own source points and the
    # model they support), from a start 0.1 off in each coordinate; the plane fit from the file's
    # centre (the plane's pattern centre at the map's middle against the file's)
    for name, fn, start in (("vote_from_0.1_off", s.fit_pc, pc_file - 0.1),
                            ("fit_geometry_from_0.1_off", s.fit_geometry, pc_file - 0.1),
                            ("fit_plane_from_file_pc", s.fit_plane, pc_file)):
        s.set_geometry(pc=tuple(start))
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        out = fn()
        torch.cuda.synchronize()
        fits[name] = {"s": round(time.perf_counter() - t1, 3),
                      "off": round(float(np.abs(np.array(out["pc"]) - pc_file).max()), 5)}
        for k in ("model", "n_patterns"):
            if k in out:
                fits[name][k] = out[k]
        s.set_geometry(pc=tuple(pc_file), plane_kind="none")
    split = {}
    if a.kernel_split:  # device time by kernel over 5 calls in each form (CUPTI through torch.profiler)
        from torch.profiler import ProfilerActivity, profile

        for prec in ("f32", "bf16"):
            s.configure(precision=prec)
            s.index()
            torch.cuda.synchronize()
            with profile(activities=[ProfilerActivity.CUDA]) as prof:
                for _ in range(5):
                    s.index()
                torch.cuda.synchronize()
            rows_ = [(ev.key, ev.count, ev.self_device_time_total) for ev in prof.key_averages()
                     if ev.self_device_time_total > 0]
            total = sum(r[2] for r in rows_)
            rows_.sort(key=lambda r: -r[2])
            split[prec] = [{"kernel": k[:80], "launches": c, "us_per_call": round(t / 5, 1),
                            "share": round(t / total, 4)} for k, c, t in rows_[:12]]
            print(f"kernel split, precision {prec}, 5 index() calls, {total / 5:.0f} us of device time a call:",
                  file=sys.stderr)
            for r in split[prec]:
                print(f"  {r['share'] * 100:5.1f} %  {r['us_per_call']:8.1f} us/call  {r['launches']:3d}  {r['kernel']}",
                      file=sys.stderr)
        s.configure(precision="f32")
    s.close()
    line = {"metric": "patterns/s indexed, kikuchipy's nickel scan (55x75 of 60x60), L=64 one pass, 1 B200",
            "value": one["value"], "unit": "patterns/s", "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
            "higher_is_better": True, "dtype": "bf16+f32", "data": "kikuchipy nickel_ebsd_large (real, h5ebsd)",
            "config": {"workload": "nickel scan 55x75 of 60x60 u8, Ni master 501^2 (m-3m), defaults (precision f32, "
                                   "the drop-in form; bf16_* the BF16 form); timed from the patterns on the host to the "
                                   "results on the host (Solver.index)", "patterns": n},
            "one_pass": one, "two_sweeps": two, "bf16_one_pass": one_bf16, "bf16_two_sweeps": two_bf16,
            "nlpar_7x7": averaged, "nickel_and_gan": phases, "fits": fits, "open_s": round(t_open, 3),
            **({"kernel_split": split} if split else {}),
            "reference_published": {"one_pass": 22700, "two_sweeps": 67000, "median_deg": 0.32, "within_3deg": 0.99,
                                     "mean_ncc": 0.53, "nlpar_mean_ncc": 0.62, "nickel_of_two_phases": 0.999,
                                     "hardware": "desktop GPU"}}
    print(json.dumps(line), flush=True)


def match_main(a):
    """The dictionary match alone (zeb_match_bf16: BF16 tcgen05 GEMM with each pattern's eight best
    kept by the epilogue) on random unit rows: --patterns patterns × --entries entries ×
    --components values (the PCA configuration's shape by default: 16 384 × 65 536 × 512). Prints
    the kernel's TFLOP/s (CUDA events over --steps launches after --warmup)."""
    import ctypes

    import torch

    from zebsdsolve_b200 import _native as N
    from zebsdsolve_b200.dictionary import panel

    n, m, k = min(a.patterns, 16384), a.entries, a.components
    g = torch.Generator(device="cuda").manual_seed(7)
    x = torch.randn(n, k, generator=g, device="cuda")
    x /= x.norm(dim=1, keepdim=True)
    d = torch.randn(m, k, generator=g, device="cuda")
    d /= d.norm(dim=1, keepdim=True)
    xp, dp = panel(x), panel(d)
    sl = N.load().zeb_match_slices(n, m, k, 1)
    cv = torch.empty(n * sl * 8, device="cuda")
    ci = torch.empty(n * sl * 8, dtype=torch.int32, device="cuda")
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    P = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    sp = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def run():
        N.call("zeb_match_bf16", P(xp), n, P(dp), m, k, sl, P(cv), P(ci), P(st), sp)

    for _ in range(max(a.warmup, 1)):
        run()
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record()
    for _ in range(a.steps):
        run()
    t1.record()
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    ms = t0.elapsed_time(t1) / a.steps
    tf = 2.0 * n * m * k / (ms / 1e3) / 1e12
    print(json.dumps({"metric": "dictionary match TFLOP/s (BF16 tcgen05, top 8 kept in the epilogue), 1 B200",
                      "value": round(tf, 1), "unit": "TFLOP/s", "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
                      "ms_per_step": round(ms, 3), "higher_is_better": True, "dtype": "bf16", "data": "synthetic",
                      "config": {"workload": f"{n} patterns x {m} entries x {k} values, random unit rows",
                                 "slices": sl}}), flush=True)


def relaunch(a):
    """`--gpus N` (N > 1) run directly: the same command under torch.distributed.run, one process
    per GPU of this node (rendezvous on 127.0.0.1); returns its exit status."""
    import socket

    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={a.gpus}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


if __name__ == "__main__":
    args = parse()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(relaunch(args))
    if args.impl == "reference":
        reference_main(args)
    elif args.workload == "adjoint":
        adjoint_main(args)
    elif args.workload == "uneven":
        uneven_main(args)
    elif args.workload == "pcfit":
        pcfit_main(args)
    elif args.workload == "plane":
        plane_main(args)
    elif args.workload == "large":
        large_main(args)
    elif args.workload == "nickel":
        nickel_main(args)
    elif args.workload == "match":
        match_main(args)
    elif args.workload == "target":
        target_main(args)
    else:
        device_main(args)
