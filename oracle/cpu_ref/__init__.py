"""The C++ FP32 restatement of the oracle's per-pattern path (cpu_ref.cpp), timed on the host cores
as the CPU baseline (test and measurement infrastructure: only tests/, the bench's CPU legs and
smoke() use it; the product never does).

CpuRef(scan) takes an oracle.pipeline.Scan (the oracle's FP64 tables for one phase, bandwidth and
detector) and runs Scan.index's steps in single precision with host threads over the patterns:
index(raws, ts) gives, per stored pattern, the refined orientation reduced to the fundamental zone,
its NCC, NMI, last improving step, and the spherical peak's score.
"""
import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SRC = HERE / "cpu_ref.cpp"
LIB = HERE / "libcpu_ref.so"

# x86-64-v3 (AVX2, FMA): what the hosts here and the GPU boxes run, so the library built in one
# place runs in the other; complex products by the textbook formula (finite values throughout)
FLAGS = ["-O3", "-std=c++17", "-march=x86-64-v3", "-fcx-limited-range", "-pthread", "-fPIC", "-shared"]


def build(force=False):
    """Compile cpu_ref.cpp into libcpu_ref.so beside it (g++, std::thread); returns the path."""
    if force or not LIB.exists() or LIB.stat().st_mtime < SRC.stat().st_mtime:
        cmd = [os.environ.get("CXX", "g++"), *FLAGS, str(SRC), "-o", str(LIB)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"cpu_ref build failed:\n{r.stderr}")
    return LIB


F = ctypes.POINTER(ctypes.c_float)


class _Tables(ctypes.Structure):
    _fields_ = [("h", ctypes.c_int), ("w", ctypes.c_int), ("static_bg", F), ("dynamic", ctypes.c_int),
                ("sigma", ctypes.c_float), ("mask", ctypes.c_float * 3), ("c0", ctypes.c_float * 3),
                ("c1", ctypes.c_float * 3), ("c2", ctypes.c_float * 3), ("L", ctypes.c_int), ("n_theta", ctypes.c_int),
                ("n_phi", ctypes.c_int), ("dirs", F), ("glw", F), ("plm", F), ("n", ctypes.c_int), ("nc", ctypes.c_int),
                ("fold", ctypes.c_int), ("mu_max", ctypes.c_int), ("wig", F), ("f", F), ("rden", F),
                ("side", ctypes.c_int), ("grad", F), ("sheets", F), ("iters", ctypes.c_int),
                ("max_step", ctypes.c_float), ("nmi_bins", ctypes.c_int)]


def _f32(a):
    return np.ascontiguousarray(np.asarray(a), np.float32)


def _ptr(a):
    return a.ctypes.data_as(F) if a is not None else None


class CpuRef:
    """The scan's tables in FP32 for the C++ path (kept alive with the struct that points at them)."""

    def __init__(self, scan):
        from .. import spherical as osp

        if scan.dynamic != "none" and scan.sigma > 0 and int(scan.sigma // 6) >= 2:
            raise ValueError("cpu_ref: the wide background blur (sigma >= 12 pixels) is not restated")
        self.scan = scan
        tb, pt = scan.tb, scan.pt
        self._keep = {
            "static": _f32(scan.static.reshape(-1)) if scan.static is not None else None,
            "dirs": _f32(tb.grid.directions().reshape(-1)),
            "glw": _f32(tb.grid.w),
            "plm": _f32(tb.grid.plm),
            "wig": _f32(np.concatenate([b.reshape(-1) for b in osp._wigner_blocks(tb)])),
            "f": _f32(np.stack([np.real(pt.f), np.imag(pt.f)], -1).reshape(-1)),
            "rden": _f32(scan.rden.reshape(-1)),
            "grad": _f32(scan.grad.reshape(-1)),
            "sheets": _f32(scan.sheets.reshape(-1)),
        }
        k = self._keep
        c0, c1, c2 = scan.frame
        self.t = _Tables(
            h=scan.h, w=scan.w, static_bg=_ptr(k["static"]),
            dynamic={"none": 0, "subtract": 1, "divide": 2}[scan.dynamic] if scan.sigma > 0 else 0,
            sigma=float(scan.sigma), mask=(ctypes.c_float * 3)(*map(float, scan.mask)),
            c0=(ctypes.c_float * 3)(*map(float, c0)), c1=(ctypes.c_float * 3)(*map(float, c1)),
            c2=(ctypes.c_float * 3)(*map(float, c2)), L=tb.L, n_theta=tb.n_theta, n_phi=tb.n_phi,
            dirs=_ptr(k["dirs"]), glw=_ptr(k["glw"]), plm=_ptr(k["plm"]), n=tb.n, nc=pt.nc, fold=pt.fold,
            mu_max=pt.mu_max, wig=_ptr(k["wig"]), f=_ptr(k["f"]), rden=_ptr(k["rden"]), side=scan.side,
            grad=_ptr(k["grad"]), sheets=_ptr(k["sheets"]), iters=scan.iters if scan.refine_on else 0,
            max_step=float(scan.max_step), nmi_bins=scan.nmi_bins)
        self.lib = ctypes.CDLL(str(build()))
        self.lib.zcr_index.argtypes = [ctypes.POINTER(_Tables), ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_int]
        self.lib.zcr_index.restype = ctypes.c_int
        self.lib.zcr_threads.restype = ctypes.c_int

    def threads(self):
        return int(self.lib.zcr_threads())

    def index(self, raws, ts=None, threads=0):
        """raws: stored u16 patterns [n][h][w]; ts: their detector positions [n][3] (pixels; the
        map centre's by default); threads: host threads (0: one a hardware thread).
        Returns a list of records like Scan.index's (q in the fundamental zone, ncc, nmi, step,
        peak_score)."""
        from .. import sym as osym

        raws = np.ascontiguousarray(np.asarray(raws), np.uint16).reshape(-1, self.scan.h * self.scan.w)
        n = raws.shape[0]
        ts = np.ascontiguousarray(np.broadcast_to(self.scan.t0 if ts is None else np.asarray(ts, np.float64),
                                                  (n, 3)), np.float64)
        out = np.zeros((n, 8), np.float32)
        self.lib.zcr_index(ctypes.byref(self.t), n, raws.ctypes.data, ts.ctypes.data, out.ctypes.data, int(threads))
        q = [osym.to_fz(x, self.scan.rotations) for x in out[:, :4].astype(np.float64)]
        return [{"q": q[i], "ncc": float(out[i, 4]), "nmi": float(out[i, 5]), "step": float(out[i, 6]),
                 "peak_score": float(out[i, 7])} for i in range(n)]
