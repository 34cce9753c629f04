"""The C++ FP32 restatement of the path (oracle/cpu_ref, the CPU baseline the bench times) against
the FP64 oracle it restates (oracle/pipeline.py Scan.index), pattern by pattern, on the host.

A seeded 432 master (151², SH <= 28), patterns simulated by the oracle's projection at uniform
orientations with Poisson counts, the reference's default filters, L = 16 and 32. Bounds (FP32
against FP64): the refined orientation within 0.05° (modulo the group), NCC within 1e-4, the
peak's score within 1e-5, NMI within 5e-3 (a pixel may change histogram bin).
"""
import math

import numpy as np
import pytest

import oracle.cpu_ref as ocr
import oracle.detector as od
import oracle.geometry as og
import oracle.pipeline as opl
import oracle.sym as osym


@pytest.fixture(scope="module")
def master():
    from zebsdsolve_b200 import synthetic as syn

    sheets = np.asarray(syn.master_sheets(3, side=151, lmax=28, group="432", device="cpu"), np.float64)
    return sheets.reshape(-1), syn.group_matrices("432"), syn.uniform_quaternions(np.random.default_rng(5), 6)


@pytest.mark.parametrize("L,h", [(16, 40), (32, 48)])
def test_cpu_ref_equals_the_oracle(master, L, h):
    sheets, ops, qs = master
    geo = og.Geometry(pc=(0.5, 0.3, 0.6), sample_tilt_deg=70.0)
    scan = opl.Scan(sheets, 151, ops, geo, h, h, L)
    rng = np.random.default_rng(L)
    raws = []
    for q in qs:
        p = od.project(scan.sheets, 151, scan.frame, scan.t0, q, h, h)
        p = 1000 * (0.6 + 0.4 * (p - p.min()) / (p.max() - p.min()))
        raws.append(np.minimum(rng.poisson(p), 65535).astype(np.uint16))
    raws = np.stack(raws)
    want = [scan.index(r) for r in raws]
    got = ocr.CpuRef(scan).index(raws, threads=2)
    for a, b in zip(got, want):
        dis = math.degrees(float(osym.disorientation(np.asarray(a["q"])[None], np.asarray(b["q"])[None],
                                                     scan.rotations)[0]))
        assert dis <= 0.05, dis
        assert abs(a["ncc"] - b["ncc"]) <= 1e-4, (a["ncc"], b["ncc"])
        assert abs(a["peak_score"] - b["peak_score"]) <= 1e-5, (a["peak_score"], b["peak_score"])
        assert abs(a["nmi"] - b["nmi"]) <= 5e-3, (a["nmi"], b["nmi"])
