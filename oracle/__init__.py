"""CPU oracle for the spherical cross-correlation indexing path (TEST INFRASTRUCTURE).

This package is a plain NumPy (float64) restatement of the reference's algorithm, written
from zebsdsolve 0.2.8's Zig host math (`src/sh.zig`, `src/master.zig`, `src/lambert.zig`,
`src/geometry.zig`, `src/rot.zig`, `src/sym.zig`, `src/spherical.zig`, `src/engine.zig`)
and its WGSL compute kernels (`shaders/common.wgsl`, `sphere.wgsl`, `so3.wgsl`,
`detector.wgsl`, `mastersph.wgsl`, `prep.wgsl`).  Every function cites the reference
file:line it follows.

It is the oracle, never the product: only `tests/`, `__graft_entry__.smoke()` and the
`cpu_baseline` / `--impl reference` legs of `bench.py` may import it.  The product path
(`zebsdsolve_b200`) never imports it and fails loudly when its CUDA library is missing.

Pinning: the reference engine cannot be built here (Zig and wgpu-native are absent and its
GPU path needs a graphics API), so the oracle is pinned by the reference's own known-answer
tests restated as pytest cases (the `test` blocks of `sh.zig`, `lambert.zig`,
`geometry.zig`, `settings.zig`, `master.zig`) and by the reference's test data read as
plain arrays.  Bit-level parity with the reference's FP32 WGSL arithmetic is not pinned:
the reference's tests themselves only pin it through tolerances.
"""
