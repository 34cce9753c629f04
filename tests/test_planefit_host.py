"""The plane fit's host arithmetic (zebsdsolve_b200.planefit) against the oracle's scalar
restatement of planefit.zig: each pattern's NCC, gradient and Gauss–Newton matrix from its 43
sums (localOf), the damped systems (damped), the batched pivoted elimination (solve), and the
information a pattern holds on its source with its rotation profiled out."""
import numpy as np

import oracle.detector as od
from zebsdsolve_b200 import planefit as pf


def _sums(rng, n):
    """43 sums of plausible patterns: n pixels, values and directions drawn at random."""
    out = np.zeros((n, 43), np.float32)
    for b in range(n):
        m = rng.normal(size=500)
        e = 0.6 * m + rng.normal(size=500)
        e = (e - e.mean()) / np.linalg.norm(e - e.mean())
        d = rng.normal(size=(500, 6))
        s = [500.0, m.sum(), (m * m).sum(), (m * e).sum()]
        s += list(d.sum(0)) + list((m[:, None] * d).sum(0)) + list((e[:, None] * d).sum(0))
        s += [(d[:, i] * d[:, j]).sum() for i in range(6) for j in range(i, 6)]
        out[b] = s
    return out


def test_local_of_matches_oracle():
    rng = np.random.default_rng(1)
    S = _sums(rng, 12)
    S[5, 1:] = 0  # a flat simulation: no variance, not ok
    ok, ncc, g, H = pf.local_of(S)
    for b in range(len(S)):
        ref = od.local_of(S[b].astype(np.float64))
        if ref is None:
            assert not ok[b] and ncc[b] == 0 and not g[b].any()
            continue
        assert ok[b]
        assert abs(ncc[b] - ref[0]) < 1e-12 and np.allclose(g[b], ref[1], rtol=1e-10, atol=1e-12)
        assert np.allclose(H[b], ref[2], rtol=1e-10, atol=1e-12)


def test_batched_elimination_matches_the_scalar_one():
    rng = np.random.default_rng(2)
    for k in (3, 6):
        A = rng.normal(size=(40, k, k))
        A[7] = 0  # singular
        A[8, :, 0] = 0
        b = rng.normal(size=(40, k))
        x, ok = pf.solve_batch(A, b)
        for i in range(40):
            ref = od.solve_pivot(A[i], b[i]) if k == 6 else None
            if i in (7, 8):
                assert not ok[i] and not x[i].any()
                continue
            assert ok[i] and np.allclose(A[i] @ x[i], b[i], atol=1e-9)
            if ref is not None:
                assert np.allclose(x[i], ref, rtol=1e-12, atol=1e-12)


def test_damped_systems_match_oracle():
    rng = np.random.default_rng(3)
    S = _sums(rng, 6)
    ok, ncc, g, H = pf.local_of(S)
    lam = rng.uniform(1e-4, 1e2, 6)
    A6, g6 = pf.damped(6, H, g, lam)
    for b in range(6):
        rA, rg = od.damped(H[b], g[b], lam[b])
        assert np.array_equal(A6[b], rA) and np.array_equal(g6[b], rg)
    A3, g3 = pf.damped(3, H, g, lam)
    assert np.array_equal(g3, g[:, 3:])
    tr = np.trace(H[:, 3:, 3:], axis1=1, axis2=2)
    assert np.allclose(np.diagonal(A3, axis1=1, axis2=2),
                       np.diagonal(H[:, 3:, 3:], axis1=1, axis2=2) * (1 + lam[:, None]) + 1e-9 * tr[:, None] + 1e-30)


def test_profiled_information_is_the_schur_complement():
    rng = np.random.default_rng(4)
    S = _sums(rng, 8)
    ok, ncc, g, H = pf.local_of(S)
    St, gt, good = pf.profiled(H, g)
    assert good.all()
    for b in range(8):
        B = H[b, 3:, 3:] + np.eye(3) * (1e-9 * np.trace(H[b, 3:, 3:]) + 1e-30)
        want = H[b, :3, :3] - H[b, :3, 3:] @ np.linalg.solve(B, H[b, 3:, :3])
        assert np.allclose(St[b], 0.5 * (want + want.T), rtol=1e-9, atol=1e-12)
        assert np.allclose(gt[b], g[b, :3] - H[b, :3, 3:] @ np.linalg.solve(B, g[b, 3:]), rtol=1e-9, atol=1e-12)
