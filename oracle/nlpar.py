"""Non-local pattern averaging: oracle restatement of zebsdsolve `shaders/nlpar.wgsl` and
`src/nlpar.zig` over a whole map at once (test infrastructure — what zeb_nlpar and the engine's
windows are tested against, never part of the product path).

For a map of stored patterns P[r, c] (FP64): σ²(i) = ½ min over the eight nearest neighbours of
the mean squared difference (0 without neighbours); then `passes` passes, each over the
(2·radius + 1)² window of every cell: d²(i, j) on the current patterns; e(i, j) = Σ_u (a_i[u] −
a_j[u − o])² σ²(i + u) from each average's shares a of the stored patterns (σ²(i) + σ²(j) in the
first pass); w = 1 where d² ≤ e, exp(−sqrt(N/2)(d²/e − 1)/λ²) where e > 0, else 0; the cell's own
weight 1; the average Σ w P / Σ w and its shares Σ w a_j[· − o] / Σ w. Returns the averages and
each cell's shares over (2·radius·passes + 1)² offsets (nlpar.wgsl:1-45, 96-243).
"""
import math

import numpy as np


def _moved(a, dy, dx, fill):
    """b[y, x] = a[y + dy, x + dx] over the first two axes, `fill` off the map."""
    out = np.full(a.shape, fill, dtype=a.dtype)
    rows, cols = a.shape[:2]
    ys, yd = slice(max(dy, 0), rows + min(dy, 0)), slice(max(-dy, 0), rows + min(-dy, 0))
    xs, xd = slice(max(dx, 0), cols + min(dx, 0)), slice(max(-dx, 0), cols + min(-dx, 0))
    out[yd, xd] = a[ys, xs]
    return out


def average(pats, radius, passes, lam):
    """pats [rows, cols, h, w] → (averages [rows, cols, h, w], shares [rows, cols, S, S])."""
    rows, cols = pats.shape[:2]
    P = pats.reshape(rows, cols, -1).astype(np.float64)
    npx = P.shape[-1]
    reach = radius * passes
    S = 2 * reach + 1
    on = np.ones((rows, cols), bool)

    def d2(A, dy, dx):
        return ((A - _moved(A, dy, dx, 0.0)) ** 2).mean(-1)

    # the stored patterns' noise
    least = np.full((rows, cols), np.inf)
    for dy in (-1, 0, 1):
        for dx in (-1, 0, 1):
            if dy or dx:
                least = np.minimum(least, np.where(_moved(on, dy, dx, False), d2(P, dy, dx), np.inf))
    sig = 0.5 * np.where(np.isfinite(least), least, 0.0)
    # σ² of the stored pattern at each offset u from each cell: [rows, cols, S, S]
    sig_at = np.zeros((rows, cols, S, S))
    for uy in range(-reach, reach + 1):
        for ux in range(-reach, reach + 1):
            sig_at[:, :, uy + reach, ux + reach] = _moved(sig, uy, ux, 0.0)
    shares = np.zeros((rows, cols, S, S))
    shares[:, :, reach, reach] = 1.0
    offsets = [(dy, dx) for dy in range(-radius, radius + 1) for dx in range(-radius, radius + 1) if dy or dx]
    for _ in range(passes):
        total = np.ones((rows, cols))
        acc = P.copy()
        new = shares.copy()
        for dy, dx in offsets:
            # the neighbour's shares, seen from this cell: theirs[u] = a_j[u − o]
            theirs = _moved(shares, dy, dx, 0.0)
            theirs = np.roll(np.roll(theirs, dy, axis=2), dx, axis=3)
            if dy > 0:
                theirs[:, :, :dy, :] = 0
            elif dy < 0:
                theirs[:, :, dy:, :] = 0
            if dx > 0:
                theirs[:, :, :, :dx] = 0
            elif dx < 0:
                theirs[:, :, :, dx:] = 0
            e = ((shares - theirs) ** 2 * sig_at).sum((2, 3))
            d = d2(P, dy, dx)
            with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
                w = np.where(d <= e, 1.0, np.where(e > 0, np.exp(-math.sqrt(npx / 2) * (d / e - 1) / lam ** 2), 0.0))
            w = np.where(_moved(on, dy, dx, False), w, 0.0)
            acc += w[..., None] * _moved(P, dy, dx, 0.0)
            new += w[..., None, None] * theirs
            total += w
        P = acc / total[..., None]
        shares = new / total[..., None, None]
    return P.reshape(pats.shape), shares
