"""Pattern preprocessing (oracle restatement of zebsdsolve `src/prep.zig` and `shaders/prep.wgsl`):
unpack, static background, dynamic (Gaussian) background, zero mean / unit norm under the mask.
Statistics in float64; the blur weights follow the kernels' definitions."""
import math

import numpy as np


def masked(h, w, mask):
    """prep.wgsl:399-403 — boolean [h, w] of the pixels under the circular mask."""
    r = np.arange(h)[:, None] - mask[0]
    c = np.arange(w)[None, :] - mask[1]
    if mask[2] <= 0:
        return np.ones((h, w), bool)
    return r * r + c * c <= mask[2]


def blur_direct(img, sigma):
    """prep.zig:108-118, prep.wgsl:87-164 — separable Gaussian (taps to ceil(3σ)), renormalized
    over the taps inside the image."""
    radius = max(1, int(math.ceil(3 * sigma)))
    k0 = 1.0 / (2 * sigma * sigma)
    out = np.asarray(img, np.float64)
    for axis in (1, 0):
        n = out.shape[axis]
        x = np.arange(n)
        d = np.abs(x[:, None] - x[None, :])
        g = np.where(d <= radius, np.exp(-(d * d) * k0), 0.0)
        g = g / g.sum(1, keepdims=True)
        out = out @ g.T if axis == 1 else g @ out
    return out


def _cell(jr, n, s):
    """prep.wgsl:176-183 — centre and width of coarse cell jr along an axis of n pixels."""
    lo = jr * s
    hi = lo + s
    if jr >= 0 and lo < n:
        hi = min(hi, n)
    return 0.5 * (lo + hi - 1), float(hi - lo)


def blur_wide(img, sigma):
    """prep.zig:120-139, prep.wgsl:165-284 — the wide Gaussian from box sums: boxes of s = ⌊σ/6⌋
    pixels, a coarse Gaussian over the box sums, and a narrow spread of deviation s back to the
    pixels; sums and counts are carried together and divided at the end."""
    img = np.asarray(img, np.float64)
    h, w = img.shape
    s = int(math.floor(sigma / 6))
    coarse_sigma = math.sqrt(sigma * sigma - s * s - (s * s - 1) / 12)
    cpad = 3
    radius = int(math.ceil(4 * coarse_sigma))
    kx = 1.0 / (2 * coarse_sigma * coarse_sigma)
    kz = 1.0 / (2 * s * s)
    hs = (h + s - 1) // s
    ws = (w + s - 1) // s
    wp = ws + 2 * cpad
    hp = hs + 2 * cpad
    box = np.zeros((hs, ws, 2))
    for i in range(hs):
        for j in range(ws):
            r1 = min((i + 1) * s, h)
            c1 = min((j + 1) * s, w)
            box[i, j, 0] = img[i * s:r1, j * s:c1].sum()
            box[i, j, 1] = (r1 - i * s) * (c1 - j * s)
    rows = np.zeros((hs, wp, 2))
    for t in range(wp):
        c = _cell(t - cpad, w, s)[0]
        j0 = max(int(math.floor((c - radius) / s)), 0)
        j1 = min(int(math.floor((c + radius) / s)), ws - 1)
        for j in range(j0, j1 + 1):
            d = _cell(j, w, s)[0] - c
            rows[:, t] += math.exp(-d * d * kx) * box[:, j]
    cols = np.zeros((hp, wp, 2))
    for t in range(hp):
        c = _cell(t - cpad, h, s)[0]
        i0 = max(int(math.floor((c - radius) / s)), 0)
        i1 = min(int(math.floor((c + radius) / s)), hs - 1)
        for i in range(i0, i1 + 1):
            d = _cell(i, h, s)[0] - c
            cols[t] += math.exp(-d * d * kx) * rows[i]
    spread = np.zeros((hp, w, 2))
    for x in range(w):
        own = x // s
        for t in range(2 * cpad + 1):
            cx, cw = _cell(own + t - cpad, w, s)
            d = x - cx
            spread[:, x] += cw * math.exp(-d * d * kz) * cols[:, own + t]
    out = np.zeros((h, w))
    for y in range(h):
        own = y // s
        acc = np.zeros((w, 2))
        for t in range(2 * cpad + 1):
            cy, cw = _cell(own + t - cpad, h, s)
            d = y - cy
            acc += cw * math.exp(-d * d * kz) * spread[own + t]
        out[y] = acc[:, 0] / acc[:, 1]
    return out


def blur(img, sigma):
    """prep.zig:108-140 — direct below σ = 12 pixels, else from box sums."""
    if math.floor(sigma / 6) < 2:
        return blur_direct(img, sigma)
    return blur_wide(img, sigma)


def normalize(img, mask):
    """prep.wgsl:405-443 — zero mean and unit norm under the mask, zero outside it."""
    h, w = img.shape
    m = masked(h, w, mask)
    v = np.asarray(img, np.float64)
    mean = v[m].sum() / max(m.sum(), 1)
    out = np.where(m, v - mean, 0.0)
    ss = (out * out).sum()
    return out / math.sqrt(max(ss, 1e-30))


def stretch(img):
    """prep.wgsl stretch — an image to [0, 1] between its extremes (float32)."""
    f = np.float32
    v = np.asarray(img, f)
    lo, hi = v.min(), v.max()
    k = f(1) / max(f(hi - lo), f(1e-20))
    return ((v - lo) * k).astype(f)


def clahe(img, tiles, bins, clip):
    """prep.wgsl clahe_hist / clahe_cdf / clahe_apply (prep.zig:167-188) on one image, float32
    as the kernels round: the image stretched to [0, 1]; padded by reflection at its top and left
    to a whole number of tiles; each tile's histogram clipped at clip × the mean count per level,
    the cut spread evenly (the remainder one count each to the first levels) and cumulated; each
    pixel from its four nearest tiles' tables, between its two nearest levels."""
    f = np.float32
    v = stretch(img)
    h, w = v.shape
    pad_h, pad_w = (tiles - h % tiles) % tiles, (tiles - w % tiles) % tiles
    th, tw = max(1, (h + pad_h) // tiles), max(1, (w + pad_w) // tiles)

    def reflect(i, n, pad):
        if n <= 1:
            return np.zeros_like(i)
        x = np.abs(i - pad)
        x = np.where(x >= n, 2 * n - 2 - x, x)
        return np.clip(x, 0, n - 1)

    py, px = np.arange(h + pad_h), np.arange(w + pad_w)
    padded = np.clip(v[reflect(py, h, pad_h)][:, reflect(px, w, pad_w)], f(0), f(1))
    top = f(bins - 1)
    level = np.clip(padded * top, f(0), top).astype(np.int64)
    hist = np.zeros((tiles, tiles, bins), np.int64)
    np.add.at(hist, ((py // th)[:, None].repeat(len(px), 1), (px // tw)[None, :].repeat(len(py), 0), level), 1)
    voxels, nb = f(max(th * tw, 1)), f(bins)
    limit = max(f(f(f(clip) * voxels) / nb), f(1))
    cdf = np.empty((tiles, tiles, bins), f)
    for ty in range(tiles):
        for tx in range(tiles):
            c = np.minimum(hist[ty, tx].astype(f), limit)
            sumc = f(0)
            for x in c:
                sumc = f(sumc + x)
            clipped = f(voxels - sumc)
            residual = int(f(clipped - f(nb * f(np.floor(f(clipped / nb))))))
            redist = f(f(clipped - f(residual)) / nb)
            acc = f(0)
            for i in range(bins):
                ci = f(c[i] + redist)
                if i < residual:
                    ci = f(ci + f(1))
                acc = f(acc + ci)
                cdf[ty, tx, i] = min(max(f(acc / voxels), f(0)), f(1))

    def mix(a, b, t):
        return (a * (f(1) - t)).astype(f) + (b * t).astype(f)

    tl = f(tiles - 1)
    gy = ((np.arange(h, dtype=f) + f(0.5)) / f(h) * tl).astype(f)
    gx = ((np.arange(w, dtype=f) + f(0.5)) / f(w) * tl).astype(f)
    y0, x0 = np.floor(gy).astype(np.int64), np.floor(gx).astype(np.int64)
    y1, x1 = np.minimum(y0 + 1, tiles - 1), np.minimum(x0 + 1, tiles - 1)
    fy, fx = (gy - y0.astype(f))[:, None], (gx - x0.astype(f))[None, :]
    vv = np.clip(v, f(0), f(1))
    bf = (vv * f(bins - 1)).astype(f)
    b0 = np.clip(np.floor(bf), 0, bins - 2).astype(np.int64)
    fb = (bf - b0.astype(f)).astype(f)

    def look(yy, xx):
        t = cdf[yy[:, None], xx[None, :]]
        lo = np.take_along_axis(t, b0[..., None], -1)[..., 0]
        hi = np.take_along_axis(t, b0[..., None] + 1, -1)[..., 0]
        return mix(lo, hi, fb)

    return mix(mix(look(y0, x0), look(y0, x1), fx), mix(look(y1, x0), look(y1, x1), fx), fy).astype(f)


def run(raw, static=None, dynamic="subtract", dynamic_sigma=0.0, mask=(0.0, 0.0, 0.0), do_normalize=True,
        clahe_opts=None, bandpass=None):
    """prep.zig:143-204, 263-272 — one pattern [h, w] (any integer or float dtype) through the
    filter chain: static background, dynamic background, CLAHE (clahe_opts = (tiles, bins,
    clip)), band pass (bandpass = (fine, coarse) deviations in pixels: the fine blur less the
    coarse, the fine one skipped below 0.05), then the mask and normalization."""
    img = np.asarray(raw).astype(np.float64)
    if static is not None:
        img = img - np.asarray(static, np.float64)
    if dynamic != "none" and dynamic_sigma > 0:
        bg = blur(img, dynamic_sigma)
        img = img - bg if dynamic == "subtract" else img / np.maximum(bg, 1e-6)
    if clahe_opts is not None:
        img = clahe(img, *clahe_opts).astype(np.float64)
    if bandpass is not None and bandpass[1] > 0:
        fine = blur(img, bandpass[0]) if bandpass[0] > 0.05 else img
        img = fine - blur(img, bandpass[1])
    if do_normalize:
        img = normalize(img, mask)
    return img


def reduced_shape(h, w, factor):
    """reduce.zig:12-19 — floor(size / factor) each way."""
    return int(math.floor(h / factor + 1e-9)), int(math.floor(w / factor + 1e-9))


def reduce(pixels, factor):
    """reduce.zig:44-131 — one pattern reduced by `factor`: for a whole factor the mean of each
    k × k block; otherwise area resampling (each output pixel the average of the source area it
    covers, partly covered pixels weighted by the part). From the top-left corner; the remainder
    of the last row and column is dropped. FP64."""
    p = np.asarray(pixels, np.float64)
    H, W = p.shape
    h, w = reduced_shape(H, W, factor)
    if abs(factor - round(factor)) < 1e-9:
        k = int(round(factor))
        return p[: h * k, : w * k].reshape(h, k, w, k).sum((1, 3)) / (k * k)

    def weights(n_out, n_src):
        # M[o, s]: the part of source pixel s inside output pixel o's span [o·f, (o+1)·f)
        M = np.zeros((n_out, n_src))
        for o in range(n_out):
            x0, x1 = o * factor, (o + 1) * factor
            j = int(math.floor(x0))
            while j < x1 - 1e-12 and j < n_src:
                M[o, j] = min(x1, j + 1) - max(x0, j)
                j += 1
        return M

    return weights(h, H) @ p @ weights(w, W).T / (factor * factor)
