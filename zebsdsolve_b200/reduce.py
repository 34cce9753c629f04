"""Host-side reduction of one image by `settings.binning` (reduce.zig:44-131): the k × k blocks'
means for a whole factor, area resampling for any other; floor(size / factor) each way from the
top-left corner. The patterns themselves are reduced on the device as they are unpacked
(`zeb_prep_reduced`); this serves the static background, which is averaged on the host."""
import math

import numpy as np


def reduced_shape(h, w, factor):
    """reduce.zig:12-19"""
    return int(math.floor(h / factor + 1e-9)), int(math.floor(w / factor + 1e-9))


def _weights(n_out, n_src, factor):
    m = np.zeros((n_out, n_src))
    for o in range(n_out):
        x0, x1 = o * factor, (o + 1) * factor
        j = int(math.floor(x0))
        while j < x1 - 1e-12 and j < n_src:
            m[o, j] = min(x1, j + 1) - max(x0, j)
            j += 1
    return m


def reduce_image(img, factor):
    a = np.asarray(img, np.float64)
    if factor == 1:
        return a
    h, w = reduced_shape(a.shape[0], a.shape[1], factor)
    if abs(factor - round(factor)) < 1e-9:
        k = int(round(factor))
        return a[: h * k, : w * k].reshape(h, k, w, k).sum((1, 3)) / (k * k)
    return _weights(h, a.shape[0], factor) @ a @ _weights(w, a.shape[1], factor).T / (factor * factor)
