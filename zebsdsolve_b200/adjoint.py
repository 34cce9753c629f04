"""Refinement of six unknowns per pattern on the detector: the source's shift (equivalently its
pattern centre) and the crystal's orientation (config 3; the per-pattern step of the reference's
plane fit, `planefit.zig:570-622` settle with k = 6, Winkelmann et al. / kikuchipy's
refine_orientation_projection_center).

`ProjectedNCC` is the detector projection + NCC as a `torch.autograd.Function`: forward and
backward are the CUDA kernels of `zeb_det6` (mode 0 and mode 1); the backward recomputes the
projection of every pixel from the parameters instead of keeping the projected patterns.
`refine6` runs the reference's Levenberg–Marquardt settle over all the given patterns at once,
with the damped 6 × 6 solve in FP64 on the device (`zeb_solve6`) and the Gauss–Newton matrix
from the reference's 43 sums (`zeb_det6` mode 2); the gradient is the reference's (the gradient
table's) or the exact adjoint's (the kernel behind ProjectedNCC's backward).
"""
import ctypes

import numpy as np
import torch

from . import _native as N
from .device import ptr, stream_ptr


class Plan:
    """What a batch of patterns needs besides its parameters: preprocessed patterns, items,
    frame, and the master's pair tables."""

    def __init__(self, pats, items, frame, vpair, gpair, side, pixels=None):
        self.pats, self.items, self.frame = pats, items, frame
        self.vpair, self.gpair, self.side = vpair, gpair, side
        self.pixels = pixels  # the frame's masked-pixel list (zeb_mask_list), or None
        self.n = items.shape[0]

    def run(self, mode, x, q0):
        width = (1, 7, 43, 61)[mode]
        out = torch.empty(self.n * width, dtype=torch.float32, device=x.device)
        if self.pixels is not None:
            N.call("zeb_det6_list", mode, ptr(self.pats), ptr(self.items), self.n, ctypes.byref(self.frame),
                   ptr(self.pixels), self.pixels.numel(), ptr(self.vpair), ptr(self.gpair), self.side, ptr(x), ptr(q0),
                   ptr(out), stream_ptr())
        else:
            N.call("zeb_det6", mode, ptr(self.pats), ptr(self.items), self.n, ctypes.byref(self.frame),
                   ptr(self.vpair), ptr(self.gpair), self.side, ptr(x), ptr(q0), ptr(out), stream_ptr())
        return out.view(self.n, width) if width > 1 else out


class ProjectedNCC(torch.autograd.Function):
    """NCC[b] of pattern b with the master projected at x[b] = (δt (pixels), φ (radians)) about
    its base orientation q0[b]; backward by the hand-written adjoint kernel."""

    @staticmethod
    def forward(ctx, x, q0, plan):
        x = x.detach().to(torch.float32).contiguous()
        q0 = q0.detach().to(torch.float32).contiguous()
        ctx.save_for_backward(x, q0)
        ctx.plan = plan
        return plan.run(0, x, q0).clone()

    @staticmethod
    def backward(ctx, grad_out):
        x, q0 = ctx.saved_tensors
        res = ctx.plan.run(1, x, q0)  # the projection recomputed, its derivatives summed
        return grad_out.to(torch.float32)[:, None] * res[:, :6], None, None


def projected_ncc(x, q0, plan):
    return ProjectedNCC.apply(x, q0, plan)


def pc_jacobian(geo, rows, cols):
    """∂t/∂(pcx, pcy, pcz) of the source's place t = R·(0.5 − pcy·rows, 0.5 − pcx·cols, pcz·rows)
    (geometry.zig:153-161): a 3 × 3 matrix, columns per pattern-centre coordinate."""
    R = geo.rotation()
    return np.stack([R @ np.array([0.0, -cols, 0.0]), R @ np.array([-rows, 0.0, 0.0]), R @ np.array([0.0, 0.0, rows])],
                    1)


def _qmul(a, b):
    aw, ax, ay, az = a.unbind(-1)
    bw, bx, by, bz = b.unbind(-1)
    return torch.stack([aw * bw - ax * bx - ay * by - az * bz, aw * bx + ax * bw + ay * bz - az * by,
                        aw * by - ax * bz + ay * bw + az * bx, aw * bz + ax * by - ay * bx + az * bw], -1)


def _qstd(q):
    n = torch.linalg.norm(q, dim=-1, keepdim=True)
    n = torch.where(n == 0, torch.ones_like(n), n)
    return q / n * torch.where(q[..., :1] < 0, -1.0, 1.0)


def _exp(phi):
    """rot.zig:192-198 — exp of rotation vectors."""
    th2 = (phi * phi).sum(-1, keepdim=True)
    th = torch.sqrt(th2)
    k = torch.where(th < 1e-6, 0.5 - th2 / 48.0, torch.sin(0.5 * th) / torch.where(th < 1e-6, torch.ones_like(th), th))
    return torch.cat([torch.cos(0.5 * th), k * phi], -1)


def local_of(s):
    """planefit.zig:176-200 (localOf) for every pattern, FP64: (ok, NCC, g [n,6], H [n,6,6])
    from the 43 sums [n, 43]."""
    s = s.to(torch.float64)
    n = torch.clamp(s[:, 0], min=1.0)
    mean = s[:, 1] / n
    var_n = s[:, 2] - n * mean * mean
    ok = var_n > 1e-12
    inv = torch.where(ok, torch.rsqrt(torch.where(ok, var_n, torch.ones_like(var_n))), torch.zeros_like(var_n))
    ncc = s[:, 3] * inv
    sd = s[:, 4:10]
    au = (s[:, 10:16] - mean[:, None] * sd) * inv[:, None]
    g = (s[:, 16:22] - ncc[:, None] * au) * inv[:, None]
    iu = torch.triu_indices(6, 6)
    P = torch.zeros(s.shape[0], 6, 6, dtype=torch.float64, device=s.device)
    P[:, iu[0], iu[1]] = s[:, 22:43]
    P = P + torch.triu(P, 1).transpose(1, 2)
    H = (P - sd[:, :, None] * sd[:, None, :] / n[:, None, None] - au[:, :, None] * au[:, None, :]) * (inv * inv)[:, None, None]
    ncc = torch.where(ok, ncc, torch.full_like(ncc, -2.0))
    return ok, ncc, g, H


def adjoint_gradient(s):
    """∂NCC/∂x from the one-pass sums of zeb_det6 mode 3 [n, 61] (FP64): the NCC's statistics
    (sums 0-3) with the exact derivatives' ΣD', ΣM·D', Σe·D' (sums 43-60), by the formula of
    planefit.zig:176-200 (au = (ΣM·D' − mean·ΣD')/σ, g = (Σe·D' − NCC·au)/σ)."""
    s = s.to(torch.float64)
    n = torch.clamp(s[:, 0], min=1.0)
    mean = s[:, 1] / n
    var_n = s[:, 2] - n * mean * mean
    ok = var_n > 1e-12
    inv = torch.where(ok, torch.rsqrt(torch.where(ok, var_n, torch.ones_like(var_n))), torch.zeros_like(var_n))
    ncc = s[:, 3] * inv
    au = (s[:, 49:55] - mean[:, None] * s[:, 43:49]) * inv[:, None]
    return (s[:, 55:61] - ncc[:, None] * au) * inv[:, None]


def refine6(plan, q0, trust, most=60, gradient="reference"):
    """planefit.zig:570-622 (settle, k = 6) over every pattern of `plan` at once: λ from 1e-3;
    each round every pattern's damped step (its shift clamped to ±trust pixels, its rotation
    exp(d)·q) is kept where its own NCC rose (λ ← max(λ/3, 1e-4)), else λ ← min(5λ, 1e8); until
    a round gains the patterns' mean NCC less than 1e-7 (a round in which every step overshot
    goes again while some λ < 1e8) or after `most` rounds. gradient: "reference" (the gradient
    table's, as the reference) or "adjoint" (the exact derivative of the forward, ProjectedNCC's
    backward: the derivatives of its adjoint kernel summed in the same pass as the GN sums, mode 3).
    Returns (q [n,4] f64, shift [n,3] f64 pixels, NCC [n], rounds)."""
    dev = q0.device
    n = plan.n
    q = _qstd(q0.to(torch.float64))
    shift = torch.zeros(n, 3, dtype=torch.float64, device=dev)

    def local(qq, ss):
        x = torch.cat([ss, torch.zeros(n, 3, dtype=torch.float64, device=dev)], 1).to(torch.float32).contiguous()
        qf = qq.to(torch.float32).contiguous()
        if gradient == "adjoint":
            # one pass: the GN sums and the adjoint's derivatives of the same projection
            sums = plan.run(3, x, qf)
            ok, ncc, _, H = local_of(sums[:, :43])
            g = torch.where(ok[:, None], adjoint_gradient(sums), torch.zeros_like(H[:, 0]))
            return ok, ncc, g, H
        return local_of(plan.run(2, x, qf))

    keep = local(q, shift)
    lam = torch.full((n,), 1e-3, dtype=torch.float64, device=dev)
    count = max(n, 1)
    eye = torch.eye(6, dtype=torch.float64, device=dev)
    rounds = 0
    while rounds < most:
        H, g = keep[3], keep[2]
        tr = torch.diagonal(H, dim1=1, dim2=2).sum(-1)
        A = H + eye * (torch.diagonal(H, dim1=1, dim2=2) * lam[:, None])[:, :, None] + eye * (1e-9 * tr + 1e-30)[:, None, None]
        A = A.contiguous()
        b = g.contiguous()
        d = torch.empty(n, 6, dtype=torch.float64, device=dev)
        ok = torch.empty(n, dtype=torch.int32, device=dev)
        N.call("zeb_solve6", ptr(A), ptr(b), n, ptr(d), ptr(ok), stream_ptr())
        good = (ok != 0) & keep[0]
        st = torch.where(good[:, None], torch.clamp(shift + d[:, :3], -trust, trust), shift)
        qt = torch.where(good[:, None], _qstd(_qmul(_exp(d[:, 3:]), q)), q)
        now = local(qt, st)
        better = now[1] > keep[1]
        gain = float(torch.where(better, now[1] - keep[1], torch.zeros_like(lam)).sum())
        kept = int(better.sum())
        damp = int((~better & (lam < 1e8)).sum())
        q = torch.where(better[:, None], qt, q)
        shift = torch.where(better[:, None], st, shift)
        keep = tuple(torch.where(better.view(-1, *([1] * (k.dim() - 1))), nw, k) for k, nw in zip(keep, now))
        lam = torch.where(better, torch.clamp(lam / 3, min=1e-4), torch.clamp(lam * 5, max=1e8))
        if kept == 0 and damp > 0:  # (every step overshot: they go again, damped more)
            rounds += 1
            continue
        if gain / count < 1e-7:  # (the round that ends the loop is not counted, as the reference's)
            break
        rounds += 1
    return q, shift, keep[1], rounds
