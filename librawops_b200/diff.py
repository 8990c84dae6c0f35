"""Differentiable render: torch.autograd Functions over the CUDA adjoints.

    plane (h, w)  --BilinearDemosaic or MenonDemosaic-->  camera RGB  --PointStages(wb, stops,
    matrix, curve knots)-->  working RGB  --DetailBoost(strength, eps)-->  out

Each Function's forward and backward are the hand-written kernels of
csrc/diff.cu (include/rawengine_b200.h, re_diff_*), launched on torch's current
stream; there is no autograd-traced fallback.  The curve's Bezier controls and
end slopes are derived from the knot values with torch operations
(`curve_controls`, the tangent rule of ToneOps.cpp:795-816), so gradients with
respect to the knots flow through them by autograd.  `RecipeModel` bundles the
parameters; `fit_recipe` fits them to a target render with Adam.
"""
from __future__ import annotations

import ctypes as C
import math

import torch

from ._capi import DiffPointParams, check, lib

PROPHOTO, REC2020 = 0, 1


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def quad_code(colours) -> int:
    """Packs the colours (0 R, 1 G, 2 B) of the 2x2 CFA cell at the plane origin."""
    return sum(int(c) << (2 * i) for i, c in enumerate(colours))


# ------------------------------------------------------------------ demosaic

class BilinearDemosaic(torch.autograd.Function):
    """Bilinear demosaic of a normalized sensor plane (RawEngine.cpp:299-344)."""

    @staticmethod
    def forward(ctx, plane, quad: int):
        plane = plane.contiguous()
        h, w = plane.shape
        out = torch.empty((h, w, 3), dtype=torch.float32, device=plane.device)
        check(lib().re_diff_bilinear_forward(_ptr(plane), w, w, h, quad, _ptr(out), _stream()))
        ctx.quad = quad
        ctx.shape = (h, w)
        return out

    @staticmethod
    def backward(ctx, grad):
        grad = grad.contiguous()
        h, w = ctx.shape
        dplane = torch.empty((h, w), dtype=torch.float32, device=grad.device)
        check(lib().re_diff_bilinear_backward(_ptr(grad), w, h, ctx.quad, _ptr(dplane), w, _stream()))
        return dplane, None


class MenonDemosaic(torch.autograd.Function):
    """Menon demosaic of a normalized sensor plane (MenonDemosaic.cpp:97-173,
    mirrored borders).  The forward decides the directions; the backward is
    the transpose with those directions frozen."""

    @staticmethod
    def forward(ctx, plane, quad: int):
        plane = plane.contiguous()
        h, w = plane.shape
        out = torch.empty((h, w, 3), dtype=torch.float32, device=plane.device)
        dirs = torch.empty((h, w), dtype=torch.uint8, device=plane.device)
        check(lib().re_diff_menon_forward(_ptr(plane), w, w, h, quad, _ptr(out), _ptr(dirs), _stream()))
        ctx.save_for_backward(dirs)
        ctx.quad = quad
        return out

    @staticmethod
    def backward(ctx, grad):
        (dirs,) = ctx.saved_tensors
        grad = grad.contiguous()
        h, w = dirs.shape
        dplane = torch.empty((h, w), dtype=torch.float32, device=grad.device)
        check(lib().re_diff_menon_backward(_ptr(grad), w, h, ctx.quad, _ptr(dirs), _ptr(dplane), w, _stream()))
        return dplane, None


def menon_directions(plane, quad: int):
    """The direction map of MenonDemosaic's forward (1 = horizontal)."""
    plane = plane.contiguous()
    h, w = plane.shape
    out = torch.empty((h, w, 3), dtype=torch.float32, device=plane.device)
    dirs = torch.empty((h, w), dtype=torch.uint8, device=plane.device)
    check(lib().re_diff_menon_forward(_ptr(plane), w, w, h, quad, _ptr(out), _ptr(dirs), _stream()))
    return dirs


# --------------------------------------------------------------------- curve

def curve_controls(kx: torch.Tensor, ky: torch.Tensor):
    """Bezier controls c0, c1 and end slopes of the shape-preserving cubic
    (ToneOps.cpp:795-816), differentiable in ky: tangent = the smaller-magnitude
    neighbouring slope, zero on a sign change or a flat neighbour."""
    h = kx[1:] - kx[:-1]
    s = (ky[1:] - ky[:-1]) / h
    a, b = s[:-1], s[1:]
    flat = (a == 0) | (b == 0) | (torch.signbit(a) != torch.signbit(b))
    inner = torch.where(flat, torch.zeros_like(a), torch.where(a.abs() <= b.abs(), a, b))
    m = torch.cat([s[:1], inner, s[-1:]])
    c0 = ky[:-1] + h * m[:-1] / 3
    c1 = ky[1:] - h * m[1:] / 3
    return c0, c1, s[0], s[-1]


class PointStages(torch.autograd.Function):
    """WB -> exposure multiplier -> 3x3 -> master curve, per pixel."""

    @staticmethod
    def forward(ctx, x, wb, exposure, matrix, kx, ky, c0, c1, s_first, s_last):
        x = x.contiguous()
        scalars = torch.cat([wb.detach().reshape(3), exposure.detach().reshape(1), matrix.detach().reshape(9),
                             s_first.detach().reshape(1), s_last.detach().reshape(1)]).float().contiguous()
        knots = [t.detach().float().contiguous() for t in (kx, ky, c0, c1)]
        y = torch.empty_like(x)
        p = PointStages._params(scalars, knots)
        check(lib().re_diff_point_forward(_ptr(x), x.numel() // 3, C.byref(p), _ptr(y), _stream()))
        ctx.save_for_backward(x, scalars, *knots)
        ctx.n = kx.numel()
        return y

    @staticmethod
    def _params(scalars, knots):
        p = DiffPointParams()
        p.scalars = scalars.data_ptr()
        p.knots = knots[0].numel()
        p.kx, p.ky, p.c0, p.c1 = (t.data_ptr() for t in knots)
        return p

    @staticmethod
    def backward(ctx, grad):
        x, scalars, kx, ky, c0, c1 = ctx.saved_tensors
        p = PointStages._params(scalars, [kx, ky, c0, c1])
        n = ctx.n
        grad = grad.contiguous()
        g = torch.zeros(int(lib().re_diff_point_grad_count(n)), dtype=torch.float64, device=x.device)
        dx = torch.empty_like(x)
        check(lib().re_diff_point_backward(_ptr(x), _ptr(grad), x.numel() // 3, C.byref(p), _ptr(dx), _ptr(g),
                                           _stream()))
        gf = g.float()
        gk = gf[13:]
        return (dx, gf[0:3], gf[3], gf[4:13].reshape(3, 3), None, gk[:n], gk[n:2 * n - 1],
                gk[2 * n - 1:3 * n - 2], gk[3 * n - 2], gk[3 * n - 1])


def point_stages(x, wb, stops, matrix, kx, ky):
    """Point stages with the exposure in stops and the curve given by its knots."""
    c0, c1, sf, sl = curve_controls(kx, ky)
    exposure = torch.exp2(stops)
    return PointStages.apply(x, wb, exposure, matrix, kx, ky, c0, c1, sf, sl)


# -------------------------------------------------------------- detail boost

class DetailBoost(torch.autograd.Function):
    """out = v + strength (v - GF(v)), GF the self-guided working-Y guided filter.

    `eps` is a one-element float64 tensor: the kernels take its value by value
    (read on the host once per call) and the backward returns its gradient."""

    @staticmethod
    def forward(ctx, v, strength, eps, radius: int, space: int):
        v = v.contiguous()
        h, w = v.shape[:2]
        k = strength.detach().float().reshape(1).contiguous()
        e = float(eps.detach())
        out = torch.empty_like(v)
        check(lib().re_diff_detail_forward(_ptr(v), w, h, radius, e, _ptr(k), space, _ptr(out), _stream()))
        ctx.save_for_backward(v, k)
        ctx.args = (radius, e, space, eps.dtype)
        return out

    @staticmethod
    def backward(ctx, grad):
        v, k = ctx.saved_tensors
        radius, e, space, eps_dtype = ctx.args
        h, w = v.shape[:2]
        grad = grad.contiguous()
        dv = torch.empty_like(v)
        dk = torch.zeros(2, dtype=torch.float64, device=v.device)     # d strength, d eps
        check(lib().re_diff_detail_backward(_ptr(v), _ptr(grad), w, h, radius, e, _ptr(k), space, _ptr(dv),
                                            _ptr(dk), C.c_void_p(dk.data_ptr() + 8), _stream()))
        return dv, dk[0].float(), dk[1].to(eps_dtype), None, None


# --------------------------------------------------------------------- model

class RecipeModel(torch.nn.Module):
    """The differentiable render (bilinear, or Menon with directions frozen
    from the forward) with learnable recipe parameters: WB gains,
    exposure stops, the 3x3 camera->working matrix, the master-curve knot values
    (knot positions fixed), the detail-boost strength and the guided filter's
    epsilon (learned as its natural logarithm, float64, so that it stays
    positive)."""

    def __init__(self, quad, kx, ky, wb=(1.0, 1.0, 1.0), stops=0.0, matrix=None, strength=0.0, radius=16,
                 eps=1e-3, space=PROPHOTO, device="cuda", demosaic="bilinear"):
        super().__init__()
        f = dict(dtype=torch.float32, device=device)
        if demosaic not in ("bilinear", "menon"):
            raise ValueError("demosaic must be 'bilinear' or 'menon'")
        self.demosaic = demosaic
        self.quad = quad_code(quad)
        self.radius, self.space = radius, space
        self.register_buffer("kx", torch.tensor(kx, **f))
        self.wb = torch.nn.Parameter(torch.tensor(wb, **f))
        self.stops = torch.nn.Parameter(torch.tensor(float(stops), **f))
        m = torch.eye(3) if matrix is None else torch.as_tensor(matrix, dtype=torch.float32)
        self.matrix = torch.nn.Parameter(m.to(**f).clone())
        self.ky = torch.nn.Parameter(torch.tensor(ky, **f))
        self.strength = torch.nn.Parameter(torch.tensor(float(strength), **f))
        self.log_eps = torch.nn.Parameter(torch.tensor(math.log(eps), dtype=torch.float64, device=device))

    @property
    def eps(self) -> float:
        return math.exp(float(self.log_eps.detach()))

    def forward(self, plane):
        x = (MenonDemosaic if self.demosaic == "menon" else BilinearDemosaic).apply(plane, self.quad)
        v = point_stages(x, self.wb, self.stops, self.matrix, self.kx, self.ky)
        return DetailBoost.apply(v, self.strength, torch.exp(self.log_eps), self.radius, self.space)


def fit_recipe(model: RecipeModel, planes, targets, steps: int = 200, lr: float = 0.01, params=None):
    """Adam on the mean squared error between model(plane) and target over a
    list of frames; returns the loss history."""
    opt = torch.optim.Adam(params if params is not None else model.parameters(), lr=lr)
    history = []
    for _ in range(steps):
        opt.zero_grad(set_to_none=True)
        loss = sum(torch.mean((model(p) - t) ** 2) for p, t in zip(planes, targets)) / len(planes)
        loss.backward()
        opt.step()
        history.append(float(loss.detach()))
    return history

