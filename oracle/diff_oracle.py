"""Float64 CPU restatement of the differentiable render and its adjoint.

TEST INFRASTRUCTURE ONLY: the CUDA adjoints in librawops_b200/csrc/diff.cu are
checked against this module (and this module against central finite
differences) in tests/; nothing in the product imports it.

The reference has no gradients; the forward model restates its arithmetic on
the path:

* bilinear demosaic of the normalized sensor plane over the active area
  (RawEngine.cpp:299-344): own channel = sample, other channels = mean of the
  same-colour samples in the 3x3 clipped to the active area;
* or Menon demosaic (MenonDemosaic.cpp:97-173) with mirrored borders: the
  forward decides the directions, and with those directions held fixed the
  demosaic is linear in the samples, so its adjoint is that linear map's
  transpose;
* white balance x_c * g_c (RawEngine.cpp:417-431), exposure * 2^stops
  (RawEngine.cpp:488-500), a 3x3 matrix (RawEngine.cpp:539-545);
* the master curve of ExtendedCurvesNode with ShapePreservingCubic
  interpolation (ToneOps.cpp:795-844): slopes, min-magnitude tangents (zero
  on a sign change or a flat neighbour), cubic Bezier per segment, linear
  extrapolation outside the knots -- here with the knot y values as
  parameters;
* a detail boost out = v + k (v - GF(v)) with the self-guided working-Y guided
  filter of SpatialOps.cpp:168-287 (box means over the clipped (2r+1)^2
  window with actual counts, a = cov/(var+eps), b = mean_p - a mean_I,
  q = mean(a) I + mean(b)).

Every function takes and returns float64 arrays; `backward_*` return the
adjoints (vector-Jacobian products) for a given output gradient.
"""
from __future__ import annotations

import numpy as np

PATTERN_COLORS = [(0, 1, 1, 2), (2, 1, 1, 0), (1, 0, 2, 1), (1, 2, 0, 1)]
Y_WEIGHTS = {0: (0.28807112822929337, 0.00008565396060525903),   # ProPhoto (wr, wb)
             1: (0.26270021201126703, 0.059301716469861945)}     # Rec.2020


def colour_map(h: int, w: int, quad) -> np.ndarray:
    """Colour (0 R, 1 G, 2 B) of each site; quad[(y&1)*2+(x&1)] relative to the active origin."""
    y = np.arange(h)[:, None] & 1
    x = np.arange(w)[None, :] & 1
    return np.asarray(quad)[y * 2 + x]


# ------------------------------------------------------------------ demosaic

def bilinear_forward(s: np.ndarray, quad) -> np.ndarray:
    h, w = s.shape
    col = colour_map(h, w, quad)
    out = np.zeros((h, w, 3))
    for c in range(3):
        m = (col == c).astype(np.float64)
        sp = np.pad(s * m, 1)
        mp = np.pad(m, 1)
        tot = sum(sp[1 + dy:1 + dy + h, 1 + dx:1 + dx + w] for dy in (-1, 0, 1) for dx in (-1, 0, 1))
        cnt = sum(mp[1 + dy:1 + dy + h, 1 + dx:1 + dx + w] for dy in (-1, 0, 1) for dx in (-1, 0, 1))
        avg = np.divide(tot, cnt, out=np.zeros_like(tot), where=cnt > 0)
        out[..., c] = np.where(col == c, s, avg)
    return out


def bilinear_backward(dout: np.ndarray, quad) -> np.ndarray:
    h, w = dout.shape[:2]
    col = colour_map(h, w, quad)
    ds = np.zeros((h, w))
    for c in range(3):
        m = (col == c).astype(np.float64)
        mp = np.pad(m, 1)
        cnt = sum(mp[1 + dy:1 + dy + h, 1 + dx:1 + dx + w] for dy in (-1, 0, 1) for dx in (-1, 0, 1))
        # pixels of another colour average their c-neighbours: scatter dout/cnt back
        g = np.where((col != c) & (cnt > 0), dout[..., c] / np.maximum(cnt, 1), 0.0)
        gp = np.pad(g, 1)
        spread = sum(gp[1 + dy:1 + dy + h, 1 + dx:1 + dx + w] for dy in (-1, 0, 1) for dx in (-1, 0, 1))
        ds += m * (dout[..., c] + spread)
    return ds


# --------------------------------------------------------------------- curve

def curve_controls(kx, ky):
    """Slopes, tangents and Bezier controls of ToneOps.cpp:795-816."""
    kx, ky = np.asarray(kx, np.float64), np.asarray(ky, np.float64)
    h = np.diff(kx)
    s = np.diff(ky) / h
    m = np.empty(len(kx))
    m[0], m[-1] = s[0], s[-1]
    a, b = s[:-1], s[1:]
    flat = (a == 0) | (b == 0) | (np.signbit(a) != np.signbit(b))
    m[1:-1] = np.where(flat, 0.0, np.copysign(np.minimum(np.abs(a), np.abs(b)), a))
    c0 = ky[:-1] + h * m[:-1] / 3
    c1 = ky[1:] - h * m[1:] / 3
    return h, s, m, c0, c1


def curve_forward(v: np.ndarray, kx, ky) -> np.ndarray:
    kx, ky = np.asarray(kx, np.float64), np.asarray(ky, np.float64)
    h, s, m, c0, c1 = curve_controls(kx, ky)
    n = len(kx)
    i = np.clip(np.searchsorted(kx, v, side="right") - 1, 0, n - 2)
    t = (v - kx[i]) / h[i]
    u = 1 - t
    bez = u ** 3 * ky[i] + 3 * u * u * t * c0[i] + 3 * u * t * t * c1[i] + t ** 3 * ky[i + 1]
    left = ky[0] + (v - kx[0]) * s[0]
    right = ky[-1] + (v - kx[-1]) * s[-1]
    return np.where(v < kx[0], left, np.where(v > kx[-1], right, bez))


def curve_derivative(v, kx, ky):
    kx, ky = np.asarray(kx, np.float64), np.asarray(ky, np.float64)
    h, s, m, c0, c1 = curve_controls(kx, ky)
    n = len(kx)
    i = np.clip(np.searchsorted(kx, v, side="right") - 1, 0, n - 2)
    t = (v - kx[i]) / h[i]
    u = 1 - t
    dbdt = 3 * (u * u * (c0[i] - ky[i]) + 2 * u * t * (c1[i] - c0[i]) + t * t * (ky[i + 1] - c1[i]))
    return np.where(v < kx[0], s[0], np.where(v > kx[-1], s[-1], dbdt / h[i]))


def curve_backward_knots(v, dout, kx, ky) -> np.ndarray:
    """d loss / d ky through the Bezier values, the controls and the tangents
    (the tangent rule's min/sign branches are fixed at the evaluation point)."""
    kx, ky = np.asarray(kx, np.float64), np.asarray(ky, np.float64)
    n = len(kx)
    h, s, m, c0, c1 = curve_controls(kx, ky)
    v, dout = v.ravel(), dout.ravel()
    i = np.clip(np.searchsorted(kx, v, side="right") - 1, 0, n - 2)
    t = (v - kx[i]) / h[i]
    u = 1 - t
    inside = (v >= kx[0]) & (v <= kx[-1])
    g_y = np.zeros(n)
    g_c0 = np.zeros(n - 1)
    g_c1 = np.zeros(n - 1)
    g_s = np.zeros(n - 1)
    np.add.at(g_y, i[inside], (dout * u ** 3)[inside])
    np.add.at(g_y, i[inside] + 1, (dout * t ** 3)[inside])
    np.add.at(g_c0, i[inside], (dout * 3 * u * u * t)[inside])
    np.add.at(g_c1, i[inside], (dout * 3 * u * t * t)[inside])
    lo, hi = v < kx[0], v > kx[-1]
    g_y[0] += dout[lo].sum()
    g_s[0] += (dout * (v - kx[0]))[lo].sum()
    g_y[-1] += dout[hi].sum()
    g_s[-1] += (dout * (v - kx[-1]))[hi].sum()
    # controls -> knots and tangents; tangents -> slopes; slopes -> knots
    g_y[:-1] += g_c0
    g_y[1:] += g_c1
    g_m = np.zeros(n)
    g_m[:-1] += g_c0 * h / 3
    g_m[1:] -= g_c1 * h / 3
    g_s[0] += g_m[0]
    g_s[-1] += g_m[-1]
    a, b = s[:-1], s[1:]
    flat = (a == 0) | (b == 0) | (np.signbit(a) != np.signbit(b))
    pick_a = np.abs(a) <= np.abs(b)
    for j in range(1, n - 1):
        if flat[j - 1]:
            continue
        if pick_a[j - 1]:
            g_s[j - 1] += g_m[j]
        else:
            # m = copysign(|b|, a) and sign(a) == sign(b) here, so dm/db = 1
            g_s[j] += g_m[j]
    g_y[1:] += g_s / h
    g_y[:-1] -= g_s / h
    return g_y


# ---------------------------------------------------------------- point stages

def point_forward(x: np.ndarray, wb, stops, M, kx, ky) -> np.ndarray:
    z = x * np.asarray(wb)[None, None, :] * 2.0 ** stops
    y = np.einsum("ij,hwj->hwi", np.asarray(M, np.float64), z)
    return curve_forward(y, kx, ky)


def point_backward(x, dout, wb, stops, M, kx, ky):
    """Returns (dx, dwb, dstops, dM, dky)."""
    wb, M = np.asarray(wb, np.float64), np.asarray(M, np.float64)
    e = 2.0 ** stops
    t1 = x * wb[None, None, :]
    z = t1 * e
    y = np.einsum("ij,hwj->hwi", M, z)
    dy = dout * curve_derivative(y, kx, ky)
    dky = curve_backward_knots(y, dout, kx, ky)
    dM = np.einsum("hwi,hwj->ij", dy, z)
    dz = np.einsum("ij,hwi->hwj", M, dy)
    de = (dz * t1).sum()
    dstops = de * e * np.log(2.0)
    dt1 = dz * e
    dwb = (dt1 * x).sum(axis=(0, 1))
    dx = dt1 * wb[None, None, :]
    return dx, dwb, dstops, dM, dky


# -------------------------------------------------------------- detail boost

def _box(a: np.ndarray, r: int) -> np.ndarray:
    """Clipped box sum over (2r+1)^2 (leading two axes)."""
    h, w = a.shape[:2]
    c = np.cumsum(np.cumsum(np.pad(a, [(1, 0), (1, 0)] + [(0, 0)] * (a.ndim - 2)), 0), 1)
    y0 = np.clip(np.arange(h) - r, 0, h)
    y1 = np.clip(np.arange(h) + r + 1, 0, h)
    x0 = np.clip(np.arange(w) - r, 0, w)
    x1 = np.clip(np.arange(w) + r + 1, 0, w)
    return (c[y1][:, x1] - c[y0][:, x1] - c[y1][:, x0] + c[y0][:, x0])


def _count(h, w, r):
    ny = np.minimum(np.arange(h) + r, h - 1) - np.maximum(np.arange(h) - r, 0) + 1
    nx = np.minimum(np.arange(w) + r, w - 1) - np.maximum(np.arange(w) - r, 0) + 1
    return (ny[:, None] * nx[None, :]).astype(np.float64)


def _guide(p, space):
    wr, wb = Y_WEIGHTS[space]
    return (p[..., 1] + wr * (p[..., 0] - p[..., 1])) + wb * (p[..., 2] - p[..., 1])


def guided_forward(p: np.ndarray, r: int, eps: float, space: int = 0):
    h, w = p.shape[:2]
    n = _count(h, w, r)
    I = _guide(p, space)
    mI = _box(I, r) / n
    mII = _box(I * I, r) / n
    mp = _box(p, r) / n[..., None]
    mIp = _box(I[..., None] * p, r) / n[..., None]
    var = mII - mI * mI
    cov = mIp - mI[..., None] * mp
    a = cov / (var + eps)[..., None]
    b = mp - a * mI[..., None]
    ma = _box(a, r) / n[..., None]
    mb = _box(b, r) / n[..., None]
    q = ma * I[..., None] + mb
    return q, (n, I, mI, mII, mp, mIp, var, cov, a, b, ma, mb)


def detail_forward(p: np.ndarray, r: int, eps: float, k: float, space: int = 0) -> np.ndarray:
    q, _ = guided_forward(p, r, eps, space)
    return p + k * (p - q)


def detail_backward(p: np.ndarray, dout: np.ndarray, r: int, eps: float, k: float, space: int = 0):
    """Returns (dp, dk, deps).  epsilon enters each centre only through
    var + eps, so d/d eps is the sum over centres of the variance adjoint."""
    q, (n, I, mI, mII, mp, mIp, var, cov, a, b, ma, mb) = guided_forward(p, r, eps, space)
    dk = float(((p - q) * dout).sum())
    dq = -k * dout
    dp = (1 + k) * dout
    dI = (ma * dq).sum(-1)
    da = _box(dq * I[..., None] / n[..., None], r)
    db = _box(dq / n[..., None], r)
    inv = 1.0 / (var + eps)
    dmp = db.copy()
    dA = da - db * mI[..., None]
    dmI = -(db * a).sum(-1)
    dcov = dA * inv[..., None]
    dvar = -(dA * cov).sum(-1) * inv * inv
    deps = float(dvar.sum())
    dmIp = dcov
    dmI += -(dcov * mp).sum(-1)
    dmp += -dcov * mI[..., None]
    dmII = dvar
    dmI += -2 * mI * dvar
    BI = _box(dmI / n, r)
    BII = _box(dmII / n, r)
    Bp = _box(dmp / n[..., None], r)
    BIp = _box(dmIp / n[..., None], r)
    dp += Bp + I[..., None] * BIp
    dI += BI + 2 * I * BII + (p * BIp).sum(-1)
    wr, wb = Y_WEIGHTS[space]
    dp += dI[..., None] * np.array([wr, 1 - wr - wb, wb])[None, None, :]
    return dp, dk, deps


# ------------------------------------------------------------------ Menon

def _mirror(i, n):
    """MenonDemosaic.cpp:60-66: reflection about the edge samples."""
    i = np.asarray(i)
    if n == 1:
        return np.zeros_like(i)
    period = 2 * (n - 1)
    f = np.mod(i, period)
    return np.where(f < n, f, period - f)


def _taps(h, w, dx, dy):
    """Flat indices of the mirrored samples at offset (dx, dy) of every site."""
    y = _mirror(np.arange(h) + dy, h)[:, None]
    x = _mirror(np.arange(w) + dx, w)[None, :]
    return (y * w + x).reshape(-1)


CLASSIFIER = [(0, 2, 1.0), (-2, 2, 1.0), (-1, 1, 1.0), (0, 0, 3.0), (-2, 0, 3.0), (-1, -1, 1.0), (0, -2, 1.0),
              (-2, -2, 1.0)]


def menon_directions(s: np.ndarray, quad) -> np.ndarray:
    """The horizontal flags of MenonDemosaic.cpp:107-147 (1 at green sites)."""
    h, w = s.shape
    c = colour_map(h, w, quad)
    f = s.reshape(-1)
    at = lambda dx, dy: f[_taps(h, w, dx, dy)].reshape(h, w)
    gh = 0.5 * (at(-1, 0) + at(1, 0)) + 0.5 * s - 0.25 * (at(-2, 0) + at(2, 0))
    gv = 0.5 * (at(0, -1) + at(0, 1)) + 0.5 * s - 0.25 * (at(0, -2) + at(0, 2))
    ng = c != 1
    ch = np.where(ng, s - gh, 0.0)
    cv = np.where(ng, s - gv, 0.0)
    dh = np.abs(ch - ch.reshape(-1)[_taps(h, w, 2, 0)].reshape(h, w))
    dv = np.abs(cv - cv.reshape(-1)[_taps(h, w, 0, 2)].reshape(h, w))

    def grad(p, dx, dy):   # zero outside the image, no mirror
        out = np.zeros_like(p)
        ys, xs = slice(max(0, -dy), min(h, h - dy)), slice(max(0, -dx), min(w, w - dx))
        yd, xd = slice(max(0, dy), min(h, h + dy)), slice(max(0, dx), min(w, w + dx))
        out[ys, xs] = p[yd, xd]
        return out
    hh = np.zeros_like(s)
    vv = np.zeros_like(s)
    for tx, ty, wt in CLASSIFIER:
        hh = hh + wt * grad(dh, tx, ty)
        vv = vv + wt * grad(dv, ty, tx)
    return np.where(ng, (vv >= hh).astype(np.uint8), 1).astype(np.uint8)


def menon_forward(s: np.ndarray, quad, horizontal=None):
    """MenonDemosaic.cpp:97-173 on a float64 plane with mirrored borders;
    returns (rgb, horizontal).  With `horizontal` given, those directions are
    used (the linear map the adjoint transposes)."""
    h, w = s.shape
    c = colour_map(h, w, quad)
    if horizontal is None:
        horizontal = menon_directions(s, quad)
    f = s.reshape(-1)
    at = lambda p, dx, dy: p.reshape(-1)[_taps(h, w, dx, dy)].reshape(h, w)
    gh = 0.5 * (at(f, -1, 0) + at(f, 1, 0)) + 0.5 * s - 0.25 * (at(f, -2, 0) + at(f, 2, 0))
    gv = 0.5 * (at(f, 0, -1) + at(f, 0, 1)) + 0.5 * s - 0.25 * (at(f, 0, -2) + at(f, 0, 2))
    green = np.where(c == 1, s, np.where(horizontal == 1, gh, gv))
    mean = lambda p, dx, dy: 0.5 * (at(p, -dx, -dy) + at(p, dx, dy))
    red_h = colour_map(h, w + 1, quad)[:, 1:] == 0          # colour(x + 1, y) == R
    # (green + mean(raw)) - mean(green), in the reference's order
    along = lambda p, horiz: np.where(horiz, mean(p, 1, 0), mean(p, 0, 1))
    red = np.where(c == 0, s, np.where(c == 1, (green + along(f, red_h)) - along(green, red_h), 0.0))
    blue = np.where(c == 2, s, np.where(c == 1, (green + along(f, ~red_h)) - along(green, ~red_h), 0.0))
    Hd = horizontal == 1
    rr = np.where(c == 2, (blue + along(red, Hd)) - along(blue, Hd), red)
    bb = np.where(c == 0, (red + along(blue, Hd)) - along(red, Hd), blue)
    return np.stack([rr, green, bb], -1), horizontal


def _scatter(h, w, g, dx, dy, weight):
    """Transpose of p -> weight * p[mirror(offset)]: adds weight * g at the tapped sites."""
    out = np.zeros(h * w)
    np.add.at(out, _taps(h, w, dx, dy), (weight * g).reshape(-1))
    return out.reshape(h, w)


def menon_backward(dout: np.ndarray, quad, horizontal) -> np.ndarray:
    """The transpose of the frozen-direction Menon demosaic: d loss / d s."""
    h, w = horizontal.shape
    c = colour_map(h, w, quad)
    dR, dG, dB = dout[..., 0], dout[..., 1], dout[..., 2]
    H = horizontal == 1
    # final step: rr = blue + (mean(red) - mean(blue)) at B sites, bb = red - (...) at R sites
    dd = np.where(c == 2, dR, 0.0) - np.where(c == 0, dB, 0.0)          # d loss / d dred
    dred = np.where(c != 2, dR, 0.0) + np.where(c == 0, dB, 0.0)
    dblue = np.where(c != 0, dB, 0.0) + np.where(c == 2, dR, 0.0)
    for dx, dy, sel in ((1, 0, H), (0, 1, ~H)):
        g = np.where(sel, dd, 0.0)
        for sx, sy in ((-dx, -dy), (dx, dy)):
            dred += _scatter(h, w, g, sx, sy, 0.5)
            dblue -= _scatter(h, w, g, sx, sy, 0.5)
    # red / blue at green sites: green + mean(s) - mean(green); own sites: s
    ds = np.where(c == 0, dred, 0.0) + np.where(c == 2, dblue, 0.0)
    dgreen = dG + np.where(c == 1, dred + dblue, 0.0)
    red_h = colour_map(h, w + 1, quad)[:, 1:] == 0
    for g, along_x in ((np.where(c == 1, dred, 0.0), red_h), (np.where(c == 1, dblue, 0.0), ~red_h)):
        for dx, dy, sel in ((1, 0, along_x), (0, 1, ~along_x)):
            gg = np.where(sel, g, 0.0)
            for sx, sy in ((-dx, -dy), (dx, dy)):
                ds += _scatter(h, w, gg, sx, sy, 0.5)
                dgreen -= _scatter(h, w, gg, sx, sy, 0.5)
    # green: s at green sites, gh or gv elsewhere
    ds += np.where(c == 1, dgreen, 0.0)
    dgh = np.where((c != 1) & H, dgreen, 0.0)
    dgv = np.where((c != 1) & ~H, dgreen, 0.0)
    for g, ax in ((dgh, 0), (dgv, 1)):
        ds += 0.5 * g
        for k, wt in ((1, 0.5), (2, -0.25)):
            for sgn in (-1, 1):
                dx, dy = (sgn * k, 0) if ax == 0 else (0, sgn * k)
                ds += _scatter(h, w, g, dx, dy, wt)
    return ds


# ----------------------------------------------------------------- full model

def _demosaic(s, quad, demosaic, horizontal=None):
    if demosaic == "menon":
        return menon_forward(s, quad, horizontal)[0]
    return bilinear_forward(s, quad)


def render_forward(s, quad, wb, stops, M, kx, ky, r, eps, k, space=0, demosaic="bilinear", horizontal=None):
    x = _demosaic(s, quad, demosaic, horizontal)
    v = point_forward(x, wb, stops, M, kx, ky)
    return detail_forward(v, r, eps, k, space)


def render_backward(s, dout, quad, wb, stops, M, kx, ky, r, eps, k, space=0, demosaic="bilinear", horizontal=None):
    """Gradients of sum(dout * render) w.r.t. (s, wb, stops, M, ky, k, eps);
    a Menon demosaic's directions are held at `horizontal` (default: the
    forward's)."""
    if demosaic == "menon" and horizontal is None:
        horizontal = menon_directions(s, quad)
    x = _demosaic(s, quad, demosaic, horizontal)
    v = point_forward(x, wb, stops, M, kx, ky)
    dv, dk, deps = detail_backward(v, dout, r, eps, k, space)
    dx, dwb, dstops, dM, dky = point_backward(x, dv, wb, stops, M, kx, ky)
    ds = menon_backward(dx, quad, horizontal) if demosaic == "menon" else bilinear_backward(dx, quad)
    return ds, dwb, dstops, dM, dky, dk, deps
