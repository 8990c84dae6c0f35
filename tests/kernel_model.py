"""CPU model of the Menon render kernel's on-chip indexing (render_raw.cu).

The GPU kernel keeps each Menon plane in shared memory over a *virtual*
window around its output tile, stores mirrored values at out-of-area virtual
positions and skips positions a partial tile does not need.  This model runs
exactly that index arithmetic with bounds-checked NumPy planes initialised to
NaN, so that

* every shared-memory index the kernel forms is proven in bounds for the tile
  geometries exercised (tiny active areas, multiple mirror folds, partial
  tiles, odd origins), and
* no read touches an entry the kernel never wrote (NaN would propagate), and
* the values equal the oracle's bit for bit.

It is test infrastructure: the kernel is never generated from it.
"""
from __future__ import annotations

import numpy as np

TW, TH = 32, 16          # MN_TW, MN_TH
PATTERNS = [(0, 1, 1, 2), (2, 1, 1, 0), (1, 0, 2, 1), (1, 2, 0, 1)]


class Plane:
    def __init__(self, w, h, ox, oy, dtype=np.float64):
        self.a = np.full((h, w), np.nan, dtype)
        self.ox, self.oy = ox, oy

    def idx(self, x, y):
        i, j = y - self.oy, x - self.ox
        if not (0 <= i < self.a.shape[0] and 0 <= j < self.a.shape[1]):
            raise IndexError(f"shared-memory index ({j},{i}) outside {self.a.shape[::-1]}")
        return i, j

    def get(self, x, y):
        v = self.a[self.idx(x, y)]
        if np.isnan(v):
            raise ValueError(f"read of unwritten entry at ({x},{y})")
        return float(v)

    def set(self, x, y, v):
        self.a[self.idx(x, y)] = v


def mirror(v, origin, size):
    if origin <= v < origin + size:
        return v
    if size == 1:
        return origin
    period = 2 * (size - 1)
    folded = (v - origin) % period
    return origin + (folded if folded < size else period - folded)


def model_render(meta, samples, viewport, fast=True):
    """meta: dict(width,height,stride,pattern,phase_x,phase_y,active,black,white)."""
    ax, ay, aw, ah = meta["active"]
    stride = meta["stride"]
    pat = PATTERNS[meta["pattern"]]
    px, py = meta["phase_x"], meta["phase_y"]

    def site(x, y):
        return (((y & 1) + py) & 1) * 2 + (((x & 1) + px) & 1)

    def color(x, y):
        return pat[site(x, y)]

    def sample(x, y):
        assert ax <= x < ax + aw and ay <= y < ay + ah, "global read outside active area"
        s = site(x, y)
        code = np.float32(samples[y * stride + x])
        num = np.float32(code - np.float32(meta["black"][s]))
        return float(np.float32(num / np.float32(meta["white"][s] - meta["black"][s])))

    ox, oy, ow, oh = viewport
    out = np.zeros((oh, ow, 3), np.float32)
    inside = lambda x, y: ax <= x < ax + aw and ay <= y < ay + ah
    gx0, gy0 = ox & ~1, oy & ~1
    for by in range((oy + oh - gy0 + TH - 1) // TH):
        for bx in range((ox + ow - gx0 + TW - 1) // TW):
            x0, y0 = gx0 + bx * TW, gy0 + by * TH
            xe, ye = min(x0 + TW, ox + ow), min(y0 + TH, oy + oh)
            if (fast and x0 - 6 >= ax and y0 - 6 >= ay and x0 + TW + 6 <= ax + aw
                    and y0 + TH + 6 <= ay + ah):
                _fast_tile(meta, sample, color, x0, y0, viewport, out)
                continue
            needed = lambda x, y, rx, ry: x < xe + rx and y < ye + ry
            mx = lambda x: mirror(x, ax, aw)
            my = lambda y: mirror(y, ay, ah)
            raw = Plane(TW + 12, TH + 12, x0 - 6, y0 - 6, np.float64)
            ch = Plane(TW + 8, TH + 8, x0 - 4, y0 - 4)
            cv = Plane(TW + 8, TH + 8, x0 - 4, y0 - 4)
            dh = Plane(TW + 6, TH + 8, x0 - 4, y0 - 4)
            dv = Plane(TW + 8, TH + 6, x0 - 4, y0 - 4)
            green = Plane(TW + 4, TH + 4, x0 - 2, y0 - 2)
            horiz = Plane(TW + 4, TH + 4, x0 - 2, y0 - 2)
            red = Plane(TW + 2, TH + 2, x0 - 1, y0 - 1)
            blue = Plane(TW + 2, TH + 2, x0 - 1, y0 - 1)
            for j in range(TH + 12):
                for i in range(TW + 12):
                    vx, vy = x0 - 6 + i, y0 - 6 + j
                    if needed(vx, vy, 6, 6):
                        raw.set(vx, vy, sample(mx(vx), my(vy)))

            def five(x, y, dx, dy):
                m2, m1 = raw.get(x - 2 * dx, y - 2 * dy), raw.get(x - dx, y - dy)
                p1, p2 = raw.get(x + dx, y + dy), raw.get(x + 2 * dx, y + 2 * dy)
                own = raw.get(x, y)
                return (0.5 * (m1 + p1) + 0.5 * own) - 0.25 * (m2 + p2)

            for j in range(TH + 8):
                for i in range(TW + 8):
                    vx, vy = x0 - 4 + i, y0 - 4 + j
                    if not needed(vx, vy, 4, 4):
                        continue
                    x, y = mx(vx), my(vy)
                    h = v = 0.0
                    if color(x, y) != 1:
                        own = raw.get(x, y)
                        h, v = own - five(x, y, 1, 0), own - five(x, y, 0, 1)
                    ch.set(vx, vy, h)
                    cv.set(vx, vy, v)
            for j in range(TH + 8):
                for i in range(TW + 6):
                    x, y = x0 - 4 + i, y0 - 4 + j
                    if needed(x, y, 2, 4):
                        dh.set(x, y, abs(ch.get(x, y) - ch.get(x + 2, y)) if inside(x, y) else 0.0)
            for j in range(TH + 6):
                for i in range(TW + 8):
                    x, y = x0 - 4 + i, y0 - 4 + j
                    if needed(x, y, 4, 2):
                        dv.set(x, y, abs(cv.get(x, y) - cv.get(x, y + 2)) if inside(x, y) else 0.0)
            terms = [(0, 2, 1), (-2, 2, 1), (-1, 1, 1), (0, 0, 3), (-2, 0, 3), (-1, -1, 1),
                     (0, -2, 1), (-2, -2, 1)]
            for j in range(TH + 4):
                for i in range(TW + 4):
                    vx, vy = x0 - 2 + i, y0 - 2 + j
                    if not needed(vx, vy, 2, 2):
                        continue
                    x, y = mx(vx), my(vy)
                    if color(x, y) == 1:
                        horiz.set(vx, vy, 1.0)
                        green.set(vx, vy, raw.get(x, y))
                        continue
                    h = v = 0.0
                    for tx, ty, w in terms:
                        h += w * dh.get(x + tx, y + ty)
                        v += w * dv.get(x + ty, y + tx)
                    hz = v >= h
                    horiz.set(vx, vy, 1.0 if hz else 0.0)
                    green.set(vx, vy, five(x, y, 1, 0) if hz else five(x, y, 0, 1))
            pm = lambda p, x, y, dx, dy: 0.5 * (p.get(x - dx, y - dy) + p.get(x + dx, y + dy))
            for j in range(TH + 2):
                for i in range(TW + 2):
                    vx, vy = x0 - 1 + i, y0 - 1 + j
                    if not needed(vx, vy, 1, 1):
                        continue
                    x, y = mx(vx), my(vy)
                    own = color(x, y)
                    rr = bb = 0.0
                    if own == 0:
                        rr = raw.get(x, y)
                    if own == 2:
                        bb = raw.get(x, y)
                    if own == 1:
                        rh = color(x + 1, y) == 0
                        dx, dy = (1, 0) if rh else (0, 1)
                        g = green.get(x, y)
                        rr = (g + pm(raw, x, y, dx, dy)) - pm(green, x, y, dx, dy)
                        bb = (g + pm(raw, x, y, dy, dx)) - pm(green, x, y, dy, dx)
                    red.set(vx, vy, rr)
                    blue.set(vx, vy, bb)
            for y in range(max(y0, oy), ye):
                for x in range(max(x0, ox), xe):
                    own = color(x, y)
                    hz = horiz.get(x, y) != 0
                    dx, dy = (1, 0) if hz else (0, 1)
                    rr, bb = red.get(x, y), blue.get(x, y)
                    if own == 2:
                        rr = (bb + pm(red, x, y, dx, dy)) - pm(blue, x, y, dx, dy)
                    if own == 0:
                        bb = (rr + pm(blue, x, y, dx, dy)) - pm(red, x, y, dx, dy)
                    out[y - oy, x - ox] = (rr, green.get(x, y), bb)
    return out


def _fast_tile(meta, sample, color, x0, y0, viewport, out):
    """The interior quad path (menon_fast in render_raw.cu): class-packed chroma
    planes on the quad grid, full-resolution green/red/blue, the kernel's strides
    and neighbour offsets."""
    ox, oy, ow, oh = viewport
    RW, RH, GW, GH = TW + 12, TH + 12, TW + 4, TH + 4
    QW, QH = (TW + 8) // 2, (TH + 8) // 2
    QN = QW * QH
    lay = [color(x0 + (k & 1), y0 + (k >> 1)) for k in range(4)]
    AX = 0 if lay[0] != 1 else 1          # column of the first row's non-green
    BX = 1 - AX

    def flat(n):
        return Plane(n, 1, 0, 0)

    raw = flat(RW * RH)
    ng = {name: flat(QN) for name in ("ghA", "ghB", "gvA", "gvB", "chA", "chB", "cvA", "cvB",
                                      "dhA", "dhB", "dvA", "dvB")}
    green, horiz = flat(GW * GH), flat(GW * GH)
    for i in range(RW * RH):
        raw.set(i, 0, sample(x0 - 6 + i % RW, y0 - 6 + i // RW))
    half = lambda a, b: 0.5 * (a + b)
    R = lambda i: raw.get(i, 0)

    def five(i, d):
        return (half(R(i - d), R(i + d)) + 0.5 * R(i)) - 0.25 * (R(i - 2 * d) + R(i + 2 * d))

    for q in range(QN):
        qx, qy = q % QW, q // QW
        ra = (2 * qy + 2) * RW + 2 * qx + AX + 2
        rb = (2 * qy + 3) * RW + 2 * qx + BX + 2
        ha, va, hb, vb = five(ra, 1), five(ra, RW), five(rb, 1), five(rb, RW)
        ng["ghA"].set(q, 0, ha); ng["gvA"].set(q, 0, va)
        ng["chA"].set(q, 0, R(ra) - ha); ng["cvA"].set(q, 0, R(ra) - va)
        ng["ghB"].set(q, 0, hb); ng["gvB"].set(q, 0, vb)
        ng["chB"].set(q, 0, R(rb) - hb); ng["cvB"].set(q, 0, R(rb) - vb)
    G = lambda name, i: ng[name].get(i, 0)
    for q in range(QN):
        qx, qy = q % QW, q // QW
        if qx < QW - 1:
            ng["dhA"].set(q, 0, abs(G("chA", q) - G("chA", q + 1)))
            ng["dhB"].set(q, 0, abs(G("chB", q) - G("chB", q + 1)))
        if qy < QH - 1:
            ng["dvA"].set(q, 0, abs(G("cvA", q) - G("cvA", q + QW)))
            ng["dvB"].set(q, 0, abs(G("cvB", q) - G("cvB", q + QW)))
    for k in range((QW - 2) * (QH - 2)):
        qx, qy = k % (QW - 2) + 1, k // (QW - 2) + 1
        q = qy * QW + qx
        termsA = [(("dhA", q + QW), ("dvA", q + 1), 1), (("dhA", q + QW - 1), ("dvA", q - QW + 1), 1),
                  (("dhB", q - BX), ("dvB", q - QW + AX), 1), (("dhA", q), ("dvA", q), 3),
                  (("dhA", q - 1), ("dvA", q - QW), 3), (("dhB", q - QW - BX), ("dvB", q - QW - BX), 1),
                  (("dhA", q - QW), ("dvA", q - 1), 1), (("dhA", q - QW - 1), ("dvA", q - QW - 1), 1)]
        termsB = [(("dhB", q + QW), ("dvB", q + 1), 1), (("dhB", q + QW - 1), ("dvB", q - QW + 1), 1),
                  (("dhA", q + QW - AX), ("dvA", q + BX), 1), (("dhB", q), ("dvB", q), 3),
                  (("dhB", q - 1), ("dvB", q - QW), 3), (("dhA", q - AX), ("dvA", q - AX), 1),
                  (("dhB", q - QW), ("dvB", q - 1), 1), (("dhB", q - QW - 1), ("dvB", q - QW - 1), 1)]
        hz = []
        for terms in (termsA, termsB):
            h = v = 0.0
            for (hn, hi), (vn, vi), w in terms:
                h += w * G(hn, hi)
                v += w * G(vn, vi)
            hz.append(v >= h)
        ga = (2 * qy - 2) * GW + 2 * qx - 2 + AX
        gb = (2 * qy - 1) * GW + 2 * qx - 2 + BX
        g0 = (2 * qy - 2) * GW + 2 * qx - 2 + BX
        g1 = (2 * qy - 1) * GW + 2 * qx - 2 + AX
        horiz.set(ga, 0, float(hz[0])); horiz.set(gb, 0, float(hz[1]))
        horiz.set(g0, 0, 1.0); horiz.set(g1, 0, 1.0)
        green.set(ga, 0, G("ghA", q) if hz[0] else G("gvA", q))
        green.set(gb, 0, G("ghB", q) if hz[1] else G("gvB", q))
        green.set(g0, 0, R((2 * qy + 2) * RW + 2 * qx + 2 + BX))
        green.set(g1, 0, R((2 * qy + 3) * RW + 2 * qx + 2 + AX))
    red, blue = flat(GW * GH), flat(GW * GH)
    for q in range((GW // 2) * (GH // 2)):
        qx, qy = q % (GW // 2), q // (GW // 2)
        for k in range(4):
            i, j = k & 1, k >> 1
            gx, gy = 2 * qx + i, 2 * qy + j
            if gx == 0 or gx == GW - 1 or gy == 0 or gy == GH - 1:
                continue
            pg = gy * GW + gx
            pr = (gy + 4) * RW + gx + 4
            rr = bb = 0.0
            if lay[k] == 0:
                rr = R(pr)
            if lay[k] == 2:
                bb = R(pr)
            if lay[k] == 1:
                red_h = lay[(j << 1) | (i ^ 1)] == 0
                dr, dg = (1, 1) if red_h else (RW, GW)
                br, bg = (RW, GW) if red_h else (1, 1)
                g = green.get(pg, 0)
                rr = (g + half(R(pr - dr), R(pr + dr))) - half(green.get(pg - dg, 0), green.get(pg + dg, 0))
                bb = (g + half(R(pr - br), R(pr + br))) - half(green.get(pg - bg, 0), green.get(pg + bg, 0))
            red.set(pg, 0, rr); blue.set(pg, 0, bb)
    for q in range((TW // 2) * (TH // 2)):
        qx, qy = q % (TW // 2), q // (TW // 2)
        for k in range(4):
            i, j = k & 1, k >> 1
            x, y = x0 + 2 * qx + i, y0 + 2 * qy + j
            pg = (2 * qy + j + 2) * GW + 2 * qx + i + 2
            d = 1 if horiz.get(pg, 0) else GW
            rr, bb = red.get(pg, 0), blue.get(pg, 0)
            if lay[k] == 2:
                rr = (bb + half(red.get(pg - d, 0), red.get(pg + d, 0))) - half(blue.get(pg - d, 0), blue.get(pg + d, 0))
            if lay[k] == 0:
                bb = (rr + half(blue.get(pg - d, 0), blue.get(pg + d, 0))) - half(red.get(pg - d, 0), red.get(pg + d, 0))
            if ox <= x < ox + ow and oy <= y < oy + oh:
                out[y - oy, x - ox] = (rr, green.get(pg, 0), bb)
