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


def _floor_half(v):
    return v // 2


def _pos_at(i, j, dx, dy):
    return ((j + dy) & 1) * 2 + ((i + dx) & 1)


def _quad_at(i, j, dx, dy, w):
    return _floor_half(j + dy) * w + _floor_half(i + dx)


def _fast_tile(meta, sample, color, x0, y0, viewport, out):
    """The interior quad path (menon_fast in render_raw.cu): every plane stored
    by quad position (raw at all four positions, chroma/gradients/green/
    directions at the non-green positions A and B, red/blue at the green
    positions G0 and G1), the kernel's strides, neighbour offsets and the
    epilogue's warp/lane mapping."""
    ox, oy, ow, oh = viewport
    RQW, RQH = (TW + 12) // 2, (TH + 12) // 2
    QW, QH = (TW + 8) // 2, (TH + 8) // 2
    GQW, GQH = QW - 2, QH - 2
    RQN, QN, GQN = RQW * RQH, QW * QH, GQW * GQH
    lay = [color(x0 + (k & 1), y0 + (k >> 1)) for k in range(4)]
    AX = 0 if lay[0] != 1 else 1          # column of the first row's non-green
    BX = 1 - AX

    def flat(n):
        return Plane(n, 1, 0, 0)

    raw = [flat(RQN) for _ in range(4)]
    ng = {name: flat(QN) for name in ("ghA", "ghB", "gvA", "gvB", "chA", "chB", "cvA", "cvB",
                                      "dhA", "dhB", "dvA", "dvB")}
    green, horiz = [flat(GQN), flat(GQN)], [flat(GQN), flat(GQN)]
    for q in range(RQN):
        qx, qy = q % RQW, q // RQW
        for k in range(4):
            raw[k].set(q, 0, sample(x0 - 6 + 2 * qx + (k & 1), y0 - 6 + 2 * qy + (k >> 1)))
    half = lambda a, b: 0.5 * (a + b)

    def R(i, j, dx, dy, rq):
        return raw[_pos_at(i, j, dx, dy)].get(rq + _quad_at(i, j, dx, dy, RQW), 0)

    def five(i, j, dx, dy, rq):
        return ((half(R(i, j, -dx, -dy, rq), R(i, j, dx, dy, rq)) + 0.5 * R(i, j, 0, 0, rq))
                - 0.25 * (R(i, j, -2 * dx, -2 * dy, rq) + R(i, j, 2 * dx, 2 * dy, rq)))

    for q in range(QN):
        qx, qy = q % QW, q // QW
        rq = (qy + 1) * RQW + qx + 1
        sa, sb = R(AX, 0, 0, 0, rq), R(BX, 1, 0, 0, rq)
        ha, va = five(AX, 0, 1, 0, rq), five(AX, 0, 0, 1, rq)
        hb, vb = five(BX, 1, 1, 0, rq), five(BX, 1, 0, 1, rq)
        ng["ghA"].set(q, 0, ha); ng["gvA"].set(q, 0, va)
        ng["chA"].set(q, 0, sa - ha); ng["cvA"].set(q, 0, sa - va)
        ng["ghB"].set(q, 0, hb); ng["gvB"].set(q, 0, vb)
        ng["chB"].set(q, 0, sb - hb); ng["cvB"].set(q, 0, sb - vb)
    G = lambda name, i: ng[name].get(i, 0)
    for q in range(QN):
        qx, qy = q % QW, q // QW
        if qx < QW - 1:
            ng["dhA"].set(q, 0, abs(G("chA", q) - G("chA", q + 1)))
            ng["dhB"].set(q, 0, abs(G("chB", q) - G("chB", q + 1)))
        if qy < QH - 1:
            ng["dvA"].set(q, 0, abs(G("cvA", q) - G("cvA", q + QW)))
            ng["dvB"].set(q, 0, abs(G("cvB", q) - G("cvB", q + QW)))
    for k in range(GQN):
        qx, qy = k % GQW + 1, k // GQW + 1
        q = qy * QW + qx
        termsA = [(("dhA", q + QW), ("dvA", q + 1), 1), (("dhA", q + QW - 1), ("dvA", q - QW + 1), 1),
                  (("dhB", q - BX), ("dvB", q - QW + AX), 1), (("dhA", q), ("dvA", q), 3),
                  (("dhA", q - 1), ("dvA", q - QW), 3), (("dhB", q - QW - BX), ("dvB", q - QW - BX), 1),
                  (("dhA", q - QW), ("dvA", q - 1), 1), (("dhA", q - QW - 1), ("dvA", q - QW - 1), 1)]
        termsB = [(("dhB", q + QW), ("dvB", q + 1), 1), (("dhB", q + QW - 1), ("dvB", q - QW + 1), 1),
                  (("dhA", q + QW - AX), ("dvA", q + BX), 1), (("dhB", q), ("dvB", q), 3),
                  (("dhB", q - 1), ("dvB", q - QW), 3), (("dhA", q - AX), ("dvA", q - AX), 1),
                  (("dhB", q - QW), ("dvB", q - 1), 1), (("dhB", q - QW - 1), ("dvB", q - QW - 1), 1)]
        for site, terms in enumerate((termsA, termsB)):
            h = v = 0.0
            for (hn, hi), (vn, vi), w in terms:
                h += w * G(hn, hi)
                v += w * G(vn, vi)
            hz = v >= h
            horiz[site].set(k, 0, float(hz))
            green[site].set(k, 0, G("ghA" if site == 0 else "ghB", q) if hz else G("gvA" if site == 0 else "gvB", q))

    def Gn(i, j, dx, dy, k):
        p = _pos_at(i, j, dx, dy)
        assert p in (AX, 2 + BX), "green_q reads a non-green position"
        return green[p >> 1].get(k + _quad_at(i, j, dx, dy, GQW), 0)

    rb = [flat(GQN) for _ in range(4)]      # red G0, red G1, blue G0, blue G1
    for k in range(GQN):
        qx, qy = k % GQW, k // GQW
        rq = (qy + 2) * RQW + qx + 2
        for gi, (i, j) in enumerate(((BX, 0), (AX, 1))):
            px, py = 2 * qx - 2 + i, 2 * qy - 2 + j
            if not (-1 <= px <= TW and -1 <= py <= TH):
                continue
            red_h = lay[(j << 1) | (i ^ 1)] == 0
            rx, ry = (1, 0) if red_h else (0, 1)
            bx, by = 1 - rx, 1 - ry
            g = R(i, j, 0, 0, rq)
            rr = (g + half(R(i, j, -rx, -ry, rq), R(i, j, rx, ry, rq))) - half(Gn(i, j, -rx, -ry, k), Gn(i, j, rx, ry, k))
            bb = (g + half(R(i, j, -bx, -by, rq), R(i, j, bx, by, rq))) - half(Gn(i, j, -bx, -by, k), Gn(i, j, bx, by, k))
            rb[gi].set(k, 0, rr)
            rb[2 + gi].set(k, 0, bb)
    for t in range(256):
        w, lane = t >> 5, t & 31
        row = w + (TH // 2) * (lane >> 4)
        qx, qy = lane & 15, row >> 1
        j = w & 1
        assert row & 1 == j
        k = (qy + 1) * GQW + qx + 1
        rq = (qy + 3) * RQW + qx + 3
        ni = AX if j == 0 else BX
        gi = 1 - ni
        px = {}
        # green position of the row
        px[gi] = (rb[j].get(k, 0), R(gi, j, 0, 0, rq), rb[2 + j].get(k, 0))
        hz = horiz[j].get(k, 0) != 0
        plane = j if hz else 1 - j
        om = k + (_quad_at(ni, j, -1, 0, GQW) if hz else _quad_at(ni, j, 0, -1, GQW))
        op = k + (_quad_at(ni, j, 1, 0, GQW) if hz else _quad_at(ni, j, 0, 1, GQW))
        red, blue = rb[plane], rb[2 + plane]
        s = R(ni, j, 0, 0, rq)
        if lay[2 * j + ni] == 2:
            rr = (s + half(red.get(om, 0), red.get(op, 0))) - half(blue.get(om, 0), blue.get(op, 0))
            px[ni] = (rr, green[j].get(k, 0), s)
        else:
            bb = (s + half(blue.get(om, 0), blue.get(op, 0))) - half(red.get(om, 0), red.get(op, 0))
            px[ni] = (s, green[j].get(k, 0), bb)
        for i in range(2):
            x, y = x0 + 2 * qx + i, y0 + row
            if ox <= x < ox + ow and oy <= y < oy + oh:
                out[y - oy, x - ox] = px[i]
