"""CPU model of the strip-streaming spatial kernels' indexing (spatial.cu).

gf_strip_kernel and ls_strip_kernel keep their window sums in skewed
shared-memory planes, a ring of row sums per CTA in global memory and a few
registers per thread.  This model runs the same index arithmetic -- tasks,
bands, the four phases per block of R rows, the skew, the ring slots -- with
bounds-checked NumPy arrays that are poisoned with NaN whenever their contents
become dead, so that

* every shared-memory, ring, input and output index the kernels form is
  proven in bounds for the geometries exercised (several strips and bands,
  partial last strips and bands, images narrower and shorter than a strip,
  radii up to 32),
* no read sees an entry that the current block did not write (NaN would
  propagate into the result), and
* every output pixel is written exactly once, with the values of the oracle.

Threads are vectorized: one NumPy lane per thread of a phase.  It is test
infrastructure: the kernels are never generated from it.
"""
from __future__ import annotations

import numpy as np

PROPHOTO = (0.28807112822929337, 0.00008565396060525903)
REC2020 = (0.26270021201126703, 0.059301716469861945)


class Flat:
    """A bounds-checked, poisonable flat array (a shared-memory plane or ring)."""

    def __init__(self, n, dtype=np.float64):
        self.a = np.full(n, np.nan, dtype) if dtype == np.float64 else np.full(n, -(1 << 30), dtype)
        self.dtype = dtype

    def poison(self):
        self.a[:] = np.nan if self.dtype == np.float64 else -(1 << 30)

    def _check(self, idx):
        idx = np.asarray(idx)
        if idx.size and (idx.min() < 0 or idx.max() >= self.a.size):
            raise IndexError(f"index {idx.min()}..{idx.max()} outside {self.a.size}")
        return idx

    def get(self, idx):
        v = self.a[self._check(idx)]
        bad = np.isnan(v) if self.dtype == np.float64 else v == -(1 << 30)
        if np.any(bad):
            raise ValueError("read of an entry this block did not write")
        return v

    def set(self, idx, v):
        self.a[self._check(idx)] = v


def sk(j, K):
    return j + j // K


def plane_len(n, K):
    return n + n // K + 1


def extent(c, r, n):
    return np.minimum(n - 1, c + r) - np.maximum(0, c - r) + 1


def band_height(height, strips, ctas, halo):
    bands = max(1, ctas // strips)
    th = (height + bands - 1) // bands
    th = max(th, max(16, 2 * halo))
    return min(th, height)


def block_sums(plane, plen, rows, nb, m, K, bs):
    """block_sums<NT, K, M>: bs[(i*M + k)*nb + b] = plane (i, k) over [bK, bK + K)."""
    for i in range(rows):
        for b in range(nb):
            base = i * m * plen + b * (K + 1)
            for k in range(m):
                bs.set((i * m + k) * nb + b, plane.get(base + k * plen + np.arange(K)).sum())


def window_start(plane, row_base, plen, bs, bs_base, nb, c0, r, m, K):
    """window_start<K, M> for an array of segment starts c0 (multiples of K)."""
    b0, q = c0 // K, (2 * r + 1) // K
    S = np.zeros((c0.size, m))
    for b in range(q):
        for k in range(m):
            S[:, k] += bs.get(bs_base + k * nb + b0 + b)
    for j in range(q * K, 2 * r + 1):
        for k in range(m):
            S[:, k] += plane.get(row_base + k * plen + sk(c0 + j, K))
    return S


def _load(img, x, y, mask):
    """Input pixels of columns x (where mask) at row y; zero elsewhere."""
    h, w = img.shape[:2]
    if not (0 <= y < h):
        raise IndexError(f"input row {y} outside {h}")
    out = np.zeros((x.size, 3), np.float64)
    xs = x[mask]
    if xs.size and (xs.min() < 0 or xs.max() >= w):
        raise IndexError("input column outside the image")
    out[mask] = img[y, xs].astype(np.float64)
    return out


def guided_filter(img, r, eps, space=0, NT=256, R=4, K=8, ctas=8):
    """The output of gf_strip_kernel<NT, R, K> on `img` (h, w, 3) float32."""
    img = np.ascontiguousarray(img, np.float32)
    H, W = img.shape[:2]
    wr, wb = PROPHOTO if space == 0 else REC2020
    tw = NT - 4 * r
    assert tw > 0
    strips = (W + tw - 1) // tw
    th = band_height(H, strips, ctas, 2 * r)
    tasks = strips * ((H + th - 1) // th)
    grid = min(tasks, ctas)
    c1p = plane_len(NT, K)
    c2 = tw + 2 * r
    c2p = c2 + c2 // K + 1
    period = 2 * r + 1
    out = np.full((H, W, 3), np.nan, np.float32)
    written = np.zeros((H, W), np.int32)
    tid = np.arange(NT)

    def moments(x, y):
        mask = (x >= 0) & (x < W)
        p = _load(img, x, y, mask)
        yy = p[:, 1] + wr * (p[:, 0] - p[:, 1]) + wb * (p[:, 2] - p[:, 1])
        m = np.stack([p[:, 0], p[:, 1], p[:, 2], yy * p[:, 0], yy * p[:, 1], yy * p[:, 2]], 1)
        m[~mask] = 0
        return m

    nbv, nba = NT // K, c2 // K
    for cta in range(grid):
        vb = Flat(R * 6 * c1p)       # also H2b
        ab = Flat(R * 6 * c2p)
        bs = Flat(R * 6 * nbv)
        ring = Flat(period * 6 * tw)
        for task in range(cta, tasks, grid):
            band, strip = task // strips, task % strips
            x0, y0 = strip * tw, band * th
            y1 = min(H, y0 + th)
            xa = x0 - 2 * r
            tc0 = max(0, y0 - r)
            t_end = y1 - 1 + r
            last_centre = min(H - 1, t_end)
            V = np.zeros((NT, 6))
            for y in range(max(0, tc0 - r), min(H - 1, tc0 + r - 1) + 1):
                V += moments(xa + tid, y)
            Q = np.zeros((tw, 6))
            for tb in range(tc0, t_end + 1, R):
                rows = min(R, last_centre - tb + 1)
                vb.poison()
                for i in range(max(rows, 0)):           # phase A
                    t = tb + i
                    if t + r <= H - 1:
                        V += moments(xa + tid, t + r)
                    if t - r - 1 >= max(0, tc0 - r):
                        V -= moments(xa + tid, t - r - 1)
                    for k in range(6):
                        vb.set(i * 6 * c1p + k * c1p + sk(tid, K), V[:, k])
                ab.poison()
                bs.poison()
                block_sums(vb, c1p, max(rows, 0), nbv, 6, K, bs)
                segs = (c2 + K - 1) // K
                for i in range(max(rows, 0)):           # phase B (lanes = segments)
                    t = tb + i
                    c0 = np.arange(segs) * K
                    S = window_start(vb, i * 6 * c1p, c1p, bs, i * 6 * nbv, nbv, c0, r, 6, K)
                    wy = float(extent(t, r, H))
                    for d in range(K):
                        c = c0 + d
                        live = c < c2
                        if d:
                            for k in range(6):
                                S[live, k] += (vb.get(i * 6 * c1p + k * c1p + sk(c[live] + 2 * r, K)) -
                                               vb.get(i * 6 * c1p + k * c1p + sk(c[live] - 1, K)))
                        xc = x0 - r + c
                        inside = live & (xc >= 0) & (xc < W)
                        zero = live & ~inside
                        for k in range(6):
                            ab.set(i * 6 * c2p + k * c2p + sk(c[zero], K), 0.0)
                        if not inside.any():
                            continue
                        s = S[inside]
                        inv_n = 1.0 / (extent(xc[inside], r, W).astype(np.float64) * wy)
                        sy = s[:, 1] + wr * (s[:, 0] - s[:, 1]) + wb * (s[:, 2] - s[:, 1])
                        syy = s[:, 4] + wr * (s[:, 3] - s[:, 4]) + wb * (s[:, 5] - s[:, 4])
                        my = sy * inv_n
                        var = np.maximum(syy * inv_n - my * my, 0.0)
                        inv = 1.0 / (var + eps)
                        for ch in range(3):
                            mp = s[:, ch] * inv_n
                            a = (s[:, 3 + ch] * inv_n - my * mp) * inv
                            b = mp - a * my
                            ab.set(i * 6 * c2p + ch * c2p + sk(c[inside], K), a)
                            ab.set(i * 6 * c2p + (3 + ch) * c2p + sk(c[inside], K), b)
                vb.poison()                              # Vb is dead; H2b aliases it
                bs.poison()
                block_sums(ab, c2p, max(rows, 0), nba, 6, K, bs)
                segs_c = (tw + K - 1) // K
                for i in range(max(rows, 0)):           # phase C
                    o0 = np.arange(segs_c) * K
                    S = window_start(ab, i * 6 * c2p, c2p, bs, i * 6 * nba, nba, o0, r, 6, K)
                    for d in range(K):
                        o = o0 + d
                        live = o < tw
                        if d:
                            for k in range(6):
                                S[live, k] += (ab.get(i * 6 * c2p + k * c2p + sk(o[live] + 2 * r, K)) -
                                               ab.get(i * 6 * c2p + k * c2p + sk(o[live] - 1, K)))
                        for k in range(6):
                            vb.set(i * 6 * c1p + k * c1p + sk(o[live], K), S[live, k])
                steps = min(R, t_end - tb + 1)
                lanes = np.arange(tw)
                for i in range(steps):                  # phase D (lanes = output columns)
                    t = tb + i
                    slot = (t % period) * 6 * tw
                    h = None
                    if t <= last_centre:
                        h = np.stack([vb.get(i * 6 * c1p + k * c1p + sk(lanes, K)) for k in range(6)], 1)
                        Q += h
                    if t - period >= tc0:
                        Q -= np.stack([ring.get(slot + k * tw + lanes) for k in range(6)], 1)
                    if t <= last_centre:
                        for k in range(6):
                            ring.set(slot + k * tw + lanes, h[:, k])
                    yo = t - r
                    x = x0 + lanes
                    emit = (x < W) & (yo >= y0) & (yo < y1)
                    if not emit.any():
                        continue
                    xs = x[emit]
                    p = img[yo, xs].astype(np.float64)
                    Y = p[:, 1] + wr * (p[:, 0] - p[:, 1]) + wb * (p[:, 2] - p[:, 1])
                    inv_n = 1.0 / (extent(xs, r, W).astype(np.float64) * float(extent(yo, r, H)))
                    qq = Q[emit]
                    for ch in range(3):
                        q = (qq[:, ch] * inv_n) * Y + qq[:, 3 + ch] * inv_n
                        out[yo, xs, ch] = np.where(q - p[:, ch] == 0, img[yo, xs, ch], q.astype(np.float32))
                    written[yo, xs] += 1
    assert np.all(written == 1), "every output pixel is written exactly once"
    return out


def local_statistics(img, r, NT=256, R=4, K=8, ctas=8):
    """(mean, variance, count) of ls_strip_kernel on `img` (h, w, 3) float32."""
    img = np.ascontiguousarray(img, np.float32)
    H, W = img.shape[:2]
    tw = NT - 2 * r
    strips = (W + tw - 1) // tw
    th = band_height(H, strips, ctas, r)
    tasks = strips * ((H + th - 1) // th)
    grid = min(tasks, ctas)
    c1p = plane_len(NT, K)
    mean = np.full((H, W, 3), np.nan)
    var = np.full((H, W, 3), np.nan)
    cnt = np.full((H, W, 3), -1, np.int64)
    written = np.zeros((H, W), np.int32)
    tid = np.arange(NT)
    nblk = NT // K
    for cta in range(grid):
        vb = Flat(R * 6 * c1p)
        nb = Flat(R * 3 * c1p, np.int64)
        bsv = Flat(R * 6 * nblk)
        bsn = Flat(R * 3 * nblk, np.int64)
        for task in range(cta, tasks, grid):
            band, strip = task // strips, task % strips
            x0, y0 = strip * tw, band * th
            y1 = min(H, y0 + th)
            first = img[y0, x0].astype(np.float64)
            shift = np.where(np.isfinite(first), first, 0.0)
            x = x0 - r + tid
            inside = (x >= 0) & (x < W)
            s1 = np.zeros((NT, 3))
            s2 = np.zeros((NT, 3))
            n = np.zeros((NT, 3), np.int64)

            def add(y, sign):
                p = _load(img, x, y, inside)
                fin = np.isfinite(p) & inside[:, None]
                d = np.where(fin, p - shift, 0.0)
                s1[:] += sign * d
                s2[:] += sign * d * d
                n[:] += sign * fin

            for y in range(max(0, y0 - r), min(H - 1, y0 + r - 1) + 1):
                add(y, 1)
            for tb in range(y0, y1, R):
                rows = min(R, y1 - tb)
                vb.poison()
                nb.poison()
                for i in range(rows):
                    t = tb + i
                    if t + r <= H - 1:
                        add(t + r, 1)
                    if t - r - 1 >= max(0, y0 - r):
                        add(t - r - 1, -1)
                    for c in range(3):
                        vb.set(i * 6 * c1p + c * c1p + sk(tid, K), s1[:, c])
                        vb.set(i * 6 * c1p + (3 + c) * c1p + sk(tid, K), s2[:, c])
                        nb.set(i * 3 * c1p + c * c1p + sk(tid, K), n[:, c])
                bsv.poison()
                bsn.poison()
                block_sums(vb, c1p, rows, nblk, 6, K, bsv)
                block_sums(nb, c1p, rows, nblk, 3, K, bsn)
                segs = (tw + K - 1) // K
                for i in range(rows):
                    t = tb + i
                    o0 = np.arange(segs) * K
                    S = window_start(vb, i * 6 * c1p, c1p, bsv, i * 6 * nblk, nblk, o0, r, 6, K)
                    N = window_start(nb, i * 3 * c1p, c1p, bsn, i * 3 * nblk, nblk, o0, r, 3, K).astype(np.int64)
                    for d in range(K):
                        o = o0 + d
                        live = o < tw
                        if d:
                            for k in range(6):
                                S[live, k] += (vb.get(i * 6 * c1p + k * c1p + sk(o[live] + 2 * r, K)) -
                                               vb.get(i * 6 * c1p + k * c1p + sk(o[live] - 1, K)))
                            for c in range(3):
                                N[live, c] += (nb.get(i * 3 * c1p + c * c1p + sk(o[live] + 2 * r, K)) -
                                               nb.get(i * 3 * c1p + c * c1p + sk(o[live] - 1, K)))
                        xo = x0 + o
                        emit = live & (xo < W)
                        if not emit.any():
                            continue
                        xs = xo[emit]
                        ss, nn = S[emit], N[emit]
                        with np.errstate(invalid="ignore", divide="ignore"):
                            m = ss[:, :3] / nn
                            v = np.maximum((ss[:, 3:] - ss[:, :3] * m) / nn, 0.0)
                        m = np.where(nn == 0, np.nan, shift + m)
                        v = np.where(nn == 0, np.nan, v)
                        mean[t, xs] = m
                        var[t, xs] = v
                        cnt[t, xs] = nn
                        written[t, xs] += 1
    assert np.all(written == 1), "every output pixel is written exactly once"
    return mean, var, cnt
