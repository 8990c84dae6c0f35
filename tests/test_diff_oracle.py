"""The float64 adjoint restatement (oracle/diff_oracle.py) against central
finite differences of its own forward model (CPU)."""
import numpy as np

from oracle import diff_oracle as D


def _case(seed=0, h=14, w=17):
    rng = np.random.default_rng(seed)
    return dict(s=rng.uniform(0.05, 0.9, (h, w)), quad=(2, 1, 1, 0), wb=np.array([1.8, 1.0, 1.4]), stops=0.3,
                M=np.array([[1.5, -0.3, -0.2], [-0.2, 1.4, -0.2], [0.05, -0.4, 1.35]]),
                kx=np.array([0, 0.1, 0.3, 0.6, 1.0, 1.6]), ky=np.array([0, 0.18, 0.4, 0.62, 0.85, 1.05]),
                r=2, eps=1e-3, k=0.5, dout=rng.normal(size=(h, w, 3)))


def _fd(fun, x, step):
    x = np.array(x, dtype=float)
    out = np.zeros_like(x)
    for i in np.ndindex(x.shape):
        xp, xm = x.copy(), x.copy()
        xp[i] += step
        xm[i] -= step
        out[i] = (fun(xp) - fun(xm)) / (2 * step)
    return out


def test_adjoint_matches_central_differences():
    c = _case()
    quad, kx, r, eps, dout = c["quad"], c["kx"], c["r"], c["eps"], c["dout"]

    def f(s, wb, stops, M, ky, k):
        return float((D.render_forward(s, quad, wb, stops, M, kx, ky, r, eps, k) * dout).sum())

    g = D.render_backward(c["s"], dout, quad, c["wb"], c["stops"], c["M"], kx, c["ky"], r, eps, c["k"])
    args = [c["s"], c["wb"], c["stops"], c["M"], c["ky"], c["k"]]
    for j, name in enumerate(["s", "wb", "stops", "M", "ky", "k"]):
        def fj(z, j=j):
            a = list(args)
            a[j] = z if np.ndim(args[j]) else float(z)
            return f(*a)
        fd = _fd(fj, args[j], 1e-6)
        err = np.max(np.abs(fd - g[j])) / max(1e-12, np.max(np.abs(fd)))
        assert err < 1e-6, (name, err)


def test_bilinear_adjoint_is_transpose():
    rng = np.random.default_rng(4)
    for quad in [(0, 1, 1, 2), (1, 0, 2, 1), (1, 2, 0, 1), (2, 1, 1, 0)]:
        s = rng.normal(size=(9, 11))
        d = rng.normal(size=(9, 11, 3))
        lhs = float((D.bilinear_forward(s, quad) * d).sum())
        rhs = float((s * D.bilinear_backward(d, quad)).sum())
        assert abs(lhs - rhs) < 1e-10 * max(1.0, abs(lhs))


def test_eps_adjoint_matches_central_differences():
    c = _case(seed=2)
    quad, kx, r, dout = c["quad"], c["kx"], c["r"], c["dout"]
    for eps in (1e-4, 1e-3, 1e-2):
        def f(e):
            return float((D.render_forward(c["s"], quad, c["wb"], c["stops"], c["M"], kx, c["ky"], r, e, c["k"])
                          * dout).sum())
        g = D.render_backward(c["s"], dout, quad, c["wb"], c["stops"], c["M"], kx, c["ky"], r, eps, c["k"])[6]
        step = 1e-4 * eps
        fd = (f(eps + step) - f(eps - step)) / (2 * step)
        assert abs(g - fd) <= 1e-6 * abs(fd), (eps, g, fd)


def _menon_quad(pattern, phase):
    cols = D.PATTERN_COLORS[pattern]
    return [cols[(((yy + phase[1]) & 1) * 2 + ((xx + phase[0]) & 1))] for yy in (0, 1) for xx in (0, 1)]


def test_menon_forward_matches_c_restatement(oracle):
    """The float64 Menon of the differentiable model equals the C restatement
    (pinned to the reference's frozen vectors) bit for bit after the float32
    cast, on every pattern and phase."""
    from oracle.oracle import RawSpec
    rng = np.random.default_rng(1)
    h, w = 23, 31
    for pat in range(4):
        for ph in ((0, 0), (1, 0), (0, 1), (1, 1)):
            codes = rng.integers(600, 15000, (h, w)).astype(np.uint16)
            spec = RawSpec(w, h, codes.reshape(-1), w, pat, ph[0], ph[1], (0, 0, w, h), (512,) * 4, (16383,) * 4)
            want = np.asarray(oracle.demosaic(spec, (0, 0, w, h), True), np.float32)
            plane = ((codes.astype(np.float32) - np.float32(512)) / np.float32(16383 - 512)).astype(np.float64)
            got, _ = D.menon_forward(plane, _menon_quad(pat, ph))
            assert np.array_equal(got.astype(np.float32).view(np.uint32), want.view(np.uint32)), (pat, ph)


def test_menon_adjoint_is_transpose():
    rng = np.random.default_rng(2)
    for h, w in ((9, 11), (14, 17), (2, 5), (3, 3), (1, 6)):
        for quad in [(0, 1, 1, 2), (1, 0, 2, 1), (1, 2, 0, 1), (2, 1, 1, 0)]:
            s = rng.normal(size=(h, w))
            u = rng.normal(size=(h, w, 3))
            H = D.menon_directions(s, quad)
            lhs = float((D.menon_forward(s, quad, H)[0] * u).sum())
            rhs = float((s * D.menon_backward(u, quad, H)).sum())
            assert abs(lhs - rhs) < 1e-10 * max(1.0, abs(lhs)), (h, w, quad)


def test_menon_render_adjoint_matches_central_differences():
    """Full model with a Menon demosaic, directions frozen at the forward's."""
    c = _case(seed=5)
    quad, kx, r, eps, dout = c["quad"], c["kx"], c["r"], c["eps"], c["dout"]
    H = D.menon_directions(c["s"], quad)

    def f(s, wb, stops, M, ky, k):
        return float((D.render_forward(s, quad, wb, stops, M, kx, ky, r, eps, k, demosaic="menon", horizontal=H)
                      * dout).sum())

    g = D.render_backward(c["s"], dout, quad, c["wb"], c["stops"], c["M"], kx, c["ky"], r, eps, c["k"],
                          demosaic="menon", horizontal=H)
    args = [c["s"], c["wb"], c["stops"], c["M"], c["ky"], c["k"]]
    for j, name in enumerate(["s", "wb", "stops", "M", "ky", "k"]):
        def fj(z, j=j):
            a = list(args)
            a[j] = z if np.ndim(args[j]) else float(z)
            return f(*a)
        fd = _fd(fj, args[j], 1e-6)
        err = np.max(np.abs(fd - g[j])) / max(1e-12, np.max(np.abs(fd)))
        assert err < 1e-6, (name, err)
