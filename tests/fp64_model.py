"""An FP64 restatement of the encoder's objective for the tests: every site of every plane, the site positions and the
bilinear rule in double u-space (src/objective.cu:97-118, src/sample.cuh:43-178), the features [c][s][s c], the affine
decoder, the per-output weights and the per-plane site weights, all in float64. It is the smooth function the
finite-difference checks differentiate and the FP64 reference the mixed-precision form's errors are measured against.
Test infrastructure: nothing in the product imports it."""
import numpy as np

ROT4 = np.array([(-0.375, -0.125), (-0.125, 0.375), (0.125, -0.375), (0.375, 0.125)])


def site_offsets(k, px, py):
    """(dx, dy) of site j = 1..k of every pixel (px, py): arrays of shape (k, n)."""
    n = px.size
    if k == 0:
        return np.zeros((0, n)), np.zeros((0, n))
    if k == 2:
        dx = np.array([-0.25, 0.25])[:, None].repeat(n, 1)
        dy = np.array([0.25, -0.25])[:, None].repeat(n, 1)
        return dx, dy
    base = ROT4 if k == 4 else np.array([(0.25, 0.25)])
    turns = (py & 1) * 2 + (px & 1)
    dx = np.empty((k, n))
    dy = np.empty((k, n))
    for j in range(k):
        ox = np.full(n, base[j, 0])
        oy = np.full(n, base[j, 1])
        for r in range(3):
            m = turns > r
            ox[m], oy[m] = -oy[m], ox[m].copy()
        dx[j], dy[j] = ox, oy
    return dx, dy


def bilinear(plane, w, h, c, u, v):
    """plane (h w c, float64) at u-space (u, v) arrays: the four taps clamped, weights in double."""
    x = u * w - 0.5
    y = v * h - 0.5
    xf = np.floor(x)
    yf = np.floor(y)
    fx = (x - xf)[:, None]
    fy = (y - yf)[:, None]
    x0 = np.clip(xf.astype(np.int64), 0, w - 1)
    x1 = np.clip(xf.astype(np.int64) + 1, 0, w - 1)
    y0 = np.clip(yf.astype(np.int64), 0, h - 1)
    y1 = np.clip(yf.astype(np.int64) + 1, 0, h - 1)
    p = plane.reshape(h, w, c)
    return ((1 - fx) * (1 - fy) * p[y0, x0] + fx * (1 - fy) * p[y0, x1] + (1 - fx) * fy * p[y1, x0] +
            fx * fy * p[y1, x1])


def plane_residuals(layout, src, v0, v1, W, b, c0, c1, k):
    """The residuals decode - target at every site of one plane: (sites, nout), centres first then site j = 1..k."""
    w0, h0, w1, h1 = layout
    nout = W.shape[0]
    py, px = np.divmod(np.arange(w0 * h0), w0)
    dx, dy = site_offsets(k, px, py)
    out = []
    for j in range(k + 1):
        ox = np.zeros(px.size) if j == 0 else dx[j - 1]
        oy = np.zeros(px.size) if j == 0 else dy[j - 1]
        u = (px + 0.5 + ox) / w0
        v = (py + 0.5 + oy) / h0
        c = bilinear(v1, w1, h1, c1, u, v)
        if j == 0:
            s = v0.reshape(-1, c0).astype(np.float64)
            t = src.reshape(-1, nout).astype(np.float64)
        else:
            s = bilinear(v0, w0, h0, c0, u, v)
            t = bilinear(src, w0, h0, nout, u, v)
        phi = np.concatenate([c, s, (s[:, :, None] * c[:, None, :]).reshape(-1, c0 * c1)], axis=1)
        out.append(phi @ W.T + b - t)
    return np.concatenate(out, axis=0)


def objective(mat, v0s, v1s, W, b, cw, k):
    """E, normalised as the encoder normalises it."""
    num = den = 0.0
    for i, lay in enumerate(mat.planes):
        r = plane_residuals(lay, mat.chain[i], v0s[i], v1s[i], W, b, mat.c0, mat.c1, k)
        num += mat.per_site[i] * float(np.sum((r * r) @ cw))
        den += mat.per_site[i] * lay[0] * lay[1] * (1 + k)
    return num / (float(np.sum(cw)) * den)
