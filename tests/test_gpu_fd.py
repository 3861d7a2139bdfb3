"""The decode's adjoint against central finite differences, as the adjoint check of the 4 x 1024 x 1024 material
(c0 2, c1 4) specifies it: a 64 x 64 crop of that material (its four textures cropped at the top-left, with their own
mip chain), FP64 differences with step h = 1e-3 along 256 random unit directions (numpy's default_rng).

- The gradient (nntc_b200_objective_gradient: J^T diag(cw) r gathered per texel for both latents, 2 cw (A x - rhs)
  for the decoder) against (E(x + h d) - E(x - h d)) / 2h of the FP64 objective (tests/fp64_model.py), along
  directions over every parameter at once (both latents of every plane, the decoder's weights and biases).
- The Gauss-Newton operators J^T diag(cw) J of blocks (b) and (c') applied matrix-free on the device
  (nntc_b200_probe_jtj_level1 / _level0): d . H d against |J d|^2_cw with J d = (r(x + h d) - r(x - h d)) / 2h of
  the FP64 residuals (exact up to rounding: the decode is linear in either latent alone), 128 directions a level."""
import ctypes as C

import numpy as np
import pytest

import fp64_model as F
from nntc_b200 import abi, check, lib, materials
from nntc_b200.session import Session

pytestmark = pytest.mark.gpu

H = 1e-3
DIRECTIONS = 256


def crop_material():
    full = materials.config(2)
    tex = [t[:64, :64].copy() for t in full.textures]
    return materials.Material("4x64x64 crop of 4x1024x1024 pbr", tex, full.c0, full.c1, full.k).build()


def state(mat, rng):
    nin, nout = abi.feature_count(mat.c0, mat.c1), mat.nout
    v0 = [(rng.random(p[0] * p[1] * mat.c0) * 2 - 1).astype(np.float32) for p in mat.planes]
    v1 = [(rng.random(p[2] * p[3] * mat.c1) * 2 - 1).astype(np.float32) for p in mat.planes]
    W = (rng.standard_normal((nout, nin)) * 0.3).astype(np.float32)
    b = rng.random(nout).astype(np.float32)
    return v0, v1, W, b


def test_gradient_vs_central_differences():
    mat = crop_material()
    rng = np.random.default_rng(2)
    v0, v1, W, b = state(mat, rng)
    cw = np.ones(mat.nout)
    k = mat.k
    with Session(mat) as s:
        for i in range(len(mat.planes)):
            s.set_planes(i, v0[i], v1[i])
        s.set_decoder(W, b)
        s.set_grids(np.full(mat.c0, -1.0), np.full(mat.c0, 1.0))
        g0 = [np.zeros(v.size) for v in v0]
        g1 = [np.zeros(v.size) for v in v1]
        gd = np.zeros(mat.nout * (W.shape[1] + 1))
        pp = lambda arrs: (C.POINTER(C.c_double) * len(arrs))(*[a.ctypes.data_as(C.POINTER(C.c_double)) for a in arrs])
        check(lib().nntc_b200_objective_gradient(s.d, C.byref(s.m), k, s.per_site, pp(g0), pp(g1),
                                                 gd.ctypes.data_as(C.POINTER(C.c_double))), "gradient")
    sizes = [v.size for v in v0] + [v.size for v in v1] + [gd.size]
    g = np.concatenate(g0 + g1 + [gd])
    x0 = np.concatenate([v.astype(np.float64) for v in v0] + [v.astype(np.float64) for v in v1] +
                        [np.concatenate([W.astype(np.float64), b.astype(np.float64)[:, None]], axis=1).ravel()])
    np_ = len(mat.planes)

    def E(x):
        parts = np.split(x, np.cumsum(sizes)[:-1])
        dec = parts[-1].reshape(mat.nout, -1)
        return F.objective(mat, parts[:np_], parts[np_:2 * np_], dec[:, :-1], dec[:, -1], cw, k)

    gnorm = np.linalg.norm(g)
    worst = 0.0
    for _ in range(DIRECTIONS):
        d = rng.standard_normal(x0.size)
        d /= np.linalg.norm(d)
        fd = (E(x0 + H * d) - E(x0 - H * d)) / (2 * H)
        worst = max(worst, abs(fd - g @ d) / gnorm)
    assert worst <= 1e-5, worst


@pytest.mark.parametrize("level0", [False, True])
def test_gauss_newton_operator_vs_central_differences(level0):
    mat = crop_material()
    rng = np.random.default_rng(3 + level0)
    v0, v1, W, b = state(mat, rng)
    cw = np.ones(mat.nout)
    k = mat.k
    worst = 0.0
    with Session(mat) as s:
        for i in range(len(mat.planes)):
            s.set_planes(i, v0[i], v1[i])
        s.set_decoder(W, b)
        s.set_grids(np.full(mat.c0, -1.0), np.full(mat.c0, 1.0))
        probe = lib().nntc_b200_probe_jtj_level0 if level0 else lib().nntc_b200_probe_jtj_level1
        per_plane = DIRECTIONS // 2 // len(mat.planes) + 1
        for i, lay in enumerate(mat.planes):
            base0 = v0[i].astype(np.float64)
            base1 = v1[i].astype(np.float64)
            n = base0.size if level0 else base1.size
            for _ in range(per_plane):
                d = rng.standard_normal(n)
                d /= np.linalg.norm(d)
                y = np.zeros(n)
                check(probe(s.d, k, i, d.ctypes.data_as(C.POINTER(C.c_double)),
                            y.ctypes.data_as(C.POINTER(C.c_double)), n), "jtj")

                def r(sign):
                    a0 = base0 + sign * H * d if level0 else base0
                    a1 = base1 if level0 else base1 + sign * H * d
                    return F.plane_residuals(lay, mat.chain[i], a0, a1, W.astype(np.float64),
                                             b.astype(np.float64), mat.c0, mat.c1, k)

                jd = (r(1) - r(-1)) / (2 * H)
                q_fd = float(np.sum((jd * jd) @ cw))
                worst = max(worst, abs(d @ y - q_fd) / max(q_fd, 1e-300))
    assert worst <= 1e-5, worst
