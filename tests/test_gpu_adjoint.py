"""The decode's derivatives, checked two ways on a B200 (block (b) over level 1, block (c') over level 0).

- The assembled stencil against the fused forward/adjoint operator: H x from the stencil the assembly stored (the
  reference's per-texel blocks, src/solve_level1.cu:259-581) and from nntc_b200_probe_jtj_level{1,0}, which apply
  J^T diag(cw) J site by site without assembling anything, agree to 1e-12 relative on random vectors.
- The assembled gradient against central finite differences of the objective: for a random direction d the change of
  a plane's E between v + h d and v - h d is 4 g.d / (sum cw x sites) (E is quadratic in level 1), to 1e-6 relative
  (the objective samples in double, the assembly in float)."""
import ctypes as C

import numpy as np
import pytest

from nntc_b200 import check, lib, materials
from nntc_b200.session import Session

pytestmark = pytest.mark.gpu

SLOT_OFFSETS = [(0, 0), (1, 0), (-1, 1), (0, 1), (1, 1)]   # self, right, down-left, down, down-right


def random_state(mat, seed):
    rng = np.random.default_rng(seed)
    nin = mat.c1 + mat.c0 + mat.c0 * mat.c1
    nout = 3 * len(mat.textures)
    w = (rng.standard_normal((nout, nin)) * 0.3).astype(np.float32)
    b = rng.random(nout).astype(np.float32)
    v0 = [(rng.random(p[0] * p[1] * mat.c0) * 2 - 1).astype(np.float32) for p in mat.planes]
    v1 = [(rng.random(p[2] * p[3] * mat.c1) * 2 - 1).astype(np.float32) for p in mat.planes]
    return w, b, v0, v1


def stencil_product(stencil, x, w, h, c):
    """y = H x from the reference-ordered stencil [texel][slot][i][j] (owned blocks and the neighbours' transposes)."""
    S = stencil.reshape(h, w, 5, c, c)
    X = x.reshape(h, w, c)
    y = np.einsum("yxij,yxj->yxi", S[:, :, 0], X)
    for slot, (dx, dy) in enumerate(SLOT_OFFSETS):
        if slot == 0:
            continue
        for ty in range(h):
            for tx in range(w):
                fx, fy = tx + dx, ty + dy
                if 0 <= fx < w and 0 <= fy < h:
                    y[ty, tx] += S[ty, tx, slot] @ X[fy, fx]          # this texel's block times its neighbour
                    y[fy, fx] += S[ty, tx, slot].T @ X[ty, tx]        # the neighbour's row: the transpose
    return y.ravel()


@pytest.mark.parametrize("level0", [False, True])
@pytest.mark.parametrize("textures,c0,c1,w,h", [(2, 4, 4, 72, 40), (1, 2, 4, 61, 37), (2, 3, 2, 64, 64)])
def test_matrix_free_operator_matches_the_assembled_stencil(textures, c0, c1, w, h, level0):
    mat = materials.small(80 + w, w, h, textures=textures, c0=c0, c1=c1)
    dw, db, v0, v1 = random_state(mat, w + 7 * h)
    rng = np.random.default_rng(3)
    probe = lib().nntc_b200_probe_jtj_level0 if level0 else lib().nntc_b200_probe_jtj_level1
    with Session(mat) as s:
        for i in range(len(mat.planes)):
            s.set_planes(i, v0[i], v1[i])
        s.set_decoder(dw, db)
        s.set_grids(np.full(c0, -1.0), np.full(c0, 1.0))
        s.block(level0)   # assembles every plane's stencil of that latent
        c = c0 if level0 else c1
        for i, p in enumerate(mat.planes):
            uw, uh = (p[0], p[1]) if level0 else (p[2], p[3])
            ws = s.workspace(i, level0)
            for _ in range(2):
                x = rng.standard_normal(uw * uh * c)
                want = stencil_product(ws["stencil"], x, uw, uh, c)
                got = np.zeros_like(x)
                check(probe(s.d, 4, i, x.ctypes.data_as(C.POINTER(C.c_double)),
                            got.ctypes.data_as(C.POINTER(C.c_double)), got.size), "jtj")
                assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max(), (i, np.abs(got - want).max())


@pytest.mark.parametrize("level0", [False, True])
@pytest.mark.parametrize("textures,c0,c1,w,h", [(2, 4, 4, 72, 40), (1, 2, 4, 61, 37)])
def test_gradient_matches_central_differences(textures, c0, c1, w, h, level0):
    mat = materials.small(90 + w, w, h, textures=textures, c0=c0, c1=c1)
    dw, db, v0, v1 = random_state(mat, 5 * w + h)
    rng = np.random.default_rng(4)
    k = 4
    with Session(mat) as s:
        for i in range(len(mat.planes)):
            s.set_planes(i, v0[i], v1[i])
        s.set_decoder(dw, db)
        s.set_grids(np.full(c0, -1.0), np.full(c0, 1.0))
        s.block(level0)   # assembles the gradient at the planes as set, then the solve moves them
        sum_cw = float(np.sum(np.array(s.m.cw[: s.m.nout], np.float64)))
        for i, p in enumerate(mat.planes[:2]):
            g = s.workspace(i, level0)["grad"]
            prev = (v0 if level0 else v1)[i]   # the point the gradient was assembled at
            d = rng.standard_normal(prev.size)
            hstep = 1e-3
            vp = (prev + hstep * d).astype(np.float32)
            vm = (prev - hstep * d).astype(np.float32)
            put = (lambda v: s.set_planes(i, v0=v)) if level0 else (lambda v: s.set_planes(i, v1=v))
            put(vp)
            ep = s.objective(k).e_plane[i]
            put(vm)
            em = s.objective(k).e_plane[i]
            put(prev)
            delta = (vp.astype(np.float64) - vm.astype(np.float64)) / 2.0
            sites = float(p[0]) * float(p[1]) * (1 + k)
            fd = (ep - em) * sum_cw * sites / 4.0
            gd = float(g @ delta)
            assert abs(fd - gd) <= 1e-6 * abs(gd), (i, fd, gd)
