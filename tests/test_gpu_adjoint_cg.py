"""The adjoint form's conjugate gradients on a B200: blocks (b) and (c') with (H + lambda I) p applied matrix-free in
FP32 (adjoint_cg.cu) against the same blocks on the assembled FP64 stencil, from the same state.

- The operator: one CG product of the matrix-free form equals the stencil's product on the same direction to FP32
  rounding (checked through a whole solve: the same gradient and diagonal blocks are assembled by both, bit for bit,
  and the corrections agree to the FP32 stop, 1e-6 of the right-hand side, amplified at most by the condition of the
  preconditioned system; the bar is 1e-3 of the correction's largest entry).
- Only the diagonal blocks and the gradient are assembled: those are the stencil form's, bit for bit."""
import ctypes as C

import numpy as np
import pytest

from nntc_b200 import abi, check, lib, materials
from nntc_b200.session import Session

pytestmark = pytest.mark.gpu


def setup(s, mat, rng, c0, c1):
    nin, nout = abi.feature_count(c0, c1), 3 * len(mat.textures)
    s.set_decoder((rng.standard_normal((nout, nin)) * 0.3).astype(np.float32), rng.random(nout).astype(np.float32))
    s.set_grids(np.full(c0, -1.0), np.full(c0, 1.0))
    for i, p in enumerate(mat.planes):
        s.set_planes(i, (rng.random(p[0] * p[1] * c0) * 2 - 1).astype(np.float32),
                     (rng.random(p[2] * p[3] * c1) * 2 - 1).astype(np.float32))


@pytest.mark.parametrize("level0", [False, True])
@pytest.mark.parametrize("textures,c0,c1,w,h,k", [(2, 2, 4, 72, 56, 4), (4, 4, 4, 64, 64, 4), (1, 3, 2, 37, 29, 2),
                                                  (2, 1, 3, 40, 24, 0)])
def test_matrix_free_cg_vs_stencil(level0, textures, c0, c1, w, h, k):
    mat = materials.small(w + h + c0, w, h, textures=textures, c0=c0, c1=c1, k=k)
    out = {}
    for adjoint in (0, 1):
        with Session(mat) as s:
            setup(s, mat, np.random.default_rng(w * h), c0, c1)
            check(lib().nntc_b200_set_option(s.d, abi.OPT_ADJOINT_CG, adjoint), "option")
            rep, _ = s.block(level0, k=k)
            out[adjoint] = [s.workspace(i, level0) for i in range(len(mat.planes))], rep
    (ws0, rep0), (ws1, rep1) = out[0], out[1]
    c = c0 if level0 else c1
    for i in range(len(mat.planes)):
        assert np.array_equal(ws0[i]["grad"], ws1[i]["grad"]), f"plane {i} gradient"
        t = ws0[i]["grad"].size // c
        diag0 = ws0[i]["stencil"].reshape(t, 5, c, c)[:, 0]
        diag1 = ws1[i]["stencil"].reshape(t, 5, c, c)[:, 0]
        assert np.array_equal(diag0, diag1), f"plane {i} diagonal blocks"
        assert rep0[i].lambda_ == rep1[i].lambda_
        x0, x1 = ws0[i]["x"], ws1[i]["x"]
        scale = max(np.abs(x0).max(), 1e-30)
        assert np.abs(x1 - x0).max() <= 1e-3 * scale, (i, np.abs(x1 - x0).max() / scale, rep0[i].iterations,
                                                      rep1[i].iterations)
