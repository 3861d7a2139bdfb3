"""Block (c) of the `--l0 palette` mode, the CUDA path against the reference's own CPU arm on the same state.

The per-texel palette search (src/solve_level0.cu:75-327) moves level 0 only to palette values, strictly downhill and
colour by colour, so its result is bytes: level 0's values and indices, and the moved counts, must be identical."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from nntc_b200 import abi, check, lib, materials
from nntc_b200.session import Session

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("textures,c0,c1,w,h,bits", [(1, 2, 4, 61, 37, 3), (2, 1, 2, 40, 24, 4), (2, 3, 2, 33, 21, 2)])
def test_palette_search_vs_reference(textures, c0, c1, w, h, bits):
    try:
        O.RefSession.lib()
    except FileNotFoundError:
        pytest.skip("the reference CPU arm is not built")
    mat = materials.small(60 + w, w, h, textures=textures, c0=c0, c1=c1)
    m = abi.make_model(mat, l0_bc8=False)
    levels = (1 << bits) - 1
    for c in range(c0):
        m.bits0[c] = bits
        m.palette0_len[c] = levels + 1
        for k in range(levels + 1):
            m.palette0[c][k] = -1.0 + 2.0 * (k / levels)
    rng = np.random.default_rng(w * h)
    nin, nout = m.nin, m.nout
    dw = (rng.standard_normal((nout, nin)) * 0.3).astype(np.float32)
    db = rng.random(nout).astype(np.float32)
    m.has_decoder = 1
    for i, x in enumerate(dw.ravel()):
        m.dec_w[i] = float(x)
    for i, x in enumerate(db):
        m.dec_b[i] = float(x)
    m.has_lo1 = 1
    for c in range(c1):
        m.lo1[c], m.hi1[c] = -1.0, 1.0
    pal = np.array([[m.palette0[c][k] for k in range(levels + 1)] for c in range(c0)], np.float32)
    k0 = [rng.integers(0, levels + 1, p[0] * p[1] * c0).astype(np.uint8) for p in mat.planes]
    v0 = [pal[np.arange(kk.size) % c0, kk] for kk in k0]
    v1 = [(rng.random(p[2] * p[3] * c1) * 2 - 1).astype(np.float32) for p in mat.planes]

    ref = O.RefSession(mat, m, threads=1)
    try:
        for i in range(len(mat.planes)):
            ref.set_planes(i, v0[i], v1[i])
            ref.set_indices(i, k0=k0[i])
        ref.sync_in()
        rrep = (abi.Level0Report * len(mat.planes))()
        ref.L.ref_solve_level0_palette(ref.h, 4, 2, C.cast(rrep, C.c_void_p))
        want = [ref.planes(i) for i in range(len(mat.planes))]
    finally:
        ref.close()

    with Session(mat, model=m) as s:
        check(lib().nntc_b200_upload_decoder(s.d, C.byref(s.m)), "decoder")
        check(lib().nntc_b200_upload_grids(s.d, C.byref(s.m)), "grids")
        for i in range(len(mat.planes)):
            s.set_planes(i, v0[i], v1[i])
            kk = np.ascontiguousarray(k0[i])
            check(lib().nntc_b200_level0_upload_indices(s.d, i, O.u8ptr(kk), kk.size), "indices")
        rep = (abi.Level0Report * len(mat.planes))()
        ms = C.c_double()
        check(lib().nntc_b200_solve_level0_all(s.d, C.byref(s.m), 4, 2, rep, C.byref(ms)), "palette search")
        for i in range(len(mat.planes)):
            assert np.array_equal(s.get_v0(i), want[i][0]), f"plane {i} values"
            assert np.array_equal(s.get_k0(i), want[i][2]), f"plane {i} indices"
            assert rep[i].moved_total == rrep[i].moved_total, (i, rep[i].moved_total, rrep[i].moved_total)
