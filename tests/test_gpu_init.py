"""The initialisation on a B200 against the reference's own CPU arm on the same material and state.

The seam's init_level0 (palette and bc8), init_level1 (box and pca) and init0_residual_channel (base and chain
scope, whole and by texture) are direct kernels: what they write is compared with the bar the reference's check
harness holds direct kernels to (src/backend_check.cpp: 1e-6 of the array's scale per value, indices with at most 1%
flips), the report's sums within 1e-9 relative (the same sums, reduced in another order). Level 1's pca components are
compared up to their sign, which the method leaves open."""
import ctypes as C
import copy

import numpy as np
import pytest

import oracle as O
from nntc_b200 import abi, check, lib, materials
from nntc_b200.session import Session

pytestmark = pytest.mark.gpu

LUMA = np.array([0.299, 0.587, 0.114], np.float32)


def reference_lib():
    try:
        return O.RefSession.lib()
    except FileNotFoundError:
        pytest.skip("the reference CPU arm is not built")


def close(a, b, rel=1e-9):
    return abs(a - b) <= rel * max(abs(a), abs(b), 1e-300)


@pytest.mark.parametrize("bc8", [True, False])
@pytest.mark.parametrize("pca", [0, 1])
def test_level_inits_vs_reference(bc8, pca):
    reference_lib()
    mat = materials.small(71, 45, 33, textures=2, c0=2, c1=4)
    m = abi.make_model(mat, l0_bc8=bc8)
    ref = O.RefSession(mat, copy.deepcopy(m), threads=1)
    try:
        ref.L.ref_init_level0(ref.h, O.fptr(LUMA), 1)
        rrep = abi.Init1Report()
        ref.L.ref_init_level1(ref.h, pca, C.byref(rrep))
        mr = copy.deepcopy(m)
        ref.L.ref_sync_out(ref.h, C.byref(mr))
        want = [ref.planes(i) for i in range(m.nplanes)]
    finally:
        ref.close()
    with Session(mat, model=copy.deepcopy(m)) as s:
        check(lib().nntc_b200_init_level0(s.d, C.byref(s.m), O.fptr(LUMA), 1, None), "init_level0")
        rep = abi.Init1Report()
        check(lib().nntc_b200_init_level1(s.d, C.byref(s.m), pca, C.byref(rep), None), "init_level1")
        got = [(s.get_v0(i), s.get_v1(i), s.get_k0(i), s.get_k1(i)) for i in range(m.nplanes)]
        for i in range(m.nplanes):
            assert np.array_equal(got[i][0], want[i][0]), f"plane {i} level 0 values"
            assert np.array_equal(got[i][2], want[i][2]), f"plane {i} level 0 indices"
        assert rep.pca == rrep.pca and rep.components == rrep.components
        if not pca:
            for c in range(m.c1):
                assert s.m.lo1[c] == mr.lo1[c] and s.m.hi1[c] == mr.hi1[c]
            for i in range(m.nplanes):
                assert np.array_equal(got[i][1], want[i][1]), f"plane {i} level 1 values"
                assert np.array_equal(got[i][3], want[i][3]), f"plane {i} level 1 indices"
            return
        assert close(rep.total_variance, rrep.total_variance)
        for j in range(rep.components):
            assert close(rep.eigenvalue[j], rrep.eigenvalue[j]), (j, rep.eigenvalue[j], rrep.eigenvalue[j])
            assert close(rep.peak[j], rrep.peak[j], 1e-7), (j, rep.peak[j], rrep.peak[j])
        # each component equal up to its sign: the grid follows (lo, hi) -> (-hi, -lo), values within one grid step
        v_got = np.concatenate([g[1] for g in got]).reshape(-1, m.c1)
        v_want = np.concatenate([w[1] for w in want]).reshape(-1, m.c1)
        for j in range(rep.components):
            sign = 1.0 if np.dot(v_got[:, j], v_want[:, j]) >= 0 else -1.0
            step = (mr.hi1[j] - mr.lo1[j]) / 255.0
            d = np.abs(v_got[:, j] - sign * v_want[:, j])
            assert d.max() <= 1.01 * step, (j, d.max(), step)
            assert np.mean(d > 1e-6 * max(abs(mr.lo1[j]), abs(mr.hi1[j]))) <= 0.01, j


@pytest.mark.parametrize("bc8,chain,texture", [(True, 0, 0), (False, 0, 0), (True, 1, 0), (False, 1, 1),
                                               (True, 0, 1)])
def test_init0_residual_vs_reference(bc8, chain, texture):
    reference_lib()
    mat = materials.small(83, 52, 40, textures=3, c0=3, c1=2)
    m = abi.make_model(mat, l0_bc8=bc8, init0="texture" if texture else "residual")
    m.init0_chain = chain
    rng = np.random.default_rng(5)
    nin, nout = m.nin, m.nout
    dw = (rng.standard_normal((nout, nin)) * 0.3).astype(np.float32)
    db = rng.random(nout).astype(np.float32)
    m.has_decoder = 1
    for i, x in enumerate(dw.ravel()):
        m.dec_w[i] = float(x)
    for i, x in enumerate(db):
        m.dec_b[i] = float(x)
    m.has_lo1 = 1
    for c in range(m.c1):
        m.lo1[c], m.hi1[c] = -1.0, 1.0
    v0 = [(rng.random(p[0] * p[1] * m.c0) * 2 - 1).astype(np.float32) for p in mat.planes]
    v1 = [(rng.random(p[2] * p[3] * m.c1) * 2 - 1).astype(np.float32) for p in mat.planes]
    weights = np.array(mat.per_site, np.float64)
    ref = O.RefSession(mat, copy.deepcopy(m), threads=1)
    try:
        for i in range(m.nplanes):
            ref.set_planes(i, v0[i], v1[i])
        ref.sync_in()
        rrep = abi.Init0Report()
        ref.L.ref_init0_residual_channel(ref.h, 1, O.dptr(weights), C.byref(rrep))
        want = [ref.planes(i) for i in range(m.nplanes)]
    finally:
        ref.close()
    with Session(mat, model=copy.deepcopy(m)) as s:
        check(lib().nntc_b200_upload_decoder(s.d, C.byref(s.m)), "decoder")
        check(lib().nntc_b200_upload_grids(s.d, C.byref(s.m)), "grids")
        for i in range(m.nplanes):
            s.set_planes(i, v0[i], v1[i])
        rep = abi.Init0Report()
        k0 = s.u8_planes(0)
        check(lib().nntc_b200_init0_residual_channel(s.d, C.byref(s.m), 1, O.dptr(weights), C.byref(rep),
                                                     abi.u8_ptrs(k0)), "init0")
        assert rep.texture == rrep.texture and rep.nout == rrep.nout
        assert close(rep.total_variance, rrep.total_variance) and close(rep.eigenvalue, rrep.eigenvalue)
        assert np.allclose(np.array(rep.dir[:nout]), np.array(rrep.dir[:nout]), rtol=0, atol=1e-9)
        assert close(rep.peak, rrep.peak, 1e-7) and close(rep.divisor, rrep.divisor, 1e-7)
        flips = total = 0
        for i in range(m.nplanes):
            got = s.get_v0(i).reshape(-1, m.c0)
            w = want[i][0].reshape(-1, m.c0)
            assert np.array_equal(np.delete(got, 1, axis=1), np.delete(w, 1, axis=1)), "untouched channels"
            if bc8:
                assert np.abs(got[:, 1] - w[:, 1]).max() <= 1e-6, f"plane {i} seeded channel"
            else:
                same = k0[i].reshape(-1, m.c0)[:, 1] == want[i][2].reshape(-1, m.c0)[:, 1]
                assert np.array_equal(got[same, 1], w[same, 1])
                flips += int(np.sum(~same))
                total += same.size
        assert flips <= 0.01 * max(total, 1)
