"""The C restatement (oracle/nntc_oracle.c) pinned against golden vectors the reference's own CPU arm produced
(tests/golden/make_golden.py). Per-texel and per-block work must be bit-exact; sums taken in a different order than
the reference's chunked reductions (the objective, the normal equations, the CG inner products) within 1e-12 / 1e-9.
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O


def state(g, tag):
    textures, c0, c1, k = (int(x) for x in g["shape"])
    planes = []
    for i, (w0, h0, w1, h1) in enumerate(g["layout"]):
        planes.append((int(w0), int(h0), int(w1), int(h1), g[f"src.{i}"], g[f"{tag}.v0.{i}"], g[f"{tag}.v1.{i}"]))
    return O.State(planes, c0, c1, 3 * textures, k, g[f"{tag}.dec_w"], g[f"{tag}.dec_b"],
                   np.ones(3 * textures, np.float32))


def normalised_e(g, st, tag):
    per_site = g["per_site"]
    num = den = 0.0
    for i in range(len(g["layout"])):
        out = np.zeros(3)
        O.oracle().orc_objective_plane(C.byref(st.plane(i)), C.byref(st.dec), O.dptr(out))
        w0, h0 = g["layout"][i][:2]
        sites = float(w0) * float(h0) * (1 + st.k)
        num += per_site[i] * out[0]
        den += per_site[i] * sites
    return num / (st.nout * den)


@pytest.mark.parametrize("tag", ["s0", "s2", "s7"])
def test_objective(case, tag):
    name, g = case
    st = state(g, tag)
    e = normalised_e(g, st, tag)
    assert abs(e - g[f"{tag}.objective"][0]) <= 1e-12 * abs(g[f"{tag}.objective"][0])


def test_normal_equations_and_decoder(case):
    name, g = case
    st = state(g, "s0")
    ne = g["s0.normal_equations"]
    acc = np.zeros_like(ne)
    for i in range(len(g["layout"])):
        e = np.zeros_like(ne)
        O.oracle().orc_normal_equations_plane(C.byref(st.plane(i)), C.byref(st.dec), O.dptr(e))
        acc += g["per_site"][i] * e
    assert np.allclose(acc, ne, rtol=1e-12, atol=1e-15 * np.abs(ne).max())
    # The ladder on the reference's own sums gives the reference's decoder bit for bit.
    nin, nout = st.nin, st.nout
    w = np.zeros(nout * nin, np.float32)
    b = np.zeros(nout, np.float32)
    sites = sum(float(p[0]) * float(p[1]) * (1 + st.k) * g["per_site"][i] for i, p in enumerate(g["layout"]))
    O.oracle().orc_decoder_solve(O.dptr(ne), nin, nout, O.fptr(st.cw), 1.0 / (nout * sites), 1, 0, O.fptr(w),
                                 O.fptr(b))
    assert np.array_equal(w, g["s1.dec_w"]) and np.array_equal(b, g["s1.dec_b"])


@pytest.mark.parametrize("level0", [False, True])
def test_assembly_bit_exact(case, level0):
    name, g = case
    tag, key = ("s3", "s3.level0") if level0 else ("s2", "s2.level1")
    st = state(g, tag)
    c = st.c0 if level0 else st.c1
    mono = np.zeros(15 * 16)
    O.oracle().orc_monomials(C.byref(st.dec), 1 if level0 else 0, O.dptr(mono))
    for i, (w0, h0, w1, h1) in enumerate(g["layout"]):
        t = (w0 * h0) if level0 else (w1 * h1)
        sten = np.zeros(t * 5 * c * c)
        grad = np.zeros(t * c)
        O.oracle().orc_assemble(C.byref(st.plane(i)), C.byref(st.dec), 1 if level0 else 0, O.dptr(mono),
                                O.dptr(sten), O.dptr(grad))
        assert np.array_equal(sten, g[f"{key}.stencil.{i}"]), f"plane {i} stencil"
        assert np.array_equal(grad, g[f"{key}.grad.{i}"]), f"plane {i} gradient"


@pytest.mark.parametrize("level0", [False, True])
def test_pcg(case, level0):
    name, g = case
    key = "s3.level0" if level0 else "s2.level1"
    textures, c0, c1, k = (int(x) for x in g["shape"])
    c = c0 if level0 else c1
    for i, (w0, h0, w1, h1) in enumerate(g["layout"]):
        w, h = (w0, h0) if level0 else (w1, h1)
        lam = g[f"{key}.lambda"][i]
        diag = np.zeros(4)
        O.oracle().orc_diag(O.dptr(g[f"{key}.stencil.{i}"]), w * h, c, 1e-4, O.dptr(diag))
        assert abs(diag[3] - lam) <= 1e-13 * abs(lam)
        x = np.zeros(w * h * c)
        res = np.zeros(1)
        it = O.oracle().orc_pcg(O.dptr(g[f"{key}.stencil.{i}"]), O.dptr(g[f"{key}.grad.{i}"]), int(w), int(h), c,
                                float(lam), O.dptr(x), O.dptr(res))
        ref = g[f"{key}.x.{i}"]
        assert it == g[f"{key}.iterations"][i]
        assert np.allclose(x, ref, rtol=1e-9, atol=1e-12 * max(1e-300, np.abs(ref).max()))


@pytest.mark.parametrize("level0", [False, True])
def test_quantised_sweeps_bit_exact(case, level0):
    name, g = case
    key, before, after = ("s6.level0", "s6", "s7") if level0 else ("s5.level1", "s5", "s6")
    textures, c0, c1, k = (int(x) for x in g["shape"])
    c = c0 if level0 else c1
    lo = g[f"{before}.lo0"] if level0 else g[f"{before}.lo1"]
    hi = g[f"{before}.hi0"] if level0 else g[f"{before}.hi1"]
    for i, (w0, h0, w1, h1) in enumerate(g["layout"]):
        w, h = (w0, h0) if level0 else (w1, h1)
        v = g[f"{before}.v0.{i}" if level0 else f"{before}.v1.{i}"].copy()
        kk = g[f"{before}.k0.{i}" if level0 else f"{before}.k1.{i}"].copy()
        prev = v.copy()
        x = np.zeros(w * h * c)
        moved = O.oracle().orc_quant_sweeps(O.dptr(g[f"{key}.stencil.{i}"]), O.dptr(g[f"{key}.grad.{i}"]),
                                            O.fptr(prev), int(w), int(h), c, float(g[f"{key}.lambda"][i]), O.fptr(lo),
                                            O.fptr(hi), 8, 4, O.dptr(x), O.fptr(v), O.u8ptr(kk))
        assert moved == g[f"{key}.moved"][i]
        assert np.array_equal(v, g[f"{after}.v0.{i}" if level0 else f"{after}.v1.{i}"])
        assert np.array_equal(kk, g[f"{after}.k0.{i}" if level0 else f"{after}.k1.{i}"])


def test_bc_seed_and_refine_bit_exact(case):
    name, g = case
    textures, c0, c1, k = (int(x) for x in g["shape"])
    bits = (C.c_int * 4)(8, 8, 8, 8)
    lo0, hi0 = g["s8.lo0"], g["s8.hi0"]
    for i, (w0, h0, w1, h1) in enumerate(g["layout"]):
        w0, h0 = int(w0), int(h0)
        k0 = g[f"s7.k0.{i}"]
        blocks = ((w0 + 3) // 4) * ((h0 + 3) // 4)
        ep = np.zeros(blocks * c0 * 2, np.uint8)
        sel = np.zeros(blocks * c0 * 16, np.uint8)
        O.oracle().orc_bc_seed(O.u8ptr(k0), w0, h0, c0, bits, O.u8ptr(ep), O.u8ptr(sel))
        assert np.array_equal(ep, g[f"s7.seed.ep.{i}"]) and np.array_equal(sel, g[f"s7.seed.sel.{i}"])
        # the decode of the seed, then one refinement pass of four colours from the reference's own stencil
        prev = g[f"s7.refine_in.prev.{i}"]
        v0 = np.zeros(w0 * h0 * c0, np.float32)
        kk = np.zeros(w0 * h0 * c0, np.uint8)
        delta = np.zeros(w0 * h0 * c0)
        O.oracle().orc_bc_decode(O.u8ptr(ep), O.u8ptr(sel), O.fptr(lo0), O.fptr(hi0), w0, h0, c0, O.fptr(prev),
                                 O.fptr(v0), O.u8ptr(kk), O.dptr(delta))
        assert np.array_equal(v0, g[f"s8.v0.{i}"]) and np.array_equal(kk, g[f"s8.k0.{i}"])
        assert np.array_equal(delta, g[f"s7.refine_in.x.{i}"])
        improved = C.c_longlong(0)
        for colour in range(4):
            O.oracle().orc_bc_refine_colour(O.dptr(g[f"s7.refine_in.stencil.{i}"]), O.dptr(g[f"s7.refine_in.grad.{i}"]),
                                            O.fptr(prev), O.fptr(lo0), O.fptr(hi0), w0, h0, c0, colour, O.u8ptr(ep),
                                            O.u8ptr(sel), O.dptr(delta), O.fptr(v0), O.u8ptr(kk), C.byref(improved))
        assert np.array_equal(ep, g[f"s8.refined.ep.{i}"]), f"plane {i} endpoints"
        assert np.array_equal(sel, g[f"s8.refined.sel.{i}"]), f"plane {i} selectors"
        assert np.array_equal(v0, g[f"s9.v0.{i}"]) and np.array_equal(delta, g[f"s8.refined.x.{i}"])


def test_grid_round_trip():
    L = O.oracle()
    for bits in (4, 5, 6, 7, 8):
        for k in range((1 << bits)):
            v = L.orc_grid_value(-0.7, 1.3, bits, k)
            assert L.orc_grid_index(-0.7, 1.3, bits, v) == k
