"""CUDA path vs the reference, kernel by kernel, through the C ABI on a B200.

Against the golden vectors the reference's own CPU arm produced (tests/golden): the per-texel and per-block work -
the stencil and gradient assembly of both latents, the quantised sweeps, the BC seed, decode and refinement - must be
BIT-EXACT; what the reference reduces in another order (the objective, the normal equations, the CG inner products)
within 1e-12 relative, the CG correction within 1e-9 relative and the decoder within 1e-5 of its largest coefficient.
Against the C restatement (oracle/nntc_oracle.c) the same bars at larger, ragged, multi-plane sizes."""
import ctypes as C

import numpy as np
import pytest

from nntc_b200 import abi, materials
from nntc_b200.session import Session

import oracle as O

pytestmark = pytest.mark.gpu


def material_of(g):
    textures, c0, c1, k = (int(x) for x in g["shape"])
    layout = [tuple(int(v) for v in p) for p in g["layout"]]
    mat = materials.Material("golden", [np.zeros((layout[0][1], layout[0][0], 3), np.uint8)] * textures, c0, c1, k)
    mat.planes = layout
    mat.chain = [g[f"src.{i}"].reshape(p[1], p[0], 3 * textures) for i, p in enumerate(layout)]
    mat.per_site = list(g["per_site"])
    return mat


def load(s, g, tag):
    for i in range(s.m.nplanes):
        s.set_planes(i, g[f"{tag}.v0.{i}"], g[f"{tag}.v1.{i}"])
        k0 = np.ascontiguousarray(g[f"{tag}.k0.{i}"])
        k1 = np.ascontiguousarray(g[f"{tag}.k1.{i}"])
        from nntc_b200 import lib
        lib().nntc_b200_level0_upload_indices(s.d, i, O.u8ptr(k0), k0.size)
        lib().nntc_b200_level1_upload_indices(s.d, i, O.u8ptr(k1), k1.size)
    if np.any(g[f"{tag}.dec_w"]) or np.any(g[f"{tag}.dec_b"]):
        s.set_decoder(g[f"{tag}.dec_w"], g[f"{tag}.dec_b"])
    s.set_grids(g[f"{tag}.lo0"], g[f"{tag}.hi0"], g[f"{tag}.lo1"] if g[f"{tag}.lo1"].any() else None,
                g[f"{tag}.hi1"] if g[f"{tag}.hi1"].any() else None)


@pytest.fixture
def session(case):
    name, g = case
    s = Session(material_of(g))
    yield s, g
    s.close()


def test_objective_vs_reference(session):
    s, g = session
    for tag in ("s0", "s2", "s7"):
        load(s, g, tag)
        r = s.objective()
        ref = g[f"{tag}.objective"]
        assert abs(r.e - ref[0]) <= 1e-12 * abs(ref[0])
        assert abs(r.centre_mse - ref[1]) <= 1e-12 * abs(ref[1])
        assert abs(r.sampled_mse - ref[2]) <= 1e-12 * abs(ref[2])


def test_decoder_vs_reference(session):
    s, g = session
    load(s, g, "s0")
    s.m.has_decoder = 0
    s.solve_decoder()
    ne = s.normal_equations()
    ref = g["s0.normal_equations"]
    assert np.allclose(ne, ref, rtol=1e-12, atol=1e-14 * np.abs(ref).max())
    w, b = s.decoder()
    scale = max(np.abs(g["s1.dec_w"]).max(), np.abs(g["s1.dec_b"]).max())
    assert np.abs(w.ravel() - g["s1.dec_w"]).max() <= 1e-5 * scale
    assert np.abs(b - g["s1.dec_b"]).max() <= 1e-5 * scale


@pytest.mark.parametrize("level0", [False, True])
def test_block_solve_vs_reference(session, level0):
    s, g = session
    tag, key = ("s3", "s3.level0") if level0 else ("s2", "s2.level1")
    load(s, g, tag)
    rep, _ = s.block(level0)
    for i in range(s.m.nplanes):
        ws = s.workspace(i, level0)
        assert np.array_equal(ws["stencil"], g[f"{key}.stencil.{i}"]), f"plane {i} stencil"
        assert np.array_equal(ws["grad"], g[f"{key}.grad.{i}"]), f"plane {i} gradient"
        assert np.array_equal(ws["precond"], g[f"{key}.precond.{i}"]) or np.allclose(
            ws["precond"], g[f"{key}.precond.{i}"], rtol=1e-6)
        ref = g[f"{key}.x.{i}"]
        assert np.allclose(ws["x"], ref, rtol=1e-9, atol=1e-12 * max(1e-300, np.abs(ref).max()))
        assert rep[i].iterations == g[f"{key}.iterations"][i]
        assert abs(rep[i].lambda_ - g[f"{key}.lambda"][i]) <= 1e-13 * abs(g[f"{key}.lambda"][i])
    after = "s4" if level0 else "s3"
    for i in range(s.m.nplanes):
        got = s.get_v0(i) if level0 else s.get_v1(i)
        want = g[f"{after}.v0.{i}" if level0 else f"{after}.v1.{i}"]
        assert np.allclose(got, want, rtol=0, atol=1e-6)


@pytest.mark.parametrize("level0", [False, True])
def test_quantised_sweeps_vs_reference(session, level0):
    s, g = session
    before, after = ("s6", "s7") if level0 else ("s5", "s6")
    load(s, g, before)
    rep, _ = s.block(level0, sweeps=4)
    for i in range(s.m.nplanes):
        got_v = s.get_v0(i) if level0 else s.get_v1(i)
        got_k = s.get_k0(i) if level0 else s.get_k1(i)
        assert np.array_equal(got_v, g[f"{after}.v0.{i}" if level0 else f"{after}.v1.{i}"])
        assert np.array_equal(got_k, g[f"{after}.k0.{i}" if level0 else f"{after}.k1.{i}"])
        key = "s6.level0" if level0 else "s5.level1"
        assert rep[i].moved == g[f"{key}.moved"][i]


def test_bc_seed_and_refine_vs_reference(session):
    s, g = session
    from nntc_b200 import lib, check
    load(s, g, "s7")
    k0 = [np.ascontiguousarray(g[f"s7.k0.{i}"]) for i in range(s.m.nplanes)]
    ms = C.c_double()
    check(lib().nntc_b200_bc_pack_prepare(s.d, C.byref(s.m), 4, 1, abi.u8_ptrs(k0), C.byref(ms)), "prepare")
    eps = [np.zeros(g[f"s7.seed.ep.{i}"].size, np.uint8) for i in range(s.m.nplanes)]
    sels = [np.zeros(g[f"s7.seed.sel.{i}"].size, np.uint8) for i in range(s.m.nplanes)]
    check(lib().nntc_b200_bc_state_save(s.d, C.byref(s.m), abi.u8_ptrs(eps), abi.u8_ptrs(sels)), "save")
    for i in range(s.m.nplanes):
        assert np.array_equal(eps[i], g[f"s7.seed.ep.{i}"]) and np.array_equal(sels[i], g[f"s7.seed.sel.{i}"])
        ws = s.workspace(i, True)
        assert np.array_equal(ws["stencil"], g[f"s7.refine_in.stencil.{i}"])
        assert np.array_equal(ws["x"], g[f"s7.refine_in.x.{i}"])
        assert np.array_equal(s.get_v0(i), g[f"s8.v0.{i}"])
    rep = (abi.BcReport * 1)()
    check(lib().nntc_b200_bc_refine(s.d, C.byref(s.m), 1, rep, C.byref(ms)), "refine")
    check(lib().nntc_b200_bc_state_save(s.d, C.byref(s.m), abi.u8_ptrs(eps), abi.u8_ptrs(sels)), "save")
    for i in range(s.m.nplanes):
        assert np.array_equal(eps[i], g[f"s8.refined.ep.{i}"]), f"plane {i} endpoints"
        assert np.array_equal(sels[i], g[f"s8.refined.sel.{i}"]), f"plane {i} selectors"
        assert np.array_equal(s.get_v0(i), g[f"s9.v0.{i}"])
        assert np.array_equal(s.get_k0(i), g[f"s9.k0.{i}"])


# ---- against the C restatement, at larger and ragged sizes ----------------------------------------------------------

SIZES = [(1, 2, 4, 61, 37), (4, 4, 4, 72, 40), (6, 4, 4, 48, 44), (2, 1, 2, 33, 21)]


def random_state(mat, seed):
    rng = np.random.default_rng(seed)
    nin = mat.c1 + mat.c0 + mat.c0 * mat.c1
    nout = 3 * len(mat.textures)
    w = (rng.standard_normal((nout, nin)) * 0.3).astype(np.float32)
    b = rng.random(nout).astype(np.float32)
    v0 = [(rng.random(p[0] * p[1] * mat.c0) * 2 - 1).astype(np.float32) for p in mat.planes]
    v1 = [(rng.random(p[2] * p[3] * mat.c1) * 2 - 1).astype(np.float32) for p in mat.planes]
    return w, b, v0, v1


# power-of-two planes: level 1 at exactly a quarter, whose interior texels take the gather's visit tables
POW2 = [(2, 4, 4, 64, 64), (1, 2, 3, 128, 64)]


@pytest.mark.parametrize("textures,c0,c1,w,h", SIZES + POW2)
def test_assembly_and_objective_vs_oracle(textures, c0, c1, w, h):
    mat = materials.small(21 + w, w, h, textures=textures, c0=c0, c1=c1)
    dw, db, v0, v1 = random_state(mat, w * h)
    with Session(mat) as s:
        for i in range(len(mat.planes)):
            s.set_planes(i, v0[i], v1[i])
        s.set_decoder(dw, db)
        s.set_grids(np.full(c0, -1.0), np.full(c0, 1.0))
        st = O.State([(p[0], p[1], p[2], p[3], mat.chain[i], v0[i], v1[i]) for i, p in enumerate(mat.planes)], c0,
                     c1, 3 * textures, 4, dw, db, np.ones(3 * textures, np.float32))
        r = s.objective()
        num = den = 0.0
        for i, p in enumerate(mat.planes):
            out = np.zeros(3)
            O.oracle().orc_objective_plane(C.byref(st.plane(i)), C.byref(st.dec), O.dptr(out))
            num += mat.per_site[i] * out[0]
            den += mat.per_site[i] * p[0] * p[1] * 5
        assert abs(r.e - num / (3 * textures * den)) <= 1e-12 * r.e
        for level0 in (False, True):
            s.block(level0)
            mono = np.zeros(15 * 16)
            O.oracle().orc_monomials(C.byref(st.dec), int(level0), O.dptr(mono))
            c = c0 if level0 else c1
            for i, p in enumerate(mat.planes):
                t = p[0] * p[1] if level0 else p[2] * p[3]
                sten, grad = np.zeros(t * 5 * c * c), np.zeros(t * c)
                # block (b) ran first and moved level 1, which block (c') then assembled against
                if level0:
                    st.v1(i)[:] = s.get_v1(i)
                O.oracle().orc_assemble(C.byref(st.plane(i)), C.byref(st.dec), int(level0), O.dptr(mono),
                                        O.dptr(sten), O.dptr(grad))
                ws = s.workspace(i, level0)
                assert np.array_equal(ws["stencil"], sten) and np.array_equal(ws["grad"], grad), (level0, i)


@pytest.mark.parametrize("textures,c0,c1,w,h", SIZES + [(1, 3, 2, 45, 29)])
def test_bc_refine_vs_oracle(textures, c0, c1, w, h):
    from nntc_b200 import lib, check
    mat = materials.small(31 + w, w, h, textures=textures, c0=c0, c1=c1)
    dw, db, v0, v1 = random_state(mat, 7 * w + h)
    lo0 = np.full(c0, -0.9, np.float32)
    hi0 = np.full(c0, 1.1, np.float32)
    with Session(mat) as s:
        for i in range(len(mat.planes)):
            s.set_planes(i, v0[i], v1[i])
        s.set_decoder(dw, db)
        s.set_grids(lo0, hi0)
        s.m.has_decoder = 1
        s.block(True, sweeps=2)   # v0 onto the grid
        k0 = [s.get_k0(i) for i in range(len(mat.planes))]
        ms = C.c_double()
        check(lib().nntc_b200_bc_pack_prepare(s.d, C.byref(s.m), 4, 1, abi.u8_ptrs(k0), C.byref(ms)), "prepare")
        ins = [s.workspace(i, True) for i in range(len(mat.planes))]
        v0s = [s.get_v0(i) for i in range(len(mat.planes))]
        eps = [np.zeros(((p[0] + 3) // 4) * ((p[1] + 3) // 4) * c0 * 2, np.uint8) for p in mat.planes]
        sels = [np.zeros(e.size * 8, np.uint8) for e in eps]
        check(lib().nntc_b200_bc_state_save(s.d, C.byref(s.m), abi.u8_ptrs(eps), abi.u8_ptrs(sels)), "save")
        rep = (abi.BcReport * 2)()
        check(lib().nntc_b200_bc_refine(s.d, C.byref(s.m), 2, rep, C.byref(ms)), "refine")
        geps = [e.copy() for e in eps]
        gsels = [q.copy() for q in sels]
        check(lib().nntc_b200_bc_state_save(s.d, C.byref(s.m), abi.u8_ptrs(geps), abi.u8_ptrs(gsels)), "save")
        for i, p in enumerate(mat.planes):
            delta = ins[i]["x"].copy()
            v = v0s[i].copy()
            kk = np.zeros(v.size, np.uint8)
            imp = C.c_longlong(0)
            for _ in range(2):
                for colour in range(4):
                    O.oracle().orc_bc_refine_colour(O.dptr(ins[i]["stencil"]), O.dptr(ins[i]["grad"]),
                                                    O.fptr(ins[i]["prev"]), O.fptr(lo0), O.fptr(hi0), p[0], p[1], c0,
                                                    colour, O.u8ptr(eps[i]), O.u8ptr(sels[i]), O.dptr(delta),
                                                    O.fptr(v), O.u8ptr(kk), C.byref(imp))
            assert np.array_equal(geps[i], eps[i]) and np.array_equal(gsels[i], sels[i]), f"plane {i}"
            assert np.array_equal(s.get_v0(i), v)


@pytest.mark.parametrize("textures,c0,c1,w,h", [(4, 4, 4, 72, 40), (1, 3, 2, 45, 29)] + POW2)
def test_assembly_shapes_agree_bit_for_bit(textures, c0, c1, w, h):
    """The per-site + per-(texel, slot) assembly and the reference-shaped per-texel gather give the same bits."""
    from nntc_b200 import lib
    mat = materials.small(41 + w, w, h, textures=textures, c0=c0, c1=c1)
    dw, db, v0, v1 = random_state(mat, 3 * w + h)
    out = []
    for shaped in (0, 1):
        with Session(mat) as s:
            assert lib().nntc_b200_set_option(s.d, 0, shaped) == 0
            for i in range(len(mat.planes)):
                s.set_planes(i, v0[i], v1[i])
            s.set_decoder(dw, db)
            s.set_grids(np.full(c0, -1.0), np.full(c0, 1.0))
            s.block(False)
            s.block(True)
            out.append([(s.workspace(i, False), s.workspace(i, True)) for i in range(len(mat.planes))])
    for (a1, a0), (b1, b0) in zip(*out):
        for key in ("stencil", "grad", "x"):
            assert np.array_equal(a1[key], b1[key]) and np.array_equal(a0[key], b0[key]), key
