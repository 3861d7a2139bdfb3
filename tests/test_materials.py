"""The synthetic inputs and the layout: seeded, deterministic, and laid out exactly as the reference lays out a chain
(checked against the reference's own build_plane_sizes / build_mip_weights / image_box when oracle/_ref is built)."""
import ctypes as C
import os
import zlib

import numpy as np
import pytest

from nntc_b200 import materials as M

import oracle as O


def test_generator_is_seeded():
    a = M.small(5, 40, 24, textures=4)
    b = M.small(5, 40, 24, textures=4)
    for x, y in zip(a.textures, b.textures):
        assert np.array_equal(x, y)
    c = M.small(6, 40, 24, textures=4)
    assert not np.array_equal(a.textures[0], c.textures[0])


@pytest.mark.parametrize("index,shape,textures,c0", [(0, (256, 256), 1, 2), (1, (512, 512), 4, 2)])
def test_configs(index, shape, textures, c0):
    m = M.config(index)
    assert m.textures[0].shape[:2] == shape and len(m.textures) == textures and m.c0 == c0 and m.c1 == 4
    assert len(m.chain) == len(m.planes)
    assert abs(sum(p * s * (1 + m.k) for p, s in zip(m.per_site, [q[0] * q[1] for q in m.planes])) - 1.0) < 1e-12


@pytest.mark.parametrize("w,h", [(256, 256), (2048, 1024), (20, 12), (64, 4), (1, 1), (4096, 4096)])
def test_layout_against_reference(w, h):
    if not os.path.exists(O.REF_SO):
        pytest.skip("reference CPU arm not built")
    L = O.RefSession.lib()
    L.ref_layout.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_char_p, C.c_double,
                             C.POINTER(C.c_int), C.POINTER(C.c_double)]
    sizes = (C.c_int * 64)()
    ps = (C.c_double * 16)()
    n = L.ref_layout(w, h, 8, 1, 4, b"pixels", 0.5, sizes, ps)
    mine = M.plane_sizes(w, h, 8, True)
    weights = M.mip_weights(mine)
    assert n == len(mine)
    for i, p in enumerate(mine):
        assert tuple(sizes[4 * i: 4 * i + 4]) == p
        assert ps[i] == weights[i]


@pytest.mark.parametrize("w,h,textures,mip_min", [(52, 36, 2, 8), (33, 21, 4, 1), (40, 9, 6, 1), (61, 37, 2, 1)])
def test_chain_against_reference(w, h, textures, mip_min):
    if not os.path.exists(O.REF_SO):
        pytest.skip("reference CPU arm not built")
    L = O.RefSession.lib()
    L.ref_source_chain.argtypes = [C.POINTER(C.c_float), C.c_int, C.c_int, C.c_int, C.c_int,
                                   C.POINTER(C.POINTER(C.c_float))]
    mat = M.small(9, w, h, textures=textures, mip_min=mip_min)
    nc = 3 * textures
    outs = [np.zeros((p[1], p[0], nc), np.float32) for p in mat.planes[1:]]
    arr = (C.POINTER(C.c_float) * len(outs))(*[O.fptr(o) for o in outs])
    base = np.ascontiguousarray(mat.chain[0])
    L.ref_source_chain(O.fptr(base), base.shape[1], base.shape[0], nc, len(outs), arr)
    for a, b in zip(outs, mat.chain[1:]):
        assert np.array_equal(a, b)


def test_png_round_trip(tmp_path):
    img = M.small(2, 17, 9).textures[0]
    p = tmp_path / "x.png"
    M.write_png(str(p), img)
    data = p.read_bytes()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    idat = data[data.index(b"IDAT") + 4:data.index(b"IEND") - 8]
    raw = zlib.decompress(idat)
    rows = np.frombuffer(raw, np.uint8).reshape(9, 1 + 17 * 3)
    assert np.array_equal(rows[:, 1:].reshape(9, 17, 3), img)
