"""An encode on a B200 written to disk as the reference's asset, and read back.

The encode's shipped state (nntc_b200_encode_on_device with its output buffers: both levels' indices and the refined
BC endpoints and selectors) goes through nntc_b200_write_asset; reading the files back (nntc_b200/asset.py) must give
the same indices, endpoints and selectors, and the descriptor the same decoder and grids, bit for bit. The writer
re-checks every level-1 index against its published grid, so an index the encode left off its grid fails here too."""
import ctypes as C

import numpy as np
import pytest

from nntc_b200 import abi, asset, lib, materials
from nntc_b200.session import Session

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("textures,c0,c1,w,h", [(2, 2, 4, 32, 24), (1, 3, 3, 40, 28)])
def test_encode_to_asset_round_trip(tmp_path, textures, c0, c1, w, h):
    mat = materials.small(31 + w, w, h, textures=textures, c0=c0, c1=c1)
    with Session(mat) as s:
        args = abi.EncodeArgs()
        lib().nntc_b200_encode_defaults(C.byref(args))
        args.rounds = 4
        _, out = s.encode(args, outputs=True)
        prefix = str(tmp_path / "mat")
        s.write_asset(prefix, out)
        m = s.m
        a = asset.read_asset(prefix + "_nntc.json")
        m2, k1, k0, ep, sel = asset.model_from_asset(a)
        for i in range(m.nplanes):
            assert np.array_equal(k1[i], out["k1"][i]), i
            assert np.array_equal(ep[i], out["ep"][i]), i
            assert np.array_equal(sel[i], out["sel"][i]), i
        n = m.nout * m.nin
        assert np.array_equal(np.array(m2.dec_w[:n], np.float32), np.array(m.dec_w[:n], np.float32))
        assert np.array_equal(np.array(m2.dec_b[:m.nout], np.float32), np.array(m.dec_b[:m.nout], np.float32))
        for c in range(m.c1):
            assert (m2.lo1[c], m2.hi1[c]) == (m.lo1[c], m.hi1[c])
        for c in range(m.c0):
            assert (m2.lo0[c], m2.hi0[c]) == (m.lo0[c], m.hi0[c])
