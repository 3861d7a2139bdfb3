"""The source chain built on the device from the base plane, against the host-built chain (which
tests/test_materials.py pins to the reference's own image_box loop): bit for bit, at even, odd and one-texel-wide
levels, and through a whole encode."""
import numpy as np
import pytest

from nntc_b200 import NntcError, materials
from nntc_b200.session import Session

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("w,h,textures", [(64, 64, 1), (61, 37, 2), (33, 21, 4), (40, 9, 6)])
def test_chain_from_base_is_bit_exact(w, h, textures):
    mat = materials.small(70 + w, w, h, textures=textures, mip_min=1)
    with Session(mat, from_base=True) as s:
        for i, ch in enumerate(mat.chain):
            got = s.get_source(i)
            want = np.ascontiguousarray(ch, np.float32).ravel()
            assert got.view(np.uint32).tolist() == want.view(np.uint32).tolist(), f"plane {i} {mat.planes[i]}"


def test_encode_from_base_matches_full_upload():
    mat = materials.small(5, 72, 40, textures=2, c0=4, c1=4)
    with Session(mat) as a, Session(mat, from_base=True) as b:
        ra, rb = a.encode(), b.encode()
        assert ra.e_ship == rb.e_ship
        assert list(ra.psnr[:2]) == list(rb.psnr[:2])


def test_from_base_rejects_a_chain_that_is_not_the_box_halving():
    mat = materials.small(6, 32, 32, textures=1)
    from nntc_b200 import abi
    m = abi.make_model(mat)
    m.w0[1] = m.w0[1] + 1   # not the floor halving of plane 0
    with pytest.raises(NntcError):
        Session(mat, model=m, from_base=True)
