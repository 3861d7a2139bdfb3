"""The C-ABI library on the CPU: it loads, exports every entry point include/nntc_b200.h declares, and its structs
have the sizes the Python mirror assumes. No compute call is made (there is no GPU here)."""
import ctypes as C
import os
import re

import pytest

import nntc_b200
from nntc_b200 import abi

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "nntc_b200.h")


def declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(nntc_b200_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = nntc_b200.lib()
    names = declared()
    assert len(names) >= 50
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_every_declared_symbol_has_a_python_prototype():
    assert set(declared()) <= set(nntc_b200.PROTOTYPES)


def test_struct_sizes_match_the_mirror():
    out = (C.c_size_t * 16)()
    n = nntc_b200.lib().nntc_b200_abi_sizes(out, 16)
    mirror = [abi.Model, abi.DeviceInfo, abi.PlaneReport, abi.Level0Report, abi.Objective, abi.Init1Report,
              abi.Init0Report, abi.BcReport, abi.EncodeArgs, abi.EncodeResult]
    assert n == len(mirror)
    for i, t in enumerate(mirror):
        assert out[i] == C.sizeof(t), t.__name__


def test_encode_defaults_are_the_references():
    a = abi.EncodeArgs()
    nntc_b200.lib().nntc_b200_encode_defaults(C.byref(a))
    # src/options.h:82-163
    assert (a.k, a.rounds, a.q1_start, a.q1_sweeps, a.range_pct, a.bc_refine, a.bc_refine_after, a.bc_outer) == (
        4, 20, 3, 4, 1, 4, 0, 2)
    assert a.tol == pytest.approx(1e-4) and a.ridge == pytest.approx(1e-4)


def test_stencil_monomials_is_pure_host():
    L = nntc_b200.lib()
    assert [L.nntc_b200_stencil_monomials(c) for c in (1, 2, 3, 4)] == [3, 6, 10, 15]


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(nntc_b200, "_lib", None)
    monkeypatch.setattr(nntc_b200, "LIBRARY", str(tmp_path / "absent.so"))
    with pytest.raises(nntc_b200.NntcError):
        nntc_b200.lib()


@pytest.mark.parametrize("field,value,what", [("c0", 5, "channel"), ("textures", 7, "textures"), ("nin", 3, "nin"),
                                               ("nplanes", 0, "planes"), ("bits1", 9, "bits1")])
def test_device_create_rejects_a_bad_model_before_any_device_work(field, value, what):
    """Validation runs on the host first: a model the encoder cannot take is refused with a message, no GPU needed."""
    import ctypes as C

    import numpy as np

    from nntc_b200 import abi, lib, materials

    mat = materials.small(1, 24, 16, textures=1)
    m = abi.make_model(mat)
    setattr(m, field, value)
    chain = [np.ascontiguousarray(c, np.float32) for c in mat.chain]
    h = C.c_void_p()
    assert lib().nntc_b200_device_create(C.byref(m), abi.float_ptrs(chain), C.byref(h)) == 1
    assert not h.value
    assert lib().nntc_b200_last_error().decode()


def test_device_create_from_base_rejects_a_chain_that_is_not_the_box_halving():
    import ctypes as C

    import numpy as np

    from nntc_b200 import abi, lib, materials

    mat = materials.small(2, 32, 32, textures=1)
    m = abi.make_model(mat)
    m.w0[1] += 1
    base = np.ascontiguousarray(mat.chain[0], np.float32).ravel()
    h = C.c_void_p()
    assert lib().nntc_b200_device_create_from_base(C.byref(m), base.ctypes.data_as(C.POINTER(C.c_float)),
                                                   C.byref(h)) == 1
    assert "halving" in lib().nntc_b200_last_error().decode()
