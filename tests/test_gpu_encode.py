"""Whole encodes on a B200.

- The drop-in: the reference's own host (main.cpp) linked against libnntc_b200.so in place of its CUDA arm, run under
  its per-kernel harness (--backend check), which mirrors every seam call into the reference's CPU arm and compares.
  Every call must agree; the one accepted difference is device_memory, a byte count of a layout this library chose
  differently on purpose (structure-of-arrays stencil, batched reductions).
- The encoder's own round loop (nntc_b200_encode_on_device) against the reference CPU encoder on the same input:
  per-texture PSNR within 0.05 dB.
- Full-size properties: every stored index re-quantises to itself, the decoded BC blocks are the plane, E after the
  loop is below E at the start."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from nntc_b200 import abi, check, lib, materials
from nntc_b200.session import Session

import oracle as O

pytestmark = pytest.mark.gpu


def run(cmd, timeout=600):
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    return p.returncode, p.stdout + p.stderr


def harness_table(text):
    rows = {}
    for line in text.splitlines():
        m = re.match(r"\s+(\S[\w ]*?)\s+(\d+)\s+(\d+)\s+(\d+)\s+(\d+)\s+(\d+)\s+(\S+)\s*$", line)
        if m:
            rows[m.group(1).strip()] = tuple(int(m.group(i)) for i in range(2, 7))
    return rows


@pytest.mark.parametrize("spec", [
    dict(seed=3, w=64, h=64, textures=1, args=[]),
    dict(seed=5, w=64, h=48, textures=4, args=["--c0", "4", "--c1", "4"]),
    dict(seed=7, w=20, h=12, textures=1, args=[]),
    dict(seed=9, w=40, h=36, textures=2, args=["--c0", "3", "--c1", "2"]),
])
def test_reference_harness_through_the_dropin(tmp_path, spec):
    if not os.path.exists(O.DROPIN_ENCODER):
        pytest.skip("the drop-in encoder is not built (oracle/Makefile dropin)")
    mat = materials.small(spec["seed"], spec["w"], spec["h"], textures=spec["textures"])
    pngs = materials.save_material(mat, str(tmp_path / "in"))
    rc, out = run([O.DROPIN_ENCODER, *pngs, "-o", str(tmp_path / "out") + "/", "--backend", "check", *spec["args"]])
    rows = harness_table(out)
    assert "objective_eval" in rows and "bc refinement colour passes" in rows, out[-3000:]
    for name, (calls, ok, flips, mismatches, missing) in rows.items():
        assert flips == 0, (name, out[-2000:])
        if name != "device_memory":
            assert mismatches == 0 and ok == calls, (name, out[-2000:])


def reference_psnr(pngs, tmp_path, extra=()):
    rc, out = run([O.REF_ENCODER, *pngs, "-o", str(tmp_path / "ref") + "/", "--backend", "cpu", *extra], 900)
    assert rc == 0, out[-2000:]
    return [float(x) for x in re.findall(r"psnr\s+texture \d+\s+([\d.]+) dB", out)]


@pytest.mark.parametrize("index", [0, 1])
def test_encode_psnr_vs_reference(tmp_path, index):
    if not os.path.exists(O.REF_ENCODER):
        pytest.skip("the reference CPU encoder is not built")
    mat = materials.config(index)
    pngs = materials.save_material(mat, str(tmp_path / "in"))
    with Session(mat) as s:
        r = s.encode()
    ref = reference_psnr(pngs, tmp_path)
    ours = list(r.psnr[: len(mat.textures)])
    assert len(ref) == len(ours)
    for a, b in zip(ours, ref):
        assert abs(a - b) <= 0.05, (ours, ref)
    assert r.e_ship < r.e_init


def test_full_size_properties():
    mat = materials.config(2)   # 4 x 1024 x 1024, c0 2 c1 4
    with Session(mat) as s:
        args = abi.EncodeArgs()
        lib().nntc_b200_encode_defaults(C.byref(args))
        r = abi.EncodeResult()
        np_ = s.m.nplanes
        k0 = s.u8_planes(0)
        k1 = s.u8_planes(1)
        eps = [np.zeros(((p[0] + 3) // 4) * ((p[1] + 3) // 4) * mat.c0 * 2, np.uint8) for p in mat.planes]
        sels = [np.zeros(e.size * 8, np.uint8) for e in eps]
        check(lib().nntc_b200_encode_on_device(s.d, C.byref(s.m), C.byref(args), s.per_site, C.byref(r),
                                               abi.u8_ptrs(k0), abi.u8_ptrs(k1), abi.u8_ptrs(eps), abi.u8_ptrs(sels)),
              "encode")
        assert r.e_ship < r.e_after_rounds * 1.5 and r.e_ship < r.e_init
        for i in range(np_):
            # level 1 is on its grid: every value is exactly the grid value of its index
            v1 = s.get_v1(i).reshape(-1, mat.c1)
            kk = k1[i].reshape(-1, mat.c1)
            for c in range(mat.c1):
                want = np.array([O.oracle().orc_grid_value(s.m.lo1[c], s.m.hi1[c], 8, int(q)) for q in range(256)],
                                np.float32)
                assert np.array_equal(v1[:, c], want[kk[:, c]])
            # level 0 is the decode of the BC blocks (src/refine_bc.cu:155-174)
            w0, h0 = mat.planes[i][0], mat.planes[i][1]
            v = np.zeros(w0 * h0 * mat.c0, np.float32)
            kb = np.zeros(v.size, np.uint8)
            dl = np.zeros(v.size)
            prev = np.zeros(v.size, np.float32)
            lo0 = np.array(s.m.lo0[: mat.c0], np.float32)
            hi0 = np.array(s.m.hi0[: mat.c0], np.float32)
            O.oracle().orc_bc_decode(O.u8ptr(eps[i]), O.u8ptr(sels[i]), O.fptr(lo0), O.fptr(hi0), w0, h0, mat.c0,
                                     O.fptr(prev), O.fptr(v), O.u8ptr(kb), O.dptr(dl))
            assert np.array_equal(v, s.get_v0(i))
            assert np.array_equal(kb, k0[i])
