"""The asset writer (nntc_b200_write_asset) against the reference's own assets.

tests/golden/assets holds assets the reference encoder wrote (tests/golden/make_golden_asset.py), one per layout the
format distinguishes: a block-compressed level 0 of one to four channels (BC4, BC5, BC5 + BC4, BC5 + BC5), a padded
source, a palette-mode level 0 stored uncompressed and one packed by the seed pack, a single stored level. Each is read
back (nntc_b200/asset.py), its state handed to the writer, and the writer's output compared with the reference's:

- every .dds file byte for byte (header, level order, block and texel bytes);
- every descriptor key a reader needs, with the same value (floats as float32, exactly); the prose keys are the
  writer's own and are not compared.

Where the reference's own reader of the format (tools/dds_decode.py) is present it reads the re-written asset too and
must report what it reports for the reference's."""
import ctypes as C
import json
import os
import re
import shutil
import subprocess
import sys

import numpy as np
import pytest
from PIL import Image

from nntc_b200 import NntcError, abi, check, lib, materials
from nntc_b200 import asset as A
from conftest import reference_file

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "assets")
CASES = json.load(open(os.path.join(GOLDEN, "cases.json")))
REF_READER = reference_file("tools", "dds_decode.py")


def indices_from_blocks(m, ep, sel):
    """Level 0's indices from lossless blocks (palette mode at 1-3 bits, where the decoded byte is k 255 / levels)."""
    k0 = []
    for i in range(m.nplanes):
        w, h = m.w0[i], m.h0[i]
        bx = (w + 3) // 4
        e = ep[i].reshape(-1, m.c0, 2).astype(np.int32)
        s = sel[i].reshape(-1, m.c0, 16)
        k = np.zeros((h, w, m.c0), np.uint8)
        for c in range(m.c0):
            levels = (1 << m.bits0[c]) - 1
            for y in range(h):
                for x in range(w):
                    b = (y // 4) * bx + x // 4
                    r0, r1, j = e[b, c, 0], e[b, c, 1], s[b, c, (y % 4) * 4 + x % 4]
                    if r0 > r1:
                        pal = [r0, r1] + [((8 - t) * r0 + (t - 1) * r1) / 7.0 for t in range(2, 8)]
                    else:
                        pal = [r0, r1] + [((6 - t) * r0 + (t - 1) * r1) / 5.0 for t in range(2, 6)] + [0, 255]
                    k[y, x, c] = int(round(pal[j] * levels / 255.0))
        k0.append(k.ravel())
    return k0


def descriptors(case):
    return sorted(f for f in os.listdir(os.path.join(GOLDEN, case)) if f.endswith("_nntc.json"))


def rewrite(case, out_dir, jname=None):
    src = os.path.join(GOLDEN, case)
    jname = jname or descriptors(case)[0]
    a = A.read_asset(os.path.join(src, jname))
    m, k1, k0, ep, sel = A.model_from_asset(a)
    if m.bc0 and not m.l0_bc8:
        # palette mode packs k0 itself: hand the writer the indices, not the blocks
        k0, ep, sel = indices_from_blocks(m, ep, sel), None, None
    js = a.descriptor
    prefix = os.path.join(out_dir, jname[: -len("_nntc.json")])
    sizes = A.write_asset(m, prefix, k1, k0=k0, ep=ep, sel=sel,
                          source_size=(js["source"]["width"], js["source"]["height"]))
    return src, jname, prefix, sizes


def required(js):
    """The descriptor's keys a reader needs (the format specification's required ones), prose left out."""
    out = {k: js[k] for k in ("format", "decode", "block", "lod_bias_level1")}
    out["source"] = {k: v for k, v in js["source"].items() if k != "inputs"}
    tex = []
    for t in js["textures"]:
        e = {k: t[k] for k in ("level", "width", "height", "dxgi_format", "dxgi_format_id", "channels_used",
                               "channels_stored", "bits_per_channel", "mip_count", "mip_sizes")}
        e["file"] = t.get("file")
        e["files"] = t.get("files")
        e["bc_palette"] = t.get("bc_palette")
        d = dict(t["dequantise"])
        d.pop("note")
        e["dequantise"] = d
        tex.append(e)
    out["textures"] = tex
    dec = {k: js["decoder"][k] for k in ("type", "terms", "C0", "C1", "nin", "nout", "hidden", "output",
                                        "activation", "leak")}
    dec["layers"] = js["decoder"]["layers"]
    out["decoder"] = dec
    return out


def as_f32(x):
    if isinstance(x, float):
        return float(np.float32(x))
    if isinstance(x, list):
        return [as_f32(v) for v in x]
    if isinstance(x, dict):
        return {k: as_f32(v) for k, v in x.items()}
    return x


@pytest.mark.parametrize("case,jname", [(c, j) for c in sorted(CASES) for j in descriptors(c)])
def test_rewritten_asset_is_the_references(tmp_path, case, jname):
    src, jname, prefix, sizes = rewrite(case, str(tmp_path), jname)
    stem = jname[: -len("_nntc.json")]
    ours_dds = sorted(f for f in os.listdir(str(tmp_path)) if f.endswith(".dds"))
    theirs_dds = sorted(f for f in os.listdir(src) if f.endswith(".dds") and f[len(stem):].startswith("_lat"))
    assert ours_dds == theirs_dds, (case, ours_dds, theirs_dds)
    for f in ours_dds:
        ours = open(os.path.join(str(tmp_path), f), "rb").read()
        theirs = open(os.path.join(src, f), "rb").read()
        assert ours == theirs, (case, f, len(ours), len(theirs))
    ours = json.load(open(prefix + "_nntc.json"))
    theirs = json.load(open(os.path.join(src, jname)))
    assert as_f32(required(ours)) == as_f32(required(theirs)), case
    dds = sum(os.path.getsize(os.path.join(str(tmp_path), f)) for f in ours_dds)
    assert sizes[0] + sizes[1] == dds and sizes[2] == os.path.getsize(prefix + "_nntc.json")


def test_writer_refuses_what_the_reference_refuses(tmp_path):
    src = os.path.join(GOLDEN, "bc8_c2_padded")
    a = A.read_asset(os.path.join(src, "tex0_nntc.json"))
    m, k1, k0, ep, sel = A.model_from_asset(a)
    bad = tmp_path / "bad"
    bad.mkdir()
    # a decoder weight that is not finite: nothing is written
    m.dec_w[3] = float("nan")
    with pytest.raises(NntcError):
        A.write_asset(m, str(bad / "x"), k1, ep=ep, sel=sel, source_size=(22, 14))
    assert os.listdir(str(bad)) == []
    m.dec_w[3] = 0.5
    # a level-1 grid on which a stored index no longer reads back as itself
    m.lo1[0] = m.hi1[0]
    with pytest.raises(NntcError):
        A.write_asset(m, str(bad / "x"), k1, ep=ep, sel=sel, source_size=(22, 14))
    assert "read back" in lib().nntc_b200_last_error().decode()


@pytest.mark.skipif(not os.path.exists(REF_READER), reason="the reference's reader of the format is not present")
@pytest.mark.parametrize("case", ["bc8_c3_t2", "palette_plain", "palette_bc"])
def test_reference_reader_takes_the_rewritten_asset(tmp_path, case):
    spec = CASES[case]
    mat = materials.small(spec["seed"], spec["w"], spec["h"], textures=spec["textures"])
    pngs = materials.save_material(mat, str(tmp_path / "in"))
    ref_dir = tmp_path / "ref"
    shutil.copytree(os.path.join(GOLDEN, case), str(ref_dir))
    ours_dir = tmp_path / "ours"
    ours_dir.mkdir()
    _, _, prefix, _ = rewrite(case, str(ours_dir))

    def reader(pre, *args):
        p = subprocess.run([sys.executable, REF_READER, pre, *args], capture_output=True, text=True, timeout=300)
        return p.returncode, p.stdout

    for args in (["--grid"], ["--psnr", *pngs]):
        rc_ours, out_ours = reader(prefix, *args)
        rc_ref, out_ref = reader(str(ref_dir / "tex0"), *args)
        assert rc_ours == 0 and rc_ref == 0, (out_ours, out_ref)
        strip = lambda s: [l for l in s.splitlines() if "tex0" not in l]  # noqa: E731  (lines naming the path differ)
        assert strip(out_ours) == strip(out_ref), (out_ours, out_ref)
    # this package's own decoder of the format agrees with the reference's reader (which prints two decimals)
    quoted = [float(re.search(r"psnr ([0-9.]+) dB", l).group(1)) for l in out_ref.splitlines()
              if re.match(r"\s*texture \d+:", l)]
    sources = [np.asarray(Image.open(p).convert("RGB")) for p in pngs]
    ours = A.psnr(A.read_asset(prefix + "_nntc.json"), sources)
    assert len(quoted) == len(ours) and all(abs(a - b) <= 0.0051 for a, b in zip(ours, quoted)), (ours, quoted)


REF_EXAMPLES = reference_file("examples")
SHIPPED = ["m1_m4_c0_3_c1_4", "pavingstones141_1k_c0_4"]


@pytest.mark.skipif(not os.path.isdir(REF_EXAMPLES), reason="the reference's example assets are not present")
@pytest.mark.parametrize("stem", SHIPPED)
def test_rewritten_shipped_example_is_the_references(tmp_path, stem):
    """The example assets the reference ships (a 512 x 512 four-texture material at C0 = 3 and a 1K five-texture one at
    C0 = 4), re-written from their own state: the same .dds bytes and the same descriptor keys."""
    jpath = os.path.join(REF_EXAMPLES, stem + "_nntc.json")
    if not os.path.exists(jpath):
        pytest.skip(f"{stem} is not among the reference's examples")
    a = A.read_asset(jpath)
    m, k1, k0, ep, sel = A.model_from_asset(a)
    js = a.descriptor
    prefix = str(tmp_path / stem)
    A.write_asset(m, prefix, k1, k0=k0, ep=ep, sel=sel, source_size=(js["source"]["width"], js["source"]["height"]))
    for f in sorted(os.listdir(str(tmp_path))):
        if f.endswith(".dds"):
            assert open(os.path.join(str(tmp_path), f), "rb").read() == open(os.path.join(REF_EXAMPLES, f), "rb").read(), f
    assert as_f32(required(json.load(open(prefix + "_nntc.json")))) == as_f32(required(js))


@pytest.mark.parametrize("case", ["bc8_c1", "bc8_c3_t2", "bc8_c4_t4", "palette_bc"])
def test_bc_pack_blocks_gives_the_files_blocks(case):
    """nntc_b200_bc_pack_blocks (the seam's host pack, src/export.cpp:333-370) turns each plane's endpoints and
    selectors into the reference's file bytes; on a lossless palette-mode plane its error against k0 is the float
    rounding of the palette (the decoded entry is a float division by 7, the exact value a double one)."""
    src = os.path.join(GOLDEN, case)
    a = A.read_asset(os.path.join(src, descriptors(case)[0]))
    m, k1, k0, ep, sel = A.model_from_asset(a)
    lossless = not m.l0_bc8
    if lossless:
        k0 = indices_from_blocks(m, ep, sel)
    for i in range(m.nplanes):
        files = [np.zeros(len(f.levels[i]), np.uint8) for f in a.level0]
        se, n = C.c_double(0.0), C.c_size_t(0)
        kk = np.ascontiguousarray(k0[i]) if lossless else None
        check(lib().nntc_b200_bc_pack_blocks(C.byref(m), i, ep[i].ctypes.data_as(C.POINTER(C.c_uint8)),
                                             sel[i].ctypes.data_as(C.POINTER(C.c_uint8)),
                                             kk.ctypes.data_as(C.POINTER(C.c_uint8)) if kk is not None else None,
                                             abi.u8_ptrs(files), C.byref(se), C.byref(n)), "bc_pack_blocks")
        for f, mine in zip(a.level0, files):
            assert mine.tobytes() == f.levels[i], (case, i)
        if lossless:
            assert se.value <= 1e-9 * n.value and n.value == m.w0[i] * m.h0[i] * m.c0
