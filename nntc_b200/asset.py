"""The asset on disk: ``nntc_b200_write_asset`` for Python callers, and a reader of the same files.

The layout is the reference's (src/export.cpp:89-146 and 470-812; its specification is the reference's
docs/FORMAT.md): level 0 as one .dds file, or two for a block-compressed level 0 of three or four channels (BC5 + BC4,
BC5 + BC5), level 1 as one uncompressed .dds, and a JSON descriptor with the extents, the bits, the dequantisation of
both levels and the decoder. The reader here parses what the writer writes: the DX10 header, the mip levels and the
descriptor, and recovers the indices and the BC endpoints and selectors from the bytes.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import struct
from dataclasses import dataclass, field

import numpy as np

from . import abi, check, lib

DXGI = {61: ("R8_UNORM", 1), 49: ("R8G8_UNORM", 2), 28: ("R8G8B8A8_UNORM", 4), 80: ("BC4_UNORM", 8), 83: ("BC5_UNORM", 16)}


def write_asset(model: abi.Model, prefix: str, k1, k0=None, ep=None, sel=None, source_size=None,
                json_path: str | None = None):
    """Write the asset of one encode. k1 (and k0 / ep / sel) are per-plane uint8 arrays, the base first; a
    block-compressed level 0 takes ep/sel (the refined blocks) or, without them, packs k0. Returns the bytes written
    for level 0's file(s), level 1's file and the descriptor."""
    n = model.nplanes
    keep = []

    def ptrs(arrays):
        if arrays is None:
            return None
        arrs = [np.ascontiguousarray(a, dtype=np.uint8) for a in arrays]
        keep.append(arrs)
        if len(arrs) != n:
            raise ValueError(f"{len(arrs)} planes given, the model has {n}")
        return abi.u8_ptrs(arrs)

    sw, sh = source_size if source_size is not None else (model.width, model.height)
    sizes = (C.c_size_t * 3)()
    check(lib().nntc_b200_write_asset(C.byref(model), ptrs(k0), ptrs(k1), ptrs(ep), ptrs(sel), int(sw), int(sh),
                                      prefix.encode(), json_path.encode() if json_path else None, sizes),
          "write_asset")
    return tuple(sizes)


@dataclass
class DdsFile:
    width: int
    height: int
    dxgi: int
    flags: int
    size_field: int
    caps: int
    levels: list = field(default_factory=list)   # bytes of each stored level, the base first

    @property
    def block_bytes(self):
        return DXGI[self.dxgi][1]

    @property
    def compressed(self):
        return self.dxgi in (80, 83)


def read_dds(path: str, sizes) -> DdsFile:
    """A DX10 .dds of the asset: its header fields and the bytes of each level at the given [w, h] sizes."""
    raw = open(path, "rb").read()
    hd = struct.unpack("<37I", raw[:148])
    if hd[0] != 0x20534444 or hd[1] != 124 or hd[21] != 0x30315844:
        raise ValueError(f"{path}: not a DX10 .dds")
    f = DdsFile(width=hd[4], height=hd[3], dxgi=hd[32], flags=hd[2], size_field=hd[5], caps=hd[27])
    if f.dxgi not in DXGI or hd[33] != 3 or hd[35] != 1:
        raise ValueError(f"{path}: not a 2D texture of a format the asset uses")
    if hd[7] != len(sizes) or [f.width, f.height] != list(sizes[0]):
        raise ValueError(f"{path}: {hd[7]} levels of {f.width}x{f.height}, the descriptor lists {sizes}")
    chain = len(sizes) > 1
    want_flags = 0x1007 | (0x20000 if chain else 0) | (0x80000 if f.compressed else 0x8)
    want_size = (((f.width + 3) // 4) * ((f.height + 3) // 4) * f.block_bytes if f.compressed
                 else f.width * f.block_bytes)
    if f.flags != want_flags or f.caps != (0x401008 if chain else 0x1000) or f.size_field != want_size:
        raise ValueError(f"{path}: header flags, caps or size field do not describe the stored levels")
    at = 148
    for w, h in sizes:
        n = ((w + 3) // 4) * ((h + 3) // 4) * f.block_bytes if f.compressed else w * h * f.block_bytes
        f.levels.append(raw[at:at + n])
        at += n
    if at != len(raw):
        raise ValueError(f"{path}: {len(raw) - at} bytes past the last level")
    return f


def bc4_fields(blocks: bytes, nblocks: int, stride: int, offset: int):
    """Endpoints (nblocks x 2) and selectors (nblocks x 16) of the BC4 blocks at `offset` within each `stride` bytes."""
    b = np.frombuffer(blocks, np.uint8).reshape(nblocks, stride)[:, offset:offset + 8]
    ep = b[:, :2].copy()
    bits = np.zeros(nblocks, np.uint64)
    for i in range(6):
        bits |= b[:, 2 + i].astype(np.uint64) << np.uint64(8 * i)
    sel = np.stack([(bits >> np.uint64(3 * t)) & np.uint64(7) for t in range(16)], axis=1).astype(np.uint8)
    return ep, sel


@dataclass
class Asset:
    descriptor: dict
    level0: list          # DdsFile per level-0 file
    level1: DdsFile


def read_asset(json_path: str) -> Asset:
    js = json.load(open(json_path))
    here = os.path.dirname(os.path.abspath(json_path))
    t0, t1 = js["textures"]
    names0 = [e["file"] if isinstance(e, dict) else e for e in t0["files"]] if "files" in t0 else [t0["file"]]
    l0 = [read_dds(os.path.join(here, n), t0["mip_sizes"]) for n in names0]
    l1 = read_dds(os.path.join(here, t1["file"]), t1["mip_sizes"])
    return Asset(js, l0, l1)


def model_from_asset(a: Asset):
    """The model, level 1's indices and level 0's state (ep/sel for a block-compressed level 0, else k0) an asset holds:
    what write_asset needs to write the same asset again."""
    js = a.descriptor
    t0, t1 = js["textures"]
    dec = js["decoder"]
    m = abi.Model()
    m.textures = js["decode"]["textures_out"]
    m.nout = dec["nout"]
    m.width, m.height = js["decode"]["width"], js["decode"]["height"]
    m.c0, m.c1 = dec["C0"], dec["C1"]
    for c in range(m.c0):
        m.bits0[c] = t0["bits_per_channel"][c]
    m.bits1 = t1["bits_per_channel"][0]
    m.bc0 = 1 if a.level0[0].compressed else 0
    m.l0_bc8 = 1 if t0["dequantise"]["kind"] == "range" else 0
    m.nin = dec["nin"]
    m.nplanes = len(t0["mip_sizes"])
    for i, ((w0, h0), (w1, h1)) in enumerate(zip(t0["mip_sizes"], t1["mip_sizes"])):
        m.w0[i], m.h0[i], m.w1[i], m.h1[i] = w0, h0, w1, h1
    for r in range(m.nout):
        m.cw[r] = 1.0
    layer = dec["layers"][0]
    m.has_decoder = 1
    for i, x in enumerate(layer["weights"]):
        m.dec_w[i] = x
    for i, x in enumerate(layer["bias"]):
        m.dec_b[i] = x
    m.has_lo1 = 1
    for c in range(m.c1):
        m.lo1[c], m.hi1[c] = t1["dequantise"]["lo"][c], t1["dequantise"]["hi"][c]
    if m.l0_bc8:
        m.has_lo0 = 1
        for c in range(m.c0):
            m.lo0[c], m.hi0[c] = t0["dequantise"]["lo"][c], t0["dequantise"]["hi"][c]
    else:
        for c in range(m.c0):
            pal = t0["dequantise"]["palette"][c]
            m.palette0_len[c] = len(pal)
            for k, x in enumerate(pal):
                m.palette0[c][k] = x
    stored1 = a.level1.block_bytes
    k1 = []
    for i, lv in enumerate(a.level1.levels):
        b = np.frombuffer(lv, np.uint8).reshape(-1, stored1)[:, :m.c1]
        k1.append((b >> (8 - m.bits1)).astype(np.uint8).ravel())
    k0 = ep = sel = None
    if m.bc0:
        ep, sel = [], []
        for i in range(m.nplanes):
            nb = ((m.w0[i] + 3) // 4) * ((m.h0[i] + 3) // 4)
            e = np.zeros((nb, m.c0, 2), np.uint8)
            s = np.zeros((nb, m.c0, 16), np.uint8)
            for f, df in enumerate(a.level0):
                nc = 1 if df.dxgi == 80 else 2
                for c in range(nc):
                    e[:, 2 * f + c], s[:, 2 * f + c] = bc4_fields(df.levels[i], nb, df.block_bytes, 8 * c)
            ep.append(e.ravel())
            sel.append(s.ravel())
    else:
        stored0 = a.level0[0].block_bytes
        k0 = []
        for i, lv in enumerate(a.level0[0].levels):
            b = np.frombuffer(lv, np.uint8).reshape(-1, stored0)[:, :m.c0].astype(np.int32)
            shift = np.array([8 - m.bits0[c] for c in range(m.c0)], np.int32)
            k0.append((b >> shift).astype(np.uint8).ravel())
    return m, k1, k0, ep, sel


def _bc4_plane(blocks: bytes, w: int, h: int, stride: int, offset: int) -> np.ndarray:
    """One channel of a BC4/BC5 level as the float bytes the standard palette decodes to (h x w)."""
    bx, by = (w + 3) // 4, (h + 3) // 4
    ep, sel = bc4_fields(blocks, bx * by, stride, offset)
    r0, r1 = ep[:, 0].astype(np.float64), ep[:, 1].astype(np.float64)
    pal = np.empty((bx * by, 8))
    pal[:, 0], pal[:, 1] = r0, r1
    wide = r0 > r1
    for i in range(2, 8):
        six = ((6 - i) * r0 + (i - 1) * r1) / 5.0 if i < 6 else np.full_like(r0, 0.0 if i == 6 else 255.0)
        pal[:, i] = np.where(wide, ((8 - i) * r0 + (i - 1) * r1) / 7.0, six)
    texel = np.take_along_axis(pal, sel.astype(np.intp), axis=1)            # (blocks, 16), row-major in the block
    img = texel.reshape(by, bx, 4, 4).transpose(0, 2, 1, 3).reshape(by * 4, bx * 4)
    return img[:h, :w]


def sampled_bytes(a: Asset, level: int, mip: int) -> np.ndarray:
    """What a UNORM sampler holds for one texture at one mip, in bytes (h x w x channels_used, float)."""
    tex = a.descriptor["textures"][level]
    w, h = tex["mip_sizes"][mip]
    used = tex["channels_used"]
    if level == 0 and a.level0[0].compressed:
        planes = []
        for f in a.level0:
            nc = 1 if f.dxgi == 80 else 2
            planes += [_bc4_plane(f.levels[mip], w, h, f.block_bytes, 8 * c) for c in range(nc)]
        return np.stack(planes, axis=-1)[:, :, :used]
    f = a.level0[0] if level == 0 else a.level1
    return np.frombuffer(f.levels[mip], np.uint8).reshape(h, w, f.block_bytes)[:, :, :used].astype(np.float64)


def decode(a: Asset, mip: int = 0) -> np.ndarray:
    """The material one mip of the asset decodes to, at level 0's texel centres: level 0 read at the texel, level 1
    sampled bilinearly with clamped taps, both dequantised after sampling (lo + byte / 255 (hi - lo)), phi in the
    descriptor's term order, out = W phi + b, saturated and rounded half up to 8 bits. h x w x 3T bytes."""
    js = a.descriptor
    t0, t1 = js["textures"]
    dec = js["decoder"]
    if dec["type"] != "bilinear" or dec["terms"].split() != ["a", "b", "sc"] or dec["hidden"]:
        raise ValueError("a decoder this format does not describe")

    def value(level, tex):
        dq = tex["dequantise"]
        lo = np.asarray(dq["lo"], np.float64)[None, None, :]
        hi = np.asarray(dq["hi"], np.float64)[None, None, :]
        return lo + sampled_bytes(a, level, mip) / 255.0 * (hi - lo)

    s = value(0, t0)
    z1 = value(1, t1)
    h, w = s.shape[:2]
    h1, w1 = z1.shape[:2]
    x = (np.arange(w) + 0.5) / w * w1 - 0.5
    y = (np.arange(h) + 0.5) / h * h1 - 0.5
    xf, yf = np.floor(x), np.floor(y)
    fx, fy = (x - xf)[None, :, None], (y - yf)[:, None, None]
    xa, xb = np.clip(xf.astype(int), 0, w1 - 1), np.clip(xf.astype(int) + 1, 0, w1 - 1)
    ya, yb = np.clip(yf.astype(int), 0, h1 - 1), np.clip(yf.astype(int) + 1, 0, h1 - 1)
    c = (z1[ya][:, xa] * (1 - fx) + z1[ya][:, xb] * fx) * (1 - fy) + (z1[yb][:, xa] * (1 - fx) + z1[yb][:, xb] * fx) * fy
    c0, c1 = dec["C0"], dec["C1"]
    phi = np.concatenate([c, s, (s[:, :, :, None] * c[:, :, None, :]).reshape(h, w, c0 * c1)], axis=-1)
    layer = dec["layers"][0]
    W = np.asarray(layer["weights"], np.float64).reshape(layer["rows"], layer["cols"])
    out = phi @ W.T + np.asarray(layer["bias"], np.float64)
    return np.floor(np.clip(out, 0.0, 1.0) * 255.0 + 0.5).astype(np.uint8)


def psnr(a: Asset, sources) -> list:
    """Per texture, the PSNR of the decoded base level against its source image (h x w x 3 bytes) over the source's
    extent (the asset may be padded)."""
    img = decode(a, 0).astype(np.float64)
    out = []
    for t, src in enumerate(sources):
        src = np.asarray(src, np.float64)
        h, w = src.shape[:2]
        mse = float(np.mean((img[:h, :w, 3 * t:3 * t + 3] - src) ** 2))
        out.append(10.0 * np.log10(255.0 * 255.0 / mse) if mse > 0 else 100.0)
    return out
