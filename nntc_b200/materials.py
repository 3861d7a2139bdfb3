"""Seeded synthetic materials and the encoder's plane layout.

The reference encodes real photographs; the benchmark configurations stand in for them with seeded synthetic
textures whose recipe is fixed here (every choice the recipe leaves open is pinned in this file and nowhere else):

* ``value_noise``: a lattice of U[0,1) values per octave, smoothstep-weighted bilinear interpolation, base period
  halved per octave, amplitude multiplied by the persistence per octave, normalised by the amplitude sum.
* ``noise_rects`` (the 256x256 single-texture case): one 5-octave field per RGB channel (base period 64, persistence
  0.5) plus 8 axis-aligned rectangles (corners uniform over the image, fill U[0,1)^3) blended at alpha 0.6.
* ``pbr_material`` (the correlated 4- and 6-texture cases): a height field H from 6-octave value noise; Color = a
  3-stop random gradient lookup of H plus N(0, 6) byte jitter; Normal = the tangent-space normal of H from central
  differences (edge-clamped) at strength 4, the slope taken per 1/16 of the base period, packed as (n + 1) * 127.5;
  Roughness = 255 (0.3 + 0.5 H); AO = 255 (1 - 0.6 max(0, blur_r8(H) - H)) with blur_r8 a separable box of radius 8
  with clamped edges; and for the six-texture case Metalness = 255 [H > 0.7] and Displacement = 255 H.

Every texture is quantised to uint8 by round-to-nearest and read back as byte * (1/255) in float32, which is how the
reference loads an image (src/image.h:149-151). The layout and the source chain follow src/mips.cpp:25-40 and
src/image.h:335-366; the per-site mip weight follows src/mips.cpp:141-169.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

BLOCK = 4
MAX_MIP_LEVELS = 12


def value_noise(rng: np.random.Generator, h: int, w: int, octaves: int, period: float, persistence: float = 0.5):
    out = np.zeros((h, w), np.float64)
    amp, total, p = 1.0, 0.0, float(period)
    ys = np.arange(h, dtype=np.float64)
    xs = np.arange(w, dtype=np.float64)
    for _ in range(octaves):
        gh, gw = int(math.ceil(h / p)) + 2, int(math.ceil(w / p)) + 2
        lattice = rng.random((gh, gw))
        fy, fx = ys / p, xs / p
        iy, ix = np.floor(fy).astype(np.int64), np.floor(fx).astype(np.int64)
        ty, tx = fy - iy, fx - ix
        sy, sx = ty * ty * (3 - 2 * ty), tx * tx * (3 - 2 * tx)
        a = lattice[iy][:, ix]
        b = lattice[iy][:, ix + 1]
        c = lattice[iy + 1][:, ix]
        d = lattice[iy + 1][:, ix + 1]
        top = a + (b - a) * sx[None, :]
        bot = c + (d - c) * sx[None, :]
        out += amp * (top + (bot - top) * sy[:, None])
        total += amp
        amp *= persistence
        p = max(p / 2.0, 1.0)
    return out / total


def _to_u8(x):
    return np.clip(np.rint(x), 0, 255).astype(np.uint8)


def noise_rects(seed: int, size: int = 256):
    """One RGB8 texture: 5-octave value noise per channel plus 8 blended rectangles."""
    rng = np.random.default_rng(seed)
    img = np.stack([value_noise(rng, size, size, 5, 64.0, 0.5) for _ in range(3)], axis=-1)
    for _ in range(8):
        xa, xb = np.sort(rng.random(2) * size)
        ya, yb = np.sort(rng.random(2) * size)
        fill = rng.random(3)
        x0, x1, y0, y1 = int(xa), int(math.ceil(xb)), int(ya), int(math.ceil(yb))
        img[y0:y1, x0:x1] = 0.4 * img[y0:y1, x0:x1] + 0.6 * fill
    return [_to_u8(img * 255.0)]


def _box_blur_clamped(x, r):
    def along(a, axis):
        n = a.shape[axis]
        idx = np.arange(n)
        pad = np.take(a, np.clip(np.arange(-r - 1, n + r), 0, n - 1), axis=axis)
        c = np.cumsum(pad, axis=axis)
        hi = np.take(c, idx + 2 * r + 1, axis=axis)
        lo = np.take(c, idx, axis=axis)
        return (hi - lo) / (2 * r + 1)

    return along(along(x, 0), 1)


def pbr_material(seed: int, width: int, height: int, period: float = 128.0, six: bool = False):
    """The correlated material: Color, Normal, Roughness, AO (and Metalness, Displacement when six)."""
    rng = np.random.default_rng(seed)
    H = value_noise(rng, height, width, 6, period, 0.5)
    stops = rng.random((3, 3)) * 255.0
    t = np.clip(H, 0.0, 1.0) * 2.0
    lo = np.minimum(t.astype(np.int64), 1)
    f = (t - lo)[..., None]
    color = stops[lo] * (1 - f) + stops[lo + 1] * f
    color = color + rng.normal(0.0, 6.0, color.shape)
    slope = period / 16.0
    gx = np.empty_like(H)
    gy = np.empty_like(H)
    gx[:, 1:-1] = (H[:, 2:] - H[:, :-2]) * 0.5
    gx[:, 0] = H[:, 1] - H[:, 0]
    gx[:, -1] = H[:, -1] - H[:, -2]
    gy[1:-1, :] = (H[2:, :] - H[:-2, :]) * 0.5
    gy[0, :] = H[1, :] - H[0, :]
    gy[-1, :] = H[-1, :] - H[-2, :]
    n = np.stack([-4.0 * slope * gx, -4.0 * slope * gy, np.ones_like(H)], axis=-1)
    n /= np.linalg.norm(n, axis=-1, keepdims=True)
    normal = (n + 1.0) * 127.5
    rough = np.repeat((255.0 * (0.3 + 0.5 * H))[..., None], 3, axis=-1)
    ao = 255.0 * (1.0 - 0.6 * np.maximum(0.0, _box_blur_clamped(H, 8) - H))
    ao = np.repeat(ao[..., None], 3, axis=-1)
    tex = [color, normal, rough, ao]
    if six:
        tex.append(np.repeat((255.0 * (H > 0.7))[..., None], 3, axis=-1))
        tex.append(np.repeat((255.0 * H)[..., None], 3, axis=-1))
    return [_to_u8(x) for x in tex]


def mip_dim(n: int) -> int:
    return n // 2 if n // 2 > 0 else 1


def mip_count(w: int, h: int, min_size: int) -> int:
    n = 0
    while n < MAX_MIP_LEVELS and w // 2 >= min_size and h // 2 >= min_size:
        w //= 2
        h //= 2
        n += 1
    return n


def plane_sizes(width: int, height: int, mip_min: int = 8, mips: bool = True):
    """[(w0, h0, w1, h1)] base first, as src/mips.cpp:25-40 lays them out."""
    levels = mip_count(width, height, mip_min) if mips else 0
    planes = [(width, height, width // BLOCK, height // BLOCK)]
    for _ in range(levels):
        w0, h0, w1, h1 = planes[-1]
        planes.append((mip_dim(w0), mip_dim(h0), mip_dim(w1), mip_dim(h1)))
    return planes


def mip_weights(planes, kind: str = "pixels", mix: float = 0.5, k: int = 4):
    """The per-site mip weight of every plane (src/mips.cpp:141-169)."""
    n = len(planes)
    if n == 1:
        return [1.0]
    r = [0.0] * n
    total = 0.0
    for m in range(1, n):
        pixels = float(planes[m][0]) * float(planes[m][1])
        r[m] = 1.0 if kind == "uniform" else (math.sqrt(pixels) if kind == "sqrt" else pixels)
        total += r[m]
    share = [1.0 - mix] + [mix * r[m] / total if total > 0 else 0.0 for m in range(1, n)]
    out = []
    for m in range(n):
        sites = float(planes[m][0]) * float(planes[m][1]) * float(1 + k)
        out.append(share[m] / sites if sites > 0 else 0.0)
    return out


def pack_textures(textures):
    """3T interleaved float32 channels in [0,1], byte * (1/255) as the reference loads them."""
    inv = np.float32(1.0) / np.float32(255.0)
    return np.concatenate([t.astype(np.float32) * inv for t in textures], axis=-1)


def box_down(img):
    """One level of the default chain: the 2x2 box of src/image.h:343-366, in the same float32 order."""
    h, w, nc = img.shape
    oh, ow = mip_dim(h), mip_dim(w)
    xs = np.arange(ow)
    ys = np.arange(oh)
    xa = np.where(2 * xs < w, 2 * xs, w - 1)
    xb = np.where(2 * xs + 1 < w, 2 * xs + 1, w - 1)
    ya = np.where(2 * ys < h, 2 * ys, h - 1)
    yb = np.where(2 * ys + 1 < h, 2 * ys + 1, h - 1)
    a = img[ya][:, xa]
    b = img[ya][:, xb]
    c = img[yb][:, xa]
    d = img[yb][:, xb]
    return (np.float32(0.25) * ((a + b) + (c + d))).astype(np.float32)


def source_chain(base, planes):
    chain = [np.ascontiguousarray(base, np.float32)]
    for _ in range(1, len(planes)):
        chain.append(box_down(chain[-1]))
    return chain


@dataclass
class Material:
    name: str
    textures: list
    c0: int = 2
    c1: int = 4
    k: int = 4
    mip_min: int = 8
    planes: list = field(default_factory=list)
    chain: list = field(default_factory=list)
    per_site: list = field(default_factory=list)

    @property
    def width(self):
        return self.textures[0].shape[1]

    @property
    def height(self):
        return self.textures[0].shape[0]

    @property
    def nout(self):
        return 3 * len(self.textures)

    def build(self):
        self.planes = plane_sizes(self.width, self.height, self.mip_min, True)
        self.chain = source_chain(pack_textures(self.textures), self.planes)
        self.per_site = mip_weights(self.planes, "pixels", 0.5, self.k)
        return self

    @property
    def chain_pixels(self):
        return sum(p[0] * p[1] for p in self.planes)


# The benchmark configurations, by what they are.
def config(index: int, seed: int = 0) -> Material:
    if index == 0:
        return Material("1x256x256 noise+rects c0=2 c1=4", noise_rects(seed, 256), 2, 4).build()
    if index == 1:
        return Material("4x512x512 pbr c0=2 c1=4", pbr_material(seed, 512, 512, 128.0), 2, 4).build()
    if index == 2:
        return Material("4x1024x1024 pbr c0=2 c1=4", pbr_material(seed, 1024, 1024, 128.0), 2, 4).build()
    if index == 3:
        return Material("4x2048x1024 pbr c0=4 c1=4", pbr_material(seed, 2048, 1024, 128.0), 4, 4).build()
    if index == 4:
        return Material("6x4096x4096 pbr c0=4 c1=4", pbr_material(seed, 4096, 4096, 512.0, six=True), 4, 4).build()
    raise ValueError(index)


def small(seed: int, width: int, height: int, textures: int = 1, c0: int = 2, c1: int = 4, k: int = 4,
          mip_min: int = 8) -> Material:
    """A small material of the same recipe for parity tests (any size, including ragged ones)."""
    if textures == 1:
        rng = np.random.default_rng(seed)
        img = np.stack([value_noise(rng, height, width, 4, max(4.0, min(width, height) / 4.0)) for _ in range(3)], -1)
        tex = [_to_u8(img * 255.0)]
    else:
        tex = pbr_material(seed, width, height, max(8.0, min(width, height) / 2.0), six=textures > 4)[:textures]
    return Material(f"{textures}x{width}x{height}", tex, c0, c1, k, mip_min).build()


def write_png(path: str, rgb8, level: int = 6) -> None:
    """An 8-bit RGB PNG (zlib-compressed, filter 0 rows): what the reference's encoder reads as its input."""
    import struct
    import zlib

    a = np.ascontiguousarray(rgb8, np.uint8)
    h, w, _ = a.shape
    raw = b"".join(b"\x00" + a[y].tobytes() for y in range(h))

    def chunk(tag, data):
        return struct.pack(">I", len(data)) + tag + data + struct.pack(">I", zlib.crc32(tag + data) & 0xFFFFFFFF)

    with open(path, "wb") as f:
        f.write(b"\x89PNG\r\n\x1a\n")
        f.write(chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 2, 0, 0, 0)))
        f.write(chunk(b"IDAT", zlib.compress(raw, level)))
        f.write(chunk(b"IEND", b""))


def save_material(material, directory: str, level: int = 6):
    """The material's textures as PNGs (zlib level `level`), in order; returns the paths."""
    import os

    os.makedirs(directory, exist_ok=True)
    paths = []
    for i, t in enumerate(material.textures):
        p = os.path.join(directory, f"tex{i}.png")
        write_png(p, t, level)
        paths.append(p)
    return paths
