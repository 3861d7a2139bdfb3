"""Golden assets from the REFERENCE encoder itself: oracle/_ref/nntc_encode_cpu (the reference's own host and CPU arm,
built by oracle/Makefile from its sources) encodes small seeded materials in each level-0 / level-1 layout the format
distinguishes, and its .dds files and JSON descriptor are kept under tests/golden/assets/<case>/. The asset writer's
tests re-write each one from the state it holds and compare the bytes.

    python tests/golden/make_golden_asset.py      (needs oracle/_ref built; rewrites tests/golden/assets/)
"""
from __future__ import annotations

import json
import os
import shutil
import subprocess
import sys
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from nntc_b200 import materials  # noqa: E402
import oracle as O  # noqa: E402

OUT = os.path.join(ROOT, "tests", "golden", "assets")

# seed, size and texture count of the material (nntc_b200/materials.py small()), and the encoder's layout arguments
CASES = {
    "bc8_c2_padded": dict(seed=11, w=22, h=14, textures=1, args=[]),
    "bc8_c3_t2": dict(seed=12, w=40, h=36, textures=2, args=["--c0", "3", "--c1", "3", "--bits1", "6"]),
    "bc8_c4_t4": dict(seed=13, w=64, h=48, textures=4, args=["--c0", "4", "--c1", "4"]),
    "bc8_c1": dict(seed=14, w=32, h=32, textures=1, args=["--c0", "1", "--c1", "2", "--bits1", "5"]),
    "palette_plain": dict(seed=15, w=32, h=24, textures=1, args=["--l0", "palette", "--bits0", "2", "--bc0", "0",
                                                                 "--c1", "1"]),
    "palette_bc": dict(seed=16, w=36, h=28, textures=1, args=["--l0", "palette", "--bits0", "3", "--c0", "3"]),
    "one_level": dict(seed=17, w=24, h=24, textures=1, args=["--mips", "0"]),
    "bc8_twin": dict(seed=18, w=24, h=20, textures=1, args=["--bc0", "both"]),
}


def main():
    if not os.path.exists(O.REF_ENCODER):
        raise SystemExit(f"{O.REF_ENCODER} is not built (make -C oracle)")
    shutil.rmtree(OUT, ignore_errors=True)
    os.makedirs(OUT)
    for name, spec in CASES.items():
        with tempfile.TemporaryDirectory() as tmp:
            mat = materials.small(spec["seed"], spec["w"], spec["h"], textures=spec["textures"])
            pngs = materials.save_material(mat, os.path.join(tmp, "in"))
            out = os.path.join(tmp, "out")
            p = subprocess.run([O.REF_ENCODER, *pngs, "-o", out + "/", "--backend", "cpu", "--quiet", *spec["args"]],
                               capture_output=True, text=True, timeout=600)
            if p.returncode != 0:
                raise SystemExit(f"{name}: the reference encoder failed\n{p.stdout}{p.stderr}")
            dst = os.path.join(OUT, name)
            os.makedirs(dst)
            for f in sorted(os.listdir(out)):
                if f.endswith(".dds") or f.endswith("_nntc.json"):
                    shutil.copy(os.path.join(out, f), os.path.join(dst, f))
            print(name, sorted(os.listdir(dst)))
    with open(os.path.join(OUT, "cases.json"), "w") as f:
        json.dump(CASES, f, indent=1)


if __name__ == "__main__":
    main()
