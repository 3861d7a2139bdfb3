"""The reference CPU encoder this repository builds (oracle/_ref/nntc_encode_cpu, from the reference's own sources by
oracle/Makefile) against the known answers the reference publishes for its own test image (tests/tiny.png in the
reference tree; the table of docs/CPU_BACKEND_PLAN.md, "texture PSNR (both backends)"): the per-texture PSNR the
encoder reports for the default path, --l0 palette and --c0 4 --c1 4. This pins the build the parity tests lean on; it
reads the reference tree where that is present and is skipped elsewhere."""
import os
import re
import subprocess

import pytest

import oracle as O
from conftest import reference_file

TINY = reference_file("tests", "tiny.png")


@pytest.mark.skipif(not (os.path.exists(O.REF_ENCODER) and os.path.exists(TINY)),
                    reason="needs the reference CPU encoder built and the reference's tiny.png")
@pytest.mark.parametrize("args,psnr", [([], 33.89), (["--l0", "palette"], 28.89), (["--c0", "4", "--c1", "4"], 39.66)])
def test_reference_build_reproduces_published_psnr(tmp_path, args, psnr):
    p = subprocess.run([O.REF_ENCODER, TINY, "-o", str(tmp_path) + "/", "--backend", "cpu", *args],
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    m = re.search(r"^\s*psnr\s+texture 0\s+([0-9.]+) dB", p.stdout, re.M)
    assert m, p.stdout[-3000:]
    assert float(m.group(1)) == psnr
