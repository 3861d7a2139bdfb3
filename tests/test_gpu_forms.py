"""Whole encodes of the two forms on a B200, and parity at the larger configurations.

- The adjoint + mixed-precision form (tensor-core normal equations, FP32 stencils and FP32-product conjugate
  gradients, FP32 objective, the joint pass along the adjoint's gradient) against the plain form on the same material:
  per-texture PSNR within 0.05 dB; the joint pass never leaves the shipped E above where it started (it is kept only
  when E falls and no texture's base-level PSNR falls by more than 0.01 dB).
- The 4 x 1024 x 1024 material (c0 2, c1 4): the plain form against the reference's own CPU encoder
  (oracle/_ref/nntc_encode_cpu), per-texture PSNR within 0.05 dB.
- The 4 x 2048 x 1024 material (c0 4, c1 4): both forms against the reference's own CUDA encoder
  (oracle/_ref/nntc_encode_cuda, its sources unmodified, run on the same B200), per-texture PSNR within 0.05 dB."""
import os
import re
import subprocess

import numpy as np
import pytest

import oracle as O
from nntc_b200 import abi, lib, materials
from nntc_b200.session import Session

pytestmark = pytest.mark.gpu

REF_CUDA = os.path.join(os.path.dirname(O.REF_ENCODER), "nntc_encode_cuda")


def encode(mat, form):
    a = abi.EncodeArgs()
    lib().nntc_b200_encode_defaults(a)
    a.form = form
    with Session(mat) as s:
        return s.encode(a)


def reference_psnr(exe, backend, mat, tmp_path):
    pngs = materials.save_material(mat, str(tmp_path / "in"), level=1)
    p = subprocess.run([exe, *pngs, "-o", str(tmp_path / backend) + "/", "--backend", backend, "--c0", str(mat.c0),
                        "--c1", str(mat.c1), "--png", "0", "-j", str(os.cpu_count() or 1)],
                       capture_output=True, text=True, timeout=1500)
    assert p.returncode == 0, (p.stdout + p.stderr)[-2000:]
    return [float(x) for x in re.findall(r"psnr\s+texture \d+\s+([\d.]+) dB", p.stdout)]


@pytest.mark.parametrize("index", [1, 2])
def test_adjoint_form_vs_plain(index):
    mat = materials.config(index)
    plain = encode(mat, 0)
    adj = encode(mat, 1)
    nt = len(mat.textures)
    a, b = list(adj.psnr[:nt]), list(plain.psnr[:nt])
    assert all(abs(x - y) <= 0.05 for x, y in zip(a, b)), (a, b)
    if adj.e_before_joint > 0:
        assert adj.e_ship <= adj.e_before_joint * (1 + 1e-12), (adj.e_ship, adj.e_before_joint, adj.joint_taken)
        if adj.joint_taken == 1:
            assert adj.e_joint < adj.e_before_joint


def test_config2_plain_vs_reference_cpu(tmp_path):
    if not os.path.exists(O.REF_ENCODER):
        pytest.skip("the reference CPU encoder is not built")
    mat = materials.config(2)
    ours = list(encode(mat, 0).psnr[: len(mat.textures)])
    ref = reference_psnr(O.REF_ENCODER, "cpu", mat, tmp_path)
    assert len(ref) == len(ours)
    assert all(abs(x - y) <= 0.05 for x, y in zip(ours, ref)), (ours, ref)


@pytest.mark.parametrize("form", [0, 1])
def test_config3_vs_reference_cuda(tmp_path, form):
    if not os.path.exists(REF_CUDA):
        pytest.skip("the reference CUDA encoder is not built")
    mat = materials.config(3)
    ours = list(encode(mat, form).psnr[: len(mat.textures)])
    ref = reference_psnr(REF_CUDA, "cuda", mat, tmp_path)
    assert len(ref) == len(ours)
    assert all(abs(x - y) <= 0.05 for x, y in zip(ours, ref)), (ours, ref)
