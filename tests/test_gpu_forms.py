"""Whole encodes of the two forms on a B200, and parity at the larger configurations.

- The adjoint + mixed-precision form (tensor-core normal equations, FP32 stencils and FP32-product conjugate
  gradients, FP32 objective, the joint pass along the adjoint's gradient) against the plain form on the same material.
  The precision switches alone (the form without its joint pass) are held two-sided: per-texture PSNR within 0.05 dB.
  The joint pass is an extra descent step the plain form does not take; it is kept only when the shipped E falls and no
  texture's base-level PSNR falls by more than 0.01 dB, so the whole form is held one-sided: no texture more than
  0.05 dB below the plain form (a texture may gain more). The joint pass never leaves the shipped E above where it
  started.
- The precision switches with the matrix-free conjugate-gradient products (NNTC_B200_OPT_ADJOINT_CG) against the plain
  form: per-texture PSNR within 0.05 dB.
- The 4 x 1024 x 1024 material (c0 2, c1 4): the plain form against the reference's own CPU encoder
  (oracle/_ref/nntc_encode_cpu), per-texture PSNR within 0.05 dB.
- The 4 x 2048 x 1024 material (c0 4, c1 4): against the reference's own CUDA encoder (oracle/_ref/nntc_encode_cuda,
  its sources unmodified, run on the same B200): the plain form and the precision switches within 0.05 dB, the
  adjoint form no texture more than 0.05 dB below."""
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


MIXED = (abi.OPT_MIXED_PRECISION_GRAM, abi.OPT_MIXED_OBJECTIVE, abi.OPT_FP32_STENCIL)


def encode(mat, form, options=()):
    a = abi.EncodeArgs()
    lib().nntc_b200_encode_defaults(a)
    a.form = form
    with Session(mat) as s:
        for o in options:
            assert lib().nntc_b200_set_option(s.d, o, 1) == 0
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
    nt = len(mat.textures)
    plain = list(encode(mat, 0).psnr[:nt])
    mixed = list(encode(mat, 0, MIXED).psnr[:nt])
    adj = encode(mat, 1)
    assert all(abs(x - y) <= 0.05 for x, y in zip(mixed, plain)), (mixed, plain)
    a = list(adj.psnr[:nt])
    assert all(x >= y - 0.05 for x, y in zip(a, plain)), (a, plain, adj.joint_taken)
    if adj.e_before_joint > 0:
        assert adj.e_ship <= adj.e_before_joint * (1 + 1e-12), (adj.e_ship, adj.e_before_joint, adj.joint_taken)
        if adj.joint_taken == 1:
            assert adj.e_joint < adj.e_before_joint


@pytest.mark.parametrize("index", [1, 2])
def test_matrix_free_cg_vs_plain(index):
    """The precision switches with the conjugate gradients' products matrix-free (the decode's forward pass and its
    adjoint, no off-diagonal stencil blocks for the CG; the quantised sweeps keep the assembled stencil): per-texture
    PSNR within 0.05 dB of the plain form."""
    mat = materials.config(index)
    nt = len(mat.textures)
    plain = list(encode(mat, 0).psnr[:nt])
    free = list(encode(mat, 0, MIXED + (abi.OPT_ADJOINT_CG,)).psnr[:nt])
    assert all(abs(x - y) <= 0.05 for x, y in zip(free, plain)), (free, plain)


def test_config2_plain_vs_reference_cpu(tmp_path):
    if not os.path.exists(O.REF_ENCODER):
        pytest.skip("the reference CPU encoder is not built")
    mat = materials.config(2)
    ours = list(encode(mat, 0).psnr[: len(mat.textures)])
    ref = reference_psnr(O.REF_ENCODER, "cpu", mat, tmp_path)
    assert len(ref) == len(ours)
    assert all(abs(x - y) <= 0.05 for x, y in zip(ours, ref)), (ours, ref)


@pytest.fixture(scope="module")
def config3_reference(tmp_path_factory):
    if not os.path.exists(REF_CUDA):
        pytest.skip("the reference CUDA encoder is not built")
    mat = materials.config(3)
    return mat, reference_psnr(REF_CUDA, "cuda", mat, tmp_path_factory.mktemp("ref3"))


@pytest.mark.parametrize("variant", ["plain", "mixed", "adjoint"])
def test_config3_vs_reference_cuda(config3_reference, variant):
    mat, ref = config3_reference
    form, options = {"plain": (0, ()), "mixed": (0, MIXED), "adjoint": (1, ())}[variant]
    ours = list(encode(mat, form, options).psnr[: len(mat.textures)])
    assert len(ref) == len(ours)
    if variant == "adjoint":
        assert all(x >= y - 0.05 for x, y in zip(ours, ref)), (ours, ref)
    else:
        assert all(abs(x - y) <= 0.05 for x, y in zip(ours, ref)), (ours, ref)
