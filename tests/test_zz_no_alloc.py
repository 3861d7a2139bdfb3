"""nntc_b200_objective_plane_noalloc against nntc_b200_objective_eval, through the C ABI on a B200.

The no-allocation entry point reads one plane from the caller's own device buffers (torch tensors here) and writes
its three raw sums into caller memory, with a static device array as its only scratch. It runs the same two kernels
as the device-model objective on a one-plane launch, so the plane's normalised figures must agree with the ones
nntc_b200_objective_eval reports for that plane within TOL relative (in practice they are the same bits). Each plane
is evaluated twice in a row, so a second call that read anything left over from the first would show.

This file is named to be collected last: it must pass alone and after every other test in the same process."""
import numpy as np
import pytest

from nntc_b200 import NntcError, abi, check, lib, materials
from nntc_b200.session import Session

pytestmark = pytest.mark.gpu

TOL = 1e-12   # relative


def call(v0, v1, src, w, b, cw, sums, plane, m, k, stream):
    w0, h0, w1, h1 = plane
    return lib().nntc_b200_objective_plane_noalloc(
        v0.data_ptr(), w0, h0, m.c0, v1.data_ptr(), w1, h1, m.c1, src.data_ptr(), m.nout, w.data_ptr(),
        b.data_ptr(), cw.data_ptr(), m.nin, k, sums.data_ptr(), stream)


def close(a, b):
    return abs(a - b) <= TOL * max(abs(a), abs(b))


@pytest.mark.parametrize("textures,c0,c1,w,h,k", [(2, 4, 4, 72, 40, 4), (1, 2, 4, 61, 37, 4), (6, 4, 4, 48, 44, 1),
                                                  (3, 3, 2, 50, 34, 2), (2, 1, 3, 40, 28, 0)])
def test_noalloc_matches_objective_eval(textures, c0, c1, w, h, k):
    import torch

    mat = materials.small(50 + w, w, h, textures=textures, c0=c0, c1=c1)
    rng = np.random.default_rng(w * 31 + h)
    nin, nout = abi.feature_count(c0, c1), 3 * textures
    dw = (rng.standard_normal((nout, nin)) * 0.3).astype(np.float32)
    db = rng.random(nout).astype(np.float32)
    v0 = [(rng.random(p[0] * p[1] * c0) * 2 - 1).astype(np.float32) for p in mat.planes]
    v1 = [(rng.random(p[2] * p[3] * c1) * 2 - 1).astype(np.float32) for p in mat.planes]
    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream(dev).cuda_stream
    with Session(mat) as s:
        for i in range(len(mat.planes)):
            s.set_planes(i, v0[i], v1[i])
        s.set_decoder(dw, db)
        ref = s.objective(k)
        m = s.m
        cw_host = np.array(m.cw[:nout], np.float32)
        weights = torch.from_numpy(np.array(m.dec_w[: nout * nin], np.float32)).to(dev)
        bias = torch.from_numpy(np.array(m.dec_b[:nout], np.float32)).to(dev)
        cw = torch.from_numpy(cw_host).to(dev)
        sum_cw = 0.0
        for c in range(nout):
            sum_cw += float(cw_host[c])
        for i, p in enumerate(mat.planes):
            t0 = torch.from_numpy(v0[i]).to(dev)
            t1 = torch.from_numpy(v1[i]).to(dev)
            src = torch.from_numpy(np.ascontiguousarray(mat.chain[i], np.float32).ravel()).to(dev)
            pixels = float(p[0]) * float(p[1])
            for rep in range(2):
                sums = torch.full((3,), float("nan"), dtype=torch.float64, device=dev)
                check(call(t0, t1, src, weights, bias, cw, sums, p, m, k, stream), "objective_plane_noalloc")
                torch.cuda.synchronize(dev)
                out = sums.cpu().numpy()
                assert close(out[0] / (sum_cw * (pixels * (1 + k))), ref.e_plane[i]), (i, rep)
                assert close(out[1] / (pixels * nout), ref.centre_plane[i]), (i, rep)
                if i == 0 and k > 0:
                    assert close(out[2] / (pixels * nout * k), ref.sampled_mse), rep
                elif k == 0:
                    assert out[2] == 0.0, rep   # no fractional sites: their sum is an exact zero


def test_noalloc_rejects_a_plane_above_its_limit():
    import torch

    dev = torch.device("cuda:0")
    f = torch.zeros(64, dtype=torch.float32, device=dev)
    sums = torch.zeros(3, dtype=torch.float64, device=dev)
    side = 4097   # 4097 x 4097 pixels is above the 4096 x 4096 the static scratch holds
    st = lib().nntc_b200_objective_plane_noalloc(f.data_ptr(), side, side, 2, f.data_ptr(), 4, 4, 4, f.data_ptr(), 3,
                                                 f.data_ptr(), f.data_ptr(), f.data_ptr(), 14, 4, sums.data_ptr(),
                                                 torch.cuda.current_stream(dev).cuda_stream)
    assert st == 1   # NNTC_B200_ERR_ARG, before any device work
    assert "above the limit" in lib().nntc_b200_last_error().decode()
    with pytest.raises(NntcError):
        check(st, "objective_plane_noalloc")
