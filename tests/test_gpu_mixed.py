"""The mixed-precision decoder fit on a B200: block (a)'s normal equations on the tcgen05 tensor cores (BF16 hi + lo
split site rows, FP32 accumulators in tensor memory, FP64 across batches of 256 sites) against the same sums formed
exactly (products of floats are exact in double, summed in FP64), on the same state.

Bars: every entry of the system within 2e-6 of the largest entry of its kind (the split holds each factor to about
2^-17 of itself); the decoder the device Cholesky solves from it within 1e-4 relative of the FP64 form's decoder
(relative to the largest coefficient of the same output row), which is the bar the mixed-precision form is held to
against the FP64 oracle; and the tensor-core sums are the same bits on a second run (fixed-order reduction)."""
import ctypes as C

import numpy as np
import pytest

from nntc_b200 import abi, check, lib, materials
from nntc_b200.session import Session

pytestmark = pytest.mark.gpu


def state(seed, w, h, textures, c0, c1, k=4):
    mat = materials.small(seed, w, h, textures=textures, c0=c0, c1=c1, k=k)
    rng = np.random.default_rng(seed)
    v0 = [(rng.random(p[0] * p[1] * c0) * 2 - 1).astype(np.float32) for p in mat.planes]
    v1 = [(rng.random(p[2] * p[3] * c1) * 2 - 1).astype(np.float32) for p in mat.planes]
    return mat, v0, v1


def solve(s, mixed, k):
    check(lib().nntc_b200_set_option(s.d, abi.OPT_MIXED_PRECISION_GRAM, 1 if mixed else 0), "option")
    s.m.has_decoder = 0
    s.solve_decoder(k)
    w, b = s.decoder()
    return s.normal_equations(), np.concatenate([w.reshape(s.m.nout, -1), b.reshape(-1, 1)], axis=1)


@pytest.mark.parametrize("textures,c0,c1,w,h,k", [(4, 4, 4, 128, 96, 4), (6, 4, 4, 70, 52, 4), (1, 2, 4, 64, 64, 4),
                                                  (2, 3, 2, 45, 31, 2), (3, 1, 1, 33, 20, 0)])
def test_tensor_core_normal_equations_vs_fp64(textures, c0, c1, w, h, k):
    mat, v0, v1 = state(w * h + textures, w, h, textures, c0, c1, k)
    with Session(mat) as s:
        for i in range(len(mat.planes)):
            s.set_planes(i, v0[i], v1[i])
        s.set_grids(np.full(c0, -1.0), np.full(c0, 1.0))
        ne64, x64 = solve(s, False, k)
        ne_tc, x_tc = solve(s, True, k)
        ne_tc2, _ = solve(s, True, k)
    mm = abi.feature_count(c0, c1) + 1
    tri = mm * (mm + 1) // 2
    for part in (slice(0, tri), slice(tri, ne64.size)):
        scale = np.abs(ne64[part]).max()
        err = np.abs(ne_tc[part] - ne64[part]).max()
        assert err <= 2e-6 * scale, (err / scale)
    assert np.array_equal(ne_tc, ne_tc2), "the tensor-core sums are not reproducible"
    row_scale = np.abs(x64).max(axis=1, keepdims=True)
    rel = np.abs(x_tc - x64) / row_scale
    assert rel.max() <= 1e-4, rel.max()


def test_precision_report_against_fp64():
    """The adjoint form's errors against the FP64 form after an encode of a small material (c0 = c1 = 4): the decoder
    from the tensor-core sums and one block (b) and (c') solve on the FP32 stencil, each within 1e-4 relative."""
    mat = materials.small(31, 96, 80, textures=4, c0=4, c1=4)
    with Session(mat) as s:
        a = abi.EncodeArgs()
        lib().nntc_b200_encode_defaults(a)
        a.form = 1
        s.encode(a)
        rep = s.precision_report()
    assert rep["decoder"] <= 1e-4 and rep["level1"] <= 1e-4 and rep["level0"] <= 1e-4, rep


@pytest.mark.parametrize("textures,c0,c1,w,h,k", [(4, 4, 4, 128, 96, 4), (6, 4, 4, 70, 52, 4), (2, 2, 4, 64, 48, 2),
                                                  (3, 3, 2, 45, 31, 1)])
def test_fp32_objective_vs_fp64(textures, c0, c1, w, h, k):
    """The adjoint form's objective (the decode in FP32 with fused multiply-adds, each site's squared residuals summed in
    FP32, the sites' sums in FP64) against the FP64 objective on the same state and decoder: E and every plane's E
    within 1e-6 relative."""
    mat, v0, v1 = state(w * h + 7 * textures, w, h, textures, c0, c1, k)
    rng = np.random.default_rng(w + h)
    nin, nout = abi.feature_count(c0, c1), 3 * textures
    with Session(mat) as s:
        for i in range(len(mat.planes)):
            s.set_planes(i, v0[i], v1[i])
        s.set_decoder(rng.standard_normal((nout, nin)) * 0.2, rng.random(nout) * 0.5)
        out = []
        for mixed in (0, 1):
            check(lib().nntc_b200_set_option(s.d, abi.OPT_MIXED_OBJECTIVE, mixed), "option")
            r = s.objective(k)
            out.append((r.e, list(r.e_plane[: len(mat.planes)]), r.centre_mse, r.sampled_mse))
    (e64, p64, c64, s64), (e32, p32, c32, s32) = out
    assert abs(e32 - e64) <= 1e-6 * e64, (e32, e64)
    for a, b in zip(p32, p64):
        assert abs(a - b) <= 1e-6 * b, (a, b)
    assert abs(c32 - c64) <= 1e-6 * c64 and abs(s32 - s64) <= 1e-6 * max(s64, 1e-300)


@pytest.mark.parametrize("textures,c0,c1,w,h", [(4, 4, 4, 128, 96), (2, 4, 4, 64, 64), (3, 2, 4, 70, 52),
                                                (1, 3, 2, 45, 31)])
def test_fp32_stencil_vs_fp64(textures, c0, c1, w, h):
    """The adjoint form's FP32 assembly (fused site terms, one thread per texel gathering all five slots, the stencil
    stored per texel block) against the FP64 assembly on the same state: every plane's stencil within 1e-5 of its
    largest coefficient and its gradient within 1e-5 of its largest entry, both levels, across interior (tabled) and
    border texels."""
    mat, v0, v1 = state(w * h + 11 * textures, w, h, textures, c0, c1)
    rng = np.random.default_rng(w * 3 + h)
    nin, nout = abi.feature_count(c0, c1), 3 * textures
    with Session(mat) as s:
        for i in range(len(mat.planes)):
            s.set_planes(i, v0[i], v1[i])
        s.set_decoder(rng.standard_normal((nout, nin)) * 0.3, rng.random(nout))
        s.set_grids(np.full(c0, -1.0), np.full(c0, 1.0), np.full(c1, -1.0), np.full(c1, 1.0))
        for level0 in (False, True):
            got = []
            for mixed in (0, 1):
                check(lib().nntc_b200_set_option(s.d, abi.OPT_FP32_STENCIL, mixed), "option")
                for i in range(len(mat.planes)):
                    s.set_planes(i, v0[i], v1[i])
                s.block(level0, k=4)
                got.append([s.workspace(i, level0) for i in range(len(mat.planes))])
            for i, (a, b) in enumerate(zip(got[0], got[1])):
                for key in ("stencil", "grad"):
                    scale = np.abs(a[key]).max()
                    err = np.abs(b[key] - a[key]).max()
                    assert err <= 1e-5 * scale, (level0, i, key, err / max(scale, 1e-300))


@pytest.mark.parametrize("textures,c0,c1,w,h,k", [(4, 4, 4, 128, 96, 4), (6, 4, 4, 70, 52, 4), (2, 2, 4, 64, 48, 2)])
def test_objective_with_normal_equations(textures, c0, c1, w, h, k):
    """The adjoint form's round-closing pass (the tensor-core normal equations and E of the current decoder from one
    pass over the sites) against the two passes it replaces, on the same state: the normal equations the same bits as
    the tensor-core pass alone, E and every plane's E within 1e-12 of the FP32 objective (the same per-site values,
    their FP64 sums in another order)."""
    mat, v0, v1 = state(w * h + 13 * textures, w, h, textures, c0, c1, k)
    rng = np.random.default_rng(w + 2 * h)
    nin, nout = abi.feature_count(c0, c1), 3 * textures
    with Session(mat) as s:
        for i in range(len(mat.planes)):
            s.set_planes(i, v0[i], v1[i])
        s.set_decoder(rng.standard_normal((nout, nin)) * 0.2, rng.random(nout) * 0.5)
        for opt in (abi.OPT_MIXED_PRECISION_GRAM, abi.OPT_MIXED_OBJECTIVE):
            check(lib().nntc_b200_set_option(s.d, opt, 1), "option")
        ref = s.objective(k)
        w_keep, b_keep = s.decoder()
        s.solve_decoder(k)                      # the tensor-core normal equations alone (and a solve)
        ne_alone = s.normal_equations()
        s.set_decoder(w_keep, b_keep)
        got = abi.Objective()
        check(lib().nntc_b200_probe_objective_with_normal_equations(s.d, C.byref(s.m), k, s.per_site, C.byref(got)),
              "fused")
        ne_fused = s.normal_equations()
    assert np.array_equal(ne_fused, ne_alone)
    assert abs(got.e - ref.e) <= 1e-12 * ref.e, (got.e, ref.e)
    for i in range(len(mat.planes)):
        assert abs(got.e_plane[i] - ref.e_plane[i]) <= 1e-12 * ref.e_plane[i], (i, got.e_plane[i], ref.e_plane[i])
