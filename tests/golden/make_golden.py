"""Golden vectors from the REFERENCE itself: its CPU arm (src/cpu/*.cpp, built into oracle/_ref/libnntc_ref.so by
oracle/Makefile from the reference sources) driven seam call by seam call through a short encode of two small seeded
materials. Every step records the state it started from and what the reference computed, so each kernel of the C
restatement (oracle/nntc_oracle.c) and of the CUDA path can be replayed against it in isolation.

    python tests/golden/make_golden.py      (needs oracle/_ref built; rewrites tests/golden/*.npz)
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from nntc_b200 import abi, materials  # noqa: E402
import oracle as O  # noqa: E402

CASES = {
    "t1_c0_2": dict(seed=11, w=32, h=24, textures=1, c0=2, c1=4),
    "t2_c0_4": dict(seed=13, w=24, h=20, textures=2, c0=4, c1=4),
}
LUMA = np.array([0.299, 0.587, 0.114], np.float32)


def model_arrays(m):
    nin, nout = m.nin, m.nout
    return dict(dec_w=np.array(m.dec_w[: nout * nin], np.float32), dec_b=np.array(m.dec_b[:nout], np.float32),
                lo0=np.array(m.lo0[: m.c0], np.float32), hi0=np.array(m.hi0[: m.c0], np.float32),
                lo1=np.array(m.lo1[: m.c1], np.float32), hi1=np.array(m.hi1[: m.c1], np.float32))


def snapshot(s, tag, out):
    s.sync_out()
    for k, v in model_arrays(s.m).items():
        out[f"{tag}.{k}"] = v
    for i in range(s.m.nplanes):
        v0, v1, k0, k1 = s.planes(i)
        out[f"{tag}.v0.{i}"] = v0
        out[f"{tag}.v1.{i}"] = v1
        out[f"{tag}.k0.{i}"] = k0
        out[f"{tag}.k1.{i}"] = k1


def objective(s, k=4):
    r = abi.Objective()
    s.L.ref_objective(s.h, k, s.per_site, C.byref(r))
    return np.array([r.e, r.centre_mse, r.sampled_mse] + list(r.e_plane[: s.m.nplanes]), np.float64)


def make(name, seed, w, h, textures, c0, c1):
    mat = materials.small(seed, w, h, textures=textures, c0=c0, c1=c1)
    m = abi.make_model(mat)
    s = O.RefSession(mat, m, threads=1)
    out = {}
    out["layout"] = np.array([[p[0], p[1], p[2], p[3]] for p in mat.planes], np.int32)
    out["per_site"] = np.array(mat.per_site, np.float64)
    out["shape"] = np.array([textures, c0, c1, 4], np.int32)
    for i, ch in enumerate(mat.chain):
        out[f"src.{i}"] = ch.ravel()
    s.L.ref_init_level0(s.h, O.fptr(LUMA), 0)
    s.L.ref_init_level1(s.h, 0, C.byref(abi.Init1Report()))
    snapshot(s, "s0", out)
    out["s0.objective"] = objective(s)
    s.L.ref_solve_decoder(s.h, 4, s.per_site)
    ne = np.zeros(4096, np.float64)
    n = s.L.ref_normal_equations(s.h, O.dptr(ne))
    out["s0.normal_equations"] = ne[:n]
    snapshot(s, "s1", out)
    s.L.ref_init0_residual_channel(s.h, 0, s.per_site, C.byref(abi.Init0Report()))
    s.L.ref_solve_decoder(s.h, 4, s.per_site)
    snapshot(s, "s2", out)
    out["s2.objective"] = objective(s)
    rep = (abi.PlaneReport * m.nplanes)()
    s.L.ref_solve_block(s.h, 0, 4, 1e-4, 0, rep)
    out["s2.level1.iterations"] = np.array([r.iterations for r in rep], np.int32)
    out["s2.level1.lambda"] = np.array([r.lambda_ for r in rep], np.float64)
    for i in range(m.nplanes):
        ws = s.workspace(i, False)
        for k, v in ws.items():
            out[f"s2.level1.{k}.{i}"] = v
    snapshot(s, "s3", out)
    s.L.ref_solve_block(s.h, 1, 4, 1e-4, 0, rep)
    out["s3.level0.iterations"] = np.array([r.iterations for r in rep], np.int32)
    out["s3.level0.lambda"] = np.array([r.lambda_ for r in rep], np.float64)
    for i in range(m.nplanes):
        ws = s.workspace(i, True)
        for k, v in ws.items():
            out[f"s3.level0.{k}.{i}"] = v
    snapshot(s, "s4", out)
    s.L.ref_grid(s.h, 1, 1)
    s.L.ref_grid(s.h, 3, 1)
    snapshot(s, "s5", out)
    s.L.ref_solve_block(s.h, 0, 4, 1e-4, 4, rep)
    out["s5.level1.moved"] = np.array([r.moved for r in rep], np.int64)
    out["s5.level1.lambda"] = np.array([r.lambda_ for r in rep], np.float64)
    for i in range(m.nplanes):
        ws = s.workspace(i, False)
        out[f"s5.level1.stencil.{i}"] = ws["stencil"]
        out[f"s5.level1.grad.{i}"] = ws["grad"]
    snapshot(s, "s6", out)
    s.L.ref_solve_block(s.h, 1, 4, 1e-4, 4, rep)
    out["s6.level0.moved"] = np.array([r.moved for r in rep], np.int64)
    out["s6.level0.lambda"] = np.array([r.lambda_ for r in rep], np.float64)
    for i in range(m.nplanes):
        ws = s.workspace(i, True)
        out[f"s6.level0.stencil.{i}"] = ws["stencil"]
        out[f"s6.level0.grad.{i}"] = ws["grad"]
    s.L.ref_solve_decoder(s.h, 4, s.per_site)
    snapshot(s, "s7", out)
    out["s7.objective"] = objective(s)
    for i in range(m.nplanes):   # the host mirror the seed pack reads is the device's indices (src/main.cpp:2436)
        s.set_indices(i, k0=s.planes(i)[2])
    s.L.ref_bc_prepare(s.h, 4, 1)
    for i in range(m.nplanes):
        ep, sel = s.bc_state(i)
        out[f"s7.seed.ep.{i}"] = ep
        out[f"s7.seed.sel.{i}"] = sel
        ws = s.workspace(i, True)
        for k, v in ws.items():
            out[f"s7.refine_in.{k}.{i}"] = v
    snapshot(s, "s8", out)
    s.L.ref_bc_refine(s.h, 1, C.byref((abi.BcReport * 1)()))
    for i in range(m.nplanes):
        ep, sel = s.bc_state(i)
        out[f"s8.refined.ep.{i}"] = ep
        out[f"s8.refined.sel.{i}"] = sel
        ws = s.workspace(i, True)
        out[f"s8.refined.x.{i}"] = ws["x"]
    snapshot(s, "s9", out)
    s.close()
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), f"{name}.npz")
    np.savez_compressed(path, **out)
    return path


if __name__ == "__main__":
    for name, spec in CASES.items():
        p = make(name, **spec)
        print(p, os.path.getsize(p))
