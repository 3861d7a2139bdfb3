"""ctypes access to the checkers: this repository's C restatement (_build/libnntc_oracle.so) and the reference's own CPU
arm (_ref/libnntc_ref.so, built from the reference sources by oracle/Makefile).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg, never by the
product.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libnntc_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libnntc_ref.so")
REF_ENCODER = os.path.join(HERE, "_ref", "nntc_encode_cpu")
DROPIN_ENCODER = os.path.join(HERE, "_ref", "nntc_encode_b200")

_PF = C.POINTER(C.c_float)
_PD = C.POINTER(C.c_double)
_PU8 = C.POINTER(C.c_uint8)


class Plane(C.Structure):
    _fields_ = [("w0", C.c_int), ("h0", C.c_int), ("w1", C.c_int), ("h1", C.c_int), ("src", _PF), ("v0", _PF),
                ("v1", _PF)]


class Decoder(C.Structure):
    _fields_ = [("c0", C.c_int), ("c1", C.c_int), ("nin", C.c_int), ("nout", C.c_int), ("k", C.c_int), ("w", _PF),
                ("b", _PF), ("cw", _PF)]


def fptr(a):
    return a.ctypes.data_as(_PF)


def dptr(a):
    return a.ctypes.data_as(_PD)


def u8ptr(a):
    return a.ctypes.data_as(_PU8)


_oracle = None


def oracle():
    """The C restatement, built on first use if it is missing."""
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_SO):
            subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
        L = C.CDLL(ORACLE_SO)
        L.orc_grid_value.restype = C.c_float
        L.orc_grid_value.argtypes = [C.c_float, C.c_float, C.c_int, C.c_int]
        L.orc_grid_index.argtypes = [C.c_float, C.c_float, C.c_int, C.c_float]
        L.orc_objective_plane.argtypes = [C.POINTER(Plane), C.POINTER(Decoder), _PD]
        L.orc_decode_plane.argtypes = [C.POINTER(Plane), C.POINTER(Decoder), _PU8]
        L.orc_normal_equations_plane.argtypes = [C.POINTER(Plane), C.POINTER(Decoder), _PD]
        L.orc_decoder_solve.argtypes = [_PD, C.c_int, C.c_int, _PF, C.c_double, C.c_int, C.c_int, _PF, _PF]
        L.orc_monomials.argtypes = [C.POINTER(Decoder), C.c_int, _PD]
        L.orc_assemble.argtypes = [C.POINTER(Plane), C.POINTER(Decoder), C.c_int, _PD, _PD, _PD]
        L.orc_diag.argtypes = [_PD, C.c_size_t, C.c_int, C.c_double, _PD]
        L.orc_pcg.argtypes = [_PD, _PD, C.c_int, C.c_int, C.c_int, C.c_double, _PD, _PD]
        L.orc_quant_sweeps.restype = C.c_longlong
        L.orc_quant_sweeps.argtypes = [_PD, _PD, _PF, C.c_int, C.c_int, C.c_int, C.c_double, _PF, _PF, C.c_int,
                                       C.c_int, _PD, _PF, _PU8]
        L.orc_bc_seed.argtypes = [_PU8, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int), _PU8, _PU8]
        L.orc_bc_decode.argtypes = [_PU8, _PU8, _PF, _PF, C.c_int, C.c_int, C.c_int, _PF, _PF, _PU8, _PD]
        L.orc_bc_refine_colour.restype = C.c_double
        L.orc_bc_refine_colour.argtypes = [_PD, _PD, _PF, _PF, _PF, C.c_int, C.c_int, C.c_int, C.c_int, _PU8, _PU8,
                                           _PD, _PF, _PU8, C.POINTER(C.c_longlong)]
        L.orc_init_level1_box.argtypes = [_PF, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _PF]
        L.orc_residual.argtypes = [C.POINTER(Plane), C.POINTER(Decoder), _PF]
        _oracle = L
    return _oracle


class State:
    """Plane arrays and a decoder in the oracle's POD form (the arrays are kept alive here)."""

    def __init__(self, planes, c0, c1, nout, k, w, b, cw):
        self.arrays = []
        self.planes = []
        for (w0, h0, w1, h1, src, v0, v1) in planes:
            src = np.ascontiguousarray(src, np.float32).ravel()
            v0 = np.ascontiguousarray(v0, np.float32).ravel().copy()
            v1 = np.ascontiguousarray(v1, np.float32).ravel().copy()
            self.arrays += [src, v0, v1]
            self.planes.append((Plane(w0, h0, w1, h1, fptr(src), fptr(v0), fptr(v1)), src, v0, v1))
        self.w = np.ascontiguousarray(w, np.float32).ravel()
        self.b = np.ascontiguousarray(b, np.float32).ravel()
        self.cw = np.ascontiguousarray(cw, np.float32).ravel()
        nin = c1 + c0 + c0 * c1
        self.dec = Decoder(c0, c1, nin, nout, k, fptr(self.w), fptr(self.b), fptr(self.cw))
        self.c0, self.c1, self.nin, self.nout, self.k = c0, c1, nin, nout, k

    def plane(self, i):
        return self.planes[i][0]

    def v0(self, i):
        return self.planes[i][2]

    def v1(self, i):
        return self.planes[i][3]


class RefSession:
    """One model on the reference's own CPU arm, seam call by seam call (oracle/ref_shim.cpp)."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not os.path.exists(REF_SO):
                raise FileNotFoundError(f"{REF_SO} is not built (oracle/Makefile `ref`, needs the reference sources)")
            L = C.CDLL(REF_SO)
            L.ref_open.restype = C.c_void_p
            L.ref_open.argtypes = [C.c_void_p, C.POINTER(_PF), C.c_int]
            for n in ("ref_close",):
                getattr(L, n).argtypes = [C.c_void_p]
            L.ref_sync_in.argtypes = [C.c_void_p, C.c_void_p]
            L.ref_sync_out.argtypes = [C.c_void_p, C.c_void_p]
            L.ref_set_planes.argtypes = [C.c_void_p, C.c_int, _PF, _PF]
            L.ref_set_indices.argtypes = [C.c_void_p, C.c_int, _PU8, _PU8]
            L.ref_get_planes.argtypes = [C.c_void_p, C.c_int, _PF, _PF, _PU8, _PU8]
            L.ref_get_host_indices.argtypes = [C.c_void_p, C.c_int, _PU8, _PU8]
            L.ref_objective.argtypes = [C.c_void_p, C.c_int, _PD, C.c_void_p]
            L.ref_decode.argtypes = [C.c_void_p, C.c_int, _PU8]
            L.ref_solve_decoder.argtypes = [C.c_void_p, C.c_int, _PD]
            L.ref_normal_equations.argtypes = [C.c_void_p, _PD]
            L.ref_solve_block.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_int, C.c_void_p]
            L.ref_assemble_for_refine.argtypes = [C.c_void_p, C.c_int]
            L.ref_monomials.argtypes = [C.c_void_p, C.c_int, _PD]
            L.ref_workspace.argtypes = [C.c_void_p, C.c_int, C.c_int, _PD, _PD, _PF, _PD, _PF]
            L.ref_set_workspace0.argtypes = [C.c_void_p, C.c_int, _PD, _PD, _PD, _PF]
            L.ref_bc_prepare.argtypes = [C.c_void_p, C.c_int, C.c_int]
            L.ref_bc_refine.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
            L.ref_bc_state.argtypes = [C.c_void_p, C.c_int, _PU8, _PU8]
            L.ref_bc_set_state.argtypes = [C.c_void_p, C.c_int, _PU8, _PU8]
            L.ref_pack_seed.argtypes = [C.c_void_p, C.c_int, _PU8, _PU8]
            L.ref_init_level0.argtypes = [C.c_void_p, _PF, C.c_int]
            L.ref_init_level1.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
            L.ref_init0_residual_channel.argtypes = [C.c_void_p, C.c_int, _PD, C.c_void_p]
            L.ref_grid.argtypes = [C.c_void_p, C.c_int, C.c_int]
            L.ref_solve_level0_palette.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p]
            cls._lib = L
        return cls._lib

    def __init__(self, material, model, threads=1):
        self.L = self.lib()
        self.m = model
        self.material = material
        self._chain = [np.ascontiguousarray(c, np.float32) for c in material.chain]
        arr = (_PF * len(self._chain))(*[fptr(c) for c in self._chain])
        self.h = self.L.ref_open(C.byref(model), arr, threads)
        self.per_site = (C.c_double * len(material.per_site))(*material.per_site)

    def close(self):
        if self.h:
            self.L.ref_close(self.h)
            self.h = None

    def n0(self, i):
        return self.m.w0[i] * self.m.h0[i]

    def n1(self, i):
        return self.m.w1[i] * self.m.h1[i]

    def sync_in(self):
        self.L.ref_sync_in(self.h, C.byref(self.m))

    def sync_out(self):
        self.L.ref_sync_out(self.h, C.byref(self.m))

    def planes(self, i):
        v0 = np.zeros(self.n0(i) * self.m.c0, np.float32)
        v1 = np.zeros(self.n1(i) * self.m.c1, np.float32)
        k0 = np.zeros(self.n0(i) * self.m.c0, np.uint8)
        k1 = np.zeros(self.n1(i) * self.m.c1, np.uint8)
        self.L.ref_get_planes(self.h, i, fptr(v0), fptr(v1), u8ptr(k0), u8ptr(k1))
        return v0, v1, k0, k1

    def set_planes(self, i, v0=None, v1=None):
        a0 = None if v0 is None else np.ascontiguousarray(v0, np.float32)
        a1 = None if v1 is None else np.ascontiguousarray(v1, np.float32)
        self.L.ref_set_planes(self.h, i, None if a0 is None else fptr(a0), None if a1 is None else fptr(a1))

    def set_indices(self, i, k0=None, k1=None):
        a0 = None if k0 is None else np.ascontiguousarray(k0, np.uint8)
        a1 = None if k1 is None else np.ascontiguousarray(k1, np.uint8)
        self.L.ref_set_indices(self.h, i, None if a0 is None else u8ptr(a0), None if a1 is None else u8ptr(a1))

    def workspace(self, i, level0):
        w, h = (self.m.w0[i], self.m.h0[i]) if level0 else (self.m.w1[i], self.m.h1[i])
        c = self.m.c0 if level0 else self.m.c1
        t = w * h
        out = dict(stencil=np.zeros(t * 5 * c * c), grad=np.zeros(t * c), precond=np.zeros(t * c * c, np.float32),
                   x=np.zeros(t * c), prev=np.zeros(t * c, np.float32))
        self.L.ref_workspace(self.h, i, 1 if level0 else 0, dptr(out["stencil"]), dptr(out["grad"]),
                             fptr(out["precond"]), dptr(out["x"]), fptr(out["prev"]))
        return out

    def bc_state(self, i):
        blocks = ((self.m.w0[i] + 3) // 4) * ((self.m.h0[i] + 3) // 4)
        ep = np.zeros(blocks * self.m.c0 * 2, np.uint8)
        sel = np.zeros(blocks * self.m.c0 * 16, np.uint8)
        self.L.ref_bc_state(self.h, i, u8ptr(ep), u8ptr(sel))
        return ep, sel
