"""A device model of one material on the GPU, driven through the C ABI (the host side of the seam, for Python callers).

Mirrors the reference's host usage of its device seam (src/main.cpp:1930-2743): create the device model from a
material's source chain, then call seam functions or the whole encode. Every call goes to libnntc_b200.so.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi, check, lib


class Session:
    def __init__(self, material, model: abi.Model | None = None, from_base: bool = False):
        """from_base: upload the base plane only and build the rest of the source chain on the device."""
        self.material = material
        self.m = model if model is not None else abi.make_model(material)
        self._chain = [np.ascontiguousarray(c, np.float32) for c in material.chain]
        self.per_site = (C.c_double * len(material.per_site))(*material.per_site)
        handle = C.c_void_p()
        if from_base:
            base = self._chain[0].ravel()
            check(lib().nntc_b200_device_create_from_base(C.byref(self.m), base.ctypes.data_as(C.POINTER(C.c_float)),
                                                           C.byref(handle)), "device_create_from_base")
        else:
            check(lib().nntc_b200_device_create(C.byref(self.m), abi.float_ptrs(self._chain), C.byref(handle)),
                  "device_create")
        self.d = handle

    def close(self):
        if self.d:
            lib().nntc_b200_device_destroy(self.d)
            self.d = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- sizes
    def n0(self, i):
        return self.m.w0[i] * self.m.h0[i]

    def n1(self, i):
        return self.m.w1[i] * self.m.h1[i]

    def u8_planes(self, level):
        c = self.m.c0 if level == 0 else self.m.c1
        return [np.zeros((self.n0(i) if level == 0 else self.n1(i)) * c, np.uint8) for i in range(self.m.nplanes)]

    def get_source(self, i):
        a = np.zeros(self.n0(i) * self.m.nout, np.float32)
        check(lib().nntc_b200_probe_source(self.d, i, a.ctypes.data_as(C.POINTER(C.c_float)), a.size), "probe_source")
        return a

    # ---- transfers
    def set_planes(self, i, v0=None, v1=None):
        if v0 is not None:
            a = np.ascontiguousarray(v0, np.float32).ravel()
            check(lib().nntc_b200_level0_upload(self.d, i, a.ctypes.data_as(abi.C.POINTER(C.c_float)), a.size),
                  "level0_upload")
        if v1 is not None:
            a = np.ascontiguousarray(v1, np.float32).ravel()
            check(lib().nntc_b200_level1_upload(self.d, i, a.ctypes.data_as(abi.C.POINTER(C.c_float)), a.size),
                  "level1_upload")

    def get_v0(self, i):
        a = np.zeros(self.n0(i) * self.m.c0, np.float32)
        check(lib().nntc_b200_level0_download_values(self.d, i, a.ctypes.data_as(C.POINTER(C.c_float)), a.size), "")
        return a

    def get_v1(self, i):
        a = np.zeros(self.n1(i) * self.m.c1, np.float32)
        check(lib().nntc_b200_level1_download(self.d, i, a.ctypes.data_as(C.POINTER(C.c_float)), a.size), "")
        return a

    def get_k0(self, i):
        a = np.zeros(self.n0(i) * self.m.c0, np.uint8)
        check(lib().nntc_b200_level0_download(self.d, i, a.ctypes.data_as(C.POINTER(C.c_uint8)), a.size), "")
        return a

    def get_k1(self, i):
        a = np.zeros(self.n1(i) * self.m.c1, np.uint8)
        check(lib().nntc_b200_level1_download_indices(self.d, i, a.ctypes.data_as(C.POINTER(C.c_uint8)), a.size), "")
        return a

    def set_decoder(self, w, b):
        self.m.has_decoder = 1
        w = np.asarray(w, np.float32).ravel()
        b = np.asarray(b, np.float32).ravel()
        for i, x in enumerate(w):
            self.m.dec_w[i] = float(x)
        for i, x in enumerate(b):
            self.m.dec_b[i] = float(x)
        check(lib().nntc_b200_upload_decoder(self.d, C.byref(self.m)), "upload_decoder")

    def decoder(self):
        nin, nout = self.m.nin, self.m.nout
        w = np.array(self.m.dec_w[: nout * nin], np.float32).reshape(nout, nin)
        b = np.array(self.m.dec_b[:nout], np.float32)
        return w, b

    def set_grids(self, lo0=None, hi0=None, lo1=None, hi1=None):
        if lo0 is not None:
            self.m.has_lo0 = 1
            for c in range(self.m.c0):
                self.m.lo0[c], self.m.hi0[c] = float(lo0[c]), float(hi0[c])
        if lo1 is not None:
            self.m.has_lo1 = 1
            for c in range(self.m.c1):
                self.m.lo1[c], self.m.hi1[c] = float(lo1[c]), float(hi1[c])
        check(lib().nntc_b200_upload_grids(self.d, C.byref(self.m)), "upload_grids")

    # ---- seam calls
    def objective(self, k=4):
        r = abi.Objective()
        check(lib().nntc_b200_objective_eval(self.d, C.byref(self.m), k, self.per_site, C.byref(r)), "objective")
        return r

    def solve_decoder(self, k=4):
        ms = C.c_double()
        check(lib().nntc_b200_solve_decoder(self.d, C.byref(self.m), k, self.per_site, C.byref(ms)), "solve_decoder")
        return ms.value

    def normal_equations(self):
        mm = self.m.nin + 1
        n = mm * (mm + 1) // 2 + self.m.nout * mm
        a = np.zeros(n, np.float64)
        check(lib().nntc_b200_probe_normal_equations(self.d, a.ctypes.data_as(C.POINTER(C.c_double)), n), "probe")
        return a

    def block(self, level0: bool, sweeps: int = 0, k=4, ridge=1e-4):
        rep = (abi.PlaneReport * self.m.nplanes)()
        ms = C.c_double()
        L = lib()
        if level0:
            f = L.nntc_b200_sweep_level0_cont_all if sweeps else L.nntc_b200_solve_level0_cont_all
        else:
            f = L.nntc_b200_sweep_level1_all if sweeps else L.nntc_b200_solve_level1_all
        if sweeps:
            check(f(self.d, C.byref(self.m), k, ridge, sweeps, rep, C.byref(ms)), "sweep")
        else:
            check(f(self.d, C.byref(self.m), k, ridge, rep, C.byref(ms)), "solve")
        return list(rep), ms.value

    def workspace(self, i, level0):
        w, h = (self.m.w0[i], self.m.h0[i]) if level0 else (self.m.w1[i], self.m.h1[i])
        c = self.m.c0 if level0 else self.m.c1
        t = w * h
        st = np.zeros(t * 5 * c * c, np.float64)
        g = np.zeros(t * c, np.float64)
        pc = np.zeros(t * c * c, np.float32)
        x = np.zeros(t * c, np.float64)
        prev = np.zeros(t * c, np.float32)
        P = lambda a, ty: a.ctypes.data_as(C.POINTER(ty))
        check(lib().nntc_b200_probe_workspace(self.d, i, 1 if level0 else 0, P(st, C.c_double), P(g, C.c_double),
                                              P(pc, C.c_float), P(x, C.c_double), P(prev, C.c_float)), "workspace")
        return dict(stencil=st, grad=g, precond=pc, x=x, prev=prev)

    def encode(self, args: abi.EncodeArgs | None = None, outputs: bool = False):
        """The whole encode (nntc_b200_encode_on_device). With outputs, also returns the shipped state per plane: level
        0's and level 1's indices and, under bc8, the refined endpoints and selectors - what write_asset takes."""
        if args is None:
            args = abi.EncodeArgs()
            lib().nntc_b200_encode_defaults(C.byref(args))
        r = abi.EncodeResult()
        out = None
        ptrs = (None, None, None, None)
        if outputs:
            m, n = self.m, self.m.nplanes
            blocks = [((m.w0[i] + 3) // 4) * ((m.h0[i] + 3) // 4) for i in range(n)]
            out = dict(k0=[np.zeros(self.n0(i) * m.c0, np.uint8) for i in range(n)],
                       k1=[np.zeros(self.n1(i) * m.c1, np.uint8) for i in range(n)],
                       ep=[np.zeros(b * m.c0 * 2, np.uint8) for b in blocks] if m.l0_bc8 else None,
                       sel=[np.zeros(b * m.c0 * 16, np.uint8) for b in blocks] if m.l0_bc8 else None)
            ptrs = tuple(abi.u8_ptrs(out[k]) if out[k] is not None else None for k in ("k0", "k1", "ep", "sel"))
        check(lib().nntc_b200_encode_on_device(self.d, C.byref(self.m), C.byref(args), self.per_site, C.byref(r),
                                               *ptrs), "encode")
        return (r, out) if outputs else r

    def write_asset(self, prefix: str, outputs: dict, source_size=None, json_path: str | None = None):
        """The encode's result as the reference's asset on disk (nntc_b200_write_asset): PREFIX_lat0*.dds,
        PREFIX_lat1.dds and PREFIX_nntc.json. outputs: what encode(outputs=True) returned."""
        from . import asset
        return asset.write_asset(self.m, prefix, outputs["k1"], k0=outputs["k0"], ep=outputs["ep"],
                                 sel=outputs["sel"], source_size=source_size, json_path=json_path)

    def precision_report(self, k=4):
        """The adjoint form's mixed precision against the FP64 form, from this session's current state (both latents,
        their indices and the decoder are put back afterwards):

        - `decoder`: the decoder solved from the tensor-core normal equations (BF16 hi + lo, FP32 accumulation)
          against the one solved from the FP64 sums, the largest difference of a coefficient relative to the largest
          coefficient of its output row;
        - `level1`, `level0`: one block (b) / block (c') solve with the FP32 stencil against the FP64 stencil, the
          largest difference of the correction relative to the correction's largest entry, over every plane (level 0
          under bc8 only)."""
        L = lib()
        m = self.m
        n = m.nplanes
        v0 = [self.get_v0(i) for i in range(n)]
        v1 = [self.get_v1(i) for i in range(n)]
        k0 = [self.get_k0(i) for i in range(n)]
        k1 = [self.get_k1(i) for i in range(n)]
        saved = abi.Model.from_buffer_copy(m)

        def restore():
            C.memmove(C.addressof(m), C.addressof(saved), C.sizeof(m))
            check(L.nntc_b200_upload_decoder(self.d, C.byref(m)), "decoder")
            check(L.nntc_b200_upload_grids(self.d, C.byref(m)), "grids")
            for i in range(n):
                self.set_planes(i, v0[i], v1[i])
                L.nntc_b200_level0_upload_indices(self.d, i, k0[i].ctypes.data_as(C.POINTER(C.c_uint8)), k0[i].size)
                L.nntc_b200_level1_upload_indices(self.d, i, k1[i].ctypes.data_as(C.POINTER(C.c_uint8)), k1[i].size)

        def options(value):
            for opt in (abi.OPT_MIXED_PRECISION_GRAM, abi.OPT_FP32_STENCIL):
                check(L.nntc_b200_set_option(self.d, opt, value), "option")

        out = {}
        dec = []
        for mixed in (0, 1):
            restore()
            options(mixed)
            m.has_decoder = 0
            self.solve_decoder(k)
            w, b = self.decoder()
            dec.append(np.concatenate([w, b[:, None]], axis=1).astype(np.float64))
        out["decoder"] = float((np.abs(dec[1] - dec[0]) / np.abs(dec[0]).max(axis=1, keepdims=True)).max())
        for level0 in ((False, True) if m.l0_bc8 else (False,)):
            xs = []
            for mixed in (0, 1):
                restore()
                options(mixed)
                self.block(level0, k=k)
                per = []
                for i in range(n):
                    c = m.c0 if level0 else m.c1
                    t = self.n0(i) if level0 else self.n1(i)
                    x = np.zeros(t * c)
                    check(L.nntc_b200_probe_workspace(self.d, i, 1 if level0 else 0, None, None, None,
                                                      x.ctypes.data_as(C.POINTER(C.c_double)), None), "workspace")
                    per.append(x)
                xs.append(per)
            worst = 0.0
            for x64, x32 in zip(xs[0], xs[1]):
                scale = np.abs(x64).max()
                if scale > 0:
                    worst = max(worst, float(np.abs(x32 - x64).max() / scale))
            out["level0" if level0 else "level1"] = worst
        options(0)
        restore()
        return out
