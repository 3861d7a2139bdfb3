"""ctypes mirror of include/nntc_b200.h, and the model POD built from a material.

The structs here are field-for-field copies of the header's; a layout test checks their sizes against the library's
own ``sizeof`` (nntc_b200_abi_sizes) so the two cannot drift apart.
"""
from __future__ import annotations

import ctypes as C

MAX_PLANES = 13
MAX_CHANNELS = 4
MAX_NIN = 24
MAX_NOUT = 18


class Model(C.Structure):
    _fields_ = [
        ("textures", C.c_int), ("nout", C.c_int), ("width", C.c_int), ("height", C.c_int),
        ("c0", C.c_int), ("c1", C.c_int), ("bits0", C.c_int * MAX_CHANNELS), ("bits1", C.c_int),
        ("bc0", C.c_int), ("l0_bc8", C.c_int), ("init0_residual", C.c_int), ("init0_texture", C.c_int),
        ("init0_chain", C.c_int), ("nin", C.c_int), ("nplanes", C.c_int),
        ("w0", C.c_int * MAX_PLANES), ("h0", C.c_int * MAX_PLANES),
        ("w1", C.c_int * MAX_PLANES), ("h1", C.c_int * MAX_PLANES),
        ("cw", C.c_float * MAX_NOUT), ("has_decoder", C.c_int),
        ("dec_w", C.c_float * (MAX_NOUT * MAX_NIN)), ("dec_b", C.c_float * MAX_NOUT),
        ("palette0_len", C.c_int * MAX_CHANNELS), ("palette0", (C.c_float * 16) * MAX_CHANNELS),
        ("has_lo0", C.c_int), ("has_lo1", C.c_int),
        ("lo0", C.c_float * MAX_CHANNELS), ("hi0", C.c_float * MAX_CHANNELS),
        ("lo1", C.c_float * MAX_CHANNELS), ("hi1", C.c_float * MAX_CHANNELS),
    ]


class DeviceInfo(C.Structure):
    _fields_ = [("name", C.c_char * 256), ("major", C.c_int), ("minor", C.c_int), ("error", C.c_char * 512)]


class PlaneReport(C.Structure):
    _fields_ = [
        ("iterations", C.c_int), ("residual", C.c_double), ("lambda_", C.c_double), ("min_diag", C.c_double),
        ("max_diag", C.c_double), ("ms_assemble", C.c_double), ("ms_precond", C.c_double), ("ms_cg", C.c_double),
        ("moved_values", C.c_longlong), ("delta2", C.c_double), ("plane2", C.c_double),
        ("lo", C.c_float * MAX_CHANNELS), ("hi", C.c_float * MAX_CHANNELS), ("quantised", C.c_int),
        ("sweeps", C.c_int), ("moved", C.c_longlong), ("ms_sweeps", C.c_double),
    ]


class Level0Report(C.Structure):
    _fields_ = [("moved", C.c_longlong * 4), ("moved_total", C.c_longlong), ("ms", C.c_double), ("joint", C.c_int),
                ("states", C.c_longlong)]


class Objective(C.Structure):
    _fields_ = [("e", C.c_double), ("e_plane", C.c_double * MAX_PLANES), ("centre_mse", C.c_double),
                ("sampled_mse", C.c_double), ("centre_plane", C.c_double * MAX_PLANES), ("ms", C.c_double)]


class Init1Report(C.Structure):
    _fields_ = [("pca", C.c_int), ("components", C.c_int), ("eigenvalue", C.c_double * 4),
                ("peak", C.c_double * 4), ("total_variance", C.c_double)]


class Init0Report(C.Structure):
    _fields_ = [("eigenvalue", C.c_double), ("total_variance", C.c_double), ("share", C.c_double),
                ("peak", C.c_double), ("divisor", C.c_double), ("dir", C.c_double * MAX_NOUT), ("nout", C.c_int),
                ("texture", C.c_int)]


class BcReport(C.Structure):
    _fields_ = [("pass_", C.c_int), ("blocks", C.c_longlong), ("improved", C.c_longlong), ("delta_e", C.c_double),
                ("ms", C.c_double)]


class EncodeArgs(C.Structure):
    _fields_ = [("k", C.c_int), ("rounds", C.c_int), ("tol", C.c_double), ("q1_start", C.c_int),
                ("q1_sweeps", C.c_int), ("range_pct", C.c_int), ("ridge", C.c_double), ("sweeps", C.c_int),
                ("init_pca", C.c_int), ("bc_refine", C.c_int), ("bc_refine_after", C.c_int), ("bc_outer", C.c_int),
                ("luma", C.c_float * 3), ("form", C.c_int)]


class EncodeResult(C.Structure):
    _fields_ = [("rounds_used", C.c_int), ("stop", C.c_int), ("outer_taken", C.c_int), ("e_init", C.c_double),
                ("e_after_rounds", C.c_double), ("e_ship", C.c_double), ("centre_mse", C.c_double),
                ("sampled_mse", C.c_double), ("psnr", C.c_double * 6), ("ms_a", C.c_double), ("ms_b", C.c_double),
                ("ms_c", C.c_double), ("ms_e", C.c_double), ("ms_pack", C.c_double), ("ms_refine", C.c_double),
                ("ms_total", C.c_double), ("objective_passes", C.c_longlong), ("joint_taken", C.c_int),
                ("e_before_joint", C.c_double), ("e_joint", C.c_double), ("ms_joint", C.c_double)]


# nntc_b200_set_option's options (include/nntc_b200.h, enum nntc_b200_option)
OPT_REFERENCE_SHAPED_ASSEMBLY = 0
OPT_MIXED_PRECISION_GRAM = 1
OPT_ADJOINT_CG = 2
OPT_MIXED_OBJECTIVE = 3
OPT_FP32_STENCIL = 4


def feature_count(c0: int, c1: int) -> int:
    return c1 + c0 + c0 * c1


def make_model(material, l0_bc8: bool = True, init0: str = "residual", bits1: int = 8, cw=None) -> Model:
    """The model a default encode of this material starts from (src/main.cpp:1838-1915)."""
    m = Model()
    T = len(material.textures)
    m.textures = T
    m.nout = 3 * T
    m.width, m.height = material.width, material.height
    m.c0, m.c1 = material.c0, material.c1
    for c in range(MAX_CHANNELS):
        m.bits0[c] = 8 if l0_bc8 else 3
    m.bits1 = bits1
    m.bc0 = 1
    m.l0_bc8 = 1 if l0_bc8 else 0
    m.init0_residual = 1 if init0 in ("residual", "texture") else 0
    m.init0_texture = 1 if init0 == "texture" else 0
    m.init0_chain = 0
    m.nin = feature_count(m.c0, m.c1)
    m.nplanes = len(material.planes)
    for i, (w0, h0, w1, h1) in enumerate(material.planes):
        m.w0[i], m.h0[i], m.w1[i], m.h1[i] = w0, h0, w1, h1
    for c in range(m.nout):
        m.cw[c] = 1.0 if cw is None else float(cw[c])
    m.has_decoder = 0
    if l0_bc8:
        m.has_lo0 = 1
        for c in range(m.c0):
            m.lo0[c], m.hi0[c] = -1.0, 1.0
    else:
        for c in range(m.c0):
            levels = (1 << m.bits0[c]) - 1
            m.palette0_len[c] = levels + 1
            for k in range(levels + 1):
                m.palette0[c][k] = -1.0 + 2.0 * (k / levels)
    m.has_lo1 = 0
    return m


def float_ptrs(arrays):
    """A const float* const* over a list of contiguous float32 arrays (kept alive by the caller)."""
    return (C.POINTER(C.c_float) * len(arrays))(*[a.ctypes.data_as(C.POINTER(C.c_float)) for a in arrays])


def u8_ptrs(arrays):
    return (C.POINTER(C.c_uint8) * len(arrays))(*[a.ctypes.data_as(C.POINTER(C.c_uint8)) for a in arrays])
