"""nntc_b200: the NNTC encoder's hot path for B200 (sm_100a), behind the reference's device-seam interface.

The product is ``libnntc_b200.so`` (C ABI, include/nntc_b200.h). This package only loads it and declares its
prototypes for Python callers (tests, the benchmark); there is no Python or CPU implementation of any kernel, and
``lib()`` raises if the library was not built.
"""
from __future__ import annotations

import ctypes as C
import os

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY = os.path.join(HERE, "libnntc_b200.so")

_lib = None

_P = C.c_void_p
_I = C.c_int
_D = C.c_double
_S = C.c_size_t
_PF = C.POINTER(C.c_float)
_PD = C.POINTER(C.c_double)
_PU8 = C.POINTER(C.c_uint8)
_PPF = C.POINTER(_PF)
_PPU8 = C.POINTER(_PU8)
_PPD = C.POINTER(_PD)
_M = C.POINTER(abi.Model)

PROTOTYPES = {
    "nntc_b200_last_error": (C.c_char_p, []),
    "nntc_b200_version": (_I, []),
    "nntc_b200_abi_sizes": (_I, [C.POINTER(_S), _I]),
    "nntc_b200_device_select": (_I, [_I, C.POINTER(abi.DeviceInfo)]),
    "nntc_b200_device_create": (_I, [_M, _PPF, C.POINTER(_P)]),
    "nntc_b200_device_create_from_base": (_I, [_M, _PF, C.POINTER(_P)]),
    "nntc_b200_device_destroy": (None, [_P]),
    "nntc_b200_device_memory": (_S, [_P]),
    "nntc_b200_init_level0": (_I, [_P, _M, _PF, _I, _PPU8]),
    "nntc_b200_init_level1": (_I, [_P, _M, _I, C.POINTER(abi.Init1Report), _PPU8]),
    "nntc_b200_init0_residual_channel": (_I, [_P, _M, _I, _PD, C.POINTER(abi.Init0Report), _PPU8]),
    "nntc_b200_quantise_level1": (_I, [_P, _M, _I, _PPU8]),
    "nntc_b200_freeze_level1_grid": (_I, [_P, _M, _I, _PPU8]),
    "nntc_b200_quantise_level0": (_I, [_P, _M, _I, _PPU8]),
    "nntc_b200_freeze_level0_grid": (_I, [_P, _M, _I, _PPU8]),
    "nntc_b200_snap_level0_on_grid": (_I, [_P, _M, _PPU8]),
    "nntc_b200_stencil_monomials": (_I, [_I]),
    "nntc_b200_solve_decoder": (_I, [_P, _M, _I, _PD, _PD]),
    "nntc_b200_decoder_ridge_tally": (None, [C.POINTER(C.c_longlong)]),
    "nntc_b200_solve_level1_all": (_I, [_P, _M, _I, _D, C.POINTER(abi.PlaneReport), _PD]),
    "nntc_b200_sweep_level1_all": (_I, [_P, _M, _I, _D, _I, C.POINTER(abi.PlaneReport), _PD]),
    "nntc_b200_solve_level0_cont_all": (_I, [_P, _M, _I, _D, C.POINTER(abi.PlaneReport), _PD]),
    "nntc_b200_sweep_level0_cont_all": (_I, [_P, _M, _I, _D, _I, C.POINTER(abi.PlaneReport), _PD]),
    "nntc_b200_assemble_level0_for_refine": (_I, [_P, _M, _I, _PD]),
    "nntc_b200_level1_download_indices": (_I, [_P, _I, _PU8, _S]),
    "nntc_b200_level1_upload": (_I, [_P, _I, _PF, _S]),
    "nntc_b200_level1_upload_indices": (_I, [_P, _I, _PU8, _S]),
    "nntc_b200_level0_upload_indices": (_I, [_P, _I, _PU8, _S]),
    "nntc_b200_upload_decoder": (_I, [_P, _M]),
    "nntc_b200_upload_grids": (_I, [_P, _M]),
    "nntc_b200_level1_download": (_I, [_P, _I, _PF, _S]),
    "nntc_b200_level1_delta": (_I, [_P, _I, _PD, _S]),
    "nntc_b200_level1_poke": (_I, [_P, _I, _S, C.c_float]),
    "nntc_b200_level1_range": (_I, [_P, _I, _PF, _PF]),
    "nntc_b200_solve_level1_dense_host": (_I, [_P, _M, _I, _I, _D, _PF, _S, _PD, _I]),
    "nntc_b200_level0_download": (_I, [_P, _I, _PU8, _S]),
    "nntc_b200_level0_upload": (_I, [_P, _I, _PF, _S]),
    "nntc_b200_level0_download_values": (_I, [_P, _I, _PF, _S]),
    "nntc_b200_solve_level0_all": (_I, [_P, _M, _I, _I, C.POINTER(abi.Level0Report), _PD]),
    "nntc_b200_decode_plane": (_I, [_P, _M, _I, _PU8, _S]),
    "nntc_b200_objective_eval": (_I, [_P, _M, _I, _PD, C.POINTER(abi.Objective)]),
    "nntc_b200_objective_total_ms": (_D, []),
    "nntc_b200_objective_passes": (C.c_longlong, []),
    "nntc_b200_objective_check_host": (_I, [_P, _M, _I, _PD, C.POINTER(abi.Objective)]),
    "nntc_b200_bc_pack_prepare": (_I, [_P, _M, _I, _I, _PPU8, _PD]),
    "nntc_b200_bc_refine": (_I, [_P, _M, _I, C.POINTER(abi.BcReport), _PD]),
    "nntc_b200_bc_state_save": (_I, [_P, _M, _PPU8, _PPU8]),
    "nntc_b200_bc_state_restore": (_I, [_P, _M, _PPU8, _PPU8]),
    "nntc_b200_bc_pack_blocks": (_I, [_M, _I, _PU8, _PU8, _PU8, _PPU8, _PD, C.POINTER(_S)]),
    "nntc_b200_write_asset": (_I, [_M, _PPU8, _PPU8, _PPU8, _PPU8, _I, _I, C.c_char_p, C.c_char_p, C.POINTER(_S)]),
    "nntc_b200_encode_defaults": (None, [C.POINTER(abi.EncodeArgs)]),
    "nntc_b200_encode_on_device": (_I, [_P, _M, C.POINTER(abi.EncodeArgs), _PD, C.POINTER(abi.EncodeResult),
                                        _PPU8, _PPU8, _PPU8, _PPU8]),
    "nntc_b200_set_option": (_I, [_P, _I, _I]),
    "nntc_b200_objective_gradient": (_I, [_P, _M, _I, _PD, _PPD, _PPD, _PD]),
    "nntc_b200_measure_fma_peaks": (_I, [_PD, _PD]),
    "nntc_b200_probe_normal_equations": (_I, [_P, _PD, _S]),
    "nntc_b200_probe_objective_with_normal_equations": (_I, [_P, _P, _I, _PD, _P]),
    "nntc_b200_probe_workspace": (_I, [_P, _I, _I, _PD, _PD, _PF, _PD, _PF]),
    "nntc_b200_probe_monomials": (_I, [_P, _I, _PD, _S]),
    "nntc_b200_probe_source": (_I, [_P, _I, _PF, _S]),
    "nntc_b200_probe_jtj_level1": (_I, [_P, _I, _I, _PD, _PD, _S]),
    "nntc_b200_probe_jtj_level0": (_I, [_P, _I, _I, _PD, _PD, _S]),
}


class NntcError(RuntimeError):
    pass


def lib():
    """The loaded C ABI library. Raises if it was not built: there is no other implementation to fall back on."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBRARY):
            raise NntcError(f"{LIBRARY} is missing: build it with `make -C {HERE}` (needs nvcc for sm_100a)")
        handle = C.CDLL(LIBRARY)
        for name, (res, args) in PROTOTYPES.items():
            f = getattr(handle, name)
            f.restype = res
            f.argtypes = args
        _lib = handle
    return _lib


def check(status: int, what: str = "") -> None:
    if status != 0:
        msg = lib().nntc_b200_last_error().decode(errors="replace")
        raise NntcError(f"{what}: status {status}: {msg}")

PROTOTYPES.update({
    "nntc_b200_objective_plane_noalloc": (_I, [_P, _I, _I, _I, _P, _I, _I, _I, _P, _I, _P, _P, _P, _I, _I, _P, _P]),
    "nntc_b200_launch_count": (C.c_longlong, []),
    "nntc_b200_kernel_timing": (_I, [_P, _I]),
    "nntc_b200_kernel_stats": (_I, [_P, _I, C.POINTER(C.c_longlong), _PD, _I]),
})

KERNELS = ["objective", "normal_equations", "assemble_level1", "assemble_level0", "cg_matvec", "quant_sweep",
           "bc_refine"]
