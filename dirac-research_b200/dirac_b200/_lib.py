"""ctypes binding of libdiracgpu.so, the sm_100a C ABI declared in include/dirac_gpu.h.

The library is built in place (``make -C dirac-research_b200``).  Importing this module
fails loudly when it is missing: there is no CPU fallback for any entry point.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "libdiracgpu.so")

DGPU_OK = 0
DGPU_ERR_SIZE = -2
ERRORS = {
    -1: "DGPU_ERR_ARG",
    -2: "DGPU_ERR_SIZE",
    -3: "DGPU_ERR_CUDA",
    -4: "DGPU_ERR_NOMEM",
    -5: "DGPU_ERR_DEVICE",
}


class DgpuError(RuntimeError):
    """A libdiracgpu entry point returned a negative status."""

    def __init__(self, code, what=""):
        self.code = code
        name = ERRORS.get(code, str(code))
        detail = ""
        if code == -3 and _lib is not None:
            detail = " (" + _lib.dgpu_last_error().decode(errors="replace") + ")"
        super().__init__(f"{what}: {name}{detail}")


_lib = None

c_int = ctypes.c_int
c_void_p = ctypes.c_void_p
c_size_t = ctypes.c_size_t
P_int = ctypes.POINTER(ctypes.c_int)
P_void = ctypes.POINTER(ctypes.c_void_p)

# name -> (restype, argtypes); mirrors include/dirac_gpu.h
SIGNATURES = {
    "dgpu_version": (ctypes.c_char_p, []),
    "dgpu_device_check": (c_int, []),
    "dgpu_last_error": (ctypes.c_char_p, []),
    "dgpu_launch_count": (ctypes.c_ulonglong, []),
    "dgpu_dwt_scratch_bytes": (c_size_t, [c_int, c_int, c_int]),
    "dgpu_wavelet_transform": (
        c_int,
        [c_int, c_int, c_int, c_void_p, c_int, c_int, c_int, c_void_p, c_int, c_int, c_int,
         c_void_p, c_size_t, c_void_p],
    ),
    "dgpu_wavelet_transform_batch": (
        c_int,
        [c_int, c_int, P_int, P_int, P_void, P_int, P_int, P_int, P_void, P_int, P_int, P_int,
         c_void_p, c_size_t, c_void_p],
    ),
    "dgpu_wavelet_transform_static": (
        c_int,
        [c_int, c_int, c_int, c_void_p, c_int, c_int, c_int, c_void_p, c_int, c_int, c_int, c_void_p],
    ),
    "dgpu_wavelet_transform_host": (
        c_int,
        [c_int, c_int, c_int, c_void_p, c_int, c_int, c_int, c_void_p, c_int, c_int, c_int],
    ),
    "dgpu_upconvert": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_void_p, c_int, c_void_p]),
    "dgpu_upconvert_batch": (c_int, [c_int, P_void, P_int, P_int, P_int, P_int, P_void, P_int, c_void_p]),
    "dgpu_downconvert": (c_int, [c_void_p, c_int, c_int, c_int, c_void_p, c_int, c_void_p]),
    "dgpu_downconvert_batch": (c_int, [c_int, P_void, P_int, P_int, P_int, P_void, P_int, c_void_p]),
    "dgpu_clip": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_void_p]),
    "dgpu_cwm_filter": (c_int, [c_void_p, c_int, c_void_p, c_int, c_int, c_int, c_int, c_void_p]),
    "dgpu_rect_lp_filter": (c_int, [c_void_p, c_int, c_int, c_int, ctypes.c_float, c_int, c_void_p, c_void_p]),
    "dgpu_diag_lp_filter": (c_int, [c_void_p, c_int, c_int, c_int, ctypes.c_float, c_int, c_void_p, c_void_p]),
    "dgpu_motion_compensate": (
        c_int,
        [c_int, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
         P_void, P_int, P_void, P_void, c_int, c_int, c_void_p],
    ),
    "dgpu_motion_compensate_weighted": (
        c_int,
        [c_int, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
         P_void, P_int, P_void, P_void, c_int, c_int, c_int, c_int, c_int, c_void_p],
    ),
    "dgpu_me_depth": (c_int, [c_int, c_int]),
    "dgpu_measure_int_rate": (c_int, [c_void_p]),
    "dgpu_me_profile": (c_int, [c_int, c_void_p, c_void_p]),
    "dgpu_me_set_occupancy": (c_int, [c_int]),
    "dgpu_me_set_unit_lifetime": (c_int, [c_int]),
    "dgpu_set_blocking_waits": (c_int, [c_int]),
    "dgpu_debug_wavefront": (c_int, [c_int, ctypes.c_longlong, c_void_p, c_void_p, c_void_p, c_void_p]),
    "dgpu_me_workspace_bytes": (c_size_t, [c_int, c_int, c_int, c_void_p, c_int]),
    "dgpu_me_batch_workspace_bytes": (c_size_t, [c_int, c_int, c_int, c_void_p, c_int, c_int, P_int, c_int]),
    "dgpu_motion_estimate_batch": (
        c_int,
        [c_int, c_int, c_int, c_void_p, c_int, c_int, P_void, c_int, P_int, P_int, P_int, c_void_p, c_int,
         P_void, P_void, P_void, P_void, P_void, P_void, c_void_p, c_size_t, c_void_p],
    ),
    "dgpu_motion_estimate": (
        c_int,
        [c_int, c_int, c_int, c_void_p, c_int, P_void, P_void, P_void, c_int, ctypes.c_float, c_int,
         c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_size_t, c_void_p],
    ),
    "dgpu_quant_factor4": (c_int, [c_int]),
    "dgpu_band_weights": (c_int, [c_int, c_int, c_int, c_int, c_int, c_int, ctypes.c_float, ctypes.c_float, c_int,
                                  c_void_p]),
    "dgpu_code_blocks": (c_int, [c_int, c_int, c_int, c_int, c_void_p]),
    "dgpu_code_residue_workspace_bytes": (c_size_t, [c_int, P_int, P_int, P_int, P_int, P_int]),
    "dgpu_code_residue_batch": (
        c_int,
        [c_int, P_int, P_int, P_void, P_int, P_int, c_void_p, c_void_p, c_void_p, P_int, P_int, P_int, P_int,
         c_void_p, P_void, c_void_p, c_size_t, c_void_p],
    ),
    "dgpu_encoder_device_bytes": (c_size_t, [c_void_p, c_int]),
    "dgpu_encoder_create": (c_int, [c_void_p, c_int, c_void_p, P_void]),
    "dgpu_encoder_destroy": (c_int, [c_void_p]),
    "dgpu_encoder_reset": (c_int, [c_void_p]),
    "dgpu_encoder_profile": (c_int, [c_void_p, c_int, c_void_p, c_void_p]),
    "dgpu_encoder_load": (c_int, [c_void_p, P_void, c_int]),
    "dgpu_encoder_end_sequence": (c_int, [c_void_p]),
    "dgpu_encoder_code_next": (c_int, [c_void_p, c_void_p, c_void_p]),
    "dgpu_encoder_code_next_adaptive": (c_int, [c_void_p, c_void_p, c_void_p]),
    "dgpu_encoder_prepare_next": (c_int, [c_void_p, c_void_p]),
    "dgpu_encoder_finish_next": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "dgpu_encoder_code_adaptive": (c_int, [c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_size_t, c_void_p,
                                           c_void_p, c_void_p, c_void_p]),
    "dgpu_encoder_adaptive_data": (c_int, [c_void_p, c_void_p, c_size_t, c_void_p]),
    "dgpu_encoder_item_bytes": (c_size_t, [c_void_p, c_int, c_int, c_int]),
    "dgpu_encoder_read": (c_int, [c_void_p, c_int, c_int, c_int, c_void_p, c_size_t, c_int]),
    "dgpu_batch_device_bytes": (c_size_t, [c_int, c_void_p, c_void_p]),
    "dgpu_batch_create": (c_int, [c_int, c_void_p, c_void_p, c_void_p, P_void]),
    "dgpu_batch_destroy": (c_int, [c_void_p]),
    "dgpu_batch_planes": (c_int, [c_void_p, c_int, P_void]),
    "dgpu_batch_load": (c_int, [c_void_p, c_int, P_void, c_int]),
    "dgpu_batch_run": (c_int, [c_void_p]),
    "dgpu_batch_stage_times": (c_int, [c_void_p, c_void_p]),
    "dgpu_batch_item_bytes": (c_size_t, [c_void_p, c_int, c_int, c_int]),
    "dgpu_batch_read": (c_int, [c_void_p, c_int, c_int, c_int, c_void_p, c_size_t, c_int]),
    "dgpu_encoder_group_device_bytes": (c_size_t, [P_void, c_int]),
    "dgpu_encoder_group_create": (c_int, [P_void, c_int, P_void]),
    "dgpu_encoder_group_destroy": (c_int, [c_void_p]),
    "dgpu_encoder_group_estimate": (c_int, [c_void_p, P_int]),
    "dgpu_encoders_estimate": (c_int, [P_void, c_int, c_void_p, c_size_t, c_void_p, P_int]),
    "dgpu_dequantise_batch": (
        c_int, [c_int, P_int, P_int, P_void, P_void, P_int, P_int, P_int, P_int, P_int, c_void_p, c_void_p],
    ),
    "dgpu_dequantise_batch16": (
        c_int, [c_int, P_int, P_int, P_void, P_void, P_int, P_int, P_int, P_int, P_int, c_void_p, c_void_p],
    ),
    "dgpu_decoder_device_bytes": (c_size_t, [c_void_p, c_int]),
    "dgpu_decoder_create": (c_int, [c_void_p, c_int, c_void_p, P_void]),
    "dgpu_decoder_destroy": (c_int, [c_void_p]),
    "dgpu_decoder_decode": (c_int, [c_void_p, c_void_p]),
    "dgpu_decoder_release": (c_int, [c_void_p, c_int]),
    "dgpu_decoder_item_bytes": (c_size_t, [c_void_p, c_int, c_int, c_int]),
    "dgpu_decoder_read": (c_int, [c_void_p, c_int, c_int, c_int, c_void_p, c_size_t, c_int]),
    "dgpu_code_bands_host": (
        c_int, [c_int, P_int, P_int, P_void, P_int, P_int, P_int, P_int, P_int, c_void_p, c_void_p, c_size_t, P_int],
    ),
    "dgpu_code_bands_host16": (
        c_int, [c_int, P_int, P_int, P_void, P_int, P_int, P_int, P_int, P_int, c_void_p, c_void_p, c_size_t, P_int],
    ),
    "dgpu_code_bands_vlc_host": (
        c_int,
        [c_int, P_int, P_int, P_void, P_int, P_int, P_int, P_int, P_int, c_void_p, c_void_p, c_size_t, P_int, c_void_p],
    ),
    "dgpu_decode_bands_host": (
        c_int, [c_int, P_int, P_int, P_int, P_int, P_int, c_void_p, c_size_t, P_int, c_int, P_void, c_void_p],
    ),
    "dgpu_code_bands_vlc": (c_int, [c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                    c_void_p, c_size_t, c_void_p, c_void_p, c_void_p, c_size_t, c_void_p]),
    "dgpu_entropy_init": (c_int, [c_int, c_void_p]),
    "dgpu_entropy_factors": (c_int, [c_int, c_void_p, c_int, c_int, c_void_p]),
    "dgpu_entropy_update": (c_int, [c_int, c_void_p, c_int, c_int, c_int, P_int, P_int, P_int]),
}


class BlockParams(ctypes.Structure):
    """dgpu_block_params: luma overlapped-block parameters and superblock counts."""

    _fields_ = [(n, ctypes.c_int) for n in
                ("precision", "xblen", "yblen", "xbsep", "ybsep", "xnum_sb", "ynum_sb")]


def load(path=LIB_PATH):
    """Load the library (once) and declare every entry point's signature."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(
            f"{path} is missing: build it with `make -C dirac-research_b200` "
            "(the Dirac GPU path has no CPU fallback)"
        )
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc, what):
    if rc != DGPU_OK:
        raise DgpuError(rc, what)
    return rc


def int_array(values):
    return (ctypes.c_int * len(values))(*values)


def ptr_array(values):
    return (ctypes.c_void_p * len(values))(*values)
