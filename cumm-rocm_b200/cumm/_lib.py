"""ctypes binding of libcumm_b200.so (C ABI declared in include/cumm_b200.h).

The structures below mirror ``sc_conv_params`` / ``sc_gemm_params`` field by
field.  Status codes map to the reference's exception types
(include/tensorview/core/common.h:102-183): SC_INVALID_ARG -> ValueError,
everything else -> RuntimeError.
"""
import ctypes
import os
import threading
from pathlib import Path

SC_OK, SC_INVALID_ARG, SC_RUNTIME, SC_CUDA, SC_DEVICE = 0, 1, 2, 3, 4
SC_ALGO_TCGEN05, SC_ALGO_SIMT = 0, 1
SC_FLAG_SYNC_CHECK = 1

_LIB_PATH = Path(__file__).resolve().parent / "libcumm_b200.so"

EXPORTS = (
    "sc_conv_implicit_gemm", "sc_conv_workspace_size", "sc_gemm_matmul", "sc_gemm_workspace_size",
    "sc_pairs_workspace_size", "sc_build_subm_pairs", "sc_build_conv_outputs",
    "sc_build_conv_pairs", "sc_sort_masks_split", "sc_sort_workspace_size",
    "sc_check_device_error", "sc_last_error", "sc_version", "sc_sort_indices",
    "sc_conv_wgrad_static_scratch", "sc_gather_rows", "sc_scatter_add_rows",
    "sc_tile_order", "sc_tile_order_workspace_size",
)

c_i32, c_i64, c_u32, c_f32, c_vp = (ctypes.c_int32, ctypes.c_int64, ctypes.c_uint32,
                                    ctypes.c_float, ctypes.c_void_p)


class ConvParamsC(ctypes.Structure):
    _fields_ = [
        ("op_type", c_i32), ("algo", c_i32), ("dtype_input", c_i32), ("dtype_weight", c_i32),
        ("dtype_output", c_i32), ("tile_m", c_i32), ("tile_k", c_i32), ("kv", c_i32),
        ("n_in", c_i64), ("n_out", c_i64), ("C", c_i64), ("K", c_i64), ("N", c_i64),
        ("input", c_vp), ("weight", c_vp), ("output", c_vp), ("indices", c_vp),
        ("mask", c_vp), ("mask_count", c_i64), ("mask_argsort", c_vp),
        ("mask_output", c_vp), ("mask_output_count", c_i64), ("mask_filter", c_u32),
        ("reverse_mask", c_i32), ("mask_width", c_i32), ("alpha", c_f32), ("beta", c_f32),
        ("act_alpha", c_f32), ("act_beta", c_f32), ("act_type", c_i32), ("bias", c_vp),
        ("output_add", c_vp), ("scale", c_vp), ("split_k_slices", c_i32), ("flags", c_i32),
        ("workspace", c_vp), ("workspace_bytes", c_i64), ("stream", c_vp),
        ("indices_sorted", c_vp), ("tile_n", c_i32), ("tile_order", c_vp),
    ]


class GemmParamsC(ctypes.Structure):
    _fields_ = [
        ("dtype_a", c_i32), ("dtype_b", c_i32), ("dtype_c", c_i32), ("trans_a", c_i32),
        ("trans_b", c_i32), ("trans_c", c_i32), ("shuffle_type", c_i32), ("algo", c_i32),
        ("m", c_i64), ("n", c_i64), ("k", c_i64), ("a", c_vp), ("lda", c_i64), ("b", c_vp),
        ("ldb", c_i64), ("c", c_vp), ("ldc", c_i64), ("d", c_vp), ("ldd", c_i64),
        ("a_inds", c_vp), ("b_inds", c_vp), ("c_inds", c_vp), ("a_rows", c_i64),
        ("b_rows", c_i64), ("alpha", c_f32), ("beta", c_f32), ("act_alpha", c_f32),
        ("act_beta", c_f32), ("act_type", c_i32), ("split_k_slices", c_i32), ("flags", c_i32),
        ("workspace", c_vp), ("workspace_bytes", c_i64), ("stream", c_vp),
    ]


_lock = threading.Lock()
_lib = None


def lib_path() -> Path:
    return _LIB_PATH


def load() -> ctypes.CDLL:
    """Loads the library (once).  Raises RuntimeError if it is missing."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not _LIB_PATH.exists():
            raise RuntimeError(
                f"{_LIB_PATH} not found: build it with `python cumm-rocm_b200/build.py` "
                "(there is no CPU fallback)")
        lib = ctypes.CDLL(str(_LIB_PATH))
        P = ctypes.POINTER
        lib.sc_conv_implicit_gemm.argtypes = [P(ConvParamsC)]
        lib.sc_conv_workspace_size.argtypes = [P(ConvParamsC), P(c_i64)]
        lib.sc_gemm_matmul.argtypes = [P(GemmParamsC)]
        lib.sc_gemm_workspace_size.argtypes = [P(GemmParamsC), P(c_i64)]
        lib.sc_pairs_workspace_size.argtypes = [c_i64, c_i32, c_i32, P(c_i64)]
        lib.sc_build_subm_pairs.argtypes = [c_vp, c_i64, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp,
                                            c_vp, c_i64, c_vp]
        lib.sc_build_conv_outputs.argtypes = [c_vp, c_i64, c_i32, c_vp, c_vp, c_vp, c_vp, c_vp,
                                              c_vp, P(c_i64), c_vp, c_i64, c_vp]
        lib.sc_build_conv_pairs.argtypes = [c_vp, c_i64, c_i32, c_vp, c_vp, c_vp, c_vp, c_vp,
                                            c_i64, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_i64,
                                            c_vp]
        lib.sc_sort_masks_split.argtypes = [c_vp, c_i64, c_u32, c_vp, c_vp, c_i64, c_vp]
        lib.sc_sort_workspace_size.argtypes = [c_i64, P(c_i64)]
        lib.sc_check_device_error.argtypes = [c_vp, P(c_i32)]
        lib.sc_sort_indices.argtypes = [c_vp, c_i32, c_i64, c_vp, c_vp, c_vp]
        lib.sc_tile_order_workspace_size.argtypes = [c_i64, P(c_i64)]
        lib.sc_tile_order.argtypes = [c_vp, c_i64, c_u32, c_i32, c_i32, c_vp, c_vp, c_i64, c_vp]
        lib.sc_gather_rows.argtypes = [c_vp, c_vp, c_i64, c_vp, c_i64, c_i64, c_i32, c_i32, c_vp]
        lib.sc_scatter_add_rows.argtypes = [c_vp, c_i64, c_vp, c_vp, c_i64, c_i64, c_i32, c_i32,
                                            c_i32, c_vp]
        lib.sc_last_error.restype = ctypes.c_char_p
        lib.sc_version.restype = ctypes.c_char_p
        for name in EXPORTS:
            if name not in ("sc_last_error", "sc_version"):
                getattr(lib, name).restype = c_i32
        _lib = lib
        return lib


def check(rc: int):
    """Raises the reference's exception type for a non-zero status."""
    if rc == SC_OK:
        return
    msg = load().sc_last_error().decode(errors="replace")
    if rc == SC_INVALID_ARG:
        raise ValueError(msg)
    raise RuntimeError(msg)


def device_error_bits(stream: int = 0) -> int:
    bits = c_i32(0)
    check(load().sc_check_device_error(c_vp(stream), ctypes.byref(bits)))
    return int(bits.value)


def require_cuda():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("cumm B200 kernels need a CUDA device (there is no CPU fallback)")
