"""ConvMainUnitTest: the sparse-convolution operator of cumm, served by the
sm_100a kernels of libcumm_b200.so.

Reference surface: ``ConvMainUnitTest().implicit_gemm2(params: tv.gemm.ConvParams)``
(cumm/conv/main.py:483-745) with the prologue of
cumm/conv/nvrtc_code.py:20-196, plus ``get_all_conv_algo_desp``
(cumm/conv/main.py:983-1050) and ``extract_mnk`` (main.py:467-481).
Only the mask-sparse (implicit GEMM over indice pairs) path exists here; the
dense NHWC path of the reference is out of scope.
"""
import ctypes
import threading
from typing import Dict, List, Tuple

import torch

from .. import _lib
from .. import tensorview as tv
from ..tensorview.gemm import (SIMT_ALGOS, TENSOR_OP_ALGOS, Activation, ConvAlgoDesp,
                               ConvOpType, ConvParams)


def implicit_gemm_mnk(op_type: ConvOpType, N: int, C: int, K: int, kv: int) -> Tuple[int, int, int]:
    """(m, n, k) of the mask-sparse implicit GEMM (include/tensorview/gemm/core/utils.h:63-76)."""
    op = ConvOpType(op_type)
    if op == ConvOpType.kForward:
        return N, K, C * kv
    if op == ConvOpType.kBackwardInput:
        return N, C, K * kv
    return K, C * kv, N


class _Workspace:
    """Per (device, stream) scratch buffer grown on demand (the C ABI never
    allocates; the reference allocates ``tv::empty`` when no workspace is
    given, cumm/conv/nvrtc_code.py:181-196)."""

    def __init__(self):
        self._bufs: Dict[Tuple[int, int], torch.Tensor] = {}
        self._lock = threading.Lock()

    def get(self, device: int, stream: int, nbytes: int) -> torch.Tensor:
        key = (device, stream)
        with self._lock:
            buf = self._bufs.get(key)
            if buf is None or buf.numel() < nbytes:
                buf = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=f"cuda:{device}")
                self._bufs[key] = buf
            return buf


_WS = _Workspace()


def _ptr(t: tv.Tensor):
    return None if t is None or t.empty() else t.byte_pointer()


def _algo_code(desp) -> int:
    if desp.algo in SIMT_ALGOS:
        return _lib.SC_ALGO_SIMT
    if desp.algo in TENSOR_OP_ALGOS:
        return _lib.SC_ALGO_TCGEN05
    raise RuntimeError(f"Can't Found Algorithm for params: {desp.algo}")


def _check_dense(t: tv.Tensor, name: str):
    if not t.empty() and not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    if not t.empty() and t.device < 0:
        raise ValueError(f"{name} must be a CUDA tensor")


def build_conv_params_c(params: ConvParams) -> Tuple[_lib.ConvParamsC, dict]:
    """Validates a ConvParams and packs it into the C struct (no launch)."""
    desp = params.conv_algo_desp
    if not desp.mask_sparse:
        raise RuntimeError("Can't Found Algorithm: only mask_sparse convolutions are supported")
    inp, w, out = params.input, params.weight, params.output
    if inp.ndim != 2:
        raise RuntimeError("error: input must be [N, C]")
    if w.ndim != 3:
        raise RuntimeError("error: weight must be [K, kv, C]")
    if out.ndim != 2:
        raise RuntimeError("error: output must be [N, K]")
    K = w.dim(0)
    kv = w.dim(1)
    C = inp.dim(1)
    if out.dim(1) != K:
        raise RuntimeError("error: output.dim(1) != weight.dim(0)")
    if w.dim(2) != C:
        raise RuntimeError("error: weight.dim(2) != input.dim(1)")
    for t, n in ((inp, "input"), (w, "weight"), (out, "output"), (params.indices, "indices"),
                 (params.mask, "mask"), (params.mask_argsort, "mask_argsort"),
                 (params.mask_output, "mask_output"), (params.bias, "bias"),
                 (params.scale, "scale"), (params.output_add, "output_add")):
        _check_dense(t, n)
    if params.indices.empty():
        raise RuntimeError("error: indices must not be empty")
    if params.indices.ndim != 2 or params.indices.dim(0) != kv:
        raise RuntimeError(f"error: indices shape {params.indices.shape} != [{kv}, -1]")
    if not params.scale.empty() and params.scale.dtype != tv.float32:
        raise ValueError("scale must be float32 [K]")
    op = ConvOpType(desp.op_type)
    cp = _lib.ConvParamsC()
    cp.op_type = int(op)
    cp.algo = _algo_code(desp)
    cp.dtype_input = inp.dtype
    cp.dtype_weight = w.dtype
    cp.dtype_output = out.dtype
    cp.tile_m = int(desp.tile_shape[0])
    cp.tile_k = int(desp.tile_shape[2])
    cp.kv = kv
    cp.n_in = inp.dim(0)
    cp.n_out = out.dim(0)
    cp.C = C
    cp.K = K
    cp.N = params.indices.dim(1)
    cp.input = _ptr(inp)
    cp.weight = _ptr(w)
    cp.output = _ptr(out)
    cp.indices = _ptr(params.indices)
    cp.mask = _ptr(params.mask)
    cp.mask_count = params.mask.size
    cp.mask_argsort = _ptr(params.mask_argsort)
    cp.mask_output = _ptr(params.mask_output)
    cp.mask_output_count = params.mask_output.size
    cp.mask_filter = int(params.mask_filter) & 0xffffffff
    cp.reverse_mask = 1 if params.reverse_mask else 0
    cp.mask_width = int(params.mask_width)
    cp.alpha = float(params.alpha)
    cp.beta = float(params.beta)
    cp.act_alpha = float(params.act_alpha)
    cp.act_beta = float(params.act_beta)
    cp.act_type = int(params.act_type)
    cp.bias = _ptr(params.bias)
    cp.output_add = _ptr(params.output_add)
    cp.scale = _ptr(params.scale)
    cp.split_k_slices = int(params.split_k_slices)
    cp.flags = 0
    cp.stream = int(params.stream) if params.stream else None
    isorted = getattr(params, "indices_sorted", None)
    if isorted is not None and not isorted.empty():
        if list(isorted.shape) != list(params.indices.shape):
            raise ValueError("indices_sorted must have the shape of indices")
        _check_dense(isorted, "indices_sorted")
        cp.indices_sorted = isorted.byte_pointer()
    cp.tile_n = int(getattr(params, "tile_n", 0) or 0)
    torder = getattr(params, "tile_order", None)
    if torder is not None and not torder.empty():
        n_rows = int(params.indices.shape[1])
        if torder.dtype != tv.int32 or list(torder.shape) != [(n_rows + 127) // 128]:
            raise ValueError("tile_order must be int32 [ceil(N / 128)]")
        _check_dense(torder, "tile_order")
        cp.tile_order = torder.byte_pointer()
    return cp, {"kv": kv, "C": C, "K": K}


class ConvMainUnitTest:
    """Sparse convolution entry points (reference class of the same name)."""

    def __init__(self, sync_check: bool = False):
        # sync_check: synchronise after each launch and raise on a device error word
        self.sync_check = sync_check

    @staticmethod
    def extract_mnk(op_type: int, N: int, C: int, K: int, kernel_volume: int,
                    in_prod: int = -1, out_prod: int = -1, mask_sparse: bool = True):
        if not mask_sparse:
            raise RuntimeError("only mask_sparse is supported")
        return list(implicit_gemm_mnk(ConvOpType(op_type), N, C, K, kernel_volume))

    @staticmethod
    def get_all_conv_algo_desp() -> List[ConvAlgoDesp]:
        return get_all_conv_algo_desp()

    def implicit_gemm2(self, params: ConvParams) -> None:
        _lib.require_cuda()
        lib = _lib.load()
        cp, info = build_conv_params_c(params)
        if self.sync_check:
            cp.flags |= _lib.SC_FLAG_SYNC_CHECK
        need = ctypes.c_int64(0)
        _lib.check(lib.sc_conv_workspace_size(ctypes.byref(cp), ctypes.byref(need)))
        if need.value > 0:
            ws = params.workspace
            if ws.empty():
                dev = params.output.device if params.output.device >= 0 else 0
                buf = _WS.get(dev, int(params.stream or 0), need.value)
                cp.workspace = buf.data_ptr()
                cp.workspace_bytes = buf.numel()
            else:
                if ws.nbytes < need.value:
                    raise RuntimeError(f"workspace at least {need.value} bytes.")
                cp.workspace = ws.byte_pointer()
                cp.workspace_bytes = ws.nbytes
        if params.timer is not None and getattr(params.timer, "enable", False):
            with params.timer.record(repr(params.conv_algo_desp), int(params.stream or 0)):
                rc = lib.sc_conv_implicit_gemm(ctypes.byref(cp))
        else:
            rc = lib.sc_conv_implicit_gemm(ctypes.byref(cp))
        _lib.check(rc)

    # the reference keeps a stale kwarg-style implicit_gemm (main_real.py:184);
    # here it is the same operator as implicit_gemm2
    implicit_gemm = implicit_gemm2


def _desp(op: ConvOpType, algo: str, dt_in: int, dt_w: int, dt_out: int, tile: Tuple[int, int, int],
          epa: int) -> ConvAlgoDesp:
    d = ConvAlgoDesp(3, op)
    iwo = [dt_in, dt_w, dt_out]
    inv = ConvAlgoDesp.gemm_abc_012_to_iwo(op)
    d.dtype_a, d.dtype_b, d.dtype_c = iwo[inv[0]], iwo[inv[1]], iwo[inv[2]]
    d.tile_shape = tile
    d.warp_tile_shape = (tile[0] // 2, tile[1] // 2, tile[2])
    d.num_stage = 4
    d.dacc = tv.float32
    d.dcomp = tv.float32
    d.algo = algo
    d.tensorop = (-1, -1, -1) if algo in SIMT_ALGOS else (128, tile[1], 16)
    # trans flags of the mask-sparse GEMM views (cumm/conv/params.py:61-69)
    d.trans_a = op == ConvOpType.kBackwardWeight
    d.trans_b = op != ConvOpType.kBackwardInput
    d.trans_c = False
    d.element_per_access_a = epa
    d.element_per_access_b = epa
    d.element_per_access_c = epa
    d.mask_sparse = True
    d.increment_k_first = True
    d.split_k_serial = op == ConvOpType.kBackwardWeight
    return d


_ALL_CONV_DESPS: List[ConvAlgoDesp] = []


def get_all_conv_algo_desp() -> List[ConvAlgoDesp]:
    """Every conv algorithm this build serves.  tile_shape[0] is the mask
    granularity (rows OR-ed into one mask word; 32, 64 or 128); the tcgen05
    kernels always compute 128-row tiles and gate rows by their sub-tile's mask.
    Built once; callers get their own list."""
    if not _ALL_CONV_DESPS:
        _ALL_CONV_DESPS.extend(_build_conv_algo_desps())
    return list(_ALL_CONV_DESPS)


def _build_conv_algo_desps() -> List[ConvAlgoDesp]:
    res: List[ConvAlgoDesp] = []
    bf16, f16, f32, e4m3 = tv.bfloat16, tv.float16, tv.float32, tv.float_e4m3
    for tm in (128, 64, 32):
        for dt in (bf16, f16):
            res.append(_desp(ConvOpType.kForward, "Tcgen05", dt, dt, dt, (tm, 128, 64), 8))
            res.append(_desp(ConvOpType.kForward, "Tcgen05", dt, dt, f32, (tm, 128, 64), 8))
            res.append(_desp(ConvOpType.kBackwardInput, "Tcgen05", dt, dt, dt, (tm, 128, 64), 8))
        res.append(_desp(ConvOpType.kForward, "Tcgen05", e4m3, e4m3, bf16, (tm, 128, 128), 16))
        res.append(_desp(ConvOpType.kForward, "Simt", f32, f32, f32, (tm, 32, 32), 1))
        res.append(_desp(ConvOpType.kBackwardInput, "Simt", f32, f32, f32, (tm, 32, 32), 1))
    for dw in (bf16, f32):
        res.append(_desp(ConvOpType.kBackwardWeight, "Tcgen05", bf16, dw, bf16, (128, 128, 64), 8))
    res.append(_desp(ConvOpType.kBackwardWeight, "Simt", f32, f32, f32, (32, 32, 32), 1))
    return res
