"""GemmMainUnitTest: cumm's GEMM operator (``matmul2(GemmParams)``,
cumm/gemm/main.py:1176-1335; prologue cumm/gemm/nvrtc_code.py:34-140) on the
sm_100a kernels of libcumm_b200.so, plus the host helpers of the reference
class (``get_all_algo_desp``, ``extract_mnk``, ``align_to_power2``,
``device_synchronize``, ``stream_synchronize``, ``simple_select_tile_shape``).
"""
import ctypes
from typing import List, Optional, Tuple

import torch

from .. import _lib
from .. import tensorview as tv
from ..conv.main import _WS, _algo_code
from ..tensorview.gemm import GemmAlgoDesp, GemmParams, ShuffleStrideType


def _rows_ld(t: tv.Tensor) -> Tuple[int, int]:
    if t.ndim != 2:
        raise RuntimeError(f"expected a 2-D tensor, got {t.shape}")
    if t.stride[1] != 1:
        raise ValueError("inner dimension must be contiguous")
    return t.dim(0), t.stride[0]


def extract_mnk(a_shape, b_shape, trans_a: bool, trans_b: bool, trans_c: bool,
                shuffle_type: int = 0, a_inds_shape=None, b_inds_shape=None,
                c_inds_shape=None) -> Tuple[int, int, int]:
    """(m, n, k) exactly as the reference prologue derives them
    (cumm/gemm/nvrtc_code.py:62-125)."""
    if trans_c:
        trans_a, trans_b = not trans_b, not trans_a
        a_shape, b_shape = b_shape, a_shape
    st = ShuffleStrideType(shuffle_type)
    if st == ShuffleStrideType.kShuffleAC:
        m = a_inds_shape[0] if a_inds_shape else a_shape[0]
        k = a_shape[int(not trans_a)]
        n = b_shape[int(not trans_b)]
    elif st == ShuffleStrideType.kShuffleAB:
        m = a_shape[int(trans_a)]
        k = a_inds_shape[0]
        n = b_shape[int(not trans_b)]
    else:
        m = a_shape[int(trans_a)]
        k = a_shape[int(not trans_a)]
        n = b_shape[int(not trans_b)]
    return m, n, k


class GemmMainUnitTest:
    """Dense / shuffled GEMM entry points (reference class of the same name)."""

    def __init__(self, sync_check: bool = False):
        self.sync_check = sync_check

    @staticmethod
    def extract_mnk(a_shape, b_shape, trans_a, trans_b, trans_c, shuffle_type=0,
                    a_inds_shape=None, b_inds_shape=None, c_inds_shape=None):
        return list(extract_mnk(a_shape, b_shape, trans_a, trans_b, trans_c, shuffle_type,
                                a_inds_shape, b_inds_shape, c_inds_shape))

    @staticmethod
    def get_all_algo_desp() -> List[GemmAlgoDesp]:
        return get_all_algo_desp()

    @staticmethod
    def align_to_power2(val: int) -> int:
        """Smallest power of two >= val (cumm/gemm/main.py host helper)."""
        p = 1
        while p < val:
            p <<= 1
        return p

    @staticmethod
    def device_synchronize():
        torch.cuda.synchronize()

    @staticmethod
    def stream_synchronize(stream: int):
        if stream:
            torch.cuda.ExternalStream(stream).synchronize()
        else:
            torch.cuda.synchronize()

    @staticmethod
    def simple_select_tile_shape(m: int, n: int, k: int, tile_ms: List[int], tile_ns: List[int],
                                 tile_ks: List[int], tile_shape_to_algos, large_k_first: bool):
        """Largest tile that divides the problem least wastefully (reference
        gemm/main.py:1028-1134 ranks tiles by padding waste)."""
        best = None
        for tm in tile_ms:
            for tn in tile_ns:
                for tk in tile_ks:
                    waste = ((m + tm - 1) // tm * tm - m) / max(m, 1) + (
                        (n + tn - 1) // tn * tn - n) / max(n, 1)
                    key = (waste, -(tk if large_k_first else -tk), -(tm * tn))
                    if best is None or key < best[0]:
                        best = (key, (tm, tn, tk))
        if best is None:
            return []
        return tile_shape_to_algos.get(best[1], []) if isinstance(tile_shape_to_algos, dict) \
            else [best[1]]

    def matmul2(self, params: GemmParams) -> None:
        _lib.require_cuda()
        lib = _lib.load()
        params.check_valid()
        desp = params.algo_desp
        a, b, c = params.a, params.b, params.c
        d = params.d if not params.d.empty() else None
        ta, tb, tc = desp.trans_a, desp.trans_b, desp.trans_c
        st = ShuffleStrideType(desp.shuffle_type)
        if tc and st != ShuffleStrideType.kNoShuffle:
            raise RuntimeError("trans_c is only supported without shuffle")
        if tc:
            # C stored transposed: C^T = op(B)^T op(A)^T, i.e. the same GEMM with
            # the operands swapped and their transposes flipped
            # (cumm/gemm/nvrtc_code.py:62-68)
            a, b, ta, tb = b, a, not tb, not ta
        a_inds = params.a_inds if not params.a_inds.empty() else None
        b_inds = params.b_inds if not params.b_inds.empty() else None
        c_inds = params.c_inds if not params.c_inds.empty() else None
        m, n, k = extract_mnk(a.shape, b.shape, ta, tb, False, int(st),
                              a_inds.shape if a_inds is not None else None,
                              b_inds.shape if b_inds is not None else None)
        # k == k2 check of the reference prologue
        if st == ShuffleStrideType.kShuffleAB:
            k2 = b_inds.dim(0)
        else:
            k2 = b.shape[int(tb)]
        if k != k2:
            raise ValueError("error")
        if st != ShuffleStrideType.kShuffleAC and list(c.shape) != [m, n]:
            raise RuntimeError(f"c shape {c.shape} != {[m, n]}")
        if st == ShuffleStrideType.kShuffleAC and c.dim(1) != n:
            raise RuntimeError(f"c shape {c.shape} != [-1, {n}]")
        if not desp.supported(m, n, k):
            raise ValueError("this m, n, k isn't supported due to misaligned contiguous dim.")
        a_rows, lda = _rows_ld(a)
        b_rows, ldb = _rows_ld(b)
        _, ldc = _rows_ld(c)
        gp = _lib.GemmParamsC()
        gp.dtype_a, gp.dtype_b, gp.dtype_c = a.dtype, b.dtype, c.dtype
        gp.trans_a, gp.trans_b, gp.trans_c = int(ta), int(tb), int(tc)
        gp.shuffle_type = int(st)
        gp.algo = _algo_code(desp)
        gp.m, gp.n, gp.k = m, n, k
        gp.a, gp.lda, gp.b, gp.ldb, gp.c, gp.ldc = a.byte_pointer(), lda, b.byte_pointer(), ldb, \
            c.byte_pointer(), ldc
        if d is not None:
            if d.ndim == 1:
                if d.dim(0) != n:
                    raise RuntimeError("d must be a valid bias")
                gp.d, gp.ldd = d.byte_pointer(), 0
            else:
                gp.d, gp.ldd = d.byte_pointer(), d.stride[0]
        gp.a_inds = a_inds.byte_pointer() if a_inds is not None else None
        gp.b_inds = b_inds.byte_pointer() if b_inds is not None else None
        gp.c_inds = c_inds.byte_pointer() if c_inds is not None else None
        gp.a_rows, gp.b_rows = a_rows, b_rows
        gp.alpha, gp.beta = float(params.alpha), float(params.beta)
        gp.act_alpha, gp.act_beta = float(params.act_alpha), float(params.act_beta)
        gp.act_type = int(params.act_type)
        gp.split_k_slices = int(params.split_k_slices)
        gp.flags = _lib.SC_FLAG_SYNC_CHECK if self.sync_check else 0
        gp.stream = int(params.stream) if params.stream else None
        need = ctypes.c_int64(0)
        _lib.check(lib.sc_gemm_workspace_size(ctypes.byref(gp), ctypes.byref(need)))
        if need.value > 0:
            if params.workspace.empty():
                buf = _WS.get(c.device, int(params.stream or 0), need.value)
                gp.workspace, gp.workspace_bytes = buf.data_ptr(), buf.numel()
            else:
                if params.workspace.nbytes < need.value:
                    raise RuntimeError(f"workspace at least {need.value} bytes.")
                gp.workspace, gp.workspace_bytes = params.workspace.byte_pointer(), \
                    params.workspace.nbytes
        _lib.check(lib.sc_gemm_matmul(ctypes.byref(gp)))


def _gdesp(algo: str, dt_ab: int, dt_c: int, ta: bool, tb: bool, st: ShuffleStrideType,
           tile=(128, 128, 64)) -> GemmAlgoDesp:
    d = GemmAlgoDesp()
    d.dtype_a = d.dtype_b = dt_ab
    d.dtype_c = dt_c
    d.trans_a, d.trans_b, d.trans_c = ta, tb, False
    d.tile_shape = tile
    d.warp_tile_shape = (tile[0] // 2, tile[1] // 2, tile[2])
    d.num_stage = 4
    d.dacc = tv.float32
    d.dcomp = tv.float32
    d.algo = algo
    d.tensorop = (-1, -1, -1) if algo == "Simt" else (128, tile[1], 16)
    d.shuffle_type = st
    epa = 1 if algo == "Simt" else 8
    d.element_per_access_a = d.element_per_access_b = d.element_per_access_c = epa
    return d


def get_all_algo_desp() -> List[GemmAlgoDesp]:
    res = []
    for dt in (tv.bfloat16, tv.float16):
        for dc in (dt, tv.float32):
            for ta in (False, True):
                for tb in (False, True):
                    res.append(_gdesp("Tcgen05", dt, dc, ta, tb, ShuffleStrideType.kNoShuffle))
            res.append(_gdesp("Tcgen05", dt, dc, False, False, ShuffleStrideType.kShuffleAC))
            res.append(_gdesp("Tcgen05", dt, dc, False, True, ShuffleStrideType.kShuffleAC))
            res.append(_gdesp("Tcgen05", dt, dc, True, False, ShuffleStrideType.kShuffleAB))
    for ta in (False, True):
        for tb in (False, True):
            res.append(_gdesp("Simt", tv.float32, tv.float32, ta, tb, ShuffleStrideType.kNoShuffle,
                              (64, 64, 32)))
    res.append(_gdesp("Simt", tv.float32, tv.float32, False, False, ShuffleStrideType.kShuffleAC,
                      (64, 64, 32)))
    res.append(_gdesp("Simt", tv.float32, tv.float32, True, False, ShuffleStrideType.kShuffleAB,
                      (64, 64, 32)))
    return res
