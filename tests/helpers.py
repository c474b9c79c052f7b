"""Shared helpers for the GPU parity tests: builds ConvParams the way the
reference driver does (cumm/conv/main_real_spconv.py:228-294) and runs them
through ConvMainUnitTest.implicit_gemm2."""
import numpy as np
import torch

from cumm import tensorview as tv
from cumm.conv.main import ConvMainUnitTest, get_all_conv_algo_desp
from cumm.tensorview.gemm import ConvOpType, ConvParams

TORCH = {tv.float32: torch.float32, tv.float16: torch.float16, tv.bfloat16: torch.bfloat16,
         tv.float_e4m3: torch.float8_e4m3fn}


def find_desp(op, algo, dt_in, dt_w, dt_out, tile_m=128):
    for d in get_all_conv_algo_desp():
        if (d.op_type == op and d.algo == algo and d.dtype_input == dt_in and
                d.dtype_weight == dt_w and d.dtype_output == dt_out and d.tile_shape[0] == tile_m):
            return d
    raise KeyError((op, algo, dt_in, dt_w, dt_out, tile_m))


def dev(x, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    return t if dtype is None else t.to(dtype)


def u32(x):
    """uint32 numpy -> int32 torch storage tagged uint32."""
    return tv.Tensor(dev(np.asarray(x, np.uint32).view(np.int32)), tv.uint32)


def i32(x):
    return tv.Tensor(dev(np.asarray(x, np.int32)), tv.int32)


def conv(op, desp, inp, weight, out, indices, mask, argsort, mask_output=None, mask_filter=0xffffffff,
         reverse_mask=False, mask_width=-1, alpha=1.0, beta=0.0, bias=None, scale=None,
         output_add=None, act_type=0, act_alpha=0.0, sync_check=True, sorted_indices=False, tile_n=0):
    """inp / weight / out are torch tensors (already on the GPU).  With
    sorted_indices the index table permuted into argsort order is passed as
    well (ConvParams.indices_sorted), which selects the kernels that read it
    (the strand kernel for 128-byte rows, N % 4 == 0 and tile_n <= 64)."""
    p = ConvParams(3, op)
    p.conv_algo_desp = desp
    p.input = tv.Tensor(inp, desp.dtype_input)
    p.weight = tv.Tensor(weight, desp.dtype_weight)
    p.output = tv.Tensor(out, desp.dtype_output)
    p.indices = i32(indices)
    p.mask = u32(mask)
    p.mask_argsort = i32(argsort)
    if sorted_indices:
        p.indices_sorted = i32(np.ascontiguousarray(np.asarray(indices)[:, np.asarray(argsort)]))
    if tile_n:
        p.tile_n = tile_n
    if mask_output is not None:
        p.mask_output = mask_output
    p.mask_filter = mask_filter
    p.reverse_mask = reverse_mask
    p.mask_width = mask_width
    p.alpha, p.beta = alpha, beta
    p.act_type, p.act_alpha = act_type, act_alpha
    if bias is not None:
        p.bias = tv.Tensor(bias)
    if scale is not None:
        p.scale = tv.Tensor(scale)
    if output_add is not None:
        p.output_add = tv.Tensor(output_add)
    ConvMainUnitTest(sync_check=sync_check).implicit_gemm2(p)
    return p


def to64(t):
    return t.float().cpu().numpy().astype(np.float64)
