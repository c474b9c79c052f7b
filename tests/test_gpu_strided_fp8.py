"""Stride-2 downsample (3x3x3, pad 1, C 64 -> 128) on the 200k-voxel LiDAR-like
cloud: BF16 and FP8-E4M3 forward through ConvMainUnitTest.implicit_gemm2
against the FP64 oracle.

Tolerances (norm-relative): the kernel's own error, measured against FP64 on
the same rounded / quantized operands, is <= 2e-3 for both variants (bf16
output rounding dominates).  Against FP64 on the unrounded fp32 inputs the
BF16 path stays <= 5e-3 and the FP8 path (3 mantissa bits per operand) <= 6e-2."""
import numpy as np
import pytest
import torch

from cumm import tensorview as tv
from cumm import voxelgen as vg
from cumm.precision import quantize_act_fp8, quantize_weight_fp8
from cumm.spconv_ops import build_pair_table
from cumm.tensorview.gemm import ConvOpType
from oracle import conv_oracle as co
from tests.helpers import conv, find_desp, to64

pytestmark = pytest.mark.gpu

TOL_KERNEL = 2e-3
TOL_BF16_TOTAL = 5e-3
TOL_FP8_TOTAL = 6e-2


@pytest.fixture(scope="module")
def layer():
    coords = torch.from_numpy(vg.lidar_voxels(200_000, seed=3)).cuda()
    pt = build_pair_table(coords, vg.KITTI_SHAPE, ksize=(3, 3, 3), stride=(2, 2, 2),
                          padding=(1, 1, 1), subm=False)
    rng = np.random.default_rng(3)
    x = torch.from_numpy(rng.standard_normal((200_000, 64)).astype(np.float32)).cuda()
    w = torch.from_numpy(vg.kaiming_uniform(128, 27, 64, 3)).cuda()
    pf = pt.pairs_fwd.cpu().numpy()
    ref32 = co.fwd_gather_gemm_scatter(x.double().cpu().numpy(), w.double().cpu().numpy(), pf)
    return pt, x, w, pf, ref32


def _run(pt, xin, win, dt, scale=None):
    out = torch.zeros((pt.n_out, 128), dtype=torch.bfloat16, device="cuda")
    ms = pt.masks_fwd[0].cpu().numpy().view(np.uint32)
    order = pt.argsorts_fwd[0].cpu().numpy()
    conv(ConvOpType.kForward, find_desp(ConvOpType.kForward, "Tcgen05", dt, dt, tv.bfloat16, 128),
         xin, win, out, pt.pairs_fwd.cpu().numpy(), ms, order, scale=scale)
    return out


def test_strided_pairs_shape(layer):
    pt, _, _, pf, _ = layer
    # every output of a stride-2 pad-1 3x3x3 conv has at least one input pair
    assert pt.n_out > 0 and pf.shape == (27, pt.n_out)
    assert ((pf >= 0).sum(0) > 0).all()


def test_bf16_downsample(layer):
    pt, x, w, pf, ref32 = layer
    xb, wb = x.bfloat16(), w.bfloat16()
    out = to64(_run(pt, xb, wb, tv.bfloat16))
    ref_b = co.fwd_gather_gemm_scatter(to64(xb), to64(wb), pf)
    nr, mr, ma = co.rel_err(out, ref_b)
    assert nr <= TOL_KERNEL, (nr, mr, ma)
    nr, mr, ma = co.rel_err(out, ref32)
    assert nr <= TOL_BF16_TOTAL, (nr, mr, ma)


def test_fp8_downsample(layer):
    pt, x, w, pf, ref32 = layer
    xq, sx = quantize_act_fp8(x)
    wq, sw = quantize_weight_fp8(w, sx)
    out = to64(_run(pt, xq, wq, tv.float_e4m3, scale=sw))
    ref_q = co.fwd_gather_gemm_scatter(to64(xq), to64(wq), pf) * sw.double().cpu().numpy()[None, :]
    nr, mr, ma = co.rel_err(out, ref_q)
    assert nr <= TOL_KERNEL, (nr, mr, ma)
    nr, mr, ma = co.rel_err(out, ref32)
    assert nr <= TOL_FP8_TOTAL, (nr, mr, ma)
