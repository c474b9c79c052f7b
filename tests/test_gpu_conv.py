"""GPU parity of the sparse conv kernels (through the C ABI via
ConvMainUnitTest.implicit_gemm2) against the FP64 oracle."""
import numpy as np
import pytest
import torch

from cumm import tensorview as tv
from cumm import voxelgen as vg
from cumm.tensorview.gemm import ConvOpType
from oracle import conv_oracle as co
from oracle import pairs_oracle as po
from tests.helpers import TORCH, conv, dev, find_desp, to64, u32

pytestmark = pytest.mark.gpu

TOL_16 = 2e-3   # bf16/f16 operands, fp32 accumulation: norm-relative vs FP64
TOL_32 = 1e-5   # fp32 SIMT path


def _cloud(n, grid=24, seed=0):
    return vg.uniform_voxels(n, grid, seed)


def _subm(n, grid, seed):
    coords = _cloud(n, grid, seed)
    pf, pb, m = po.subm_pairs(coords, (grid, grid, grid))
    return coords, pf, pb, m


def _assert_close(y, ref, tol):
    nr, mr, ma = co.rel_err(y, ref)
    assert nr <= tol, (nr, mr, ma)


@pytest.mark.parametrize("dt", [tv.bfloat16, tv.float16])
@pytest.mark.parametrize("n,grid,C,K", [(3000, 24, 64, 64), (1000, 16, 32, 48), (777, 16, 16, 16),
                                        (2000, 20, 128, 128), (500, 12, 96, 32)])
@pytest.mark.parametrize("tile_m", [128, 32])
@pytest.mark.parametrize("sorted_idx", [False, True])
def test_fwd_tcgen05(dt, n, grid, C, K, tile_m, sorted_idx):
    coords, pf, pb, m = _subm(n, grid, n)
    rng = np.random.default_rng(1)
    x = rng.standard_normal((n, C)).astype(np.float32)
    w = vg.kaiming_uniform(K, 27, C, 2)
    xt, wt = dev(x, TORCH[dt]), dev(w, TORCH[dt])
    ms, order = po.sort_by_key_split(m, 0xffffffff)
    out = torch.zeros((n, K), dtype=TORCH[dt], device="cuda")
    mo = tv.zeros([(n + tile_m - 1) // tile_m], tv.uint32, 0)
    conv(ConvOpType.kForward, find_desp(ConvOpType.kForward, "Tcgen05", dt, dt, dt, tile_m),
         xt, wt, out, pf, ms, order, mask_output=mo, sorted_indices=sorted_idx)
    ref, mo_ref = co.conv_fwd_masked(to64(xt), to64(wt), pf, ms, order, tile_m)
    _assert_close(to64(out), ref, TOL_16)
    assert np.array_equal(mo.numpy(), mo_ref)


@pytest.mark.parametrize("dt", [tv.bfloat16, tv.float16])
@pytest.mark.parametrize("n,grid,C,K", [(3000, 24, 64, 64), (1000, 16, 48, 32), (600, 12, 16, 16),
                                        (1500, 16, 64, 128), (1200, 16, 32, 64)])
@pytest.mark.parametrize("sorted_idx", [False, True])
def test_dgrad_tcgen05(dt, n, grid, C, K, sorted_idx):
    coords, pf, pb, m = _subm(n, grid, n + 1)
    rng = np.random.default_rng(3)
    dy = rng.standard_normal((n, K)).astype(np.float32)
    w = vg.kaiming_uniform(K, 27, C, 4)
    dyt, wt = dev(dy, TORCH[dt]), dev(w, TORCH[dt])
    ms, order = po.sort_by_key_split(m, 0xffffffff)
    din = torch.zeros((n, C), dtype=TORCH[dt], device="cuda")
    conv(ConvOpType.kBackwardInput,
         find_desp(ConvOpType.kBackwardInput, "Tcgen05", dt, dt, dt, 128),
         din, wt, dyt, pb, ms, order, reverse_mask=True, sorted_indices=sorted_idx)
    ref = co.conv_dgrad_masked(to64(dyt), to64(wt), pb, ms, order, 128, reverse_mask=True)
    _assert_close(to64(din), ref, TOL_16)


@pytest.mark.parametrize("dw_dt", [tv.bfloat16, tv.float32])
@pytest.mark.parametrize("n,grid,C,K", [(3000, 24, 64, 64), (1500, 16, 32, 32), (800, 12, 128, 64),
                                        (700, 12, 16, 16)])
def test_wgrad_tcgen05(dw_dt, n, grid, C, K):
    coords, pf, pb, m = _subm(n, grid, n + 2)
    rng = np.random.default_rng(5)
    x = rng.standard_normal((n, C)).astype(np.float32)
    dy = rng.standard_normal((n, K)).astype(np.float32)
    xt, dyt = dev(x, torch.bfloat16), dev(dy, torch.bfloat16)
    ms, order = po.sort_by_key_split(m, 0xffffffff)
    mo = co.tile_masks(ms, 128).astype(np.uint32)
    dw = torch.zeros((K, 27, C), dtype=TORCH[dw_dt], device="cuda")
    desp = find_desp(ConvOpType.kBackwardWeight, "Tcgen05", tv.bfloat16, dw_dt, tv.bfloat16, 128)
    conv(ConvOpType.kBackwardWeight, desp, xt, dw, dyt, pf, mo, order, mask_width=128)
    ref = co.conv_wgrad_masked(to64(dyt), to64(xt), pf, mo, 128, order, 27)
    _assert_close(to64(dw), ref, TOL_16 if dw_dt == tv.bfloat16 else 2e-5)


def test_wgrad_fp32_dw_at_element_offset():
    """An fp32 dW view that starts 4 bytes past a 16-byte boundary cannot take
    the in-place accumulation (its v4 reductions need 16-byte alignment); it
    goes through the workspace and the finalize kernel and gives the aligned
    result."""
    n, grid, C, K = 3000, 24, 64, 64
    coords, pf, pb, m = _subm(n, grid, 21)
    rng = np.random.default_rng(21)
    xt = dev(rng.standard_normal((n, C)).astype(np.float32), torch.bfloat16)
    dyt = dev(rng.standard_normal((n, K)).astype(np.float32), torch.bfloat16)
    ms, order = po.sort_by_key_split(m, 0xffffffff)
    mo = co.tile_masks(ms, 128).astype(np.uint32)
    desp = find_desp(ConvOpType.kBackwardWeight, "Tcgen05", tv.bfloat16, tv.float32, tv.bfloat16, 128)
    dw = torch.zeros((K, 27, C), dtype=torch.float32, device="cuda")
    conv(ConvOpType.kBackwardWeight, desp, xt, dw, dyt, pf, mo, order, mask_width=128)
    buf = torch.full((K * 27 * C + 1,), 5.0, dtype=torch.float32, device="cuda")
    dw_off = buf[1:].view(K, 27, C)
    assert dw_off.data_ptr() % 16 == 4
    conv(ConvOpType.kBackwardWeight, desp, xt, dw_off, dyt, pf, mo, order, mask_width=128)
    nr, _, _ = co.rel_err(to64(dw_off), to64(dw))
    assert nr < 1e-6, nr
    assert buf[0].item() == 5.0
    ref = co.conv_wgrad_masked(to64(dyt), to64(xt), pf, mo, 128, order, 27)
    _assert_close(to64(dw_off), ref, 2e-5)


def test_fwd_output_add_scale_bias_epilogue():
    """The reference's int8-inference epilogue form with a residual operand:
    out = act(scale * acc + alpha * bias + beta * output_add)
    (cumm/conv/nvrtc_code.py:78-99, cumm/gemm/output_op/linear.py:300-392;
    the int8 clamp does not apply to a floating-point output)."""
    n, grid, C, K = 2500, 20, 64, 64
    coords, pf, pb, m = _subm(n, grid, 22)
    rng = np.random.default_rng(22)
    x = rng.standard_normal((n, C)).astype(np.float32)
    w = vg.kaiming_uniform(K, 27, C, 22)
    xt, wt = dev(x, torch.bfloat16), dev(w, torch.bfloat16)
    scale = dev((0.5 + rng.random(K)).astype(np.float32))
    bias = dev(rng.standard_normal(K).astype(np.float32), torch.bfloat16)
    res = dev(rng.standard_normal((n, K)).astype(np.float32), torch.bfloat16)
    ms, order = po.sort_by_key_split(m, 0xffffffff)
    desp = find_desp(ConvOpType.kForward, "Tcgen05", tv.bfloat16, tv.bfloat16, tv.bfloat16, 128)
    for act_type, act_alpha in ((0, 0.0), (1, 0.0), (3, 0.2)):
        out = torch.full((n, K), 9.0, dtype=torch.bfloat16, device="cuda")
        conv(ConvOpType.kForward, desp, xt, wt, out, pf, ms, order, alpha=0.75, beta=0.5, bias=bias,
             scale=scale, output_add=res, act_type=act_type, act_alpha=act_alpha)
        ref, _ = co.conv_fwd_masked(to64(xt), to64(wt), pf, ms, order, 128, alpha=0.75, beta=0.5,
                                    bias=to64(bias), scale=to64(scale), output_add=to64(res),
                                    act_type=act_type, act_alpha=act_alpha)
        _assert_close(to64(out), ref, TOL_16)
    # output_add without scale is the reference's "only int8 inference" error
    out = torch.zeros((n, K), dtype=torch.bfloat16, device="cuda")
    with pytest.raises(ValueError, match="output_add"):
        conv(ConvOpType.kForward, desp, xt, wt, out, pf, ms, order, output_add=res)


def test_split_two_launches_equals_single():
    """MaskSplitImplicitGemm: split filters with beta=1 on the second launch
    (main_real_spconv.py:273-294) equals one launch with all offsets."""
    n, grid, C, K = 4000, 24, 64, 64
    coords, pf, pb, m = _subm(n, grid, 9)
    rng = np.random.default_rng(9)
    xt = dev(rng.standard_normal((n, C)).astype(np.float32), torch.bfloat16)
    wt = dev(vg.kaiming_uniform(K, 27, C, 9), torch.bfloat16)
    desp = find_desp(ConvOpType.kForward, "Tcgen05", tv.bfloat16, tv.bfloat16, tv.float32, 128)
    out1 = torch.zeros((n, K), dtype=torch.float32, device="cuda")
    ms, order = po.sort_by_key_split(m, 0xffffffff)
    conv(ConvOpType.kForward, desp, xt, wt, out1, pf, ms, order)
    out2 = torch.zeros((n, K), dtype=torch.float32, device="cuda")
    for j, sm in enumerate(po.split_masks(27, 2)):
        msj, oj = po.sort_by_key_split(m, sm)
        conv(ConvOpType.kForward, desp, xt, wt, out2, pf, msj, oj, mask_filter=sm,
             beta=1.0 if j else 0.0)
    _assert_close(to64(out2), to64(out1), 1e-6)
    ref = co.fwd_gather_gemm_scatter(to64(xt), to64(wt), pf)
    _assert_close(to64(out1), ref, 1e-5)


def test_fwd_epilogue_bias_act():
    n, grid, C, K = 1500, 16, 32, 64
    coords, pf, pb, m = _subm(n, grid, 10)
    rng = np.random.default_rng(10)
    xt = dev(rng.standard_normal((n, C)).astype(np.float32), torch.bfloat16)
    wt = dev(vg.kaiming_uniform(K, 27, C, 10), torch.bfloat16)
    bias = dev(rng.standard_normal(K).astype(np.float32), torch.bfloat16)
    ms, order = po.sort_by_key_split(m, 0xffffffff)
    desp = find_desp(ConvOpType.kForward, "Tcgen05", tv.bfloat16, tv.bfloat16, tv.bfloat16, 128)
    for act_type, act_alpha in ((1, 0.0), (3, 0.1), (2, 0.0)):
        out = torch.zeros((n, K), dtype=torch.bfloat16, device="cuda")
        conv(ConvOpType.kForward, desp, xt, wt, out, pf, ms, order, alpha=0.5, beta=1.0,
             bias=bias, act_type=act_type, act_alpha=act_alpha)
        ref, _ = co.conv_fwd_masked(to64(xt), to64(wt), pf, ms, order, 128, alpha=0.5, beta=1.0,
                                    bias=to64(bias), act_type=act_type, act_alpha=act_alpha)
        _assert_close(to64(out), ref, TOL_16)


def test_fwd_fp8_scale_epilogue():
    n, grid, C, K = 2000, 20, 64, 128
    coords, pf, pb, m = _subm(n, grid, 11)
    rng = np.random.default_rng(11)
    x = rng.standard_normal((n, C)).astype(np.float32)
    w = vg.kaiming_uniform(K, 27, C, 11)
    sx = np.abs(x).max() / 448.0
    sw = np.abs(w).reshape(K, -1).max(1) / 448.0
    xq = dev(x / sx, torch.float8_e4m3fn)
    wq = dev(w / sw[:, None, None], torch.float8_e4m3fn)
    scale = dev((sx * sw).astype(np.float32))
    ms, order = po.sort_by_key_split(m, 0xffffffff)
    out = torch.zeros((n, K), dtype=torch.bfloat16, device="cuda")
    desp = find_desp(ConvOpType.kForward, "Tcgen05", tv.float_e4m3, tv.float_e4m3, tv.bfloat16, 128)
    conv(ConvOpType.kForward, desp, xq, wq, out, pf, ms, order, scale=scale)
    ref, _ = co.conv_fwd_masked(to64(xq), to64(wq), pf, ms, order, 128,
                                scale=(sx * sw).astype(np.float64))
    _assert_close(to64(out), ref, TOL_16)


@pytest.mark.parametrize("op", [ConvOpType.kForward, ConvOpType.kBackwardInput,
                                ConvOpType.kBackwardWeight])
def test_simt_fp32(op):
    """The fp32 path meets 1e-5 norm-relative (20k voxels in 64^3, C=K=32 is
    the workload; a smaller cloud keeps the test short)."""
    n, grid, C, K = 5000, 40, 32, 32
    coords, pf, pb, m = _subm(n, grid, 12)
    rng = np.random.default_rng(12)
    x = rng.standard_normal((n, C)).astype(np.float32)
    w = vg.kaiming_uniform(K, 27, C, 12)
    dy = rng.standard_normal((n, K)).astype(np.float32)
    ms, order = po.sort_by_key_split(m, 0xffffffff)
    desp = find_desp(op, "Simt", tv.float32, tv.float32, tv.float32, 32 if op != 2 else 32)
    if op == ConvOpType.kForward:
        out = torch.zeros((n, K), device="cuda")
        conv(op, desp, dev(x), dev(w), out, pf, ms, order)
        ref, _ = co.conv_fwd_masked(x, w, pf, ms, order, 32)
        _assert_close(to64(out), ref, TOL_32)
    elif op == ConvOpType.kBackwardInput:
        din = torch.zeros((n, C), device="cuda")
        conv(op, desp, din, dev(w), dev(dy), pb, ms, order, reverse_mask=True)
        ref = co.conv_dgrad_masked(dy, w, pb, ms, order, 32, reverse_mask=True)
        _assert_close(to64(din), ref, TOL_32)
    else:
        mo = co.tile_masks(ms, 32).astype(np.uint32)
        dw = torch.zeros((K, 27, C), device="cuda")
        conv(op, desp, dev(x), dw, dev(dy), pf, mo, order, mask_width=32)
        ref = co.conv_wgrad_masked(dy, x, pf, mo, 32, order, 27)
        _assert_close(to64(dw), ref, TOL_32)


def test_edge_cases():
    desp = find_desp(ConvOpType.kForward, "Tcgen05", tv.bfloat16, tv.bfloat16, tv.bfloat16, 128)
    # all-empty masks: outputs get the epilogue of a zero accumulator (beta * bias)
    n, C, K = 300, 64, 64
    pf = np.full((27, n), -1, np.int32)
    m = np.zeros(n, np.uint32)
    order = np.arange(n, dtype=np.int32)
    x = dev(np.ones((n, C), np.float32), torch.bfloat16)
    w = dev(np.ones((K, 27, C), np.float32), torch.bfloat16)
    out = torch.full((n, K), 7.0, dtype=torch.bfloat16, device="cuda")
    conv(ConvOpType.kForward, desp, x, w, out, pf, m, order)
    assert torch.all(out == 0)
    # dgrad with empty masks writes nothing
    din = torch.full((n, C), 3.0, dtype=torch.bfloat16, device="cuda")
    dd = find_desp(ConvOpType.kBackwardInput, "Tcgen05", tv.bfloat16, tv.bfloat16, tv.bfloat16, 128)
    conv(ConvOpType.kBackwardInput, dd, din, w, out, pf, m, order, reverse_mask=True)
    assert torch.all(din == 3.0)
    # N = 0: an empty index table is rejected like the reference prologue
    # (TV_ASSERT_RT_ERR(!indices.empty()), cumm/conv/nvrtc_code.py:123-125)
    e = torch.zeros((0, C), dtype=torch.bfloat16, device="cuda")
    eo = torch.zeros((0, K), dtype=torch.bfloat16, device="cuda")
    with pytest.raises(RuntimeError, match="indices"):
        conv(ConvOpType.kForward, desp, e, w, eo, np.zeros((27, 0), np.int32),
             np.zeros(0, np.uint32), np.zeros(0, np.int32))
    # ragged: N not a multiple of the tile, one row
    pf1 = np.full((27, 1), -1, np.int32)
    pf1[13, 0] = 0
    x1 = dev(np.full((1, C), 2.0, np.float32), torch.bfloat16)
    o1 = torch.zeros((1, K), dtype=torch.bfloat16, device="cuda")
    conv(ConvOpType.kForward, desp, x1, w, o1, pf1, np.array([1 << 13], np.uint32),
         np.zeros(1, np.int32))
    assert torch.all(o1.float() == 2.0 * C)


def test_bad_index_reported():
    """A gather index beyond the input raises a device error instead of reading
    out of bounds (the kernel checks every index and zero-fills)."""
    n, C, K = 256, 64, 64
    desp = find_desp(ConvOpType.kForward, "Tcgen05", tv.bfloat16, tv.bfloat16, tv.bfloat16, 128)
    pf = np.full((27, n), -1, np.int32)
    pf[13] = np.arange(n)
    pf[13, 5] = n + 100  # out of range
    m = np.full(n, 1 << 13, np.uint32)
    x = dev(np.ones((n, C), np.float32), torch.bfloat16)
    w = dev(np.ones((K, 27, C), np.float32), torch.bfloat16)
    out = torch.zeros((n, K), dtype=torch.bfloat16, device="cuda")
    with pytest.raises(RuntimeError, match="device error"):
        conv(ConvOpType.kForward, desp, x, w, out, pf, m, np.arange(n, dtype=np.int32))


@pytest.mark.parametrize("seed", [0])
def test_lidar_200k_fwd_dgrad_wgrad(seed):
    """The 200k-voxel LiDAR-like C=K=64 bf16 layer: fwd, dgrad, wgrad against
    the FP64 oracle at 2e-3."""
    n, C, K = 200000, 64, 64
    coords = vg.lidar_voxels(n, seed=seed)
    pf, pb, m = po.subm_pairs(coords, vg.KITTI_SHAPE)
    ms, order = po.sort_by_key_split(m, 0xffffffff)
    rng = np.random.default_rng(seed)
    xt = dev(rng.standard_normal((n, C)).astype(np.float32), torch.bfloat16)
    wt = dev(vg.kaiming_uniform(K, 27, C, seed), torch.bfloat16)
    dyt = dev(rng.standard_normal((n, K)).astype(np.float32), torch.bfloat16)
    out = torch.zeros((n, K), dtype=torch.bfloat16, device="cuda")
    mo = tv.zeros([(n + 127) // 128], tv.uint32, 0)
    conv(ConvOpType.kForward,
         find_desp(ConvOpType.kForward, "Tcgen05", tv.bfloat16, tv.bfloat16, tv.bfloat16, 128),
         xt, wt, out, pf, ms, order, mask_output=mo)
    x64, w64, dy64 = to64(xt), to64(wt), to64(dyt)
    ref = co.fwd_gather_gemm_scatter(x64, w64, pf)
    _assert_close(to64(out), ref, TOL_16)
    din = torch.zeros((n, C), dtype=torch.bfloat16, device="cuda")
    conv(ConvOpType.kBackwardInput,
         find_desp(ConvOpType.kBackwardInput, "Tcgen05", tv.bfloat16, tv.bfloat16, tv.bfloat16, 128),
         din, wt, dyt, pb, ms, order, reverse_mask=True)
    _assert_close(to64(din), co.dgrad_gather_gemm_scatter(dy64, w64, pb), TOL_16)
    dw = torch.zeros((K, 27, C), dtype=torch.float32, device="cuda")
    conv(ConvOpType.kBackwardWeight,
         find_desp(ConvOpType.kBackwardWeight, "Tcgen05", tv.bfloat16, tv.float32, tv.bfloat16, 128),
         xt, dw, dyt, pf, mo.numpy(), order, mask_width=128)
    _assert_close(to64(dw), co.wgrad_gather_gemm_scatter(dy64, x64, pf), TOL_16)


def test_lidar_200k_bench_path():
    """The exact call sequence bench.py times, at its full size, against the
    FP64 oracle: the GPU pair build, indices_sorted (the forward and
    backward-input kernels then copy whole tiles' index slices with
    cp.async.bulk), the forward's mask_output feeding backward-weight, and an
    fp32 dW accumulated in place (alpha 1, beta 0, every offset)."""
    from cumm.conv.main import ConvMainUnitTest
    from cumm.spconv_ops import build_pair_table
    from cumm.tensorview.gemm import ConvParams
    n, C, K = 200000, 64, 64
    coords = vg.lidar_voxels(n, seed=0)
    pt = build_pair_table(torch.from_numpy(coords).cuda(), vg.KITTI_SHAPE)
    pf, pb, m = po.subm_pairs(coords, vg.KITTI_SHAPE)
    assert np.array_equal(pt.pairs_fwd.cpu().numpy(), pf)
    assert np.array_equal(pt.pairs_bwd.cpu().numpy(), pb)
    rng = np.random.default_rng(0)
    xt = dev(rng.standard_normal((n, C)).astype(np.float32), torch.bfloat16)
    dyt = dev(rng.standard_normal((n, K)).astype(np.float32), torch.bfloat16)
    wt = dev(vg.kaiming_uniform(K, 27, C, 0), torch.bfloat16)
    out = torch.empty((n, K), dtype=torch.bfloat16, device="cuda")
    din = torch.empty((n, C), dtype=torch.bfloat16, device="cuda")
    dw = torch.full((K, 27, C), 3.0, dtype=torch.float32, device="cuda")
    mo = torch.empty(((n + 127) // 128,), dtype=torch.int32, device="cuda")
    for op in (ConvOpType.kForward, ConvOpType.kBackwardInput, ConvOpType.kBackwardWeight):
        p = ConvParams(3, op)
        p.conv_algo_desp = find_desp(op, "Tcgen05", tv.bfloat16,
                                     tv.float32 if op == ConvOpType.kBackwardWeight else tv.bfloat16,
                                     tv.bfloat16, 128)
        if op == ConvOpType.kForward:
            p.input, p.weight, p.output = tv.Tensor(xt), tv.Tensor(wt), tv.Tensor(out)
            p.indices = tv.Tensor(pt.pairs_fwd)
            p.mask = tv.Tensor(pt.masks_fwd[0], tv.uint32)
            p.mask_output = tv.Tensor(mo, tv.uint32)
        elif op == ConvOpType.kBackwardInput:
            p.input, p.weight, p.output = tv.Tensor(din), tv.Tensor(wt), tv.Tensor(dyt)
            p.indices = tv.Tensor(pt.pairs_bwd)
            p.mask = tv.Tensor(pt.masks_fwd[0], tv.uint32)
            p.reverse_mask = True
        else:
            p.input, p.weight, p.output = tv.Tensor(xt), tv.Tensor(dw), tv.Tensor(dyt)
            p.indices = tv.Tensor(pt.pairs_fwd)
            p.mask = tv.Tensor(mo, tv.uint32)
            p.mask_width = 128
        p.mask_argsort = tv.Tensor(pt.argsorts_fwd[0])
        p.indices_sorted = tv.Tensor(pt.sorted_indices("bwd" if op == ConvOpType.kBackwardInput else "fwd"))
        ConvMainUnitTest(sync_check=True).implicit_gemm2(p)
    torch.cuda.synchronize()
    ms = pt.masks_fwd[0].cpu().numpy().view(np.uint32)
    order = pt.argsorts_fwd[0].cpu().numpy()
    x64, w64, dy64 = to64(xt), to64(wt), to64(dyt)
    ref, mo_ref = co.conv_fwd_masked(x64, w64, pf, ms, order, 128)
    _assert_close(to64(out), ref, TOL_16)
    assert np.array_equal(mo.cpu().numpy().view(np.uint32), mo_ref)
    _assert_close(to64(din), co.dgrad_gather_gemm_scatter(dy64, w64, pb), TOL_16)
    _assert_close(to64(dw), co.wgrad_gather_gemm_scatter(dy64, x64, pf), TOL_16)
    _assert_close(to64(dw), co.conv_wgrad_masked(dy64, x64, pf, mo_ref, 128, order, 27), TOL_16)


@pytest.mark.parametrize("n", [30000, 30001])
def test_sorted_index_table_identical(n):
    """ConvParams.indices_sorted (coalesced index table) gives bit-identical
    results for fwd, dgrad and wgrad.  With N % 4 == 0 the forward and
    backward-input kernels copy each whole tile's index slices with
    cp.async.bulk (and gate them in the producers); with N % 4 != 0 the
    slices are not 16-byte aligned and every row is loaded and gated by the
    index loaders."""
    import torch as _t
    from cumm.spconv_ops import build_pair_table
    C, K = 64, 64
    coords = vg.lidar_voxels(n, seed=5)
    pt = build_pair_table(_t.from_numpy(coords).cuda(), vg.KITTI_SHAPE)
    rng = np.random.default_rng(5)
    x = dev(rng.standard_normal((n, C)).astype(np.float32), torch.bfloat16)
    w = dev(vg.kaiming_uniform(K, 27, C, 5), torch.bfloat16)
    dy = dev(rng.standard_normal((n, K)).astype(np.float32), torch.bfloat16)
    m = pt.masks_fwd[0].cpu().numpy().view(np.uint32)
    order = pt.argsorts_fwd[0].cpu().numpy()
    from cumm.conv.main import ConvMainUnitTest
    from cumm.tensorview.gemm import ConvParams
    outs = []
    for use_sorted in (False, True):
        res = []
        for op, dw_dt in ((ConvOpType.kForward, tv.bfloat16), (ConvOpType.kBackwardInput, tv.bfloat16),
                          (ConvOpType.kBackwardWeight, tv.float32)):
            p = ConvParams(3, op)
            p.conv_algo_desp = find_desp(op, "Tcgen05", tv.bfloat16, dw_dt, tv.bfloat16, 128)
            if op == ConvOpType.kForward:
                o = torch.zeros((n, K), dtype=torch.bfloat16, device="cuda")
                p.input, p.weight, p.output = tv.Tensor(x), tv.Tensor(w), tv.Tensor(o)
                p.indices = tv.Tensor(pt.pairs_fwd)
                p.mask = tv.Tensor(pt.masks_fwd[0], tv.uint32)
                if use_sorted:
                    p.indices_sorted = tv.Tensor(pt.sorted_indices("fwd"))
            elif op == ConvOpType.kBackwardInput:
                o = torch.zeros((n, C), dtype=torch.bfloat16, device="cuda")
                p.input, p.weight, p.output = tv.Tensor(o), tv.Tensor(w), tv.Tensor(dy)
                p.indices = tv.Tensor(pt.pairs_bwd)
                p.mask = tv.Tensor(pt.masks_fwd[0], tv.uint32)
                p.reverse_mask = True
                if use_sorted:
                    p.indices_sorted = tv.Tensor(pt.sorted_indices("bwd"))
            else:
                o = torch.zeros((K, 27, C), dtype=torch.float32, device="cuda")
                mo = co.tile_masks(m, 128).astype(np.uint32)
                p.input, p.weight, p.output = tv.Tensor(x), tv.Tensor(o), tv.Tensor(dy)
                p.indices = tv.Tensor(pt.pairs_fwd)
                p.mask = u32(mo)
                p.mask_width = 128
                if use_sorted:
                    p.indices_sorted = tv.Tensor(pt.sorted_indices("fwd"))
            p.mask_argsort = tv.Tensor(pt.argsorts_fwd[0])
            ConvMainUnitTest(sync_check=True).implicit_gemm2(p)
            res.append(o.float().cpu())
        outs.append(res)
    assert torch.equal(outs[0][0], outs[1][0])
    assert torch.equal(outs[0][1], outs[1][1])
    # wgrad accumulates per-CTA partial sums with fp32 atomics: equal up to the
    # (run-to-run) summation order
    nr = (torch.linalg.norm(outs[0][2] - outs[1][2]) / torch.linalg.norm(outs[0][2])).item()
    assert nr < 1e-6, nr


@pytest.mark.parametrize("n,grid,C,K,tile_n,tile_m", [
    (4000, 24, 64, 64, 0, 128), (4000, 24, 64, 64, 32, 64), (4000, 24, 64, 64, 16, 32),
    (2000, 20, 128, 64, 0, 128), (2000, 20, 64, 128, 64, 128), (2000, 20, 128, 128, 64, 32),
    (4, 8, 64, 64, 0, 128), (132, 10, 64, 64, 0, 128),
    # 64-byte rows (SWIZZLE_64B stages, four per strand): C = 32 forward, K = 32 backward-input
    (4000, 24, 32, 32, 0, 128), (4000, 24, 32, 64, 32, 64), (3000, 20, 64, 32, 16, 32), (132, 10, 32, 32, 0, 128)])
def test_strand_kernel_shapes(n, grid, C, K, tile_n, tile_m):
    """Forward and backward-input through the strand kernel (sorted index
    table, 128-byte rows, column tiles <= 64): several chunks per offset
    (C = 128), several column tiles (K = 128 with tile_n 64), sub-tile masks
    (tile_shape[0] 32 / 64) with mask_output, a split mask_filter with beta = 1
    on the second launch, and tiny and ragged N, against the FP64 oracle."""
    coords, pf, pb, m = _subm(n, grid, n + 7)
    rng = np.random.default_rng(n)
    xt = dev(rng.standard_normal((n, C)).astype(np.float32), torch.bfloat16)
    wt = dev(vg.kaiming_uniform(K, 27, C, n), torch.bfloat16)
    dyt = dev(rng.standard_normal((n, K)).astype(np.float32), torch.bfloat16)
    ms, order = po.sort_by_key_split(m, 0xffffffff)
    desp = find_desp(ConvOpType.kForward, "Tcgen05", tv.bfloat16, tv.bfloat16, tv.float32, tile_m)
    out = torch.zeros((n, K), dtype=torch.float32, device="cuda")
    mo = tv.zeros([(n + tile_m - 1) // tile_m], tv.uint32, 0)
    conv(ConvOpType.kForward, desp, xt, wt, out, pf, ms, order, mask_output=mo, sorted_indices=True,
         tile_n=tile_n)
    ref, mo_ref = co.conv_fwd_masked(to64(xt), to64(wt), pf, ms, order, tile_m)
    _assert_close(to64(out), ref, TOL_16)
    assert np.array_equal(mo.numpy(), mo_ref)
    # MaskSplitImplicitGemm form: two launches over the split masks, beta 1 on the second
    out2 = torch.zeros((n, K), dtype=torch.float32, device="cuda")
    for j, sm in enumerate(po.split_masks(27, 2)):
        msj, oj = po.sort_by_key_split(m, sm)
        conv(ConvOpType.kForward, desp, xt, wt, out2, pf, msj, oj, mask_filter=sm, beta=1.0 if j else 0.0,
             sorted_indices=True, tile_n=tile_n)
    _assert_close(to64(out2), ref, TOL_16)
    dd = find_desp(ConvOpType.kBackwardInput, "Tcgen05", tv.bfloat16, tv.bfloat16, tv.bfloat16, tile_m)
    din = torch.zeros((n, C), dtype=torch.bfloat16, device="cuda")
    conv(ConvOpType.kBackwardInput, dd, din, wt, dyt, pb, ms, order, reverse_mask=True, sorted_indices=True,
         tile_n=tile_n if C % max(tile_n, 1) == 0 else 0)
    _assert_close(to64(din), co.conv_dgrad_masked(to64(dyt), to64(wt), pb, ms, order, tile_m, reverse_mask=True),
                  TOL_16)


def test_strand_kernel_fp8_and_bad_index():
    """E4M3 operands with 128-byte rows (C = 128) and the scale epilogue on the
    strand kernel, and a bad index in the sorted table reported as a device
    error instead of being gathered."""
    n, grid, C, K = 2000, 20, 128, 64
    coords, pf, pb, m = _subm(n, grid, 31)
    rng = np.random.default_rng(31)
    x = rng.standard_normal((n, C)).astype(np.float32)
    w = vg.kaiming_uniform(K, 27, C, 31)
    sx = np.abs(x).max() / 448.0
    sw = np.abs(w).reshape(K, -1).max(1) / 448.0
    xq = dev(x / sx, torch.float8_e4m3fn)
    wq = dev(w / sw[:, None, None], torch.float8_e4m3fn)
    scale = dev((sx * sw).astype(np.float32))
    ms, order = po.sort_by_key_split(m, 0xffffffff)
    out = torch.zeros((n, K), dtype=torch.bfloat16, device="cuda")
    desp = find_desp(ConvOpType.kForward, "Tcgen05", tv.float_e4m3, tv.float_e4m3, tv.bfloat16, 128)
    conv(ConvOpType.kForward, desp, xq, wq, out, pf, ms, order, scale=scale, sorted_indices=True)
    ref, _ = co.conv_fwd_masked(to64(xq), to64(wq), pf, ms, order, 128, scale=(sx * sw).astype(np.float64))
    _assert_close(to64(out), ref, TOL_16)
    bad = pf.copy()
    r = int(order[5])
    k = int(np.nonzero(pf[:, r] >= 0)[0][0])
    bad[k, r] = n + 50
    xb = dev(rng.standard_normal((n, 64)).astype(np.float32), torch.bfloat16)
    wb = dev(vg.kaiming_uniform(64, 27, 64, 1), torch.bfloat16)
    ob = torch.zeros((n, 64), dtype=torch.bfloat16, device="cuda")
    db = find_desp(ConvOpType.kForward, "Tcgen05", tv.bfloat16, tv.bfloat16, tv.bfloat16, 128)
    with pytest.raises(RuntimeError, match="device error"):
        conv(ConvOpType.kForward, db, xb, wb, ob, bad, ms, order, sorted_indices=True)


@pytest.mark.parametrize("use_sorted", [True, False])
def test_tile_schedule_does_not_change_results(use_sorted):
    """With a tile order (PairTable.tile_order) the forward hands its 128-row
    tiles out heaviest first; without one it deals them in mask order, and
    without a workspace (optional for the forward) it also reads the unsorted
    index table on the row-gather kernel.  Each tile is computed by one
    pipeline alone, so all give bit-identical outputs and mask_output, and
    match the FP64 oracle."""
    import ctypes
    from cumm import _lib
    from cumm.conv.main import ConvMainUnitTest, build_conv_params_c
    from cumm.spconv_ops import build_pair_table
    from cumm.tensorview.gemm import ConvParams
    n, C, K = 40000, 64, 64
    coords = vg.lidar_voxels(n, seed=11)
    pt = build_pair_table(torch.from_numpy(coords).cuda(), vg.KITTI_SHAPE)
    rng = np.random.default_rng(11)
    x = dev(rng.standard_normal((n, C)).astype(np.float32), torch.bfloat16)
    w = dev(vg.kaiming_uniform(K, 27, C, 11), torch.bfloat16)
    outs, mos = [], []
    for with_ws in (True, False, "given"):
        p = ConvParams(3, ConvOpType.kForward)
        p.conv_algo_desp = find_desp(ConvOpType.kForward, "Tcgen05", tv.bfloat16, tv.bfloat16, tv.bfloat16, 32)
        o = torch.full((n, K), float("nan"), dtype=torch.bfloat16, device="cuda")
        mo = tv.zeros([(n + 31) // 32], tv.uint32, 0)
        p.input, p.weight, p.output = tv.Tensor(x), tv.Tensor(w), tv.Tensor(o)
        p.indices = tv.Tensor(pt.pairs_fwd)
        p.mask = tv.Tensor(pt.masks_fwd[0], tv.uint32)
        p.mask_argsort = tv.Tensor(pt.argsorts_fwd[0])
        p.mask_output = mo
        if use_sorted:
            p.indices_sorted = tv.Tensor(pt.sorted_indices("fwd"))
        if with_ws == "given":
            p.tile_order = tv.Tensor(pt.tile_order("fwd"))
        if with_ws:
            ConvMainUnitTest(sync_check=True).implicit_gemm2(p)
        else:
            cp, _info = build_conv_params_c(p)
            cp.flags |= _lib.SC_FLAG_SYNC_CHECK
            cp.workspace, cp.workspace_bytes = None, 0
            _lib.check(_lib.load().sc_conv_implicit_gemm(ctypes.byref(cp)))
        torch.cuda.synchronize()
        outs.append(o.float().cpu())
        mos.append(mo.numpy().copy())
    assert not torch.isnan(outs[0]).any()
    assert torch.equal(outs[0], outs[1]) and torch.equal(outs[0], outs[2])
    assert np.array_equal(mos[0], mos[1]) and np.array_equal(mos[0], mos[2])
    m = pt.masks_fwd[0].cpu().numpy().view(np.uint32)
    order = pt.argsorts_fwd[0].cpu().numpy()
    ref, mo_ref = co.conv_fwd_masked(to64(x), to64(w), pt.pairs_fwd.cpu().numpy(), m, order, 32)
    _assert_close(outs[0].double().numpy(), ref, TOL_16)
    assert np.array_equal(mos[0], mo_ref)



def test_tile_order_is_largest_first_permutation():
    """SpconvOps.tile_order: a permutation of the 128-row tiles with their
    offset counts (popcount of the OR-ed masks, mask_filter applied)
    non-increasing; the reverse (backward-input) count gives the same counts
    for kv-bit masks; a ragged last tile and a split filter included."""
    from cumm.spconv_ops import SpconvOps
    for n, filt in ((30001, 0xffffffff), (5000, 0x3fff), (77, 0xffffffff)):
        coords, pf, pb, m = _subm(n, 40 if n > 1000 else 8, n)
        ms, order = po.sort_by_key_split(m, 0xffffffff)
        md = torch.from_numpy(ms.view(np.int32)).cuda()
        tiles = (n + 127) // 128
        pc = np.array([bin(int(np.bitwise_or.reduce(ms[t * 128:(t + 1) * 128])) & filt).count("1")
                       for t in range(tiles)])
        for rev in (False, True):
            o = SpconvOps.tile_order(md, 27, filt, rev).cpu().numpy()
            assert sorted(o.tolist()) == list(range(tiles))
            assert np.all(np.diff(pc[o]) <= 0), (n, rev)


def test_tile_order_bad_entry_reported():
    """A caller-supplied tile_order entry outside the row tiles sets the
    bad-index bit (reported as a device error) instead of being followed."""
    import torch as _t
    from cumm.conv.main import ConvMainUnitTest
    from cumm.spconv_ops import build_pair_table
    from cumm.tensorview.gemm import ConvParams
    n, C, K = 4000, 64, 64
    coords = vg.lidar_voxels(n, seed=3)
    pt = build_pair_table(_t.from_numpy(coords).cuda(), vg.KITTI_SHAPE)
    x = dev(np.random.default_rng(3).standard_normal((n, C)).astype(np.float32), torch.bfloat16)
    w = dev(vg.kaiming_uniform(K, 27, C, 3), torch.bfloat16)
    for use_sorted in (True, False):
        p = ConvParams(3, ConvOpType.kForward)
        p.conv_algo_desp = find_desp(ConvOpType.kForward, "Tcgen05", tv.bfloat16, tv.bfloat16, tv.bfloat16, 128)
        o = torch.zeros((n, K), dtype=torch.bfloat16, device="cuda")
        p.input, p.weight, p.output = tv.Tensor(x), tv.Tensor(w), tv.Tensor(o)
        p.indices = tv.Tensor(pt.pairs_fwd)
        p.mask = tv.Tensor(pt.masks_fwd[0], tv.uint32)
        p.mask_argsort = tv.Tensor(pt.argsorts_fwd[0])
        if use_sorted:
            p.indices_sorted = tv.Tensor(pt.sorted_indices("fwd"))
        bad = pt.tile_order("fwd").clone()
        bad[3] = -5
        p.tile_order = tv.Tensor(bad)
        with pytest.raises(RuntimeError, match="device error"):
            ConvMainUnitTest(sync_check=True).implicit_gemm2(p)



@pytest.mark.parametrize("n,K,tile_m", [(6000, 64, 128), (2000, 128, 32), (132, 64, 128)])
def test_strand_kernel_e4m3_64byte_rows(n, K, tile_m):
    """E4M3 with C = 64 (64-byte rows): the strand kernel with SWIZZLE_64B
    stages (four per strand), per-output-channel scale epilogue, several column
    tiles (K = 128), mask_output, against the FP64 oracle on the rounded
    operands."""
    C = 64
    coords, pf, pb, m = _subm(n, 26 if n > 1000 else 10, n + 3)
    rng = np.random.default_rng(n)
    x = rng.standard_normal((n, C)).astype(np.float32)
    w = vg.kaiming_uniform(K, 27, C, n)
    sx = np.abs(x).max() / 448.0
    sw = np.abs(w).reshape(K, -1).max(1) / 448.0
    xq = dev(x / sx, torch.float8_e4m3fn)
    wq = dev(w / sw[:, None, None], torch.float8_e4m3fn)
    scale = dev((sx * sw).astype(np.float32))
    ms, order = po.sort_by_key_split(m, 0xffffffff)
    out = torch.zeros((n, K), dtype=torch.bfloat16, device="cuda")
    mo = tv.zeros([(n + tile_m - 1) // tile_m], tv.uint32, 0)
    desp = find_desp(ConvOpType.kForward, "Tcgen05", tv.float_e4m3, tv.float_e4m3, tv.bfloat16, tile_m)
    conv(ConvOpType.kForward, desp, xq, wq, out, pf, ms, order, scale=scale, sorted_indices=True,
         mask_output=mo, tile_n=64 if K > 64 else 0)
    ref, mo_ref = co.conv_fwd_masked(to64(xq), to64(wq), pf, ms, order, tile_m,
                                     scale=(sx * sw).astype(np.float64))
    _assert_close(to64(out), ref, TOL_16)
    assert np.array_equal(mo.numpy(), mo_ref)


def test_tile_order_backward_input_and_split_masks():
    """The largest-first order made for the forward masks serves the
    submanifold backward-input (reverse_mask) and each mask split of the
    MaskSplitImplicitGemm form: results are bit-identical to calls without an
    order (tiles in mask order) and match the FP64 oracle."""
    import ctypes
    from cumm import _lib
    from cumm.conv.main import ConvMainUnitTest, build_conv_params_c
    from cumm.spconv_ops import build_pair_table
    from cumm.tensorview.gemm import ConvParams
    n, C, K = 36000, 64, 64
    coords = vg.lidar_voxels(n, seed=21)
    pt = build_pair_table(torch.from_numpy(coords).cuda(), vg.KITTI_SHAPE, num_split=2)
    rng = np.random.default_rng(21)
    w = dev(vg.kaiming_uniform(K, 27, C, 21), torch.bfloat16)
    dy = dev(rng.standard_normal((n, K)).astype(np.float32), torch.bfloat16)
    x = dev(rng.standard_normal((n, C)).astype(np.float32), torch.bfloat16)

    def call(p, given):
        if given:
            ConvMainUnitTest(sync_check=True).implicit_gemm2(p)
        else:
            cp, _info = build_conv_params_c(p)
            cp.flags |= _lib.SC_FLAG_SYNC_CHECK
            cp.tile_order = None
            lib = _lib.load()
            need = ctypes.c_int64(0)
            _lib.check(lib.sc_conv_workspace_size(ctypes.byref(cp), ctypes.byref(need)))
            ws = torch.empty(max(need.value, 256), dtype=torch.uint8, device="cuda")
            # a workspace but no order: the call orders the tiles itself
            cp.workspace, cp.workspace_bytes = ws.data_ptr(), ws.numel()
            _lib.check(lib.sc_conv_implicit_gemm(ctypes.byref(cp)))
        torch.cuda.synchronize()

    dins, outs = [], []
    for given in (True, False):
        din = torch.zeros((n, C), dtype=torch.bfloat16, device="cuda")
        out = torch.zeros((n, K), dtype=torch.float32, device="cuda")
        for j in range(2):
            p = ConvParams(3, ConvOpType.kBackwardInput)
            p.conv_algo_desp = find_desp(ConvOpType.kBackwardInput, "Tcgen05", tv.bfloat16, tv.bfloat16,
                                         tv.bfloat16, 128)
            p.input, p.weight, p.output = tv.Tensor(din), tv.Tensor(w), tv.Tensor(dy)
            p.indices = tv.Tensor(pt.pairs_bwd)
            p.mask = tv.Tensor(pt.masks_fwd[j], tv.uint32)
            p.mask_argsort = tv.Tensor(pt.argsorts_fwd[j])
            p.indices_sorted = tv.Tensor(pt.sorted_indices("bwd", j))
            p.reverse_mask = True
            p.mask_filter = pt.split_masks[j]
            p.beta = 1.0 if j else 0.0
            if given:
                p.tile_order = tv.Tensor(pt.tile_order("bwd", j))
            call(p, given)
            q = ConvParams(3, ConvOpType.kForward)
            q.conv_algo_desp = find_desp(ConvOpType.kForward, "Tcgen05", tv.bfloat16, tv.bfloat16, tv.float32, 128)
            q.input, q.weight, q.output = tv.Tensor(x), tv.Tensor(w), tv.Tensor(out)
            q.indices = tv.Tensor(pt.pairs_fwd)
            q.mask = tv.Tensor(pt.masks_fwd[j], tv.uint32)
            q.mask_argsort = tv.Tensor(pt.argsorts_fwd[j])
            q.indices_sorted = tv.Tensor(pt.sorted_indices("fwd", j))
            q.mask_filter = pt.split_masks[j]
            q.beta = 1.0 if j else 0.0
            if given:
                q.tile_order = tv.Tensor(pt.tile_order("fwd", j))
            call(q, given)
        dins.append(din.float().cpu())
        outs.append(out.cpu())
    assert torch.equal(dins[0], dins[1])
    assert torch.equal(outs[0], outs[1])
    pf, pb = pt.pairs_fwd.cpu().numpy(), pt.pairs_bwd.cpu().numpy()
    # the split backward-input writes bf16 dIn twice (the second launch adds
    # to the rounded first half), so it carries two bf16 roundings: twice the
    # one-launch tolerance; the forward accumulates into fp32
    _assert_close(dins[0].double().numpy(), co.dgrad_gather_gemm_scatter(to64(dy), to64(w), pb), 2 * TOL_16)
    _assert_close(outs[0].double().numpy(), co.fwd_gather_gemm_scatter(to64(x), to64(w), pf), TOL_16)



def test_default_path_builds_sorted_table():
    """A call without indices_sorted builds the sorted index table in its
    workspace and runs the strand kernel: bit-identical to the call given the
    table.  With a workspace too small for the table (the forward's is
    optional) it reads the unsorted table on the row-gather kernel, equal up to
    fp32 summation order."""
    import ctypes
    from cumm import _lib
    from cumm.conv.main import ConvMainUnitTest, build_conv_params_c
    from cumm.spconv_ops import build_pair_table
    from cumm.tensorview.gemm import ConvParams
    n, C, K = 30000, 64, 64
    coords = vg.lidar_voxels(n, seed=17)
    pt = build_pair_table(torch.from_numpy(coords).cuda(), vg.KITTI_SHAPE)
    rng = np.random.default_rng(17)
    x = dev(rng.standard_normal((n, C)).astype(np.float32), torch.bfloat16)
    w = dev(vg.kaiming_uniform(K, 27, C, 17), torch.bfloat16)
    outs = []
    for mode in ("given", "default", "small_ws"):
        p = ConvParams(3, ConvOpType.kForward)
        p.conv_algo_desp = find_desp(ConvOpType.kForward, "Tcgen05", tv.bfloat16, tv.bfloat16, tv.float32, 128)
        o = torch.full((n, K), float("nan"), dtype=torch.float32, device="cuda")
        p.input, p.weight, p.output = tv.Tensor(x), tv.Tensor(w), tv.Tensor(o)
        p.indices = tv.Tensor(pt.pairs_fwd)
        p.mask = tv.Tensor(pt.masks_fwd[0], tv.uint32)
        p.mask_argsort = tv.Tensor(pt.argsorts_fwd[0])
        if mode == "given":
            p.indices_sorted = tv.Tensor(pt.sorted_indices("fwd"))
        if mode != "small_ws":
            ConvMainUnitTest(sync_check=True).implicit_gemm2(p)
        else:
            cp, _info = build_conv_params_c(p)
            cp.flags |= _lib.SC_FLAG_SYNC_CHECK
            ws = torch.empty(256, dtype=torch.uint8, device="cuda")
            cp.workspace, cp.workspace_bytes = ws.data_ptr(), 256
            _lib.check(_lib.load().sc_conv_implicit_gemm(ctypes.byref(cp)))
        torch.cuda.synchronize()
        outs.append(o.cpu())
    assert torch.equal(outs[0], outs[1])
    nr = ((outs[2] - outs[0]).norm() / outs[0].norm()).item()
    assert nr < 1e-6, nr
    ref = co.fwd_gather_gemm_scatter(to64(x), to64(w), pt.pairs_fwd.cpu().numpy())
    _assert_close(outs[0].double().numpy(), ref, TOL_16)
