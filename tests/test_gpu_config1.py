"""The plain correctness layer: 20,000 unique voxels drawn uniformly without
replacement from a 64^3 grid (seeded), C = K = 32, fp32 features ~N(0, 1),
Kaiming-uniform weights [K, 27, C]; pair table and masks bit-exact with the
CPU builder, forward within 1e-5 (norm-relative) of the reference's CPU
gather-GEMM-scatter (cumm/conv/main_real_spconv.py:309-325)."""
import numpy as np
import pytest
import torch

from cumm import tensorview as tv
from cumm import voxelgen as vg
from cumm.spconv_ops import build_pair_table
from cumm.tensorview.gemm import ConvOpType
from oracle import conv_oracle as co
from oracle import pairs_oracle as po
from tests.helpers import conv, dev, find_desp, to64

pytestmark = pytest.mark.gpu


def test_config1_pairs_and_forward():
    n, grid, C, K = 20_000, 64, 32, 32
    coords = vg.uniform_voxels(n, grid, 0)
    pt = build_pair_table(torch.from_numpy(coords).cuda(), (grid, grid, grid))
    pf, pb, m = po.subm_pairs(coords, (grid, grid, grid))
    assert np.array_equal(pt.pairs_fwd.cpu().numpy(), pf)
    assert np.array_equal(pt.pairs_bwd.cpu().numpy(), pb)
    ms, order = po.sort_by_key_split(m, 0xffffffff)
    assert np.array_equal(pt.masks_fwd[0].cpu().numpy().view(np.uint32), ms)
    assert np.array_equal(pt.argsorts_fwd[0].cpu().numpy(), order)
    rng = np.random.default_rng(0)
    x = rng.standard_normal((n, C)).astype(np.float32)
    w = vg.kaiming_uniform(K, 27, C, 0)
    out = torch.zeros((n, K), dtype=torch.float32, device="cuda")
    conv(ConvOpType.kForward, find_desp(ConvOpType.kForward, "Simt", tv.float32, tv.float32, tv.float32, 128),
         dev(x), dev(w), out, pf, ms, order)
    ref = co.fwd_gather_gemm_scatter(x.astype(np.float64), w.astype(np.float64), pf)
    nr, mr, ma = co.rel_err(to64(out), ref)
    assert nr <= 1e-5, (nr, mr, ma)
    # the bf16 tensor-core path on the same layer, against FP64 of its rounded operands
    xb, wb = dev(x, torch.bfloat16), dev(w, torch.bfloat16)
    outb = torch.zeros((n, K), dtype=torch.float32, device="cuda")
    conv(ConvOpType.kForward, find_desp(ConvOpType.kForward, "Tcgen05", tv.bfloat16, tv.bfloat16, tv.float32, 128),
         xb, wb, outb, pf, ms, order)
    nr, mr, ma = co.rel_err(to64(outb), co.fwd_gather_gemm_scatter(to64(xb), to64(wb), pf))
    assert nr <= 1e-5, (nr, mr, ma)
