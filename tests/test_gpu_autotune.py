"""Backward-weight split-K (ConvParams.split_k_slices = the kernel's row
splits) and the autotuner that picks it: every candidate gives the same dW
(up to fp32 atomic order) and matches the oracle."""
import numpy as np
import pytest
import torch

from cumm import voxelgen as vg
from cumm.autotune import ConvAutotuner, WgradConfig, run_wgrad, wgrad_candidates
from cumm.spconv_ops import build_pair_table
from oracle import conv_oracle as co
from tests.helpers import to64

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def layer():
    n = 20_000
    coords = torch.from_numpy(vg.lidar_voxels(n, seed=21)).cuda()
    pt = build_pair_table(coords, vg.KITTI_SHAPE)
    rng = np.random.default_rng(21)
    x = torch.from_numpy(rng.standard_normal((n, 64)).astype(np.float32)).cuda().bfloat16()
    dy = torch.from_numpy(rng.standard_normal((n, 64)).astype(np.float32)).cuda().bfloat16()
    w = torch.from_numpy(vg.kaiming_uniform(64, 27, 64, 21)).cuda().bfloat16()
    out = torch.empty((n, 64), dtype=torch.bfloat16, device="cuda")
    mo = torch.empty(((n + 127) // 128,), dtype=torch.int32, device="cuda")
    # forward with mask_output: the reduced masks backward-weight reads
    from cumm import tensorview as tv
    from cumm.conv.main import ConvMainUnitTest
    from cumm.tensorview.gemm import ConvOpType, ConvParams
    from tests.helpers import find_desp
    p = ConvParams(3, ConvOpType.kForward)
    p.conv_algo_desp = find_desp(ConvOpType.kForward, "Tcgen05", tv.bfloat16, tv.bfloat16, tv.bfloat16, 128)
    p.input, p.weight, p.output = tv.Tensor(x), tv.Tensor(w), tv.Tensor(out)
    p.indices = tv.Tensor(pt.pairs_fwd)
    p.mask = tv.Tensor(pt.masks_fwd[0], tv.uint32)
    p.mask_argsort = tv.Tensor(pt.argsorts_fwd[0])
    p.mask_output = tv.Tensor(mo, tv.uint32)
    ConvMainUnitTest(sync_check=True).implicit_gemm2(p)
    return pt, x, dy, mo


@pytest.mark.parametrize("split_k", [0, 1, 16, 74, 148])
def test_wgrad_split_k_same_result(layer, split_k):
    pt, x, dy, mo = layer
    ref_dw = torch.empty((64, 27, 64), dtype=torch.float32, device="cuda")
    run_wgrad(WgradConfig(0), x, dy, ref_dw, pt, mo)
    dw = torch.empty((64, 27, 64), dtype=torch.float32, device="cuda")
    run_wgrad(WgradConfig(split_k), x, dy, dw, pt, mo)
    torch.cuda.synchronize()
    nr, _, _ = co.rel_err(to64(dw), to64(ref_dw))
    assert nr <= 1e-6, nr
    ref = co.wgrad_gather_gemm_scatter(to64(dy), to64(x), pt.pairs_fwd.cpu().numpy())
    nr, mr, ma = co.rel_err(to64(dw), ref)
    assert nr <= 2e-5, (nr, mr, ma)


def test_tuner_picks_and_caches_split_k(layer):
    pt, x, dy, mo = layer
    tuner = ConvAutotuner(iters=2)
    dw = torch.empty((64, 27, 64), dtype=torch.float32, device="cuda")
    cfg = tuner.tune_wgrad(x.shape[0], 64, 64, 12, lambda c: run_wgrad(c, x, dy, dw, pt, mo))
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    assert cfg in wgrad_candidates(sms)
    assert len(tuner.last_timings) == 4
    again = tuner.tune_wgrad(x.shape[0], 64, 64, 12, lambda c: pytest.fail("re-tuned"))
    assert again == cfg
