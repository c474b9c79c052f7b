"""Grouped forward of several clouds (one pair build + one conv launch per mask
split, captured in a CUDA graph) against each cloud run alone and the oracle."""
import numpy as np
import pytest
import torch

from cumm import voxelgen as vg
from cumm.autotune import ConvAutotuner, FwdConfig, run_forward
from cumm.batch import GroupedSubmConv
from cumm.spconv_ops import build_pair_table
from oracle import conv_oracle as co
from tests.helpers import to64

pytestmark = pytest.mark.gpu

SIZES = [3000, 7000, 1500, 9000, 500]


@pytest.fixture(scope="module")
def clouds():
    coords = [torch.from_numpy(vg.lidar_voxels(n, seed=40 + i)).cuda() for i, n in enumerate(SIZES)]
    rng = np.random.default_rng(4)
    feats = [torch.from_numpy(rng.standard_normal((n, 64)).astype(np.float32)).cuda().bfloat16()
             for n in SIZES]
    w = torch.from_numpy(vg.kaiming_uniform(64, 27, 64, 4)).cuda().bfloat16()
    alone = []
    for c, x in zip(coords, feats):
        out = torch.empty((x.shape[0], 64), dtype=torch.bfloat16, device="cuda")
        run_forward(FwdConfig(1, 0), x, w, out, {1: build_pair_table(c, vg.KITTI_SHAPE)})
        alone.append(out)
    torch.cuda.synchronize()
    return coords, feats, w, alone


@pytest.mark.parametrize("cfg", [FwdConfig(1, 0), FwdConfig(2, 0), FwdConfig(1, 32)])
def test_grouped_graph_matches_alone(clouds, cfg):
    coords, feats, w, alone = clouds
    tuner = ConvAutotuner()
    g = GroupedSubmConv(coords, vg.KITTI_SHAPE, w, tuner=tuner)
    g.cfg = cfg
    y1 = g(torch.cat(feats, 0)).clone()
    y2 = g().clone()  # replay with the same inputs
    assert torch.equal(y1, y2)
    for yi, ai in zip(g.split(y1), alone):
        if cfg.num_split == 1:
            # same rows, same offsets in the same order: bit-identical to the cloud alone
            assert torch.equal(yi, ai)
        else:
            # two launches round the partial sum to bf16 once more
            nr, _, _ = co.rel_err(to64(yi), to64(ai))
            assert nr <= 4e-3


def test_grouped_vs_oracle_and_tuner(clouds):
    coords, feats, w, alone = clouds
    tuner = ConvAutotuner(iters=2)
    g = GroupedSubmConv(coords, vg.KITTI_SHAPE, w, tuner=tuner)
    cfg = g.tune()
    assert cfg in {FwdConfig(1, 0), FwdConfig(2, 0), FwdConfig(1, 32)}
    assert set(tuner.last_timings) == {"split1_tnauto", "split2_tnauto", "split1_tn32"}
    y = g(torch.cat(feats, 0))
    torch.cuda.synchronize()
    pt = g.tables[cfg.num_split]
    ref = co.fwd_gather_gemm_scatter(to64(torch.cat(feats, 0)), to64(w), pt.pairs_fwd.cpu().numpy())
    nr, mr, ma = co.rel_err(to64(y), ref)
    assert nr <= 2e-3, (nr, mr, ma)
    # no pair crosses a cloud boundary
    pf = pt.pairs_fwd.cpu().numpy()
    owner = np.repeat(np.arange(len(SIZES)), SIZES)
    rows = np.nonzero(pf >= 0)
    assert (owner[pf[rows]] == owner[rows[1]]).all()
