"""GPU pair / mask builder and split argsort: bit-exact against the CPU oracle."""
import numpy as np
import pytest
import torch

from cumm import voxelgen as vg
from cumm.spconv_ops import SpconvOps, build_pair_table
from oracle import conv_oracle as co
from oracle import pairs_oracle as po

pytestmark = pytest.mark.gpu


def _u(t):
    return t.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("n,seed", [(1000, 0), (20000, 1), (200000, 2)])
def test_subm_pairs_bit_exact(n, seed):
    coords = vg.lidar_voxels(n, seed=seed) if n >= 20000 else vg.uniform_voxels(n, 32, seed)
    spatial = vg.KITTI_SHAPE if n >= 20000 else (32, 32, 32)
    pt = build_pair_table(torch.from_numpy(coords).cuda(), spatial, num_split=2)
    pf, pb, m = po.subm_pairs(coords, spatial)
    assert np.array_equal(pt.pairs_fwd.cpu().numpy(), pf)
    assert np.array_equal(pt.pairs_bwd.cpu().numpy(), pb)
    for j, sm in enumerate(po.split_masks(27, 2)):
        ms, order = po.sort_by_key_split(m, sm)
        assert np.array_equal(pt.argsorts_fwd[j].cpu().numpy(), order)
        assert np.array_equal(_u(pt.masks_fwd[j]), ms)


def test_uniform_20k_64cube():
    coords = vg.uniform_voxels(20000, 64, 0)
    pt = build_pair_table(torch.from_numpy(coords).cuda(), (64, 64, 64))
    pf, pb, m = po.subm_pairs(coords, (64, 64, 64))
    assert np.array_equal(pt.pairs_fwd.cpu().numpy(), pf)
    ms, order = po.sort_by_key_split(m, 0xffffffff)
    assert np.array_equal(pt.argsorts_fwd[0].cpu().numpy(), order)
    assert np.array_equal(_u(pt.masks_fwd[0]), ms)


@pytest.mark.parametrize("n,seed,batch", [(3000, 3, 1), (200000, 4, 1), (5000, 5, 3)])
def test_strided_pairs_bit_exact(n, seed, batch):
    if batch == 1:
        coords = vg.lidar_voxels(n, seed=seed)
    else:
        coords = np.concatenate([vg.lidar_voxels(n // batch, seed=seed + b, batch=b)
                                 for b in range(batch)], 0)
    spatial = vg.KITTI_SHAPE
    pt = build_pair_table(torch.from_numpy(coords).cuda(), spatial, stride=(2, 2, 2),
                          padding=(1, 1, 1), subm=False, batch_size=batch)
    out, pf, pb, mf, mb, osp = po.conv_pairs(coords, batch, spatial)
    assert pt.out_spatial == osp
    assert np.array_equal(pt.out_inds.cpu().numpy(), out)
    assert np.array_equal(pt.pairs_fwd.cpu().numpy(), pf)
    assert np.array_equal(pt.pairs_bwd.cpu().numpy(), pb)
    ms, order = po.sort_by_key_split(mf, 0xffffffff)
    assert np.array_equal(pt.argsorts_fwd[0].cpu().numpy(), order)
    msb, orderb = po.sort_by_key_split(mb, 0xffffffff)
    assert np.array_equal(pt.argsorts_bwd[0].cpu().numpy(), orderb)
    assert np.array_equal(_u(pt.masks_bwd[0]), msb)


def test_sort_large_keys_stable():
    rng = np.random.default_rng(7)
    data = rng.integers(0, 1 << 27, 300001).astype(np.uint32)
    t = torch.from_numpy(data.view(np.int32)).cuda()
    for sm in (0xffffffff, 0b111, 0b1111111111111 << 14):
        tt = t.clone()
        order = SpconvOps.sort_1d_by_key_split(tt, sm)
        s, o = po.sort_by_key_split(data, sm)
        assert np.array_equal(order.cpu().numpy(), o)
        assert np.array_equal(tt.cpu().numpy().view(np.uint32), s)


@pytest.mark.parametrize("n,seed,dil", [(20000, 6, 1), (5000, 7, 2)])
def test_subm_invariants_the_reference_caller_relies_on(n, seed, dil):
    """Properties of a submanifold pair table that the reference's driver
    depends on (cumm/conv/main_real_spconv.py:79-105): every voxel is its own
    centre neighbour, so the centre bit 1 << (kv // 2) is set in every mask
    (the driver seeds the split masks with it, :83-84) and the centre column
    is the identity; the table is symmetric, pairs_bwd[k] == pairs_fwd[kv-1-k]
    (offset k from an output is offset kv-1-k from its input, which is what
    lets backward-input reuse the forward's masks with reverse_mask); and the
    mask bit k is set exactly where pairs_fwd[k] != -1."""
    coords = vg.lidar_voxels(n, seed=seed)
    pt = build_pair_table(torch.from_numpy(coords).cuda(), vg.KITTI_SHAPE,
                          dilation=(dil, dil, dil))
    pf = pt.pairs_fwd.cpu().numpy()
    pb = pt.pairs_bwd.cpu().numpy()
    kv = pf.shape[0]
    assert kv == 27
    assert np.array_equal(pb, pf[::-1])
    assert np.array_equal(pf[kv // 2], np.arange(n, dtype=np.int32))
    order = pt.argsorts_fwd[0].cpu().numpy()
    ms = _u(pt.masks_fwd[0])
    assert np.all(ms & np.uint32(1 << (kv // 2)))
    m = np.zeros(n, np.uint32)
    m[order] = ms
    bits = ((m[None, :] >> np.arange(kv, dtype=np.uint32)[:, None]) & 1).astype(bool)
    assert np.array_equal(bits, pf >= 0)
    # the reverse-mask relation: brev(mask) >> (32 - kv) is the mask of pairs_bwd
    rev = co.brev_shift(m, kv)
    bits_b = ((rev[None, :] >> np.arange(kv, dtype=np.int64)[:, None]) & 1).astype(bool)
    assert np.array_equal(bits_b, pb >= 0)
