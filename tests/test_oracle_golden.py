"""Pins the CPU oracle (oracle/) against the golden fixtures (dense conv3d in
float64, tests/golden/make_golden.py) and a brute-force pair enumeration."""
import itertools

import numpy as np
import pytest

from oracle import conv_oracle as co
from oracle import pairs_oracle as po

CASES = ["subm_k3", "subm_k3_batch2", "subm_k3_dil2", "subm_k311", "conv_s2", "conv_s2_batch2",
         "conv_k2s2"]


def _load(golden_dir, name):
    return dict(np.load(golden_dir / f"{name}.npz"))


def _pairs(g):
    coords = g["coords"]
    ks, st, pd, dl = (tuple(int(v) for v in g[k]) for k in ("ksize", "stride", "padding", "dilation"))
    if bool(g["subm"]):
        pf, pb, m = po.subm_pairs(coords, tuple(g["spatial"]), ks, dl)
        return coords, pf, pb, m, m
    out, pf, pb, mf, mb, _ = po.conv_pairs(coords, int(g["batch"]), tuple(g["spatial"]), ks, st, pd, dl)
    return out, pf, pb, mf, mb


@pytest.mark.parametrize("name", CASES)
def test_golden_gather_gemm_scatter(golden_dir, name):
    g = _load(golden_dir, name)
    out_coords, pf, pb, mf, mb = _pairs(g)
    assert np.array_equal(out_coords, g["out_coords"])
    out = co.fwd_gather_gemm_scatter(g["feats"], g["weight"], pf)
    np.testing.assert_allclose(out, g["out"], rtol=1e-10, atol=1e-10)
    din = co.dgrad_gather_gemm_scatter(g["grad_out"], g["weight"], pb)
    np.testing.assert_allclose(din, g["grad_in"], rtol=1e-10, atol=1e-10)
    dw = co.wgrad_gather_gemm_scatter(g["grad_out"], g["feats"], pf)
    np.testing.assert_allclose(dw, g["grad_w"], rtol=1e-10, atol=1e-10)


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("tile_m", [32, 128])
@pytest.mark.parametrize("num_split", [1, 2])
def test_golden_masked_semantics(golden_dir, name, tile_m, num_split):
    """The kernel-semantics oracle (sorted masks, tile masks, permuted store,
    split launches with beta=1) reproduces the dense conv."""
    g = _load(golden_dir, name)
    out_coords, pf, pb, mf, mb = _pairs(g)
    kv = pf.shape[0]
    subm = bool(g["subm"])
    n_out, n_in = pf.shape[1], pb.shape[1]
    out = None
    din = None
    dw = None
    for j, sm in enumerate(po.split_masks(kv, num_split)):
        ms, order = po.sort_by_key_split(mf, sm)
        out, mo = co.conv_fwd_masked(g["feats"], g["weight"], pf, ms, order, tile_m, sm,
                                     out_prev=out if j else None, beta=1.0 if j else 0.0)
        if subm:
            din = co.conv_dgrad_masked(g["grad_out"], g["weight"], pb, ms, order, tile_m, sm,
                                       True, din_prev=din if j else None, beta=1.0 if j else 0.0)
        else:
            msb, orderb = po.sort_by_key_split(mb, sm)
            din = co.conv_dgrad_masked(g["grad_out"], g["weight"], pb, msb, orderb, tile_m, sm,
                                       False, din_prev=din if j else None, beta=1.0 if j else 0.0)
        dw = co.conv_wgrad_masked(g["grad_out"], g["feats"], pf, mo, tile_m, order, kv, sm,
                                  dw_prev=dw if j else None, beta=1.0 if j else 0.0)
    np.testing.assert_allclose(out, g["out"], rtol=1e-10, atol=1e-10)
    np.testing.assert_allclose(din, g["grad_in"], rtol=1e-10, atol=1e-10)
    np.testing.assert_allclose(dw, g["grad_w"], rtol=1e-10, atol=1e-10)


def test_pairs_bruteforce():
    rng = np.random.default_rng(0)
    sp = (5, 6, 7)
    lin = np.sort(rng.choice(np.prod(sp), 60, replace=False))
    coords = np.stack([np.zeros_like(lin), lin // 42, (lin // 7) % 6, lin % 7], 1).astype(np.int32)
    pf, pb, m = po.subm_pairs(coords, sp)
    where = {tuple(c[1:]): i for i, c in enumerate(coords)}
    for i, c in enumerate(coords):
        for k, (a, b, d) in enumerate(itertools.product(range(3), range(3), range(3))):
            j = where.get((c[1] + a - 1, c[2] + b - 1, c[3] + d - 1), -1)
            assert pf[k, i] == j
            assert ((int(m[i]) >> k) & 1) == (j >= 0)
            if j >= 0:
                assert pb[k, j] == i
    # centre always present; dgrad mask = reversed fwd mask for submanifold convs
    assert np.all((m >> 13) & 1)
    mb = (pb >= 0).astype(np.int64)
    mb = (mb << np.arange(27)[:, None]).sum(0)
    assert np.array_equal(mb, co.brev_shift(m, 27))


def test_sort_split_stable():
    rng = np.random.default_rng(1)
    data = rng.integers(0, 1 << 27, 1000).astype(np.uint32)
    for sm in po.split_masks(27, 2):
        s, order = po.sort_by_key_split(data, sm)
        key = s.astype(np.int64) & sm
        assert np.all(np.diff(key) >= 0)
        assert np.array_equal(s, data[order])
        # stability: equal keys keep their original order
        for kval in np.unique(key)[:20]:
            idx = order[key == kval]
            assert np.all(np.diff(idx) > 0)


def test_permutation_invariance_and_adjoint():
    """Output does not depend on how ties of mask_argsort are ordered, and
    dgrad is the adjoint of fwd: <fwd(x), y> == <x, dgrad(y)>."""
    rng = np.random.default_rng(2)
    sp = (8, 9, 10)
    lin = np.sort(rng.choice(np.prod(sp), 200, replace=False))
    coords = np.stack([np.zeros_like(lin), lin // 90, (lin // 10) % 9, lin % 10], 1).astype(np.int32)
    pf, pb, m = po.subm_pairs(coords, sp)
    x = rng.standard_normal((200, 4))
    y = rng.standard_normal((200, 6))
    w = rng.standard_normal((6, 27, 4))
    ms, order = po.sort_by_key_split(m, 0xffffffff)
    out, _ = co.conv_fwd_masked(x, w, pf, ms, order, 64)
    perm = rng.permutation(200)
    out2, _ = co.conv_fwd_masked(x, w, pf, m[perm], perm.astype(np.int32), 64)
    np.testing.assert_allclose(out, out2, rtol=1e-12, atol=1e-12)
    din = co.conv_dgrad_masked(y, w, pb, ms, order, 64, reverse_mask=True)
    assert abs(np.sum(out * y) - np.sum(x * din)) < 1e-9 * max(1.0, abs(np.sum(out * y)))


def test_epilogue_ops():
    rng = np.random.default_rng(3)
    acc = rng.standard_normal((5, 4))
    prev = rng.standard_normal((10, 4))
    rows = np.array([1, 3, 5, 7, 9])
    v = co.epilogue(acc, rows, prev, 2.0, 0.5, co.ACT_LEAKY, 0.1)
    ref = 2.0 * acc + 0.5 * prev[rows]
    np.testing.assert_allclose(v, np.where(ref >= 0, ref, 0.1 * ref))
    scale = rng.standard_normal(4)
    bias = rng.standard_normal(4)
    v = co.epilogue(acc, rows, prev, 2.0, 0.5, co.ACT_RELU, scale=scale, bias=bias)
    np.testing.assert_allclose(v, np.maximum(scale * acc + 2.0 * bias + 0.5 * prev[rows], 0))


def test_subm_invariants_oracle_builder():
    """The oracle pair builder keeps the submanifold invariants the reference
    driver relies on (cumm/conv/main_real_spconv.py:79-105): centre bit set in
    every mask, identity centre column, pairs_bwd[k] == pairs_fwd[kv-1-k], and
    brev(mask) >> (32 - kv) marking exactly the pairs of pairs_bwd."""
    from cumm import voxelgen as vg
    coords = vg.lidar_voxels(6000, seed=3)
    for dil in (1, 2):
        pf, pb, m = po.subm_pairs(coords, vg.KITTI_SHAPE, dilation=(dil, dil, dil))
        kv = pf.shape[0]
        assert np.array_equal(pb, pf[::-1])
        assert np.array_equal(pf[kv // 2], np.arange(coords.shape[0], dtype=np.int32))
        assert np.all(m.astype(np.int64) & (1 << (kv // 2)))
        bits = ((m.astype(np.int64)[None, :] >> np.arange(kv)[:, None]) & 1).astype(bool)
        assert np.array_equal(bits, pf >= 0)
        rev = co.brev_shift(m, kv)
        bits_b = ((rev[None, :] >> np.arange(kv)[:, None]) & 1).astype(bool)
        assert np.array_equal(bits_b, pb >= 0)
