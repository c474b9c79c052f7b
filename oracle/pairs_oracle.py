"""CPU oracle of the indice-pair / mask builder and the split mask argsort.

TEST INFRASTRUCTURE ONLY (see oracle/conv_oracle.py).  The reference's builder
lives in spconv (SpconvOps.generate_subm_conv_inds / sort_1d_by_key_split,
called at cumm/conv/main_real_spconv.py:79-145), which is not part of the
reference tree and pins no version: its outputs are UNPINNED.  The semantics
restated here are the ones observable at those call sites (dense
[2, kv, N] pair layout with -1 fill, mask bit k <=> pair exists, centre bit
always set for submanifold convs, dgrad through reverse_mask) plus the
cross-correlation offset order of a dense conv3d, which tests/golden pins.
The algorithm is independent of the GPU one: sorted linear keys and binary
search instead of a hash table.
"""
from typing import List, Sequence, Tuple

import numpy as np


def _lin(b, z, y, x, shape) -> np.ndarray:
    return ((b.astype(np.int64) * shape[0] + z) * shape[1] + y) * shape[2] + x


def _lookup(keys_sorted: np.ndarray, order: np.ndarray, q: np.ndarray, valid: np.ndarray) -> np.ndarray:
    pos = np.searchsorted(keys_sorted, q)
    pos_c = np.minimum(pos, max(len(keys_sorted) - 1, 0))
    hit = valid & (pos < len(keys_sorted))
    if len(keys_sorted):
        hit &= keys_sorted[pos_c] == q
    else:
        hit &= False
    return np.where(hit, order[pos_c] if len(order) else -1, -1).astype(np.int32)


def offsets(ksize: Sequence[int]) -> List[Tuple[int, int, int]]:
    return [(a, c, d) for a in range(ksize[0]) for c in range(ksize[1]) for d in range(ksize[2])]


def subm_pairs(coords: np.ndarray, spatial: Sequence[int], ksize=(3, 3, 3), dilation=(1, 1, 1)):
    """Returns (pairs_fwd [kv, N], pairs_bwd [kv, N], mask [N] uint32)."""
    n = coords.shape[0]
    b, z, y, x = (coords[:, i].astype(np.int64) for i in range(4))
    keys = _lin(b, z, y, x, spatial)
    order = np.argsort(keys, kind="stable")
    ks = keys[order]
    offs = offsets(ksize)
    kv = len(offs)
    pf = np.full((kv, n), -1, np.int32)
    pb = np.full((kv, n), -1, np.int32)
    mask = np.zeros(n, np.int64)
    for k, (a, c, d) in enumerate(offs):
        zz = z + (a - ksize[0] // 2) * dilation[0]
        yy = y + (c - ksize[1] // 2) * dilation[1]
        xx = x + (d - ksize[2] // 2) * dilation[2]
        ok = (zz >= 0) & (yy >= 0) & (xx >= 0) & (zz < spatial[0]) & (yy < spatial[1]) & \
             (xx < spatial[2])
        j = _lookup(ks, order, _lin(b, zz, yy, xx, spatial), ok)
        pf[k] = j
        hit = j >= 0
        pb[k][j[hit]] = np.nonzero(hit)[0]
        mask |= hit.astype(np.int64) << k
    return pf, pb, mask.astype(np.uint32)


def conv_out_spatial(spatial, ksize, stride, padding, dilation) -> List[int]:
    return [(spatial[d] + 2 * padding[d] - dilation[d] * (ksize[d] - 1) - 1) // stride[d] + 1
            for d in range(3)]


def conv_pairs(coords: np.ndarray, batch: int, spatial, ksize=(3, 3, 3), stride=(2, 2, 2),
               padding=(1, 1, 1), dilation=(1, 1, 1)):
    """Strided sparse conv: returns (out_coords [n_out, 4] in ascending
    (batch, z, y, x) order, pairs_fwd [kv, n_out], pairs_bwd [kv, n_in],
    mask_fwd [n_out], mask_bwd [n_in], out_spatial)."""
    osp = conv_out_spatial(spatial, ksize, stride, padding, dilation)
    n = coords.shape[0]
    b, z, y, x = (coords[:, i].astype(np.int64) for i in range(4))
    offs = offsets(ksize)
    kv = len(offs)
    cand = np.full((kv, n), -1, np.int64)
    for k, (a, c, d) in enumerate(offs):
        tz = z + padding[0] - a * dilation[0]
        ty = y + padding[1] - c * dilation[1]
        tx = x + padding[2] - d * dilation[2]
        ok = (tz >= 0) & (ty >= 0) & (tx >= 0) & (tz % stride[0] == 0) & (ty % stride[1] == 0) & \
             (tx % stride[2] == 0)
        oz, oy, ox = tz // stride[0], ty // stride[1], tx // stride[2]
        ok &= (oz < osp[0]) & (oy < osp[1]) & (ox < osp[2])
        cand[k] = np.where(ok, _lin(b, oz, oy, ox, osp), -1)
    uk = np.unique(cand[cand >= 0])
    n_out = uk.shape[0]
    out = np.zeros((n_out, 4), np.int32)
    rem = uk.copy()
    out[:, 3] = rem % osp[2]
    rem //= osp[2]
    out[:, 2] = rem % osp[1]
    rem //= osp[1]
    out[:, 1] = rem % osp[0]
    out[:, 0] = rem // osp[0]
    pf = np.full((kv, n_out), -1, np.int32)
    pb = np.full((kv, n), -1, np.int32)
    mf = np.zeros(n_out, np.int64)
    mb = np.zeros(n, np.int64)
    for k in range(kv):
        ok = cand[k] >= 0
        o = np.searchsorted(uk, cand[k][ok]).astype(np.int32)
        i = np.nonzero(ok)[0].astype(np.int32)
        pb[k][i] = o
        pf[k][o] = i
        mb[i] |= 1 << k
        mf[o] |= 1 << k
    return out, pf, pb, mf.astype(np.uint32), mb.astype(np.uint32), osp


def sort_by_key_split(data: np.ndarray, split_mask: int) -> Tuple[np.ndarray, np.ndarray]:
    """Stable argsort of data by (data & split_mask); returns (sorted data, argsort)."""
    d = data.astype(np.int64) & 0xffffffff
    key = d & (int(split_mask) & 0xffffffff)
    order = np.argsort(key, kind="stable").astype(np.int32)
    return d[order].astype(np.uint32), order


def split_masks(kv: int, num_split: int) -> List[int]:
    if num_split == 1:
        return [0xffffffff]
    half = kv // 2 + 1
    return [(1 << half) - 1, ((1 << kv) - 1) & ~((1 << half) - 1)]
