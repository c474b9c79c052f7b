"""Generates the golden fixtures that pin the CPU oracle.

The reference has no golden vectors for this path and cannot run here, so the
fixtures come from an independent evaluation of the same operator: dense
torch.nn.functional.conv3d (cross-correlation) in float64 on the voxel grid,
with features scattered to the active sites and, for the backward passes, the
upstream gradient zero outside the active output sites.  A submanifold conv
equals that dense conv read back at the active sites; a strided sparse conv
equals it read back at every output site whose window holds an active input.

Run:  python tests/golden/make_golden.py   (writes tests/golden/*.npz)
"""
from pathlib import Path

import numpy as np
import torch
import torch.nn.functional as F

HERE = Path(__file__).resolve().parent


def _dense_case(name, coords, spatial, batch, C, K, ksize, stride, padding, dilation, subm, seed):
    rng = np.random.default_rng(seed)
    n = coords.shape[0]
    kv = int(np.prod(ksize))
    feats = rng.standard_normal((n, C))
    weight = rng.uniform(-0.5, 0.5, (K, kv, C))
    w_t = torch.from_numpy(weight.reshape(K, *ksize, C)).permute(0, 4, 1, 2, 3).contiguous()
    x = torch.zeros((batch, C, *spatial), dtype=torch.float64)
    b, z, y, xx = (torch.from_numpy(coords[:, i].astype(np.int64)) for i in range(4))
    x[b, :, z, y, xx] = torch.from_numpy(feats)
    x.requires_grad_(True)
    w_t.requires_grad_(True)
    out = F.conv3d(x, w_t, stride=stride, padding=padding, dilation=dilation)
    if subm:
        out_coords = coords
    else:
        # active output sites: windows holding at least one active input
        occ = torch.zeros((batch, 1, *spatial), dtype=torch.float64)
        occ[b, 0, z, y, xx] = 1.0
        ones = torch.ones((1, 1, *ksize), dtype=torch.float64)
        hit = F.conv3d(occ, ones, stride=stride, padding=padding, dilation=dilation)[:, 0] > 0
        out_coords = torch.nonzero(hit).numpy().astype(np.int32)  # sorted (b, z, y, x)
    ob, oz, oy, ox = (torch.from_numpy(out_coords[:, i].astype(np.int64)) for i in range(4))
    out_sparse = out[ob, :, oz, oy, ox]
    g_sparse = torch.from_numpy(rng.standard_normal(out_sparse.shape))
    g = torch.zeros_like(out)
    g[ob, :, oz, oy, ox] = g_sparse
    (out * g).sum().backward()
    grad_in = x.grad[b, :, z, y, xx]
    grad_w = w_t.grad.permute(0, 2, 3, 4, 1).reshape(K, kv, C)
    np.savez_compressed(
        HERE / f"{name}.npz", coords=coords, spatial=np.array(spatial), batch=batch,
        ksize=np.array(ksize), stride=np.array(stride), padding=np.array(padding),
        dilation=np.array(dilation), subm=subm, feats=feats, weight=weight,
        out_coords=out_coords, out=out_sparse.detach().numpy(), grad_out=g_sparse.numpy(),
        grad_in=grad_in.detach().numpy(), grad_w=grad_w.detach().numpy())


def _coords(n, spatial, batch, seed):
    rng = np.random.default_rng(seed)
    per = int(np.prod(spatial))
    lin = np.sort(rng.choice(per * batch, n, replace=False))
    b = lin // per
    r = lin % per
    z = r // (spatial[1] * spatial[2])
    y = (r // spatial[2]) % spatial[1]
    x = r % spatial[2]
    return np.stack([b, z, y, x], 1).astype(np.int32)


def main():
    sp = (10, 12, 14)
    _dense_case("subm_k3", _coords(300, sp, 1, 1), sp, 1, 8, 16, (3, 3, 3), (1, 1, 1),
                (1, 1, 1), (1, 1, 1), True, 11)
    _dense_case("subm_k3_batch2", _coords(400, sp, 2, 2), sp, 2, 16, 8, (3, 3, 3), (1, 1, 1),
                (1, 1, 1), (1, 1, 1), True, 12)
    _dense_case("subm_k3_dil2", _coords(250, sp, 1, 3), sp, 1, 8, 8, (3, 3, 3), (1, 1, 1),
                (2, 2, 2), (2, 2, 2), True, 13)
    _dense_case("subm_k311", _coords(200, sp, 1, 4), sp, 1, 8, 16, (3, 1, 1), (1, 1, 1),
                (1, 0, 0), (1, 1, 1), True, 14)
    _dense_case("conv_s2", _coords(300, sp, 1, 5), sp, 1, 8, 16, (3, 3, 3), (2, 2, 2),
                (1, 1, 1), (1, 1, 1), False, 15)
    _dense_case("conv_s2_batch2", _coords(350, (9, 11, 13), 2, 6), (9, 11, 13), 2, 8, 8,
                (3, 3, 3), (2, 2, 2), (1, 1, 1), (1, 1, 1), False, 16)
    _dense_case("conv_k2s2", _coords(300, sp, 1, 7), sp, 1, 8, 8, (2, 2, 2), (2, 2, 2),
                (0, 0, 0), (1, 1, 1), False, 17)


if __name__ == "__main__":
    main()
