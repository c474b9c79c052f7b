"""Standalone gather / scatter-add (GatherAll / ScatterAll, the reference's
cumm/gemm/gather.py:390-620) on the GPU: bit-exact against numpy / torch
indexing, the way the reference's own driver checks them
(cumm/gemm/main_real.py:776-860: c_ref = a[inds] for gather, c_ref[inds] = a
from zeros for scatter)."""
import numpy as np
import pytest
import torch

from cumm import tensorview as tv
from cumm.gemm.gather import GatherAll, ScatterAll

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", [torch.float32, torch.bfloat16, torch.float16, torch.uint8])
@pytest.mark.parametrize("m,k", [(64000, 128), (1000, 126), (777, 64), (5, 3), (0, 16)])
def test_gather_bit_exact(dtype, m, k):
    rng = np.random.default_rng(m + k)
    rows = max(m, 1)
    if dtype == torch.uint8:
        a = torch.from_numpy(rng.integers(0, 255, (rows, k)).astype(np.uint8))
    else:
        a = torch.from_numpy(rng.uniform(-2, 2, size=(rows, k)).astype(np.float32)).to(dtype)
    inds = rng.permutation(rows)[:m].astype(np.int32)
    g = GatherAll()
    row_bytes = k * a.element_size()
    ran = 0
    for bpa in (16, 8, 4):
        if row_bytes % bpa:
            continue
        c_d = torch.full((m, k), 7, dtype=dtype, device="cuda")
        g.gather(tv.Tensor(c_d), tv.Tensor(a.cuda()), tv.Tensor(torch.from_numpy(inds).cuda()),
                 bytes_per_access=bpa, num_threads=128, sync_check=True)
        ref = a[torch.from_numpy(inds).long()]
        assert torch.equal(c_d.cpu().view(torch.uint8), ref.contiguous().view(torch.uint8)), bpa
        ran += 1
    assert ran or row_bytes % 4


def test_gather_reference_keys_and_edge_indices():
    g = GatherAll()
    m, k = 4096, 64
    a = torch.randn(m, k, device="cuda")
    inds = torch.randperm(m, device="cuda").int()
    inds[7] = -1  # a zero row
    c = torch.empty(m, k, device="cuda")
    n = 0
    for p in g.get_all_gather_params():
        if not g.supported(p[2], k, tv.float32) or p[3] != 256 or p[0] != 4:
            continue
        c.fill_(3.0)
        g.gather(tv.Tensor(c), tv.Tensor(a), tv.Tensor(inds), *p, sync_check=True)
        ref = a[inds.clamp(min=0).long()]
        ref[7] = 0
        assert torch.equal(c, ref), p
        n += 1
    assert n >= 3
    with pytest.raises(RuntimeError, match="sutable"):
        g.gather(tv.Tensor(c), tv.Tensor(a), tv.Tensor(inds), 3, 64, 16, 256)
    bad = inds.clone()
    bad[100] = m + 5  # outside the input: reported, read as a zero row
    with pytest.raises(RuntimeError, match="device error"):
        g.gather(tv.Tensor(c), tv.Tensor(a), tv.Tensor(bad), sync_check=True)


@pytest.mark.parametrize("dtype", [torch.float32, torch.bfloat16, torch.float16])
@pytest.mark.parametrize("m,k", [(64000, 256), (3000, 64), (513, 40)])
def test_scatter_add_bit_exact(dtype, m, k):
    rng = np.random.default_rng(m * 3 + k)
    n_out = m + 1000
    a = torch.from_numpy(rng.uniform(-2, 2, size=(m, k)).astype(np.float32)).to(dtype)
    base = torch.from_numpy(rng.uniform(-2, 2, size=(n_out, k)).astype(np.float32)).to(dtype)
    inds = rng.permutation(n_out)[:m].astype(np.int32)
    inds[3] = -1  # skipped
    out = base.cuda()
    ScatterAll().scatter(tv.Tensor(out), tv.Tensor(a.cuda()), tv.Tensor(torch.from_numpy(inds).cuda()),
                         sync_check=True)
    ref = base.clone()
    keep = inds >= 0
    ii = torch.from_numpy(inds[keep]).long()
    src = torch.from_numpy(np.nonzero(keep)[0])
    ref[ii] = (base[ii].float() + a[src].float()).to(dtype)
    assert torch.equal(out.cpu().view(torch.uint8), ref.view(torch.uint8))


def test_scatter_reference_form():
    """The reference driver's check: scatter into zeros equals c_ref[inds] = a
    (cumm/gemm/main_real.py:846-860)."""
    m, k = 64000, 256
    rng = np.random.default_rng(12315)
    a = rng.uniform(-2, 2, size=[m, k]).astype(np.float32)
    inds = np.arange(m, dtype=np.int32)
    rng.shuffle(inds)
    c_ref = np.zeros_like(a)
    c_ref[inds] = a
    s = ScatterAll()
    n = 0
    for p in s.get_all_scatter_params():
        if not s.supported_scatter(*p, k, tv.float32) or p[0] != 8:
            continue
        c = torch.zeros(m, k, device="cuda")
        s.scatter(tv.Tensor(c), tv.Tensor(torch.from_numpy(a).cuda()),
                  tv.Tensor(torch.from_numpy(inds).cuda()), *p, sync_check=True)
        assert np.array_equal(c.cpu().numpy(), c_ref), p
        n += 1
    assert n >= 3
