"""GemmMainUnitTest.matmul2 parity (NoShuffle / ShuffleAC / ShuffleAB) against
the FP64 oracle, mirroring cumm/gemm/main_real.py:193-229."""
import numpy as np
import pytest
import torch

from cumm import tensorview as tv
from cumm.gemm.main import GemmMainUnitTest, get_all_algo_desp
from cumm.tensorview.gemm import GemmParams, ShuffleStrideType
from oracle import conv_oracle as co

pytestmark = pytest.mark.gpu


def _desp(algo, dt, dc, ta, tb, st):
    for d in get_all_algo_desp():
        if (d.algo == algo and d.dtype_a == dt and d.dtype_c == dc and d.trans_a == ta and
                d.trans_b == tb and d.shuffle_type == st):
            return d
    raise KeyError


def _t(x, dt):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda().to(dt)


def _run(desp, a, b, c, d=None, a_inds=None, b_inds=None, c_inds=None, alpha=1.0, beta=0.0, act=0,
         split_k=1):
    p = GemmParams()
    p.split_k_slices = split_k
    p.algo_desp = desp
    p.a, p.b, p.c = tv.Tensor(a), tv.Tensor(b), tv.Tensor(c)
    if d is not None:
        p.d = tv.Tensor(d)
    for name, v in (("a_inds", a_inds), ("b_inds", b_inds), ("c_inds", c_inds)):
        if v is not None:
            setattr(p, name, tv.Tensor(torch.from_numpy(v.astype(np.int32)).cuda()))
    p.alpha, p.beta, p.act_type = alpha, beta, act
    GemmMainUnitTest(sync_check=True).matmul2(p)


def _f64(t):
    return t.float().cpu().numpy().astype(np.float64)


@pytest.mark.parametrize("dt,dc", [(torch.bfloat16, torch.bfloat16), (torch.float16, torch.float32)])
@pytest.mark.parametrize("ta,tb", [(False, False), (False, True), (True, False), (True, True)])
@pytest.mark.parametrize("m,n,k", [(1000, 128, 256), (300, 64, 96), (64, 256, 1000)])
def test_dense(dt, dc, ta, tb, m, n, k):
    rng = np.random.default_rng(m + n + k)
    a = rng.standard_normal((k, m) if ta else (m, k)).astype(np.float32)
    b = rng.standard_normal((n, k) if tb else (k, n)).astype(np.float32)
    at, bt = _t(a, dt), _t(b, dt)
    c = torch.zeros((m, n), dtype=dc, device="cuda")
    tvd = {torch.bfloat16: tv.bfloat16, torch.float16: tv.float16, torch.float32: tv.float32}
    desp = _desp("Tcgen05", tvd[dt], tvd[dc], ta, tb, ShuffleStrideType.kNoShuffle)
    if not desp.supported(m, n, k):
        # misaligned contiguous dimension: rejected like the reference prologue
        with pytest.raises(ValueError, match="misaligned"):
            _run(desp, at, bt, c)
        return
    _run(desp, at, bt, c)
    ref = co.gemm(_f64(at), _f64(bt), ta, tb)
    nr, _, _ = co.rel_err(_f64(c), ref)
    assert nr < 2e-3


def test_shuffle_ac_and_ab():
    rng = np.random.default_rng(0)
    m_rows, k, n = 5000, 128, 64
    a = rng.standard_normal((m_rows, k)).astype(np.float32)
    b = rng.standard_normal((k, n)).astype(np.float32)
    a_inds = rng.choice(m_rows, 3000, replace=False)
    c_inds = rng.choice(4000, 3000, replace=False)
    at, bt = _t(a, torch.bfloat16), _t(b, torch.bfloat16)
    c = torch.zeros((4000, n), dtype=torch.bfloat16, device="cuda")
    _run(_desp("Tcgen05", tv.bfloat16, tv.bfloat16, False, False, ShuffleStrideType.kShuffleAC),
         at, bt, c, a_inds=a_inds, c_inds=c_inds)
    ref = co.gemm(_f64(at), _f64(bt), shuffle=1, a_inds=a_inds, c_inds=c_inds,
                  c_prev=np.zeros((4000, n)))
    assert co.rel_err(_f64(c), ref)[0] < 2e-3
    # ShuffleAB: C = A[a_inds]^T B[b_inds] (the native wgrad)
    K_out, C_in = 64, 128
    do = _t(rng.standard_normal((m_rows, K_out)).astype(np.float32), torch.bfloat16)
    xi = _t(rng.standard_normal((m_rows, C_in)).astype(np.float32), torch.bfloat16)
    ai = rng.choice(m_rows, 2500, replace=False)
    bi = rng.choice(m_rows, 2500, replace=False)
    c2 = torch.zeros((K_out, C_in), dtype=torch.float32, device="cuda")
    _run(_desp("Tcgen05", tv.bfloat16, tv.float32, True, False, ShuffleStrideType.kShuffleAB),
         do, xi, c2, a_inds=ai, b_inds=bi)
    ref2 = co.gemm(_f64(do), _f64(xi), shuffle=2, a_inds=ai, b_inds=bi)
    assert co.rel_err(_f64(c2), ref2)[0] < 2e-3


def test_simt_fp32_and_epilogue():
    rng = np.random.default_rng(1)
    m, n, k = 257, 65, 129
    a = rng.standard_normal((m, k)).astype(np.float32)
    b = rng.standard_normal((k, n)).astype(np.float32)
    d = rng.standard_normal(n).astype(np.float32)
    at, bt, dt_ = _t(a, torch.float32), _t(b, torch.float32), _t(d, torch.float32)
    c = torch.zeros((m, n), device="cuda")
    _run(_desp("Simt", tv.float32, tv.float32, False, False, ShuffleStrideType.kNoShuffle), at, bt,
         c, d=dt_, alpha=0.5, beta=2.0, act=1)
    ref = co.gemm(a, b, d=d, alpha=0.5, beta=2.0, act_type=1)
    assert co.rel_err(_f64(c), ref)[0] < 1e-5


TVD = {torch.bfloat16: tv.bfloat16, torch.float16: tv.float16, torch.float32: tv.float32}


@pytest.mark.parametrize("ta,tb", [(False, False), (False, True), (True, False), (True, True)])
@pytest.mark.parametrize("m,n,k,split", [(333, 200, 200, 1), (128, 256, 64, 1), (1, 8, 8, 1),
                                         (517, 520, 1000, 3), (256, 512, 4096, 8), (100, 48, 40, 4)])
def test_dense_tcgen05_shapes_and_split_k(ta, tb, m, n, k, split):
    """The dense tcgen05 GEMM (2-D TMA tiles of 128 x 256, K blocks of 64,
    either operand read in place K- or MN-major): ragged m / n / k (TMA zero
    fill, guarded stores) and parallel split-K into an fp32 workspace."""
    rng = np.random.default_rng(m * 7 + n + k + split)
    a = rng.standard_normal((k, m) if ta else (m, k)).astype(np.float32)
    b = rng.standard_normal((n, k) if tb else (k, n)).astype(np.float32)
    at, bt = _t(a, torch.bfloat16), _t(b, torch.bfloat16)
    c = torch.full((m, n), 5.0, dtype=torch.float32, device="cuda")
    desp = _desp("Tcgen05", tv.bfloat16, tv.float32, ta, tb, ShuffleStrideType.kNoShuffle)
    if not desp.supported(m, n, k):
        pytest.skip("contiguous dimension not a multiple of 8 elements (reference rejects it)")
    _run(desp, at, bt, c, split_k=split)
    ref = co.gemm(_f64(at), _f64(bt), ta, tb)
    nr, mr, _ = co.rel_err(_f64(c), ref)
    assert nr < 1e-5 if split == 1 else nr < 2e-5, (nr, mr)


@pytest.mark.parametrize("split", [1, 4])
@pytest.mark.parametrize("dc", [torch.bfloat16, torch.float16, torch.float32])
def test_dense_tcgen05_epilogue(split, dc):
    """act(alpha * A B + beta * D) with D a matrix or a [n] bias, on both the
    direct epilogue and the split-K finalize pass."""
    rng = np.random.default_rng(3)
    m, n, k = 300, 320, 256
    dt = torch.float16 if dc == torch.float16 else torch.bfloat16
    at = _t(rng.standard_normal((m, k)).astype(np.float32), dt)
    bt = _t(rng.standard_normal((k, n)).astype(np.float32), dt)
    desp = _desp("Tcgen05", TVD[dt], TVD[dc], False, False, ShuffleStrideType.kNoShuffle)
    dm = rng.standard_normal((m, n)).astype(np.float32)
    bias = rng.standard_normal(n).astype(np.float32)
    for d, act in ((dm, 1), (bias, 3), (None, 2)):
        c = torch.zeros((m, n), dtype=dc, device="cuda")
        dd = None if d is None else _t(d, dc)
        _run(desp, at, bt, c, d=dd, alpha=0.5, beta=1.5 if d is not None else 0.0, act=act, split_k=split)
        ref = co.gemm(_f64(at), _f64(bt), d=None if d is None else _f64(dd), alpha=0.5,
                      beta=1.5 if d is not None else 0.0, act_type=act)
        assert co.rel_err(_f64(c), ref)[0] < (2e-3 if dc != torch.float32 else 1e-5), (act, split)


def test_dense_trans_c_and_shuffle_ab_split_k():
    """trans_c (C stored transposed: the operands swap, cumm/gemm/nvrtc_code.py
    prologue) and split-K on ShuffleAB (row splits of the reduction-gather
    kernel)."""
    rng = np.random.default_rng(4)
    m, n, k = 200, 136, 512
    at = _t(rng.standard_normal((m, k)).astype(np.float32), torch.bfloat16)
    bt = _t(rng.standard_normal((k, n)).astype(np.float32), torch.bfloat16)
    d = GemmMainUnitTest.get_all_algo_desp()
    desp = [x for x in d if x.algo == "Tcgen05" and x.dtype_a == tv.bfloat16 and x.dtype_c == tv.float32
            and not x.trans_a and not x.trans_b and x.shuffle_type == ShuffleStrideType.kNoShuffle][0]
    import copy
    desp_c = copy.copy(desp)
    desp_c.trans_c = True
    ct = torch.zeros((n, m), dtype=torch.float32, device="cuda")
    _run(desp_c, at, bt, ct)
    ref = co.gemm(_f64(at), _f64(bt))
    assert co.rel_err(_f64(ct).T, ref)[0] < 1e-5
    m_rows, K_out, C_in = 6000, 64, 128
    do = _t(rng.standard_normal((m_rows, K_out)).astype(np.float32), torch.bfloat16)
    xi = _t(rng.standard_normal((m_rows, C_in)).astype(np.float32), torch.bfloat16)
    ai = rng.choice(m_rows, 5000, replace=False)
    bi = rng.choice(m_rows, 5000, replace=False)
    ref2 = co.gemm(_f64(do), _f64(xi), shuffle=2, a_inds=ai, b_inds=bi)
    for split in (1, 16, 64):
        c2 = torch.zeros((K_out, C_in), dtype=torch.float32, device="cuda")
        _run(_desp("Tcgen05", tv.bfloat16, tv.float32, True, False, ShuffleStrideType.kShuffleAB),
             do, xi, c2, a_inds=ai, b_inds=bi, split_k=split)
        assert co.rel_err(_f64(c2), ref2)[0] < 2e-5, split
    # ShuffleAC has no split-K (the reference's message)
    c3 = torch.zeros((4000, n), dtype=torch.bfloat16, device="cuda")
    with pytest.raises(RuntimeError, match="splitk"):
        _run(_desp("Tcgen05", tv.bfloat16, tv.bfloat16, False, False, ShuffleStrideType.kShuffleAC), at, bt, c3,
             a_inds=rng.choice(m, 100, replace=False), c_inds=rng.choice(4000, 100, replace=False), split_k=2)
