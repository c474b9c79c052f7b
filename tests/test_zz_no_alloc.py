"""sc_conv_wgrad_static_scratch: backward weight with the library's static
device scratch instead of a caller workspace, checked against
sc_conv_implicit_gemm (the entry point that takes a workspace) through the
C ABI.  Two calls in a row with different gradients: the second result shows
the scratch was cleared between calls."""
import ctypes

import numpy as np
import pytest
import torch

from cumm import _lib
from cumm import tensorview as tv
from cumm import voxelgen as vg
from cumm.conv.main import build_conv_params_c
from cumm.tensorview.gemm import ConvOpType, ConvParams
from oracle import conv_oracle as co
from oracle import pairs_oracle as po
from tests.helpers import dev, find_desp, i32, to64, u32

MAX_FLOATS = 1 << 21


def _wgrad_params(x, dw, dy, pf, mo, order, beta=0.0, mask_filter=0xffffffff):
    desp = find_desp(ConvOpType.kBackwardWeight, "Tcgen05", tv.bfloat16,
                     tv.float32 if dw.dtype == torch.float32 else tv.bfloat16, tv.bfloat16, 128)
    p = ConvParams(3, ConvOpType.kBackwardWeight)
    p.conv_algo_desp = desp
    p.input = tv.Tensor(x, desp.dtype_input)
    p.weight = tv.Tensor(dw, desp.dtype_weight)
    p.output = tv.Tensor(dy, desp.dtype_output)
    p.indices = i32(pf)
    p.mask = u32(mo)
    p.mask_argsort = i32(order)
    p.mask_width = 128
    p.beta = beta
    p.mask_filter = mask_filter
    cp, _ = build_conv_params_c(p)
    cp.flags |= _lib.SC_FLAG_SYNC_CHECK
    return cp, p


def _with_workspace(x, dw, dy, pf, mo, order, **kw):
    lib = _lib.load()
    cp, keep = _wgrad_params(x, dw, dy, pf, mo, order, **kw)
    need = ctypes.c_int64(0)
    _lib.check(lib.sc_conv_workspace_size(ctypes.byref(cp), ctypes.byref(need)))
    ws = torch.empty(need.value, dtype=torch.uint8, device="cuda")
    cp.workspace = ws.data_ptr()
    cp.workspace_bytes = ws.numel()
    _lib.check(lib.sc_conv_implicit_gemm(ctypes.byref(cp)))
    torch.cuda.synchronize()


def _static(x, dw, dy, pf, mo, order, **kw):
    lib = _lib.load()
    cp, keep = _wgrad_params(x, dw, dy, pf, mo, order, **kw)
    _lib.check(lib.sc_conv_wgrad_static_scratch(ctypes.byref(cp)))
    torch.cuda.synchronize()


def _fake_params(op, C, K, kv, n=1000):
    """Params with non-null dummy pointers: the checks under test run before
    any device access."""
    cp = _lib.ConvParamsC()
    cp.op_type = int(op)
    cp.algo = _lib.SC_ALGO_TCGEN05
    cp.dtype_input = cp.dtype_output = tv.bfloat16
    cp.dtype_weight = tv.float32
    cp.tile_m, cp.tile_k, cp.kv = 128, 32, kv
    cp.n_in = cp.n_out = cp.N = n
    cp.C, cp.K = C, K
    cp.input = cp.weight = cp.output = cp.indices = cp.mask = cp.mask_argsort = 0x1000
    cp.mask_count = n
    cp.mask_filter = 0xffffffff
    cp.mask_width = 128
    cp.alpha = 1.0
    return cp


def test_static_scratch_rejects_without_device_work():
    lib = _lib.load()
    # 256 * 27 * 320 floats > 2**21
    cp = _fake_params(ConvOpType.kBackwardWeight, 320, 256, 27)
    assert lib.sc_conv_wgrad_static_scratch(ctypes.byref(cp)) == _lib.SC_INVALID_ARG
    assert b"exceeds the static wgrad scratch" in lib.sc_last_error()
    cp = _fake_params(ConvOpType.kForward, 64, 64, 27)
    assert lib.sc_conv_wgrad_static_scratch(ctypes.byref(cp)) == _lib.SC_INVALID_ARG
    cp = _fake_params(ConvOpType.kBackwardWeight, 64, 64, 27)
    cp.workspace = 0x2000
    cp.workspace_bytes = 1 << 20
    assert lib.sc_conv_wgrad_static_scratch(ctypes.byref(cp)) == _lib.SC_INVALID_ARG


# Routes through the entry point: an fp32 dW with alpha 1, beta 0 and every
# offset selected accumulates in dW itself ("direct"); beta != 0 from a
# nonzero dW, or a mask_filter that leaves an offset out, accumulates in the
# static scratch and finalizes into dW ("beta", "filter").  bf16 dW always
# goes through the scratch.
ROUTES = {"direct": dict(), "beta": dict(beta=0.5), "filter": dict(mask_filter=0xffffffff & ~(1 << 13))}


@pytest.mark.gpu
@pytest.mark.parametrize("dw_dt,route", [(torch.float32, "direct"), (torch.float32, "beta"),
                                         (torch.float32, "filter"), (torch.bfloat16, "direct"),
                                         (torch.bfloat16, "beta")])
@pytest.mark.parametrize("n,grid,C,K", [(3000, 24, 64, 64), (900, 12, 128, 64), (700, 12, 16, 16)])
def test_static_scratch_matches_workspace_entry(dw_dt, route, n, grid, C, K):
    assert K * 27 * C <= MAX_FLOATS
    kw = ROUTES[route]
    coords = vg.uniform_voxels(n, grid, n + 11)
    pf, pb, m = po.subm_pairs(coords, (grid, grid, grid))
    ms, order = po.sort_by_key_split(m, 0xffffffff)
    mo = co.tile_masks(ms, 128).astype(np.uint32)
    rng = np.random.default_rng(n)
    x = dev(rng.standard_normal((n, C)).astype(np.float32), torch.bfloat16)
    dys = [dev(rng.standard_normal((n, K)).astype(np.float32), torch.bfloat16) for _ in range(2)]
    # the starting dW: zero for beta 0 and every offset selected, else nonzero
    # (beta reads it; offsets outside mask_filter must keep it)
    start = torch.zeros((K, 27, C), dtype=dw_dt, device="cuda") if route == "direct" else \
        dev(rng.standard_normal((K, 27, C)).astype(np.float32), dw_dt)
    refs = []
    for dy in dys:
        dw_ref = start.clone()
        _with_workspace(x, dw_ref, dy, pf, mo, order, **kw)
        refs.append(dw_ref)
    # two static-scratch calls back to back
    outs = [start.clone() for _ in range(2)]
    for dy, dw in zip(dys, outs):
        _static(x, dw, dy, pf, mo, order, **kw)
    for call, (dy, dw, dw_ref) in enumerate(zip(dys, outs, refs)):
        # fp32 atomics may add the per-CTA partial sums in another order
        nr, mr, ma = co.rel_err(to64(dw), to64(dw_ref))
        assert nr <= (1e-6 if dw_dt == torch.float32 else 4e-3), (call, nr, mr, ma)
        ref = co.conv_wgrad_masked(to64(dy), to64(x), pf, mo, 128, order, 27,
                                   mask_filter=kw.get("mask_filter", 0xffffffff), dw_prev=to64(start),
                                   beta=kw.get("beta", 0.0))
        nr, mr, ma = co.rel_err(to64(dw), ref)
        assert nr <= (2e-5 if dw_dt == torch.float32 else 2e-3), (call, nr, mr, ma)
        if route == "filter":
            assert torch.equal(dw[:, 13], start[:, 13]), call
