"""CPU oracle for the mask-implicit-GEMM sparse convolution path.

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and by
bench.py's CPU-baseline / reference arm as the checker or the timed CPU
algorithm.  Nothing in the library (cumm-rocm_b200/) imports it; the product
path has no CPU fallback.

Parity status: the reference (cumm 0.8.2) cannot be built or imported here
(pccm / spconv missing) and ships no golden vectors for this path, so parity
against the reference's own outputs is UNPINNED.  This oracle is instead
pinned against an independent evaluation of the same operator: dense
torch.nn.functional.conv3d on the voxel grid (tests/golden/, generated by
tests/golden/make_golden.py), which the reference's own dense-conv driver uses
as its check (cumm/conv/main_real.py:120-146).

Restated algorithms (FP64 unless noted):
* gather-GEMM-scatter forward / backward-input / backward-weight of
  cumm/conv/main_real_spconv.py:309-403 (``*_gather_gemm_scatter``; fp32 when
  timed as the CPU baseline, as in the reference);
* the exact mask-implicit-GEMM kernel semantics (``conv_*_masked``): tile
  masks OR-ed over tile_shape[0] sorted rows and AND-ed with mask_filter
  (cumm/conv/kernel.py:844-866), bit reversal for backward-input
  (kernel.py:883-889), skipped empty dgrad tiles (kernel.py:875-882), gathers
  through indices[k][mask_argsort[r]] with -1 = zero (cumm/conv/sparse_iters.py:318-356,
  625-648), permuted store to mask_argsort[r] (cumm/gemm/out_iters.py:537-551),
  wgrad rows gated by mask[r // mask_width] (cumm/gemm/blockmma/mma.py:607-648);
* epilogues LinearCombination act(alpha*acc + beta*src) and the scale/bias op
  act(scale*acc + alpha*bias + beta*src) (cumm/gemm/output_op/linear.py:107-129,
  300-392) with activations of cumm/gemm/gemmmath/__init__.py:185-210.
"""
from typing import Optional, Tuple

import numpy as np

ACT_NONE, ACT_RELU, ACT_SIGMOID, ACT_LEAKY = 0, 1, 2, 3


def act(x: np.ndarray, act_type: int, a: float = 0.0) -> np.ndarray:
    if act_type == ACT_RELU:
        return np.maximum(x, 0)
    if act_type == ACT_SIGMOID:
        return 1.0 / (1.0 + np.exp(-x))
    if act_type == ACT_LEAKY:
        return np.where(x >= 0, x, x * a)
    return x


def _u32(x) -> np.ndarray:
    return np.asarray(x).astype(np.int64) & 0xffffffff


def brev_shift(m: np.ndarray, kv: int) -> np.ndarray:
    """__brev(m) >> (32 - kv) for uint32 values."""
    m = _u32(m)
    out = np.zeros_like(m)
    for b in range(kv):
        out |= ((m >> b) & 1) << (kv - 1 - b)
    # bits >= kv of m land below bit 0 after the shift and vanish
    return out


def tile_masks(mask_sorted: np.ndarray, tile_m: int) -> np.ndarray:
    m = _u32(mask_sorted)
    M = m.shape[0]
    if M == 0:
        return np.zeros(0, np.int64)
    starts = np.arange(0, M, tile_m)
    return np.bitwise_or.reduceat(m, starts)


def epilogue(acc: np.ndarray, rows_out: np.ndarray, out_prev: Optional[np.ndarray], alpha: float,
             beta: float, act_type: int = 0, act_alpha: float = 0.0, bias: Optional[np.ndarray] = None,
             scale: Optional[np.ndarray] = None, output_add: Optional[np.ndarray] = None) -> np.ndarray:
    """Values written to rows ``rows_out`` (acc is [len(rows_out), n])."""
    if scale is not None:
        v = scale[None, :] * acc
        if bias is not None:
            v = v + alpha * bias[None, :]
        src = output_add if output_add is not None else out_prev
        if beta != 0 and src is not None:
            v = v + beta * src[rows_out]
    else:
        v = alpha * acc
        if beta != 0:
            if bias is not None:
                v = v + beta * bias[None, :]
            elif out_prev is not None:
                v = v + beta * out_prev[rows_out]
    return act(v, act_type, act_alpha)


def conv_fwd_masked(inp: np.ndarray, weight: np.ndarray, indices: np.ndarray, mask_sorted: np.ndarray,
                    argsort: np.ndarray, tile_m: int = 128, mask_filter: int = 0xffffffff,
                    out_prev: Optional[np.ndarray] = None, alpha: float = 1.0, beta: float = 0.0,
                    act_type: int = 0, act_alpha: float = 0.0, bias=None, scale=None,
                    output_add=None) -> Tuple[np.ndarray, np.ndarray]:
    """Forward: returns (output [N, K] fp64, mask_output [ceil(N/tile_m)] uint32).
    weight is [K, kv, C]; indices is [kv, N]."""
    K, kv, C = weight.shape
    N = indices.shape[1]
    inp = inp.astype(np.float64)
    w = weight.astype(np.float64)
    tm = tile_masks(mask_sorted, tile_m) & (int(mask_filter) & 0xffffffff)
    gate = tm[np.arange(N) // tile_m] if N else np.zeros(0, np.int64)
    acc = np.zeros((N, K), np.float64)
    sig = np.asarray(argsort).astype(np.int64)
    for k in range(kv):
        rows = np.nonzero((gate >> k) & 1)[0]
        if rows.size == 0:
            continue
        idx = indices[k][sig[rows]]
        ok = idx >= 0
        acc[rows[ok]] += inp[idx[ok]] @ w[:, k, :].T
    out = np.zeros((N, K), np.float64) if out_prev is None else out_prev.astype(np.float64).copy()
    out[sig] = epilogue(acc, sig, out_prev if out_prev is None else out_prev.astype(np.float64),
                        alpha, beta, act_type, act_alpha,
                        None if bias is None else bias.astype(np.float64),
                        None if scale is None else scale.astype(np.float64),
                        None if output_add is None else output_add.astype(np.float64))
    return out, tm.astype(np.uint32)


def conv_dgrad_masked(dout: np.ndarray, weight: np.ndarray, indices: np.ndarray,
                      mask_sorted: np.ndarray, argsort: np.ndarray, tile_m: int = 128,
                      mask_filter: int = 0xffffffff, reverse_mask: bool = True,
                      din_prev: Optional[np.ndarray] = None, alpha: float = 1.0, beta: float = 0.0,
                      act_type: int = 0, act_alpha: float = 0.0) -> np.ndarray:
    """Backward-input: din [N, C] with din[sigma(r)] = sum_k dout[indices[k][sigma(r)]] @ W[:, k, :]."""
    K, kv, C = weight.shape
    N = indices.shape[1]
    dout = dout.astype(np.float64)
    w = weight.astype(np.float64)
    tm = tile_masks(mask_sorted, tile_m) & (int(mask_filter) & 0xffffffff)
    tile_nonzero = tm != 0
    if reverse_mask:
        tm = brev_shift(tm, kv)
    gate = tm[np.arange(N) // tile_m] if N else np.zeros(0, np.int64)
    acc = np.zeros((N, C), np.float64)
    sig = np.asarray(argsort).astype(np.int64)
    for k in range(kv):
        rows = np.nonzero((gate >> k) & 1)[0]
        if rows.size == 0:
            continue
        idx = indices[k][sig[rows]]
        ok = idx >= 0
        acc[rows[ok]] += dout[idx[ok]] @ w[:, k, :]
    din = np.zeros((N, C), np.float64) if din_prev is None else din_prev.astype(np.float64).copy()
    written = tile_nonzero[np.arange(N) // tile_m] if N else np.zeros(0, bool)
    rows_w = np.nonzero(written)[0]
    prev = None if din_prev is None else din_prev.astype(np.float64)
    din[sig[rows_w]] = epilogue(acc[rows_w], sig[rows_w], prev, alpha, beta, act_type, act_alpha)
    return din


def conv_wgrad_masked(dout: np.ndarray, inp: np.ndarray, indices: np.ndarray, mask_reduced: np.ndarray,
                      mask_width: int, argsort: np.ndarray, kv: int, mask_filter: int = 0xffffffff,
                      dw_prev: Optional[np.ndarray] = None, alpha: float = 1.0,
                      beta: float = 0.0) -> np.ndarray:
    """Backward-weight: dW [K, kv, C]; offsets outside mask_filter keep dw_prev."""
    N = indices.shape[1]
    K = dout.shape[1]
    C = inp.shape[1]
    dout = dout.astype(np.float64)
    inp = inp.astype(np.float64)
    words = _u32(mask_reduced)
    r = np.arange(N)
    wi = r // mask_width
    word = np.where(wi < words.shape[0], words[np.minimum(wi, max(words.shape[0] - 1, 0))], 0) \
        if N else np.zeros(0, np.int64)
    word = word & (int(mask_filter) & 0xffffffff)
    sig = np.asarray(argsort).astype(np.int64)
    acc = np.zeros((K, kv, C), np.float64)
    for k in range(kv):
        rows = np.nonzero((word >> k) & 1)[0]
        if rows.size == 0:
            continue
        s = sig[rows]
        idx = indices[k][s]
        ok = idx >= 0
        acc[:, k, :] = dout[s[ok]].T @ inp[idx[ok]]
    dw = np.zeros((K, kv, C), np.float64) if dw_prev is None else dw_prev.astype(np.float64).copy()
    for k in range(kv):
        if (int(mask_filter) >> k) & 1:
            v = alpha * acc[:, k, :]
            if beta != 0 and dw_prev is not None:
                v = v + beta * dw_prev[:, k, :].astype(np.float64)
            dw[:, k, :] = v
    return dw


# ------------------------------------------------------------------ reference CPU algorithm
def fwd_gather_gemm_scatter(inp: np.ndarray, weight: np.ndarray, pairs_fwd: np.ndarray,
                            dtype=np.float64) -> np.ndarray:
    """out[o] += in[i] @ W_k^T for every pair (i, o, k) (main_real_spconv.py:309-325)."""
    K, kv, C = weight.shape
    N = pairs_fwd.shape[1]
    out = np.zeros((N, K), dtype)
    inp = inp.astype(dtype, copy=False)
    w = weight.astype(dtype, copy=False)
    for k in range(kv):
        o = np.nonzero(pairs_fwd[k] >= 0)[0]
        if o.size == 0:
            continue
        out[o] += inp[pairs_fwd[k][o]] @ w[:, k, :].T
    return out


def dgrad_gather_gemm_scatter(dout: np.ndarray, weight: np.ndarray, pairs_bwd: np.ndarray,
                              dtype=np.float64) -> np.ndarray:
    """din[i] += dout[o] @ W_k (main_real_spconv.py:347-365)."""
    K, kv, C = weight.shape
    N = pairs_bwd.shape[1]
    din = np.zeros((N, C), dtype)
    dout = dout.astype(dtype, copy=False)
    w = weight.astype(dtype, copy=False)
    for k in range(kv):
        i = np.nonzero(pairs_bwd[k] >= 0)[0]
        if i.size == 0:
            continue
        din[i] += dout[pairs_bwd[k][i]] @ w[:, k, :]
    return din


def wgrad_gather_gemm_scatter(dout: np.ndarray, inp: np.ndarray, pairs_fwd: np.ndarray,
                              dtype=np.float64) -> np.ndarray:
    """dW_k = dout[o]^T @ in[i] (main_real_spconv.py:375-397)."""
    kv, N = pairs_fwd.shape
    K = dout.shape[1]
    C = inp.shape[1]
    dw = np.zeros((K, kv, C), dtype)
    dout = dout.astype(dtype, copy=False)
    inp = inp.astype(dtype, copy=False)
    for k in range(kv):
        o = np.nonzero(pairs_fwd[k] >= 0)[0]
        if o.size == 0:
            continue
        dw[:, k, :] = dout[o].T @ inp[pairs_fwd[k][o]]
    return dw


# ------------------------------------------------------------------ GEMM (matmul2)
def gemm(a: np.ndarray, b: np.ndarray, trans_a=False, trans_b=False, shuffle: int = 0,
         a_inds=None, b_inds=None, c_inds=None, c_prev=None, d=None, alpha=1.0, beta=0.0,
         act_type=0, act_alpha=0.0) -> np.ndarray:
    """C = act(alpha op(A) op(B) + beta D) with ShuffleAC / ShuffleAB
    (cumm/gemm/main_real.py:136, 206-229)."""
    a = a.astype(np.float64)
    b = b.astype(np.float64)
    if shuffle == 2:
        prod = a[a_inds].T @ b[b_inds]
    elif shuffle == 1:
        aa = a[a_inds] if a_inds is not None else a
        prod = aa @ (b.T if trans_b else b)
    else:
        prod = (a.T if trans_a else a) @ (b.T if trans_b else b)
    if shuffle == 1:
        c = c_prev.astype(np.float64).copy()
        src = d.astype(np.float64) if d is not None else c_prev.astype(np.float64)
        rows = np.asarray(c_inds)
        v = alpha * prod
        if beta != 0:
            v = v + beta * (src[None, :] if src.ndim == 1 else src[rows])
        c[rows] = act(v, act_type, act_alpha)
        return c
    v = alpha * prod
    if beta != 0:
        src = d if d is not None else c_prev
        src = src.astype(np.float64)
        v = v + beta * (src[None, :] if src.ndim == 1 else src)
    return act(v, act_type, act_alpha)


def rel_err(y: np.ndarray, ref: np.ndarray) -> Tuple[float, float, float]:
    """(norm-relative, max-relative with a 1e-3 * max|ref| floor, max-abs)."""
    y = y.astype(np.float64)
    ref = ref.astype(np.float64)
    diff = np.abs(y - ref)
    nr = float(np.linalg.norm(diff) / max(np.linalg.norm(ref), 1e-300))
    floor = 1e-3 * max(float(np.abs(ref).max()) if ref.size else 0.0, 1e-300)
    mr = float((diff / np.maximum(np.abs(ref), floor)).max()) if ref.size else 0.0
    ma = float(diff.max()) if ref.size else 0.0
    return nr, mr, ma
