"""FP8-E4M3 operands for the forward conv: quantizers and an error/throughput
report for the stride-2 downsample layer.

Scales follow the reference's int8 inference epilogue (Int8Inference,
cumm/gemm/output_op/linear.py:185-392: ``act(scale[n] * acc + alpha * bias[n] +
beta * src)`` with a per-output-channel ``scale``):

* activations get one scale per 64-channel tile of the input features
  (``s_x[t] = amax(x[:, tile t]) / 448``);
* that tile scale is folded into the weights' input channels, and the folded
  weights get one scale per output channel (``s_w[n] = amax(w'[n]) / 448``).

Then ``sum_c x[., c] w[n, ., c] = s_w[n] * sum_c q_x[., c] q_w[n, ., c]``, so the
kernel accumulates raw E4M3 products in fp32 and applies ``s_w`` in the epilogue
(ConvParams.scale) with no per-row work.

``python -m cumm.precision`` builds the 200k-voxel LiDAR-like cloud, runs the
3x3x3 stride-2 pad-1 downsample (C 64 -> 128) in BF16 and FP8 on the GPU and
prints one JSON line: per variant the error against an FP64 gather-GEMM-scatter on
the same rounded / quantized operands (the kernel's error) and against FP64 on the
fp32 inputs (including operand rounding), FP8 against the BF16 path, and forward
TFLOP/s (norm-relative, max-relative with a 1e-3 * max|ref| floor, max-abs).
"""
from typing import Tuple

import numpy as np
import torch

E4M3_MAX = 448.0


def quantize_act_fp8(x: torch.Tensor, ctile: int = 64) -> Tuple[torch.Tensor, torch.Tensor]:
    """x [N, C] float -> (q [N, C] float8_e4m3fn, s [ceil(C / ctile)] fp32)."""
    n, c = x.shape
    nt = (c + ctile - 1) // ctile
    xf = x.float()
    s = torch.empty(nt, dtype=torch.float32, device=x.device)
    q = torch.empty_like(xf)
    for t in range(nt):
        sl = slice(t * ctile, min((t + 1) * ctile, c))
        amax = xf[:, sl].abs().max() if n else torch.tensor(0.0, device=x.device)
        s[t] = torch.clamp(amax / E4M3_MAX, min=1e-12)
        q[:, sl] = xf[:, sl] / s[t]
    return q.to(torch.float8_e4m3fn), s


def quantize_weight_fp8(w: torch.Tensor, act_scale: torch.Tensor = None,
                        ctile: int = 64) -> Tuple[torch.Tensor, torch.Tensor]:
    """w [K, kv, C] float -> (q [K, kv, C] float8_e4m3fn, s [K] fp32).  With
    ``act_scale`` (from quantize_act_fp8) the activation tile scales are folded
    into the input channels first, so ``s`` is the whole epilogue scale."""
    wf = w.float()
    if act_scale is not None:
        c = wf.shape[2]
        per_c = act_scale.repeat_interleave(ctile)[:c]
        wf = wf * per_c[None, None, :]
    amax = wf.abs().reshape(wf.shape[0], -1).max(1).values
    s = torch.clamp(amax / E4M3_MAX, min=1e-12)
    return (wf / s[:, None, None]).to(torch.float8_e4m3fn), s.float().contiguous()


def rel_err(y: torch.Tensor, ref: torch.Tensor) -> Tuple[float, float, float]:
    """(norm-relative, max-relative with a 1e-3 * max|ref| floor, max-abs)."""
    diff = (y - ref).abs()
    nr = float(diff.norm() / ref.norm().clamp_min(1e-300))
    floor = 1e-3 * float(ref.abs().max()) if ref.numel() else 1.0
    mr = float((diff / ref.abs().clamp_min(max(floor, 1e-300))).max()) if ref.numel() else 0.0
    return nr, mr, float(diff.max()) if ref.numel() else 0.0


def main(seed: int = 0, n_vox: int = 200_000, c_in: int = 64, c_out: int = 128) -> dict:
    import json

    from cumm import tensorview as tv
    from cumm import voxelgen as vg
    from cumm.conv.main import ConvMainUnitTest, get_all_conv_algo_desp
    from cumm.spconv_ops import build_pair_table
    from cumm.tensorview.gemm import ConvOpType, ConvParams

    dev = torch.device("cuda")
    coords = torch.from_numpy(vg.lidar_voxels(n_vox, seed=seed)).to(dev)
    pt = build_pair_table(coords, vg.KITTI_SHAPE, ksize=(3, 3, 3), stride=(2, 2, 2),
                          padding=(1, 1, 1), subm=False)
    n_out = pt.n_out
    rng = np.random.default_rng(seed)
    x = torch.from_numpy(rng.standard_normal((n_vox, c_in)).astype(np.float32)).to(dev)
    w = torch.from_numpy(vg.kaiming_uniform(c_out, 27, c_in, seed)).to(dev)
    P = pt.pair_count()
    flops = 2.0 * P * c_in * c_out

    def desp(dt_in, dt_out):
        for d in get_all_conv_algo_desp():
            if (d.op_type == ConvOpType.kForward and d.algo == "Tcgen05" and d.dtype_input == dt_in
                    and d.dtype_weight == dt_in and d.dtype_output == dt_out and d.tile_shape[0] == 128):
                return d
        raise KeyError((dt_in, dt_out))

    def run(xin, win, dt_in, scale=None):
        out = torch.empty((n_out, c_out), dtype=torch.bfloat16, device=dev)
        p = ConvParams(3, ConvOpType.kForward)
        p.conv_algo_desp = desp(dt_in, tv.bfloat16)
        p.input, p.weight, p.output = tv.Tensor(xin, dt_in), tv.Tensor(win, dt_in), tv.Tensor(out)
        p.indices = tv.Tensor(pt.pairs_fwd)
        p.mask = tv.Tensor(pt.masks_fwd[0], tv.uint32)
        p.mask_argsort = tv.Tensor(pt.argsorts_fwd[0])
        p.indices_sorted = tv.Tensor(pt.sorted_indices("fwd"))
        if scale is not None:
            p.scale = tv.Tensor(scale)
        cm = ConvMainUnitTest()
        flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
        for _ in range(3):
            cm.implicit_gemm2(p)
        torch.cuda.synchronize()
        ts = []
        for _ in range(20):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            cm.implicit_gemm2(p)
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return out, float(np.median(ts))

    xb, wb = x.bfloat16(), w.bfloat16()
    out_b, ms_b = run(xb, wb, tv.bfloat16)
    xq, sx = quantize_act_fp8(x)
    wq, sw = quantize_weight_fp8(w, sx)
    out_q, ms_q = run(xq, wq, tv.float_e4m3, scale=sw)

    def gather_gemm_fp64(xd, wd):
        """FP64 gather-GEMM-scatter (torch, on the GPU): out[o] += x[i] @ W_k^T."""
        ref = torch.zeros((n_out, c_out), dtype=torch.float64, device=dev)
        for k in range(pt.kv):
            o = torch.nonzero(pt.pairs_fwd[k] >= 0).squeeze(1)
            if o.numel():
                ref.index_add_(0, o, xd[pt.pairs_fwd[k][o].long()] @ wd[:, k, :].T)
        return ref

    ref = gather_gemm_fp64(x.double(), w.double())                    # fp32 operands
    ref_b = gather_gemm_fp64(xb.double(), wb.double())                # the bf16 operands
    ref_q = gather_gemm_fp64(xq.double(), wq.double()) * sw.double()[None, :]  # the E4M3 operands
    ob, oq = out_b.double(), out_q.double()
    keys = ("norm_rel", "max_rel", "max_abs")
    res = {
        "workload": f"conv3x3x3_s2p1_lidar{n_vox // 1000}k_c{c_in}k{c_out}_fwd",
        "voxels_in": n_vox, "voxels_out": int(n_out), "pairs": int(P), "gflop": flops / 1e9,
        "bf16": {"kernel_vs_fp64": dict(zip(keys, rel_err(ob, ref_b))),
                 "total_vs_fp64_of_fp32_inputs": dict(zip(keys, rel_err(ob, ref))),
                 "ms": ms_b, "tflops": flops / (ms_b * 1e-3) / 1e12},
        "fp8_e4m3": {"kernel_vs_fp64": dict(zip(keys, rel_err(oq, ref_q))),
                     "total_vs_fp64_of_fp32_inputs": dict(zip(keys, rel_err(oq, ref))),
                     "ms": ms_q, "tflops": flops / (ms_q * 1e-3) / 1e12},
        "fp8_vs_bf16_path": dict(zip(keys, rel_err(oq, ob))),
        "note": "kernel_vs_fp64: FP64 on the same (rounded / quantized) operands; total: FP64 "
                "on the fp32 inputs, so it includes operand rounding",
    }
    print(json.dumps(res), flush=True)
    return res


if __name__ == "__main__":
    main()
