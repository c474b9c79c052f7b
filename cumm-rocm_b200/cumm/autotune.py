"""Autotuner for the mask-implicit-GEMM convolution.  Forward: the mask split
(MaskImplicitGemm = 1 launch, MaskSplitImplicitGemm = 2 launches over the two
halves of the kernel offsets, spconv's ConvAlgo choice) and the output-column
tile (ConvAlgoDesp tile_shape[1], ConvParams.tile_n).  Backward-weight: the
split-K count (ConvParams.split_k_slices = the kernel's row splits).  Each
candidate is timed on the caller's own workload with CUDA events and the
winner is cached per workload signature (rows rounded up to a power of two,
C, K, dtype).

The reference picks its kernel from a fixed if-tree over tile shapes
(cumm/conv/main.py:483-745, 'Can't Found Algorithm' when none fits); here the
candidates all compute the same result and only their speed differs.
"""
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Sequence, Tuple

import torch

from cumm import tensorview as tv
from cumm.conv.main import ConvMainUnitTest, get_all_conv_algo_desp
from cumm.tensorview.gemm import ConvOpType, ConvParams


@dataclass(frozen=True)
class FwdConfig:
    num_split: int = 1   # 1: one launch with the full mask; 2: two launches, beta = 1 on the second
    tile_n: int = 0      # 0: widest column tile

    def __str__(self):
        return f"split{self.num_split}_tn{self.tile_n or 'auto'}"


@dataclass(frozen=True)
class WgradConfig:
    split_k: int = 0     # row splits of the backward-weight kernel; 0: about one CTA per SM

    def __str__(self):
        return f"splitk{self.split_k or 'auto'}"


def wgrad_candidates(num_sms: int) -> List[WgradConfig]:
    return [WgradConfig(0), WgradConfig(max(1, num_sms // 4)), WgradConfig(max(1, num_sms // 2)),
            WgradConfig(num_sms)]


def fwd_candidates(K: int) -> List[FwdConfig]:
    res = [FwdConfig(1, 0), FwdConfig(2, 0)]
    if K % 32 == 0 and K // 2 >= 16:
        res.append(FwdConfig(1, K // 2))
    return res


def _desp(dt_in, dt_out):
    for d in get_all_conv_algo_desp():
        if (d.op_type == ConvOpType.kForward and d.algo == "Tcgen05" and d.dtype_input == dt_in
                and d.dtype_weight == dt_in and d.dtype_output == dt_out and d.tile_shape[0] == 128):
            return d
    raise KeyError((dt_in, dt_out))


def run_forward(cfg: FwdConfig, x: torch.Tensor, w: torch.Tensor, out: torch.Tensor, tables: Dict,
                dt_in=tv.bfloat16, dt_out=tv.bfloat16, stream: int = 0, cm: ConvMainUnitTest = None,
                act_type: int = 0, scale: torch.Tensor = None):
    """Forward conv of one (possibly batched) cloud with configuration `cfg`.
    `tables[num_split]` is the PairTable built with that split count.
    act_type / scale: epilogue activation and per-output-channel scale (E4M3)."""
    pt = tables[cfg.num_split]
    cm = cm or ConvMainUnitTest()
    desp = _desp(dt_in, dt_out)
    for j in range(cfg.num_split):
        p = ConvParams(3, ConvOpType.kForward)
        p.conv_algo_desp = desp
        p.input, p.weight, p.output = tv.Tensor(x, dt_in), tv.Tensor(w, dt_in), tv.Tensor(out, dt_out)
        p.indices = tv.Tensor(pt.pairs_fwd)
        p.mask = tv.Tensor(pt.masks_fwd[j], tv.uint32)
        p.mask_argsort = tv.Tensor(pt.argsorts_fwd[j])
        p.indices_sorted = tv.Tensor(pt.sorted_indices("fwd", j))
        p.tile_order = tv.Tensor(pt.tile_order("fwd", j))
        p.mask_filter = pt.split_masks[j] if cfg.num_split > 1 else 0xffffffff
        p.beta = 1.0 if j > 0 else 0.0
        p.tile_n = cfg.tile_n
        if scale is not None:
            p.scale = tv.Tensor(scale)
        if act_type and j == cfg.num_split - 1:
            p.act_type = act_type
        p.stream = stream or torch.cuda.current_stream().cuda_stream
        cm.implicit_gemm2(p)


def run_wgrad(cfg: WgradConfig, x: torch.Tensor, dy: torch.Tensor, dw: torch.Tensor, pt,
              mask_output: torch.Tensor, dt_in=tv.bfloat16, stream: int = 0,
              cm: ConvMainUnitTest = None):
    """Backward-weight of one cloud: dw [K, kv, C] (fp32 or dt_in) from input
    x [N, C] and output gradient dy [N, K] over PairTable pt; mask_output is
    the forward's per-128-row mask words."""
    cm = cm or ConvMainUnitTest()
    dt_w = tv.float32 if dw.dtype == torch.float32 else dt_in
    desp = None
    for d in get_all_conv_algo_desp():
        if (d.op_type == ConvOpType.kBackwardWeight and d.algo == "Tcgen05" and d.dtype_input == dt_in
                and d.dtype_weight == dt_w and d.dtype_output == dt_in):
            desp = d
            break
    if desp is None:
        raise KeyError((dt_in, dt_w))
    p = ConvParams(3, ConvOpType.kBackwardWeight)
    p.conv_algo_desp = desp
    p.input, p.weight, p.output = tv.Tensor(x, dt_in), tv.Tensor(dw, dt_w), tv.Tensor(dy, dt_in)
    p.indices = tv.Tensor(pt.pairs_fwd)
    p.mask = tv.Tensor(mask_output, tv.uint32)
    p.mask_argsort = tv.Tensor(pt.argsorts_fwd[0])
    p.indices_sorted = tv.Tensor(pt.sorted_indices("fwd"))
    p.mask_width = 128
    p.split_k_slices = cfg.split_k if cfg.split_k > 1 else 1
    p.stream = stream or torch.cuda.current_stream().cuda_stream
    cm.implicit_gemm2(p)


@dataclass
class ConvAutotuner:
    iters: int = 5
    cache: Dict[Tuple, FwdConfig] = field(default_factory=dict)
    last_timings: Dict[str, float] = field(default_factory=dict)

    @staticmethod
    def key(n_rows: int, C: int, K: int, dt) -> Tuple:
        b = 1
        while b < n_rows:
            b <<= 1
        return ("fwd", b, C, K, int(dt))

    def tune_forward(self, n_rows: int, C: int, K: int, dt, run: Callable[[FwdConfig], None],
                     candidates: Sequence[FwdConfig] = None) -> FwdConfig:
        """run(cfg) must launch one forward of the workload with `cfg` on the
        current stream.  Returns (and caches) the fastest candidate."""
        return self._tune(self.key(n_rows, C, K, dt), list(candidates or fwd_candidates(K)), run)

    def tune_wgrad(self, n_rows: int, C: int, K: int, dt, run: Callable[[WgradConfig], None],
                   candidates: Sequence[WgradConfig] = None) -> WgradConfig:
        """run(cfg) must launch one backward-weight of the workload with `cfg`
        on the current stream.  Returns (and caches) the fastest candidate."""
        if candidates is None:
            candidates = wgrad_candidates(torch.cuda.get_device_properties(
                torch.cuda.current_device()).multi_processor_count)
        k = ("wgrad",) + self.key(n_rows, C, K, dt)[1:]
        return self._tune(k, list(candidates), run)

    def _tune(self, k: Tuple, cands: List, run: Callable):
        if k in self.cache:
            return self.cache[k]
        times = {}
        for cfg in cands:
            run(cfg)  # warm-up (first-call set-up, L2)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(self.iters):
                run(cfg)
            e1.record()
            torch.cuda.synchronize()
            times[str(cfg)] = e0.elapsed_time(e1) / self.iters
        best = min(cands, key=lambda c: times[str(c)])
        self.cache[k] = best
        self.last_timings = times
        return best
