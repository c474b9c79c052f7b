"""Many point clouds in one grouped forward: the clouds are concatenated into
one batched voxel set (the batch index is part of every hash key, so no pair
ever joins two clouds), one pair-table build and one persistent conv launch
(per mask split) cover every tile of every cloud, and the whole sequence is
captured once in a CUDA graph and replayed.

This is the batched form of spconv's per-batch SparseConvTensor (the reference
drives one cloud per call, cumm/conv/main_real_spconv.py:228-294).  Rows of the
output are the rows of the concatenated input, so cloud i's result is the row
range offsets[i]:offsets[i+1].

``python -m cumm.batch`` runs 64 LiDAR-like clouds (lognormal voxel counts,
median 40k, sigma 0.8, clipped to [5k, 300k]) through a submanifold 3x3x3
C = K = 64 bf16 layer, grouped + graph-replayed vs 64 sequential per-cloud
calls, and prints one JSON line.
"""
from typing import Dict, List, Optional, Sequence

import numpy as np
import torch

from cumm import tensorview as tv
from cumm.autotune import ConvAutotuner, FwdConfig, run_forward
from cumm.conv.main import ConvMainUnitTest
from cumm.spconv_ops import build_pair_table


def concat_clouds(coords_list: Sequence[torch.Tensor]):
    """[n_i, 4] (batch, z, y, x) per cloud -> ([sum n_i, 4] with batch = cloud
    index, offsets [len + 1])."""
    parts, offs = [], [0]
    for i, c in enumerate(coords_list):
        c = c.clone()
        c[:, 0] = i
        parts.append(c)
        offs.append(offs[-1] + c.shape[0])
    return torch.cat(parts, 0).contiguous(), offs


class GroupedSubmConv:
    """Forward of one submanifold layer over a fixed set of clouds.

    The voxel coordinates are fixed at construction (static device buffers);
    features are copied into a static input buffer per call.  capture() records
    pair-table build + conv launches in a CUDA graph; __call__ replays it."""

    def __init__(self, coords_list: Sequence[torch.Tensor], spatial_shape: Sequence[int],
                 weight: torch.Tensor, ksize=(3, 3, 3), tuner: Optional[ConvAutotuner] = None,
                 build_pairs_in_graph: bool = True):
        self.dev = weight.device
        self.coords, self.offsets = concat_clouds([c.to(self.dev) for c in coords_list])
        self.n = self.coords.shape[0]
        self.spatial = list(spatial_shape)
        self.ksize = ksize
        self.weight = weight
        self.K, _, self.C = weight.shape
        self.x = torch.zeros((self.n, self.C), dtype=weight.dtype, device=self.dev)
        self.out = torch.empty((self.n, self.K), dtype=weight.dtype, device=self.dev)
        self.tuner = tuner or ConvAutotuner()
        self.build_pairs_in_graph = build_pairs_in_graph
        self.cfg: Optional[FwdConfig] = None
        self.tables: Dict[int, object] = {}
        self.graph: Optional[torch.cuda.CUDAGraph] = None
        self.cm = ConvMainUnitTest()

    def _build(self, splits: Sequence[int]):
        for s in splits:
            pt = build_pair_table(self.coords, self.spatial, ksize=self.ksize, num_split=s)
            pt.sorted_indices("fwd", 0)
            if s == 2:
                pt.sorted_indices("fwd", 1)
            self.tables[s] = pt

    def _dt(self):
        return tv.bfloat16 if self.weight.dtype == torch.bfloat16 else tv.float16

    def tune(self) -> FwdConfig:
        self._build((1, 2))
        dt = self._dt()
        self.cfg = self.tuner.tune_forward(
            self.n, self.C, self.K, dt,
            lambda cfg: run_forward(cfg, self.x, self.weight, self.out, self.tables, dt, dt, cm=self.cm))
        return self.cfg

    def _body(self):
        dt = self._dt()
        if self.build_pairs_in_graph:
            self.tables = {}
            self._build((self.cfg.num_split,))
        run_forward(self.cfg, self.x, self.weight, self.out, self.tables, dt, dt, cm=self.cm)

    def capture(self):
        if self.cfg is None:
            self.tune()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            self._body()  # eager warm-up on the capture stream (first-call set-up)
        torch.cuda.current_stream().wait_stream(s)
        torch.cuda.synchronize()
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self._body()
        torch.cuda.synchronize()

    def __call__(self, x: Optional[torch.Tensor] = None) -> torch.Tensor:
        if x is not None:
            self.x.copy_(x, non_blocking=True)
        if self.graph is None:
            self.capture()
        self.graph.replay()
        return self.out

    def split(self, y: torch.Tensor) -> List[torch.Tensor]:
        return [y[self.offsets[i]:self.offsets[i + 1]] for i in range(len(self.offsets) - 1)]


def lognormal_counts(n: int, median: float, sigma: float, lo: int, hi: int, seed: int) -> List[int]:
    rng = np.random.default_rng(seed)
    return [int(v) for v in np.clip(np.round(median * np.exp(sigma * rng.standard_normal(n))), lo, hi)]


def main(n_clouds: int = 64, median: int = 40_000, sigma: float = 0.8, C: int = 64, K: int = 64,
         seed: int = 0, reps: int = 5, verbose: bool = True, keep: bool = False) -> dict:
    """Config-4 comparison: grouped + graph-replayed vs sequential per-cloud
    calls.  Returns the result dict (printed as one JSON line when verbose);
    with keep=True it also holds "state": the clouds, features, weight and the
    grouped output split per cloud, for an outside check of the numbers."""
    import json

    from cumm import voxelgen as vg
    from cumm.autotune import FwdConfig

    dev = torch.device("cuda")
    counts = lognormal_counts(n_clouds, median, sigma, 5_000, 300_000, seed)
    coords = [torch.from_numpy(vg.lidar_voxels(n, seed=seed + i + 1)).to(dev) for i, n in enumerate(counts)]
    rng = np.random.default_rng(seed)
    feats = [torch.from_numpy(rng.standard_normal((n, C)).astype(np.float32)).to(dev).bfloat16()
             for n in counts]
    w = torch.from_numpy(vg.kaiming_uniform(K, 27, C, seed)).to(dev).bfloat16()
    cm = ConvMainUnitTest()

    # plain path: one cloud per call (pair build + forward), default stream
    outs_seq = [torch.empty((n, K), dtype=torch.bfloat16, device=dev) for n in counts]
    pairs_total = 0

    def sequential(with_pairs=True, tables=None):
        nonlocal pairs_total
        for i in range(n_clouds):
            pt = build_pair_table(coords[i], vg.KITTI_SHAPE) if with_pairs else tables[i]
            run_forward(FwdConfig(1, 0), feats[i], w, outs_seq[i], {1: pt}, cm=cm)

    sequential()
    tables = [build_pair_table(c, vg.KITTI_SHAPE) for c in coords]
    for t in tables:
        t.sorted_indices("fwd")
    pairs_total = sum(t.pair_count() for t in tables)
    flops = 2.0 * pairs_total * C * K

    def timed(fn, n):
        fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(n):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n

    ms_seq = timed(lambda: sequential(True), reps)
    ms_seq_conv = timed(lambda: sequential(False, tables), reps)

    grouped = GroupedSubmConv(coords, vg.KITTI_SHAPE, w)
    cfg = grouped.tune()
    tune_ms = dict(grouped.tuner.last_timings)
    xcat = torch.cat(feats, 0)
    grouped.x.copy_(xcat)
    grouped.capture()
    ms_grp = timed(lambda: grouped(), reps * 4)
    conv_only = GroupedSubmConv(coords, vg.KITTI_SHAPE, w, tuner=grouped.tuner, build_pairs_in_graph=False)
    conv_only.tune()
    conv_only.x.copy_(xcat)
    conv_only.capture()
    ms_grp_conv = timed(lambda: conv_only(), reps * 4)

    y = grouped(xcat)
    torch.cuda.synchronize()
    sequential(False, tables)
    torch.cuda.synchronize()
    worst = 0.0
    for i, yi in enumerate(grouped.split(y)):
        d = (yi.float() - outs_seq[i].float()).norm() / outs_seq[i].float().norm().clamp_min(1e-30)
        worst = max(worst, float(d))
    res = {
        "workload": f"batched{n_clouds}_lognormal_median{median // 1000}k_subm3x3x3_c{C}k{K}_bf16_fwd",
        "clouds": n_clouds, "voxels": int(sum(counts)), "voxels_min": min(counts),
        "voxels_max": max(counts), "pairs": int(pairs_total), "gflop": flops / 1e9,
        "autotune": {"chosen": str(cfg), "ms": tune_ms},
        "layer_with_pair_build": {"sequential_ms": ms_seq, "grouped_graph_ms": ms_grp,
                                  "speedup": ms_seq / ms_grp,
                                  "grouped_tflops": flops / (ms_grp * 1e-3) / 1e12},
        "conv_only": {"sequential_ms": ms_seq_conv, "grouped_graph_ms": ms_grp_conv,
                      "speedup": ms_seq_conv / ms_grp_conv,
                      "grouped_tflops": flops / (ms_grp_conv * 1e-3) / 1e12},
        "max_norm_rel_grouped_vs_sequential": worst,
    }
    if verbose:
        print(json.dumps(res), flush=True)
    if keep:
        res["state"] = {"coords": coords, "feats": feats, "weight": w, "outputs": grouped.split(y)}
    return res


if __name__ == "__main__":
    main()
