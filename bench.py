"""Benchmark: mask-implicit-GEMM sparse conv on B200 (one training step of the
200k-voxel LiDAR-like submanifold 3x3x3 layer, C = K = 64, bf16 operands,
fp32 accumulation: forward + backward-input + backward-weight).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

* ``value``: whole-job algorithmic TFLOP/s, 3 * 2 * P * C * K per step (P =
  valid voxel pairs; padded MMA rows are not counted), inputs resident in HBM,
  per-step CUDA events on the launching stream around the three C-ABI calls,
  L2 flushed (256 MB write) between steps, max over ranks.
* ``e2e``: the same metric through the public API with host buffers: per step
  the pinned-host coordinates, features and upstream gradient are copied in,
  the pair table is built on the GPU, the three ops run, and output, input
  gradient and weight gradient are copied back.  Consecutive steps are
  pipelined over an upload, a compute and a download stream (full-duplex
  copies overlap the next and previous steps' compute).
* ``cpu_baseline`` / ``--impl reference``: the reference's own CPU algorithm
  for this path (numpy gather-GEMM-scatter, cumm/conv/main_real_spconv.py:309-403)
  restated in oracle/conv_oracle.py, fp32, BLAS on all host cores.
* ``batched`` (N = 1): 64 LiDAR-like clouds (lognormal voxel counts, median
  40k, sigma 0.8, clipped to [5k, 300k]) through the same subm 3x3x3 C = K = 64
  bf16 layer: one grouped persistent launch replayed from a CUDA graph vs 64
  sequential one-cloud calls (the reference's plain path), with and without
  the pair build; the grouped result is checked against the FP64 oracle.
* ``served`` (N = 1): the 10-layer sparse encoder served at 800 req/s
  (Poisson arrivals, clouds of 10k-400k voxels) in plain one-request-at-a-time
  mode and with continuous batching: p50 / p99 latency and voxels/s of both,
  and both modes' capacity (``saturated``: every request arriving at once);
  every layer of one request is checked against the FP64 oracle, and that
  request's result alone equals its result inside the mix.
Multi-GPU: independent clouds per rank (weak scaling, no collective on the
data path).
"""
import argparse
import ctypes
import json
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "cumm-rocm_b200"))

N_VOX, C, K, KV = 200_000, 64, 64, 27
REF_BUDGET_S = 120.0  # CPU seconds for a whole --impl reference run
WORKLOAD = "subm3x3x3_lidar200k_c64k64_bf16_fwd_dgrad_wgrad"


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d["bf16_tflops"], d["hbm_gbs"], "measured"
    return 1590.0, 6650.0, "fallback"


class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sms, maxs, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sms.append(float(f[1]))
                maxs.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sms)) if sms else None,
                "sm_max_mhz": float(max(maxs)) if maxs else None,
                "samples": len(sms), "reasons": sorted(reasons)}


KERNEL_SOURCE = {"conv_fwd": "conv_rowgather.cu", "conv_dgrad": "conv_rowgather.cu",
                 "conv_wgrad": "conv_wgrad.cu"}


def source_sha(kernel: str) -> str:
    import hashlib
    src = ROOT / "cumm-rocm_b200" / "csrc" / KERNEL_SOURCE[kernel]
    return hashlib.sha256(src.read_bytes()).hexdigest()[:16]


def recorded_traffic(kernel: str):
    """DRAM bytes per launch of `kernel` from the ncu capture recorded in
    profiles/traffic.json, used only when the capture was taken of the
    current kernel source (its sha256 prefix is stored with the bytes);
    otherwise None and a note saying the capture is stale."""
    tfile = ROOT / "profiles" / "traffic.json"
    if not tfile.exists():
        return None, "no ncu capture recorded"
    rec = json.loads(tfile.read_text()).get(kernel)
    if not isinstance(rec, dict):
        return None, "no ncu capture recorded for this kernel"
    if rec.get("source_sha") != source_sha(kernel):
        return None, f"recorded capture ({rec.get('bytes')} B) was taken of an older kernel source"
    return rec["bytes"], f"ncu capture of the current source ({rec.get('capture', '')})"


def max_over_ranks(x: float, dist, device) -> float:
    """The slowest rank's value (every rank takes part; identity at N = 1)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_tflops(flops_per_rank_step: float, world: int, ms: float) -> float:
    """Replicas: every rank runs its own cloud, so the job does world x the
    per-rank work in the slowest rank's time."""
    return flops_per_rank_step * world / (ms * 1e-3) / 1e12


def cpu_reference_step(x, w, dy, pf, pb):
    """fp32 numpy gather-GEMM-scatter fwd + dgrad + wgrad (the reference's CPU path)."""
    from oracle import conv_oracle as co
    out = co.fwd_gather_gemm_scatter(x, w, pf, np.float32)
    din = co.dgrad_gather_gemm_scatter(dy, w, pb, np.float32)
    dw = co.wgrad_gather_gemm_scatter(dy, x, pf, np.float32)
    return out, din, dw


def _cpu_data(seed):
    from cumm import voxelgen as vg
    from oracle import pairs_oracle as po
    coords = vg.lidar_voxels(N_VOX, seed=seed)
    pf, pb, m = po.subm_pairs(coords, vg.KITTI_SHAPE)
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((N_VOX, C)).astype(np.float32)
    dy = rng.standard_normal((N_VOX, K)).astype(np.float32)
    w = vg.kaiming_uniform(K, KV, C, seed)
    return coords, pf, pb, m, x, dy, w


def _sample_step(x, w, dy, pf, pb, rows):
    """One sample of the step on the first `rows` output (and input) rows:
    fwd / dgrad / wgrad restricted to the pairs of those rows."""
    return cpu_reference_step(x, w, dy, pf[:, :rows], pb[:, :rows])


def run_reference(args, rank, world):
    """The reference's CPU algorithm (numpy fp32 gather-GEMM-scatter on all
    host cores) on the same layer.  Each step is a bounded sample: the first
    R rows' pairs, with R sized from a timed probe so that warm-up + steps take
    about REF_BUDGET_S seconds; FLOP are counted on the sampled pairs."""
    if rank != 0:
        return None
    threads = os.cpu_count() or 1
    coords, pf, pb, m, x, dy, w = _cpu_data(0)
    n_steps = max(1, args.steps) + max(0, args.warmup)
    probe = min(N_VOX, 8_000)
    t0 = time.perf_counter()
    _sample_step(x, w, dy, pf, pb, probe)
    t_probe = max(time.perf_counter() - t0, 1e-4)
    rows = int(min(N_VOX, max(probe, probe * (REF_BUDGET_S / n_steps) / t_probe)))
    P = int((pf[:, :rows] >= 0).sum() + (pb[:, :rows] >= 0).sum() + (pf[:, :rows] >= 0).sum())
    flops = 2.0 * P * C * K  # fwd + dgrad + wgrad over the sampled pairs
    for _ in range(args.warmup):
        _sample_step(x, w, dy, pf, pb, rows)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        _sample_step(x, w, dy, pf, pb, rows)
        times.append(time.perf_counter() - t0)
    t = float(np.mean(times))
    v = flops / t / 1e12
    sample = (f"first {rows} of {N_VOX} rows per step (fwd / dgrad / wgrad over their pairs), "
              f"numpy fp32 gather-GEMM-scatter (oracle/conv_oracle.py), BLAS on all host cores")
    line = {
        "metric": "implicit-GEMM spconv TFLOP/s (% BF16 peak)", "value": v, "unit": "TFLOP/s",
        "impl": "reference", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "voxels": N_VOX, "pairs": int((pf >= 0).sum()), "C": C, "K": K,
                   "parallelism": "cpu", "sampled_rows": rows},
        "cpu_baseline": {"value": v, "unit": "TFLOP/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": v, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return line


def run_batched(reps: int = 3) -> dict:
    """Config 4: grouped + graph-replayed forward over 64 clouds vs sequential
    per-cloud calls (cumm.batch)."""
    from cumm import batch
    res = batch.main(reps=reps, verbose=False, keep=True)
    return res


def run_served(rate: float = 800.0, n_req: int = 160, seed: int = 0) -> dict:
    """Config 5: one point of the serving sweep, plain vs continuous, on the
    same seeded request stream (cumm.serve)."""
    import torch

    from cumm import serve as sv
    from cumm import voxelgen as vg
    enc = sv.SparseEncoder(vg.KITTI_SHAPE, seed=seed)
    pool = sv.make_pool(k=16, seed=seed)
    # warm-up: kernels loaded, and the caching allocator of every pass stream
    # holds the buffers of the largest passes (growing it synchronizes)
    sv.serve(enc, sv.make_requests(8, 1000.0, seed + 99, pool=pool), continuous=False)
    for _ in range(2):
        sv.serve(enc, sv.make_requests(n_req, 1e7, seed + 98, pool=pool), continuous=True)
        sv.serve(enc, sv.make_requests(96, 5000.0, seed + 97, pool=pool), continuous=True)
    out = {"rate_req_s": rate, "requests": n_req,
           "encoder": "subm16x2,down32,subm32,down64,subm64x2,down128,subm128x2 (ReLU), bf16"}
    for continuous in (False, True):
        reqs = sv.make_requests(n_req, rate, seed + int(rate), pool=pool)
        st = sv.serve(enc, reqs, continuous=continuous, keep_outputs=continuous)
        out["continuous" if continuous else "plain"] = {
            k: st[k] for k in ("p50_ms", "p99_ms", "voxels_per_s", "makespan_s", "passes", "mean_batch")}
        if continuous:
            mixed = reqs
    out["voxels_per_s_ratio"] = out["continuous"]["voxels_per_s"] / out["plain"]["voxels_per_s"]
    # capacity: the same number of requests all arriving at once, so neither
    # mode waits for arrivals (at 800 req/s continuous batching keeps pace with
    # the arrivals and its voxels/s is the offered load)
    sat = {}
    for continuous in (False, True):
        reqs = sv.make_requests(n_req, 1e7, seed + 7, pool=pool)
        st = sv.serve(enc, reqs, continuous=continuous)
        sat["continuous" if continuous else "plain"] = {
            k: st[k] for k in ("p50_ms", "p99_ms", "voxels_per_s", "makespan_s", "passes", "mean_batch")}
    sat["voxels_per_s_ratio"] = sat["continuous"]["voxels_per_s"] / sat["plain"]["voxels_per_s"]
    out["saturated"] = sat
    # one request alone vs inside the mix (the check below compares them)
    small = min(mixed, key=lambda r: r.n)
    alone = sv.Request(small.rid, 0.0, small.coords, small.feats)
    sv.serve(enc, [alone], continuous=False, keep_outputs=True)
    torch.cuda.synchronize()
    out["_check"] = (enc, small, alone)
    return out


def run_aux(peak_tf: float, peak_bw: float) -> dict:
    """Kernels beside the conv step, timed with CUDA events (L2-resident
    inputs unless stated): the dense tcgen05 matmul2 on an 8192^3 bf16 GEMM
    (cuBLAS through torch.matmul on the same shape for context), a tall-K
    ShuffleAB GEMM (200k gathered rows, the native backward-weight form), and
    the standalone gather / scatter-add on 128-byte rows (4M rows: 512 MB,
    HBM-bound)."""
    import torch

    from cumm import tensorview as tv
    from cumm.gemm.gather import GatherAll, ScatterAll
    from cumm.gemm.main import GemmMainUnitTest, get_all_algo_desp
    from cumm.tensorview.gemm import GemmParams, ShuffleStrideType

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    def desp(st, ta, tb, dc):
        for d in get_all_algo_desp():
            if (d.algo == "Tcgen05" and d.dtype_a == tv.bfloat16 and d.dtype_c == dc and d.trans_a == ta
                    and d.trans_b == tb and d.shuffle_type == st):
                return d
        raise KeyError(st)

    out = {}
    g = GemmMainUnitTest()
    n = 8192
    a = torch.randn(n, n, device="cuda").bfloat16()
    b = torch.randn(n, n, device="cuda").bfloat16()
    c = torch.empty(n, n, device="cuda", dtype=torch.bfloat16)
    p = GemmParams()
    p.algo_desp = desp(ShuffleStrideType.kNoShuffle, False, False, tv.bfloat16)
    p.a, p.b, p.c = tv.Tensor(a), tv.Tensor(b), tv.Tensor(c)
    ms = timed(lambda: g.matmul2(p), 10)
    ms_cublas = timed(lambda: torch.matmul(a, b, out=c), 10)
    fl = 2.0 * n ** 3
    out["dense_gemm_8192_bf16"] = {"ms": ms, "tflops": fl / ms / 1e9, "frac_of_peak": fl / ms / 1e9 / peak_tf,
                                   "cublas_ms": ms_cublas, "cublas_tflops": fl / ms_cublas / 1e9}
    rows, ko, ci = 200_000, 64, 128
    do = torch.randn(rows, ko, device="cuda").bfloat16()
    xi = torch.randn(rows, ci, device="cuda").bfloat16()
    perm = torch.randperm(rows, device="cuda").int()
    c2 = torch.empty(ko, ci, device="cuda")
    p2 = GemmParams()
    p2.algo_desp = desp(ShuffleStrideType.kShuffleAB, True, False, tv.float32)
    p2.a, p2.b, p2.c = tv.Tensor(do), tv.Tensor(xi), tv.Tensor(c2)
    p2.a_inds, p2.b_inds = tv.Tensor(perm), tv.Tensor(torch.randperm(rows, device="cuda").int())
    ms2 = timed(lambda: g.matmul2(p2), 20)
    fl2 = 2.0 * rows * ko * ci
    out["shuffle_ab_tallk_200k_64x128_bf16"] = {"ms": ms2, "tflops": fl2 / ms2 / 1e9,
                                                 "frac_of_peak": fl2 / ms2 / 1e9 / peak_tf}
    m = 4_000_000
    src = torch.randn(m, 64, device="cuda").bfloat16()
    dst = torch.empty_like(src)
    idx = torch.randperm(m, device="cuda").int()
    ga, sa = GatherAll(), ScatterAll()
    msg = timed(lambda: ga.gather(tv.Tensor(dst), tv.Tensor(src), tv.Tensor(idx)), 10)
    by = 2.0 * m * 128 + m * 4
    out["gather_4M_rows_128B"] = {"ms": msg, "gbs": by / msg / 1e6, "frac_of_hbm": by / msg / 1e6 / peak_bw}
    msc = timed(lambda: sa.scatter(tv.Tensor(dst), tv.Tensor(src), tv.Tensor(idx)), 10)
    by = 3.0 * m * 128 + m * 4
    out["scatter_add_4M_rows_128B"] = {"ms": msc, "gbs": by / msc / 1e6, "frac_of_hbm": by / msc / 1e6 / peak_bw}
    del a, b, c, src, dst
    torch.cuda.empty_cache()
    return out


def check_batched_and_served(batched: dict, served: dict) -> None:
    """The checker: FP64 oracle errors of the batched result (smallest cloud)
    and of every encoder layer of one served request, and alone-vs-mix
    identity of that request.  Fills the dicts' "max_norm_rel_vs_fp64" keys."""
    import torch

    from cumm import voxelgen as vg
    from oracle import conv_oracle as co
    from oracle import pairs_oracle as po

    def to64(t):
        return t.float().cpu().numpy().astype(np.float64)

    if batched is not None:
        st = batched.pop("state")
        i = int(np.argmin([c.shape[0] for c in st["coords"]]))
        c = st["coords"][i].cpu().numpy()
        pf, _, _ = po.subm_pairs(c, vg.KITTI_SHAPE)
        ref = co.fwd_gather_gemm_scatter(to64(st["feats"][i]), to64(st["weight"]), pf)
        nr, mr, _ = co.rel_err(to64(st["outputs"][i]), ref)
        batched["checked_cloud_voxels"] = int(c.shape[0])
        batched["max_norm_rel_vs_fp64"] = float(nr)
    if served is not None:
        enc, mixed, alone = served.pop("_check")
        served["alone_equals_mix"] = bool(torch.equal(mixed.out, alone.out) and
                                          torch.equal(mixed.out_coords, alone.out_coords))
        rec = []
        enc.forward(alone.coords.cuda(), alone.feats.cuda(), record=rec)
        torch.cuda.synchronize()
        worst = 0.0
        for li, (x, pt, y) in enumerate(rec):
            ref = np.maximum(co.fwd_gather_gemm_scatter(to64(x), to64(enc.wb[li]), pt.pairs_fwd.cpu().numpy()), 0.0)
            worst = max(worst, co.rel_err(to64(y), ref)[0])
        served["checked_request_voxels"] = int(alone.n)
        served["max_norm_rel_vs_fp64"] = float(worst)


def run_b200(args, rank, world, dist):
    import torch

    from cumm import _lib
    from cumm import tensorview as tv
    from cumm import voxelgen as vg
    from cumm.conv.main import build_conv_params_c, get_all_conv_algo_desp
    from cumm.spconv_ops import build_pair_table
    from cumm.tensorview.gemm import ConvOpType, ConvParams

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    lib = _lib.load()
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream

    seed = rank
    coords_np = vg.lidar_voxels(N_VOX, seed=seed)
    rng = np.random.default_rng(seed)
    x_np = rng.standard_normal((N_VOX, C)).astype(np.float32)
    dy_np = rng.standard_normal((N_VOX, K)).astype(np.float32)
    w_np = vg.kaiming_uniform(K, KV, C, seed)
    coords = torch.from_numpy(coords_np).to(dev)
    x = torch.from_numpy(x_np).to(dev).bfloat16()
    dy = torch.from_numpy(dy_np).to(dev).bfloat16()
    w = torch.from_numpy(w_np).to(dev).bfloat16()
    pt = build_pair_table(coords, vg.KITTI_SHAPE)
    P = pt.pair_count()
    flops_op = 2.0 * P * C * K

    def desp_for(op, dt_w=tv.bfloat16):
        for d in get_all_conv_algo_desp():
            if (d.op_type == op and d.algo == "Tcgen05" and d.dtype_input == tv.bfloat16 and
                    d.dtype_weight == dt_w and d.dtype_output == tv.bfloat16 and
                    d.tile_shape[0] == 128):
                return d
        raise KeyError(op)

    out = torch.empty((N_VOX, K), dtype=torch.bfloat16, device=dev)
    din = torch.empty((N_VOX, C), dtype=torch.bfloat16, device=dev)
    dw = torch.empty((K, KV, C), dtype=torch.float32, device=dev)
    mask_out = torch.empty(((N_VOX + 127) // 128,), dtype=torch.int32, device=dev)

    def make(op, pt_, x_, w_, out_, dy_, din_, dw_, mo_):
        p = ConvParams(3, op)
        p.conv_algo_desp = desp_for(op, tv.float32 if op == ConvOpType.kBackwardWeight else tv.bfloat16)
        if op == ConvOpType.kForward:
            p.input, p.weight, p.output = tv.Tensor(x_), tv.Tensor(w_), tv.Tensor(out_)
            p.indices = tv.Tensor(pt_.pairs_fwd)
            p.mask = tv.Tensor(pt_.masks_fwd[0], tv.uint32)
            p.mask_output = tv.Tensor(mo_, tv.uint32)
        elif op == ConvOpType.kBackwardInput:
            p.input, p.weight, p.output = tv.Tensor(din_), tv.Tensor(w_), tv.Tensor(dy_)
            p.indices = tv.Tensor(pt_.pairs_bwd)
            p.mask = tv.Tensor(pt_.masks_fwd[0], tv.uint32)
            p.reverse_mask = True
        else:
            p.input, p.weight, p.output = tv.Tensor(x_), tv.Tensor(dw_), tv.Tensor(dy_)
            p.indices = tv.Tensor(pt_.pairs_fwd)
            p.mask = tv.Tensor(mo_, tv.uint32)
            p.mask_width = 128
        p.mask_argsort = tv.Tensor(pt_.argsorts_fwd[0])
        p.indices_sorted = tv.Tensor(pt_.sorted_indices(
            "bwd" if op == ConvOpType.kBackwardInput else "fwd"))
        if op != ConvOpType.kBackwardWeight:
            p.tile_order = tv.Tensor(pt_.tile_order("fwd"))
        p.stream = sptr
        cp, _ = build_conv_params_c(p)
        need = ctypes.c_int64(0)
        _lib.check(lib.sc_conv_workspace_size(ctypes.byref(cp), ctypes.byref(need)))
        ws = torch.empty(max(need.value, 256), dtype=torch.uint8, device=dev)
        cp.workspace, cp.workspace_bytes = ws.data_ptr(), ws.numel()
        return cp, ws

    ops = [make(op, pt, x, w, out, dy, din, dw, mask_out)
           for op in (ConvOpType.kForward, ConvOpType.kBackwardInput, ConvOpType.kBackwardWeight)]
    call = lib.sc_conv_implicit_gemm

    def step():
        for cp, _ in ops:
            rc = call(ctypes.byref(cp))
            if rc:
                _lib.check(rc)

    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    bits = _lib.device_error_bits(sptr)
    if bits:
        raise RuntimeError(f"device error word {bits} during warm-up")

    n_ev = args.steps
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(n_ev)]
    sampler = ClockSampler(local)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    time.sleep(0.3)
    for s in range(n_ev):
        flush.zero_()
        e = evs[s]
        e[0].record(stream)
        for i, (cp, _) in enumerate(ops):
            rc = call(ctypes.byref(cp))
            if rc:
                _lib.check(rc)
            e[i + 1].record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    if dist is not None:
        dist.barrier()
    per_op = np.array([[evs[s][i].elapsed_time(evs[s][i + 1]) for i in range(3)]
                       for s in range(n_ev)])  # ms
    ms_op = per_op.mean(0)
    ms_step = float(per_op.sum(1).mean())
    bits = _lib.device_error_bits(sptr)
    if bits:
        raise RuntimeError(f"device error word {bits} during timing")
    ms_max = max_over_ranks(ms_step, dist, dev)
    value = whole_job_tflops(3 * flops_op, world, ms_max)

    # ---------------------------------------------------------------- end to end (public API)
    coords_h = torch.from_numpy(coords_np).pin_memory()
    x_h = torch.from_numpy(x_np).bfloat16().pin_memory()
    dy_h = torch.from_numpy(dy_np).bfloat16().pin_memory()
    from cumm.conv.main import ConvMainUnitTest
    cmt = ConvMainUnitTest()
    # Steps are pipelined over three streams (uploads, compute, downloads):
    # step s+1's inputs go up while step s computes and step s-1's results
    # come down.  Step s reuses the device and pinned host buffers of step
    # s - NBUF once that step's results are down; with two sets the upload ->
    # compute -> download chain of one step would pace every second step, with
    # three the host link is the limit.  Every step still copies its inputs in
    # and its results out inside the timed region.
    NBUF = 3
    s_in, s_comp, s_out = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
    bufs = []
    for _ in range(NBUF):
        bufs.append({
            "cd": torch.empty_like(coords_h, device=dev), "xd": torch.empty_like(x_h, device=dev),
            "dyd": torch.empty_like(dy_h, device=dev),
            "outd": torch.empty((N_VOX, K), dtype=torch.bfloat16, device=dev),
            "dind": torch.empty((N_VOX, C), dtype=torch.bfloat16, device=dev),
            "dwd": torch.empty((K, KV, C), dtype=torch.float32, device=dev),
            "mod": torch.empty(((N_VOX + 127) // 128,), dtype=torch.int32, device=dev),
            "out_h": torch.empty((N_VOX, K), dtype=torch.bfloat16).pin_memory(),
            "din_h": torch.empty((N_VOX, C), dtype=torch.bfloat16).pin_memory(),
            "dw_h": torch.empty((K, KV, C), dtype=torch.float32).pin_memory(),
            "ev_in": torch.cuda.Event(), "ev_fwd": torch.cuda.Event(),
            "ev_done": torch.cuda.Event(), "ev_free": torch.cuda.Event(),
        })

    def e2e_step(step: int):
        b = bufs[step % NBUF]
        with torch.cuda.stream(s_in):
            if step >= NBUF:
                s_in.wait_event(b["ev_free"])
            b["cd"].copy_(coords_h, non_blocking=True)
            b["xd"].copy_(x_h, non_blocking=True)
            b["dyd"].copy_(dy_h, non_blocking=True)
            b["ev_in"].record(s_in)
        with torch.cuda.stream(s_comp):
            s_comp.wait_event(b["ev_in"])
            if step >= NBUF:
                s_comp.wait_event(b["ev_free"])
            cptr = s_comp.cuda_stream
            ptd = build_pair_table(b["cd"], vg.KITTI_SHAPE)
            for op in (ConvOpType.kForward, ConvOpType.kBackwardInput, ConvOpType.kBackwardWeight):
                p = ConvParams(3, op)
                p.conv_algo_desp = desp_for(op, tv.float32 if op == ConvOpType.kBackwardWeight
                                            else tv.bfloat16)
                if op == ConvOpType.kForward:
                    p.input, p.weight, p.output = tv.Tensor(b["xd"]), tv.Tensor(w), tv.Tensor(b["outd"])
                    p.indices = tv.Tensor(ptd.pairs_fwd)
                    p.mask = tv.Tensor(ptd.masks_fwd[0], tv.uint32)
                    p.mask_output = tv.Tensor(b["mod"], tv.uint32)
                elif op == ConvOpType.kBackwardInput:
                    p.input, p.weight, p.output = tv.Tensor(b["dind"]), tv.Tensor(w), tv.Tensor(b["dyd"])
                    p.indices = tv.Tensor(ptd.pairs_bwd)
                    p.mask = tv.Tensor(ptd.masks_fwd[0], tv.uint32)
                    p.reverse_mask = True
                else:
                    p.input, p.weight, p.output = tv.Tensor(b["xd"]), tv.Tensor(b["dwd"]), tv.Tensor(b["dyd"])
                    p.indices = tv.Tensor(ptd.pairs_fwd)
                    p.mask = tv.Tensor(b["mod"], tv.uint32)
                    p.mask_width = 128
                p.mask_argsort = tv.Tensor(ptd.argsorts_fwd[0])
                p.indices_sorted = tv.Tensor(ptd.sorted_indices(
                    "bwd" if op == ConvOpType.kBackwardInput else "fwd"))
                if op != ConvOpType.kBackwardWeight:
                    p.tile_order = tv.Tensor(ptd.tile_order("fwd"))
                p.stream = cptr
                cmt.implicit_gemm2(p)
                if op == ConvOpType.kForward:
                    b["ev_fwd"].record(s_comp)
            b["ev_done"].record(s_comp)
        with torch.cuda.stream(s_out):
            s_out.wait_event(b["ev_fwd"])
            b["out_h"].copy_(b["outd"], non_blocking=True)
            s_out.wait_event(b["ev_done"])
            b["din_h"].copy_(b["dind"], non_blocking=True)
            b["dw_h"].copy_(b["dwd"], non_blocking=True)
            b["ev_free"].record(s_out)

    n_e2e = 0 if args.no_e2e else max(3, min(args.steps, 20))
    for st in range(NBUF if n_e2e else 0):
        e2e_step(st)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(s_in)
    for st in range(n_e2e):
        e2e_step(st)
    e1.record(s_out)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / max(n_e2e, 1)
    out_h, din_h, dw_h = bufs[0]["out_h"], bufs[0]["din_h"], bufs[0]["dw_h"]
    e2e_ms = max_over_ranks(e2e_ms, dist, dev)
    e2e_value = whole_job_tflops(3 * flops_op, world, e2e_ms)
    h2d = coords_h.numel() * 4 + x_h.numel() * 2 + dy_h.numel() * 2
    d2h = out_h.numel() * 2 + din_h.numel() * 2 + dw_h.numel() * 4

    # ---------------------------------------------------------------- roofline of the dominant kernel
    names = ["conv_fwd", "conv_dgrad", "conv_wgrad"]
    dom = int(np.argmax(ms_op))
    peak_tf, peak_bw, peak_kind = _peaks()
    achieved = flops_op / (ms_op[dom] * 1e-3) / 1e12
    traffic, traffic_note = recorded_traffic(names[dom])
    # algorithmic bytes of one op: features in + out (or dOut + In for wgrad),
    # weights, the [kv, N] index table, masks and argsort
    alg_bytes = (N_VOX * C * 2 + N_VOX * K * 2 + KV * C * K * (4 if dom == 2 else 2)
                 + KV * N_VOX * 4 + 2 * N_VOX * 4)
    hbm_achieved = alg_bytes / (ms_op[dom] * 1e-3) / 1e9
    roofline = {"bound": "tensor", "kernel": names[dom], "achieved": achieved, "peak": peak_tf,
                "unit": "TFLOP/s", "frac": achieved / peak_tf, "peak_kind": peak_kind,
                "traffic": traffic, "traffic_note": traffic_note,
                "hbm": {"algorithmic_bytes": alg_bytes, "achieved_gbs": hbm_achieved,
                        "peak_gbs": peak_bw, "frac": hbm_achieved / peak_bw}}

    # ---------------------------------------------------------------- batched / served forms (N = 1)
    batched = served = aux = None
    if world == 1 and not args.no_aux:
        aux = run_aux(*_peaks()[:2])
    if world == 1 and not args.no_batched:
        batched = run_batched()
    if world == 1 and not args.no_served:
        served = run_served()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        check_batched_and_served(batched, served)
        _, pf, pb, _, xc, dyc, wc = _cpu_data(0)
        t0 = time.perf_counter()
        cpu_reference_step(xc, wc, dyc, pf, pb)
        tc = time.perf_counter() - t0
        Pc = int((pf >= 0).sum())
        cpu = {"value": 3 * 2.0 * Pc * C * K / tc / 1e12, "unit": "TFLOP/s",
               "cores": os.cpu_count(), "kind": "port",
               "sample": "one full step (fwd+dgrad+wgrad) of the same 200k-voxel layer, numpy "
                         "fp32 gather-GEMM-scatter, BLAS on all host cores"}

    # objects kept only for the checker
    if batched is not None:
        batched.pop("state", None)
    if served is not None:
        served.pop("_check", None)

    if rank == 0:
        line = {
            "metric": "implicit-GEMM spconv TFLOP/s (% BF16 peak)", "value": value,
            "unit": "TFLOP/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "bf16", "data": "synthetic",
            "config": {"workload": WORKLOAD, "voxels": N_VOX, "pairs": P, "C": C, "K": K,
                       "kernel": "3x3x3 subm", "l2": "flushed (256 MB write) between steps",
                       "parallelism": f"replicas{world}"},
            "per_op_ms": {names[i]: float(ms_op[i]) for i in range(3)},
            "per_op_tflops": {names[i]: flops_op / (ms_op[i] * 1e-3) / 1e12 for i in range(3)},
            "pct_bf16_peak": value / world / peak_tf,
            "roofline": roofline,
            "e2e": None if n_e2e == 0 else {
                "value": e2e_value, "unit": "TFLOP/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms,
                "steps": n_e2e, "pipelined_streams": 3, "buffer_sets": NBUF},
            "cpu_baseline": cpu,
            "batched": batched,
            "aux": aux,
            "served": served,
            # this library's kernels per timed step: strand forward, strand
            # backward-input, backward-weight (the dW memset is a cudaMemsetAsync)
            "gpu_launches": 3 * args.steps,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end loop (profiling)")
    ap.add_argument("--no-batched", action="store_true", help="skip the 64-cloud grouped vs sequential run")
    ap.add_argument("--no-served", action="store_true", help="skip the serving point (800 req/s)")
    ap.add_argument("--no-aux", action="store_true", help="skip the GEMM / gather / scatter timings")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if world > 1 and args.impl == "b200":
        import datetime

        import torch
        import torch.distributed as dist_mod
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist_mod.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = dist_mod
    try:
        if args.impl == "reference":
            if rank == 0:
                run_reference(args, rank, world)
        else:
            run_b200(args, rank, world, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
