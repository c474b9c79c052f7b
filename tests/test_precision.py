"""FP8-E4M3 quantizers of cumm.precision (CPU)."""
import numpy as np
import torch

from cumm.precision import quantize_act_fp8, quantize_weight_fp8


def test_fp8_scales_fold_exactly():
    """The activation tile scale folded into the weights reproduces the
    unquantized product up to E4M3 rounding only (checked on the CPU)."""
    rng = np.random.default_rng(0)
    x = torch.from_numpy(rng.standard_normal((512, 128)).astype(np.float32) * 3.0)
    w = torch.from_numpy(rng.standard_normal((32, 27, 128)).astype(np.float32) * 0.05)
    xq, sx = quantize_act_fp8(x)
    wq, sw = quantize_weight_fp8(w, sx)
    assert sx.shape == (2,) and sw.shape == (32,)
    y = (xq.double() @ wq.double()[:, 5, :].T) * sw.double()[None, :]
    ref = x.double() @ w.double()[:, 5, :].T
    assert float((y - ref).norm() / ref.norm()) < 6e-2
