"""tv.Tensor for the B200 build: a thin wrapper over a torch tensor that keeps
the reference's dtype integers (include/tensorview/dtypes.h:39-62,
cumm/tensorview/__init__.py:40-62), device convention (-1 = CPU, >= 0 = CUDA
device) and the Tensor methods the conv / GEMM path uses
(cumm/core_cc/tensorview_bind.pyi:227-420).

Unsigned 32/16/64-bit tensors are stored in the same-width signed torch dtype
(torch has few kernels for unsigned types) and re-tagged; ``numpy()`` returns
the unsigned view.
"""
from typing import List, Optional, Sequence, Union

import numpy as np
import torch

from . import gemm  # noqa: F401  (tv.gemm.ConvParams etc.)

bool_ = 5
float16 = 7
float32 = 0
float64 = 4
int8 = 3
int16 = 2
int32 = 1
int64 = 8
uint8 = 6
uint16 = 9
uint32 = 10
uint64 = 11
bfloat16 = 12
tf32 = 13
float_e4m3 = 14
float_e5m2 = 15
custom64 = 103
unknown = -1

_TV_TO_TORCH = {
    float32: torch.float32, int32: torch.int32, int16: torch.int16, int8: torch.int8,
    float64: torch.float64, bool_: torch.bool, uint8: torch.uint8, float16: torch.float16,
    int64: torch.int64, uint16: torch.int16, uint32: torch.int32, uint64: torch.int64,
    bfloat16: torch.bfloat16, float_e4m3: torch.float8_e4m3fn, float_e5m2: torch.float8_e5m2,
    custom64: torch.int64,
}
_TORCH_TO_TV = {
    torch.float32: float32, torch.int32: int32, torch.int16: int16, torch.int8: int8,
    torch.float64: float64, torch.bool: bool_, torch.uint8: uint8, torch.float16: float16,
    torch.int64: int64, torch.bfloat16: bfloat16, torch.float8_e4m3fn: float_e4m3,
    torch.float8_e5m2: float_e5m2,
}
_NP_VIEW = {uint16: np.uint16, uint32: np.uint32, uint64: np.uint64}
_BITS = {float32: 32, int32: 32, int16: 16, int8: 8, float64: 64, bool_: 8, uint8: 8,
         float16: 16, int64: 64, uint16: 16, uint32: 32, uint64: 64, bfloat16: 16, tf32: 32,
         float_e4m3: 8, float_e5m2: 8, custom64: 64}


def tvdtype_bitsize(dtype: int) -> int:
    return _BITS[dtype]


def tvdtype_itemsize(dtype: int) -> int:
    return _BITS[dtype] // 8


itemsize_of = tvdtype_itemsize


def _np_to_tv(dt: np.dtype) -> int:
    dt = np.dtype(dt)
    table = {np.dtype(np.float32): float32, np.dtype(np.int32): int32,
             np.dtype(np.int16): int16, np.dtype(np.int8): int8, np.dtype(np.float64): float64,
             np.dtype(np.bool_): bool_, np.dtype(np.uint8): uint8, np.dtype(np.float16): float16,
             np.dtype(np.int64): int64, np.dtype(np.uint16): uint16,
             np.dtype(np.uint32): uint32, np.dtype(np.uint64): uint64}
    if dt not in table:
        raise ValueError(f"unsupported numpy dtype {dt}")
    return table[dt]


def _device_str(device: int) -> str:
    return "cpu" if device < 0 else f"cuda:{device}"


class Tensor:
    """tv.Tensor: torch-backed storage plus a tv dtype tag."""

    __slots__ = ("_t", "_dtype")

    def __init__(self, t: Optional[torch.Tensor] = None, dtype: Optional[int] = None):
        self._t = t
        if t is None:
            self._dtype = unknown
        else:
            self._dtype = dtype if dtype is not None else _TORCH_TO_TV[t.dtype]

    # -- construction helpers -------------------------------------------------------
    @staticmethod
    def from_torch(t: torch.Tensor, dtype: Optional[int] = None) -> "Tensor":
        return Tensor(t, dtype)

    def torch(self) -> torch.Tensor:
        """The underlying torch tensor (unsigned types appear as signed)."""
        return self._t

    # -- properties -------------------------------------------------------------------
    @property
    def shape(self) -> List[int]:
        return [] if self._t is None else list(self._t.shape)

    @property
    def stride(self) -> List[int]:
        return [] if self._t is None else list(self._t.stride())

    @property
    def dtype(self) -> int:
        return self._dtype

    @property
    def size(self) -> int:
        return 0 if self._t is None else self._t.numel()

    @property
    def itemsize(self) -> int:
        return tvdtype_itemsize(self._dtype)

    @property
    def ndim(self) -> int:
        return 0 if self._t is None else self._t.dim()

    @property
    def device(self) -> int:
        if self._t is None or self._t.device.type == "cpu":
            return -1
        return self._t.device.index

    @property
    def pinned(self) -> bool:
        return self._t is not None and self._t.device.type == "cpu" and self._t.is_pinned()

    @property
    def nbytes(self) -> int:
        return self.size * self.itemsize

    def bytesize(self) -> int:
        return self.nbytes

    def empty(self) -> bool:
        return self._t is None or self._t.numel() == 0

    def is_contiguous(self) -> bool:
        return self._t is not None and self._t.is_contiguous()

    def dim(self, axis: int) -> int:
        return self._t.shape[axis]

    def byte_pointer(self) -> int:
        return 0 if self._t is None else self._t.data_ptr()

    def data_ptr(self) -> int:
        return self.byte_pointer()

    # -- views / copies ---------------------------------------------------------------
    def view(self, views: Sequence[int]) -> "Tensor":
        return Tensor(self._t.view(*views), self._dtype)

    def slice_first_axis(self, start: int, end: int) -> "Tensor":
        return Tensor(self._t[start:end], self._dtype)

    def __getitem__(self, idx) -> "Tensor":
        return Tensor(self._t[idx], self._dtype)

    def select(self, dim: int, index: int) -> "Tensor":
        return Tensor(self._t.select(dim, index), self._dtype)

    def unsqueeze(self, axis: int) -> "Tensor":
        return Tensor(self._t.unsqueeze(axis), self._dtype)

    def squeeze(self, axis: Optional[int] = None) -> "Tensor":
        return Tensor(self._t.squeeze() if axis is None else self._t.squeeze(axis), self._dtype)

    def transpose(self, d0: int, d1: int) -> "Tensor":
        return Tensor(self._t.transpose(d0, d1), self._dtype)

    @property
    def T(self) -> "Tensor":
        return self.transpose(0, 1)

    def clone(self, pinned: bool = False) -> "Tensor":
        return Tensor(self._t.clone(), self._dtype)

    def cpu(self, ctx=None) -> "Tensor":
        return Tensor(self._t.cpu(), self._dtype)

    def cuda(self, ctx=None) -> "Tensor":
        return Tensor(self._t.cuda(), self._dtype)

    def copy_(self, other: "Tensor", ctx=None) -> None:
        self._t.copy_(other._t)

    def zero_(self, ctx=None) -> "Tensor":
        self._t.zero_()
        return self

    def fill_int_(self, val: int, ctx=None) -> "Tensor":
        if self._dtype in _NP_VIEW and val >= 2 ** (tvdtype_bitsize(self._dtype) - 1):
            val -= 2 ** tvdtype_bitsize(self._dtype)
        self._t.fill_(int(val))
        return self

    def fill_float_(self, val: float, ctx=None) -> "Tensor":
        self._t.fill_(float(val))
        return self

    def numpy(self) -> np.ndarray:
        t = self._t.detach()
        if t.device.type != "cpu":
            t = t.cpu()
        if self._dtype == bfloat16:
            return t.float().numpy()
        if self._dtype in (float_e4m3, float_e5m2):
            return t.float().numpy()
        arr = t.contiguous().numpy()
        if self._dtype in _NP_VIEW:
            arr = arr.view(_NP_VIEW[self._dtype])
        return arr

    def numpy_view(self) -> np.ndarray:
        if self.device >= 0:
            raise ValueError("numpy_view needs a CPU tensor")
        return self.numpy()

    def __repr__(self) -> str:
        return f"tv.Tensor(shape={self.shape}, dtype={self._dtype}, device={self.device})"


def from_numpy(arr: np.ndarray) -> Tensor:
    dt = _np_to_tv(arr.dtype)
    arr = np.ascontiguousarray(arr)
    if dt in _NP_VIEW:
        signed = {uint16: np.int16, uint32: np.int32, uint64: np.int64}[dt]
        arr = arr.view(signed)
    return Tensor(torch.from_numpy(arr.copy()), dt)


def from_torch(t: torch.Tensor, dtype: Optional[int] = None) -> Tensor:
    return Tensor(t, dtype)


def empty(shape: Sequence[int], dtype: int = float32, device: int = -1, pinned: bool = False,
          managed: bool = False) -> Tensor:
    t = torch.empty(list(shape), dtype=_TV_TO_TORCH[dtype], device=_device_str(device),
                    pin_memory=pinned and device < 0)
    return Tensor(t, dtype)


def zeros(shape: Sequence[int], dtype: int = float32, device: int = -1, pinned: bool = False,
          managed: bool = False) -> Tensor:
    t = torch.zeros(list(shape), dtype=_TV_TO_TORCH[dtype], device=_device_str(device),
                    pin_memory=pinned and device < 0)
    return Tensor(t, dtype)


def full(shape: Sequence[int], val: Union[int, float], dtype: int = float32, device: int = -1,
         pinned: bool = False, managed: bool = False) -> Tensor:
    t = zeros(shape, dtype, device, pinned)
    if dtype in (float32, float64, float16, bfloat16):
        return t.fill_float_(val)
    return t.fill_int_(val)


def cat_first_axis(tens: List[Tensor]) -> Tensor:
    return Tensor(torch.cat([t._t for t in tens], 0), tens[0].dtype)


def get_compute_capability(index: int = -1):
    if not torch.cuda.is_available():
        return (-1, -1)
    return torch.cuda.get_device_capability(max(index, 0))


def is_cpu_only() -> bool:
    return not torch.cuda.is_available()


def torch_dtype(dtype: int):
    return _TV_TO_TORCH[dtype]


def tv_dtype(dt) -> int:
    return _TORCH_TO_TV[dt]


class KernelTimer:
    """CUDA-event pair recorder keyed by name (reference: tv::CUDAKernelTimer,
    include/tensorview/profile/cuda_profiler.h:225-405; Python wrapper
    cumm/tensorview/__init__.py:545-620)."""

    def __init__(self, enable: bool = True):
        self.enable = enable and torch.cuda.is_available()
        self._pairs = {}

    def record(self, name: str, stream: int = 0):
        timer = self

        class _Ctx:
            def __enter__(self_inner):
                if timer.enable:
                    s = torch.cuda.ExternalStream(stream) if stream else torch.cuda.current_stream()
                    self_inner.s = s
                    self_inner.e0 = torch.cuda.Event(enable_timing=True)
                    self_inner.e1 = torch.cuda.Event(enable_timing=True)
                    self_inner.e0.record(s)
                return self_inner

            def __exit__(self_inner, *exc):
                if timer.enable:
                    self_inner.e1.record(self_inner.s)
                    timer._pairs.setdefault(name, []).append((self_inner.e0, self_inner.e1))
                return False

        return _Ctx()

    def get_all_pair_time(self):
        torch.cuda.synchronize()
        return {k: sum(a.elapsed_time(b) for a, b in v) for k, v in self._pairs.items()}
