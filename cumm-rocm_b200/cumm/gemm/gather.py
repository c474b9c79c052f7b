"""Standalone row gather / scatter-add: the reference's ``GatherAll`` and
``ScatterAll`` (cumm/gemm/gather.py:390-620) over ``sc_gather_rows`` /
``sc_scatter_add_rows`` of libcumm_b200.so.

    GatherAll().gather(output, input, indices, tile_m, tile_k_bytes,
                       bytes_per_access, num_threads, stream=0)
        output[i] = input[indices[i]]            (m = indices.dim(0))
    ScatterAll().scatter(output, input, indices, tile_m, tile_k_bytes,
                         bytes_per_access, num_threads, stream=0)
        output[indices[i]] += input[i]

The launch parameters are the reference's tuning keys: ``tile_m`` and
``tile_k_bytes`` are accepted when the reference's table holds the key (the
B200 kernel sizes its own tiles), ``bytes_per_access`` is the access width and
``num_threads`` the block size.  ``gather`` / ``scatter`` also take the
parameters as keywords and default to the widest access that divides the row.
"""
import ctypes
from typing import List, Optional, Tuple

from .. import _lib
from .. import tensorview as tv


def _gather_keys() -> List[Tuple[int, int, int, int]]:
    """(tile_m, tile_k_bytes, bytes_per_access, num_threads) of the
    reference's gather table (gather.py:397-417)."""
    keys = []
    for tk in (4, 8, 16, 32, 64, 128, 256, 512, 1024, 2048):
        for tm in (1, 2, 4, 8):
            for bpa in (4, 8, 16):
                for nt in (64, 128, 256):
                    if nt * bpa > tk * tm:
                        continue
                    keys.append((tm, tk, bpa, nt))
    return keys


def _scatter_keys() -> List[Tuple[int, int, int, int]]:
    """Keys of the reference's scatter table (gather.py:500-523)."""
    keys = []
    for tk in (64, 128, 256, 512, 1024, 2048):
        for tm in (1, 2, 4, 8):
            for bpa in (4, 8, 16):
                for nt in (128, 256):
                    if nt * bpa > tk * tm:
                        continue
                    keys.append((tm, tk, bpa, nt))
    return keys


def _widest_access(row_bytes: int, *ptrs: int) -> int:
    for bpa in (16, 8, 4):
        if row_bytes % bpa == 0 and all(p % bpa == 0 for p in ptrs):
            return bpa
    raise RuntimeError("not supported. use supported() to check first")


def _check_2d(output: tv.Tensor, input: tv.Tensor):
    if not (input.ndim == 2 and output.ndim == 2 and input.dim(1) == output.dim(1)):
        raise RuntimeError("error")
    if input.dtype != output.dtype:
        raise RuntimeError("error")
    for t in (input, output):
        if t.stride[1] != 1 or t.stride[0] != t.dim(1):
            raise ValueError("gather / scatter rows must be contiguous")


def _sync(stream: int):
    import torch
    if stream:
        torch.cuda.ExternalStream(stream).synchronize()
    else:
        torch.cuda.synchronize()


class GatherAll:
    """output[i] = input[indices[i]] on the B200 gather kernel."""

    def __init__(self):
        self._keys = set(_gather_keys())

    @staticmethod
    def get_all_gather_params() -> List[Tuple[int, int, int, int]]:
        return _gather_keys()

    @staticmethod
    def supported(bytes_per_access: int, channel_size: int, dtype: int) -> bool:
        return (channel_size * tv.tvdtype_itemsize(dtype)) % bytes_per_access == 0

    @staticmethod
    def stream_synchronize(stream: int = 0):
        _sync(stream)

    def gather(self, output: tv.Tensor, input: tv.Tensor, indices: tv.Tensor,
               tile_m: Optional[int] = None, tile_k_bytes: Optional[int] = None,
               bytes_per_access: Optional[int] = None, num_threads: Optional[int] = None,
               stream: int = 0, sync_check: bool = False):
        _lib.require_cuda()
        _check_2d(output, input)
        m = indices.dim(0)
        if output.dim(0) < m:
            raise RuntimeError("error: output has fewer rows than indices")
        row_bytes = input.dim(1) * input.itemsize
        if tile_m is not None:
            if (tile_m, tile_k_bytes, bytes_per_access, num_threads) not in self._keys:
                raise RuntimeError("can't find a sutable gather")
        bpa = bytes_per_access or _widest_access(row_bytes, input.data_ptr(), output.data_ptr())
        nt = num_threads or 256
        lib = _lib.load()
        _lib.check(lib.sc_gather_rows(ctypes.c_void_p(output.data_ptr()), ctypes.c_void_p(input.data_ptr()),
                                      input.dim(0), ctypes.c_void_p(indices.data_ptr()), m, row_bytes,
                                      bpa, nt, ctypes.c_void_p(stream)))
        if sync_check:
            bits = _lib.device_error_bits(stream)
            if bits:
                raise RuntimeError(f"device error word {bits} (1 = index outside the input)")


class ScatterAll:
    """output[indices[i]] += input[i] on the B200 scatter kernel (fp32 like the
    reference; fp16 / bf16 added in fp32 and rounded once)."""

    def __init__(self):
        self._keys = set(_scatter_keys())

    @staticmethod
    def get_all_scatter_params() -> List[Tuple[int, int, int, int]]:
        return _scatter_keys()

    def supported_scatter(self, tile_m: int, tile_k_bytes: int, bytes_per_access: int,
                          num_threads: int, channel_size: int, dtype: int) -> bool:
        if (tile_m, tile_k_bytes, bytes_per_access, num_threads) not in self._keys:
            return False
        if dtype not in (tv.float32, tv.float16, tv.bfloat16):
            return False
        return (channel_size * tv.tvdtype_itemsize(dtype)) % bytes_per_access == 0

    @staticmethod
    def stream_synchronize(stream: int = 0):
        _sync(stream)

    def scatter(self, output: tv.Tensor, input: tv.Tensor, indices: tv.Tensor,
                tile_m: Optional[int] = None, tile_k_bytes: Optional[int] = None,
                bytes_per_access: Optional[int] = None, num_threads: Optional[int] = None,
                stream: int = 0, sync_check: bool = False):
        _lib.require_cuda()
        _check_2d(output, input)
        m = indices.dim(0)
        if input.dim(0) < m:
            raise RuntimeError("error: input has fewer rows than indices")
        row_bytes = input.dim(1) * input.itemsize
        if tile_m is not None:
            if (tile_m, tile_k_bytes, bytes_per_access, num_threads) not in self._keys:
                raise RuntimeError("can't find a sutable scatter")
        bpa = bytes_per_access or _widest_access(row_bytes, input.data_ptr(), output.data_ptr())
        nt = num_threads or 256
        lib = _lib.load()
        _lib.check(lib.sc_scatter_add_rows(ctypes.c_void_p(output.data_ptr()), output.dim(0),
                                           ctypes.c_void_p(input.data_ptr()),
                                           ctypes.c_void_p(indices.data_ptr()), m, input.dim(1),
                                           int(input.dtype), bpa, nt, ctypes.c_void_p(stream)))
        if sync_check:
            bits = _lib.device_error_bits(stream)
            if bits:
                raise RuntimeError(f"device error word {bits} (1 = index outside the output)")
