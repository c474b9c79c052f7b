"""Indice-pair / mask builder and mask argsort for the mask-implicit-GEMM
convolution, on the GPU kernels of libcumm_b200.so.

The reference consumes these from spconv (``SpconvOps.generate_subm_conv_inds``
and ``SpconvOps.sort_1d_by_key_split``, called at
cumm/conv/main_real_spconv.py:79-145); spconv is not part of the reference
tree, so the semantics are defined here (and restated on the CPU in
oracle/pairs_oracle.py):

* offsets k = (kz * KY + ky) * KX + kx over the kernel box, cross-correlation
  (the same indexing as ``torch.nn.functional.conv3d`` with a [K, C, kz, ky, kx]
  weight);
* ``pairs[0][k][o]`` = input index feeding output o through offset k (-1 if
  none), ``pairs[1][k][i]`` = output index fed by input i through offset k;
* ``mask_fwd[o]`` bit k <=> pairs[0][k][o] >= 0, ``mask_bwd[i]`` bit k <=>
  pairs[1][k][i] >= 0; for submanifold convs mask_bwd is the bit-reversed
  mask_fwd, which the backward-input kernel derives with ``reverse_mask``;
* strided-conv outputs are numbered in ascending (batch, z, y, x) order.
"""
import ctypes
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import torch

from . import _lib
from . import tensorview as tv

# split masks of spconv's two-way MaskSplitImplicitGemm (main_real_spconv.py:120-121)
SPLIT_MASKS_27 = (0b11111111111111, 0b1111111111111 << 14)


def _vp(t: torch.Tensor):
    return ctypes.c_void_p(t.data_ptr()) if t is not None and t.numel() > 0 else None


def _i32x3(v: Sequence[int]) -> torch.Tensor:
    return torch.tensor(list(v), dtype=torch.int32)


def _stream(stream: int):
    return ctypes.c_void_p(stream) if stream else (
        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))


def _ws(nbytes: int, device) -> torch.Tensor:
    return torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device)


def _t(x):
    return x.torch() if isinstance(x, tv.Tensor) else x


class SpconvOps:
    """GPU pair builder with spconv's operation names."""

    @staticmethod
    def generate_subm_conv_inds(indices, indice_pairs, indice_pair_mask, spatial_shape: Sequence[int],
                                ksize: Sequence[int], dilation: Sequence[int] = (1, 1, 1),
                                indice_num_per_loc=None, split_masks: Optional[Sequence[int]] = None,
                                stream: int = 0) -> int:
        """Fills ``indice_pairs`` [2, kv, N] int32 and ``indice_pair_mask``
        [S, N] uint32 (S = 1, or 2 with ``split_masks``: row j holds
        mask & split_masks[j]) for a submanifold conv; returns N."""
        _lib.require_cuda()
        lib = _lib.load()
        coords = _t(indices)
        pairs = _t(indice_pairs)
        masks = _t(indice_pair_mask)
        n = coords.shape[0]
        kv = int(ksize[0] * ksize[1] * ksize[2])
        if tuple(pairs.shape) != (2, kv, n) or pairs.dtype != torch.int32:
            raise ValueError(f"indice_pairs must be int32 [2, {kv}, {n}]")
        dev = coords.device
        need = ctypes.c_int64(0)
        _lib.check(lib.sc_pairs_workspace_size(n, kv, 1, ctypes.byref(need)))
        ws = _ws(need.value, dev)
        sp, ks, dl = _i32x3(spatial_shape), _i32x3(ksize), _i32x3(dilation)
        mask_full = torch.empty(n, dtype=torch.int32, device=dev)
        s = _stream(stream)
        _lib.check(lib.sc_build_subm_pairs(
            _vp(coords), n, ctypes.c_void_p(sp.data_ptr()), ctypes.c_void_p(ks.data_ptr()),
            ctypes.c_void_p(dl.data_ptr()), _vp(pairs[0]), _vp(pairs[1]), _vp(mask_full), _vp(ws),
            ws.numel(), s))
        if split_masks is None:
            masks[0].copy_(mask_full)
        else:
            for j, sm in enumerate(split_masks):
                masks[j].copy_(mask_full & _as_i32(sm))
        if indice_num_per_loc is not None:
            _t(indice_num_per_loc).copy_((pairs[0] >= 0).sum(1).to(torch.int32))
        return n

    @staticmethod
    def generate_conv_inds(indices, batch_size: int, spatial_shape: Sequence[int],
                           ksize: Sequence[int], stride: Sequence[int], padding: Sequence[int],
                           dilation: Sequence[int] = (1, 1, 1), stream: int = 0):
        """Regular (strided) sparse conv: returns (out_inds [n_out, 4],
        pairs_fwd [kv, n_out], pairs_bwd [kv, n_in], mask_fwd [n_out],
        mask_bwd [n_in], out_spatial_shape).  Synchronises once (n_out sizes
        the outputs)."""
        _lib.require_cuda()
        lib = _lib.load()
        coords = _t(indices)
        n = coords.shape[0]
        dev = coords.device
        kv = int(ksize[0] * ksize[1] * ksize[2])
        need = ctypes.c_int64(0)
        _lib.check(lib.sc_pairs_workspace_size(n, kv, 0, ctypes.byref(need)))
        ws = _ws(need.value, dev)
        sp, ks, st, pd, dl = (_i32x3(spatial_shape), _i32x3(ksize), _i32x3(stride), _i32x3(padding),
                              _i32x3(dilation))
        out_sp = torch.zeros(3, dtype=torch.int32)
        n_out = ctypes.c_int64(0)
        s = _stream(stream)
        args = (ctypes.c_void_p(sp.data_ptr()), ctypes.c_void_p(ks.data_ptr()),
                ctypes.c_void_p(st.data_ptr()), ctypes.c_void_p(pd.data_ptr()),
                ctypes.c_void_p(dl.data_ptr()))
        _lib.check(lib.sc_build_conv_outputs(_vp(coords), n, batch_size, *args,
                                             ctypes.c_void_p(out_sp.data_ptr()),
                                             ctypes.byref(n_out), _vp(ws), ws.numel(), s))
        no = int(n_out.value)
        out_inds = torch.empty((no, 4), dtype=torch.int32, device=dev)
        pf = torch.empty((kv, no), dtype=torch.int32, device=dev)
        pb = torch.empty((kv, n), dtype=torch.int32, device=dev)
        mf = torch.empty(no, dtype=torch.int32, device=dev)
        mb = torch.empty(n, dtype=torch.int32, device=dev)
        _lib.check(lib.sc_build_conv_pairs(_vp(coords), n, batch_size, *args, no, _vp(out_inds),
                                           _vp(pf), _vp(pb), _vp(mf), _vp(mb), _vp(ws), ws.numel(),
                                           s))
        return out_inds, pf, pb, mf, mb, [int(x) for x in out_sp]

    @staticmethod
    def sort_1d_by_key_split(data, mask, stream: int = 0):
        """Stable sort of ``data`` (uint32 [N], in place) by ``data & mask``;
        returns the argsort (int32 [N]).  ``mask`` is an int or a one-element
        tensor (reference call: main_real_spconv.py:141-145)."""
        _lib.require_cuda()
        lib = _lib.load()
        d = _t(data)
        if isinstance(mask, (tv.Tensor, torch.Tensor)):
            m = int(_t(mask).reshape(-1)[0].item()) & 0xffffffff
        else:
            m = int(mask) & 0xffffffff
        n = d.numel()
        out = torch.empty(n, dtype=torch.int32, device=d.device)
        need = ctypes.c_int64(0)
        _lib.check(lib.sc_sort_workspace_size(n, ctypes.byref(need)))
        ws = _ws(need.value, d.device)
        _lib.check(lib.sc_sort_masks_split(_vp(d), n, ctypes.c_uint32(m), _vp(out), _vp(ws),
                                           ws.numel(), _stream(stream)))
        if isinstance(data, tv.Tensor):
            return tv.Tensor(out, tv.int32)
        return out

    @staticmethod
    def sort_1d_by_key(data, stream: int = 0):
        return SpconvOps.sort_1d_by_key_split(data, 0xffffffff, stream)

    @staticmethod
    def sort_indices(indices, argsort, stream: int = 0):
        """indices [kv, N] permuted into argsort order: out[k][r] =
        indices[k][argsort[r]] (the optional ConvParams.indices_sorted)."""
        _lib.require_cuda()
        lib = _lib.load()
        ind, srt = _t(indices), _t(argsort)
        kv, n = ind.shape
        out = torch.empty_like(ind)
        _lib.check(lib.sc_sort_indices(_vp(ind), kv, n, _vp(srt), _vp(out), _stream(stream)))
        if isinstance(indices, tv.Tensor):
            return tv.Tensor(out, tv.int32)
        return out


    @staticmethod
    def tile_order(mask, kv: int, mask_filter: int = 0xffffffff, reverse: bool = False,
                   stream: int = 0):
        """Largest-first order of the 128-row tiles of the sorted masks (the
        optional ConvParams.tile_order): tiles by the number of offsets their
        OR-ed masks visit, heaviest first."""
        _lib.require_cuda()
        lib = _lib.load()
        m = _t(mask)
        n = int(m.numel())
        out = torch.empty(((n + 127) // 128,), dtype=torch.int32, device=m.device)
        need = ctypes.c_int64(0)
        _lib.check(lib.sc_tile_order_workspace_size(n, ctypes.byref(need)))
        ws = torch.empty((max(int(need.value), 1),), dtype=torch.uint8, device=m.device)
        _lib.check(lib.sc_tile_order(_vp(m), n, ctypes.c_uint32(mask_filter & 0xffffffff), kv,
                                     1 if reverse else 0, _vp(out), _vp(ws), ws.numel(),
                                     _stream(stream)))
        if isinstance(mask, tv.Tensor):
            return tv.Tensor(out, tv.int32)
        return out


def _as_i32(v: int) -> int:
    v &= 0xffffffff
    return v - (1 << 32) if v >= (1 << 31) else v


@dataclass
class PairTable:
    """Device-resident pair tables of one sparse conv layer (the inputs of
    ConvParams for fwd / dgrad / wgrad)."""
    n_in: int
    n_out: int
    kv: int
    subm: bool
    pairs_fwd: torch.Tensor            # [kv, n_out] int32
    pairs_bwd: torch.Tensor            # [kv, n_in] int32
    masks_fwd: List[torch.Tensor]      # per split: sorted masks [n_out] (int32 storage of uint32)
    argsorts_fwd: List[torch.Tensor]   # per split: [n_out] int32
    masks_bwd: List[torch.Tensor] = field(default_factory=list)   # strided only
    argsorts_bwd: List[torch.Tensor] = field(default_factory=list)
    split_masks: List[int] = field(default_factory=list)
    out_inds: Optional[torch.Tensor] = None
    out_spatial: Optional[List[int]] = None

    def pair_count(self) -> int:
        """P = number of valid (input, output) pairs."""
        return int((self.pairs_fwd >= 0).sum().item())

    def sorted_indices(self, which: str = "fwd", split: int = 0) -> torch.Tensor:
        """Index table of `which` ('fwd' or 'bwd') permuted into the argsort
        order the matching convolution uses: forward and backward-weight walk
        pairs_fwd in argsorts_fwd order; backward-input walks pairs_bwd in
        argsorts_fwd order (submanifold, reverse_mask) or argsorts_bwd order
        (strided).  Cached per (which, split)."""
        cache = self.__dict__.setdefault("_sorted_cache", {})
        key = (which, split)
        if key not in cache:
            if which == "fwd":
                cache[key] = SpconvOps.sort_indices(self.pairs_fwd, self.argsorts_fwd[split])
            else:
                order = self.argsorts_fwd[split] if self.subm else self.argsorts_bwd[split]
                cache[key] = SpconvOps.sort_indices(self.pairs_bwd, order)
        return cache[key]

    def tile_order(self, which: str = "fwd", split: int = 0) -> torch.Tensor:
        """Largest-first tile order (ConvParams.tile_order) for the masks
        `which` uses: forward and (submanifold) backward-input share
        masks_fwd[split], whose offset counts are the same in both directions;
        a strided backward-input uses masks_bwd[split].  Cached per (which,
        split)."""
        cache = self.__dict__.setdefault("_order_cache", {})
        key = ("fwd" if which == "fwd" or self.subm else "bwd", split)
        if key not in cache:
            masks = self.masks_fwd if key[0] == "fwd" else self.masks_bwd
            cache[key] = SpconvOps.tile_order(masks[split], self.kv, self.split_masks[split]
                                              if self.split_masks else 0xffffffff)
        return cache[key]


def build_pair_table(coords: torch.Tensor, spatial_shape: Sequence[int], ksize=(3, 3, 3),
                     stride=(1, 1, 1), padding=(1, 1, 1), dilation=(1, 1, 1), subm: bool = True,
                     batch_size: int = 1, num_split: int = 1, stream: int = 0) -> PairTable:
    """Builds pairs, masks and (split) argsorts for one layer on the GPU, the
    way spconv's get_indice_pairs_implicit_gemm prepares them for
    MaskImplicitGemm (num_split 1) or MaskSplitImplicitGemm (num_split 2)."""
    kv = int(ksize[0] * ksize[1] * ksize[2])
    if num_split == 1:
        splits = [0xffffffff]
    elif num_split == 2:
        half = kv // 2 + 1
        splits = [(1 << half) - 1, ((1 << kv) - 1) & ~((1 << half) - 1)]
    else:
        raise ValueError("num_split must be 1 or 2")
    dev = coords.device
    n = coords.shape[0]
    if subm:
        pairs = torch.empty((2, kv, n), dtype=torch.int32, device=dev)
        m = torch.empty((1, n), dtype=torch.int32, device=dev)
        SpconvOps.generate_subm_conv_inds(coords, pairs, m, spatial_shape, ksize, dilation,
                                          stream=stream)
        masks, sorts = [], []
        for sm in splits:
            mm = m[0].clone()
            sorts.append(SpconvOps.sort_1d_by_key_split(mm, sm, stream))
            masks.append(mm)
        return PairTable(n, n, kv, True, pairs[0], pairs[1], masks, sorts, split_masks=splits,
                         out_inds=coords, out_spatial=list(spatial_shape))
    out_inds, pf, pb, mf, mb, out_sp = SpconvOps.generate_conv_inds(
        coords, batch_size, spatial_shape, ksize, stride, padding, dilation, stream)
    masks, sorts, masks_b, sorts_b = [], [], [], []
    for sm in splits:
        mm = mf.clone()
        sorts.append(SpconvOps.sort_1d_by_key_split(mm, sm, stream))
        masks.append(mm)
        mb2 = mb.clone()
        sorts_b.append(SpconvOps.sort_1d_by_key_split(mb2, sm, stream))
        masks_b.append(mb2)
    return PairTable(n, out_inds.shape[0], kv, False, pf, pb, masks, sorts, masks_b, sorts_b,
                     splits, out_inds, out_sp)
