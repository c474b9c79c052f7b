"""tv.gemm: enums, algorithm descriptors and parameter structs of the GEMM /
sparse-conv operator surface (reference: include/tensorview/gemm/core/params.h:24-428,
constants.h:20-57, pybind stubs cumm/core_cc/tensorview_bind.pyi:596-929).
"""
import enum
from typing import List, Tuple


class ConvOpType(enum.IntEnum):
    kForward = 0
    kBackwardInput = 1
    kBackwardWeight = 2


class ConvMode(enum.IntEnum):
    kConvolution = 0
    kCrossCorrelation = 1


class ConvIterAlgo(enum.IntEnum):
    kAnalytic = 0
    kOptimized = 1


class ConvLayoutType(enum.IntEnum):
    kChannelFirst = 0
    kChannelLast = 1
    kSpatialFirst = 2


class ShuffleStrideType(enum.IntEnum):
    kNoShuffle = 0
    kShuffleAC = 1
    kShuffleAB = 2


class SparseConvAlgo(enum.IntEnum):
    kNative = 0
    kMaskImplicitGemm = 1
    kMaskSplitImplicitGemm = 2


class Activation(enum.IntEnum):
    kNone = 0
    kReLU = 1
    kSigmoid = 2
    kLeakyReLU = 3


# algo strings: the reference's tensor-op families map to the tcgen05 kernels
# on sm_100a; "Simt" is the fp32 FFMA family.
TENSOR_OP_ALGOS = ("Tcgen05", "Turing", "Ampere", "Volta")
SIMT_ALGOS = ("Simt",)

_SHORT = {0: "f32", 1: "s32", 2: "s16", 3: "s8", 4: "f64", 5: "b1", 6: "u8", 7: "f16",
          8: "s64", 9: "u16", 10: "u32", 11: "u64", 12: "bf16", 13: "tf32", 14: "e4m3",
          15: "e5m2"}


class GemmAlgoDesp:
    """Mirror of tv::gemm::GemmAlgoDesp (params.h:24-164)."""

    def __init__(self):
        self.dtype_a = -1
        self.dtype_b = -1
        self.dtype_c = -1
        self.trans_a_ = -1
        self.trans_b_ = -1
        self.trans_c_ = -1
        self.tile_shape: Tuple[int, int, int] = (-1, -1, -1)
        self.warp_tile_shape: Tuple[int, int, int] = (-1, -1, -1)
        self.num_stage = -1
        self.dacc = -1
        self.dcomp = -1
        self.algo = ""
        self.tensorop: Tuple[int, int, int] = (-1, -1, -1)
        self.split_k_serial_ = 0
        self.split_k_parallel_ = 0
        self.shuffle_type = ShuffleStrideType.kNoShuffle
        self.element_per_access_a = -1
        self.element_per_access_b = -1
        self.element_per_access_c = -1
        self.access_per_vector = 1
        self.is_nvrtc = False
        self.min_arch = (0, 0)

    # bool views of the int fields
    @property
    def trans_a(self) -> bool:
        return self.trans_a_ == 1

    @trans_a.setter
    def trans_a(self, v: bool):
        self.trans_a_ = 1 if v else 0

    @property
    def trans_b(self) -> bool:
        return self.trans_b_ == 1

    @trans_b.setter
    def trans_b(self, v: bool):
        self.trans_b_ = 1 if v else 0

    @property
    def trans_c(self) -> bool:
        return self.trans_c_ == 1

    @trans_c.setter
    def trans_c(self, v: bool):
        self.trans_c_ = 1 if v else 0

    @property
    def split_k_serial(self) -> bool:
        return self.split_k_serial_ == 1

    @split_k_serial.setter
    def split_k_serial(self, v: bool):
        self.split_k_serial_ = 1 if v else 0

    @property
    def split_k_parallel(self) -> bool:
        return self.split_k_parallel_ == 1

    @split_k_parallel.setter
    def split_k_parallel(self, v: bool):
        self.split_k_parallel_ = 1 if v else 0

    def check_valid(self):
        if self.trans_a_ == -1 or self.trans_b_ == -1 or self.trans_c_ == -1 or not self.algo:
            raise RuntimeError("trans_a, trans_b, trans_c and algo must be set")
        for i in range(3):
            if self.tile_shape[i] <= 0 or self.warp_tile_shape[i] <= 0:
                raise RuntimeError(
                    f"tile_shape and warp_tile_shape must be set, but they are "
                    f"{self.tile_shape} {self.warp_tile_shape}")
        if self.algo not in ("Simt", "SimtDP4A", "SimtDP2A"):
            for i in range(3):
                if self.tensorop[i] <= 0:
                    raise RuntimeError(f"tensorop must be set, but they are {self.tensorop}")
        if self.dtype_a == -1 or self.dtype_b == -1 or self.dtype_c == -1:
            raise RuntimeError("dacc and dcomp must be set to valid value")
        if self.dacc == -1 or self.dcomp == -1:
            raise RuntimeError("dacc and dcomp must be set to valid value")
        if self.num_stage <= 0:
            raise RuntimeError("num_stage must larger than zero")

    def __repr__(self) -> str:
        self.check_valid()
        s = (f"{self.algo}_{_SHORT.get(self.dtype_a)}{_SHORT.get(self.dtype_b)}"
             f"{_SHORT.get(self.dtype_c)}{_SHORT.get(self.dacc)}{_SHORT.get(self.dcomp)}")
        s += ("n" if self.trans_a else "t") + ("n" if self.trans_b else "t") + (
            "n" if self.trans_c else "t")
        ts, wts = self.tile_shape, self.warp_tile_shape
        s += f"_m{ts[0]}n{ts[1]}k{ts[2]}m{wts[0]}n{wts[1]}k{wts[2]}A{self.access_per_vector}"
        if self.tensorop[0] != -1:
            s += f"T{self.tensorop[0]}{self.tensorop[1]}{self.tensorop[2]}"
        s += f"_{self.num_stage}{int(self.split_k_serial)}{int(self.split_k_parallel)}"
        if self.shuffle_type != ShuffleStrideType.kNoShuffle:
            s += f"_S{int(self.shuffle_type)}"
        return s

    def copy(self):
        import copy
        return copy.copy(self)

    def supported(self, m: int, n: int, k: int) -> bool:
        lda = m if self.trans_a else k
        ldb = k if self.trans_b else n
        ldc = m if self.trans_c else n
        return self.supported_ldx(lda, ldb, ldc)

    def supported_ldx(self, lda: int, ldb: int, ldc: int) -> bool:
        res = True
        if self.element_per_access_a > 0:
            res &= lda % self.element_per_access_a == 0
        if self.element_per_access_b > 0:
            res &= ldb % self.element_per_access_b == 0
        if self.element_per_access_c > 0:
            res &= ldc % self.element_per_access_c == 0
        return res

    def query_workspace_size(self, m: int, n: int, k: int, split_k_slices: int) -> int:
        """Bytes of workspace the sm_100a GEMM kernels need (no split-K
        semaphores: the reduction-over-rows path accumulates in an fp32 [m, n]
        buffer; a row-major B for the row-gather path is transposed once)."""
        from . import itemsize_of
        if self.algo in SIMT_ALGOS or self.dtype_a == 0:
            return 0
        es = itemsize_of(self.dtype_a)
        rowmajor_a = self.shuffle_type == ShuffleStrideType.kShuffleAC or (
            self.shuffle_type == ShuffleStrideType.kNoShuffle and not self.trans_a)
        if rowmajor_a:
            return 0 if self.trans_b else _a256(n * k * es)
        b = _a256(m * n * 4)
        if self.trans_b:
            b += _a256(n * k * es)
        return b


def _a256(x: int) -> int:
    return (x + 255) & ~255


class ConvAlgoDesp(GemmAlgoDesp):
    """Mirror of tv::gemm::ConvAlgoDesp (params.h:166-327)."""

    def __init__(self, ndim: int, op_type: ConvOpType):
        super().__init__()
        self.ndim = ndim
        self.op_type = ConvOpType(op_type)
        self.iter_algo = ConvIterAlgo.kOptimized
        self.layout_i = ConvLayoutType.kChannelLast
        self.layout_w = ConvLayoutType.kChannelLast
        self.layout_o = ConvLayoutType.kChannelLast
        self.interleave_i = 1
        self.interleave_w = 1
        self.interleave_o = 1
        self.mask_sparse = False
        self.increment_k_first = False
        self.is_int8_inference = False
        self.dynamic_mask = False

    @staticmethod
    def conv_iwo_012_to_abc(op_type: ConvOpType) -> List[int]:
        return {0: [0, 1, 2], 1: [2, 1, 0], 2: [1, 2, 0]}[int(op_type)]

    @staticmethod
    def gemm_abc_012_to_iwo(op_type: ConvOpType) -> List[int]:
        return {0: [0, 1, 2], 1: [2, 1, 0], 2: [2, 0, 1]}[int(op_type)]

    def _abc(self):
        return [self.dtype_a, self.dtype_b, self.dtype_c]

    @property
    def dtype_input(self) -> int:
        return self._abc()[self.conv_iwo_012_to_abc(self.op_type)[0]]

    @property
    def dtype_weight(self) -> int:
        return self._abc()[self.conv_iwo_012_to_abc(self.op_type)[1]]

    @property
    def dtype_output(self) -> int:
        return self._abc()[self.conv_iwo_012_to_abc(self.op_type)[2]]

    def __repr__(self) -> str:
        s = super().__repr__()
        s += f"_C{self.ndim}{int(self.op_type)}{int(self.iter_algo)}"
        li = "F" if self.layout_i == ConvLayoutType.kChannelFirst else "L"
        lw = "F" if self.layout_w == ConvLayoutType.kChannelFirst else "L"
        lo = "F" if self.layout_o == ConvLayoutType.kChannelFirst else "L"
        s += li + lw + lo
        if self.mask_sparse:
            s += "_" + ("SK" if self.increment_k_first else "SF")
        if self.dynamic_mask:
            s += "D"
        if self.is_int8_inference:
            s += "_S8"
        return s

    def supported(self, m: int, n: int, k: int, C: int, K: int, mask_width: int) -> bool:
        res = GemmAlgoDesp.supported(self, m, n, k)
        if self.mask_sparse:
            if self.op_type == ConvOpType.kForward:
                res &= C % self.element_per_access_a == 0
            elif self.op_type == ConvOpType.kBackwardInput:
                res &= K % self.element_per_access_a == 0
            else:
                res &= mask_width % self.tile_shape[2] == 0
                res &= K % self.element_per_access_a == 0
                res &= C % self.element_per_access_b == 0
        return res

    def query_conv_workspace_size(self, m: int, n: int, k: int, split_k_slices: int,
                                  kv: int) -> int:
        """Bytes of workspace the sm_100a conv kernels use: the tensor-core
        forward and backward-input kernels keep a 256-byte tile counter for
        their dynamic scheduler (forward runs without it, dealing tiles
        statically); backward-input also stages the weight transposed
        ([C, kv, K]); backward-weight accumulates dW in fp32 ([K, kv, C])."""
        from . import itemsize_of
        if self.op_type == ConvOpType.kForward:
            return 0 if self.algo in SIMT_ALGOS else 256
        if self.op_type == ConvOpType.kBackwardInput:
            # mnk = (N, C, K * kv)
            C, K = n, k // kv
            if self.algo in SIMT_ALGOS:
                return 0
            return 256 + _a256(K * kv * C * itemsize_of(self.dtype_a))
        # mnk = (K, C * kv, N)
        K, C = m, n // kv
        return _a256(K * kv * C * 4)

    def supported_ldx_conv(self, ldi: int, ldw: int, ldo: int) -> bool:
        epas = [self.element_per_access_a, self.element_per_access_b, self.element_per_access_c]
        idx = self.conv_iwo_012_to_abc(self.op_type)
        res = True
        for ld, j in zip((ldi, ldw, ldo), idx):
            if epas[j] > 0:
                res &= ld % epas[j] == 0
        return res


class GemmParams:
    """Mirror of tv::gemm::GemmParams (params.h:329-390)."""

    def __init__(self, timer=None):
        from . import Tensor
        self.algo_desp = GemmAlgoDesp()
        self._a = Tensor()
        self._b = Tensor()
        self._c = Tensor()
        self._d = Tensor()
        self.split_k_slices = 1
        self.workspace = Tensor()
        self.a_inds = Tensor()
        self.b_inds = Tensor()
        self.c_inds = Tensor()
        self.alpha = 1.0
        self.beta = 0.0
        self.act_alpha = 0.0
        self.act_beta = 0.0
        self.act_type = Activation.kNone
        self.stream = 0
        self.timer = timer

    def check_valid(self):
        self.algo_desp.check_valid()
        if self._a.empty() or self._b.empty() or self._c.empty():
            raise RuntimeError("a,b,c must not empty")
        if self.algo_desp.shuffle_type == ShuffleStrideType.kShuffleAC:
            if self.c_inds.empty():
                raise RuntimeError("a_inds,c_inds tensor must not empty")
        elif self.algo_desp.shuffle_type == ShuffleStrideType.kShuffleAB:
            if self.a_inds.empty() or self.b_inds.empty():
                raise RuntimeError("a_inds,b_inds tensor must not empty")

    @property
    def a(self):
        return self._a

    @a.setter
    def a(self, v):
        self._a = v
        self.algo_desp.dtype_a = v.dtype

    @property
    def b(self):
        return self._b

    @b.setter
    def b(self, v):
        self._b = v
        self.algo_desp.dtype_b = v.dtype

    @property
    def c(self):
        return self._c

    @c.setter
    def c(self, v):
        self._c = v
        self.algo_desp.dtype_c = v.dtype

    @property
    def d(self):
        return self._d

    @d.setter
    def d(self, v):
        if v.dtype != self._c.dtype:
            raise RuntimeError("d dtype must equal to c")
        self._d = v


class ConvParams:
    """Mirror of tv::gemm::ConvParams (params.h:392-428)."""

    def __init__(self, ndim: int, op_type: ConvOpType, timer=None):
        from . import Tensor
        self.conv_algo_desp = ConvAlgoDesp(ndim, op_type)
        self.input = Tensor()
        self.weight = Tensor()
        self.output = Tensor()
        self.output_add = Tensor()
        self.bias = Tensor()
        self.scale = Tensor()
        self.split_k_slices = 1
        self.padding: List[int] = []
        self.stride: List[int] = []
        self.dilation: List[int] = []
        self.alpha = 1.0
        self.beta = 0.0
        self.act_alpha = 0.0
        self.act_beta = 0.0
        self.act_type = Activation.kNone
        self.mask_width = -1
        self.mask_filter = 0xffffffff
        self.reverse_mask = False
        self.verbose = False
        self.mask_int_count = 1
        self.timer = timer
        self.workspace = Tensor()
        self.mask = Tensor()
        self.mask_argsort = Tensor()
        self.indices = Tensor()
        self.mask_output = Tensor()
        self.stream = 0
        # extension (no counterpart in the reference): indices permuted into
        # mask_argsort order (SpconvOps.sort_indices); lets the kernels read
        # the index table coalesced; results are identical
        self.indices_sorted = Tensor()
        # extension: output-column tile of the tcgen05 fwd / dgrad kernels
        # (0 = widest); set by cumm.autotune, results are identical
        self.tile_n = 0
        # extension: the order in which the tcgen05 fwd / dgrad kernels take
        # their 128-row tiles (SpconvOps.tile_order, heaviest first); without
        # it each call computes that order; results are identical
        self.tile_order = Tensor()
