"""CPU tests of the host side: the C ABI library loads and exports every
symbol include/cumm_b200.h declares, argument validation maps to the
reference's exception types, and the Python mirror of the reference
interface (tv.Tensor, descriptors, mnk helpers) behaves like cumm's."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest
import torch

from cumm import _lib
from cumm import tensorview as tv
from cumm.conv.main import ConvMainUnitTest, get_all_conv_algo_desp, implicit_gemm_mnk
from cumm.gemm.main import GemmMainUnitTest, extract_mnk, get_all_algo_desp
from cumm.tensorview.gemm import ConvAlgoDesp, ConvOpType, ConvParams, GemmAlgoDesp

ROOT = Path(__file__).resolve().parent.parent


def _declared():
    text = (ROOT / "include" / "cumm_b200.h").read_text()
    return sorted(set(re.findall(r"^(?:int|const char \*)\s*(sc_\w+)\(", text, re.M)))


def test_library_exports_header_symbols():
    lib = _lib.load()
    names = _declared()
    assert len(names) >= 13
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(_lib.EXPORTS)
    assert lib.sc_version().decode().startswith("cumm_b200")


def _fake_conv(op=0, **kw):
    cp = _lib.ConvParamsC()
    cp.op_type, cp.algo = op, _lib.SC_ALGO_TCGEN05
    cp.dtype_input = cp.dtype_weight = cp.dtype_output = tv.bfloat16
    cp.tile_m, cp.tile_k, cp.kv = 128, 64, 27
    cp.n_in = cp.n_out = cp.N = 1000
    cp.C = cp.K = 64
    for f in ("input", "weight", "output", "indices", "mask", "mask_argsort"):
        setattr(cp, f, 0x1000)
    cp.mask_count = 1000
    cp.mask_width = 128
    for k, v in kw.items():
        setattr(cp, k, v)
    return cp


def _ws(cp):
    lib = _lib.load()
    n = ctypes.c_int64(-1)
    rc = lib.sc_conv_workspace_size(ctypes.byref(cp), ctypes.byref(n))
    return rc, n.value, lib.sc_last_error().decode()


def test_conv_validation_codes():
    # fwd (optional workspace): the tile counter head, then the sorted index
    # table the call builds for the strand kernel when none is given
    # (kv x N int32, rounded up to 256 bytes)
    own = ((27 * 1000 * 4 + 255) // 256) * 256
    assert _ws(_fake_conv())[:2] == (0, 256 + own)
    rc, n, _ = _ws(_fake_conv(1))
    assert rc == 0 and n == 256 + 64 * 27 * 64 * 2 + own  # dgrad: + transposed weight
    # with indices_sorted given, or a layer the strand kernel does not take
    # (N % 4 != 0), no table is built
    assert _ws(_fake_conv(indices_sorted=0x3000))[:2] == (0, 256)
    assert _ws(_fake_conv(N=1001, n_in=1001, n_out=1001, mask_count=1001))[:2] == (0, 256)
    rc, n, _ = _ws(_fake_conv(2))
    assert rc == 0 and n == 64 * 27 * 64 * 4          # wgrad: fp32 accumulation (no own sorted
    # table: building it costs more than the faster index loaders save)
    rc, _, msg = _ws(_fake_conv(0, N=999))
    assert rc == _lib.SC_RUNTIME and "output.dim(0)" in msg
    rc, _, msg = _ws(_fake_conv(2, mask_width=100))
    assert rc == _lib.SC_RUNTIME and "mask_width" in msg
    rc, _, msg = _ws(_fake_conv(0, C=20))
    assert rc == _lib.SC_RUNTIME and "Can't Found Algorithm" in msg
    rc, _, msg = _ws(_fake_conv(0, indices=None))
    assert rc == _lib.SC_RUNTIME
    rc, _, msg = _ws(_fake_conv(0, tile_m=256))
    assert rc == _lib.SC_RUNTIME
    rc, _, msg = _ws(_fake_conv(0, output_add=0x2000))
    assert rc == _lib.SC_INVALID_ARG
    with pytest.raises(ValueError):
        _lib.check(_lib.SC_INVALID_ARG)
    with pytest.raises(RuntimeError):
        _lib.check(_lib.SC_RUNTIME)


def test_misaligned_tensors_rejected_before_launch():
    """A tensor view that does not start on a 16-byte boundary is an argument
    error of the tcgen05 path (its kernels move 16-byte units), reported by the
    host checks before any device access: these dummy pointers are never
    dereferenced."""
    lib = _lib.load()
    for op, field in ((0, "input"), (0, "weight"), (0, "output"), (1, "input"), (1, "weight"),
                      (1, "output"), (2, "input"), (2, "output")):
        cp = _fake_conv(op, **{field: 0x1000 + 4})
        rc, _, msg = _ws(cp)
        assert rc == _lib.SC_INVALID_ARG and "16-byte boundary" in msg and field in msg, (op, field, msg)
        cp.workspace, cp.workspace_bytes = 0x100000, 1 << 24
        assert lib.sc_conv_implicit_gemm(ctypes.byref(cp)) == _lib.SC_INVALID_ARG, (op, field)
    rc, _, msg = _ws(_fake_conv(0, bias=0x2000 + 8))
    assert rc == _lib.SC_INVALID_ARG and "bias" in msg
    # backward weight may write a dW view at any 4-byte offset (scalar stores
    # through the workspace and the finalize kernel)
    cp = _fake_conv(2, weight=0x1000 + 4)
    cp.dtype_weight = tv.float32
    assert _ws(cp)[0] == 0
    # the fp32 SIMT path reads scalars only
    cp = _fake_conv(0, input=0x1000 + 4)
    cp.algo = _lib.SC_ALGO_SIMT
    cp.dtype_input = cp.dtype_weight = cp.dtype_output = tv.float32
    assert _ws(cp)[0] == 0


def test_null_params():
    lib = _lib.load()
    assert lib.sc_conv_implicit_gemm(None) == _lib.SC_INVALID_ARG
    assert lib.sc_gemm_matmul(None) == _lib.SC_INVALID_ARG


def test_tensor_mirror():
    a = np.arange(12, dtype=np.uint32).reshape(3, 4) | np.uint32(1 << 31)
    t = tv.from_numpy(a)
    assert t.dtype == tv.uint32 and t.shape == [3, 4] and t.dim(1) == 4 and t.device == -1
    assert np.array_equal(t.numpy(), a)
    assert t.slice_first_axis(1, 2).shape == [1, 4]
    z = tv.zeros([5], tv.bfloat16)
    assert z.itemsize == 2 and z.numpy().sum() == 0
    f = tv.full([2, 2], 0xffffffff, tv.uint32)
    assert np.all(f.numpy() == 0xffffffff)
    assert tv.Tensor().empty()


def test_descriptors_and_mnk():
    d = ConvAlgoDesp(3, ConvOpType.kBackwardWeight)
    assert d.conv_iwo_012_to_abc(ConvOpType.kBackwardInput) == [2, 1, 0]
    assert d.gemm_abc_012_to_iwo(ConvOpType.kBackwardWeight) == [2, 0, 1]
    assert implicit_gemm_mnk(ConvOpType.kForward, 100, 32, 64, 27) == (100, 64, 32 * 27)
    assert implicit_gemm_mnk(ConvOpType.kBackwardInput, 100, 32, 64, 27) == (100, 32, 64 * 27)
    assert implicit_gemm_mnk(ConvOpType.kBackwardWeight, 100, 32, 64, 27) == (64, 32 * 27, 100)
    assert ConvMainUnitTest.extract_mnk(0, 100, 32, 64, 27) == [100, 64, 864]
    desps = get_all_conv_algo_desp()
    assert len(desps) > 10
    for dd in desps:
        name = repr(dd)
        assert dd.mask_sparse and ("_SK" in name)
    fwd = [x for x in desps if x.op_type == ConvOpType.kForward and x.algo == "Tcgen05"][0]
    assert fwd.supported(1000, 64, 64 * 27, 64, 64, 128)
    wg = [x for x in desps if x.op_type == ConvOpType.kBackwardWeight and x.algo == "Tcgen05"][0]
    assert not wg.supported(64, 64 * 27, 1000, 64, 64, 100)
    assert wg.query_conv_workspace_size(64, 64 * 27, 1000, 1, 27) == 64 * 27 * 64 * 4
    assert extract_mnk([100, 32], [32, 48], False, False, False) == (100, 48, 32)
    assert extract_mnk([32, 100], [48, 32], True, True, False) == (100, 48, 32)
    assert extract_mnk([1000, 64], [1000, 32], True, False, False, 2, [500]) == (64, 32, 500)
    assert GemmMainUnitTest.align_to_power2(100) == 128
    gd = get_all_algo_desp()
    assert any(x.shuffle_type == 1 for x in gd) and any(x.shuffle_type == 2 for x in gd)
    g = GemmAlgoDesp()
    with pytest.raises(RuntimeError):
        g.check_valid()


def test_ops_need_cuda_no_cpu_fallback():
    if torch.cuda.is_available():
        pytest.skip("has a GPU")
    p = ConvParams(3, ConvOpType.kForward)
    with pytest.raises(RuntimeError, match="CUDA device"):
        ConvMainUnitTest().implicit_gemm2(p)



def test_tile_order_entry_validation():
    """sc_tile_order_workspace_size and the argument checks of sc_tile_order
    (made before any device call)."""
    lib = _lib.load()
    n = ctypes.c_int64(-1)
    assert lib.sc_tile_order_workspace_size(1000, ctypes.byref(n)) == 0 and n.value == 256 + 256
    assert lib.sc_tile_order_workspace_size(200000, ctypes.byref(n)) == 0
    assert n.value == 256 + ((1563 * 4 + 255) // 256) * 256
    assert lib.sc_tile_order_workspace_size(-1, ctypes.byref(n)) == _lib.SC_INVALID_ARG
    assert lib.sc_tile_order(None, 1000, 0xffffffff, 27, 0, 0x1000, 0x2000, 4096, None) == _lib.SC_INVALID_ARG
    assert lib.sc_tile_order(0x1000, 1000, 0xffffffff, 40, 0, 0x1000, 0x2000, 4096, None) == _lib.SC_INVALID_ARG
    rc = lib.sc_tile_order(0x1000, 1000, 0xffffffff, 27, 0, 0x3000, 0x2000, 100, None)
    assert rc == _lib.SC_RUNTIME and "workspace at least" in lib.sc_last_error().decode()
    assert lib.sc_tile_order(None, 0, 0xffffffff, 27, 0, None, None, 0, None) == 0



def test_misaligned_tile_order_rejected():
    """A tile_order that is not 4-byte aligned is an argument error before any
    launch (the kernels read it as int32)."""
    rc, _, msg = _ws(_fake_conv(0, tile_order=0x1002))
    assert rc == _lib.SC_INVALID_ARG and "tile_order" in msg
    assert _ws(_fake_conv(0, tile_order=0x1004))[0] == 0


def test_own_sorted_table_predicate():
    """The workspace a forward reports includes the sorted index table it
    builds for the strand kernel exactly when that kernel takes the layer:
    64-byte rows or whole 128-byte blocks, a column tile <= 64 and N % 4 == 0."""
    own = ((27 * 1000 * 4 + 255) // 256) * 256
    cases = [
        (dict(C=32), True),                      # 64-byte rows
        (dict(C=128), True),                     # two 128-byte blocks per offset
        (dict(C=16), False),                     # 32-byte rows: packed row-gather path
        (dict(K=128), False),                    # widest column tile 128
        (dict(K=128, tile_n=64), True),          # column tile 64
        (dict(C=96), False),                     # 192-byte rows
    ]
    for kw, builds in cases:
        rc, n, msg = _ws(_fake_conv(0, **kw))
        assert rc == 0, (kw, msg)
        assert n == 256 + (own if builds else 0), (kw, n)
