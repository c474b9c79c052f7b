"""cumm (B200 build): mask-implicit-GEMM sparse convolution and dense GEMM on
sm_100a, behind the operator surface of cumm 0.8.2
(``cumm.conv.main.ConvMainUnitTest.implicit_gemm2``,
``cumm.gemm.main.GemmMainUnitTest.matmul2``, ``cumm.tensorview``).

The compute path is ``libcumm_b200.so`` (hand-written sm_100a kernels behind a
C ABI, ``include/cumm_b200.h``); PyTorch provides device memory and streams.
There is no CPU fallback: every op raises when the library cannot be loaded
or no CUDA device is present.
"""
__version__ = "0.1.0"
