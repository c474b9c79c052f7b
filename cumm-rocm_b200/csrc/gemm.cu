// gemm.cu - dense / shuffled GEMM (the reference's GemmMainUnitTest.matmul2,
// cumm/gemm/main.py:1176-1335) on sm_100a.
//
//   NoShuffle: C = act(alpha * op(A) @ op(B) + beta * D)
//   ShuffleAC: C[c_inds[i]] = act(alpha * A[a_inds[i]] @ op(B) + beta * D[c_inds[i]])
//   ShuffleAB: C = act(alpha * A[a_inds]^T @ B[b_inds] + beta * D)
// (shape rules: cumm/gemm/nvrtc_code.py:80-125).
//
// 16-bit operands run on tcgen05 kernels:
//   * NoShuffle is the dense GEMM of gemm_dense.cu (2-D TMA tiles, either
//     operand read in place K- or MN-major, optional parallel split-K);
//   * ShuffleAC is the row-gather
//     kernel in GEMM mode (kv = 1, one 128-byte K chunk per stage, TMEM
//     accumulator, permuted-store epilogue); B is consumed K-major, so a
//     row-major [k, n] B is transposed once into the workspace;
//   * transposed A (NoShuffle with trans_a, ShuffleAB) reduces over gathered
//     rows and is the backward-weight kernel in GEMM mode (MN-major operands,
//     fp32 workspace, finalize epilogue).
// Shapes those kernels do not tile (unaligned leading dimensions, n not a
// multiple of 16, ...) and fp32 operands use the SIMT FFMA kernel below.
#include "kernels.h"

namespace scb {
namespace {

template <typename T>
__device__ __forceinline__ float ld_elem(const uint8_t *base, int64_t idx) {
  return to_f32(reinterpret_cast<const T *>(base)[idx]);
}

// 64x64 output tile per CTA, 256 threads, 4x4 outputs per thread.
template <typename T, typename TOut>
__global__ void __launch_bounds__(256) simt_gemm_kernel(const GemmArgs A) {
  __shared__ float sA[32][65];
  __shared__ float sB[32][65];
  const int tid = threadIdx.x;
  const int64_t i0 = static_cast<int64_t>(blockIdx.y) * 64;
  const int64_t j0 = static_cast<int64_t>(blockIdx.x) * 64;
  const int ti = tid >> 4;  // rows ti + 16 r
  const int tj = tid & 15;  // cols tj + 16 c
  float acc[4][4];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[r][c] = 0.f;
  for (int64_t k0 = 0; k0 < A.k; k0 += 32) {
    __syncthreads();
    for (int e = tid; e < 32 * 64; e += 256) {
      const int kk = e / 64, ii = e % 64;
      const int64_t i = i0 + ii, kx = k0 + kk;
      float v = 0.f;
      if (i < A.m && kx < A.k) {
        int64_t off;
        if (A.shuffle == 2) {
          const int row = A.a_inds ? A.a_inds[kx] : static_cast<int>(kx);
          off = (row >= 0 && row < A.a_rows) ? static_cast<int64_t>(row) * A.lda + i : -1;
        } else if (A.shuffle == 1) {
          const int row = A.a_inds ? A.a_inds[i] : static_cast<int>(i);
          off = (row >= 0 && row < A.a_rows) ? static_cast<int64_t>(row) * A.lda + kx : -1;
        } else {
          off = A.trans_a ? kx * A.lda + i : i * A.lda + kx;
        }
        if (off >= 0) v = ld_elem<T>(A.a, off);
        else atomicOr(A.err, kErrBadIndex);
      }
      sA[kk][ii] = v;
    }
    for (int e = tid; e < 32 * 64; e += 256) {
      const int kk = e / 64, jj = e % 64;
      const int64_t j = j0 + jj, kx = k0 + kk;
      float v = 0.f;
      if (j < A.n && kx < A.k) {
        int64_t off;
        if (A.shuffle == 2) {
          const int row = A.b_inds ? A.b_inds[kx] : static_cast<int>(kx);
          off = (row >= 0 && row < A.b_rows) ? static_cast<int64_t>(row) * A.ldb + j : -1;
        } else {
          off = A.trans_b ? j * A.ldb + kx : kx * A.ldb + j;
        }
        if (off >= 0) v = ld_elem<T>(A.b, off);
        else atomicOr(A.err, kErrBadIndex);
      }
      sB[kk][jj] = v;
    }
    __syncthreads();
#pragma unroll 8
    for (int kk = 0; kk < 32; ++kk) {
      float av[4], bv[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) av[r] = sA[kk][ti + 16 * r];
#pragma unroll
      for (int c = 0; c < 4; ++c) bv[c] = sB[kk][tj + 16 * c];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[r][c] = fmaf(av[r], bv[c], acc[r][c]);
    }
  }
  const EpiParams &e = A.epi;
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int64_t i = i0 + ti + 16 * r;
    if (i >= A.m) continue;
    int64_t orow = i;
    if (A.shuffle == 1 && A.c_inds) {
      orow = A.c_inds[i];
      if (orow < 0) continue;
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int64_t j = j0 + tj + 16 * c;
      if (j >= A.n) continue;
      float v = e.alpha * acc[r][c];
      if (e.beta != 0.f && e.src != nullptr)
        v = fmaf(e.beta, to_f32(static_cast<const TOut *>(e.src)[orow * e.src_ld + j]), v);
      static_cast<TOut *>(A.c)[orow * A.ldc + j] = from_f32<TOut>(apply_act(v, e.act_type, e.act_alpha));
    }
  }
}

template <typename T>
__global__ void transpose2d_kernel(const T *src, int64_t ld_src, T *dst, int64_t rows,
                                   int64_t cols) {
  // dst[cols, rows] (dense) = src[rows, cols]^T
  const int64_t total = rows * cols;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = i / cols, c = i % cols;
    dst[c * rows + r] = src[r * ld_src + c];
  }
}

int64_t align256(int64_t x) { return (x + 255) & ~static_cast<int64_t>(255); }

// Which tcgen05 kernel can run this GEMM: 0 none (SIMT), 1 row-gather,
// 2 reduction-gather, 3 dense.
int tc_route(const GemmArgs &a) {
  if (dense_gemm_supported(a)) return 3;
  if (a.in_dtype != 12 && a.in_dtype != 7) return 0;
  if (a.out_dtype != 0 && a.out_dtype != 7 && a.out_dtype != 12) return 0;
  const int64_t es = 2;
  const bool rowmajor_a = a.shuffle == 1 || (a.shuffle == 0 && !a.trans_a);
  if (rowmajor_a) {
    if ((a.k * es) % 16 || (a.lda * es) % 16) return 0;
    if (a.n % 16) return 0;
    if (a.ldc % 8 || (a.epi.src && a.epi.src_ld % 8)) return 0;
    if (reinterpret_cast<uintptr_t>(a.a) % 16 || reinterpret_cast<uintptr_t>(a.c) % 16) return 0;
    return 1;
  }
  // reduction over rows: A [k, m], B [k, n]
  if (a.m > 256) return 0;
  if (!(a.n % 64 == 0 || a.n == 16 || a.n == 32)) return 0;
  if ((a.lda * es) % 16 || (a.ldb * es) % 16 || (a.m * es) % 16) return 0;
  if (a.trans_b && a.shuffle == 2) return 0;
  if (reinterpret_cast<uintptr_t>(a.a) % 16 || reinterpret_cast<uintptr_t>(a.b) % 16) return 0;
  return 2;
}

template <typename T, typename TOut>
cudaError_t launch_simt(const GemmArgs &a, cudaStream_t s) {
  dim3 grid(static_cast<unsigned>((a.n + 63) / 64), static_cast<unsigned>((a.m + 63) / 64));
  simt_gemm_kernel<T, TOut><<<grid, 256, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_simt_any(const GemmArgs &a, cudaStream_t s) {
  if (a.in_dtype == 0 && a.out_dtype == 0) return launch_simt<float, float>(a, s);
  if (a.in_dtype == 12 && a.out_dtype == 12) return launch_simt<__nv_bfloat16, __nv_bfloat16>(a, s);
  if (a.in_dtype == 7 && a.out_dtype == 7) return launch_simt<__half, __half>(a, s);
  if (a.in_dtype == 12 && a.out_dtype == 0) return launch_simt<__nv_bfloat16, float>(a, s);
  if (a.in_dtype == 7 && a.out_dtype == 0) return launch_simt<__half, float>(a, s);
  return cudaErrorInvalidValue;
}

}  // namespace

int64_t gemm_workspace_bytes(const GemmArgs &a) {
  const int route = tc_route(a);
  if (route == 3) return dense_gemm_splits(a) > 1 ? align256(a.m * a.n * 4) : 0;
  if (route == 1) return a.trans_b ? 0 : align256(a.n * a.k * 2);
  if (route == 2) {
    int64_t b = align256(a.m * a.n * 4);
    if (a.trans_b) b += align256(a.n * a.k * 2);
    return b;
  }
  return 0;
}

cudaError_t launch_gemm(const GemmArgs &a, int num_sms, cudaStream_t s) {
  if (a.m == 0 || a.n == 0) return cudaSuccess;
  const int route = tc_route(a);
  if (route == 0) return launch_simt_any(a, s);
  uint8_t *ws = reinterpret_cast<uint8_t *>(a.ws);
  if (route == 3) {
    // a shape the tensor maps cannot describe runs on the SIMT kernel
    if (dense_gemm_splits(a) <= 1) {
      cudaError_t e = launch_dense_gemm(a, nullptr, num_sms, s);
      return e == cudaErrorInvalidValue ? launch_simt_any(a, s) : e;
    }
    // parallel split-K: partial tiles add into a zeroed fp32 [m, n], then the
    // finalize pass applies act(alpha * sum + beta * D) and converts
    float *acc = reinterpret_cast<float *>(ws);
    cudaError_t e = cudaMemsetAsync(acc, 0, a.m * a.n * 4, s);
    if (e != cudaSuccess) return e;
    e = launch_dense_gemm(a, acc, num_sms, s);
    if (e == cudaErrorInvalidValue) return launch_simt_any(a, s);
    if (e != cudaSuccess) return e;
    return launch_wgrad_finalize(acc, a.c, a.ldc, a.out_dtype, static_cast<int>(a.m), 1,
                                 static_cast<int>(a.n), 1u, a.epi, s);
  }
  if (route == 1) {
    const uint8_t *bt = a.b;
    int64_t ldbt = a.ldb;
    if (!a.trans_b) {
      // B [k, n] -> Bt [n, k]
      const int64_t total = a.k * a.n;
      int blocks = static_cast<int>((total + 255) / 256);
      if (blocks > 8192) blocks = 8192;
      transpose2d_kernel<uint16_t><<<blocks, 256, 0, s>>>(
          reinterpret_cast<const uint16_t *>(a.b), a.ldb, reinterpret_cast<uint16_t *>(ws), a.k,
          a.n);
      bt = ws;
      ldbt = a.k;
    }
    ConvRowGatherArgs g{};
    g.a_base = a.a;
    g.a_rows = a.shuffle == 1 ? a.a_rows : a.m;
    g.a_row_bytes = static_cast<int>(a.k * 2);
    g.a_row_stride = a.lda * 2;
    g.b_base = bt;
    g.b_row_stride = ldbt * 2;
    g.b_off_stride = 0;
    g.n_total = static_cast<int>(a.n);
    int bn = static_cast<int>(a.n);
    int tiles = 1;
    while (bn > 256 || bn % 16) {
      ++tiles;
      while (a.n % tiles || (a.n / tiles) % 16) ++tiles;
      bn = static_cast<int>(a.n / tiles);
    }
    g.BN = bn;
    g.n_tiles = tiles;
    g.M = a.m;
    g.kv = 1;
    g.mask = nullptr;
    g.argsort = a.shuffle == 1 ? a.c_inds : nullptr;
    g.indices = nullptr;
    g.a_inds = a.shuffle == 1 ? a.a_inds : nullptr;
    g.mask_out = nullptr;
    g.tile_m_desp = 128;
    g.mask_filter = 1u;
    g.reverse = 0;
    g.is_fwd = 1;
    g.out = a.c;
    g.out_ld = a.ldc;
    g.out_rows = a.shuffle == 1 ? 0x7fffffff : a.m;
    g.in_dtype = a.in_dtype;
    g.out_dtype = a.out_dtype;
    g.epi = a.epi;
    g.err = a.err;
    return launch_conv_rowgather(g, num_sms, s);
  }
  // route 2: C[m, n] = A[rows]^T B[rows]
  float *acc = reinterpret_cast<float *>(ws);
  const uint8_t *bb = a.b;
  int64_t ldbb = a.ldb;
  if (a.trans_b) {
    // B [n, k] -> [k, n]
    uint8_t *bt = ws + align256(a.m * a.n * 4);
    const int64_t total = a.k * a.n;
    int blocks = static_cast<int>((total + 255) / 256);
    if (blocks > 8192) blocks = 8192;
    transpose2d_kernel<uint16_t><<<blocks, 256, 0, s>>>(reinterpret_cast<const uint16_t *>(a.b),
                                                        a.ldb, reinterpret_cast<uint16_t *>(bt),
                                                        a.n, a.k);
    bb = bt;
    ldbb = a.n;
  }
  cudaError_t e = cudaMemsetAsync(acc, 0, a.m * a.n * 4, s);
  if (e != cudaSuccess) return e;
  ConvWgradArgs w{};
  w.dout = a.a;
  w.dout_rows = a.shuffle == 2 ? a.a_rows : a.k;
  w.dout_ld = a.lda;
  w.input = bb;
  w.in_rows = a.shuffle == 2 ? a.b_rows : a.k;
  w.in_ld = ldbb;
  w.K = static_cast<int>(a.m);
  w.C = static_cast<int>(a.n);
  w.kv = 1;
  w.N = a.k;
  w.mask = nullptr;
  w.mask_count = 0;
  w.mask_width = 1;
  w.mask_filter = 1u;
  w.argsort = a.shuffle == 2 ? a.a_inds : nullptr;
  w.indices = nullptr;
  w.b_inds = a.shuffle == 2 ? a.b_inds : nullptr;
  w.ws = acc;
  w.in_dtype = a.in_dtype;
  w.err = a.err;
  w.split_k = a.split_k > 1 ? a.split_k : 0;
  e = launch_conv_wgrad(w, num_sms, s);
  if (e != cudaSuccess) return e;
  return launch_wgrad_finalize(acc, a.c, a.ldc, a.out_dtype, static_cast<int>(a.m), 1,
                               static_cast<int>(a.n), 1u, a.epi, s);
}

}  // namespace scb
