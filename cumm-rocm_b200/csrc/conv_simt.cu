// conv_simt.cu - fp32 mask-implicit-GEMM sparse convolution with FFMA.
//
// The fp32 path (reference algo "Simt", cumm/gemm/algospec/simt.py) keeps full
// fp32 products so results stay within 1e-5 of an fp64 evaluation; tensor-core
// tf32 would not.  Semantics are those of the tcgen05 kernels:
//   fwd / dgrad: one CTA per tile_shape[0]-row tile of the sorted rows; the tile
//     mask (OR of the rows' masks AND mask_filter, reversed for dgrad with
//     reverse_mask) selects the offsets (cumm/conv/kernel.py:844-889); row r
//     gathers A[indices[k][sigma(r)]] and the result goes to row sigma(r).
//   wgrad: dW[:, k, :] += dOut[sigma(r)]^T In[indices[k][sigma(r)]] over rows r
//     whose reduced mask word mask[r / mask_width] has bit k
//     (cumm/gemm/blockmma/mma.py:580-765), accumulated into an fp32 workspace.
#include "kernels.h"

namespace scb {
namespace {

constexpr int kSimtThreads = 128;

__global__ void __launch_bounds__(kSimtThreads) simt_fwd_kernel(const ConvSimtArgs A, int TM,
                                                                int n_red, int n_out) {
  // n_red: reduction length per offset (C for fwd, K for dgrad); n_out: output columns
  extern __shared__ float sm[];
  float *sA = sm;                    // [TM][33]
  float *sB = sA + 128 * 33;         // [32 cols][33]
  __shared__ uint32_t s_km;
  __shared__ int s_sig[128];
  const int tid = threadIdx.x;
  const int64_t row0 = static_cast<int64_t>(blockIdx.x) * TM;
  if (tid == 0) s_km = 0;
  __syncthreads();
  uint32_t m = 0;
  int sig = -1;
  if (tid < TM && row0 + tid < A.M) {
    m = A.mask[row0 + tid];
    sig = A.argsort[row0 + tid];
    if (sig < 0 || sig >= A.M) {
      atomicOr(A.err, kErrBadIndex);
      sig = -1;
    }
  }
  if (tid < 128) s_sig[tid] = sig;
  if (m) atomicOr(&s_km, m);
  __syncthreads();
  uint32_t km = s_km & A.mask_filter;
  if (A.op == 0 && A.mask_out != nullptr && tid == 0) A.mask_out[blockIdx.x] = km;
  if (A.op == 1 && km == 0) return;  // dgrad early exit (kernel.py:875-882)
  if (A.op == 1 && A.reverse) km = __brev(km) >> (32 - A.kv);

  const int cg = tid & 7;   // column group: cols cg + 8 j
  const int rgp = tid >> 3; // row group: rows rgp + 16 i
  const int n_rows_i = (TM + 15) / 16;
  for (int nb = 0; nb < n_out; nb += 32) {
    float acc[8][4];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[i][j] = 0.f;
    uint32_t mm = km;
    while (mm) {
      const int k = __ffs(mm) - 1;
      mm &= mm - 1;
      for (int c0 = 0; c0 < n_red; c0 += 32) {
        __syncthreads();
        // gather A: TM rows x 32 reduction elements
        for (int e = tid; e < TM * 32; e += kSimtThreads) {
          const int r = e >> 5, c = e & 31;
          float v = 0.f;
          const int sg = s_sig[r];
          if (sg >= 0 && c0 + c < n_red) {
            const int idx = A.indices[static_cast<int64_t>(k) * A.M + sg];
            if (idx >= 0 && idx < A.a_rows)
              v = A.a[static_cast<int64_t>(idx) * n_red + c0 + c];
            else if (idx >= A.a_rows || idx < -1)
              atomicOr(A.err, kErrBadIndex);
          }
          sA[r * 33 + c] = v;
        }
        // B: 32 output columns x 32 reduction elements of offset k
        for (int e = tid; e < 32 * 32; e += kSimtThreads) {
          const int n = e >> 5, c = e & 31;
          float v = 0.f;
          if (nb + n < n_out && c0 + c < n_red) {
            if (A.op == 0)  // W[n, k, c]
              v = A.b[(static_cast<int64_t>(nb + n) * A.kv + k) * n_red + c0 + c];
            else            // dgrad: W[c_red, k, n] with n = input channel
              v = A.b[(static_cast<int64_t>(c0 + c) * A.kv + k) * n_out + nb + n];
          }
          sB[n * 33 + c] = v;
        }
        __syncthreads();
#pragma unroll 4
        for (int c = 0; c < 32; ++c) {
          float bv[4];
#pragma unroll
          for (int j = 0; j < 4; ++j) bv[j] = sB[(cg + 8 * j) * 33 + c];
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            if (i < n_rows_i) {
              const float av = sA[(rgp + 16 * i) * 33 + c];
#pragma unroll
              for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(av, bv[j], acc[i][j]);
            }
          }
        }
      }
    }
    // epilogue
    const EpiParams &e = A.epi;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int r = rgp + 16 * i;
      if (i >= n_rows_i || r >= TM) continue;
      const int sg = s_sig[r];
      if (sg < 0) continue;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int n = nb + cg + 8 * j;
        if (n >= n_out) continue;
        float v;
        const float *src = static_cast<const float *>(e.src);
        const bool use_src = e.beta != 0.f && src != nullptr;
        if (e.mode == 1) {
          const float sc = e.scale ? e.scale[n] : 1.f;
          v = sc * acc[i][j] + (e.bias ? e.alpha * static_cast<const float *>(e.bias)[n] : 0.f);
        } else {
          v = e.alpha * acc[i][j];
        }
        if (use_src) v = fmaf(e.beta, src[static_cast<int64_t>(sg) * e.src_ld + n], v);
        A.out[static_cast<int64_t>(sg) * n_out + n] = apply_act(v, e.act_type, e.act_alpha);
      }
    }
  }
}

// grid: (kv, ceil(K/32) * ceil(C/32), row splits)
__global__ void __launch_bounds__(kSimtThreads) simt_wgrad_kernel(const ConvSimtArgs A,
                                                                  int rows_per_split) {
  __shared__ float sO[32][33];
  __shared__ float sI[32][33];
  const int k = blockIdx.x;
  const int ncb = (A.C + 31) / 32;
  const int n0 = (blockIdx.y / ncb) * 32;
  const int c0 = (blockIdx.y % ncb) * 32;
  const int64_t r_begin = static_cast<int64_t>(blockIdx.z) * rows_per_split;
  const int64_t r_end = min(r_begin + rows_per_split, A.M);
  const int tid = threadIdx.x;
  if (!((A.mask_filter >> k) & 1u)) return;
  const int tc = tid & 31;   // channel
  const int tn = tid >> 5;   // n group: n = tn + 4 j
  float acc[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) acc[j] = 0.f;
  for (int64_t rb = r_begin; rb < r_end; rb += 32) {
    __syncthreads();
    for (int e = tid; e < 32 * 32; e += kSimtThreads) {
      const int r = e >> 5, x = e & 31;
      const int64_t row = rb + r;
      float ov = 0.f, iv = 0.f;
      if (row < r_end) {
        const int64_t wi = row / A.mask_width;
        const uint32_t word = wi < A.mask_count ? A.mask[wi] : 0u;
        const int sg = A.argsort[row];
        if (sg >= 0 && sg < A.M) {
          if (n0 + x < A.K) ov = A.a[static_cast<int64_t>(sg) * A.K + n0 + x];
          if (((word >> k) & 1u) && c0 + x < A.C) {
            const int idx = A.indices[static_cast<int64_t>(k) * A.M + sg];
            if (idx >= 0 && idx < A.b_rows) iv = A.b[static_cast<int64_t>(idx) * A.C + c0 + x];
            else if (idx >= A.b_rows || idx < -1) atomicOr(A.err, kErrBadIndex);
          }
        } else {
          atomicOr(A.err, kErrBadIndex);
        }
      }
      sO[r][x] = ov;
      sI[r][x] = iv;
    }
    __syncthreads();
#pragma unroll 4
    for (int r = 0; r < 32; ++r) {
      const float iv = sI[r][tc];
#pragma unroll
      for (int j = 0; j < 8; ++j) acc[j] = fmaf(sO[r][tn + 4 * j], iv, acc[j]);
    }
  }
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const int n = n0 + tn + 4 * j;
    const int c = c0 + tc;
    if (n < A.K && c < A.C) atomicAdd(A.out + (static_cast<int64_t>(n) * A.kv + k) * A.C + c, acc[j]);
  }
}

}  // namespace

cudaError_t launch_conv_simt(const ConvSimtArgs &a, cudaStream_t stream) {
  if (a.M == 0) return cudaSuccess;
  if (a.op == 2) {
    const int rows_per_split = 2048;
    const int splits = static_cast<int>((a.M + rows_per_split - 1) / rows_per_split);
    dim3 grid(a.kv, ((a.K + 31) / 32) * ((a.C + 31) / 32), splits);
    simt_wgrad_kernel<<<grid, kSimtThreads, 0, stream>>>(a, rows_per_split);
    return cudaGetLastError();
  }
  const int TM = a.tile_m_desp;
  const int64_t tiles = (a.M + TM - 1) / TM;
  const int n_red = a.op == 0 ? a.C : a.K;
  const int n_out = a.op == 0 ? a.K : a.C;
  const size_t smem = (128 * 33 + 32 * 33) * sizeof(float);
  simt_fwd_kernel<<<static_cast<unsigned>(tiles), kSimtThreads, smem, stream>>>(a, TM, n_red,
                                                                                 n_out);
  return cudaGetLastError();
}

}  // namespace scb
