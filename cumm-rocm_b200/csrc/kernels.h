// kernels.h - host-side launch interfaces between the C ABI (api.cu) and the
// kernel translation units.  No torch types; plain pointers and sizes.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "common.cuh"

namespace scb {

// Encodes a 2-D SWIZZLE_128B TMA tensor map over a row-major [outer, inner]
// tensor (row stride in bytes) with a box of box_outer rows x 128 bytes.
// Returns false when TMA cannot describe the tensor (alignment, sizes).
bool encode_tmap_2d(void *out_map, int dtype, const void *base, uint64_t inner, uint64_t outer,
                    uint64_t row_stride_bytes, uint32_t box_inner, uint32_t box_outer,
                    int swizzle_bytes = 128);

// Device address (current device) of four 128-byte rows of zeros that
// tile::gather4 reads in place of a group of four absent rows (index -1):
// out-of-range gather rows cost the TMA unit several times an in-range row.
// Looked up once per device; nullptr if the lookup fails.
const void *zero_rows_address();
constexpr int kZeroRows = 512;
// First row of a group of four zero rows for gather `c` of thread slot `t`.
__device__ __forceinline__ int zero_group(uint32_t t, uint32_t c) {
  return static_cast<int>(((t * 37u + c * 101u) & (kZeroRows / 4 - 1)) * 4u);
}

// ------------------------------------------------------------------ conv fwd / dgrad (tcgen05)
// Row-gather implicit GEMM: for every 128-row tile of the sorted row order,
//   out[sigma(r), n] = epi( sum_{k in tile mask} sum_c A[idx[k][sigma(r)], c] * B[n, k, c] )
// A = input (fwd) or dOut (dgrad) rows; B = weight [K, kv, C] (fwd) or its
// transpose [C, kv, K] (dgrad).
struct ConvRowGatherArgs {
  const uint8_t *a_base;
  int64_t a_rows;
  int a_row_bytes;           // bytes of one A row (reduction elements per offset * esize)
  int64_t a_row_stride;      // bytes between A rows
  const uint8_t *b_base;
  int64_t b_row_stride;      // bytes between B rows (kv * reduction * esize)
  int b_off_stride;          // bytes between offsets inside a B row
  int n_total;               // GEMM N
  int BN;                    // N tile (multiple of 16, <= 256)
  int n_tiles;
  int64_t M;                 // rows (indices.dim(1))
  int kv;
  const uint32_t *mask;
  const int32_t *argsort;
  const int32_t *indices;
  uint32_t *mask_out;
  int tile_m_desp;           // 32, 64 or 128
  uint32_t mask_filter;
  int reverse;
  int is_fwd;
  void *out;
  int64_t out_ld;
  int in_dtype;              // 12 bf16, 7 f16, 14 e4m3 (kind::f8f6f4)
  int out_dtype;             // SC_* dtype of out/src/bias
  EpiParams epi;
  int *err;
  // dense / ShuffleAC GEMM mode (indices == nullptr, kv == 1, mask == nullptr):
  // A row of sorted row r = a_inds ? a_inds[r] : r, output row = argsort ? argsort[r] : r
  const int32_t *a_inds;
  int64_t out_rows;          // bound for output rows
  const int32_t *idx_sorted; // optional [kv, M]: indices[k][argsort[r]]
  int *tile_counter;         // optional, zero at launch: tiles handed out dynamically
  // optional largest-first tile schedule given by the caller (order_given
  // set): ceil(M / 128) ints, a permutation of the row tiles.  tile_counter,
  // when set, is zeroed by the launcher.
  const int32_t *tile_order;
  int order_given;
  int m_tiles;               // ceil(M / 128), set by the launcher
  // backward-input with B = the [K, kv, C] weight itself: the slab of offset
  // k is rows j (reduction) x columns k * C + c (n), read MN-major by the
  // tensor core (no transposed copy); needs 16-bit data, red % 64 == 0 and
  // BN % 64 == 0 on the TMA gather path
  int b_mn;
};
cudaError_t launch_conv_rowgather(const ConvRowGatherArgs &a, int num_sms, cudaStream_t stream);
// head: 34 zeroed ints; tile_pc: m_tiles ints of scratch; order: m_tiles ints
cudaError_t launch_tile_order(const uint32_t *mask, int64_t M, uint32_t filter, int reverse, int kv,
                              int *head, int32_t *tile_pc, int32_t *order, cudaStream_t stream);

// dgrad weight transposition W[K, kv, C] -> Wt[C, kv, K] (16-bit or 8-bit elements)
cudaError_t launch_transpose_weight(const void *w, void *wt, int K, int kv, int C, int esize,
                                    cudaStream_t stream);

// ------------------------------------------------------------------ conv wgrad (tcgen05)
// dW[K, kv, C] (fp32 workspace accumulation) = sum over rows of
//   dOut[sigma(r)]^T x In[idx[k][sigma(r)]], rows gated by mask[r / mask_width].
struct ConvWgradArgs {
  const uint8_t *dout;       // [rows_out, K]
  int64_t dout_rows;
  int64_t dout_ld;           // elements
  const uint8_t *input;      // [rows_in, C]
  int64_t in_rows;
  int64_t in_ld;             // elements
  int K;
  int C;
  int kv;
  int64_t N;                 // rows (indices.dim(1))
  const uint32_t *mask;      // reduced masks (fwd mask_output)
  int64_t mask_count;
  int mask_width;
  uint32_t mask_filter;
  const int32_t *argsort;
  const int32_t *indices;
  float *ws;                 // [K, kv, C] fp32, zeroed
  int in_dtype;              // 12 bf16 or 7 f16 (dOut and input)
  int *err;
  // ShuffleAB GEMM mode (indices == nullptr, kv == 1): input row of sorted row r
  // is b_inds ? b_inds[r] : r; dOut row is argsort ? argsort[r] : r; mask may be null
  const int32_t *b_inds;
  const int32_t *idx_sorted; // optional [kv, N]: indices[k][argsort[r]]
  int split_k;               // row splits (grid.x); 0 = about one CTA per SM
};
cudaError_t launch_conv_wgrad(const ConvWgradArgs &a, int num_sms, cudaStream_t stream);

// out[K, kv, C] = act(alpha * ws + beta * src) for offsets in mask_filter
// (others untouched); src rows have stride src_ld (0 = [C] bias row), out rows
// have stride out_ld (elements, per K row).
cudaError_t launch_wgrad_finalize(const float *ws, void *out, int64_t out_ld, int out_dtype,
                                  int K, int kv, int C, uint32_t mask_filter, const EpiParams &e,
                                  cudaStream_t stream);

// ------------------------------------------------------------------ SIMT fp32 conv
struct ConvSimtArgs {
  int op;                    // 0 fwd, 1 dgrad, 2 wgrad
  const float *a;            // gathered operand (fwd: input, dgrad: dout, wgrad: dout)
  int64_t a_rows;
  const float *b;            // fwd/dgrad: weight [K, kv, C]; wgrad: input [rows, C]
  int64_t b_rows;
  float *out;                // fwd: [.., K]; dgrad: [.., C]; wgrad: ws [K, kv, C]
  int C, K, kv;
  int64_t M;
  const uint32_t *mask;
  int64_t mask_count;
  const int32_t *argsort;
  const int32_t *indices;
  uint32_t *mask_out;
  int tile_m_desp;
  int mask_width;
  uint32_t mask_filter;
  int reverse;
  EpiParams epi;
  int *err;
};
cudaError_t launch_conv_simt(const ConvSimtArgs &a, cudaStream_t stream);

// ------------------------------------------------------------------ GEMM
struct GemmArgs {
  int shuffle;               // 0 none, 1 AC, 2 AB
  int trans_a, trans_b;
  int64_t m, n, k;
  const uint8_t *a;
  int64_t lda;
  const uint8_t *b;
  int64_t ldb;
  void *c;
  int64_t ldc;
  const int32_t *a_inds, *b_inds, *c_inds;
  int64_t a_rows, b_rows;
  int in_dtype;              // SC_BFLOAT16 / SC_FLOAT16 / SC_FLOAT32
  int out_dtype;
  EpiParams epi;
  float *ws;                 // fp32 [m, n] accumulation workspace (ShuffleAB, split-K)
  int *err;
  int split_k;               // K splits (1 = none): dense route and ShuffleAB only
};
cudaError_t launch_gemm(const GemmArgs &a, int num_sms, cudaStream_t stream);
int64_t gemm_workspace_bytes(const GemmArgs &a);
// Dense tcgen05 GEMM (NoShuffle, 16-bit operands): whether it takes `a`, its
// K-split count, and the launch (split_ws: zeroed fp32 [m, n] when splits > 1).
bool dense_gemm_supported(const GemmArgs &a);
int dense_gemm_splits(const GemmArgs &a);
cudaError_t launch_dense_gemm(const GemmArgs &a, float *split_ws, int num_sms, cudaStream_t stream);

// ------------------------------------------------------------------ gather / scatter
// out[i] = in[indices[i]] (rows of row_bytes bytes), and
// out[indices[i]] += in[i] (rows of `channels` elements of dtype 0 / 7 / 12).
cudaError_t launch_gather_rows(void *out, const void *in, int64_t in_rows, const int32_t *indices,
                               int64_t m, int64_t row_bytes, int bytes_per_access, int threads,
                               int num_sms, int *err, cudaStream_t s);
cudaError_t launch_scatter_add_rows(void *out, int64_t out_rows, const void *in, const int32_t *indices,
                                    int64_t m, int64_t channels, int dtype, int bytes_per_access,
                                    int threads, int num_sms, int *err, cudaStream_t s);

// ------------------------------------------------------------------ pair builder
struct PairBuildArgs {
  const int32_t *coords;
  int64_t n_in;
  int batch;
  int spatial[3];
  int ksize[3];
  int stride[3];
  int padding[3];
  int dilation[3];
  int out_spatial[3];
  int subm;
  int *err;
};
int64_t pairs_workspace_bytes(int64_t n_in, int kv, int subm);
cudaError_t build_subm_pairs(const PairBuildArgs &a, int32_t *pairs_fwd, int32_t *pairs_bwd,
                             uint32_t *mask_fwd, void *ws, int64_t ws_bytes, cudaStream_t s);
cudaError_t build_conv_outputs(const PairBuildArgs &a, int64_t *n_out, void *ws,
                               int64_t ws_bytes, cudaStream_t s);
cudaError_t build_conv_pairs(const PairBuildArgs &a, int64_t n_out, int32_t *out_coords,
                             int32_t *pairs_fwd, int32_t *pairs_bwd, uint32_t *mask_fwd,
                             uint32_t *mask_bwd, void *ws, int64_t ws_bytes, cudaStream_t s);
int64_t sort_workspace_bytes(int64_t n);
cudaError_t sort_indices(const int32_t *indices, int kv, int64_t n, const int32_t *argsort,
                         int32_t *out, cudaStream_t s);
cudaError_t sort_masks_split(uint32_t *data, int64_t n, uint32_t split_mask, int32_t *argsort,
                             void *ws, int64_t ws_bytes, cudaStream_t s);

}  // namespace scb
