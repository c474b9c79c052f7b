/*
 * cumm_b200.h - C ABI of the B200 (sm_100a) mask-implicit-GEMM sparse
 * convolution and dense GEMM library (libcumm_b200.so).
 *
 * Every entry point takes plain device pointers, sizes and a CUDA stream,
 * returns an int status and never frees caller memory.  Status codes:
 *   SC_OK (0)            success
 *   SC_INVALID_ARG (1)   argument validation failed (reference: TV_THROW_INVALID_ARG
 *                        -> Python ValueError, include/tensorview/core/common.h:102-141)
 *   SC_RUNTIME (2)       unsupported configuration / "Can't Found Algorithm"
 *                        (cumm/conv/main.py:733-744) -> Python RuntimeError
 *   SC_CUDA (3)          a CUDA runtime call failed (TV_CHECK_CUDA_ERR_V2,
 *                        include/tensorview/core/common.h:170-183)
 *   SC_DEVICE (4)        a kernel reported an error word (bad gather index,
 *                        hash table full, bounded wait expired)
 * sc_last_error() returns the thread-local message of the last failure.
 *
 * All launches are asynchronous on the given stream; no entry point
 * synchronises unless SC_FLAG_SYNC_CHECK is set in `flags`.
 */
#ifndef CUMM_B200_H_
#define CUMM_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SC_OK 0
#define SC_INVALID_ARG 1
#define SC_RUNTIME 2
#define SC_CUDA 3
#define SC_DEVICE 4

/* dtype codes: identical to tv::DType (include/tensorview/dtypes.h:39-62). */
#define SC_FLOAT32 0
#define SC_INT32 1
#define SC_FLOAT16 7
#define SC_UINT32 10
#define SC_BFLOAT16 12
#define SC_FLOAT_E4M3 14

/* ConvOpType (include/tensorview/gemm/core/constants.h:20). */
#define SC_CONV_FORWARD 0
#define SC_CONV_BACKWARD_INPUT 1
#define SC_CONV_BACKWARD_WEIGHT 2

/* Activation (include/tensorview/gemm/core/constants.h:39-57). */
#define SC_ACT_NONE 0
#define SC_ACT_RELU 1
#define SC_ACT_SIGMOID 2
#define SC_ACT_LEAKY_RELU 3

/* Kernel family selector (replaces GemmAlgoDesp::algo strings). */
#define SC_ALGO_TCGEN05 0 /* tcgen05.mma + TMEM accumulators (bf16/f16/e4m3) */
#define SC_ALGO_SIMT 1    /* fp32 FFMA kernel (fp32 operands, exact-ish path) */

/* ShuffleStrideType (constants.h:34). */
#define SC_SHUFFLE_NONE 0
#define SC_SHUFFLE_AC 1
#define SC_SHUFFLE_AB 2

/* flags */
#define SC_FLAG_SYNC_CHECK 1 /* synchronise the stream and check the device error word */

/*
 * POD mirror of tv::gemm::ConvParams + ConvAlgoDesp for the mask-sparse path
 * (include/tensorview/gemm/core/params.h:166-327, 392-428; field list in
 * cumm/core_cc/tensorview_bind.pyi:887-929).  Tensor semantics:
 *   input  [n_in, C]     (written by BACKWARD_INPUT)
 *   weight [K, kv, C]    (written by BACKWARD_WEIGHT, dtype_weight may be f32)
 *   output [n_out, K]    (written by FORWARD)
 *   indices [kv, N] int32, -1 = no pair; N = indices.dim(1)
 *   mask [>= rows] uint32 (sorted, consistent with mask_argsort)
 *   mask_argsort [N] int32
 *   mask_output [ceil(N / tile_m)] uint32 (FORWARD writes, BACKWARD_WEIGHT reads
 *   through `mask` with mask_width rows per word)
 * With SC_ALGO_TCGEN05, input, output, bias, output_add and (forward,
 * backward-input) weight must start on a 16-byte boundary, else
 * SC_INVALID_ARG; a backward-weight dW may start at any element.
 */
typedef struct sc_conv_params {
  int32_t op_type;
  int32_t algo;
  int32_t dtype_input;
  int32_t dtype_weight;
  int32_t dtype_output;
  int32_t tile_m;    /* mask granularity = ConvAlgoDesp.tile_shape[0] */
  int32_t tile_k;    /* ConvAlgoDesp.tile_shape[2] (wgrad mask_width check) */
  int32_t kv;
  int64_t n_in;
  int64_t n_out;
  int64_t C;
  int64_t K;
  int64_t N; /* indices.dim(1) */
  void *input;
  void *weight;
  void *output;
  const int32_t *indices;
  const uint32_t *mask;
  int64_t mask_count;
  const int32_t *mask_argsort;
  uint32_t *mask_output;
  int64_t mask_output_count;
  uint32_t mask_filter;
  int32_t reverse_mask;
  int32_t mask_width;
  float alpha;
  float beta;
  float act_alpha;
  float act_beta;
  int32_t act_type;
  const void *bias;       /* [K], dtype_output; replaces the source operand */
  const void *output_add; /* [n_out, K] source operand when given */
  const float *scale;     /* [K] fp32 per-output-channel scale (e4m3 inference epilogue) */
  int32_t split_k_slices;
  int32_t flags;
  void *workspace;
  int64_t workspace_bytes;
  void *stream; /* cudaStream_t */
  /* Optional (may be NULL): indices permuted into mask_argsort order,
   * indices_sorted[k][r] = indices[k][mask_argsort[r]] ([kv, N] int32), as
   * produced by sc_sort_indices.  With it the kernels read the index table
   * coalesced instead of through the argsort indirection; results are
   * identical.  Without it, a forward / backward-input call whose layer the
   * strand kernel takes builds the table at the end of its workspace (the
   * size sc_conv_workspace_size reports includes it); pass it when a pair
   * table serves several calls. */
  const int32_t *indices_sorted;
  /* Output-column tile of the tcgen05 forward / backward-input kernels (the
   * reference's ConvAlgoDesp tile_shape[1]): 0 picks the widest tile (all
   * columns up to 256); otherwise a multiple of 16, <= 256, dividing the
   * output width (K forward, C backward-input), else SC_INVALID_ARG. */
  int32_t tile_n;
  /* Optional (may be NULL): the order in which the tcgen05 forward /
   * backward-input kernels take their 128-row tiles, ceil(N / 128) int32
   * entries, a permutation of 0 .. ceil(N / 128) - 1 as sc_tile_order writes
   * it.  Results do not depend on it.  Without it the tiles are taken in
   * mask order.  An entry outside the range sets error bit 1 and its tile is
   * skipped (the permutation property itself is not checked). */
  const int32_t *tile_order;
} sc_conv_params;

/*
 * POD mirror of tv::gemm::GemmParams (params.h:329-390) for matmul2
 * (cumm/gemm/main.py:1176-1335, cumm/gemm/nvrtc_code.py:34-274):
 *   C = act(alpha * op(A) @ op(B) + beta * D)
 * A is [m, k] ([k, m] when trans_a), B is [k, n] ([n, k] when trans_b),
 * C is [m, n]; D is C's shape or a [n] bias (d_is_bias).
 * ShuffleAC: C[c_inds[i]] = A[a_inds[i]] @ B (m = len(a_inds)).
 * ShuffleAB: C = A[a_inds]^T @ B[b_inds] (k = len(a_inds)).
 */
typedef struct sc_gemm_params {
  int32_t dtype_a;
  int32_t dtype_b;
  int32_t dtype_c;
  int32_t trans_a;
  int32_t trans_b;
  int32_t trans_c;
  int32_t shuffle_type;
  int32_t algo;
  int64_t m;
  int64_t n;
  int64_t k;
  const void *a;
  int64_t lda;
  const void *b;
  int64_t ldb;
  void *c;
  int64_t ldc;
  const void *d;
  int64_t ldd; /* 0 => d is a [n] bias broadcast over rows */
  const int32_t *a_inds;
  const int32_t *b_inds;
  const int32_t *c_inds;
  int64_t a_rows; /* rows of the physical A buffer (bounds for a_inds) */
  int64_t b_rows; /* rows of the physical B buffer (bounds for b_inds) */
  float alpha;
  float beta;
  float act_alpha;
  float act_beta;
  int32_t act_type;
  int32_t split_k_slices;
  int32_t flags;
  void *workspace;
  int64_t workspace_bytes;
  void *stream;
} sc_gemm_params;

/* Replaces ConvMainUnitTest.implicit_gemm2 (cumm/conv/main.py:483-745) together
 * with its prologue nvrtc_conv_template (cumm/conv/nvrtc_code.py:20-196). */
int sc_conv_implicit_gemm(const sc_conv_params *p);

/* Replaces ConvAlgoDesp::query_conv_workspace_size (params.h:286-307):
 * bytes of workspace sc_conv_implicit_gemm needs for these params. */
int sc_conv_workspace_size(const sc_conv_params *p, int64_t *bytes);

/*
 * Backward weight without a caller workspace.  No counterpart in the
 * reference: implicit_gemm2 allocates a missing workspace itself
 * (cumm/conv/nvrtc_code.py:181-196), this library never allocates.
 * Same params and results as sc_conv_implicit_gemm with op_type
 * SC_CONV_BACKWARD_WEIGHT; workspace must be NULL / 0.  The fp32 [K, kv, C]
 * accumulator lives in a static 8 MiB device array of this library, so
 * K * kv * C must be <= 2097152 (else SC_INVALID_ARG); an fp32 dW with
 * alpha 1, beta 0 and every offset in mask_filter is accumulated in dW itself
 * and leaves the array untouched.  Nothing has to start
 * at zero: each call clears the part it uses on p->stream before the kernel.
 * The first call on a device (with that device current) looks up the array's
 * address and caches it; make that first call before any stream capture
 * starts, and do not call cudaDeviceReset on that device afterwards (the
 * module reloads at a new address and the cached one is stale).  There is
 * one array per device: calls that may run at the same time on one device
 * (different streams or host threads) race on it and give wrong gradients;
 * calls queued on one stream are safe.
 */
int sc_conv_wgrad_static_scratch(const sc_conv_params *p);

/* Replaces GemmMainUnitTest.matmul2 (cumm/gemm/main.py:1176-1335). */
int sc_gemm_matmul(const sc_gemm_params *p);

/* Replaces GemmAlgoDesp::query_workspace_size (params.h:115-132). */
int sc_gemm_workspace_size(const sc_gemm_params *p, int64_t *bytes);

/*
 * Indice-pair / mask builder.  Replaces spconv's
 * SpconvOps.generate_subm_conv_inds / generate_conv_inds (called at
 * cumm/conv/main_real_spconv.py:79-105) over cumm's linear-probing hash table
 * (include/tensorview/hash/linear.cu.h:557-840).
 *   coords [n_in, 4] int32 (batch, z, y, x); spatial [3] = (D, H, W)
 *   pairs_fwd [kv, n_out] and pairs_bwd [kv, n_in] int32 (filled with -1 here)
 *   mask_fwd [n_out] and mask_bwd [n_in] uint32
 * Submanifold: n_out == n_in and out coords == in coords.
 * Workspace is queried with sc_pairs_workspace_size.
 */
int sc_pairs_workspace_size(int64_t n_in, int32_t kv, int32_t subm, int64_t *bytes);

int sc_build_subm_pairs(const int32_t *coords, int64_t n_in, const int32_t *spatial,
                        const int32_t *ksize, const int32_t *dilation,
                        int32_t *pairs_fwd, int32_t *pairs_bwd, uint32_t *mask_fwd,
                        void *workspace, int64_t workspace_bytes, void *stream);

/* Strided / regular sparse conv, pass 1: number of unique output voxels.
 * out_spatial [3] receives the output grid shape.  Synchronises the stream
 * (the output count sizes the caller's allocations). */
int sc_build_conv_outputs(const int32_t *coords, int64_t n_in, int32_t batch,
                          const int32_t *spatial, const int32_t *ksize,
                          const int32_t *stride, const int32_t *padding,
                          const int32_t *dilation, int32_t *out_spatial,
                          int64_t *n_out, void *workspace, int64_t workspace_bytes,
                          void *stream);

/* Pass 2: output coords [n_out, 4] in canonical (batch, z, y, x) order and the
 * pair tables / masks.  Must follow sc_build_conv_outputs with the same workspace. */
int sc_build_conv_pairs(const int32_t *coords, int64_t n_in, int32_t batch,
                        const int32_t *spatial, const int32_t *ksize,
                        const int32_t *stride, const int32_t *padding,
                        const int32_t *dilation, int64_t n_out, int32_t *out_coords,
                        int32_t *pairs_fwd, int32_t *pairs_bwd, uint32_t *mask_fwd,
                        uint32_t *mask_bwd, void *workspace, int64_t workspace_bytes,
                        void *stream);

/* Replaces SpconvOps.sort_1d_by_key_split (main_real_spconv.py:138-145):
 * stable sort of `data` [n] uint32 in place by key (data & split_mask);
 * argsort [n] int32 receives the permutation. */
int sc_sort_masks_split(uint32_t *data, int64_t n, uint32_t split_mask, int32_t *argsort,
                        void *workspace, int64_t workspace_bytes, void *stream);
int sc_sort_workspace_size(int64_t n, int64_t *bytes);

/* indices_sorted[k][r] = indices[k][argsort[r]] for k < kv, r < N (a gather
 * kernel on `stream`; prepares sc_conv_params.indices_sorted for a pair table
 * that is reused by several convolutions). */
int sc_sort_indices(const int32_t *indices, int32_t kv, int64_t N, const int32_t *argsort,
                    int32_t *indices_sorted, void *stream);

/* Largest-first tile order for sc_conv_params.tile_order: the 128-row tiles
 * of the mask-sorted rows ordered by the number of offsets they visit
 * (popcount of the OR of their mask words AND mask_filter), heaviest first;
 * ties in any order.  reverse = 1 gives the backward-input count (brev of the
 * mask, kv bits), which equals the forward one for masks of kv bits, so one
 * order serves both directions of a submanifold layer.  The workspace (size
 * from sc_tile_order_workspace_size) is scratch of this call.  Asynchronous
 * on `stream`. */
int sc_tile_order_workspace_size(int64_t N, int64_t *bytes);
int sc_tile_order(const uint32_t *mask, int64_t N, uint32_t mask_filter, int32_t kv, int32_t reverse,
                  int32_t *tile_order, void *workspace, int64_t workspace_bytes, void *stream);

/*
 * Standalone row gather and scatter-add.  Replace the reference's
 * GatherAll.gather / ScatterAll.scatter (cumm/gemm/gather.py:390-620; kernels
 * GatherKernelV2 and ScatterKernel, gather.py:125-331):
 *   sc_gather_rows:      out[i, :] = in[indices[i], :] for i < m, rows of
 *                        row_bytes bytes (any dtype)
 *   sc_scatter_add_rows: out[indices[i], :] += in[i, :] for i < m, rows of
 *                        `channels` elements of dtype SC_FLOAT32 (the
 *                        reference's only scatter dtype), SC_FLOAT16 or
 *                        SC_BFLOAT16 (added in fp32, rounded once)
 * bytes_per_access (4, 8 or 16) must divide the row's bytes and the base
 * addresses; num_threads (64, 128 or 256) is the block size.  As in the
 * reference, scatter-add reads, adds and writes each row once without
 * atomics, so the indices of one call must be distinct.  Index -1 gives a zero
 * row (gather) or skips the row (scatter-add); any other index outside
 * [0, in_rows) / [0, out_rows) sets the device error word's bad-index bit and
 * is treated like -1.
 */
int sc_gather_rows(void *out, const void *in, int64_t in_rows, const int32_t *indices, int64_t m,
                   int64_t row_bytes, int32_t bytes_per_access, int32_t num_threads, void *stream);
int sc_scatter_add_rows(void *out, int64_t out_rows, const void *in, const int32_t *indices,
                        int64_t m, int64_t channels, int32_t dtype, int32_t bytes_per_access,
                        int32_t num_threads, void *stream);

/* Device error word of the current device: returns the accumulated error bits
 * (0 = none) after synchronising `stream`, and clears them. */
int sc_check_device_error(void *stream, int32_t *bits);

/* Thread-local message of the last failed call ("" when none). */
const char *sc_last_error(void);

/* Library version string. */
const char *sc_version(void);

#ifdef __cplusplus
}
#endif

#endif /* CUMM_B200_H_ */
