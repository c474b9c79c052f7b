// conv_rowgather.cu - mask-implicit-GEMM sparse convolution, forward and
// backward-input, on sm_100a tensor cores.
//
// Semantics follow the reference conv kernel (cumm/conv/kernel.py:737-1090):
//   * rows are visited in mask_argsort order; a 128-row tile's mask is the OR
//     of its rows' masks AND mask_filter (kernel.py:844-866); backward-input
//     reverses it with brev(kmask) >> (32 - kv) (kernel.py:883-889) and skips
//     tiles whose mask is zero (kernel.py:875-882);
//   * for every offset k set in the tile mask, row r gathers
//     A[indices[k][sigma(r)]] (zero when the index is -1,
//     cumm/conv/sparse_iters.py:318-356, 625-648) and multiplies with the
//     weight slab of offset k (cumm/gemm/blockmma/mma.py:445-578);
//   * the epilogue writes row r to output row sigma(r) (permuted store,
//     cumm/gemm/out_iters.py:537-551) with act(alpha*acc + beta*src).
// The reference accumulates mask_output words per tile_shape[0] rows; here the
// compute tile is always 128 rows and the mask of each tile_shape[0]-row
// sub-tile (32/64/128) gates its own rows, which keeps results identical to a
// tile_shape[0]-row kernel even for masks inconsistent with the index table.
//
// B200 design (persistent, warp-specialised; tiles drawn from a per-call
// counter so CTAs that drew small tiles come back for more):
//   epilogue warps   TMEM -> registers -> act(alpha acc + beta src) -> row
//                    mask_argsort[r] (permuted store)
//   producer warps   A rows of each (offset, 128-byte column block) chunk by
//                    TMA tile::gather4 (4 rows per lane, SWIZZLE_128B or
//                    SWIZZLE_64B by address; index -1 reads as zero rows, each
//                    group of 4 gated by its 32-row sub-tile mask) and the
//                    weight slab by 2-D TMA boxes (backward-input: the [K, kv,
//                    C] weight itself, read MN-major); shorter rows (16 / 32
//                    bytes, several offsets packed per 128-byte row) by
//                    16-byte cp.async instead
//   loader warps     tile masks (OR, mask_filter, brev for backward-input),
//                    mask_output, and the tile's [offset][row] index table into
//                    a shared-memory ring: with the sorted table one 512-byte
//                    cp.async.bulk per offset, else all loads of a row issued
//                    together; the next tile is drawn one tile ahead
//   MMA warp         TMEM allocator + single-thread tcgen05.mma issuer into a
//                    double-buffered fp32 TMEM accumulator (128 lanes x BN)
// Layouts (Layout<kPair>): one 17-warp CTA per SM, or on the gather path two
// 11-warp CTAs per SM (4 producers, 2 loaders): measured on B200 the TMA
// gather rate is per issuing CTA, so two CTAs per SM gather ~1.5x the rows
// per cycle, which the kernel, bound by that rate, turns into ~12 % less time.
// Every mbarrier wait is bounded (globaltimer) and raises a CTA abort flag
// plus kErrWaitTimeout instead of spinning forever.
#include <cuda.h>

#include <mutex>

#include "kernels.h"

namespace scb {

// Source of the all-zero gathers: kZeroRows 128-byte rows of zeros.  Each
// gather picks its group of four from a spread of addresses, so the reads do
// not all land on one L2 slice.
__device__ __align__(1024) uint8_t g_zero_rows[kZeroRows * 128];

const void *zero_rows_address() {
  static std::mutex mu;
  static const void *addr[64] = {nullptr};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lk(mu);
  if (addr[dev] == nullptr) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_zero_rows) != cudaSuccess) return nullptr;
    addr[dev] = p;
  }
  return addr[dev];
}

namespace {

constexpr int kTileM = 128;

struct Meta {
  int nchunks;
  int n_active;
  uint32_t tilemask;
  int tile;  // tile index of this ring slot, -1 = no more tiles
  uint32_t sub[4];  // offsets active in each 32-row group (sub-tile mask, filtered)
  int k_list[32];
};

struct KParams {
  CUtensorMap tmap_a;  // gathered rows [a_rows, red] (TMA path)
  CUtensorMap tmap_b;  // B rows [n_total, kv * red] (TMA path)
  // four rows of zeros with tmap_a's box and swizzle: a gather whose four
  // rows are all -1 reads these instead (out-of-range gather rows cost the
  // TMA unit several times an in-range row)
  CUtensorMap tmap_zero;
  int zero_ok;
  ConvRowGatherArgs a;
  int64_t num_tiles;
  int cpo;            // chunks per offset (a_row_bytes >= 128), else 0
  int opc;            // offsets packed per chunk (a_row_bytes < 128)
  int upo;            // 16-byte units per packed offset segment
  int stages;
  uint32_t stage_bytes;
  uint32_t b_off;
  uint32_t idx_off;
  uint32_t idx_buf_bytes;
  uint32_t bar_off;
  uint32_t tmem_cols;
  uint32_t idesc;
  int row_bytes;  // bytes of one operand row in a stage: 128 (SWIZZLE_128B) or 64 (SWIZZLE_64B)
  int bulk_idx;   // sorted index table copied by 512-byte bulk copies (16-byte aligned rows)
  int b_mn;       // weight slab is MN-major: BN / 64 boxes of 64 reduction rows x 64 columns
};

__device__ __forceinline__ void flag_error(int *err, int bits) { atomicOr(err, bits); }

// ------------------------------------------------------------------ largest-first tile schedule
// A 128-row tile costs one chunk per (offset it visits, column block), and on
// the mask-sorted rows that count varies from a few offsets to all of them.
// Handing tiles out in mask order leaves the pipelines that drew the heavy
// tiles running alone at the end; handing them out heaviest first (the LPT
// rule) evens the pipelines out.  This kernel writes that order: one warp per
// tile ORs the tile's mask words (the kernels' tile mask: mask_filter, and
// brev for backward-input) and counts its offsets into the block's histogram,
// which the block adds to the global one; the last block to finish turns the
// histogram into descending bin starts and places every tile (a counting
// sort; the order inside a bin is arbitrary and does not affect any result,
// since each tile is computed by one pipeline alone).
constexpr int kOrderWarps = 32;

__global__ void __launch_bounds__(kOrderWarps * 32)
    tile_order_kernel(const uint32_t *__restrict__ mask, int64_t M, uint32_t filter, int reverse, int kv,
                      int64_t m_tiles, int *__restrict__ head, int32_t *__restrict__ tile_pc,
                      int32_t *__restrict__ order) {
  int *hist = head;        // [33]
  int *done = head + 33;   // blocks finished
  __shared__ int bins[33];
  __shared__ int last;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x < 33) bins[threadIdx.x] = 0;
  __syncthreads();
  const int64_t t = static_cast<int64_t>(blockIdx.x) * kOrderWarps + warp;
  if (t < m_tiles) {
    uint32_t v = 0u;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int64_t rq = t * kTileM + q * 32 + lane;
      if (rq < M) v |= mask ? __ldg(mask + rq) : 1u;
    }
#pragma unroll
    for (int sh = 16; sh > 0; sh >>= 1) v |= __shfl_xor_sync(0xffffffffu, v, sh);
    uint32_t tm = v & filter;
    if (reverse) tm = __brev(tm) >> (32 - kv);
    if (lane == 0) {
      const int pc = __popc(tm);
      tile_pc[t] = pc;
      atomicAdd(&bins[pc], 1);
    }
  }
  __syncthreads();
  if (threadIdx.x < 33 && bins[threadIdx.x] != 0) atomicAdd(hist + threadIdx.x, bins[threadIdx.x]);
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(done, 1) == static_cast<int>(gridDim.x) - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  if (threadIdx.x < 33) bins[threadIdx.x] = __ldcg(hist + threadIdx.x);
  __syncthreads();
  if (threadIdx.x == 0) {
    int acc = 0;
    for (int b = 32; b >= 0; --b) {
      const int c = bins[b];
      bins[b] = acc;
      acc += c;
    }
  }
  __syncthreads();
  // eight tiles per thread per pass, loads first
  constexpr int kPer = 8;
  for (int64_t base = 0; base < m_tiles; base += static_cast<int64_t>(blockDim.x) * kPer) {
    int pc[kPer];
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
      const int64_t i = base + j * static_cast<int64_t>(blockDim.x) + threadIdx.x;
      pc[j] = i < m_tiles ? __ldcg(tile_pc + i) : -1;
    }
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
      if (pc[j] < 0) continue;
      const int64_t i = base + j * static_cast<int64_t>(blockDim.x) + threadIdx.x;
      order[atomicAdd(&bins[pc[j]], 1)] = static_cast<int32_t>(i);
    }
  }
}

// Tile (row tile x column tile) at schedule position d: the d-th of the
// largest-first order when it exists, else d itself.  An order entry outside
// the row tiles (a caller-supplied order) sets the bad-index bit and maps to
// the first row tile past the end, whose rows all lie beyond M, so every
// role skips it.
__device__ __forceinline__ int64_t scheduled_tile(const ConvRowGatherArgs &A, int64_t d) {
  if (A.tile_order == nullptr) return d;
  const int64_t q = d / A.n_tiles;
  uint32_t mt = static_cast<uint32_t>(__ldg(A.tile_order + q));
  if (mt >= static_cast<uint32_t>(A.m_tiles)) {
    atomicOr(A.err, kErrBadIndex);
    mt = static_cast<uint32_t>(A.m_tiles);
  }
  return static_cast<int64_t>(mt) * A.n_tiles + (d - q * A.n_tiles);
}


// ------------------------------------------------------------------ epilogue helpers
template <int n, typename TOut>
__device__ __forceinline__ void load_src(const TOut *p, float *v) {
  if constexpr (sizeof(TOut) == 4) {
#pragma unroll
  for (int i = 0; i < n; i += 4) {
    const float4 q = *reinterpret_cast<const float4 *>(p + i);
    v[i] = q.x; v[i + 1] = q.y; v[i + 2] = q.z; v[i + 3] = q.w;
  }
  } else {
#pragma unroll
  for (int i = 0; i < n; i += 8) {
    const uint4 q = *reinterpret_cast<const uint4 *>(p + i);
    const TOut *h = reinterpret_cast<const TOut *>(&q);
#pragma unroll
    for (int j = 0; j < 8; ++j) v[i + j] = to_f32(h[j]);
  }
  }
}

// One 32-byte store (a whole DRAM sector: no partial-sector merge in L2).
__device__ __forceinline__ void st_global_v8(void *p, const uint32_t *w) {
  asm volatile("st.global.v8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(p), "r"(w[0]), "r"(w[1]), "r"(w[2]),
               "r"(w[3]), "r"(w[4]), "r"(w[5]), "r"(w[6]), "r"(w[7])
               : "memory");
}

// Stores n values to p: 32-byte stores when p is 32-byte aligned, else 16-byte.
template <int n, typename TOut>
__device__ __forceinline__ void store_row(TOut *p, const float *v) {
  constexpr int kPer32 = 32 / sizeof(TOut);  // values per 32 bytes
  static_assert(n % kPer32 == 0, "row chunk must be whole 32-byte units");
  const bool a32 = (reinterpret_cast<uintptr_t>(p) & 31u) == 0;
#pragma unroll
  for (int i = 0; i < n; i += kPer32) {
    uint32_t w[8];
    if constexpr (sizeof(TOut) == 4) {
#pragma unroll
      for (int j = 0; j < 8; ++j) w[j] = __float_as_uint(v[i + j]);
    } else {
      TOut *h = reinterpret_cast<TOut *>(w);
#pragma unroll
      for (int j = 0; j < 16; ++j) h[j] = from_f32<TOut>(v[i + j]);
    }
    if (a32) {
      st_global_v8(p + i, w);
    } else {
      *reinterpret_cast<uint4 *>(p + i) = make_uint4(w[0], w[1], w[2], w[3]);
      *reinterpret_cast<uint4 *>(p + i + kPer32 / 2) = make_uint4(w[4], w[5], w[6], w[7]);
    }
  }
}

// Applies the epilogue to `n` (16 or 32) consecutive columns starting at column
// `col` of output row `orow` and stores them.
template <int n, typename TOut>
__device__ __forceinline__ void epilogue_cols(const KParams &P, float *acc, int64_t orow, int col) {
  const EpiParams &e = P.a.epi;
  float src[n];
  const bool use_src = e.beta != 0.f && e.src != nullptr;
  if (use_src) {
    const TOut *s = reinterpret_cast<const TOut *>(e.src) + orow * e.src_ld + col;
    load_src<n, TOut>(s, src);
  }
  if (e.mode == 1) {
    float bias[n];
    if (e.bias != nullptr) load_src<n, TOut>(reinterpret_cast<const TOut *>(e.bias) + col, bias);
#pragma unroll
    for (int i = 0; i < n; ++i) {
      float sc = e.scale != nullptr ? __ldg(e.scale + col + i) : 1.f;
      float v = sc * acc[i] + (e.bias != nullptr ? e.alpha * bias[i] : 0.f);
      if (use_src) v = fmaf(e.beta, src[i], v);
      acc[i] = apply_act(v, e.act_type, e.act_alpha);
    }
  } else {
#pragma unroll
    for (int i = 0; i < n; ++i) {
      float v = e.alpha * acc[i];
      if (use_src) v = fmaf(e.beta, src[i], v);
      acc[i] = apply_act(v, e.act_type, e.act_alpha);
    }
  }
  TOut *dst = reinterpret_cast<TOut *>(P.a.out) + orow * P.a.out_ld + col;
  store_row<n, TOut>(dst, acc);
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// ------------------------------------------------------------------ kernel
// Warp roles (17 warps):
// Two layouts.  Single (one CTA per SM, 17 warps): warps 0-3 epilogue, 4-11
// producers, 12-15 index loaders, 16 MMA; 3-deep index ring.  Pair (two
// CTAs per SM, 11 warps each, for the gather path when two fit): warps 0-3
// epilogue, 4-7 producers, 8-9 index loaders (2 rows per thread), 10 MMA;
// 2-deep index ring.  Measured on B200: two CTAs per SM gather ~1.5x the
// rows per cycle of one (the TMA gather rate is per issuing CTA, not per SM).
constexpr int kEpiWarps = 4;  // warps 0-3 in both layouts
constexpr int kProdWarp0 = 4;
template <bool kPair> struct Layout {
  static constexpr int kProdWarps = kPair ? 4 : 8;
  static constexpr int kLoadWarp0 = kProdWarp0 + kProdWarps;
  static constexpr int kLoadWarps = kPair ? 2 : 4;
  static constexpr int kMmaWarp = kLoadWarp0 + kLoadWarps;
  static constexpr int kThreads = (kMmaWarp + 1) * 32;
  static constexpr int kIdxStages = kPair ? 2 : 3;
  static constexpr int kRowsPer = kTileM / (kLoadWarps * 32);
};

// Registers: single layout 17 warps (5 per SMSP) x 96; pair layout 2 x 11
// warps (up to 6 per SMSP) x 80 = 15360 of an SMSP's 16K registers.
template <bool kF8, typename TOut, bool kTma, bool kGather, bool kPair>
__global__ void __maxnreg__(kPair ? 80 : 96)
    conv_rowgather_kernel(const __grid_constant__ KParams P) {
  constexpr int kProdWarps = Layout<kPair>::kProdWarps;
  constexpr int kLoadWarp0 = Layout<kPair>::kLoadWarp0;
  constexpr int kLoadWarps = Layout<kPair>::kLoadWarps;
  constexpr int kMmaWarp = Layout<kPair>::kMmaWarp;
  constexpr int kIdxStages = Layout<kPair>::kIdxStages;
  constexpr int kRowsPer = Layout<kPair>::kRowsPer;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw_u32 = smem_u32(smem_raw);
  const uint32_t pad = (1024u - (raw_u32 & 1023u)) & 1023u;
  uint8_t *smem = smem_raw + pad;
  const uint32_t smem_base = raw_u32 + pad;

  const int S = P.stages;
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + P.bar_off);
  uint64_t *full_bar = bars;
  uint64_t *empty_bar = bars + S;
  uint64_t *idx_full = bars + 2 * S;
  uint64_t *idx_empty = idx_full + kIdxStages;
  uint64_t *acc_full = idx_empty + kIdxStages;
  uint64_t *acc_empty = acc_full + 2;
  uint64_t *drain_bar = acc_empty + 2;
  uint64_t *tile_bar = drain_bar + 1;  // [2]: tile of accumulator buffer b announced
  uint64_t *sched_bar = tile_bar + 2;  // [4]: next tile drawn by loader warp 0
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(sched_bar + 4);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);
  volatile int *acc_tile = abort_flag + 1;    // [2]: tile held by accumulator buffer b
  volatile int *sched_tile = acc_tile + 2;    // [4]: tile of loader iteration i (slot i & 3)

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const ConvRowGatherArgs &A = P.a;

  if (threadIdx.x == 0) {
    for (int i = 0; i < S; ++i) {
      // gather: one arrive.expect_tx per producer warp; cp.async: the 32
      // lanes of the stage's producer warp (cp.async.mbarrier.arrive.noinc)
      // plus, with TMA, one arrive.expect_tx for the weight slab
      mbar_init(&full_bar[i], kGather ? kProdWarps : 32 + (kTma ? 1 : 0));
      mbar_init(&empty_bar[i], 1);
    }
    for (int i = 0; i < kIdxStages; ++i) {
      mbar_init(&idx_full[i], kLoadWarps * 32);
      mbar_init(&idx_empty[i], (kGather ? kProdWarps : min(S, kProdWarps)) + 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(&acc_full[i], 1);
      mbar_init(&acc_empty[i], 128);
    }
    mbar_init(drain_bar, 1);
    mbar_init(&tile_bar[0], 1);
    mbar_init(&tile_bar[1], 1);
    for (int i = 0; i < 4; ++i) mbar_init(&sched_bar[i], 1);
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == kMmaWarp) {
    tmem_alloc(tmem_slot, P.tmem_cols);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  if (warp >= kLoadWarp0 && warp < kLoadWarp0 + kLoadWarps) {
    // ---------------------------------------------------------------- index loaders
    // kLoadWarps warps, kRowsPer rows of the tile per thread (row t + i * 32 kLoadWarps)
    const int t = threadIdx.x - kLoadWarp0 * 32;
    const int lw = t >> 5;
    int next_draw = -1;  // lane 0 of loader warp 0: counter value drawn one tile ahead, or -1
    for (int it = 0;; ++it) {
      const int b = it % kIdxStages;
      const uint32_t ph = (it / kIdxStages) & 1;
      if (!mbar_wait(&idx_empty[b], ph ^ 1, abort_flag)) {
        flag_error(A.err, kErrWaitTimeout);
        break;
      }
      uint8_t *buf = smem + P.idx_off + b * P.idx_buf_bytes;
      int *tab = reinterpret_cast<int *>(buf);
      Meta *meta = reinterpret_cast<Meta *>(buf + A.kv * kTileM * 4);
      // Next tile: from the launch-wide counter when there is one (CTAs that
      // drew small tiles come back for more, which evens out the per-CTA
      // work), else every gridDim.x-th tile.  Lane 0 of loader warp 0 draws
      // it and publishes it through slot it & 3 (store, then arrive); the
      // other loader warps take it with a bounded wait.  A reader can trail
      // the drawer by two iterations at most (the drawer's idx_empty wait for
      // iteration i + 2 needs every loader thread's idx_full arrival for
      // i - 1), so four slots are never overwritten before they are read.
      int tile;
      if (lw == 0) {
        int t = -1;
        if (lane == 0) {
          const int64_t d = A.tile_counter
                                ? static_cast<int64_t>(next_draw >= 0 ? next_draw : atomicAdd(A.tile_counter, 1))
                                : static_cast<int64_t>(blockIdx.x) + static_cast<int64_t>(it) * gridDim.x;
          t = d < P.num_tiles ? static_cast<int>(scheduled_tile(A, d)) : -1;
          // While more tiles remain than there are CTAs, the following tile is
          // drawn now, so the atomic's round trip overlaps this tile's loads;
          // near the end (or on a grid with few tiles) a CTA holding two
          // tiles would idle the others, so it draws when it needs one.
          next_draw = -1;
          if (A.tile_counter && t >= 0 && d + 2 * static_cast<int64_t>(gridDim.x) < P.num_tiles)
            next_draw = atomicAdd(A.tile_counter, 1);
          sched_tile[it & 3] = t;
          mbar_arrive(&sched_bar[it & 3]);
        }
        tile = __shfl_sync(0xffffffffu, t, 0);
      } else {
        if (!mbar_wait(&sched_bar[it & 3], (it >> 2) & 1, abort_flag)) {
          flag_error(A.err, kErrWaitTimeout);
          break;
        }
        tile = sched_tile[it & 3];
      }
      if (tile < 0) {
        if (t == 0) meta->tile = -1;
        mbar_arrive(&idx_full[b]);
        break;
      }
      const int64_t tile_m = tile / A.n_tiles;
      const int n_tile = static_cast<int>(tile % A.n_tiles);
      uint32_t g0 = 0, g1 = 0, g2 = 0, g3 = 0, tm = 0;
      // Sorted table and whole 128-row tile with 16-byte aligned slices:
      // each offset's 128 indices are one 512-byte bulk copy that completes
      // on idx_full, and the producers apply the sub-tile masks; otherwise
      // every thread loads, gates and stores its rows' indices.
      const bool bulk = kGather && P.bulk_idx && (tile_m + 1) * kTileM <= A.M;
      if (bulk && lw == 0) {
        if (lane == 0) mbar_expect_tx(&idx_full[b], static_cast<uint32_t>(A.kv) * kTileM * 4);
        __syncwarp();
        if (lane < A.kv)
          bulk_copy_g2s(smem_u32(tab + lane * kTileM),
                        A.idx_sorted + static_cast<int64_t>(lane) * A.M + tile_m * kTileM, kTileM * 4,
                        &idx_full[b]);
      }
#pragma unroll 1
      for (int rr = 0; rr < kRowsPer; ++rr) {
        if (bulk && rr > 0) break;
        const int r = t + rr * (kLoadWarps * 32);  // row inside the tile
        const int64_t row_g = tile_m * kTileM + r;
        const bool valid = row_g < A.M;
        // Every index of the row (all kv offsets) is loaded up front and stored
        // unconditionally below, so the loads leave together: one memory round
        // trip per row.  With the sorted table row_g is already the sorted row;
        // otherwise sigma(row) comes first (argsort), then the kv loads.
        int pre[32];
        if (bulk) {
        } else if (A.idx_sorted) {
#pragma unroll
          for (int k = 0; k < 32; ++k)
            pre[k] = (valid && k < A.kv) ? __ldg(A.idx_sorted + static_cast<int64_t>(k) * A.M + row_g)
                                         : -1;
        } else {
          int sig = valid ? (A.argsort ? __ldg(A.argsort + row_g) : static_cast<int>(row_g)) : -1;
          if (valid && (sig < 0 || sig >= A.out_rows)) {
            flag_error(A.err, kErrBadIndex);
            sig = -1;
          }
          int ident = -1;
          if (!A.indices && sig >= 0) ident = A.a_inds ? __ldg(A.a_inds + row_g) : static_cast<int>(row_g);
#pragma unroll
          for (int k = 0; k < 32; ++k)
            pre[k] = (sig >= 0 && k < A.kv)
                         ? (A.indices ? __ldg(A.indices + static_cast<int64_t>(k) * A.M + sig) : ident)
                         : -1;
        }
        if (rr == 0) {
          // every loader warp reduces all four 32-row groups itself (no
          // cross-warp barrier, so an aborted warp can never strand the others)
          uint32_t gq[4];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int64_t rq = tile_m * kTileM + q * 32 + lane;
            uint32_t v = rq < A.M ? (A.mask ? __ldg(A.mask + rq) : 1u) : 0u;
#pragma unroll
            for (int sh = 16; sh > 0; sh >>= 1) v |= __shfl_xor_sync(0xffffffffu, v, sh);
            gq[q] = v;
          }
          g0 = gq[0];
          g1 = gq[1];
          g2 = gq[2];
          g3 = gq[3];
          tm = (g0 | g1 | g2 | g3) & A.mask_filter;
          if (A.is_fwd && A.mask_out != nullptr && n_tile == 0 && t == 0) {
            const int nsub = kTileM / A.tile_m_desp;
            for (int d = 0; d < nsub; ++d) {
              const int64_t start = tile_m * kTileM + d * A.tile_m_desp;
              if (start >= A.M) break;
              uint32_t w;
              if (nsub == 4) w = d == 0 ? g0 : d == 1 ? g1 : d == 2 ? g2 : g3;
              else if (nsub == 2) w = d == 0 ? (g0 | g1) : (g2 | g3);
              else w = g0 | g1 | g2 | g3;
              A.mask_out[start / A.tile_m_desp] = w & A.mask_filter;
            }
          }
          if (A.reverse) tm = __brev(tm) >> (32 - A.kv);
        }
        const int lr = r >> 5;  // 32-row group of this row
        uint32_t sub;
        if (A.tile_m_desp == 32) {
          sub = lr == 0 ? g0 : lr == 1 ? g1 : lr == 2 ? g2 : g3;
        } else if (A.tile_m_desp == 64) {
          sub = lr < 2 ? (g0 | g1) : (g2 | g3);
        } else {
          sub = g0 | g1 | g2 | g3;
        }
        sub &= A.mask_filter;
        if (A.reverse) sub = __brev(sub) >> (32 - A.kv);
        // tab[k][r]: index of row r for offset k (-1 where the row's sub-tile
        // mask lacks k).  Written for every offset, whatever the tile mask: a
        // select, not a branch, so no load is deferred to its use.
        if (!bulk) {
#pragma unroll
          for (int k = 0; k < 32; ++k) {
            if (k < A.kv) {
              int v = ((sub >> k) & 1u) ? pre[k] : -1;
              if (v < -1 || v >= A.a_rows) {
                flag_error(A.err, kErrBadIndex);
                v = -1;
              }
              tab[k * kTileM + r] = v;
            }
          }
          // a later bulk copy (async proxy) may overwrite these stores
          fence_proxy_async_smem();
        }
      }
      if (t == 0) {
        const int na = __popc(tm);
        int s = 0;
        uint32_t mm = tm;
        while (mm) {
          const int k = __ffs(mm) - 1;
          mm &= mm - 1;
          meta->k_list[s++] = k;
        }
        meta->n_active = na;
        meta->tilemask = tm;
        meta->tile = tile;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          uint32_t sq;
          if (A.tile_m_desp == 32) sq = q == 0 ? g0 : q == 1 ? g1 : q == 2 ? g2 : g3;
          else if (A.tile_m_desp == 64) sq = q < 2 ? (g0 | g1) : (g2 | g3);
          else sq = g0 | g1 | g2 | g3;
          sq &= A.mask_filter;
          if (A.reverse) sq = __brev(sq) >> (32 - A.kv);
          meta->sub[q] = sq;
        }
        meta->nchunks = P.cpo > 0 ? na * P.cpo : (na + P.opc - 1) / P.opc;
      }
      mbar_arrive(&idx_full[b]);
    }
  } else if (warp >= kProdWarp0 && warp < kProdWarp0 + kProdWarps) {
    // ---------------------------------------------------------------- producers
    const int pw = warp - kProdWarp0;
    if constexpr (kGather) {
    // TMA gather: all kProdWarps warps serve every chunk; lanes 0-3 of warp pw
    // each issue one tile::gather4 (4 rows x 128 bytes, SWIZZLE_128B by
    // address) for rows [16 pw, 16 pw + 16) of the stage.  An index of -1 is
    // an out-of-range row and lands as zeros.  Lane 0 of every warp arrives
    // with expect_tx for its 2 KB (one warp in turn adds the weight slab), so
    // a stage completes on kProdWarps arrivals plus the copied bytes.  Every
    // warp arrives once per use of stage s and empty phase n cannot complete
    // before all of them did, so no warp runs two phases ahead of a wait.
    // (Measured on B200: 8 warps of gather4 fill a 16 KB stage in ~740
    // cycles; per-thread cp.async arrivals serialise on the barrier word.)
    const int esz = kF8 ? 1 : 2;
    const int rb = P.row_bytes;  // 128, or 64 for 64-byte rows (SWIZZLE_64B stages)
    const int box = rb / esz;
    const uint32_t a_tx = (kTileM / kProdWarps) * static_cast<uint32_t>(rb);
    const uint32_t b_tx = static_cast<uint32_t>(A.BN) * rb;
    const int r0 = pw * (kTileM / kProdWarps) + lane * 4;
    int it = 0;
    uint32_t stage = 0, eph = 0, gchunk = 0;
    bool ok = true;
    for (; ok; ++it) {
      const int b = it % kIdxStages;
      const uint32_t ph = (it / kIdxStages) & 1;
      if (!__all_sync(0xffffffffu, mbar_wait(&idx_full[b], ph, abort_flag))) {
        if (lane == 0) flag_error(A.err, kErrWaitTimeout);
        break;
      }
      const uint8_t *buf = smem + P.idx_off + b * P.idx_buf_bytes;
      const int *tab = reinterpret_cast<const int *>(buf);
      const Meta *meta = reinterpret_cast<const Meta *>(buf + A.kv * kTileM * 4);
      const int tile = meta->tile;
      if (tile < 0) break;
      const int nch = meta->nchunks;
      const int n0 = (tile % A.n_tiles) * A.BN;
      for (int j = 0; j < nch; ++j) {
        const uint32_t s = stage;
        const int slot_a = j / P.cpo;
        const int cb = j - slot_a * P.cpo;
        const int k = meta->k_list[slot_a];
        const uint32_t sA = smem_base + s * P.stage_bytes;
        if (!__all_sync(0xffffffffu, mbar_wait(&empty_bar[s], eph ^ 1, abort_flag))) {
          if (lane == 0) flag_error(A.err, kErrWaitTimeout);
          ok = false;
          break;
        }
        if (lane == 0) {
          if (static_cast<int>(gchunk % kProdWarps) == pw) {
            mbar_arrive_expect_tx(&full_bar[s], a_tx + b_tx);
            if (P.b_mn) {
              // rows j = cb * 64 .. + 63 of the weight, columns k * C + n0 + 64 q
              for (int q = 0; q < A.BN / 64; ++q)
                tma_load_2d(sA + P.b_off + q * 8192, &P.tmap_b, k * (A.b_off_stride / esz) + n0 + 64 * q,
                            cb * 64, &full_bar[s]);
            } else {
              tma_load_2d(sA + P.b_off, &P.tmap_b, k * (A.b_off_stride / esz) + cb * box, n0,
                          &full_bar[s]);
            }
          } else {
            mbar_arrive_expect_tx(&full_bar[s], a_tx);
          }
        }
        __syncwarp();
        if (lane < (kTileM / kProdWarps) / 4) {
          int4 q = *reinterpret_cast<const int4 *>(tab + k * kTileM + r0);
          // rows r0..r0+3 share a 32-row group: gate by its sub-tile mask
          // (bulk-copied tables are ungated) and check the indices
          if (!((meta->sub[r0 >> 5] >> k) & 1u)) q = make_int4(-1, -1, -1, -1);
          const bool bad = q.x < -1 || q.x >= A.a_rows || q.y < -1 || q.y >= A.a_rows ||
                           q.z < -1 || q.z >= A.a_rows || q.w < -1 || q.w >= A.a_rows;
          if (bad) {
            flag_error(A.err, kErrBadIndex);
            q = make_int4(-1, -1, -1, -1);
          }
          if (P.zero_ok && (q.x & q.y & q.z & q.w) == -1) {
            const int z = zero_group(blockIdx.x * 32 + pw * 8 + lane, gchunk);
            tma_gather4(sA + r0 * rb, &P.tmap_zero, 0, z, z + 1, z + 2, z + 3, &full_bar[s]);
          }
          else
            tma_gather4(sA + r0 * rb, &P.tmap_a, cb * box, q.x, q.y, q.z, q.w, &full_bar[s]);
        }
        ++gchunk;
        if (++stage == static_cast<uint32_t>(S)) {
          stage = 0;
          eph ^= 1u;
        }
      }
      if (!ok) break;
      __syncwarp();
      if (lane == 0) mbar_arrive(&idx_empty[b]);
    }
    } else {
    // Producer warp pw owns shared-memory stage pw (S <= kProdWarps stages;
    // warps beyond S stay idle) and fills every chunk c with c % S == pw
    // alone: lane owns 16-byte unit u of rows rg + 4 i (i < 32).  The S stages
    // are filled concurrently and the per-stage synchronisation is amortised
    // over 32 copies per lane.  One owner per stage also keeps every empty-
    // barrier wait exactly one phase ahead of the MMA warp (a parity wait
    // cannot tell phase k from k + 2).
    // Rows with a pair are fetched with 16-byte cp.async; rows without one are
    // zero-filled cp.async (src-size 0, no memory request).  With TMA the
    // weight slab is one 2-D tiled load issued by lane 0.
    const int u = lane & 7;
    const int rg = lane >> 3;
    const int esz = kF8 ? 1 : 2;
    const int box = 128 / esz;
    const uint32_t b_tx = static_cast<uint32_t>(A.BN) * 128;
    int it = 0;
    uint32_t c_base = 0;  // chunks of all previous tiles
    bool ok = pw < S;
    for (; ok; ++it) {
      const int b = it % kIdxStages;
      const uint32_t ph = (it / kIdxStages) & 1;
      int w_ok = 1;
      if (lane == 0) w_ok = mbar_wait(&idx_full[b], ph, abort_flag) ? 1 : 0;
      w_ok = __shfl_sync(0xffffffffu, w_ok, 0);
      if (!w_ok) {
        if (lane == 0) flag_error(A.err, kErrWaitTimeout);
        break;
      }
      const uint8_t *buf = smem + P.idx_off + b * P.idx_buf_bytes;
      const int *tab = reinterpret_cast<const int *>(buf);
      const Meta *meta = reinterpret_cast<const Meta *>(buf + A.kv * kTileM * 4);
      const int tile = meta->tile;
      if (tile < 0) break;
      const int nch = meta->nchunks;
      const int na = meta->n_active;
      const int n0 = (tile % A.n_tiles) * A.BN;
      const uint32_t uS = static_cast<uint32_t>(S);
      const int j0 = static_cast<int>((static_cast<uint32_t>(pw) + uS - c_base % uS) % uS);
      for (int j = j0; j < nch; j += S) {
        const uint32_t c = c_base + static_cast<uint32_t>(j);
        const uint32_t s = static_cast<uint32_t>(pw);  // == c % S
        const uint32_t eph = (c / uS) & 1u;
        int slot_a, cb;
        if (P.cpo > 0) {
          slot_a = j / P.cpo;
          cb = j - slot_a * P.cpo;
        } else {
          slot_a = 0;
          cb = 0;
        }
        int e_ok = 1;
        const uint32_t sA = smem_base + s * P.stage_bytes;
        const uint32_t sB = sA + P.b_off;
        if (lane == 0) {
          e_ok = mbar_wait(&empty_bar[s], eph ^ 1, abort_flag) ? 1 : 0;
          if constexpr (kTma) {
            if (e_ok) {
              mbar_arrive_expect_tx(&full_bar[s], b_tx);
              const int xb = meta->k_list[slot_a] * (A.b_off_stride / esz) + cb * box;
              tma_load_2d(sB, &P.tmap_b, xb, n0, &full_bar[s]);
            }
          }
        }
        e_ok = __shfl_sync(0xffffffffu, e_ok, 0);
        if (!e_ok) {
          if (lane == 0) flag_error(A.err, kErrWaitTimeout);
          ok = false;
          break;
        }
        int slot, byte0;
        if (P.cpo > 0) {
          slot = slot_a;
          byte0 = cb * 128 + u * 16;
        } else {
          slot = j * P.opc + u / P.upo;
          byte0 = (u % P.upo) * 16;
        }
        const bool slot_ok = slot < na && byte0 < A.a_row_bytes;
        const int *trow = tab + (slot_ok ? meta->k_list[slot] : 0) * kTileM;
        const uint8_t *abase = A.a_base + byte0;
#pragma unroll 8
        for (int i = 0; i < kTileM / 4; ++i) {
          const int r = rg + 4 * i;
          const int idx = slot_ok ? trow[r] : -1;
          const uint32_t dst = sA + sw128(r, u);
          if (idx >= 0)
            cp_async_16(dst, abase + static_cast<int64_t>(idx) * A.a_row_stride, 16u);
          else
            cp_async_16(dst, A.a_base, 0u);  // zero fill, no memory request
        }
        if constexpr (!kTma) {
          // B: BN rows x 8 units over the warp's 32 lanes
          for (int q = lane; q < A.BN * 8; q += 32) {
            const int n = q >> 3;
            const int uu = q & 7;
            int kb, bbyte;
            if (P.cpo > 0) {
              kb = meta->k_list[slot];
              bbyte = cb * 128 + uu * 16;
            } else {
              const int sl = j * P.opc + uu / P.upo;
              kb = sl < na ? meta->k_list[sl] : -1;
              bbyte = (uu % P.upo) * 16;
            }
            const int ng = n0 + n;
            const uint32_t dst = sB + sw128(n, uu);
            if (kb >= 0 && ng < A.n_total && bbyte < A.a_row_bytes) {
              cp_async_16(dst,
                          A.b_base + static_cast<int64_t>(ng) * A.b_row_stride +
                              static_cast<int64_t>(kb) * A.b_off_stride + bbyte,
                          16u);
            } else {
              cp_async_16(dst, A.b_base, 0u);  // zero fill, no memory request
            }
          }
        }
        // the stage's full barrier counts each lane once its copies land
        cp_async_mbar_arrive_noinc(&full_bar[s]);
      }
      if (!ok) break;
      c_base += static_cast<uint32_t>(nch);
      __syncwarp();
      if (lane == 0) mbar_arrive(&idx_empty[b]);
    }
    cp_async_wait_all();
    }
  } else if (warp == kMmaWarp) {
    // ---------------------------------------------------------------- MMA issuer
    if (lane == 0) {
      int it = 0;
      uint32_t stage = 0, fph = 0;
      bool issued = false;
      // 8-row swizzle atoms: 1024 bytes apart for 128-byte rows (SWIZZLE_128B),
      // 512 for 64-byte rows (SWIZZLE_64B); one MMA per 32 bytes of K
      const uint64_t a_desc0 = P.row_bytes == 64 ? make_sdesc_l(smem_base, 16, 512, 4u)
                                                 : make_sdesc(smem_base, 16, 1024);
      const int mmas = P.row_bytes / 32;
      // B of stage 0 and its step per MMA (descriptor units of 16 bytes):
      // K-major B advances 32 bytes inside its rows; MN-major B (64-wide
      // column atoms 8 KB apart) advances 16 rows = 2 KB
      const uint64_t b_desc0 = P.b_mn ? make_sdesc(smem_base + P.b_off, 8192, 1024)
                                      : a_desc0 + static_cast<uint64_t>(P.b_off >> 4);
      const uint64_t b_kstep = P.b_mn ? 128 : 2;
      for (;; ++it) {
        const int b = it % kIdxStages;
        const uint32_t ph = (it / kIdxStages) & 1;
        if (!mbar_wait(&idx_full[b], ph, abort_flag)) {
          flag_error(A.err, kErrWaitTimeout);
          break;
        }
        const Meta *meta =
            reinterpret_cast<const Meta *>(smem + P.idx_off + b * P.idx_buf_bytes + A.kv * kTileM * 4);
        const int nch = meta->nchunks;
        const int tile = meta->tile;
        mbar_arrive(&idx_empty[b]);
        const int ab = it & 1;
        const uint32_t aph = (it >> 1) & 1;
        if (!mbar_wait(&acc_empty[ab], aph ^ 1, abort_flag)) {
          flag_error(A.err, kErrWaitTimeout);
          break;
        }
        tc_fence_after();
        // announce the buffer's tile to the epilogue (the plain arrive
        // releases the store to the epilogue's wait); -1 ends the epilogue
        acc_tile[ab] = tile;
        mbar_arrive(&tile_bar[ab]);
        if (tile < 0) break;
        const uint32_t d = tmem_base + static_cast<uint32_t>(ab * A.BN);
        if (nch == 0) {
          mbar_arrive(&acc_full[ab]);
          continue;
        }
        bool ok = true;
        for (int j = 0; j < nch; ++j) {
          const uint32_t s = stage;
          if (!mbar_wait(&full_bar[s], fph, abort_flag)) {
            flag_error(A.err, kErrWaitTimeout);
            ok = false;
            break;
          }
          tc_fence_after();
          const uint64_t ad0 = a_desc0 + static_cast<uint64_t>((s * P.stage_bytes) >> 4);
          const uint64_t bd0 = b_desc0 + static_cast<uint64_t>((s * P.stage_bytes) >> 4);
#pragma unroll
          for (int kk = 0; kk < 4; ++kk) {
            if (kk >= mmas) break;
            // K advances 32 bytes inside the swizzle atom (start address >> 4)
            const uint64_t ad = ad0 + static_cast<uint64_t>(kk * 2);
            const uint64_t bd = bd0 + static_cast<uint64_t>(kk) * b_kstep;
            if constexpr (kF8)
              mma_f8(d, ad, bd, P.idesc, (j | kk) != 0 ? 1u : 0u);
            else
              mma_f16(d, ad, bd, P.idesc, (j | kk) != 0 ? 1u : 0u);
          }
          issued = true;
          mma_commit(&empty_bar[s]);
          if (++stage == static_cast<uint32_t>(S)) {
            stage = 0;
            fph ^= 1u;
          }
        }
        if (!ok) break;
        mma_commit(&acc_full[ab]);
      }
      if (issued) {
        // make sure no tcgen05.mma is in flight before TMEM is released
        mma_commit(drain_bar);
        int never = 0;
        if (!mbar_wait(drain_bar, 0, reinterpret_cast<volatile int *>(&never)))
          flag_error(A.err, kErrWaitTimeout);
      }
    }
  } else if (warp < kEpiWarps) {
    // ---------------------------------------------------------------- epilogue (warps 0-3)
    const int r = threadIdx.x;  // TMEM lane == tile row
    const uint32_t lane_base = static_cast<uint32_t>(warp * 32) << 16;
    for (int it = 0;; ++it) {
      const int ab = it & 1;
      const uint32_t aph = (it >> 1) & 1;
      if (!mbar_wait(&tile_bar[ab], aph, abort_flag)) {
        flag_error(A.err, kErrWaitTimeout);
        break;
      }
      const int tile = acc_tile[ab];
      if (tile < 0) break;
      const int64_t tile_m = tile / A.n_tiles;
      const int n0 = static_cast<int>(tile % A.n_tiles) * A.BN;
      const int64_t row_g = tile_m * kTileM + r;
      const bool valid = row_g < A.M;
      int sig = valid ? (A.argsort ? __ldg(A.argsort + row_g) : static_cast<int>(row_g)) : -1;
      if (sig >= A.out_rows) sig = -1;
      uint32_t km = 0;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int64_t rr = tile_m * kTileM + q * 32 + lane;
        if (rr < A.M) km |= A.mask ? __ldg(A.mask + rr) : 1u;
      }
#pragma unroll
      for (int s = 16; s > 0; s >>= 1) km |= __shfl_xor_sync(0xffffffffu, km, s);
      km &= A.mask_filter;
      if (!mbar_wait(&acc_full[ab], aph, abort_flag)) {
        flag_error(A.err, kErrWaitTimeout);
        break;
      }
      tc_fence_after();
      const bool write = valid && sig >= 0 && (A.is_fwd || km != 0);
      const uint32_t tbase = tmem_base + lane_base + static_cast<uint32_t>(ab * A.BN);
      for (int cc = 0; cc < A.BN; cc += 16) {
        float acc[16];
        if (km != 0) {
          tmem_ld16(tbase + cc, acc);
        } else {
#pragma unroll
          for (int i = 0; i < 16; ++i) acc[i] = 0.f;
        }
        if (write) epilogue_cols<16, TOut>(P, acc, sig, n0 + cc);
      }
      tc_fence_before();
      mbar_arrive(&acc_empty[ab]);
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == kMmaWarp) {
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem_base, P.tmem_cols);
  }
}

// ------------------------------------------------------------------ strand kernel
// Forward / backward-input over 128-byte (SWIZZLE_128B) or 64-byte
// (SWIZZLE_64B: C = 64 e4m3, C = 32 bf16 / f16) gathered rows with several
// independent pipelines ("strands") per SM: two CTAs per SM, each running
// kStrands strands.  A strand owns kSProd producer warps, its own ring of
// P.stages stages (128 gathered rows + the weight slab; as many as fit, 2 of
// 24 KB for 128-byte rows at BN = 64, 4 of 12 KB for 64-byte rows), one MMA
// warp and a double-buffered TMEM accumulator; the four epilogue warps of the
// CTA serve both strands.  The kernel is bound by the latency of its rings
// (each stage needs a producer -> MMA -> producer round trip), so the ring
// depth that shared memory allows sets its speed.  Measured on B200: one tcgen05.mma stream (one issuing warp)
// completes an M = 128, K = 16 MMA about every 170 cycles whatever N is, and
// one producer ring (its warps, stages and barriers) fills ~18-30 bytes per
// cycle; both rates grow with the number of independent streams on the SM
// (four MMA warps: ~5450 FLOP/clk/SM at N = 64; four rings of four TMA warps:
// ~65 B/clk/SM), which the strands provide.  Tiles are taken in the
// largest-first order when one is given (strand_tile), else round-robin.  Every role derives its tiles' masks itself (the
// tile's mask words OR-ed per 32-row group), and the producers read each
// gather's four indices straight from the sorted index table, so the strands
// share no index ring.  Needs indices_sorted (16-byte aligned, M % 4 == 0)
// and BN <= 64.
constexpr int kStrands = 2;
constexpr int kSProd = 4;
constexpr int kSMaxStages = 4;  // stages per strand: 2 of 24 KB (128-byte rows), 4 of 12 KB (64-byte rows)
constexpr int kSWarps = kEpiWarps + kStrands * (kSProd + 1);  // 14
constexpr int kSThreads = kSWarps * 32;
constexpr int kSBars = 2 * kSMaxStages + 7;  // barriers per strand
constexpr uint32_t kSTmemCols = 256;      // per CTA: kStrands x 2 buffers x BN (<= 64)

struct TileMasks {
  uint32_t g[4];    // OR of each 32-row group (unfiltered)
  uint32_t sub[4];  // mask gating each 32-row group (descriptor tile, filtered, reversed for dgrad)
  uint32_t tm;      // offsets the tile visits (filtered, reversed for dgrad)
};

// Lane l loads the mask words of rows q * 32 + l (q < 4) of a 128-row tile.
__device__ __forceinline__ void load_mask_words(const ConvRowGatherArgs &A, int64_t tile_m, int lane,
                                                uint32_t (&w)[4]) {
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int64_t rq = tile_m * kTileM + q * 32 + lane;
    w[q] = rq < A.M ? (A.mask ? __ldg(A.mask + rq) : 1u) : 0u;
  }
}

// Warp-wide: the tile's group ORs, sub-tile masks and tile mask (kernel.py:844-889).
__device__ __forceinline__ TileMasks reduce_masks(const ConvRowGatherArgs &A, const uint32_t (&w)[4]) {
  TileMasks t;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    uint32_t v = w[q];
#pragma unroll
    for (int sh = 16; sh > 0; sh >>= 1) v |= __shfl_xor_sync(0xffffffffu, v, sh);
    t.g[q] = v;
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    uint32_t sq;
    if (A.tile_m_desp == 32) sq = t.g[q];
    else if (A.tile_m_desp == 64) sq = q < 2 ? (t.g[0] | t.g[1]) : (t.g[2] | t.g[3]);
    else sq = t.g[0] | t.g[1] | t.g[2] | t.g[3];
    sq &= A.mask_filter;
    if (A.reverse) sq = __brev(sq) >> (32 - A.kv);
    t.sub[q] = sq;
  }
  uint32_t tm = (t.g[0] | t.g[1] | t.g[2] | t.g[3]) & A.mask_filter;
  if (A.reverse) tm = __brev(tm) >> (32 - A.kv);
  t.tm = tm;
  return t;
}

// The it-th tile of the strand at schedule position pos, or -1 past the end.
// With the largest-first order the positions take the tiles in a snake
// (0 .. nstr-1, then nstr-1 .. 0, ...), so the strand that drew the heaviest
// tile of one round draws the lightest of the next; without it, every nstr-th
// tile.
__device__ __forceinline__ int64_t strand_tile(const KParams &P, int64_t pos, int64_t nstr, int64_t it) {
  if (P.a.tile_order == nullptr) {
    const int64_t d = it * nstr + pos;
    return d < P.num_tiles ? d : -1;
  }
  const int64_t d = it * nstr + ((it & 1) ? nstr - 1 - pos : pos);
  return d < P.num_tiles ? scheduled_tile(P.a, d) : -1;
}

template <bool kF8, typename TOut, bool kWide>
__global__ void __maxnreg__(72) conv_strand_kernel(const __grid_constant__ KParams P) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw_u32 = smem_u32(smem_raw);
  const uint32_t pad = (1024u - (raw_u32 & 1023u)) & 1023u;
  uint8_t *smem = smem_raw + pad;
  const uint32_t smem_base = raw_u32 + pad;
  const ConvRowGatherArgs &A = P.a;
  // kWide: 128-byte rows (SWIZZLE_128B), two 24 KB stages per strand; else
  // 64-byte rows (SWIZZLE_64B), four 12 KB stages
  constexpr int S = kWide ? 2 : 4;
  constexpr int rb = kWide ? 128 : 64;
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + P.bar_off);
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + kStrands * kSBars);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);
  volatile int *acc_tile = abort_flag + 1;  // [kStrands][2]: tile held by accumulator buffer

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStrands; ++s) {
      uint64_t *b = bars + s * kSBars;
      for (int i = 0; i < S; ++i) {
        mbar_init(&b[i], kSProd);  // full: one arrive.expect_tx per producer warp
        mbar_init(&b[S + i], 1);   // empty: the MMA commit
      }
      mbar_init(&b[2 * S + 0], 1);    // acc_full[0]
      mbar_init(&b[2 * S + 1], 1);    // acc_full[1]
      mbar_init(&b[2 * S + 2], 128);  // acc_empty[0]
      mbar_init(&b[2 * S + 3], 128);  // acc_empty[1]
      mbar_init(&b[2 * S + 4], 1);    // tile_bar[0]
      mbar_init(&b[2 * S + 5], 1);    // tile_bar[1]
      mbar_init(&b[2 * S + 6], 1);    // drain
    }
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 0) {
    tmem_alloc(tmem_slot, kSTmemCols);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  const int64_t nstr = static_cast<int64_t>(gridDim.x) * kStrands;

  if (warp >= kEpiWarps) {
    const int sw = warp - kEpiWarps;
    const int s = sw / (kSProd + 1);
    const int role = sw % (kSProd + 1);  // < kSProd: producer warp, kSProd: MMA warp
    uint64_t *full = bars + s * kSBars;
    uint64_t *empty = full + S;
    uint64_t *acc_full = full + 2 * S;
    uint64_t *acc_empty = acc_full + 2;
    uint64_t *tile_bar = acc_full + 4;
    uint64_t *drain_bar = acc_full + 6;
    // this strand's position in the schedule: consecutive positions sit on
    // consecutive CTAs (so on different SMs)
    const int64_t pos = static_cast<int64_t>(s) * gridDim.x + blockIdx.x;
    const uint32_t ring = smem_base + static_cast<uint32_t>(s * S) * P.stage_bytes;
    uint32_t w[4] = {0u, 0u, 0u, 0u};
    {
      const int64_t t0 = strand_tile(P, pos, nstr, 0);
      if (t0 >= 0) load_mask_words(A, t0 / A.n_tiles, lane, w);
    }
    if (role < kSProd) {
      // ---------------------------------------------------------------- producers
      // Warp pw gathers rows [32 pw, 32 pw + 32) of every chunk: lanes 0-7
      // each take the four sorted indices of their rows for the chunk's
      // offset (gated by the row group's sub-tile mask; rows past M read as
      // -1) and issue one tile::gather4.  The warp whose turn it is adds the
      // weight slab.  A cursor runs two chunks ahead of the chunk being
      // issued and loads their indices, so an index load's latency overlaps
      // the two chunks before it.
      const int pw = role;
      const int esz = kF8 ? 1 : 2;
      const int box = rb / esz;
      const uint32_t a_tx = 32u * static_cast<uint32_t>(rb);
      const uint32_t b_tx = static_cast<uint32_t>(A.BN) * static_cast<uint32_t>(rb);
      const int r0 = pw * 32 + lane * 4;
      // cursor (warp-uniform): tile (the strand's c_it-th), offsets not
      // started yet, current offset / column block
      int64_t c_it = -1, c_tile = -1, c_tile_m = 0;
      uint32_t c_mm = 0u, c_sub = 0u;
      int c_k = 0, c_cb = 0, c_n0 = 0;
      bool c_valid = true;
      // enters the following tiles until one visits an offset (writing
      // mask_output for each tile entered)
      auto next_tile = [&]() {
        for (;;) {
          c_tile = strand_tile(P, pos, nstr, ++c_it);
          if (c_tile < 0) {
            c_valid = false;
            return;
          }
          const TileMasks t = reduce_masks(A, w);
          const int64_t t_next = strand_tile(P, pos, nstr, c_it + 1);
          if (t_next >= 0) load_mask_words(A, t_next / A.n_tiles, lane, w);
          c_tile_m = c_tile / A.n_tiles;
          const int n_tile = static_cast<int>(c_tile % A.n_tiles);
          c_n0 = n_tile * A.BN;
          if (pw == 0 && lane == 0 && A.is_fwd && A.mask_out != nullptr && n_tile == 0) {
            const int nsub = kTileM / A.tile_m_desp;
            for (int d = 0; d < nsub; ++d) {
              const int64_t start = c_tile_m * kTileM + d * A.tile_m_desp;
              if (start >= A.M) break;
              uint32_t wd;
              if (nsub == 4) wd = t.g[d];
              else if (nsub == 2) wd = d == 0 ? (t.g[0] | t.g[1]) : (t.g[2] | t.g[3]);
              else wd = t.g[0] | t.g[1] | t.g[2] | t.g[3];
              A.mask_out[start / A.tile_m_desp] = wd & A.mask_filter;
            }
          }
          // rows of lanes 0-7 lie in 32-row group pw
          c_sub = pw == 0 ? t.sub[0] : pw == 1 ? t.sub[1] : pw == 2 ? t.sub[2] : t.sub[3];
          if (t.tm != 0u) {
            c_k = __ffs(t.tm) - 1;
            c_mm = t.tm & (t.tm - 1u);
            c_cb = 0;
            return;
          }
        }
      };
      auto advance = [&]() {
        if (++c_cb < P.cpo) return;
        c_cb = 0;
        if (c_mm != 0u) {
          c_k = __ffs(c_mm) - 1;
          c_mm &= c_mm - 1u;
          return;
        }
        next_tile();
      };
      // this lane's four indices of the cursor's chunk (checked when issued,
      // so the load stays in flight until then)
      auto load_q = [&]() {
        int4 q = make_int4(-1, -1, -1, -1);
        const int64_t rg = c_tile_m * kTileM + r0;
        if (lane < 8 && rg < A.M && ((c_sub >> c_k) & 1u))
          q = __ldg(reinterpret_cast<const int4 *>(A.idx_sorted + static_cast<int64_t>(c_k) * A.M + rg));
        return q;
      };
      next_tile();
      // slots 0 (the chunk to issue) and 1 (the next one)
      int4 q0 = make_int4(-1, -1, -1, -1), q1 = q0;
      int k0 = 0, cb0 = 0, n00 = 0, k1 = 0, cb1 = 0, n01 = 0;
      bool v0 = c_valid, v1 = false;
      if (c_valid) {
        q0 = load_q();
        k0 = c_k; cb0 = c_cb; n00 = c_n0;
        advance();
        v1 = c_valid;
        if (c_valid) {
          q1 = load_q();
          k1 = c_k; cb1 = c_cb; n01 = c_n0;
          advance();
        }
      }
      uint32_t stage = 0, eph = 0, gchunk = 0;
      while (v0) {
        // the chunk two ahead: load its indices now
        int4 q2 = make_int4(-1, -1, -1, -1);
        int k2 = 0, cb2 = 0, n02 = 0;
        const bool v2 = c_valid;
        if (v2) {
          q2 = load_q();
          k2 = c_k; cb2 = c_cb; n02 = c_n0;
          advance();
        }
        if (!__all_sync(0xffffffffu, mbar_wait(&empty[stage], eph ^ 1u, abort_flag))) {
          if (lane == 0) flag_error(A.err, kErrWaitTimeout);
          break;
        }
        const uint32_t sA = ring + stage * P.stage_bytes;
        if (lane == 0) {
          if (static_cast<int>(gchunk % kSProd) == pw) {
            mbar_arrive_expect_tx(&full[stage], a_tx + b_tx);
            if (P.b_mn) {
              for (int qq = 0; qq < A.BN / 64; ++qq)
                tma_load_2d(sA + P.b_off + qq * 8192, &P.tmap_b, k0 * (A.b_off_stride / esz) + n00 + 64 * qq,
                            cb0 * 64, &full[stage]);
            } else {
              tma_load_2d(sA + P.b_off, &P.tmap_b, k0 * (A.b_off_stride / esz) + cb0 * box, n00, &full[stage]);
            }
          } else {
            mbar_arrive_expect_tx(&full[stage], a_tx);
          }
        }
        __syncwarp();
        if (lane < 8) {
          if (q0.x < -1 || q0.x >= A.a_rows || q0.y < -1 || q0.y >= A.a_rows || q0.z < -1 || q0.z >= A.a_rows ||
              q0.w < -1 || q0.w >= A.a_rows) {
            flag_error(A.err, kErrBadIndex);
            q0 = make_int4(-1, -1, -1, -1);
          }
          if (P.zero_ok && (q0.x & q0.y & q0.z & q0.w) == -1) {
            const int z = zero_group(blockIdx.x * 64 + warp * 8 + lane, gchunk);
            tma_gather4(sA + r0 * rb, &P.tmap_zero, 0, z, z + 1, z + 2, z + 3, &full[stage]);
          }
          else
            tma_gather4(sA + r0 * rb, &P.tmap_a, cb0 * box, q0.x, q0.y, q0.z, q0.w, &full[stage]);
        }
        ++gchunk;
        if (++stage == static_cast<uint32_t>(S)) {
          stage = 0;
          eph ^= 1u;
        }
        q0 = q1; k0 = k1; cb0 = cb1; n00 = n01; v0 = v1;
        q1 = q2; k1 = k2; cb1 = cb2; n01 = n02; v1 = v2;
      }
    } else {
      // ---------------------------------------------------------------- MMA warp
      const uint64_t b_kstep = P.b_mn ? 128 : 2;
      // 8-row swizzle atoms 1024 bytes apart (SWIZZLE_128B) or 512 (SWIZZLE_64B);
      // one MMA per 32 bytes of K
      constexpr uint32_t sbo = kWide ? 1024u : 512u;
      constexpr uint32_t swz = kWide ? 2u : 4u;
      constexpr int mmas = rb / 32;
      uint32_t stage = 0, fph = 0;
      bool issued = false, ok = true;
      for (int it = 0;; ++it) {
        const int64_t tile = strand_tile(P, pos, nstr, it);
        const bool have = tile >= 0;
        int nch = 0;
        if (have) {
          const TileMasks tmk = reduce_masks(A, w);
          const int64_t t_next = strand_tile(P, pos, nstr, it + 1);
          if (t_next >= 0) load_mask_words(A, t_next / A.n_tiles, lane, w);
          nch = __popc(tmk.tm) * P.cpo;
        }
        if (lane == 0) {
          const int ab = it & 1;
          const uint32_t aph = (it >> 1) & 1;
          if (!mbar_wait(&acc_empty[ab], aph ^ 1u, abort_flag)) {
            flag_error(A.err, kErrWaitTimeout);
            ok = false;
          } else {
            tc_fence_after();
            // announce the buffer's tile to the epilogue; -1 ends it
            acc_tile[s * 2 + ab] = have ? static_cast<int>(tile) : -1;
            mbar_arrive(&tile_bar[ab]);
            if (have) {
              const uint32_t d = tmem_base + static_cast<uint32_t>(s * 128 + ab * A.BN);
              for (int j = 0; j < nch; ++j) {
                if (!mbar_wait(&full[stage], fph, abort_flag)) {
                  flag_error(A.err, kErrWaitTimeout);
                  ok = false;
                  break;
                }
                tc_fence_after();
                const uint32_t sA = ring + stage * P.stage_bytes;
                const uint64_t ad = make_sdesc_l(sA, 16, sbo, swz);
                const uint64_t bd = P.b_mn ? make_sdesc(sA + P.b_off, 8192, 1024)
                                           : make_sdesc_l(sA + P.b_off, 16, sbo, swz);
#pragma unroll
                for (int kk = 0; kk < mmas; ++kk) {
                  if constexpr (kF8)
                    mma_f8(d, ad + static_cast<uint64_t>(kk * 2), bd + static_cast<uint64_t>(kk) * b_kstep, P.idesc,
                           (j | kk) != 0 ? 1u : 0u);
                  else
                    mma_f16(d, ad + static_cast<uint64_t>(kk * 2), bd + static_cast<uint64_t>(kk) * b_kstep, P.idesc,
                            (j | kk) != 0 ? 1u : 0u);
                }
                issued = true;
                mma_commit(&empty[stage]);
                if (++stage == static_cast<uint32_t>(S)) {
                  stage = 0;
                  fph ^= 1u;
                }
              }
              if (ok) {
                if (nch == 0) mbar_arrive(&acc_full[ab]);
                else mma_commit(&acc_full[ab]);
              }
            }
          }
        }
        ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
        if (!ok || !have) break;
      }
      if (lane == 0 && issued) {
        // no tcgen05.mma may be in flight when TMEM is released
        mma_commit(drain_bar);
        int never = 0;
        if (!mbar_wait(drain_bar, 0, reinterpret_cast<volatile int *>(&never))) flag_error(A.err, kErrWaitTimeout);
      }
    }
  } else {
    // ---------------------------------------------------------------- epilogue (warps 0-3)
    // Takes the strands' accumulators in turn; thread r owns TMEM lane r (tile row r).
    const int r = threadIdx.x;
    const uint32_t lane_base = static_cast<uint32_t>(warp * 32) << 16;
    int its[kStrands];
    bool done[kStrands];
    for (int s = 0; s < kStrands; ++s) {
      its[s] = 0;
      done[s] = false;
    }
    int n_done = 0;
    bool ok = true;
    while (n_done < kStrands && ok) {
      for (int s = 0; s < kStrands && ok; ++s) {
        if (done[s]) continue;
        uint64_t *acc_full = bars + s * kSBars + 2 * S;
        uint64_t *acc_empty = acc_full + 2;
        uint64_t *tile_bar = acc_full + 4;
        const int ab = its[s] & 1;
        const uint32_t aph = (its[s] >> 1) & 1;
        if (!mbar_wait(&tile_bar[ab], aph, abort_flag)) {
          flag_error(A.err, kErrWaitTimeout);
          ok = false;
          break;
        }
        const int tile = acc_tile[s * 2 + ab];
        if (tile < 0) {
          done[s] = true;
          ++n_done;
          continue;
        }
        const int64_t tile_m = tile / A.n_tiles;
        const int n0 = static_cast<int>(tile % A.n_tiles) * A.BN;
        const int64_t row_g = tile_m * kTileM + r;
        const bool valid = row_g < A.M;
        int sig = valid ? (A.argsort ? __ldg(A.argsort + row_g) : static_cast<int>(row_g)) : -1;
        if (sig >= A.out_rows) sig = -1;
        uint32_t km = 0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int64_t rr = tile_m * kTileM + q * 32 + lane;
          if (rr < A.M) km |= A.mask ? __ldg(A.mask + rr) : 1u;
        }
#pragma unroll
        for (int sh = 16; sh > 0; sh >>= 1) km |= __shfl_xor_sync(0xffffffffu, km, sh);
        km &= A.mask_filter;
        if (!mbar_wait(&acc_full[ab], aph, abort_flag)) {
          flag_error(A.err, kErrWaitTimeout);
          ok = false;
          break;
        }
        tc_fence_after();
        const bool write = valid && sig >= 0 && (A.is_fwd || km != 0);
        const uint32_t tbase = tmem_base + lane_base + static_cast<uint32_t>(s * 128 + ab * A.BN);
        for (int cc = 0; cc < A.BN; cc += 16) {
          float acc[16];
          if (km != 0) {
            tmem_ld16(tbase + cc, acc);
          } else {
#pragma unroll
            for (int i = 0; i < 16; ++i) acc[i] = 0.f;
          }
          if (write) epilogue_cols<16, TOut>(P, acc, sig, n0 + cc);
        }
        tc_fence_before();
        mbar_arrive(&acc_empty[ab]);
        ++its[s];
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem_base, kSTmemCols);
  }
}

template <bool kF8, typename TOut>
cudaError_t launch_strands(const KParams &P, int grid, size_t smem, cudaStream_t stream) {
  void (*kern)(KParams) = P.row_bytes == 128 ? conv_strand_kernel<kF8, TOut, true>
                                             : conv_strand_kernel<kF8, TOut, false>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  kern<<<grid, kSThreads, smem, stream>>>(P);
  return cudaGetLastError();
}

template <bool kF8, typename TOut>
cudaError_t launch_typed(const KParams &P, bool tma, bool gather, bool pair, int grid, size_t smem,
                         cudaStream_t stream) {
  void (*kern)(KParams) =
      gather ? (pair ? conv_rowgather_kernel<kF8, TOut, true, true, true>
                     : conv_rowgather_kernel<kF8, TOut, true, true, false>)
      : tma  ? conv_rowgather_kernel<kF8, TOut, true, false, false>
             : conv_rowgather_kernel<kF8, TOut, false, false, false>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  kern<<<grid, pair ? Layout<true>::kThreads : Layout<false>::kThreads, smem, stream>>>(P);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_tile_order(const uint32_t *mask, int64_t M, uint32_t filter, int reverse, int kv,
                              int *head, int32_t *tile_pc, int32_t *order, cudaStream_t stream) {
  const int64_t m_tiles = (M + kTileM - 1) / kTileM;
  if (m_tiles == 0) return cudaSuccess;
  const int64_t blocks = (m_tiles + kOrderWarps - 1) / kOrderWarps;
  tile_order_kernel<<<static_cast<unsigned>(blocks), kOrderWarps * 32, 0, stream>>>(
      mask, M, filter, reverse, kv, m_tiles, head, tile_pc, order);
  return cudaGetLastError();
}

namespace {
// Zeroes the row-gather kernel's tile counter (the strand kernel has none).
cudaError_t prepare_schedule(const ConvRowGatherArgs &a, bool counter, cudaStream_t stream) {
  if (!counter || a.tile_counter == nullptr) return cudaSuccess;
  return cudaMemsetAsync(a.tile_counter, 0, sizeof(int), stream);
}
}  // namespace

cudaError_t launch_conv_rowgather(const ConvRowGatherArgs &a, int num_sms, cudaStream_t stream) {
  KParams P;
  P.a = a;
  const int64_t m_tiles = (a.M + kTileM - 1) / kTileM;
  P.a.m_tiles = static_cast<int>(m_tiles);
  P.num_tiles = m_tiles * a.n_tiles;
  const int esz = a.in_dtype == 14 ? 1 : 2;
  const uint64_t red = static_cast<uint64_t>(a.a_row_bytes) / esz;
  // 64-byte rows (C = 64 e4m3, C = 32 bf16 / f16): one offset per stage in
  // SWIZZLE_64B layout, filled by TMA gather4 like the 128-byte case, when
  // both tensor maps encode; otherwise offsets are packed into 128-byte rows
  // and filled with cp.async
  bool tma = false, gather = false;
  P.row_bytes = 128;
  P.bulk_idx = a.idx_sorted != nullptr && reinterpret_cast<uintptr_t>(a.idx_sorted) % 16 == 0 &&
               a.M % 4 == 0;
  if (a.a_row_bytes == 64 && a.kv > 1 && a.a_rows > 0 &&
      encode_tmap_2d(&P.tmap_b, a.in_dtype, a.b_base, red * a.kv, a.n_total,
                     static_cast<uint64_t>(a.b_row_stride), 64u / esz, a.BN, 64) &&
      encode_tmap_2d(&P.tmap_a, a.in_dtype, a.a_base, red, static_cast<uint64_t>(a.a_rows),
                     static_cast<uint64_t>(a.a_row_stride), 64u / esz, 1, 64)) {
    tma = gather = true;
    P.row_bytes = 64;
    P.cpo = 1;
    P.opc = 1;
    P.upo = 4;
  } else if (a.a_row_bytes >= 128 || a.kv == 1) {
    P.cpo = (a.a_row_bytes + 127) / 128;
    P.opc = 1;
    P.upo = 8;
  } else {
    P.cpo = 0;
    P.opc = 128 / a.a_row_bytes;
    P.upo = a.a_row_bytes / 16;
  }
  // TMA weight slabs: whole 128-byte reduction chunks (no packing of small offsets)
  P.b_mn = a.b_mn;
  if (P.cpo > 0 && P.row_bytes == 128) {
    const uint32_t box = 128u / esz;
    // MN-major weight: [red rows, kv * n_total columns], 64 x 64 boxes
    tma = a.b_mn ? encode_tmap_2d(&P.tmap_b, a.in_dtype, a.b_base,
                                  static_cast<uint64_t>(a.n_total) * a.kv, red,
                                  static_cast<uint64_t>(a.b_row_stride), 64, 64)
                 : encode_tmap_2d(&P.tmap_b, a.in_dtype, a.b_base, red * a.kv, a.n_total,
                                  static_cast<uint64_t>(a.b_row_stride), box, a.BN);
    // gathered A rows: [a_rows, red] with one-row boxes (tile::gather4)
    if (tma && a.a_row_bytes >= 128 && a.a_rows > 0)
      gather = encode_tmap_2d(&P.tmap_a, a.in_dtype, a.a_base, red, static_cast<uint64_t>(a.a_rows),
                              static_cast<uint64_t>(a.a_row_stride), box, 1);
  }
  // zero rows with the same box and swizzle as the gathered rows
  P.zero_ok = 0;
  if (gather) {
    const void *z = zero_rows_address();
    const uint32_t zbox = static_cast<uint32_t>(P.row_bytes) / esz;
    P.zero_ok = z != nullptr && encode_tmap_2d(&P.tmap_zero, a.in_dtype, z, zbox, kZeroRows,
                                               static_cast<uint64_t>(P.row_bytes), zbox, 1, P.row_bytes)
                    ? 1 : 0;
  }
  // the MN-major weight slab is only read by the TMA gather path
  if (a.b_mn && (!gather || a.BN % 64 != 0 || esz != 2)) return cudaErrorInvalidConfiguration;
  const uint32_t a_bytes = kTileM * static_cast<uint32_t>(P.row_bytes);
  const uint32_t b_bytes = static_cast<uint32_t>(a.BN) * P.row_bytes;
  P.stage_bytes = a_bytes + b_bytes;
  P.b_off = a_bytes;
  // Strands (two independent pipelines per CTA, two CTAs per SM) on the TMA
  // gather path of 128-byte rows with the sorted index table and BN <= 64
  // (TMEM: 2 strands x 2 buffers x BN columns per CTA).
  if (gather && P.bulk_idx && a.BN <= 64 && !(P.row_bytes == 64 && a.b_mn)) {
    if (P.num_tiles == 0) return cudaSuccess;
    // two CTAs per SM (113 KB each): two stages per strand with 128-byte rows
    // (24 KB at BN 64), four with 64-byte rows (12 KB)
    const int stages = P.row_bytes == 128 ? 2 : 4;
    P.stages = stages;
    P.tmem_cols = kSTmemCols;
    P.bar_off = P.stage_bytes * kStrands * stages;
    const size_t smem = 1024 + P.bar_off + 512;
    const int64_t ctas = (P.num_tiles + kStrands - 1) / kStrands;
    const int grid = static_cast<int>(ctas < 2 * num_sms ? ctas : 2 * num_sms);
    {
      const cudaError_t e = prepare_schedule(a, false, stream);
      if (e != cudaSuccess) return e;
    }
    if (a.in_dtype == 14) {
      P.idesc = make_idesc(128, a.BN, 0u, false, false);
      switch (a.out_dtype) {
        case 0: return launch_strands<true, float>(P, grid, smem, stream);
        case 7: return launch_strands<true, __half>(P, grid, smem, stream);
        default: return launch_strands<true, __nv_bfloat16>(P, grid, smem, stream);
      }
    }
    P.idesc = make_idesc(128, a.BN, a.in_dtype == 12 ? 1u : 0u, false, a.b_mn != 0);
    switch (a.out_dtype) {
      case 0: return launch_strands<false, float>(P, grid, smem, stream);
      case 7: return launch_strands<false, __half>(P, grid, smem, stream);
      case 12: return launch_strands<false, __nv_bfloat16>(P, grid, smem, stream);
      default: return cudaErrorInvalidValue;
    }
  }
  P.idx_buf_bytes = ((static_cast<uint32_t>(a.kv) * kTileM * 4 + sizeof(Meta)) + 127u) & ~127u;
  uint32_t cols = 32;
  while (cols < static_cast<uint32_t>(2 * a.BN)) cols <<= 1;
  P.tmem_cols = cols;
  const uint32_t bar_bytes = 512;
  // dynamic shared memory of one CTA: 227 KB alone on an SM, 113 KB for two
  // per SM; 1 KB of it is slack for the 1024-byte alignment of the stages
  auto stages_for = [&](uint32_t limit, int idx_stages) {
    const int64_t budget = static_cast<int64_t>(limit) - 1024 - P.idx_buf_bytes * idx_stages - bar_bytes;
    const int64_t st = budget / P.stage_bytes;
    return static_cast<int>(st > 8 ? 8 : st);
  };
  const uint32_t kLimitSingle = 227u * 1024u, kLimitPair = 113u * 1024u;
  // two CTAs per SM on the gather path when both fit (TMEM: 2 x 2 BN columns)
  // with at least 3 stages each
  const bool pair = gather && cols <= 256 && stages_for(kLimitPair, Layout<true>::kIdxStages) >= 3;
  const int idx_stages = pair ? Layout<true>::kIdxStages : Layout<false>::kIdxStages;
  const int stages = stages_for(pair ? kLimitPair : kLimitSingle, idx_stages);
  if (stages < 2) return cudaErrorInvalidConfiguration;
  P.stages = stages;
  P.idx_off = P.stage_bytes * stages;
  P.bar_off = P.idx_off + P.idx_buf_bytes * idx_stages;
  const size_t smem = 1024 + P.bar_off + bar_bytes;
  if (P.num_tiles == 0) return cudaSuccess;
  {
    const cudaError_t e = prepare_schedule(a, true, stream);
    if (e != cudaSuccess) return e;
  }
  const int64_t ctas = static_cast<int64_t>(pair ? 2 : 1) * num_sms;
  const int grid = static_cast<int>(P.num_tiles < ctas ? P.num_tiles : ctas);
  if (a.in_dtype == 14) {
    P.idesc = make_idesc(128, a.BN, 0u, false, false);
    switch (a.out_dtype) {
      case 0: return launch_typed<true, float>(P, tma, gather, pair, grid, smem, stream);
      case 7: return launch_typed<true, __half>(P, tma, gather, pair, grid, smem, stream);
      default: return launch_typed<true, __nv_bfloat16>(P, tma, gather, pair, grid, smem, stream);
    }
  }
  P.idesc = make_idesc(128, a.BN, a.in_dtype == 12 ? 1u : 0u, false, a.b_mn != 0);
  switch (a.out_dtype) {
    case 0: return launch_typed<false, float>(P, tma, gather, pair, grid, smem, stream);
    case 7: return launch_typed<false, __half>(P, tma, gather, pair, grid, smem, stream);
    case 12: return launch_typed<false, __nv_bfloat16>(P, tma, gather, pair, grid, smem, stream);
    default: break;
  }
  return cudaErrorInvalidValue;
}

}  // namespace scb
