// conv_wgrad.cu - mask-implicit-GEMM sparse convolution, backward-weight, on
// sm_100a tensor cores.
//
// Semantics follow the reference's wgrad path (cumm/gemm/blockmma/mma.py:580-765,
// cumm/conv/sparse_iters.py:284-316, cumm/conv/kernel.py:890-897):
//   dW[:, k, :] = sum over sorted rows r whose reduced mask word
//                 mask[r / mask_width] has bit k (and k in mask_filter) of
//                 dOut[sigma(r)]^T x In[indices[k][sigma(r)]]
// with sigma = mask_argsort and In rows of index -1 contributing zero.
// Offsets outside mask_filter are left untouched (kernel.py:893-896).
//
// B200 design: the reduction runs over gathered rows, so both operands are
// staged MN-major: a 64-row chunk of gathered input rows (two 128-byte atoms =
// 128 MN-elements: one or more filters' channels) is the M side and the
// matching 64 dOut rows are the N side.  Every CTA owns a group of M-tiles
// (up to 512 TMEM columns of fp32 accumulators) and every splits-th row
// chunk; TMEM accumulates over the whole range, and the epilogue adds the
// CTA's partial dW into an fp32 workspace with red.global.add.v4.f32 (split
// over rows without a serial semaphore, so there is no inter-CTA spin).  A
// finalize kernel applies alpha/beta and converts to the weight dtype.
// Warp roles: epilogue, producers (TMA tile::gather4 of the input rows per
// stage and of the chunk's dOut rows once per chunk when rows are whole
// 128-byte blocks, 16-byte cp.async otherwise), index loaders, and one TMEM
// allocator + tcgen05.mma issuer.  On the gather path with 64 dOut columns
// two 11-warp CTAs share an SM (M-tile groups of <= 256 TMEM columns);
// otherwise one 17-warp CTA per SM (Layout below).
#include <cuda.h>

#include "kernels.h"

namespace scb {
namespace {

// Two layouts.  Single (one CTA per SM, 17 warps, 96 registers): warps 0-3
// epilogue, 4-11 producers, 12-15 index loaders (one row and one filter
// parity per thread), 16 MMA; index tables of up to 32 filters.  Pair (two
// CTAs per SM, 11 warps each, 80 registers; gather path with 64 dOut columns
// and M-tile groups of <= 4 tiles = 256 TMEM columns): warps 0-3 epilogue,
// 4-7 producers, 8-9 index loaders (one row, every filter of the group per
// thread), 10 MMA; index tables of 8 filters.  The TMA gather rate is per
// issuing CTA, so two CTAs on an SM gather faster than one.
constexpr int kEpiWarps = 4;     // warps 0-3 in both layouts
constexpr int kProdWarp0 = 4;
template <bool kPair> struct Layout {
  static constexpr int kProdWarps = kPair ? 4 : 8;
  static constexpr int kLoadWarp0 = kProdWarp0 + kProdWarps;
  static constexpr int kLoadWarps = kPair ? 2 : 4;
  static constexpr int kMmaWarp = kLoadWarp0 + kLoadWarps;
  static constexpr int kThreads = (kMmaWarp + 1) * 32;
  static constexpr int kTabF = kPair ? 8 : 32;  // filters of an index table
  // index loader thread: filters k_lo + par + kFStride q (q < kNQ), par being
  // the thread's filter parity in the single layout
  static constexpr int kFStride = kPair ? 1 : 2;
  static constexpr int kNQ = kPair ? 8 : 16;
};
constexpr int kIdxStages = 4;
constexpr int kMaxBBufs = 4;  // dOut buffers of the gather path (2 or 4 per launch)
constexpr int kRows = 64;  // reduction rows per stage

struct WMeta {
  int n_active;
  uint32_t active_bits;  // bit j -> M-tile t0 + j active for this chunk
  uint32_t grp[4];
};
__host__ __device__ constexpr uint32_t kScratchOff(int tab_f) {
  return static_cast<uint32_t>(((tab_f * kRows + kRows) * 4 + sizeof(WMeta) + 15) & ~15u);
}

struct WParams {
  CUtensorMap tmap_in;    // input rows [in_rows, C], one-row boxes (gather path)
  CUtensorMap tmap_dout;  // dOut rows [dout_rows, K], one-row boxes (gather path)
  CUtensorMap tmap_zero;  // four zero rows: gathers whose rows are all -1 read these
  int zero_ok;
  ConvWgradArgs a;
  int n_chunks;        // ceil(N / 64)
  int chunks_per_cta;
  int n_groups;
  int tiles_per_group;
  int n_mtiles;
  int n_atoms;
  int cpa;             // 64-element c-blocks per filter (C >= 64), else 0
  int fpa;             // filters per atom (C < 64)
  int upf;             // 16-byte units per filter segment (C < 64)
  int n_mma;           // MMA N (K rounded up to 64)
  int mw_shift;        // log2(mask_width) when it is a power of two, else -1
  int stages;
  uint32_t stage_bytes;
  uint32_t b_off;
  uint32_t bbuf_off;      // gather path: n_bbuf dOut buffers of n_b_atoms x 8 KB
  uint32_t n_bbuf;
  uint32_t idx_off;
  uint32_t idx_buf_bytes;
  uint32_t bar_off;
  uint32_t tmem_cols;
  uint32_t idesc;
};

__device__ __forceinline__ void flag_error(int *err, int bits) { atomicOr(err, bits); }

// Four consecutive fp32 atomic adds (address 16-byte aligned).
__device__ __forceinline__ void red_add_v4(float *p, float a, float b, float c, float d) {
  asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(a), "f"(b), "f"(c),
               "f"(d)
               : "memory");
}

// Filter and channel of element e (0..63) of atom a.
__device__ __forceinline__ void atom_elem(const WParams &P, int a, int e, int &k, int &c) {
  if (P.cpa > 0) {
    k = a / P.cpa;
    c = (a % P.cpa) * 64 + e;
  } else {
    const int C = P.a.C;
    k = a * P.fpa + e / C;
    c = e % C;
  }
}

// M-tiles of group g: n_mtiles / n_groups each, and the remainder goes to
// the outer groups first (0, last, 1, last - 1, ...).  The middle offsets of
// a kernel carry the most pairs (a submanifold conv's centre and, on surfaces,
// its in-plane neighbours), so the middle groups get fewer tiles: 14 tiles in
// 4 groups are 4 + 3 + 3 + 4, not 4 + 4 + 4 + 2.  No group exceeds
// tiles_per_group (the TMEM columns of a CTA).
__device__ __forceinline__ void group_filters(const WParams &P, int g, int &k_lo, int &k_hi,
                                              int &t0, int &t1) {
  const int n = P.n_groups;
  const int base = P.n_mtiles / n, rem = P.n_mtiles % n;
  auto size = [&](int q) {
    const int m = n - 1 - q;
    const int rank = q < m ? 2 * q : 2 * m + 1;  // order 0, n-1, 1, n-2, ...
    return base + (rank < rem ? 1 : 0);
  };
  int s = 0;
  for (int q = 0; q < g; ++q) s += size(q);
  t0 = s;
  t1 = min(s + size(g), P.n_mtiles);
  const int a0 = 2 * t0;
  const int a1 = min(2 * t1, P.n_atoms);  // exclusive
  if (P.cpa > 0) {
    k_lo = a0 / P.cpa;
    k_hi = (a1 - 1) / P.cpa + 1;
  } else {
    k_lo = a0 * P.fpa;
    k_hi = min(a1 * P.fpa, P.a.kv);
  }
}

// Filter range covered by M-tile t.
__device__ __forceinline__ uint32_t tile_filter_bits(const WParams &P, int t) {
  const int a0 = 2 * t;
  const int a1 = min(2 * t + 2, P.n_atoms);
  int lo, hi;
  if (P.cpa > 0) {
    lo = a0 / P.cpa;
    hi = (a1 - 1) / P.cpa + 1;
  } else {
    lo = a0 * P.fpa;
    hi = min(a1 * P.fpa, P.a.kv);
  }
  const uint32_t upto_hi = hi >= 32 ? 0xffffffffu : ((1u << hi) - 1u);
  return upto_hi & ~((1u << lo) - 1u);
}

// Registers: single 17 warps (5 per SM sub-partition) x 96; pair 2 x 11 warps
// (6 per sub-partition) x 80 = 15360 of a sub-partition's 16384.
template <bool kGather, bool kPair>
__global__ void __maxnreg__(kPair ? 80 : 96) conv_wgrad_kernel(const __grid_constant__ WParams P) {
  constexpr int kProdWarps = Layout<kPair>::kProdWarps;
  constexpr int kLoadWarp0 = Layout<kPair>::kLoadWarp0;
  constexpr int kLoadWarps = Layout<kPair>::kLoadWarps;
  constexpr int kMmaWarp = Layout<kPair>::kMmaWarp;
  constexpr int kTabF = Layout<kPair>::kTabF;
  constexpr int kFStride = Layout<kPair>::kFStride;
  constexpr int kNQ = Layout<kPair>::kNQ;
  // producer rings: the pair layout's epilogue warps are the second ring's
  // producers until the mainloop ends
  constexpr int kRings = kPair ? 2 : 1;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw_u32 = smem_u32(smem_raw);
  const uint32_t pad = (1024u - (raw_u32 & 1023u)) & 1023u;
  uint8_t *smem = smem_raw + pad;
  const uint32_t smem_base = raw_u32 + pad;
  const ConvWgradArgs &A = P.a;

  const int S = P.stages;
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + P.bar_off);
  uint64_t *full_bar = bars;
  uint64_t *empty_bar = bars + S;
  uint64_t *idx_full = bars + 2 * S;
  uint64_t *idx_empty = idx_full + kIdxStages;
  uint64_t *acc_full = idx_empty + kIdxStages;
  uint64_t *drain_bar = acc_full + 1;
  uint64_t *bfull = drain_bar + 1;   // gather path: dOut buffer b loaded
  uint64_t *bempty = bfull + kMaxBBufs;  // gather path: dOut buffer b consumed
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bempty + kMaxBBufs);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);
  uint32_t *used_tiles = reinterpret_cast<uint32_t *>(tmem_slot + 2);
  uint32_t *tile_fbits = used_tiles + 1;  // [16]: filters of M-tile t0 + j

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int g = blockIdx.y;
  int k_lo, k_hi, t0, t1;
  group_filters(P, g, k_lo, k_hi, t0, t1);
  // chunks are dealt round-robin (c = x, x + splits, ...): rows are sorted by
  // mask, so contiguous ranges would give some CTAs only the dense chunks
  const int c_begin = blockIdx.x;
  const int c_end = P.n_chunks;
  const int c_step = gridDim.x;

  if (threadIdx.x == 0) {
    for (int i = 0; i < S; ++i) {
      // gather: one arrive.expect_tx per producer warp; cp.async: the 32
      // lanes of the stage's producer warp (cp.async.mbarrier.arrive.noinc)
      mbar_init(&full_bar[i], kGather ? kProdWarps : 32);
      mbar_init(&empty_bar[i], 1);
    }
    for (int i = 0; i < kIdxStages; ++i) {
      mbar_init(&idx_full[i], kLoadWarps * 32);
      mbar_init(&idx_empty[i], (kGather ? kProdWarps : min(S, kProdWarps)) + 1);
    }
    mbar_init(acc_full, 1);
    mbar_init(drain_bar, 1);
    for (int i = 0; i < kMaxBBufs; ++i) {
      mbar_init(&bfull[i], kProdWarps);
      mbar_init(&bempty[i], 1);
    }
    *abort_flag = 0;
    *used_tiles = 0;
    for (int j = 0; j < 16; ++j) tile_fbits[j] = t0 + j < t1 ? tile_filter_bits(P, t0 + j) : 0u;
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

  // ---------------------------------------------------------------- TMA gather producer loop
  // Producer warps of ring `ring` serve every stage of that ring: warp pw
  // owns rows [kRpw pw, kRpw pw + kRpw) of each 64-row atom; lane l < 2 kGpw
  // issues one tile::gather4 for rows kRpw pw + 4 (l % kGpw) .. +3 of atom
  // l / kGpw (input rows of the atom's filter; a group of four absent rows
  // reads the zero tensor).  The chunk's 64 dOut rows are the same for every
  // M-tile, so they are gathered once per chunk into one of the ring's dOut
  // buffers (lanes l < kGpw n_b_atoms, same row split), released by the MMA
  // after the chunk's last tile.  Lane 0 of each warp arrives with
  // expect_tx for its bytes.  With two rings (pair layout) ring r takes the
  // CTA's chunks it = r, r + 2, ... (index buffers it % 4: 0 and 2 for ring
  // 0, 1 and 3 for ring 1), and owns half of the stages and dOut buffers.
  auto produce_gather = [&](int pw, int ring) {
    constexpr int kRpw = kRows / kProdWarps;  // rows per warp: 8 single, 16 pair
    constexpr int kGpw = kRpw / 4;            // gathers per atom per warp
    const int n_b_atoms = P.n_mma / 64;
    const uint32_t Sr = static_cast<uint32_t>(S / kRings);
    const uint32_t NBr = P.n_bbuf / kRings;
    const int rq = pw * kRpw + (lane % kGpw) * 4;
    uint32_t stage = 0, eph = 0, bb = 0, bph = 0;  // this ring's stage / dOut buffer and phases
    bool ok = true;
    int it = ring;
    for (int c = c_begin + ring * c_step; c < c_end && ok; c += kRings * c_step, it += kRings) {
      const int b = it % kIdxStages;
      const uint32_t ph = (it / kIdxStages) & 1;
      if (!__all_sync(0xffffffffu, mbar_wait(&idx_full[b], ph, abort_flag))) {
        if (lane == 0) flag_error(A.err, kErrWaitTimeout);
        break;
      }
      const uint8_t *buf = smem + P.idx_off + b * P.idx_buf_bytes;
      const int *tab = reinterpret_cast<const int *>(buf);
      const int *sig_tab = tab + kTabF * kRows;
      const WMeta *meta = reinterpret_cast<const WMeta *>(sig_tab + kRows);
      uint32_t bits = meta->active_bits;
      if (bits) {
        const uint32_t bi = static_cast<uint32_t>(ring) * NBr + bb;
        if (!__all_sync(0xffffffffu, mbar_wait(&bempty[bi], bph ^ 1u, abort_flag))) {
          if (lane == 0) flag_error(A.err, kErrWaitTimeout);
          break;
        }
        if (lane == 0) mbar_arrive_expect_tx(&bfull[bi], static_cast<uint32_t>(n_b_atoms * kRpw) * 128u);
        __syncwarp();
        if (lane < kGpw * n_b_atoms) {
          const int na = lane / kGpw;
          const int4 q = *reinterpret_cast<const int4 *>(sig_tab + rq);
          const uint32_t dst = smem_base + P.bbuf_off + bi * (n_b_atoms * 8192u) + na * 8192u + rq * 128;
          if (P.zero_ok && (q.x & q.y & q.z & q.w) == -1) {
            const int z = zero_group(blockIdx.x * 64 + pw * 8 + lane, static_cast<uint32_t>(it));
            tma_gather4(dst, &P.tmap_zero, 0, z, z + 1, z + 2, z + 3, &bfull[bi]);
          }
          else
            tma_gather4(dst, &P.tmap_dout, na * 64, q.x, q.y, q.z, q.w, &bfull[bi]);
        }
        if (++bb == NBr) {
          bb = 0;
          bph ^= 1u;
        }
      }
      while (bits) {
        const int jt = __ffs(bits) - 1;
        bits &= bits - 1;
        const int tt = t0 + jt;
        const uint32_t s = static_cast<uint32_t>(ring) * Sr + stage;
        if (!__all_sync(0xffffffffu, mbar_wait(&empty_bar[s], eph ^ 1, abort_flag))) {
          if (lane == 0) flag_error(A.err, kErrWaitTimeout);
          ok = false;
          break;
        }
        if (++stage == Sr) {
          stage = 0;
          eph ^= 1u;
        }
        if (lane == 0) mbar_arrive_expect_tx(&full_bar[s], 2u * kRpw * 128u);
        __syncwarp();
        if (lane < 2 * kGpw) {
          const int a = 2 * tt + lane / kGpw;
          const int k = a / P.cpa;
          int4 q = make_int4(-1, -1, -1, -1);
          if (a < P.n_atoms && k < A.kv)
            q = *reinterpret_cast<const int4 *>(tab + (k - k_lo) * kRows + rq);
          const uint32_t dst = smem_base + s * P.stage_bytes + (lane / kGpw) * 8192u + rq * 128;
          if (P.zero_ok && (q.x & q.y & q.z & q.w) == -1) {
            const int z = zero_group(blockIdx.x * 64 + pw * 8 + lane, s + static_cast<uint32_t>(it));
            tma_gather4(dst, &P.tmap_zero, 0, z, z + 1, z + 2, z + 3, &full_bar[s]);
          }
          else
            tma_gather4(dst, &P.tmap_in, (a % P.cpa) * 64, q.x, q.y, q.z, q.w, &full_bar[s]);
        }
      }
      if (!ok) break;
      __syncwarp();
      if (lane == 0) mbar_arrive(&idx_empty[b]);
    }
  };

  // ---------------------------------------------------------------- dW reduction
  // TMEM lane m holds M element m of every tile; the warp that reads lane
  // quadrant q (lanes 32 q .. 32 q + 31) turns its 32 lanes x 32 columns
  // through a private shared-memory tile (the stage buffers are idle once the
  // MMA warp drained), so that a lane then owns 4 consecutive channels of one
  // column and adds them with one red.global.add.v4.f32 (a quarter of the
  // scalar atomics).  It reduces the CTA's used tiles j = j0, j0 + jstep, ...;
  // in the pair layout the epilogue warps take the even tiles and ring 0's
  // producer warps (same quadrants, idle once their ring is done) the odd ones.
  // Only __syncwarp is used: a warp whose wait ran out never strands the others.
  auto reduce_tiles = [&](int q, int j0, int jstep) {
    if (!mbar_wait(acc_full, 0, abort_flag)) {
      flag_error(A.err, kErrWaitTimeout);
      return;
    }
    tc_fence_after();
    const uint32_t used = *reinterpret_cast<volatile uint32_t *>(used_tiles);
    const uint32_t lane_base = static_cast<uint32_t>(q * 32) << 16;
    float *tb = reinterpret_cast<float *>(smem) + warp * (32 * 33);
    const int h = q >> 1;               // atom of this warp's 32 M elements
    const int e_base = (q & 1) * 32;    // first element of the warp inside the atom
    for (int j = j0; j < t1 - t0; j += jstep) {
      if (!((used >> j) & 1u)) continue;
      const int a = 2 * (t0 + j) + h;
      for (int n0 = 0; n0 < P.n_mma; n0 += 32) {
        float v[32];
        tmem_ld32(tmem_base + lane_base + static_cast<uint32_t>(j * P.n_mma + n0), v);
#pragma unroll
        for (int i = 0; i < 32; ++i) tb[i * 33 + lane] = v[i];
        __syncwarp();
        // lane = (channel quad c4, column nsub): the 8 lanes of one column
        // cover the warp's 32 consecutive channels, so each instruction adds
        // 4 whole 128-byte dW lines instead of 32 scattered 16-byte pieces
        // (reads of tb are conflict-free: bank = nsub + 4 c4 + const)
        const int c4 = lane & 7, nsub = lane >> 3;
        if (a < P.n_atoms) {
          int k = 0, ch = 0;
          atom_elem(P, a, e_base + 4 * c4, k, ch);
          if (k < A.kv && ((A.mask_filter >> k) & 1u)) {
#pragma unroll
            for (int cc = 0; cc < 8; ++cc) {
              const int col = cc * 4 + nsub;
              const int n = n0 + col;
              if (n < A.K) {
                const float *src = tb + col * 33 + 4 * c4;
                red_add_v4(A.ws + (static_cast<int64_t>(n) * A.kv + k) * A.C + ch, src[0], src[1], src[2],
                           src[3]);
              }
            }
          }
        }
        __syncwarp();
      }
    }
  };

  if (warp >= kLoadWarp0 && warp < kLoadWarp0 + kLoadWarps) {
    // ---------------------------------------------------------------- index loaders
    const int t = threadIdx.x - kLoadWarp0 * 32;
    const int r = t & 63;                  // row of the chunk
    const int par = kPair ? 0 : (t >> 6);  // filter parity of this thread (single layout)
    bool async_done = false;
    if constexpr (kPair) {
      if (A.idx_sorted != nullptr) {
        // Asynchronous form (pair layout, sorted index table).  The argsort
        // entry, the two mask words and the group's index values of this
        // thread's row are cp.async copies into the chunk's index buffer,
        // issued kAhead chunks before the chunk is gated and published, so
        // the memory round trips of consecutive chunks overlap.  A thread
        // copies and then gates only its own row's values, so
        // cp.async.wait_group alone orders them; the idx_full arrival
        // publishes the gated table.  Two of the four buffers in flight as
        // copies leave two published ahead of the producers (three in flight
        // left too few published and was slower).
        constexpr int kAhead = 2;
        static_assert(kAhead < kIdxStages, "a buffer is refilled only after its chunk is published");
        const uint32_t scr_off = kScratchOff(kTabF);
        // copies of iteration j into buffer j % kIdxStages (an empty commit
        // group past the last chunk); false when the buffer wait ran out
        auto issue = [&](int j) -> bool {
          const int64_t c = static_cast<int64_t>(c_begin) + static_cast<int64_t>(j) * c_step;
          if (c < c_end) {
            const int b = j % kIdxStages;
            const uint32_t ph = (j / kIdxStages) & 1;
            if (!mbar_wait(&idx_empty[b], ph ^ 1, abort_flag)) {
              cp_async_commit();
              return false;
            }
            const uint32_t base = smem_u32(smem + P.idx_off + b * P.idx_buf_bytes);
            const int64_t row = c * kRows + r;
            const int64_t row2 = c * kRows + (r ^ 32);
            const bool valid = row < A.N;
            if (A.argsort)
              cp_async_4(base + (kTabF * kRows + r) * 4, A.argsort + (valid ? row : 0), valid ? 4u : 0u);
            if (A.mask) {
              int64_t wi = P.mw_shift >= 0 ? row >> P.mw_shift : row / A.mask_width;
              bool ok1 = valid && wi < A.mask_count;
              cp_async_4(base + scr_off + r * 4, A.mask + (ok1 ? wi : 0), ok1 ? 4u : 0u);
              wi = P.mw_shift >= 0 ? row2 >> P.mw_shift : row2 / A.mask_width;
              ok1 = row2 < A.N && wi < A.mask_count;
              cp_async_4(base + scr_off + (kRows + r) * 4, A.mask + (ok1 ? wi : 0), ok1 ? 4u : 0u);
            }
#pragma unroll
            for (int q = 0; q < kNQ; ++q) {
              const int k = k_lo + q;
              if (k < k_hi)
                cp_async_4(base + ((k - k_lo) * kRows + r) * 4,
                           A.idx_sorted + (valid ? static_cast<int64_t>(k) * A.N + row : 0), valid ? 4u : 0u);
            }
          }
          cp_async_commit();
          return true;
        };
        bool ok = true;
#pragma unroll 1
        for (int j = 0; j < kAhead && ok; ++j) ok = issue(j);
#pragma unroll 1
        for (int it = 0; ok; ++it) {
          const int64_t c = static_cast<int64_t>(c_begin) + static_cast<int64_t>(it) * c_step;
          if (c >= c_end) break;
          cp_async_wait<kAhead - 1>();  // this thread's copies of iteration it have landed
          const int b = it % kIdxStages;
          uint8_t *buf = smem + P.idx_off + b * P.idx_buf_bytes;
          int *tab = reinterpret_cast<int *>(buf);
          int *sig_tab = tab + kTabF * kRows;
          WMeta *meta = reinterpret_cast<WMeta *>(sig_tab + kRows);
          const uint32_t *scr = reinterpret_cast<const uint32_t *>(buf + scr_off);
          const int64_t row = c * kRows + r;
          const int64_t row2 = c * kRows + (r ^ 32);
          const bool valid = row < A.N;
          int sig = valid ? (A.argsort ? sig_tab[r] : static_cast<int>(row)) : -1;
          uint32_t word, w_other;
          if (A.mask) {
            word = scr[r];
            w_other = scr[kRows + r];
          } else {
            word = valid ? 0xffffffffu : 0u;
            w_other = row2 < A.N ? 0xffffffffu : 0u;
          }
          if (valid && (sig < 0 || sig >= A.dout_rows)) {
            flag_error(A.err, kErrBadIndex);
            sig = -1;
          }
          word &= A.mask_filter;
          w_other &= A.mask_filter;
          uint32_t cm = word | w_other;
#pragma unroll
          for (int s = 16; s > 0; s >>= 1) cm |= __shfl_xor_sync(0xffffffffu, cm, s);
          sig_tab[r] = sig;
#pragma unroll
          for (int q = 0; q < kNQ; ++q) {
            const int k = k_lo + q;
            if (k < k_hi) {
              int v = tab[q * kRows + r];
              v = (((word >> k) & 1u) && sig >= 0) ? v : -1;
              if (v < -1 || v >= A.in_rows) {
                flag_error(A.err, kErrBadIndex);
                v = -1;
              }
              tab[q * kRows + r] = v;
            }
          }
          if (t < 32) {
            const bool on = lane < t1 - t0 && (tile_fbits[lane] & cm) != 0;
            const uint32_t bits = __ballot_sync(0xffffffffu, on);
            if (t == 0) {
              meta->active_bits = bits;
              meta->n_active = __popc(bits);
            }
          }
          mbar_arrive(&idx_full[b]);
          if (!issue(it + kAhead)) ok = false;
        }
        cp_async_wait_all();
        if (!ok) flag_error(A.err, kErrWaitTimeout);
        async_done = true;
      }
    }
    // synchronous form (single layout, or no sorted table): every load of a
    // chunk is issued before any result is used
    int it = 0;
    for (int c = async_done ? c_end : c_begin; c < c_end; c += c_step, ++it) {
      const int b = it % kIdxStages;
      const uint32_t ph = (it / kIdxStages) & 1;
      if (!mbar_wait(&idx_empty[b], ph ^ 1, abort_flag)) {
        flag_error(A.err, kErrWaitTimeout);
        break;
      }
      uint8_t *buf = smem + P.idx_off + b * P.idx_buf_bytes;
      int *tab = reinterpret_cast<int *>(buf);          // [kTabF][64]
      int *sig_tab = tab + kTabF * kRows;                // [64]
      WMeta *meta = reinterpret_cast<WMeta *>(sig_tab + kRows);
      const int64_t row = static_cast<int64_t>(c) * kRows + r;
      const int64_t row2 = static_cast<int64_t>(c) * kRows + (r ^ 32);
      const bool valid = row < A.N;
      // Every load of the chunk leaves before any result is used (argsort,
      // the mask words of this row and of its partner row r ^ 32, and with
      // the sorted table the indices): one memory round trip per chunk.
      int sig = valid ? (A.argsort ? __ldg(A.argsort + row) : static_cast<int>(row)) : -1;
      uint32_t word = 0, w_other = 0;
      if (A.mask) {
        if (valid) {
          const int64_t wi = P.mw_shift >= 0 ? row >> P.mw_shift : row / A.mask_width;
          if (wi < A.mask_count) word = __ldg(A.mask + wi);
        }
        if (row2 < A.N) {
          const int64_t wi = P.mw_shift >= 0 ? row2 >> P.mw_shift : row2 / A.mask_width;
          if (wi < A.mask_count) w_other = __ldg(A.mask + wi);
        }
      } else {
        word = valid ? 0xffffffffu : 0u;
        w_other = row2 < A.N ? 0xffffffffu : 0u;
      }
      int vals[kNQ];
#pragma unroll
      for (int q = 0; q < kNQ; ++q) {
        const int k = k_lo + kFStride * q + par;
        vals[q] = (A.idx_sorted && valid && k < k_hi)  // coalesced: row is the sorted row
                      ? __ldg(A.idx_sorted + static_cast<int64_t>(k) * A.N + row)
                      : -1;
      }
      if (valid && (sig < 0 || sig >= A.dout_rows)) {
        flag_error(A.err, kErrBadIndex);
        sig = -1;
      }
      if (!A.idx_sorted) {  // indices of the unsorted table are read at row sigma(r)
#pragma unroll
        for (int q = 0; q < kNQ; ++q) {
          const int k = k_lo + kFStride * q + par;
          int v = -1;
          if (k < k_hi && sig >= 0) {
            if (A.indices) v = __ldg(A.indices + static_cast<int64_t>(k) * A.N + sig);
            else v = A.b_inds ? __ldg(A.b_inds + row) : static_cast<int>(row);
          }
          vals[q] = v;
        }
      }
      word &= A.mask_filter;
      w_other &= A.mask_filter;
      // this warp covers rows (r & 32) .. +31 and read the words of the
      // partner rows r ^ 32 too (rows r and r ^ 32 share a mask word unless
      // mask_width < 64), so the OR over the warp is the chunk's mask, with
      // no cross-warp barrier
      uint32_t cm = word | w_other;
#pragma unroll
      for (int s = 16; s > 0; s >>= 1) cm |= __shfl_xor_sync(0xffffffffu, cm, s);
      if (par == 0) sig_tab[r] = sig;
#pragma unroll
      for (int q = 0; q < kNQ; ++q) {
        const int k = k_lo + kFStride * q + par;
        if (k < k_hi) {
          int v = (((word >> k) & 1u) && sig >= 0) ? vals[q] : -1;
          if (v < -1 || v >= A.in_rows) {
            flag_error(A.err, kErrBadIndex);
            v = -1;
          }
          tab[(k - k_lo) * kRows + r] = v;
        }
      }
      if (t < 32) {
        // lane j tests M-tile t0 + j against the chunk mask
        const bool on = lane < t1 - t0 && (tile_fbits[lane] & cm) != 0;
        const uint32_t bits = __ballot_sync(0xffffffffu, on);
        if (t == 0) {
          meta->active_bits = bits;
          meta->n_active = __popc(bits);
        }
      }
      mbar_arrive(&idx_full[b]);
    }
  } else if (warp >= kProdWarp0 && warp < kProdWarp0 + kProdWarps) {
    // ---------------------------------------------------------------- producers
    // Producer warp pw owns shared-memory stage pw (S <= kProdWarps; warps
    // beyond S stay idle) and fills every stage index g with g % S == pw
    // alone: lane owns 16-byte unit u of rows rg + 4 i (i < 16) of every
    // atom.  One owner per stage keeps each empty-barrier wait exactly one
    // phase ahead of the MMA warp.
    // Gathered rows with a pair use cp.async, the others are zero-filled
    // cp.async (src-size 0, no memory request).
    const int pw = warp - kProdWarp0;
    if constexpr (kGather) {
      produce_gather(pw, 0);
      if constexpr (kPair) reduce_tiles(pw, 1, 2);
    } else {
    const int u = lane & 7;
    const int rg = lane >> 3;
    int it = 0;
    uint32_t st_base = 0;  // stages of all previous chunks
    bool ok = pw < S;
    const uint32_t uS = static_cast<uint32_t>(S);
    const int n_b_atoms = P.n_mma / 64;
    for (int c = c_begin; c < c_end && ok; c += c_step, ++it) {
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
      const int *sig_tab = tab + kTabF * kRows;
      const WMeta *meta = reinterpret_cast<const WMeta *>(sig_tab + kRows);
      uint32_t bits = meta->active_bits;
      uint32_t local = 0;  // index of the stage inside this chunk
      while (bits) {
        const int jt = __ffs(bits) - 1;
        bits &= bits - 1;
        const uint32_t g_stage = st_base + local;
        ++local;
        if (g_stage % uS != static_cast<uint32_t>(pw)) continue;
        const int tt = t0 + jt;
        const uint32_t s = static_cast<uint32_t>(pw);  // == g_stage % S
        const uint32_t eph = (g_stage / uS) & 1u;
        int e_ok = 1;
        if (lane == 0) e_ok = mbar_wait(&empty_bar[s], eph ^ 1, abort_flag) ? 1 : 0;
        e_ok = __shfl_sync(0xffffffffu, e_ok, 0);
        if (!e_ok) {
          if (lane == 0) flag_error(A.err, kErrWaitTimeout);
          ok = false;
          break;
        }
        const uint32_t sA = smem_base + s * P.stage_bytes;
        const uint32_t sB = sA + P.b_off;
        // M side: two atoms x 64 rows
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int a = 2 * tt + h;
          int k, byte0;
          if (P.cpa > 0) {
            k = a / P.cpa;
            byte0 = (a % P.cpa) * 128 + u * 16;
          } else {
            k = a * P.fpa + u / P.upf;
            byte0 = (u % P.upf) * 16;
          }
          const bool atom_ok = a < P.n_atoms && k < A.kv;
          const int *trow = tab + (k - k_lo) * kRows;
#pragma unroll 4
          for (int i = 0; i < kRows / 4; ++i) {
            const int r = rg + 4 * i;
            const int idx = atom_ok ? trow[r] : -1;
            const uint32_t dst = sA + h * 8192 + sw128(r, u);
            if (idx >= 0)
              cp_async_16(dst, A.input + static_cast<int64_t>(idx) * A.in_ld * 2 + byte0, 16u);
            else
              cp_async_16(dst, A.input, 0u);  // zero fill, no memory request
          }
        }
        // N side: n_b_atoms atoms x 64 rows of dOut[sigma(r)]
        for (int na = 0; na < n_b_atoms; ++na) {
          const bool col_ok = na * 64 + u * 8 < A.K;
#pragma unroll 4
          for (int i = 0; i < kRows / 4; ++i) {
            const int r = rg + 4 * i;
            const int sg = sig_tab[r];
            const uint32_t dst = sB + na * 8192 + sw128(r, u);
            if (col_ok && sg >= 0)
              cp_async_16(dst, A.dout + static_cast<int64_t>(sg) * A.dout_ld * 2 + na * 128 + u * 16,
                          16u);
            else
              cp_async_16(dst, A.dout, 0u);  // zero fill, no memory request
          }
        }
        cp_async_mbar_arrive_noinc(&full_bar[s]);
      }
      if (!ok) break;
      st_base += local;
      __syncwarp();
      if (lane == 0) mbar_arrive(&idx_empty[b]);
    }
    cp_async_wait_all();
    }
  } else if (warp == kMmaWarp) {
    // ---------------------------------------------------------------- MMA issuer
    if (lane == 0) {
      int it = 0;
      // stage, full phase, dOut buffer and its phase of the ring of the
      // current chunk (c) and of the other ring (o); the rings alternate
      // chunk by chunk, so the two sets swap after every chunk (scalars, so
      // they stay in registers)
      uint32_t stage = 0, fph = 0, bb = 0, bph = 0;
      uint32_t stage_o = 0, fph_o = 0, bb_o = 0, bph_o = 0;
      const uint32_t Sr = static_cast<uint32_t>(S / kRings);
      const uint32_t NBr = P.n_bbuf / kRings;
      uint32_t started = 0;
      bool ok = true;
      for (int c = c_begin; c < c_end && ok; c += c_step, ++it) {
        const int ring = kRings == 2 ? (it & 1) : 0;
        const int b = it % kIdxStages;
        const uint32_t ph = (it / kIdxStages) & 1;
        if (!mbar_wait(&idx_full[b], ph, abort_flag)) {
          flag_error(A.err, kErrWaitTimeout);
          break;
        }
        const WMeta *meta = reinterpret_cast<const WMeta *>(smem + P.idx_off + b * P.idx_buf_bytes +
                                                            (kTabF * kRows + kRows) * 4);
        uint32_t bits = meta->active_bits;
        mbar_arrive(&idx_empty[b]);
        uint32_t sBg = 0;
        const bool chunk_used = bits != 0;
        const uint32_t bi = static_cast<uint32_t>(ring) * NBr + bb;
        if (kGather && chunk_used) {
          if (!mbar_wait(&bfull[bi], bph, abort_flag)) {
            flag_error(A.err, kErrWaitTimeout);
            break;
          }
          sBg = smem_base + P.bbuf_off + bi * ((P.n_mma / 64) * 8192u);
        }
        while (bits) {
          const int j = __ffs(bits) - 1;
          bits &= bits - 1;
          const uint32_t s = static_cast<uint32_t>(ring) * Sr + stage;
          if (!mbar_wait(&full_bar[s], fph, abort_flag)) {
            flag_error(A.err, kErrWaitTimeout);
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t sA = smem_base + s * P.stage_bytes;
          const uint32_t sB = kGather ? sBg : sA + P.b_off;
          const uint32_t d = tmem_base + static_cast<uint32_t>(j * P.n_mma);
#pragma unroll
          for (int kk = 0; kk < 4; ++kk) {
            const uint64_t ad = make_sdesc(sA + kk * 2048, 8192, 1024);
            const uint64_t bd = make_sdesc(sB + kk * 2048, 8192, 1024);
            const uint32_t acc = ((started >> j) & 1u) || kk > 0 ? 1u : 0u;
            mma_f16(d, ad, bd, P.idesc, acc);
          }
          started |= 1u << j;
          mma_commit(&empty_bar[s]);
          if (++stage == Sr) {
            stage = 0;
            fph ^= 1u;
          }
        }
        if (kGather && chunk_used && ok) {
          mma_commit(&bempty[bi]);  // dOut buffer free once these MMAs finish
          if (++bb == NBr) {
            bb = 0;
            bph ^= 1u;
          }
        }
        if constexpr (kRings == 2) {
          uint32_t x;
          x = stage; stage = stage_o; stage_o = x;
          x = fph; fph = fph_o; fph_o = x;
          x = bb; bb = bb_o; bb_o = x;
          x = bph; bph = bph_o; bph_o = x;
        }
      }
      if (started) {
        // all MMAs complete before the epilogue reads TMEM
        mma_commit(drain_bar);
        int never = 0;
        if (!mbar_wait(drain_bar, 0, reinterpret_cast<volatile int *>(&never))) {
          flag_error(A.err, kErrWaitTimeout);
          started = 0;
        }
        tc_fence_after();
      }
      *used_tiles = started;
      tc_fence_before();
      mbar_arrive(acc_full);  // release: used_tiles and the finished accumulators
    }
  } else if (warp < kEpiWarps) {
    // ---------------------------------------------------------------- epilogue (warps 0-3)
    // In the pair layout these warps first produce for the second ring.
    if constexpr (kGather && kPair) produce_gather(warp, 1);
    reduce_tiles(warp, 0, kPair ? 2 : 1);
  }

  tc_fence_before();
  __syncthreads();
  if (warp == kMmaWarp) {
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem_base, P.tmem_cols);
  }
}

template <typename TOut>
__global__ void wgrad_finalize_kernel(const float *ws, TOut *out, int64_t out_ld, int64_t total,
                                      int kv, int C, uint32_t mask_filter, EpiParams e) {
  const int64_t row_len = static_cast<int64_t>(kv) * C;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t row = i / row_len;
    const int64_t col = i % row_len;
    const int k = static_cast<int>(col / C);
    if (!((mask_filter >> k) & 1u)) continue;
    float v = e.alpha * ws[i];
    if (e.beta != 0.f && e.src != nullptr)
      v = fmaf(e.beta, to_f32(static_cast<const TOut *>(e.src)[row * e.src_ld + col]), v);
    out[row * out_ld + col] = from_f32<TOut>(apply_act(v, e.act_type, e.act_alpha));
  }
}

template <typename T>
__global__ void transpose_weight_kernel(const T *w, T *wt, int K, int kv, int C) {
  // w[K, kv, C] -> wt[C, kv, K]
  const int64_t total = static_cast<int64_t>(K) * kv * C;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int c = static_cast<int>(i % C);
    const int k = static_cast<int>((i / C) % kv);
    const int ko = static_cast<int>(i / (static_cast<int64_t>(C) * kv));
    wt[(static_cast<int64_t>(c) * kv + k) * K + ko] = w[i];
  }
}

}  // namespace

cudaError_t launch_conv_wgrad(const ConvWgradArgs &a, int num_sms, cudaStream_t stream) {
  WParams P;
  P.a = a;
  P.n_chunks = static_cast<int>((a.N + kRows - 1) / kRows);
  if (P.n_chunks == 0) return cudaSuccess;
  if (a.C >= 64) {
    P.cpa = a.C / 64;
    P.fpa = 1;
    P.upf = 8;
    P.n_atoms = a.kv * P.cpa;
  } else {
    P.cpa = 0;
    P.fpa = 64 / a.C;
    P.upf = a.C / 8;
    P.n_atoms = (a.kv + P.fpa - 1) / P.fpa;
  }
  P.n_mtiles = (P.n_atoms + 1) / 2;
  P.n_mma = ((a.K + 63) / 64) * 64;
  P.mw_shift = -1;
  for (int sh = 0; sh < 31; ++sh)
    if (a.mask_width == (1 << sh)) P.mw_shift = sh;
  // gather path: whole 128-byte row blocks on both sides and tensor maps for
  // the input and dOut rows (else 16-byte cp.async gathers)
  bool gather = P.cpa > 0 && a.K % 64 == 0 && (a.in_dtype == 12 || a.in_dtype == 7) &&
                a.in_rows > 0 && a.dout_rows > 0;
  if (gather)
    gather = encode_tmap_2d(&P.tmap_in, a.in_dtype, a.input, static_cast<uint64_t>(a.C),
                            static_cast<uint64_t>(a.in_rows), static_cast<uint64_t>(a.in_ld) * 2, 64, 1) &&
             encode_tmap_2d(&P.tmap_dout, a.in_dtype, a.dout, static_cast<uint64_t>(a.K),
                            static_cast<uint64_t>(a.dout_rows), static_cast<uint64_t>(a.dout_ld) * 2, 64, 1);
  P.zero_ok = 0;
  if (gather) {
    const void *z = zero_rows_address();
    P.zero_ok = z != nullptr && encode_tmap_2d(&P.tmap_zero, a.in_dtype, z, 64, kZeroRows, 128, 64, 1) ? 1 : 0;
  }
  const uint32_t a_bytes = 2 * 8192;
  const uint32_t b_bytes = static_cast<uint32_t>(P.n_mma / 64) * 8192;
  P.stage_bytes = gather ? a_bytes : a_bytes + b_bytes;
  P.b_off = a_bytes;
  const uint32_t bar_bytes = 512;
  auto idx_buf_for = [](bool pr) {
    const int f = pr ? Layout<true>::kTabF : Layout<false>::kTabF;
    return static_cast<uint32_t>((kScratchOff(f) + 2 * kRows * 4 + 127) & ~size_t(127));
  };
  // stages that fit beside the index ring, barriers and dOut buffers in one
  // CTA's dynamic shared memory: 227 KB alone on an SM, 113 KB for one of two
  // (1 KB of it is slack for the 1024-byte alignment of the stages)
  auto stages_for = [&](bool pr, uint32_t bbuf_bytes) {
    const int64_t limit = pr ? 113 * 1024 : 227 * 1024;
    const int64_t budget = limit - 1024 - static_cast<int64_t>(idx_buf_for(pr)) * kIdxStages -
                           bar_bytes - static_cast<int64_t>(bbuf_bytes);
    const int64_t st = budget > 0 ? budget / P.stage_bytes : 0;
    return static_cast<int>(st > 8 ? 8 : st);
  };
  // Two CTAs per SM on the gather path with 64 dOut columns, when each of
  // their two producer rings gets two stages and two dOut buffers in 113 KB.
  const bool pair = gather && P.n_mma == 64 && stages_for(true, kMaxBBufs * b_bytes) >= 4;
  // The producers can run n_bbuf - 1 chunks ahead of the MMA (a chunk's dOut
  // buffer is released after its last M-tile): four buffers when that still
  // leaves four stages, else two (one ring).
  P.n_bbuf = gather ? (pair || stages_for(false, kMaxBBufs * b_bytes) >= 4 ? kMaxBBufs : 2) : 1;
  const uint32_t bbuf_bytes = gather ? P.n_bbuf * b_bytes : 0;
  int stages = stages_for(pair, bbuf_bytes);
  if (pair) stages &= ~1;  // an equal share per ring
  if (stages < 2) return cudaErrorInvalidConfiguration;
  P.idx_buf_bytes = idx_buf_for(pair);
  // M-tile groups: TMEM columns per CTA (512, or 256 for each of a pair)
  int per_group = (pair ? 256 : 512) / P.n_mma;
  if (per_group > 16) per_group = 16;
  if (per_group > P.n_mtiles) per_group = P.n_mtiles;
  // as few groups as TMEM allows, then equal shares (14 tiles: 7 + 7, not 8 + 6)
  const int n_groups = (P.n_mtiles + per_group - 1) / per_group;
  per_group = (P.n_mtiles + n_groups - 1) / n_groups;
  P.tiles_per_group = per_group;
  P.n_groups = (P.n_mtiles + per_group - 1) / per_group;
  // row splits: the caller's split_k_slices, else about one CTA per SM (two
  // per SM in the pair layout)
  const int ctas = (pair ? 2 : 1) * num_sms;
  int splits = a.split_k > 0 ? a.split_k : (ctas + P.n_groups - 1) / P.n_groups;
  if (splits > P.n_chunks) splits = P.n_chunks;
  P.chunks_per_cta = (P.n_chunks + splits - 1) / splits;
  splits = (P.n_chunks + P.chunks_per_cta - 1) / P.chunks_per_cta;
  P.stages = stages;
  P.bbuf_off = P.stage_bytes * stages;
  P.idx_off = P.bbuf_off + bbuf_bytes;
  P.bar_off = P.idx_off + P.idx_buf_bytes * kIdxStages;
  const size_t smem = 1024 + P.bar_off + bar_bytes;
  uint32_t cols = 32;
  while (cols < static_cast<uint32_t>(per_group * P.n_mma)) cols <<= 1;
  P.tmem_cols = cols;
  P.idesc = make_idesc(128, P.n_mma, a.in_dtype == 12 ? 1u : 0u, true, true);
  void (*kern)(WParams) = pair     ? conv_wgrad_kernel<true, true>
                          : gather ? conv_wgrad_kernel<true, false>
                                   : conv_wgrad_kernel<false, false>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  dim3 grid(splits, P.n_groups);
  kern<<<grid, pair ? Layout<true>::kThreads : Layout<false>::kThreads, smem, stream>>>(P);
  return cudaGetLastError();
}

cudaError_t launch_wgrad_finalize(const float *ws, void *out, int64_t out_ld, int out_dtype,
                                  int K, int kv, int C, uint32_t mask_filter, const EpiParams &e,
                                  cudaStream_t stream) {
  const int64_t total = static_cast<int64_t>(K) * kv * C;
  const int threads = 256;
  int blocks = static_cast<int>((total + threads - 1) / threads);
  if (blocks > 4096) blocks = 4096;
  if (blocks < 1) blocks = 1;
  switch (out_dtype) {
    case 0:
      wgrad_finalize_kernel<float><<<blocks, threads, 0, stream>>>(
          ws, static_cast<float *>(out), out_ld, total, kv, C, mask_filter, e);
      break;
    case 7:
      wgrad_finalize_kernel<__half><<<blocks, threads, 0, stream>>>(
          ws, static_cast<__half *>(out), out_ld, total, kv, C, mask_filter, e);
      break;
    case 12:
      wgrad_finalize_kernel<__nv_bfloat16><<<blocks, threads, 0, stream>>>(
          ws, static_cast<__nv_bfloat16 *>(out), out_ld, total, kv, C, mask_filter, e);
      break;
    default:
      return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_transpose_weight(const void *w, void *wt, int K, int kv, int C, int esize,
                                    cudaStream_t stream) {
  const int64_t total = static_cast<int64_t>(K) * kv * C;
  const int threads = 256;
  int blocks = static_cast<int>((total + threads - 1) / threads);
  if (blocks > 4096) blocks = 4096;
  if (blocks < 1) blocks = 1;
  if (esize == 2)
    transpose_weight_kernel<uint16_t><<<blocks, threads, 0, stream>>>(
        static_cast<const uint16_t *>(w), static_cast<uint16_t *>(wt), K, kv, C);
  else if (esize == 1)
    transpose_weight_kernel<uint8_t><<<blocks, threads, 0, stream>>>(
        static_cast<const uint8_t *>(w), static_cast<uint8_t *>(wt), K, kv, C);
  else if (esize == 4)
    transpose_weight_kernel<float><<<blocks, threads, 0, stream>>>(
        static_cast<const float *>(w), static_cast<float *>(wt), K, kv, C);
  else
    return cudaErrorInvalidValue;
  return cudaGetLastError();
}

}  // namespace scb
