// gemm_dense.cu - dense GEMM of matmul2 (NoShuffle, 16-bit operands) on
// sm_100a tensor cores.
//
//   C[m, n] = act(alpha * op(A) @ op(B) + beta * D)
// with op(A) = A [m, k] or A^T (A stored [k, m]) and op(B) = B [k, n] or B^T
// (B stored [n, k]) -- the reference's GemmMainUnitTest.matmul2 without a
// shuffle (cumm/gemm/main.py:1176-1335, kernel cumm/gemm/kernel.py:586-940;
// split-K as in cumm/gemm/nvrtc_code.py:68-75 and params.h:115-132, here as a
// parallel reduction into an fp32 workspace instead of the serial semaphore).
//
// B200 design: persistent CTAs (one per SM) walk (128 x 256 output tile,
// K split) work units.  Warp 4 loads 128 x 64 A and 256 x 64 B blocks with
// 2-D TMA boxes into a 4-stage ring (48 KB per stage, SWIZZLE_128B); a
// row-major operand is K-major for the tensor core and a transposed one is
// read in place as MN-major (no copy).  Warp 5 issues tcgen05.mma (M = 128,
// N = 256, K = 16; one issuing warp completes such an MMA about as fast as
// the tensor pipe runs it) into a double-buffered 128 x 256 fp32 TMEM
// accumulator, so warps 0-3 run the epilogue of one tile while the next one
// accumulates.  The epilogue applies act(alpha acc + beta D) and stores
// 32-byte row segments, or with split-K adds its partial tile into an fp32
// workspace with red.global.add.v4.f32 (a finalize pass applies the
// epilogue).  Rows and columns past m / n / k are TMA zero fill on the loads
// and skipped on the stores.  Every mbarrier wait is bounded.
#include <cuda.h>

#include "kernels.h"

namespace scb {
namespace {

constexpr int kBM = 128, kBN = 256, kBK = 64;
constexpr int kStages = 4;
constexpr int kThreads = 192;  // warps 0-3 epilogue, 4 TMA producer, 5 MMA issuer
constexpr int kGroupM = 16;    // row tiles per raster group
constexpr uint32_t kABytes = kBM * kBK * 2;  // 16 KB
constexpr uint32_t kBBytes = kBN * kBK * 2;  // 32 KB
constexpr uint32_t kStageBytes = kABytes + kBBytes;

struct DParams {
  CUtensorMap ta;
  CUtensorMap tb;
  GemmArgs g;
  int a_mn, b_mn;  // operand is MN-major (stored transposed relative to the MMA's K-major form)
  int64_t m_tiles, n_tiles, units;
  int splits, kb_per_split, kblocks;
  uint32_t bar_off;
  uint32_t idesc;
  float *ws;  // split-K: fp32 [m, n] (ld n), zeroed; else null
};

__device__ __forceinline__ void flag_error(int *err, int bits) { atomicOr(err, bits); }

// Output tile -> (row tile, column tile).  Tiles are walked in groups of
// kGroupM row tiles, column by column inside a group, so the tiles that the
// persistent CTAs hold at one time (one each) cover a compact block: at
// 8192^3, 16 row tiles x ~10 column tiles = 34 MB of A and 42 MB of B, which
// stay in L2 instead of B streaming from HBM once per 4.6 row tiles.
__device__ __forceinline__ void tile_mn(const DParams &P, int64_t tile, int64_t &mt, int64_t &nt) {
  const int64_t per_group = static_cast<int64_t>(kGroupM) * P.n_tiles;
  const int64_t g = tile / per_group;
  const int64_t first = g * kGroupM;
  const int64_t gm = P.m_tiles - first < kGroupM ? P.m_tiles - first : kGroupM;
  const int64_t r = tile - g * per_group;
  mt = first + r % gm;
  nt = r / gm;
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

__device__ __forceinline__ void red_add_v4(float *p, float a, float b, float c, float d) {
  asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(a), "f"(b), "f"(c), "f"(d)
               : "memory");
}

__device__ __forceinline__ void st_global_v8(void *p, const uint32_t *w) {
  asm volatile("st.global.v8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(p), "r"(w[0]), "r"(w[1]), "r"(w[2]),
               "r"(w[3]), "r"(w[4]), "r"(w[5]), "r"(w[6]), "r"(w[7])
               : "memory");
}

// Epilogue of 16 accumulator columns [col0, col0 + 16) of output row `row`.
template <typename TOut>
__device__ __forceinline__ void store16(const DParams &P, int64_t row, int64_t col0, float *acc) {
  const GemmArgs &G = P.g;
  const EpiParams &e = G.epi;
  const int64_t ncol = G.n - col0 < 16 ? G.n - col0 : 16;
  if (P.ws != nullptr) {
    float *w = P.ws + row * G.n + col0;
    if (ncol == 16 && (G.n & 3) == 0) {
#pragma unroll
      for (int i = 0; i < 16; i += 4) red_add_v4(w + i, acc[i], acc[i + 1], acc[i + 2], acc[i + 3]);
    } else {
      for (int i = 0; i < ncol; ++i) atomicAdd(w + i, acc[i]);
    }
    return;
  }
  const bool use_src = e.beta != 0.f && e.src != nullptr;
  const TOut *src = use_src ? static_cast<const TOut *>(e.src) + row * e.src_ld + col0 : nullptr;
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    float v = e.alpha * acc[i];
    if (use_src && i < ncol) v = fmaf(e.beta, to_f32(src[i]), v);
    acc[i] = apply_act(v, e.act_type, e.act_alpha);
  }
  TOut *dst = static_cast<TOut *>(G.c) + row * G.ldc + col0;
  constexpr int kPer32 = 32 / sizeof(TOut);
  if (ncol == 16 && (reinterpret_cast<uintptr_t>(dst) & 31u) == 0) {
#pragma unroll
    for (int i = 0; i < 16; i += kPer32) {
      uint32_t w[8];
      if constexpr (sizeof(TOut) == 4) {
#pragma unroll
        for (int j = 0; j < 8; ++j) w[j] = __float_as_uint(acc[i + j]);
      } else {
        TOut *h = reinterpret_cast<TOut *>(w);
#pragma unroll
        for (int j = 0; j < 16; ++j) h[j] = from_f32<TOut>(acc[i + j]);
      }
      st_global_v8(dst + i, w);
    }
  } else {
    for (int i = 0; i < ncol; ++i) dst[i] = from_f32<TOut>(acc[i]);
  }
}

template <typename TOut>
__global__ void __launch_bounds__(kThreads, 1) dense_gemm_kernel(const __grid_constant__ DParams P) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw_u32 = smem_u32(smem_raw);
  const uint32_t pad = (1024u - (raw_u32 & 1023u)) & 1023u;
  uint8_t *smem = smem_raw + pad;
  const uint32_t smem_base = raw_u32 + pad;
  const GemmArgs &G = P.g;

  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + P.bar_off);
  uint64_t *full = bars;
  uint64_t *empty = bars + kStages;
  uint64_t *acc_full = empty + kStages;
  uint64_t *acc_empty = acc_full + 2;
  uint64_t *tile_bar = acc_empty + 2;
  uint64_t *drain_bar = tile_bar + 2;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(drain_bar + 1);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);
  volatile long long *acc_unit = reinterpret_cast<volatile long long *>(tmem_slot + 2);  // [2]
  volatile int *acc_nkb = reinterpret_cast<volatile int *>(tmem_slot + 6);              // [2]

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int i = 0; i < kStages; ++i) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(&acc_full[i], 1);
      mbar_init(&acc_empty[i], 128);
      mbar_init(&tile_bar[i], 1);
    }
    mbar_init(drain_bar, 1);
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 5) {
    tmem_alloc(tmem_slot, 512);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  if (warp == 4) {
    // ---------------------------------------------------------------- TMA producer
    if (lane == 0) {
      uint32_t stage = 0, eph = 0;
      bool ok = true;
      for (int64_t u = blockIdx.x; u < P.units && ok; u += gridDim.x) {
        const int64_t tile = u / P.splits;
        const int ks = static_cast<int>(u % P.splits);
        int64_t mt, nt;
        tile_mn(P, tile, mt, nt);
        const int m0 = static_cast<int>(mt * kBM);
        const int n0 = static_cast<int>(nt * kBN);
        const int kb0 = ks * P.kb_per_split;
        const int kb1 = min(P.kblocks, kb0 + P.kb_per_split);
        for (int kb = kb0; kb < kb1; ++kb) {
          if (!mbar_wait(&empty[stage], eph ^ 1u, abort_flag)) {
            flag_error(G.err, kErrWaitTimeout);
            ok = false;
            break;
          }
          const uint32_t sA = smem_base + stage * kStageBytes;
          const uint32_t sB = sA + kABytes;
          const int k0 = kb * kBK;
          mbar_arrive_expect_tx(&full[stage], kStageBytes);
          if (P.a_mn) {
            tma_load_2d(sA, &P.ta, m0, k0, &full[stage]);
            tma_load_2d(sA + 8192, &P.ta, m0 + 64, k0, &full[stage]);
          } else {
            tma_load_2d(sA, &P.ta, k0, m0, &full[stage]);
          }
          if (P.b_mn) {
#pragma unroll
            for (int q = 0; q < 4; ++q) tma_load_2d(sB + q * 8192, &P.tb, n0 + 64 * q, k0, &full[stage]);
          } else {
            tma_load_2d(sB, &P.tb, k0, n0, &full[stage]);
          }
          if (++stage == kStages) {
            stage = 0;
            eph ^= 1u;
          }
        }
      }
    }
  } else if (warp == 5) {
    // ---------------------------------------------------------------- MMA issuer
    if (lane == 0) {
      uint32_t stage = 0, fph = 0;
      bool issued = false, ok = true;
      int it = 0;
      for (int64_t u = blockIdx.x;; u += gridDim.x, ++it) {
        const bool have = u < P.units;
        const int ab = it & 1;
        const uint32_t aph = (it >> 1) & 1;
        if (!mbar_wait(&acc_empty[ab], aph ^ 1u, abort_flag)) {
          flag_error(G.err, kErrWaitTimeout);
          break;
        }
        tc_fence_after();
        int nkb = 0;
        if (have) {
          const int ks = static_cast<int>(u % P.splits);
          const int kb0 = ks * P.kb_per_split;
          nkb = max(0, min(P.kblocks, kb0 + P.kb_per_split) - kb0);
        }
        acc_unit[ab] = have ? u : -1;
        acc_nkb[ab] = nkb;
        mbar_arrive(&tile_bar[ab]);
        if (!have) break;
        const uint32_t d = tmem_base + static_cast<uint32_t>(ab * kBN);
        for (int j = 0; j < nkb; ++j) {
          if (!mbar_wait(&full[stage], fph, abort_flag)) {
            flag_error(G.err, kErrWaitTimeout);
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t sA = smem_base + stage * kStageBytes;
          const uint32_t sB = sA + kABytes;
#pragma unroll
          for (int kk = 0; kk < 4; ++kk) {
            // K advances 16 elements: 32 bytes inside a K-major row, 16 rows
            // (2 KB) of an MN-major atom
            const uint64_t ad = P.a_mn ? make_sdesc(sA + kk * 2048, 8192, 1024) : make_sdesc(sA + kk * 32, 16, 1024);
            const uint64_t bd = P.b_mn ? make_sdesc(sB + kk * 2048, 8192, 1024) : make_sdesc(sB + kk * 32, 16, 1024);
            mma_f16(d, ad, bd, P.idesc, (j | kk) != 0 ? 1u : 0u);
          }
          issued = true;
          mma_commit(&empty[stage]);
          if (++stage == kStages) {
            stage = 0;
            fph ^= 1u;
          }
        }
        if (!ok) break;
        if (nkb == 0) mbar_arrive(&acc_full[ab]);
        else mma_commit(&acc_full[ab]);
      }
      if (issued) {
        mma_commit(drain_bar);
        int never = 0;
        if (!mbar_wait(drain_bar, 0, reinterpret_cast<volatile int *>(&never))) flag_error(G.err, kErrWaitTimeout);
      }
    }
  } else {
    // ---------------------------------------------------------------- epilogue (warps 0-3)
    const uint32_t lane_base = static_cast<uint32_t>(warp * 32) << 16;
    for (int it = 0;; ++it) {
      const int ab = it & 1;
      const uint32_t aph = (it >> 1) & 1;
      if (!mbar_wait(&tile_bar[ab], aph, abort_flag)) {
        flag_error(G.err, kErrWaitTimeout);
        break;
      }
      const long long u = acc_unit[ab];
      if (u < 0) break;
      const int nkb = acc_nkb[ab];
      if (!mbar_wait(&acc_full[ab], aph, abort_flag)) {
        flag_error(G.err, kErrWaitTimeout);
        break;
      }
      tc_fence_after();
      const int64_t tile = u / P.splits;
      int64_t mt, nt;
      tile_mn(P, tile, mt, nt);
      const int64_t row = mt * kBM + threadIdx.x;
      const int64_t nb = nt * kBN;
      for (int cc = 0; cc < kBN; cc += 16) {
        if (nb + cc >= G.n) break;  // warp-uniform
        float acc[16];
        if (nkb > 0) {
          tmem_ld16(tmem_base + lane_base + static_cast<uint32_t>(ab * kBN + cc), acc);
        } else {
#pragma unroll
          for (int i = 0; i < 16; ++i) acc[i] = 0.f;
        }
        if (row < G.m) store16<TOut>(P, row, nb + cc, acc);
      }
      tc_fence_before();
      mbar_arrive(&acc_empty[ab]);
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 5) {
    tc_fence_after();
    tmem_dealloc(tmem_base, 512);
  }
}

}  // namespace

bool dense_gemm_supported(const GemmArgs &a) {
  if (a.shuffle != 0) return false;
  if (a.in_dtype != 12 && a.in_dtype != 7) return false;
  if (a.out_dtype != 0 && a.out_dtype != 7 && a.out_dtype != 12) return false;
  if ((a.lda * 2) % 16 || (a.ldb * 2) % 16) return false;
  if (reinterpret_cast<uintptr_t>(a.a) % 16 || reinterpret_cast<uintptr_t>(a.b) % 16) return false;
  if (a.m <= 0 || a.n <= 0 || a.k < 0) return false;
  return true;
}

int dense_gemm_splits(const GemmArgs &a) {
  const int64_t kblocks = (a.k + kBK - 1) / kBK;
  int s = a.split_k > 1 ? a.split_k : 1;
  if (s > kblocks) s = static_cast<int>(kblocks > 0 ? kblocks : 1);
  return s;
}

cudaError_t launch_dense_gemm(const GemmArgs &a, float *split_ws, int num_sms, cudaStream_t stream) {
  DParams P;
  P.g = a;
  P.a_mn = a.trans_a ? 1 : 0;
  P.b_mn = a.trans_b ? 0 : 1;
  // A: [m, k] (K-major, 64 x 128 boxes) or stored [k, m] (MN-major, 64 x 64 boxes)
  const bool ok_a = P.a_mn ? encode_tmap_2d(&P.ta, a.in_dtype, a.a, static_cast<uint64_t>(a.m),
                                            static_cast<uint64_t>(a.k > 0 ? a.k : 1),
                                            static_cast<uint64_t>(a.lda) * 2, 64, 64)
                           : encode_tmap_2d(&P.ta, a.in_dtype, a.a, static_cast<uint64_t>(a.k > 0 ? a.k : 1),
                                            static_cast<uint64_t>(a.m), static_cast<uint64_t>(a.lda) * 2, 64, kBM);
  // B: stored [n, k] (K-major, 64 x 256 boxes) or [k, n] (MN-major, 64 x 64 boxes)
  const bool ok_b = P.b_mn ? encode_tmap_2d(&P.tb, a.in_dtype, a.b, static_cast<uint64_t>(a.n),
                                            static_cast<uint64_t>(a.k > 0 ? a.k : 1),
                                            static_cast<uint64_t>(a.ldb) * 2, 64, 64)
                           : encode_tmap_2d(&P.tb, a.in_dtype, a.b, static_cast<uint64_t>(a.k > 0 ? a.k : 1),
                                            static_cast<uint64_t>(a.n), static_cast<uint64_t>(a.ldb) * 2, 64, kBN);
  if (!ok_a || !ok_b) return cudaErrorInvalidValue;
  const int64_t m_tiles = (a.m + kBM - 1) / kBM;
  P.m_tiles = m_tiles;
  P.n_tiles = (a.n + kBN - 1) / kBN;
  P.kblocks = static_cast<int>((a.k + kBK - 1) / kBK);
  P.splits = dense_gemm_splits(a);
  P.kb_per_split = P.kblocks > 0 ? (P.kblocks + P.splits - 1) / P.splits : 0;
  P.units = m_tiles * P.n_tiles * P.splits;
  P.ws = P.splits > 1 ? split_ws : nullptr;
  P.bar_off = kStages * kStageBytes;
  P.idesc = make_idesc(kBM, kBN, a.in_dtype == 12 ? 1u : 0u, P.a_mn != 0, P.b_mn != 0);
  const size_t smem = 1024 + P.bar_off + 256;
  const int grid = static_cast<int>(P.units < num_sms ? P.units : num_sms);
  void (*kern)(DParams);
  switch (a.out_dtype) {
    case 0: kern = dense_gemm_kernel<float>; break;
    case 7: kern = dense_gemm_kernel<__half>; break;
    case 12: kern = dense_gemm_kernel<__nv_bfloat16>; break;
    default: return cudaErrorInvalidValue;
  }
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  kern<<<grid, kThreads, smem, stream>>>(P);
  return cudaGetLastError();
}

}  // namespace scb
