// pairs.cu - indice-pair / mask builder on the GPU.
//
// Replaces spconv's generate_subm_conv_inds / generate_conv_inds and
// sort_1d_by_key_split as they are used by the reference driver
// (cumm/conv/main_real_spconv.py:72-145), over a linear-probing hash table in
// the style of cumm's LinearHashTableSplit (include/tensorview/hash/linear.cu.h:557-840):
// keys are linearised voxel coordinates (int64, empty slot = -1), slot =
// MurmurHash3 64-bit finaliser(key) & (capacity - 1), collisions probe
// linearly.  Unlike the reference's unbounded `while (true)` probe loops
// (linear.cu.h:229,381) every probe here stops after `capacity` steps and
// reports kErrHashFull.
//
// Conventions (cross-correlation, matching torch.nn.functional.conv3d):
//   coords[i] = (batch, z, y, x); offset k = (kz * KY + ky) * KX + kx;
//   submanifold: pairs_fwd[k][i] = index of the voxel at
//     coord(i) + ((kz, ky, kx) - ksize // 2) * dilation, or -1;
//   strided: output o receives input i through offset k iff
//     coord(i) = o * stride - padding + (kz, ky, kx) * dilation;
//   pairs_bwd[k][i] = o such that pairs_fwd[k][o] = i;
//   mask_fwd[o] bit k <=> pairs_fwd[k][o] >= 0; mask_bwd[i] bit k <=> pairs_bwd[k][i] >= 0.
// Strided outputs are numbered in ascending linearised (batch, z, y, x) order
// (the reference numbers them by an atomic counter, i.e. nondeterministically,
// hash.cu.h:201-213; the canonical order makes the table reproducible).
#include "kernels.h"

namespace scb {
namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ uint64_t fmix64(uint64_t k) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdull;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ull;
  k ^= k >> 33;
  return k;
}

struct Table {
  unsigned long long *keys;  // -1 = empty
  int *vals;
  int64_t cap;               // power of two
};

__device__ __forceinline__ bool table_insert(const Table &t, long long key, int val, int *err) {
  uint64_t slot = fmix64(static_cast<uint64_t>(key)) & static_cast<uint64_t>(t.cap - 1);
  for (int64_t step = 0; step < t.cap; ++step) {
    const unsigned long long prev =
        atomicCAS(t.keys + slot, ~0ull, static_cast<unsigned long long>(key));
    if (prev == ~0ull || prev == static_cast<unsigned long long>(key)) {
      if (t.vals) atomicMin(t.vals + slot, val);
      return true;
    }
    slot = (slot + 1) & static_cast<uint64_t>(t.cap - 1);
  }
  atomicOr(err, kErrHashFull);
  return false;
}

__device__ __forceinline__ int table_lookup(const Table &t, long long key) {
  uint64_t slot = fmix64(static_cast<uint64_t>(key)) & static_cast<uint64_t>(t.cap - 1);
  for (int64_t step = 0; step < t.cap; ++step) {
    const unsigned long long k = t.keys[slot];
    if (k == static_cast<unsigned long long>(key)) return t.vals[slot];
    if (k == ~0ull) return -1;
    slot = (slot + 1) & static_cast<uint64_t>(t.cap - 1);
  }
  return -1;
}

__global__ void table_clear(Table t) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < t.cap;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    t.keys[i] = ~0ull;
    if (t.vals) t.vals[i] = 0x7fffffff;
  }
}

struct Geom {
  int spatial[3];
  int ksize[3];
  int stride[3];
  int padding[3];
  int dilation[3];
  int out_spatial[3];
  int kv;
};

__device__ __forceinline__ long long lin_key(int b, int z, int y, int x, const int *sp) {
  return ((static_cast<long long>(b) * sp[0] + z) * sp[1] + y) * sp[2] + x;
}

__global__ void insert_coords(const int32_t *coords, int64_t n, Geom g, Table t, int *err) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int b = coords[i * 4], z = coords[i * 4 + 1], y = coords[i * 4 + 2],
              x = coords[i * 4 + 3];
    if (b < 0 || z < 0 || y < 0 || x < 0 || z >= g.spatial[0] || y >= g.spatial[1] ||
        x >= g.spatial[2]) {
      atomicOr(err, kErrBadIndex);
      continue;
    }
    table_insert(t, lin_key(b, z, y, x, g.spatial), static_cast<int>(i), err);
  }
}

__global__ void fill_i32(int32_t *p, int64_t n, int32_t v) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    p[i] = v;
}

__global__ void subm_pairs_kernel(const int32_t *coords, int64_t n, Geom g, Table t,
                                  int32_t *pairs_fwd, int32_t *pairs_bwd, uint32_t *mask_fwd) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int b = coords[i * 4], z = coords[i * 4 + 1], y = coords[i * 4 + 2],
              x = coords[i * 4 + 3];
    uint32_t m = 0;
    int k = 0;
    for (int a = 0; a < g.ksize[0]; ++a) {
      for (int c = 0; c < g.ksize[1]; ++c) {
        for (int d = 0; d < g.ksize[2]; ++d, ++k) {
          const int zz = z + (a - g.ksize[0] / 2) * g.dilation[0];
          const int yy = y + (c - g.ksize[1] / 2) * g.dilation[1];
          const int xx = x + (d - g.ksize[2] / 2) * g.dilation[2];
          int j = -1;
          if (zz >= 0 && yy >= 0 && xx >= 0 && zz < g.spatial[0] && yy < g.spatial[1] &&
              xx < g.spatial[2])
            j = table_lookup(t, lin_key(b, zz, yy, xx, g.spatial));
          pairs_fwd[static_cast<int64_t>(k) * n + i] = j;
          if (j >= 0) {
            m |= 1u << k;
            pairs_bwd[static_cast<int64_t>(k) * n + j] = static_cast<int>(i);
          }
        }
      }
    }
    mask_fwd[i] = m;
  }
}

// Output coordinate of input (z,y,x) through offset (a,c,d); false if none.
__device__ __forceinline__ bool out_coord(const Geom &g, int z, int y, int x, int a, int c, int d,
                                          int &oz, int &oy, int &ox) {
  const int tz = z + g.padding[0] - a * g.dilation[0];
  const int ty = y + g.padding[1] - c * g.dilation[1];
  const int tx = x + g.padding[2] - d * g.dilation[2];
  if (tz < 0 || ty < 0 || tx < 0) return false;
  if (tz % g.stride[0] || ty % g.stride[1] || tx % g.stride[2]) return false;
  oz = tz / g.stride[0];
  oy = ty / g.stride[1];
  ox = tx / g.stride[2];
  return oz < g.out_spatial[0] && oy < g.out_spatial[1] && ox < g.out_spatial[2];
}

__global__ void conv_candidates(const int32_t *coords, int64_t n, Geom g, Table t, int *err) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int b = coords[i * 4], z = coords[i * 4 + 1], y = coords[i * 4 + 2],
              x = coords[i * 4 + 3];
    for (int a = 0; a < g.ksize[0]; ++a)
      for (int c = 0; c < g.ksize[1]; ++c)
        for (int d = 0; d < g.ksize[2]; ++d) {
          int oz, oy, ox;
          if (out_coord(g, z, y, x, a, c, d, oz, oy, ox))
            table_insert(t, lin_key(b, oz, oy, ox, g.out_spatial), 0, err);
        }
  }
}

__global__ void collect_keys(Table t, unsigned long long *out, int *count) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < t.cap;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const unsigned long long k = t.keys[i];
    if (k != ~0ull) out[atomicAdd(count, 1)] = k;
  }
}

__global__ void decode_and_insert(const unsigned long long *keys, int64_t n_out, Geom g, Table t,
                                  int32_t *out_coords, int *err) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n_out;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    long long k = static_cast<long long>(keys[i]);
    const int x = static_cast<int>(k % g.out_spatial[2]);
    k /= g.out_spatial[2];
    const int y = static_cast<int>(k % g.out_spatial[1]);
    k /= g.out_spatial[1];
    const int z = static_cast<int>(k % g.out_spatial[0]);
    const int b = static_cast<int>(k / g.out_spatial[0]);
    out_coords[i * 4] = b;
    out_coords[i * 4 + 1] = z;
    out_coords[i * 4 + 2] = y;
    out_coords[i * 4 + 3] = x;
    table_insert(t, static_cast<long long>(keys[i]), static_cast<int>(i), err);
  }
}

__global__ void conv_pairs_kernel(const int32_t *coords, int64_t n, int64_t n_out, Geom g, Table t,
                                  int32_t *pairs_fwd, int32_t *pairs_bwd, uint32_t *mask_fwd,
                                  uint32_t *mask_bwd) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int b = coords[i * 4], z = coords[i * 4 + 1], y = coords[i * 4 + 2],
              x = coords[i * 4 + 3];
    uint32_t m = 0;
    int k = 0;
    for (int a = 0; a < g.ksize[0]; ++a)
      for (int c = 0; c < g.ksize[1]; ++c)
        for (int d = 0; d < g.ksize[2]; ++d, ++k) {
          int oz, oy, ox;
          int o = -1;
          if (out_coord(g, z, y, x, a, c, d, oz, oy, ox))
            o = table_lookup(t, lin_key(b, oz, oy, ox, g.out_spatial));
          pairs_bwd[static_cast<int64_t>(k) * n + i] = o;
          if (o >= 0) {
            m |= 1u << k;
            pairs_fwd[static_cast<int64_t>(k) * n_out + o] = static_cast<int>(i);
            atomicOr(mask_fwd + o, 1u << k);
          }
        }
    mask_bwd[i] = m;
  }
}

// ------------------------------------------------------------------ stable LSD radix sort
// 8-bit digits; each pass: per-tile digit histograms, one exclusive scan,
// then an order-preserving scatter (tiles of 4096 items, 8 warps x 512).
constexpr int kSortTile = 4096;
constexpr int kSortWarps = 8;

template <typename K>
__global__ void radix_hist(const K *keys, int64_t n, int shift, uint32_t *hist, int nblocks) {
  __shared__ uint32_t h[256];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) h[i] = 0;
  __syncthreads();
  const int64_t base = static_cast<int64_t>(blockIdx.x) * kSortTile;
  for (int i = threadIdx.x; i < kSortTile; i += blockDim.x) {
    const int64_t j = base + i;
    if (j < n) atomicAdd(&h[(keys[j] >> shift) & 255u], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 256; i += blockDim.x)
    hist[static_cast<int64_t>(i) * nblocks + blockIdx.x] = h[i];
}

// single-block exclusive scan of `n` uint32 in place
__global__ void scan_exclusive(uint32_t *a, int64_t n) {
  __shared__ uint32_t warp_sums[32];
  __shared__ uint32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int64_t base = 0; base < n; base += blockDim.x) {
    const int64_t i = base + threadIdx.x;
    uint32_t v = i < n ? a[i] : 0u;
    uint32_t x = v;
#pragma unroll
    for (int s = 1; s < 32; s <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, s);
      if (lane >= s) x += y;
    }
    if (lane == 31) warp_sums[w] = x;
    __syncthreads();
    if (w == 0) {
      uint32_t ws = lane < static_cast<int>(blockDim.x >> 5) ? warp_sums[lane] : 0u;
#pragma unroll
      for (int s = 1; s < 32; s <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, ws, s);
        if (lane >= s) ws += y;
      }
      warp_sums[lane] = ws;
    }
    __syncthreads();
    const uint32_t prefix = (w > 0 ? warp_sums[w - 1] : 0u) + carry;
    if (i < n) a[i] = prefix + x - v;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = prefix + x;
    __syncthreads();
  }
}

template <typename K>
__global__ void radix_scatter(const K *keys, const int32_t *vals, K *keys_out, int32_t *vals_out,
                              int64_t n, int shift, const uint32_t *hist, int nblocks) {
  __shared__ uint32_t wh[kSortWarps][256];
  __shared__ uint32_t base_off[256];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t tile0 = static_cast<int64_t>(blockIdx.x) * kSortTile;
  const int per_warp = kSortTile / kSortWarps;
  const int64_t w0 = tile0 + static_cast<int64_t>(w) * per_warp;
  for (int i = lane; i < 256; i += 32) wh[w][i] = 0;
  __syncwarp();
  for (int i = lane; i < per_warp; i += 32) {
    const int64_t j = w0 + i;
    if (j < n) atomicAdd(&wh[w][(keys[j] >> shift) & 255u], 1u);
  }
  __syncthreads();
  // exclusive prefix over warps per digit, plus the global base of this tile
  for (int d = threadIdx.x; d < 256; d += blockDim.x) {
    uint32_t run = hist[static_cast<int64_t>(d) * nblocks + blockIdx.x];
    for (int ww = 0; ww < kSortWarps; ++ww) {
      const uint32_t c = wh[ww][d];
      wh[ww][d] = run;
      run += c;
    }
    base_off[d] = 0;
  }
  __syncthreads();
  const unsigned lt = (1u << lane) - 1u;
  for (int i = 0; i < per_warp; i += 32) {
    const int64_t j = w0 + i + lane;
    const bool v = j < n;
    const uint32_t d = v ? static_cast<uint32_t>((keys[j] >> shift) & 255u) : 256u + lane;
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const uint32_t rank = __popc(peers & lt);
    uint32_t pos = 0;
    if (v) pos = wh[w][d] + rank;
    __syncwarp();
    if (v && rank == 0) wh[w][d] += __popc(peers);
    __syncwarp();
    if (v) {
      keys_out[pos] = keys[j];
      vals_out[pos] = vals[j];
    }
  }
}

__global__ void iota_kernel(int32_t *p, int64_t n) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    p[i] = static_cast<int32_t>(i);
}

__global__ void masked_keys(const uint32_t *data, uint32_t *keys, int64_t n, uint32_t m) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    keys[i] = data[i] & m;
}

__global__ void permute_u32(const uint32_t *src, const int32_t *perm, uint32_t *dst, int64_t n) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    dst[i] = src[perm[i]];
}

inline int grid_for(int64_t n) {
  int64_t b = (n + kThreads - 1) / kThreads;
  if (b > 65535) b = 65535;
  if (b < 1) b = 1;
  return static_cast<int>(b);
}

int64_t align_up(int64_t x) { return (x + 255) & ~static_cast<int64_t>(255); }

int64_t radix_ws_bytes(int64_t n, int key_bytes) {
  const int64_t nblocks = (n + kSortTile - 1) / kSortTile;
  return align_up(n * key_bytes) + align_up(n * 4) + align_up(256 * nblocks * 4);
}

// Sorts (keys, vals) stably by the low `bits` bits of the keys.  The sorted
// result ends in (keys, vals) again.  ws: radix_ws_bytes(n, sizeof(K)).
template <typename K>
cudaError_t radix_sort(K *keys, int32_t *vals, int64_t n, int bits, uint8_t *ws,
                       cudaStream_t s) {
  if (n <= 1) return cudaSuccess;
  const int nblocks = static_cast<int>((n + kSortTile - 1) / kSortTile);
  K *k2 = reinterpret_cast<K *>(ws);
  int32_t *v2 = reinterpret_cast<int32_t *>(ws + align_up(n * sizeof(K)));
  uint32_t *hist = reinterpret_cast<uint32_t *>(ws + align_up(n * sizeof(K)) + align_up(n * 4));
  K *src_k = keys, *dst_k = k2;
  int32_t *src_v = vals, *dst_v = v2;
  int passes = (bits + 7) / 8;
  if (passes < 1) passes = 1;
  for (int p = 0; p < passes; ++p) {
    const int shift = 8 * p;
    radix_hist<K><<<nblocks, 256, 0, s>>>(src_k, n, shift, hist, nblocks);
    scan_exclusive<<<1, 1024, 0, s>>>(hist, static_cast<int64_t>(256) * nblocks);
    radix_scatter<K><<<nblocks, 32 * kSortWarps, 0, s>>>(src_k, src_v, dst_k, dst_v, n, shift,
                                                         hist, nblocks);
    K *tk = src_k; src_k = dst_k; dst_k = tk;
    int32_t *tv = src_v; src_v = dst_v; dst_v = tv;
  }
  if (src_k != keys) {
    cudaMemcpyAsync(keys, src_k, n * sizeof(K), cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(vals, src_v, n * 4, cudaMemcpyDeviceToDevice, s);
  }
  return cudaGetLastError();
}

int64_t next_pow2(int64_t x) {
  int64_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

Geom make_geom(const PairBuildArgs &a) {
  Geom g;
  for (int d = 0; d < 3; ++d) {
    g.spatial[d] = a.spatial[d];
    g.ksize[d] = a.ksize[d];
    g.stride[d] = a.stride[d];
    g.padding[d] = a.padding[d];
    g.dilation[d] = a.dilation[d];
    g.out_spatial[d] = a.out_spatial[d];
  }
  g.kv = a.ksize[0] * a.ksize[1] * a.ksize[2];
  return g;
}

struct ConvWs {
  Table set;                   // output key set (no values), later output index table
  unsigned long long *ukeys;   // unique keys
  int32_t *uvals;
  int *counter;
  uint8_t *sort_ws;
};

}  // namespace

int64_t pairs_workspace_bytes(int64_t n_in, int kv, int subm) {
  if (subm) {
    const int64_t cap = next_pow2(2 * (n_in > 0 ? n_in : 1));
    return align_up(cap * 8) + align_up(cap * 4) + 256;
  }
  // strided: kv bounds outputs_per_input from above
  const int64_t max_out = n_in * kv;
  const int64_t cap = next_pow2(2 * (max_out > 0 ? max_out : 1));
  return align_up(cap * 8) + align_up(cap * 4) + align_up(max_out * 8) + align_up(max_out * 4) +
         256 + radix_ws_bytes(max_out, 8);
}

static ConvWs carve_conv_ws(void *ws, int64_t n_in, int kv) {
  ConvWs w;
  const int64_t max_out = n_in * kv;
  const int64_t cap = next_pow2(2 * (max_out > 0 ? max_out : 1));
  uint8_t *p = static_cast<uint8_t *>(ws);
  w.set.keys = reinterpret_cast<unsigned long long *>(p);
  p += align_up(cap * 8);
  w.set.vals = reinterpret_cast<int *>(p);
  p += align_up(cap * 4);
  w.set.cap = cap;
  w.ukeys = reinterpret_cast<unsigned long long *>(p);
  p += align_up(max_out * 8);
  w.uvals = reinterpret_cast<int32_t *>(p);
  p += align_up(max_out * 4);
  w.counter = reinterpret_cast<int *>(p);
  p += 256;
  w.sort_ws = p;
  return w;
}

cudaError_t build_subm_pairs(const PairBuildArgs &a, int32_t *pairs_fwd, int32_t *pairs_bwd,
                             uint32_t *mask_fwd, void *ws, int64_t ws_bytes, cudaStream_t s) {
  const Geom g = make_geom(a);
  const int64_t n = a.n_in;
  if (n == 0) return cudaSuccess;
  Table t;
  t.cap = next_pow2(2 * n);
  uint8_t *p = static_cast<uint8_t *>(ws);
  t.keys = reinterpret_cast<unsigned long long *>(p);
  t.vals = reinterpret_cast<int *>(p + align_up(t.cap * 8));
  if (ws_bytes < pairs_workspace_bytes(n, g.kv, 1)) return cudaErrorInvalidValue;
  table_clear<<<grid_for(t.cap), kThreads, 0, s>>>(t);
  insert_coords<<<grid_for(n), kThreads, 0, s>>>(a.coords, n, g, t, a.err);
  fill_i32<<<grid_for(n * g.kv), kThreads, 0, s>>>(pairs_bwd, n * g.kv, -1);
  subm_pairs_kernel<<<grid_for(n), kThreads, 0, s>>>(a.coords, n, g, t, pairs_fwd, pairs_bwd,
                                                     mask_fwd);
  return cudaGetLastError();
}

cudaError_t build_conv_outputs(const PairBuildArgs &a, int64_t *n_out, void *ws, int64_t ws_bytes,
                               cudaStream_t s) {
  const Geom g = make_geom(a);
  const int64_t n = a.n_in;
  *n_out = 0;
  if (n == 0) return cudaSuccess;
  if (ws_bytes < pairs_workspace_bytes(n, g.kv, 0)) return cudaErrorInvalidValue;
  ConvWs w = carve_conv_ws(ws, n, g.kv);
  Table set = w.set;
  table_clear<<<grid_for(set.cap), kThreads, 0, s>>>(set);
  cudaMemsetAsync(w.counter, 0, 4, s);
  Table keys_only = set;
  keys_only.vals = nullptr;
  conv_candidates<<<grid_for(n), kThreads, 0, s>>>(a.coords, n, g, keys_only, a.err);
  collect_keys<<<grid_for(set.cap), kThreads, 0, s>>>(set, w.ukeys, w.counter);
  int count = 0;
  cudaError_t e = cudaMemcpyAsync(&count, w.counter, 4, cudaMemcpyDeviceToHost, s);
  if (e != cudaSuccess) return e;
  e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return e;
  const long long total = static_cast<long long>(a.batch) * g.out_spatial[0] * g.out_spatial[1] *
                          g.out_spatial[2];
  int bits = 1;
  while (bits < 63 && (1ll << bits) < total) ++bits;
  iota_kernel<<<grid_for(count), kThreads, 0, s>>>(w.uvals, count);
  e = radix_sort<unsigned long long>(w.ukeys, w.uvals, count, bits, w.sort_ws, s);
  if (e != cudaSuccess) return e;
  *n_out = count;
  return cudaGetLastError();
}

cudaError_t build_conv_pairs(const PairBuildArgs &a, int64_t n_out, int32_t *out_coords,
                             int32_t *pairs_fwd, int32_t *pairs_bwd, uint32_t *mask_fwd,
                             uint32_t *mask_bwd, void *ws, int64_t ws_bytes, cudaStream_t s) {
  const Geom g = make_geom(a);
  const int64_t n = a.n_in;
  if (n == 0) return cudaSuccess;
  if (ws_bytes < pairs_workspace_bytes(n, g.kv, 0)) return cudaErrorInvalidValue;
  ConvWs w = carve_conv_ws(ws, n, g.kv);
  Table t = w.set;
  table_clear<<<grid_for(t.cap), kThreads, 0, s>>>(t);
  decode_and_insert<<<grid_for(n_out), kThreads, 0, s>>>(w.ukeys, n_out, g, t, out_coords, a.err);
  fill_i32<<<grid_for(n_out * g.kv), kThreads, 0, s>>>(pairs_fwd, n_out * g.kv, -1);
  cudaMemsetAsync(mask_fwd, 0, n_out * 4, s);
  conv_pairs_kernel<<<grid_for(n), kThreads, 0, s>>>(a.coords, n, n_out, g, t, pairs_fwd,
                                                     pairs_bwd, mask_fwd, mask_bwd);
  return cudaGetLastError();
}

namespace {
__global__ void sort_indices_kernel(const int32_t *indices, int kv, int64_t n,
                                    const int32_t *argsort, int32_t *out, int *err) {
  const int64_t total = static_cast<int64_t>(kv) * n;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t k = i / n, r = i % n;
    const int sig = argsort[r];
    out[i] = (sig >= 0 && sig < n) ? indices[k * n + sig] : -1;
  }
}
}  // namespace

cudaError_t sort_indices(const int32_t *indices, int kv, int64_t n, const int32_t *argsort,
                         int32_t *out, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  sort_indices_kernel<<<grid_for(static_cast<int64_t>(kv) * n), kThreads, 0, s>>>(
      indices, kv, n, argsort, out, nullptr);
  return cudaGetLastError();
}

int64_t sort_workspace_bytes(int64_t n) { return align_up(n * 4) + radix_ws_bytes(n, 4); }

cudaError_t sort_masks_split(uint32_t *data, int64_t n, uint32_t split_mask, int32_t *argsort,
                             void *ws, int64_t ws_bytes, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  if (ws_bytes < sort_workspace_bytes(n)) return cudaErrorInvalidValue;
  uint8_t *p = static_cast<uint8_t *>(ws);
  uint32_t *keys = reinterpret_cast<uint32_t *>(p);
  uint8_t *rws = p + align_up(n * 4);
  masked_keys<<<grid_for(n), kThreads, 0, s>>>(data, keys, n, split_mask);
  iota_kernel<<<grid_for(n), kThreads, 0, s>>>(argsort, n);
  const int bits = split_mask == 0 ? 1 : 32 - __builtin_clz(split_mask);
  cudaError_t e = radix_sort<uint32_t>(keys, argsort, n, bits, rws, s);
  if (e != cudaSuccess) return e;
  // data <- data[argsort] (full masks, sorted by their masked key); keys buffer
  // is free again and holds the copy
  cudaMemcpyAsync(keys, data, n * 4, cudaMemcpyDeviceToDevice, s);
  permute_u32<<<grid_for(n), kThreads, 0, s>>>(keys, argsort, data, n);
  return cudaGetLastError();
}

}  // namespace scb
