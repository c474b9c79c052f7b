// gather.cu - standalone row gather and row scatter-add.
//
// Semantics follow the reference's gather / scatter kernels
// (cumm/gemm/gather.py:29-390, iterators cumm/gemm/frozen/mask_iters.py):
//   gather:      out[i, :] = in[indices[i], :]            i < m
//   scatter-add: out[indices[i], :] += in[i, :]           i < m
// Rows are row_bytes long and moved in bytes_per_access units (4, 8 or 16
// bytes, the reference's access widths).  Like the reference, scatter-add is a
// plain read-add-write per row, so the indices of one call must be distinct.
// Additions to the reference's contract: index -1 writes a zero row (gather)
// or leaves the row alone (scatter); any other index outside the table is
// reported in the device error word (bit 1) and treated like -1 instead of
// being read or written out of bounds.
//
// B200 design: these are HBM copies (no reuse, no arithmetic to speak of), so
// the kernel keeps many independent 16-byte accesses in flight: a row is
// covered by `tpr` consecutive lanes (a 128-byte row by 8 lanes, so every
// warp access is four whole 128-byte lines), each thread handles kRows rows
// per iteration with all loads issued before any store, and the grid is a
// whole number of waves over the SMs.
#include "kernels.h"

namespace scb {
namespace {

constexpr int kRows = 4;  // rows in flight per thread

template <int VB>
struct Vec;
template <> struct Vec<4> { using T = uint32_t; };
template <> struct Vec<8> { using T = uint2; };
template <> struct Vec<16> { using T = uint4; };

template <int VB>
__device__ __forceinline__ typename Vec<VB>::T ld_nc(const uint8_t *p) {
  using T = typename Vec<VB>::T;
  return __ldg(reinterpret_cast<const T *>(p));
}

template <int VB>
__device__ __forceinline__ typename Vec<VB>::T zero_vec() {
  using T = typename Vec<VB>::T;
  T z;
  memset(&z, 0, sizeof(T));
  return z;
}

// Loads an index and checks it: -1 (and any invalid value, which also sets
// the error bit) comes back as -1.
__device__ __forceinline__ int64_t checked_index(const int32_t *indices, int64_t i, int64_t rows,
                                                 int *err) {
  const int v = __ldg(indices + i);
  if (v == -1) return -1;
  if (v < 0 || v >= rows) {
    atomicOr(err, kErrBadIndex);
    return -1;
  }
  return v;
}

template <int VB>
__global__ void __launch_bounds__(256) gather_rows_kernel(uint8_t *__restrict__ out,
                                                          const uint8_t *__restrict__ in, int64_t in_rows,
                                                          const int32_t *__restrict__ indices, int64_t m,
                                                          int64_t row_bytes, int tpr, int *err) {
  using T = typename Vec<VB>::T;
  const int64_t upr = row_bytes / VB;                       // units per row
  const int lane_u = threadIdx.x % tpr;                     // unit column of this thread
  const int64_t rows_per_block = blockDim.x / tpr;
  const int64_t row0 = static_cast<int64_t>(blockIdx.x) * rows_per_block * kRows + threadIdx.x / tpr;
  const int64_t row_step = static_cast<int64_t>(gridDim.x) * rows_per_block * kRows;
  for (int64_t base = row0; base < m; base += row_step) {
    int64_t src[kRows];
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
      const int64_t i = base + r * rows_per_block;
      src[r] = i < m ? checked_index(indices, i, in_rows, err) : -1;
    }
    for (int64_t u = lane_u; u < upr; u += tpr) {
      T v[kRows];
#pragma unroll
      for (int r = 0; r < kRows; ++r)
        v[r] = src[r] >= 0 ? ld_nc<VB>(in + src[r] * row_bytes + u * VB) : zero_vec<VB>();
#pragma unroll
      for (int r = 0; r < kRows; ++r) {
        const int64_t i = base + r * rows_per_block;
        if (i < m) *reinterpret_cast<T *>(out + i * row_bytes + u * VB) = v[r];
      }
    }
  }
}

template <typename E>
__device__ __forceinline__ void add_units(uint32_t &o, uint32_t a) {
  if constexpr (sizeof(E) == 4) {
    o = __float_as_uint(__uint_as_float(o) + __uint_as_float(a));
  } else {
    E x[2], y[2];
    memcpy(x, &o, 4);
    memcpy(y, &a, 4);
#pragma unroll
    for (int j = 0; j < 2; ++j) x[j] = from_f32<E>(to_f32(x[j]) + to_f32(y[j]));
    memcpy(&o, x, 4);
  }
}

template <int VB, typename E>
__global__ void __launch_bounds__(256) scatter_add_rows_kernel(uint8_t *__restrict__ out, int64_t out_rows,
                                                               const uint8_t *__restrict__ in,
                                                               const int32_t *__restrict__ indices, int64_t m,
                                                               int64_t row_bytes, int tpr, int *err) {
  using T = typename Vec<VB>::T;
  constexpr int kWords = VB / 4;
  const int64_t upr = row_bytes / VB;
  const int lane_u = threadIdx.x % tpr;
  const int64_t rows_per_block = blockDim.x / tpr;
  const int64_t row0 = static_cast<int64_t>(blockIdx.x) * rows_per_block * kRows + threadIdx.x / tpr;
  const int64_t row_step = static_cast<int64_t>(gridDim.x) * rows_per_block * kRows;
  for (int64_t base = row0; base < m; base += row_step) {
    int64_t dst[kRows];
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
      const int64_t i = base + r * rows_per_block;
      dst[r] = i < m ? checked_index(indices, i, out_rows, err) : -1;
    }
    for (int64_t u = lane_u; u < upr; u += tpr) {
      T a[kRows], o[kRows];
#pragma unroll
      for (int r = 0; r < kRows; ++r) {
        const int64_t i = base + r * rows_per_block;
        if (dst[r] >= 0) {
          a[r] = ld_nc<VB>(in + i * row_bytes + u * VB);
          o[r] = *reinterpret_cast<const T *>(out + dst[r] * row_bytes + u * VB);
        }
      }
#pragma unroll
      for (int r = 0; r < kRows; ++r) {
        if (dst[r] < 0) continue;
        uint32_t *ow = reinterpret_cast<uint32_t *>(&o[r]);
        const uint32_t *aw = reinterpret_cast<const uint32_t *>(&a[r]);
#pragma unroll
        for (int w = 0; w < kWords; ++w) add_units<E>(ow[w], aw[w]);
        *reinterpret_cast<T *>(out + dst[r] * row_bytes + u * VB) = o[r];
      }
    }
  }
}

// Threads per row: enough lanes to cover the row's units, a power of two,
// at most a warp.
int threads_per_row(int64_t upr) {
  int t = 1;
  while (t < upr && t < 32) t <<= 1;
  return t;
}

int grid_for(int64_t m, int threads, int tpr, int num_sms) {
  const int64_t rows_per_block = threads / tpr;
  const int64_t blocks = (m + rows_per_block * kRows - 1) / (rows_per_block * kRows);
  // at most 8 waves of 2048 / threads blocks per SM
  const int64_t cap = static_cast<int64_t>(num_sms) * (2048 / threads) * 8;
  return static_cast<int>(blocks < cap ? (blocks > 0 ? blocks : 1) : cap);
}

}  // namespace

cudaError_t launch_gather_rows(void *out, const void *in, int64_t in_rows, const int32_t *indices,
                               int64_t m, int64_t row_bytes, int bytes_per_access, int threads,
                               int num_sms, int *err, cudaStream_t s) {
  if (m == 0 || row_bytes == 0) return cudaSuccess;
  const int tpr = threads_per_row(row_bytes / bytes_per_access);
  const int grid = grid_for(m, threads, tpr, num_sms);
  auto *o = static_cast<uint8_t *>(out);
  const auto *i = static_cast<const uint8_t *>(in);
  switch (bytes_per_access) {
    case 16: gather_rows_kernel<16><<<grid, threads, 0, s>>>(o, i, in_rows, indices, m, row_bytes, tpr, err); break;
    case 8: gather_rows_kernel<8><<<grid, threads, 0, s>>>(o, i, in_rows, indices, m, row_bytes, tpr, err); break;
    case 4: gather_rows_kernel<4><<<grid, threads, 0, s>>>(o, i, in_rows, indices, m, row_bytes, tpr, err); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_scatter_add_rows(void *out, int64_t out_rows, const void *in, const int32_t *indices,
                                    int64_t m, int64_t channels, int dtype, int bytes_per_access,
                                    int threads, int num_sms, int *err, cudaStream_t s) {
  const int es = dtype == 0 ? 4 : 2;
  const int64_t row_bytes = channels * es;
  if (m == 0 || row_bytes == 0) return cudaSuccess;
  const int tpr = threads_per_row(row_bytes / bytes_per_access);
  const int grid = grid_for(m, threads, tpr, num_sms);
  auto *o = static_cast<uint8_t *>(out);
  const auto *i = static_cast<const uint8_t *>(in);
#define SCB_SCATTER(VB, E)                                                                         \
  scatter_add_rows_kernel<VB, E><<<grid, threads, 0, s>>>(o, out_rows, i, indices, m, row_bytes, tpr, err)
#define SCB_SCATTER_VB(E)                  \
  switch (bytes_per_access) {              \
    case 16: SCB_SCATTER(16, E); break;    \
    case 8: SCB_SCATTER(8, E); break;      \
    case 4: SCB_SCATTER(4, E); break;      \
    default: return cudaErrorInvalidValue; \
  }
  switch (dtype) {
    case 0: SCB_SCATTER_VB(float); break;
    case 7: SCB_SCATTER_VB(__half); break;
    case 12: SCB_SCATTER_VB(__nv_bfloat16); break;
    default: return cudaErrorInvalidValue;
  }
#undef SCB_SCATTER_VB
#undef SCB_SCATTER
  return cudaGetLastError();
}

}  // namespace scb
