// api.cu - the C ABI (include/cumm_b200.h): argument validation, workspace
// sizing and kernel dispatch for the sparse convolution and GEMM entry points.
//
// Validation mirrors the reference prologues (cumm/conv/nvrtc_code.py:20-196,
// cumm/gemm/nvrtc_code.py:34-140): shape / dtype checks raise SC_INVALID_ARG
// or SC_RUNTIME with the reference's wording where one exists; a configuration
// no kernel covers reports "Can't Found Algorithm" (cumm/conv/main.py:733-744).
// Unlike the reference (which allocates missing workspaces with tv::empty,
// nvrtc_code.py:181-196) this library never allocates: callers query the size
// and pass the buffer.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/cumm_b200.h"
#include "kernels.h"

namespace {

thread_local std::string g_last_error;

__device__ int g_device_error_word[1];

constexpr int kMaxDevices = 64;
std::mutex g_dev_mu;
int *g_err_ptr[kMaxDevices] = {nullptr};
int g_num_sms[kMaxDevices] = {0};

int fail(int code, const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

int cuda_fail(cudaError_t e, const char *what) {
  return fail(SC_CUDA, "%s: CUDA error %d (%s)", what, static_cast<int>(e), cudaGetErrorString(e));
}

// Device-side error word and SM count of the current device (set up once per device).
int device_state(int **err, int *sms) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) return fail(SC_RUNTIME, "device index %d out of range", dev);
  std::lock_guard<std::mutex> lk(g_dev_mu);
  if (g_err_ptr[dev] == nullptr) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_device_error_word);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(error word)");
    int n = 0;
    e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute");
    g_err_ptr[dev] = static_cast<int *>(p);
    g_num_sms[dev] = n;
  }
  *err = g_err_ptr[dev];
  *sms = g_num_sms[dev];
  return SC_OK;
}

int esize(int dt) {
  switch (dt) {
    case SC_FLOAT32: return 4;
    case SC_FLOAT16: return 2;
    case SC_BFLOAT16: return 2;
    case SC_FLOAT_E4M3: return 1;
    default: return 0;
  }
}

const char *dtype_name(int dt) {
  switch (dt) {
    case SC_FLOAT32: return "float32";
    case SC_FLOAT16: return "float16";
    case SC_BFLOAT16: return "bfloat16";
    case SC_FLOAT_E4M3: return "float_e4m3";
    case SC_INT32: return "int32";
    default: return "unknown";
  }
}

int sync_check(cudaStream_t s) {
  int32_t bits = 0;
  int rc = sc_check_device_error(s, &bits);
  if (rc != SC_OK) return rc;
  if (bits) return fail(SC_DEVICE, "device error word 0x%x (1 bad index, 2 wait timeout, 4 hash full)", bits);
  return SC_OK;
}

bool is16(int dt) { return dt == SC_BFLOAT16 || dt == SC_FLOAT16; }

// The tensor-core kernels move whole 16-byte units (TMA boxes and gathers,
// 16-byte cp.async, uint4 / float4 epilogue loads and stores, v4 reductions).
bool aligned16(const void *q) { return reinterpret_cast<uintptr_t>(q) % 16 == 0; }

int64_t align256(int64_t x) { return (x + 255) & ~static_cast<int64_t>(255); }

// Reduction row width accepted by the row-gather kernel (bytes per offset).
bool rowgather_width_ok(int64_t bytes) {
  if (bytes % 16) return false;
  return bytes >= 128 || bytes == 16 || bytes == 32 || bytes == 64;
}

struct ConvPlan {
  bool simt = false;
  int64_t ws_bytes = 0;  // what sc_conv_workspace_size reports
  int64_t ws_min = 0;    // what a call cannot run without
};

// Workspace of the tcgen05 forward / backward-input kernels: a 256-byte head
// (the tile counter of the row-gather kernel's dynamic scheduler, zeroed per
// call), for backward-input without an MN-major weight the transposed
// [C, kv, K] weight, and, when the caller gives no indices_sorted and the
// strand kernel can take the layer, the index table permuted into argsort
// order (kv x N int32) that this call writes itself.
constexpr int64_t kSchedBytes = 256;

// Output-column tile of the tcgen05 forward / backward-input kernels.
int64_t column_tile(int64_t ncols, int32_t tile_n) {
  if (tile_n > 0) return tile_n;
  int64_t bn = ncols;
  int tiles = 1;
  while (bn > 256 || bn % 16) {
    ++tiles;
    while (ncols % tiles || (ncols / tiles) % 16) ++tiles;
    bn = ncols / tiles;
  }
  return bn;
}

// Bytes of the sorted index table a forward / backward-input call builds for
// the strand kernel when the caller passes none (0 when the strand kernel
// would not take the layer: rows of 64 bytes or whole 128-byte blocks,
// column tile <= 64, N % 4 == 0).  Building it costs one gather of kv x N
// ints; the strand kernel then runs ~2x faster than the row-gather kernel
// reading the unsorted table through the argsort.
int64_t own_sorted_bytes(const sc_conv_params *p, int es) {
  if (p->indices_sorted != nullptr || p->N <= 0 || p->N % 4 != 0) return 0;
  const bool fwd = p->op_type == SC_CONV_FORWARD;
  const int64_t rb = (fwd ? p->C : p->K) * es;
  const int64_t ncols = fwd ? p->K : p->C;
  if (!((rb == 64 && p->kv > 1) || (rb >= 128 && rb % 128 == 0))) return 0;
  if (column_tile(ncols, p->tile_n) > 64) return 0;
  return align256(static_cast<int64_t>(p->kv) * p->N * 4);
}

int plan_conv(const sc_conv_params *p, ConvPlan *plan) {
  if (p == nullptr) return fail(SC_INVALID_ARG, "params is null");
  const int op = p->op_type;
  if (op < 0 || op > 2) return fail(SC_RUNTIME, "unknown op type %d", op);
  if (p->kv < 1 || p->kv > 32)
    return fail(SC_RUNTIME, "kernel volume %d not supported (1..32; dynamic masks are out of scope)", p->kv);
  if (p->indices == nullptr) return fail(SC_RUNTIME, "error: indices must not be empty");
  if (p->mask == nullptr) return fail(SC_RUNTIME, "error: mask must not be empty");
  if (p->mask_argsort == nullptr) return fail(SC_RUNTIME, "error: mask_argsort must not be empty");
  if (p->input == nullptr || p->weight == nullptr || p->output == nullptr)
    return fail(SC_INVALID_ARG, "input, weight and output must not be empty");
  if (p->C <= 0 || p->K <= 0 || p->N < 0) return fail(SC_INVALID_ARG, "bad sizes C=%lld K=%lld N=%lld",
                                                      (long long)p->C, (long long)p->K, (long long)p->N);
  if (op == SC_CONV_FORWARD || op == SC_CONV_BACKWARD_WEIGHT) {
    if (p->N != p->n_out) return fail(SC_RUNTIME, "error: N (%lld) != output.dim(0) (%lld)",
                                      (long long)p->N, (long long)p->n_out);
  } else {
    if (p->N != p->n_in) return fail(SC_RUNTIME, "error: N (%lld) != input.dim(0) (%lld)",
                                     (long long)p->N, (long long)p->n_in);
  }
  if (op == SC_CONV_BACKWARD_WEIGHT) {
    if (p->mask_width <= 0 || p->tile_k <= 0 || p->mask_width % p->tile_k)
      return fail(SC_RUNTIME, "error: mask_width (%d) must be > 0 and a multiple of tile_shape[2] (%d)",
                  p->mask_width, p->tile_k);
    const int64_t need = (p->N + p->mask_width - 1) / p->mask_width;
    if (p->mask_count < need)
      return fail(SC_RUNTIME, "error: mask.dim(0) (%lld) < num_reduced_mask (%lld)",
                  (long long)p->mask_count, (long long)need);
  } else {
    if (p->mask_count < p->N)
      return fail(SC_INVALID_ARG, "mask has %lld entries, needs %lld", (long long)p->mask_count,
                  (long long)p->N);
    if (p->tile_m != 32 && p->tile_m != 64 && p->tile_m != 128)
      return fail(SC_RUNTIME, "Can't Found Algorithm: tile_shape[0]=%d (supported 32, 64, 128)", p->tile_m);
    if (op == SC_CONV_FORWARD && p->mask_output != nullptr) {
      const int64_t need = (p->N + p->tile_m - 1) / p->tile_m;
      if (p->mask_output_count < need)
        return fail(SC_INVALID_ARG, "mask_output has %lld words, needs %lld",
                    (long long)p->mask_output_count, (long long)need);
    }
  }
  if (p->output_add != nullptr && p->scale == nullptr)
    return fail(SC_INVALID_ARG, "only int8 inference support output_add not empty ");
  if (p->split_k_slices > 1 && op != SC_CONV_BACKWARD_WEIGHT)
    return fail(SC_RUNTIME, "algo don't support splitk but you provide split_k_slices > 1. %d",
                p->split_k_slices);
  const int di = p->dtype_input, dw = p->dtype_weight, dout = p->dtype_output;
  if (p->algo == SC_ALGO_SIMT) {
    if (di != SC_FLOAT32 || dw != SC_FLOAT32 || dout != SC_FLOAT32)
      return fail(SC_RUNTIME, "Can't Found Algorithm: Simt kernels take float32 operands (%s %s %s)",
                  dtype_name(di), dtype_name(dw), dtype_name(dout));
    plan->simt = true;
    if (op == SC_CONV_BACKWARD_WEIGHT) plan->ws_bytes = plan->ws_min = align256(p->K * p->kv * p->C * 4);
    return SC_OK;
  }
  if (p->algo != SC_ALGO_TCGEN05) return fail(SC_RUNTIME, "Can't Found Algorithm: unknown algo %d", p->algo);
  // Every tensor a tcgen05 kernel reads or writes in 16-byte units must start
  // on a 16-byte boundary; a misaligned view is an argument error here rather
  // than a misaligned access on the device.  (Backward weight writes dW with
  // scalar stores unless it can accumulate into it directly, which checks
  // dW's alignment itself.)
  {
    const bool wg = op == SC_CONV_BACKWARD_WEIGHT;
    const void *need[5] = {p->input, p->output, wg ? nullptr : p->weight, p->bias, p->output_add};
    const char *names[5] = {"input", "output", "weight", "bias", "output_add"};
    for (int i = 0; i < 5; ++i)
      if (!aligned16(need[i]))
        return fail(SC_INVALID_ARG, "%s must start on a 16-byte boundary for the tcgen05 kernels (address %p)",
                    names[i], need[i]);
  }
  if (reinterpret_cast<uintptr_t>(p->tile_order) % 4 != 0)
    return fail(SC_INVALID_ARG, "tile_order must be 4-byte aligned (address %p)",
                static_cast<const void *>(p->tile_order));
  if (p->tile_n != 0 && op != SC_CONV_BACKWARD_WEIGHT) {
    const int64_t ncols = op == SC_CONV_FORWARD ? p->K : p->C;
    if (p->tile_n < 16 || p->tile_n > 256 || p->tile_n % 16 || ncols % p->tile_n)
      return fail(SC_INVALID_ARG, "tile_n %d must be a multiple of 16, <= 256, dividing %lld",
                  p->tile_n, (long long)ncols);
  }
  if (op == SC_CONV_FORWARD) {
    const bool f8 = di == SC_FLOAT_E4M3 && dw == SC_FLOAT_E4M3;
    const bool f16 = is16(di) && dw == di;
    if (!(f8 || f16) || !(dout == SC_FLOAT32 || is16(dout)) || (f16 && dout != di && dout != SC_FLOAT32))
      return fail(SC_RUNTIME, "Can't Found Algorithm for params: %s %s %s", dtype_name(di),
                  dtype_name(dw), dtype_name(dout));
    if (!rowgather_width_ok(p->C * esize(di)) || p->K % 16)
      return fail(SC_RUNTIME, "Can't Found Algorithm: C=%lld K=%lld not tiled by the tcgen05 kernel "
                  "(C*sizeof in {16,32,64} or a multiple of 16 >= 128 bytes; K %% 16 == 0)",
                  (long long)p->C, (long long)p->K);
    // optional: without it tiles are dealt statically and the unsorted table is read
    plan->ws_bytes = kSchedBytes + own_sorted_bytes(p, esize(di));
    return SC_OK;
  }
  if (op == SC_CONV_BACKWARD_INPUT) {
    if (!is16(di) || dw != di || dout != di)
      return fail(SC_RUNTIME, "Can't Found Algorithm for params: %s %s %s", dtype_name(di),
                  dtype_name(dw), dtype_name(dout));
    if (!rowgather_width_ok(p->K * esize(di)) || p->C % 16)
      return fail(SC_RUNTIME, "Can't Found Algorithm: K=%lld C=%lld not tiled by the tcgen05 kernel",
                  (long long)p->K, (long long)p->C);
    plan->ws_min = kSchedBytes + align256(p->K * p->kv * p->C * esize(di));
    plan->ws_bytes = plan->ws_min + own_sorted_bytes(p, esize(di));
    return SC_OK;
  }
  // backward weight
  if (!is16(di) || dout != di || !(dw == SC_BFLOAT16 || dw == SC_FLOAT32 || dw == SC_FLOAT16))
    return fail(SC_RUNTIME, "Can't Found Algorithm for params: %s %s %s", dtype_name(di),
                dtype_name(dw), dtype_name(dout));
  if (!(p->C % 64 == 0 || p->C == 8 || p->C == 16 || p->C == 32) || p->K % 8 || p->K > 256)
    return fail(SC_RUNTIME, "Can't Found Algorithm: C=%lld K=%lld not tiled by the tcgen05 wgrad kernel",
                (long long)p->C, (long long)p->K);
  plan->ws_bytes = align256(p->K * p->kv * p->C * 4);
  plan->ws_min = plan->ws_bytes;
  return SC_OK;
}

scb::EpiParams conv_epi(const sc_conv_params *p, int64_t out_cols) {
  scb::EpiParams e{};
  e.alpha = p->alpha;
  e.beta = p->beta;
  e.act_alpha = p->act_alpha;
  e.act_beta = p->act_beta;
  e.act_type = p->act_type;
  e.scale = p->scale;
  if (p->scale != nullptr) {
    e.mode = 1;
    e.bias = p->bias;
    if (p->output_add) {
      e.src = p->output_add;
      e.src_ld = out_cols;
    } else {
      e.src = nullptr;  // filled by the caller with the output
      e.src_ld = out_cols;
    }
  } else {
    e.mode = 0;
    e.bias = nullptr;
    if (p->bias) {
      e.src = p->bias;
      e.src_ld = 0;
    } else {
      e.src = nullptr;
      e.src_ld = out_cols;
    }
  }
  return e;
}

}  // namespace

extern "C" {

const char *sc_last_error(void) { return g_last_error.c_str(); }

const char *sc_version(void) { return "cumm_b200 0.1.0 (sm_100a)"; }

int sc_check_device_error(void *stream, int32_t *bits) {
  int *err = nullptr;
  int sms = 0;
  int rc = device_state(&err, &sms);
  if (rc != SC_OK) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(e, "cudaStreamSynchronize");
  int v = 0;
  e = cudaMemcpy(&v, err, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "read device error word");
  if (v) {
    const int zero = 0;
    e = cudaMemcpy(err, &zero, sizeof(int), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e, "clear device error word");
  }
  if (bits) *bits = v;
  return SC_OK;
}

int sc_conv_workspace_size(const sc_conv_params *p, int64_t *bytes) {
  ConvPlan plan;
  int rc = plan_conv(p, &plan);
  if (rc != SC_OK) return rc;
  *bytes = plan.ws_bytes;
  return SC_OK;
}

int sc_conv_implicit_gemm(const sc_conv_params *p) {
  g_last_error.clear();
  ConvPlan plan;
  int rc = plan_conv(p, &plan);
  if (rc != SC_OK) return rc;
  if (plan.ws_min > 0 && (p->workspace == nullptr || p->workspace_bytes < plan.ws_min))
    return fail(SC_RUNTIME, "workspace at least %lld bytes.", (long long)plan.ws_min);
  int *err = nullptr;
  int sms = 0;
  rc = device_state(&err, &sms);
  if (rc != SC_OK) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(p->stream);
  const int op = p->op_type;
  cudaError_t e = cudaSuccess;
  if (plan.simt) {
    scb::ConvSimtArgs a{};
    a.op = op;
    a.C = static_cast<int>(p->C);
    a.K = static_cast<int>(p->K);
    a.kv = p->kv;
    a.M = p->N;
    a.mask = p->mask;
    a.mask_count = p->mask_count;
    a.argsort = p->mask_argsort;
    a.indices = p->indices;
    a.mask_out = op == SC_CONV_FORWARD ? p->mask_output : nullptr;
    a.tile_m_desp = p->tile_m;
    a.mask_width = p->mask_width;
    a.mask_filter = p->mask_filter;
    a.reverse = p->reverse_mask;
    a.err = err;
    if (op == SC_CONV_FORWARD) {
      a.a = static_cast<const float *>(p->input);
      a.a_rows = p->n_in;
      a.b = static_cast<const float *>(p->weight);
      a.out = static_cast<float *>(p->output);
      a.epi = conv_epi(p, p->K);
      if (a.epi.src == nullptr) a.epi.src = p->output;
    } else if (op == SC_CONV_BACKWARD_INPUT) {
      a.a = static_cast<const float *>(p->output);
      a.a_rows = p->n_out;
      a.b = static_cast<const float *>(p->weight);
      a.out = static_cast<float *>(p->input);
      a.epi = conv_epi(p, p->C);
      if (a.epi.src == nullptr) a.epi.src = p->input;
    } else {
      a.a = static_cast<const float *>(p->output);
      a.a_rows = p->n_out;
      a.b = static_cast<const float *>(p->input);
      a.b_rows = p->n_in;
      a.out = static_cast<float *>(p->workspace);
      e = cudaMemsetAsync(p->workspace, 0, p->K * p->kv * p->C * 4, s);
      if (e != cudaSuccess) return cuda_fail(e, "zero workspace");
    }
    e = scb::launch_conv_simt(a, s);
    if (e != cudaSuccess) return cuda_fail(e, "conv_simt launch");
    if (op == SC_CONV_BACKWARD_WEIGHT) {
      scb::EpiParams ep{};
      ep.alpha = p->alpha;
      ep.beta = p->beta;
      ep.act_type = 0;
      ep.src = p->weight;
      ep.src_ld = p->kv * p->C;
      e = scb::launch_wgrad_finalize(static_cast<const float *>(p->workspace), p->weight,
                                     p->kv * p->C, SC_FLOAT32, static_cast<int>(p->K), p->kv,
                                     static_cast<int>(p->C), p->mask_filter, ep, s);
      if (e != cudaSuccess) return cuda_fail(e, "wgrad finalize launch");
    }
  } else if (op == SC_CONV_FORWARD || op == SC_CONV_BACKWARD_INPUT) {
    const bool fwd = op == SC_CONV_FORWARD;
    const int es = esize(p->dtype_input);
    const int64_t red = fwd ? p->C : p->K;    // reduction elements per offset
    const int64_t ncols = fwd ? p->K : p->C;  // output columns
    scb::ConvRowGatherArgs a{};
    uint8_t *ws = static_cast<uint8_t *>(p->workspace);
    // the tile counter in the workspace head (zeroed by the launcher); a
    // largest-first order only when the caller gives one (computing it per
    // call costs about what it saves)
    if (ws != nullptr && p->workspace_bytes >= kSchedBytes) a.tile_counter = reinterpret_cast<int *>(ws);
    if (p->tile_order != nullptr) {
      a.tile_order = p->tile_order;
      a.order_given = 1;
    }
    a.a_base = static_cast<const uint8_t *>(fwd ? p->input : p->output);
    a.a_rows = fwd ? p->n_in : p->n_out;
    a.a_row_bytes = static_cast<int>(red * es);
    a.a_row_stride = red * es;
    const int64_t bn = column_tile(ncols, p->tile_n);
    const int tiles = static_cast<int>(ncols / bn);
    // backward-input reads the weight MN-major when the slabs are whole
    // 64 x 64 boxes of 16-bit data, else from a transposed [C, kv, K] copy
    const bool b_mn = !fwd && es == 2 && red % 64 == 0 && bn % 64 == 0 && p->n_out > 0 &&
                      reinterpret_cast<uintptr_t>(p->weight) % 16 == 0;
    if (fwd || b_mn) {
      a.b_base = static_cast<const uint8_t *>(p->weight);
    } else {
      e = scb::launch_transpose_weight(p->weight, ws + kSchedBytes, static_cast<int>(p->K), p->kv,
                                       static_cast<int>(p->C), es, s);
      if (e != cudaSuccess) return cuda_fail(e, "weight transpose launch");
      a.b_base = ws + kSchedBytes;
    }
    a.b_mn = b_mn ? 1 : 0;
    // B rows: [n, kv, red] (K-major), or for b_mn the weight's [red, kv, n]
    a.b_row_stride = static_cast<int64_t>(p->kv) * (b_mn ? ncols : red) * es;
    a.b_off_stride = static_cast<int>((b_mn ? ncols : red) * es);
    a.n_total = static_cast<int>(ncols);
    a.BN = static_cast<int>(bn);
    a.n_tiles = tiles;
    a.M = p->N;
    a.kv = p->kv;
    a.mask = p->mask;
    a.argsort = p->mask_argsort;
    a.indices = p->indices;
    a.a_inds = nullptr;
    a.idx_sorted = p->indices_sorted;
    // no sorted table given: build one at the end of the workspace when the
    // strand kernel can take the layer (results are the same either way)
    const int64_t own = own_sorted_bytes(p, es);
    if (own > 0 && ws != nullptr && p->workspace_bytes >= plan.ws_bytes) {
      int32_t *tab = reinterpret_cast<int32_t *>(ws + plan.ws_bytes - own);
      e = scb::sort_indices(p->indices, p->kv, p->N, p->mask_argsort, tab, s);
      if (e != cudaSuccess) return cuda_fail(e, "sorted index table");
      a.idx_sorted = tab;
    }
    a.mask_out = fwd ? p->mask_output : nullptr;
    a.tile_m_desp = p->tile_m;
    a.mask_filter = p->mask_filter;
    a.reverse = (!fwd && p->reverse_mask) ? 1 : 0;
    a.is_fwd = fwd ? 1 : 0;
    a.out = fwd ? p->output : p->input;
    a.out_ld = ncols;
    a.out_rows = p->N;
    a.in_dtype = p->dtype_input;
    a.out_dtype = fwd ? p->dtype_output : p->dtype_input;
    a.epi = conv_epi(p, ncols);
    if (a.epi.src == nullptr) a.epi.src = a.out;
    a.err = err;
    e = scb::launch_conv_rowgather(a, sms, s);
    if (e != cudaSuccess) return cuda_fail(e, "conv row-gather launch");
  } else {
    // dW = 1 * sum with beta = 0 into an fp32 [K, kv, C] weight covering every
    // offset: the kernel accumulates straight into dW (bit-identical to the
    // workspace + finalize route, which computes alpha * ws with alpha = 1).
    // Its red.global.add.v4.f32 needs a 16-byte aligned dW; any other dW goes
    // through the workspace and the finalize kernel's scalar stores.
    const uint32_t all_offsets = p->kv >= 32 ? 0xffffffffu : ((1u << p->kv) - 1u);
    const bool direct = p->dtype_weight == SC_FLOAT32 && p->alpha == 1.f && p->beta == 0.f &&
                        (p->mask_filter & all_offsets) == all_offsets && aligned16(p->weight);
    float *acc = static_cast<float *>(direct ? p->weight : p->workspace);
    e = cudaMemsetAsync(acc, 0, p->K * p->kv * p->C * 4, s);
    if (e != cudaSuccess) return cuda_fail(e, "zero workspace");
    scb::ConvWgradArgs a{};
    a.dout = static_cast<const uint8_t *>(p->output);
    a.dout_rows = p->n_out;
    a.dout_ld = p->K;
    a.input = static_cast<const uint8_t *>(p->input);
    a.in_rows = p->n_in;
    a.in_ld = p->C;
    a.K = static_cast<int>(p->K);
    a.C = static_cast<int>(p->C);
    a.kv = p->kv;
    a.N = p->N;
    a.mask = p->mask;
    a.mask_count = p->mask_count;
    a.mask_width = p->mask_width;
    a.mask_filter = p->mask_filter;
    a.argsort = p->mask_argsort;
    a.indices = p->indices;
    a.ws = acc;
    a.err = err;
    a.b_inds = nullptr;
    a.idx_sorted = p->indices_sorted;
    a.in_dtype = p->dtype_input;
    a.split_k = p->split_k_slices > 1 ? p->split_k_slices : 0;
    e = scb::launch_conv_wgrad(a, sms, s);
    if (e != cudaSuccess) return cuda_fail(e, "conv wgrad launch");
    if (direct) {
      if (p->flags & SC_FLAG_SYNC_CHECK) return sync_check(s);
      return SC_OK;
    }
    scb::EpiParams ep{};
    ep.alpha = p->alpha;
    ep.beta = p->beta;
    ep.act_type = 0;
    ep.src = p->weight;
    ep.src_ld = p->kv * p->C;
    e = scb::launch_wgrad_finalize(static_cast<const float *>(p->workspace), p->weight,
                                   p->kv * p->C, p->dtype_weight, static_cast<int>(p->K), p->kv,
                                   static_cast<int>(p->C), p->mask_filter, ep, s);
    if (e != cudaSuccess) return cuda_fail(e, "wgrad finalize launch");
  }
  if (p->flags & SC_FLAG_SYNC_CHECK) return sync_check(s);
  return SC_OK;
}

// ------------------------------------------------ backward weight, static scratch
// The weight-gradient kernels accumulate into an fp32 [K, kv, C] buffer.  This
// entry point takes that buffer from a file-scope device array instead of the
// caller's workspace, so a caller with no device allocator still gets dW.
}  // extern "C"

namespace {
constexpr int64_t kStaticScratchFloats = int64_t(1) << 21;  // 8 MiB of fp32
static __device__ __align__(256) float g_wgrad_scratch[kStaticScratchFloats];
float *g_scratch_ptr[kMaxDevices] = {nullptr};

// Address of this device's copy of g_wgrad_scratch, looked up once per device
// (with that device current) and cached.  cudaDeviceReset after that first
// lookup is unsupported: the module would reload at another address.
int scratch_address(float **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) return fail(SC_RUNTIME, "device index %d out of range", dev);
  std::lock_guard<std::mutex> lk(g_dev_mu);
  if (g_scratch_ptr[dev] == nullptr) {
    void *ptr = nullptr;
    e = cudaGetSymbolAddress(&ptr, g_wgrad_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(wgrad scratch)");
    g_scratch_ptr[dev] = static_cast<float *>(ptr);
  }
  *out = g_scratch_ptr[dev];
  return SC_OK;
}
}  // namespace

extern "C" {

int sc_conv_wgrad_static_scratch(const sc_conv_params *p) {
  g_last_error.clear();
  if (p == nullptr) return fail(SC_INVALID_ARG, "params is null");
  if (p->op_type != SC_CONV_BACKWARD_WEIGHT)
    return fail(SC_INVALID_ARG, "sc_conv_wgrad_static_scratch runs backward weight only (op_type %d)",
                p->op_type);
  if (p->workspace != nullptr || p->workspace_bytes != 0)
    return fail(SC_INVALID_ARG, "sc_conv_wgrad_static_scratch takes no workspace (it uses its own scratch)");
  ConvPlan plan;
  int rc = plan_conv(p, &plan);
  if (rc != SC_OK) return rc;
  const int64_t floats = p->K * p->kv * p->C;
  if (floats > kStaticScratchFloats)
    return fail(SC_INVALID_ARG,
                "K*kv*C = %lld exceeds the static wgrad scratch of %lld floats (8 MiB); "
                "use sc_conv_implicit_gemm with a workspace",
                (long long)floats, (long long)kStaticScratchFloats);
  float *scratch = nullptr;
  rc = scratch_address(&scratch);
  if (rc != SC_OK) return rc;
  sc_conv_params q = *p;
  q.workspace = scratch;
  q.workspace_bytes = kStaticScratchFloats * 4;
  return sc_conv_implicit_gemm(&q);
}

// ------------------------------------------------------------------ GEMM
static int plan_gemm(const sc_gemm_params *p, scb::GemmArgs *a) {
  if (p == nullptr) return fail(SC_INVALID_ARG, "params is null");
  if (p->a == nullptr || p->b == nullptr || p->c == nullptr)
    return fail(SC_RUNTIME, "a,b,c must not empty");
  if (p->shuffle_type == SC_SHUFFLE_AC && p->c_inds == nullptr)
    return fail(SC_RUNTIME, "a_inds,c_inds tensor must not empty");
  if (p->shuffle_type == SC_SHUFFLE_AB && (p->a_inds == nullptr || p->b_inds == nullptr))
    return fail(SC_RUNTIME, "a_inds,b_inds tensor must not empty");
  if (p->shuffle_type == SC_SHUFFLE_AC && p->trans_a)
    return fail(SC_RUNTIME, "a of shuffle AB must be row major");
  if (p->shuffle_type == SC_SHUFFLE_AB && !(p->trans_a && !p->trans_b))
    return fail(SC_RUNTIME, "shuffle AB must be nt, i.e. backward weight");
  if (p->shuffle_type < 0 || p->shuffle_type > 2) return fail(SC_RUNTIME, "unknown shuffle type");
  if (p->split_k_slices > 1 && p->shuffle_type == SC_SHUFFLE_AC)
    return fail(SC_RUNTIME, "algo don't support splitk but you provide split_k_slices > 1. %d", p->split_k_slices);
  if (p->m < 0 || p->n < 0 || p->k < 0) return fail(SC_INVALID_ARG, "bad m, n, k");
  const int di = p->dtype_a;
  if (p->dtype_b != di) return fail(SC_RUNTIME, "Can't Found Algorithm: dtype_a != dtype_b");
  if (!(di == SC_FLOAT32 || is16(di))) return fail(SC_RUNTIME, "Can't Found Algorithm: dtype %s", dtype_name(di));
  if (!(p->dtype_c == SC_FLOAT32 || p->dtype_c == di))
    return fail(SC_RUNTIME, "Can't Found Algorithm: dtype_c %s", dtype_name(p->dtype_c));
  if (p->algo == SC_ALGO_SIMT && di != SC_FLOAT32)
    return fail(SC_RUNTIME, "Can't Found Algorithm: Simt kernels take float32 operands");
  *a = scb::GemmArgs{};
  a->shuffle = p->shuffle_type;
  a->trans_a = p->trans_a;
  a->trans_b = p->trans_b;
  a->m = p->m;
  a->n = p->n;
  a->k = p->k;
  a->a = static_cast<const uint8_t *>(p->a);
  a->lda = p->lda;
  a->b = static_cast<const uint8_t *>(p->b);
  a->ldb = p->ldb;
  a->c = p->c;
  a->ldc = p->ldc;
  a->a_inds = p->a_inds;
  a->b_inds = p->b_inds;
  a->c_inds = p->c_inds;
  a->a_rows = p->a_rows;
  a->b_rows = p->b_rows;
  a->in_dtype = di;
  a->out_dtype = p->dtype_c;
  a->epi.alpha = p->alpha;
  a->epi.beta = p->beta;
  a->epi.act_alpha = p->act_alpha;
  a->epi.act_beta = p->act_beta;
  a->epi.act_type = p->act_type;
  a->epi.mode = 0;
  a->epi.src = p->d != nullptr ? p->d : p->c;
  a->epi.src_ld = p->d != nullptr ? p->ldd : p->ldc;
  a->split_k = p->split_k_slices > 1 ? p->split_k_slices : 1;
  if (a->split_k > 1 && !(scb::dense_gemm_supported(*a) || p->shuffle_type == SC_SHUFFLE_AB))
    return fail(SC_RUNTIME, "algo don't support splitk but you provide split_k_slices > 1. %d", p->split_k_slices);
  return SC_OK;
}

int sc_gemm_workspace_size(const sc_gemm_params *p, int64_t *bytes) {
  scb::GemmArgs a;
  int rc = plan_gemm(p, &a);
  if (rc != SC_OK) return rc;
  *bytes = scb::gemm_workspace_bytes(a);
  return SC_OK;
}

int sc_gemm_matmul(const sc_gemm_params *p) {
  g_last_error.clear();
  scb::GemmArgs a;
  int rc = plan_gemm(p, &a);
  if (rc != SC_OK) return rc;
  const int64_t need = scb::gemm_workspace_bytes(a);
  if (need > 0 && (p->workspace == nullptr || p->workspace_bytes < need))
    return fail(SC_RUNTIME, "workspace at least %lld bytes.", (long long)need);
  a.ws = static_cast<float *>(p->workspace);
  int sms = 0;
  rc = device_state(&a.err, &sms);
  if (rc != SC_OK) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(p->stream);
  cudaError_t e = scb::launch_gemm(a, sms, s);
  if (e != cudaSuccess) return cuda_fail(e, "gemm launch");
  if (p->flags & SC_FLAG_SYNC_CHECK) return sync_check(s);
  return SC_OK;
}

// ------------------------------------------------------------------ gather / scatter
static int check_rows_args(const void *out, const void *in, const int32_t *indices, int64_t m,
                           int64_t row_bytes, int32_t bpa, int32_t threads) {
  if (m < 0 || row_bytes < 0) return fail(SC_INVALID_ARG, "bad m / row size");
  if (bpa != 4 && bpa != 8 && bpa != 16)
    return fail(SC_INVALID_ARG, "bytes_per_access %d must be 4, 8 or 16", bpa);
  if (threads != 64 && threads != 128 && threads != 256)
    return fail(SC_INVALID_ARG, "num_threads %d must be 64, 128 or 256", threads);
  if (row_bytes % bpa) return fail(SC_RUNTIME, "not supported. use supported() to check first");
  if (m > 0 && row_bytes > 0 && (out == nullptr || in == nullptr || indices == nullptr))
    return fail(SC_INVALID_ARG, "output, input and indices must not be empty");
  if (reinterpret_cast<uintptr_t>(out) % bpa || reinterpret_cast<uintptr_t>(in) % bpa)
    return fail(SC_INVALID_ARG, "output and input must be aligned to bytes_per_access (%d)", bpa);
  return SC_OK;
}

int sc_gather_rows(void *out, const void *in, int64_t in_rows, const int32_t *indices, int64_t m,
                   int64_t row_bytes, int32_t bytes_per_access, int32_t num_threads, void *stream) {
  g_last_error.clear();
  int rc = check_rows_args(out, in, indices, m, row_bytes, bytes_per_access, num_threads);
  if (rc != SC_OK) return rc;
  int *err = nullptr;
  int sms = 0;
  rc = device_state(&err, &sms);
  if (rc != SC_OK) return rc;
  cudaError_t e = scb::launch_gather_rows(out, in, in_rows, indices, m, row_bytes, bytes_per_access,
                                          num_threads, sms, err, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_fail(e, "gather launch");
  return SC_OK;
}

int sc_scatter_add_rows(void *out, int64_t out_rows, const void *in, const int32_t *indices,
                        int64_t m, int64_t channels, int32_t dtype, int32_t bytes_per_access,
                        int32_t num_threads, void *stream) {
  g_last_error.clear();
  if (dtype != SC_FLOAT32 && !is16(dtype))
    return fail(SC_RUNTIME, "can't find a sutable scatter: dtype %s", dtype_name(dtype));
  int rc = check_rows_args(out, in, indices, m, channels * esize(dtype), bytes_per_access, num_threads);
  if (rc != SC_OK) return rc;
  int *err = nullptr;
  int sms = 0;
  rc = device_state(&err, &sms);
  if (rc != SC_OK) return rc;
  cudaError_t e = scb::launch_scatter_add_rows(out, out_rows, in, indices, m, channels, dtype,
                                               bytes_per_access, num_threads, sms, err,
                                               static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_fail(e, "scatter launch");
  return SC_OK;
}

// ------------------------------------------------------------------ pairs
int sc_pairs_workspace_size(int64_t n_in, int32_t kv, int32_t subm, int64_t *bytes) {
  if (n_in < 0 || kv < 1 || kv > 32) return fail(SC_INVALID_ARG, "bad n_in / kv");
  *bytes = scb::pairs_workspace_bytes(n_in, kv, subm);
  return SC_OK;
}

static int fill_pair_args(scb::PairBuildArgs *a, const int32_t *coords, int64_t n_in, int32_t batch,
                          const int32_t *spatial, const int32_t *ksize, const int32_t *stride,
                          const int32_t *padding, const int32_t *dilation, int subm) {
  if (n_in > 0 && coords == nullptr) return fail(SC_INVALID_ARG, "coords is null");
  if (spatial == nullptr || ksize == nullptr) return fail(SC_INVALID_ARG, "spatial/ksize null");
  *a = scb::PairBuildArgs{};
  a->coords = coords;
  a->n_in = n_in;
  a->batch = batch;
  a->subm = subm;
  int kv = 1;
  for (int d = 0; d < 3; ++d) {
    a->spatial[d] = spatial[d];
    a->ksize[d] = ksize[d];
    a->stride[d] = stride ? stride[d] : 1;
    a->padding[d] = padding ? padding[d] : 0;
    a->dilation[d] = dilation ? dilation[d] : 1;
    if (a->spatial[d] <= 0 || a->ksize[d] <= 0 || a->stride[d] <= 0 || a->dilation[d] <= 0 ||
        a->padding[d] < 0)
      return fail(SC_INVALID_ARG, "bad spatial / ksize / stride / padding / dilation");
    kv *= a->ksize[d];
    a->out_spatial[d] = subm ? a->spatial[d]
                             : (a->spatial[d] + 2 * a->padding[d] - a->dilation[d] * (a->ksize[d] - 1) - 1) /
                                       a->stride[d] + 1;
    if (a->out_spatial[d] <= 0) return fail(SC_INVALID_ARG, "empty output grid");
  }
  if (kv > 32) return fail(SC_RUNTIME, "kernel volume %d > 32 not supported", kv);
  if (subm) {
    for (int d = 0; d < 3; ++d)
      if (a->ksize[d] % 2 == 0) return fail(SC_INVALID_ARG, "submanifold conv needs odd kernel sizes");
  }
  return SC_OK;
}

int sc_build_subm_pairs(const int32_t *coords, int64_t n_in, const int32_t *spatial,
                        const int32_t *ksize, const int32_t *dilation, int32_t *pairs_fwd,
                        int32_t *pairs_bwd, uint32_t *mask_fwd, void *workspace,
                        int64_t workspace_bytes, void *stream) {
  g_last_error.clear();
  scb::PairBuildArgs a;
  int rc = fill_pair_args(&a, coords, n_in, 1, spatial, ksize, nullptr, nullptr, dilation, 1);
  if (rc != SC_OK) return rc;
  const int kv = a.ksize[0] * a.ksize[1] * a.ksize[2];
  if (workspace_bytes < scb::pairs_workspace_bytes(n_in, kv, 1))
    return fail(SC_RUNTIME, "workspace at least %lld bytes.",
                (long long)scb::pairs_workspace_bytes(n_in, kv, 1));
  int sms = 0;
  rc = device_state(&a.err, &sms);
  if (rc != SC_OK) return rc;
  cudaError_t e = scb::build_subm_pairs(a, pairs_fwd, pairs_bwd, mask_fwd, workspace,
                                        workspace_bytes, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_fail(e, "build_subm_pairs");
  return SC_OK;
}

int sc_build_conv_outputs(const int32_t *coords, int64_t n_in, int32_t batch, const int32_t *spatial,
                          const int32_t *ksize, const int32_t *stride, const int32_t *padding,
                          const int32_t *dilation, int32_t *out_spatial, int64_t *n_out,
                          void *workspace, int64_t workspace_bytes, void *stream) {
  g_last_error.clear();
  scb::PairBuildArgs a;
  int rc = fill_pair_args(&a, coords, n_in, batch, spatial, ksize, stride, padding, dilation, 0);
  if (rc != SC_OK) return rc;
  const int kv = a.ksize[0] * a.ksize[1] * a.ksize[2];
  if (workspace_bytes < scb::pairs_workspace_bytes(n_in, kv, 0))
    return fail(SC_RUNTIME, "workspace at least %lld bytes.",
                (long long)scb::pairs_workspace_bytes(n_in, kv, 0));
  int sms = 0;
  rc = device_state(&a.err, &sms);
  if (rc != SC_OK) return rc;
  for (int d = 0; d < 3; ++d) out_spatial[d] = a.out_spatial[d];
  cudaError_t e = scb::build_conv_outputs(a, n_out, workspace, workspace_bytes,
                                          static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_fail(e, "build_conv_outputs");
  return sync_check(static_cast<cudaStream_t>(stream));
}

int sc_build_conv_pairs(const int32_t *coords, int64_t n_in, int32_t batch, const int32_t *spatial,
                        const int32_t *ksize, const int32_t *stride, const int32_t *padding,
                        const int32_t *dilation, int64_t n_out, int32_t *out_coords,
                        int32_t *pairs_fwd, int32_t *pairs_bwd, uint32_t *mask_fwd,
                        uint32_t *mask_bwd, void *workspace, int64_t workspace_bytes,
                        void *stream) {
  g_last_error.clear();
  scb::PairBuildArgs a;
  int rc = fill_pair_args(&a, coords, n_in, batch, spatial, ksize, stride, padding, dilation, 0);
  if (rc != SC_OK) return rc;
  const int kv = a.ksize[0] * a.ksize[1] * a.ksize[2];
  if (workspace_bytes < scb::pairs_workspace_bytes(n_in, kv, 0))
    return fail(SC_RUNTIME, "workspace at least %lld bytes.",
                (long long)scb::pairs_workspace_bytes(n_in, kv, 0));
  int sms = 0;
  rc = device_state(&a.err, &sms);
  if (rc != SC_OK) return rc;
  cudaError_t e = scb::build_conv_pairs(a, n_out, out_coords, pairs_fwd, pairs_bwd, mask_fwd,
                                        mask_bwd, workspace, workspace_bytes,
                                        static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_fail(e, "build_conv_pairs");
  return SC_OK;
}

int sc_sort_indices(const int32_t *indices, int32_t kv, int64_t N, const int32_t *argsort,
                    int32_t *indices_sorted, void *stream) {
  g_last_error.clear();
  if (N > 0 && (indices == nullptr || argsort == nullptr || indices_sorted == nullptr))
    return fail(SC_INVALID_ARG, "null indices / argsort / output");
  if (kv < 1 || kv > 32 || N < 0) return fail(SC_INVALID_ARG, "bad kv / N");
  cudaError_t e = scb::sort_indices(indices, kv, N, argsort, indices_sorted,
                                    static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_fail(e, "sort_indices");
  return SC_OK;
}

int sc_tile_order_workspace_size(int64_t N, int64_t *bytes) {
  g_last_error.clear();
  if (bytes == nullptr) return fail(SC_INVALID_ARG, "bytes is null");
  if (N < 0) return fail(SC_INVALID_ARG, "N must be >= 0");
  *bytes = kSchedBytes + align256((N + 127) / 128 * 4);
  return SC_OK;
}

int sc_tile_order(const uint32_t *mask, int64_t N, uint32_t mask_filter, int32_t kv, int32_t reverse,
                  int32_t *tile_order, void *workspace, int64_t workspace_bytes, void *stream) {
  g_last_error.clear();
  if (N < 0) return fail(SC_INVALID_ARG, "N must be >= 0");
  if (N == 0) return SC_OK;
  if (mask == nullptr || tile_order == nullptr) return fail(SC_INVALID_ARG, "mask and tile_order must not be null");
  if (kv < 1 || kv > 32) return fail(SC_INVALID_ARG, "kernel volume %d not supported (1..32)", kv);
  const int64_t need = kSchedBytes + align256((N + 127) / 128 * 4);
  if (workspace == nullptr || workspace_bytes < need)
    return fail(SC_RUNTIME, "workspace at least %lld bytes.", (long long)need);
  int *err = nullptr;
  int sms = 0;
  int rc = device_state(&err, &sms);
  if (rc != SC_OK) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  uint8_t *ws = static_cast<uint8_t *>(workspace);
  cudaError_t e = cudaMemsetAsync(ws, 0, 34 * sizeof(int), s);
  if (e != cudaSuccess) return cuda_fail(e, "zero tile order histogram");
  e = scb::launch_tile_order(mask, N, mask_filter, reverse ? 1 : 0, kv, reinterpret_cast<int *>(ws),
                             reinterpret_cast<int32_t *>(ws + kSchedBytes), tile_order, s);
  if (e != cudaSuccess) return cuda_fail(e, "tile order launch");
  return SC_OK;
}

int sc_sort_workspace_size(int64_t n, int64_t *bytes) {
  if (n < 0) return fail(SC_INVALID_ARG, "bad n");
  *bytes = scb::sort_workspace_bytes(n);
  return SC_OK;
}

int sc_sort_masks_split(uint32_t *data, int64_t n, uint32_t split_mask, int32_t *argsort,
                        void *workspace, int64_t workspace_bytes, void *stream) {
  g_last_error.clear();
  if (n > 0 && (data == nullptr || argsort == nullptr)) return fail(SC_INVALID_ARG, "null data/argsort");
  if (n >= 0x7fffffff) return fail(SC_INVALID_ARG, "n too large for int32 argsort");
  if (workspace_bytes < scb::sort_workspace_bytes(n))
    return fail(SC_RUNTIME, "workspace at least %lld bytes.", (long long)scb::sort_workspace_bytes(n));
  cudaError_t e = scb::sort_masks_split(data, n, split_mask, argsort, workspace, workspace_bytes,
                                        static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_fail(e, "sort_masks_split");
  return SC_OK;
}

}  // extern "C"
