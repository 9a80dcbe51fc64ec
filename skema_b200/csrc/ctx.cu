// ctx.cu -- the C ABI of include/skema_c.h: context lifecycle, parameter
// resolution, map orientation, sketch import/export and dispatch of the
// linear update to the kernels of the other translation units.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <string>

#include "internal.h"

namespace skema {

static thread_local std::string g_create_error;

// The message skema_last_error(NULL) returns: failures of skema_create and
// of the file calls, which have no context.
void set_thread_error(const std::string& msg) { g_create_error = msg; }

void fail(int status, const std::string& msg) { throw Error{status, msg}; }

void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    (void)cudaGetLastError();  // a failed call (e.g. cudaMalloc) must not fail the next launch check
    const int st = (e == cudaErrorMemoryAllocation) ? SKEMA_ENOMEM
                   : (e == cudaErrorNoDevice || e == cudaErrorNoKernelImageForDevice ||
                      e == cudaErrorInsufficientDriver)
                       ? SKEMA_ENOKERNEL
                       : SKEMA_ECUDA;
    fail(st, std::string(what) + ": " + cudaGetErrorString(e));
  }
}

// Writes the limit of every bounded device wait (ns; <= 0: the 2 s default)
// into the context's status block, ordered on the context stream.
static void set_wait_limit(skema_ctx* c, int64_t ns) {
  const unsigned long long v = ns > 0 ? (unsigned long long)ns : tc_default_wait_ns();
  SKEMA_CUDA(cudaMemcpyAsync(c->dev_err + 2, &v, sizeof(v), cudaMemcpyHostToDevice, c->stream));
  SKEMA_CUDA(cudaStreamSynchronize(c->stream));
}

void check_device_error(skema_ctx* c) {
  if (!c->dev_err_armed || !c->dev_err) return;
  int h = 0;
  SKEMA_CUDA(cudaMemcpyAsync(&h, c->dev_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  SKEMA_CUDA(cudaStreamSynchronize(c->stream));
  c->dev_err_armed = false;
  if (h != 0) {
    SKEMA_CUDA(cudaMemsetAsync(c->dev_err, 0, sizeof(int), c->stream));
    SKEMA_CUDA(cudaStreamSynchronize(c->stream));
    fail(SKEMA_ETIMEOUT, "a tensor-core kernel gave up waiting on its pipeline; the sketches are invalid");
  }
}

// Fails with SKEMA_ENOMEM when growing a context buffer from `have` to
// `want` bytes would take the context's workspace and staging above the limit
// set by skema_set_workspace_limit.
static void check_ws_limit(const skema_ctx* c, size_t have, size_t want) {
  if (c->ws_limit == 0) return;
  const size_t total = c->ws_bytes + c->stage_bytes - have + want;
  if (total > c->ws_limit)
    fail(SKEMA_ENOMEM, "workspace of " + std::to_string(total) + " bytes needed, above the limit of " +
                           std::to_string(c->ws_limit) + " bytes set by skema_set_workspace_limit");
}

void* workspace(skema_ctx* c, size_t bytes) {
  if (bytes <= c->ws_bytes) return c->ws;
  check_ws_limit(c, c->ws_bytes, std::max<size_t>(bytes, 1 << 20));
  if (c->ws) {
    SKEMA_CUDA(cudaStreamSynchronize(c->stream));
    SKEMA_CUDA(cudaFree(c->ws));
    c->ws = nullptr;
    c->ws_bytes = 0;
  }
  const size_t b = std::max<size_t>(bytes, 1 << 20);
  SKEMA_CUDA(cudaMalloc(&c->ws, b));
  c->ws_bytes = b;
  return c->ws;
}

// A pitched copy whose rows lie back to back on both sides goes as one
// linear copy: the copy engines move one long run much faster than the same
// bytes as many short rows (a 1e6 x 81 row-major sketch has 324-byte rows).
static cudaError_t copy2d(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width, size_t height,
                          cudaMemcpyKind kind, cudaStream_t st) {
  if (dpitch == width && spitch == width) return cudaMemcpyAsync(dst, src, width * height, kind, st);
  return cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, height, kind, st);
}

void* staging(skema_ctx* c, size_t bytes) {
  if (bytes <= c->stage_bytes) return c->stage;
  check_ws_limit(c, c->stage_bytes, std::max<size_t>(bytes, 1 << 20));
  if (c->stage) {
    SKEMA_CUDA(cudaStreamSynchronize(c->stream));
    SKEMA_CUDA(cudaFree(c->stage));
    c->stage = nullptr;
    c->stage_bytes = 0;
  }
  const size_t b = std::max<size_t>(bytes, 1 << 20);
  SKEMA_CUDA(cudaMalloc(&c->stage, b));
  c->stage_bytes = b;
  return c->stage;
}

bool y_rows_clean(const skema_ctx* c, int64_t a, int64_t b) {
  for (const Interval& iv : c->y_written)
    if (iv.a < b && a < iv.b) return false;
  return true;
}

void y_rows_mark(skema_ctx* c, int64_t a, int64_t b) {
  if (a >= b) return;
  std::vector<Interval>& v = c->y_written;
  v.push_back({a, b});
  std::sort(v.begin(), v.end(), [](const Interval& x, const Interval& y) { return x.a < y.a; });
  std::vector<Interval> out;
  for (const Interval& iv : v) {
    if (!out.empty() && iv.a <= out.back().b)
      out.back().b = std::max(out.back().b, iv.b);
    else
      out.push_back(iv);
  }
  v.swap(out);
}

// Y is column-major (m x k, ld = m): rows [a, b) are one strip per column.
static void y_zero_rows(skema_ctx* c, int64_t a, int64_t b) {
  if (a >= b) return;
  SKEMA_CUDA(cudaMemset2DAsync(c->Y + a, sizeof(float) * (size_t)c->m, 0, sizeof(float) * (size_t)(b - a),
                               (size_t)c->k, c->stream));
}

void y_materialize(skema_ctx* c) {
  int64_t at = 0;
  for (const Interval& iv : c->y_written) {
    if (iv.a > at) y_zero_rows(c, at, iv.a);
    at = std::max(at, iv.b);
  }
  if (at < c->m) y_zero_rows(c, at, c->m);
  c->y_written.assign(1, Interval{0, c->m});
}

float y_beta(skema_ctx* c, int64_t a, int64_t b, float nu) {
  if (y_rows_clean(c, a, b)) return 0.f;
  // Rows of [a, b) not written since the reset still hold whatever Y held
  // before it: zero them, so that beta = nu scales zeros there.
  int64_t at = a;
  for (const Interval& iv : c->y_written) {
    if (iv.b <= a || iv.a >= b) continue;
    if (iv.a > at) y_zero_rows(c, at, iv.a);
    at = std::max(at, iv.b);
  }
  if (at < b) y_zero_rows(c, at, b);
  y_rows_mark(c, a, b);
  return nu;
}

void xz_materialize(skema_ctx* c, cudaStream_t stream) {
  if (!c->xz_pending) return;
  if (c->X) SKEMA_CUDA(cudaMemsetAsync(c->X, 0, sizeof(float) * (size_t)(c->k * c->n), stream));
  if (c->Z) SKEMA_CUDA(cudaMemsetAsync(c->Z, 0, sizeof(float) * (size_t)(c->s * c->s), stream));
  c->xz_pending = false;
}

const char* const kStageNames[ST_COUNT] = {"update.omega",   "update.psi",    "update.upsilon",
                                            "update.phi",     "update.entries", "update.window",
                                            "update.fused",   "update.daxpy",  "approx.orth",
                                            "approx.core",    "approx.svd",    "approx.vectors"};

static cudaEvent_t pool_event(skema_ctx* c) {
  if (!c->event_pool.empty()) {
    cudaEvent_t e = c->event_pool.back();
    c->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  SKEMA_CUDA(cudaEventCreate(&e));
  return e;
}

StageScope::StageScope(skema_ctx* c, int stage) : StageScope(c, stage, c->stream) {}

StageScope::StageScope(skema_ctx* c, int stage, cudaStream_t stream) : c_(c), stage_(stage), stream_(stream) {
  // an NVTX range per stage (host-side: a profiler that records NVTX shows
  // the stage around its launches; without one the call is a no-op)
  nvtxRangePushA(kStageNames[stage]);
  if (!c_->timing) return;
  a_ = pool_event(c_);
  SKEMA_CUDA(cudaEventRecord(a_, stream_));
}

StageScope::~StageScope() {
  nvtxRangePop();
  if (!a_) return;
  cudaEvent_t b = nullptr;
  if (!c_->event_pool.empty()) {
    b = c_->event_pool.back();
    c_->event_pool.pop_back();
  } else if (cudaEventCreate(&b) != cudaSuccess) {
    return;
  }
  if (cudaEventRecord(b, stream_) != cudaSuccess) return;
  c_->pending.push_back(PendingTimer{stage_, a_, b});
}

static void drain_timers(skema_ctx* c) {
  if (c->pending.empty()) return;
  SKEMA_CUDA(cudaStreamSynchronize(c->stream));
  for (const PendingTimer& t : c->pending) {
    float ms = 0.f;
    SKEMA_CUDA(cudaEventElapsedTime(&ms, t.a, t.b));
    c->stage_ms[t.stage] += ms;
    c->stage_n[t.stage] += 1;
    c->event_pool.push_back(t.a);
    c->event_pool.push_back(t.b);
  }
  c->pending.clear();
}

static void free_all(skema_ctx* c) {
  for (const PendingTimer& t : c->pending) {
    cudaEventDestroy(t.a);
    cudaEventDestroy(t.b);
  }
  c->pending.clear();
  for (cudaEvent_t e : c->event_pool) cudaEventDestroy(e);
  c->event_pool.clear();
  map_free(c->ups);
  map_free(c->omg);
  map_free(c->phi);
  map_free(c->psi);
  if (c->X) cudaFree(c->X);
  if (c->Y) cudaFree(c->Y);
  if (c->Z) cudaFree(c->Z);
  if (c->ws) cudaFree(c->ws);
  if (c->stage) cudaFree(c->stage);
  if (c->op16) cudaFree(c->op16);
  residual_free(c);
  if (c->op8) cudaFree(c->op8);
  if (c->fp8_win) cudaFree(c->fp8_win);
  if (c->dev_err) cudaFree(c->dev_err);
  c->X = c->Y = c->Z = nullptr;
  c->ws = c->stage = c->op16 = c->op8 = nullptr;
  c->fp8_win = nullptr;
  c->dev_err = nullptr;
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
  c->own_stream = nullptr;
  if (c->side) cudaStreamDestroy(c->side);
  if (c->fork_ev) cudaEventDestroy(c->fork_ev);
  if (c->join_ev) cudaEventDestroy(c->join_ev);
  for (cudaEvent_t& e : c->pipe_ev) {
    if (e) cudaEventDestroy(e);
    e = nullptr;
  }
  for (cudaEvent_t& e : c->stage_ev) {
    if (e) cudaEventDestroy(e);
    e = nullptr;
  }
  c->side = nullptr;
  c->fork_ev = c->join_ev = nullptr;
}

// Runs f, converting library errors into a status and remembering the message.
template <typename F>
static int guarded(skema_ctx* c, F&& f) {
  if (!c) return SKEMA_EINVAL;
  try {
    SKEMA_CUDA(cudaSetDevice(c->dev));
    if (!c->xz_defer) xz_materialize(c, c->stream);
    f();
    c->err.clear();
    return SKEMA_OK;
  } catch (const Error& e) {
    c->err = e.msg;
    return e.status;
  } catch (const std::bad_alloc&) {
    c->err = "host allocation failed";
    return SKEMA_ENOMEM;
  } catch (...) {
    c->err = "unexpected C++ exception";
    return SKEMA_ECUDA;
  }
}

static void set_map(Map& mp, int kind, int64_t nrow, int64_t ncol, bool transposed,
                    int32_t seed) {
  mp.kind = kind;
  mp.nrow = nrow;
  mp.ncol = ncol;
  mp.transposed = transposed;
  mp.lrows = transposed ? ncol : nrow;
  mp.lcols = transposed ? nrow : ncol;
  mp.seed = (uint32_t)seed;
}

// Orientation rules of SketchySVD's ctor (src/Skema_SketchySVD.cpp:30-95) and
// SketchySPD's ctor (src/Skema_SketchySVD.cpp:769-775).
static void plan_maps(skema_ctx* c) {
  const skema_params& p = c->p;
  const int kind = p.dim_redux;
  if (c->spd) {
    // Omega(ncol, range, seeds[0]) applied as Y = A * Omega (:896-903):
    // logical Omega~ = stored^T (k x n).
    set_map(c->omg, kind, c->n, c->k, true, p.seeds[0]);
    return;
  }
  const bool gauss_sparse = p.issparse && kind == SKEMA_MAP_GAUSS;
  const bool omega_t = p.issparse != 0;
  set_map(c->ups, kind, gauss_sparse ? c->m : c->k, gauss_sparse ? c->k : c->m, gauss_sparse,
          p.seeds[0]);
  set_map(c->omg, kind, omega_t ? c->n : c->k, omega_t ? c->k : c->n, omega_t, p.seeds[1]);
  set_map(c->phi, kind, gauss_sparse ? c->m : c->s, gauss_sparse ? c->s : c->m, gauss_sparse,
          p.seeds[2]);
  set_map(c->psi, kind, omega_t ? c->n : c->s, omega_t ? c->s : c->n, omega_t, p.seeds[3]);
}

static void check_dense_args(const void* A, int64_t ld, int32_t layout, int64_t rows,
                             int64_t cols, int32_t mem) {
  if (layout != SKEMA_COL_MAJOR && layout != SKEMA_ROW_MAJOR) fail(SKEMA_EINVAL, "bad layout");
  if (mem != SKEMA_MEM_DEVICE && mem != SKEMA_MEM_HOST) fail(SKEMA_EINVAL, "bad mem kind");
  if (rows > 0 && cols > 0 && !A) fail(SKEMA_EINVAL, "null matrix pointer");
  const int64_t need = (layout == SKEMA_COL_MAJOR) ? rows : cols;
  if (rows > 0 && cols > 0 && ld < need) fail(SKEMA_EINVAL, "leading dimension too small");
}

}  // namespace skema

using namespace skema;

extern "C" {

int skema_params_init(skema_params* p) {
  if (!p) return SKEMA_EINVAL;
  std::memset(p, 0, sizeof(*p));
  p->matrix_m = 0;
  p->matrix_n = 0;
  p->rank = 1;
  p->sketch_range = 1;
  p->sketch_core = 1;
  p->window = 1;
  p->sketch_eta = 1.0;
  p->sketch_nu = 1.0;
  p->seeds[0] = 0;
  p->seeds[1] = 1;
  p->seeds[2] = 2;
  p->seeds[3] = 3;
  p->dim_redux = SKEMA_MAP_GAUSS;
  p->issparse = 0;
  p->issymmetric = 0;
  p->force_three_sketch = 0;
  p->kernel_func = SKEMA_KERNEL_NONE;
  p->kernel_gamma = 1.0;
  p->precision = SKEMA_PREC_FP32;
  p->device = 0;
  p->spd_approx = SKEMA_SPD_NYSTROM;
  return SKEMA_OK;
}

int skema_create(const skema_params* p, skema_ctx** out) {
  g_create_error.clear();
  if (!p || !out) {
    g_create_error = "null argument";
    return SKEMA_EINVAL;
  }
  *out = nullptr;
  skema_ctx* c = new (std::nothrow) skema_ctx();
  if (!c) return SKEMA_ENOMEM;
  c->p = *p;
  try {
    if (p->matrix_m <= 0 || p->matrix_n <= 0) fail(SKEMA_EINVAL, "matrix_m and matrix_n must be > 0");
    if (p->rank < 1) fail(SKEMA_EINVAL, "rank must be >= 1");
    if (p->window < 1) fail(SKEMA_EINVAL, "window must be >= 1");
    if (p->dim_redux != SKEMA_MAP_GAUSS && p->dim_redux != SKEMA_MAP_SPARSE_SIGN)
      fail(SKEMA_EINVAL, "dim_redux must be gauss or sparse-sign");
    if (p->kernel_func != SKEMA_KERNEL_NONE && p->kernel_func != SKEMA_KERNEL_GAUSSRBF)
      fail(SKEMA_EINVAL, "kernel_func must be none or gaussrbf");
    if (p->precision < SKEMA_PREC_FP32 || p->precision > SKEMA_PREC_FP8)
      fail(SKEMA_EINVAL, "precision must be fp32, bf16 or fp8");
    if (p->kernel_func == SKEMA_KERNEL_GAUSSRBF && p->issparse)
      fail(SKEMA_EUNSUPPORTED, "Gauss RBF kernel on a sparse input (the reference exits here too)");
    if (p->kernel_func == SKEMA_KERNEL_GAUSSRBF && p->matrix_m != p->matrix_n)
      fail(SKEMA_EINVAL, "kernel input needs matrix_n == matrix_m");
    if (!(p->kernel_gamma >= 0.0)) fail(SKEMA_EINVAL, "kernel_gamma must be >= 0");
    c->m = p->matrix_m;
    c->n = p->matrix_n;
    // range/core defaults (src/Skema_SketchySVD.cpp:20-24)
    c->k = p->sketch_range < p->rank ? 4 * p->rank + 1 : p->sketch_range;
    c->s = p->sketch_core < p->rank ? 2 * c->k + 1 : p->sketch_core;
    c->w = p->window;
    c->spd = p->issymmetric && !p->force_three_sketch;
    if (c->n >= (int64_t(1) << 31) || c->m >= (int64_t(1) << 40) || c->k >= (1 << 20) ||
        c->s >= (1 << 20))
      fail(SKEMA_EINVAL, "dimension out of supported range");
    int ndev = 0;
    cuda_check(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
    if (p->device < 0 || p->device >= ndev) fail(SKEMA_EINVAL, "device ordinal out of range");
    c->dev = p->device;
    SKEMA_CUDA(cudaSetDevice(c->dev));
    cudaDeviceProp prop;
    SKEMA_CUDA(cudaGetDeviceProperties(&prop, c->dev));
    c->sm_count = prop.multiProcessorCount;
    c->cc_major = prop.major;
    c->cc_minor = prop.minor;
    if (prop.major != 10) fail(SKEMA_ENOKERNEL, "this build carries sm_100a code only");
    SKEMA_CUDA(cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking));
    c->stream = c->own_stream;
    SKEMA_CUDA(cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking));
    SKEMA_CUDA(cudaEventCreateWithFlags(&c->fork_ev, cudaEventDisableTiming));
    SKEMA_CUDA(cudaEventCreateWithFlags(&c->join_ev, cudaEventDisableTiming));
    for (cudaEvent_t& e : c->pipe_ev) SKEMA_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    for (cudaEvent_t& e : c->stage_ev) SKEMA_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    c->pipe_xt_sms = 0;
    c->pipe_windows = 2;
    if (const char* v = std::getenv("SKEMA_DENSE_PIPE_SMS")) c->pipe_xt_sms = std::max(0, std::atoi(v));
    if (const char* v = std::getenv("SKEMA_DENSE_PIPE_WINDOWS")) c->pipe_windows = std::max(1, std::atoi(v));
    if (c->pipe_xt_sms >= c->sm_count) c->pipe_xt_sms = 0;
    c->ssign_bin_kb = 128;
    if (const char* v = std::getenv("SKEMA_SSIGN_BIN_KB")) c->ssign_bin_kb = std::min(220, std::max(16, std::atoi(v)));
    c->ssign_batch = 4;
    c->xt_store_thread = true;
    if (const char* v = std::getenv("SKEMA_XT_STORE_THREAD")) c->xt_store_thread = std::atoi(v) != 0;
    if (const char* v = std::getenv("SKEMA_SSIGN_BATCH")) c->ssign_batch = std::atoi(v);
    plan_maps(c);
    if (c->spd) {
      map_generate(c, c->omg, p->precision);
    } else {
      map_generate(c, c->ups, p->precision);
      map_generate(c, c->omg, p->precision);
      map_generate(c, c->phi, p->precision);
      map_generate(c, c->psi, p->precision);
      if (p->dim_redux == SKEMA_MAP_SPARSE_SIGN) {
        map_build_inverse(c, c->ups);
        map_build_inverse(c, c->phi);
      }
      tc_prepare_maps(c);
    }
    // device status block: int status at [0], the wait limit (ns) at [2..3]
    SKEMA_CUDA(cudaMalloc(&c->dev_err, 4 * sizeof(int)));
    SKEMA_CUDA(cudaMemsetAsync(c->dev_err, 0, 4 * sizeof(int), c->stream));
    set_wait_limit(c, 0);
    if (!c->spd) {
      SKEMA_CUDA(cudaMalloc(&c->X, sizeof(float) * (size_t)(c->k * c->n)));
      SKEMA_CUDA(cudaMalloc(&c->Z, sizeof(float) * (size_t)(c->s * c->s)));
    }
    SKEMA_CUDA(cudaMalloc(&c->Y, sizeof(float) * (size_t)(c->m * c->k)));
    if (c->X) SKEMA_CUDA(cudaMemsetAsync(c->X, 0, sizeof(float) * (size_t)(c->k * c->n), c->stream));
    if (c->Z) SKEMA_CUDA(cudaMemsetAsync(c->Z, 0, sizeof(float) * (size_t)(c->s * c->s), c->stream));
    SKEMA_CUDA(cudaMemsetAsync(c->Y, 0, sizeof(float) * (size_t)(c->m * c->k), c->stream));
    SKEMA_CUDA(cudaStreamSynchronize(c->stream));
  } catch (const Error& e) {
    g_create_error = e.msg;
    free_all(c);
    delete c;
    return e.status;
  } catch (const std::bad_alloc&) {
    g_create_error = "host allocation failed";
    free_all(c);
    delete c;
    return SKEMA_ENOMEM;
  }
  *out = c;
  return SKEMA_OK;
}

int skema_destroy(skema_ctx* c) {
  if (!c) return SKEMA_OK;
  cudaSetDevice(c->dev);
  if (c->stream) cudaStreamSynchronize(c->stream);
  free_all(c);
  delete c;
  return SKEMA_OK;
}

const char* skema_last_error(const skema_ctx* c) {
  if (!c) return g_create_error.c_str();
  return c->err.c_str();
}

int skema_get_dims(const skema_ctx* c, int64_t* range, int64_t* core, int32_t* spd) {
  if (!c) return SKEMA_EINVAL;
  if (range) *range = c->k;
  if (core) *core = c->s;
  if (spd) *spd = c->spd ? 1 : 0;
  return SKEMA_OK;
}

int skema_reset(skema_ctx* c) {
  return guarded(c, [&] {
    // X and Z are zeroed by the next call (xz_materialize), Y lazily: the
    // update kernels treat rows not written since the reset as zero
    // (write-only), and y_materialize() clears the rest before Y is read
    // back or factorised.
    c->xz_pending = c->X || c->Z;
    c->y_written.clear();
  });
}

int skema_linear_update_dense(skema_ctx* c, const float* A, int64_t ld, int32_t layout,
                              int64_t row0, int64_t nrows, int32_t mem) {
  return guarded(c, [&] {
    if (c->p.kernel_func != SKEMA_KERNEL_NONE)
      fail(SKEMA_ESTATE, "context expects kernel points: use skema_linear_update_rbf");
    if (c->p.issparse) fail(SKEMA_ESTATE, "context was created for a CSR input");
    if (row0 < 0 || nrows < 0 || row0 + nrows > c->m) fail(SKEMA_EINVAL, "row range outside A");
    check_dense_args(A, ld, layout, nrows, c->n, mem);
    if (nrows == 0) return;
    if (mem == SKEMA_MEM_DEVICE) {
      Mat a{A, layout == SKEMA_COL_MAJOR ? 1 : ld, layout == SKEMA_COL_MAJOR ? ld : 1};
      dense_update(c, a, row0, nrows);
      return;
    }
    // Host input: staged window by window through two slots. The uploads
    // run on the side stream and each window's update on the context stream
    // once its upload has landed, so window w + 1 crosses PCIe while window
    // w is sketched; a slot is refilled only after the update that read it.
    // The device path sees a column-major w x n block (ld = w) or a
    // row-major one (ld = n).
    const int64_t W = c->w;
    const bool two = nrows > W;
    const size_t win_bytes = (sizeof(float) * (size_t)(std::min(W, nrows) * c->n) + 255) / 256 * 256;
    char* slots = (char*)staging(c, two ? 2 * win_bytes : win_bytes);
    cudaEvent_t up[2] = {c->stage_ev[0], c->stage_ev[1]}, used[2] = {c->stage_ev[2], c->stage_ev[3]};
    SKEMA_CUDA(cudaEventRecord(c->fork_ev, c->stream));
    SKEMA_CUDA(cudaStreamWaitEvent(c->side, c->fork_ev, 0));
    for (int64_t r = 0, i = 0; r < nrows; r += W, ++i) {
      const int64_t wr = std::min(W, nrows - r);
      const int sl = (int)(i & 1);
      float* buf = (float*)(slots + sl * win_bytes);
      if (i >= 2) SKEMA_CUDA(cudaStreamWaitEvent(c->side, used[sl], 0));
      if (layout == SKEMA_COL_MAJOR)
        SKEMA_CUDA(copy2d(buf, sizeof(float) * wr, A + r, sizeof(float) * ld, sizeof(float) * wr, c->n,
                          cudaMemcpyHostToDevice, c->side));
      else
        SKEMA_CUDA(copy2d(buf, sizeof(float) * c->n, A + r * ld, sizeof(float) * ld, sizeof(float) * c->n, wr,
                          cudaMemcpyHostToDevice, c->side));
      SKEMA_CUDA(cudaEventRecord(up[sl], c->side));
      SKEMA_CUDA(cudaStreamWaitEvent(c->stream, up[sl], 0));
      const Mat a = layout == SKEMA_COL_MAJOR ? Mat{buf, 1, wr} : Mat{buf, c->n, 1};
      dense_update(c, a, row0 + r, wr);
      SKEMA_CUDA(cudaEventRecord(used[sl], c->stream));
    }
  });
}

int skema_linear_update_csr(skema_ctx* c, const int64_t* rowptr, const int32_t* col,
                            const float* val, int64_t row0, int64_t nrows, int32_t mem) {
  if (!c) return SKEMA_EINVAL;
  struct Defer {  // csr_update zeroes a pending X / Z itself
    skema_ctx* c;
    ~Defer() { c->xz_defer = false; }
  } defer{c};
  c->xz_defer = true;
  return guarded(c, [&] {
    if (!c->p.issparse) fail(SKEMA_ESTATE, "context was created for a dense input");
    if (row0 < 0 || nrows < 0 || row0 + nrows > c->m) fail(SKEMA_EINVAL, "row range outside A");
    if (mem != SKEMA_MEM_DEVICE && mem != SKEMA_MEM_HOST) fail(SKEMA_EINVAL, "bad mem kind");
    if (nrows == 0) return;
    if (!rowptr) fail(SKEMA_EINVAL, "null rowptr");
    if (mem == SKEMA_MEM_DEVICE) {
      csr_update(c, rowptr, col, val, 0, row0, nrows);
      return;
    }
    const int64_t base = rowptr[0];
    const int64_t nnz = rowptr[nrows] - base;
    if (nnz < 0) fail(SKEMA_EINVAL, "rowptr is decreasing");
    if (nnz > 0 && (!col || !val)) fail(SKEMA_EINVAL, "null col/val");
    const size_t rp_bytes = sizeof(int64_t) * (size_t)(nrows + 1);
    const size_t rp_pad = (rp_bytes + 255) / 256 * 256;
    const size_t c_bytes = sizeof(int32_t) * (size_t)nnz;
    const size_t c_pad = (c_bytes + 255) / 256 * 256;
    char* buf = (char*)staging(c, rp_pad + c_pad + sizeof(float) * (size_t)nnz + 256);
    int64_t* d_rp = (int64_t*)buf;
    int32_t* d_col = (int32_t*)(buf + rp_pad);
    float* d_val = (float*)(buf + rp_pad + c_pad);
    SKEMA_CUDA(cudaMemcpyAsync(d_rp, rowptr, rp_bytes, cudaMemcpyHostToDevice, c->stream));
    if (nnz > 0) {
      SKEMA_CUDA(cudaMemcpyAsync(d_col, col + base, c_bytes, cudaMemcpyHostToDevice, c->stream));
      SKEMA_CUDA(cudaMemcpyAsync(d_val, val + base, sizeof(float) * (size_t)nnz,
                                 cudaMemcpyHostToDevice, c->stream));
    }
    // the row map is checked on the host while the copies run (their sizes
    // depend only on its ends); a decreasing map waits for them, so the
    // caller's buffers are no longer read, and nothing is launched
    for (int64_t i = 0; i < nrows; ++i)
      if (rowptr[i + 1] < rowptr[i]) {
        SKEMA_CUDA(cudaStreamSynchronize(c->stream));
        fail(SKEMA_EINVAL, "rowptr is decreasing");
      }
    csr_update(c, d_rp, d_col, d_val, base, row0, nrows);
  });
}

int skema_linear_update_rbf(skema_ctx* c, const float* pts, int64_t ld, int32_t layout,
                            int64_t npts, int64_t d, int64_t row0, int64_t nrows, int32_t mem) {
  return guarded(c, [&] {
    if (c->p.kernel_func != SKEMA_KERNEL_GAUSSRBF)
      fail(SKEMA_ESTATE, "context was not created with kernel_func = gaussrbf");
    if (npts != c->m) fail(SKEMA_EINVAL, "npts must equal matrix_m");
    if (d <= 0) fail(SKEMA_EINVAL, "d must be > 0");
    if (row0 < 0 || nrows < 0 || row0 + nrows > c->m) fail(SKEMA_EINVAL, "row range outside K");
    check_dense_args(pts, ld, layout, npts, d, mem);
    if (nrows == 0) return;
    if (mem == SKEMA_MEM_DEVICE) {
      Mat P{pts, layout == SKEMA_COL_MAJOR ? 1 : ld, layout == SKEMA_COL_MAJOR ? ld : 1};
      rbf_update(c, P, npts, d, row0, nrows);
      return;
    }
    float* buf = (float*)staging(c, sizeof(float) * (size_t)(npts * d));
    if (layout == SKEMA_COL_MAJOR) {
      SKEMA_CUDA(copy2d(buf, sizeof(float) * npts, pts, sizeof(float) * ld,
                                   sizeof(float) * npts, d, cudaMemcpyHostToDevice, c->stream));
      rbf_update(c, Mat{buf, 1, npts}, npts, d, row0, nrows);
    } else {
      SKEMA_CUDA(copy2d(buf, sizeof(float) * d, pts, sizeof(float) * ld,
                                   sizeof(float) * d, npts, cudaMemcpyHostToDevice, c->stream));
      rbf_update(c, Mat{buf, d, 1}, npts, d, row0, nrows);
    }
  });
}

int skema_low_rank_approx_rows(skema_ctx* c, int64_t row0, int64_t nrows, skema_allreduce_fn allreduce,
                               void* user, double* U, double* S, double* V, int32_t mem) {
  return guarded(c, [&] {
    if (mem != SKEMA_MEM_DEVICE && mem != SKEMA_MEM_HOST) fail(SKEMA_EINVAL, "bad mem kind");
    if (c->spd) fail(SKEMA_EUNSUPPORTED, "SketchySPD contexts take skema_low_rank_approx");
    if (!allreduce) fail(SKEMA_EINVAL, "null all-reduce callback");
    if (row0 < 0 || nrows < 0 || row0 + nrows > c->m) fail(SKEMA_EINVAL, "row range outside A");
    if (c->k > c->n || c->k > c->m) fail(SKEMA_EINVAL, "range must not exceed min(m, n)");
    if (c->s < c->k) fail(SKEMA_EINVAL, "core must be >= range");
    const int64_t r = c->p.rank;
    if (r > c->k) fail(SKEMA_EINVAL, "rank must not exceed range");
    check_device_error(c);
    if (mem == SKEMA_MEM_DEVICE) {
      low_rank_approx_sharded(c, row0, nrows, allreduce, user, U, S, V);
      return;
    }
    const size_t ub = sizeof(double) * (size_t)(nrows * r), vb = sizeof(double) * (size_t)(c->n * r);
    char* buf = (char*)staging(c, ub + vb + sizeof(double) * (size_t)r + 512);
    double* dU = (double*)buf;
    double* dV = (double*)(buf + (ub + 255) / 256 * 256);
    double* dS = (double*)(buf + (ub + 255) / 256 * 256 + (vb + 255) / 256 * 256);
    low_rank_approx_sharded(c, row0, nrows, allreduce, user, U ? dU : nullptr, S ? dS : nullptr, V ? dV : nullptr);
    if (U && ub) SKEMA_CUDA(cudaMemcpyAsync(U, dU, ub, cudaMemcpyDeviceToHost, c->stream));
    if (V) SKEMA_CUDA(cudaMemcpyAsync(V, dV, vb, cudaMemcpyDeviceToHost, c->stream));
    if (S) SKEMA_CUDA(cudaMemcpyAsync(S, dS, sizeof(double) * (size_t)r, cudaMemcpyDeviceToHost, c->stream));
    SKEMA_CUDA(cudaStreamSynchronize(c->stream));
  });
}

int skema_low_rank_approx(skema_ctx* c, double* U, double* S, double* V, int32_t mem) {
  return guarded(c, [&] {
    if (mem != SKEMA_MEM_DEVICE && mem != SKEMA_MEM_HOST) fail(SKEMA_EINVAL, "bad mem kind");
    if (c->spd) {
      if (c->p.spd_approx != SKEMA_SPD_NYSTROM && c->p.spd_approx != SKEMA_SPD_REFERENCE_STEPS)
        fail(SKEMA_EINVAL, "spd_approx must be SKEMA_SPD_NYSTROM or SKEMA_SPD_REFERENCE_STEPS");
      if (c->m != c->n) fail(SKEMA_EINVAL, "SketchySPD needs a square matrix");
      if (c->k > c->m) fail(SKEMA_EINVAL, "range must not exceed the matrix size");
      if (c->p.rank > c->k) fail(SKEMA_EINVAL, "rank must not exceed range");
      check_device_error(c);
      const int64_t r = c->p.rank;
      if (mem == SKEMA_MEM_DEVICE) {
        spd_low_rank_approx(c, U, S);
        if (c->keep_factors && U && S) residual_keep(c, nullptr, S, U);  // the one-sided form's V is U
        return;
      }
      const size_t ub = sizeof(double) * (size_t)(c->m * r);
      char* buf = (char*)staging(c, ub + sizeof(double) * (size_t)r + 512);
      double* dU = (double*)buf;
      double* dS = (double*)(buf + (ub + 255) / 256 * 256);
      const bool keep = c->keep_factors;
      spd_low_rank_approx(c, (U || keep) ? dU : nullptr, (S || keep) ? dS : nullptr);
      if (keep) residual_keep(c, nullptr, dS, dU);
      if (U) SKEMA_CUDA(cudaMemcpyAsync(U, dU, ub, cudaMemcpyDeviceToHost, c->stream));
      if (S) SKEMA_CUDA(cudaMemcpyAsync(S, dS, sizeof(double) * (size_t)r, cudaMemcpyDeviceToHost, c->stream));
      SKEMA_CUDA(cudaStreamSynchronize(c->stream));
      return;
    }
    if (c->k > c->n || c->k > c->m) fail(SKEMA_EINVAL, "range must not exceed min(m, n)");
    if (c->s < c->k) fail(SKEMA_EINVAL, "core must be >= range");
    const int64_t r = c->p.rank;
    if (r > c->k) fail(SKEMA_EINVAL, "rank must not exceed range");
    check_device_error(c);
    if (mem == SKEMA_MEM_DEVICE) {
      low_rank_approx(c, U, S, V);
      if (c->keep_factors && U && S && V) residual_keep(c, U, S, V);
      return;
    }
    const size_t ub = sizeof(double) * (size_t)(c->m * r), vb = sizeof(double) * (size_t)(c->n * r);
    char* buf = (char*)staging(c, ub + vb + sizeof(double) * (size_t)r + 512);
    double* dU = (double*)buf;
    double* dV = (double*)(buf + (ub + 255) / 256 * 256);
    double* dS = (double*)(buf + (ub + 255) / 256 * 256 + (vb + 255) / 256 * 256);
    const bool keep = c->keep_factors;
    low_rank_approx(c, (U || keep) ? dU : nullptr, (S || keep) ? dS : nullptr, (V || keep) ? dV : nullptr);
    if (keep) residual_keep(c, dU, dS, dV);
    if (U) SKEMA_CUDA(cudaMemcpyAsync(U, dU, ub, cudaMemcpyDeviceToHost, c->stream));
    if (V) SKEMA_CUDA(cudaMemcpyAsync(V, dV, vb, cudaMemcpyDeviceToHost, c->stream));
    if (S) SKEMA_CUDA(cudaMemcpyAsync(S, dS, sizeof(double) * (size_t)r, cudaMemcpyDeviceToHost, c->stream));
    SKEMA_CUDA(cudaStreamSynchronize(c->stream));
  });
}

// ---- residual pass ----------------------------------------------------------
int skema_set_keep_factors(skema_ctx* c, int32_t on) {
  return guarded(c, [&] {
    c->keep_factors = on != 0;
    if (!c->keep_factors) c->res_factors_kept = false;
  });
}

int skema_residuals_begin(skema_ctx* c, const double* U, const double* S, const double* V, int32_t mem) {
  return guarded(c, [&] {
    if (mem != SKEMA_MEM_DEVICE && mem != SKEMA_MEM_HOST) fail(SKEMA_EINVAL, "bad mem kind");
    if (!U && !S && !V) {  // the factors the last approximation kept on the device
      residual_begin_kept(c);
      return;
    }
    if (!S || !V || (!c->spd && !U)) fail(SKEMA_EINVAL, "null U, S or V");
    const int64_t r = c->p.rank;
    if (mem == SKEMA_MEM_DEVICE) {
      residual_begin(c, U, S, V);
      return;
    }
    const size_t ub = c->spd ? 0 : sizeof(double) * (size_t)(c->m * r);
    const size_t vb = sizeof(double) * (size_t)(c->n * r), sb = sizeof(double) * (size_t)r;
    const size_t up = (ub + 255) / 256 * 256, vp = (vb + 255) / 256 * 256;
    char* buf = (char*)staging(c, up + vp + sb + 256);
    double* dU = (double*)buf;
    double* dV = (double*)(buf + up);
    double* dS = (double*)(buf + up + vp);
    if (!c->spd) SKEMA_CUDA(cudaMemcpyAsync(dU, U, ub, cudaMemcpyHostToDevice, c->stream));
    SKEMA_CUDA(cudaMemcpyAsync(dV, V, vb, cudaMemcpyHostToDevice, c->stream));
    SKEMA_CUDA(cudaMemcpyAsync(dS, S, sb, cudaMemcpyHostToDevice, c->stream));
    residual_begin(c, dU, dS, dV);
    // the staging buffer is reused by the next host-input call
    SKEMA_CUDA(cudaStreamSynchronize(c->stream));
  });
}

namespace {
// Routes the update entry points to the residual pass for one call.
struct ResidualRoute {
  skema_ctx* c;
  explicit ResidualRoute(skema_ctx* cc) : c(cc) { c->residual_pass = true; }
  ~ResidualRoute() { c->residual_pass = false; }
};
int no_pass(skema_ctx* c) {
  return guarded(c, [&] { fail(SKEMA_ESTATE, "no residual pass open: call skema_residuals_begin first"); });
}
}  // namespace

int skema_residuals_update_dense(skema_ctx* c, const float* A, int64_t ld, int32_t layout, int64_t row0,
                                 int64_t nrows, int32_t mem) {
  if (!c || !c->res_ready) return c ? no_pass(c) : SKEMA_EINVAL;
  ResidualRoute route(c);
  return skema_linear_update_dense(c, A, ld, layout, row0, nrows, mem);
}

int skema_residuals_update_csr(skema_ctx* c, const int64_t* rowptr, const int32_t* col, const float* val,
                               int64_t row0, int64_t nrows, int32_t mem) {
  if (!c || !c->res_ready) return c ? no_pass(c) : SKEMA_EINVAL;
  ResidualRoute route(c);
  return skema_linear_update_csr(c, rowptr, col, val, row0, nrows, mem);
}

int skema_residuals_update_rbf(skema_ctx* c, const float* pts, int64_t ld, int32_t layout, int64_t npts, int64_t d,
                               int64_t row0, int64_t nrows, int32_t mem) {
  if (!c || !c->res_ready) return c ? no_pass(c) : SKEMA_EINVAL;
  ResidualRoute route(c);
  return skema_linear_update_rbf(c, pts, ld, layout, npts, d, row0, nrows, mem);
}

int skema_residuals_finish(skema_ctx* c, double* rnorms, int32_t mem) {
  return guarded(c, [&] {
    if (mem != SKEMA_MEM_DEVICE && mem != SKEMA_MEM_HOST) fail(SKEMA_EINVAL, "bad mem kind");
    if (!rnorms) fail(SKEMA_EINVAL, "null rnorms");
    if (!c->res_ready) fail(SKEMA_ESTATE, "no residual pass open: call skema_residuals_begin first");
    check_device_error(c);
    const int64_t r = c->p.rank;
    if (mem == SKEMA_MEM_DEVICE) {
      residual_finish(c, rnorms);
      return;
    }
    double* d = (double*)staging(c, sizeof(double) * (size_t)r + 256);
    residual_finish(c, d);
    SKEMA_CUDA(cudaMemcpyAsync(rnorms, d, sizeof(double) * (size_t)r, cudaMemcpyDeviceToHost, c->stream));
    SKEMA_CUDA(cudaStreamSynchronize(c->stream));
  });
}

static void sketch_shape(const skema_ctx* c, int32_t which, float** p, int64_t* rows, int64_t* cols) {
  switch (which) {
    case SKEMA_SKETCH_X:
      *p = c->X, *rows = c->k, *cols = c->n;
      break;
    case SKEMA_SKETCH_Y:
      *p = c->Y, *rows = c->m, *cols = c->k;
      break;
    case SKEMA_SKETCH_Z:
      *p = c->Z, *rows = c->s, *cols = c->s;
      break;
    default:
      fail(SKEMA_EINVAL, "which must be X, Y or Z");
  }
  if (!*p) fail(SKEMA_ESTATE, "this context has no such sketch (SketchySPD keeps Y only)");
}

// X and Z are kept row-major, Y column-major (LayoutLeft, ld = m).
static bool sketch_row_major(int32_t which) { return which != SKEMA_SKETCH_Y; }

int skema_get_sketch(skema_ctx* c, int32_t which, float* buf, int64_t ld, int32_t layout,
                     int32_t mem) {
  return guarded(c, [&] {
    float* src;
    int64_t rows, cols;
    sketch_shape(c, which, &src, &rows, &cols);
    check_dense_args(buf, ld, layout, rows, cols, mem);
    check_device_error(c);
    if (which == SKEMA_SKETCH_Y) y_materialize(c);
    const bool irow = sketch_row_major(which);
    const int64_t inner = irow ? cols : rows, outer = irow ? rows : cols;
    const Mat sm = irow ? Mat{src, cols, 1} : Mat{src, 1, rows};
    const bool want_row = layout == SKEMA_ROW_MAJOR;
    const cudaMemcpyKind kind = mem == SKEMA_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    if (want_row == irow) {
      SKEMA_CUDA(copy2d(buf, sizeof(float) * ld, src, sizeof(float) * inner,
                                   sizeof(float) * inner, outer, kind, c->stream));
    } else if (mem == SKEMA_MEM_DEVICE) {
      copy_block(c, sm, want_row ? MatOut{buf, ld, 1} : MatOut{buf, 1, ld}, rows, cols);
    } else {
      // The transposed copy goes out in chunks of the host layout's outer
      // dimension through two staging slots: the side stream transposes
      // chunk i + 1 while the context stream copies chunk i to the host, so
      // the transposes hide behind the PCIe copy.
      const int64_t tin = want_row ? cols : rows, tout = want_row ? rows : cols;
      const int64_t och = std::max<int64_t>(1, std::min<int64_t>(tout, ((int64_t)8 << 20) / tin));
      const size_t slot_bytes = (sizeof(float) * (size_t)(och * tin) + 255) / 256 * 256;
      char* tmp = (char*)staging(c, 2 * slot_bytes);
      cudaEvent_t tr_done[2] = {c->stage_ev[0], c->stage_ev[1]}, out_done[2] = {c->stage_ev[2], c->stage_ev[3]};
      SKEMA_CUDA(cudaEventRecord(c->fork_ev, c->stream));
      SKEMA_CUDA(cudaStreamWaitEvent(c->side, c->fork_ev, 0));
      for (int64_t o0 = 0, i = 0; o0 < tout; o0 += och, ++i) {
        const int64_t n = std::min(och, tout - o0);
        const int sl = (int)(i & 1);
        float* slot = (float*)(tmp + sl * slot_bytes);
        if (i >= 2) SKEMA_CUDA(cudaStreamWaitEvent(c->side, out_done[sl], 0));
        // the chunk's outer dimension is the one contiguous in the stored sketch
        if (tin <= 256)
          transpose_narrow(c, sm.p + o0, n, tin, want_row ? sm.cs : sm.rs, slot, c->side);
        else if (want_row)
          copy_block(c, Mat{sm.p + o0 * sm.rs, sm.rs, sm.cs}, MatOut{slot, cols, 1}, n, cols, c->side);
        else
          copy_block(c, Mat{sm.p + o0 * sm.cs, sm.rs, sm.cs}, MatOut{slot, 1, rows}, rows, n, c->side);
        SKEMA_CUDA(cudaEventRecord(tr_done[sl], c->side));
        SKEMA_CUDA(cudaStreamWaitEvent(c->stream, tr_done[sl], 0));
        SKEMA_CUDA(copy2d(buf + o0 * ld, sizeof(float) * ld, slot, sizeof(float) * tin,
                                     sizeof(float) * tin, n, cudaMemcpyDeviceToHost, c->stream));
        SKEMA_CUDA(cudaEventRecord(out_done[sl], c->stream));
      }
    }
    if (mem == SKEMA_MEM_HOST) SKEMA_CUDA(cudaStreamSynchronize(c->stream));
  });
}

int skema_set_sketch(skema_ctx* c, int32_t which, const float* buf, int64_t ld, int32_t layout,
                     int32_t mem) {
  return guarded(c, [&] {
    float* dst;
    int64_t rows, cols;
    sketch_shape(c, which, &dst, &rows, &cols);
    check_dense_args(buf, ld, layout, rows, cols, mem);
    const bool irow = sketch_row_major(which);
    const int64_t inner = irow ? cols : rows, outer = irow ? rows : cols;
    const MatOut dm = irow ? MatOut{dst, cols, 1} : MatOut{dst, 1, rows};
    const bool have_row = layout == SKEMA_ROW_MAJOR;
    const cudaMemcpyKind kind = mem == SKEMA_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    if (have_row == irow) {
      SKEMA_CUDA(copy2d(dst, sizeof(float) * inner, buf, sizeof(float) * ld,
                                   sizeof(float) * inner, outer, kind, c->stream));
    } else if (mem == SKEMA_MEM_DEVICE) {
      copy_block(c, have_row ? Mat{buf, ld, 1} : Mat{buf, 1, ld}, dm, rows, cols);
    } else {
      const int64_t tin = have_row ? cols : rows, tout = have_row ? rows : cols;
      float* tmp = (float*)staging(c, sizeof(float) * (size_t)(rows * cols));
      SKEMA_CUDA(copy2d(tmp, sizeof(float) * tin, buf, sizeof(float) * ld,
                                   sizeof(float) * tin, tout, cudaMemcpyHostToDevice, c->stream));
      copy_block(c, have_row ? Mat{tmp, cols, 1} : Mat{tmp, 1, rows}, dm, rows, cols);
    }
    if (which == SKEMA_SKETCH_Y) {
      c->y_written.clear();
      y_rows_mark(c, 0, c->m);
    }
    SKEMA_CUDA(cudaStreamSynchronize(c->stream));
  });
}

static Map* map_of(skema_ctx* c, int32_t which) {
  Map* mp = nullptr;
  switch (which) {
    case SKEMA_UPSILON: mp = &c->ups; break;
    case SKEMA_OMEGA: mp = &c->omg; break;
    case SKEMA_PHI: mp = &c->phi; break;
    case SKEMA_PSI: mp = &c->psi; break;
    default: fail(SKEMA_EINVAL, "which must be UPSILON, OMEGA, PHI or PSI");
  }
  if (mp->nrow == 0) fail(SKEMA_ESTATE, "this context has no such map (SketchySPD keeps Omega only)");
  return mp;
}

int skema_map_info(const skema_ctx* cc, int32_t which, int64_t* nrow, int64_t* ncol,
                   int32_t* zeta, int32_t* transposed) {
  skema_ctx* c = const_cast<skema_ctx*>(cc);
  return guarded(c, [&] {
    Map* mp = map_of(c, which);
    if (nrow) *nrow = mp->nrow;
    if (ncol) *ncol = mp->ncol;
    if (zeta) *zeta = mp->kind == SKEMA_MAP_SPARSE_SIGN ? mp->zeta : 0;
    // The reference's init_transposed flag: SketchySPD's Omega is built
    // without it even though it is applied as A * Omega.
    if (transposed) *transposed = (mp->transposed && !c->spd) ? 1 : 0;
  });
}

}  // extern "C"

namespace skema {
void map_export(skema_ctx* c, Map& mp, double* values, int32_t* indices);
void map_import(skema_ctx* c, Map& mp, const double* values, const int32_t* indices);
}  // namespace skema

extern "C" {

int skema_map_export(skema_ctx* c, int32_t which, double* values, int32_t* indices) {
  return guarded(c, [&] {
    Map* mp = map_of(c, which);
    map_export(c, *mp, values, indices);
  });
}

int skema_map_import(skema_ctx* c, int32_t which, const double* values, const int32_t* indices) {
  return guarded(c, [&] {
    Map* mp = map_of(c, which);
    map_import(c, *mp, values, indices);
    tc_prepare_maps(c);
  });
}

int skema_rbf_sketch_fwd(skema_ctx* c, const float* pts, int64_t npts, int64_t d, double gamma,
                         const float* omega, int64_t k, float* Y) {
  return guarded(c, [&] {
    if (npts <= 0 || d <= 0 || k <= 0) fail(SKEMA_EINVAL, "npts, d and k must be > 0");
    if (!pts || !omega || !Y) fail(SKEMA_EINVAL, "null pointer");
    if (!(gamma >= 0.0)) fail(SKEMA_EINVAL, "gamma must be >= 0");
    rbf_fwd(c, pts, npts, d, gamma, omega, k, Y);
  });
}

int skema_rbf_sketch_vjp(skema_ctx* c, const float* pts, int64_t npts, int64_t d, double gamma,
                         const float* omega, int64_t k, const float* Ybar, float* dpts,
                         double* dgamma) {
  return guarded(c, [&] {
    if (npts <= 0 || d <= 0 || k <= 0) fail(SKEMA_EINVAL, "npts, d and k must be > 0");
    if (!pts || !omega || !Ybar || !dpts || !dgamma) fail(SKEMA_EINVAL, "null pointer");
    if (!(gamma >= 0.0)) fail(SKEMA_EINVAL, "gamma must be >= 0");
    rbf_vjp(c, pts, npts, d, gamma, omega, k, Ybar, dpts, dgamma);
  });
}

int skema_synchronize(skema_ctx* c) {
  return guarded(c, [&] {
    SKEMA_CUDA(cudaStreamSynchronize(c->stream));
    check_device_error(c);
  });
}

int skema_set_stream(skema_ctx* c, void* stream) {
  return guarded(c, [&] {
    SKEMA_CUDA(cudaStreamSynchronize(c->stream));
    check_device_error(c);
    c->stream = stream ? (cudaStream_t)stream : c->own_stream;
  });
}

int skema_get_stream(const skema_ctx* c, void** stream) {
  if (!c || !stream) return SKEMA_EINVAL;
  *stream = (void*)c->stream;
  return SKEMA_OK;
}

int skema_set_wait_limit(skema_ctx* c, int64_t ns) {
  return guarded(c, [&] {
    SKEMA_CUDA(cudaStreamSynchronize(c->stream));
    check_device_error(c);
    set_wait_limit(c, ns);
  });
}

int skema_set_workspace_limit(skema_ctx* c, int64_t bytes) {
  return guarded(c, [&] {
    if (bytes < 0) fail(SKEMA_EINVAL, "workspace limit must be >= 0");
    c->ws_limit = (size_t)bytes;
  });
}

int64_t skema_launch_count(const skema_ctx* c) { return c ? c->launches : -1; }

int skema_timing_enable(skema_ctx* c, int32_t on) {
  return guarded(c, [&] {
    drain_timers(c);
    for (int i = 0; i < ST_COUNT; ++i) {
      c->stage_ms[i] = 0.0;
      c->stage_n[i] = 0;
    }
    c->timing = on != 0;
  });
}

int skema_timing_get(skema_ctx* c, const char* stage, double* ms, int64_t* count) {
  return guarded(c, [&] {
    if (!stage) fail(SKEMA_EINVAL, "null stage name");
    drain_timers(c);
    if (std::strcmp(stage, "approx.svd_sweeps") == 0) {
      if (ms) *ms = 0.0;
      if (count) *count = c->svd_sweeps;
      return;
    }
    for (int i = 0; i < ST_COUNT; ++i) {
      if (std::strcmp(stage, kStageNames[i]) == 0) {
        if (ms) *ms = c->stage_ms[i];
        if (count) *count = c->stage_n[i];
        return;
      }
    }
    fail(SKEMA_EINVAL, std::string("unknown stage ") + stage);
  });
}

}  // extern "C"
