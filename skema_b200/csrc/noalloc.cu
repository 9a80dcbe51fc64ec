// noalloc.cu -- skema_rbf_sketch_fwd_noalloc: the RBF-kernel sketch forward
// pass (Y = K Omega^T) for callers that must not allocate device memory.
//
// The regular entry point (skema_rbf_sketch_fwd) builds kernel row blocks in
// the context's workspace, which it grows with cudaMalloc on first use. Some
// callers cannot let a library allocate: a host framework that owns all
// device memory through its own pool or memory cap, or a latency-critical
// loop where cudaMalloc's implicit device-wide synchronisation would stall
// other streams. This variant takes its scratch from one fixed array in the
// library image instead and allocates nothing, at the price of smaller row
// blocks (more, smaller launches).
//
// The scratch is kNoAllocScratchFloats floats (16 MiB); every GPU that loads
// the library holds it until the process exits. All calls on a device share
// it and it keeps the last call's contents. Nothing in it needs to start at
// zero: each kernel row block is fully written before it is read. Calls that
// overlap on the GPU (different streams or contexts at the same time) race
// on the array and must be serialised by the caller.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "internal.h"

namespace skema {

void rbf_window_block(skema_ctx* c, Mat P, int64_t N, int64_t d, float gamma, int64_t R0,
                      int64_t wr, float* out, int64_t ldo);

constexpr int64_t kNoAllocScratchFloats = int64_t(1) << 22;  // 16 MiB
constexpr int kMaxDevices = 64;

static __device__ __align__(256) float g_noalloc_scratch[kNoAllocScratchFloats];

static float* g_scratch_addr[kMaxDevices];
static std::once_flag g_scratch_once[kMaxDevices];
static cudaError_t g_scratch_err[kMaxDevices];

// Device address of the scratch array on the current device (which must be
// `dev`). The host-side name g_noalloc_scratch is only a stand-in for the
// symbol, not a device address, so the address is looked up once per
// device with that device current.
static float* noalloc_scratch(int dev) {
  if (dev < 0 || dev >= kMaxDevices) fail(SKEMA_EINVAL, "device ordinal beyond the no-alloc scratch table");
  std::call_once(g_scratch_once[dev], [dev] {
    void* p = nullptr;
    g_scratch_err[dev] = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    g_scratch_addr[dev] = static_cast<float*>(p);
  });
  cuda_check(g_scratch_err[dev], "cudaGetSymbolAddress(no-alloc scratch)");
  return g_scratch_addr[dev];
}

}  // namespace skema

using namespace skema;

extern "C" int skema_rbf_sketch_fwd_noalloc(skema_ctx* c, const float* pts, int64_t npts, int64_t d,
                                            double gamma, const float* omega, int64_t k, float* Y) {
  if (!c) return SKEMA_EINVAL;
  try {
    SKEMA_CUDA(cudaSetDevice(c->dev));
    if (npts <= 0 || d <= 0 || k <= 0) fail(SKEMA_EINVAL, "npts, d and k must be > 0");
    if (!pts || !omega || !Y) fail(SKEMA_EINVAL, "null pointer");
    if (!(gamma >= 0.0)) fail(SKEMA_EINVAL, "gamma must be >= 0");
    if (npts > kNoAllocScratchFloats)
      fail(SKEMA_EINVAL, "npts exceeds the no-alloc scratch: at most 4194304 points (one kernel row "
                         "of npts floats must fit in the 16 MiB static array)");
    float* Kw = noalloc_scratch(c->dev);
    const int64_t N = npts;
    const int64_t wb = std::min<int64_t>(N, kNoAllocScratchFloats / N);  // rows per kernel block
    const Mat P{pts, d, 1};
    for (int64_t r = 0; r < N; r += wb) {
      const int64_t wr = std::min(wb, N - r);
      rbf_window_block(c, P, N, d, (float)gamma, r, wr, Kw, N);
      // Y(r:r+wr, :) = K_w Omega~^T with Omega~ (k x N) row-major
      sgemm(c, wr, k, N, 1.f, Mat{Kw, N, 1}, Mat{omega, 1, N}, 0.f, MatOut{Y + r * k, k, 1});
    }
    c->err.clear();
    return SKEMA_OK;
  } catch (const Error& e) {
    c->err = e.msg;
    return e.status;
  } catch (...) {
    c->err = "unexpected C++ exception";
    return SKEMA_ECUDA;
  }
}
