// tc_host.h -- host-side pieces shared by the tensor-core forms of the
// sketch (dense windows in dense_tc.cu, Gauss-RBF windows in rbf_tc.cu).
#pragma once
#include <cuda_bf16.h>

#include "internal.h"
#include "tc_gemm.cuh"
#include "tma.h"

namespace skema {

inline int64_t pad8(int64_t x) { return (x + 7) / 8 * 8; }

// A split of K into ks ranges of kchunk (a multiple of the kernel's K
// step), or, with streamk > 0, a stream-K schedule over streamk CTAs (each
// takes an equal run of the tiles' K-steps). Either split adds partial sums
// atomically into outputs scaled beforehand.
struct Plan {
  int ks;
  int64_t kchunk;
  int streamk = 0;
  bool split() const { return ks > 1 || streamk > 0; }
};
// Stream-K over `ctas` CTAs (at most one per SM).
Plan plan_streamk(const skema_ctx* c, int ctas);
// Split that minimises waves x (k-steps per split + fill) for a product
// bound by the tensor pipe, one CTA per SM.
Plan plan_split(const skema_ctx* c, int64_t tiles, int64_t K, int max_ks);

tc::OutSpec out_spec();

CUtensorMap tmap_bf16(const void* base, uint64_t d0, uint64_t d1, uint64_t st1, uint32_t b0, uint32_t b1);

// FP32 strided block -> BF16 with D(i, j) at D[i * drs + j * dcs].
void to_bf16(skema_ctx* c, Mat src, int64_t rows, int64_t cols, __nv_bfloat16* D, int64_t drs, int64_t dcs);
// BF16 column-major (ld16) <- FP32 column-major (ld32), rows x cols; T16lo
// (when given, ld16) receives the BF16 rounding of the remainder.
void t32_to_t16(skema_ctx* c, const float* T32, int64_t ld32, __nv_bfloat16* T16, __nv_bfloat16* T16lo, int64_t ld16,
                int64_t rows, int64_t cols);

// The window's columns of the BF16 Upsilon~ / Phi~ copies as TMA operands:
// in place when R0 is a multiple of 8 (16-byte aligned), else converted
// into scratch taken from *sp (k x wp and s x wp, 256-byte aligned).
struct TcSlices {
  const __nv_bfloat16* U16;
  const __nv_bfloat16* F16;
  int64_t ldm;
};
TcSlices tc_window_slices(skema_ctx* c, int64_t R0, int64_t wr, char** sp);
size_t tc_slice_bytes(const skema_ctx* c, int64_t wr);

// Z = beta Z + eta Phi~(:, rows) T for T (BF16, K x s column-major, ld
// ldT) over K rows whose Phi~ columns are sl.F16, as Z^T = T^T Phi~^T on
// the tensor cores.
void tc_z_update(skema_ctx* c, const __nv_bfloat16* T16, int64_t ldT, const TcSlices& sl, int64_t K, float beta);

}  // namespace skema
