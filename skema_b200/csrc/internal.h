// internal.h -- private declarations shared by the library's translation
// units: the context, map storage and the launchers of every kernel.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <utility>
#include <vector>

#include "../../include/skema_c.h"

namespace skema {

// Thrown inside the library only; converted to a status at the C boundary.
struct Error {
  int status;
  std::string msg;
};

[[noreturn]] void fail(int status, const std::string& msg);
void cuda_check(cudaError_t e, const char* what);
#define SKEMA_CUDA(call) ::skema::cuda_check((call), #call)
// After a kernel launch: reports launch-configuration errors.
#define SKEMA_LAUNCHED(ctx) \
  do {                      \
    ::skema::cuda_check(cudaGetLastError(), "kernel launch"); \
    (ctx)->launches++;      \
  } while (0)

// A random map on the device.
//
// `nrow x ncol` is the stored shape of the reference's DimRedux ctor; the
// map is `transposed` when that ctor got init_transposed=true
// (src/Skema_SketchySVD.cpp:30-95). `lrows x lcols` is the logical operator
// the sketch formulas use: Upsilon~ (k x m), Omega~ (k x n), Phi~ (s x m),
// Psi~ (s x n); logical = stored^T when transposed.
struct Map {
  int kind = SKEMA_MAP_GAUSS;
  int64_t nrow = 0, ncol = 0;
  bool transposed = false;
  int64_t lrows = 0, lcols = 0;
  uint32_t seed = 0;
  double maxval = 0.0;
  int zeta = 0;
  // Gauss: FP32 values; logical (r, c) at f32[r*rs + c*cs].
  float* f32 = nullptr;
  int64_t rs = 0, cs = 0;
  // Gauss, tensor-core forms: logical rows in row-major BF16 / FP8 copies.
  void* lowp = nullptr;
  // SparseSign: stored rows, zeta packed entries each: column | sign << 31.
  uint32_t* packed = nullptr;
  // Stored-transposed SparseSign with zeta == 8 and ncol <= 128, as eight
  // 16-bit entries per stored row (16 bytes): (column * 128) | sign << 15,
  // the byte offset of the column's bin in a warp's bin-major accumulator
  // (the streaming Y kernel's map format).
  void* packed16 = nullptr;
  // SparseSign maps that are row-sparse over the input rows (Upsilon, Phi of
  // the three-sketch): (input row, map row, sign) triples sorted by input
  // row, on the host and on the device.
  std::vector<int64_t> inv_row;   // host, sorted input rows
  int64_t* d_inv_row = nullptr;   // device copy of inv_row
  uint32_t* d_inv_rs = nullptr;   // device: map row | sign << 31
};

struct Interval {
  int64_t a, b;
};

enum Stage {
  ST_OMEGA = 0,
  ST_PSI,
  ST_UPSILON,
  ST_PHI,
  ST_ENTRIES,
  ST_WINDOW,
  ST_FUSED,
  ST_DAXPY,
  ST_A_ORTH,     // orthonormal bases of Y and X^T
  ST_A_CORE,     // the core matrix: Phi Q, Psi P, their QR and the solves
  ST_A_SVD,      // the core matrix's SVD
  ST_A_VECTORS,  // U = Q Uc, V = P Vc
  ST_COUNT
};
extern const char* const kStageNames[ST_COUNT];

struct PendingTimer {
  int stage;
  cudaEvent_t a, b;
};

}  // namespace skema

struct skema_ctx {
  skema_params p;
  int64_t m = 0, n = 0, k = 0, s = 0, w = 1;
  bool spd = false;     // SketchySPD: only Y = A Omega
  int dev = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  // Side stream for work that runs beside a kernel on `stream` within one
  // call (forked from and joined back to `stream` before the call returns).
  cudaStream_t side = nullptr;
  cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
  // Hand-offs between the two streams of the BF16 dense pipeline (window
  // copies ready / released, one pair per copy buffer).
  cudaEvent_t pipe_ev[4] = {nullptr, nullptr, nullptr, nullptr};
  // host staging through two slots (uploads and transposed fetches): slot i
  // filled / slot i read, i = 0, 1
  cudaEvent_t stage_ev[4] = {nullptr, nullptr, nullptr, nullptr};
  std::string err;
  int64_t launches = 0;
  skema::Map ups, omg, phi, psi;
  // Sketches, FP32: X k x n and Z s x s row-major; Y m x k column-major
  // (ld = m, the reference's LayoutLeft).
  float* X = nullptr;
  float* Y = nullptr;
  float* Z = nullptr;
  // Rows of Y written since the last reset (merged, sorted intervals).
  std::vector<skema::Interval> y_written;
  // X and Z are zeroed lazily after a reset: every entry point zeroes them
  // on `stream` first (xz_materialize), except the CSR update, which zeroes
  // them on the side stream beside its Y kernel when it touches them.
  bool xz_pending = false;
  bool xz_defer = false;
  // Workspace (grown on demand, owned).
  void* ws = nullptr;
  size_t ws_bytes = 0;
  void* stage = nullptr;  // host-input staging
  size_t stage_bytes = 0;
  size_t ws_limit = 0;    // cap on ws_bytes + stage_bytes (0: none)
  int sm_count = 148;
  // Upper bound on the CTAs of one tensor-core launch (0: one per SM); set
  // while the dense pipeline splits the SMs between its two streams.
  int tc_cta_cap = 0;
  // Dense BF16 / FP8 pipeline: SMs given to the X^T product (0: no
  // pipeline, the products run one after another on all SMs) and windows
  // per [Y | T] group. Defaults set at creation; SKEMA_DENSE_PIPE_SMS and
  // SKEMA_DENSE_PIPE_WINDOWS override them.
  int pipe_xt_sms = 0;
  int64_t pipe_windows = 2;
  // Shared memory per SM for the CSR x SparseSign Y kernel's bins, in KB
  // (it sets the warps per SM; the rest of the unified L1 / shared memory
  // stays L1). SKEMA_SSIGN_BIN_KB overrides the default.
  int ssign_bin_kb = 128;
  // Nonzeros each lane of that kernel loads ahead per step (2, 4, 6 or 8);
  // SKEMA_SSIGN_BATCH overrides the default.
  int ssign_batch = 4;
  // X^T product from an FP32 window: a thread of its own issues the BF16
  // window copy's stores (true, 2-3 % faster X^T) or a converter thread
  // does (false); SKEMA_XT_STORE_THREAD=1|0 overrides the default.
  bool xt_store_thread = true;
  int cc_major = 0, cc_minor = 0;
  // BF16 tensor-core form: Omega~ and Psi~ stacked as one (k+s) x n
  // row-major operand (ld_op16), Upsilon~ / Phi~ copies in Map::lowp with
  // ld_maps16; padded row strides are multiples of 8 elements.
  void* op16 = nullptr;
  int64_t ld_op16 = 0, ld_maps16 = 0;
  // FP8 form: the Gauss maps are held on the E4M3 grid scaled by
  // fp8_map_scale (a power of two, so every map value is exact in FP8, BF16
  // and FP32 alike); op8 is E4M3(fp8_map_scale [Omega~; Psi~]), (k+s) x n
  // row-major with ld_op8 (a multiple of 16 bytes). fp8_win holds, on the
  // device, the amax bits of the current window's A and the product scale
  // 1 / (scale_A * fp8_map_scale) of its [Y | T] GEMM.
  void* op8 = nullptr;
  int64_t ld_op8 = 0;
  float fp8_map_scale = 1.f;
  uint32_t* fp8_win = nullptr;
  int64_t fp8_win_cap = 1;  // windows fp8_win has room for (amax and scale each)
  // Residual pass (skema_residuals_*): the approximation's U and V as
  // row-major FP64 copies (m x r, n x r), S, the accumulated A^T U (n x r,
  // row-major) and the per-column sums of squares of A V - U S. While
  // residual_pass is set, the update entry points feed the residual pass
  // instead of the sketches.
  double* res_U = nullptr;
  double* res_V = nullptr;
  double* res_S = nullptr;
  double* res_AtU = nullptr;
  double* res_sq = nullptr;
  bool res_ready = false;
  // skema_set_keep_factors: each low_rank_approx also loads its U, S, V into
  // the residual buffers (res_factors_kept then holds), so a residual pass
  // can open on them without a host copy
  bool keep_factors = false;
  bool res_factors_kept = false;
  bool residual_pass = false;
  // Device status block of the bounded waits in the tensor-core kernels:
  // dev_err[0] non-zero when a wait timed out (checked at the next
  // synchronising call); dev_err[2..3] the wait limit in ns (64-bit).
  int* dev_err = nullptr;
  bool dev_err_armed = false;
  // stage timers
  bool timing = false;
  std::vector<skema::PendingTimer> pending;
  std::vector<cudaEvent_t> event_pool;
  // Sweeps of the last core-matrix SVD (the Jacobi iteration's count).
  int64_t svd_sweeps = 0;
  double stage_ms[skema::ST_COUNT] = {0};
  int64_t stage_n[skema::ST_COUNT] = {0};
};

namespace skema {

// Records CUDA events around the launches of one stage while timing is on.
class StageScope {
 public:
  StageScope(skema_ctx* c, int stage);
  StageScope(skema_ctx* c, int stage, cudaStream_t stream);
  ~StageScope();
  StageScope(const StageScope&) = delete;
  StageScope& operator=(const StageScope&) = delete;

 private:
  skema_ctx* c_;
  int stage_;
  cudaStream_t stream_;
  cudaEvent_t a_ = nullptr;
};

void* workspace(skema_ctx* c, size_t bytes);
void* staging(skema_ctx* c, size_t bytes);
bool y_rows_clean(const skema_ctx* c, int64_t a, int64_t b);
void y_rows_mark(skema_ctx* c, int64_t a, int64_t b);
// Zero every Y row not written since the last reset.
void y_materialize(skema_ctx* c);
// The beta an update of Y rows [a, b) applies on the context stream: 0 when
// no row of the range was written since the reset (the kernel then writes
// without reading), else nu, after the range's unwritten rows were zeroed.
float y_beta(skema_ctx* c, int64_t a, int64_t b, float nu);
// Zero X and Z on `stream` if a reset left them pending.
void xz_materialize(skema_ctx* c, cudaStream_t stream);

// ---- maps (maps.cu) ----
void map_generate(skema_ctx* c, Map& mp, int precision);
void map_free(Map& mp);
void map_build_inverse(skema_ctx* c, Map& mp);

// ---- FP32 SIMT GEMM (gemm_f32.cu) ----
// C(i,j) = alpha * sum_kk A(i,kk) B(kk,j) + beta * C(i,j), every operand
// addressed by (row stride, col stride). With splitk > 1 the K range is
// split over grid.z and partial results are added atomically (requires the
// caller to have applied beta beforehand; beta is ignored).
struct Mat {
  const float* p;
  int64_t rs, cs;
};
struct MatOut {
  float* p;
  int64_t rs, cs;
};
void sgemm(skema_ctx* c, int64_t M, int64_t N, int64_t K, float alpha, Mat A,
           Mat B, float beta, MatOut C, int splitk = 1);
// The same product, with the K dimension split when the output tiles would
// fill less than two waves: the splits write partial products into part
// (capacity part_floats; at most 16 splits of 1024 or more) and one pass
// sums them in a fixed order into C. Without room it falls back to sgemm.
void sgemm_split(skema_ctx* c, int64_t M, int64_t N, int64_t K, float alpha, Mat A, Mat B, float beta, MatOut C,
                 float* part, int64_t part_floats);
// C = beta * C over an M x N strided block.
void scale_block(skema_ctx* c, MatOut C, int64_t M, int64_t N, float beta, cudaStream_t stream = nullptr);
// dst(i,j) = alpha * src(i,j) + beta * dst(i,j) over M x N (beta 0: no read).
void axpby_block(skema_ctx* c, Mat src, MatOut dst, int64_t M, int64_t N,
                 float alpha, float beta);
// Copy a strided FP32 block into another strided block.
void copy_block(skema_ctx* c, Mat src, MatOut dst, int64_t M, int64_t N);
void copy_block(skema_ctx* c, Mat src, MatOut dst, int64_t M, int64_t N, cudaStream_t st);
// dst[l * ns + s] = src[l + s * ss] (l < nl, s < ns <= 256) on stream st.
void transpose_narrow(skema_ctx* c, const float* src, int64_t nl, int64_t ns, int64_t ss, float* dst,
                      cudaStream_t st);

// ---- dense update (dense.cu) ----
// One call of skema_linear_update_dense on device data.
void dense_update(skema_ctx* c, Mat A, int64_t row0, int64_t nrows);
// Per-window body shared with the RBF path: A_w holds rows [R0, R0+wr) of
// the input; T is the scratch returned for dense_scratch_bytes(c, wr).
void dense_window(skema_ctx* c, Mat Aw, int64_t R0, int64_t wr, float* T);
size_t dense_scratch_bytes(const skema_ctx* c, int64_t wr);

// ---- BF16 tensor-core form (dense_tc.cu) ----
bool tc_available(const skema_ctx* c);
void tc_prepare_maps(skema_ctx* c);
size_t tc_scratch_bytes(const skema_ctx* c, int64_t wr);
void tc_dense_window(skema_ctx* c, Mat Aw, int64_t R0, int64_t wr, void* scratch);
// All windows of one dense call in the tensor-core forms ([Y | T] and Z per
// group of windows).
void tc_dense_update(skema_ctx* c, Mat A, int64_t row0, int64_t nrows);
// Reads the tensor-core status word (synchronises the stream) and fails with
// SKEMA_ETIMEOUT if a kernel gave up on a wait since the last check.
void check_device_error(skema_ctx* c);
// The default limit of one bounded device wait, in ns.
unsigned long long tc_default_wait_ns();

// ---- sparse paths (sparse.cu) ----
void csr_update(skema_ctx* c, const int64_t* rowptr, const int32_t* col,
                const float* val, int64_t col_offset, int64_t row0,
                int64_t nrows);
void dense_ssign_window(skema_ctx* c, Mat Aw, int64_t R0, int64_t wr);
void spd_ssign_window(skema_ctx* c, Mat Aw, int64_t R0, int64_t wr);

// ---- RBF, BF16 tensor-core form without a stored kernel (rbf_tc.cu) ----
bool rbf_tc_supported(const skema_ctx* c, int64_t d);
void rbf_tc_update(skema_ctx* c, Mat P, int64_t npts, int64_t d, int64_t row0, int64_t nrows);
// The standalone forward / adjoint pair in the same form (d <= 64, k <= 192).
bool rbf_pair_tc_supported(const skema_ctx* c, int64_t d, int64_t k, double gamma);
void rbf_fwd_tc(skema_ctx* c, const float* pts, int64_t N, int64_t d, double gamma, const float* omega, int64_t k,
                float* Y);
void rbf_vjp_tc(skema_ctx* c, const float* pts, int64_t N, int64_t d, double gamma, const float* omega, int64_t k,
                const float* Ybar, float* dpts, double* dgamma);

// ---- RBF (rbf.cu) ----
void rbf_update(skema_ctx* c, Mat P, int64_t npts, int64_t d, int64_t row0,
                int64_t nrows);
void rbf_fwd(skema_ctx* c, const float* pts, int64_t N, int64_t d,
             double gamma, const float* omega, int64_t k, float* Y);
void rbf_vjp(skema_ctx* c, const float* pts, int64_t N, int64_t d,
             double gamma, const float* omega, int64_t k, const float* Ybar,
             float* dpts, double* dgamma);

// ---- FP64 approximation (approx.cu) ----
void low_rank_approx(skema_ctx* c, double* U, double* S, double* V);
// Rows [row0, row0 + nrows) of a row-block sharded sketch, sums over the
// ranks through fn (skema_low_rank_approx_rows).
void low_rank_approx_sharded(skema_ctx* c, int64_t row0, int64_t nrows, skema_allreduce_fn fn, void* user,
                             double* U, double* S, double* V);
// SketchySPD: U (m x rank, column-major) and S (rank), device pointers (either may be NULL).
void spd_low_rank_approx(skema_ctx* c, double* U, double* S);
// C = alpha A B + beta C in FP64 (A FP32, exact in FP64), strided operands.
void dgemm_f32_f64(skema_ctx* c, int64_t M, int64_t N, int64_t K, double alpha, const float* A, int64_t ars,
                   int64_t acs, const double* B, int64_t brs, int64_t bcs, double beta, double* C, int64_t crs,
                   int64_t ccs);

// ---- residual norms (residuals.cu) ----
// U (m x r), S (r), V (n x r) column-major, device pointers.
void residual_begin(skema_ctx* c, const double* U, const double* S, const double* V);
// Loads device U (m x r, column-major; unused for SketchySPD), S and V into
// the residual buffers and marks them as the kept factors.
void residual_keep(skema_ctx* c, const double* U, const double* S, const double* V);
// Opens a residual pass on the kept factors (SKEMA_ESTATE without them).
void residual_begin_kept(skema_ctx* c);
void residual_dense(skema_ctx* c, Mat A, int64_t row0, int64_t nrows);
void residual_csr(skema_ctx* c, const int64_t* rowptr, const int32_t* col, const float* val, int64_t col_offset,
                  int64_t row0, int64_t nrows);
void residual_rbf(skema_ctx* c, Mat P, int64_t npts, int64_t d, int64_t row0, int64_t nrows);
// rnorms (r doubles, device pointer).
void residual_finish(skema_ctx* c, double* rnorms);
void residual_free(skema_ctx* c);

}  // namespace skema
