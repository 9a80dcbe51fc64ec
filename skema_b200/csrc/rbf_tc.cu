// rbf_tc.cu -- the BF16 tensor-core form of the Gauss-RBF kernel sketch
// (SketchySVD over the kernel matrix K(i, j) = exp(-gamma ||x_i - x_j||^2),
// the window of src/Skema_Window.hpp:90-107 and the kernel of
// src/Skema_Kernel.cpp:6-81, diagonal forced to 1 as at :62-68). K is never
// stored: the kernel rows of a call are sketched by two passes of
// rbf_sketch_kernel (tc_rbf.cuh) that regenerate its tiles from the points:
//   row pass     [Y | T] = K(rows, :) [Omega~; Psi~]^T   query = the rows
//   column pass  X^T = nu^G X^T + eta sum_w nu^(G-1-w) K_w^T Upsilon~_w^T
//                                                        query = all points
// then Z^T = nu^G Z^T + eta T^T Phi~^T on the dense tensor-core GEMM, with
// window w's T rows weighted by nu^(G-1-w) (one group of G windows per
// call when nu > 0, see rbf_tc_update).
// Distances come from the Gram expansion ||x_i||^2 + ||x_j||^2 - 2 x_i.x_j
// of the BF16-rounded points (FP32 accumulation), clamped at 0; the point
// norms are those of the same rounded points, so a point's distance to
// itself is 0 up to accumulation order and the diagonal is set exactly.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "tc_host.h"
#include "tc_rbf.cuh"

namespace skema {

namespace {

constexpr float kLog2e = 1.4426950408889634f;

// Points (N x d FP32, strided) -> X16 (N x dp BF16 row-major, zero padded)
// and c_p = -gamma log2(e) ||bf16(x_p)||^2; c is -inf for p in [N, npad).
__global__ void rbf_prep_kernel(const float* __restrict__ P, int64_t prs, int64_t pcs, int64_t N, int64_t d,
                                int64_t dp, float gl, __nv_bfloat16* __restrict__ X16, float* __restrict__ cval,
                                int64_t npad) {
  const int lane = threadIdx.x & 31;
  const int64_t w0 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t p = w0; p < npad; p += nw) {
    if (p >= N) {
      if (lane == 0) cval[p] = -INFINITY;
      continue;
    }
    float sum = 0.f;
    for (int64_t f = lane; f < dp; f += 32) {
      const float v = f < d ? P[p * prs + f * pcs] : 0.f;
      const __nv_bfloat16 b = __float2bfloat16(v);
      X16[p * dp + f] = b;
      const float fb = __bfloat162float(b);
      sum = fmaf(fb, fb, sum);
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if (lane == 0) cval[p] = -gl * sum;
  }
}

// Key constants of the column pass: c of rows [R0, R0 + nr) plus the
// log2 window weight (G - 1 - i / W) * log2w of row i (windows of W rows, G
// of them), -inf from nr up to npad.
__global__ void rbf_key_c_kernel(const float* __restrict__ cval, int64_t R0, int64_t nr, int64_t W, int64_t G,
                                 float log2w, float* __restrict__ out, int64_t npad) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < npad; i += (int64_t)gridDim.x * blockDim.x) {
    float v = -INFINITY;
    if (i < nr) {
      v = cval[R0 + i];
      const int64_t e = G - 1 - i / W;
      if (log2w != 0.f && e > 0) v += (float)e * log2w;
    }
    out[i] = v;
  }
}

template <int NC1, int NC2, int DK, int S>
void launch_rbf(skema_ctx* c, const CUtensorMap& tq, const CUtensorMap& tk, const CUtensorMap& tv1,
                const CUtensorMap& tv2, const tc::RbfArgs& a, const tc::OutSpec& o) {
  constexpr uint32_t Q_BYTES = DK * tc::RBF_BQ * 128;
  constexpr uint32_t STAGE = ((DK * tc::RBF_BJ * 128 + (NC1 + NC2) * 128 + 256 + 1023) / 1024) * 1024;
  const size_t smem = Q_BYTES + (size_t)S * STAGE + 2 * tc::RBF_BQ * 128 + 1024 + 256;
  auto kern = tc::rbf_sketch_kernel<NC1, NC2, DK, S>;
  SKEMA_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int64_t units = (int64_t)a.qtiles * a.nchunks * a.ksplit;
  if (units <= 0 || a.nblocks <= 0) return;
  if (units > 0x7fffffff) fail(SKEMA_EINVAL, "kernel-sketch grid too large");
  const int grid = (int)std::min<int64_t>(units, c->sm_count);
  kern<<<grid, tc::kThreads, smem, c->stream>>>(tq, tk, tv1, tv2, a, o, c->dev_err);
  SKEMA_LAUNCHED(c);
  c->dev_err_armed = true;
}

// Output-column chunks of one pass: (NC1, NC2) = (256, 144) with two key /
// value stages, or (256, 16) with three.
template <int DK>
void run_pass(skema_ctx* c, bool narrow, const CUtensorMap& tq, const CUtensorMap& tk, const void* V, int64_t vcols,
              int64_t vrows, int64_t vld, const tc::RbfArgs& a, const tc::OutSpec& o) {
  const CUtensorMap tv1 = tmap_bf16(V, (uint64_t)vcols, (uint64_t)vrows, (uint64_t)vld * 2, 64, 256);
  if (narrow) {
    const CUtensorMap tv2 = tmap_bf16(V, (uint64_t)vcols, (uint64_t)vrows, (uint64_t)vld * 2, 64, 16);
    launch_rbf<256, 16, DK, 3>(c, tq, tk, tv1, tv2, a, o);
  } else {
    const CUtensorMap tv2 = tmap_bf16(V, (uint64_t)vcols, (uint64_t)vrows, (uint64_t)vld * 2, 64, 144);
    launch_rbf<256, 144, DK, 2>(c, tq, tk, tv1, tv2, a, o);
  }
}

}  // namespace

bool rbf_tc_supported(const skema_ctx* c, int64_t d) {
  return tc_available(c) && d >= 1 && d <= 128 && c->k <= 448 && c->n == c->m;
}

// All windows of the call in one row pass, one column pass and one Z
// product when nu > 0: the per-window sequence X = nu X + eta x_w (likewise
// Z) over G windows equals X = nu^G X + eta sum_w nu^(G-1-w) x_w, so window
// w's kernel rows carry the weight nu^(G-1-w) -- in the key constants of the
// column pass and in the T rows that feed Z -- while its Y rows get eta
// alone. Other nu take one window at a time (G = 1).
void rbf_tc_update(skema_ctx* c, Mat P, int64_t N, int64_t d, int64_t row0, int64_t nrows) {
  const float eta = (float)c->p.sketch_eta, nu = (float)c->p.sketch_nu;
  const float gl = (float)c->p.kernel_gamma * kLog2e;
  const int64_t k = c->k, s = c->s, m = c->m, W = c->w;
  const int DK = d <= 64 ? 1 : 2;
  const int64_t dp = 64 * DK;
  const int64_t npad = (N + tc::RBF_BJ - 1) / tc::RBF_BJ * tc::RBF_BJ;
  const int64_t nwin = (nrows + W - 1) / W;
  const bool fold = nu > 0.f;
  const float log2nu = (fold && nu != 1.f) ? std::log2(nu) : 0.f;
  const int64_t gwin = fold ? nwin : 1;            // windows per group
  const int64_t gmax = std::min(nrows, gwin * W);  // rows per group
  const int64_t gp = pad8(gmax);
  const int64_t gpad = (gmax + tc::RBF_BJ - 1) / tc::RBF_BJ * tc::RBF_BJ;
  auto rup = [](size_t b) { return (b + 255) / 256 * 256; };
  const size_t b_x16 = rup(sizeof(__nv_bfloat16) * (size_t)(N * dp));
  const size_t b_c = rup(sizeof(float) * (size_t)npad);
  const size_t b_ck = rup(sizeof(float) * (size_t)gpad);
  const size_t b_t16 = 2 * rup(sizeof(__nv_bfloat16) * (size_t)(gp * s));  // T16 and its remainder
  const size_t b_t32 = rup(sizeof(float) * (size_t)(gp * s));
  char* ws = static_cast<char*>(workspace(c, b_x16 + b_c + b_ck + b_t16 + b_t32 + tc_slice_bytes(c, gmax)));
  __nv_bfloat16* X16 = reinterpret_cast<__nv_bfloat16*>(ws);
  float* cval = reinterpret_cast<float*>(ws + b_x16);
  float* ckey = reinterpret_cast<float*>(ws + b_x16 + b_c);
  __nv_bfloat16* T16 = reinterpret_cast<__nv_bfloat16*>(ws + b_x16 + b_c + b_ck);
  __nv_bfloat16* T16lo = reinterpret_cast<__nv_bfloat16*>(ws + b_x16 + b_c + b_ck + b_t16 / 2);
  float* T32 = reinterpret_cast<float*>(ws + b_x16 + b_c + b_ck + b_t16);
  char* slice_sp = ws + b_x16 + b_c + b_ck + b_t16 + b_t32;

  {
    StageScope st(c, ST_WINDOW);
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((npad * 32 + 255) / 256, c->sm_count * 16));
    rbf_prep_kernel<<<grid, 256, 0, c->stream>>>(P.p, P.rs, P.cs, N, d, dp, gl, X16, cval, npad);
    SKEMA_LAUNCHED(c);
  }
  const CUtensorMap tq = tmap_bf16(X16, (uint64_t)dp, (uint64_t)N, (uint64_t)dp * 2, 64, tc::RBF_BQ);
  const CUtensorMap tk = tmap_bf16(X16, (uint64_t)dp, (uint64_t)N, (uint64_t)dp * 2, 64, tc::RBF_BJ);

  for (int64_t g0 = 0; g0 < nwin; g0 += gwin) {
    const int64_t R0 = row0 + g0 * W;
    const int64_t nr = std::min(gwin * W, nrows - g0 * W);  // rows of this group
    const int64_t G = (nr + W - 1) / W;                      // windows of this group
    const int64_t ldT = pad8(nr);
    const float nuG = fold ? std::pow(nu, (float)G) : nu;    // G = 1 when not folded
    const float ybeta = y_beta(c, R0, R0 + nr, nu);  // rows written before get the nu term
    char* sp = slice_sp;
    const TcSlices sl = tc_window_slices(c, R0, nr, &sp);
    {  // row pass: [Y | T] = K(rows, :) [Omega~; Psi~]^T, T rows weighted per window
      StageScope st(c, ST_FUSED);
      tc::RbfArgs a;
      a.nq = nr, a.qbase = R0, a.kbase = 0;
      a.nblocks = npad / tc::RBF_BJ;
      a.qtiles = (int)((nr + tc::RBF_BQ - 1) / tc::RBF_BQ);
      a.chunk_cols = 272;
      a.nchunks = (int)((k + s + 271) / 272);
      const Plan pl = plan_split(c, (int64_t)a.qtiles * a.nchunks, npad, 16);
      a.bchunk = pl.kchunk / tc::RBF_BJ;
      a.ksplit = (int)((a.nblocks + a.bchunk - 1) / a.bchunk);
      a.cq = cval + R0, a.ckey = cval, a.two_g = 2.f * gl;
      a.klog2w = 0.f, a.kwlen = W, a.knwin = 1;
      tc::OutSpec o = out_spec();
      o.p0 = c->Y + R0, o.rs0 = 1, o.cs0 = m, o.alpha0 = eta, o.beta0 = ybeta;
      o.rows = nr, o.split = k, o.ncols = k + s;
      o.row_log2w = log2nu, o.row_wlen = W, o.row_nwin = G;
      if (a.ksplit == 1) {
        o.p1 = T16, o.p1lo = T16lo, o.rs1 = 1, o.cs1 = ldT;
      } else {
        scale_block(c, MatOut{c->Y + R0, 1, m}, nr, k, ybeta);
        SKEMA_CUDA(cudaMemsetAsync(T32, 0, sizeof(float) * (size_t)(ldT * s), c->stream));
        o.atomic0 = 1, o.beta0 = 0.f;
        o.p1f = T32, o.rs1 = 1, o.cs1 = ldT, o.atomic1 = 1;
      }
      if (DK == 1)
        run_pass<1>(c, true, tq, tk, c->op16, N, k + s, c->ld_op16, a, o);
      else
        run_pass<2>(c, true, tq, tk, c->op16, N, k + s, c->ld_op16, a, o);
      if (a.ksplit > 1) t32_to_t16(c, T32, ldT, T16, T16lo, ldT, nr, s);
    }
    y_rows_mark(c, R0, R0 + nr);
    {  // column pass: X^T = nu^G X^T + eta sum_w nu^(G-1-w) K_w^T Upsilon~_w^T
      StageScope st(c, ST_UPSILON);
      const int64_t kpad = (nr + tc::RBF_BJ - 1) / tc::RBF_BJ * tc::RBF_BJ;
      rbf_key_c_kernel<<<(int)std::max<int64_t>(1, std::min<int64_t>((kpad + 255) / 256, c->sm_count * 8)), 256, 0,
                         c->stream>>>(cval, R0, nr, W, G, log2nu, ckey, kpad);
      SKEMA_LAUNCHED(c);
      const bool narrow = k <= 272;
      tc::RbfArgs a;
      a.nq = N, a.qbase = 0, a.kbase = R0;
      a.nblocks = kpad / tc::RBF_BJ;
      a.qtiles = (int)((N + tc::RBF_BQ - 1) / tc::RBF_BQ);
      a.chunk_cols = narrow ? 272 : 400;
      a.nchunks = (int)((k + a.chunk_cols - 1) / a.chunk_cols);
      const Plan pl = plan_split(c, (int64_t)a.qtiles * a.nchunks, kpad, 8);
      a.bchunk = pl.kchunk / tc::RBF_BJ;
      a.ksplit = (int)((a.nblocks + a.bchunk - 1) / a.bchunk);
      a.cq = cval, a.ckey = ckey, a.two_g = 2.f * gl;
      a.klog2w = log2nu, a.kwlen = W, a.knwin = G;
      tc::OutSpec o = out_spec();
      o.p0 = c->X, o.rs0 = 1, o.cs0 = c->n, o.alpha0 = eta, o.beta0 = nuG;
      o.rows = N, o.split = k, o.ncols = k;
      if (a.ksplit > 1) {
        scale_block(c, MatOut{c->X, c->n, 1}, k, c->n, nuG);
        o.atomic0 = 1, o.beta0 = 0.f;
      }
      if (DK == 1)
        run_pass<1>(c, narrow, tq, tk, sl.U16, nr, k, sl.ldm, a, o);
      else
        run_pass<2>(c, narrow, tq, tk, sl.U16, nr, k, sl.ldm, a, o);
    }
    // T in two BF16 parts (about 16 significant bits); the second Z product
    // is small next to the passes and lowers the singular-value error of
    // the kernel form by about a fifth
    tc_z_update(c, T16, ldT, sl, nr, nuG);
    tc_z_update(c, T16lo, ldT, sl, nr, 1.f);
  }
}

// ---------------------------------------------------------------------------
// The standalone forward / adjoint pair (skema_rbf_sketch_fwd / _vjp) in the
// BF16 form: Y = K Omega^T by rbf_sketch_kernel (queries and keys all
// points, V = Omega), the adjoint by two passes of rbf_vjp_kernel.
namespace {

// E X + E^T X and the row / column sums of E -> dL/dx (FP32 points, d
// columns, S with leading dimension d).
__global__ void rbf_pair_dx_kernel(const float* __restrict__ P, int64_t N, int64_t d, float gamma,
                                   const float* __restrict__ rsum, const float* __restrict__ csum,
                                   const float* __restrict__ S, float* __restrict__ dX) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < N * d; q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = q / d;
    dX[q] = -2.f * gamma * ((rsum[i] + csum[i]) * P[q] - S[q]);
  }
}

struct PairPrep {
  __nv_bfloat16* X16;
  float* cval;
  int64_t npad;
};

// Points -> BF16 rows (d padded to 64) and their constants; scratch from *sp.
PairPrep pair_prep(skema_ctx* c, const float* pts, int64_t N, int64_t d, float gl, char** sp) {
  auto take = [&](size_t b) {
    char* p = *sp;
    *sp += (b + 255) / 256 * 256;
    return p;
  };
  PairPrep pp;
  pp.npad = (N + tc::RBF_BJ - 1) / tc::RBF_BJ * tc::RBF_BJ;
  pp.X16 = reinterpret_cast<__nv_bfloat16*>(take(sizeof(__nv_bfloat16) * (size_t)(N * 64)));
  pp.cval = reinterpret_cast<float*>(take(sizeof(float) * (size_t)pp.npad));
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((pp.npad * 32 + 255) / 256, c->sm_count * 16));
  rbf_prep_kernel<<<grid, 256, 0, c->stream>>>(pts, d, 1, N, d, 64, gl, pp.X16, pp.cval, pp.npad);
  SKEMA_LAUNCHED(c);
  return pp;
}

size_t pair_prep_bytes(int64_t N) {
  const int64_t npad = (N + 63) / 64 * 64;
  return sizeof(__nv_bfloat16) * (size_t)(N * 64) + sizeof(float) * (size_t)npad + 512;
}

template <int KK>
void launch_vjp(skema_ctx* c, const CUtensorMap& tqx, const CUtensorMap& tkx, const CUtensorMap& tqa,
                const CUtensorMap& tkb, const CUtensorMap& txt, const tc::RbfVjpArgs& a) {
  constexpr uint32_t STAGE = ((64 * 128 + KK * 64 * 128 + 64 * 128 + 256 + 1023) / 1024) * 1024;
  const size_t smem = 128 * 128 + KK * 128 * 128 + 3 * (size_t)STAGE + 1024 + 256;
  auto kern = tc::rbf_vjp_kernel<1, KK>;
  SKEMA_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int64_t units = (int64_t)a.qtiles * a.ksplit;
  const int grid = (int)std::min<int64_t>(units, c->sm_count);
  kern<<<grid, tc::kThreads, smem, c->stream>>>(tqx, tkx, tqa, tkb, txt, a, c->dev_err);
  SKEMA_LAUNCHED(c);
  c->dev_err_armed = true;
}

}  // namespace

bool rbf_pair_tc_supported(const skema_ctx* c, int64_t d, int64_t k, double gamma) {
  return c->p.precision == SKEMA_PREC_BF16 && tc_available(c) && d >= 1 && d <= 64 && k >= 1 && k <= 192 &&
         gamma > 0.0;
}

void rbf_fwd_tc(skema_ctx* c, const float* pts, int64_t N, int64_t d, double gamma, const float* omega, int64_t k,
                float* Y) {
  const float gl = (float)gamma * kLog2e;
  const int64_t ldN = pad8(N);
  char* ws = static_cast<char*>(workspace(c, pair_prep_bytes(N) + sizeof(__nv_bfloat16) * (size_t)(k * ldN) + 256));
  char* sp = ws;
  const PairPrep pp = pair_prep(c, pts, N, d, gl, &sp);
  __nv_bfloat16* Om16 = reinterpret_cast<__nv_bfloat16*>(sp);  // k x N row-major, ld pad8(N)
  to_bf16(c, Mat{omega, N, 1}, k, N, Om16, ldN, 1);
  const CUtensorMap tq = tmap_bf16(pp.X16, 64, (uint64_t)N, 128, 64, tc::RBF_BQ);
  const CUtensorMap tk = tmap_bf16(pp.X16, 64, (uint64_t)N, 128, 64, tc::RBF_BJ);
  tc::RbfArgs a;
  a.nq = N, a.qbase = 0, a.kbase = 0;
  a.nblocks = pp.npad / tc::RBF_BJ;
  a.qtiles = (int)((N + tc::RBF_BQ - 1) / tc::RBF_BQ);
  const bool small = k <= 144;
  a.chunk_cols = small ? 144 : k <= 272 ? 272 : 400;
  a.nchunks = (int)((k + a.chunk_cols - 1) / a.chunk_cols);
  const Plan pl = plan_split(c, (int64_t)a.qtiles * a.nchunks, pp.npad, 16);
  a.bchunk = pl.kchunk / tc::RBF_BJ;
  a.ksplit = (int)((a.nblocks + a.bchunk - 1) / a.bchunk);
  a.cq = pp.cval, a.ckey = pp.cval, a.two_g = 2.f * gl;
  a.klog2w = 0.f, a.kwlen = 1, a.knwin = 1;
  tc::OutSpec o = out_spec();
  o.p0 = Y, o.rs0 = k, o.cs0 = 1, o.alpha0 = 1.f, o.beta0 = 0.f;
  o.rows = N, o.split = k, o.ncols = k;
  if (a.ksplit > 1) {
    SKEMA_CUDA(cudaMemsetAsync(Y, 0, sizeof(float) * (size_t)(N * k), c->stream));
    o.atomic0 = 1;
  }
  const CUtensorMap tv1 = tmap_bf16(Om16, (uint64_t)N, (uint64_t)k, (uint64_t)ldN * 2, 64, small ? 128 : 256);
  if (small) {
    const CUtensorMap tv2 = tmap_bf16(Om16, (uint64_t)N, (uint64_t)k, (uint64_t)ldN * 2, 64, 16);
    launch_rbf<128, 16, 1, 3>(c, tq, tk, tv1, tv2, a, o);
  } else {
    run_pass<1>(c, k <= 272, tq, tk, Om16, N, k, ldN, a, o);
  }
}

void rbf_vjp_tc(skema_ctx* c, const float* pts, int64_t N, int64_t d, double gamma, const float* omega, int64_t k,
                const float* Ybar, float* dpts, double* dgamma) {
  const float gl = (float)gamma * kLog2e;
  const int KK = (int)((k + 63) / 64);
  const int64_t kp = 64 * KK, ldN = pad8(N);
  auto rup = [](size_t b) { return (b + 255) / 256 * 256; };
  const size_t b_xt = rup(sizeof(__nv_bfloat16) * (size_t)(64 * ldN));
  const size_t b_a = rup(sizeof(__nv_bfloat16) * (size_t)(N * kp));
  const size_t b_s = rup(sizeof(float) * (size_t)(N * d));
  const size_t b_v = rup(sizeof(float) * (size_t)N);
  char* ws = static_cast<char*>(workspace(c, pair_prep_bytes(N) + b_xt + 2 * b_a + b_s + 2 * b_v));
  char* sp = ws;
  const PairPrep pp = pair_prep(c, pts, N, d, gl, &sp);
  __nv_bfloat16* XT16 = reinterpret_cast<__nv_bfloat16*>(sp);  // 64 x N: features as rows
  __nv_bfloat16* Yb16 = reinterpret_cast<__nv_bfloat16*>(sp + b_xt);        // N x kp
  __nv_bfloat16* OmT16 = reinterpret_cast<__nv_bfloat16*>(sp + b_xt + b_a);  // N x kp
  float* S = reinterpret_cast<float*>(sp + b_xt + 2 * b_a);
  float* rs = reinterpret_cast<float*>(sp + b_xt + 2 * b_a + b_s);
  float* cs = reinterpret_cast<float*>(sp + b_xt + 2 * b_a + b_s + b_v);
  // zero padding (features >= d, columns >= k) and the accumulators
  SKEMA_CUDA(cudaMemsetAsync(XT16, 0, b_xt + 2 * b_a + b_s + 2 * b_v, c->stream));
  SKEMA_CUDA(cudaMemsetAsync(dgamma, 0, sizeof(double), c->stream));
  to_bf16(c, Mat{pts, d, 1}, N, d, XT16, 1, ldN);
  to_bf16(c, Mat{Ybar, k, 1}, N, k, Yb16, kp, 1);
  to_bf16(c, Mat{omega, 1, N}, N, k, OmT16, kp, 1);
  const CUtensorMap tqx = tmap_bf16(pp.X16, 64, (uint64_t)N, 128, 64, tc::RBF_BQ);
  const CUtensorMap tkx = tmap_bf16(pp.X16, 64, (uint64_t)N, 128, 64, tc::RBF_BJ);
  const CUtensorMap txt = tmap_bf16(XT16, (uint64_t)N, 64, (uint64_t)ldN * 2, 64, 64);
  const CUtensorMap tyq = tmap_bf16(Yb16, (uint64_t)kp, (uint64_t)N, (uint64_t)kp * 2, 64, tc::RBF_BQ);
  const CUtensorMap tyk = tmap_bf16(Yb16, (uint64_t)kp, (uint64_t)N, (uint64_t)kp * 2, 64, tc::RBF_BJ);
  const CUtensorMap toq = tmap_bf16(OmT16, (uint64_t)kp, (uint64_t)N, (uint64_t)kp * 2, 64, tc::RBF_BQ);
  const CUtensorMap tok = tmap_bf16(OmT16, (uint64_t)kp, (uint64_t)N, (uint64_t)kp * 2, 64, tc::RBF_BJ);
  tc::RbfVjpArgs a;
  a.N = N;
  a.nblocks = pp.npad / tc::RBF_BJ;
  a.qtiles = (int)((N + tc::RBF_BQ - 1) / tc::RBF_BQ);
  const Plan pl = plan_split(c, a.qtiles, pp.npad, 8);
  a.bchunk = pl.kchunk / tc::RBF_BJ;
  a.ksplit = (int)((a.nblocks + a.bchunk - 1) / a.bchunk);
  a.cval = pp.cval, a.two_g = 2.f * gl, a.inv_g = 1.f / gl;
  a.S = S, a.d = d;
  for (int pass = 0; pass < 2; ++pass) {
    a.rsum = pass == 0 ? rs : cs;
    a.dgamma = pass == 0 ? dgamma : nullptr;
    const CUtensorMap& tqa = pass == 0 ? tyq : toq;
    const CUtensorMap& tkb = pass == 0 ? tok : tyk;
    if (KK == 1)
      launch_vjp<1>(c, tqx, tkx, tqa, tkb, txt, a);
    else if (KK == 2)
      launch_vjp<2>(c, tqx, tkx, tqa, tkb, txt, a);
    else
      launch_vjp<3>(c, tqx, tkx, tqa, tkb, txt, a);
  }
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((N * d + 255) / 256, c->sm_count * 16));
  rbf_pair_dx_kernel<<<grid, 256, 0, c->stream>>>(pts, N, d, (float)gamma, rs, cs, S, dpts);
  SKEMA_LAUNCHED(c);
}

}  // namespace skema
