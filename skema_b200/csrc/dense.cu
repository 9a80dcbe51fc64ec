// dense.cu -- SketchySVD::linear_update over a dense input
// (src/Skema_SketchySVD.cpp:120-246) with update(dense, Gauss)
// (src/Skema_SketchySVD.cpp:256-268), FP32 form, and the dispatch to the
// SparseSign, SketchySPD and tensor-core forms.
//
// Per window A_w (rows [R0, R0+wr)):
//   Y(R0:R0+wr, :) = nu*Y + eta * A_w Omega~^T          (k columns)
//   T              =            A_w Psi~^T              (s columns, scratch)
//   X              = nu*X + eta * Upsilon~(:, w) A_w
//   Z              = nu*Z + eta * Phi~(:, w) T
// Z uses the association Phi~_w (A_w Psi~^T): 2*wr*n*s + 2*s*s*wr flops per
// window instead of the reference's (Phi~_w A_w) Psi~^T with
// 2*s*wr*n + 2*s*s*n; both equal Phi~_w A_w Psi~^T.
#include <cuda_runtime.h>

#include <algorithm>

#include "internal.h"

namespace skema {

static int splitk_for(const skema_ctx* c, int64_t M, int64_t N, int64_t K) {
  const int64_t tiles = ((M + 127) / 128) * ((N + 127) / 128);
  int64_t sk = (2 * c->sm_count + tiles - 1) / tiles;
  sk = std::min<int64_t>(sk, std::max<int64_t>(1, K / 256));
  return (int)std::max<int64_t>(1, sk);
}

// Room for the K-split partial products of the window's three large
// products (at most about 13 M values on the 200k x 20k case), after T.
constexpr int64_t kSplitPartFloats = (int64_t)16 << 20;
static int64_t t_floats(const skema_ctx* c, int64_t wr) { return (wr * c->s + 63) / 64 * 64; }

// The Gauss three-sketch body for one window. T is wr x s scratch, followed
// by kSplitPartFloats for sgemm_split.
static void gauss_window(skema_ctx* c, Mat Aw, int64_t R0, int64_t wr, float* T) {
  float* part = T + t_floats(c, wr);
  const float eta = (float)c->p.sketch_eta, nu = (float)c->p.sketch_nu;
  const Map& U = c->ups;
  const Map& O = c->omg;
  const Map& F = c->phi;
  const Map& P = c->psi;
  const float ybeta = y_beta(c, R0, R0 + wr, nu);
  {  // Y rows: B(kk=j, col=r) = Omega~(r, j)
    StageScope st(c, ST_OMEGA);
    sgemm_split(c, wr, c->k, c->n, eta, Aw, Mat{O.f32, O.cs, O.rs}, ybeta, MatOut{c->Y + R0, 1, c->m}, part,
                kSplitPartFloats);
  }
  y_rows_mark(c, R0, R0 + wr);
  {  // T = A_w Psi~^T
    StageScope st(c, ST_PSI);
    sgemm_split(c, wr, c->s, c->n, 1.f, Aw, Mat{P.f32, P.cs, P.rs}, 0.f, MatOut{T, c->s, 1}, part,
                kSplitPartFloats);
  }
  {  // X = nu X + eta Upsilon~(:, R0:R0+wr) A_w
    StageScope st(c, ST_UPSILON);
    sgemm_split(c, c->k, c->n, wr, eta, Mat{U.f32 + R0 * U.cs, U.rs, U.cs}, Aw, nu, MatOut{c->X, c->n, 1}, part,
                kSplitPartFloats);
  }
  {  // Z = nu Z + eta Phi~(:, R0:R0+wr) T
    StageScope st(c, ST_PHI);
    scale_block(c, MatOut{c->Z, c->s, 1}, c->s, c->s, nu);
    sgemm(c, c->s, c->s, wr, eta, Mat{F.f32 + R0 * F.cs, F.rs, F.cs}, Mat{T, c->s, 1}, 1.f,
          MatOut{c->Z, c->s, 1}, splitk_for(c, c->s, c->s, wr));
  }
}

// SketchySPD, Gauss: Y(w,:) = nu*Y + eta * A_w Omega (Omega stored n x k).
static void spd_gauss_window(skema_ctx* c, Mat Aw, int64_t R0, int64_t wr) {
  const float eta = (float)c->p.sketch_eta, nu = (float)c->p.sketch_nu;
  const Map& O = c->omg;
  const float ybeta = y_beta(c, R0, R0 + wr, nu);
  sgemm(c, wr, c->k, c->n, eta, Aw, Mat{O.f32, O.cs, O.rs}, ybeta, MatOut{c->Y + R0, 1, c->m});
  y_rows_mark(c, R0, R0 + wr);
}

void spd_ssign_window(skema_ctx* c, Mat Aw, int64_t R0, int64_t wr);

void dense_window(skema_ctx* c, Mat Aw, int64_t R0, int64_t wr, float* T) {
  if (c->spd) {
    if (c->p.dim_redux == SKEMA_MAP_GAUSS)
      spd_gauss_window(c, Aw, R0, wr);
    else
      spd_ssign_window(c, Aw, R0, wr);
    return;
  }
  if (c->p.dim_redux == SKEMA_MAP_SPARSE_SIGN) {
    dense_ssign_window(c, Aw, R0, wr);
    return;
  }
  if (c->p.precision != SKEMA_PREC_FP32) {
    if (!tc_available(c)) fail(SKEMA_EUNSUPPORTED, "this precision is not available for this sketch");
    tc_dense_window(c, Aw, R0, wr, T);
    return;
  }
  gauss_window(c, Aw, R0, wr, T);
}

size_t dense_scratch_bytes(const skema_ctx* c, int64_t wr) {
  if (c->spd || c->p.dim_redux == SKEMA_MAP_SPARSE_SIGN) return 256;
  if (tc_available(c)) return tc_scratch_bytes(c, wr);
  return sizeof(float) * (size_t)(t_floats(c, wr) + kSplitPartFloats) + 256;
}

void dense_update(skema_ctx* c, Mat A, int64_t row0, int64_t nrows) {
  if (c->residual_pass) {
    residual_dense(c, A, row0, nrows);
    return;
  }
  if (!c->spd && c->p.dim_redux == SKEMA_MAP_GAUSS && c->p.precision != SKEMA_PREC_FP32) {
    if (!tc_available(c)) fail(SKEMA_EUNSUPPORTED, "this precision is not available for this sketch");
    tc_dense_update(c, A, row0, nrows);
    return;
  }
  const int64_t W = c->w;
  float* T = (float*)workspace(c, dense_scratch_bytes(c, std::min(W, nrows)));
  for (int64_t r = 0; r < nrows; r += W) {
    const int64_t wr = std::min(W, nrows - r);
    Mat Aw{A.p + r * A.rs, A.rs, A.cs};
    dense_window(c, Aw, row0 + r, wr, T);
  }
}

}  // namespace skema
