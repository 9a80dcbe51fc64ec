// residuals.cu -- residual norms of the fixed-rank approximation
// (Skema::residuals with map_A_by_window, src/Skema_Residuals.hpp:58-110,
// 160-217, as called by SketchySVD::compute_residuals,
// src/Skema_SketchySVD.cpp:719-727). For U (m x r), S (r), V (n x r):
//   rnorm_j = || [ (A^T U - V S)(:, j) ; (A V - U S)(:, j) ] ||_2 .
// A is streamed again in row blocks, as for the sketch update. A block's
// rows of A V are complete within the block, so each block adds its share
// of the column sums of squares of A V - U S and drops the rows; A^T U is a
// sum over blocks and is accumulated, and its difference with V S is formed
// at the end. The SketchySPD form (src/Skema_Residuals.hpp:112-158) has no
// A^T U part and uses V in place of U. FP64 throughout (the FP32 input
// values are exact in FP64).
#include <cuda_runtime.h>

#include <algorithm>

#include "internal.h"

namespace skema {

void rbf_window_block(skema_ctx* c, Mat P, int64_t N, int64_t d, float gamma, int64_t R0, int64_t wr, float* out,
                      int64_t ldo);

namespace {

int grid_of(const skema_ctx* c, int64_t work, int per_sm) {
  return (int)std::max<int64_t>(1, std::min<int64_t>(work, (int64_t)c->sm_count * per_sm));
}

// Column-major (ld) -> row-major rows x r.
__global__ void cm_to_rm_kernel(const double* __restrict__ S, int64_t ld, int64_t rows, int64_t r,
                                double* __restrict__ D) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < rows * r;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = q / r, j = q - i * r;
    D[q] = S[i + j * ld];
  }
}

// sq[j] += sum_i (M[i*r + j] - B[i*r + j] * S[j])^2 over rows i < rows.
// Threads: 32 lanes over columns (chunks of 32), 8 rows per block step.
__global__ void __launch_bounds__(256)
    colsumsq_diff_kernel(const double* __restrict__ M, const double* __restrict__ B, const double* __restrict__ S,
                         int64_t rows, int64_t r, double* __restrict__ sq) {
  const int lane = threadIdx.x & 31, ty = threadIdx.x >> 5;
  for (int64_t c0 = 0; c0 < r; c0 += 32) {
    const int64_t j = c0 + lane;
    if (j >= r) continue;
    const double s = S[j];
    double acc = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * 8 + ty; i < rows; i += (int64_t)gridDim.x * 8) {
      const double d = M[i * r + j] - B[i * r + j] * s;
      acc = fma(d, d, acc);
    }
    atomicAdd(sq + j, acc);
  }
}

// CSR rows [0, nrows) (absolute offsets rowptr - col_offset into col/val),
// global rows R0 + i: a warp per row and 32 columns of r per pass. Each
// nonzero (i, j, a) adds a V(j, :) to the row's A V and a U(i, :) to
// A^T U(j, :) (FP64 atomics); the row's (A V - U S)^2 goes to sq.
__global__ void __launch_bounds__(256)
    csr_residual_kernel(const int64_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                        const float* __restrict__ val, int64_t col_offset, int64_t nrows, int64_t R0, int64_t ncol,
                        const double* __restrict__ U, const double* __restrict__ V, const double* __restrict__ S,
                        int64_t r, double* __restrict__ AtU, double* __restrict__ sq) {
  const int lane = threadIdx.x & 31;
  const int64_t w0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t c0 = 0; c0 < r; c0 += 32) {
    const int64_t j = c0 + lane;
    const bool lj = j < r;
    const double s = lj ? S[j] : 0.0;
    double acc = 0.0;
    for (int64_t i = w0; i < nrows; i += nw) {
      const double u = lj ? U[(R0 + i) * r + j] : 0.0;
      double av = 0.0;
      const int64_t b = rowptr[i] - col_offset, e = rowptr[i + 1] - col_offset;
      for (int64_t p = b; p < e; ++p) {
        const int32_t cj = col[p];
        if ((uint64_t)cj >= (uint64_t)ncol) continue;
        const double a = (double)val[p];
        if (lj) {
          av = fma(a, V[(int64_t)cj * r + j], av);
          if (AtU) atomicAdd(AtU + (int64_t)cj * r + j, a * u);
        }
      }
      const double d = av - u * s;
      acc = fma(d, d, acc);
    }
    if (lj) atomicAdd(sq + j, acc);
  }
}

__global__ void sqrt_kernel(const double* __restrict__ a, double* __restrict__ out, int64_t r) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < r; j += (int64_t)gridDim.x * blockDim.x)
    out[j] = sqrt(a[j]);
}

void need_ready(const skema_ctx* c) {
  if (!c->res_ready) fail(SKEMA_ESTATE, "no residual pass open: call skema_residuals_begin first");
}

}  // namespace

void residual_free(skema_ctx* c) {
  for (double** p : {&c->res_U, &c->res_V, &c->res_S, &c->res_AtU, &c->res_sq}) {
    if (*p) cudaFree(*p);
    *p = nullptr;
  }
  c->res_ready = false;
}

// Allocates the residual buffers once and loads U, S, V into them.
static void residual_load(skema_ctx* c, const double* U, const double* S, const double* V) {
  const int64_t m = c->m, n = c->n, r = c->p.rank;
  if (!c->res_V) {
    SKEMA_CUDA(cudaMalloc(&c->res_V, sizeof(double) * (size_t)(n * r)));
    SKEMA_CUDA(cudaMalloc(&c->res_S, sizeof(double) * (size_t)r));
    SKEMA_CUDA(cudaMalloc(&c->res_sq, sizeof(double) * (size_t)r));
    if (!c->spd) {
      SKEMA_CUDA(cudaMalloc(&c->res_U, sizeof(double) * (size_t)(m * r)));
      SKEMA_CUDA(cudaMalloc(&c->res_AtU, sizeof(double) * (size_t)(n * r)));
    }
  }
  cm_to_rm_kernel<<<grid_of(c, (n * r + 255) / 256, 16), 256, 0, c->stream>>>(V, n, n, r, c->res_V);
  SKEMA_LAUNCHED(c);
  if (!c->spd) {
    cm_to_rm_kernel<<<grid_of(c, (m * r + 255) / 256, 16), 256, 0, c->stream>>>(U, m, m, r, c->res_U);
    SKEMA_LAUNCHED(c);
  }
  SKEMA_CUDA(cudaMemcpyAsync(c->res_S, S, sizeof(double) * (size_t)r, cudaMemcpyDeviceToDevice, c->stream));
}

// Zeroes the pass's sums over the loaded factors and opens it.
static void residual_open(skema_ctx* c) {
  const int64_t n = c->n, r = c->p.rank;
  if (!c->spd) SKEMA_CUDA(cudaMemsetAsync(c->res_AtU, 0, sizeof(double) * (size_t)(n * r), c->stream));
  SKEMA_CUDA(cudaMemsetAsync(c->res_sq, 0, sizeof(double) * (size_t)r, c->stream));
  c->res_ready = true;
}

void residual_begin(skema_ctx* c, const double* U, const double* S, const double* V) {
  residual_load(c, U, S, V);
  c->res_factors_kept = false;  // these factors are the caller's, not an approximation's
  residual_open(c);
}

void residual_keep(skema_ctx* c, const double* U, const double* S, const double* V) {
  residual_load(c, U, S, V);
  c->res_factors_kept = true;
}

void residual_begin_kept(skema_ctx* c) {
  if (!c->res_factors_kept)
    fail(SKEMA_ESTATE, "no kept factors: enable skema_set_keep_factors before skema_low_rank_approx");
  residual_open(c);
}

// Rows [row0, row0 + nrows) of a dense A, in windows of params.window rows
// (map_A_by_window): A_w V -> (A_w V - U_w S)^2 into the sums; A^T U += A_w^T U_w.
void residual_dense(skema_ctx* c, Mat A, int64_t row0, int64_t nrows) {
  need_ready(c);
  const int64_t n = c->n, r = c->p.rank, W = c->w;
  const double* Urows = c->spd ? c->res_V : c->res_U;  // SPD: A V - V S
  double* AVw = static_cast<double*>(workspace(c, sizeof(double) * (size_t)(std::min(W, nrows) * r)));
  for (int64_t q = 0; q < nrows; q += W) {
    const int64_t wr = std::min(W, nrows - q), R0 = row0 + q;
    const float* Ap = A.p + q * A.rs;
    // AV_w (wr x r, row-major) = A_w V
    dgemm_f32_f64(c, wr, r, n, 1.0, Ap, A.rs, A.cs, c->res_V, r, 1, 0.0, AVw, r, 1);
    colsumsq_diff_kernel<<<grid_of(c, (wr + 7) / 8, 8), 256, 0, c->stream>>>(AVw, Urows + R0 * r, c->res_S, wr, r,
                                                                             c->res_sq);
    SKEMA_LAUNCHED(c);
    // A^T U (n x r, row-major) += A_w^T U_w
    if (!c->spd) dgemm_f32_f64(c, n, r, wr, 1.0, Ap, A.cs, A.rs, c->res_U + R0 * r, r, 1, 1.0, c->res_AtU, r, 1);
  }
}

void residual_csr(skema_ctx* c, const int64_t* rowptr, const int32_t* col, const float* val, int64_t col_offset,
                  int64_t row0, int64_t nrows) {
  need_ready(c);
  const int64_t r = c->p.rank;
  const int grid = grid_of(c, (nrows * 32 + 255) / 256, 16);
  // A^T U with FP64 atomics. Two alternatives measured slower on the
  // 1e6 x 1e5, 1e7-entry pass (19 ms with the atomics): a kernel that owned
  // column blocks of A^T U in shared memory (every CTA walked all rows of
  // the call; 49 ms), and a transposed (CSC) copy of the call's rows built
  // with counting atomics and summed a warp per column (27 ms).
  csr_residual_kernel<<<grid, 256, 0, c->stream>>>(rowptr, col, val, col_offset, nrows, row0, c->n,
                                                   c->spd ? c->res_V : c->res_U, c->res_V, c->res_S, r,
                                                   c->spd ? nullptr : c->res_AtU, c->res_sq);
  SKEMA_LAUNCHED(c);
}

// Kernel rows of the Gauss RBF input, a window at a time (the window of
// GaussRBFWindow::get, src/Skema_Window.hpp:90-107), then the dense pass.
void residual_rbf(skema_ctx* c, Mat P, int64_t npts, int64_t d, int64_t row0, int64_t nrows) {
  need_ready(c);
  const int64_t W = c->w;
  const int64_t wmax = std::min(W, nrows);
  const size_t kbytes = (sizeof(float) * (size_t)(wmax * npts) + 255) / 256 * 256;
  const size_t avbytes = sizeof(double) * (size_t)(wmax * c->p.rank);
  // K rows after the A V scratch of residual_dense, in one workspace
  char* ws = static_cast<char*>(workspace(c, avbytes + kbytes + 256));
  float* Kw = reinterpret_cast<float*>(ws + (avbytes + 255) / 256 * 256);
  for (int64_t q = 0; q < nrows; q += W) {
    const int64_t wr = std::min(W, nrows - q), R0 = row0 + q;
    rbf_window_block(c, P, npts, d, (float)c->p.kernel_gamma, R0, wr, Kw, npts);
    residual_dense(c, Mat{Kw, npts, 1}, R0, wr);
  }
}

void residual_finish(skema_ctx* c, double* rnorms) {
  need_ready(c);
  const int64_t n = c->n, r = c->p.rank;
  if (!c->spd) {
    // (A^T U - V S)^2 column sums join those of A V - U S
    colsumsq_diff_kernel<<<grid_of(c, (n + 7) / 8, 8), 256, 0, c->stream>>>(c->res_AtU, c->res_V, c->res_S, n, r,
                                                                            c->res_sq);
    SKEMA_LAUNCHED(c);
  }
  sqrt_kernel<<<1, 256, 0, c->stream>>>(c->res_sq, rnorms, r);
  SKEMA_LAUNCHED(c);
  c->res_ready = false;
}

}  // namespace skema
