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

// A^T U for a call's CSR rows through the transposed structure (CSC),
// without atomics on A^T U: count the entries of each column, scan the
// counts into column offsets, place each entry's row and value in its
// column, then a warp per column sums a U(i, :) over the column's entries
// (U row-major, r values per row, coalesced over the lanes) and adds the
// sum to A^T U(c, :), which no other warp touches.
__global__ void csr_col_count_kernel(const int32_t* __restrict__ col, int64_t b0, int64_t e0, int64_t ncol,
                                     int* __restrict__ cnt) {
  for (int64_t p = b0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < e0; p += (int64_t)gridDim.x * blockDim.x) {
    const int32_t c = col[p];
    if ((uint64_t)c < (uint64_t)ncol) atomicAdd(cnt + c, 1);
  }
}

// colptr[0..n] = exclusive prefix sum of cnt[0..n) (one CTA of 1024 threads:
// each thread sums a contiguous chunk, the chunk sums are scanned in shared
// memory, then each thread writes its chunk's offsets).
__global__ void __launch_bounds__(1024) scan_counts_kernel(const int* __restrict__ cnt, int64_t n,
                                                           int64_t* __restrict__ colptr) {
  __shared__ int64_t part[1024];
  const int64_t per = (n + blockDim.x - 1) / blockDim.x;
  const int64_t a = threadIdx.x * per, b = min(n, a + per);
  int64_t sum = 0;
  for (int64_t q = a; q < b; ++q) sum += cnt[q];
  part[threadIdx.x] = sum;
  __syncthreads();
  if (threadIdx.x == 0) {
    int64_t run = 0;
    for (int t = 0; t < (int)blockDim.x; ++t) {
      const int64_t v = part[t];
      part[t] = run;
      run += v;
    }
    colptr[n] = run;
  }
  __syncthreads();
  int64_t run = part[threadIdx.x];
  for (int64_t q = a; q < b; ++q) {
    colptr[q] = run;
    run += cnt[q];
  }
}

__global__ void csr_to_csc_kernel(const int64_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                                  const float* __restrict__ val, int64_t col_offset, int64_t nrows, int64_t ncol,
                                  const int64_t* __restrict__ colptr, int* __restrict__ fill,
                                  int32_t* __restrict__ rows_t, float* __restrict__ vals_t) {
  const int lane = threadIdx.x & 31;
  const int64_t w0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t i = w0; i < nrows; i += nw) {
    const int64_t b = rowptr[i] - col_offset, e = rowptr[i + 1] - col_offset;
    for (int64_t p = b + lane; p < e; p += 32) {
      const int32_t c = col[p];
      if ((uint64_t)c >= (uint64_t)ncol) continue;
      const int64_t q = colptr[c] + atomicAdd(fill + c, 1);
      rows_t[q] = (int32_t)i;
      vals_t[q] = val[p];
    }
  }
}

__global__ void csc_atu_kernel(const int64_t* __restrict__ colptr, const int32_t* __restrict__ rows_t,
                               const float* __restrict__ vals_t, int64_t ncol, int64_t R0,
                               const double* __restrict__ U, int64_t r, double* __restrict__ AtU) {
  const int lane = threadIdx.x & 31;
  const int64_t w0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t c = w0; c < ncol; c += nw) {
    const int64_t b = colptr[c], e = colptr[c + 1];
    if (b == e) continue;
    for (int64_t j0 = 0; j0 < r; j0 += 32) {
      const int64_t j = j0 + lane;
      if (j >= r) break;
      double acc = 0.0;
      for (int64_t q = b; q < e; ++q) acc = fma((double)vals_t[q], U[(R0 + rows_t[q]) * r + j], acc);
      AtU[c * r + j] += acc;
    }
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

void residual_begin(skema_ctx* c, const double* U, const double* S, const double* V) {
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
    SKEMA_CUDA(cudaMemsetAsync(c->res_AtU, 0, sizeof(double) * (size_t)(n * r), c->stream));
  }
  SKEMA_CUDA(cudaMemcpyAsync(c->res_S, S, sizeof(double) * (size_t)r, cudaMemcpyDeviceToDevice, c->stream));
  SKEMA_CUDA(cudaMemsetAsync(c->res_sq, 0, sizeof(double) * (size_t)r, c->stream));
  c->res_ready = true;
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
  // the transposed structure keeps call-local rows as int32
  const bool transpose = !c->spd && nrows < ((int64_t)1 << 31);
  // A V and its column sums of squares, a warp per row (with FP64 atomics
  // into A^T U when the call is too large to transpose)
  csr_residual_kernel<<<grid, 256, 0, c->stream>>>(rowptr, col, val, col_offset, nrows, row0, c->n,
                                                   c->spd ? c->res_V : c->res_U, c->res_V, c->res_S, r,
                                                   (c->spd || transpose) ? nullptr : c->res_AtU, c->res_sq);
  SKEMA_LAUNCHED(c);
  if (!transpose || nrows == 0) return;
  // A^T U through the call's transposed structure (the FP64 atomics of one
  // warp per row into A^T U took about 12 ms for 1e7 entries at r = 20; a
  // kernel that owned column blocks of A^T U in shared memory had every CTA
  // walk all rows of the call and ran 2.5x longer)
  int64_t ends[2];
  SKEMA_CUDA(cudaMemcpyAsync(&ends[0], rowptr, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream));
  SKEMA_CUDA(cudaMemcpyAsync(&ends[1], rowptr + nrows, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream));
  SKEMA_CUDA(cudaStreamSynchronize(c->stream));
  const int64_t b0 = ends[0] - col_offset, e0 = ends[1] - col_offset, nnz = e0 - b0, n = c->n;
  if (nnz <= 0) return;
  auto rup = [](size_t b) { return (b + 255) / 256 * 256; };
  const size_t b_cnt = rup(sizeof(int) * (size_t)n), b_ptr = rup(sizeof(int64_t) * (size_t)(n + 1));
  const size_t b_rows = rup(sizeof(int32_t) * (size_t)nnz), b_vals = rup(sizeof(float) * (size_t)nnz);
  char* ws = static_cast<char*>(workspace(c, 2 * b_cnt + b_ptr + b_rows + b_vals));
  int* cnt = reinterpret_cast<int*>(ws);
  int* fill = reinterpret_cast<int*>(ws + b_cnt);
  int64_t* colptr = reinterpret_cast<int64_t*>(ws + 2 * b_cnt);
  int32_t* rows_t = reinterpret_cast<int32_t*>(ws + 2 * b_cnt + b_ptr);
  float* vals_t = reinterpret_cast<float*>(ws + 2 * b_cnt + b_ptr + b_rows);
  SKEMA_CUDA(cudaMemsetAsync(cnt, 0, 2 * b_cnt, c->stream));  // cnt and fill
  csr_col_count_kernel<<<grid_of(c, (nnz + 255) / 256, 16), 256, 0, c->stream>>>(col, b0, e0, n, cnt);
  SKEMA_LAUNCHED(c);
  scan_counts_kernel<<<1, 1024, 0, c->stream>>>(cnt, n, colptr);
  SKEMA_LAUNCHED(c);
  csr_to_csc_kernel<<<grid, 256, 0, c->stream>>>(rowptr, col, val, col_offset, nrows, n, colptr, fill, rows_t,
                                                 vals_t);
  SKEMA_LAUNCHED(c);
  csc_atu_kernel<<<grid_of(c, (n * 32 + 255) / 256, 16), 256, 0, c->stream>>>(colptr, rows_t, vals_t, n, row0,
                                                                               c->res_U, r, c->res_AtU);
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
