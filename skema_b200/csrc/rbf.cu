// rbf.cu -- the Gauss RBF kernel input (GaussRBFWindow::get +
// GaussRBF::compute, src/Skema_Window.hpp:90-107, src/Skema_Kernel.cpp:6-81)
// and the standalone kernel-sketch forward/VJP pair.
//
// K(i, j) = exp(-gamma * sum_f (x_if - x_jf)^2) with explicit differences
// (the reference's formula, src/Skema_Kernel.cpp:37-44), and K(i, i) = 1
// (src/Skema_Kernel.cpp:62-74). Kernel rows are produced a window at a time
// into a scratch block and consumed by the dense sketch of the same window;
// the window is reused for the next one, so K never exists as a whole.
//
// VJP of Y = K Omega~^T with respect to gamma and the points, given
// Ybar = dL/dY:  M = Ybar Omega~,  E = M o K,
//   dL/dgamma = -sum_ij E_ij d_ij^2,
//   dL/dx_i   = -2 gamma sum_j (E_ij + E_ji)(x_i - x_j)
//             = -2 gamma [ (rowsum(E)_i + colsum(E)_i) x_i - (E X)_i - (E^T X)_i ].
// Kernel tiles are recomputed in the backward pass, never stored.
#include <cuda_runtime.h>

#include <algorithm>

#include "internal.h"

namespace skema {

size_t dense_scratch_bytes(const skema_ctx* c, int64_t wr);
void dense_window(skema_ctx* c, Mat Aw, int64_t R0, int64_t wr, float* T);

namespace {

constexpr int TT = 64;  // tile edge
constexpr int TD = 16;  // feature chunk

// MODE 0: out(i, j) = K.  MODE 1: out(i, j) <- out(i, j) * K (E = M o K) and
// accumulate -sum E d^2 into *dgamma, rowsum(E) into rsum[R0+i] and
// colsum(E) into csum[j].
template <int MODE>
__global__ void __launch_bounds__(256)
    rbf_tile_kernel(const float* __restrict__ P, int64_t prs, int64_t pcs, int64_t N, int64_t d,
                    float gamma, int64_t R0, int64_t wr, float* __restrict__ out, int64_t ldo,
                    double* __restrict__ dgamma, float* __restrict__ rsum, float* __restrict__ csum) {
  __shared__ float xi[TD][TT + 1];
  __shared__ float xj[TD][TT + 1];
  __shared__ float red[256];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int64_t tiles_j = (N + TT - 1) / TT;
  const int64_t tiles_i = (wr + TT - 1) / TT;
  for (int64_t tile = blockIdx.x; tile < tiles_i * tiles_j; tile += gridDim.x) {
    const int64_t i0 = (tile / tiles_j) * TT, j0 = (tile % tiles_j) * TT;
    float acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) acc[a][b] = 0.f;
    for (int64_t f0 = 0; f0 < d; f0 += TD) {
      for (int q = threadIdx.x; q < TD * TT; q += 256) {
        const int ff = q / TT, rr = q % TT;
        const int64_t f = f0 + ff;
        const int64_t gi = R0 + i0 + rr, gj = j0 + rr;
        xi[ff][rr] = (f < d && i0 + rr < wr) ? P[gi * prs + f * pcs] : 0.f;
        xj[ff][rr] = (f < d && gj < N) ? P[gj * prs + f * pcs] : 0.f;
      }
      __syncthreads();
#pragma unroll
      for (int ff = 0; ff < TD; ++ff) {
        float a[4], b[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          a[u] = xi[ff][ty + 16 * u];
          b[u] = xj[ff][tx + 16 * u];
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int v = 0; v < 4; ++v) {
            const float df = a[u] - b[v];
            acc[u][v] = fmaf(df, df, acc[u][v]);
          }
      }
      __syncthreads();
    }
    float gpart = 0.f;
    float rpart[4] = {0.f, 0.f, 0.f, 0.f};
    float cpart[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int64_t li = i0 + ty + 16 * u;
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const int64_t gj = j0 + tx + 16 * v;
        if (li < wr && gj < N) {
          const bool diag = (gj == R0 + li);
          const float kv = diag ? 1.f : expf(-gamma * acc[u][v]);
          float* op = out + li * ldo + gj;
          if (MODE == 0) {
            *op = kv;
          } else {
            const float e = *op * kv;
            *op = e;
            if (!diag) gpart += e * acc[u][v];
            rpart[u] += e;
            cpart[v] += e;
          }
        }
      }
    }
    if (MODE == 1) {
      // block reduction of the gamma partial
      red[threadIdx.x] = gpart;
      __syncthreads();
      for (int st = 128; st > 0; st >>= 1) {
        if (threadIdx.x < st) red[threadIdx.x] += red[threadIdx.x + st];
        __syncthreads();
      }
      if (threadIdx.x == 0) atomicAdd(dgamma, -(double)red[0]);
      __syncthreads();
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int64_t li = i0 + ty + 16 * u;
        float r = rpart[u];
        // reduce over tx (16 lanes of one half-warp share ty)
        for (int o = 8; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
        if (tx == 0 && li < wr) atomicAdd(rsum + R0 + li, r);
      }
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const int64_t gj = j0 + tx + 16 * v;
        if (gj < N && cpart[v] != 0.f) atomicAdd(csum + gj, cpart[v]);
      }
    }
  }
}

// dX = -2 gamma * (r o X - S), r = rsum + csum (N), S = S1 + S2 (N x d).
__global__ void rbf_dx_kernel(const float* __restrict__ P, int64_t prs, int64_t pcs, int64_t N,
                              int64_t d, float gamma, const float* __restrict__ rsum,
                              const float* __restrict__ csum, const float* __restrict__ S,
                              float* __restrict__ dX) {
  const int64_t total = N * d;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = q / d, f = q - i * d;
    const float r = rsum[i] + csum[i];
    dX[q] = -2.f * gamma * (r * P[i * prs + f * pcs] - S[q]);
  }
}

int grid_cap(const skema_ctx* c, int64_t want, int per_sm) {
  return (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)c->sm_count * per_sm));
}

void launch_tile(skema_ctx* c, int mode, Mat P, int64_t N, int64_t d, float gamma, int64_t R0,
                 int64_t wr, float* out, int64_t ldo, double* dg, float* rs, float* cs) {
  const int64_t tiles = ((wr + TT - 1) / TT) * ((N + TT - 1) / TT);
  const int grid = grid_cap(c, tiles, 8);
  if (mode == 0)
    rbf_tile_kernel<0><<<grid, 256, 0, c->stream>>>(P.p, P.rs, P.cs, N, d, gamma, R0, wr, out, ldo,
                                                    dg, rs, cs);
  else
    rbf_tile_kernel<1><<<grid, 256, 0, c->stream>>>(P.p, P.rs, P.cs, N, d, gamma, R0, wr, out, ldo,
                                                    dg, rs, cs);
  SKEMA_LAUNCHED(c);
}

// Rows per scratch block so that a w x N FP32 block stays near 1 GiB.
int64_t rows_per_block(int64_t N, int64_t cap_rows) {
  const int64_t budget = (int64_t)1 << 28;  // floats
  return std::max<int64_t>(1, std::min<int64_t>(cap_rows, budget / std::max<int64_t>(N, 1)));
}

}  // namespace

void rbf_window_block(skema_ctx* c, Mat P, int64_t N, int64_t d, float gamma, int64_t R0,
                      int64_t wr, float* out, int64_t ldo) {
  launch_tile(c, 0, P, N, d, gamma, R0, wr, out, ldo, nullptr, nullptr, nullptr);
}

void rbf_update(skema_ctx* c, Mat P, int64_t npts, int64_t d, int64_t row0, int64_t nrows) {
  if (c->residual_pass) {
    residual_rbf(c, P, npts, d, row0, nrows);
    return;
  }
  if (!c->spd && c->p.precision == SKEMA_PREC_BF16 && rbf_tc_supported(c, d)) {
    // tensor-core form: kernel tiles regenerated inside the sketch kernels
    rbf_tc_update(c, P, npts, d, row0, nrows);
    return;
  }
  const int64_t W = c->w;
  const int64_t N = npts;
  const float gamma = (float)c->p.kernel_gamma;
  const int64_t wmax = std::min(W, nrows);
  const size_t kbytes = (sizeof(float) * (size_t)(wmax * N) + 255) / 256 * 256;
  char* ws = (char*)workspace(c, kbytes + dense_scratch_bytes(c, wmax));
  float* Kw = (float*)ws;
  float* T = (float*)(ws + kbytes);
  for (int64_t r = 0; r < nrows; r += W) {
    const int64_t wr = std::min(W, nrows - r);
    const int64_t R0 = row0 + r;
    {
      StageScope st(c, ST_WINDOW);
      launch_tile(c, 0, P, N, d, gamma, R0, wr, Kw, N, nullptr, nullptr, nullptr);
    }
    dense_window(c, Mat{Kw, N, 1}, R0, wr, T);
  }
}

// Room for the K-split partial products of the FP32 forward and adjoint
// (a window's rows times k or d, at most 16 splits).
constexpr int64_t kRbfPartFloats = (int64_t)4 << 20;

void rbf_fwd(skema_ctx* c, const float* pts, int64_t N, int64_t d, double gamma,
             const float* omega, int64_t k, float* Y) {
  if (rbf_pair_tc_supported(c, d, k, gamma)) {
    rbf_fwd_tc(c, pts, N, d, gamma, omega, k, Y);
    return;
  }
  const Mat P{pts, d, 1};
  const int64_t wb = rows_per_block(N, N);
  const size_t kb = (sizeof(float) * (size_t)(wb * N) + 255) / 256 * 256;
  char* ws = (char*)workspace(c, kb + sizeof(float) * (size_t)kRbfPartFloats);
  float* Kw = (float*)ws;
  float* part = (float*)(ws + kb);  // K-split partial products
  for (int64_t r = 0; r < N; r += wb) {
    const int64_t wr = std::min(wb, N - r);
    launch_tile(c, 0, P, N, d, (float)gamma, r, wr, Kw, N, nullptr, nullptr, nullptr);
    // Y(r:r+wr, :) = K_w Omega~^T ; B(kk=j, col=q) = omega[q*N + j]
    sgemm_split(c, wr, k, N, 1.f, Mat{Kw, N, 1}, Mat{omega, 1, N}, 0.f, MatOut{Y + r * k, k, 1}, part,
                kRbfPartFloats);
  }
}

void rbf_vjp(skema_ctx* c, const float* pts, int64_t N, int64_t d, double gamma,
             const float* omega, int64_t k, const float* Ybar, float* dpts, double* dgamma) {
  if (rbf_pair_tc_supported(c, d, k, gamma)) {
    rbf_vjp_tc(c, pts, N, d, gamma, omega, k, Ybar, dpts, dgamma);
    return;
  }
  const Mat P{pts, d, 1};
  const int64_t wb = rows_per_block(N, N);
  const size_t eb = (sizeof(float) * (size_t)(wb * N) + 255) / 256 * 256;
  const size_t vb = (sizeof(float) * (size_t)N + 255) / 256 * 256;
  const size_t sb = (sizeof(float) * (size_t)(N * d) + 255) / 256 * 256;
  char* ws = (char*)workspace(c, eb + 2 * vb + sb + sizeof(float) * (size_t)kRbfPartFloats);
  float* E = (float*)ws;
  float* rs = (float*)(ws + eb);
  float* cs = (float*)(ws + eb + vb);
  float* S = (float*)(ws + eb + 2 * vb);
  float* part = (float*)(ws + eb + 2 * vb + sb);  // K-split partial products
  SKEMA_CUDA(cudaMemsetAsync(rs, 0, 2 * vb + sb, c->stream));
  SKEMA_CUDA(cudaMemsetAsync(dgamma, 0, sizeof(double), c->stream));
  for (int64_t r = 0; r < N; r += wb) {
    const int64_t wr = std::min(wb, N - r);
    // M_w = Ybar_w Omega~   (wr x N)
    sgemm(c, wr, N, k, 1.f, Mat{Ybar + r * k, k, 1}, Mat{omega, N, 1}, 0.f, MatOut{E, N, 1});
    // E_w = M_w o K_w, with the gamma / row / column partial sums
    launch_tile(c, 1, P, N, d, (float)gamma, r, wr, E, N, dgamma, rs, cs);
    // S(r:r+wr, :) += E_w X ;  S += E_w^T X_w
    sgemm_split(c, wr, d, N, 1.f, Mat{E, N, 1}, Mat{pts, d, 1}, 1.f, MatOut{S + r * d, d, 1}, part, kRbfPartFloats);
    sgemm(c, N, d, wr, 1.f, Mat{E, 1, N}, Mat{pts + r * d, d, 1}, 1.f, MatOut{S, d, 1});
  }
  rbf_dx_kernel<<<grid_cap(c, (N * d + 255) / 256, 16), 256, 0, c->stream>>>(
      pts, d, 1, N, d, (float)gamma, rs, cs, S, dpts);
  SKEMA_LAUNCHED(c);
}

}  // namespace skema
