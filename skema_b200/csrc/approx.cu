// approx.cu -- SketchySVD::initial_approx + low_rank_approx
// (src/Skema_SketchySVD.cpp:338-664) on the device, in FP64.
//
//   P = orth(X^T)          (reference: dgeqrf+dorgqr, :355-357)
//   Q = orth(Y)            (:381-383; here Y is not overwritten)
//   [U1, T1] = qr(Phi~ Q)  (:409, :453)
//   [U2, T2] = qr(Psi~ P)  (:430, :476)
//   Z2 = U1^T Z U2         (:500, :515)
//   Z2 = T1 \ Z2           (dgels on the triangular T1, :532)
//   C  = (T2 \ Z2^T)^T     (:549-562)
//   [Uc, S, Vc] = svd(C)   (dgesvd, :609)
//   U = Q Uc(:, 1:r), V = P Vc(:, 1:r), S(1:r)   (:627, :645, :657-660)
//
// orth/qr use CholeskyQR2 (Gram on the device, Cholesky in one CTA, triangular
// solve of the rows), with the shifted CholeskyQR pre-pass of Fukaya,
// Kannan, Nakatsukasa, Yamamoto and Yanagisawa (SIAM J. Sci. Comput. 2020)
// when the Gram matrix is not numerically positive definite. The Q factor
// equals Householder's up to column signs, so S is unchanged and U, V match
// LAPACK's up to sign. The SVD of the k x k core is a one-sided (Hestenes)
// Jacobi SVD with round-robin pair ordering in one CTA.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <initializer_list>
#include <limits>
#include <memory>
#include <vector>

#include "internal.h"

namespace skema {

namespace {

// ---------------------------------------------------------------- DGEMM ----
// C(i,j) = alpha * sum A(i,kk) B(kk,j) + beta*C(i,j); A, B may be float or
// double; FP64 accumulation. 64x64 tile, 4x4 per thread, split-K atomic.
template <typename TA, typename TB, bool ATOMIC>
__global__ void __launch_bounds__(256)
    dgemm_kernel(int64_t M, int64_t N, int64_t K, double alpha, const TA* __restrict__ A,
                 int64_t ars, int64_t acs, const TB* __restrict__ B, int64_t brs, int64_t bcs,
                 double beta, double* __restrict__ C, int64_t crs, int64_t ccs, int64_t kchunk) {
  __shared__ double As[8][64 + 1];
  __shared__ double Bs[8][64 + 1];
  const int tid = threadIdx.x;
  const int64_t m0 = (int64_t)blockIdx.x * 64, n0 = (int64_t)blockIdx.y * 64;
  const int64_t kb = (int64_t)blockIdx.z * kchunk, ke = min(K, kb + kchunk);
  if (kb >= ke) return;
  const bool am = (ars == 1);
  const bool bn = (bcs == 1);
  // 512 elements per operand tile: 2 per thread
  int la_m[2], la_k[2], lb_n[2], lb_k[2];
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const int e = tid + 256 * q;
    if (am) { la_m[q] = e & 63; la_k[q] = e >> 6; } else { la_k[q] = e & 7; la_m[q] = e >> 3; }
    if (bn) { lb_n[q] = e & 63; lb_k[q] = e >> 6; } else { lb_k[q] = e & 7; lb_n[q] = e >> 3; }
  }
  const int tx = tid & 15, ty = tid >> 4;
  double acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
  for (int64_t k0 = kb; k0 < ke; k0 += 8) {
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int64_t gm = m0 + la_m[q], gk = k0 + la_k[q];
      As[la_k[q]][la_m[q]] = (gm < M && gk < ke) ? (double)A[gm * ars + gk * acs] : 0.0;
      const int64_t gn = n0 + lb_n[q], gk2 = k0 + lb_k[q];
      Bs[lb_k[q]][lb_n[q]] = (gn < N && gk2 < ke) ? (double)B[gk2 * brs + gn * bcs] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 8; ++kk) {
      double a[4], b[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        a[u] = As[kk][ty + 16 * u];
        b[u] = Bs[kk][tx + 16 * u];
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int64_t gm = m0 + ty + 16 * i;
    if (gm >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int64_t gn = n0 + tx + 16 * j;
      if (gn >= N) continue;
      double* cp = C + gm * crs + gn * ccs;
      if (ATOMIC)
        atomicAdd(cp, alpha * acc[i][j]);
      else
        *cp = (beta == 0.0) ? alpha * acc[i][j] : fma(beta, *cp, alpha * acc[i][j]);
    }
  }
}

template <typename TA, typename TB>
void dgemm(skema_ctx* c, int64_t M, int64_t N, int64_t K, double alpha, const TA* A, int64_t ars,
           int64_t acs, const TB* B, int64_t brs, int64_t bcs, double beta, double* C, int64_t crs,
           int64_t ccs, bool allow_split = true);

__global__ void dscale_kernel(double* C, int64_t crs, int64_t ccs, int64_t M, int64_t N, double b) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < M * N;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = q % M, j = q / M;
    double* p = C + i * crs + j * ccs;
    *p = (b == 0.0) ? 0.0 : b * *p;
  }
}

template <typename TA, typename TB>
void dgemm(skema_ctx* c, int64_t M, int64_t N, int64_t K, double alpha, const TA* A, int64_t ars,
           int64_t acs, const TB* B, int64_t brs, int64_t bcs, double beta, double* C, int64_t crs,
           int64_t ccs, bool allow_split) {
  if (M <= 0 || N <= 0) return;
  const int64_t tiles = ((M + 63) / 64) * ((N + 63) / 64);
  int64_t split = 1;
  if (allow_split && tiles < 2 * c->sm_count && K >= 512)
    split = std::min<int64_t>((2 * c->sm_count + tiles - 1) / tiles, K / 256);
  if (split > 1) {
    dscale_kernel<<<(int)std::min<int64_t>((M * N + 255) / 256, 4096), 256, 0, c->stream>>>(
        C, crs, ccs, M, N, beta);
    SKEMA_LAUNCHED(c);
  }
  int64_t kchunk = (K + split - 1) / split;
  kchunk = (kchunk + 7) / 8 * 8;
  const int64_t gz = std::max<int64_t>(1, (K + kchunk - 1) / kchunk);
  if ((N + 63) / 64 > 65535) fail(SKEMA_EUNSUPPORTED, "dgemm: N too large");
  dim3 grid((unsigned)((M + 63) / 64), (unsigned)((N + 63) / 64), (unsigned)gz);
  if (split > 1)
    dgemm_kernel<TA, TB, true><<<grid, 256, 0, c->stream>>>(M, N, K, alpha, A, ars, acs, B, brs,
                                                            bcs, beta, C, crs, ccs, kchunk);
  else
    dgemm_kernel<TA, TB, false><<<grid, 256, 0, c->stream>>>(M, N, K, alpha, A, ars, acs, B, brs,
                                                             bcs, beta, C, crs, ccs, kchunk);
  SKEMA_LAUNCHED(c);
}

// ----------------------------------------- tall-skinny FP64 products -------
// Both run on the FP64 tensor cores: mma.sync m8n8k4 (D = A B + C, 8 x 4 by
// 4 x 8). Per lane: A holds element (lane / 4, lane % 4), B element
// (lane % 4, lane / 4), C / D elements (lane / 4, 2 (lane % 4) + i), i < 2.
__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

// G += A^T A for a tall column-major A (rows x k, ld lda, k <= 256; T float
// or double, widened to FP64 exactly). The k x k product is cut into 32 x 32
// tiles and only the tiles on or above the diagonal are formed (6 of 9 at
// k <= 96), each by P warps of the CTA that split the CTA's rows four at a
// time; a warp holds its tile as 4 x 4 MMA blocks. For a step of four rows
// the A fragment of column block c is A(r + lane % 4, c + lane / 4) and
// the B fragment of the same block is the same value, so a tile reads its
// two column ranges once per step. The partial tiles go to G (column-major
// k x k, zeroed beforehand) with atomics, mirrored below the diagonal.
//
// The same kernel forms C = A^T B for two tall matrices with the same rows
// (SYM = false: A rows x ka, B rows x kb, every 32 x 32 tile of the ka x kb
// product; C column-major with ld ka), which is how a dense map meets a
// tall basis (Phi~ Q = (Phi~^T)^T Q).
template <typename TA, typename TB, bool SYM>
__global__ void __launch_bounds__(512) atb_mma_kernel(const TA* __restrict__ A, int64_t lda, int ka,
                                                      const TB* __restrict__ B, int64_t ldb, int kb, int64_t rows,
                                                      double* __restrict__ G, int64_t rows_per_cta, int P) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nia = (ka + 31) >> 5, njb = (kb + 31) >> 5;
  const int ntiles = SYM ? nia * (nia + 1) / 2 : nia * njb;
  // blockIdx.y takes a group of tiles when they do not all fit one CTA
  const int per_cta = (int)(blockDim.x >> 5) / P;
  const int tile = (int)blockIdx.y * per_cta + warp / P, part = warp % P;
  if (tile >= ntiles) return;
  int ti, tj;
  if (SYM) {  // tile -> (ti, tj), ti <= tj, row-major over the upper triangle
    ti = 0, tj = tile;
    while (tj >= nia - ti) {
      tj -= nia - ti;
      ++ti;
    }
    tj += ti;
  } else {
    ti = tile / njb, tj = tile - (tile / njb) * njb;
  }
  const int64_t r0 = (int64_t)blockIdx.x * rows_per_cta, r1 = min(rows, r0 + rows_per_cta);
  const int lr = lane & 3, lc = lane >> 2;
  const TA* ci[4];
  const TB* cj[4];
  bool vi[4], vj[4];
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    const int coli = 32 * ti + 8 * m + lc, colj = 32 * tj + 8 * m + lc;
    vi[m] = coli < ka;
    vj[m] = colj < kb;
    ci[m] = A + (int64_t)(vi[m] ? coli : 0) * lda;
    cj[m] = B + (int64_t)(vj[m] ? colj : 0) * ldb;
  }
  double acc[4][4][2];
#pragma unroll
  for (int m = 0; m < 4; ++m)
#pragma unroll
    for (int n = 0; n < 4; ++n) acc[m][n][0] = acc[m][n][1] = 0.0;
  // two steps of four rows per iteration: their 16 loads are in flight
  // together before the 32 MMAs that use them
  const bool diag = SYM && ti == tj;
  for (int64_t r = r0 + 4 * part; r < r1; r += 8 * P) {
    double a[2][4], b[2][4];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int64_t row = r + 4 * P * u + lr;
      const bool rv = row < r1;
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        a[u][m] = (rv && vi[m]) ? (double)ci[m][row] : 0.0;
        b[u][m] = (!diag && rv && vj[m]) ? (double)cj[m][row] : 0.0;
      }
    }
#pragma unroll
    for (int u = 0; u < 2; ++u)
#pragma unroll
      for (int m = 0; m < 4; ++m)
#pragma unroll
        for (int n = 0; n < 4; ++n) dmma(acc[m][n], a[u][m], diag ? a[u][n] : b[u][n]);
  }
#pragma unroll
  for (int m = 0; m < 4; ++m)
#pragma unroll
    for (int n = 0; n < 4; ++n)
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int gi = 32 * ti + 8 * m + lc, gj = 32 * tj + 8 * n + 2 * lr + i;
        if (gi >= ka || gj >= kb) continue;
        atomicAdd(G + gi + (int64_t)gj * ka, acc[m][n][i]);
        if (SYM && ti != tj) atomicAdd(G + gj + (int64_t)gi * ka, acc[m][n][i]);
      }
}

// C = A B for a tall column-major A (rows x k, ld lda; T float or double)
// and a small B (k x n2, column-major ld ldb, k, n2 <= 8 NB). B stays in
// shared memory for the CTA's life as 4-row slices laid out for its MMA
// fragments; each warp takes 16-row tiles (two MMA row blocks) of C with
// every column block in registers. UPPER: B is upper triangular, so column
// block nb only needs the rows of B up to its last column and the K steps
// past it are skipped (about half the work for Q R^{-1}). C is column-major
// (ld ldc) and written, not accumulated.
template <typename T, int NB, bool UPPER>
__global__ void __launch_bounds__(256) tsm_mma_kernel(const T* __restrict__ A, int64_t lda, int64_t rows, int k,
                                                      const double* __restrict__ B, int64_t ldb, int n2,
                                                      double* __restrict__ C, int64_t ldc, int col0) {
  // B and C are the columns [col0, col0 + n2) of the whole product (col0
  // places them against the triangle for UPPER)
  extern __shared__ double tsm_smem[];
  // Bs[kk * ldbs + col], ldbs = 8 NB + 4 (mod 16) so a fragment's 4 x 8
  // reads hit 16 distinct bank pairs per half-warp
  constexpr int ldbs = (8 * NB + 15) / 16 * 16 + 4;
  const int kp = (k + 3) & ~3;
  for (int q = threadIdx.x; q < kp * 8 * NB; q += blockDim.x) {
    const int kk = q / (8 * NB), col = q - kk * (8 * NB);
    tsm_smem[kk * ldbs + col] = (kk < k && col < n2) ? B[kk + (int64_t)col * ldb] : 0.0;
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
  const int lr = lane & 3, lc = lane >> 2;
  for (int64_t r0 = ((int64_t)blockIdx.x * nwarp + warp) * 16; r0 < rows; r0 += (int64_t)gridDim.x * nwarp * 16) {
    double acc[2][NB][2];
#pragma unroll
    for (int m = 0; m < 2; ++m)
#pragma unroll
      for (int n = 0; n < NB; ++n) acc[m][n][0] = acc[m][n][1] = 0.0;
    const int64_t ra = r0 + lc, rb = r0 + 8 + lc;
    const bool va = ra < rows, vb = rb < rows;
    // eight K steps per batch: their 16 loads of A are in flight together
    for (int kb = 0; kb < kp; kb += 32) {
      double a0[8], a1[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int kk = kb + 4 * j + lr;
        const bool kv = kk < k;
        a0[j] = (va && kv) ? (double)A[ra + (int64_t)kk * lda] : 0.0;
        a1[j] = (vb && kv) ? (double)A[rb + (int64_t)kk * lda] : 0.0;
      }
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int k0 = kb + 4 * j;
        if (k0 >= kp) break;
        const double* bs = tsm_smem + (k0 + lr) * ldbs + lc;
#pragma unroll
        for (int n = 0; n < NB; ++n) {
          if (UPPER && col0 + 8 * n + 7 < k0) continue;  // B(k0.., block n) is zero
          const double b = bs[8 * n];
          dmma(acc[0][n], a0[j], b);
          dmma(acc[1][n], a1[j], b);
        }
      }
    }
#pragma unroll
    for (int m = 0; m < 2; ++m) {
      const int64_t row = r0 + 8 * m + lc;
      if (row >= rows) continue;
#pragma unroll
      for (int n = 0; n < NB; ++n)
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          const int col = 8 * n + 2 * lr + i;
          if (col < n2) C[row + (int64_t)col * ldc] = acc[m][n][i];
        }
    }
  }
}

// C (ka x kb, column-major, zeroed beforehand) += A^T B, or the Gram matrix
// A^T A when B is null (its upper tiles only).
template <typename TA, typename TB>
void launch_atb_mma(skema_ctx* c, const TA* A, int64_t lda, int64_t ka, const TB* B, int64_t ldb, int64_t kb,
                    int64_t rows, double* G) {
  const int nia = (int)((ka + 31) / 32), njb = (int)((kb + 31) / 32);
  const int tiles = B ? nia * njb : nia * (nia + 1) / 2;
  // up to 16 warps per CTA: P warps per tile when the tiles leave room,
  // else groups of 16 tiles over blockIdx.y
  const int P = std::max(1, 16 / tiles);
  const int per_cta = std::min(tiles, 16 / P);
  const int groups = (tiles + per_cta - 1) / per_cta;
  const int64_t ctas = std::max<int64_t>(1, std::min<int64_t>((rows + 1023) / 1024, (int64_t)c->sm_count));
  const int64_t per = ((rows + ctas - 1) / ctas + 3) / 4 * 4;
  const dim3 grid((unsigned)((rows + per - 1) / per), (unsigned)groups);
  if (B)
    atb_mma_kernel<TA, TB, false><<<grid, 32 * per_cta * P, 0, c->stream>>>(A, lda, (int)ka, B, ldb, (int)kb, rows,
                                                                             G, per, P);
  else
    atb_mma_kernel<TA, TA, true><<<grid, 32 * per_cta * P, 0, c->stream>>>(A, lda, (int)ka, A, lda, (int)ka, rows,
                                                                            G, per, P);
  SKEMA_LAUNCHED(c);
}

template <typename T, int NB>
void launch_tsm_nb(skema_ctx* c, const T* A, int64_t lda, int64_t rows, int64_t k, const double* B, int64_t ldb,
                   int64_t n2, double* C, int64_t ldc, bool upper, int col0) {
  constexpr int ldbs = (8 * NB + 15) / 16 * 16 + 4;
  const size_t smem = sizeof(double) * (size_t)(((k + 3) & ~3) * ldbs);
  auto kern = upper ? tsm_mma_kernel<T, NB, true> : tsm_mma_kernel<T, NB, false>;
  SKEMA_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int64_t tiles = (rows + 15) / 16;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((tiles + 7) / 8, 4 * (int64_t)c->sm_count));
  kern<<<grid, 256, smem, c->stream>>>(A, lda, rows, (int)k, B, ldb, (int)n2, C, ldc, col0);
  SKEMA_LAUNCHED(c);
}

// G (k x k, column-major) = A^T A for column-major A (rows x k, ld lda).
constexpr int64_t kTallMaxK = 256;  // the tensor-core tall products take k up to this
template <typename T>
void gram_t(skema_ctx* c, const T* A, int64_t lda, int64_t rows, int64_t k, double* G) {
  SKEMA_CUDA(cudaMemsetAsync(G, 0, sizeof(double) * (size_t)(k * k), c->stream));
  if (rows > 0) launch_atb_mma<T, T>(c, A, lda, k, static_cast<const T*>(nullptr), 0, k, rows, G);
}
void gram(skema_ctx* c, const double* A, int64_t lda, int64_t rows, int64_t k, double* G) {
  if (rows <= 0) {  // an empty row block (a rank without rows) adds nothing
    SKEMA_CUDA(cudaMemsetAsync(G, 0, sizeof(double) * (size_t)(k * k), c->stream));
    return;
  }
  if (k > kTallMaxK) {
    dgemm<double, double>(c, k, k, rows, 1.0, A, lda, 1, A, 1, lda, 0.0, G, 1, k);
    return;
  }
  gram_t<double>(c, A, lda, rows, k, G);
}

// Column block width of the tall product: B's k x (8 NB) slice (padded)
// stays in shared memory, at most 220 KB.
int tsm_chunk_blocks(int64_t k) {
  const int64_t kp = (k + 3) & ~3;
  for (int nb = 16; nb > 1; --nb) {
    const int64_t ldbs = (8 * nb + 15) / 16 * 16 + 4;
    if (kp * ldbs * (int64_t)sizeof(double) <= 220 * 1024) return nb;
  }
  return 1;
}

// C (rows x n2) = A (rows x k) B (k x n2), all column-major; upper: B is
// upper triangular (its zeros below the diagonal are not read). Column
// blocks of B beyond what shared memory holds go in further launches.
template <typename T>
void tall_times_small_t(skema_ctx* c, const T* A, int64_t lda, int64_t rows, int64_t k, const double* B,
                        int64_t ldb, int64_t n2, double* C, int64_t ldc, bool upper) {
  const int64_t chunk = 8 * (int64_t)tsm_chunk_blocks(k);
  for (int64_t c0 = 0; c0 < n2; c0 += chunk) {
    const int64_t w = std::min(chunk, n2 - c0);
    const double* Bc = B + c0 * ldb;
    double* Cc = C + c0 * ldc;
    const int col0 = (int)c0;
    switch ((w + 7) / 8) {
      case 1: launch_tsm_nb<T, 1>(c, A, lda, rows, k, Bc, ldb, w, Cc, ldc, upper, col0); break;
      case 2: launch_tsm_nb<T, 2>(c, A, lda, rows, k, Bc, ldb, w, Cc, ldc, upper, col0); break;
      case 3: launch_tsm_nb<T, 3>(c, A, lda, rows, k, Bc, ldb, w, Cc, ldc, upper, col0); break;
      case 4: launch_tsm_nb<T, 4>(c, A, lda, rows, k, Bc, ldb, w, Cc, ldc, upper, col0); break;
      case 5: launch_tsm_nb<T, 5>(c, A, lda, rows, k, Bc, ldb, w, Cc, ldc, upper, col0); break;
      case 6: launch_tsm_nb<T, 6>(c, A, lda, rows, k, Bc, ldb, w, Cc, ldc, upper, col0); break;
      case 7: launch_tsm_nb<T, 7>(c, A, lda, rows, k, Bc, ldb, w, Cc, ldc, upper, col0); break;
      case 8: launch_tsm_nb<T, 8>(c, A, lda, rows, k, Bc, ldb, w, Cc, ldc, upper, col0); break;
      case 9: launch_tsm_nb<T, 9>(c, A, lda, rows, k, Bc, ldb, w, Cc, ldc, upper, col0); break;
      case 10: launch_tsm_nb<T, 10>(c, A, lda, rows, k, Bc, ldb, w, Cc, ldc, upper, col0); break;
      case 11: launch_tsm_nb<T, 11>(c, A, lda, rows, k, Bc, ldb, w, Cc, ldc, upper, col0); break;
      case 12: launch_tsm_nb<T, 12>(c, A, lda, rows, k, Bc, ldb, w, Cc, ldc, upper, col0); break;
      case 13: launch_tsm_nb<T, 13>(c, A, lda, rows, k, Bc, ldb, w, Cc, ldc, upper, col0); break;
      case 14: launch_tsm_nb<T, 14>(c, A, lda, rows, k, Bc, ldb, w, Cc, ldc, upper, col0); break;
      case 15: launch_tsm_nb<T, 15>(c, A, lda, rows, k, Bc, ldb, w, Cc, ldc, upper, col0); break;
      default: launch_tsm_nb<T, 16>(c, A, lda, rows, k, Bc, ldb, w, Cc, ldc, upper, col0); break;
    }
  }
}
void tall_times_small(skema_ctx* c, const double* A, int64_t lda, int64_t rows, int64_t k, const double* B,
                      int64_t ldb, int64_t n2, double* C, int64_t ldc, bool upper = false) {
  if (rows <= 0 || n2 <= 0) return;
  if (k > kTallMaxK) {
    dgemm<double, double>(c, rows, n2, k, 1.0, A, 1, lda, B, 1, ldb, 0.0, C, 1, ldc, false);
    return;
  }
  tall_times_small_t<double>(c, A, lda, rows, k, B, ldb, n2, C, ldc, upper);
}

// ----------------------------------------------------- conversions ----------
__global__ void f2d_kernel(const float* __restrict__ S, int64_t srs, int64_t scs,
                           double* __restrict__ D, int64_t drs, int64_t dcs, int64_t M, int64_t N) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < M * N;
       q += (int64_t)gridDim.x * blockDim.x) {
    int64_t i, j;
    if (drs == 1) { i = q % M; j = q / M; } else { i = q / N; j = q % N; }
    D[i * drs + j * dcs] = (double)S[i * srs + j * scs];
  }
}

// ----------------------------------------------------------- Cholesky -------
// In place on the lower triangle of the column-major k x k G (one CTA).
// status[0] = 0 ok, j+1 if the j-th pivot was not positive.
__global__ void cholesky_kernel(double* G, int64_t k, int* status) {
  __shared__ double piv;
  __shared__ int bad;
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
  for (int64_t j = 0; j < k; ++j) {
    if (threadIdx.x == 0) {
      const double d = G[j + j * k];
      if (!(d > 0.0) && !bad) bad = (int)(j + 1);
      piv = (d > 0.0) ? sqrt(d) : 1.0;
      G[j + j * k] = piv;
    }
    __syncthreads();
    if (bad) break;
    for (int64_t i = j + 1 + threadIdx.x; i < k; i += blockDim.x) G[i + j * k] /= piv;
    __syncthreads();
    // trailing update of the lower triangle: G(a, b) -= L(a, j) L(b, j), b > j, a >= b
    const int64_t rem = k - j - 1;
    for (int64_t q = threadIdx.x; q < rem * rem; q += blockDim.x) {
      const int64_t a = j + 1 + q % rem, b = j + 1 + q / rem;
      if (a >= b) G[a + b * k] -= G[a + j * k] * G[b + j * k];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) status[0] = bad;
}

// R (upper, column-major k x k) = L^T from the factored lower triangle of G.
__global__ void lower_to_upper_kernel(const double* G, double* R, int64_t k) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < k * k;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = q % k, j = q / k;
    R[i + j * k] = (i <= j) ? G[j + i * k] : 0.0;
  }
}

// Solve R X = B in place for upper-triangular R (column-major k x k) and B
// (k x nrhs, column stride ldb): one warp per right-hand side.
__global__ void trsm_upper_kernel(const double* __restrict__ R, int64_t k, double* B, int64_t ldb,
                                  int64_t nrhs) {
  const int lane = threadIdx.x & 31;
  const int64_t col = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (col >= nrhs) return;
  double* x = B + col * ldb;
  for (int64_t i = k - 1; i >= 0; --i) {
    double s = 0.0;
    for (int64_t l = i + 1 + lane; l < k; l += 32) s += R[i + l * k] * x[l];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) x[i] = (x[i] - s) / R[i + i * k];
    __syncwarp();
  }
}

// Packed triangles in shared memory. Upper: column j holds rows 0..j from
// j (j + 1) / 2. Lower: column j holds rows j..k-1 from j k - j (j - 1) / 2.
__device__ __forceinline__ int up_off(int j) { return j * (j + 1) / 2; }
__device__ __forceinline__ int lo_off(int j, int k) { return j * k - j * (j - 1) / 2; }

// Largest k for which one packed triangle plus k doubles fits the 200 KB
// that the single-CTA kernels below use.
constexpr int kPackedMaxK = 225;
size_t packed_smem_bytes(int64_t k) { return sizeof(double) * (size_t)(k * (k + 1) / 2 + k); }

// Value v of the register array b (v known only at run time) without a
// local-memory copy: a chain of selects the compiler keeps in registers.
template <int VMAX>
__device__ __forceinline__ double pick(const double (&b)[VMAX], int v) {
  double r = 0.0;
#pragma unroll
  for (int q = 0; q < VMAX; ++q)
    if (q == v) r = b[q];
  return r;
}

// Solve R X = B in place, R upper triangular (column-major k x k, k <=
// min(32 VMAX, kPackedMaxK)) and B k x nrhs (column stride ldb). R is held
// packed in shared memory with the reciprocals of its diagonal; one warp
// per right-hand side keeps its column in registers (entry i in lane i % 32,
// slot i / 32) and eliminates column by column: x_i = b_i / R(i, i), then
// b_l -= R(l, i) x_i for l < i.
template <int VMAX>
__global__ void __launch_bounds__(256) trsm_upper_packed_kernel(const double* __restrict__ R, int k, double* B,
                                                                int64_t ldb, int nrhs) {
  extern __shared__ double tp_smem[];
  double* Rp = tp_smem;
  double* inv = Rp + k * (k + 1) / 2;
  for (int q = threadIdx.x; q < k * k; q += blockDim.x) {
    const int i = q % k, j = q / k;
    if (i <= j) Rp[up_off(j) + i] = R[q];
  }
  for (int i = threadIdx.x; i < k; i += blockDim.x) inv[i] = 1.0 / R[i + (int64_t)i * k];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int col = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (col >= nrhs) return;
  double* x = B + (int64_t)col * ldb;
  double b[VMAX];
#pragma unroll
  for (int v = 0; v < VMAX; ++v) {
    const int i = lane + 32 * v;
    b[v] = i < k ? x[i] : 0.0;
  }
  for (int i = k - 1; i >= 0; --i) {
    const double xi = __shfl_sync(0xffffffffu, pick(b, i >> 5) * inv[i], i & 31);
    const double* rc = Rp + up_off(i);
#pragma unroll
    for (int v = 0; v < VMAX; ++v) {
      const int l = lane + 32 * v;
      if (l < i)
        b[v] = fma(-rc[l], xi, b[v]);
      else if (l == i)
        b[v] = xi;
    }
  }
#pragma unroll
  for (int v = 0; v < VMAX; ++v) {
    const int i = lane + 32 * v;
    if (i < k) x[i] = b[v];
  }
}

// Cholesky of the symmetric positive definite G (column-major k x k, lower
// triangle read) with its factor and inverse: R = L^T and Rinv = R^{-1}
// (both upper, column-major k x k, zeros below the diagonal). One CTA of
// 1024 threads, the lower triangle packed in shared memory. Right-looking:
// step j subtracts L(a, j) L(b, j) / d_j from the trailing triangle using
// the unscaled column, so one barrier per column suffices; the columns are
// scaled by sqrt(d_j) afterwards. L^{-1} comes from forward substitution of
// the unit vectors (one warp per column, the column in registers), and
// Rinv(j, i) = L^{-1}(i, j). G is read completely before anything is
// written, so Rinv may alias G. status[0] = 0, or j + 1 when the j-th pivot
// is not positive (R and Rinv are then not written).
template <int VMAX>
__global__ void __launch_bounds__(1024) chol_factor_kernel(const double* G, int k, double* R, double* Rinv,
                                                           int* status) {
  extern __shared__ double cf_smem[];
  double* L = cf_smem;
  double* aux = L + k * (k + 1) / 2;  // pivots, then their reciprocals
  for (int q = threadIdx.x; q < k * k; q += blockDim.x) {
    const int i = q % k, j = q / k;
    if (i >= j) L[lo_off(j, k) + i - j] = G[q];
  }
  __syncthreads();
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  int bad = 0;
  for (int j = 0; j < k; ++j) {
    const double d = L[lo_off(j, k)];
    if (!(d > 0.0)) {  // every thread reads the same pivot: a uniform exit
      bad = j + 1;
      break;
    }
    const double dinv = 1.0 / d;
    const double* colj = L + lo_off(j, k) - j;  // colj[a] = L(a, j)
    for (int b = j + 1 + ty; b < k; b += 32) {
      const double lbj = colj[b] * dinv;
      double* colb = L + lo_off(b, k) - b;
      for (int a = b + tx; a < k; a += 32) colb[a] = fma(-colj[a], lbj, colb[a]);
    }
    __syncthreads();
  }
  if (bad) {
    if (threadIdx.x == 0) status[0] = bad;
    return;
  }
  for (int j = threadIdx.x; j < k; j += blockDim.x) aux[j] = sqrt(L[lo_off(j, k)]);
  __syncthreads();
  for (int j = ty; j < k; j += 32) {
    const double p = aux[j];
    double* colj = L + lo_off(j, k) - j;
    for (int i = j + tx; i < k; i += 32) colj[i] = (i == j) ? p : colj[i] / p;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < k * k; q += blockDim.x) {
    const int i = q % k, j = q / k;
    R[q] = (i <= j) ? L[lo_off(i, k) + j - i] : 0.0;
  }
  for (int j = threadIdx.x; j < k; j += blockDim.x) aux[j] = 1.0 / aux[j];
  __syncthreads();
  for (int j = ty; j < k; j += 32) {
    double b[VMAX];
#pragma unroll
    for (int v = 0; v < VMAX; ++v) b[v] = (tx + 32 * v == j) ? 1.0 : 0.0;
    for (int l = j; l < k; ++l) {
      const double yl = __shfl_sync(0xffffffffu, pick(b, l >> 5) * aux[l], l & 31);
      const double* coll = L + lo_off(l, k) - l;
#pragma unroll
      for (int v = 0; v < VMAX; ++v) {
        const int i = tx + 32 * v;
        if (i > l && i < k)
          b[v] = fma(-coll[i], yl, b[v]);
        else if (i == l)
          b[v] = yl;
      }
    }
#pragma unroll
    for (int v = 0; v < VMAX; ++v) {
      const int i = tx + 32 * v;
      if (i < k) Rinv[j + (int64_t)i * k] = (i >= j) ? b[v] : 0.0;
    }
  }
  if (threadIdx.x == 0) status[0] = 0;
}

// D = S^T for column-major k x k matrices.
__global__ void dtranspose_kernel(const double* __restrict__ S, double* __restrict__ D, int64_t k) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < k * k;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = q % k, j = q / k;
    D[i + j * k] = S[j + i * k];
  }
}

__global__ void identity_kernel(double* I, int64_t k) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < k * k;
       q += (int64_t)gridDim.x * blockDim.x)
    I[q] = (q % k == q / k) ? 1.0 : 0.0;
}

// G(j, j) += shift
__global__ void shift_diag_kernel(double* G, int64_t k, const double* fro2, double factor) {
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j < k) G[j + j * k] += factor * fro2[0];
}

__global__ void trace_kernel(const double* G, int64_t k, double* out) {
  __shared__ double red[256];
  double s = 0.0;
  for (int64_t j = threadIdx.x; j < k; j += blockDim.x) s += G[j + j * k];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int st = 128; st > 0; st >>= 1) {
    if (threadIdx.x < st) red[threadIdx.x] += red[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = red[0];
}

// --------------------------------------------------- sparse-sign maps ------
// out(r, :) = sum_t sign_rt Q(c_rt, :) for a row-sparse map (R x m, zeta per
// row); Q is m x k column-major (ldq), out R x k column-major (ldo).
__global__ void rowsparse_apply_kernel(const uint32_t* __restrict__ mp, int zeta, int64_t R,
                                       const double* __restrict__ Q, int64_t ldq, int64_t k,
                                       double* __restrict__ out, int64_t ldo, int64_t q0, int64_t qrows) {
  // Q holds rows [q0, q0 + qrows) of the operand; map entries elsewhere
  // belong to other row blocks
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < R * k;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = q % R, j = q / R;
    double a = 0.0;
    for (int t = 0; t < zeta; ++t) {
      const uint32_t w = mp[r * zeta + t];
      const int64_t row = (int64_t)(w & 0x7fffffffu) - q0;
      if ((uint64_t)row >= (uint64_t)qrows) continue;
      const double v = Q[row + j * ldq];
      a += (w >> 31) ? -v : v;
    }
    out[r + j * ldo] = a;
  }
}

// out(c_jt, :) += sign_jt P(j, :) for a stored-transposed map (n rows, zeta
// entries over R columns); out is R x k column-major, zeroed by the caller.
__global__ void colsparse_apply_kernel(const uint32_t* __restrict__ mp, int zeta, int64_t n,
                                       const double* __restrict__ P, int64_t ldp, int64_t k,
                                       double* __restrict__ out, int64_t ldo) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n * k;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = q % n, col = q / n;
    const double v = P[j + col * ldp];
    for (int t = 0; t < zeta; ++t) {
      const uint32_t w = mp[j * zeta + t];
      atomicAdd(out + (int64_t)(w & 0x7fffffffu) + col * ldo, (w >> 31) ? -v : v);
    }
  }
}

// The same product with a private copy of out per CTA in shared memory: the
// CTA's stored rows add into it with shared-memory atomics (few collisions:
// out has R x k entries), then each entry goes to out with one global atomic
// per CTA. Used when out fits in shared memory; the kernel above turns every
// map entry into a global atomic on out's few entries.
__global__ void colsparse_apply_smem_kernel(const uint32_t* __restrict__ mp, int zeta, int64_t n,
                                            const double* __restrict__ P, int64_t ldp, int64_t k,
                                            double* __restrict__ out, int64_t ldo, int64_t R) {
  extern __shared__ double priv[];  // R x k, column-major (ld R)
  for (int64_t q = threadIdx.x; q < R * k; q += blockDim.x) priv[q] = 0.0;
  __syncthreads();
  const int64_t per = (n + gridDim.x - 1) / gridDim.x;
  const int64_t j0 = (int64_t)blockIdx.x * per, j1 = min(n, j0 + per);
  const int64_t span = j1 > j0 ? j1 - j0 : 0;
  for (int64_t q = threadIdx.x; q < span * k; q += blockDim.x) {
    const int64_t j = j0 + q % span, col = q / span;  // consecutive threads: consecutive rows j
    const double v = P[j + col * ldp];
    for (int t = 0; t < zeta; ++t) {
      const uint32_t w = mp[j * zeta + t];
      atomicAdd(priv + (int64_t)(w & 0x7fffffffu) + col * R, (w >> 31) ? -v : v);
    }
  }
  __syncthreads();
  for (int64_t q = threadIdx.x; q < R * k; q += blockDim.x) {
    const double a = priv[q];
    if (a != 0.0) atomicAdd(out + (q % R) + (q / R) * ldo, a);
  }
}

// ------------------------------------------------------ Jacobi SVD ---------
// One-sided Jacobi on the column-major k x k A (overwritten by A V = U S),
// V accumulated (column-major k x k). One CTA; each half-warp rotates one
// pair of a round-robin round, and a sweep ends the loop when it made no
// rotation (every pair within tol of orthogonal).
// A and V are worked on in shared memory (2 k^2 doubles, k <= 114), copied
// in at the start and out at the end; every rotation reads and writes two
// columns of each, so global memory would put an L2 round trip on every
// step.
__global__ void __launch_bounds__(1024) jacobi_svd_kernel(double* Ag, double* Vg, int64_t k64, int max_sweeps,
                                                            double tol, int* sweeps_out) {
  __shared__ int rotated;
  extern __shared__ double jac_smem[];
  const int k = (int)k64;
  double* A = jac_smem;
  double* V = jac_smem + (size_t)k * k;
  for (int q = threadIdx.x; q < k * k; q += blockDim.x) {
    A[q] = Ag[q];
    V[q] = (q % k == q / k) ? 1.0 : 0.0;
  }
  // a pair per half-warp: 64 pairs at a time, all of them for k <= 128
  const int hl = threadIdx.x & 15, slot = threadIdx.x >> 4, nslot = blockDim.x >> 4;
  const unsigned hmask = (threadIdx.x & 16) ? 0xffff0000u : 0x0000ffffu;
  const int kp = (k + 1) & ~1;  // even number of players
  int sweep = 0;
  for (; sweep < max_sweeps; ++sweep) {
    if (threadIdx.x == 0) rotated = 0;
    __syncthreads();
    for (int round = 0; round < kp - 1; ++round) {
      for (int pr = slot; pr < kp / 2; pr += nslot) {
        // round-robin pairing: player kp-1 stays, the others rotate
        int p, q;
        if (pr == 0) {
          p = round;
          q = kp - 1;
        } else {
          p = round + pr;
          if (p >= kp - 1) p -= kp - 1;
          q = round - pr;
          if (q < 0) q += kp - 1;
        }
        if (p > q) {
          const int t = p;
          p = q;
          q = t;
        }
        if (q >= k) continue;  // bye
        double* ap = A + (size_t)p * k;
        double* aq = A + (size_t)q * k;
        double al = 0.0, be = 0.0, ga = 0.0;
        for (int i = hl; i < k; i += 16) {
          const double x = ap[i], y = aq[i];
          al = fma(x, x, al);
          be = fma(y, y, be);
          ga = fma(x, y, ga);
        }
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) {
          al += __shfl_xor_sync(hmask, al, o);
          be += __shfl_xor_sync(hmask, be, o);
          ga += __shfl_xor_sync(hmask, ga, o);
        }
        // converged pair: |gamma| <= tol sqrt(alpha beta), compared squared
        if (ga == 0.0 || ga * ga <= (tol * tol) * (al * be)) continue;
        if (hl == 0) rotated = 1;
        // tan of the rotation angle, the smaller root of t^2 + 2 zeta t - 1
        // with zeta = d / h, d = beta - alpha, h = 2 gamma, written as
        // t = sign(d) h / (|d| + sqrt(d^2 + h^2)): one square root and one
        // division on the chain that every round waits for
        const double d = be - al, h = 2.0 * ga;
        const double t = (d >= 0.0 ? h : -h) / (fabs(d) + sqrt(fma(d, d, h * h)));
        const double cs = rsqrt(fma(t, t, 1.0)), sn = cs * t;
        for (int i = hl; i < k; i += 16) {
          const double x = ap[i], y = aq[i];
          ap[i] = cs * x - sn * y;
          aq[i] = sn * x + cs * y;
        }
        double* vp = V + (size_t)p * k;
        double* vq = V + (size_t)q * k;
        for (int i = hl; i < k; i += 16) {
          const double x = vp[i], y = vq[i];
          vp[i] = cs * x - sn * y;
          vq[i] = sn * x + cs * y;
        }
      }
      __syncthreads();
    }
    const bool more = rotated != 0;
    __syncthreads();
    if (!more) break;
  }
  if (threadIdx.x == 0) sweeps_out[0] = sweep;
  __syncthreads();
  for (int q = threadIdx.x; q < k * k; q += blockDim.x) {
    Ag[q] = A[q];
    Vg[q] = V[q];
  }
}

// Block one-sided Jacobi for a k x k problem too large for one CTA's shared
// memory. The columns are cut into nb blocks of bs (the last ones short or
// empty). An outer round pairs the blocks round-robin; each CTA takes one
// pair (I, J), copies the up to 2 bs columns of A and V into shared memory,
// runs one inner sweep of the one-sided Jacobi rotations over all pairs of
// those columns (a half-warp per pair, as in the single-CTA kernel), and
// writes them back. rotated[0] is set when any rotation was made. nb - 1
// outer rounds make an outer sweep, after which every pair of columns has
// met; sweeps continue until one makes no rotation.
__global__ void __launch_bounds__(1024) jacobi_block_kernel(double* __restrict__ Ag, double* __restrict__ Vg, int k,
                                                            int bs, int nb, int round, double tol,
                                                            int* __restrict__ rotated) {
  extern __shared__ double jb_smem[];
  __shared__ int any;
  // this CTA's pair of blocks in the round-robin round
  const int pr = blockIdx.x;
  int bi, bj;
  if (pr == 0) {
    bi = round;
    bj = nb - 1;
  } else {
    bi = round + pr;
    if (bi >= nb - 1) bi -= nb - 1;
    bj = round - pr;
    if (bj < 0) bj += nb - 1;
  }
  // local column c < 2 bs: block bi's columns, then block bj's
  auto gcol = [&](int c) { return c < bs ? bi * bs + c : bj * bs + (c - bs); };
  double* A = jb_smem;                       // 2 bs columns of length k
  double* V = jb_smem + (size_t)2 * bs * k;  // same for V
  for (int q = threadIdx.x; q < 2 * bs * k; q += blockDim.x) {
    const int c = q / k, i = q - c * k, g = gcol(c);
    const bool in = g < k;
    A[q] = in ? Ag[(size_t)g * k + i] : 0.0;
    V[q] = in ? Vg[(size_t)g * k + i] : 0.0;
  }
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  const int hl = threadIdx.x & 15, slot = threadIdx.x >> 4, nslot = blockDim.x >> 4;
  const unsigned hmask = (threadIdx.x & 16) ? 0xffff0000u : 0x0000ffffu;
  const int np = 2 * bs;  // even number of local players
  for (int r = 0; r < np - 1; ++r) {
    for (int pp = slot; pp < np / 2; pp += nslot) {
      int p, q;
      if (pp == 0) {
        p = r;
        q = np - 1;
      } else {
        p = r + pp;
        if (p >= np - 1) p -= np - 1;
        q = r - pp;
        if (q < 0) q += np - 1;
      }
      if (gcol(p) >= k || gcol(q) >= k) continue;  // an absent column
      double* ap = A + (size_t)p * k;
      double* aq = A + (size_t)q * k;
      double al = 0.0, be = 0.0, ga = 0.0;
      for (int i = hl; i < k; i += 16) {
        const double x = ap[i], y = aq[i];
        al = fma(x, x, al);
        be = fma(y, y, be);
        ga = fma(x, y, ga);
      }
#pragma unroll
      for (int o = 8; o > 0; o >>= 1) {
        al += __shfl_xor_sync(hmask, al, o);
        be += __shfl_xor_sync(hmask, be, o);
        ga += __shfl_xor_sync(hmask, ga, o);
      }
      if (ga == 0.0 || ga * ga <= (tol * tol) * (al * be)) continue;
      if (hl == 0) any = 1;
      const double d = be - al, h = 2.0 * ga;
      const double t = (d >= 0.0 ? h : -h) / (fabs(d) + sqrt(fma(d, d, h * h)));
      const double cs = rsqrt(fma(t, t, 1.0)), sn = cs * t;
      for (int i = hl; i < k; i += 16) {
        const double x = ap[i], y = aq[i];
        ap[i] = cs * x - sn * y;
        aq[i] = sn * x + cs * y;
      }
      double* vp = V + (size_t)p * k;
      double* vq = V + (size_t)q * k;
      for (int i = hl; i < k; i += 16) {
        const double x = vp[i], y = vq[i];
        vp[i] = cs * x - sn * y;
        vq[i] = sn * x + cs * y;
      }
    }
    __syncthreads();
  }
  for (int q = threadIdx.x; q < 2 * bs * k; q += blockDim.x) {
    const int c = q / k, i = q - c * k, g = gcol(c);
    if (g < k) {
      Ag[(size_t)g * k + i] = A[q];
      Vg[(size_t)g * k + i] = V[q];
    }
  }
  if (threadIdx.x == 0 && any) atomicExch(rotated, 1);
}

__global__ void store_int_kernel(int* dst, int v) { *dst = v; }

// One-sided Jacobi for k above the single-CTA size: block sweeps driven
// from the host, each outer sweep's rotation flag read back once.
void jacobi_svd_blocked(skema_ctx* c, double* A, double* V, int64_t k, int max_sweeps, double tol,
                        int* sweeps_out) {
  // columns per block: 8, or fewer where two blocks of A and V would not fit
  // about 200 KB. Small blocks put more CTAs on each round (nb / 2) for the
  // same pairs per outer sweep: at k = 201, 8 columns (13 CTAs a round) took
  // 10.5 ms against 15.1 ms for 31 columns (4 CTAs), 12 and 16 about 11.2 ms,
  // 6 and 4 11.1 and 11.8 ms.
  const int bs = (int)std::max<int64_t>(
      2, std::min<int64_t>(8, (200 * 1024) / (4 * (int64_t)sizeof(double) * k)));
  int nb = (int)((k + bs - 1) / bs);
  nb += nb & 1;  // an even number of players
  const size_t smem = sizeof(double) * (size_t)(4 * bs * k);
  SKEMA_CUDA(cudaFuncSetAttribute(jacobi_block_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  identity_kernel<<<(unsigned)std::min<int64_t>((k * k + 255) / 256, 4096), 256, 0, c->stream>>>(V, k);
  SKEMA_LAUNCHED(c);
  int* flag = sweeps_out + 2;  // the caller's status block has room after the sweep count
  int sweep = 0;
  for (; sweep < max_sweeps; ++sweep) {
    SKEMA_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), c->stream));
    for (int r = 0; r < nb - 1; ++r) {
      jacobi_block_kernel<<<nb / 2, 1024, smem, c->stream>>>(A, V, (int)k, bs, nb, r, tol, flag);
      SKEMA_LAUNCHED(c);
    }
    int h = 0;
    SKEMA_CUDA(cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    SKEMA_CUDA(cudaStreamSynchronize(c->stream));
    if (!h) break;
  }
  store_int_kernel<<<1, 1, 0, c->stream>>>(sweeps_out, sweep);
  SKEMA_LAUNCHED(c);
}

// The SVD kernel for a k x k problem: shared memory when A and V fit.
void jacobi_svd(skema_ctx* c, double* A, double* V, int64_t k, int max_sweeps, double tol, int* sweeps_out) {
  const size_t smem = sizeof(double) * (size_t)(2 * k * k);
  // a half-warp per pair of a round: (k + 1) / 2 pairs, at most 64 at a time
  const int threads = (int)std::min<int64_t>(1024, ((k + 1) / 2 * 16 + 31) / 32 * 32);
  if (smem <= 200 * 1024) {
    SKEMA_CUDA(cudaFuncSetAttribute(jacobi_svd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    jacobi_svd_kernel<<<1, threads, smem, c->stream>>>(A, V, k, max_sweeps, tol, sweeps_out);
    SKEMA_LAUNCHED(c);
    return;
  }
  // larger k: block sweeps in shared memory (a single CTA working on A and
  // V in global memory took 51 ms at k = 201, with every rotation waiting
  // on L2)
  jacobi_svd_blocked(c, A, V, k, max_sweeps, tol, sweeps_out);
}

// sigma_j = ||a_j||, ranks by descending sigma (ties by index), then
// U(:, rank) = a_j / sigma_j, Vout(:, rank) = v_j, S(rank) = sigma_j.
__global__ void svd_finish_kernel(const double* A, const double* V, int64_t k, double* U,
                                  double* Vout, double* S, double* sig) {
  for (int64_t j = threadIdx.x; j < k; j += blockDim.x) {
    double s = 0.0;
    for (int64_t i = 0; i < k; ++i) s += A[i + j * k] * A[i + j * k];
    sig[j] = sqrt(s);
  }
  __syncthreads();
  for (int64_t j = threadIdx.x; j < k; j += blockDim.x) {
    int64_t rank = 0;
    const double sj = sig[j];
    for (int64_t l = 0; l < k; ++l)
      if (sig[l] > sj || (sig[l] == sj && l < j)) ++rank;
    S[rank] = sj;
    const double inv = sj > 0.0 ? 1.0 / sj : 0.0;
    for (int64_t i = 0; i < k; ++i) {
      U[i + rank * k] = A[i + j * k] * inv;
      Vout[i + rank * k] = V[i + j * k];
    }
  }
}

// ------------------------------------------------------------ helpers ------
// Buffers of one approximation call, carved from the context's workspace
// (grown once, then reused by every later call: no allocation per call).
class Carve {
 public:
  Carve(skema_ctx* c, std::initializer_list<size_t> bytes) {
    size_t total = 0;
    for (size_t b : bytes) total += round(b);
    base_ = static_cast<char*>(workspace(c, total));
    at_ = base_;
  }
  double* take(size_t bytes) {
    char* p = at_;
    at_ += round(bytes);
    return reinterpret_cast<double*>(p);
  }

 private:
  static size_t round(size_t b) { return (std::max<size_t>(b, 16) + 255) / 256 * 256; }
  char* base_;
  char* at_;
};

int g1(const skema_ctx* c, int64_t total) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, (int64_t)c->sm_count * 16));
}

// R X = B in place for upper-triangular R (k x k) and B (k x nrhs, ld ldb):
// the packed shared-memory kernel when R fits, else one warp per right-hand
// side reading R from global memory.
void trsm_upper(skema_ctx* c, const double* R, int64_t k, double* B, int64_t ldb, int64_t nrhs) {
  if (nrhs <= 0 || k <= 0) return;
  if (k <= kPackedMaxK) {
    const size_t smem = packed_smem_bytes(k);
    const int grid = (int)((nrhs + 7) / 8);
    auto launch = [&](auto kern) {
      SKEMA_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      kern<<<grid, 256, smem, c->stream>>>(R, (int)k, B, ldb, (int)nrhs);
    };
    if (k <= 32)
      launch(trsm_upper_packed_kernel<1>);
    else if (k <= 64)
      launch(trsm_upper_packed_kernel<2>);
    else if (k <= 128)
      launch(trsm_upper_packed_kernel<4>);
    else
      launch(trsm_upper_packed_kernel<8>);
  } else {
    trsm_upper_kernel<<<(int)((nrhs * 32 + 255) / 256), 256, 0, c->stream>>>(R, k, B, ldb, nrhs);
  }
  SKEMA_LAUNCHED(c);
}

// Cholesky G = L L^T of the k x k G with R = L^T and Rinv = R^{-1} (Rinv may
// alias G); st[0] as chol_factor_kernel sets it, read by the caller. G is
// consumed. When the factorisation fails R and Rinv hold no meaning.
void chol_inverse(skema_ctx* c, double* G, int64_t k, double* R, double* Rinv, int* st) {
  if (k <= kPackedMaxK) {
    const size_t smem = packed_smem_bytes(k);
    auto launch = [&](auto kern) {
      SKEMA_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      kern<<<1, 1024, smem, c->stream>>>(G, (int)k, R, Rinv, st);
    };
    if (k <= 32)
      launch(chol_factor_kernel<1>);
    else if (k <= 64)
      launch(chol_factor_kernel<2>);
    else if (k <= 128)
      launch(chol_factor_kernel<4>);
    else
      launch(chol_factor_kernel<8>);
    SKEMA_LAUNCHED(c);
    return;
  }
  cholesky_kernel<<<1, 1024, 0, c->stream>>>(G, k, st);
  SKEMA_LAUNCHED(c);
  lower_to_upper_kernel<<<g1(c, k * k), 256, 0, c->stream>>>(G, R, k);
  SKEMA_LAUNCHED(c);
  identity_kernel<<<g1(c, k * k), 256, 0, c->stream>>>(Rinv, k);
  SKEMA_LAUNCHED(c);
  trsm_upper(c, R, k, Rinv, k, k);
}

// In-place CholeskyQR2 (+ shifted pre-pass if needed) of the column-major
// rows x k matrix Qm (ld = rows). On return Rout (k x k, upper, column-major)
// holds R with Q_in = Q_out R. False when a Cholesky failed even after the
// shifted pass (the columns are numerically dependent); Qm then holds the
// input times an invertible upper-triangular matrix (the same column space).
bool cholqr_try(skema_ctx* c, double* Qm, int64_t rows, int64_t k, double* Rout, double* work,
                int* dstatus) {
  double* G = work;            // k x k
  double* R = work + k * k;    // k x k
  double* Racc = work + 2 * k * k;
  double* fro2 = work + 3 * k * k;
  identity_kernel<<<g1(c, k * k), 256, 0, c->stream>>>(Racc, k);
  SKEMA_LAUNCHED(c);
  int passes_left = 2;
  bool shifted = false;
  // each pass writes Q R^{-1} into the other of the two buffers
  double* cur = Qm;
  double* nxt = work + 3 * k * k + 8;
  while (passes_left > 0) {
    // G = Q^T Q
    gram(c, cur, rows, rows, k, G);
    chol_inverse(c, G, k, R, G, dstatus);
    int st = 0;
    SKEMA_CUDA(cudaMemcpyAsync(&st, dstatus, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    SKEMA_CUDA(cudaStreamSynchronize(c->stream));
    if (st != 0) {
      if (shifted) {
        if (cur != Qm)
          SKEMA_CUDA(cudaMemcpyAsync(Qm, cur, sizeof(double) * (size_t)(rows * k), cudaMemcpyDeviceToDevice,
                                     c->stream));
        return false;
      }
      // shifted CholeskyQR: G + s I with s = 11 (rows*k + k(k+1)) u ||Q||_F^2
      gram(c, cur, rows, rows, k, G);
      trace_kernel<<<1, 256, 0, c->stream>>>(G, k, fro2);
      SKEMA_LAUNCHED(c);
      const double u = 1.1102230246251565e-16;
      shift_diag_kernel<<<(int)((k + 255) / 256), 256, 0, c->stream>>>(
          G, k, fro2, 11.0 * ((double)rows * k + (double)k * (k + 1)) * u);
      SKEMA_LAUNCHED(c);
      chol_inverse(c, G, k, R, G, dstatus);
      SKEMA_CUDA(cudaMemcpyAsync(&st, dstatus, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
      SKEMA_CUDA(cudaStreamSynchronize(c->stream));
      if (st != 0) {
        if (cur != Qm)
          SKEMA_CUDA(cudaMemcpyAsync(Qm, cur, sizeof(double) * (size_t)(rows * k), cudaMemcpyDeviceToDevice,
                                     c->stream));
        return false;
      }
      shifted = true;
      passes_left = 3;  // shifted pass + CholeskyQR2
    }
    // Q <- Q R^{-1} with G = R^{-1} (upper): next <- cur * Rinv (rows x k)
    tall_times_small(c, cur, rows, rows, k, G, k, k, nxt, rows, true);
    std::swap(cur, nxt);
    // Racc <- R * Racc
    double* tmp = Rout;
    dgemm<double, double>(c, k, k, k, 1.0, R, 1, k, Racc, 1, k, 0.0, tmp, 1, k, false);
    SKEMA_CUDA(cudaMemcpyAsync(Racc, tmp, sizeof(double) * (size_t)(k * k),
                               cudaMemcpyDeviceToDevice, c->stream));
    --passes_left;
  }
  if (cur != Qm)
    SKEMA_CUDA(cudaMemcpyAsync(Qm, cur, sizeof(double) * (size_t)(rows * k), cudaMemcpyDeviceToDevice, c->stream));
  SKEMA_CUDA(cudaMemcpyAsync(Rout, Racc, sizeof(double) * (size_t)(k * k), cudaMemcpyDeviceToDevice,
                             c->stream));
  return true;
}

void cholqr(skema_ctx* c, double* Qm, int64_t rows, int64_t k, double* Rout, double* work, int* dstatus) {
  if (!cholqr_try(c, Qm, rows, k, Rout, work, dstatus))
    fail(SKEMA_ENOTPD, "Cholesky of the Gram matrix failed after the shifted pass");
}

// 3 k^2 + 8 for cholqr's small matrices, rows x k for its second buffer,
// 3 k^2 + 8 more for orth's eigen-decomposition.
size_t cholqr_work_doubles(int64_t rows, int64_t k) { return (size_t)(6 * k * k + 16 + rows * k); }

// Uniform values on [-1, 1) from SplitMix64 (Steele, Lea and Flood, OOPSLA
// 2014) of (seed + index): the completion directions of orth.
__global__ void fill_uniform_kernel(double* __restrict__ W, int64_t cnt, uint64_t seed) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < cnt; q += (int64_t)gridDim.x * blockDim.x) {
    uint64_t z = seed + 0x9e3779b97f4a7c15ull * (uint64_t)(q + 1);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    z ^= z >> 31;
    W[q] = (double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
  }
}

// An orthonormal basis Q (rows x k, in place) whose first columns span the
// column space of the input, as dgeqrf + dorgqr give (src/Skema_SketchySVD.cpp:
// 355-357, 381-383) also for inputs of rank below k. CholeskyQR2 first; when
// the columns are numerically dependent, the eigen-decomposition of the
// Gram matrix gives the independent directions (eigenvalues above 1e-12 of
// the largest), which are orthonormalised, and the remaining columns are
// completed with pseudo-random directions orthogonalised against them twice
// (block Gram-Schmidt) and then among themselves. Householder QR completes
// the basis with other orthonormal columns of the same complement; the
// fixed-rank approximation does not depend on that choice beyond the rank
// of the sketch.
void orth(skema_ctx* c, double* Qm, int64_t rows, int64_t k, double* Rscratch, double* work, int* dstatus) {
  if (cholqr_try(c, Qm, rows, k, Rscratch, work, dstatus)) return;
  double* T = work + 3 * k * k + 8;              // rows x k
  double* G = T + rows * k;                      // k x k
  double* V = G + k * k;                         // k x k
  double* Vs = V + k * k;                        // k x k (sorted)
  double* Sv = Vs + k * k;                       // k
  double* sig = Sv + k;                          // k
  dgemm<double, double>(c, k, k, rows, 1.0, Qm, rows, 1, Qm, 1, rows, 0.0, G, 1, k);
  jacobi_svd(c, G, V, k, 60, 1e-15, dstatus + 1);
  // G V = U diag(lambda) with U = V for the symmetric positive semidefinite G
  svd_finish_kernel<<<1, 256, 0, c->stream>>>(G, V, k, Rscratch /*U, unused*/, Vs, Sv, sig);
  SKEMA_LAUNCHED(c);
  std::vector<double> lam(k), vs((size_t)(k * k));
  SKEMA_CUDA(cudaMemcpyAsync(lam.data(), Sv, sizeof(double) * (size_t)k, cudaMemcpyDeviceToHost, c->stream));
  SKEMA_CUDA(cudaMemcpyAsync(vs.data(), Vs, sizeof(double) * (size_t)(k * k), cudaMemcpyDeviceToHost, c->stream));
  SKEMA_CUDA(cudaStreamSynchronize(c->stream));
  int64_t r = 0;
  while (r < k && lam[r] > 1e-12 * lam[0]) ++r;
  if (r == 0) fail(SKEMA_ENOTPD, "the sketch is zero: no direction to orthonormalise");
  // B = V_r diag(lambda_r^-1/2): Q V_r B has orthonormal columns up to rounding
  for (int64_t j = 0; j < r; ++j) {
    const double sc = 1.0 / std::sqrt(lam[j]);
    for (int64_t i = 0; i < k; ++i) vs[i + j * k] *= sc;
  }
  SKEMA_CUDA(cudaMemcpyAsync(G, vs.data(), sizeof(double) * (size_t)(k * r), cudaMemcpyHostToDevice, c->stream));
  dgemm<double, double>(c, rows, r, k, 1.0, Qm, 1, rows, G, 1, k, 0.0, T, 1, rows, false);
  SKEMA_CUDA(cudaMemcpyAsync(Qm, T, sizeof(double) * (size_t)(rows * r), cudaMemcpyDeviceToDevice, c->stream));
  // stream order keeps the host vectors' copies complete before they go out of scope
  SKEMA_CUDA(cudaStreamSynchronize(c->stream));
  cholqr(c, Qm, rows, r, Rscratch, work, dstatus);  // well conditioned now
  if (r == k) return;
  double* W = Qm + r * rows;  // columns r .. k-1
  const int64_t kr = k - r;
  fill_uniform_kernel<<<g1(c, rows * kr), 256, 0, c->stream>>>(W, rows * kr, 0x5eed5eedull + (uint64_t)k);
  SKEMA_LAUNCHED(c);
  for (int pass = 0; pass < 2; ++pass) {
    // W <- W - Q2 (Q2^T W)
    dgemm<double, double>(c, r, kr, rows, 1.0, Qm, rows, 1, W, 1, rows, 0.0, G, 1, r);
    dgemm<double, double>(c, rows, kr, r, -1.0, Qm, 1, rows, G, 1, r, 1.0, W, 1, rows, false);
  }
  cholqr(c, W, rows, kr, Rscratch, work, dstatus);
}

// In-place sum over the ranks of a row-block sharded sketch (device
// memory, after the context's stream has finished writing it), through the
// caller's all-reduce; nothing for a single context.
struct RankSum {
  skema_allreduce_fn fn = nullptr;
  void* user = nullptr;
  bool on() const { return fn != nullptr; }
  void operator()(skema_ctx* c, double* buf, int64_t count) const {
    if (!fn) return;
    SKEMA_CUDA(cudaStreamSynchronize(c->stream));
    if (fn(buf, count, user) != 0) fail(SKEMA_ECOLLECTIVE, "the all-reduce callback reported a failure");
  }
};

// The orthonormal basis of orth() for the FP32 sketch S (rows x k,
// column-major ld lds), left as Qm Tout with Tout upper triangular (k x k):
// the first CholeskyQR pass reads S itself (its products are exact in
// FP64) and writes Qm = S R1^{-1}; the second pass only factors
// Qm^T Qm = R2^T R2 and returns Tout = R2^{-1}, so the last product with
// the tall matrix is folded by the caller into the small matrices it
// multiplies the basis by anyway. When a Cholesky factor does not exist,
// orth() makes the basis explicit in Qm from the FP64 matrix at hand and
// Tout = I. With a rank sum, S is this rank's row block of a sharded
// sketch: both Gram matrices are summed over the ranks before their
// Cholesky, Qm is the block's rows of the basis, and a missing factor
// fails (SKEMA_ENOTPD) on every rank alike, since the explicit fallback
// needs the whole matrix.
void orth_lazy(skema_ctx* c, const float* S, int64_t lds, double* Qm, int64_t rows, int64_t k, double* Tout,
               double* Rscratch, double* work, int* dstatus, const RankSum& rsum = RankSum{}) {
  double* G = work;
  double* R = work + k * k;
  auto factor = [&] {
    chol_inverse(c, G, k, R, G, dstatus);
    int st = 0;
    SKEMA_CUDA(cudaMemcpyAsync(&st, dstatus, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    SKEMA_CUDA(cudaStreamSynchronize(c->stream));
    return st == 0;
  };
  auto explicit_basis = [&] {
    if (rsum.on())
      fail(SKEMA_ENOTPD, "the sharded sketch is rank deficient: CholeskyQR needs full column rank");
    orth(c, Qm, rows, k, Rscratch, work, dstatus);
    identity_kernel<<<g1(c, k * k), 256, 0, c->stream>>>(Tout, k);
    SKEMA_LAUNCHED(c);
  };
  if (k <= kTallMaxK || rows <= 0) {
    gram_t<float>(c, S, lds, rows, k, G);
  } else {
    dgemm<float, float>(c, k, k, rows, 1.0, S, lds, 1, S, 1, lds, 0.0, G, 1, k);
  }
  rsum(c, G, k * k);
  if (!factor()) {
    f2d_kernel<<<g1(c, rows * k), 256, 0, c->stream>>>(S, 1, lds, Qm, 1, rows, rows, k);
    SKEMA_LAUNCHED(c);
    explicit_basis();
    return;
  }
  // Qm = S R1^{-1} (G holds R1^{-1})
  if (rows <= 0) {
  } else if (k <= kTallMaxK) {
    tall_times_small_t<float>(c, S, lds, rows, k, G, k, k, Qm, rows, true);
  } else {
    dgemm<float, double>(c, rows, k, k, 1.0, S, 1, lds, G, 1, k, 0.0, Qm, 1, rows, false);
  }
  gram(c, Qm, rows, rows, k, G);
  rsum(c, G, k * k);
  if (!factor()) {
    explicit_basis();
    return;
  }
  SKEMA_CUDA(cudaMemcpyAsync(Tout, G, sizeof(double) * (size_t)(k * k), cudaMemcpyDeviceToDevice, c->stream));
}

// out (R x k, column-major ld R) = Map~ (R x cols) * Qm (cols x k, column-major ld cols)
// out (R x k, column-major) = M Q for the map's logical R x cols matrix M
// and rows [q0, q0 + qrows) of Q held in Qm (column-major, ld qrows): the
// block's share of M Q, which sums over the row blocks to the whole.
void apply_map_rows(skema_ctx* c, const Map& mp, const double* Qm, int64_t q0, int64_t qrows, int64_t k,
                    double* out) {
  const int64_t R = mp.lrows;
  if (qrows <= 0) {
    SKEMA_CUDA(cudaMemsetAsync(out, 0, sizeof(double) * (size_t)(R * k), c->stream));
    return;
  }
  if (mp.kind == SKEMA_MAP_GAUSS) {
    if (mp.cs == 1 && R <= kTallMaxK * 4 && k <= kTallMaxK) {
      // M(:, rows) Q = (M(:, rows)^T)^T Q: the map's logical rows are
      // contiguous over the operand's rows, a tall column-major matrix
      SKEMA_CUDA(cudaMemsetAsync(out, 0, sizeof(double) * (size_t)(R * k), c->stream));
      launch_atb_mma<float, double>(c, mp.f32 + q0, mp.rs, R, Qm, qrows, k, qrows, out);
      return;
    }
    dgemm<float, double>(c, R, k, qrows, 1.0, mp.f32 + q0 * mp.cs, mp.rs, mp.cs, Qm, 1, qrows, 0.0, out, 1, R);
    return;
  }
  if (!mp.transposed) {
    rowsparse_apply_kernel<<<g1(c, R * k), 256, 0, c->stream>>>(mp.packed, mp.zeta, R, Qm, qrows, k, out, R, q0,
                                                                 qrows);
    SKEMA_LAUNCHED(c);
  } else {
    // stored rows are the operand's rows: the block's stored rows only
    const uint32_t* mpb = mp.packed + q0 * mp.zeta;
    SKEMA_CUDA(cudaMemsetAsync(out, 0, sizeof(double) * (size_t)(R * k), c->stream));
    const size_t priv = sizeof(double) * (size_t)(R * k);
    if (priv <= 200 * 1024) {
      SKEMA_CUDA(cudaFuncSetAttribute(colsparse_apply_smem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)priv));
      colsparse_apply_smem_kernel<<<c->sm_count, 1024, priv, c->stream>>>(mpb, mp.zeta, qrows, Qm, qrows, k, out,
                                                                            R, R);
    } else {
      colsparse_apply_kernel<<<g1(c, qrows * k), 256, 0, c->stream>>>(mpb, mp.zeta, qrows, Qm, qrows, k, out, R);
    }
    SKEMA_LAUNCHED(c);
  }
}

void apply_map(skema_ctx* c, const Map& mp, const double* Qm, int64_t cols, int64_t k, double* out) {
  apply_map_rows(c, mp, Qm, 0, cols, k, out);
}

// ---- SketchySPD pieces -----------------------------------------------------
// Stored SparseSign rows (zeta entries: column | sign << 31) -> dense n x k
// (column-major, ld n, zeroed beforehand); duplicate entries add up.
__global__ void ssign_dense_kernel(const uint32_t* __restrict__ packed, int zeta, int64_t n, double* __restrict__ D) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    for (int t = 0; t < zeta; ++t) {
      const uint32_t w = packed[i * zeta + t];
      D[i + (int64_t)(w & 0x7fffffffu) * n] += (w >> 31) ? -1.0 : 1.0;
    }
}
// SparseSignDimRedux::axpy as the reference runs it (`*=`): each stored entry
// multiplies its Y entry by eta * sign, a duplicate entry twice.
__global__ void ssign_scale_kernel(const uint32_t* __restrict__ packed, int zeta, int64_t n, double* __restrict__ Y,
                                   int64_t ldy, double eta) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    for (int t = 0; t < zeta; ++t) {
      const uint32_t w = packed[i * zeta + t];
      Y[i + (int64_t)(w & 0x7fffffffu) * ldy] *= eta * ((w >> 31) ? -1.0 : 1.0);
    }
}
__global__ void daxpy_kernel(double* __restrict__ Y, const double* __restrict__ X, int64_t cnt, double a) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < cnt; q += (int64_t)gridDim.x * blockDim.x)
    Y[q] += a * X[q];
}
// C = (B + B^T) / 2, column-major k x k.
__global__ void symmetrize_kernel(const double* __restrict__ B, double* __restrict__ C, int64_t k) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < k * k; q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = q % k, j = q / k;
    C[q] = 0.5 * (B[i + j * k] + B[j + i * k]);
  }
}
// out_j = max(0, S_j^2 - sub): squared singular values of E less the shift.
__global__ void spd_eig_kernel(const double* __restrict__ S, double* __restrict__ out, int64_t r, double sub) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < r; j += (int64_t)gridDim.x * blockDim.x)
    out[j] = fmax(0.0, S[j] * S[j] - sub);
}

}  // namespace

// SketchySPD::low_rank_approx (src/Skema_SketchySVD.cpp:935-1151) in FP64 on
// the device, with Omega the stored n x k map and Y the m x k sketch (m = n):
//   nu = ||Y||_2 (from the largest eigenvalue of Y^T Y), eta = eps nu (below)
//   Y_eta = Y + eta Omega   (REFERENCE_STEPS with SparseSign: each stored map
//                            entry multiplies its Y entry by eta * sign)
//   B = Omega^T Y_eta, R^T R = (B + B^T) / 2 (upper Cholesky, as dpotrf 'U')
//   E = Y_eta R^{-1}        (REFERENCE_STEPS: the unshifted Y, :1094-1103)
//   U S V^T = svd(E)        (CholeskyQR2 of E, then a Jacobi SVD of its R)
//   U <- U(:, 1:r), S_j <- max(0, S_j^2 - eta)   (REFERENCE_STEPS: - nu)
// The reference takes eta from the norm of a buffer dgesvd has already
// overwritten (:964-965), a value that depends on the LAPACK build; its
// steps here use eps ||Y||_2, the value its comment states, which enters at
// the level of eps. The Nystrom form shifts by the FP32 epsilon times
// ||Y||_2, because Y is held in FP32: a shift below the rounding of Y leaves
// B indefinite for spectra that decay to zero.
void spd_low_rank_approx(skema_ctx* c, double* Uout, double* Sout) {
  const int64_t m = c->m, n = c->n, k = c->k, r = c->p.rank;
  const bool ref_steps = c->p.spd_approx == SKEMA_SPD_REFERENCE_STEPS;
  const Map& O = c->omg;
  y_materialize(c);
  const size_t b_mk = sizeof(double) * (size_t)(m * k), b_nk = sizeof(double) * (size_t)(n * k);
  const size_t b_w = sizeof(double) * cholqr_work_doubles(m, k);
  const size_t b_small = sizeof(double) * (size_t)(8 * k * k + 4 * k + 64);
  Carve cv(c, {b_mk, b_mk, b_nk, b_w, b_small, 16});
  double* Yd = cv.take(b_mk);
  double* Ye = cv.take(b_mk);
  double* Od = cv.take(b_nk);
  double* W = cv.take(b_w);
  double* G = cv.take(b_small);  // k x k
  double* R = G + k * k;        // k x k
  double* Rinv = R + k * k;     // k x k
  double* Cw = Rinv + k * k;    // k x k
  double* Vc = Cw + k * k;      // k x k
  double* Uc = Vc + k * k;      // k x k
  double* Vt = Uc + k * k;      // k x k
  double* RE = Vt + k * k;      // k x k
  double* Sv = RE + k * k;      // k
  double* sig = Sv + k;         // k
  int* st = reinterpret_cast<int*>(cv.take(16));

  f2d_kernel<<<g1(c, m * k), 256, 0, c->stream>>>(c->Y, 1, m, Yd, 1, m, m, k);
  SKEMA_LAUNCHED(c);
  if (O.kind == SKEMA_MAP_GAUSS) {
    // stored (i, j) = logical (j, i)
    f2d_kernel<<<g1(c, n * k), 256, 0, c->stream>>>(O.f32, O.cs, O.rs, Od, 1, n, n, k);
  } else {
    SKEMA_CUDA(cudaMemsetAsync(Od, 0, sizeof(double) * (size_t)(n * k), c->stream));
    ssign_dense_kernel<<<g1(c, n), 256, 0, c->stream>>>(O.packed, O.zeta, n, Od);
  }
  SKEMA_LAUNCHED(c);

  // nu = ||Y||_2 = sqrt(lambda_max(Y^T Y))
  dgemm<double, double>(c, k, k, m, 1.0, Yd, m, 1, Yd, 1, m, 0.0, G, 1, k);
  jacobi_svd(c, G, Vc, k, 60, 1e-15, st + 1);
  svd_finish_kernel<<<1, 256, 0, c->stream>>>(G, Vc, k, Uc, Vt, Sv, sig);
  SKEMA_LAUNCHED(c);
  double lmax = 0.0;
  SKEMA_CUDA(cudaMemcpyAsync(&lmax, Sv, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  SKEMA_CUDA(cudaStreamSynchronize(c->stream));
  const double nu = std::sqrt(std::max(lmax, 0.0));
  // the Nystrom shift covers the rounding of Y, which is held in FP32 here
  // (the reference holds Y in FP64 and shifts by the FP64 epsilon)
  const double eta =
      (ref_steps ? std::numeric_limits<double>::epsilon() : (double)std::numeric_limits<float>::epsilon()) * nu;

  // Y_eta
  SKEMA_CUDA(cudaMemcpyAsync(Ye, Yd, sizeof(double) * (size_t)(m * k), cudaMemcpyDeviceToDevice, c->stream));
  if (ref_steps && O.kind == SKEMA_MAP_SPARSE_SIGN) {
    ssign_scale_kernel<<<g1(c, n), 256, 0, c->stream>>>(O.packed, O.zeta, n, Ye, m, eta);
  } else {
    daxpy_kernel<<<g1(c, m * k), 256, 0, c->stream>>>(Ye, Od, m * k, eta);
  }
  SKEMA_LAUNCHED(c);
  // B = Omega^T Y_eta; R^T R = (B + B^T) / 2
  dgemm<double, double>(c, k, k, n, 1.0, Od, n, 1, Ye, 1, m, 0.0, Cw, 1, k);
  symmetrize_kernel<<<g1(c, k * k), 256, 0, c->stream>>>(Cw, G, k);
  SKEMA_LAUNCHED(c);
  chol_inverse(c, G, k, R, Rinv, st);
  int bad = 0;
  SKEMA_CUDA(cudaMemcpyAsync(&bad, st, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  SKEMA_CUDA(cudaStreamSynchronize(c->stream));
  if (bad != 0) fail(SKEMA_ENOTPD, "SketchySPD: (B + B^T) / 2 is not positive definite (dpotrf would fail)");
  // E = (Y_eta or Y) R^{-1}, into Yd's buffer when it is no longer needed
  double* E = ref_steps ? Ye : Yd;
  const double* src = ref_steps ? Yd : Ye;
  dgemm<double, double>(c, m, k, k, 1.0, src, 1, m, Rinv, 1, k, 0.0, E, 1, m, false);
  // svd(E) = Q svd(R_E)
  cholqr(c, E, m, k, RE, W, st);
  SKEMA_CUDA(cudaMemcpyAsync(Cw, RE, sizeof(double) * (size_t)(k * k), cudaMemcpyDeviceToDevice, c->stream));
  jacobi_svd(c, Cw, Vc, k, 60, 1e-15, st + 1);
  svd_finish_kernel<<<1, 256, 0, c->stream>>>(Cw, Vc, k, Uc, Vt, Sv, sig);
  SKEMA_LAUNCHED(c);
  if (Uout) dgemm<double, double>(c, m, r, k, 1.0, E, 1, m, Uc, 1, k, 0.0, Uout, 1, m, false);
  if (Sout) {
    spd_eig_kernel<<<1, 256, 0, c->stream>>>(Sv, Sout, r, ref_steps ? nu : eta);
    SKEMA_LAUNCHED(c);
  }
  SKEMA_CUDA(cudaStreamSynchronize(c->stream));
}

void dgemm_f32_f64(skema_ctx* c, int64_t M, int64_t N, int64_t K, double alpha, const float* A, int64_t ars,
                   int64_t acs, const double* B, int64_t brs, int64_t bcs, double beta, double* C, int64_t crs,
                   int64_t ccs) {
  dgemm<float, double>(c, M, N, K, alpha, A, ars, acs, B, brs, bcs, beta, C, crs, ccs);
}

// The fixed-rank approximation from Y's rows [row0, row0 + nrows) with
// the sums over row blocks taken by rsum (a row-block sharded sketch whose
// X and Z are already summed), or from all of Y (rsum off, the whole
// range). U (nrows x rank, column-major ld nrows) gets the block's rows.
void low_rank_approx_rows(skema_ctx* c, int64_t row0, int64_t nrows, const RankSum& rsum, double* Uout,
                          double* Sout, double* Vout) {
  const int64_t m = nrows, n = c->n, k = c->k, s = c->s, r = c->p.rank;
  y_materialize(c);
  const size_t b_q = sizeof(double) * (size_t)(m * k), b_p = sizeof(double) * (size_t)(n * k);
  const size_t b_w = sizeof(double) * cholqr_work_doubles(std::max(m, std::max(n, s)), k);
  const size_t b_u = sizeof(double) * (size_t)(s * k);
  const size_t b_small = sizeof(double) * (size_t)(12 * k * k + s * s + k * s + 4 * k + 64);
  Carve cv(c, {b_q, b_p, b_w, b_u, b_u, b_small, 16});
  double* Q = cv.take(b_q);
  double* P = cv.take(b_p);
  double* W = cv.take(b_w);
  double* U1 = cv.take(b_u);
  double* U2 = cv.take(b_u);
  double* T1 = cv.take(b_small);
  double* T2 = T1 + k * k;
  double* Z1 = T2 + k * k;         // k x s
  double* Z2 = Z1 + k * s;         // k x k
  double* Z2t = Z2 + k * k;        // k x k
  double* Uc = Z2t + k * k;        // k x k
  double* Vc = Uc + k * k;         // k x k
  double* Sv = Vc + k * k;         // k
  double* sig = Sv + k;            // k
  double* Zd = sig + k;            // s x s
  double* TQ = Zd + s * s;         // k x k: the basis of Y is Q TQ
  double* TP = TQ + k * k;         // k x k: the basis of X^T is P TP
  double* WU = TP + k * k;         // k x r
  double* WV = WU + k * k;         // k x r
  int* st = reinterpret_cast<int*>(cv.take(16));

  auto orth_scope = std::make_unique<StageScope>(c, ST_A_ORTH);
  f2d_kernel<<<g1(c, s * s), 256, 0, c->stream>>>(c->Z, s, 1, Zd, 1, s, s, s);
  SKEMA_LAUNCHED(c);
  // bases of Y (m x k, column-major) and X^T (n x k: X is k x n row-major),
  // as Q TQ and P TP
  orth_lazy(c, c->X, n, P, n, k, TP, T1, W, st);  // T1 used as scratch R here
  orth_lazy(c, c->Y + row0, c->m, Q, m, k, TQ, T1, W, st, rsum);
  orth_scope.reset();
  auto core_scope = std::make_unique<StageScope>(c, ST_A_CORE);
  // U1 = Phi~ Q TQ (s x k), U2 = Psi~ P TP (s x k); W holds Phi~ Q, Psi~ P
  apply_map_rows(c, c->phi, Q, row0, m, k, W);
  rsum(c, W, s * k);
  tall_times_small(c, W, s, s, k, TQ, k, k, U1, s, true);
  apply_map(c, c->psi, P, n, k, W);
  tall_times_small(c, W, s, s, k, TP, k, k, U2, s, true);
  cholqr(c, U1, s, k, T1, W, st);
  cholqr(c, U2, s, k, T2, W, st);
  // Z1 = U1^T Z (k x s); Z2 = Z1 U2 (k x k)
  dgemm<double, double>(c, k, s, s, 1.0, U1, s, 1, Zd, 1, s, 0.0, Z1, 1, k);
  dgemm<double, double>(c, k, k, s, 1.0, Z1, 1, k, U2, 1, s, 0.0, Z2, 1, k);
  // Z2 = T1 \ Z2
  trsm_upper(c, T1, k, Z2, k, k);
  // C^T = T2 \ Z2^T
  dtranspose_kernel<<<g1(c, k * k), 256, 0, c->stream>>>(Z2, Z2t, k);
  SKEMA_LAUNCHED(c);
  trsm_upper(c, T2, k, Z2t, k, k);
  // C = (Z2t)^T: copy into Uc's slot as the Jacobi working matrix
  double* C = Uc;
  core_scope.reset();
  {
    StageScope sc(c, ST_A_SVD);
    double* Cw = W;  // k x k working copy
    dtranspose_kernel<<<g1(c, k * k), 256, 0, c->stream>>>(Z2t, Cw, k);
    SKEMA_LAUNCHED(c);
    jacobi_svd(c, Cw, Vc, k, 60, 1e-15, st + 1);
    svd_finish_kernel<<<1, 256, 0, c->stream>>>(Cw, Vc, k, C, Z2 /*Vout*/, Sv, sig);
    SKEMA_LAUNCHED(c);
  }
  {
    StageScope sc(c, ST_A_VECTORS);
    // U = Q TQ Uc(:, 1:r), V = P TP Vc(:, 1:r), S = S(1:r)
    if (Uout) {
      tall_times_small(c, TQ, k, k, k, C, k, r, WU, k);
      tall_times_small(c, Q, m, m, k, WU, k, r, Uout, m);
    }
    if (Vout) {
      tall_times_small(c, TP, k, k, k, Z2, k, r, WV, k);
      tall_times_small(c, P, n, n, k, WV, k, r, Vout, n);
    }
    if (Sout)
      SKEMA_CUDA(cudaMemcpyAsync(Sout, Sv, sizeof(double) * (size_t)r, cudaMemcpyDeviceToDevice, c->stream));
  }
  int sweeps = 0;
  SKEMA_CUDA(cudaMemcpyAsync(&sweeps, st + 1, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  SKEMA_CUDA(cudaStreamSynchronize(c->stream));
  c->svd_sweeps = sweeps;
}

void low_rank_approx(skema_ctx* c, double* Uout, double* Sout, double* Vout) {
  low_rank_approx_rows(c, 0, c->m, RankSum{}, Uout, Sout, Vout);
}

void low_rank_approx_sharded(skema_ctx* c, int64_t row0, int64_t nrows, skema_allreduce_fn fn, void* user,
                             double* Uout, double* Sout, double* Vout) {
  RankSum rs;
  rs.fn = fn;
  rs.user = user;
  low_rank_approx_rows(c, row0, nrows, rs, Uout, Sout, Vout);
}

}  // namespace skema
