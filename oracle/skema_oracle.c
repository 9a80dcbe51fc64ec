/*
 * skema_oracle.c -- TEST INFRASTRUCTURE ONLY. CPU restatement of the
 * reference's SketchySVD sketch path, used as the checker for the CUDA
 * library (tests, smoke check and the CPU baseline of the benchmark). The
 * product library never links, loads or calls this file.
 *
 * What is restated here (integer-exact or FP64 parts):
 *   - Philox4x32-10 (Salmon et al., SC'11), written independently of the
 *     library's philox.h so that the two implementations check each other;
 *   - the map entry formulas: Gauss entries uniform on [-maxval, maxval),
 *     maxval = sqrt(2 ln(nrow*ncol)) (src/Skema_DimRedux.hpp:112,115), and
 *     SparseSign rows of zeta = max(2,min(ncol,8)) sorted indices drawn with
 *     replacement plus +-1 values (src/Skema_DimRedux.hpp:205-251);
 *   - the CRS x SparseSign update (src/Skema_SketchySVD.cpp:319-335 with
 *     src/Skema_DimRedux_SparseSign.cpp:53-111, 125-155) as a Gustavson
 *     sparse product in FP64, and the dense x SparseSign products
 *     (src/Skema_DimRedux_SparseSign.cpp:9-51);
 *   - the Gauss RBF kernel window with explicit differences and the forced
 *     unit diagonal (src/Skema_Kernel.cpp:6-81).
 * The dense FP64 GEMM/LAPACK parts live in oracle/sketchy_oracle.py (numpy
 * and scipy LAPACK, the routines the reference calls).
 *
 * Build: oracle/Makefile (gcc -O2 -fopenmp -shared).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

/* ---------------- Philox4x32-10 ---------------------------------------- */
static void ph_round(uint32_t ctr[4], const uint32_t key[2]) {
  uint64_t p0 = (uint64_t)0xD2511F53u * ctr[0];
  uint64_t p1 = (uint64_t)0xCD9E8D57u * ctr[2];
  uint32_t out0 = (uint32_t)(p1 >> 32) ^ ctr[1] ^ key[0];
  uint32_t out1 = (uint32_t)p1;
  uint32_t out2 = (uint32_t)(p0 >> 32) ^ ctr[3] ^ key[1];
  uint32_t out3 = (uint32_t)p0;
  ctr[0] = out0;
  ctr[1] = out1;
  ctr[2] = out2;
  ctr[3] = out3;
}

void oracle_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2],
                          uint32_t out[4]) {
  uint32_t ctr[4] = {ctr_in[0], ctr_in[1], ctr_in[2], ctr_in[3]};
  uint32_t key[2] = {key_in[0], key_in[1]};
  int r;
  for (r = 0; r < 10; ++r) {
    if (r > 0) {
      key[0] += 0x9E3779B9u;
      key[1] += 0xBB67AE85u;
    }
    ph_round(ctr, key);
  }
  memcpy(out, ctr, sizeof(ctr));
}

#define KEY1 0x534B454Du
#define TAG_GAUSS 0x47415553u
#define TAG_SSIGN 0x53534731u

/* Gauss map entry e = i + j*nrow of an nrow x ncol map. */
static double gauss_value(uint32_t seed, uint64_t e, double maxval) {
  uint64_t blk = e / 2;
  uint32_t ctr[4] = {(uint32_t)(blk & 0xffffffffu), (uint32_t)(blk >> 32),
                     TAG_GAUSS, 0u};
  uint32_t key[2] = {seed, KEY1};
  uint32_t o[4];
  uint64_t hi, lo, bits;
  int64_t b, c;
  oracle_philox4x32_10(ctr, key, o);
  if (e % 2 == 0) {
    hi = o[0];
    lo = o[1];
  } else {
    hi = o[2];
    lo = o[3];
  }
  bits = (hi << 32) | lo;
  b = (int64_t)(bits >> 11);
  c = 2 * b - ((int64_t)1 << 53);
  return maxval * ldexp((double)c, -53);
}

double oracle_gauss_maxval(int64_t nrow, int64_t ncol) {
  /* GaussDimRedux: maxval = sqrt(2 * log(nrow * ncol)) with size_t product
   * (src/Skema_DimRedux.hpp:112). */
  return sqrt(2.0 * log((double)((uint64_t)nrow * (uint64_t)ncol)));
}

/* Fill a column-major nrow x ncol Gauss map (double). */
void oracle_gauss_map(uint32_t seed, int64_t nrow, int64_t ncol, double* out) {
  double maxval = oracle_gauss_maxval(nrow, ncol);
  int64_t total = nrow * ncol;
  int64_t e;
#pragma omp parallel for schedule(static)
  for (e = 0; e < total; ++e) out[e] = gauss_value(seed, (uint64_t)e, maxval);
}

int oracle_zeta(int64_t ncol) {
  int64_t z = ncol < 8 ? ncol : 8;
  return (int)(z < 2 ? 2 : z);
}

static int cmp_u32(const void* a, const void* b) {
  uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
  return (x > y) - (x < y);
}

/* SparseSign map: nrow stored rows, zeta entries each over [0,ncol).
 * idx[r*zeta + t] sorted ascending within a row; val = +-1.0. */
void oracle_sparse_sign_map(uint32_t seed, int64_t nrow, int64_t ncol,
                            int32_t* idx, double* val) {
  int zeta = oracle_zeta(ncol);
  int64_t r;
#pragma omp parallel for schedule(static)
  for (r = 0; r < nrow; ++r) {
    uint32_t key[2] = {seed, KEY1};
    uint32_t c0[4] = {(uint32_t)((uint64_t)r & 0xffffffffu),
                      (uint32_t)((uint64_t)r >> 32), TAG_SSIGN, 0u};
    uint32_t c1[4] = {c0[0], c0[1], TAG_SSIGN, 1u};
    uint32_t c2[4] = {c0[0], c0[1], TAG_SSIGN, 2u};
    uint32_t a[4], b[4], s[4], draws[8], sorted[8];
    int t;
    oracle_philox4x32_10(c0, key, a);
    oracle_philox4x32_10(c1, key, b);
    oracle_philox4x32_10(c2, key, s);
    memcpy(draws, a, sizeof(a));
    memcpy(draws + 4, b, sizeof(b));
    for (t = 0; t < zeta; ++t)
      sorted[t] = (uint32_t)(((uint64_t)draws[t] * (uint64_t)ncol) >> 32);
    qsort(sorted, (size_t)zeta, sizeof(uint32_t), cmp_u32);
    for (t = 0; t < zeta; ++t) {
      idx[r * zeta + t] = (int32_t)sorted[t];
      val[r * zeta + t] = ((s[0] >> t) & 1u) ? -1.0 : 1.0;
    }
  }
}

/* ---------------- CRS x SparseSign update (one window) ------------------
 * Inputs: the CRS window rows [0,w) (rowptr relative, w+1 entries), the
 * window's absolute first row `row0`, matrix dims m x n.
 * Maps: Upsilon (k x m, zeta_u per row), Phi (s x m), both row-sparse over m;
 *       Omega stored n x k and Psi stored n x s (init_transposed, zeta per
 *       stored row over k / s).
 * Outputs (FP64, overwritten): x (k x n, row-major), y (w x k, row-major),
 *       z (s x s, row-major).
 * Follows update(crs, SparseSign) (src/Skema_SketchySVD.cpp:319-335):
 *   x = Upsilon(:,idx) * A_w    (col_subview + spgemm + densify)
 *   y = A_w * Omega             (spgemm)
 *   w = Phi(:,idx) * A_w
 *   z = w * Psi                 (dense x sparse)
 */
void oracle_csr_sparse_sign_window(
    int64_t m, int64_t n, int64_t row0, int64_t w, const int64_t* rowptr,
    const int32_t* col, const double* val, int64_t k, int64_t s,
    const int32_t* ups_idx, const double* ups_val, int zeta_u,
    const int32_t* omg_idx, const double* omg_val, int zeta_o,
    const int32_t* phi_idx, const double* phi_val, int zeta_p,
    const int32_t* psi_idx, const double* psi_val, int zeta_s, double* x,
    double* y, double* z) {
  int64_t i, r;
  (void)m;
  memset(x, 0, sizeof(double) * (size_t)(k * n));
  memset(y, 0, sizeof(double) * (size_t)(w * k));
  memset(z, 0, sizeof(double) * (size_t)(s * s));
  /* y = A_w * Omega (row i of A_w times the n x k stored map). */
#pragma omp parallel for schedule(dynamic, 256)
  for (i = 0; i < w; ++i) {
    int64_t p;
    for (p = rowptr[i] - rowptr[0]; p < rowptr[i + 1] - rowptr[0]; ++p) {
      int64_t j = col[p];
      int t;
      for (t = 0; t < zeta_o; ++t)
        y[i * k + omg_idx[j * zeta_o + t]] += val[p] * omg_val[j * zeta_o + t];
    }
  }
  /* x = Upsilon(:, idx) * A_w : row r gathers the A rows its entries hit. */
#pragma omp parallel for schedule(dynamic, 4)
  for (r = 0; r < k; ++r) {
    int t;
    for (t = 0; t < zeta_u; ++t) {
      int64_t c = ups_idx[r * zeta_u + t];
      if (c >= row0 && c < row0 + w) {
        int64_t li = c - row0, p;
        for (p = rowptr[li] - rowptr[0]; p < rowptr[li + 1] - rowptr[0]; ++p)
          x[r * n + col[p]] += ups_val[r * zeta_u + t] * val[p];
      }
    }
  }
  /* w = Phi(:, idx) * A_w (sparse rows), then z = w * Psi. */
#pragma omp parallel for schedule(dynamic, 4)
  for (r = 0; r < s; ++r) {
    double* wrow = (double*)calloc((size_t)n, sizeof(double));
    unsigned char* touched = (unsigned char*)calloc((size_t)n, 1);
    int64_t* list = (int64_t*)malloc(sizeof(int64_t) * 64);
    int64_t nlist = 0, cap = 64, q;
    int t;
    for (t = 0; t < zeta_p; ++t) {
      int64_t c = phi_idx[r * zeta_p + t];
      if (c >= row0 && c < row0 + w) {
        int64_t li = c - row0, p;
        for (p = rowptr[li] - rowptr[0]; p < rowptr[li + 1] - rowptr[0]; ++p) {
          int64_t j = col[p];
          wrow[j] += phi_val[r * zeta_p + t] * val[p];
          if (!touched[j]) {
            touched[j] = 1;
            if (nlist == cap) {
              cap *= 2;
              list = (int64_t*)realloc(list, sizeof(int64_t) * (size_t)cap);
            }
            list[nlist++] = j;
          }
        }
      }
    }
    for (q = 0; q < nlist; ++q) {
      int64_t j = list[q];
      int u;
      for (u = 0; u < zeta_s; ++u)
        z[r * s + psi_idx[j * zeta_s + u]] += wrow[j] * psi_val[j * zeta_s + u];
    }
    free(list);
    free(touched);
    free(wrow);
  }
}

/* y = A_w * Omega for a CRS window only (the dominant term; used by the
 * timed CPU baseline on a row sample). */
void oracle_csr_sparse_sign_y(int64_t w, const int64_t* rowptr,
                              const int32_t* col, const double* val, int64_t k,
                              const int32_t* omg_idx, const double* omg_val,
                              int zeta_o, double* y) {
  int64_t i;
#pragma omp parallel for schedule(dynamic, 256)
  for (i = 0; i < w; ++i) {
    int64_t p;
    memset(y + i * k, 0, sizeof(double) * (size_t)k);
    for (p = rowptr[i] - rowptr[0]; p < rowptr[i + 1] - rowptr[0]; ++p) {
      int64_t j = col[p];
      int t;
      for (t = 0; t < zeta_o; ++t)
        y[i * k + omg_idx[j * zeta_o + t]] += val[p] * omg_val[j * zeta_o + t];
    }
  }
}

/* ---------------- dense x SparseSign products ---------------------------
 * M is a row-sparse map R x C (zeta per row over C). B is dense C x N,
 * column-major with leading dimension ldb, restricted to columns [c0,c0+cw)
 * of M (col_subview, src/Skema_DimRedux_SparseSign.cpp:125-155):
 *   out (R x N, row-major) = M(:, c0:c0+cw) * B
 */
void oracle_rowsparse_times_dense(int64_t R, int zeta, const int32_t* idx,
                                  const double* v, int64_t c0, int64_t cw,
                                  const double* B, int64_t ldb, int64_t N,
                                  double* out) {
  int64_t r;
#pragma omp parallel for schedule(static)
  for (r = 0; r < R; ++r) {
    int64_t j;
    int t;
    for (j = 0; j < N; ++j) out[r * N + j] = 0.0;
    for (t = 0; t < zeta; ++t) {
      int64_t c = idx[r * zeta + t];
      if (c >= c0 && c < c0 + cw) {
        for (j = 0; j < N; ++j) out[r * N + j] += v[r * zeta + t] * B[(c - c0) + j * ldb];
      }
    }
  }
}

/* out (W x R, row-major) = B * M^T where B is W x C column-major (ldb) and
 * M is row-sparse R x C: out(i, r) = sum_t M(r, c_t) B(i, c_t). */
void oracle_dense_times_rowsparse_t(int64_t W, const double* B, int64_t ldb,
                                    int64_t R, int zeta, const int32_t* idx,
                                    const double* v, double* out) {
  int64_t i;
#pragma omp parallel for schedule(static)
  for (i = 0; i < W; ++i) {
    int64_t r;
    for (r = 0; r < R; ++r) {
      double acc = 0.0;
      int t;
      for (t = 0; t < zeta; ++t) acc += v[r * zeta + t] * B[i + (int64_t)idx[r * zeta + t] * ldb];
      out[i * R + r] = acc;
    }
  }
}

/* ---------------- Gauss RBF kernel window -------------------------------
 * K(i, j) = exp(-gamma * sum_f (X(r0+i,f) - X(j,f))^2) for i < w, j < N with
 * explicit differences, then K(i, r0+i) = 1 (src/Skema_Kernel.cpp:30-74).
 * X is N x d column-major (ldx); out is w x N row-major.
 */
void oracle_rbf_window(const double* X, int64_t ldx, int64_t N, int64_t d,
                       double gamma, int64_t r0, int64_t w, double* out) {
  int64_t i;
#pragma omp parallel for schedule(static)
  for (i = 0; i < w; ++i) {
    int64_t j;
    for (j = 0; j < N; ++j) {
      double acc = 0.0;
      int64_t f;
      for (f = 0; f < d; ++f) {
        double diff = X[(r0 + i) + f * ldx] - X[j + f * ldx];
        acc += diff * diff;
      }
      out[i * N + j] = exp(-1.0 * gamma * acc);
    }
    out[i * N + (r0 + i)] = 1.0;
  }
}

int oracle_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
