// sparse.cu -- the sparse-map and sparse-input forms of the sketch update.
//
//   CSR x SparseSign (update(crs, SparseSign), src/Skema_SketchySVD.cpp:319-335):
//     y_i  = sum_j a_ij Omega(j, :)      Omega stored n x k, zeta per row
//     X(r,:) += sign * A(c, :)           for each Upsilon entry (r, c) in the window
//     Z(r,:) += sign * A(c, :) Psi       for each Phi entry (r, c) in the window
//   The reference forms these with spgemm + densify
//   (src/Skema_DimRedux_SparseSign.cpp:53-111) after a serial col_subview
//   (:125-155). Here all windows of a call are handled by two launches: a
//   streaming kernel for Y (the HBM-bound part: every nonzero read once, every
//   Y row written once) and a tiny kernel for the X/Z entries, whose window
//   weights eta*nu^(W-1-w) reproduce the per-window axpy sequence.
//   CSR x Gauss (src/Skema_SketchySVD.cpp:296-316), dense x SparseSign
//   (:271-293) and the SketchySPD updates (:896-932) follow.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "internal.h"

namespace skema {

namespace {

int grid_cap(const skema_ctx* c, int64_t want, int per_sm) {
  return (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)c->sm_count * per_sm));
}

// ---------------------------------------------------------------------------
// Y rows for a CSR window block times a stored-transposed SparseSign map.
// One warp owns a tile of R consecutive rows; the tile's k-wide output rows
// accumulate in shared memory (one shared atomic per (nonzero, map entry)),
// then stream out once. Nonzeros are read with streaming loads, the map
// (zeta words per input column) through the read-only path.
// ---------------------------------------------------------------------------
constexpr int YUNR = 2;

template <bool Z8>
__global__ void __launch_bounds__(256)
    csr_ssign_y_kernel(const int64_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                       const float* __restrict__ val, int64_t col_offset, int64_t nrows,
                       const uint32_t* __restrict__ omg, int zeta, int k, int ncol,
                       float* __restrict__ Y,
                       float alpha, float beta, int R) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
  int64_t* srp_all = reinterpret_cast<int64_t*>(smem_raw);
  int64_t* srp = srp_all + warp * 32;
  float* acc = reinterpret_cast<float*>(smem_raw + sizeof(int64_t) * 32 * nw) + (size_t)warp * R * k;
  for (int q = lane; q < R * k; q += 32) acc[q] = 0.f;
  __syncwarp();
  const int64_t ntiles = (nrows + R - 1) / R;
  for (int64_t tile = (int64_t)blockIdx.x * nw + warp; tile < ntiles;
       tile += (int64_t)gridDim.x * nw) {
    const int64_t i0 = tile * R;
    const int rr = (int)min((int64_t)R, nrows - i0);
    if (lane <= rr) srp[lane] = __ldg(rowptr + i0 + lane) - col_offset;
    __syncwarp();
    const int64_t S = srp[0], E = srp[rr];
    for (int64_t base = S; base < E; base += 32 * YUNR) {
      int32_t jj[YUNR];
      float vv[YUNR];
      int rl[YUNR];
#pragma unroll
      for (int u = 0; u < YUNR; ++u) {
        const int64_t e = base + u * 32 + lane;
        const bool ok = e < E;
        jj[u] = ok ? __ldcs(col + e) : -1;
        if ((unsigned)jj[u] >= (unsigned)ncol) jj[u] = -1;  // columns outside [0, n) are ignored
        vv[u] = ok ? __ldcs(val + e) : 0.f;
        // largest l with srp[l] <= e (srp[rr] = E > e)
        int lo = 0, hi = rr;
        while (hi - lo > 1) {
          const int mid = (lo + hi) >> 1;
          if (srp[mid] <= e) lo = mid; else hi = mid;
        }
        rl[u] = lo;
      }
      if (Z8) {
        uint4 w0[YUNR], w1[YUNR];
#pragma unroll
        for (int u = 0; u < YUNR; ++u) {
          if (jj[u] >= 0) {
            const uint4* op = reinterpret_cast<const uint4*>(omg + (int64_t)jj[u] * 8);
            w0[u] = __ldg(op);
            w1[u] = __ldg(op + 1);
          }
        }
#pragma unroll
        for (int u = 0; u < YUNR; ++u) {
          if (jj[u] >= 0) {
            float* a = acc + rl[u] * k;
            const float v = vv[u];
            const uint32_t w[8] = {w0[u].x, w0[u].y, w0[u].z, w0[u].w,
                                   w1[u].x, w1[u].y, w1[u].z, w1[u].w};
#pragma unroll
            for (int t = 0; t < 8; ++t)
              atomicAdd(a + (w[t] & 0x7fffffffu), (w[t] >> 31) ? -v : v);
          }
        }
      } else {
#pragma unroll
        for (int u = 0; u < YUNR; ++u) {
          if (jj[u] >= 0) {
            float* a = acc + rl[u] * k;
            const float v = vv[u];
            for (int t = 0; t < zeta; ++t) {
              const uint32_t w = __ldg(omg + (int64_t)jj[u] * zeta + t);
              atomicAdd(a + (w & 0x7fffffffu), (w >> 31) ? -v : v);
            }
          }
        }
      }
    }
    __syncwarp();
    for (int l = 0; l < rr; ++l) {
      float* yrow = Y + (i0 + l) * (int64_t)k;
      float* arow = acc + l * k;
      for (int cc = lane; cc < k; cc += 32) {
        const float a = arow[cc];
        arow[cc] = 0.f;
        if (beta == 0.f)
          __stcs(yrow + cc, alpha * a);
        else
          yrow[cc] = fmaf(beta, yrow[cc], alpha * a);
      }
    }
    __syncwarp();
  }
}

// X and Z contributions of the Upsilon / Phi entries whose input row lies
// in the call's rows. One warp per entry.
__global__ void csr_ssign_entries_kernel(
    const int64_t* __restrict__ rowptr, const int32_t* __restrict__ col,
    const float* __restrict__ val, int64_t col_offset, int64_t row0, int64_t W, int64_t nwin,
    float eta, float nu, const int64_t* __restrict__ u_row, const uint32_t* __restrict__ u_rs,
    int64_t nu_ent, const int64_t* __restrict__ p_row, const uint32_t* __restrict__ p_rs,
    int64_t np_ent, const uint32_t* __restrict__ psi, int zeta_s, float* __restrict__ X, int64_t n,
    float* __restrict__ Z, int64_t s) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t e = gw; e < nu_ent + np_ent; e += nwarps) {
    const bool is_u = e < nu_ent;
    const int64_t ee = is_u ? e : e - nu_ent;
    const int64_t li = (is_u ? u_row[ee] : p_row[ee]) - row0;
    const uint32_t rsw = is_u ? u_rs[ee] : p_rs[ee];
    const int64_t r = rsw & 0x7fffffffu;
    const int64_t wi = li / W;
    float wgt = eta;
    if (nu != 1.f) wgt = (float)((double)eta * pow((double)nu, (double)(nwin - 1 - wi)));
    if (rsw >> 31) wgt = -wgt;
    const int64_t b = rowptr[li] - col_offset, en = rowptr[li + 1] - col_offset;
    if (is_u) {
      for (int64_t q = b + lane; q < en; q += 32)
        if ((uint64_t)col[q] < (uint64_t)n) atomicAdd(X + r * n + col[q], wgt * val[q]);
    } else {
      const int64_t pairs = (en - b) * zeta_s;
      for (int64_t q = lane; q < pairs; q += 32) {
        const int64_t p = b + q / zeta_s;
        const int t = (int)(q % zeta_s);
        if ((uint64_t)col[p] >= (uint64_t)n) continue;
        const uint32_t w = psi[(int64_t)col[p] * zeta_s + t];
        const float v = wgt * val[p];
        atomicAdd(Z + r * s + (w & 0x7fffffffu), (w >> 31) ? -v : v);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// CSR x Gauss: Y rows by a warp-per-row SpMM against the stored n x k map
// (rows contiguous); X^T / W^T by atomic scatter of map rows.
// ---------------------------------------------------------------------------
__global__ void csr_gauss_y_kernel(const int64_t* __restrict__ rowptr,
                                   const int32_t* __restrict__ col, const float* __restrict__ val,
                                   int64_t col_offset, int64_t nrows, int64_t ncol,
                                   const float* __restrict__ mapT /* n x k rows */, int64_t k,
                                   float* __restrict__ Y, float alpha, float beta) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t i = gw; i < nrows; i += nwarps) {
    const int64_t b = rowptr[i] - col_offset, e = rowptr[i + 1] - col_offset;
    for (int64_t c0 = 0; c0 < k; c0 += 128) {
      float a[4] = {0.f, 0.f, 0.f, 0.f};
      for (int64_t p = b; p < e; ++p) {
        const float v = val[p];
        if ((uint64_t)col[p] >= (uint64_t)ncol) continue;
        const float* mrow = mapT + (int64_t)col[p] * k;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int64_t cc = c0 + lane + 32 * u;
          if (cc < k) a[u] = fmaf(v, __ldg(mrow + cc), a[u]);
        }
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int64_t cc = c0 + lane + 32 * u;
        if (cc < k) {
          float* yp = Y + i * k + cc;
          *yp = (beta == 0.f) ? alpha * a[u] : fmaf(beta, *yp, alpha * a[u]);
        }
      }
    }
  }
}

// out^T(j, :) += alpha * a_ij * map_rows(R0 + i, :) for every nonzero; out is
// stored with (row stride ors, col stride ocs) for logical out(r, j).
__global__ void csr_gauss_scatter_kernel(const int64_t* __restrict__ rowptr,
                                         const int32_t* __restrict__ col,
                                         const float* __restrict__ val, int64_t col_offset,
                                         int64_t nrows, int64_t ncol, const float* __restrict__ maprows,
                                         int64_t kk, float* __restrict__ out, int64_t ors,
                                         int64_t ocs, float alpha) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t i = gw; i < nrows; i += nwarps) {
    const int64_t b = rowptr[i] - col_offset, e = rowptr[i + 1] - col_offset;
    const float* mrow = maprows + i * kk;
    for (int64_t p = b; p < e; ++p) {
      const float v = alpha * val[p];
      const int64_t j = col[p];
      if ((uint64_t)j >= (uint64_t)ncol) continue;
      for (int64_t r = lane; r < kk; r += 32) atomicAdd(out + r * ors + j * ocs, v * mrow[r]);
    }
  }
}

// ---------------------------------------------------------------------------
// Dense window x SparseSign (three-sketch, dense input, update(dense,
// SparseSign) src/Skema_SketchySVD.cpp:271-293).
// Y(R0+i, r) = beta*Y + alpha * sum_t sign_rt A_w(i, c_rt) for the k x n
// row-sparse Omega~. Block: 32 rows x all r, staged in shared memory.
// ---------------------------------------------------------------------------
__global__ void dense_ssign_y_kernel(const float* __restrict__ A, int64_t ars, int64_t acs,
                                     int64_t wr, const uint32_t* __restrict__ omg, int zeta,
                                     int64_t k, float* __restrict__ Y, float alpha, float beta) {
  extern __shared__ float st[];  // 32 x k
  const int ti = threadIdx.x & 31, tr = threadIdx.x >> 5, nr = blockDim.x >> 5;
  for (int64_t i0 = (int64_t)blockIdx.x * 32; i0 < wr; i0 += (int64_t)gridDim.x * 32) {
    const int64_t i = i0 + ti;
    for (int64_t r = tr; r < k; r += nr) {
      float a = 0.f;
      if (i < wr) {
        for (int t = 0; t < zeta; ++t) {
          const uint32_t w = __ldg(omg + r * zeta + t);
          const float v = __ldg(A + i * ars + (int64_t)(w & 0x7fffffffu) * acs);
          a += (w >> 31) ? -v : v;
        }
      }
      st[ti * k + r] = a;
    }
    __syncthreads();
    const int64_t rows = min((int64_t)32, wr - i0);
    for (int64_t q = threadIdx.x; q < rows * k; q += blockDim.x) {
      const int64_t l = q / k, r = q - l * k;
      float* yp = Y + (i0 + l) * k + r;
      const float v = alpha * st[l * k + r];
      *yp = (beta == 0.f) ? v : fmaf(beta, *yp, v);
    }
    __syncthreads();
  }
}

// X(r, :) += wgt * A_w(li, :) for the Upsilon entries in the window, and
// Z(r, :) += wgt * sum_u sign A_w(li, c_{r'' u}) for the Phi entries.
__global__ void dense_ssign_entries_kernel(const float* __restrict__ A, int64_t ars, int64_t acs,
                                           int64_t R0, float eta, const int64_t* __restrict__ u_row,
                                           const uint32_t* __restrict__ u_rs, int64_t nu_ent,
                                           const int64_t* __restrict__ p_row,
                                           const uint32_t* __restrict__ p_rs, int64_t np_ent,
                                           const uint32_t* __restrict__ psi, int zeta_s,
                                           float* __restrict__ X, int64_t n, float* __restrict__ Z,
                                           int64_t s) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t e = gw; e < nu_ent + np_ent; e += nwarps) {
    const bool is_u = e < nu_ent;
    const int64_t ee = is_u ? e : e - nu_ent;
    const int64_t li = (is_u ? u_row[ee] : p_row[ee]) - R0;
    const uint32_t rsw = is_u ? u_rs[ee] : p_rs[ee];
    const int64_t r = rsw & 0x7fffffffu;
    const float wgt = (rsw >> 31) ? -eta : eta;
    const float* arow = A + li * ars;
    if (is_u) {
      for (int64_t j = lane; j < n; j += 32) atomicAdd(X + r * n + j, wgt * arow[j * acs]);
    } else {
      for (int64_t r2 = lane; r2 < s; r2 += 32) {
        float a = 0.f;
        for (int t = 0; t < zeta_s; ++t) {
          const uint32_t w = psi[r2 * zeta_s + t];
          const float v = arow[(int64_t)(w & 0x7fffffffu) * acs];
          a += (w >> 31) ? -v : v;
        }
        atomicAdd(Z + r * s + r2, wgt * a);
      }
    }
  }
}

// SketchySPD with a SparseSign Omega stored n x k (zeta per input column):
// Y(R0+i, :) = beta*Y + alpha * sum_j A_w(i, j) Omega(j, :). One thread per
// row, accumulating its k-row in shared memory (odd stride: no bank clash).
__global__ void dense_colsparse_y_kernel(const float* __restrict__ A, int64_t ars, int64_t acs,
                                         int64_t wr, int64_t n, const uint32_t* __restrict__ omg,
                                         int zeta, int64_t k, int64_t kp, float* __restrict__ Y,
                                         float alpha, float beta) {
  extern __shared__ float acc[];  // blockDim.x x kp
  float* my = acc + (int64_t)threadIdx.x * kp;
  for (int64_t i0 = (int64_t)blockIdx.x * blockDim.x; i0 < wr; i0 += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = i0 + threadIdx.x;
    for (int64_t r = 0; r < k; ++r) my[r] = 0.f;
    if (i < wr) {
      for (int64_t j = 0; j < n; ++j) {
        const float v = __ldg(A + i * ars + j * acs);
        for (int t = 0; t < zeta; ++t) {
          const uint32_t w = __ldg(omg + j * zeta + t);
          my[w & 0x7fffffffu] += (w >> 31) ? -v : v;
        }
      }
      for (int64_t r = 0; r < k; ++r) {
        float* yp = Y + i * k + r;
        *yp = (beta == 0.f) ? alpha * my[r] : fmaf(beta, *yp, alpha * my[r]);
      }
    }
  }
}

// Index range of the sorted inverse entries with input row in [a, b).
std::pair<int64_t, int64_t> entry_range(const Map& mp, int64_t a, int64_t b) {
  const auto lo = std::lower_bound(mp.inv_row.begin(), mp.inv_row.end(), a);
  const auto hi = std::lower_bound(mp.inv_row.begin(), mp.inv_row.end(), b);
  return {lo - mp.inv_row.begin(), hi - mp.inv_row.begin()};
}

void launch_csr_ssign_y(skema_ctx* c, const int64_t* rowptr, const int32_t* col, const float* val,
                        int64_t col_offset, int64_t nrows, const Map& O, float* Yrows, float alpha,
                        float beta) {
  const int k = (int)c->k;
  // rows per warp tile: ~6 KB of accumulators per warp, at most 31 rows
  int R = (int)std::max<int64_t>(1, std::min<int64_t>(31, 6144 / (4 * (int64_t)k)));
  int nw = 8;
  size_t smem = sizeof(int64_t) * 32 * nw + sizeof(float) * (size_t)nw * R * k;
  while (smem > 200 * 1024 && nw > 1) {
    nw >>= 1;
    smem = sizeof(int64_t) * 32 * nw + sizeof(float) * (size_t)nw * R * k;
  }
  if (smem > 200 * 1024) fail(SKEMA_EUNSUPPORTED, "sketch range too large for the sparse-sign kernel");
  const int64_t ntiles = (nrows + R - 1) / R;
  const int64_t blocks_want = (ntiles + nw - 1) / nw;
  int per_sm = 1;
  cudaFuncAttributes fa;
  if (O.zeta == 8) {
    SKEMA_CUDA(cudaFuncSetAttribute(csr_ssign_y_kernel<true>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    SKEMA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, csr_ssign_y_kernel<true>,
                                                             32 * nw, smem));
  } else {
    SKEMA_CUDA(cudaFuncSetAttribute(csr_ssign_y_kernel<false>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    SKEMA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, csr_ssign_y_kernel<false>,
                                                             32 * nw, smem));
  }
  (void)fa;
  const int grid = grid_cap(c, blocks_want, std::max(1, per_sm));
  if (O.zeta == 8)
    csr_ssign_y_kernel<true><<<grid, 32 * nw, smem, c->stream>>>(
        rowptr, col, val, col_offset, nrows, O.packed, 8, k, (int)c->n, Yrows, alpha, beta, R);
  else
    csr_ssign_y_kernel<false><<<grid, 32 * nw, smem, c->stream>>>(
        rowptr, col, val, col_offset, nrows, O.packed, O.zeta, k, (int)c->n, Yrows, alpha, beta, R);
  SKEMA_LAUNCHED(c);
}

}  // namespace

// ---------------------------------------------------------------------------
void csr_update(skema_ctx* c, const int64_t* rowptr, const int32_t* col, const float* val,
                int64_t col_offset, int64_t row0, int64_t nrows) {
  const float eta = (float)c->p.sketch_eta, nu = (float)c->p.sketch_nu;
  const int64_t W = c->w;
  const int64_t nwin = (nrows + W - 1) / W;
  const bool clean = y_rows_clean(c, row0, row0 + nrows);
  const float ybeta = clean ? 0.f : nu;
  float* Yrows = c->Y + row0 * c->k;

  if (c->p.dim_redux == SKEMA_MAP_SPARSE_SIGN) {
    {
      StageScope st(c, ST_OMEGA);
      launch_csr_ssign_y(c, rowptr, col, val, col_offset, nrows, c->omg, Yrows, eta, ybeta);
    }
    y_rows_mark(c, row0, row0 + nrows);
    if (c->spd) return;
    if (nu != 1.f) {
      StageScope st(c, ST_DAXPY);
      const float sc = (float)std::pow((double)nu, (double)nwin);
      scale_block(c, MatOut{c->X, c->n, 1}, c->k, c->n, sc);
      scale_block(c, MatOut{c->Z, c->s, 1}, c->s, c->s, sc);
    }
    const auto ur = entry_range(c->ups, row0, row0 + nrows);
    const auto pr = entry_range(c->phi, row0, row0 + nrows);
    const int64_t nue = ur.second - ur.first, npe = pr.second - pr.first;
    if (nue + npe > 0) {
      StageScope st(c, ST_ENTRIES);
      const int threads = 256;
      const int grid = grid_cap(c, (nue + npe + 7) / 8, 8);
      csr_ssign_entries_kernel<<<grid, threads, 0, c->stream>>>(
          rowptr, col, val, col_offset, row0, W, nwin, eta, nu, c->ups.d_inv_row + ur.first,
          c->ups.d_inv_rs + ur.first, nue, c->phi.d_inv_row + pr.first, c->phi.d_inv_rs + pr.first,
          npe, c->psi.packed, c->psi.zeta, c->X, c->n, c->Z, c->s);
      SKEMA_LAUNCHED(c);
    }
    return;
  }

  // Gauss maps, all stored transposed (src/Skema_SketchySVD.cpp:296-316):
  // stored rows contiguous, logical (r, j) at f32[r + j*lrows].
  const int threads = 256;
  for (int64_t r = 0; r < nrows; r += W) {
    const int64_t wr = std::min(W, nrows - r);
    const int64_t R0 = row0 + r;
    const float yb = y_rows_clean(c, R0, R0 + wr) ? 0.f : nu;
    csr_gauss_y_kernel<<<grid_cap(c, (wr + 7) / 8, 16), threads, 0, c->stream>>>(
        rowptr + r, col, val, col_offset, wr, c->n, c->omg.f32, c->k, c->Y + R0 * c->k, eta, yb);
    SKEMA_LAUNCHED(c);
    y_rows_mark(c, R0, R0 + wr);
    if (c->spd) continue;
    // X = nu X + eta (A_w^T Upsilon_stored(R0:R0+wr, :))^T
    scale_block(c, MatOut{c->X, c->n, 1}, c->k, c->n, nu);
    csr_gauss_scatter_kernel<<<grid_cap(c, (wr + 7) / 8, 16), threads, 0, c->stream>>>(
        rowptr + r, col, val, col_offset, wr, c->n, c->ups.f32 + R0 * c->k, c->k, c->X, c->n, 1, eta);
    SKEMA_LAUNCHED(c);
    // W^T = A_w^T Phi_stored(R0:R0+wr, :) in scratch (n x s), then
    // Z = nu Z + eta W Psi_stored.
    float* Wt = (float*)workspace(c, sizeof(float) * (size_t)(c->n * c->s));
    SKEMA_CUDA(cudaMemsetAsync(Wt, 0, sizeof(float) * (size_t)(c->n * c->s), c->stream));
    csr_gauss_scatter_kernel<<<grid_cap(c, (wr + 7) / 8, 16), threads, 0, c->stream>>>(
        rowptr + r, col, val, col_offset, wr, c->n, c->phi.f32 + R0 * c->s, c->s, Wt, 1, c->s, 1.f);
    SKEMA_LAUNCHED(c);
    scale_block(c, MatOut{c->Z, c->s, 1}, c->s, c->s, nu);
    const int64_t tiles = ((c->s + 127) / 128) * ((c->s + 127) / 128);
    int sk = (int)std::max<int64_t>(1, std::min<int64_t>((2 * c->sm_count + tiles - 1) / tiles, c->n / 256));
    sgemm(c, c->s, c->s, c->n, eta, Mat{Wt, 1, c->s}, Mat{c->psi.f32, c->psi.cs, c->psi.rs}, 1.f,
          MatOut{c->Z, c->s, 1}, std::max(1, sk));
  }
}

void dense_ssign_window(skema_ctx* c, Mat Aw, int64_t R0, int64_t wr) {
  const float eta = (float)c->p.sketch_eta, nu = (float)c->p.sketch_nu;
  const float ybeta = y_rows_clean(c, R0, R0 + wr) ? 0.f : nu;
  const size_t smem = sizeof(float) * 32 * (size_t)c->k;
  if (smem > 200 * 1024) fail(SKEMA_EUNSUPPORTED, "sketch range too large for the dense sparse-sign kernel");
  SKEMA_CUDA(cudaFuncSetAttribute(dense_ssign_y_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem));
  dense_ssign_y_kernel<<<grid_cap(c, (wr + 31) / 32, 4), 256, smem, c->stream>>>(
      Aw.p, Aw.rs, Aw.cs, wr, c->omg.packed, c->omg.zeta, c->k, c->Y + R0 * c->k, eta, ybeta);
  SKEMA_LAUNCHED(c);
  y_rows_mark(c, R0, R0 + wr);
  scale_block(c, MatOut{c->X, c->n, 1}, c->k, c->n, nu);
  scale_block(c, MatOut{c->Z, c->s, 1}, c->s, c->s, nu);
  const auto ur = entry_range(c->ups, R0, R0 + wr);
  const auto pr = entry_range(c->phi, R0, R0 + wr);
  const int64_t nue = ur.second - ur.first, npe = pr.second - pr.first;
  if (nue + npe == 0) return;
  dense_ssign_entries_kernel<<<grid_cap(c, (nue + npe + 7) / 8, 8), 256, 0, c->stream>>>(
      Aw.p, Aw.rs, Aw.cs, R0, eta, c->ups.d_inv_row + ur.first, c->ups.d_inv_rs + ur.first, nue,
      c->phi.d_inv_row + pr.first, c->phi.d_inv_rs + pr.first, npe, c->psi.packed, c->psi.zeta, c->X,
      c->n, c->Z, c->s);
  SKEMA_LAUNCHED(c);
}

void spd_ssign_window(skema_ctx* c, Mat Aw, int64_t R0, int64_t wr) {
  const float eta = (float)c->p.sketch_eta, nu = (float)c->p.sketch_nu;
  const float ybeta = y_rows_clean(c, R0, R0 + wr) ? 0.f : nu;
  const int64_t kp = c->k | 1;
  int threads = 128;
  while (threads > 32 && sizeof(float) * (size_t)(threads * kp) > 200 * 1024) threads >>= 1;
  const size_t smem = sizeof(float) * (size_t)(threads * kp);
  if (smem > 200 * 1024) fail(SKEMA_EUNSUPPORTED, "sketch range too large for the SPD sparse-sign kernel");
  SKEMA_CUDA(cudaFuncSetAttribute(dense_colsparse_y_kernel,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  dense_colsparse_y_kernel<<<grid_cap(c, (wr + threads - 1) / threads, 4), threads, smem, c->stream>>>(
      Aw.p, Aw.rs, Aw.cs, wr, c->n, c->omg.packed, c->omg.zeta, c->k, kp, c->Y + R0 * c->k, eta,
      ybeta);
  SKEMA_LAUNCHED(c);
  y_rows_mark(c, R0, R0 + wr);
}

}  // namespace skema
