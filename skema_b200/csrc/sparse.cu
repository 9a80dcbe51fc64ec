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
//   Y element written once) and a tiny kernel for the X/Z entries, whose window
//   weights eta*nu^(W-1-w) reproduce the per-window axpy sequence.
//   CSR x Gauss (src/Skema_SketchySVD.cpp:296-316), dense x SparseSign
//   (:271-293) and the SketchySPD updates (:896-932) follow.
//
// Y is column-major (m x k, ld = m), the reference's LayoutLeft.
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
// Y rows of a CSR block times a stored-transposed SparseSign map (n rows of
// zeta entries over k columns).
//
// One thread per input row. Each warp owns 32 consecutive rows and a
// bin-major accumulator acc[r * 32 + lane] in shared memory: lane l adds
// +-a_ij into the k bins of its own row only, so the updates need no
// atomics and every shared access of a warp hits 32 distinct banks. After
// the rows are done, bin r of the 32 rows is one coalesced 128-byte store
// into the column-major Y. Nonzeros go through the read-only path (the
// warp's 32 rows are contiguous in col/val, so L1 serves the lanes' strided
// walk). This general form reads zeta 32-bit map words per input column
// (column | sign << 31); csr_ssign_y16_kernel below is the form for zeta = 8
// and k <= 256.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void ssign_apply(float* __restrict__ my, const uint32_t* __restrict__ omg32, int zeta,
                                            int32_t j, float a) {
  for (int t = 0; t < zeta; ++t) {
    const uint32_t w = __ldg(omg32 + (int64_t)j * zeta + t);
    my[(w & 0x7fffffffu) * 32] += (w >> 31) ? -a : a;
  }
}

template <int UNR>
__global__ void __launch_bounds__(128)
    csr_ssign_y_kernel(const int64_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                       const float* __restrict__ val, int64_t col_offset, int64_t nrows,
                       const uint32_t* __restrict__ omg32,
                       int zeta, int k, int ncol, float* __restrict__ Y, int64_t ldy, float alpha,
                       float beta) {
  extern __shared__ float acc_all[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  float* my = acc_all + (size_t)warp * k * 32 + lane;  // bins of this lane's row: my[r * 32]
  for (int r = 0; r < k; ++r) my[r * 32] = 0.f;
  const int64_t ntiles = (nrows + 31) / 32;
  for (int64_t tile = (int64_t)blockIdx.x * nw + warp; tile < ntiles;
       tile += (int64_t)gridDim.x * nw) {
    const int64_t i = tile * 32 + lane;
    const bool live = i < nrows;
    int64_t b = live ? __ldg(rowptr + i) - col_offset : 0;
    int64_t e = __shfl_down_sync(0xffffffffu, b, 1);
    if (lane == 31 || i + 1 >= nrows) e = live ? __ldg(rowptr + i + 1) - col_offset : 0;
    int64_t p = b;
    for (; p + UNR <= e; p += UNR) {
      int32_t jj[UNR];
      float aa[UNR];
#pragma unroll
      for (int u = 0; u < UNR; ++u) {
        jj[u] = __ldg(col + p + u);
        aa[u] = __ldg(val + p + u);
      }
#pragma unroll
      for (int u = 0; u < UNR; ++u)
        if ((unsigned)jj[u] < (unsigned)ncol) ssign_apply(my, omg32, zeta, jj[u], aa[u]);
    }
    for (; p < e; ++p) {
      const int32_t j = __ldg(col + p);
      if ((unsigned)j < (unsigned)ncol) ssign_apply(my, omg32, zeta, j, __ldg(val + p));
    }
    if (live) {
      float* yp = Y + i;
      for (int r = 0; r < k; ++r) {
        const float v = my[r * 32];
        my[r * 32] = 0.f;
        if (beta == 0.f)
          __stcs(yp + r * ldy, alpha * v);
        else
          yp[r * ldy] = fmaf(beta, yp[r * ldy], alpha * v);
      }
    }
  }
}

// The same Y rows for the map's 16-bit offset form (zeta = 8, k <= 256):
// each entry is the byte offset of its bin in the warp's accumulator, the
// sign in bit 15 and a same-bin-as-previous flag in bit 0 (pack16_kernel).
// Per nonzero the eight bin loads are issued together, then the eight stores
// in entry order; a flagged entry adds to the previous entry's sum instead of
// its own (stale) load, so every bin still sees its additions in entry order
// and Y is bit-identical to one read-modify-write per entry.
// The work is pipelined across each warp's tiles: the next tile's row range
// is loaded when a tile starts and its first U nonzeros with the current
// tile's last batch, so their latency overlaps the apply and the write-out.
// Map rows are gathered through L2 only (.cg): 1e7 random 16-byte gathers
// would otherwise evict the col/val lines that the lanes' row walks reuse
// from L1. The write-out moves four bins per 16-byte access (lane -> bin
// r0 + lane / 8, rows 4 (lane % 8) .. + 3) and clears them in the same pass.
// The launch keeps about 128 KB of bins per SM and gives the rest of the
// unified L1 / shared memory to L1, which the row walks need (measured on the
// 1e6 x 1e5, 1e7-nonzero case: 48 KB less L1 cost 8 %, 96 KB less 34 %).
__device__ __forceinline__ float bin_ld(uint32_t addr) {
  float x;
  asm volatile("ld.shared.f32 %0, [%1];" : "=f"(x) : "r"(addr) : "memory");
  return x;
}
__device__ __forceinline__ void bin_st(uint32_t addr, float v) {
  asm volatile("st.shared.f32 [%0], %1;" ::"r"(addr), "f"(v) : "memory");
}

__device__ __forceinline__ void ssign_apply8(uint32_t base, uint4 wv, float a) {
  const uint32_t abits = __float_as_uint(a);
  const uint32_t e[8] = {wv.x & 0xffffu, wv.x >> 16, wv.y & 0xffffu, wv.y >> 16,
                         wv.z & 0xffffu, wv.z >> 16, wv.w & 0xffffu, wv.w >> 16};
  float v[8];
#pragma unroll
  for (int t = 0; t < 8; ++t) v[t] = bin_ld(base + (e[t] & 0x7f80u));
  float prev = 0.f;
#pragma unroll
  for (int t = 0; t < 8; ++t) {
    const float nv = ((e[t] & 1u) ? prev : v[t]) + __uint_as_float(abits ^ ((e[t] << 16) & 0x80000000u));
    bin_st(base + (e[t] & 0x7f80u), nv);
    prev = nv;
  }
}

// (A form with one red.shared.add per map entry instead of the load and
// store measured 30 % slower: 0.170 against 0.131 ms on the 1e6 x 1e5 case.)
template <int U>
__global__ void __launch_bounds__(128)
    csr_ssign_y16_kernel(const int64_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                         const float* __restrict__ val, int64_t col_offset, int64_t nrows,
                         const uint4* __restrict__ omg16, int k, int ncol, float* __restrict__ Y, int64_t ldy,
                         float alpha, float beta) {
  extern __shared__ __align__(16) float acc_all[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  float* bins = acc_all + (size_t)warp * k * 32;
  const uint32_t base = (uint32_t)__cvta_generic_to_shared(bins + lane);
  float4* bins4 = reinterpret_cast<float4*>(bins);
  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int q = lane; q < k * 8; q += 32) bins4[q] = z4;
  __syncwarp();
  const int64_t ntiles = (nrows + 31) / 32;
  const int64_t tstride = (int64_t)gridDim.x * nw;
  const bool vec = (reinterpret_cast<uintptr_t>(Y) & 15) == 0 && ldy % 4 == 0;
  int64_t tile = (int64_t)blockIdx.x * nw + warp;
  auto row_range = [&](int64_t t, int64_t& b, int64_t& e) {
    const int64_t i = t * 32 + lane;
    b = 0, e = 0;
    if (t < ntiles && i < nrows) b = __ldg(rowptr + i) - col_offset, e = __ldg(rowptr + i + 1) - col_offset;
  };
  auto load_batch = [&](int64_t q0, int64_t q1, int32_t* jj, float* aa) {
#pragma unroll
    for (int u = 0; u < U; ++u) {
      jj[u] = -1, aa[u] = 0.f;
      if (q0 + u < q1) jj[u] = __ldcs(col + q0 + u), aa[u] = __ldcs(val + q0 + u);
    }
  };
  int64_t b, e;
  row_range(tile, b, e);
  int32_t jj[U];
  float aa[U];
  load_batch(b, e, jj, aa);
  for (; tile < ntiles; tile += tstride) {
    int64_t nb, ne;
    row_range(tile + tstride, nb, ne);
    for (int64_t p = b;; p += U) {
      uint4 ww[U];
#pragma unroll
      for (int u = 0; u < U; ++u)
        ww[u] = (unsigned)jj[u] < (unsigned)ncol ? __ldcg(omg16 + jj[u]) : make_uint4(0u, 0u, 0u, 0u);
      // the next batch: the rest of this row, else the next tile's first
      const bool more = p + U < e;
      int32_t j2[U];
      float a2[U];
      load_batch(more ? p + U : nb, more ? e : ne, j2, a2);
#pragma unroll
      for (int u = 0; u < U; ++u)
        if ((unsigned)jj[u] < (unsigned)ncol) ssign_apply8(base, ww[u], aa[u] * alpha);
#pragma unroll
      for (int u = 0; u < U; ++u) jj[u] = j2[u], aa[u] = a2[u];
      if (!more) break;
    }
    __syncwarp();
    const int64_t r0 = tile * 32;
    if (vec && r0 + 32 <= nrows) {
      const int sub = lane >> 3, q4 = lane & 7;
      float* yp = Y + r0 + 4 * q4 + (int64_t)sub * ldy;
      for (int r = sub; r < k; r += 4, yp += 4 * ldy) {
        float4* bp = bins4 + r * 8 + q4;
        float4 v = *bp;
        *bp = z4;
        float4* y4 = reinterpret_cast<float4*>(yp);
        if (beta == 0.f) {
          __stcs(y4, v);
        } else {
          const float4 o = *y4;
          v.x = fmaf(beta, o.x, v.x), v.y = fmaf(beta, o.y, v.y), v.z = fmaf(beta, o.z, v.z),
          v.w = fmaf(beta, o.w, v.w);
          *y4 = v;
        }
      }
    } else {
      const int64_t i = r0 + lane;
      if (i < nrows) {
        float* yp = Y + i;
        if (beta == 0.f) {
          for (int r = 0; r < k; ++r, yp += ldy) __stcs(yp, bins[r * 32 + lane]);
        } else {
          for (int r = 0; r < k; ++r, yp += ldy) *yp = fmaf(beta, *yp, bins[r * 32 + lane]);
        }
      }
      __syncwarp();
      for (int q = lane; q < k * 8; q += 32) bins4[q] = z4;
    }
    __syncwarp();
    b = nb, e = ne;
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
                                   float* __restrict__ Y, int64_t ldy, float alpha, float beta) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t i = gw; i < nrows; i += nwarps) {
    const int64_t b = rowptr[i] - col_offset, e = rowptr[i + 1] - col_offset;
    for (int64_t c0 = 0; c0 < k; c0 += 128) {
      float a[4] = {0.f, 0.f, 0.f, 0.f};
      for (int64_t p = b; p < e; ++p) {
        if ((uint64_t)col[p] >= (uint64_t)ncol) continue;
        const float v = val[p];
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
          float* yp = Y + i + cc * ldy;
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
                                         int64_t nrows, int64_t ncol,
                                         const float* __restrict__ maprows, int64_t kk,
                                         float* __restrict__ out, int64_t ors, int64_t ocs,
                                         float alpha) {
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
// row-sparse Omega~: thread (row, map row), consecutive threads on
// consecutive rows (coalesced gathers from a column-major window and
// coalesced stores into the column-major Y).
// ---------------------------------------------------------------------------
__global__ void dense_ssign_y_kernel(const float* __restrict__ A, int64_t ars, int64_t acs,
                                     int64_t wr, const uint32_t* __restrict__ omg, int zeta,
                                     int64_t k, float* __restrict__ Y, int64_t ldy, float alpha,
                                     float beta) {
  const int64_t total = wr * k;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = q / wr, i = q - r * wr;
    float a = 0.f;
    for (int t = 0; t < zeta; ++t) {
      const uint32_t w = __ldg(omg + r * zeta + t);
      const float v = __ldg(A + i * ars + (int64_t)(w & 0x7fffffffu) * acs);
      a += (w >> 31) ? -v : v;
    }
    float* yp = Y + i + r * ldy;
    *yp = (beta == 0.f) ? alpha * a : fmaf(beta, *yp, alpha * a);
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
// row with bin-major accumulators acc[r * blockDim + tid] (conflict free).
__global__ void dense_colsparse_y_kernel(const float* __restrict__ A, int64_t ars, int64_t acs,
                                         int64_t wr, int64_t n, const uint32_t* __restrict__ omg,
                                         int zeta, int64_t k, float* __restrict__ Y, int64_t ldy,
                                         float alpha, float beta) {
  extern __shared__ float acc[];
  float* my = acc + threadIdx.x;
  const int nt = blockDim.x;
  for (int64_t i0 = (int64_t)blockIdx.x * nt; i0 < wr; i0 += (int64_t)gridDim.x * nt) {
    const int64_t i = i0 + threadIdx.x;
    for (int64_t r = 0; r < k; ++r) my[r * nt] = 0.f;
    if (i < wr) {
      for (int64_t j = 0; j < n; ++j) {
        const float v = __ldg(A + i * ars + j * acs);
        for (int t = 0; t < zeta; ++t) {
          const uint32_t w = __ldg(omg + j * zeta + t);
          my[(int64_t)(w & 0x7fffffffu) * nt] += (w >> 31) ? -v : v;
        }
      }
      for (int64_t r = 0; r < k; ++r) {
        float* yp = Y + i + r * ldy;
        *yp = (beta == 0.f) ? alpha * my[r * nt] : fmaf(beta, *yp, alpha * my[r * nt]);
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

}  // namespace

template <int UNR>
void launch_csr_ssign_y_variant(skema_ctx* c, int warps_per_block, const int64_t* rowptr,
                                const int32_t* col, const float* val, int64_t col_offset,
                                int64_t nrows, const Map& O, float* Y, int64_t ldy, float alpha,
                                float beta) {
  const int k = (int)c->k;
  const size_t smem = sizeof(float) * 32 * (size_t)k * warps_per_block;
  auto kern = csr_ssign_y_kernel<UNR>;
  SKEMA_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 1;
  SKEMA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * warps_per_block, smem));
  const int64_t tiles = (nrows + 31) / 32;
  const int grid = grid_cap(c, (tiles + warps_per_block - 1) / warps_per_block, std::max(1, per_sm));
  kern<<<grid, 32 * warps_per_block, smem, c->stream>>>(rowptr, col, val, col_offset, nrows, O.packed, O.zeta,
                                                        k, (int)c->n, Y, ldy, alpha, beta);
  SKEMA_LAUNCHED(c);
}

template <int U>
static void launch_csr_ssign_y16(skema_ctx* c, const int64_t* rowptr, const int32_t* col, const float* val,
                                 int64_t col_offset, int64_t nrows, const Map& O, float* Y, int64_t ldy, float alpha,
                                 float beta) {
  const int k = (int)c->k;
  // warps per block: the most warps within the bin budget per SM (about
  // 128 KB), in the fewest blocks (k = 81: 4 x 3 = 12 warps; k = 161:
  // 2 x 3 = 6; k = 256: 4 x 1)
  const size_t budget = (size_t)c->ssign_bin_kb * 1024;
  int wpb = 1;
  {
    const size_t per_warp = sizeof(float) * 32 * (size_t)k;
    int best = 0;
    for (int w = 4; w >= 1; w >>= 1) {
      const int warps = w * (int)(budget / (per_warp * w));
      if (warps > best) best = warps, wpb = w;
    }
  }
  const size_t smem = sizeof(float) * 32 * (size_t)k * wpb;
  auto kern = csr_ssign_y16_kernel<U>;
  SKEMA_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  // the bin budget per SM; the carve-out leaves the rest of the unified
  // L1 / shared memory to L1
  int smem_sm = 0;
  SKEMA_CUDA(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, c->dev));
  const int per_sm = (int)std::max<size_t>(1, budget / smem);
  const int carve = (int)std::min<size_t>(100, (per_sm * (smem + 1024) * 100 + smem_sm - 1) / std::max(1, smem_sm) + 2);
  SKEMA_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, carve));
  const int64_t tiles = (nrows + 31) / 32;
  const int grid = grid_cap(c, (tiles + wpb - 1) / wpb, per_sm);
  kern<<<grid, 32 * wpb, smem, c->stream>>>(rowptr, col, val, col_offset, nrows,
                                            static_cast<const uint4*>(O.packed16), k, (int)c->n, Y, ldy, alpha,
                                            beta);
  SKEMA_LAUNCHED(c);
}

static void launch_csr_ssign_y(skema_ctx* c, const int64_t* rowptr, const int32_t* col,
                               const float* val, int64_t col_offset, int64_t nrows, const Map& O,
                               float* Y, int64_t ldy, float alpha, float beta) {
  if (O.packed16) {  // zeta = 8, k <= 256: at most 32 KB of bins per warp
    switch (c->ssign_batch) {
      case 2: launch_csr_ssign_y16<2>(c, rowptr, col, val, col_offset, nrows, O, Y, ldy, alpha, beta); break;
      case 6: launch_csr_ssign_y16<6>(c, rowptr, col, val, col_offset, nrows, O, Y, ldy, alpha, beta); break;
      case 8: launch_csr_ssign_y16<8>(c, rowptr, col, val, col_offset, nrows, O, Y, ldy, alpha, beta); break;
      default: launch_csr_ssign_y16<4>(c, rowptr, col, val, col_offset, nrows, O, Y, ldy, alpha, beta); break;
    }
    return;
  }
  // general form: up to 4 warps within 96 KB of bins per block; one warp's
  // bins (32 k floats) must fit the 200 KB limit
  int wpb = 4;
  while (wpb > 1 && sizeof(float) * 32 * (size_t)c->k * wpb > 96 * 1024) wpb >>= 1;
  if (sizeof(float) * 32 * (size_t)c->k * wpb > 200 * 1024)
    fail(SKEMA_EUNSUPPORTED, "sketch range too large for the sparse-sign kernel");
  launch_csr_ssign_y_variant<4>(c, wpb, rowptr, col, val, col_offset, nrows, O, Y, ldy, alpha, beta);
}

// ---------------------------------------------------------------------------
void csr_update(skema_ctx* c, const int64_t* rowptr, const int32_t* col, const float* val,
                int64_t col_offset, int64_t row0, int64_t nrows) {
  if (c->residual_pass) {
    residual_csr(c, rowptr, col, val, col_offset, row0, nrows);
    return;
  }
  const float eta = (float)c->p.sketch_eta, nu = (float)c->p.sketch_nu;
  const int64_t W = c->w;
  const int64_t nwin = (nrows + W - 1) / W;
  const float ybeta = y_beta(c, row0, row0 + nrows, nu);

  if (c->p.dim_redux == SKEMA_MAP_SPARSE_SIGN) {
    // X / Z (zeroing after a reset, the nu scaling and the Upsilon / Phi
    // entries) touch neither Y nor anything the Y kernel reads: they run on
    // the side stream, forked before the Y launch and joined after it,
    // beside the Y kernel.
    const auto ur = entry_range(c->ups, row0, row0 + nrows);
    const auto pr = entry_range(c->phi, row0, row0 + nrows);
    const int64_t nue = c->spd ? 0 : ur.second - ur.first, npe = c->spd ? 0 : pr.second - pr.first;
    const bool side = c->xz_pending || (!c->spd && (nu != 1.f || nue + npe > 0));
    if (side) SKEMA_CUDA(cudaEventRecord(c->fork_ev, c->stream));
    {
      StageScope st(c, ST_OMEGA);
      launch_csr_ssign_y(c, rowptr, col, val, col_offset, nrows, c->omg, c->Y + row0, c->m, eta, ybeta);
    }
    y_rows_mark(c, row0, row0 + nrows);
    if (!side) return;
    SKEMA_CUDA(cudaStreamWaitEvent(c->side, c->fork_ev, 0));
    xz_materialize(c, c->side);
    if (c->spd) {
      SKEMA_CUDA(cudaEventRecord(c->join_ev, c->side));
      SKEMA_CUDA(cudaStreamWaitEvent(c->stream, c->join_ev, 0));
      return;
    }
    if (nu != 1.f) {
      StageScope st(c, ST_DAXPY, c->side);
      const float sc = (float)std::pow((double)nu, (double)nwin);
      scale_block(c, MatOut{c->X, c->n, 1}, c->k, c->n, sc, c->side);
      scale_block(c, MatOut{c->Z, c->s, 1}, c->s, c->s, sc, c->side);
    }
    if (nue + npe > 0) {
      StageScope st(c, ST_ENTRIES, c->side);
      const int grid = grid_cap(c, (nue + npe + 7) / 8, 8);
      csr_ssign_entries_kernel<<<grid, 256, 0, c->side>>>(
          rowptr, col, val, col_offset, row0, W, nwin, eta, nu, c->ups.d_inv_row + ur.first,
          c->ups.d_inv_rs + ur.first, nue, c->phi.d_inv_row + pr.first, c->phi.d_inv_rs + pr.first,
          npe, c->psi.packed, c->psi.zeta, c->X, c->n, c->Z, c->s);
      SKEMA_LAUNCHED(c);
    }
    SKEMA_CUDA(cudaEventRecord(c->join_ev, c->side));
    SKEMA_CUDA(cudaStreamWaitEvent(c->stream, c->join_ev, 0));
    return;
  }

  xz_materialize(c, c->stream);
  // Gauss maps, all stored transposed (src/Skema_SketchySVD.cpp:296-316):
  // stored rows contiguous, logical (r, j) at f32[r + j*lrows].
  const int threads = 256;
  for (int64_t r = 0; r < nrows; r += W) {
    const int64_t wr = std::min(W, nrows - r);
    const int64_t R0 = row0 + r;
    const float yb = y_beta(c, R0, R0 + wr, nu);
    {
      StageScope st(c, ST_OMEGA);
      csr_gauss_y_kernel<<<grid_cap(c, (wr + 7) / 8, 16), threads, 0, c->stream>>>(
          rowptr + r, col, val, col_offset, wr, c->n, c->omg.f32, c->k, c->Y + R0, c->m, eta, yb);
      SKEMA_LAUNCHED(c);
    }
    y_rows_mark(c, R0, R0 + wr);
    if (c->spd) continue;
    {  // X = nu X + eta (A_w^T Upsilon_stored(R0:R0+wr, :))^T
      StageScope st(c, ST_UPSILON);
      scale_block(c, MatOut{c->X, c->n, 1}, c->k, c->n, nu);
      csr_gauss_scatter_kernel<<<grid_cap(c, (wr + 7) / 8, 16), threads, 0, c->stream>>>(
          rowptr + r, col, val, col_offset, wr, c->n, c->ups.f32 + R0 * c->k, c->k, c->X, c->n, 1, eta);
      SKEMA_LAUNCHED(c);
    }
    // W^T = A_w^T Phi_stored(R0:R0+wr, :) in scratch (n x s), then
    // Z = nu Z + eta W Psi_stored.
    StageScope st(c, ST_PHI);
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
  const float ybeta = y_beta(c, R0, R0 + wr, nu);
  {
    StageScope st(c, ST_OMEGA);
    dense_ssign_y_kernel<<<grid_cap(c, (wr * c->k + 255) / 256, 16), 256, 0, c->stream>>>(
        Aw.p, Aw.rs, Aw.cs, wr, c->omg.packed, c->omg.zeta, c->k, c->Y + R0, c->m, eta, ybeta);
    SKEMA_LAUNCHED(c);
  }
  y_rows_mark(c, R0, R0 + wr);
  scale_block(c, MatOut{c->X, c->n, 1}, c->k, c->n, nu);
  scale_block(c, MatOut{c->Z, c->s, 1}, c->s, c->s, nu);
  const auto ur = entry_range(c->ups, R0, R0 + wr);
  const auto pr = entry_range(c->phi, R0, R0 + wr);
  const int64_t nue = ur.second - ur.first, npe = pr.second - pr.first;
  if (nue + npe == 0) return;
  StageScope st(c, ST_ENTRIES);
  dense_ssign_entries_kernel<<<grid_cap(c, (nue + npe + 7) / 8, 8), 256, 0, c->stream>>>(
      Aw.p, Aw.rs, Aw.cs, R0, eta, c->ups.d_inv_row + ur.first, c->ups.d_inv_rs + ur.first, nue,
      c->phi.d_inv_row + pr.first, c->phi.d_inv_rs + pr.first, npe, c->psi.packed, c->psi.zeta, c->X,
      c->n, c->Z, c->s);
  SKEMA_LAUNCHED(c);
}

void spd_ssign_window(skema_ctx* c, Mat Aw, int64_t R0, int64_t wr) {
  const float eta = (float)c->p.sketch_eta, nu = (float)c->p.sketch_nu;
  const float ybeta = y_beta(c, R0, R0 + wr, nu);
  int threads = 128;
  while (threads > 32 && sizeof(float) * (size_t)(threads * c->k) > 200 * 1024) threads >>= 1;
  const size_t smem = sizeof(float) * (size_t)(threads * c->k);
  if (smem > 200 * 1024) fail(SKEMA_EUNSUPPORTED, "sketch range too large for the SPD sparse-sign kernel");
  SKEMA_CUDA(cudaFuncSetAttribute(dense_colsparse_y_kernel,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  StageScope st(c, ST_OMEGA);
  dense_colsparse_y_kernel<<<grid_cap(c, (wr + threads - 1) / threads, 4), threads, smem, c->stream>>>(
      Aw.p, Aw.rs, Aw.cs, wr, c->n, c->omg.packed, c->omg.zeta, c->k, c->Y + R0, c->m, eta, ybeta);
  SKEMA_LAUNCHED(c);
  y_rows_mark(c, R0, R0 + wr);
}

}  // namespace skema
