// dimredux.cu -- standalone random maps with their lmap / rmap products:
// GaussDimRedux and SparseSignDimRedux (src/Skema_DimRedux.hpp:60-268,
// src/Skema_DimRedux_Gauss.cpp:10-99, src/Skema_DimRedux_SparseSign.cpp:9-111).
//
// A map is generated exactly as a context's map of the same kind, shape and
// seed (maps.cu), so a caller can apply the sketch operators by hand. The
// products are stated without the reference's conventions:
//   lmap:  C = alpha op(M(:, idx)) op(B) + beta C     (idx: stored columns)
//   rmap:  C = alpha op(A) op(M(idx, :)) + beta C     (idx: stored rows)
// with op() chosen by 'N' / 'T'; the C++ layer (include/skema.hpp) maps the
// reference's calls, with its init_transposed swap and its transposed CRS
// results, onto these. A SparseSign map is expanded once into a dense FP32
// copy (duplicate entries summed, as KokkosSparse does) and then multiplies
// like a Gauss map: these products are utilities, not the streaming path.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "internal.h"

struct skema_dimredux {
  skema_ctx* c = nullptr;  // device, stream and workspace (a context without sketches)
  skema::Map map;
  float* dense = nullptr;  // SparseSign: stored nrow x ncol, row-major, expanded on first use
  std::string err;
};

namespace skema {

void map_export(skema_ctx* c, Map& mp, double* values, int32_t* indices);

namespace {

int grid1d(const skema_ctx* c, int64_t total, int threads) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((total + threads - 1) / threads, (int64_t)c->sm_count * 16));
}

// Dense row-major copy of a SparseSign map: one thread per stored row adds
// its zeta signs in entry order.
__global__ void ssign_expand_kernel(const uint32_t* __restrict__ packed, int64_t nrow, int64_t ncol, int zeta,
                                    float* __restrict__ out) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < nrow; r += (int64_t)gridDim.x * blockDim.x) {
    float* row = out + r * ncol;
    for (int t = 0; t < zeta; ++t) {
      const uint32_t w = packed[r * zeta + t];
      row[w & 0x7fffffffu] += (w >> 31) ? -1.f : 1.f;
    }
  }
}

// out(i, :) = alpha sum_p val[p] D(col[p], :) + beta out(i, :) for the rows of
// a CSR matrix (one warp per row, lanes over the K output columns); column
// indices outside [0, ncol) are skipped.
__global__ void csr_spmm_kernel(const int64_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                                const float* __restrict__ val, int64_t nrows, int64_t ncol, Mat D, int64_t K,
                                MatOut out, float alpha, float beta) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t base = nrows > 0 ? rowptr[0] : 0;
  for (int64_t i = gw; i < nrows; i += nw) {
    const int64_t b = rowptr[i] - base, e = rowptr[i + 1] - base;
    for (int64_t j0 = 0; j0 < K; j0 += 32) {
      const int64_t j = j0 + lane;
      float a = 0.f;
      if (j < K)
        for (int64_t p = b; p < e; ++p) {
          const int64_t cc = col[p];
          if ((uint64_t)cc < (uint64_t)ncol) a = fmaf(val[p], D.p[cc * D.rs + j * D.cs], a);
        }
      if (j < K) {
        float* o = out.p + i * out.rs + j * out.cs;
        *o = (beta == 0.f) ? alpha * a : fmaf(beta, *o, alpha * a);
      }
    }
  }
}

// out(col[p], :) += alpha val[p] D(i, :) for every nonzero (i, col[p]) of a
// CSR matrix: the product with its transpose, scattered with atomics (the
// caller has applied beta to out).
__global__ void csr_t_spmm_kernel(const int64_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                                  const float* __restrict__ val, int64_t nrows, int64_t ncol, Mat D, int64_t K,
                                  MatOut out, float alpha) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t base = nrows > 0 ? rowptr[0] : 0;
  for (int64_t i = gw; i < nrows; i += nw) {
    const int64_t b = rowptr[i] - base, e = rowptr[i + 1] - base;
    for (int64_t p = b; p < e; ++p) {
      const int64_t cc = col[p];
      if ((uint64_t)cc >= (uint64_t)ncol) continue;
      const float v = alpha * val[p];
      for (int64_t j = lane; j < K; j += 32) atomicAdd(out.p + cc * out.rs + j * out.cs, v * D.p[i * D.rs + j * D.cs]);
    }
  }
}

bool trans_of(char t) {
  if (t == 'N' || t == 'n') return false;
  if (t == 'T' || t == 't') return true;
  fail(SKEMA_EINVAL, std::string("trans must be 'N' or 'T', got '") + t + "'");
}

// (rows, cols, strides) of a caller matrix descriptor on the device.
struct View {
  float* p;
  int64_t rows, cols, rs, cs;
};

View view_of(const skema_matf* m) {
  if (!m) fail(SKEMA_EINVAL, "null matrix descriptor");
  if (m->rows < 0 || m->cols < 0) fail(SKEMA_EINVAL, "negative matrix extent");
  if (m->layout != SKEMA_COL_MAJOR && m->layout != SKEMA_ROW_MAJOR) fail(SKEMA_EINVAL, "bad layout");
  const int64_t need = m->layout == SKEMA_COL_MAJOR ? m->rows : m->cols;
  if (m->rows > 0 && m->cols > 0) {
    if (!m->p) fail(SKEMA_EINVAL, "null matrix pointer");
    if (m->ld < std::max<int64_t>(need, 1)) fail(SKEMA_EINVAL, "leading dimension too small");
  }
  return m->layout == SKEMA_COL_MAJOR ? View{m->p, m->rows, m->cols, 1, m->ld} : View{m->p, m->rows, m->cols, m->ld, 1};
}

View transpose_if(View v, bool t) { return t ? View{v.p, v.cols, v.rows, v.cs, v.rs} : v; }

// Bytes a caller matrix spans from its pointer.
size_t span_bytes(const skema_matf* m) {
  if (m->rows == 0 || m->cols == 0) return 0;
  const int64_t outer = m->layout == SKEMA_COL_MAJOR ? m->cols : m->rows;
  const int64_t inner = m->layout == SKEMA_COL_MAJOR ? m->rows : m->cols;
  return sizeof(float) * (size_t)((outer - 1) * m->ld + inner);
}

// The map as a dense FP32 view (stored nrow x ncol, row-major), restricted to
// stored columns (lmap) or rows (rmap) [i0, i1) when i0 != i1.
View map_view(skema_dimredux* d, bool cols, int64_t i0, int64_t i1) {
  skema_ctx* c = d->c;
  Map& mp = d->map;
  float* base = mp.f32;  // Gauss: generated row-major (rs = ncol, cs = 1)
  if (mp.kind == SKEMA_MAP_SPARSE_SIGN) {
    if (!d->dense) {
      SKEMA_CUDA(cudaMalloc(&d->dense, sizeof(float) * (size_t)(mp.nrow * mp.ncol)));
      SKEMA_CUDA(cudaMemsetAsync(d->dense, 0, sizeof(float) * (size_t)(mp.nrow * mp.ncol), c->stream));
      ssign_expand_kernel<<<grid1d(c, mp.nrow, 256), 256, 0, c->stream>>>(mp.packed, mp.nrow, mp.ncol, mp.zeta,
                                                                         d->dense);
      SKEMA_LAUNCHED(c);
    }
    base = d->dense;
  }
  View v{base, mp.nrow, mp.ncol, mp.ncol, 1};
  if (i0 == i1) return v;
  const int64_t lim = cols ? mp.ncol : mp.nrow;
  if (i0 < 0 || i1 < i0 || i1 > lim) fail(SKEMA_EINVAL, "idx range outside the map");
  if (cols) return View{v.p + i0, v.rows, i1 - i0, v.rs, 1};
  return View{v.p + i0 * v.rs, i1 - i0, v.cols, v.rs, 1};
}

template <typename F>
int guarded_map(skema_dimredux* d, F&& f) {
  if (!d) return SKEMA_EINVAL;
  try {
    SKEMA_CUDA(cudaSetDevice(d->c->dev));
    f();
    d->err.clear();
    return SKEMA_OK;
  } catch (const Error& e) {
    d->err = e.msg;
    return e.status;
  } catch (const std::bad_alloc&) {
    d->err = "host allocation failed";
    return SKEMA_ENOMEM;
  } catch (...) {
    d->err = "unexpected C++ exception";
    return SKEMA_ECUDA;
  }
}

// Host operands are staged: the dense input (A or B) or the CSR arrays
// through the context's workspace, C through its staging buffer (C's old
// values are copied in when beta != 0).
View stage_in(skema_dimredux* d, const skema_matf* X, int32_t mem) {
  View x = view_of(X);
  if (mem == SKEMA_MEM_DEVICE) return x;
  if (mem != SKEMA_MEM_HOST) fail(SKEMA_EINVAL, "bad mem kind");
  const size_t bx = span_bytes(X);
  float* dx = static_cast<float*>(workspace(d->c, bx + 256));
  if (bx) SKEMA_CUDA(cudaMemcpyAsync(dx, X->p, bx, cudaMemcpyHostToDevice, d->c->stream));
  x.p = dx;
  return x;
}

View stage_out(skema_dimredux* d, skema_matf* C, float beta, int32_t mem) {
  View o = view_of(C);
  if (mem == SKEMA_MEM_DEVICE) return o;
  if (mem != SKEMA_MEM_HOST) fail(SKEMA_EINVAL, "bad mem kind");
  const size_t bc = span_bytes(C);
  float* dc = static_cast<float*>(staging(d->c, bc + 256));
  if (bc && beta != 0.f) SKEMA_CUDA(cudaMemcpyAsync(dc, C->p, bc, cudaMemcpyHostToDevice, d->c->stream));
  o.p = dc;
  return o;
}

void finish_host(skema_dimredux* d, skema_matf* C, const View& o, int32_t mem) {
  if (mem != SKEMA_MEM_HOST) return;
  const size_t bc = span_bytes(C);
  if (bc) SKEMA_CUDA(cudaMemcpyAsync(C->p, o.p, bc, cudaMemcpyDeviceToHost, d->c->stream));
  SKEMA_CUDA(cudaStreamSynchronize(d->c->stream));
}

void check_shape(const View& a, const View& b, const View& c) {
  if (a.cols != b.rows) fail(SKEMA_EINVAL, "inner dimensions of the product differ");
  if (c.rows != a.rows || c.cols != b.cols) fail(SKEMA_EINVAL, "output shape does not match the product");
}

// out = alpha op(S) D + beta out for a CSR S (rows x cols; op(S) = S^T when
// st) and a dense D, by the two SpMM kernels above.
void csr_times(skema_ctx* c, const skema_csrf* S, bool st, View D, View out, float alpha, float beta) {
  const int64_t inner = st ? S->rows : S->cols, orows = st ? S->cols : S->rows;
  if (D.rows != inner) fail(SKEMA_EINVAL, "inner dimensions of the product differ");
  if (out.rows != orows || out.cols != D.cols) fail(SKEMA_EINVAL, "output shape does not match the product");
  if (out.rows == 0 || out.cols == 0) return;
  const int grid = grid1d(c, S->rows * 32, 256);
  if (!st) {
    if (S->rows > 0)
      csr_spmm_kernel<<<grid, 256, 0, c->stream>>>(S->rowptr, S->col, S->val, S->rows, S->cols,
                                                   Mat{D.p, D.rs, D.cs}, D.cols, MatOut{out.p, out.rs, out.cs},
                                                   alpha, beta);
  } else {
    scale_block(c, MatOut{out.p, out.rs, out.cs}, out.rows, out.cols, beta);
    if (S->rows > 0)
      csr_t_spmm_kernel<<<grid, 256, 0, c->stream>>>(S->rowptr, S->col, S->val, S->rows, S->cols,
                                                     Mat{D.p, D.rs, D.cs}, D.cols, MatOut{out.p, out.rs, out.cs},
                                                     alpha);
  }
  SKEMA_LAUNCHED(c);
}

// A CSR operand on the device (host arrays staged through the workspace).
skema_csrf stage_csr(skema_dimredux* d, const skema_csrf* S, int32_t mem) {
  if (!S) fail(SKEMA_EINVAL, "null CSR descriptor");
  if (S->rows < 0 || S->cols < 0) fail(SKEMA_EINVAL, "negative CSR extent");
  if (S->rows > 0 && !S->rowptr) fail(SKEMA_EINVAL, "null rowptr");
  if (mem == SKEMA_MEM_DEVICE) return *S;
  if (mem != SKEMA_MEM_HOST) fail(SKEMA_EINVAL, "bad mem kind");
  if (S->rows == 0) return *S;
  const int64_t base = S->rowptr[0], nnz = S->rowptr[S->rows] - base;
  for (int64_t i = 0; i < S->rows; ++i)
    if (S->rowptr[i + 1] < S->rowptr[i]) fail(SKEMA_EINVAL, "rowptr is decreasing");
  if (nnz > 0 && (!S->col || !S->val)) fail(SKEMA_EINVAL, "null col/val");
  auto rup = [](size_t b) { return (b + 255) / 256 * 256; };
  const size_t brp = sizeof(int64_t) * (size_t)(S->rows + 1), bcol = sizeof(int32_t) * (size_t)nnz;
  char* ws = static_cast<char*>(workspace(d->c, rup(brp) + rup(bcol) + sizeof(float) * (size_t)nnz + 256));
  int64_t* rp = reinterpret_cast<int64_t*>(ws);
  int32_t* cl = reinterpret_cast<int32_t*>(ws + rup(brp));
  float* vl = reinterpret_cast<float*>(ws + rup(brp) + rup(bcol));
  skema_ctx* c = d->c;
  SKEMA_CUDA(cudaMemcpyAsync(rp, S->rowptr, brp, cudaMemcpyHostToDevice, c->stream));
  if (nnz) {
    SKEMA_CUDA(cudaMemcpyAsync(cl, S->col + base, bcol, cudaMemcpyHostToDevice, c->stream));
    SKEMA_CUDA(cudaMemcpyAsync(vl, S->val + base, sizeof(float) * (size_t)nnz, cudaMemcpyHostToDevice, c->stream));
  }
  return skema_csrf{rp, cl, vl, S->rows, S->cols};
}

}  // namespace
}  // namespace skema

using namespace skema;

extern "C" {

int skema_dimredux_create(int32_t kind, int64_t nrow, int64_t ncol, int32_t seed, int32_t device,
                          skema_dimredux** out) {
  if (!out) return SKEMA_EINVAL;
  *out = nullptr;
  if (kind != SKEMA_MAP_GAUSS && kind != SKEMA_MAP_SPARSE_SIGN) return SKEMA_EINVAL;
  if (nrow <= 0 || ncol <= 0 || ncol >= (int64_t(1) << 31) || nrow >= (int64_t(1) << 40)) return SKEMA_EINVAL;
  skema_params p;
  skema_params_init(&p);
  p.matrix_m = p.matrix_n = 1;
  p.device = device;
  skema_dimredux* d = new (std::nothrow) skema_dimredux();
  if (!d) return SKEMA_ENOMEM;
  int st = skema_create(&p, &d->c);
  if (st != SKEMA_OK) {
    delete d;
    return st;
  }
  st = guarded_map(d, [&] {
    Map& mp = d->map;
    mp.kind = kind;
    mp.nrow = nrow;
    mp.ncol = ncol;
    mp.transposed = false;
    mp.lrows = nrow;
    mp.lcols = ncol;
    mp.seed = (uint32_t)seed;
    map_generate(d->c, mp, SKEMA_PREC_FP32);
    SKEMA_CUDA(cudaStreamSynchronize(d->c->stream));
  });
  if (st != SKEMA_OK) {
    skema_dimredux_destroy(d);
    return st;
  }
  *out = d;
  return SKEMA_OK;
}

int skema_dimredux_destroy(skema_dimredux* d) {
  if (!d) return SKEMA_OK;
  if (d->c) {
    cudaSetDevice(d->c->dev);
    cudaStreamSynchronize(d->c->stream);
    map_free(d->map);
    if (d->dense) cudaFree(d->dense);
    skema_destroy(d->c);
  }
  delete d;
  return SKEMA_OK;
}

const char* skema_dimredux_last_error(const skema_dimredux* d) { return d ? d->err.c_str() : ""; }

int skema_dimredux_export(skema_dimredux* d, double* values, int32_t* indices) {
  return guarded_map(d, [&] { map_export(d->c, d->map, values, indices); });
}

int skema_dimredux_lmap(skema_dimredux* d, double alpha, const skema_matf* B, double beta, char transA, char transB,
                        int64_t idx_first, int64_t idx_second, skema_matf* C, int32_t mem) {
  return guarded_map(d, [&] {
    const bool ta = trans_of(transA), tb = trans_of(transB);
    const View in = stage_in(d, B, mem);
    const View o = stage_out(d, C, (float)beta, mem);
    const View a = transpose_if(map_view(d, true, idx_first, idx_second), ta);
    const View b = transpose_if(in, tb);
    check_shape(a, b, o);
    sgemm(d->c, a.rows, b.cols, a.cols, (float)alpha, Mat{a.p, a.rs, a.cs}, Mat{b.p, b.rs, b.cs}, (float)beta,
          MatOut{o.p, o.rs, o.cs});
    finish_host(d, C, o, mem);
  });
}

int skema_dimredux_rmap(skema_dimredux* d, double alpha, const skema_matf* A, double beta, char transA, char transB,
                        int64_t idx_first, int64_t idx_second, skema_matf* C, int32_t mem) {
  return guarded_map(d, [&] {
    const bool ta = trans_of(transA), tb = trans_of(transB);
    const View in = stage_in(d, A, mem);
    const View o = stage_out(d, C, (float)beta, mem);
    const View a = transpose_if(in, ta);
    const View b = transpose_if(map_view(d, false, idx_first, idx_second), tb);
    check_shape(a, b, o);
    sgemm(d->c, a.rows, b.cols, a.cols, (float)alpha, Mat{a.p, a.rs, a.cs}, Mat{b.p, b.rs, b.cs}, (float)beta,
          MatOut{o.p, o.rs, o.cs});
    finish_host(d, C, o, mem);
  });
}

int skema_dimredux_lmap_csr(skema_dimredux* d, double alpha, const skema_csrf* B, double beta, char transA,
                            char transB, int64_t idx_first, int64_t idx_second, skema_matf* C, int32_t mem) {
  return guarded_map(d, [&] {
    const bool ta = trans_of(transA), tb = trans_of(transB);
    const View o = stage_out(d, C, (float)beta, mem);
    const skema_csrf S = stage_csr(d, B, mem);
    const View m = transpose_if(map_view(d, true, idx_first, idx_second), ta);
    // C = op(M) op(B)  <=>  C^T = op(B)^T op(M)^T
    const View mt = transpose_if(m, true);
    const View ot = transpose_if(o, true);
    csr_times(d->c, &S, !tb, mt, ot, (float)alpha, (float)beta);
    finish_host(d, C, o, mem);
  });
}

int skema_dimredux_rmap_csr(skema_dimredux* d, double alpha, const skema_csrf* A, double beta, char transA,
                            char transB, int64_t idx_first, int64_t idx_second, skema_matf* C, int32_t mem) {
  return guarded_map(d, [&] {
    const bool ta = trans_of(transA), tb = trans_of(transB);
    const View o = stage_out(d, C, (float)beta, mem);
    const skema_csrf S = stage_csr(d, A, mem);
    const View m = transpose_if(map_view(d, false, idx_first, idx_second), tb);
    csr_times(d->c, &S, ta, m, o, (float)alpha, (float)beta);
    finish_host(d, C, o, mem);
  });
}

}  // extern "C"
