// maps.cu -- generation, import and export of the four DimRedux maps.
//
// Gauss maps (GaussDimRedux ctor, src/Skema_DimRedux.hpp:98-128) are written
// as FP32 in the layout the sketch kernels read: logical rows contiguous for
// dense and kernel inputs (the maps are the left/right GEMM operands), stored
// rows contiguous for CSR inputs (rows of the stored map are gathered per
// nonzero). SparseSign maps (src/Skema_DimRedux.hpp:191-268) are kept as
// zeta packed words per stored row: column | sign << 31.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "internal.h"
#include "philox.h"

namespace skema {

__global__ void gauss_map_kernel(float* __restrict__ out, int64_t lrows, int64_t lcols,
                                 int64_t rs, int64_t cs, int64_t nrow, int transposed,
                                 uint32_t seed, double maxval) {
  const int64_t total = lrows * lcols;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total;
       q += (int64_t)gridDim.x * blockDim.x) {
    // Walk the output buffer contiguously: q is the memory order index.
    int64_t r, c;
    if (cs == 1) {
      r = q / lcols;
      c = q - r * lcols;
    } else {
      c = q / lrows;
      r = q - c * lrows;
    }
    const int64_t i = transposed ? c : r;  // stored row
    const int64_t j = transposed ? r : c;  // stored col
    const uint64_t e = (uint64_t)(i + j * nrow);
    out[r * rs + c * cs] = (float)gauss_entry(seed, e, maxval);
  }
}

__global__ void sparse_sign_map_kernel(uint32_t* __restrict__ packed, int64_t nrow,
                                       uint32_t ncol, int zeta, uint32_t seed) {
  for (int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; row < nrow;
       row += (int64_t)gridDim.x * blockDim.x) {
    uint32_t idx[8], neg[8];
    sparse_sign_row(seed, (uint64_t)row, ncol, zeta, idx, neg);
    for (int t = 0; t < zeta; ++t) packed[row * zeta + t] = idx[t] | (neg[t] << 31);
  }
}

// Offset form of a SparseSign map with zeta = 8 and at most 256 columns:
// eight 16-bit entries per stored row, entry t
// = (column * 128) | sign << 15 | dup, i.e. the byte offset of bin `column`
// in a warp's bin-major accumulator (32 floats per bin) with the sign on top.
// The entries are stably sorted by column (generated rows already are), and
// bit 0 (dup) marks an entry whose column equals the previous entry's: the
// sketch kernel then adds it to the previous entry's sum rather than to a
// value it loaded before that sum was stored. Stable order keeps the
// additions into each bin in entry order.
__global__ void pack16_kernel(const uint32_t* __restrict__ packed, uint4* __restrict__ out, int64_t nrow) {
  for (int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; row < nrow;
       row += (int64_t)gridDim.x * blockDim.x) {
    uint32_t h[8];
    for (int t = 0; t < 8; ++t) {
      const uint32_t e = packed[row * 8 + t];
      h[t] = ((e & 0xffu) << 7) | ((e >> 31) << 15);
    }
    for (int t = 1; t < 8; ++t) {  // stable insertion sort on the column bits
      const uint32_t v = h[t];
      int u = t - 1;
      while (u >= 0 && (h[u] & 0x7f80u) > (v & 0x7f80u)) {
        h[u + 1] = h[u];
        --u;
      }
      h[u + 1] = v;
    }
    for (int t = 1; t < 8; ++t) h[t] |= (h[t] & 0x7f80u) == (h[t - 1] & 0x7f80u) ? 1u : 0u;
    out[row] = make_uint4(h[0] | (h[1] << 16), h[2] | (h[3] << 16), h[4] | (h[5] << 16), h[6] | (h[7] << 16));
  }
}

// Import path: logical FP32 layout from stored column-major doubles.
__global__ void gauss_import_kernel(float* __restrict__ out, const double* __restrict__ stored,
                                    int64_t lrows, int64_t lcols, int64_t rs, int64_t cs,
                                    int64_t nrow, int transposed) {
  const int64_t total = lrows * lcols;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = q % lrows, c = q / lrows;
    const int64_t i = transposed ? c : r;
    const int64_t j = transposed ? r : c;
    out[r * rs + c * cs] = (float)stored[i + j * nrow];
  }
}

static int grid_for(int64_t total, int threads, int sms) {
  const int64_t want = (total + threads - 1) / threads;
  return (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)sms * 32));
}

static void build_pack16(skema_ctx* c, Map& mp) {
  if (mp.kind != SKEMA_MAP_SPARSE_SIGN || !mp.transposed) return;
  if (mp.zeta != 8 || mp.ncol > 256) return;
  if (!mp.packed16) SKEMA_CUDA(cudaMalloc(&mp.packed16, sizeof(uint4) * (size_t)mp.nrow));
  pack16_kernel<<<grid_for(mp.nrow, 256, c->sm_count), 256, 0, c->stream>>>(
      mp.packed, reinterpret_cast<uint4*>(mp.packed16), mp.nrow);
  SKEMA_LAUNCHED(c);
}

static void gauss_layout(const skema_ctx* c, Map& mp) {
  if (c->p.issparse) {
    // stored rows contiguous: logical (r, col) = stored (col, r) at col*lrows + r
    mp.rs = 1;
    mp.cs = mp.lrows;
  } else {
    mp.rs = mp.lcols;
    mp.cs = 1;
  }
}

void map_generate(skema_ctx* c, Map& mp, int precision) {
  (void)precision;
  if (mp.kind == SKEMA_MAP_GAUSS) {
    mp.maxval = std::sqrt(2.0 * std::log((double)((uint64_t)mp.nrow * (uint64_t)mp.ncol)));
    gauss_layout(c, mp);
    SKEMA_CUDA(cudaMalloc(&mp.f32, sizeof(float) * (size_t)(mp.lrows * mp.lcols)));
    const int threads = 256;
    gauss_map_kernel<<<grid_for(mp.lrows * mp.lcols, threads, c->sm_count), threads, 0, c->stream>>>(
        mp.f32, mp.lrows, mp.lcols, mp.rs, mp.cs, mp.nrow, mp.transposed ? 1 : 0, mp.seed,
        mp.maxval);
    SKEMA_LAUNCHED(c);
  } else {
    mp.zeta = sparse_sign_zeta(mp.ncol);
    SKEMA_CUDA(cudaMalloc(&mp.packed, sizeof(uint32_t) * (size_t)(mp.nrow * mp.zeta)));
    const int threads = 256;
    sparse_sign_map_kernel<<<grid_for(mp.nrow, threads, c->sm_count), threads, 0, c->stream>>>(
        mp.packed, mp.nrow, (uint32_t)mp.ncol, mp.zeta, mp.seed);
    SKEMA_LAUNCHED(c);
    build_pack16(c, mp);
  }
}

void map_free(Map& mp) {
  if (mp.f32) cudaFree(mp.f32);
  if (mp.lowp) cudaFree(mp.lowp);
  if (mp.packed) cudaFree(mp.packed);
  if (mp.packed16) cudaFree(mp.packed16);
  mp.packed16 = nullptr;
  if (mp.d_inv_row) cudaFree(mp.d_inv_row);
  if (mp.d_inv_rs) cudaFree(mp.d_inv_rs);
  mp.f32 = nullptr;
  mp.lowp = nullptr;
  mp.packed = nullptr;
  mp.d_inv_row = nullptr;
  mp.d_inv_rs = nullptr;
  mp.inv_row.clear();
}

// For a SparseSign map that is row-sparse over the input rows (Upsilon~ and
// Phi~, k x m / s x m with zeta entries per map row): the list of
// (input row, map row, sign) sorted by input row, which is what
// col_subview (src/Skema_DimRedux_SparseSign.cpp:125-155) extracts per window.
void map_build_inverse(skema_ctx* c, Map& mp) {
  if (mp.kind != SKEMA_MAP_SPARSE_SIGN || mp.transposed) return;
  const int64_t ne = mp.nrow * mp.zeta;
  std::vector<uint32_t> h(ne);
  SKEMA_CUDA(cudaMemcpyAsync(h.data(), mp.packed, sizeof(uint32_t) * ne, cudaMemcpyDeviceToHost,
                             c->stream));
  SKEMA_CUDA(cudaStreamSynchronize(c->stream));
  struct Tri {
    int64_t in_row;
    uint32_t rs;
  };
  std::vector<Tri> t(ne);
  for (int64_t r = 0; r < mp.nrow; ++r)
    for (int z = 0; z < mp.zeta; ++z) {
      const uint32_t w = h[r * mp.zeta + z];
      t[r * mp.zeta + z] = Tri{(int64_t)(w & 0x7fffffffu), (uint32_t)r | (w & 0x80000000u)};
    }
  std::stable_sort(t.begin(), t.end(), [](const Tri& a, const Tri& b) { return a.in_row < b.in_row; });
  mp.inv_row.resize(ne);
  std::vector<uint32_t> rs(ne);
  for (int64_t q = 0; q < ne; ++q) {
    mp.inv_row[q] = t[q].in_row;
    rs[q] = t[q].rs;
  }
  if (mp.d_inv_row) cudaFree(mp.d_inv_row);
  if (mp.d_inv_rs) cudaFree(mp.d_inv_rs);
  mp.d_inv_row = nullptr;
  mp.d_inv_rs = nullptr;
  SKEMA_CUDA(cudaMalloc(&mp.d_inv_row, sizeof(int64_t) * std::max<int64_t>(ne, 1)));
  SKEMA_CUDA(cudaMalloc(&mp.d_inv_rs, sizeof(uint32_t) * std::max<int64_t>(ne, 1)));
  SKEMA_CUDA(cudaMemcpyAsync(mp.d_inv_row, mp.inv_row.data(), sizeof(int64_t) * ne,
                             cudaMemcpyHostToDevice, c->stream));
  SKEMA_CUDA(cudaMemcpyAsync(mp.d_inv_rs, rs.data(), sizeof(uint32_t) * ne, cudaMemcpyHostToDevice,
                             c->stream));
  SKEMA_CUDA(cudaStreamSynchronize(c->stream));
}

void map_export(skema_ctx* c, Map& mp, double* values, int32_t* indices) {
  if (mp.kind == SKEMA_MAP_GAUSS) {
    if (!values) fail(SKEMA_EINVAL, "values buffer required for a Gauss map");
    // FP32 copy back, widened; stored column-major orientation.
    const int64_t total = mp.lrows * mp.lcols;
    std::vector<float> h(total);
    SKEMA_CUDA(cudaMemcpyAsync(h.data(), mp.f32, sizeof(float) * total, cudaMemcpyDeviceToHost,
                               c->stream));
    SKEMA_CUDA(cudaStreamSynchronize(c->stream));
    for (int64_t i = 0; i < mp.nrow; ++i)
      for (int64_t j = 0; j < mp.ncol; ++j) {
        const int64_t r = mp.transposed ? j : i, col = mp.transposed ? i : j;
        values[i + j * mp.nrow] = (double)h[r * mp.rs + col * mp.cs];
      }
    return;
  }
  if (!values || !indices) fail(SKEMA_EINVAL, "values and indices required for a SparseSign map");
  const int64_t ne = mp.nrow * mp.zeta;
  std::vector<uint32_t> h(ne);
  SKEMA_CUDA(cudaMemcpyAsync(h.data(), mp.packed, sizeof(uint32_t) * ne, cudaMemcpyDeviceToHost,
                             c->stream));
  SKEMA_CUDA(cudaStreamSynchronize(c->stream));
  for (int64_t q = 0; q < ne; ++q) {
    indices[q] = (int32_t)(h[q] & 0x7fffffffu);
    values[q] = (h[q] >> 31) ? -1.0 : 1.0;
  }
}

void map_import(skema_ctx* c, Map& mp, const double* values, const int32_t* indices) {
  if (mp.kind == SKEMA_MAP_GAUSS) {
    if (!values) fail(SKEMA_EINVAL, "values buffer required for a Gauss map");
    const int64_t total = mp.nrow * mp.ncol;
    double* d = (double*)workspace(c, sizeof(double) * (size_t)total);
    SKEMA_CUDA(cudaMemcpyAsync(d, values, sizeof(double) * total, cudaMemcpyHostToDevice, c->stream));
    const int threads = 256;
    gauss_import_kernel<<<grid_for(total, threads, c->sm_count), threads, 0, c->stream>>>(
        mp.f32, d, mp.lrows, mp.lcols, mp.rs, mp.cs, mp.nrow, mp.transposed ? 1 : 0);
    SKEMA_LAUNCHED(c);
    SKEMA_CUDA(cudaStreamSynchronize(c->stream));
    return;
  }
  if (!values || !indices) fail(SKEMA_EINVAL, "values and indices required for a SparseSign map");
  const int64_t ne = mp.nrow * mp.zeta;
  std::vector<uint32_t> h(ne);
  for (int64_t q = 0; q < ne; ++q) {
    if (indices[q] < 0 || indices[q] >= mp.ncol) fail(SKEMA_EINVAL, "sparse-sign index out of range");
    if (values[q] != 1.0 && values[q] != -1.0) fail(SKEMA_EINVAL, "sparse-sign values must be +-1");
    h[q] = (uint32_t)indices[q] | (values[q] < 0 ? 0x80000000u : 0u);
  }
  SKEMA_CUDA(cudaMemcpyAsync(mp.packed, h.data(), sizeof(uint32_t) * ne, cudaMemcpyHostToDevice,
                             c->stream));
  build_pack16(c, mp);
  SKEMA_CUDA(cudaStreamSynchronize(c->stream));
  map_build_inverse(c, mp);
}

}  // namespace skema
