// dense_tc.cu -- the BF16 tensor-core form of the dense Gauss sketch
// (update(dense, Gauss), src/Skema_SketchySVD.cpp:256-268).
//
// Per window A_w (rows [R0, R0+wr)), FP32 accumulation throughout:
//   A16          = bf16(A_w)                    row-blocked (64-row blocks)
//   [Y_w | T]    = A16 [Omega~; Psi~]^T         M = wr, N = k + s, K = n
//                  (Y_w -> Y with eta / nu, T -> BF16 scratch, column-major)
//   X^T          = nu X^T + eta A16^T Upsilon~_w^T   M = n, N = k, K = wr
//   Z^T          = nu Z^T + eta T^T Phi~_w^T         M = s, N = s, K = wr
// Each product is oriented so that its output's contiguous dimension runs
// along the tile rows (TMEM lanes): Y and T are column-major, X and Z
// row-major, so X^T and Z^T are the products that store coalesced.
// The maps are kept as BF16 row-major copies (Upsilon~ k x m, Phi~ s x m,
// and Omega~ / Psi~ stacked into one (k+s) x n operand); every BF16 row
// stride is padded to a multiple of 8 elements (16 bytes) for TMA.
//
// Split-K: with one 128-row CTA per SM a product with few tiles leaves SMs
// idle (157 X tiles on 148 SMs is two waves, the second nearly empty), so K
// is split when that shortens the critical path; the split partial sums are
// added with FP32 atomics into outputs scaled by nu beforehand.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

#include "internal.h"
#include "tc_host.h"

namespace skema {

namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  if (!fn) fail(SKEMA_ENOKERNEL, "cuTensorMapEncodeTiled is not available from the driver");
  return fn;
}

}  // namespace

CUtensorMap tmap_2d(CUtensorMapDataType dtype, const void* base, uint64_t d0, uint64_t d1, uint64_t st1,
                    uint32_t b0, uint32_t b1, CUtensorMapSwizzle swizzle) {
  if (reinterpret_cast<uintptr_t>(base) % 16) fail(SKEMA_EINVAL, "TMA base address not 16-byte aligned");
  if (st1 % 16) fail(SKEMA_EINVAL, "TMA row stride not a multiple of 16 bytes");
  CUtensorMap tm;
  cuuint64_t dims[2] = {d0, d1};
  cuuint64_t strides[1] = {st1};
  cuuint32_t box[2] = {b0, b1};
  cuuint32_t es[2] = {1, 1};
  const CUresult r = encode_fn()(&tm, dtype, 2, const_cast<void*>(base), dims, strides, box, es,
                                 CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) fail(SKEMA_EINVAL, "cuTensorMapEncodeTiled rejected a 2-D tensor map");
  return tm;
}

CUtensorMap tmap_3d(CUtensorMapDataType dtype, const void* base, uint64_t d0, uint64_t d1, uint64_t d2,
                    uint64_t st1, uint64_t st2, uint32_t b0, uint32_t b1, uint32_t b2,
                    CUtensorMapSwizzle swizzle) {
  if (reinterpret_cast<uintptr_t>(base) % 16) fail(SKEMA_EINVAL, "TMA base address not 16-byte aligned");
  if (st1 % 16 || st2 % 16) fail(SKEMA_EINVAL, "TMA stride not a multiple of 16 bytes");
  CUtensorMap tm;
  cuuint64_t dims[3] = {d0, d1, d2};
  cuuint64_t strides[2] = {st1, st2};
  cuuint32_t box[3] = {b0, b1, b2};
  cuuint32_t es[3] = {1, 1, 1};
  const CUresult r = encode_fn()(&tm, dtype, 3, const_cast<void*>(base), dims, strides, box, es,
                                 CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) fail(SKEMA_EINVAL, "cuTensorMapEncodeTiled rejected a 3-D tensor map");
  return tm;
}

CUtensorMap tmap_bf16(const void* base, uint64_t d0, uint64_t d1, uint64_t st1, uint32_t b0, uint32_t b1) {
  return tmap_2d(CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, base, d0, d1, st1, b0, b1, CU_TENSOR_MAP_SWIZZLE_128B);
}

Plan plan_split(const skema_ctx* c, int64_t tiles, int64_t K, int max_ks) {
  const int64_t ksteps = (K + tc::BK - 1) / tc::BK;
  const int64_t ctas = c->tc_cta_cap > 0 ? std::min(c->tc_cta_cap, c->sm_count) : c->sm_count;
  int best = 1;
  double best_cost = 1e300;
  for (int ks = 1; ks <= max_ks; ++ks) {
    if (ks > 1 && ksteps / ks < 8) break;  // at least 8 k-steps per split
    const int64_t waves = (tiles * ks + ctas - 1) / ctas;
    // a split adds atomic partial sums to every output element; their cost
    // shows as about 12 k-steps per wave
    const double cost = (double)waves * ((double)ksteps / ks + 6.0 + (ks > 1 ? 12.0 : 0.0));
    if (cost < best_cost * 0.97) {
      best_cost = cost;
      best = ks;
    }
  }
  const int64_t kchunk = (ksteps + best - 1) / best * tc::BK;
  const int ks = (int)((K + kchunk - 1) / kchunk);
  return Plan{ks, kchunk};
}

Plan plan_streamk(const skema_ctx* c, int ctas) {
  Plan p{1, 0};
  p.streamk = std::max(1, std::min(ctas, c->sm_count));
  return p;
}

tc::OutSpec out_spec() {
  tc::OutSpec o;
  o.p0 = nullptr, o.p1 = nullptr, o.p1lo = nullptr, o.p1f = nullptr;
  o.rs0 = o.cs0 = o.rs1 = o.cs1 = 0;
  o.alpha0 = 1.f, o.beta0 = 0.f, o.alpha1 = 1.f, o.beta1 = 0.f;
  o.rows = 0, o.split = 0, o.ncols = 0;
  o.atomic0 = 0, o.atomic1 = 0;
  o.row_log2w = 0.f, o.row_wlen = 1, o.row_nwin = 1;
  o.scale = nullptr;
  o.scale_wlen = 1;
  return o;
}

namespace {

constexpr int kNT = 208;  // N tile of every product (k = 201, s = 403 pad to 208 / 416)

// 2-D FP32 map, 128-byte swizzle (box inner extent 32).
CUtensorMap tmap_f32(const void* base, uint64_t d0, uint64_t d1, uint64_t st1, uint32_t b0, uint32_t b1) {
  return tmap_2d(CU_TENSOR_MAP_DATA_TYPE_FLOAT32, base, d0, d1, st1, b0, b1, CU_TENSOR_MAP_SWIZZLE_128B);
}

// 3-D BF16 map of the row-blocked window: {64, d1, d2} with the 64-element
// lines contiguous, byte strides 128 (dim1) and d1 * 128 (dim2), box
// {64, b1, 1}.
CUtensorMap tmap_bf16_blocked(const void* base, uint64_t d1, uint64_t d2, uint32_t b1) {
  return tmap_3d(CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, base, 64, d1, d2, 128, d1 * 128, 64, b1, 1,
                 CU_TENSOR_MAP_SWIZZLE_128B);
}
// The window in BF16, row-blocked: element (i, j) of a rows x cols block at
// D[((i / 64) * cols + j) * 64 + i % 64], i.e. for each 64-row block the
// columns one after another, each a 128-byte line of 64 rows. Rows past
// `rows` in the last block are written as zeros. A TMA box of 64 rows x
// 64 or 128 columns is then one contiguous 8 or 16 KB run, read MN-major by
// the [Y|T] product and K-major by the X product.
__global__ void to_bf16_blocked_vec_kernel(const float* __restrict__ S, int64_t scs, int64_t rows,
                                           int64_t cols, __nv_bfloat16* __restrict__ D, int64_t nrb) {
  const int64_t g8 = nrb * 8;  // 8-row groups, padding included
  const int64_t total = g8 * cols;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = q / g8, i = (q - j * g8) * 8;
    const float* sp = S + i + j * scs;
    float v[8];
    if (i + 8 <= rows) {
      const float4 a = __ldcs(reinterpret_cast<const float4*>(sp));
      const float4 b = __ldcs(reinterpret_cast<const float4*>(sp + 4));
      v[0] = a.x, v[1] = a.y, v[2] = a.z, v[3] = a.w, v[4] = b.x, v[5] = b.y, v[6] = b.z, v[7] = b.w;
    } else {
      for (int t = 0; t < 8; ++t) v[t] = (i + t < rows) ? sp[t] : 0.f;
    }
    __nv_bfloat162 h[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) h[t] = __floats2bfloat162_rn(v[2 * t], v[2 * t + 1]);
    *reinterpret_cast<uint4*>(D + ((i >> 6) * cols + j) * 64 + (i & 63)) = *reinterpret_cast<const uint4*>(h);
  }
}

// The same layout from any strided FP32 block, 64 x 32 tiles through shared
// memory (reads along the source's unit stride, writes 128-byte lines).
__global__ void to_bf16_blocked_tiled_kernel(const float* __restrict__ S, int64_t srs, int64_t scs, int64_t rows,
                                             int64_t cols, __nv_bfloat16* __restrict__ D, int64_t nrb) {
  __shared__ float tile[64][33];
  const int64_t tj = (cols + 31) / 32;
  const bool s_rowfast = srs <= scs;
  for (int64_t t = blockIdx.x; t < nrb * tj; t += gridDim.x) {
    const int64_t rb = t / tj, j0 = (t - rb * tj) * 32;
    if (s_rowfast) {
      for (int q = threadIdx.y; q < 32; q += blockDim.y)
        for (int h = 0; h < 2; ++h) {
          const int r = threadIdx.x + 32 * h;
          const int64_t i = rb * 64 + r, j = j0 + q;
          tile[r][q] = (i < rows && j < cols) ? S[i * srs + j * scs] : 0.f;
        }
    } else {
      for (int r = threadIdx.y; r < 64; r += blockDim.y) {
        const int64_t i = rb * 64 + r, j = j0 + threadIdx.x;
        tile[r][threadIdx.x] = (i < rows && j < cols) ? S[i * srs + j * scs] : 0.f;
      }
    }
    __syncthreads();
    for (int q = threadIdx.y; q < 32; q += blockDim.y) {
      const int64_t j = j0 + q;
      if (j < cols) {
        const int r = 2 * threadIdx.x;
        *reinterpret_cast<__nv_bfloat162*>(D + (rb * cols + j) * 64 + r) =
            __floats2bfloat162_rn(tile[r][q], tile[r + 1][q]);
      }
    }
    __syncthreads();
  }
}

void to_bf16_blocked(skema_ctx* c, Mat src, int64_t rows, int64_t cols, __nv_bfloat16* D) {
  const int64_t nrb = (rows + 63) / 64;
  if (nrb <= 0 || cols <= 0) return;
  const bool vec = src.rs == 1 && src.cs % 4 == 0 && reinterpret_cast<uintptr_t>(src.p) % 16 == 0;
  if (vec) {
    const int64_t work = nrb * 8 * cols;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((work + 255) / 256, (int64_t)c->sm_count * 16));
    to_bf16_blocked_vec_kernel<<<grid, 256, 0, c->stream>>>(src.p, src.cs, rows, cols, D, nrb);
  } else {
    const int64_t tiles = nrb * ((cols + 31) / 32);
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(tiles, (int64_t)c->sm_count * 16));
    to_bf16_blocked_tiled_kernel<<<grid, dim3(32, 8), 0, c->stream>>>(src.p, src.rs, src.cs, rows, cols, D, nrb);
  }
  SKEMA_LAUNCHED(c);
}

// Any strided FP32 block -> BF16 with D(i, j) at D[i * drs + j * dcs], by
// 32 x 32 tiles through shared memory so that both the read (along the
// source's unit stride) and the write (along the destination's) coalesce.
__global__ void to_bf16_tiled_kernel(const float* __restrict__ S, int64_t srs, int64_t scs, int64_t rows,
                                     int64_t cols, __nv_bfloat16* __restrict__ D, int64_t drs, int64_t dcs) {
  __shared__ float tile[32][33];
  const int64_t ti = (rows + 31) / 32, tj = (cols + 31) / 32;
  const bool s_rowfast = srs <= scs;  // source unit stride along i
  const bool d_rowfast = drs <= dcs;
  for (int64_t t = blockIdx.x; t < ti * tj; t += gridDim.x) {
    const int64_t i0 = (t % ti) * 32, j0 = (t / ti) * 32;
    for (int q = threadIdx.y; q < 32; q += blockDim.y) {
      const int64_t i = s_rowfast ? i0 + threadIdx.x : i0 + q;
      const int64_t j = s_rowfast ? j0 + q : j0 + threadIdx.x;
      const float v = (i < rows && j < cols) ? S[i * srs + j * scs] : 0.f;
      if (s_rowfast)
        tile[threadIdx.x][q] = v;
      else
        tile[q][threadIdx.x] = v;
    }
    __syncthreads();
    for (int q = threadIdx.y; q < 32; q += blockDim.y) {
      const int64_t i = d_rowfast ? i0 + threadIdx.x : i0 + q;
      const int64_t j = d_rowfast ? j0 + q : j0 + threadIdx.x;
      const float v = d_rowfast ? tile[threadIdx.x][q] : tile[q][threadIdx.x];
      if (i < rows && j < cols) D[i * drs + j * dcs] = __float2bfloat16(v);
    }
    __syncthreads();
  }
}

}  // namespace

void to_bf16(skema_ctx* c, Mat src, int64_t rows, int64_t cols, __nv_bfloat16* D, int64_t drs, int64_t dcs) {
  if (rows <= 0 || cols <= 0) return;
  const int64_t tiles = ((rows + 31) / 32) * ((cols + 31) / 32);
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(tiles, (int64_t)c->sm_count * 16));
  to_bf16_tiled_kernel<<<grid, dim3(32, 8), 0, c->stream>>>(src.p, src.rs, src.cs, rows, cols, D, drs, dcs);
  SKEMA_LAUNCHED(c);
}

namespace {

// BF16 column-major (ld) <- FP32 column-major (ld), rows x cols, and the
// BF16 rounding of the remainder into L (when given).
__global__ void f32_to_bf16_cm_kernel(const float* __restrict__ S, int64_t lds, __nv_bfloat16* __restrict__ D,
                                      __nv_bfloat16* __restrict__ L, int64_t ldd, int64_t rows, int64_t cols) {
  const int64_t total = rows * cols;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = q / rows, i = q - j * rows;
    const float x = S[i + j * lds];
    const __nv_bfloat16 hi = __float2bfloat16(x);
    D[i + j * ldd] = hi;
    if (L) L[i + j * ldd] = __float2bfloat16(x - __bfloat162float(hi));
  }
}

// Persistent launch: min(units, SMs) CTAs of one per SM (the 5-stage ring
// takes 211 KB of shared memory).
// Tiles, K-steps and schedule of one launch; *grid gets the CTA count.
tc::Grid3 grid_of(const skema_ctx* c, int64_t M, int64_t N, int64_t K, int nt, int bk, const Plan& pl, int m_fast,
                  int* grid) {
  tc::Grid3 g;
  g.mtiles = (int)((M + tc::BM - 1) / tc::BM);
  g.ntiles = (int)((N + nt - 1) / nt);
  g.ksplit = pl.ks;
  g.m_fast = m_fast;
  g.ksteps = (K + bk - 1) / bk;
  g.kcsteps = pl.kchunk > 0 ? (int)(pl.kchunk / bk) : (int)g.ksteps;
  g.streamk = pl.streamk > 0 ? 1 : 0;
  const int64_t units = (int64_t)g.mtiles * g.ntiles * (g.streamk ? g.ksteps : g.ksplit);
  if (units > 0x7fffffff) fail(SKEMA_EINVAL, "tensor-core grid too large");
  *grid = (int)std::min<int64_t>(units, g.streamk ? pl.streamk : c->sm_count);
  if (c->tc_cta_cap > 0) *grid = std::min(*grid, c->tc_cta_cap);
  if (M <= 0 || N <= 0 || K <= 0) *grid = 0;
  return g;
}

template <int AMODE>
void launch_gemm(skema_ctx* c, const CUtensorMap& ta, const CUtensorMap& tb, int64_t M, int64_t N, int64_t K,
                 Plan pl, int m_fast, const tc::OutSpec& o) {
  constexpr int S = 5;
  constexpr uint32_t STAGE = ((tc::BM * tc::BK * 2 + kNT * tc::BK * 2 + 1023) / 1024) * 1024;
  const size_t smem = (size_t)S * STAGE + 1024 + 256;
  auto kern = tc::gemm_bf16_kernel<kNT, S, AMODE>;
  SKEMA_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int grid = 0;
  const tc::Grid3 g = grid_of(c, M, N, K, kNT, tc::BK, pl, m_fast, &grid);
  if (grid <= 0) return;
  kern<<<grid, tc::kThreads, smem, c->stream>>>(ta, tb, g, o, c->dev_err);
  SKEMA_LAUNCHED(c);
  c->dev_err_armed = true;
}

// X^T product straight from the FP32 window (converts it and writes A16).
template <bool AROW, int S1, int S2, bool STT>
void launch_gemm_a32_s(skema_ctx* c, const CUtensorMap& ta32, const CUtensorMap& tb, const CUtensorMap& ta16,
                       int64_t M, int64_t N, int64_t K, Plan pl, const tc::OutSpec& o, uint32_t* amax) {
  constexpr uint32_t STAGE = ((tc::BM * tc::BK * 2 + kNT * tc::BK * 2 + 1023) / 1024) * 1024;
  const size_t smem = (size_t)S1 * tc::BM * tc::BK * 4 + (size_t)S2 * STAGE + 1024 + 256;
  auto kern = amax ? tc::gemm_a32_kernel<kNT, S1, S2, AROW, true, STT>
                   : tc::gemm_a32_kernel<kNT, S1, S2, AROW, false, STT>;
  SKEMA_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int grid = 0;
  const tc::Grid3 g = grid_of(c, M, N, K, kNT, tc::BK, pl, 1, &grid);
  if (grid <= 0) return;
  kern<<<grid, STT ? tc::kThreadsA32St : tc::kThreadsA32, smem, c->stream>>>(ta32, tb, ta16, g, o, amax,
                                                                            c->dev_err);
  SKEMA_LAUNCHED(c);
  c->dev_err_armed = true;
}

// 3 FP32 + 3 BF16 stages (228 KB of shared memory). With separate FP32 and
// B producers, 4 + 2 stages took 7.2 ms per 200k x 20k step against 5.7:
// the BF16 ring, held until each tile's store has read it, is the tighter
// of the two.
template <bool AROW>
void launch_gemm_a32(skema_ctx* c, const CUtensorMap& ta32, const CUtensorMap& tb, const CUtensorMap& ta16,
                     int64_t M, int64_t N, int64_t K, Plan pl, const tc::OutSpec& o, uint32_t* amax) {
  if (c->xt_store_thread)
    launch_gemm_a32_s<AROW, 3, 3, true>(c, ta32, tb, ta16, M, N, K, pl, o, amax);
  else
    launch_gemm_a32_s<AROW, 3, 3, false>(c, ta32, tb, ta16, M, N, K, pl, o, amax);
}

// ---- FP8 form -------------------------------------------------------------
// E4M3: largest finite value 448. Scales are powers of two, so scaling is
// exact and only the rounding to the E4M3 grid loses information.
constexpr float kE4M3Max = 448.f;

__host__ __device__ inline float pow2_scale_for(float amax) {
  // largest power of two s with amax * s <= 448 (1 when amax is 0 or not finite)
  if (!(amax > 0.f) || !(amax < 3.0e38f)) return 1.f;
  const float r = kE4M3Max / amax;
  int e;
#ifdef __CUDA_ARCH__
  e = (int)((__float_as_uint(r) >> 23) & 0xffu) - 127;
#else
  uint32_t bits;
  memcpy(&bits, &r, 4);
  e = (int)((bits >> 23) & 0xffu) - 127;
#endif
  e = e < -126 ? -126 : (e > 127 ? 127 : e);
  return ldexpf(1.f, e);
}

__device__ __forceinline__ uint8_t to_e4m3(float x) {
  return (uint8_t)__nv_cvt_float_to_fp8(x, __NV_SATFINITE, __NV_E4M3);
}
__device__ __forceinline__ float from_e4m3(uint8_t b) {
  const __half_raw h = __nv_cvt_fp8_to_halfraw((__nv_fp8_storage_t)b, __NV_E4M3);
  return __half2float(__half(h));
}

// Map values onto the scaled E4M3 grid, in place: v -> e4m3(v * sm) / sm.
__global__ void fp8_round_map_kernel(float* __restrict__ v, int64_t count, float sm) {
  const float inv = 1.f / sm;  // sm is a power of two: exact
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < count; q += (int64_t)gridDim.x * blockDim.x)
    v[q] = from_e4m3(to_e4m3(v[q] * sm)) * inv;
}

// Every map value rounded to the nearest BF16 value, kept in FP32.
__global__ void bf16_round_map_kernel(float* __restrict__ v, int64_t count) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < count; q += (int64_t)gridDim.x * blockDim.x)
    v[q] = __bfloat162float(__float2bfloat16(v[q]));
}

// Logical map rows [0, rows) -> E4M3(sm * map) at D[(r0 + r) * ld + j].
__global__ void fp8_op_kernel(const float* __restrict__ f, int64_t rs, int64_t cs, int64_t rows, int64_t cols,
                              float sm, uint8_t* __restrict__ D, int64_t ld) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < rows * cols;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = q / cols, j = q - r * cols;
    D[r * ld + j] = to_e4m3(f[r * rs + j * cs] * sm);
  }
}

// max |a| over the row-blocked BF16 window (padding rows are zeros), into
// *amax as float bits.
__global__ void amax_a16_kernel(const __nv_bfloat16* __restrict__ A16, int64_t count, uint32_t* amax) {
  float mx = 0.f;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < count; q += (int64_t)gridDim.x * blockDim.x)
    mx = fmaxf(mx, fabsf(__bfloat162float(A16[q])));
  const uint32_t wm = __reduce_max_sync(0xffffffffu, __float_as_uint(mx));
  if ((threadIdx.x & 31) == 0) atomicMax(amax, wm);
}

// Row-blocked BF16 window (64-row blocks, a 128-byte line of 64 rows per
// column) -> E4M3(scale_A a) row-major with row stride ld8 bytes, by tiles
// of 64 rows x 128 columns through shared memory. A thread takes two 4 x 4
// blocks (4 rows of 4 columns: four 8-byte loads), converts them and stores
// each block row as one 32-bit word of the row-major tile; rows then leave
// as 16-byte global stores. Within a warp the lanes cover 8 row quads x 4
// column quads: the loads are 64-byte runs of 4 column lines, and with a
// tile row stride of 33 words both the word stores and the row read-out
// hit 32 distinct banks. scale_A comes from the window's amax (*amax);
// block 0 also writes the [Y | T] product scale 1 / (scale_A scale_map)
// into *scale_out.
__global__ void __launch_bounds__(256)
    a16_to_a8_kernel(const __nv_bfloat16* __restrict__ A16, int64_t rows, int64_t cols, uint8_t* __restrict__ A8,
                     int64_t ld8, const uint32_t* amax, float* scale_out, float smap) {
  constexpr int TC = 128, W = TC / 4 + 1;  // tile columns; shared row stride in 32-bit words
  __shared__ uint32_t tile[64 * W];
  const float sa = pow2_scale_for(__uint_as_float(*amax));
  if (blockIdx.x == 0 && threadIdx.x == 0) *scale_out = 1.f / (sa * smap);
  const int64_t nrb = (rows + 63) / 64, ncb = (cols + TC - 1) / TC;
  for (int64_t t = blockIdx.x; t < nrb * ncb; t += gridDim.x) {
    const int64_t rb = t / ncb, j0 = (t - rb * ncb) * TC;
    uint2 w[2][4];
#pragma unroll
    for (int v = 0; v < 2; ++v) {
      // rows 4g .. 4g+3 and columns 4cq .. 4cq+3 of the tile
      const int b = threadIdx.x + 256 * v;
      const int g = (b & 7) | (((b >> 5) & 1) << 3), cq = ((b >> 3) & 3) | ((b >> 6) << 2);
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int64_t col = j0 + 4 * cq + j;
        w[v][j] = make_uint2(0u, 0u);
        if (col < cols) w[v][j] = *reinterpret_cast<const uint2*>(A16 + (rb * cols + col) * 64 + 4 * g);
      }
    }
#pragma unroll
    for (int v = 0; v < 2; ++v) {
      const int b = threadIdx.x + 256 * v;
      const int g = (b & 7) | (((b >> 5) & 1) << 3), cq = ((b >> 3) & 3) | ((b >> 6) << 2);
      uint32_t row[4] = {0u, 0u, 0u, 0u};
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const __nv_bfloat162 lo = *reinterpret_cast<const __nv_bfloat162*>(&w[v][j].x);  // rows 4g, 4g+1
        const __nv_bfloat162 hi = *reinterpret_cast<const __nv_bfloat162*>(&w[v][j].y);  // rows 4g+2, 4g+3
        row[0] |= (uint32_t)to_e4m3(__low2float(lo) * sa) << (8 * j);
        row[1] |= (uint32_t)to_e4m3(__high2float(lo) * sa) << (8 * j);
        row[2] |= (uint32_t)to_e4m3(__low2float(hi) * sa) << (8 * j);
        row[3] |= (uint32_t)to_e4m3(__high2float(hi) * sa) << (8 * j);
      }
#pragma unroll
      for (int e = 0; e < 4; ++e) tile[(4 * g + e) * W + cq] = row[e];
    }
    __syncthreads();
    // row r of the tile: TC bytes as TC / 16 pieces of 16 bytes
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int q = threadIdx.x + 256 * u, r = q >> 3, pc = q & 7;
      const int64_t i = rb * 64 + r, j = j0 + 16 * pc;
      if (i < rows && j < cols) {
        const uint32_t* src = tile + r * W + 4 * pc;
        const uint4 v = make_uint4(src[0], src[1], src[2], src[3]);
        uint8_t* dst = A8 + i * ld8 + j;
        if (j + 16 <= cols) {
          *reinterpret_cast<uint4*>(dst) = v;
        } else {
          const uint32_t vw[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
          for (int e = 0; e < 16; ++e)
            if (j + e < cols) dst[e] = (uint8_t)(vw[e >> 2] >> (8 * (e & 3)));
        }
      }
    }
    __syncthreads();
  }
}

CUtensorMap tmap_u8(const void* base, uint64_t d0, uint64_t d1, uint64_t st1, uint32_t b0, uint32_t b1) {
  return tmap_2d(CU_TENSOR_MAP_DATA_TYPE_UINT8, base, d0, d1, st1, b0, b1, CU_TENSOR_MAP_SWIZZLE_128B);
}

// [Y | T] in FP8: K split in multiples of the kernel's 128-element stage.
Plan plan_fp8(Plan pl, int64_t K) {
  pl.kchunk = (pl.kchunk + 127) / 128 * 128;
  pl.ks = (int)((K + pl.kchunk - 1) / pl.kchunk);
  return pl;
}

void launch_gemm_fp8(skema_ctx* c, const CUtensorMap& ta, const CUtensorMap& tb, int64_t M, int64_t N, int64_t K,
                     Plan pl, const tc::OutSpec& o) {
  constexpr int S = 5;
  constexpr uint32_t STAGE = ((tc::BM * 128 + kNT * 128 + 1023) / 1024) * 1024;
  const size_t smem = (size_t)S * STAGE + 1024 + 256;
  auto kern = tc::gemm_fp8_kernel<kNT, S>;
  SKEMA_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int grid = 0;
  const tc::Grid3 g = grid_of(c, M, N, K, kNT, 128, pl, 0, &grid);
  if (grid <= 0) return;
  kern<<<grid, tc::kThreads, smem, c->stream>>>(ta, tb, g, o, c->dev_err);
  SKEMA_LAUNCHED(c);
  c->dev_err_armed = true;
}

}  // namespace

void t32_to_t16(skema_ctx* c, const float* T32, int64_t ld32, __nv_bfloat16* T16, __nv_bfloat16* T16lo, int64_t ld16,
                int64_t rows, int64_t cols) {
  if (rows <= 0 || cols <= 0) return;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((rows * cols + 255) / 256, c->sm_count * 16));
  f32_to_bf16_cm_kernel<<<grid, 256, 0, c->stream>>>(T32, ld32, T16, T16lo, ld16, rows, cols);
  SKEMA_LAUNCHED(c);
}

size_t tc_slice_bytes(const skema_ctx* c, int64_t wr) {
  return sizeof(__nv_bfloat16) * (size_t)((c->k + c->s) * pad8(wr)) + 512;
}

TcSlices tc_window_slices(skema_ctx* c, int64_t R0, int64_t wr, char** sp) {
  TcSlices sl{static_cast<const __nv_bfloat16*>(c->ups.lowp) + R0,
              static_cast<const __nv_bfloat16*>(c->phi.lowp) + R0, c->ld_maps16};
  if (R0 % 8 == 0) return sl;
  const int64_t wp = pad8(wr);
  auto take = [&](size_t bytes) {
    char* p = *sp;
    *sp += (bytes + 255) / 256 * 256;
    return reinterpret_cast<__nv_bfloat16*>(p);
  };
  __nv_bfloat16* us = take(sizeof(__nv_bfloat16) * (size_t)(c->k * wp));
  __nv_bfloat16* fs = take(sizeof(__nv_bfloat16) * (size_t)(c->s * wp));
  to_bf16(c, Mat{c->ups.f32 + R0 * c->ups.cs, c->ups.rs, c->ups.cs}, c->k, wr, us, wp, 1);
  to_bf16(c, Mat{c->phi.f32 + R0 * c->phi.cs, c->phi.rs, c->phi.cs}, c->s, wr, fs, wp, 1);
  return TcSlices{us, fs, wp};
}

void tc_z_update(skema_ctx* c, const __nv_bfloat16* T16, int64_t ldT, const TcSlices& sl, int64_t K, float beta) {
  const float eta = (float)c->p.sketch_eta;
  const int64_t s = c->s;
  StageScope st(c, ST_PHI);
  const CUtensorMap ta = tmap_bf16(T16, (uint64_t)K, (uint64_t)s, (uint64_t)ldT * 2, 64, 128);
  const CUtensorMap tb = tmap_bf16(sl.F16, (uint64_t)K, (uint64_t)s, (uint64_t)sl.ldm * 2, 64, kNT);
  // Z^T has few tiles (8 at s = 403) and a long K: stream-K over 64 CTAs
  // gives every tile about eight partial sums (a K split over all SMs gave
  // 32, and their atomics dominated the product)
  const Plan pl = plan_streamk(c, 64);
  tc::OutSpec o = out_spec();
  o.p0 = c->Z, o.rs0 = 1, o.cs0 = s, o.alpha0 = eta, o.beta0 = beta;
  o.rows = s, o.split = s, o.ncols = s;
  if (pl.split()) {
    scale_block(c, MatOut{c->Z, s, 1}, s, s, beta);
    o.atomic0 = 1, o.beta0 = 0.f;
  }
  launch_gemm<tc::A_KMAJ>(c, ta, tb, s, s, K, pl, 0, o);
}

unsigned long long tc_default_wait_ns() { return tc::kWaitNs; }

bool tc_available(const skema_ctx* c) {
  if (c->p.precision == SKEMA_PREC_FP8 && !(c->op8 && c->fp8_win)) return false;
  return (c->p.precision == SKEMA_PREC_BF16 || c->p.precision == SKEMA_PREC_FP8) && c->ups.lowp && c->phi.lowp &&
         c->op16;
}

// BF16 copies of the Gauss maps for the tensor-core form (dense and kernel
// inputs); called after the maps are generated and after each map import.
void tc_prepare_maps(skema_ctx* c) {
  const bool fp8 = c->p.precision == SKEMA_PREC_FP8;
  if ((c->p.precision != SKEMA_PREC_BF16 && !fp8) || c->spd || c->p.issparse || c->p.dim_redux != SKEMA_MAP_GAUSS)
    return;
  if (fp8) {
    // one power-of-two scale for all four maps (the largest maxval bounds
    // them all), and the maps themselves moved onto that E4M3 grid, so that
    // the FP8, BF16 and FP32 uses of a map see the same values
    double mx = 0.0;
    for (const Map* M : {&c->ups, &c->omg, &c->phi, &c->psi}) mx = std::max(mx, M->maxval);
    c->fp8_map_scale = pow2_scale_for((float)mx);
    for (Map* M : {&c->ups, &c->omg, &c->phi, &c->psi}) {
      const int64_t cnt = M->lrows * M->lcols;
      const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((cnt + 255) / 256, c->sm_count * 16));
      fp8_round_map_kernel<<<grid, 256, 0, c->stream>>>(M->f32, cnt, c->fp8_map_scale);
      SKEMA_LAUNCHED(c);
    }
    const int64_t n8 = (c->n + 15) / 16 * 16;
    if (!c->op8) {
      SKEMA_CUDA(cudaMalloc(&c->op8, (size_t)((c->k + c->s) * n8)));
      SKEMA_CUDA(cudaMalloc(&c->fp8_win, 2 * sizeof(uint32_t)));
    }
    c->ld_op8 = n8;
    SKEMA_CUDA(cudaMemsetAsync(c->op8, 0, (size_t)((c->k + c->s) * n8), c->stream));
    auto conv8 = [&](const Map& M, int64_t r0) {
      const int64_t cnt = M.lrows * M.lcols;
      const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((cnt + 255) / 256, c->sm_count * 16));
      fp8_op_kernel<<<grid, 256, 0, c->stream>>>(M.f32, M.rs, M.cs, M.lrows, M.lcols, c->fp8_map_scale,
                                                 static_cast<uint8_t*>(c->op8) + r0 * n8, n8);
      SKEMA_LAUNCHED(c);
    };
    conv8(c->omg, 0);
    conv8(c->psi, c->k);
  } else {
    // BF16 form: the maps themselves move onto the BF16 grid, so that the
    // tensor-core products, the FP32 kernels and the FP64 approximation
    // (Phi~ Q, Psi~ P) all use the same map values
    for (Map* M : {&c->ups, &c->omg, &c->phi, &c->psi}) {
      const int64_t cnt = M->lrows * M->lcols;
      const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((cnt + 255) / 256, c->sm_count * 16));
      bf16_round_map_kernel<<<grid, 256, 0, c->stream>>>(M->f32, cnt);
      SKEMA_LAUNCHED(c);
    }
  }
  const int64_t mp = pad8(c->m), np = pad8(c->n);
  if (!c->ups.lowp) {
    SKEMA_CUDA(cudaMalloc(&c->ups.lowp, sizeof(__nv_bfloat16) * (size_t)(c->k * mp)));
    SKEMA_CUDA(cudaMalloc(&c->phi.lowp, sizeof(__nv_bfloat16) * (size_t)(c->s * mp)));
    SKEMA_CUDA(cudaMalloc(&c->op16, sizeof(__nv_bfloat16) * (size_t)((c->k + c->s) * np)));
  }
  c->ld_maps16 = mp;
  c->ld_op16 = np;
  auto conv = [&](const Map& M, void* dst, int64_t ld) {
    to_bf16(c, Mat{M.f32, M.rs, M.cs}, M.lrows, M.lcols, static_cast<__nv_bfloat16*>(dst), ld, 1);
  };
  conv(c->ups, c->ups.lowp, mp);
  conv(c->phi, c->phi.lowp, mp);
  conv(c->omg, c->op16, np);
  conv(c->psi, static_cast<__nv_bfloat16*>(c->op16) + c->k * np, np);
}

size_t tc_scratch_bytes(const skema_ctx* c, int64_t wr) {
  const int64_t wp = pad8(wr);
  const int64_t w64 = (wr + 63) / 64 * 64;
  size_t b = sizeof(__nv_bfloat16) * (size_t)(w64 * c->n) + 256;        // A16 (row-blocked)
  b += sizeof(__nv_bfloat16) * (size_t)(wp * c->s) + 256;               // T16
  b += sizeof(float) * (size_t)(wp * c->s) + 256;                       // T32 (split-K)
  b += tc_slice_bytes(c, wr);                                           // map slices (unaligned R0)
  if (c->p.precision == SKEMA_PREC_FP8) b += (size_t)(wr * ((c->n + 15) / 16 * 16)) + 256;  // A8
  return b;
}

namespace {

// X^T = nu X^T + eta A_w^T Upsilon~_w^T for one window, leaving bf16(A_w)
// row-blocked in A16 (zero rows up to a multiple of 64). The product reads
// the FP32 window itself (and writes A16) when TMA can address it (16-byte
// aligned base and stride); otherwise a conversion pass writes A16 first.
// amax (FP8 form) receives max |a| of the window. Returns the window's
// Upsilon~ / Phi~ slices (copies taken from *sp when R0 is unaligned).
TcSlices xt_window(skema_ctx* c, Mat Aw, int64_t R0, int64_t wr, __nv_bfloat16* A16, uint32_t* amax, char** sp) {
  const float eta = (float)c->p.sketch_eta, nu = (float)c->p.sketch_nu;
  const int64_t k = c->k, n = c->n;
  const int64_t nrb = (wr + 63) / 64;
  const bool al = reinterpret_cast<uintptr_t>(Aw.p) % 16 == 0;
  const bool a32_cm = al && Aw.rs == 1 && Aw.cs % 4 == 0;
  const bool a32_rm = al && Aw.cs == 1 && Aw.rs % 4 == 0;
  if (!a32_cm && !a32_rm) {
    StageScope st(c, ST_WINDOW);
    to_bf16_blocked(c, Aw, wr, n, A16);
    if (amax) {
      const int64_t cnt = nrb * 64 * n;
      const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((cnt + 255) / 256, c->sm_count * 8));
      amax_a16_kernel<<<grid, 256, 0, c->stream>>>(A16, cnt, amax);
      SKEMA_LAUNCHED(c);
    }
  }
  const TcSlices sl = tc_window_slices(c, R0, wr, sp);
  StageScope st(c, ST_UPSILON);
  const CUtensorMap tb = tmap_bf16(sl.U16, (uint64_t)wr, (uint64_t)k, (uint64_t)sl.ldm * 2, 64, kNT);
  // stream-K over all SMs: each X^T tile gets one or two partial sums (a K
  // split into eight ranges gave eight, and their atomics bounded the product)
  const Plan pl = plan_streamk(c, c->sm_count);
  tc::OutSpec o = out_spec();
  o.p0 = c->X, o.rs0 = 1, o.cs0 = n, o.alpha0 = eta, o.beta0 = nu;
  o.rows = n, o.split = k, o.ncols = k;
  if (pl.split()) {
    scale_block(c, MatOut{c->X, n, 1}, k, n, nu);
    o.atomic0 = 1, o.beta0 = 0.f;
  }
  const CUtensorMap ta16 = tmap_bf16_blocked(A16, (uint64_t)n, (uint64_t)nrb, 128);
  if (a32_cm) {
    const CUtensorMap ta32 = tmap_f32(Aw.p, (uint64_t)wr, (uint64_t)n, (uint64_t)Aw.cs * 4, 32, 128);
    launch_gemm_a32<false>(c, ta32, tb, ta16, n, k, wr, pl, o, amax);
  } else if (a32_rm) {
    const CUtensorMap ta32 = tmap_f32(Aw.p, (uint64_t)n, (uint64_t)wr, (uint64_t)Aw.rs * 4, 32, 64);
    launch_gemm_a32<true>(c, ta32, tb, ta16, n, k, wr, pl, o, amax);
  } else {
    launch_gemm<tc::A_KMAJ_BLK>(c, ta16, tb, n, k, wr, pl, 1, o);
  }
  return sl;
}

// A8 = e4m3(scale_A A16) row-major for rows rows, from the window's amax.
void to_a8(skema_ctx* c, const __nv_bfloat16* A16, int64_t rows, uint8_t* A8, int64_t ld8, const uint32_t* amax,
           float* scale_out) {
  StageScope st(c, ST_WINDOW);
  const int64_t tiles = ((rows + 63) / 64) * ((c->n + 127) / 128);
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(tiles, c->sm_count * 16));
  a16_to_a8_kernel<<<grid, 256, 0, c->stream>>>(A16, rows, c->n, A8, ld8, amax, scale_out, c->fp8_map_scale);
  SKEMA_LAUNCHED(c);
}

// Rows to process as one [Y | T] product: the M extent gr, with T going to
// Tdst (ld ldTd), rows weighted nu^(G-1-row/wlen); FP8 scales per wlen rows.
struct YtSpec {
  int64_t R0, gr;
  const __nv_bfloat16* A16;   // row-blocked BF16 (BF16 form)
  const uint8_t* A8;          // row-major E4M3, ld8 (FP8 form)
  int64_t ld8;
  const float* scales;        // FP8: per-window product scales
  __nv_bfloat16* Tdst;
  int64_t ldTd;
  float log2w;
  int64_t wlen, nwin;
  float* T32;                 // split-K scratch (ldTd rows per column)
};

void yt_product(skema_ctx* c, const YtSpec& y) {
  const float eta = (float)c->p.sketch_eta, nu = (float)c->p.sketch_nu;
  const int64_t k = c->k, s = c->s, n = c->n, m = c->m;
  const bool fp8 = c->p.precision == SKEMA_PREC_FP8;
  const float ybeta = y_beta(c, y.R0, y.R0 + y.gr, nu);
  StageScope st(c, ST_FUSED);
  const int64_t tiles = ((y.gr + 127) / 128) * ((k + s + kNT - 1) / kNT);
  Plan pl = plan_split(c, tiles, n, 8);
  if (fp8) pl = plan_fp8(pl, n);
  tc::OutSpec o = out_spec();
  o.p0 = c->Y + y.R0, o.rs0 = 1, o.cs0 = m, o.alpha0 = eta, o.beta0 = ybeta;
  o.rows = y.gr, o.split = k, o.ncols = k + s;
  o.row_log2w = y.log2w, o.row_wlen = y.wlen, o.row_nwin = y.nwin;
  if (!pl.split()) {
    o.p1 = y.Tdst, o.rs1 = 1, o.cs1 = y.ldTd;
  } else {
    scale_block(c, MatOut{c->Y + y.R0, 1, m}, y.gr, k, ybeta);
    SKEMA_CUDA(cudaMemsetAsync(y.T32, 0, sizeof(float) * (size_t)(y.ldTd * s), c->stream));
    o.atomic0 = 1, o.beta0 = 0.f;
    o.p1f = y.T32, o.rs1 = 1, o.cs1 = y.ldTd, o.atomic1 = 1;
  }
  if (fp8) {
    o.scale = y.scales, o.scale_wlen = y.wlen;
    const CUtensorMap ta = tmap_u8(y.A8, (uint64_t)n, (uint64_t)y.gr, (uint64_t)y.ld8, 128, 128);
    const CUtensorMap tb = tmap_u8(c->op8, (uint64_t)n, (uint64_t)(k + s), (uint64_t)c->ld_op8, 128, kNT);
    launch_gemm_fp8(c, ta, tb, y.gr, k + s, n, pl, o);
  } else {
    const CUtensorMap ta = tmap_bf16_blocked(y.A16, (uint64_t)n, (uint64_t)((y.gr + 63) / 64), 64);
    const CUtensorMap tb = tmap_bf16(c->op16, (uint64_t)n, (uint64_t)(k + s), (uint64_t)c->ld_op16 * 2, 64, kNT);
    launch_gemm<tc::A_MN_BLK>(c, ta, tb, y.gr, k + s, n, pl, 0, o);
  }
  if (pl.split()) t32_to_t16(c, y.T32, y.ldTd, y.Tdst, nullptr, y.ldTd, y.gr, s);
}

}  // namespace

// One window: X^T, [Y | T] and Z. Used for the windows of host-staged calls
// and for the kernel windows of the FP32 RBF path.
void tc_dense_window(skema_ctx* c, Mat Aw, int64_t R0, int64_t wr, void* scratch) {
  const float nu = (float)c->p.sketch_nu;
  const int64_t s = c->s, n = c->n;
  const int64_t wp = pad8(wr);
  char* sp = static_cast<char*>(scratch);
  auto take = [&](size_t bytes) {
    char* p = sp;
    sp += (bytes + 255) / 256 * 256;
    return p;
  };
  const int64_t nrb = (wr + 63) / 64;
  __nv_bfloat16* A16 = reinterpret_cast<__nv_bfloat16*>(take(sizeof(__nv_bfloat16) * (size_t)(nrb * 64 * n)));
  __nv_bfloat16* T16 = reinterpret_cast<__nv_bfloat16*>(take(sizeof(__nv_bfloat16) * (size_t)(wp * s)));
  float* T32 = reinterpret_cast<float*>(take(sizeof(float) * (size_t)(wp * s)));
  // FP8 form: the window's amax comes out of the X^T product (or a pass over
  // A16), its power-of-two scale is applied while A16 is rounded to E4M3,
  // and the [Y | T] product runs E4M3 x E4M3 with the scales undone in its
  // epilogue. X^T and Z stay on the BF16 path.
  const bool fp8 = c->p.precision == SKEMA_PREC_FP8;
  const int64_t ld8 = (n + 15) / 16 * 16;
  uint8_t* A8 = fp8 ? reinterpret_cast<uint8_t*>(take((size_t)(wr * ld8))) : nullptr;
  if (fp8) SKEMA_CUDA(cudaMemsetAsync(c->fp8_win, 0, 2 * sizeof(uint32_t), c->stream));
  const TcSlices sl = xt_window(c, Aw, R0, wr, A16, fp8 ? c->fp8_win : nullptr, &sp);
  float* scale = fp8 ? reinterpret_cast<float*>(c->fp8_win + 1) : nullptr;
  if (fp8) to_a8(c, A16, wr, A8, ld8, c->fp8_win, scale);
  YtSpec y{};
  y.R0 = R0, y.gr = wr, y.A16 = A16, y.A8 = A8, y.ld8 = ld8, y.scales = scale, y.T32 = T32;
  y.Tdst = T16, y.ldTd = wp, y.log2w = 0.f, y.wlen = wr, y.nwin = 1;
  yt_product(c, y);
  y_rows_mark(c, R0, R0 + wr);
  tc_z_update(c, T16, wp, sl, wr, nu);
}

namespace {

// Runs the launches of the helpers in its scope on `stream` with at most
// `cap` CTAs each (0: one per SM), restoring the context's own on exit.
class LaunchScope {
 public:
  LaunchScope(skema_ctx* c, cudaStream_t stream, int cap) : c_(c), stream_(c->stream), cap_(c->tc_cta_cap) {
    c->stream = stream;
    c->tc_cta_cap = cap;
  }
  ~LaunchScope() {
    c_->stream = stream_;
    c_->tc_cta_cap = cap_;
  }

 private:
  skema_ctx* c_;
  cudaStream_t stream_;
  int cap_;
};

}  // namespace

// The windows of one call. X^T runs per window (the recurrence X = nu X +
// eta x_w); [Y | T] and Z run once per group of windows: Y rows are
// disjoint, so a window's Y rows need only its own product, and Z = nu^G Z
// + eta sum_w nu^(G-1-w) Phi~_w T_w is the per-window recurrence
// (src/Skema_SketchySVD.cpp:187-189) summed, with window w's T rows
// weighted nu^(G-1-w) in the [Y | T] epilogue. One [Y | T] product over
// tens of thousands of rows needs no K split (its tile count fills the SMs
// many times over), and one Z^T product over the group avoids a product per
// window that was bound by its split-K atomics. The group's BF16 (or E4M3)
// window copies and T are kept. Windows that do not start on 64-row blocks,
// or nu <= 0, take one window at a time.
//
// Pipeline (pipe_xt_sms > 0): X^T streams the FP32 windows from HBM and
// leaves the tensor pipe mostly idle, [Y | T] reads the BF16 copies and is
// bound by the tensor pipe. X^T of group g + 1 therefore runs on the
// context stream with pipe_xt_sms CTAs while [Y | T] and Z of group g run on
// the side stream with the other SMs. Two copy buffers alternate: X^T of
// group g + 2 waits for [Y | T] of group g to finish reading its buffer.
// X and its per-window slices stay on the context stream; Y, T, Z and the
// group's slices on the side stream, so every buffer has one writer.
void tc_dense_update(skema_ctx* c, Mat A, int64_t row0, int64_t nrows) {
  const int64_t W = c->w, s = c->s, n = c->n;
  const float nu = (float)c->p.sketch_nu;
  const bool fp8 = c->p.precision == SKEMA_PREC_FP8;
  if (!(nu > 0.f) || W % 64 != 0 || nrows <= W) {
    void* ws = workspace(c, tc_scratch_bytes(c, std::min(W, nrows)));
    for (int64_t r = 0; r < nrows; r += W)
      tc_dense_window(c, Mat{A.p + r * A.rs, A.rs, A.cs}, row0 + r, std::min(W, nrows - r), ws);
    return;
  }
  const bool pipe = c->pipe_xt_sms > 0 && c->pipe_xt_sms < c->sm_count;
  const int nbuf = pipe ? 2 : 1;
  const int64_t cap_a = ((int64_t)2 << 30) / (2 * n), cap_t = ((int64_t)512 << 20) / (2 * s);
  int64_t gwin = std::max<int64_t>(1, std::min(cap_a, cap_t) / W);
  if (pipe) gwin = std::min(gwin, c->pipe_windows);
  const int64_t grows = std::min(nrows, gwin * W);
  const int64_t gwin_max = (grows + W - 1) / W;
  const int64_t ldT = pad8(grows), ld8 = (n + 15) / 16 * 16;
  auto rup = [](size_t b) { return (b + 255) / 256 * 256; };
  const size_t b_a16 = rup(sizeof(__nv_bfloat16) * (size_t)(((grows + 63) / 64) * 64 * n));
  const size_t b_a8 = fp8 ? rup((size_t)(grows * ld8)) : 0;
  const size_t b_t16 = rup(sizeof(__nv_bfloat16) * (size_t)(ldT * s));
  const size_t b_t32 = rup(sizeof(float) * (size_t)(ldT * s));
  const size_t b_gsl = rup(tc_slice_bytes(c, grows)), b_wsl = rup(tc_slice_bytes(c, W));
  char* ws = static_cast<char*>(workspace(c, nbuf * (b_a16 + b_a8) + b_t16 + b_t32 + b_gsl + b_wsl));
  __nv_bfloat16* A16b[2];
  uint8_t* A8b[2];
  for (int b = 0; b < nbuf; ++b) {
    A16b[b] = reinterpret_cast<__nv_bfloat16*>(ws + b * b_a16);
    A8b[b] = reinterpret_cast<uint8_t*>(ws + nbuf * b_a16 + b * b_a8);
  }
  char* tail = ws + nbuf * (b_a16 + b_a8);
  __nv_bfloat16* T16 = reinterpret_cast<__nv_bfloat16*>(tail);
  float* T32 = reinterpret_cast<float*>(tail + b_t16);
  char* gslice_sp = tail + b_t16 + b_t32;   // the group's slices (side stream)
  char* wslice_sp = gslice_sp + b_gsl;      // one window's slices (context stream)
  // FP8: per buffer, gwin_max window amax words then gwin_max scales
  uint32_t* amaxb[2] = {nullptr, nullptr};
  float* scalesb[2] = {nullptr, nullptr};
  if (fp8) {
    if (c->fp8_win_cap < 2 * gwin_max) {
      if (c->fp8_win) cudaFree(c->fp8_win);
      c->fp8_win = nullptr;
      c->fp8_win_cap = 0;
      SKEMA_CUDA(cudaMalloc(&c->fp8_win, sizeof(uint32_t) * (size_t)(4 * gwin_max)));
      c->fp8_win_cap = 2 * gwin_max;
    }
    for (int b = 0; b < nbuf; ++b) {
      amaxb[b] = c->fp8_win + b * 2 * gwin_max;
      scalesb[b] = reinterpret_cast<float*>(amaxb[b] + gwin_max);
    }
  }
  const cudaStream_t main_st = c->stream;
  const cudaStream_t yt_st = pipe ? c->side : c->stream;
  const int xt_cap = pipe ? c->pipe_xt_sms : 0, yt_cap = pipe ? c->sm_count - c->pipe_xt_sms : 0;
  if (pipe) {
    // the side stream starts after all earlier work of the context stream
    SKEMA_CUDA(cudaEventRecord(c->fork_ev, main_st));
    SKEMA_CUDA(cudaStreamWaitEvent(yt_st, c->fork_ev, 0));
  }
  // and the context stream continues after all of the side stream's work,
  // also when a launch below fails
  struct Join {
    skema_ctx* c;
    bool on;
    ~Join() {
      if (on && cudaEventRecord(c->join_ev, c->side) == cudaSuccess) cudaStreamWaitEvent(c->stream, c->join_ev, 0);
    }
  } join{c, pipe};
  const float log2nu = nu == 1.f ? 0.f : std::log2(nu);
  int64_t gi = 0;
  for (int64_t g0 = 0; g0 < nrows; g0 += grows, ++gi) {
    const int b = (int)(gi % nbuf);
    const int64_t gr = std::min(grows, nrows - g0), G = (gr + W - 1) / W, R0 = row0 + g0;
    __nv_bfloat16* A16 = A16b[b];
    uint8_t* A8 = A8b[b];
    {
      LaunchScope ls(c, main_st, xt_cap);
      // the buffer's previous group must have been read by its [Y | T]
      if (pipe && gi >= nbuf) SKEMA_CUDA(cudaStreamWaitEvent(main_st, c->pipe_ev[2 + b], 0));
      if (fp8) SKEMA_CUDA(cudaMemsetAsync(amaxb[b], 0, sizeof(uint32_t) * (size_t)(2 * gwin_max), main_st));
      for (int64_t w = 0; w < G; ++w) {
        const int64_t r = g0 + w * W, wr = std::min(W, nrows - r);
        __nv_bfloat16* A16w = A16 + (w * W / 64) * 64 * n;
        char* sp = wslice_sp;
        xt_window(c, Mat{A.p + r * A.rs, A.rs, A.cs}, row0 + r, wr, A16w, fp8 ? amaxb[b] + w : nullptr, &sp);
        if (fp8) to_a8(c, A16w, wr, A8 + w * W * ld8, ld8, amaxb[b] + w, scalesb[b] + w);
      }
      if (pipe) SKEMA_CUDA(cudaEventRecord(c->pipe_ev[b], main_st));
    }
    {
      LaunchScope ls(c, yt_st, yt_cap);
      if (pipe) SKEMA_CUDA(cudaStreamWaitEvent(yt_st, c->pipe_ev[b], 0));
      YtSpec y{};
      y.R0 = R0, y.gr = gr, y.A16 = A16, y.A8 = A8, y.ld8 = ld8, y.scales = scalesb[b], y.T32 = T32;
      y.Tdst = T16, y.ldTd = ldT, y.log2w = log2nu, y.wlen = W, y.nwin = G;
      yt_product(c, y);
      y_rows_mark(c, R0, R0 + gr);
      char* sp = gslice_sp;
      const TcSlices sl = tc_window_slices(c, R0, gr, &sp);
      tc_z_update(c, T16, ldT, sl, gr, std::pow(nu, (float)G));
      if (pipe) SKEMA_CUDA(cudaEventRecord(c->pipe_ev[2 + b], yt_st));
    }
  }
}

}  // namespace skema
