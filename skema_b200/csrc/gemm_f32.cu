// gemm_f32.cu -- the plain FP32 contraction used by the FP32 form of the
// sketch (the drop-in for KokkosBlas::gemm in Impl::mm,
// src/Skema_Common.hpp:32-40) plus small strided elementwise kernels.
//
// SIMT GEMM: 128x128 output tile per 256-thread CTA, 8x8 outputs per thread,
// K staged through double-buffered shared memory 8 deep. Operands are
// addressed by (row stride, col stride) so that column-major A windows,
// row-major maps and transposed views need no copies; the template picks the
// coalesced load pattern from which stride is 1. Optional split-K over
// grid.z with atomic accumulation for the small-output/large-K products.
#include <cuda_runtime.h>

#include <algorithm>

#include "internal.h"

namespace skema {

namespace {

constexpr int BM = 128, BN = 128, BK = 16, PAD = 4;
constexpr int LD = BK * BM / 256;  // elements of A (and of B) a thread stages per K step

// 16-deep K steps, one CTA per SM with the registers it wants (about 190):
// measured on the dense case's T product (8192 x 403, K = 20,000, K split
// four ways), 37.0 TFLOP/s against 32.4 for 8-deep steps at two CTAs per SM
// of 128 registers, and 35.6 for 8-deep steps at one CTA per SM.
template <bool A_M_CONTIG, bool B_N_CONTIG, bool ATOMIC>
__global__ void __launch_bounds__(256, 1)
    sgemm_kernel(int64_t M, int64_t N, int64_t K, float alpha, const float* __restrict__ A,
                 int64_t a_rs, int64_t a_cs, const float* __restrict__ B, int64_t b_rs,
                 int64_t b_cs, float beta, float* __restrict__ C, int64_t c_rs, int64_t c_cs,
                 int64_t kchunk, int64_t c_zs) {
  __shared__ __align__(16) float As[2][BK][BM + PAD];
  __shared__ __align__(16) float Bs[2][BK][BN + PAD];
  const int tid = threadIdx.x;
  const int64_t m0 = (int64_t)blockIdx.x * BM;
  const int64_t n0 = (int64_t)blockIdx.y * BN;
  const int64_t kb = (int64_t)blockIdx.z * kchunk;
  const int64_t ke = min(K, kb + kchunk);
  if (kb >= ke) return;

  // Load coordinates inside a tile.
  int la_m[LD], la_k[LD], lb_n[LD], lb_k[LD];
#pragma unroll
  for (int q = 0; q < LD; ++q) {
    if (A_M_CONTIG) {
      la_m[q] = tid & 127;
      la_k[q] = (tid >> 7) + 2 * q;
    } else {
      la_k[q] = tid % BK;
      la_m[q] = tid / BK + (256 / BK) * q;
    }
    if (B_N_CONTIG) {
      lb_n[q] = tid & 127;
      lb_k[q] = (tid >> 7) + 2 * q;
    } else {
      lb_k[q] = tid % BK;
      lb_n[q] = tid / BK + (256 / BK) * q;
    }
  }
  float ra[LD], rb[LD];
  auto load_tile = [&](int64_t k0) {
#pragma unroll
    for (int q = 0; q < LD; ++q) {
      const int64_t gm = m0 + la_m[q], gk = k0 + la_k[q];
      ra[q] = (gm < M && gk < ke) ? __ldg(A + gm * a_rs + gk * a_cs) : 0.f;
      const int64_t gn = n0 + lb_n[q], gk2 = k0 + lb_k[q];
      rb[q] = (gn < N && gk2 < ke) ? __ldg(B + gk2 * b_rs + gn * b_cs) : 0.f;
    }
  };
  auto store_tile = [&](int buf) {
#pragma unroll
    for (int q = 0; q < LD; ++q) {
      As[buf][la_k[q]][la_m[q]] = ra[q];
      Bs[buf][lb_k[q]][lb_n[q]] = rb[q];
    }
  };

  const int tx = tid & 15, ty = tid >> 4;
  float acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0.f;

  load_tile(kb);
  store_tile(0);
  __syncthreads();
  int buf = 0;
  for (int64_t k0 = kb; k0 < ke; k0 += BK) {
    const bool more = k0 + BK < ke;
    if (more) load_tile(k0 + BK);
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      const float4 a0 = *reinterpret_cast<const float4*>(&As[buf][kk][ty * 4]);
      const float4 a1 = *reinterpret_cast<const float4*>(&As[buf][kk][64 + ty * 4]);
      const float4 b0 = *reinterpret_cast<const float4*>(&Bs[buf][kk][tx * 4]);
      const float4 b1 = *reinterpret_cast<const float4*>(&Bs[buf][kk][64 + tx * 4]);
      const float a[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
      const float b[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    if (more) {
      store_tile(buf ^ 1);
      __syncthreads();
      buf ^= 1;
    }
  }

#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int64_t gm = m0 + (i < 4 ? ty * 4 + i : 64 + ty * 4 + (i - 4));
    if (gm >= M) continue;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int64_t gn = n0 + (j < 4 ? tx * 4 + j : 64 + tx * 4 + (j - 4));
      if (gn >= N) continue;
      float* cp = C + blockIdx.z * c_zs + gm * c_rs + gn * c_cs;
      const float v = alpha * acc[i][j];
      if (ATOMIC) {
        atomicAdd(cp, v);
      } else {
        *cp = (beta == 0.f) ? v : fmaf(beta, *cp, v);
      }
    }
  }
}

// C_zs: offset between the outputs of the K splits (0: all into C).
template <bool AM, bool BN_, bool AT>
void launch_sgemm(skema_ctx* c, int64_t M, int64_t N, int64_t K, float alpha, Mat A, Mat B,
                  float beta, MatOut C, int splitk, int64_t c_zs = 0) {
  int64_t kchunk = (K + splitk - 1) / splitk;
  kchunk = (kchunk + BK - 1) / BK * BK;
  const int64_t gz = (K + kchunk - 1) / kchunk;
  // M tiles on grid.x (2^31-1 limit); N in chunks of at most 65535 tiles.
  const int64_t nchunk = (int64_t)65535 * BN;
  for (int64_t nb = 0; nb < N; nb += nchunk) {
    const int64_t nn = std::min(nchunk, N - nb);
    dim3 grid((unsigned)((M + BM - 1) / BM), (unsigned)((nn + BN - 1) / BN), (unsigned)gz);
    sgemm_kernel<AM, BN_, AT><<<grid, 256, 0, c->stream>>>(
        M, nn, K, alpha, A.p, A.rs, A.cs, B.p + nb * B.cs, B.rs, B.cs, beta, C.p + nb * C.cs, C.rs,
        C.cs, kchunk, c_zs);
    SKEMA_LAUNCHED(c);
  }
}

__global__ void scale_kernel(float* __restrict__ C, int64_t rs, int64_t cs, int64_t M, int64_t N,
                             float beta) {
  const int64_t total = M * N;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total;
       q += (int64_t)gridDim.x * blockDim.x) {
    int64_t i, j;
    if (cs == 1) {
      i = q / N;
      j = q - i * N;
    } else {
      j = q / M;
      i = q - j * M;
    }
    float* p = C + i * rs + j * cs;
    *p = (beta == 0.f) ? 0.f : beta * *p;
  }
}

__global__ void axpby_kernel(const float* __restrict__ S, int64_t srs, int64_t scs,
                             float* __restrict__ D, int64_t drs, int64_t dcs, int64_t M,
                             int64_t N, float alpha, float beta) {
  const int64_t total = M * N;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total;
       q += (int64_t)gridDim.x * blockDim.x) {
    int64_t i, j;
    if (dcs == 1) {
      i = q / N;
      j = q - i * N;
    } else {
      j = q / M;
      i = q - j * M;
    }
    float* d = D + i * drs + j * dcs;
    const float v = alpha * S[i * srs + j * scs];
    *d = (beta == 0.f) ? v : fmaf(beta, *d, v);
  }
}

// Tiled transpose-capable copy through shared memory (32x32 tiles).
__global__ void copy_kernel(const float* __restrict__ S, int64_t srs, int64_t scs,
                            float* __restrict__ D, int64_t drs, int64_t dcs, int64_t M,
                            int64_t N) {
  __shared__ float t[32][33];
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  const int64_t ti = (M + 31) / 32, tj = (N + 31) / 32;
  for (int64_t tile = blockIdx.x; tile < ti * tj; tile += gridDim.x) {
  const int64_t i0 = (tile / tj) * 32, j0 = (tile % tj) * 32;
  // read: make consecutive threads follow the source's unit stride
  for (int r = ty; r < 32; r += 8) {
    const int64_t i = (scs == 1) ? i0 + r : i0 + tx;
    const int64_t j = (scs == 1) ? j0 + tx : j0 + r;
    if (i < M && j < N) {
      if (scs == 1)
        t[r][tx] = S[i * srs + j * scs];
      else
        t[tx][r] = S[i * srs + j * scs];
    }
  }
  __syncthreads();
  for (int r = ty; r < 32; r += 8) {
    const int64_t i = (dcs == 1) ? i0 + r : i0 + tx;
    const int64_t j = (dcs == 1) ? j0 + tx : j0 + r;
    if (i < M && j < N) {
      if (dcs == 1)
        D[i * drs + j * dcs] = t[r][tx];
      else
        D[i * drs + j * dcs] = t[tx][r];
    }
  }
  __syncthreads();
  }
}

// C = beta C + alpha sum_z P_z over M x N, the K-split partial products P_z
// (strides p_rs, p_cs; p_zs apart) summed in z order, so the result does not
// depend on scheduling. Consecutive threads follow C's unit stride.
__global__ void splitk_reduce_kernel(const float* __restrict__ P, int64_t p_rs, int64_t p_cs, int64_t p_zs, int nz,
                                     int64_t M, int64_t N, float alpha, float beta, float* __restrict__ C,
                                     int64_t c_rs, int64_t c_cs) {
  const int64_t total = M * N;
  const bool cm = c_rs == 1;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = cm ? q % M : q / N, j = cm ? q / M : q % N;
    const float* pp = P + i * p_rs + j * p_cs;
    float sum = 0.f;
    for (int z = 0; z < nz; ++z) sum += pp[z * p_zs];
    float* cp = C + i * c_rs + j * c_cs;
    *cp = (beta == 0.f) ? alpha * sum : fmaf(beta, *cp, alpha * sum);
  }
}

int grid1d(const skema_ctx* c, int64_t total, int threads) {
  const int64_t want = (total + threads - 1) / threads;
  return (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)c->sm_count * 16));
}

}  // namespace

void sgemm(skema_ctx* c, int64_t M, int64_t N, int64_t K, float alpha, Mat A, Mat B, float beta,
           MatOut C, int splitk) {
  if (M <= 0 || N <= 0) return;
  if (K <= 0) {
    if (splitk <= 1) scale_block(c, C, M, N, beta);
    return;
  }
  const bool am = (A.rs == 1);
  const bool bn = (B.cs == 1);
  const bool at = splitk > 1;
  if (am && bn && at) launch_sgemm<true, true, true>(c, M, N, K, alpha, A, B, beta, C, splitk);
  else if (am && bn) launch_sgemm<true, true, false>(c, M, N, K, alpha, A, B, beta, C, 1);
  else if (am && at) launch_sgemm<true, false, true>(c, M, N, K, alpha, A, B, beta, C, splitk);
  else if (am) launch_sgemm<true, false, false>(c, M, N, K, alpha, A, B, beta, C, 1);
  else if (bn && at) launch_sgemm<false, true, true>(c, M, N, K, alpha, A, B, beta, C, splitk);
  else if (bn) launch_sgemm<false, true, false>(c, M, N, K, alpha, A, B, beta, C, 1);
  else if (at) launch_sgemm<false, false, true>(c, M, N, K, alpha, A, B, beta, C, splitk);
  else launch_sgemm<false, false, false>(c, M, N, K, alpha, A, B, beta, C, 1);
}

void sgemm_split(skema_ctx* c, int64_t M, int64_t N, int64_t K, float alpha, Mat A, Mat B, float beta, MatOut C,
                 float* part, int64_t part_floats) {
  if (M <= 0 || N <= 0) return;
  // A grid of output tiles below two per SM gets about six (tile, K range)
  // units per SM (one CTA per SM at a time), each range at least 1024 deep,
  // as far as the partial buffer allows.
  const int64_t tiles = ((M + BM - 1) / BM) * ((N + BN - 1) / BN);
  const int64_t slots = 2 * (int64_t)c->sm_count;
  int64_t sk = 1;
  if (part && K > 0 && tiles < 2 * slots && N <= (int64_t)65535 * BN) {
    sk = (3 * slots + tiles - 1) / tiles;
    sk = std::min<int64_t>({sk, 16, K / 1024, part_floats / (M * N)});
  }
  if (sk < 2) {
    sgemm(c, M, N, K, alpha, A, B, beta, C);
    return;
  }
  int64_t kchunk = (K + sk - 1) / sk;
  kchunk = (kchunk + BK - 1) / BK * BK;
  const int nz = (int)((K + kchunk - 1) / kchunk);
  // partial planes in C's orientation, so the reduction reads and writes
  // along the same unit stride
  const bool cm = C.rs == 1;
  const MatOut P{part, cm ? 1 : N, cm ? M : 1};
  const int64_t pz = M * N;
  const bool am = (A.rs == 1), bn = (B.cs == 1);
  if (am && bn) launch_sgemm<true, true, false>(c, M, N, K, 1.f, A, B, 0.f, P, (int)sk, pz);
  else if (am) launch_sgemm<true, false, false>(c, M, N, K, 1.f, A, B, 0.f, P, (int)sk, pz);
  else if (bn) launch_sgemm<false, true, false>(c, M, N, K, 1.f, A, B, 0.f, P, (int)sk, pz);
  else launch_sgemm<false, false, false>(c, M, N, K, 1.f, A, B, 0.f, P, (int)sk, pz);
  splitk_reduce_kernel<<<grid1d(c, pz, 256), 256, 0, c->stream>>>(part, P.rs, P.cs, pz, nz, M, N, alpha, beta, C.p,
                                                                   C.rs, C.cs);
  SKEMA_LAUNCHED(c);
}

void scale_block(skema_ctx* c, MatOut C, int64_t M, int64_t N, float beta, cudaStream_t stream) {
  if (M <= 0 || N <= 0 || beta == 1.f) return;
  scale_kernel<<<grid1d(c, M * N, 256), 256, 0, stream ? stream : c->stream>>>(C.p, C.rs, C.cs, M, N, beta);
  SKEMA_LAUNCHED(c);
}

void axpby_block(skema_ctx* c, Mat src, MatOut dst, int64_t M, int64_t N, float alpha, float beta) {
  if (M <= 0 || N <= 0) return;
  axpby_kernel<<<grid1d(c, M * N, 256), 256, 0, c->stream>>>(src.p, src.rs, src.cs, dst.p, dst.rs,
                                                              dst.cs, M, N, alpha, beta);
  SKEMA_LAUNCHED(c);
}

// dst[l * ns + s] = src[l + s * ss] for l < nl, s < ns (ns <= 256): a block
// whose long dimension is contiguous in the source, written densely with the
// short dimension innermost (a column-major m x k sketch into row-major rows,
// or a row-major k x n one into column-major columns). A CTA takes 32 long
// indices: a warp reads 128 contiguous bytes per short index into shared
// memory (rows of an odd stride, so the stores do not collide), then the CTA
// writes the 32 ns values as one contiguous run.
__global__ void __launch_bounds__(256) narrow_transpose_kernel(const float* __restrict__ src, int64_t nl, int ns,
                                                               int64_t ss, float* __restrict__ dst) {
  extern __shared__ float nt[];  // 32 rows of ld >= ns
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int ld = ns | 1;
  for (int64_t l0 = (int64_t)blockIdx.x * 32; l0 < nl; l0 += (int64_t)gridDim.x * 32) {
    const int nr = (int)min((int64_t)32, nl - l0);
    if (tx < nr)
      for (int s = ty; s < ns; s += 8) nt[tx * ld + s] = src[l0 + tx + s * ss];
    __syncthreads();
    float* o = dst + l0 * ns;
    const int tot = nr * ns;
    for (int q = threadIdx.x; q < tot; q += blockDim.x) {
      const int r = q / ns;
      o[q] = nt[r * ld + (q - r * ns)];
    }
    __syncthreads();
  }
}

void transpose_narrow(skema_ctx* c, const float* src, int64_t nl, int64_t ns, int64_t ss, float* dst,
                      cudaStream_t st) {
  if (nl <= 0 || ns <= 0) return;
  if (ns > 256) fail(SKEMA_EINVAL, "transpose_narrow: short dimension above 256");
  const int grid = (int)std::min<int64_t>((nl + 31) / 32, (int64_t)c->sm_count * 16);
  const size_t smem = sizeof(float) * 32 * (size_t)(ns | 1);
  narrow_transpose_kernel<<<grid, 256, smem, st>>>(src, nl, (int)ns, ss, dst);
  SKEMA_LAUNCHED(c);
}

void copy_block(skema_ctx* c, Mat src, MatOut dst, int64_t M, int64_t N, cudaStream_t st) {
  if (M <= 0 || N <= 0) return;
  const int64_t tiles = ((M + 31) / 32) * ((N + 31) / 32);
  const int grid = (int)std::min<int64_t>(tiles, (int64_t)c->sm_count * 32);
  copy_kernel<<<grid, dim3(32, 8), 0, st>>>(src.p, src.rs, src.cs, dst.p, dst.rs, dst.cs, M, N);
  SKEMA_LAUNCHED(c);
}

void copy_block(skema_ctx* c, Mat src, MatOut dst, int64_t M, int64_t N) { copy_block(c, src, dst, M, N, c->stream); }

}  // namespace skema
