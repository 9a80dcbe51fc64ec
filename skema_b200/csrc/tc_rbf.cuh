// tc_rbf.cuh -- the Gauss-RBF kernel sketch without materialising K:
// O = P V with P(q, j) = exp(-gamma ||x_q - x_j||^2) generated tile by
// tile on the tensor cores (sm_100a tcgen05, TMEM accumulators, TMA).
//
// For one unit (128 "query" points q, one chunk of output columns, one
// range of 64-point "key" blocks j):
//   Gram     S = Q K_b^T            tcgen05, M = 128, N = 64, K = d (BF16)
//   kernel   P = exp2(2 g' S + c_q + c_j), with c_p = -g' ||x_p||^2 and
//            g' = gamma * log2(e), clamped at 1 (d^2 >= 0), 1 on the
//            diagonal point q == point j (the reference's window rule),
//            written as BF16 into 128-byte-swizzled shared memory
//   sketch   O += P V_b             tcgen05, M = 128, N = NC1 (+ NC2), K = 64
// where V_b holds the output columns' map entries for the 64 key points,
// K-major (one row per output column). Gram tiles of the next block are
// computed while the kernel warps exponentiate the current one, and the
// sketch product of a block runs while the next block is exponentiated.
//
//   row pass (Y / T of a window):  q = window rows, j = all points,
//                                  V = [Omega~; Psi~] (output = k + s columns)
//   column pass (X of a window):   q = all points, j = window rows,
//                                  V = Upsilon~ restricted to the window
//
// Roles (192 threads): warps 0-3 kernel-tile warps and epilogue (warp w owns
// TMEM lanes 32w..32w+31, i.e. query rows), warp 4 TMA producer, warp 5 MMA
// issuer and TMEM owner. Every wait is bounded (see tc_gemm.cuh).
#pragma once
#include "tc_gemm.cuh"

namespace skema {
namespace tc {

constexpr int RBF_BQ = 128;  // query rows per unit (TMEM lanes)
constexpr int RBF_BJ = 64;   // key points per block
constexpr uint32_t RBF_SCOL = 448;  // TMEM column of the Gram tile (O uses [0, 448))

// 2^x by the PTX ex2.approx instruction (relative error about 2^-22, far
// below the BF16 rounding of the result); 2^-inf = 0.
__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

struct RbfArgs {
  int64_t nq;          // valid query rows (rows >= nq are ignored)
  int64_t qbase;       // point index of query row 0
  int64_t kbase;       // point index of key column 0 (diagonal test)
  int64_t nblocks;     // key blocks in total (64 points each)
  int64_t bchunk;      // key blocks per split
  int qtiles, nchunks, ksplit;
  int chunk_cols;      // output columns per chunk (NC1 + NC2)
  const float* cq;     // c_p of the query points, indexed by query row
  const float* ckey;   // c_p of the key points, indexed by key column, padded with -inf
  float two_g;         // 2 * gamma * log2(e)
  // Window weights folded into ckey (key column j of window j / kwlen, of
  // knwin, carries + (knwin - 1 - j / kwlen) * klog2w); the forced diagonal
  // entry is that weight instead of 1. klog2w = 0: unweighted.
  float klog2w;
  int64_t kwlen, knwin;
};

template <int NC1, int NC2, int DK, int RBF_S>
__global__ void __launch_bounds__(kThreads, 1)
    rbf_sketch_kernel(const __grid_constant__ CUtensorMap tmQ, const __grid_constant__ CUtensorMap tmK,
                      const __grid_constant__ CUtensorMap tmV1, const __grid_constant__ CUtensorMap tmV2,
                      RbfArgs a, OutSpec o, int* err) {
  constexpr int NC = NC1 + NC2;
  static_assert(NC1 % 16 == 0 && NC1 <= 256 && NC2 % 16 == 0 && NC2 <= 256, "chunk tiles");
  static_assert(NC <= (int)RBF_SCOL, "O and the Gram tile share TMEM");
  constexpr uint32_t Q_BYTES = DK * RBF_BQ * 128;      // DK sub-tiles of 64 d-values
  constexpr uint32_t K_BYTES = DK * RBF_BJ * 128;
  constexpr uint32_t V_BYTES = NC * 128;               // NC rows of 64 key values
  constexpr uint32_t STAGE = ((K_BYTES + V_BYTES + 256 + 1023) / 1024) * 1024;  // + c_key of the block
  constexpr uint32_t P_BYTES = RBF_BQ * 128;           // 128 rows of 64 BF16
  // With a chunk of at most 384 columns, P (128 x 64 BF16 = 32 TMEM columns)
  // is double-buffered in TMEM at columns 384 and 416 and the sketch MMA
  // reads it from there, which leaves shared memory to the V operand alone;
  // wider chunks keep P in shared memory.
  constexpr bool PT = NC <= 384;
  constexpr uint32_t P_TCOL = 384;
  // Q (128 x 64 DK BF16 = 32 DK columns) goes to TMEM at columns NC.. as well
  // when it fits below P: the Gram MMA then reads only K from shared memory.
  // The kernel-tile warps copy it there at the start of each unit and free
  // its shared-memory copy at once.
  constexpr bool QT = PT && NC + 32 * DK <= (int)P_TCOL;
  constexpr uint32_t Q_TCOL = NC;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  unsigned char* qs = smem;
  unsigned char* st = qs + Q_BYTES;
  unsigned char* ps = st + RBF_S * STAGE;
  uint64_t* bar = reinterpret_cast<uint64_t*>(ps + 2 * P_BYTES);
  uint64_t* qfull = bar + 0;
  uint64_t* qempty = bar + 1;
  uint64_t* full = bar + 2;              // [RBF_S]
  uint64_t* empty = full + RBF_S;        // [RBF_S]
  uint64_t* sfull = empty + RBF_S;
  uint64_t* sfree = sfull + 1;
  uint64_t* pfull = sfree + 1;           // [2]
  uint64_t* pfree = pfull + 2;           // [2]
  uint64_t* ofull = pfree + 2;
  uint64_t* ofree = ofull + 1;
  uint64_t* qtm = ofree + 1;             // Q copied into TMEM (QT)
  uint32_t* tbase = reinterpret_cast<uint32_t*>(qtm + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int total = a.qtiles * a.nchunks * a.ksplit;

  if (threadIdx.x == 0) {
    mbar_init(qfull, 1);
    mbar_init(qempty, QT ? 128 : 1);
    mbar_init(qtm, 128);
    for (int s = 0; s < RBF_S; ++s) {
      mbar_init(full + s, 1);
      mbar_init(empty + s, 1);
    }
    mbar_init(sfull, 1);
    mbar_init(sfree, 128);
    for (int p = 0; p < 2; ++p) {
      mbar_init(pfull + p, 128);
      mbar_init(pfree + p, 1);
    }
    mbar_init(ofull, 1);
    mbar_init(ofree, 128);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 5) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tbase)),
                 "r"(512)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tbase;

  // unit t -> (query tile, chunk, key split), chunk fastest
  auto decode = [&](int t, int& qt, int& ch, int& ks, int64_t& b0, int64_t& b1) {
    ch = t % a.nchunks;
    t /= a.nchunks;
    qt = t % a.qtiles;
    ks = t / a.qtiles;
    b0 = (int64_t)ks * a.bchunk;
    b1 = min(a.nblocks, b0 + a.bchunk);
  };

  if (warp == 4 && lane == 0) {
    // ---------------- TMA producer ----------------
    uint32_t it = 0, un = 0;
    bool ok = true;
    for (int t = blockIdx.x; t < total && ok; t += gridDim.x, ++un) {
      int qt, ch, ks;
      int64_t b0, b1;
      decode(t, qt, ch, ks, b0, b1);
      if (!mbar_wait(qempty, (un & 1) ^ 1, err)) break;
      mbar_expect_tx(qfull, Q_BYTES);
#pragma unroll
      for (int dk = 0; dk < DK; ++dk)
        tma_load_2d(&tmQ, qfull, qs + dk * RBF_BQ * 128, 64 * dk, (int)(a.qbase + (int64_t)qt * RBF_BQ));
      for (int64_t b = b0; b < b1; ++b, ++it) {
        const int s = it % RBF_S;
        const uint32_t ph = (it / RBF_S) & 1;
        if (!mbar_wait(empty + s, ph ^ 1, err)) {
          ok = false;
          break;
        }
        unsigned char* sk = st + s * STAGE;
        mbar_expect_tx(full + s, K_BYTES + V_BYTES + 256);
#pragma unroll
        for (int dk = 0; dk < DK; ++dk)
          tma_load_2d(&tmK, full + s, sk + dk * RBF_BJ * 128, 64 * dk, (int)(a.kbase + b * RBF_BJ));
        tma_load_2d(&tmV1, full + s, sk + K_BYTES, (int)(b * RBF_BJ), ch * NC);
        if (NC2 > 0) tma_load_2d(&tmV2, full + s, sk + K_BYTES + NC1 * 128, (int)(b * RBF_BJ), ch * NC + NC1);
        // the 64 key constants of the block (256 bytes)
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], 256, [%2];" ::"r"(
                smem_u32(sk + K_BYTES + V_BYTES)),
            "l"(a.ckey + b * RBF_BJ), "r"(smem_u32(full + s))
            : "memory");
      }
    }
  } else if (warp == 5 && lane == 0) {
    // ---------------- MMA issuer ----------------
    constexpr uint32_t id_g = idesc_bf16(RBF_BJ, false, false);
    constexpr uint32_t id_1 = idesc_bf16(NC1, false, false);
    constexpr uint32_t id_2 = idesc_bf16(NC2 > 0 ? NC2 : 16, false, false);
    const uint32_t tS = tmem + RBF_SCOL;
    uint32_t it = 0, un = 0, g = 0, pc = 0;
    bool ok = true;
    // O += P_b V_b for the block whose P is in buffer pc % 2 and whose V is in stage s
    auto sketch = [&](int s, bool first) -> bool {
      const uint32_t pb = pc & 1;
      if (!mbar_wait(pfull + pb, (pc >> 1) & 1, err)) return false;
      tc_fence_after();
      const uint32_t pa = smem_u32(ps + pb * P_BYTES);
      const uint32_t pt = tmem + P_TCOL + pb * 32;
      const uint32_t vb = smem_u32(st + s * STAGE + K_BYTES);
#pragma unroll
      for (int kk = 0; kk < RBF_BJ / 16; ++kk) {
        const uint32_t acc = (!first || kk > 0) ? 1u : 0u;
        if (PT) {
          umma_ts(tmem, pt + kk * 8, sdesc(vb + kk * 32, 16, 1024), id_1, acc);
          if (NC2 > 0) umma_ts(tmem + NC1, pt + kk * 8, sdesc(vb + NC1 * 128 + kk * 32, 16, 1024), id_2, acc);
        } else {
          umma(tmem, sdesc(pa + kk * 32, 16, 1024), sdesc(vb + kk * 32, 16, 1024), id_1, acc);
          if (NC2 > 0)
            umma(tmem + NC1, sdesc(pa + kk * 32, 16, 1024), sdesc(vb + NC1 * 128 + kk * 32, 16, 1024), id_2, acc);
        }
      }
      umma_commit(empty + s);
      umma_commit(pfree + pb);
      ++pc;
      return true;
    };
    for (int t = blockIdx.x; t < total && ok; t += gridDim.x, ++un) {
      int qt, ch, ks;
      int64_t b0, b1;
      decode(t, qt, ch, ks, b0, b1);
      if (!mbar_wait(QT ? qtm : qfull, un & 1, err)) break;
      int prev_s = -1;
      bool first = true;
      for (int64_t b = b0; b < b1; ++b, ++it) {
        const int s = it % RBF_S;
        const uint32_t ph = (it / RBF_S) & 1;
        if (!mbar_wait(full + s, ph, err) || !mbar_wait(sfree, (g & 1) ^ 1, err)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t qa = smem_u32(qs), kb = smem_u32(st + s * STAGE);
#pragma unroll
        for (int dk = 0; dk < DK; ++dk)
#pragma unroll
          for (int kk = 0; kk < 4; ++kk) {
            const uint64_t bd = sdesc(kb + dk * RBF_BJ * 128 + kk * 32, 16, 1024);
            if (QT)
              umma_ts(tS, tmem + Q_TCOL + dk * 32 + kk * 8, bd, id_g, (dk > 0 || kk > 0) ? 1u : 0u);
            else
              umma(tS, sdesc(qa + dk * RBF_BQ * 128 + kk * 32, 16, 1024), bd, id_g, (dk > 0 || kk > 0) ? 1u : 0u);
          }
        umma_commit(sfull);
        ++g;
        if (!QT && b + 1 == b1) umma_commit(qempty);
        if (prev_s >= 0) {
          if (first && !mbar_wait(ofree, (un & 1) ^ 1, err)) {
            ok = false;
            break;
          }
          if (!sketch(prev_s, first)) {
            ok = false;
            break;
          }
          first = false;
        }
        prev_s = s;
      }
      if (!ok) break;
      if (prev_s >= 0) {
        if (first && !mbar_wait(ofree, (un & 1) ^ 1, err)) break;
        if (!sketch(prev_s, first)) break;
      }
      umma_commit(ofull);
    }
  } else if (warp < 4) {
    // ---------------- kernel tiles + epilogue ----------------
    const uint32_t lane_off = (uint32_t)(warp * 32) << 16;
    uint32_t it = 0, un = 0, g = 0, pc = 0;
    for (int t = blockIdx.x; t < total; t += gridDim.x, ++un) {
      int qt, ch, ks;
      int64_t b0, b1;
      decode(t, qt, ch, ks, b0, b1);
      const int64_t qrow = (int64_t)qt * RBF_BQ + warp * 32 + lane;  // query row of this thread
      const float cq = qrow < a.nq ? a.cq[qrow] : 0.f;
      if (QT) {
        // this thread's Q row into TMEM (the Gram MMAs of the previous unit
        // have completed: their S tiles were all read), then free the
        // shared-memory copy for the next unit's load
        if (!__all_sync(0xffffffffu, mbar_wait(qfull, un & 1, err))) break;
        const int row = warp * 32 + lane;
#pragma unroll
        for (int dk = 0; dk < DK; ++dk) {
          uint32_t qw[32];
          const unsigned char* qrowp = qs + dk * RBF_BQ * 128 + row * 128;
#pragma unroll
          for (int c = 0; c < 8; ++c) {
            const uint4 v = *reinterpret_cast<const uint4*>(qrowp + ((c ^ (row & 7)) << 4));
            qw[4 * c] = v.x, qw[4 * c + 1] = v.y, qw[4 * c + 2] = v.z, qw[4 * c + 3] = v.w;
          }
          tmem_st32(tmem + Q_TCOL + dk * 32 + lane_off, qw);
        }
        tc_fence_before();
        mbar_arrive(qtm);
        fence_proxy_async();
        mbar_arrive(qempty);
      }
      const int64_t gq = a.qbase + qrow;                              // its point index
      bool ok = true;
      for (int64_t b = b0; b < b1; ++b, ++it, ++g, ++pc) {
        if (!__all_sync(0xffffffffu, mbar_wait(sfull, g & 1, err))) {
          ok = false;
          break;
        }
        tc_fence_after();
        float sv[64];
        tmem_ld32(tmem + RBF_SCOL + lane_off, sv);
        tmem_ld32(tmem + RBF_SCOL + lane_off + 32, sv + 32);
        tc_fence_before();
        mbar_arrive(sfree);
        const uint32_t pb = pc & 1;
        if (!__all_sync(0xffffffffu, mbar_wait(pfree + pb, ((pc >> 1) & 1) ^ 1, err))) {
          ok = false;
          break;
        }
        if (PT) tc_fence_after();  // the MMA that read this P buffer has completed
        const float* ck = reinterpret_cast<const float*>(st + (it % RBF_S) * STAGE + K_BYTES + V_BYTES);
        const int64_t dcol = gq - (a.kbase + b * RBF_BJ);  // diagonal column in this block, if any
        const bool diag = __any_sync(0xffffffffu, dcol >= 0 && dcol < RBF_BJ);
        float dval = 1.f;
        if (diag && a.klog2w != 0.f && dcol >= 0 && dcol < RBF_BJ) {
          const int64_t e = a.knwin - 1 - (b * RBF_BJ + dcol) / a.kwlen;
          if (e > 0) dval = exp2f((float)e * a.klog2w);
        }
        unsigned char* prow = ps + pb * P_BYTES + (warp * 32 + lane) * 128;
        const int sw = lane & 7;  // (row & 7) with row = 32 * warp + lane
        uint32_t pw[32];          // P row as BF16 pairs (TMEM form)
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          float e[8];
          const float4 k0 = reinterpret_cast<const float4*>(ck)[2 * q];
          const float4 k1 = reinterpret_cast<const float4*>(ck)[2 * q + 1];
          const float kc[8] = {k0.x, k0.y, k0.z, k0.w, k1.x, k1.y, k1.z, k1.w};
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            const int col = 8 * q + u;
            const float x = fminf(fmaf(a.two_g, sv[col], cq + kc[u]), 0.f);
            e[u] = ex2_approx(x);
            if (diag && col == dcol) e[u] = dval;
          }
          __nv_bfloat162 h[4] = {__floats2bfloat162_rn(e[0], e[1]), __floats2bfloat162_rn(e[2], e[3]),
                                 __floats2bfloat162_rn(e[4], e[5]), __floats2bfloat162_rn(e[6], e[7])};
          if (PT) {
#pragma unroll
            for (int u = 0; u < 4; ++u) pw[4 * q + u] = *reinterpret_cast<const uint32_t*>(&h[u]);
          } else {
            *reinterpret_cast<uint4*>(prow + ((q ^ sw) << 4)) = *reinterpret_cast<const uint4*>(h);
          }
        }
        if (PT) {
          tmem_st32(tmem + P_TCOL + pb * 32 + lane_off, pw);
          tc_fence_before();
        } else {
          fence_proxy_async();
        }
        mbar_arrive(pfull + pb);
      }
      if (!ok) break;
      // epilogue: O (128 x NC) of this unit, output columns ch * NC + c
      if (!epilogue_unit<NC, 0>(o, tmem, 0, un & 1, ofull, ofree, qt, ch, warp, lane, err)) break;
    }
  }
  drain_on_error(err);
  if (warp == 5) {
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
  }
}

// ---------------------------------------------------------------------------
// Adjoint of Y = K Omega^T (the kernel-sketch VJP) with K regenerated tile by
// tile. Given Ybar = dL/dY, with M = Ybar Omega and E = M o K (E_ii = 0:
// the diagonal entry of K is fixed at 1 and has no gradient),
//   dL/dgamma = -sum_ij E_ij d_ij^2,
//   dL/dx_i   = -2 gamma [ (rowsum(E)_i + colsum(E)_i) x_i - (E X)_i - (E^T X)_i ].
// One pass of this kernel, for a unit of 128 query points q and a range of
// 64-point key blocks j:
//   S = X_q X_j^T   and   M = A_q B_j^T        tcgen05, N = 64, into TMEM
//   E = M o exp2(2 g' S + c_q + c_j)           four warps, in registers;
//                                              row sums of E and the dgamma
//                                              terms accumulate per thread
//   O += E X_j                                 tcgen05, N = padded d, E read
//                                              from TMEM (two 32-column buffers)
// then O, the row sums and the dgamma terms go out with FP32 / FP64
// atomics. The first pass (A = Ybar, B = Omega^T) gives E X, rowsum(E) and
// dgamma; the second (A = Omega^T, B = Ybar) sees E^T and gives E^T X and
// colsum(E). K, M and E are never stored.
struct RbfVjpArgs {
  int64_t N;          // points
  int64_t nblocks;    // 64-point key blocks (N padded)
  int64_t bchunk;     // key blocks per split
  int qtiles, ksplit;
  const float* cval;  // c_p = -g' ||bf16(x_p)||^2, -inf past N
  float two_g;        // 2 g'
  float inv_g;        // 1 / g'  (d^2 = -(2 g' S + c_q + c_j) / g')
  float* S;           // N x d, += E X
  int64_t d;
  float* rsum;        // N, += row sums of E
  double* dgamma;     // += -sum E d^2 (first pass), or nullptr
};

template <int DK, int KK>
__global__ void __launch_bounds__(kThreads, 1)
    rbf_vjp_kernel(const __grid_constant__ CUtensorMap tmQx, const __grid_constant__ CUtensorMap tmKx,
                   const __grid_constant__ CUtensorMap tmQa, const __grid_constant__ CUtensorMap tmKb,
                   const __grid_constant__ CUtensorMap tmXt, RbfVjpArgs a, int* err) {
  constexpr int NS = 3;                     // key stages
  constexpr int DP = 64 * DK;               // padded features = output columns
  constexpr uint32_t QX = DK * RBF_BQ * 128;
  constexpr uint32_t QA = KK * RBF_BQ * 128;
  constexpr uint32_t KX = DK * RBF_BJ * 128;
  constexpr uint32_t KB = KK * RBF_BJ * 128;
  constexpr uint32_t XT = DP * 128;         // DP rows of 64 keys
  constexpr uint32_t STAGE = ((KX + KB + XT + 256 + 1023) / 1024) * 1024;
  constexpr uint32_t TS = 128, TM = 192;    // TMEM columns of S and M; O at 0
  constexpr uint32_t TE = 64;               // E buffers (BF16 pairs) at 64 and 96
  // The unit's query rows (X_q: 32 DK columns, A_q: 32 KK columns) are
  // copied into TMEM at its start by the E warps, so the S and M MMAs read
  // only the key-side operands from shared memory.
  constexpr uint32_t TQX = 256, TQA = TQX + 32 * DK;
  static_assert(TQA + 32 * KK <= 512, "query rows must fit TMEM");
  static_assert(DK == 1, "one 64-row box of X^T per key block");
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  unsigned char* qx = smem;
  unsigned char* qa = qx + QX;
  unsigned char* st = qa + QA;
  uint64_t* bar = reinterpret_cast<uint64_t*>(st + NS * STAGE);
  uint64_t* qfull = bar + 0;
  uint64_t* qempty = bar + 1;
  uint64_t* full = bar + 2;
  uint64_t* empty = full + NS;
  uint64_t* sfull = empty + NS;
  uint64_t* sfree = sfull + 1;
  uint64_t* pfull = sfree + 1;
  uint64_t* pfree = pfull + 2;
  uint64_t* ofull = pfree + 2;
  uint64_t* ofree = ofull + 1;
  uint64_t* qtm = ofree + 1;  // query rows copied into TMEM
  uint32_t* tbase = reinterpret_cast<uint32_t*>(qtm + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int total = a.qtiles * a.ksplit;
  if (threadIdx.x == 0) {
    mbar_init(qfull, 1);
    mbar_init(qempty, 128);
    mbar_init(qtm, 128);
    for (int s = 0; s < NS; ++s) {
      mbar_init(full + s, 1);
      mbar_init(empty + s, 1);
    }
    mbar_init(sfull, 1);
    mbar_init(sfree, 128);
    for (int p = 0; p < 2; ++p) {
      mbar_init(pfull + p, 128);
      mbar_init(pfree + p, 1);
    }
    mbar_init(ofull, 1);
    mbar_init(ofree, 128);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 5) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tbase)),
                 "r"(512)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tbase;
  auto decode = [&](int t, int& qt, int64_t& b0, int64_t& b1) {
    qt = t % a.qtiles;
    b0 = (int64_t)(t / a.qtiles) * a.bchunk;
    b1 = min(a.nblocks, b0 + a.bchunk);
  };

  if (warp == 4 && lane == 0) {
    // ---------------- TMA producer ----------------
    uint32_t it = 0, un = 0;
    bool ok = true;
    for (int t = blockIdx.x; t < total && ok; t += gridDim.x, ++un) {
      int qt;
      int64_t b0, b1;
      decode(t, qt, b0, b1);
      if (!mbar_wait(qempty, (un & 1) ^ 1, err)) break;
      mbar_expect_tx(qfull, QX + QA);
#pragma unroll
      for (int f = 0; f < DK; ++f) tma_load_2d(&tmQx, qfull, qx + f * RBF_BQ * 128, 64 * f, qt * RBF_BQ);
#pragma unroll
      for (int f = 0; f < KK; ++f) tma_load_2d(&tmQa, qfull, qa + f * RBF_BQ * 128, 64 * f, qt * RBF_BQ);
      for (int64_t b = b0; b < b1; ++b, ++it) {
        const int s = it % NS;
        const uint32_t ph = (it / NS) & 1;
        if (!mbar_wait(empty + s, ph ^ 1, err)) {
          ok = false;
          break;
        }
        unsigned char* sk = st + s * STAGE;
        mbar_expect_tx(full + s, KX + KB + XT + 256);
        const int kb = (int)(b * RBF_BJ);
#pragma unroll
        for (int f = 0; f < DK; ++f) tma_load_2d(&tmKx, full + s, sk + f * RBF_BJ * 128, 64 * f, kb);
#pragma unroll
        for (int f = 0; f < KK; ++f) tma_load_2d(&tmKb, full + s, sk + KX + f * RBF_BJ * 128, 64 * f, kb);
        tma_load_2d(&tmXt, full + s, sk + KX + KB, kb, 0);
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], 256, [%2];" ::"r"(
                smem_u32(sk + KX + KB + XT)),
            "l"(a.cval + b * RBF_BJ), "r"(smem_u32(full + s))
            : "memory");
      }
    }
  } else if (warp == 5 && lane == 0) {
    // ---------------- MMA issuer ----------------
    constexpr uint32_t id64 = idesc_bf16(RBF_BJ, false, false);
    constexpr uint32_t idD = idesc_bf16(DP, false, false);
    uint32_t it = 0, un = 0, g = 0, pc = 0;
    bool ok = true;
    auto out_mma = [&](int s, bool first) -> bool {
      const uint32_t pb = pc & 1;
      if (!mbar_wait(pfull + pb, (pc >> 1) & 1, err)) return false;
      tc_fence_after();
      const uint32_t ea = tmem + TE + pb * 32;
      const uint32_t xb = smem_u32(st + s * STAGE + KX + KB);
#pragma unroll
      for (int kk = 0; kk < RBF_BJ / 16; ++kk)
        umma_ts(tmem, ea + kk * 8, sdesc(xb + kk * 32, 16, 1024), idD, (!first || kk > 0) ? 1u : 0u);
      umma_commit(empty + s);
      umma_commit(pfree + pb);
      ++pc;
      return true;
    };
    for (int t = blockIdx.x; t < total && ok; t += gridDim.x, ++un) {
      int qt;
      int64_t b0, b1;
      decode(t, qt, b0, b1);
      if (!mbar_wait(qtm, un & 1, err)) break;
      int prev_s = -1;
      bool first = true;
      for (int64_t b = b0; b < b1; ++b, ++it) {
        const int s = it % NS;
        const uint32_t ph = (it / NS) & 1;
        if (!mbar_wait(full + s, ph, err) || !mbar_wait(sfree, (g & 1) ^ 1, err)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t kb = smem_u32(st + s * STAGE);
#pragma unroll
        for (int f = 0; f < DK; ++f)
#pragma unroll
          for (int kk = 0; kk < 4; ++kk)
            umma_ts(tmem + TS, tmem + TQX + f * 32 + kk * 8, sdesc(kb + f * RBF_BJ * 128 + kk * 32, 16, 1024), id64,
                    (f > 0 || kk > 0) ? 1u : 0u);
#pragma unroll
        for (int f = 0; f < KK; ++f)
#pragma unroll
          for (int kk = 0; kk < 4; ++kk)
            umma_ts(tmem + TM, tmem + TQA + f * 32 + kk * 8, sdesc(kb + KX + f * RBF_BJ * 128 + kk * 32, 16, 1024),
                    id64, (f > 0 || kk > 0) ? 1u : 0u);
        umma_commit(sfull);
        ++g;
        if (prev_s >= 0) {
          if (first && !mbar_wait(ofree, (un & 1) ^ 1, err)) {
            ok = false;
            break;
          }
          if (!out_mma(prev_s, first)) {
            ok = false;
            break;
          }
          first = false;
        }
        prev_s = s;
      }
      if (!ok) break;
      if (prev_s >= 0) {
        if (first && !mbar_wait(ofree, (un & 1) ^ 1, err)) break;
        if (!out_mma(prev_s, first)) break;
      }
      umma_commit(ofull);
    }
  } else if (warp < 4) {
    // ---------------- E tiles, row sums, dgamma, epilogue ----------------
    const uint32_t lane_off = (uint32_t)(warp * 32) << 16;
    uint32_t it = 0, un = 0, g = 0, pc = 0;
    for (int t = blockIdx.x; t < total; t += gridDim.x, ++un) {
      int qt;
      int64_t b0, b1;
      decode(t, qt, b0, b1);
      const int64_t gq = (int64_t)qt * RBF_BQ + warp * 32 + lane;  // query point of this thread
      const bool live = gq < a.N;
      const float cq = live ? a.cval[gq] : 0.f;
      float rs_acc = 0.f, dg_acc = 0.f;
      {
        // this thread's X_q and A_q rows into TMEM (the S and M MMAs of the
        // previous unit have completed: their tiles were all read), then
        // free the shared-memory copies for the next unit's loads
        if (!__all_sync(0xffffffffu, mbar_wait(qfull, un & 1, err))) break;
        const int row = warp * 32 + lane;
#pragma unroll
        for (int f = 0; f < DK + KK; ++f) {
          uint32_t qw[32];
          const unsigned char* qrowp = (f < DK ? qx + f * RBF_BQ * 128 : qa + (f - DK) * RBF_BQ * 128) + row * 128;
#pragma unroll
          for (int c = 0; c < 8; ++c) {
            const uint4 v = *reinterpret_cast<const uint4*>(qrowp + ((c ^ (row & 7)) << 4));
            qw[4 * c] = v.x, qw[4 * c + 1] = v.y, qw[4 * c + 2] = v.z, qw[4 * c + 3] = v.w;
          }
          tmem_st32(tmem + TQX + f * 32 + lane_off, qw);
        }
        tc_fence_before();
        mbar_arrive(qtm);
        fence_proxy_async();
        mbar_arrive(qempty);
      }
      bool ok = true;
      for (int64_t b = b0; b < b1; ++b, ++it, ++g, ++pc) {
        if (!__all_sync(0xffffffffu, mbar_wait(sfull, g & 1, err))) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t pb = pc & 1;
        if (!__all_sync(0xffffffffu, mbar_wait(pfree + pb, ((pc >> 1) & 1) ^ 1, err))) {
          ok = false;
          break;
        }
        tc_fence_after();  // the MMA that read this E buffer has completed
        const float* ck = reinterpret_cast<const float*>(st + (it % NS) * STAGE + KX + KB + XT);
        const int64_t dcol = gq - b * RBF_BJ;  // diagonal column of this block, if any
        uint32_t ew[32];                       // the E row as BF16 pairs (TMEM form)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          float sv[32], mv[32];
          tmem_ld32(tmem + TS + lane_off + 32 * h, sv);
          tmem_ld32(tmem + TM + lane_off + 32 * h, mv);
          if (h == 1) {
            tc_fence_before();
            mbar_arrive(sfree);
          }
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const float4 k0 = reinterpret_cast<const float4*>(ck)[8 * h + 2 * q];
            const float4 k1 = reinterpret_cast<const float4*>(ck)[8 * h + 2 * q + 1];
            const float kc[8] = {k0.x, k0.y, k0.z, k0.w, k1.x, k1.y, k1.z, k1.w};
            float e[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
              const int cl = 8 * q + u, col = 32 * h + cl;
              // clamped to [-256, 0]: 2^x is 0 below -126 either way, and
              // the padding keys (c = -inf, M = 0) give 0 * x = 0, not NaN
              const float x = fmaxf(fminf(fmaf(a.two_g, sv[cl], cq + kc[u]), 0.f), -256.f);
              float ev = mv[cl] * ex2_approx(x);
              if (col == dcol) ev = 0.f;
              rs_acc += ev;
              dg_acc = fmaf(ev, x, dg_acc);
              e[u] = ev;
            }
            __nv_bfloat162 hh[4] = {__floats2bfloat162_rn(e[0], e[1]), __floats2bfloat162_rn(e[2], e[3]),
                                    __floats2bfloat162_rn(e[4], e[5]), __floats2bfloat162_rn(e[6], e[7])};
#pragma unroll
            for (int u = 0; u < 4; ++u) ew[16 * h + 4 * q + u] = *reinterpret_cast<const uint32_t*>(&hh[u]);
          }
        }
        tmem_st32(tmem + TE + pb * 32 + lane_off, ew);
        tc_fence_before();
        mbar_arrive(pfull + pb);
      }
      if (!ok) break;
      // epilogue: O = (E X)_q for this unit's key range
      if (!__all_sync(0xffffffffu, mbar_wait(ofull, un & 1, err))) break;
      tc_fence_after();
#pragma unroll
      for (int c0 = 0; c0 < DP; c0 += 32) {
        float v[32];
        tmem_ld32(tmem + lane_off + c0, v);
        if (c0 + 32 >= DP) {
          tc_fence_before();
          mbar_arrive(ofree);
        }
        if (live) {
#pragma unroll
          for (int i = 0; i < 32; ++i)
            if (c0 + i < a.d) atomicAdd(a.S + gq * a.d + c0 + i, v[i]);
        }
      }
      if (live) atomicAdd(a.rsum + gq, rs_acc);
      if (a.dgamma) {
#pragma unroll
        for (int o = 16; o; o >>= 1) dg_acc += __shfl_xor_sync(0xffffffffu, dg_acc, o);
        // -sum E d^2 = sum E x / g' with x = -g' d^2
        if (lane == 0) atomicAdd(a.dgamma, (double)dg_acc * (double)a.inv_g);
      }
    }
  }
  drain_on_error(err);
  if (warp == 5) {
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
  }
}

}  // namespace tc
}  // namespace skema
