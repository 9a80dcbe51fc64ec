// tc_gemm.cuh -- a persistent BF16 x BF16 -> FP32 tensor-core GEMM for
// sm_100a (tcgen05.mma with accumulators in TMEM, operands staged by TMA),
// used by the BF16 form of the dense sketch.
//
// Work unit: a 128 x NT output tile (NT <= 256, multiple of 16) over one
// split of K. The grid is at most one CTA per SM; CTA b takes units b,
// b + gridDim.x, ... Roles (192 threads):
//   warp 4 (one lane)  TMA producer: runs ahead over all units of the CTA,
//                      filling an S-stage shared-memory ring (one 64-wide
//                      K step of A and B per stage);
//   warp 5 (one lane)  MMA issuer: four tcgen05.mma (K = 16) per stage into
//                      one of two TMEM accumulators, alternating per unit;
//                      warp 5 also allocates and frees the TMEM columns;
//   warps 0-3          epilogue: read the finished accumulator with
//                      tcgen05.ld (warp w owns TMEM lanes 32w..32w+31), hand
//                      it back to the MMA issuer, then store.
// With two accumulators the epilogue of one unit overlaps the main loop of
// the next.
//
// Output tile rows run along TMEM lanes, so consecutive lanes of a warp own
// consecutive output rows: callers orient each product so that the output's
// contiguous dimension is the row dimension (coalesced epilogue stores).
// Operands are 128-byte-swizzled (TMA SWIZZLE_128B). A comes from one of
// three tensor-map shapes (AMode); B is K-major (rows of 64 K-elements).
//
// Every wait is bounded by a timer; on time-out the waiting thread sets
// *err, all roles stop issuing, every thread meets the final barrier, TMEM
// is freed and the kernel returns. The host reports SKEMA_ETIMEOUT.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace skema {
namespace tc {

constexpr int BM = 128;      // tile rows (TMEM lanes)
constexpr int BK = 64;       // K per stage (one 128-byte swizzle row of BF16)
constexpr int kThreads = 192;
// Every wait is bounded by the limit the context keeps in its device status
// block (err[0] status, err[2..3] the limit in ns as one 64-bit word; 2 s
// unless skema_set_wait_limit changed it).
constexpr unsigned long long kWaitNs = 2000000000ull;  // default limit per wait

// Where the A tile of a K step comes from.
enum AMode : int {
  // 2-D map {K, rows}, K innermost: one box {64, 128} at (k, m0).
  A_KMAJ = 0,
  // Row-blocked 3-D map {64, rows, K/64} (64 K-elements of a row contiguous,
  // then the rows, then the 64-blocks of K): one box {64, 128, 1} at
  // (0, m0, k/64) -- a contiguous 16 KB run.
  A_KMAJ_BLK = 1,
  // Row-blocked 3-D map {64, K, M/64} (64 M-elements contiguous, then K,
  // then the 64-blocks of M), read MN-major: two boxes {64, 64, 1} at
  // (0, k, m0/64) and (0, k, m0/64 + 1) -- two contiguous 8 KB runs.
  A_MN_BLK = 2,
};

struct OutSpec {
  // columns [0, split) of the tile row space go to p0, [split, ncols) to p1
  float* p0;
  __nv_bfloat16* p1;      // BF16 output for the second part (or nullptr)
  __nv_bfloat16* p1lo;    // with p1: the BF16 rounding of (value - p1), so p1 + p1lo
                          // carries about 16 significant bits (or nullptr)
  float* p1f;             // FP32 output for the second part (or nullptr)
  int64_t rs0, cs0, rs1, cs1;
  float alpha0, beta0, alpha1, beta1;
  int64_t rows;           // valid output rows (global row index < rows)
  int64_t split, ncols;   // valid output columns
  int atomic0;            // 1: atomicAdd alpha0*acc into p0 (split-K)
  int atomic1;            // 1: atomicAdd alpha1*acc into p1f (split-K)
  // Window weights of the second part: row r (of windows of row_wlen rows,
  // row_nwin of them) is scaled by 2^((row_nwin - 1 - r / row_wlen) *
  // row_log2w); row_log2w = 0 leaves it unweighted.
  float row_log2w;
  int64_t row_wlen, row_nwin;
  // When set, alpha0 and alpha1 of row r are multiplied by
  // scale[r / scale_wlen] (device values written by an earlier launch: the
  // FP8 form's 1 / (scale_A scale_map) of each window).
  const float* scale;
  int64_t scale_wlen;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ unsigned long long now_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait; false on time-out or when another thread already failed.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, int* err) {
  if (mbar_try(b, parity)) return true;
  const unsigned long long t0 = now_ns();
  const unsigned long long limit = *reinterpret_cast<const unsigned long long*>(err + 2);
  while (true) {
    if (mbar_try(b, parity)) return true;
    if (*(volatile int*)err) return false;
    if (now_ns() - t0 > limit) {
      atomicExch(err, 1);
      return false;
    }
  }
}
__device__ __forceinline__ void tma_load_2d(const CUtensorMap* tm, uint64_t* bar, void* dst, int c0,
                                            int c1) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
          smem_u32(dst)),
      "l"(tm), "r"(smem_u32(bar)), "r"(c0), "r"(c1)
      : "memory");
}
__device__ __forceinline__ void tma_load_3d(const CUtensorMap* tm, uint64_t* bar, void* dst, int c0, int c1,
                                            int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(
          smem_u32(dst)),
      "l"(tm), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}
__device__ __forceinline__ void tma_store_3d(const CUtensorMap* tm, const void* src, int c0, int c1, int c2) {
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%2, %3, %4}], [%1];" ::"l"(tm),
               "r"(smem_u32(src)), "r"(c0), "r"(c1), "r"(c2)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read_all() {
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
// Orders this thread's generic-proxy shared-memory writes before later
// async-proxy reads (tensor-core operands, TMA stores).
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// End of a tensor-core kernel: every thread of the CTA meets here. When a
// wait timed out anywhere (in this CTA or another), copies and tensor-core
// operations this CTA issued may still be in flight, also where the thread
// that issued them finished normally: they get a bounded 20 ms to land before
// the shared memory and TMEM they target are released. The predicate is
// reduced over the block, so every thread takes the same branch.
__device__ __forceinline__ void drain_on_error(int* err) {
  tc_fence_before();
  if (__syncthreads_or(*(volatile int*)err != 0)) {
    if (threadIdx.x == 0) {
      const unsigned long long t0 = now_ns();
      while (now_ns() - t0 < 20000000ull) __nanosleep(1000);
    }
    __syncthreads();
  }
}
// Shared-memory matrix descriptor, 128-byte swizzle, sm_100 version field.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // version
  d |= (uint64_t)2 << 61;  // SWIZZLE_128B
  return d;
}
// Instruction descriptor: BF16 x BF16 -> F32, M = 128, N = n.
__host__ __device__ constexpr uint32_t idesc_bf16(int n, bool a_mn_major, bool b_mn_major) {
  return (1u << 4)                        // D: F32
         | (1u << 7)                      // A: BF16
         | (1u << 10)                     // B: BF16
         | ((a_mn_major ? 1u : 0u) << 15) // A major
         | ((b_mn_major ? 1u : 0u) << 16) // B major
         | ((uint32_t)(n >> 3) << 17)     // N / 8
         | ((uint32_t)(BM >> 4) << 24);   // M / 16
}
// Instruction descriptor: E4M3 x E4M3 -> F32 (kind::f8f6f4), both operands
// K-major, M = 128, N = n.
__host__ __device__ constexpr uint32_t idesc_e4m3(int n) {
  return (1u << 4)                        // D: F32
         | (0u << 7)                      // A: E4M3
         | (0u << 10)                     // B: E4M3
         | ((uint32_t)(n >> 3) << 17)     // N / 8
         | ((uint32_t)(BM >> 4) << 24);   // M / 16
}
__device__ __forceinline__ void umma_f8(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, p;\n}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void umma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}
// MMA with A from TMEM (lane = row of A, K packed two BF16 per 32-bit
// column, lower half first) and B from shared memory.
__device__ __forceinline__ void umma_ts(uint32_t d, uint32_t a_tmem, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n}\n" ::"r"(d),
      "r"(a_tmem), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}
// 32 consecutive TMEM columns of this thread's lane from v, then the wait for
// the store (one asm statement, so the registers stay live until it lands).
__device__ __forceinline__ void tmem_st32(uint32_t taddr, const uint32_t* v) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,"
      "%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};\n\t"
      "tcgen05.wait::st.sync.aligned;" ::"r"(taddr),
      "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]), "r"(v[9]),
      "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15]), "r"(v[16]), "r"(v[17]), "r"(v[18]),
      "r"(v[19]), "r"(v[20]), "r"(v[21]), "r"(v[22]), "r"(v[23]), "r"(v[24]), "r"(v[25]), "r"(v[26]), "r"(v[27]),
      "r"(v[28]), "r"(v[29]), "r"(v[30]), "r"(v[31])
      : "memory");
}
// 16 consecutive TMEM columns of this thread's lane; the load and its wait
// are one asm statement so no use of the registers can precede the wait.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
// 32 consecutive columns as two loads in flight and one wait.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%32];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, "
      "[%33];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr), "r"(taddr + 16)
      : "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Work units: unit t -> (mt, nt, ks). M fastest when m_fast, else N.
// Work of a launch: mtiles x ntiles output tiles of ksteps K-steps each.
// Split mode (streamk = 0): unit t = (mt, nt, ks) covers K-steps
// [ks kcsteps, (ks + 1) kcsteps); CTA b takes units b, b + gridDim.x, ...
// Stream-K mode (streamk = 1): the tiles' K-steps in tile order are cut into
// gridDim.x equal runs and CTA b takes run b, so a tile is shared by at most
// a few CTAs and gets that many partial sums (added atomically), whatever
// the tile count is against the SM count.
struct Grid3 {
  int mtiles, ntiles, ksplit;
  int m_fast;
  int64_t ksteps;
  int kcsteps;
  int streamk;
};
__device__ __forceinline__ void decode_unit(const Grid3& g, int t, int& mt, int& nt, int& ks) {
  if (g.m_fast) {
    mt = t % g.mtiles;
    t /= g.mtiles;
    nt = t % g.ntiles;
    ks = t / g.ntiles;
  } else {
    nt = t % g.ntiles;
    t /= g.ntiles;
    mt = t % g.mtiles;
    ks = t / g.mtiles;
  }
}

// A CTA's next segment of work: tile (mt, nt) and its K-steps [kt0, kt1).
struct Sched {
  int64_t pos, end;  // stream-K: this CTA's run of K-steps
  int t;             // split mode: next unit
};
__device__ __forceinline__ void sched_init(const Grid3& g, Sched& s) {
  const int64_t T = (int64_t)g.mtiles * g.ntiles * g.ksteps;
  s.pos = T * blockIdx.x / gridDim.x;
  s.end = T * (blockIdx.x + 1) / gridDim.x;
  s.t = blockIdx.x;
}
__device__ __forceinline__ bool next_seg(const Grid3& g, Sched& s, int& mt, int& nt, int& kt0, int& kt1) {
  int ks;
  if (g.streamk) {
    if (s.pos >= s.end) return false;
    const int64_t tile = s.pos / g.ksteps;
    kt0 = (int)(s.pos - tile * g.ksteps);
    kt1 = (int)min(g.ksteps, (int64_t)kt0 + (s.end - s.pos));
    s.pos += kt1 - kt0;
    decode_unit(g, (int)tile, mt, nt, ks);
    return true;
  }
  if (s.t >= g.mtiles * g.ntiles * g.ksplit) return false;
  decode_unit(g, s.t, mt, nt, ks);
  kt0 = ks * g.kcsteps;
  kt1 = (int)min(g.ksteps, (int64_t)kt0 + g.kcsteps);
  s.t += gridDim.x;
  return true;
}

// Stores one finished 128 x NT accumulator (warps 0-3, warp w on TMEM lanes
// 32w..32w+31): waits for it, reads it 16 columns at a time, hands it back
// to the MMA issuer after the last read, and writes the columns per OutSpec.
// False when the wait failed (the warp then stops).
template <int NT, uint32_t TCOLS>
__device__ __forceinline__ bool epilogue_unit(const OutSpec& o, uint32_t tmem, uint32_t acc, uint32_t aph,
                                              uint64_t* tfull, uint64_t* tempty, int mt, int nt, int warp,
                                              int lane, int* err) {
  // tcgen05.ld is warp-collective: the whole warp reads TMEM or none of it
  if (!__all_sync(0xffffffffu, mbar_wait(tfull + acc, aph, err))) return false;
  tc_fence_after();
  const int64_t row = (int64_t)mt * BM + warp * 32 + lane;
  const uint32_t taddr = tmem + acc * TCOLS + ((uint32_t)(warp * 32) << 16);
  float alpha0 = o.alpha0, alpha1 = o.alpha1;
  if (o.scale && row < o.rows) {
    const float sc = o.scale[row / o.scale_wlen];
    alpha0 *= sc;
    alpha1 *= sc;
  }
  if (o.row_log2w != 0.f && row < o.rows) {
    const int64_t e = o.row_nwin - 1 - row / o.row_wlen;
    if (e > 0) alpha1 *= exp2f((float)e * o.row_log2w);
  }
  for (int c0 = 0; c0 < NT; c0 += 32) {
    // 32 columns per TMEM round trip (16 for an odd last chunk)
    const int w = (c0 + 32 <= NT) ? 32 : 16;
    float v[32];
    if (w == 32)
      tmem_ld32(taddr + c0, v);
    else
      tmem_ld16(taddr + c0, v);
    if (c0 + w >= NT) {
      // last read of this accumulator: hand it back before storing
      tc_fence_before();
      mbar_arrive(tempty + acc);
    }
    if (row >= o.rows) continue;
#pragma unroll
    for (int i = 0; i < 32; ++i) {
      if (i >= w) break;
      const int64_t col = (int64_t)nt * NT + c0 + i;
      if (col >= o.ncols) continue;
      if (col < o.split) {
        float* p = o.p0 + row * o.rs0 + col * o.cs0;
        if (o.atomic0)
          atomicAdd(p, alpha0 * v[i]);
        else
          *p = (o.beta0 == 0.f) ? alpha0 * v[i] : fmaf(o.beta0, *p, alpha0 * v[i]);
      } else {
        const int64_t cc = col - o.split;
        if (o.p1) {
          const float x = alpha1 * v[i];
          const __nv_bfloat16 hi = __float2bfloat16(x);
          o.p1[row * o.rs1 + cc * o.cs1] = hi;
          if (o.p1lo) o.p1lo[row * o.rs1 + cc * o.cs1] = __float2bfloat16(x - __bfloat162float(hi));
        } else if (o.p1f) {
          float* p = o.p1f + row * o.rs1 + cc * o.cs1;
          if (o.atomic1)
            atomicAdd(p, alpha1 * v[i]);
          else
            *p = (o.beta1 == 0.f) ? alpha1 * v[i] : fmaf(o.beta1, *p, alpha1 * v[i]);
        }
      }
    }
  }
  return true;
}

template <int NT, int S, int AMODE>
__global__ void __launch_bounds__(kThreads, 1)
    gemm_bf16_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                     Grid3 g, OutSpec o, int* err) {
  constexpr uint32_t A_BYTES = BM * BK * 2;  // 16 KB
  constexpr uint32_t B_BYTES = NT * BK * 2;
  constexpr uint32_t STAGE = ((A_BYTES + B_BYTES + 1023) / 1024) * 1024;
  constexpr uint32_t TCOLS = NT <= 32 ? 32 : NT <= 64 ? 64 : NT <= 128 ? 128 : 256;
  static_assert(NT % 16 == 0 && NT <= 256, "N tile");
  static_assert(2 * TCOLS <= 512, "two accumulators must fit TMEM");
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + S * STAGE);
  uint64_t* empty = full + S;
  uint64_t* tfull = empty + S;   // [2] accumulator ready (MMA -> epilogue)
  uint64_t* tempty = tfull + 2;  // [2] accumulator drained (epilogue -> MMA)
  uint32_t* tbase = reinterpret_cast<uint32_t*>(tempty + 2);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(full + s, 1);
      mbar_init(empty + s, 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(tfull + a, 1);
      mbar_init(tempty + a, 4 * 32);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 5) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tbase)),
                 "r"(2 * TCOLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tbase;

  if (warp == 4 && lane == 0) {
    // ---------------- TMA producer ----------------
    uint32_t it = 0;
    bool ok = true;
    Sched sc;
    sched_init(g, sc);
    int mt, nt, kt0, kt1;
    while (ok && next_seg(g, sc, mt, nt, kt0, kt1)) {
      const int KT = kt1 - kt0;
      for (int kt = 0; kt < KT; ++kt, ++it) {
        const int s = it % S;
        const uint32_t ph = (it / S) & 1;
        if (!mbar_wait(empty + s, ph ^ 1, err)) {
          ok = false;
          break;
        }
        unsigned char* sa = smem + s * STAGE;
        unsigned char* sb = sa + A_BYTES;
        mbar_expect_tx(full + s, A_BYTES + B_BYTES);
        const int kc = (kt0 + kt) * BK;
        if (AMODE == A_KMAJ) {
          tma_load_2d(&tmA, full + s, sa, kc, mt * BM);
        } else if (AMODE == A_KMAJ_BLK) {
          tma_load_3d(&tmA, full + s, sa, 0, mt * BM, kc / BK);
        } else {
          tma_load_3d(&tmA, full + s, sa, 0, kc, 2 * mt);
          tma_load_3d(&tmA, full + s, sa + 8192, 0, kc, 2 * mt + 1);
        }
        tma_load_2d(&tmB, full + s, sb, kc, nt * NT);
      }
    }
  } else if (warp == 5 && lane == 0) {
    // ---------------- MMA issuer ----------------
    constexpr uint32_t idesc = idesc_bf16(NT, AMODE == A_MN_BLK, false);
    uint32_t it = 0, tcount = 0;
    bool ok = true;
    Sched sc;
    sched_init(g, sc);
    int mt, nt, kt0, kt1;
    while (ok && next_seg(g, sc, mt, nt, kt0, kt1)) {
      const int KT = kt1 - kt0;
      const uint32_t acc = tcount & 1, aph = (tcount >> 1) & 1;
      if (!mbar_wait(tempty + acc, aph ^ 1, err)) break;
      tc_fence_after();
      const uint32_t d = tmem + acc * TCOLS;
      for (int kt = 0; kt < KT; ++kt, ++it) {
        const int s = it % S;
        const uint32_t ph = (it / S) & 1;
        if (!mbar_wait(full + s, ph, err)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t sa = smem_u32(smem + s * STAGE);
        const uint32_t sb = sa + A_BYTES;
#pragma unroll
        for (int kk = 0; kk < BK / 16; ++kk) {
          const uint64_t ad =
              AMODE == A_MN_BLK ? sdesc(sa + kk * 2048, 8192, 1024) : sdesc(sa + kk * 32, 16, 1024);
          const uint64_t bd = sdesc(sb + kk * 32, 16, 1024);
          umma(d, ad, bd, idesc, (kt > 0 || kk > 0) ? 1u : 0u);
        }
        umma_commit(empty + s);
      }
      if (ok) umma_commit(tfull + acc);
      ++tcount;
    }
  } else if (warp < 4) {
    // ---------------- epilogue ----------------
    uint32_t tcount = 0;
    Sched sc;
    sched_init(g, sc);
    int mt, nt, kt0, kt1;
    for (; next_seg(g, sc, mt, nt, kt0, kt1); ++tcount) {
      const uint32_t acc = tcount & 1, aph = (tcount >> 1) & 1;
      if (!epilogue_unit<NT, TCOLS>(o, tmem, acc, aph, tfull, tempty, mt, nt, warp, lane, err)) break;
    }
  }
  drain_on_error(err);
  if (warp == 5) {
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * TCOLS) : "memory");
  }
}

// ---------------------------------------------------------------------------
// The FP8 form of the same GEMM: E4M3 x E4M3 -> FP32 (tcgen05 kind::f8f6f4),
// both operands K-major from 2-D maps, 128 K-elements (one 128-byte swizzle
// row of bytes) per stage and four MMAs of K = 32 per stage. The operand
// scales are folded into the epilogue through OutSpec::scale.
template <int NT, int S>
__global__ void __launch_bounds__(kThreads, 1)
    gemm_fp8_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, Grid3 g,
                    OutSpec o, int* err) {
  constexpr int BK8 = 128;
  constexpr uint32_t A_BYTES = BM * BK8;  // 16 KB
  constexpr uint32_t B_BYTES = NT * BK8;
  constexpr uint32_t STAGE = ((A_BYTES + B_BYTES + 1023) / 1024) * 1024;
  constexpr uint32_t TCOLS = NT <= 32 ? 32 : NT <= 64 ? 64 : NT <= 128 ? 128 : 256;
  static_assert(NT % 16 == 0 && NT <= 256, "N tile");
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + S * STAGE);
  uint64_t* empty = full + S;
  uint64_t* tfull = empty + S;
  uint64_t* tempty = tfull + 2;
  uint32_t* tbase = reinterpret_cast<uint32_t*>(tempty + 2);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(full + s, 1);
      mbar_init(empty + s, 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(tfull + a, 1);
      mbar_init(tempty + a, 4 * 32);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 5) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tbase)),
                 "r"(2 * TCOLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tbase;

  if (warp == 4 && lane == 0) {
    uint32_t it = 0;
    bool ok = true;
    Sched sc;
    sched_init(g, sc);
    int mt, nt, kt0, kt1;
    while (ok && next_seg(g, sc, mt, nt, kt0, kt1)) {
      const int KT = kt1 - kt0;
      for (int kt = 0; kt < KT; ++kt, ++it) {
        const int s = it % S;
        const uint32_t ph = (it / S) & 1;
        if (!mbar_wait(empty + s, ph ^ 1, err)) {
          ok = false;
          break;
        }
        unsigned char* sa = smem + s * STAGE;
        mbar_expect_tx(full + s, A_BYTES + B_BYTES);
        const int kc = (kt0 + kt) * BK8;
        tma_load_2d(&tmA, full + s, sa, kc, mt * BM);
        tma_load_2d(&tmB, full + s, sa + A_BYTES, kc, nt * NT);
      }
    }
  } else if (warp == 5 && lane == 0) {
    constexpr uint32_t idesc = idesc_e4m3(NT);
    uint32_t it = 0, tcount = 0;
    bool ok = true;
    Sched sc;
    sched_init(g, sc);
    int mt, nt, kt0, kt1;
    while (ok && next_seg(g, sc, mt, nt, kt0, kt1)) {
      const int KT = kt1 - kt0;
      const uint32_t acc = tcount & 1, aph = (tcount >> 1) & 1;
      if (!mbar_wait(tempty + acc, aph ^ 1, err)) break;
      tc_fence_after();
      const uint32_t d = tmem + acc * TCOLS;
      for (int kt = 0; kt < KT; ++kt, ++it) {
        const int s = it % S;
        const uint32_t ph = (it / S) & 1;
        if (!mbar_wait(full + s, ph, err)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t sa = smem_u32(smem + s * STAGE);
        const uint32_t sb = sa + A_BYTES;
#pragma unroll
        for (int kk = 0; kk < BK8 / 32; ++kk)
          umma_f8(d, sdesc(sa + kk * 32, 16, 1024), sdesc(sb + kk * 32, 16, 1024), idesc,
                  (kt > 0 || kk > 0) ? 1u : 0u);
        umma_commit(empty + s);
      }
      if (ok) umma_commit(tfull + acc);
      ++tcount;
    }
  } else if (warp < 4) {
    uint32_t tcount = 0;
    Sched sc;
    sched_init(g, sc);
    int mt, nt, kt0, kt1;
    for (; next_seg(g, sc, mt, nt, kt0, kt1); ++tcount) {
      const uint32_t acc = tcount & 1, aph = (tcount >> 1) & 1;
      if (!epilogue_unit<NT, TCOLS>(o, tmem, acc, aph, tfull, tempty, mt, nt, warp, lane, err)) break;
    }
  }
  drain_on_error(err);
  if (warp == 5) {
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * TCOLS) : "memory");
  }
}

// ---------------------------------------------------------------------------
// The same GEMM with A read as FP32 and rounded to BF16 inside the kernel,
// for X^T = A_w^T Upsilon~_w^T straight from the FP32 window: M runs over
// the window's columns, K over its rows. Each K step's A tile (64 window
// rows x 128 columns) arrives by TMA as FP32; four converter warps round it
// into the 128-byte-swizzled K-major BF16 operand, and one converter thread
// stores that operand with TMA into the row-blocked BF16 copy of the window
// (A16, A_MN_BLK / A_KMAJ_BLK shape) that the [Y|T] product reads next. So
// every element of the window is read from HBM once as FP32 and written
// once as BF16, and no separate conversion pass runs.
//   AROW = false: column-major window (rows contiguous); the FP32 tile is
//                 two 128-byte-swizzled boxes {32 rows, 128 columns}.
//   AROW = true:  row-major window (columns contiguous); four boxes
//                 {32 columns, 64 rows}.
// Threads: warps 0-3 epilogue, warp 4 TMA producer of the FP32 tiles,
// warp 5 MMA issuer, warps 6-9 converters, warp 10 TMA producer of the B
// tiles, warp 11 (STT) the A16 store thread. The two producers are separate so that the FP32 loads run up to S1
// stages ahead whatever the state of the BF16 ring (one thread issuing
// both waited for a free BF16 stage before each next FP32 load, which kept
// fewer FP32 loads in flight). Rings: S1 FP32 stages (producer -> converters) and
// S2 BF16 stages (A from the converters, B by TMA -> MMA); a BF16 stage is
// free again when the MMAs that read it are done and the TMA store of its
// A tile has read it. (Copying the tile out with plain 16-byte stores
// measured slower both from the converter threads, with 4 FP32 + 2 BF16
// stages, by 9 %, and from a warp of its own, by 27 %.)
//   STT = false: converter thread 0 issues each A tile's TMA store after
//                its stage is full and releases a stage one store later.
//   STT = true:  warp 11's first lane does it: it waits for the stage to
//                be full, issues the store, waits for the store to have
//                read the stage and releases it at once.
constexpr int kThreadsA32 = 352;
constexpr int kThreadsA32St = 384;

template <int NT, int S1, int S2, bool AROW, bool AMAX, bool STT>
__global__ void __launch_bounds__(kThreadsA32St, 1)
    gemm_a32_kernel(const __grid_constant__ CUtensorMap tmA32, const __grid_constant__ CUtensorMap tmB,
                    const __grid_constant__ CUtensorMap tmA16, Grid3 g, OutSpec o, uint32_t* amax, int* err) {
  constexpr uint32_t A32_BYTES = BM * BK * 4;  // 32 KB
  constexpr uint32_t A_BYTES = BM * BK * 2;    // 16 KB
  constexpr uint32_t B_BYTES = NT * BK * 2;
  constexpr uint32_t STAGE = ((A_BYTES + B_BYTES + 1023) / 1024) * 1024;
  constexpr uint32_t TCOLS = NT <= 32 ? 32 : NT <= 64 ? 64 : NT <= 128 ? 128 : 256;
  static_assert(NT % 16 == 0 && NT <= 256, "N tile");
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  unsigned char* st32 = smem;                    // S1 x A32_BYTES
  unsigned char* stbf = smem + S1 * A32_BYTES;   // S2 x STAGE
  uint64_t* f32full = reinterpret_cast<uint64_t*>(stbf + S2 * STAGE);
  uint64_t* f32empty = f32full + S1;
  uint64_t* full = f32empty + S1;
  uint64_t* empty = full + S2;
  uint64_t* tfull = empty + S2;
  uint64_t* tempty = tfull + 2;
  uint32_t* tbase = reinterpret_cast<uint32_t*>(tempty + 2);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int s = 0; s < S1; ++s) {
      mbar_init(f32full + s, 1);
      mbar_init(f32empty + s, 128);
    }
    for (int s = 0; s < S2; ++s) {
      mbar_init(full + s, 1 + 128);  // producer (B bytes) + converters (A tile)
      mbar_init(empty + s, 2);       // MMA commit + A-tile store drained
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(tfull + a, 1);
      mbar_init(tempty + a, 4 * 32);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 5) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tbase)),
                 "r"(2 * TCOLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tbase;

  if (warp == 4 && lane == 0) {
    // ---------------- TMA producer: FP32 tiles ----------------
    uint32_t it = 0;
    bool ok = true;
    Sched sc;
    sched_init(g, sc);
    int mt, nt, kt0, kt1;
    while (ok && next_seg(g, sc, mt, nt, kt0, kt1)) {
      const int KT = kt1 - kt0;
      for (int kt = 0; kt < KT; ++kt, ++it) {
        const int s1 = it % S1;
        const uint32_t ph1 = (it / S1) & 1;
        const int kc = (kt0 + kt) * BK;
        if (!mbar_wait(f32empty + s1, ph1 ^ 1, err)) {
          ok = false;
          break;
        }
        unsigned char* a32 = st32 + s1 * A32_BYTES;
        mbar_expect_tx(f32full + s1, A32_BYTES);
        if (!AROW) {
          tma_load_2d(&tmA32, f32full + s1, a32, kc, mt * BM);
          tma_load_2d(&tmA32, f32full + s1, a32 + 16384, kc + 32, mt * BM);
        } else {
#pragma unroll
          for (int q = 0; q < 4; ++q) tma_load_2d(&tmA32, f32full + s1, a32 + q * 8192, mt * BM + 32 * q, kc);
        }
      }
    }
  } else if (warp == 10 && lane == 0) {
    // ---------------- TMA producer: B tiles ----------------
    uint32_t it = 0;
    bool ok = true;
    Sched sc;
    sched_init(g, sc);
    int mt, nt, kt0, kt1;
    while (ok && next_seg(g, sc, mt, nt, kt0, kt1)) {
      const int KT = kt1 - kt0;
      for (int kt = 0; kt < KT; ++kt, ++it) {
        const int s2 = it % S2;
        const uint32_t ph2 = (it / S2) & 1;
        const int kc = (kt0 + kt) * BK;
        if (!mbar_wait(empty + s2, ph2 ^ 1, err)) {
          ok = false;
          break;
        }
        mbar_expect_tx(full + s2, B_BYTES);
        tma_load_2d(&tmB, full + s2, stbf + s2 * STAGE + A_BYTES, kc, nt * NT);
      }
    }
  } else if (warp == 5 && lane == 0) {
    // ---------------- MMA issuer ----------------
    constexpr uint32_t idesc = idesc_bf16(NT, false, false);
    uint32_t it = 0, tcount = 0;
    bool ok = true;
    Sched sc;
    sched_init(g, sc);
    int mt, nt, kt0, kt1;
    while (ok && next_seg(g, sc, mt, nt, kt0, kt1)) {
      const int KT = kt1 - kt0;
      const uint32_t acc = tcount & 1, aph = (tcount >> 1) & 1;
      if (!mbar_wait(tempty + acc, aph ^ 1, err)) break;
      tc_fence_after();
      const uint32_t d = tmem + acc * TCOLS;
      for (int kt = 0; kt < KT; ++kt, ++it) {
        const int s2 = it % S2;
        const uint32_t ph2 = (it / S2) & 1;
        if (!mbar_wait(full + s2, ph2, err)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t sa = smem_u32(stbf + s2 * STAGE);
        const uint32_t sb = sa + A_BYTES;
#pragma unroll
        for (int kk = 0; kk < BK / 16; ++kk)
          umma(d, sdesc(sa + kk * 32, 16, 1024), sdesc(sb + kk * 32, 16, 1024), idesc, (kt > 0 || kk > 0) ? 1u : 0u);
        umma_commit(empty + s2);
      }
      if (ok) umma_commit(tfull + acc);
      ++tcount;
    }
  } else if (warp >= 6 && warp < 10) {
    // ---------------- converters ----------------
    const int ct = threadIdx.x - 6 * 32;  // A-tile line (window column) of this thread
    uint32_t it = 0;
    bool ok = true;
    float mx = 0.f;  // max |a| over every value this thread converts (FP8 form's window scale)
    int pend = -1;   // (thread 0) BF16 stage whose A-tile store is still being read
    Sched sc;
    sched_init(g, sc);
    int mt, nt, kt0, kt1;
    while (ok && next_seg(g, sc, mt, nt, kt0, kt1)) {
      const int KT = kt1 - kt0;
      for (int kt = 0; kt < KT; ++kt, ++it) {
        const int s1 = it % S1, s2 = it % S2;
        const uint32_t ph1 = (it / S1) & 1, ph2 = (it / S2) & 1;
        if (!mbar_wait(f32full + s1, ph1, err) || !mbar_wait(empty + s2, ph2 ^ 1, err)) {
          ok = false;
          break;
        }
        const unsigned char* a32 = st32 + s1 * A32_BYTES;
        unsigned char* dst = stbf + s2 * STAGE + ct * 128;
        const int sw = ct & 7;
        if (!AROW) {
          // line ct of each FP32 box holds rows 32h..32h+31 of column ct
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            const unsigned char* src = a32 + (q >> 2) * 16384 + ct * 128;
            const int c = 2 * (q & 3);
            const float4 x = *reinterpret_cast<const float4*>(src + ((c ^ sw) << 4));
            const float4 y = *reinterpret_cast<const float4*>(src + (((c + 1) ^ sw) << 4));
            if (AMAX)
              mx = fmaxf(mx, fmaxf(fmaxf(fmaxf(fabsf(x.x), fabsf(x.y)), fmaxf(fabsf(x.z), fabsf(x.w))),
                                   fmaxf(fmaxf(fabsf(y.x), fabsf(y.y)), fmaxf(fabsf(y.z), fabsf(y.w)))));
            __nv_bfloat162 h[4] = {__floats2bfloat162_rn(x.x, x.y), __floats2bfloat162_rn(x.z, x.w),
                                   __floats2bfloat162_rn(y.x, y.y), __floats2bfloat162_rn(y.z, y.w)};
            *reinterpret_cast<uint4*>(dst + ((q ^ sw) << 4)) = *reinterpret_cast<const uint4*>(h);
          }
        } else {
          // column ct lives in box ct / 32 at element ct % 32 of every line
          const unsigned char* box = a32 + (ct >> 5) * 8192;
          const int jj = ct & 31;
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            float f[8];
#pragma unroll
            for (int e = 0; e < 8; ++e) {
              const int i = 8 * q + e;
              f[e] = *reinterpret_cast<const float*>(box + i * 128 + ((((jj >> 2) ^ (i & 7))) << 4) + (jj & 3) * 4);
              if (AMAX) mx = fmaxf(mx, fabsf(f[e]));
            }
            __nv_bfloat162 h[4] = {__floats2bfloat162_rn(f[0], f[1]), __floats2bfloat162_rn(f[2], f[3]),
                                   __floats2bfloat162_rn(f[4], f[5]), __floats2bfloat162_rn(f[6], f[7])};
            *reinterpret_cast<uint4*>(dst + ((q ^ sw) << 4)) = *reinterpret_cast<const uint4*>(h);
          }
        }
        fence_proxy_async();
        mbar_arrive(f32empty + s1);
        mbar_arrive(full + s2);
        if (!STT && ct == 0) {
          // all 128 lines written (and the B tile landed): store the BF16
          // tile. The stage is released once TMA has read it; that is waited
          // for one stage later (the store before this one must be read by
          // now), so this thread never stalls on its own fresh store.
          if (!mbar_wait(full + s2, ph2, err)) {
            ok = false;
            break;
          }
          fence_proxy_async();
          const int kc = (kt0 + kt) * BK;
          tma_store_3d(&tmA16, stbf + s2 * STAGE, 0, mt * BM, kc / BK);
          bulk_commit();
          if (pend >= 0) {
            asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");
            mbar_arrive(empty + pend);
          }
          pend = s2;
        }
      }
    }
    if (!STT && ct == 0) {
      bulk_wait_all();
      if (pend >= 0) mbar_arrive(empty + pend);
    }
    if (AMAX) {
      // |a| as bits: for non-negative floats the integer order is the float
      // order, so the window's amax is one integer atomicMax per warp. Every
      // lane leaves the loop above (the waits are bounded), so the whole
      // warp meets here.
      const uint32_t wm = __reduce_max_sync(0xffffffffu, __float_as_uint(mx));
      if ((ct & 31) == 0) atomicMax(amax, wm);
    }
  } else if (STT && warp == 11 && lane == 0) {
    // ---------------- A16 store thread ----------------
    uint32_t it = 0;
    bool ok = true;
    Sched sc;
    sched_init(g, sc);
    int mt, nt, kt0, kt1;
    while (ok && next_seg(g, sc, mt, nt, kt0, kt1)) {
      const int KT = kt1 - kt0;
      for (int kt = 0; kt < KT; ++kt, ++it) {
        const int s2 = it % S2;
        const uint32_t ph2 = (it / S2) & 1;
        if (!mbar_wait(full + s2, ph2, err)) {
          ok = false;
          break;
        }
        fence_proxy_async();
        tma_store_3d(&tmA16, stbf + s2 * STAGE, 0, mt * BM, kt0 + kt);
        bulk_commit();
        bulk_wait_read_all();
        mbar_arrive(empty + s2);
      }
    }
    bulk_wait_all();
  } else if (warp < 4) {
    // ---------------- epilogue ----------------
    uint32_t tcount = 0;
    Sched sc;
    sched_init(g, sc);
    int mt, nt, kt0, kt1;
    for (; next_seg(g, sc, mt, nt, kt0, kt1); ++tcount) {
      const uint32_t acc = tcount & 1, aph = (tcount >> 1) & 1;
      if (!epilogue_unit<NT, TCOLS>(o, tmem, acc, aph, tfull, tempty, mt, nt, warp, lane, err)) break;
    }
  }
  drain_on_error(err);
  if (warp == 5) {
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * TCOLS) : "memory");
  }
}

}  // namespace tc
}  // namespace skema
