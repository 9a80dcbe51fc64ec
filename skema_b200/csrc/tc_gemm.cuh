// tc_gemm.cuh -- a BF16 x BF16 -> FP32 tensor-core GEMM for sm_100a
// (tcgen05.mma with the accumulator in TMEM, operands staged by TMA), used by
// the BF16 form of the dense sketch.
//
// One CTA computes a 128 x NT output tile (NT <= 256, multiple of 16) over
// K in steps of 64, with an S-stage shared-memory ring:
//   warp 4 (one lane)  TMA producer: waits for a free stage, posts the bytes
//                      it expects and issues the operand loads;
//   warp 5 (one lane)  MMA issuer: waits for a full stage, issues four
//                      tcgen05.mma (K = 16 each) and commits the stage back;
//                      warp 5 also allocates and frees the TMEM columns;
//   warps 0-3          epilogue: wait for the accumulator, read TMEM lanes
//                      32w..32w+31 with tcgen05.ld and write the outputs.
// Output tile rows run along TMEM lanes, so consecutive lanes of a warp own
// consecutive output rows: callers orient each product so that the output's
// contiguous dimension is the row dimension (coalesced epilogue stores).
// Operands are 128-byte-swizzled (TMA SWIZZLE_128B). A is K-major (rows of
// 64 K-elements = 128 B, 8-row groups 1024 B apart) or MN-major (lines of 64
// M-elements per K index, K-groups of 8 lines 1024 B apart, the two 64-row
// halves of the tile 8 KB apart); B is K-major.
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
constexpr unsigned long long kWaitNs = 2000000000ull;  // 2 s per wait

struct OutSpec {
  // columns [0, split) of the tile row space go to p0, [split, ncols) to p1
  float* p0;
  __nv_bfloat16* p1;      // BF16 output for the second part (or nullptr)
  float* p1f;             // FP32 output for the second part (or nullptr)
  int64_t rs0, cs0, rs1, cs1;
  float alpha0, beta0, alpha1, beta1;
  int64_t rows;           // valid output rows (global row index < rows)
  int64_t split, ncols;   // valid output columns
  int atomic0;            // 1: atomicAdd alpha0*acc into p0 (split-K)
  int atomic1;            // 1: atomicAdd alpha1*acc into p1f (split-K)
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
  while (true) {
    if (mbar_try(b, parity)) return true;
    if (*(volatile int*)err) return false;
    if (now_ns() - t0 > kWaitNs) {
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
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
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
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Tile scheduling: tile t -> (mt, nt, ks). M fastest when m_fast, else N.
struct Grid3 {
  int mtiles, ntiles, ksplit;
  int m_fast;
};

template <int NT, int S, bool A_MN>
__global__ void __launch_bounds__(kThreads, 1)
    gemm_bf16_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                     int64_t K, int64_t kchunk, Grid3 g, OutSpec o, int* err) {
  constexpr uint32_t A_BYTES = BM * BK * 2;  // 16 KB
  constexpr uint32_t B_BYTES = NT * BK * 2;
  constexpr uint32_t STAGE = ((A_BYTES + B_BYTES + 1023) / 1024) * 1024;
  constexpr uint32_t TCOLS = NT <= 32 ? 32 : NT <= 64 ? 64 : NT <= 128 ? 128 : 256;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + S * STAGE);
  uint64_t* empty = full + S;
  uint64_t* accf = empty + S;
  uint32_t* tbase = reinterpret_cast<uint32_t*>(accf + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int t = blockIdx.x;
  int mt, nt, ks;
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
  const int64_t k0 = (int64_t)ks * kchunk;
  const int64_t k1 = min(K, k0 + kchunk);
  const int KT = (int)((k1 - k0 + BK - 1) / BK);

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(full + s, 1);
      mbar_init(empty + s, 1);
    }
    mbar_init(accf, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 5) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tbase)),
                 "r"(TCOLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tbase;

  if (warp == 4 && lane == 0 && KT > 0) {
    // ---------------- TMA producer ----------------
    for (int kt = 0; kt < KT; ++kt) {
      const int s = kt % S;
      const uint32_t ph = (kt / S) & 1;
      if (!mbar_wait(empty + s, ph ^ 1, err)) break;
      unsigned char* sa = smem + s * STAGE;
      unsigned char* sb = sa + A_BYTES;
      mbar_expect_tx(full + s, A_BYTES + B_BYTES);
      const int kc = (int)(k0 + (int64_t)kt * BK);
      if (A_MN) {
        tma_load_2d(&tmA, full + s, sa, mt * BM, kc);
        tma_load_2d(&tmA, full + s, sa + 8192, mt * BM + 64, kc);
      } else {
        tma_load_2d(&tmA, full + s, sa, kc, mt * BM);
      }
      tma_load_2d(&tmB, full + s, sb, kc, nt * NT);
    }
  } else if (warp == 5 && lane == 0 && KT > 0) {
    // ---------------- MMA issuer ----------------
    constexpr uint32_t idesc = idesc_bf16(NT, A_MN, false);
    bool ok = true;
    for (int kt = 0; kt < KT; ++kt) {
      const int s = kt % S;
      const uint32_t ph = (kt / S) & 1;
      if (!mbar_wait(full + s, ph, err)) {
        ok = false;
        break;
      }
      tc_fence_after();
      const uint32_t sa = smem_u32(smem + s * STAGE);
      const uint32_t sb = sa + A_BYTES;
#pragma unroll
      for (int kk = 0; kk < BK / 16; ++kk) {
        const uint64_t ad = A_MN ? sdesc(sa + kk * 2048, 8192, 1024) : sdesc(sa + kk * 32, 16, 1024);
        const uint64_t bd = sdesc(sb + kk * 32, 16, 1024);
        umma(tmem, ad, bd, idesc, (kt > 0 || kk > 0) ? 1u : 0u);
      }
      umma_commit(empty + s);
    }
    if (ok) umma_commit(accf);
  } else if (warp < 4) {
    // ---------------- epilogue ----------------
    // tcgen05.ld is warp-collective: the whole warp reads TMEM or none of it
    const bool have = __all_sync(0xffffffffu, KT > 0 && mbar_wait(accf, 0, err));
    if (have) tc_fence_after();
    const int64_t row = (int64_t)mt * BM + warp * 32 + lane;
    const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
    for (int c0 = 0; c0 < NT; c0 += 16) {
      float v[16];
      if (have) {
        tmem_ld16(taddr + c0, v);
      } else {
#pragma unroll
        for (int i = 0; i < 16; ++i) v[i] = 0.f;
      }
      if (!have || row >= o.rows) continue;
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int64_t col = (int64_t)nt * NT + c0 + i;
        if (col >= o.ncols) continue;
        if (col < o.split) {
          float* p = o.p0 + row * o.rs0 + col * o.cs0;
          if (o.atomic0)
            atomicAdd(p, o.alpha0 * v[i]);
          else
            *p = (o.beta0 == 0.f) ? o.alpha0 * v[i] : fmaf(o.beta0, *p, o.alpha0 * v[i]);
        } else {
          const int64_t cc = col - o.split;
          if (o.p1) {
            __nv_bfloat16* p = o.p1 + row * o.rs1 + cc * o.cs1;
            *p = __float2bfloat16(o.alpha1 * v[i]);
          } else if (o.p1f) {
            float* p = o.p1f + row * o.rs1 + cc * o.cs1;
            if (o.atomic1)
              atomicAdd(p, o.alpha1 * v[i]);
            else
              *p = (o.beta1 == 0.f) ? o.alpha1 * v[i] : fmaf(o.beta1, *p, o.alpha1 * v[i]);
          }
        }
      }
    }
  }
  if ((warp == 4 || warp == 5) && lane == 0 && *(volatile int*)err) {
    // a wait timed out somewhere: give the copies and MMAs this CTA still
    // has in flight a bounded time to land before its shared memory and
    // TMEM are released
    const unsigned long long t0 = now_ns();
    while (now_ns() - t0 < 20000000ull) __nanosleep(1000);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 5) {
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TCOLS) : "memory");
  }
}

}  // namespace tc
}  // namespace skema
