// philox.h -- Philox4x32-10 counter-based generator and the map-entry
// formulas shared by the host and device code of the library.
//
// Philox4x32-10 is the generator of Salmon, Moraes, Dror and Shaw, "Parallel
// random numbers: as easy as 1, 2, 3" (SC'11): ten rounds of two 32x32->64
// multiplies with the Weyl key schedule. Being counter-based, every map entry
// is a pure function of (seed, entry index), so any thread on any device can
// generate any entry and the result is bit-identical everywhere.
//
// The reference draws its maps from Kokkos' Random_XorShift64_Pool
// (src/Skema_DimRedux.hpp:115, 232, 244). That stream cannot be reproduced
// without Kokkos, so the maps here reproduce the reference's *distributions*
// and *shapes*, not its bits:
//   Gauss:      uniform on [-maxval, maxval), maxval = sqrt(2 ln(nrow*ncol))
//               (src/Skema_DimRedux.hpp:112,115);
//   SparseSign: zeta = max(2, min(ncol, 8)) column indices per stored row,
//               drawn uniformly with replacement and sorted ascending, with
//               independent +-1 values (src/Skema_DimRedux.hpp:205-251).
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define SKEMA_HD __host__ __device__ __forceinline__
#else
#define SKEMA_HD static inline
#endif

namespace skema {

struct u32x4 {
  uint32_t v[4];
};

SKEMA_HD void mulhilo32(uint32_t a, uint32_t b, uint32_t* hi, uint32_t* lo) {
  const uint64_t p = (uint64_t)a * (uint64_t)b;
  *hi = (uint32_t)(p >> 32);
  *lo = (uint32_t)p;
}

// One Philox4x32 block with 10 rounds.
SKEMA_HD u32x4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                             uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0, lo0, hi1, lo1;
    mulhilo32(M0, c0, &hi0, &lo0);
    mulhilo32(M1, c2, &hi1, &lo1);
    const uint32_t n0 = hi1 ^ c1 ^ k0;
    const uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
    k0 += W0;
    k1 += W1;
  }
  u32x4 out;
  out.v[0] = c0;
  out.v[1] = c1;
  out.v[2] = c2;
  out.v[3] = c3;
  return out;
}

// Second key word, fixed, so that a user seed alone selects the stream.
#define SKEMA_KEY1 0x534B454Du
// Counter tags separating the Gauss and SparseSign streams of one seed.
#define SKEMA_TAG_GAUSS 0x47415553u
#define SKEMA_TAG_SSIGN 0x53534731u

// Entry e (column-major linear index i + j*nrow) of a Gauss map: the 53 high
// bits of a 64-bit draw give an integer b in [0, 2^53); the value is
// maxval * (2b - 2^53) * 2^-53. The integer and the power-of-two scaling are
// exact in double, so the only rounding is the final product -- identical on
// every IEEE-754 machine and immune to FMA contraction.
SKEMA_HD double gauss_entry(uint32_t seed, uint64_t e, double maxval) {
  const uint64_t blk = e >> 1;
  const u32x4 r = philox4x32_10((uint32_t)blk, (uint32_t)(blk >> 32),
                                SKEMA_TAG_GAUSS, 0u, seed, SKEMA_KEY1);
  const uint64_t bits = (e & 1) ? (((uint64_t)r.v[2] << 32) | r.v[3])
                                : (((uint64_t)r.v[0] << 32) | r.v[1]);
  const int64_t b = (int64_t)(bits >> 11);
  const int64_t c = 2 * b - ((int64_t)1 << 53);  // in (-2^53, 2^53)
  const double unit = (double)c * 1.1102230246251565404e-16;  // * 2^-53
  return maxval * unit;
}

// Row `row` of a SparseSign map with `ncol` columns and zeta <= 8 entries:
// fills idx[0..zeta) sorted ascending (duplicates kept) and neg[t] = 1 when
// entry t is -1. Index draw: (x * ncol) >> 32 for a 32-bit x (the
// multiply-shift range reduction of Lemire, 2019).
SKEMA_HD void sparse_sign_row(uint32_t seed, uint64_t row, uint32_t ncol,
                              int zeta, uint32_t* idx, uint32_t* neg) {
  const u32x4 a = philox4x32_10((uint32_t)row, (uint32_t)(row >> 32),
                                SKEMA_TAG_SSIGN, 0u, seed, SKEMA_KEY1);
  const u32x4 b = philox4x32_10((uint32_t)row, (uint32_t)(row >> 32),
                                SKEMA_TAG_SSIGN, 1u, seed, SKEMA_KEY1);
  const u32x4 s = philox4x32_10((uint32_t)row, (uint32_t)(row >> 32),
                                SKEMA_TAG_SSIGN, 2u, seed, SKEMA_KEY1);
  uint32_t x[8] = {a.v[0], a.v[1], a.v[2], a.v[3], b.v[0], b.v[1], b.v[2], b.v[3]};
  for (int t = 0; t < zeta; ++t) {
    idx[t] = (uint32_t)(((uint64_t)x[t] * (uint64_t)ncol) >> 32);
  }
  // insertion sort, zeta <= 8
  for (int t = 1; t < zeta; ++t) {
    const uint32_t v = idx[t];
    int u = t - 1;
    while (u >= 0 && idx[u] > v) {
      idx[u + 1] = idx[u];
      --u;
    }
    idx[u + 1] = v;
  }
  for (int t = 0; t < zeta; ++t) neg[t] = (s.v[0] >> t) & 1u;
}

SKEMA_HD int sparse_sign_zeta(int64_t ncol) {
  int64_t z = ncol < 8 ? ncol : 8;
  return (int)(z < 2 ? 2 : z);
}

}  // namespace skema
