/*
 * skema_c.h -- C ABI of the B200 SketchySVD sketch update.
 *
 * This is the drop-in boundary for Skema's streaming SketchySVD path. Every
 * entry point names the reference interface it replaces (paths are relative
 * to the jeremy-myers/skema source tree). The header is plain C: no C++
 * types, no torch types, no exceptions. Every call returns an int status
 * (skema_status); the message of the last failure on a context is returned
 * by skema_last_error().
 *
 * Conventions
 *   - Dense matrices are described by (pointer, leading dimension, layout).
 *     SKEMA_COL_MAJOR is the reference's Kokkos::LayoutLeft
 *     (src/Skema_Utils.hpp:12); SKEMA_ROW_MAJOR is also accepted.
 *   - `mem` says where caller buffers live: SKEMA_MEM_DEVICE (CUDA device
 *     pointers on the context's device) or SKEMA_MEM_HOST (host pointers;
 *     the library stages the data through device memory it owns).
 *   - One context = one CUDA stream. Calls on one context must be serialised
 *     by the caller; separate contexts are independent.
 *   - The context owns the random maps, the sketches X, Y, Z and all
 *     workspaces. Outputs go to caller-provided buffers.
 */
#ifndef SKEMA_C_H
#define SKEMA_C_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* ---- status codes ------------------------------------------------------ */
typedef enum {
  SKEMA_OK = 0,
  SKEMA_EINVAL = 1,       /* bad argument or shape                          */
  SKEMA_ENOMEM = 2,       /* device or host allocation failed               */
  SKEMA_ECUDA = 3,        /* a CUDA runtime call failed                     */
  SKEMA_ENOTPD = 4,       /* Cholesky failed even after the shifted retry   */
  SKEMA_ETIMEOUT = 5,     /* a bounded device-side wait ran out             */
  SKEMA_ESTATE = 6,       /* call not valid in the context's current state  */
  SKEMA_EUNSUPPORTED = 7, /* combination not provided by this build         */
  SKEMA_ENOKERNEL = 8,    /* no CUDA device / kernel image for this device  */
  SKEMA_ECOLLECTIVE = 9   /* the caller's all-reduce callback failed         */
} skema_status;

/* ---- enums mirroring src/Skema_Utils.hpp:38-80 ------------------------- */
enum { SKEMA_MAP_GAUSS = 0, SKEMA_MAP_SPARSE_SIGN = 1 };    /* DimRedux_Map */
enum { SKEMA_KERNEL_NONE = 0, SKEMA_KERNEL_GAUSSRBF = 1 };  /* Kernel_Map   */
/* Arithmetic of the sketch contractions (new; the reference is FP64 only).
 * With Gauss maps on a dense or kernel input, the BF16 and FP8 forms hold the
 * maps on the grid of their arithmetic (every value rounded to BF16, or to
 * E4M3 times a power-of-two scale), at creation and after each map import:
 * the tensor-core products, the FP32 kernels and the FP64 approximation then
 * all use the same maps, and skema_map_export returns those values. */
enum { SKEMA_PREC_FP32 = 0, SKEMA_PREC_BF16 = 1, SKEMA_PREC_FP8 = 2 };
/* Which map, in the order of AlgParams::seeds (src/Skema_SketchySVD.cpp:37,54,70,87). */
enum { SKEMA_UPSILON = 0, SKEMA_OMEGA = 1, SKEMA_PHI = 2, SKEMA_PSI = 3 };
enum { SKEMA_COL_MAJOR = 0, SKEMA_ROW_MAJOR = 1 };
enum { SKEMA_MEM_DEVICE = 0, SKEMA_MEM_HOST = 1 };
/* SketchySPD fixed-rank approximation (src/Skema_SketchySVD.cpp:935-1151):
 * NYSTROM (default) is the stable fixed-rank Nystrom approximation that the
 * reference's comments describe; REFERENCE_STEPS repeats the reference's
 * steps as they run (E from the unshifted Y, eigenvalues less ||Y||_2, and
 * the SparseSign shift multiplying instead of adding), for parity runs. */
enum { SKEMA_SPD_NYSTROM = 0, SKEMA_SPD_REFERENCE_STEPS = 1 };
/* Which sketch, for skema_get_sketch / skema_set_sketch. */
enum { SKEMA_SKETCH_X = 0, SKEMA_SKETCH_Y = 1, SKEMA_SKETCH_Z = 2 };

/*
 * Sketch fields of Skema::AlgParams (src/Skema_AlgParams.hpp:12-90), with the
 * same names and meaning. Defaults come from skema_params_init().
 */
typedef struct {
  int64_t matrix_m;           /* rows of A (points N for a kernel input)      */
  int64_t matrix_n;           /* cols of A (N for a kernel input)             */
  int64_t rank;               /* r                                            */
  int64_t sketch_range;       /* k; 4r+1 when < rank (Skema_SketchySVD.cpp:20) */
  int64_t sketch_core;        /* s; 2k+1 when < rank (Skema_SketchySVD.cpp:23) */
  int64_t window;             /* rows per streaming window                    */
  double sketch_eta;          /* X = nu*X + eta*x  (Skema_SketchySVD.cpp:187) */
  double sketch_nu;
  int32_t seeds[4];           /* Upsilon, Omega, Phi, Psi                     */
  int32_t dim_redux;          /* SKEMA_MAP_*                                  */
  int32_t issparse;           /* input is CSR                                 */
  int32_t issymmetric;        /* with !force_three_sketch: SketchySPD         */
  int32_t force_three_sketch;
  int32_t kernel_func;        /* SKEMA_KERNEL_*                               */
  double kernel_gamma;
  int32_t precision;          /* SKEMA_PREC_* (new)                           */
  int32_t device;             /* CUDA device ordinal                          */
  int32_t spd_approx;         /* SKEMA_SPD_* (new): SketchySPD approximation  */
} skema_params;

typedef struct skema_ctx skema_ctx;

/* Fill p with AlgParams' defaults (src/Skema_AlgParams.cpp:10-57; eta/nu 1.0
 * from src/Skema_AlgParams.cpp:275-278). */
int skema_params_init(skema_params* p);

/* SketchySVD<MatrixType,DimReduxT>::SketchySVD(const AlgParams&)
 * (src/Skema_SketchySVD.cpp:16-117) or SketchySPD::SketchySPD
 * (src/Skema_SketchySVD.cpp:759-788) when issymmetric && !force_three_sketch.
 * Generates the four maps (GaussDimRedux ctor src/Skema_DimRedux.hpp:98-128,
 * SparseSignDimRedux ctor src/Skema_DimRedux.hpp:191-268) on the device with
 * the orientation rules of src/Skema_SketchySVD.cpp:30-95, and allocates
 * zeroed sketches X (k x n), Y (m x k), Z (s x s). */
int skema_create(const skema_params* p, skema_ctx** out);

/* ~SketchySVD(): frees every device buffer the context owns. */
int skema_destroy(skema_ctx* ctx);

/* Message of the last failed call on ctx ("" if none). A NULL ctx returns the
 * message of the last failed skema_create or file call on this thread. */
const char* skema_last_error(const skema_ctx* ctx);

/* Resolved sketch sizes (range k, core s) and whether the context runs the
 * one-sketch SketchySPD variant. */
int skema_get_dims(const skema_ctx* ctx, int64_t* range, int64_t* core, int32_t* spd);

/* Zero X, Y, Z: the start of SketchySVD::linear_update
 * (src/Skema_SketchySVD.cpp:131-133). The zeroing is deferred: the next
 * call on ctx performs it first (a CSR update does it beside its Y kernel),
 * so every later call sees zero sketches. */
int skema_reset(skema_ctx* ctx);

/* SketchySVD<matrix_type,*>::linear_update + update
 * (src/Skema_SketchySVD.cpp:120-246, 256-293) for rows [row0, row0+nrows)
 * of a dense A. The rows are split into windows of params.window rows
 * (last window partial, :167-173); per window the update is
 *   X = nu*X + eta*(Upsilon_w A_w),  Y(w,:) = nu*Y(w,:) + eta*(A_w Omega^T),
 *   Z = nu*Z + eta*(Phi_w A_w Psi^T).
 * A points at row row0 of a block with leading dimension ld. Unlike the
 * reference, the sketches are not re-zeroed here: call skema_reset first to
 * get linear_update's semantics, or stream several row blocks in order. */
int skema_linear_update_dense(skema_ctx* ctx, const float* A, int64_t ld,
                              int32_t layout, int64_t row0, int64_t nrows,
                              int32_t mem);

/* SketchySVD<crs_matrix_type,*>::linear_update + update
 * (src/Skema_SketchySVD.cpp:120-246, 296-335) with the CRS window of
 * Window::get (src/Skema_Window.hpp:50-78). rowptr has nrows+1 entries
 * (absolute offsets into col/val, rowptr[0] need not be 0); col holds int32
 * column indices in [0, matrix_n). Duplicate column entries in a row are
 * summed, as KokkosSparse does. */
int skema_linear_update_csr(skema_ctx* ctx, const int64_t* rowptr,
                            const int32_t* col, const float* val, int64_t row0,
                            int64_t nrows, int32_t mem);

/* GaussRBFWindow::get + GaussRBF::compute (src/Skema_Window.hpp:90-107,
 * src/Skema_Kernel.cpp:6-81) feeding linear_update: rows [row0,row0+nrows)
 * of K(i,j) = exp(-gamma*||x_i - x_j||^2) with K(i,i) = 1, generated on the
 * device one window at a time (the whole K is never formed). pts is npts x d
 * (npts == matrix_m == matrix_n). */
int skema_linear_update_rbf(skema_ctx* ctx, const float* pts, int64_t ld,
                            int32_t layout, int64_t npts, int64_t d,
                            int64_t row0, int64_t nrows, int32_t mem);

/* SketchySVD::low_rank_approx + initial_approx
 * (src/Skema_SketchySVD.cpp:338-664), computed on the device in FP64 with
 * CholeskyQR2 in place of dgeqrf/dorgqr, triangular solves in place of the
 * dgels calls on T1/T2, and a one-sided Jacobi SVD in place of dgesvd.
 * Outputs: U (m x rank), S (rank), V (n x rank), column-major. Singular
 * vectors equal LAPACK's up to sign. Any output pointer may be NULL.
 * SketchySPD contexts: SketchySPD::low_rank_approx
 * (src/Skema_SketchySVD.cpp:935-1151) per params.spd_approx, returning the
 * eigenvectors in U (m x rank) and eigenvalues in S; V is not used. A
 * Cholesky factor that does not exist fails with SKEMA_ENOTPD (the
 * reference exits there). The sketch Y is left unchanged (the reference
 * overwrites it with E). */
int skema_low_rank_approx(skema_ctx* ctx, double* U, double* S, double* V,
                          int32_t mem);

/* In-place sum over all ranks of count doubles at buf (device memory of
 * the context's device; the context's stream has finished writing it and
 * waits for the call to return). Returns 0 on success. Every rank's call
 * sequence is the same, so the callback is a plain all-reduce (NCCL,
 * MPI, ...) on the caller's communicator. */
typedef int (*skema_allreduce_fn)(double* buf, int64_t count, void* user);

/* skema_low_rank_approx for a sketch sharded by contiguous row blocks, one
 * context per rank: this context holds Y's rows [row0, row0 + nrows) and
 * X and Z already summed over the ranks (ν-weighted as the one-process
 * window sequence has them). No counterpart in the reference, which runs
 * on one process; it is SketchySVD::low_rank_approx
 * (src/Skema_SketchySVD.cpp:338-664) with its two reductions over rows
 * made collective: the k x k Gram matrices of both CholeskyQR passes of Y
 * and the s x k product Phi~ Q are summed with `allreduce` (three calls,
 * each rank in the same order); everything else is the same k-sized
 * arithmetic on every rank. U receives the block's rows of U (nrows x
 * rank, column-major, ld nrows); S and V (n x rank) are those of the whole
 * matrix, the same on every rank up to FP64 summation order. A sketch of
 * rank below the range fails with SKEMA_ENOTPD on every rank (the
 * single-context call falls back to an eigen-decomposition that needs all
 * of Y in one place). */
int skema_low_rank_approx_rows(skema_ctx* ctx, int64_t row0, int64_t nrows, skema_allreduce_fn allreduce,
                               void* user, double* U, double* S, double* V, int32_t mem);

/* Residual norms of a fixed-rank approximation: SketchySVD::compute_residuals
 * (src/Skema_SketchySVD.cpp:719-727) with Skema::residuals and
 * map_A_by_window (src/Skema_Residuals.hpp:58-110, 160-217):
 *   rnorm_j = || [ (A^T U - V S)(:, j) ; (A V - U S)(:, j) ] ||_2,  j < rank.
 * A is streamed a second time, in the same forms as the sketch update:
 *   skema_residuals_begin(ctx, U, S, V, mem)   U (m x rank), S (rank),
 *       V (n x rank), column-major, as returned by skema_low_rank_approx
 *   skema_residuals_update_dense / _csr / _rbf(...)   arguments exactly as
 *       skema_linear_update_dense / _csr / _rbf; rows in any order, each row
 *       once; the sketches are not touched
 *   skema_residuals_finish(ctx, rnorms, mem)   rank doubles; closes the pass.
 * SketchySPD contexts take the one-sided form ||(A V - V S)(:, j)||_2
 * (src/Skema_Residuals.hpp:112-158); U may then be NULL. FP64 arithmetic.
 * An update or finish without an open pass fails with SKEMA_ESTATE.
 * U, S and V all NULL open the pass on the factors of the last
 * skema_low_rank_approx, kept on the device (skema_set_keep_factors), as
 * the reference's compute_residuals uses the uvecs, svals and vvecs its
 * low_rank_approx kept (src/Skema_SketchySVD.cpp:656-660, 719-727); without
 * kept factors that fails with SKEMA_ESTATE. Factors passed explicitly
 * replace the kept ones. */
/* on = 1: every later skema_low_rank_approx (any mem) also keeps its U, S
 * and V on the device, in buffers the context holds ((m + 2 n) rank + 2
 * rank doubles, allocated by the first one), for a residual pass opened with
 * NULL factors: no host copy of U is made. on = 0 stops keeping and drops
 * the kept factors. Off by default. */
int skema_set_keep_factors(skema_ctx* ctx, int32_t on);

int skema_residuals_begin(skema_ctx* ctx, const double* U, const double* S,
                          const double* V, int32_t mem);
int skema_residuals_update_dense(skema_ctx* ctx, const float* A, int64_t ld,
                                 int32_t layout, int64_t row0, int64_t nrows,
                                 int32_t mem);
int skema_residuals_update_csr(skema_ctx* ctx, const int64_t* rowptr,
                               const int32_t* col, const float* val,
                               int64_t row0, int64_t nrows, int32_t mem);
int skema_residuals_update_rbf(skema_ctx* ctx, const float* pts, int64_t ld,
                               int32_t layout, int64_t npts, int64_t d,
                               int64_t row0, int64_t nrows, int32_t mem);
int skema_residuals_finish(skema_ctx* ctx, double* rnorms, int32_t mem);

/* Copy one sketch out of / into the context (the reference only exposes them
 * through its debug dumps, src/Skema_SketchySVD.cpp:192-206, 235-245).
 * X is k x n, Y is m x k, Z is s x s; `layout` is the layout of buf. */
int skema_get_sketch(skema_ctx* ctx, int32_t which, float* buf, int64_t ld,
                     int32_t layout, int32_t mem);
int skema_set_sketch(skema_ctx* ctx, int32_t which, const float* buf,
                     int64_t ld, int32_t layout, int32_t mem);

/* Map dump/import (the --debug-file dumps of src/Skema_DimRedux.hpp:124-127,
 * 264-267). The map is described in its stored orientation (nrow x ncol of
 * the DimRedux ctor). Gauss: values as double, column-major nrow x ncol.
 * SparseSign: zeta entries per stored row, indices int32 and values double
 * (+-1), row r at [r*zeta, (r+1)*zeta). Query shapes with buffers NULL. */
int skema_map_info(const skema_ctx* ctx, int32_t which, int64_t* nrow,
                   int64_t* ncol, int32_t* zeta, int32_t* transposed);
int skema_map_export(skema_ctx* ctx, int32_t which, double* values,
                     int32_t* indices);
int skema_map_import(skema_ctx* ctx, int32_t which, const double* values,
                     const int32_t* indices);

/* Standalone RBF-kernel sketch (new; no reference counterpart beyond
 * GaussRBF::compute, src/Skema_Kernel.cpp:6-81):
 *   Y = K Omega^T,  K(i,j) = exp(-gamma*||x_i - x_j||^2), K(i,i) = 1,
 * with pts N x d (row-major), Omega k x N (row-major), Y N x k (row-major),
 * all device pointers, on ctx's stream. */
int skema_rbf_sketch_fwd(skema_ctx* ctx, const float* pts, int64_t npts,
                         int64_t d, double gamma, const float* omega,
                         int64_t k, float* Y);

/* Vector-Jacobian product of skema_rbf_sketch_fwd: given Ybar = dL/dY
 * (N x k, row-major), returns dL/dpts (N x d, row-major, overwritten) and
 * dL/dgamma (one double, device pointer). Kernel tiles are recomputed, never
 * stored. */
int skema_rbf_sketch_vjp(skema_ctx* ctx, const float* pts, int64_t npts,
                         int64_t d, double gamma, const float* omega,
                         int64_t k, const float* Ybar, float* dpts,
                         double* dgamma);

/* Allocation-free form of skema_rbf_sketch_fwd (no counterpart in the
 * reference): same arguments, for callers that must not have a library
 * allocate device memory -- a host framework that owns all device
 * memory through its own pool or memory cap, or a latency-critical loop in
 * which cudaMalloc's implicit device-wide synchronisation would stall other
 * streams. Instead of the context workspace it uses one static 16 MiB
 * scratch array compiled into the library (every GPU that loads the library
 * holds it until the process exits), in kernel row blocks of
 * floor(4194304 / npts) rows, and calls no cudaMalloc or cudaFree. It
 * always computes in FP32 (kernel rows by explicit differences, then an FP32
 * product), whatever the context's precision: its result is what
 * skema_rbf_sketch_fwd returns in an FP32 context, while in a BF16 context
 * skema_rbf_sketch_fwd takes the tensor-core form (d <= 64, k <= 192), whose
 * result differs from the FP32 one by the BF16 rounding (about 3e-3).
 * Limit: npts <= 4194304, else SKEMA_EINVAL. The first call on a device
 * looks up the array's device address (cudaGetSymbolAddress); make that
 * first call before any stream capture. All calls share the array: calls
 * that overlap on the GPU race and must be serialised by the caller. */
int skema_rbf_sketch_fwd_noalloc(skema_ctx* ctx, const float* pts,
                                 int64_t npts, int64_t d, double gamma,
                                 const float* omega, int64_t k, float* Y);

/* ---- standalone maps: GaussDimRedux / SparseSignDimRedux ---------------- */
/* A random map with its lmap / rmap products (src/Skema_DimRedux.hpp:60-268).
 * The map is generated on the device exactly as a context's map of the same
 * kind, stored shape nrow x ncol and seed, so a caller can apply the sketch
 * operators by hand. The products take FP32 operands and accumulate in FP32
 * (the FP32 SIMT GEMM); a SparseSign map is expanded once into a dense FP32
 * copy (duplicate entries summed) for them. The products are stated
 * without the reference's conventions -- the C++ layer in skema.hpp maps the
 * reference's calls (its init_transposed swap, its transposed CRS results)
 * onto them:
 *   lmap:  C = alpha op(M(:, idx)) op(B) + beta C   idx = stored columns
 *   rmap:  C = alpha op(A) op(M(idx, :)) + beta C   idx = stored rows
 * op(X) = X for 'N', X^T for 'T'; idx = [idx_first, idx_second), the whole
 * map when idx_first == idx_second. `mem` says where A / B and C live; every
 * descriptor's pointer follows it. */
typedef struct skema_dimredux skema_dimredux;
typedef struct {
  float* p;        /* element (0, 0)                                       */
  int64_t rows, cols, ld;
  int32_t layout;  /* SKEMA_COL_MAJOR or SKEMA_ROW_MAJOR                    */
} skema_matf;
typedef struct {
  const int64_t* rowptr; /* rows + 1 absolute offsets into col / val        */
  const int32_t* col;    /* column indices in [0, cols) (others skipped)    */
  const float* val;
  int64_t rows, cols;
} skema_csrf;
/* GaussDimRedux / SparseSignDimRedux ctor (src/Skema_DimRedux.hpp:98-128,
 * 191-268): kind SKEMA_MAP_*, stored shape nrow x ncol, seed. */
int skema_dimredux_create(int32_t kind, int64_t nrow, int64_t ncol,
                          int32_t seed, int32_t device, skema_dimredux** out);
int skema_dimredux_destroy(skema_dimredux* map);
/* Message of the last failed call on map ("" if none). */
const char* skema_dimredux_last_error(const skema_dimredux* map);
/* The map's values, as skema_map_export gives a context's map. */
int skema_dimredux_export(skema_dimredux* map, double* values,
                          int32_t* indices);
/* DimRedux::lmap / rmap on a dense operand
 * (src/Skema_DimRedux_Gauss.cpp:10-52, src/Skema_DimRedux_SparseSign.cpp:9-51). */
int skema_dimredux_lmap(skema_dimredux* map, double alpha, const skema_matf* B,
                        double beta, char transA, char transB,
                        int64_t idx_first, int64_t idx_second, skema_matf* C,
                        int32_t mem);
int skema_dimredux_rmap(skema_dimredux* map, double alpha, const skema_matf* A,
                        double beta, char transA, char transB,
                        int64_t idx_first, int64_t idx_second, skema_matf* C,
                        int32_t mem);
/* DimRedux::lmap / rmap on a CRS operand
 * (src/Skema_DimRedux_Gauss.cpp:54-99, src/Skema_DimRedux_SparseSign.cpp:53-111):
 * B (lmap) or A (rmap) is the CSR matrix; C is dense. */
int skema_dimredux_lmap_csr(skema_dimredux* map, double alpha,
                            const skema_csrf* B, double beta, char transA,
                            char transB, int64_t idx_first, int64_t idx_second,
                            skema_matf* C, int32_t mem);
int skema_dimredux_rmap_csr(skema_dimredux* map, double alpha,
                            const skema_csrf* A, double beta, char transA,
                            char transB, int64_t idx_first, int64_t idx_second,
                            skema_matf* C, int32_t mem);

/* ---- matrix files ----------------------------------------------------- */
/* Skema::read_matrix / write_matrix (src/Skema_IO.hpp:10-40,
 * src/Skema_IO.cpp:8-104), chosen by the file extension. Arrays returned by
 * the readers are allocated with malloc and released by the *_free calls.
 *   .mtx dense: MatrixMarket "matrix array" (column-major values);
 *   .mtx CRS:   MatrixMarket "matrix coordinate" (1-based; symmetric and
 *               skew-symmetric files expanded; pattern entries 1), as
 *               KokkosKernels' read_kokkos_crst_matrix reads it;
 *   .bin CRS:   int32 nrows, int64 nnz, uint64 row_map[nrows+1],
 *               int32 entries[nnz], float64 values[nnz]; ncol = nrows
 *               unless a column index is larger. A dense .bin is rejected
 *               (SKEMA_EUNSUPPORTED), as in the reference.
 * CRS rows come back sorted by column with duplicate entries summed. Errors
 * are reported by skema_last_error(NULL). The values are FP64, as the
 * reference reads them; the update entry points take FP32. */
typedef struct {
  int64_t nrow, ncol, nnz;
  int64_t* rowptr; /* nrow + 1 entries, rowptr[0] = 0 */
  int32_t* col;
  double* val;
} skema_crs;
typedef struct {
  int64_t nrow, ncol;
  double* data; /* column-major, nrow * ncol */
} skema_dense;
int skema_read_crs(const char* path, skema_crs* out);
void skema_crs_free(skema_crs* a);
int skema_read_dense(const char* path, skema_dense* out);
void skema_dense_free(skema_dense* a);
/* write_mtx / write_bin for CRS (src/Skema_IO.cpp:88-104): a .mtx file is
 * written as "coordinate real general" with 17 significant digits. */
int skema_write_crs(const char* path, const skema_crs* a);

/* Rows [row0, row0 + nrows) of a binary CRS file (.bin layout above; nrows
 * < 0: to the last row), read from their offsets without loading the rest:
 * the header and row map, then the block's entries and values. No
 * counterpart in the reference, whose read_matrix (src/Skema_IO.cpp:53-74)
 * reads the whole file; it lets each rank of a row-block sharding read
 * only its own block. out->rowptr[0] = 0; the entries of a row keep their
 * file order (not sorted, duplicates not summed: the sketch update takes
 * them as they are); out->ncol is the file's row count, or the block's
 * largest column + 1 when that is larger. Free with skema_crs_free. */
int skema_read_crs_rows(const char* path, int64_t row0, int64_t nrows, skema_crs* out);

/* Rows [row0, row0 + nrows) of a matrix file (nrows < 0: to the last row)
 * streamed into the sketches: skema_linear_update_csr / _dense over those
 * rows of A, as the reference's driver does after read_matrix
 * (driver/main.cpp:79-150, src/Skema_IO.cpp:8-74). A binary CRS file is read one
 * window of rows at a time (the context's window): the next window is read
 * and converted to FP32 on the host, into one of two pinned buffers, while
 * the device copies and sketches the previous one. A MatrixMarket file is
 * read whole first (its entries are in no row order), then streamed.
 * Kernel (Gauss-RBF) contexts take their points, not a file. */
int skema_update_from_file(skema_ctx* ctx, const char* path, int64_t row0, int64_t nrows);

/* Wait for all work queued on ctx's stream. */
int skema_synchronize(skema_ctx* ctx);

/* Use an external CUDA stream (cudaStream_t passed as void*; NULL restores
 * the context's own stream). */
int skema_set_stream(skema_ctx* ctx, void* stream);

/* Limit of every bounded device-side wait of the tensor-core kernels, in
 * nanoseconds (ns <= 0 restores the default of 2 s). A kernel whose wait runs
 * out sets the context's status word, lets the copies and tensor-core
 * operations it has in flight land for 20 ms, frees its tensor memory and
 * returns; the next synchronising call on ctx then fails with
 * SKEMA_ETIMEOUT and clears the word, and the sketches are invalid until the
 * next skema_reset. No reference counterpart: the reference has no device
 * waits. Synchronises ctx's stream. */
int skema_set_wait_limit(skema_ctx* ctx, int64_t ns);

/* Cap, in bytes, on the device workspace and staging buffers ctx may hold
 * (0: no cap, the default). A call that would grow them beyond the cap
 * fails with SKEMA_ENOMEM before allocating; buffers already held are kept.
 * The maps and sketches allocated by skema_create are not counted. No
 * reference counterpart. */
int skema_set_workspace_limit(skema_ctx* ctx, int64_t bytes);

/* The CUDA stream ctx launches on (cudaStream_t as void*): its own stream,
 * or the one given to skema_set_stream. A caller that hands the library
 * memory managed by a stream-ordered allocator records its use on this
 * stream. */
int skema_get_stream(const skema_ctx* ctx, void** stream);

/* Number of this library's kernels launched on ctx so far (for accounting). */
int64_t skema_launch_count(const skema_ctx* ctx);

/* Device-side stage timers, the counterpart of the reference's
 * timings["update"][...] / timings["approx"][...] maps
 * (src/Skema_SketchySVD.cpp:101-116), measured with CUDA events on the
 * context's stream. skema_timing_enable(ctx, 1) clears and starts them;
 * skema_timing_get synchronises and returns the accumulated milliseconds and
 * number of timed launches of one stage:
 *   "update.omega"   Y = A Omega^T (the streaming Y kernel of the sparse path)
 *   "update.psi"     T = A Psi^T
 *   "update.upsilon" X += Upsilon_w A_w
 *   "update.phi"     Z += Phi_w T
 *   "update.entries" the sparse-sign X/Z entry kernel
 *   "update.window"  kernel-window generation
 *   "update.fused"   the fused tensor-core window kernel
 *   "update.daxpy"   sketch scaling by nu
 *   "approx.orth"    orthonormal bases of Y and X^T (skema_low_rank_approx)
 *   "approx.core"    the core matrix: Phi Q, Psi P, their QR and the solves
 *   "approx.svd"     the core matrix's SVD
 *   "approx.vectors" U = Q Uc and V = P Vc
 * "approx.svd_sweeps" gives 0 ms and, as the count, the sweeps of the last
 * core-matrix SVD (one-sided Jacobi). Unknown names give SKEMA_EINVAL. */
int skema_timing_enable(skema_ctx* ctx, int32_t on);
int skema_timing_get(skema_ctx* ctx, const char* stage, double* ms, int64_t* count);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* SKEMA_C_H */
