// stream_io.cu -- matrix files read by row blocks and streamed into the
// sketch update.
//
// Skema::read_matrix (src/Skema_IO.hpp:13-21, src/Skema_IO.cpp:8-74) loads a
// whole file before the driver sketches it. The binary CRS layout
// (int32 nrows, int64 nnz, uint64 row_map[nrows + 1], int32 entries[nnz],
// float64 values[nnz]) places every row's entries at offsets the row map
// gives, so a block of rows can be read on its own: the header and row map
// first, then two positioned reads for the block's entries and values.
// skema_read_crs_rows returns such a block; skema_update_from_file streams a
// file's rows into a context one window at a time, reading and converting
// the next window on the host while the device copies and sketches the
// previous one. MatrixMarket files list entries in any order (coordinate)
// or by columns (array), so they are read whole and then streamed.
#include <cuda_runtime.h>
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cctype>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "internal.h"

namespace skema {

void set_thread_error(const std::string& msg);

namespace {

// The header and row map of a binary CRS file, and positioned reads of a
// row block's entries.
class BinCrsFile {
 public:
  explicit BinCrsFile(const char* path) {
    if (!path) fail(SKEMA_EINVAL, "null path");
    fd_ = ::open(path, O_RDONLY);
    if (fd_ < 0) fail(SKEMA_EINVAL, std::string("cannot open ") + path);
    struct stat sb;
    if (::fstat(fd_, &sb) != 0) fail(SKEMA_EINVAL, std::string("cannot stat ") + path);
    int32_t nr32 = 0;
    read_at(&nr32, 4, 0);
    read_at(&nnz_, 8, 4);
    if (nr32 < 0 || nnz_ < 0) fail(SKEMA_EINVAL, "bad binary CRS header");
    nrows_ = nr32;
    rm_.resize((size_t)nrows_ + 1);
    read_at(rm_.data(), sizeof(uint64_t) * rm_.size(), 12);
    col_off_ = 12 + (off_t)sizeof(uint64_t) * (off_t)(nrows_ + 1);
    val_off_ = col_off_ + (off_t)sizeof(int32_t) * (off_t)nnz_;
    if ((int64_t)sb.st_size != (int64_t)val_off_ + (int64_t)sizeof(double) * nnz_)
      fail(SKEMA_EINVAL, "binary CRS file size does not match its header");
    if (rm_[0] != 0 || (int64_t)rm_[nrows_] != nnz_)
      fail(SKEMA_EINVAL, "binary CRS row map does not span the entries");
    for (int64_t r = 0; r < nrows_; ++r)
      if (rm_[r + 1] < rm_[r]) fail(SKEMA_EINVAL, "binary CRS row map decreases");
  }
  ~BinCrsFile() {
    if (fd_ >= 0) ::close(fd_);
  }
  BinCrsFile(const BinCrsFile&) = delete;
  BinCrsFile& operator=(const BinCrsFile&) = delete;

  int64_t nrows() const { return nrows_; }
  int64_t first(int64_t r) const { return (int64_t)rm_[r]; }
  // Entries of rows [r0, r1): columns into col, values (FP64) into val.
  void read_block(int64_t r0, int64_t r1, int32_t* col, double* val) const {
    const int64_t a = first(r0), n = first(r1) - a;
    if (n <= 0) return;
    read_at(col, sizeof(int32_t) * (size_t)n, col_off_ + (off_t)sizeof(int32_t) * (off_t)a);
    read_at(val, sizeof(double) * (size_t)n, val_off_ + (off_t)sizeof(double) * (off_t)a);
  }

 private:
  void read_at(void* dst, size_t n, off_t off) const {
    char* p = static_cast<char*>(dst);
    while (n > 0) {
      const ssize_t got = ::pread(fd_, p, n, off);
      if (got <= 0) fail(SKEMA_EINVAL, "binary CRS file ends early");
      p += got, n -= (size_t)got, off += got;
    }
  }
  int fd_ = -1;
  int64_t nrows_ = 0, nnz_ = 0;
  std::vector<uint64_t> rm_;
  off_t col_off_ = 0, val_off_ = 0;
};

bool has_suffix(const char* path, const char* suf) {
  const size_t a = std::strlen(path), b = std::strlen(suf);
  if (a < b) return false;
  for (size_t i = 0; i < b; ++i)
    if (std::tolower((unsigned char)path[a - b + i]) != suf[i]) return false;
  return true;
}

// Two pinned host buffers for one window each (row pointers from 0, int32
// columns, FP32 values) and the events that say when the device has
// finished with them.
struct PinnedWindows {
  int64_t rows_cap = 0, nnz_cap = 0;
  int64_t* rp[2] = {nullptr, nullptr};
  int32_t* col[2] = {nullptr, nullptr};
  float* val[2] = {nullptr, nullptr};
  cudaEvent_t done[2] = {nullptr, nullptr};
  bool used[2] = {false, false};
  PinnedWindows(int64_t rows, int64_t nnz) : rows_cap(rows), nnz_cap(std::max<int64_t>(nnz, 1)) {
    for (int b = 0; b < 2; ++b) {
      SKEMA_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&rp[b]), sizeof(int64_t) * (size_t)(rows + 1),
                               cudaHostAllocDefault));
      SKEMA_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&col[b]), sizeof(int32_t) * (size_t)nnz_cap,
                               cudaHostAllocDefault));
      SKEMA_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&val[b]), sizeof(float) * (size_t)nnz_cap,
                               cudaHostAllocDefault));
      SKEMA_CUDA(cudaEventCreateWithFlags(&done[b], cudaEventDisableTiming));
    }
  }
  ~PinnedWindows() {
    for (int b = 0; b < 2; ++b) {
      if (done[b]) {
        cudaEventSynchronize(done[b]);
        cudaEventDestroy(done[b]);
      }
      if (rp[b]) cudaFreeHost(rp[b]);
      if (col[b]) cudaFreeHost(col[b]);
      if (val[b]) cudaFreeHost(val[b]);
    }
  }
  PinnedWindows(const PinnedWindows&) = delete;
  PinnedWindows& operator=(const PinnedWindows&) = delete;
};

// Rows [row0, row0 + nrows) of a binary CRS file through the context's
// update, one window at a time.
void stream_bin(skema_ctx* c, const char* path, int64_t row0, int64_t nrows) {
  const BinCrsFile f(path);
  if (nrows < 0) nrows = f.nrows() - row0;
  if (row0 < 0 || nrows < 0 || row0 + nrows > f.nrows()) fail(SKEMA_EINVAL, "row range outside the file");
  if (row0 + nrows > c->m) fail(SKEMA_EINVAL, "the file has more rows than the sketched matrix");
  if (nrows == 0) return;
  const int64_t W = std::max<int64_t>(1, std::min(c->w, nrows));
  int64_t nnz_max = 0;
  for (int64_t r = row0; r < row0 + nrows; r += W)
    nnz_max = std::max(nnz_max, f.first(std::min(row0 + nrows, r + W)) - f.first(r));
  PinnedWindows pw(W, nnz_max);
  std::vector<double> v64((size_t)std::max<int64_t>(nnz_max, 1));
  int b = 0;
  for (int64_t r = row0; r < row0 + nrows; r += W, b ^= 1) {
    const int64_t r1 = std::min(row0 + nrows, r + W), wr = r1 - r;
    // the device has finished with this buffer's previous window
    if (pw.used[b]) SKEMA_CUDA(cudaEventSynchronize(pw.done[b]));
    const int64_t a = f.first(r), nnz = f.first(r1) - a;
    for (int64_t i = 0; i <= wr; ++i) pw.rp[b][i] = f.first(r + i) - a;
    f.read_block(r, r1, pw.col[b], v64.data());
    for (int64_t q = 0; q < nnz; ++q) {
      if (pw.col[b][q] < 0 || pw.col[b][q] >= c->n) fail(SKEMA_EINVAL, "a column of the file lies outside A");
      pw.val[b][q] = (float)v64[(size_t)q];
    }
    const int st = skema_linear_update_csr(c, pw.rp[b], pw.col[b], pw.val[b], r, wr, SKEMA_MEM_HOST);
    if (st != SKEMA_OK) throw Error{st, c->err};
    SKEMA_CUDA(cudaEventRecord(pw.done[b], c->stream));
    pw.used[b] = true;
  }
}

// A MatrixMarket file read whole, then its rows [row0, row0 + nrows)
// through the update of the context's input kind.
void stream_mtx(skema_ctx* c, const char* path, int64_t row0, int64_t nrows) {
  auto check_rows = [&](int64_t total) {
    if (nrows < 0) nrows = total - row0;
    if (row0 < 0 || nrows < 0 || row0 + nrows > total) fail(SKEMA_EINVAL, "row range outside the file");
  };
  if (c->p.issparse) {
    skema_crs a{};
    int st = skema_read_crs(path, &a);
    if (st != SKEMA_OK) {
      const char* m = skema_last_error(nullptr);
      throw Error{st, m ? m : "reading the file failed"};
    }
    struct Free {
      skema_crs* a;
      ~Free() { skema_crs_free(a); }
    } fr{&a};
    check_rows(a.nrow);
    if (a.ncol > c->n) fail(SKEMA_EINVAL, "the file has more columns than the sketched matrix");
    std::vector<float> v32((size_t)std::max<int64_t>(a.nnz, 1));
    for (int64_t q = 0; q < a.nnz; ++q) v32[(size_t)q] = (float)a.val[q];
    st = skema_linear_update_csr(c, a.rowptr + row0, a.col, v32.data(), row0, nrows, SKEMA_MEM_HOST);
    if (st != SKEMA_OK) throw Error{st, c->err};
    SKEMA_CUDA(cudaStreamSynchronize(c->stream));  // v32 is pageable, but keep the order plain
    return;
  }
  if (c->p.kernel_func != SKEMA_KERNEL_NONE) fail(SKEMA_EINVAL, "a kernel context takes its points, not a matrix file");
  skema_dense d{};
  int st = skema_read_dense(path, &d);
  if (st != SKEMA_OK) {
    const char* m = skema_last_error(nullptr);
    throw Error{st, m ? m : "reading the file failed"};
  }
  struct Free {
    skema_dense* d;
    ~Free() { skema_dense_free(d); }
  } fr{&d};
  check_rows(d.nrow);
  if (d.ncol != c->n) fail(SKEMA_EINVAL, "the file's column count differs from the sketched matrix");
  // rows [row0, row0 + nrows) as FP32, column-major with ld = nrows
  std::vector<float> a32((size_t)std::max<int64_t>(nrows * d.ncol, 1));
  for (int64_t j = 0; j < d.ncol; ++j)
    for (int64_t i = 0; i < nrows; ++i) a32[(size_t)(i + j * nrows)] = (float)d.data[(row0 + i) + j * d.nrow];
  st = skema_linear_update_dense(c, a32.data(), std::max<int64_t>(nrows, 1), SKEMA_COL_MAJOR, row0, nrows,
                                 SKEMA_MEM_HOST);
  if (st != SKEMA_OK) throw Error{st, c->err};
  SKEMA_CUDA(cudaStreamSynchronize(c->stream));
}

}  // namespace
}  // namespace skema

using skema::Error;

extern "C" {

int skema_read_crs_rows(const char* path, int64_t row0, int64_t nrows, skema_crs* out) {
  if (!out) return SKEMA_EINVAL;
  *out = skema_crs{};
  try {
    const skema::BinCrsFile f(path);
    if (nrows < 0) nrows = f.nrows() - row0;
    if (row0 < 0 || nrows < 0 || row0 + nrows > f.nrows())
      skema::fail(SKEMA_EINVAL, "row range outside the file");
    const int64_t a = f.first(row0), nnz = f.first(row0 + nrows) - a;
    skema_crs r{};
    r.nrow = nrows;
    r.nnz = nnz;
    r.rowptr = static_cast<int64_t*>(std::malloc(sizeof(int64_t) * (size_t)(nrows + 1)));
    r.col = static_cast<int32_t*>(std::malloc(sizeof(int32_t) * (size_t)std::max<int64_t>(nnz, 1)));
    r.val = static_cast<double*>(std::malloc(sizeof(double) * (size_t)std::max<int64_t>(nnz, 1)));
    if (!r.rowptr || !r.col || !r.val) {
      skema_crs_free(&r);
      skema::fail(SKEMA_ENOMEM, "host allocation failed");
    }
    for (int64_t i = 0; i <= nrows; ++i) r.rowptr[i] = f.first(row0 + i) - a;
    try {
      f.read_block(row0, row0 + nrows, r.col, r.val);
    } catch (...) {
      skema_crs_free(&r);
      throw;
    }
    int64_t cmax = -1;
    for (int64_t q = 0; q < nnz; ++q) {
      if (r.col[q] < 0) {
        skema_crs_free(&r);
        skema::fail(SKEMA_EINVAL, "negative column in a binary CRS file");
      }
      cmax = std::max<int64_t>(cmax, r.col[q]);
    }
    r.ncol = std::max<int64_t>(f.nrows(), cmax + 1);
    *out = r;
    skema::set_thread_error("");
    return SKEMA_OK;
  } catch (const Error& e) {
    skema::set_thread_error(e.msg);
    return e.status;
  } catch (const std::bad_alloc&) {
    skema::set_thread_error("host allocation failed");
    return SKEMA_ENOMEM;
  }
}

int skema_update_from_file(skema_ctx* c, const char* path, int64_t row0, int64_t nrows) {
  if (!c) return SKEMA_EINVAL;
  try {
    if (!path) skema::fail(SKEMA_EINVAL, "null path");
    SKEMA_CUDA(cudaSetDevice(c->dev));
    if (skema::has_suffix(path, ".bin")) {
      if (!c->p.issparse) skema::fail(SKEMA_EUNSUPPORTED, "a binary file holds a CRS matrix; the context is dense");
      skema::stream_bin(c, path, row0, nrows);
    } else if (skema::has_suffix(path, ".mtx")) {
      skema::stream_mtx(c, path, row0, nrows);
    } else {
      skema::fail(SKEMA_EINVAL, "unknown matrix file extension (.mtx or .bin)");
    }
    c->err.clear();
    return SKEMA_OK;
  } catch (const Error& e) {
    c->err = e.msg;
    return e.status;
  } catch (const std::bad_alloc&) {
    c->err = "host allocation failed";
    return SKEMA_ENOMEM;
  }
}

}  // extern "C"
