// io.cu -- matrix files for the sketch inputs (Skema::read_matrix /
// write_matrix, src/Skema_IO.hpp:10-40, src/Skema_IO.cpp:8-104):
//   .mtx, dense:  MatrixMarket "matrix array", column-major values
//                 (read_mtx<matrix_type>, src/Skema_IO.cpp:8-51);
//   .mtx, CRS:    MatrixMarket "matrix coordinate", read as KokkosKernels'
//                 read_kokkos_crst_matrix does (src/Skema_IO.cpp:60-64):
//                 1-based indices, "symmetric" files expanded with the
//                 mirrored off-diagonal entries ("skew-symmetric" with their
//                 negatives), "pattern" entries valued 1;
//   .bin, CRS:    int32 nrows, int64 nnz, uint64 row_map[nrows+1],
//                 int32 entries[nnz], float64 values[nnz] (the layout of the
//                 reference's test/data/symmetric_sparse.bin);
//   .bin, dense:  rejected, as the reference does (src/Skema_IO.cpp:53-58).
// Rows of a CRS result are sorted by column and duplicate entries are
// summed, which is how the sketch update treats them. Host code only.
#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "internal.h"

namespace skema {

void set_thread_error(const std::string& msg);

namespace {

struct IoError {
  int code;
  std::string msg;
};
[[noreturn]] void io_fail(int code, const std::string& m) { throw IoError{code, m}; }

std::string read_file(const char* path) {
  FILE* f = std::fopen(path, "rb");
  if (!f) io_fail(SKEMA_EINVAL, std::string("cannot open ") + path + ": " + std::strerror(errno));
  std::string s;
  char buf[1 << 16];
  size_t got;
  while ((got = std::fread(buf, 1, sizeof(buf), f)) > 0) s.append(buf, got);
  std::fclose(f);
  return s;
}

bool ends_with(const std::string& s, const char* suf) {
  const size_t n = std::strlen(suf);
  return s.size() >= n && s.compare(s.size() - n, n, suf) == 0;
}

std::string lower(std::string s) {
  for (char& ch : s) ch = (char)std::tolower((unsigned char)ch);
  return s;
}

// Line cursor over a text buffer.
struct Lines {
  const std::string& s;
  size_t pos = 0;
  explicit Lines(const std::string& t) : s(t) {}
  bool next(std::string& line) {
    if (pos >= s.size()) return false;
    size_t e = s.find('\n', pos);
    if (e == std::string::npos) e = s.size();
    line.assign(s, pos, e - pos);
    if (!line.empty() && line.back() == '\r') line.pop_back();
    pos = e + 1;
    return true;
  }
};

// The MatrixMarket banner and size line; returns the banner in lower case.
std::string mm_header(Lines& L, std::string& sizeline) {
  std::string banner;
  if (!L.next(banner) || banner.size() < 2 || banner[0] != '%' || banner[1] != '%')
    io_fail(SKEMA_EINVAL, "not a MatrixMarket file (first line)");
  banner = lower(banner);
  if (banner.find("matrix") == std::string::npos) io_fail(SKEMA_EINVAL, "only MatrixMarket \"matrix\" objects are read");
  while (L.next(sizeline)) {
    size_t i = sizeline.find_first_not_of(" \t");
    if (i == std::string::npos || sizeline[i] == '%') continue;
    return banner;
  }
  io_fail(SKEMA_EINVAL, "MatrixMarket file without a size line");
}

struct Crs {
  int64_t nrow = 0, ncol = 0;
  std::vector<int64_t> rowptr;
  std::vector<int32_t> col;
  std::vector<double> val;
};

// Triplets -> CRS with rows sorted by column and duplicates summed.
Crs to_crs(int64_t nr, int64_t nc, std::vector<int64_t>& ri, std::vector<int32_t>& ci, std::vector<double>& vi) {
  const size_t ne = ri.size();
  std::vector<int64_t> cnt(nr + 1, 0);
  for (size_t e = 0; e < ne; ++e) ++cnt[ri[e] + 1];
  for (int64_t r = 0; r < nr; ++r) cnt[r + 1] += cnt[r];
  std::vector<int32_t> c1(ne);
  std::vector<double> v1(ne);
  std::vector<int64_t> fill(cnt.begin(), cnt.end() - 1);
  for (size_t e = 0; e < ne; ++e) {
    const int64_t p = fill[ri[e]]++;
    c1[p] = ci[e];
    v1[p] = vi[e];
  }
  Crs A;
  A.nrow = nr, A.ncol = nc;
  A.rowptr.assign(nr + 1, 0);
  A.col.reserve(ne);
  A.val.reserve(ne);
  std::vector<std::pair<int32_t, double>> row;
  for (int64_t r = 0; r < nr; ++r) {
    row.clear();
    for (int64_t p = cnt[r]; p < cnt[r + 1]; ++p) row.emplace_back(c1[p], v1[p]);
    std::stable_sort(row.begin(), row.end(),
                     [](const std::pair<int32_t, double>& a, const std::pair<int32_t, double>& b) {
                       return a.first < b.first;
                     });
    for (size_t q = 0; q < row.size(); ++q) {
      if (q > 0 && row[q].first == A.col.back()) {
        A.val.back() += row[q].second;
      } else {
        A.col.push_back(row[q].first);
        A.val.push_back(row[q].second);
      }
    }
    A.rowptr[r + 1] = (int64_t)A.col.size();
  }
  return A;
}

Crs read_mtx_coordinate(const std::string& text) {
  Lines L(text);
  std::string sz;
  const std::string banner = mm_header(L, sz);
  if (banner.find("coordinate") == std::string::npos)
    io_fail(SKEMA_EINVAL, "a CRS input needs a MatrixMarket \"coordinate\" file");
  if (banner.find("complex") != std::string::npos) io_fail(SKEMA_EUNSUPPORTED, "complex MatrixMarket values");
  const bool pattern = banner.find("pattern") != std::string::npos;
  const bool skew = banner.find("skew-symmetric") != std::string::npos;
  const bool sym = !skew && (banner.find("symmetric") != std::string::npos || banner.find("hermitian") != std::string::npos);
  long long nr = 0, nc = 0, ne = 0;
  if (std::sscanf(sz.c_str(), "%lld %lld %lld", &nr, &nc, &ne) != 3 || nr < 0 || nc < 0 || ne < 0)
    io_fail(SKEMA_EINVAL, "bad MatrixMarket coordinate size line");
  if (nc > 0x7fffffffLL) io_fail(SKEMA_EUNSUPPORTED, "more than 2^31 - 1 columns");
  std::vector<int64_t> ri;
  std::vector<int32_t> ci;
  std::vector<double> vi;
  ri.reserve((size_t)ne * ((sym || skew) ? 2 : 1));
  ci.reserve(ri.capacity());
  vi.reserve(ri.capacity());
  const char* p = text.c_str() + L.pos;
  const char* end = text.c_str() + text.size();
  for (long long e = 0; e < ne; ++e) {
    char* q;
    while (p < end && (*p == '%')) {  // comment lines between entries
      while (p < end && *p != '\n') ++p;
      ++p;
    }
    const long long i = std::strtoll(p, &q, 10);
    if (q == p) io_fail(SKEMA_EINVAL, "MatrixMarket coordinate file ends early");
    p = q;
    const long long j = std::strtoll(p, &q, 10);
    if (q == p) io_fail(SKEMA_EINVAL, "bad MatrixMarket coordinate entry");
    p = q;
    double v = 1.0;
    if (!pattern) {
      v = std::strtod(p, &q);
      if (q == p) io_fail(SKEMA_EINVAL, "bad MatrixMarket coordinate value");
      p = q;
    }
    if (i < 1 || i > nr || j < 1 || j > nc) io_fail(SKEMA_EINVAL, "MatrixMarket entry outside the matrix");
    ri.push_back(i - 1), ci.push_back((int32_t)(j - 1)), vi.push_back(v);
    if ((sym || skew) && i != j) {
      ri.push_back(j - 1), ci.push_back((int32_t)(i - 1)), vi.push_back(skew ? -v : v);
    }
  }
  return to_crs(nr, nc, ri, ci, vi);
}

Crs read_bin_crs(const std::string& b) {
  size_t off = 0;
  auto take = [&](void* dst, size_t n) {
    if (off + n > b.size()) io_fail(SKEMA_EINVAL, "binary CRS file ends early");
    std::memcpy(dst, b.data() + off, n);
    off += n;
  };
  int32_t nr32 = 0;
  int64_t nnz = 0;
  take(&nr32, 4);
  take(&nnz, 8);
  if (nr32 < 0 || nnz < 0) io_fail(SKEMA_EINVAL, "bad binary CRS header");
  const int64_t nr = nr32;
  std::vector<uint64_t> rm(nr + 1);
  take(rm.data(), sizeof(uint64_t) * rm.size());
  std::vector<int32_t> col(nnz);
  std::vector<double> val(nnz);
  take(col.data(), sizeof(int32_t) * col.size());
  take(val.data(), sizeof(double) * val.size());
  if (off != b.size()) io_fail(SKEMA_EINVAL, "binary CRS file has trailing bytes");
  if (rm[0] != 0 || (int64_t)rm[nr] != nnz) io_fail(SKEMA_EINVAL, "binary CRS row map does not span the entries");
  int32_t cmax = -1;
  std::vector<int64_t> ri(nnz);
  for (int64_t r = 0; r < nr; ++r) {
    if (rm[r + 1] < rm[r]) io_fail(SKEMA_EINVAL, "binary CRS row map decreases");
    for (uint64_t q = rm[r]; q < rm[r + 1]; ++q) ri[q] = r;
  }
  for (int64_t q = 0; q < nnz; ++q) {
    if (col[q] < 0) io_fail(SKEMA_EINVAL, "negative column in a binary CRS file");
    cmax = std::max(cmax, col[q]);
  }
  // the layout has no column count: square unless a column says otherwise
  const int64_t nc = std::max<int64_t>(nr, (int64_t)cmax + 1);
  return to_crs(nr, nc, ri, col, val);
}

}  // namespace
}  // namespace skema

using skema::IoError;

extern "C" {

static int io_guard(int (*body)(void*), void* arg) {
  try {
    return body(arg);
  } catch (const IoError& e) {
    skema::set_thread_error(e.msg);
    return e.code;
  } catch (const std::bad_alloc&) {
    skema::set_thread_error("host allocation failed");
    return SKEMA_ENOMEM;
  }
}

struct ReadCrsArgs {
  const char* path;
  skema_crs* out;
};

int skema_read_crs(const char* path, skema_crs* out) {
  if (!path || !out) return SKEMA_EINVAL;
  ReadCrsArgs a{path, out};
  return io_guard(
      [](void* v) -> int {
        auto* a = static_cast<ReadCrsArgs*>(v);
        const std::string p(a->path);
        skema::Crs A;
        if (skema::ends_with(skema::lower(p), ".mtx"))
          A = skema::read_mtx_coordinate(skema::read_file(a->path));
        else if (skema::ends_with(skema::lower(p), ".bin"))
          A = skema::read_bin_crs(skema::read_file(a->path));
        else
          skema::io_fail(SKEMA_EINVAL, "only .mtx and .bin files are read");
        skema_crs r{};
        r.nrow = A.nrow, r.ncol = A.ncol, r.nnz = (int64_t)A.col.size();
        r.rowptr = static_cast<int64_t*>(std::malloc(sizeof(int64_t) * (size_t)(r.nrow + 1)));
        r.col = static_cast<int32_t*>(std::malloc(sizeof(int32_t) * (size_t)std::max<int64_t>(r.nnz, 1)));
        r.val = static_cast<double*>(std::malloc(sizeof(double) * (size_t)std::max<int64_t>(r.nnz, 1)));
        if (!r.rowptr || !r.col || !r.val) {
          std::free(r.rowptr), std::free(r.col), std::free(r.val);
          throw std::bad_alloc();
        }
        std::memcpy(r.rowptr, A.rowptr.data(), sizeof(int64_t) * A.rowptr.size());
        if (r.nnz) {
          std::memcpy(r.col, A.col.data(), sizeof(int32_t) * (size_t)r.nnz);
          std::memcpy(r.val, A.val.data(), sizeof(double) * (size_t)r.nnz);
        }
        *a->out = r;
        return SKEMA_OK;
      },
      &a);
}

void skema_crs_free(skema_crs* a) {
  if (!a) return;
  std::free(a->rowptr), std::free(a->col), std::free(a->val);
  a->rowptr = nullptr, a->col = nullptr, a->val = nullptr;
  a->nrow = a->ncol = a->nnz = 0;
}

struct ReadDenseArgs {
  const char* path;
  skema_dense* out;
};

int skema_read_dense(const char* path, skema_dense* out) {
  if (!path || !out) return SKEMA_EINVAL;
  ReadDenseArgs a{path, out};
  return io_guard(
      [](void* v) -> int {
        auto* a = static_cast<ReadDenseArgs*>(v);
        const std::string p = skema::lower(a->path);
        if (skema::ends_with(p, ".bin"))
          skema::io_fail(SKEMA_EUNSUPPORTED, "only sparse binary inputs are read (a dense .bin is rejected)");
        if (!skema::ends_with(p, ".mtx")) skema::io_fail(SKEMA_EINVAL, "only .mtx and .bin files are read");
        const std::string text = skema::read_file(a->path);
        skema::Lines L(text);
        std::string sz;
        const std::string banner = skema::mm_header(L, sz);
        if (banner.find("array") == std::string::npos)
          skema::io_fail(SKEMA_EINVAL, "a dense input needs a MatrixMarket \"array\" file");
        long long nr = 0, nc = 0;
        if (std::sscanf(sz.c_str(), "%lld %lld", &nr, &nc) != 2 || nr < 0 || nc < 0)
          skema::io_fail(SKEMA_EINVAL, "bad MatrixMarket array size line");
        const size_t cnt = (size_t)nr * (size_t)nc;
        double* d = static_cast<double*>(std::malloc(sizeof(double) * std::max<size_t>(cnt, 1)));
        if (!d) throw std::bad_alloc();
        const char* q = text.c_str() + L.pos;
        for (size_t e = 0; e < cnt; ++e) {
          char* r;
          const double x = std::strtod(q, &r);
          if (r == q) {
            std::free(d);
            skema::io_fail(SKEMA_EINVAL, "MatrixMarket array file ends early");
          }
          d[e] = x;  // column-major, as the file lists them
          q = r;
        }
        a->out->nrow = nr, a->out->ncol = nc, a->out->data = d;
        return SKEMA_OK;
      },
      &a);
}

void skema_dense_free(skema_dense* a) {
  if (!a) return;
  std::free(a->data);
  a->data = nullptr;
  a->nrow = a->ncol = 0;
}

struct WriteCrsArgs {
  const char* path;
  const skema_crs* a;
};

int skema_write_crs(const char* path, const skema_crs* a) {
  if (!path || !a || a->nrow < 0 || a->ncol < 0 || !a->rowptr || (a->nnz > 0 && (!a->col || !a->val)))
    return SKEMA_EINVAL;
  WriteCrsArgs w{path, a};
  return io_guard(
      [](void* v) -> int {
        auto* w = static_cast<WriteCrsArgs*>(v);
        const skema_crs& A = *w->a;
        const std::string p = skema::lower(w->path);
        const bool bin = skema::ends_with(p, ".bin");
        if (!bin && !skema::ends_with(p, ".mtx")) skema::io_fail(SKEMA_EINVAL, "only .mtx and .bin files are written");
        if (A.rowptr[0] != 0 || A.rowptr[A.nrow] != A.nnz) skema::io_fail(SKEMA_EINVAL, "rowptr does not span nnz");
        if (bin && A.nrow > 0x7fffffffLL) skema::io_fail(SKEMA_EUNSUPPORTED, "more than 2^31 - 1 rows for .bin");
        FILE* f = std::fopen(w->path, "wb");
        if (!f) skema::io_fail(SKEMA_EINVAL, std::string("cannot create ") + w->path);
        bool ok = true;
        if (bin) {
          const int32_t nr = (int32_t)A.nrow;
          const int64_t nnz = A.nnz;
          std::vector<uint64_t> rm(A.rowptr, A.rowptr + A.nrow + 1);
          ok = std::fwrite(&nr, 4, 1, f) == 1 && std::fwrite(&nnz, 8, 1, f) == 1 &&
               std::fwrite(rm.data(), 8, rm.size(), f) == rm.size() &&
               (nnz == 0 || (std::fwrite(A.col, 4, (size_t)nnz, f) == (size_t)nnz &&
                             std::fwrite(A.val, 8, (size_t)nnz, f) == (size_t)nnz));
        } else {
          ok = std::fprintf(f, "%%%%MatrixMarket matrix coordinate real general\n%lld %lld %lld\n",
                            (long long)A.nrow, (long long)A.ncol, (long long)A.nnz) > 0;
          for (int64_t r = 0; ok && r < A.nrow; ++r)
            for (int64_t q = A.rowptr[r]; ok && q < A.rowptr[r + 1]; ++q)
              ok = std::fprintf(f, "%lld %d %.17g\n", (long long)(r + 1), A.col[q] + 1, A.val[q]) > 0;
        }
        if (std::fclose(f) != 0) ok = false;
        if (!ok) skema::io_fail(SKEMA_EINVAL, std::string("write failed: ") + w->path);
        return SKEMA_OK;
      },
      &w);
}

}  // extern "C"
