// Checks the DimRedux classes of include/skema.hpp against explicit FP64
// products of the exported maps, with the reference's conventions for each
// call (src/Skema_DimRedux_Gauss.cpp:10-99, src/Skema_DimRedux_SparseSign.cpp:
// 9-111): dense lmap op(M(:, idx)) op(B) with transA swapped by
// init_transposed; dense rmap op(A) op(M); Gauss CRS lmap (op(B) M(:, idx))^T
// and rmap op(A) M(idx, :); SparseSign CRS lmap M(:, idx) B and rmap A M.
// Prints the largest relative error and exits 0 when it is below 1e-5.
#include <cmath>
#include <cstdio>
#include <functional>
#include <iostream>

#include "skema.hpp"

namespace {

unsigned long long g_state = 88172645463325252ull;
double unif() {  // xorshift64, values in [-1, 1)
  g_state ^= g_state << 13;
  g_state ^= g_state >> 7;
  g_state ^= g_state << 17;
  return (double)(g_state >> 11) / (double)(1ull << 52) - 1.0;
}

matrix_type random_dense(size_type m, size_type n) {
  matrix_type A("A", m, n);
  for (size_type j = 0; j < n; ++j)
    for (size_type i = 0; i < m; ++i) A(i, j) = (double)(float)unif();
  return A;
}

crs_matrix_type random_crs(size_type m, size_type n, int per_row) {
  std::vector<size_type> rm(m + 1, 0);
  std::vector<int> ent;
  std::vector<double> val;
  for (size_type i = 0; i < m; ++i) {
    std::vector<int> cols;
    for (int t = 0; t < per_row; ++t) cols.push_back((int)((unif() + 1.0) * 0.5 * (double)n) % (int)n);
    std::sort(cols.begin(), cols.end());
    cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
    for (int c : cols) {
      ent.push_back(c);
      val.push_back((double)(float)unif());
    }
    rm[i + 1] = ent.size();
  }
  const size_type nnz = ent.size();
  return crs_matrix_type("S", m, n, nnz, val, rm, ent);
}

matrix_type to_dense(const crs_matrix_type& S) {
  matrix_type D("D", S.numRows(), S.numCols());
  for (size_type i = 0; i < S.numRows(); ++i)
    for (size_type p = S.row_map[i]; p < S.row_map[i + 1]; ++p) D(i, S.entries[p]) += S.values[p];
  return D;
}

matrix_type op(const matrix_type& A, char t) {
  if (t == 'N') return A;
  matrix_type B("T", A.extent(1), A.extent(0));
  for (size_type i = 0; i < A.extent(0); ++i)
    for (size_type j = 0; j < A.extent(1); ++j) B(j, i) = A(i, j);
  return B;
}

matrix_type mul(const matrix_type& A, const matrix_type& B, double alpha) {
  if (A.extent(1) != B.extent(0)) throw std::runtime_error("reference product: shapes");
  matrix_type C("C", A.extent(0), B.extent(1));
  for (size_type j = 0; j < B.extent(1); ++j)
    for (size_type k = 0; k < A.extent(1); ++k)
      for (size_type i = 0; i < A.extent(0); ++i) C(i, j) += alpha * A(i, k) * B(k, j);
  return C;
}

matrix_type cols(const matrix_type& A, range_type idx) {
  if (idx.first == idx.second) return A;
  matrix_type B("cols", A.extent(0), idx.second - idx.first);
  for (size_type j = idx.first; j < idx.second; ++j)
    for (size_type i = 0; i < A.extent(0); ++i) B(i, j - idx.first) = A(i, j);
  return B;
}

matrix_type rows(const matrix_type& A, range_type idx) { return op(cols(op(A, 'T'), idx), 'T'); }

double rel(const matrix_type& got, const matrix_type& ref) {
  if (got.extent(0) != ref.extent(0) || got.extent(1) != ref.extent(1)) return 1e30;
  double num = 0, den = 0;
  for (size_type j = 0; j < ref.extent(1); ++j)
    for (size_type i = 0; i < ref.extent(0); ++i) {
      num += (got(i, j) - ref(i, j)) * (got(i, j) - ref(i, j));
      den += ref(i, j) * ref(i, j);
    }
  return std::sqrt(num / (den > 0 ? den : 1.0));
}

template <typename Map>
matrix_type exported(const Map& M, size_type nrow, size_type ncol, bool sparse) {
  std::vector<double> v;
  std::vector<int32_t> ix;
  M.export_map(v, ix);
  matrix_type D("M", nrow, ncol);
  if (!sparse) {
    for (size_type j = 0; j < ncol; ++j)
      for (size_type i = 0; i < nrow; ++i) D(i, j) = v[i + j * nrow];
  } else {
    const size_type z = v.size() / nrow;
    for (size_type i = 0; i < nrow; ++i)
      for (size_type t = 0; t < z; ++t) D(i, ix[i * z + t]) += v[i * z + t];
  }
  return D;
}

double worst = 0.0;
void report(const std::string& what, double e) {
  std::printf("%-44s %.3e\n", what.c_str(), e);
  worst = std::max(worst, e);
}

template <typename Map>
void check_kind(bool sparse) {
  const size_type nrow = 23, ncol = 37;
  const double alpha = 1.5, beta = 0.0;
  const std::string k = sparse ? "sparse-sign" : "gauss";
  for (bool init_t : {false, true}) {
    Map M(nrow, ncol, 7, k, false, "", init_t);
    const matrix_type D = exported(M, nrow, ncol, sparse);
    for (char ta : {'N', 'T'})
      for (char tb : {'N', 'T'})
        for (range_type idx : {range_type(0, 0), range_type(4, 15)}) {
          const char eff = init_t ? (ta == 'N' ? 'T' : 'N') : ta;
          const matrix_type Mi = cols(D, idx);
          const size_type inner = eff == 'N' ? Mi.extent(1) : Mi.extent(0);
          const matrix_type B = op(random_dense(inner, 9), tb);  // op(B) is inner x 9
          const std::string tag = k + " lmap " + ta + tb + (init_t ? " init_t" : "") + (idx.first ? " idx" : "");
          report(tag, rel(M.lmap(&alpha, B, &beta, ta, tb, idx), mul(op(Mi, eff), op(B, tb), alpha)));
        }
    for (char ta : {'N', 'T'})
      for (char tb : {'N', 'T'}) {
        const size_type inner = tb == 'N' ? nrow : ncol;
        const matrix_type A = op(random_dense(11, inner), ta);  // op(A) is 11 x inner
        report(k + " rmap " + ta + tb + (init_t ? " init_t" : ""),
               rel(M.rmap(&alpha, A, &beta, ta, tb), mul(op(A, ta), op(D, tb), alpha)));
      }
  }
  Map M(nrow, ncol, 9, k);
  const matrix_type D = exported(M, nrow, ncol, sparse);
  for (range_type idx : {range_type(0, 0), range_type(3, 30)}) {
    const matrix_type Mi = cols(D, idx);
    if (!sparse) {
      for (char tb : {'N', 'T'}) {
        // (op(B) M(:, idx))^T with op(B) 13 x nrow
        const crs_matrix_type S = tb == 'N' ? random_crs(13, nrow, 4) : random_crs(nrow, 13, 3);
        const matrix_type ref = op(mul(op(to_dense(S), tb), Mi, alpha), 'T');
        report(k + " lmap crs " + tb + (idx.first ? " idx" : ""), rel(M.lmap(&alpha, S, &beta, 'N', tb, idx), ref));
      }
    } else {
      const crs_matrix_type S = random_crs(Mi.extent(1), 17, 4);
      report(k + " lmap crs" + (idx.first ? " idx" : ""),
             rel(M.lmap(&alpha, S, &beta, 'N', 'N', idx), mul(Mi, to_dense(S), 1.0)));
    }
  }
  for (range_type idx : {range_type(0, 0), range_type(2, 20)}) {
    const matrix_type Mi = sparse ? D : rows(D, idx);
    if (!sparse) {
      for (char ta : {'N', 'T'}) {
        const crs_matrix_type S = ta == 'N' ? random_crs(15, Mi.extent(0), 5) : random_crs(Mi.extent(0), 15, 2);
        report(k + " rmap crs " + ta + (idx.first ? " idx" : ""),
               rel(M.rmap(&alpha, S, &beta, ta, 'N', idx), mul(op(to_dense(S), ta), Mi, alpha)));
      }
    } else if (idx.first == 0) {
      const crs_matrix_type S = random_crs(15, nrow, 5);
      report(k + " rmap crs", rel(M.rmap(&alpha, S, &beta, 'N', 'N'), mul(to_dense(S), D, 1.0)));
    }
  }
}

}  // namespace

int main() {
  check_kind<Skema::GaussDimRedux>(false);
  check_kind<Skema::SparseSignDimRedux>(true);
  std::printf("worst %.3e\n", worst);
  return worst < 1e-5 ? 0 : 1;
}
