"""Regenerate tests/golden/kat_fixtures.npz from the reference's test data.

The reference (jeremy-myers/skema) ships small matrices with their exact
singular values under test/data/ (rectangular 32x14, symmetric 27x27 in
dense, MatrixMarket and binary CRS form, and 25 kernel points in 2-D whose
Gauss RBF kernel at gamma = 1 has the listed singular values). This script
reads them from a reference checkout and stores them as one compressed
numpy archive, so the tests run where the reference is not present.

Usage: python tests/golden/make_golden.py REFERENCE_ROOT
   or: SKEMA_REFERENCE=REFERENCE_ROOT python tests/golden/make_golden.py
"""
import os
import struct
import sys

import numpy as np

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SKEMA_REFERENCE", "")
if not REF:
    sys.exit("usage: make_golden.py REFERENCE_ROOT (or set SKEMA_REFERENCE)")
DATA = os.path.join(REF, "test", "data")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "kat_fixtures.npz")


def read_txt(name):
    return np.loadtxt(os.path.join(DATA, name), dtype=np.float64, ndmin=2)


def read_mtx(name):
    """MatrixMarket coordinate real general/symmetric -> (m, n, rows, cols, vals)."""
    with open(os.path.join(DATA, name)) as f:
        header = f.readline().lower()
        symmetric = "symmetric" in header
        line = f.readline()
        while line.startswith("%"):
            line = f.readline()
        m, n, nnz = (int(x) for x in line.split())
        rows, cols, vals = [], [], []
        for _ in range(nnz):
            i, j, v = f.readline().split()
            i, j, v = int(i) - 1, int(j) - 1, float(v)
            rows.append(i)
            cols.append(j)
            vals.append(v)
            if symmetric and i != j:
                rows.append(j)
                cols.append(i)
                vals.append(v)
    return m, n, np.array(rows), np.array(cols), np.array(vals)


def to_csr(m, rows, cols, vals):
    order = np.lexsort((cols, rows))
    rows, cols, vals = rows[order], cols[order], vals[order]
    rowptr = np.zeros(m + 1, dtype=np.int64)
    np.add.at(rowptr, rows + 1, 1)
    return np.cumsum(rowptr), cols.astype(np.int32), vals


def read_bin(name):
    """int32 nrows, int64 nnz, size_t row_map[nrows+1], int32 entries[nnz],
    double values[nnz] (the layout of the reference's .bin CRS files)."""
    raw = open(os.path.join(DATA, name), "rb").read()
    nrows, = struct.unpack_from("<i", raw, 0)
    nnz, = struct.unpack_from("<q", raw, 4)
    off = 12
    row_map = np.frombuffer(raw, dtype="<u8", count=nrows + 1, offset=off).astype(np.int64)
    off += 8 * (nrows + 1)
    entries = np.frombuffer(raw, dtype="<i4", count=nnz, offset=off).astype(np.int32)
    off += 4 * nnz
    values = np.frombuffer(raw, dtype="<f8", count=nnz, offset=off).copy()
    assert off + 8 * nnz == len(raw)
    return row_map, entries, values


def main():
    fx = {}
    fx["rect_dense"] = read_txt("rectangular_dense.txt")
    fx["rect_svals"] = read_txt("rectangular_svals.txt").ravel()
    m, n, r, c, v = read_mtx("rectangular_sparse.mtx")
    fx["rect_csr_rowptr"], fx["rect_csr_col"], fx["rect_csr_val"] = to_csr(m, r, c, v)
    fx["rect_csr_shape"] = np.array([m, n])
    fx["sym_dense"] = read_txt("symmetric_dense.txt")
    fx["sym_svals"] = read_txt("symmetric_svals.txt").ravel()
    m, n, r, c, v = read_mtx("symmetric_sparse.mtx")
    fx["sym_csr_rowptr"], fx["sym_csr_col"], fx["sym_csr_val"] = to_csr(m, r, c, v)
    fx["sym_csr_shape"] = np.array([m, n])
    fx["sym_bin_rowptr"], fx["sym_bin_col"], fx["sym_bin_val"] = read_bin("symmetric_sparse.bin")
    fx["kernel_points"] = read_txt("kernel_data.txt")
    fx["kernel_svals"] = read_txt("kernel_svals.txt").ravel()
    np.savez_compressed(OUT, **fx)
    print(f"wrote {OUT}: " + ", ".join(f"{k}{list(np.shape(v))}" for k, v in fx.items()))


if __name__ == "__main__":
    main()
