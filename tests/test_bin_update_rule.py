"""CPU check of the update rule the CSR x SparseSign Y kernel relies on.

The kernel takes the zeta = 8 map in a 16-bit offset form: per input column
eight entries (bin * 128) | sign << 15 | dup, stably sorted by bin, dup set
when an entry's bin equals the previous entry's (pack16_kernel in
skema_b200/csrc/maps.cu). Per nonzero it loads the eight bins first, then
stores the eight sums in entry order, and a flagged entry adds to the
previous entry's new sum instead of its own load (ssign_apply8 in
skema_b200/csrc/sparse.cu). This restates both in numpy float32 and checks,
bit for bit, that the result equals adding the entries one by one in their
original order, for rows with repeated bins anywhere (SparseSign draws its
indices with replacement, src/Skema_DimRedux.hpp:226-235, and imported maps
may be unsorted).
"""
import numpy as np


def pack16(idx, neg):
    """Offset form of one map row: stable sort by bin, then the dup flags."""
    h = [((int(b) & 0xFF) << 7) | (int(s) << 15) for b, s in zip(idx, neg)]
    h = sorted(h, key=lambda e: e & 0x7F80)  # Python's sort is stable
    return [e | (1 if t and (e & 0x7F80) == (h[t - 1] & 0x7F80) else 0) for t, e in enumerate(h)]


def apply_batched(bins, entries, a):
    """Eight loads, then eight stores in entry order with forwarding."""
    a = np.float32(a)
    v = [bins[(e & 0x7F80) >> 7] for e in entries]
    prev = np.float32(0)
    for t, e in enumerate(entries):
        add = -a if e & 0x8000 else a
        nv = np.float32((prev if e & 1 else v[t]) + add)
        bins[(e & 0x7F80) >> 7] = nv
        prev = nv


def apply_sequential(bins, idx, neg, a):
    a = np.float32(a)
    for b, s in zip(idx, neg):
        bins[b] = np.float32(bins[b] + (-a if s else a))


def test_batched_update_equals_sequential_bitwise():
    rng = np.random.default_rng(11)
    for trial in range(300):
        k = 81 if trial % 2 else 256
        ncols = 50
        idx = rng.integers(0, k, size=(ncols, 8))
        if trial % 3 == 0:
            idx.sort(axis=1)  # generated rows are sorted
        idx[::4, 5] = idx[::4, 1]  # repeats apart
        idx[::7, 2:6] = idx[::7, 6:7]  # four of one bin
        neg = rng.integers(0, 2, size=(ncols, 8))
        packed = [pack16(idx[j], neg[j]) for j in range(ncols)]
        b1 = np.zeros(k, dtype=np.float32)
        b2 = np.zeros(k, dtype=np.float32)
        for _ in range(12):  # the nonzeros of one row, in order
            j = int(rng.integers(0, ncols))
            a = np.float32(rng.normal() * 10.0 ** int(rng.integers(-3, 4)))
            apply_batched(b1, packed[j], a)
            apply_sequential(b2, idx[j], neg[j], a)
        assert np.array_equal(b1.view(np.uint32), b2.view(np.uint32)), trial


def test_pack16_layout():
    e = pack16([5, 3, 5, 80, 3, 3, 0, 5], [0, 1, 1, 0, 0, 1, 0, 1])
    assert [(x & 0x7F80) >> 7 for x in e] == [0, 3, 3, 3, 5, 5, 5, 80]
    assert [x & 1 for x in e] == [0, 0, 1, 1, 0, 1, 1, 0]
    # the sign travels with its entry through the stable sort
    assert [(x >> 15) & 1 for x in e] == [0, 1, 0, 1, 0, 1, 1, 0]
    assert all(x & 0x7E == 0 for x in e)  # bits 1-6 stay clear
