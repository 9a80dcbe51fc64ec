"""Python host mirror of Skema's SketchySVD interface over the C ABI.

Names and argument meanings follow the reference:

* ``AlgParams`` -- the sketch fields of ``Skema::AlgParams``
  (src/Skema_AlgParams.hpp:12-90) with the same defaults
  (src/Skema_AlgParams.cpp:10-57) and the same command-line flags and
  parsing rules (src/Skema_AlgParams.cpp:242-330, 335-600).
* ``GaussDimRedux`` / ``SparseSignDimRedux`` -- the map types
  (src/Skema_DimRedux.hpp:98-268), used as the DimReduxT selector.
* ``SketchySVD`` -- ctor, ``linear_update``, ``low_rank_approx``
  (src/Skema_SketchySVD.hpp:11-64); ``SketchySPD`` -- the one-sketch variant
  (src/Skema_SketchySVD.hpp:67-108), update only.
* ``sketchysvd(matrix, algParams)`` -- the driver entry
  (src/Skema_SketchySVD.cpp:1244, 1408), returning (U, S, V).

Inputs are numpy arrays / scipy CSR matrices (host memory, staged by the
library) or CUDA torch tensors (device memory, used in place). Every call
goes to the CUDA library; errors raise ``SkemaError``.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Any

import numpy as np

from . import _lib as L
from ._lib import SkemaError

__all__ = [
    "AlgParams",
    "GaussDimRedux",
    "SparseSignDimRedux",
    "SketchySVD",
    "SketchySPD",
    "sketchysvd",
    "rbf_sketch_fwd",
    "rbf_sketch_vjp",
    "SkemaError",
]

INT_MAX = 2**31 - 1


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


def _error(msg: str):
    # Skema::error (src/Skema_AlgParams.cpp:59-62)
    raise RuntimeError(msg)


def _find(args: list[str], flag: str) -> int:
    if flag in args:
        return args.index(flag)
    if len(flag) > 2 and flag.startswith("--") and flag[2:] in args:
        return args.index(flag[2:])
    return -1


def parse_bool(args, on, off, default):
    """src/Skema_AlgParams.cpp:335-366."""
    i = _find(args, on)
    if i >= 0:
        del args[i]
        return True
    i = _find(args, off)
    if i >= 0:
        del args[i]
        return False
    return default


def parse_int(args, flag, default, lo=0, hi=100):
    """src/Skema_AlgParams.cpp:433-474 (strtol prefix parse, 'inf' -> INT_MAX)."""
    val = default
    i = _find(args, flag)
    if i >= 0:
        if i + 1 >= len(args):
            del args[i]
            return val
        s = args[i + 1]
        if s in ("inf", "Inf"):
            val = INT_MAX
        else:
            j = 0
            t = s.strip()
            if t[:1] in "+-":
                j = 1
            while j < len(t) and t[j].isdigit():
                j += 1
            if j == 0 or (j == 1 and t[:1] in "+-"):
                _error(f"Unparseable input: {flag} {s}, must be an integer")
            val = int(t[:j])
        del args[i : i + 2]
    if val < lo or val > hi:
        _error(f"Bad input: {flag} {val},  must be in the range ({lo}, {hi})")
    return val


def parse_real(args, flag, default, lo=0.0, hi=1.0):
    """src/Skema_AlgParams.cpp:476-513."""
    val = default
    i = _find(args, flag)
    if i >= 0:
        if i + 1 >= len(args):
            del args[i]
            return val
        s = args[i + 1]
        try:
            val = float(s)
        except ValueError:
            _error(f"Unparseable input: {flag} {s}, must be a double")
        del args[i : i + 2]
    if val < lo or val > hi:
        _error(f"Bad input: {flag} {val},  must be in the range ({lo}, {hi})")
    return val


def parse_enum(args, flag, default, names):
    """src/Skema_AlgParams.cpp:368-412; returns the index into names."""
    i = _find(args, flag)
    if i >= 0:
        if i + 1 >= len(args):
            del args[i]
            return default
        v = args[i + 1]
        del args[i : i + 2]
        if v in names:
            return names.index(v)
        _error(f"Bad input: {flag} {v},  must be one of the values: {', '.join(names)}.")
    return default


def parse_string(args, flag, default):
    i = _find(args, flag)
    if i >= 0:
        if i + 1 >= len(args):
            del args[i]
            return default
        v = args[i + 1]
        del args[i : i + 2]
        return v
    return default


def parse_int_array(args, flag, default, lo=1, hi=INT_MAX):
    """src/Skema_AlgParams.cpp:549-606: '[a,b,c]' with no spaces."""
    i = _find(args, flag)
    if i < 0:
        return list(default)
    if i + 1 >= len(args):
        del args[i]
        return list(default)
    s = args[i + 1]
    if not s.startswith("["):
        _error(f"Unparseable input: {flag} {s}, must be of the form [int,...,int] with no spaces")
    body = s[1:]
    if body.endswith("]"):
        body = body[:-1]
    vals = []
    for tok in body.split(","):
        if tok == "":
            continue
        try:
            v = int(tok)
        except ValueError:
            _error(f"Unparseable input: {flag} {tok}, must be of the form [int,...,int] with no spaces")
        if v < lo or v > hi:
            _error(f"Bad input: {flag} {tok},  must be in the range ({lo}, {hi})")
        vals.append(v)
    del args[i : i + 2]
    return vals


DIM_REDUX_NAMES = ["gauss", "sparse-sign"]      # src/Skema_Utils.hpp:74-80
KERNEL_NAMES = ["none", "gaussrbf"]              # src/Skema_Utils.hpp:60-66
SOLVER_NAMES = ["isvd", "sketch", "primme"]      # src/Skema_Utils.hpp:46-52
PRECISION_NAMES = ["fp32", "bf16", "fp8"]
SPD_APPROX_NAMES = ["nystrom", "reference-steps"]


@dataclass
class AlgParams:
    """Sketch fields of Skema::AlgParams with the reference defaults."""

    solver: int = 0
    inputfilename: str = ""
    history_filename: str = ""
    debug_filename: str = ""
    issparse: bool = False
    issymmetric: bool = False
    matrix_m: int = 0
    matrix_n: int = 0
    matrix_nnz: int = 0
    rank: int = 1
    num_passes: int = 1
    print_level: int = 0
    debug: bool = False
    window: int = 1
    sketch_range: int = 1
    sketch_core: int = 1
    sketch_eta: float = 1.0
    sketch_nu: float = 1.0
    seeds: list = field(default_factory=lambda: [0, 1, 2, 3])
    force_three_sketch: bool = False
    sketch_compute_svals_iters: bool = False
    dim_redux: int = L.MAP_GAUSS
    kernel_func: int = L.KERNEL_NONE
    kernel_gamma: float = 1.0
    precision: int = L.PREC_FP32
    device: int = 0
    spd_approx: int = L.SPD_NYSTROM

    def parse(self, args: list[str]) -> None:
        """Consume the sketch flags from args, as AlgParams::parse does."""
        self.inputfilename = parse_string(args, "--input", "")
        self.debug_filename = parse_string(args, "--debug-file", "")
        self.history_filename = parse_string(args, "--history-file", "")
        self.issparse = parse_bool(args, "--sparse", "--dense", False)
        self.issymmetric = parse_bool(args, "--symmetric", "--asymmetric", False)
        self.matrix_m = parse_int(args, "--m", self.matrix_m, 0, INT_MAX)
        self.matrix_n = parse_int(args, "--n", self.matrix_n, 0, INT_MAX)
        self.rank = parse_int(args, "--rank", self.rank, 1, INT_MAX)
        self.num_passes = parse_int(args, "--num-passes", self.num_passes, 1, INT_MAX)
        self.solver = parse_enum(args, "--solver", 0, SOLVER_NAMES)
        self.print_level = parse_int(args, "--print-level", self.print_level, 0, 5)
        self.debug = parse_bool(args, "--debug", "--debug-off", False)
        self.window = parse_int(args, "--window", self.window, 1, INT_MAX)
        self.dim_redux = parse_enum(args, "--model", L.MAP_GAUSS, DIM_REDUX_NAMES)
        self.sketch_range = parse_int(args, "--range", self.sketch_range, 0, INT_MAX)
        self.sketch_core = parse_int(args, "--core", self.sketch_core, 0, INT_MAX)
        self.seeds = parse_int_array(args, "--seeds", self.seeds, 0, INT_MAX)
        self.sketch_eta = parse_real(args, "--eta", 1.0, 0.0, math.inf)
        self.sketch_nu = parse_real(args, "--nu", 1.0, 0.0, math.inf)
        self.force_three_sketch = parse_bool(args, "--force-three-sketch", "--force-three-sketch-off", False)
        self.sketch_compute_svals_iters = parse_bool(
            args, "--sketch-compute-svals-iters", "--sketch-compute-svals-iters-off", False
        )
        self.kernel_func = parse_enum(args, "--kernel", L.KERNEL_NONE, KERNEL_NAMES)
        self.kernel_gamma = parse_real(args, "--gamma", self.kernel_gamma, 0.0, math.inf)
        self.precision = parse_enum(args, "--precision", L.PREC_FP32, PRECISION_NAMES)
        self.spd_approx = parse_enum(args, "--spd-approx", L.SPD_NYSTROM, SPD_APPROX_NAMES)

    def to_c(self) -> L.Params:
        p = L.default_params()
        p.matrix_m = int(self.matrix_m)
        p.matrix_n = int(self.matrix_n)
        p.rank = int(self.rank)
        p.sketch_range = int(self.sketch_range)
        p.sketch_core = int(self.sketch_core)
        p.window = int(self.window)
        p.sketch_eta = float(self.sketch_eta)
        p.sketch_nu = float(self.sketch_nu)
        seeds = list(self.seeds) + [0, 1, 2, 3][len(self.seeds):]
        for i in range(4):
            p.seeds[i] = int(seeds[i])
        p.dim_redux = int(self.dim_redux)
        p.issparse = int(bool(self.issparse))
        p.issymmetric = int(bool(self.issymmetric))
        p.force_three_sketch = int(bool(self.force_three_sketch))
        p.kernel_func = int(self.kernel_func)
        p.kernel_gamma = float(self.kernel_gamma)
        p.precision = int(self.precision)
        p.device = int(self.device)
        p.spd_approx = int(self.spd_approx)
        return p


class GaussDimRedux:
    """DimReduxT selector: dense maps uniform on +-sqrt(2 ln(rows*cols))."""

    kind = L.MAP_GAUSS


class SparseSignDimRedux:
    """DimReduxT selector: zeta = max(2, min(ncol, 8)) +-1 entries per stored row."""

    kind = L.MAP_SPARSE_SIGN


# ---------------------------------------------------------------- helpers --
def _dense_arg(A):
    """(pointer, ld, layout, mem, keepalive) for a 2-D float32 array/tensor."""
    if _is_torch(A):
        import torch

        if A.dtype != torch.float32:
            raise TypeError("dense input must be float32")
        if A.dim() != 2:
            raise ValueError("dense input must be 2-D")
        if not A.is_cuda:
            A = A.numpy()
        else:
            if A.stride(1) == 1 and (A.stride(0) >= A.shape[1] or A.shape[0] <= 1):
                return A.data_ptr(), max(A.stride(0), A.shape[1], 1), L.ROW_MAJOR, L.MEM_DEVICE, A
            if A.stride(0) == 1 and (A.stride(1) >= A.shape[0] or A.shape[1] <= 1):
                return A.data_ptr(), max(A.stride(1), A.shape[0], 1), L.COL_MAJOR, L.MEM_DEVICE, A
            A = A.contiguous()
            return A.data_ptr(), A.shape[1], L.ROW_MAJOR, L.MEM_DEVICE, A
    A = np.asarray(A)
    if A.ndim != 2:
        raise ValueError("dense input must be 2-D")
    if A.dtype != np.float32:
        A = A.astype(np.float32)
    if A.flags.f_contiguous and not A.flags.c_contiguous:
        return A.ctypes.data, max(A.shape[0], 1), L.COL_MAJOR, L.MEM_HOST, A
    A = np.ascontiguousarray(A)
    return A.ctypes.data, max(A.shape[1], 1), L.ROW_MAJOR, L.MEM_HOST, A


def _csr_arg(A):
    """(rowptr, col, val, nrows, ncols, mem, keepalive) for a CSR input."""
    if isinstance(A, tuple):
        rowptr, col, val = A[:3]
        if _is_torch(rowptr) and rowptr.is_cuda:
            import torch

            assert rowptr.dtype == torch.int64 and col.dtype == torch.int32 and val.dtype == torch.float32
            return rowptr.data_ptr(), col.data_ptr(), val.data_ptr(), rowptr.numel() - 1, None, L.MEM_DEVICE, A
        rowptr = np.ascontiguousarray(rowptr, dtype=np.int64)
        col = np.ascontiguousarray(col, dtype=np.int32)
        val = np.ascontiguousarray(val, dtype=np.float32)
        keep = (rowptr, col, val)
        return rowptr.ctypes.data, col.ctypes.data, val.ctypes.data, len(rowptr) - 1, None, L.MEM_HOST, keep
    # scipy.sparse
    A = A.tocsr()
    rowptr = np.ascontiguousarray(A.indptr, dtype=np.int64)
    col = np.ascontiguousarray(A.indices, dtype=np.int32)
    val = np.ascontiguousarray(A.data, dtype=np.float32)
    keep = (rowptr, col, val)
    return rowptr.ctypes.data, col.ctypes.data, val.ctypes.data, A.shape[0], A.shape[1], L.MEM_HOST, keep


def _row_block(A, r0, w):
    """Rows [r0, r0 + w) of a dense (numpy / torch) or CSR (scipy or
    (rowptr, col, val)) input, as the block the update entry points take."""
    if isinstance(A, tuple):
        rowptr, col, val = A[:3]
        return (rowptr[r0:r0 + w + 1], col, val)  # absolute offsets into col / val
    return A[r0:r0 + w]


class _Context:
    def __init__(self, alg: AlgParams, dim_redux=None):
        if dim_redux is not None:
            alg.dim_redux = dim_redux.kind
        self.alg = alg
        self.lib = L.load()
        p = alg.to_c()
        h = C.c_void_p()
        st = self.lib.skema_create(C.byref(p), C.byref(h))
        if st != L.OK:
            msg = self.lib.skema_last_error(None)
            raise SkemaError(st, msg.decode() if msg else "")
        self.h = h
        k, s, spd = C.c_int64(), C.c_int64(), C.c_int32()
        self._check(self.lib.skema_get_dims(self.h, C.byref(k), C.byref(s), C.byref(spd)))
        self.range, self.core, self.spd = k.value, s.value, bool(spd.value)
        self.nrow, self.ncol, self.rank = alg.matrix_m, alg.matrix_n, alg.rank
        # like the reference, which keeps the last approximation's uvecs,
        # svals and vvecs for compute_residuals, the context keeps them on the
        # device, so the residual pass needs no host copy of U
        self._check(self.lib.skema_set_keep_factors(self.h, 1))
        stem = self.debug_stem()
        if stem:
            self.map_export_reference_dumps(stem)

    def debug_stem(self):
        """The stem of AlgParams.debug_filename, or None. Like the reference's
        --debug-file dumps (debug_filename.filename().stem(),
        src/Skema_DimRedux.hpp:124-127, src/Skema_SketchySVD.cpp:192-205), the
        files are written as <stem>_<name> in the working directory."""
        import os

        f = getattr(self.alg, "debug_filename", "")
        return os.path.splitext(os.path.basename(str(f)))[0] if f else None

    def dump_sketches(self, stem, suffix=""):
        """<stem>_X.txt, _Y.txt, _Z.txt (SketchySPD: _Y.txt) with the given
        suffix, in the reference's text format (write_dense_text)."""
        names = ((L.SKETCH_Y, "Y"),) if self.spd else ((L.SKETCH_X, "X"), (L.SKETCH_Y, "Y"), (L.SKETCH_Z, "Z"))
        for which, name in names:
            write_dense_text(f"{stem}_{name}.txt{suffix}", self.get_sketch(which))

    def _check(self, st):
        if st != L.OK:
            msg = self.lib.skema_last_error(self.h)
            raise SkemaError(st, msg.decode() if msg else "")

    def close(self):
        if getattr(self, "h", None):
            self.lib.skema_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- streaming --------------------------------------------------------
    def reset(self):
        self._check(self.lib.skema_reset(self.h))

    def update_rows(self, A, row0: int = 0, nrows: int | None = None):
        """Stream rows [row0, row0+nrows) (default: all rows of A)."""
        self._stream(A, row0, nrows, "skema_linear_update")

    def update_from_file(self, path, row0: int = 0, nrows: int | None = None):
        """Stream rows [row0, row0+nrows) of a matrix file (.bin CRS a window
        at a time, MatrixMarket after a whole read) into the sketches
        (skema_update_from_file). nrows None: to the last row of the file."""
        self._check(self.lib.skema_update_from_file(self.h, str(path).encode(), int(row0),
                                                    -1 if nrows is None else int(nrows)))

    def _stream(self, A, row0, nrows, prefix):
        self._torch_inputs_ready(*(A if isinstance(A, tuple) else (A,)))
        if self.alg.kernel_func == L.KERNEL_GAUSSRBF:
            ptr, ld, layout, mem, keep = _dense_arg(A)
            npts, d = A.shape
            nr = self.nrow - row0 if nrows is None else nrows
            self._check(getattr(self.lib, prefix + "_rbf")(self.h, ptr, ld, layout, npts, d, row0, nr, mem))
        elif self.alg.issparse:
            rp, col, val, nr_in, _, mem, keep = _csr_arg(A)
            nr = nr_in if nrows is None else nrows
            self._check(getattr(self.lib, prefix + "_csr")(self.h, rp, col, val, row0, nr, mem))
        else:
            ptr, ld, layout, mem, keep = _dense_arg(A)
            nr = A.shape[0] if nrows is None else nrows
            self._check(getattr(self.lib, prefix + "_dense")(self.h, ptr, ld, layout, row0, nr, mem))
        if mem == L.MEM_HOST:
            self.synchronize()
        del keep

    # -- residuals --------------------------------------------------------
    def residuals(self, A, U, S, V, row_blocks=None):
        """Skema::residuals (src/Skema_Residuals.hpp:160-217): per-column
        ||[A^T U - V S; A V - U S]||_2 (SketchySPD: ||A V - V S||_2) for host
        FP64 U (m x r), S (r), V (n x r); A streamed again like the update.
        U, S and V all None: the factors of the last low_rank_approx, kept
        on the device. row_blocks: optional list of (row0, A_block) pairs
        instead of A."""
        if U is None and S is None and V is None:
            self._check(self.lib.skema_residuals_begin(self.h, None, None, None, L.MEM_HOST))
        else:
            Uc = None if U is None else np.asfortranarray(np.asarray(U, dtype=np.float64))
            Sc = np.ascontiguousarray(np.asarray(S, dtype=np.float64))
            Vc = np.asfortranarray(np.asarray(V, dtype=np.float64))
            self._check(self.lib.skema_residuals_begin(self.h, None if Uc is None else Uc.ctypes.data,
                                                       Sc.ctypes.data, Vc.ctypes.data, L.MEM_HOST))
        for row0, blk in (row_blocks if row_blocks is not None else [(0, A)]):
            self._stream(blk, row0, None, "skema_residuals_update")
        out = np.empty(self.rank, dtype=np.float64)
        self._check(self.lib.skema_residuals_finish(self.h, out.ctypes.data, L.MEM_HOST))
        return out

    def compute_residuals(self, A):
        """SketchySVD::compute_residuals (src/Skema_SketchySVD.cpp:719-727):
        residual norms of the last low_rank_approx, kept as self.rnrms."""
        if getattr(self, "uvecs", None) is None:
            raise SkemaError(L.ESTATE, "compute_residuals needs a low_rank_approx first")
        try:  # the factors kept on the device
            self.rnrms = self.residuals(A, None, None, None)
        except SkemaError as e:  # replaced by factors passed to residuals() since
            if e.status != L.ESTATE:
                raise
            self.rnrms = self.residuals(A, self.uvecs, self.svals, self.vvecs)
        return self.rnrms

    def save_history(self, path=None):
        """SketchySVD::save_history (src/Skema_SketchySVD.cpp:730-755): a JSON
        object with "timings", "traces", "svals" and "rnrms", keys sorted and
        a 4-space indent as the reference's JSON writer prints it, written to
        `path`, or returned as a string when path is None. Timings hold the
        reference's keys (reference_timings)."""
        r = self.rank
        sv = getattr(self, "svals", None)
        rn = getattr(self, "rnrms", None)
        return write_history(path, np.zeros(r) if sv is None else sv, np.zeros(r) if rn is None else rn,
                             traces=getattr(self, "traces", None), timings=self.reference_timings())

    def reference_timings(self):
        """The reference's timing keys (src/Skema_SketchySVD.cpp:101-116;
        SketchySPD :776-786), in seconds, from this context's device stage
        timers (zero unless timing_enable was called, and where no stage
        corresponds): update.{upsilon, omega, phi, psi, window, daxpy} from the
        stages of the same names (the sparse-sign X / Z entry kernel under
        upsilon, the fused tensor-core window kernel under omega) and
        approx.{dgeqrf, dgels, dgesvd, dgemm} from approx.{orth, core, svd,
        vectors}."""

        def sec(*stages):
            t = 0.0
            for st in stages:
                try:
                    t += self.timing_get(st)[0] / 1e3
                except SkemaError:
                    pass
            return t

        if self.spd:
            return {"init": {"omega": 0.0},
                    "update": {"omega": sec("update.omega", "update.fused"), "window": sec("update.window"),
                               "daxpy": sec("update.daxpy")},
                    "approx": {k: 0.0 for k in ("omega", "daxpy", "norm2", "update", "dpotrf", "dgels", "dgesvd")}}
        return {"init": {k: 0.0 for k in ("upsilon", "omega", "phi", "psi")},
                "update": {"upsilon": sec("update.upsilon", "update.entries"),
                           "omega": sec("update.omega", "update.fused"), "phi": sec("update.phi"),
                           "psi": sec("update.psi"), "window": sec("update.window"), "daxpy": sec("update.daxpy")},
                "approx": {"phi": 0.0, "psi": 0.0, "dgeqrf": sec("approx.orth"), "dgels": sec("approx.core"),
                           "dgesvd": sec("approx.svd"), "dgemm": sec("approx.vectors")}}

    def linear_update(self, A):
        """SketchySVD::linear_update: zero the sketches, then stream all rows.
        With AlgParams.sketch_compute_svals_iters (and more than one window)
        the rows go one window at a time and the top-rank singular values
        after each window are kept as self.traces[str(w)]["svals"]
        (src/Skema_SketchySVD.cpp:164-216); the approximation here does not
        overwrite Y, so the later windows see the true sketch.
        With AlgParams.debug_filename the sketches are written after every
        window (<stem>_X.txt.<w>, _Y.txt.<w>, _Z.txt.<w>) and at the end
        (<stem>_X.txt, ...), as src/Skema_SketchySVD.cpp:191-205, 235-245
        write them; SketchySPD writes <stem>_Y.txt at the end only
        (src/Skema_SketchySVD.cpp:880-885). A single window of all rows
        writes none, as the reference returns before its dumps."""
        self.reset()
        self.traces = {}
        W = int(self.alg.window)
        stem = self.debug_stem()
        iters = bool(getattr(self.alg, "sketch_compute_svals_iters", False)) and not self.spd
        if W >= self.nrow:
            self.update_rows(A, 0, None)
            return
        if self.spd or not (iters or stem):
            self.update_rows(A, 0, None)
        else:
            for w, r0 in enumerate(range(0, self.nrow, W)):
                wr = min(W, self.nrow - r0)
                if self.alg.kernel_func == L.KERNEL_GAUSSRBF:
                    self.update_rows(A, r0, wr)
                else:
                    self.update_rows(_row_block(A, r0, wr), r0, wr)
                if stem:
                    self.dump_sketches(stem, f".{w}")
                if iters:
                    S = self.low_rank_approx()[1]
                    self.traces[str(w)] = {"svals": [float(x) for x in S]}
        if stem:
            self.dump_sketches(stem)

    def synchronize(self):
        self._check(self.lib.skema_synchronize(self.h))

    def launch_count(self) -> int:
        return int(self.lib.skema_launch_count(self.h))

    def timing_enable(self, on: bool = True):
        self._check(self.lib.skema_timing_enable(self.h, 1 if on else 0))

    def timing_get(self, stage: str):
        """(milliseconds, launches) accumulated for one stage."""
        ms, n = C.c_double(), C.c_int64()
        self._check(self.lib.skema_timing_get(self.h, stage.encode(), C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def set_stream(self, stream_handle: int | None):
        """Launch on an external cudaStream_t (e.g. torch's current stream).
        The stream must outlive every tensor this context has read or
        written while it was set; None returns to the context's default."""
        self._check(self.lib.skema_set_stream(self.h, stream_handle))
        self._user_stream = stream_handle or None

    # -- ordering against torch's stream ----------------------------------
    # The library launches on the context's stream (skema_get_stream). Unless
    # that is torch's current stream, a call that reads device tensors first
    # waits on the device for torch's current stream (the tensors' data are
    # complete), and the tensors are recorded on the library's stream, so
    # that torch's caching allocator reuses their memory only after the
    # library's work on them is done. A call that writes device tensors makes
    # torch's current stream wait for the library's.
    #
    # torch's allocator records an event on every recorded stream when such
    # a tensor is freed, which may be after this context is destroyed. The
    # stream the context creates for itself dies with it, so before the
    # first call on torch tensors the context is moved onto a stream from
    # torch's pool, which lives as long as the process.
    def _lib_stream(self, device):
        import torch

        if getattr(self, "_user_stream", None) is None:
            ts = getattr(self, "_torch_stream", None)
            if ts is None or ts.device != device:
                ts = torch.cuda.Stream(device=device)
                self._check(self.lib.skema_set_stream(self.h, ts.cuda_stream))
                self._torch_stream = ts
            return ts
        h = C.c_void_p()
        self._check(self.lib.skema_get_stream(self.h, C.byref(h)))
        return torch.cuda.ExternalStream(h.value or 0, device=device)

    def _cuda_tensors(self, tensors):
        return [t for t in tensors if _is_torch(t) and t.is_cuda]

    def _torch_inputs_ready(self, *tensors):
        import torch

        ts = self._cuda_tensors(tensors)
        if not ts:
            return
        lib_s, cur = self._lib_stream(ts[0].device), torch.cuda.current_stream(ts[0].device)
        if lib_s.cuda_stream == cur.cuda_stream:
            return
        lib_s.wait_stream(cur)
        for t in ts:
            t.record_stream(lib_s)

    def _torch_outputs_ready(self, *tensors):
        import torch

        ts = self._cuda_tensors(tensors)
        if not ts:
            return
        lib_s, cur = self._lib_stream(ts[0].device), torch.cuda.current_stream(ts[0].device)
        if lib_s.cuda_stream == cur.cuda_stream:
            return
        cur.wait_stream(lib_s)
        for t in ts:
            t.record_stream(lib_s)

    # -- sketches ---------------------------------------------------------
    def _sketch_shape(self, which):
        return {L.SKETCH_X: (self.range, self.ncol), L.SKETCH_Y: (self.nrow, self.range),
                L.SKETCH_Z: (self.core, self.core)}[which]

    def get_sketch(self, which, out=None):
        shape = self._sketch_shape(which)
        if out is None:
            out = np.empty(shape, dtype=np.float32)
        if _is_torch(out):
            self._torch_inputs_ready(out)
            self._check(self.lib.skema_get_sketch(self.h, which, out.data_ptr(), shape[1], L.ROW_MAJOR, L.MEM_DEVICE))
            self._torch_outputs_ready(out)
        else:
            self._check(self.lib.skema_get_sketch(self.h, which, out.ctypes.data, shape[1], L.ROW_MAJOR, L.MEM_HOST))
        return out

    def set_sketch(self, which, buf):
        shape = self._sketch_shape(which)
        if _is_torch(buf):
            self._torch_inputs_ready(buf)
            self._check(self.lib.skema_set_sketch(self.h, which, buf.data_ptr(), shape[1], L.ROW_MAJOR, L.MEM_DEVICE))
        else:
            b = np.ascontiguousarray(buf, dtype=np.float32)
            assert b.shape == shape
            self._check(self.lib.skema_set_sketch(self.h, which, b.ctypes.data, shape[1], L.ROW_MAJOR, L.MEM_HOST))

    # -- maps -------------------------------------------------------------
    def map_info(self, which):
        nr, nc, z, t = C.c_int64(), C.c_int64(), C.c_int32(), C.c_int32()
        self._check(self.lib.skema_map_info(self.h, which, C.byref(nr), C.byref(nc), C.byref(z), C.byref(t)))
        return nr.value, nc.value, z.value, bool(t.value)

    def map_export(self, which):
        """Gauss: (nrow x ncol float64 array, None); SparseSign: (values, indices)
        with zeta entries per stored row."""
        nr, nc, z, _ = self.map_info(which)
        if z == 0:
            vals = np.empty((nc, nr), dtype=np.float64)  # column-major storage
            self._check(self.lib.skema_map_export(self.h, which, vals.ctypes.data, None))
            return vals.T, None
        vals = np.empty((nr, z), dtype=np.float64)
        idx = np.empty((nr, z), dtype=np.int32)
        self._check(self.lib.skema_map_export(self.h, which, vals.ctypes.data, idx.ctypes.data))
        return vals, idx

    def map_export_reference_dumps(self, stem):
        """Write the maps as the reference's --debug-file dumps
        <stem>_{Upsilon,Omega,Phi,Psi}.{txt,mtx} (SketchySPD: Omega), in this
        context's stored orientation (write_reference_map_dump); the files
        read back with map_import_reference_dumps."""
        for which, label in MAP_LABELS.items():
            if self.spd and which != L.OMEGA:
                continue
            _, nc, z, _ = self.map_info(which)
            vals, idx = self.map_export(which)
            write_reference_map_dump(f"{stem}_{label}.mtx" if z else f"{stem}_{label}.txt", vals, idx, nc)

    def map_import_reference_dumps(self, stem):
        """Import the four maps from the reference's --debug-file dumps
        <stem>_{Upsilon,Omega,Phi,Psi}.{txt,mtx} (one map for SketchySPD:
        Omega), read by read_reference_map_dump in this context's stored
        orientation."""
        import os

        for which, label in MAP_LABELS.items():
            if self.spd and which != L.OMEGA:
                continue
            nr, nc, z, _ = self.map_info(which)
            path = f"{stem}_{label}.mtx" if z else f"{stem}_{label}.txt"
            if not os.path.exists(path):
                raise FileNotFoundError(path)
            vals, idx = read_reference_map_dump(path, nr, nc)
            self.map_import(which, vals, idx)

    def map_import(self, which, values, indices=None):
        nr, nc, z, _ = self.map_info(which)
        if z == 0:
            v = np.asfortranarray(np.asarray(values, dtype=np.float64))
            assert v.shape == (nr, nc)
            self._check(self.lib.skema_map_import(self.h, which, v.ctypes.data, None))
        else:
            v = np.ascontiguousarray(values, dtype=np.float64).reshape(nr, z)
            ix = np.ascontiguousarray(indices, dtype=np.int32).reshape(nr, z)
            self._check(self.lib.skema_map_import(self.h, which, v.ctypes.data, ix.ctypes.data))


class SketchySVD(_Context):
    """SketchySVD<MatrixType, DimReduxT> (src/Skema_SketchySVD.hpp:11-64)."""

    def get_sketches(self):
        return (self.get_sketch(L.SKETCH_X), self.get_sketch(L.SKETCH_Y), self.get_sketch(L.SKETCH_Z))

    def low_rank_approx(self, device_out=None):
        """(U m x r, S r, V n x r), FP64. device_out: optional (U, S, V) CUDA
        float64 tensors (column-major U, V) to fill in place."""
        r = self.rank
        if device_out is not None:
            U, S, V = device_out
            self._torch_inputs_ready(U, S, V)
            self._check(self.lib.skema_low_rank_approx(self.h, U.data_ptr(), S.data_ptr(), V.data_ptr(), L.MEM_DEVICE))
            self._torch_outputs_ready(U, S, V)
            return U, S, V
        U = np.empty((r, self.nrow), dtype=np.float64)
        V = np.empty((r, self.ncol), dtype=np.float64)
        S = np.empty(r, dtype=np.float64)
        self._check(self.lib.skema_low_rank_approx(self.h, U.ctypes.data, S.ctypes.data, V.ctypes.data, L.MEM_HOST))
        self.uvecs, self.svals, self.vvecs = U.T, S, V.T
        return U.T, S, V.T

    def low_rank_approx_rows(self, row0: int, nrows: int, allreduce):
        """low_rank_approx of a sketch sharded by row blocks
        (skema_low_rank_approx_rows): this context holds Y's rows [row0,
        row0 + nrows) and X, Z summed over the ranks. allreduce(ptr, count)
        sums count FP64 values at the device pointer ptr over the ranks in
        place (it is called three times, in the same order on every rank).
        Returns (U rows of the block, S, V) as numpy arrays."""
        err = []

        def cb(ptr, count, _user):
            try:
                allreduce(int(ptr), int(count))
                return 0
            except BaseException as e:  # reported as SKEMA_ECOLLECTIVE
                err.append(e)
                return 1

        fn = L.ALLREDUCE_FN(cb)
        r = self.rank
        U = np.empty((r, max(nrows, 0)), dtype=np.float64)
        V = np.empty((r, self.ncol), dtype=np.float64)
        S = np.empty(r, dtype=np.float64)
        st = self.lib.skema_low_rank_approx_rows(self.h, int(row0), int(nrows), C.cast(fn, C.c_void_p), None,
                                                 U.ctypes.data, S.ctypes.data, V.ctypes.data, L.MEM_HOST)
        if st != L.OK and err:
            raise SkemaError(st, f"all-reduce callback: {err[0]!r}") from err[0]
        self._check(st)
        return U.T, S, V.T


class SketchySPD(_Context):
    """SketchySPD<MatrixType, DimReduxT> (src/Skema_SketchySVD.hpp:67-108)."""

    def get_sketches(self):
        return self.get_sketch(L.SKETCH_Y)

    def low_rank_approx(self, device_out=None):
        """SketchySPD::low_rank_approx (src/Skema_SketchySVD.cpp:935-1151):
        (U m x r eigenvectors, S r eigenvalues), FP64, as chosen by
        AlgParams.spd_approx. device_out: optional (U, S) CUDA float64
        tensors (column-major U) to fill in place."""
        r = self.rank
        if device_out is not None:
            U, S = device_out
            self._torch_inputs_ready(U, S)
            self._check(self.lib.skema_low_rank_approx(self.h, U.data_ptr(), S.data_ptr(), None, L.MEM_DEVICE))
            self._torch_outputs_ready(U, S)
            return U, S
        U = np.empty((r, self.nrow), dtype=np.float64)
        S = np.empty(r, dtype=np.float64)
        self._check(self.lib.skema_low_rank_approx(self.h, U.ctypes.data, S.ctypes.data, None, L.MEM_HOST))
        self.uvecs, self.svals, self.vvecs = U.T, S, None
        return U.T, S

    def compute_residuals(self, A):
        """SketchySPD::compute_residuals (src/Skema_SketchySVD.cpp:1206-1213):
        ||(A U - U S)(:, j)||_2 for the last low_rank_approx."""
        if getattr(self, "uvecs", None) is None:
            raise SkemaError(L.ESTATE, "compute_residuals needs a low_rank_approx first")
        try:  # the factors kept on the device
            self.rnrms = self.residuals(A, None, None, None)
        except SkemaError as e:  # replaced by factors passed to residuals() since
            if e.status != L.ESTATE:
                raise
            self.rnrms = self.residuals(A, None, self.svals, self.uvecs)
        return self.rnrms


def read_matrix(path, sparse: bool | None = None):
    """Skema::read_matrix (src/Skema_IO.hpp:13-21) through the library's
    readers: a .bin file or (sparse=True) a MatrixMarket coordinate file
    gives a scipy CSR matrix (FP64, rows sorted, duplicates summed); a
    MatrixMarket array file gives a dense FP64 numpy array. sparse=None
    decides from the file (.bin, or a .mtx whose banner says coordinate)."""
    import scipy.sparse as sp

    lib = L.load()
    p = str(path)
    if sparse is None:
        if p.lower().endswith(".mtx"):
            with open(p, "rb") as f:
                sparse = b"coordinate" in f.readline().lower()
        else:
            sparse = True
    if sparse:
        a = L.Crs()
        st = lib.skema_read_crs(p.encode(), C.byref(a))
        if st != L.OK:
            raise SkemaError(st, lib.skema_last_error(None).decode())
        try:
            nr, nc, nnz = a.nrow, a.ncol, a.nnz
            rp = np.ctypeslib.as_array(a.rowptr, shape=(nr + 1,)).copy()
            col = np.ctypeslib.as_array(a.col, shape=(nnz,)).copy() if nnz else np.zeros(0, np.int32)
            val = np.ctypeslib.as_array(a.val, shape=(nnz,)).copy() if nnz else np.zeros(0)
        finally:
            lib.skema_crs_free(C.byref(a))
        return sp.csr_matrix((val, col, rp), shape=(nr, nc))
    d = L.Dense()
    st = lib.skema_read_dense(p.encode(), C.byref(d))
    if st != L.OK:
        raise SkemaError(st, lib.skema_last_error(None).decode())
    try:
        out = np.ctypeslib.as_array(d.data, shape=(d.ncol * d.nrow,)).reshape(d.ncol, d.nrow).T.copy() \
            if d.nrow * d.ncol else np.zeros((d.nrow, d.ncol))
    finally:
        lib.skema_dense_free(C.byref(d))
    return out


MAP_LABELS = {L.UPSILON: "Upsilon", L.OMEGA: "Omega", L.PHI: "Phi", L.PSI: "Psi"}


def write_dense_text(path, M):
    """Impl::write of a matrix or a vector (src/Skema_Common.hpp:164-184):
    a matrix as one line per row, each entry "%.16f " ; a vector as one
    "%.16f" value per line."""
    a = np.asarray(M, dtype=np.float64)
    with open(str(path), "w") as f:
        if a.ndim == 1:
            np.savetxt(f, a, fmt="%.16f", newline="\n")
        else:
            np.savetxt(f, a, fmt="%.16f", delimiter=" ", newline=" \n")


def write_reference_map_dump(path, values, indices=None, ncol=None):
    """A map in the reference's --debug-file dump formats (the writer side of
    read_reference_map_dump): Gauss values (nrow x ncol) as text lines of
    write_dense_text; SparseSign (values, indices), zeta entries per stored
    row, as a MatrixMarket coordinate file with 1-based indices, the entries
    of a row in stored order (repeated columns kept), ncol columns."""
    if indices is None:
        write_dense_text(path, values)
        return
    v = np.asarray(values, dtype=np.float64)
    ix = np.asarray(indices, dtype=np.int64)
    nr, z = v.shape
    if ncol is None:
        ncol = int(ix.max()) + 1 if ix.size else 0
    rows = np.repeat(np.arange(1, nr + 1, dtype=np.int64), z)
    with open(str(path), "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n")
        f.write(f"{nr} {int(ncol)} {nr * z}\n")
        for r, c, x in zip(rows.tolist(), (ix.reshape(-1) + 1).tolist(), v.reshape(-1).tolist()):
            f.write(f"{r} {c} {x:.17g}\n")


def read_reference_map_dump(path, nrow: int, ncol: int):
    """A map written by the reference's --debug-file dumps
    (src/Skema_DimRedux.hpp:124-127, 264-267; formats of Impl::write,
    src/Skema_Common.hpp:175-190), in its stored orientation nrow x ncol:
      <stem>_<label>.txt  GaussDimRedux: nrow lines of ncol values;
      <stem>_<label>.mtx  SparseSignDimRedux: a MatrixMarket coordinate file
                          (1-based), zeta entries per row kept as stored
                          (repeated columns are not merged).
    Returns (values, None) for Gauss (nrow x ncol float64) and
    (values, indices) (nrow x zeta) for SparseSign, the map_import forms."""
    p = str(path)
    if p.lower().endswith(".txt"):
        vals = np.loadtxt(p, dtype=np.float64, ndmin=2)
        if vals.shape != (nrow, ncol):
            raise ValueError(f"{p}: {vals.shape} values, the map is {nrow} x {ncol}")
        return vals, None
    rows, cols, vs = [], [], []
    with open(p) as f:
        header = f.readline().lower()
        if "coordinate" not in header:
            raise ValueError(f"{p}: not a MatrixMarket coordinate file")
        line = f.readline()
        while line.startswith("%") or not line.strip():
            line = f.readline()
        nr, nc, nnz = (int(t) for t in line.split()[:3])
        if (nr, nc) != (nrow, ncol):
            raise ValueError(f"{p}: {nr} x {nc}, the map is {nrow} x {ncol}")
        for line in f:
            t = line.split()
            if not t or t[0].startswith("%"):
                continue
            rows.append(int(t[0]) - 1)
            cols.append(int(t[1]) - 1)
            vs.append(float(t[2]) if len(t) > 2 else 1.0)
    if len(rows) != nnz or nnz % max(nrow, 1):
        raise ValueError(f"{p}: {len(rows)} entries, not the same count in every one of {nrow} rows")
    zeta = nnz // nrow
    order = np.argsort(np.asarray(rows), kind="stable")  # rows in file order within each row
    r = np.asarray(rows)[order]
    if np.any(r != np.repeat(np.arange(nrow), zeta)):
        raise ValueError(f"{p}: rows do not all hold {zeta} entries")
    idx = np.asarray(cols, dtype=np.int32)[order].reshape(nrow, zeta)
    val = np.asarray(vs, dtype=np.float64)[order].reshape(nrow, zeta)
    return val, idx


def read_crs_rows(path, row0: int = 0, nrows: int = -1):
    """Rows [row0, row0 + nrows) of a binary CRS file as a scipy CSR matrix
    (FP64; entries of a row in file order), read without the rest of the
    file (skema_read_crs_rows). nrows < 0 reads to the last row."""
    import scipy.sparse as sp

    lib = L.load()
    a = L.Crs()
    st = lib.skema_read_crs_rows(str(path).encode(), int(row0), int(nrows), C.byref(a))
    if st != L.OK:
        raise SkemaError(st, lib.skema_last_error(None).decode())
    try:
        nr, nc, nnz = a.nrow, a.ncol, a.nnz
        rp = np.ctypeslib.as_array(a.rowptr, shape=(nr + 1,)).copy()
        col = np.ctypeslib.as_array(a.col, shape=(nnz,)).copy() if nnz else np.zeros(0, np.int32)
        val = np.ctypeslib.as_array(a.val, shape=(nnz,)).copy() if nnz else np.zeros(0)
    finally:
        lib.skema_crs_free(C.byref(a))
    return sp.csr_matrix((val, col, rp), shape=(nr, nc))


def write_matrix(A, path):
    """Skema::write_matrix for CRS input (src/Skema_IO.cpp:88-104): a scipy
    sparse matrix to .mtx (coordinate real general) or .bin."""
    import scipy.sparse as sp

    lib = L.load()
    A = sp.csr_matrix(A)
    A.sort_indices()
    rp = np.ascontiguousarray(A.indptr, dtype=np.int64)
    col = np.ascontiguousarray(A.indices, dtype=np.int32)
    val = np.ascontiguousarray(A.data, dtype=np.float64)
    a = L.Crs(A.shape[0], A.shape[1], A.nnz, rp.ctypes.data_as(C.POINTER(C.c_int64)),
              col.ctypes.data_as(C.POINTER(C.c_int32)), val.ctypes.data_as(C.POINTER(C.c_double)))
    st = lib.skema_write_crs(str(path).encode(), C.byref(a))
    if st != L.OK:
        raise SkemaError(st, lib.skema_last_error(None).decode())


def write_history(path, svals, rnrms, update_seconds=None, traces=None, timings=None):
    """The JSON of SketchySVD::save_history (src/Skema_SketchySVD.cpp:730-755):
    {"rnrms": [...], "svals": [...], "timings": {approx, init, update},
    "traces": {...}}, keys sorted and a 4-space indent as the reference's JSON
    writer prints them. timings: the nested dict to write; by default the
    reference's SketchySVD keys (src/Skema_SketchySVD.cpp:101-116), zero
    except the update times given in update_seconds. Written to `path`
    (with a newline) unless path is None; the text is returned."""
    import json

    if timings is None:
        upd = {k: 0.0 for k in ("upsilon", "omega", "phi", "psi", "window", "daxpy")}
        upd.update(update_seconds or {})
        timings = {"init": {k: 0.0 for k in ("upsilon", "omega", "phi", "psi")}, "update": upd,
                   "approx": {k: 0.0 for k in ("phi", "psi", "dgeqrf", "dgemm", "dgels", "dgesvd")}}
    hist = {"timings": timings, "traces": dict(traces or {}), "svals": [float(x) for x in svals],
            "rnrms": [float(x) for x in rnrms]}
    text = json.dumps(hist, indent=4, sort_keys=True)
    if path is not None:
        with open(path, "w") as f:
            f.write(text + "\n")
    return text


def sketchysvd(matrix, alg: AlgParams):
    """Skema::sketchysvd (src/Skema_SketchySVD.cpp:1244-1405, 1408-1577):
    update, fixed-rank approximation, residuals and (with history_filename)
    the history file. Returns (U, S, V); the SketchySPD branch (issymmetric
    without force_three_sketch) returns (U, S, None), S the eigenvalues."""
    spd = bool(alg.issymmetric) and not bool(alg.force_three_sketch)
    with (SketchySPD if spd else SketchySVD)(alg) as sk:
        sk.linear_update(matrix)
        if spd:
            U, S = sk.low_rank_approx()
            V = None
        else:
            U, S, V = sk.low_rank_approx()
        sk.compute_residuals(matrix)
        if getattr(alg, "history_filename", ""):
            sk.save_history(alg.history_filename)
        stem = sk.debug_stem()
        if stem:  # src/Skema_SketchySVD.cpp:1386-1404, 1559-1576
            for name, M in (("U", U), ("S", S), ("V", V)):
                if M is not None and np.asarray(M).size:
                    write_dense_text(f"{stem}_{name}.txt", M)
        return U, S, V


def _ctx_for_standalone(device: int = 0, precision: int = L.PREC_FP32) -> _Context:
    alg = AlgParams(matrix_m=1, matrix_n=1, rank=1, device=device, precision=precision)
    return _Context(alg)


def rbf_sketch_fwd(pts, gamma: float, omega, ctx: _Context | None = None, precision: int = L.PREC_FP32):
    """Y = K Omega^T for device tensors pts (N x d), omega (k x N).
    precision (used when no ctx is given): PREC_BF16 takes the tensor-core
    form for d <= 64 and k <= 192 (kernel tiles from BF16 points, FP32
    accumulation), PREC_FP32 the FP32 form."""
    import torch

    own = ctx is None
    ctx = ctx or _ctx_for_standalone(pts.device.index or 0, precision)
    try:
        pts = pts.contiguous()
        omega = omega.contiguous()
        N, d = pts.shape
        k = omega.shape[0]
        Y = torch.empty((N, k), dtype=torch.float32, device=pts.device)
        ctx._torch_inputs_ready(pts, omega, Y)
        ctx._check(ctx.lib.skema_rbf_sketch_fwd(ctx.h, pts.data_ptr(), N, d, float(gamma), omega.data_ptr(), k, Y.data_ptr()))
        ctx.synchronize()
        return Y
    finally:
        if own:
            ctx.close()


def rbf_sketch_vjp(pts, gamma: float, omega, Ybar, ctx: _Context | None = None, precision: int = L.PREC_FP32):
    """(dL/dpts, dL/dgamma) of Y = K Omega^T given Ybar = dL/dY; precision
    as for rbf_sketch_fwd."""
    import torch

    own = ctx is None
    ctx = ctx or _ctx_for_standalone(pts.device.index or 0, precision)
    try:
        pts = pts.contiguous()
        omega = omega.contiguous()
        Ybar = Ybar.contiguous()
        N, d = pts.shape
        k = omega.shape[0]
        dX = torch.empty_like(pts)
        dg = torch.zeros(1, dtype=torch.float64, device=pts.device)
        ctx._torch_inputs_ready(pts, omega, Ybar, dg)
        ctx._check(ctx.lib.skema_rbf_sketch_vjp(ctx.h, pts.data_ptr(), N, d, float(gamma), omega.data_ptr(), k,
                                                Ybar.data_ptr(), dX.data_ptr(), dg.data_ptr()))
        ctx.synchronize()
        return dX, float(dg.item())
    finally:
        if own:
            ctx.close()
