"""Benchmark of the SketchySVD sketch update on B200 (one JSON line).

Default workload (sparse-sign CSR): A is CSR 1,000,000 x 100,000 FP32 with
~10 nonzeros per row at uniform random columns (duplicates merged), values
N(0,1) plus a planted rank-20 component of scale 5 sampled on the pattern;
SparseSign maps (zeta = 8), r = 20, k = 81, s = 163, windows of 10,000 rows.
One step = skema_reset + the linear update over all rows (all windows), the
inputs resident in HBM. Synthetic data, seeded.

Other workloads (--workload): dense-fp32 / dense-bf16 / dense-fp8 (A
200,000 x 20,000 FP32, r = 50, k = 201, s = 403, windows of 8,192 rows);
rbf-bf16 / rbf-fp32 (Gauss-RBF kernel of 100,000 points in 128 dimensions,
r = 64, k = 257, s = 515, windows of 4,096 rows; one step sketches all
100,000 kernel rows, the kernel's rows split over the ranks).

Parity (outside every timed region): the headline line carries `parity`,
the device's X, Y, Z of one step against the FP64 oracle over every row of
the same CSR matrix and maps (the CPU-baseline leg runs that oracle), and
every dense / kernel line carries `accuracy`, its top-r singular values
against FP64 SketchySVD on the same input and the context's own maps (FP64
device products, the oracle's approximation), or for the adjoint pair the
FP64 gradient and central finite differences of the FP64 forward.

On one GPU the default run also measures the other configurations after
the headline and reports them under `secondary`: the dense Gaussian case in
the plain FP32 form and the BF16 / FP8 forms, the RBF kernel case in FP32
and BF16, and the forward / adjoint pair in FP32 and BF16, each with its
roofline and accuracy, and the speed-ups of the precision forms over the
plain form (--no-secondary skips them).

Multi-GPU (torchrun, one rank per GPU): weak scaling by contiguous row
blocks; each rank sketches its own block of the global matrix and the
partial X and Z sketches are summed with an NCCL all-reduce (Y rows are
disjoint and stay on their rank).

--impl reference times the CPU oracle (the FP64 restatement of the
reference's algorithm) on the host cores on a bounded sample per step.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")
TRAFFIC_PATH = os.path.join(ROOT, "profiles", "traffic.json")
FALLBACK_PEAKS = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}
STAGES = ("update.omega", "update.psi", "update.upsilon", "update.phi", "update.entries",
          "update.window", "update.fused", "update.daxpy")

WORKLOADS = {
    "csr-sparse-sign": dict(m=1_000_000, n=100_000, nnz_row=10, planted=20, scale=5.0, rank=20,
                            k=81, s=163, window=10_000, seed=2, kind=1),
    "dense-fp32": dict(m=200_000, n=20_000, rank=50, k=201, s=403, window=8192, seed=3, kind=0, prec=0),
    "dense-bf16": dict(m=200_000, n=20_000, rank=50, k=201, s=403, window=8192, seed=3, kind=0, prec=1),
    "dense-fp8": dict(m=200_000, n=20_000, rank=50, k=201, s=403, window=8192, seed=3, kind=0, prec=2),
    # Gauss-RBF kernel input: 100,000 points in 128 dimensions; K (100,000^2)
    # is regenerated tile by tile inside the sketch kernels (BF16 form) or
    # materialised one 4,096-row window at a time (FP32 form)
    "rbf-bf16": dict(m=100_000, n=100_000, d=128, rank=64, k=257, s=515, window=4096, seed=4, kind=0, prec=1,
                     rbf=True),
    "rbf-fp32": dict(m=100_000, n=100_000, d=128, rank=64, k=257, s=515, window=4096, seed=4, kind=0, prec=0,
                     rbf=True),
    # the kernel-sketch forward / adjoint pair: 50,000 points in 64 dimensions
    # (same mixture recipe), Omega k = 129; one step = forward + VJP
    "rbf-vjp": dict(m=50_000, n=50_000, d=64, rank=32, k=129, s=259, window=50_000, seed=1, kind=0, vjp=True),
    "rbf-vjp-bf16": dict(m=50_000, n=50_000, d=64, rank=32, k=129, s=259, window=50_000, seed=1, kind=0, vjp=True,
                         prec=1),
}


def load_peaks():
    try:
        with open(PEAKS_PATH) as f:
            p = json.load(f)
        return p, "measured"
    except Exception:
        return dict(FALLBACK_PEAKS), "fallback"


# ------------------------------------------------------------- clocks ------
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.out = None

    def __enter__(self):
        try:
            self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.proc or not self.out:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.out.flush()
        rows = []
        with open(self.out.name) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.out.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------- synthetic ------
def make_csr_numpy(cfg, m_local, seed):
    """Seeded CSR block (numpy RNG): rowptr int64, col int32, val float32."""
    rng = np.random.default_rng(seed)
    n, nr = cfg["n"], cfg["nnz_row"]
    cols = rng.integers(0, n, size=(m_local, nr))
    cols.sort(axis=1)
    keep = np.ones_like(cols, bool)
    keep[:, 1:] = cols[:, 1:] != cols[:, :-1]
    counts = keep.sum(1)
    rowptr = np.zeros(m_local + 1, np.int64)
    rowptr[1:] = np.cumsum(counts)
    col = cols[keep].astype(np.int32)
    p = cfg["planted"]
    U = rng.standard_normal((m_local, p), dtype=np.float32)
    V = rng.standard_normal((n, p), dtype=np.float32)
    rows = np.repeat(np.arange(m_local), counts)
    val = rng.standard_normal(col.size, dtype=np.float32) + cfg["scale"] * (U[rows] * V[col]).sum(1) / np.sqrt(p)
    return rowptr, col, val.astype(np.float32)


def make_dense_torch(cfg, m_local, seed, device):
    """A = U_p diag(s) V_p^T + 1e-3 N(0,1), s_i = i^-1.5, p = 256 (FP32, column-major)."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(seed)
    m, n, p = m_local, cfg["n"], 256
    Ug = torch.randn(m, p, generator=g, device=device, dtype=torch.float64)
    Vg = torch.randn(n, p, generator=g, device=device, dtype=torch.float64)
    Uq = torch.linalg.qr(Ug)[0]
    Vq = torch.linalg.qr(Vg)[0]
    s = torch.arange(1, p + 1, device=device, dtype=torch.float64) ** -1.5
    Af = torch.empty((n, m), dtype=torch.float32, device=device)  # A^T row-major = A column-major
    blk = 2048
    for j0 in range(0, n, blk):
        j1 = min(n, j0 + blk)
        Af[j0:j1] = ((Vq[j0:j1] * s) @ Uq.T).float()
    del Ug, Vg, Uq, Vq
    Af += 1e-3 * torch.randn(Af.shape, generator=g, device=device)
    return Af.t()  # m x n view, column-major


def make_points_torch(cfg, n_pts, seed, device):
    """8-component Gaussian mixture in d dimensions: means ~ N(0, 4I), unit
    covariance, equal weights (FP32, row-major n_pts x d); and gamma =
    1 / (2 * median squared pairwise distance of a 1,000-point subsample)."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(seed)
    d = cfg["d"]
    means = 2.0 * torch.randn(8, d, generator=g, device=device)
    lab = torch.randint(0, 8, (n_pts,), generator=g, device=device)
    P = means[lab] + torch.randn(n_pts, d, generator=g, device=device)
    sub = P[torch.randperm(n_pts, generator=g, device=device)[:1000]].double()
    d2 = torch.cdist(sub, sub).pow(2)
    iu = torch.triu_indices(1000, 1000, 1, device=device)
    gamma = 1.0 / (2.0 * float(d2[iu[0], iu[1]].median()))
    return P.contiguous(), gamma


# ------------------------------------------------------------ our arm ------
def run_vjp(args, cfg, peaks, peak_kind):
    """Forward Y = K Omega^T and the VJP w.r.t. gamma and the points through
    the C ABI on device buffers; the cotangent is fixed (2 Y of the first
    forward, i.e. L = ||Y||_F^2). Ranks under torchrun run replicas."""
    import torch
    import torch.distributed as dist

    import skema_b200._lib as L
    from skema_b200.sketchy import _ctx_for_standalone

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    N, d, k = cfg["m"], cfg["d"], cfg["k"]
    P, gamma = make_points_torch(cfg, N, cfg["seed"], dev)
    g = torch.Generator(device=dev)
    g.manual_seed(5)
    Om = (2.0 * torch.rand(k, N, generator=g, device=dev) - 1.0).contiguous()
    Y = torch.empty((N, k), dtype=torch.float32, device=dev)
    dX = torch.empty_like(P)
    dg = torch.zeros(1, dtype=torch.float64, device=dev)
    prec = cfg.get("prec", 0)
    ctx = _ctx_for_standalone(local, prec)
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    lib, h = ctx.lib, ctx.h
    ctx._check(lib.skema_rbf_sketch_fwd(h, P.data_ptr(), N, d, gamma, Om.data_ptr(), k, Y.data_ptr()))
    Ybar = (2.0 * Y).contiguous()
    torch.cuda.synchronize()

    def step():
        ctx._check(lib.skema_rbf_sketch_fwd(h, P.data_ptr(), N, d, gamma, Om.data_ptr(), k, Y.data_ptr()))
        ctx._check(lib.skema_rbf_sketch_vjp(h, P.data_ptr(), N, d, gamma, Om.data_ptr(), k, Ybar.data_ptr(),
                                            dX.data_ptr(), dg.data_ptr()))

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        t0 = time.perf_counter()
        while time.perf_counter() - t0 < args.clock_lead:
            step()
            torch.cuda.synchronize()
        l0 = ctx.launch_count()
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
        launches = ctx.launch_count() - l0
        t0 = time.perf_counter()
        while time.perf_counter() - t0 < args.clock_tail:
            step()
            torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    ms_t = torch.tensor([ms], device=dev)
    if world > 1:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms = float(ms_t.item())
    # forward 2N^2(d + k) (Gram tiles + the sketch), VJP 2N^2(k + 2d) (M = Ybar Omega,
    # E X and E^T X) plus recomputed Gram tiles 2N^2 d
    flops = 2.0 * N * N * (d + k) + 2.0 * N * N * (k + 3 * d)
    if prec == 1:
        # tensor-core form: the forward is one rbf_sketch_kernel launch, the
        # adjoint two rbf_vjp_kernel passes, each with its own Gram tiles
        # (2 N^2 (d + k + d) per pass: S, M and E X); the roofline is taken
        # over the whole step against the sustained BF16 peak
        flops = 2.0 * N * N * (d + k) + 2 * 2.0 * N * N * (2 * d + k)
        pk = peaks["bf16_tflops_sustained"]
        roof = {"bound": "tensor", "achieved": flops / (ms / 1e3) / 1e12, "peak": pk, "unit": "TFLOP/s",
                "frac": flops / (ms / 1e3) / 1e12 / pk,
                "peak_source": f"bf16_tflops_sustained ({peak_kind})",
                "kernel": "rbf_sketch_kernel (forward) + 2 x rbf_vjp_kernel (adjoint)", "kernel_ms": ms,
                "algorithmic_flops_per_step": flops, "traffic": None}
    else:
        roof = {"bound": "fp32-simt", "achieved": flops / (ms / 1e3) / 1e12, "peak": 74.4, "unit": "TFLOP/s",
                "frac": flops / (ms / 1e3) / 1e12 / 74.4,
                "peak_source": "nominal FP32 SIMT (148 SMs x 128 FMA/clk x 2 x 1.965 GHz)",
                "kernel": "sgemm_kernel + rbf_tile_kernel (forward and adjoint)", "kernel_ms": ms,
                "algorithmic_flops_per_step": flops, "traffic": None}
    acc = None
    if rank == 0 and world == 1 and not args.no_accuracy:
        step()
        torch.cuda.synchronize()
        acc = vjp_accuracy(P, gamma, Om, Ybar, dX, float(dg.item()))
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        v, ns, thr = cpu_sample_vjp(cfg)
        cpu = {"value": v, "unit": "rows/s", "cores": thr, "kind": "port",
               "sample": f"forward + VJP of a {ns}-point problem (same d, k) in FP64, scaled by (N/{ns})^2",
               "host_cpu": _cpu_model(), "nproc": os.cpu_count()}
    out = {
        "metric": "sketched rows/s", "value": world * N / (ms / 1e3), "unit": "rows/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "bf16" if prec == 1 else "fp32",
        "data": "synthetic (seeded; no dataset)",
        "config": dict(config_of(args, cfg, world, 0), gamma=gamma),
        "roofline": roof, "cpu_baseline": cpu,
        "e2e": {"value": world * N / (ms / 1e3), "unit": "rows/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0, "note": "device-buffer entry points; same as value"},
        "gpu_launches": launches,
        "clocks": dict(clk.summary(), window="samples span continuous load bracketing the timed steps"),
    }
    if acc is not None:
        out["accuracy"] = acc
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return out if rank == 0 else None


def run_gpu(args, cfg, peaks, peak_kind):
    import torch
    import torch.distributed as dist

    import skema_b200 as sk

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    rbf = bool(cfg.get("rbf"))
    host_csr = None
    from skema_b200.distributed import reduce_partial_sketches, shard_rows

    if rbf:
        # the kernel's rows are sharded over the ranks (every rank holds all
        # points): total work fixed as the rank count grows
        m_glob = cfg["m"]
        row0, m_local = shard_rows(m_glob, world, rank, cfg["window"])
        P, gamma = make_points_torch(cfg, m_glob, cfg["seed"], dev)
        cfg["gamma"] = gamma
    else:
        m_local = cfg["m"]
        m_glob = m_local * world
        row0 = rank * m_local
    a = sk.AlgParams(matrix_m=m_glob, matrix_n=m_glob if rbf else cfg["n"], rank=cfg["rank"],
                     sketch_range=cfg["k"], sketch_core=cfg["s"], window=cfg["window"], dim_redux=cfg["kind"],
                     device=local)
    sparse = args.workload.startswith("csr")
    a.issparse = sparse
    a.precision = cfg.get("prec", 0)
    if rbf:
        a.kernel_func, a.kernel_gamma, a.force_three_sketch = 1, gamma, True
    ctx = sk.SketchySVD(a)
    # one non-default stream for the library's launches and the timing events
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    if rbf:
        nnz = 0
        inp = P
    elif sparse:
        # generated once on the host (numpy) and uploaded: the FP64 oracle of
        # the parity check reads the same matrix
        host_csr = make_csr_numpy(cfg, m_local, cfg["seed"] + rank)
        rowptr, col, val = (torch.from_numpy(x).to(dev) for x in host_csr)
        nnz = col.numel()
        inp = (rowptr, col, val)
    else:
        A = make_dense_torch(cfg, m_local, cfg["seed"] + rank, dev)
        nnz = m_local * cfg["n"]
        inp = A
    torch.cuda.synchronize()
    k, s, n = cfg["k"], cfg["s"], cfg["n"]
    if rbf:
        n = m_glob  # the kernel matrix is points x points (--rows shrinks both)
    Xbuf = torch.empty((k, n), dtype=torch.float32, device=dev) if world > 1 else None
    Zbuf = torch.empty((s, s), dtype=torch.float32, device=dev) if world > 1 else None

    def step():
        ctx.reset()
        ctx.update_rows(inp, row0, m_local)
        if world > 1:
            ctx.get_sketch(0, Xbuf)
            ctx.get_sketch(2, Zbuf)
            reduce_partial_sketches(Xbuf, Zbuf, m_glob, cfg["window"], float(a.sketch_nu))

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    def load_for(seconds):
        # untimed steps of the same work, so the clock samples bracket the
        # timed steps under continuous load (batches of up to 8 short steps)
        t0 = time.perf_counter()
        batch = 1
        while time.perf_counter() - t0 < seconds:
            t1 = time.perf_counter()
            for _ in range(batch):
                step()
            torch.cuda.synchronize()
            batch = 8 if time.perf_counter() - t1 < 0.05 else 1

    with ClockSampler(local) as clk:
        load_for(args.clock_lead)
        l0 = ctx.launch_count()
        ctx.timing_enable(True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
        launches = ctx.launch_count() - l0
        stages, stage_raw = {}, {}
        for name in STAGES:
            sms, scount = ctx.timing_get(name)
            if scount:
                stages[name] = round(sms / args.steps, 4)
                stage_raw[name] = (sms, scount)
        ctx.timing_enable(False)
        load_for(args.clock_tail)
    ms = e0.elapsed_time(e1) / args.steps
    ms_t = torch.tensor([ms], device=dev)
    if world > 1:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms = float(ms_t.item())
    rows_total = m_glob
    value = rows_total / (ms / 1e3)

    # roofline of the dominant kernel, from the stage timers (CUDA events on
    # the launch stream around every launch of the stage, timed steps only)
    try:
        with open(TRAFFIC_PATH) as f:
            traffic_tab = json.load(f).get(args.workload) or {}
    except Exception:
        traffic_tab = {}
    step_flops = m_local * (2 * n * (2 * k + s) + 2 * s * s)
    if rbf:
        step_flops += m_local * 2 * n * cfg["d"]  # the Gram tile of each kernel entry, once
    hbm_peak = peaks["hbm_gbs"]
    tc_peak = peaks.get("bf16_tflops_sustained", 1400.0)

    def hbm_roof(kernel, stage, bytes_per_step):
        sms, cnt = stage_raw[stage]
        per_launch = bytes_per_step * args.steps / cnt
        achieved = per_launch / (sms / cnt / 1e3) / 1e9
        return {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                "frac": achieved / hbm_peak, "peak_source": peak_kind, "kernel": kernel,
                "kernel_ms": sms / cnt, "algorithmic_bytes_per_launch": per_launch,
                "traffic": traffic_tab.get(kernel)}

    def tc_roof(kernel, stage, flops_per_step, peak, source, bound="tensor"):
        sms, cnt = stage_raw[stage]
        per_launch = flops_per_step * args.steps / cnt
        achieved = per_launch / (sms / cnt / 1e3) / 1e12
        return {"bound": bound, "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak, "peak_source": source, "kernel": kernel, "kernel_ms": sms / cnt,
                "algorithmic_flops_per_launch": per_launch, "traffic": traffic_tab.get(kernel)}

    if sparse:
        zeta = 8
        # rowptr + (col, val) per nonzero + Y rows written + the byte-packed map
        alg_bytes = (m_local + 1) * 8 + nnz * 8 + m_local * k * 4 + n * zeta
        roof = hbm_roof("csr_ssign_y16_kernel", "update.omega", alg_bytes)
    elif rbf and a.precision:
        # row pass: Gram + [Y|T] sketch per kernel entry; column pass: Gram + X
        d = cfg["d"]
        rp = tc_roof("rbf_sketch_kernel row pass", "update.fused", 2 * m_local * n * (d + k + s), tc_peak, peak_kind)
        cp = tc_roof("rbf_sketch_kernel column pass", "update.upsilon", 2 * m_local * n * (d + k), tc_peak,
                     peak_kind)
        first, second = (rp, cp) if stage_raw["update.fused"][0] >= stage_raw["update.upsilon"][0] else (cp, rp)
        roof = dict(first)
        roof["other_kernel"] = second
    elif rbf:
        roof = tc_roof("sgemm_kernel (T = K_w Psi~^T, FP32 SIMT)", "update.psi", 2 * m_local * n * s, 74.4,
                       "nominal FP32 SIMT (148 SMs x 128 FMA/clk x 2 x 1.965 GHz)", bound="fp32-simt")
    elif a.precision:
        # the two large kernels per window: [Y|T] on the tensor pipe and the X^T
        # product that streams the FP32 window (4 B read + 2 B BF16 copy written
        # per element); the one with more measured time is the roofline kernel
        if a.precision == 2:
            # E4M3 [Y|T]; no FP8 peak is measured: the dense FP8 rate is twice
            # the BF16 rate on this part, so the denominator is 2x the measured
            # sustained BF16 figure
            yt = tc_roof("gemm_fp8_kernel", "update.fused", 2 * m_local * n * (k + s), 2 * tc_peak,
                         f"2 x bf16_tflops_sustained ({peak_kind}); FP8 peak not measured")
        else:
            yt = tc_roof("gemm_bf16_kernel", "update.fused", 2 * m_local * n * (k + s), tc_peak, peak_kind)
        xa = hbm_roof("gemm_a32_kernel", "update.upsilon", m_local * n * 6)
        xa["achieved_tflops"] = 2 * m_local * n * k * args.steps / (stage_raw["update.upsilon"][0] / 1e3) / 1e12
        first, second = (yt, xa) if stage_raw["update.fused"][0] >= stage_raw["update.upsilon"][0] else (xa, yt)
        roof = dict(first)
        roof["other_kernel"] = second
    else:
        roof = tc_roof("sgemm_kernel", "update.psi", 2 * m_local * n * s, 74.4,
                       "nominal FP32 SIMT (148 SMs x 128 FMA/clk x 2 x 1.965 GHz)", bound="fp32-simt")
    if not sparse:
        roof["step_flops"] = step_flops
        roof["step_tflops"] = step_flops / (ms / 1e3) / 1e12
    roof["stages_ms_per_step"] = stages

    # end to end through the public API with pinned host buffers
    e2e = None
    if rank == 0 and sparse and not args.no_e2e:
        e2e = with_pcie_floor(e2e_sparse(ctx, inp, m_local, row0, k, s, n, args))
    elif rank == 0 and rbf and not args.no_e2e:
        e2e = with_pcie_floor(e2e_rbf(ctx, inp, m_local, row0, k, s, n, args))
    elif rank == 0 and not sparse and not args.no_e2e:
        e2e = with_pcie_floor(e2e_dense(ctx, inp, m_local, row0, k, s, n, args))

    cpu = cpu_oracle = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu, cpu_oracle = cpu_baseline(args, cfg, budget_s=args.cpu_budget, csr=host_csr if sparse else None)

    # parity of the timed workload at its full size: the device sketches of
    # one step against the FP64 oracle's over every row of the same matrix
    # and maps (the CPU baseline leg above ran it), outside the timed region
    parity = None
    if cpu_oracle is not None and not args.no_accuracy:
        step()
        parity = sparse_parity(ctx, cpu_oracle)

    # accuracy of every dense / kernel form: the top-r singular values of the
    # fixed-rank approximation against FP64 SketchySVD on the same input and
    # the context's own maps
    acc = None
    if rank == 0 and world == 1 and not sparse and not args.no_accuracy:
        step()
        _, S_dev, _ = ctx.low_rank_approx()
        S64 = fp64_sigma(ctx, inp, cfg, cfg["rank"], gamma=cfg.get("gamma") if rbf else None)
        acc = sigma_accuracy(S_dev, S64, {0: "fp32", 1: "bf16", 2: "fp8"}[a.precision])

    # the residual pass (compute_residuals, the second stream of A behind
    # Skema::sketchysvd): FP64 on the device, timed once after the bench
    # steps, rank 0 at N = 1, with the U, S, V of this step's approximation
    respass = None
    approx = None
    if rank == 0 and world == 1 and not args.no_residuals and not (rbf and a.precision):
        step()
        # the fixed-rank approximation (FP64, on the device), timed on its
        # own: CholeskyQR2 of Y and X^T, the core solve and the small SVD,
        # into device buffers (CUDA events), then once more into host memory
        r = cfg["rank"]
        n_out = m_glob if rbf else n
        Ud = torch.empty((r, m_local), dtype=torch.float64, device=dev)  # column-major m x r
        Vd = torch.empty((r, n_out), dtype=torch.float64, device=dev)
        Sd = torch.empty(r, dtype=torch.float64, device=dev)
        a0e = torch.cuda.Event(enable_timing=True)
        a1e = torch.cuda.Event(enable_timing=True)
        ctx.low_rank_approx(device_out=(Ud, Sd, Vd))  # warm
        torch.cuda.synchronize()
        ctx.timing_enable(True)
        a0e.record(stream)
        ctx.low_rank_approx(device_out=(Ud, Sd, Vd))
        a1e.record(stream)
        torch.cuda.synchronize()
        astages = {name: round(ctx.timing_get(name)[0], 3)
                   for name in ("approx.orth", "approx.core", "approx.svd", "approx.vectors")}
        sweeps = ctx.timing_get("approx.svd_sweeps")[1]
        ctx.timing_enable(False)
        t0 = time.perf_counter()
        U, S, V = ctx.low_rank_approx()
        approx = {"ms": a0e.elapsed_time(a1e), "timer": "CUDA events, outputs in device memory",
                  "stages_ms": astages, "core_svd_sweeps": sweeps,
                  "ms_with_host_copy": (time.perf_counter() - t0) * 1e3}
        r0e = torch.cuda.Event(enable_timing=True)
        r1e = torch.cuda.Event(enable_timing=True)
        r = cfg["rank"]
        # FP64 work: A V and A^T U, 2 m n r flops each (dense input); the
        # CSR form does 4 r flops per nonzero
        fl = (4.0 * nnz * r) if sparse else (4.0 * m_local * (n if not rbf else m_glob) * r)

        def timed(fn):
            torch.cuda.synchronize()
            r0e.record(stream)
            out_n = fn()
            r1e.record(stream)
            torch.cuda.synchronize()
            return out_n, r0e.elapsed_time(r1e)

        # compute_residuals' path: the factors the approximation kept on the
        # device (residuals_begin with NULL factors), once untimed, then timed
        kept = lambda: ctx.residuals(None, None, None, None, row_blocks=[(row0, inp)])
        kept()
        rn, rms = timed(kept)
        # the same pass given host U, S, V (numpy, pageable): their upload is
        # inside the timed region
        rn_h, hms = timed(lambda: ctx.residuals(None, U, S, V, row_blocks=[(row0, inp)]))
        respass = {"ms": rms, "fp64_tflops": fl / (rms / 1e3) / 1e12,
                   "rnorm_over_sigma1_max": float(np.max(rn) / S[0]),
                   "includes": "the FP64 products from the factors kept on the device by the approximation "
                               "(compute_residuals' path) + D2H of the norms",
                   "from_host_factors": {"ms": hms,
                                         "max_rel_diff": float(np.max(np.abs(rn_h - rn) / np.abs(rn))),
                                         "includes": "H2D of U, S, V (host FP64, pageable) + the same pass"}}

    out = {
        "metric": "sketched rows/s",
        "value": value,
        "unit": "rows/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "strong" if rbf else "weak",
        "vs_baseline": None,
        "dtype": {0: "fp32", 1: "bf16", 2: "fp8"}[a.precision] if not sparse else "fp32",
        "data": "synthetic (seeded; no dataset)",
        "config": config_of(args, cfg, world, nnz),
        "roofline": roof,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": launches,
        "clocks": dict(clk.summary(), window="samples span continuous load bracketing the timed steps"),
    }
    if acc is not None:
        out["accuracy"] = acc
    if parity is not None:
        out["parity"] = parity
    if respass is not None:
        out["residual_pass"] = respass
    if approx is not None:
        out["low_rank_approx"] = approx
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return out if rank == 0 else None


def config_of(args, cfg, world, nnz):
    if cfg.get("vjp"):
        return {"workload": args.workload, "points": cfg["m"], "d": cfg["d"], "k": cfg["k"],
                "step": "skema_rbf_sketch_fwd + skema_rbf_sketch_vjp, device buffers",
                "precision": "bf16 tensor-core form" if cfg.get("prec") == 1 else "fp32",
                "cotangent": "fixed 2 Y (L = ||Y||_F^2)", "parallelism": f"replicas x{world}",
                "l2": "K tiles (2.5e9 entries) recomputed per step, never stored; E blocks stream > 126 MB L2"}
    c = {"workload": args.workload, "m_per_gpu": cfg["m"], "n": cfg["m"] if cfg.get("rbf") else cfg["n"],
         "rank": cfg["rank"],
         "range_k": cfg["k"], "core_s": cfg["s"], "window": cfg["window"],
         "maps": "sparse-sign zeta=8" if cfg["kind"] == 1 else "gauss",
         "parallelism": f"row-blocks x{world}" + (" + NCCL all-reduce of X,Z" if world > 1 else "")}
    if args.workload.startswith("csr"):
        c["nnz_per_gpu"] = int(nnz)
        c["l2"] = "working set ~450 MB per step > 126 MB L2 (no flush needed)"
    elif cfg.get("rbf"):
        c["m_per_gpu"] = (cfg["m"] + world - 1) // world
        c.update({"points": cfg["m"], "d": cfg["d"], "gamma": cfg.get("gamma"),
                  "kernel": "gauss-rbf, 8-component mixture, gamma = 1/(2 median sq. distance of 1,000 points)",
                  "parallelism": f"kernel row-blocks x{world}" + (" + NCCL all-reduce of X,Z" if world > 1 else ""),
                  "l2": "maps 0.6 GB (BF16) and Y 0.1 GB per step > 126 MB L2 (no flush needed)"})
        c["kernel_stored"] = "never (tiles regenerated in the sketch kernels)" if cfg.get("prec") else \
            "one window at a time (FP32)"
    else:
        c["l2"] = "A is 16 GB per step > 126 MB L2 (no flush needed)"
    return c


_PCIE = {}


def pcie_rates():
    """Host<->device copy rates of this box (GB/s): one 1 GiB pinned buffer
    copied to and from the device, best of 3 each, CUDA events."""
    import torch

    if not _PCIE:
        nb = 1 << 30
        h = torch.empty(nb, dtype=torch.uint8).pin_memory()
        d = torch.empty(nb, dtype=torch.uint8, device="cuda")
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        for name, fn in (("h2d_gbs", lambda: d.copy_(h, non_blocking=True)),
                         ("d2h_gbs", lambda: h.copy_(d, non_blocking=True))):
            best = None
            for _ in range(3):
                torch.cuda.synchronize()
                ev[0].record()
                fn()
                ev[1].record()
                ev[1].synchronize()
                ms = ev[0].elapsed_time(ev[1])
                best = ms if best is None else min(best, ms)
            _PCIE[name] = nb / (best / 1e3) / 1e9
        del h, d
    return dict(_PCIE)


def with_pcie_floor(e2e):
    """Adds the copy-only time of the step's host<->device bytes at this box's
    measured rates, and its ratio to the e2e step."""
    r = pcie_rates()
    floor = (e2e["h2d_bytes_per_step"] / (r["h2d_gbs"] * 1e9) + e2e["d2h_bytes_per_step"] / (r["d2h_gbs"] * 1e9)) * 1e3
    e2e["pcie"] = {"h2d_gbs": r["h2d_gbs"], "d2h_gbs": r["d2h_gbs"], "copy_floor_ms": floor,
                   "floor_over_step": floor / e2e["ms_per_step"],
                   "how": "1 GiB pinned buffer to and from the device, best of 3, CUDA events"}
    return e2e


def e2e_sparse(ctx, inp, m_local, row0, k, s, n, args):
    import torch

    import skema_b200._lib as L

    rowptr, col, val = inp
    h_rp = rowptr.cpu().pin_memory()
    h_col = col.cpu().pin_memory()
    h_val = val.cpu().pin_memory()
    hX = torch.empty((k, n), dtype=torch.float32).pin_memory()
    hY = torch.empty((ctx.nrow, k), dtype=torch.float32).pin_memory()
    hZ = torch.empty((s, s), dtype=torch.float32).pin_memory()
    lib, h = ctx.lib, ctx.h

    def one():
        ctx._check(lib.skema_reset(h))
        ctx._check(lib.skema_linear_update_csr(h, h_rp.data_ptr(), h_col.data_ptr(), h_val.data_ptr(), row0,
                                               m_local, L.MEM_HOST))
        ctx._check(lib.skema_get_sketch(h, 0, hX.data_ptr(), n, L.ROW_MAJOR, L.MEM_HOST))
        ctx._check(lib.skema_get_sketch(h, 1, hY.data_ptr(), k, L.ROW_MAJOR, L.MEM_HOST))
        ctx._check(lib.skema_get_sketch(h, 2, hZ.data_ptr(), s, L.ROW_MAJOR, L.MEM_HOST))

    for _ in range(2):
        one()
    steps = max(3, min(args.steps, 10))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        one()
    torch.cuda.synchronize()
    dt = (time.perf_counter() - t0) / steps
    h2d = h_rp.numel() * 8 + h_col.numel() * 4 + h_val.numel() * 4
    d2h = (k * n + ctx.nrow * k + s * s) * 4
    return {"value": m_local / dt, "unit": "rows/s", "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h), "ms_per_step": dt * 1e3,
            "path": "skema_linear_update_csr(mem=HOST) + skema_get_sketch(X,Y,Z, mem=HOST), pinned buffers",
            "timer": "host wall clock around synchronous calls"}


def e2e_rbf(ctx, P, m_local, row0, k, s, n, args):
    import torch

    import skema_b200._lib as L

    hP = P.cpu().pin_memory()  # n x d row-major points
    d = hP.shape[1]
    hX = torch.empty((k, n), dtype=torch.float32).pin_memory()
    hY = torch.empty((ctx.nrow, k), dtype=torch.float32).pin_memory()
    hZ = torch.empty((s, s), dtype=torch.float32).pin_memory()
    lib, h = ctx.lib, ctx.h

    def one():
        ctx._check(lib.skema_reset(h))
        ctx._check(lib.skema_linear_update_rbf(h, hP.data_ptr(), d, L.ROW_MAJOR, n, d, row0, m_local, L.MEM_HOST))
        ctx._check(lib.skema_get_sketch(h, 0, hX.data_ptr(), n, L.ROW_MAJOR, L.MEM_HOST))
        ctx._check(lib.skema_get_sketch(h, 1, hY.data_ptr(), k, L.ROW_MAJOR, L.MEM_HOST))
        ctx._check(lib.skema_get_sketch(h, 2, hZ.data_ptr(), s, L.ROW_MAJOR, L.MEM_HOST))

    one()
    steps = 2
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        one()
    torch.cuda.synchronize()
    dt = (time.perf_counter() - t0) / steps
    return {"value": m_local / dt, "unit": "rows/s", "h2d_bytes_per_step": int(n * d * 4),
            "d2h_bytes_per_step": int((k * n + ctx.nrow * k + s * s) * 4), "ms_per_step": dt * 1e3,
            "path": "skema_linear_update_rbf(mem=HOST) + skema_get_sketch(X,Y,Z, mem=HOST), pinned buffers",
            "timer": "host wall clock around synchronous calls"}


def e2e_dense(ctx, A, m_local, row0, k, s, n, args):
    import torch

    import skema_b200._lib as L

    hA = A.t().contiguous().cpu().pin_memory()  # A^T row-major == A column-major (ld = m)
    hX = torch.empty((k, n), dtype=torch.float32).pin_memory()
    hY = torch.empty((ctx.nrow, k), dtype=torch.float32).pin_memory()
    hZ = torch.empty((s, s), dtype=torch.float32).pin_memory()
    lib, h = ctx.lib, ctx.h

    def one():
        ctx._check(lib.skema_reset(h))
        ctx._check(lib.skema_linear_update_dense(h, hA.data_ptr(), m_local, L.COL_MAJOR, row0, m_local,
                                                 L.MEM_HOST))
        ctx._check(lib.skema_get_sketch(h, 0, hX.data_ptr(), n, L.ROW_MAJOR, L.MEM_HOST))
        ctx._check(lib.skema_get_sketch(h, 1, hY.data_ptr(), k, L.ROW_MAJOR, L.MEM_HOST))
        ctx._check(lib.skema_get_sketch(h, 2, hZ.data_ptr(), s, L.ROW_MAJOR, L.MEM_HOST))

    one()
    steps = 2
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        one()
    torch.cuda.synchronize()
    dt = (time.perf_counter() - t0) / steps
    return {"value": m_local / dt, "unit": "rows/s", "h2d_bytes_per_step": int(m_local * n * 4),
            "d2h_bytes_per_step": int((k * n + ctx.nrow * k + s * s) * 4), "ms_per_step": dt * 1e3,
            "path": "skema_linear_update_dense(mem=HOST) + skema_get_sketch(X,Y,Z, mem=HOST), pinned buffers",
            "timer": "host wall clock around synchronous calls"}


# ------------------------------------------------------- parity checks -----
# The checker, outside every timed region: FP64 arithmetic on the same input
# and the same maps as the device run. Large FP64 products run on the device
# (torch, float64), the approximation and the sparse-sign sketches come from
# the oracle's CPU restatement.
def _rel_fro(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def sparse_parity(ctx, o):
    """Device X, Y, Z of one step against the oracle's FP64 sketches of every
    row, and the sparse-sign maps bit for bit."""
    from skema_b200 import _lib as L

    X, Y, Z = ctx.get_sketches()
    maps_equal = True
    for which, name in ((L.UPSILON, "upsilon"), (L.OMEGA, "omega"), (L.PHI, "phi"), (L.PSI, "psi")):
        vals, idx = ctx.map_export(which)
        om = o.maps[name]
        maps_equal &= bool(np.array_equal(idx, om.idx) and np.array_equal(vals, om.val))
    return {"vs": "FP64 oracle over every row of the same CSR matrix and maps (CSR x SparseSign restatement)",
            "rows": int(o.m), "bar_rel_fro": 1e-5, "rel_fro_X": _rel_fro(X, o.X), "rel_fro_Y": _rel_fro(Y, o.Y),
            "rel_fro_Z": _rel_fro(Z, o.Z), "maps_bitexact": maps_equal}


class _LogicalMap:
    """A map in the form the oracle's approximation reads (.logical)."""

    def __init__(self, logical):
        self.logical = logical


def rbf_rows64(P64, sq, gamma, r0, wr):
    """FP64 kernel rows [r0, r0 + wr): exp(-gamma d^2), d^2 >= 0, unit diagonal."""
    import torch

    d2 = (sq[r0:r0 + wr, None] + sq[None, :] - 2.0 * (P64[r0:r0 + wr] @ P64.T)).clamp_(min=0.0)
    K = torch.exp(-gamma * d2)
    idx = torch.arange(wr, device=K.device)
    K[idx, r0 + idx] = 1.0
    return K


def fp64_sigma(ctx, inp, cfg, rank, gamma=None):
    """Top-rank singular values of SketchySVD in FP64 on the same input (dense
    A, or the points of a Gauss-RBF kernel) and the context's own maps (as
    exported: FP32 values, or the BF16 / E4M3 grid of the precision forms).
    Sketches X, Y, Z by FP64 products on the device, window by window with
    eta = nu = 1; the approximation by the oracle (initial_approx +
    low_rank_approx, FP64 LAPACK) on the host."""
    import torch

    from oracle import sketchy_oracle as O
    from skema_b200 import _lib as L

    dev = inp.device
    M = {w: np.ascontiguousarray(ctx.map_export(w)[0]) for w in (L.UPSILON, L.OMEGA, L.PHI, L.PSI)}
    U, Om, F, Ps = (torch.from_numpy(M[w]).to(dev) for w in (L.UPSILON, L.OMEGA, L.PHI, L.PSI))
    k, s = U.shape[0], F.shape[0]
    m = inp.shape[0]
    n = m if gamma is not None else inp.shape[1]
    W = cfg["window"]
    X = torch.zeros((k, n), dtype=torch.float64, device=dev)
    Y = torch.empty((m, k), dtype=torch.float64, device=dev)
    Z = torch.zeros((s, s), dtype=torch.float64, device=dev)
    if gamma is not None:
        P64 = inp.double()
        sq = (P64 * P64).sum(1)
    for r0 in range(0, m, W):
        wr = min(W, m - r0)
        Aw = rbf_rows64(P64, sq, gamma, r0, wr) if gamma is not None else inp[r0:r0 + wr].double()
        X += U[:, r0:r0 + wr] @ Aw
        Y[r0:r0 + wr] = Aw @ Om.T
        Z += F[:, r0:r0 + wr] @ (Aw @ Ps.T)
        del Aw
    o = O.OracleSketch.__new__(O.OracleSketch)
    o.k, o.s, o.rank = k, s, rank
    o.X, o.Y, o.Z = X.cpu().numpy(), Y.cpu().numpy(), Z.cpu().numpy()
    o.maps = {"phi": _LogicalMap(M[L.PHI]), "psi": _LogicalMap(M[L.PSI])}
    del X, Y, Z, U, Om, F, Ps
    torch.cuda.empty_cache()
    return o.low_rank_approx()[1]


def sigma_accuracy(S, S64, form):
    d = np.abs(np.asarray(S) - S64)
    return {"vs": "FP64 SketchySVD on the same input and maps (FP64 device products, oracle approximation)",
            "form": form, "rank": int(len(S64)), "max_rel_err_sigma_i": float(np.max(d / S64)),
            "max_err_over_sigma_1": float(np.max(d) / S64[0]), "sigma_1": float(S64[0]),
            "sigma_r": float(S64[-1])}


def vjp64(P, gamma, Om, Ybar, want_grad=True, blk=2048):
    """FP64 f = <Ybar, K Omega^T> of the RBF kernel sketch on the device, row
    block by row block (K never whole), and with want_grad its exact gradient
    w.r.t. the points and gamma (the unit diagonal contributes nothing)."""
    import torch

    P64 = P.double()
    O64 = Om.double()
    Yb = Ybar.double()
    N = P64.shape[0]
    sq = (P64 * P64).sum(1)
    f = torch.zeros((), dtype=torch.float64, device=P.device)
    if want_grad:
        rows = torch.zeros(N, dtype=torch.float64, device=P.device)
        cols = torch.zeros(N, dtype=torch.float64, device=P.device)
        EX = torch.zeros_like(P64)
        EtX = torch.zeros_like(P64)
        dg = torch.zeros((), dtype=torch.float64, device=P.device)
    for r0 in range(0, N, blk):
        wr = min(blk, N - r0)
        d2 = (sq[r0:r0 + wr, None] + sq[None, :] - 2.0 * (P64[r0:r0 + wr] @ P64.T)).clamp_(min=0.0)
        K = torch.exp(-gamma * d2)
        idx = torch.arange(wr, device=P.device)
        K[idx, r0 + idx] = 1.0
        f += (Yb[r0:r0 + wr] * (K @ O64.T)).sum()
        if want_grad:
            E = (Yb[r0:r0 + wr] @ O64) * K
            E[idx, r0 + idx] = 0.0
            dg -= (E * d2).sum()
            rows[r0:r0 + wr] += E.sum(1)
            cols += E.sum(0)
            EX[r0:r0 + wr] += E @ P64
            EtX += E.T @ P64[r0:r0 + wr]
            del E
        del d2, K
    if not want_grad:
        return float(f)
    dX = -2.0 * gamma * ((rows + cols)[:, None] * P64 - EX - EtX)
    return float(f), dX, float(dg)


def vjp_accuracy(P, gamma, Om, Ybar, dX, dg, seed=7):
    """The device VJP against the FP64 gradient and against central finite
    differences of the FP64 forward (h = 1e-3 relative): along a seeded
    random direction V of the points, and in gamma."""
    import torch

    _, dX64, dg64 = vjp64(P, gamma, Om, Ybar)
    g = torch.Generator(device=P.device)
    g.manual_seed(seed)
    V = torch.randn(P.shape, generator=g, device=P.device, dtype=torch.float64)
    h = 1e-3 * float(P.double().pow(2).mean().sqrt())
    fp = vjp64(P.double() + h * V, gamma, Om, Ybar, want_grad=False)
    fm = vjp64(P.double() - h * V, gamma, Om, Ybar, want_grad=False)
    fd_x = (fp - fm) / (2 * h)
    hg = 1e-3 * gamma
    fd_g = (vjp64(P, gamma + hg, Om, Ybar, want_grad=False) - vjp64(P, gamma - hg, Om, Ybar, want_grad=False)) / (
        2 * hg)
    dir_dev = float((dX.double() * V).sum())
    dir_64 = float((dX64 * V).sum())
    rel = lambda a, b: abs(a - b) / max(abs(b), 1e-300)
    return {"vs": "FP64 gradient on the device and central FD of the FP64 forward (h = 1e-3 relative)",
            "dX_rel_fro_vs_fp64": float((dX.double() - dX64).norm() / dX64.norm()),
            "dgamma_rel_vs_fp64": rel(dg, dg64),
            "fd_direction_rel": rel(dir_dev, fd_x), "fd_gamma_rel": rel(dg, fd_g),
            "fp64_vs_fd_direction_rel": rel(dir_64, fd_x), "fp64_vs_fd_gamma_rel": rel(dg64, fd_g)}


# ------------------------------------------------------- CPU baseline ------
def cpu_sample_sparse(cfg, budget_s, seed_rows=None, csr=None):
    """Oracle (FP64 CRS x SparseSign restatement, OpenMP) on windows of the
    workload until budget_s elapses (budget_s None: all rows); returns
    (rows/s, rows, threads, oracle sketch). csr: the workload's host arrays,
    when the caller already made them."""
    import scipy.sparse as sp

    from oracle import sketchy_oracle as O

    m, n, w = cfg["m"], cfg["n"], cfg["window"]
    rows_max = seed_rows or m
    rowptr, col, val = csr if csr is not None else make_csr_numpy(cfg, rows_max, cfg["seed"])
    A = sp.csr_matrix((val.astype(np.float64), col, rowptr), shape=(rows_max, n))
    o = O.OracleSketch(m, n, cfg["rank"], w, kind=1, issparse=True, sketch_range=cfg["k"], sketch_core=cfg["s"])
    t0 = time.perf_counter()
    done = 0
    while done < rows_max and (budget_s is None or time.perf_counter() - t0 < budget_s):
        wr = min(w, rows_max - done)
        o.update_rows(A, done, wr)
        done += wr
    dt = time.perf_counter() - t0
    return done / dt, done, O.num_threads(), o


def cpu_sample_dense(cfg, budget_s):
    from oracle import sketchy_oracle as O

    m, n, w = cfg["m"], cfg["n"], cfg["window"]
    rng = np.random.default_rng(cfg["seed"])
    A = rng.standard_normal((w, n))  # one window of the same shape, FP64
    o = O.OracleSketch(m, n, cfg["rank"], w, kind=0, sketch_range=cfg["k"], sketch_core=cfg["s"])
    t0 = time.perf_counter()
    done = 0
    while done == 0 or (done < 4 * w and time.perf_counter() - t0 < budget_s):
        O.update_dense(o.maps, A, done % (m - w))  # x, y, z of one window
        done += w
    dt = time.perf_counter() - t0
    return done / dt, done, O.num_threads()


def cpu_sample_rbf(cfg, budget_s):
    """Oracle (FP64 kernel window + dense sketch restatement) on 1,024-row
    windows of a same-recipe point set until budget_s elapses."""
    from oracle import sketchy_oracle as O

    N, d, w = cfg["m"], cfg["d"], 1024
    X = O.mixture_points(N, d, seed=cfg["seed"])
    gamma = O.median_gamma(X)
    o = O.OracleSketch(N, N, cfg["rank"], w, kind=0, sketch_range=cfg["k"], sketch_core=cfg["s"],
                       kernel_gamma=gamma)
    t0 = time.perf_counter()
    done = 0
    while done == 0 or (done < 4 * w and time.perf_counter() - t0 < budget_s):
        Kw = O.rbf_window(X, gamma, done, w)
        O.update_dense(o.maps, Kw, done)
        done += w
    dt = time.perf_counter() - t0
    return done / dt, done, O.num_threads()


def cpu_sample_vjp(cfg, ns=1000):
    """Oracle FP64 forward + VJP of an ns-point problem with the workload's d
    and k; every term costs N^2 (d or k), so the full-size time is the
    sample's times (N / ns)^2. Returns (rows/s, ns, threads)."""
    from oracle import sketchy_oracle as O

    N, d, k = cfg["m"], cfg["d"], cfg["k"]
    Xs = O.mixture_points(ns, d, seed=cfg["seed"])
    gs = O.median_gamma(Xs)
    Os = np.random.default_rng(5).uniform(-1, 1, size=(k, ns))
    t0 = time.perf_counter()
    Ys = O.rbf_fwd64(Xs, gs, Os)
    O.rbf_vjp64(Xs, gs, Os, 2.0 * Ys)
    ts = time.perf_counter() - t0
    return N / (ts * (N / ns) ** 2), ns, O.num_threads()


def cpu_baseline(args, cfg, budget_s, csr=None):
    """The CPU baseline leg; for the sparse workload it runs the oracle over
    every row of the same matrix (csr) and also returns that oracle sketch,
    which the parity check compares with the device's sketches."""
    o = None
    if cfg.get("rbf"):
        v, rows, thr = cpu_sample_rbf(cfg, budget_s)
        sample = f"{rows} kernel rows (windows of 1024) of a same-recipe point set, FP64"
    elif args.workload.startswith("csr"):
        v, rows, thr, o = cpu_sample_sparse(cfg, None, csr=csr)
        sample = f"all {rows} rows ({rows // cfg['window']} windows) of the workload, FP64"
    else:
        v, rows, thr = cpu_sample_dense(cfg, budget_s)
        sample = f"{rows} rows (whole windows of {cfg['window']}) of a same-shape FP64 matrix"
    return {"value": v, "unit": "rows/s", "cores": thr, "kind": "port", "sample": sample,
            "host_cpu": _cpu_model(), "nproc": os.cpu_count()}, o


def _cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return None


def run_reference(args, cfg):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    per_step = []
    budget = max(1.0, min(10.0, 150.0 / max(1, args.steps + args.warmup)))
    rows = 0
    thr = 1
    for i in range(args.warmup + args.steps):
        if cfg.get("vjp"):
            v, ns, thr = cpu_sample_vjp(cfg)
            r = cfg["m"]
        elif cfg.get("rbf"):
            v, r, thr = cpu_sample_rbf(cfg, budget)
        elif args.workload.startswith("csr"):
            v, r, thr, _ = cpu_sample_sparse(cfg, budget, seed_rows=min(cfg["m"], 200_000))
        else:
            v, r, thr = cpu_sample_dense(cfg, budget)
        if i >= args.warmup:
            per_step.append(v)
            rows = r
    v = statistics.median(per_step)
    out = {
        "metric": "sketched rows/s", "value": v, "unit": "rows/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": rows / v * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded; no dataset)",
        **({"scaling": "strong"} if cfg.get("rbf") else {}),
        "config": config_of(args, cfg, 1, 0), "impl": "reference",
        "cpu_baseline": {"value": v, "unit": "rows/s", "cores": thr, "kind": "port",
                         "sample": f"{rows} rows per step (bounded sample), FP64 oracle restatement",
                         "host_cpu": _cpu_model(), "nproc": os.cpu_count()},
        "e2e": {"value": v, "unit": "rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


# The other configurations, measured in the default run after the headline
# (one GPU): the dense 200,000 x 20,000 Gaussian case in the plain FP32 form
# and the BF16 / FP8 precision forms, the RBF kernel case in FP32 and BF16,
# and the kernel-sketch forward / adjoint pair in FP32 and BF16. Steps per
# workload are fewer for the slow plain forms.
SECONDARY = (("dense-fp32", 3), ("dense-bf16", 10), ("dense-fp8", 10), ("rbf-fp32", 2), ("rbf-bf16", 5),
             ("rbf-vjp", 3), ("rbf-vjp-bf16", 10))


def cublas_fp32_dense_ms(cfg, reps=3):
    """ms per step of the dense FP32 sketch's products done by cuBLAS SGEMM
    (torch.matmul in FP32, TF32 off) on the same shapes: per window of W rows
    [Y_w | T] = A_w [Omega; Psi]^T, X += Upsilon_w A_w and Z += Phi_w T,
    over the m / W windows of one step. A yardstick for the plain FP32 form
    (the library's own SIMT GEMM), not a product path."""
    import torch

    dev = torch.device("cuda", 0)
    m, n, k, s, W = cfg["m"], cfg["n"], cfg["k"], cfg["s"], cfg["window"]
    g = torch.Generator(device=dev)
    g.manual_seed(1)
    A = torch.randn(W, n, generator=g, device=dev)
    OP = torch.randn(n, k + s, generator=g, device=dev)
    Ups = torch.randn(k, W, generator=g, device=dev)
    Phi = torch.randn(s, W, generator=g, device=dev)
    X = torch.zeros(k, n, device=dev)
    Z = torch.zeros(s, s, device=dev)
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        def window():
            YT = A @ OP
            X.addmm_(Ups, A)
            Z.addmm_(Phi, YT[:, k:])

        for _ in range(2):
            window()
        nwin = (m + W - 1) // W
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps * nwin):
            window()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev
        del A, OP, Ups, Phi, X, Z
        torch.cuda.empty_cache()


def run_secondary(args, peaks, peak_kind):
    import torch

    res = {}
    for wl, steps in SECONDARY:
        sub = argparse.Namespace(**vars(args))
        sub.workload, sub.steps, sub.warmup = wl, steps, 3
        sub.no_e2e = sub.no_cpu = sub.no_residuals = True
        sub.clock_lead, sub.clock_tail = 0.5, 0.1
        cfg = dict(WORKLOADS[wl])
        out = run_vjp(sub, cfg, peaks, peak_kind) if cfg.get("vjp") else run_gpu(sub, cfg, peaks, peak_kind)
        torch.cuda.empty_cache()
        roof = out["roofline"]
        keep = ("bound", "achieved", "peak", "unit", "frac", "kernel", "kernel_ms", "peak_source")
        r = {key: roof[key] for key in keep if key in roof}
        if "other_kernel" in roof:
            r["other_kernel"] = {key: roof["other_kernel"][key] for key in keep if key in roof["other_kernel"]}
        if "step_tflops" in roof:
            r["step_tflops"] = roof["step_tflops"]
        res[wl] = {"value": out["value"], "unit": out["unit"], "ms_per_step": out["ms_per_step"],
                   "steps": steps, "warmup": 3, "dtype": out["dtype"], "config": out["config"], "roofline": r,
                   "accuracy": out.get("accuracy"), "gpu_launches": out["gpu_launches"], "clocks": out["clocks"]}
    sp = lambda a, b: res[a]["ms_per_step"] / res[b]["ms_per_step"]
    res["speedups"] = {"dense_bf16_over_fp32": sp("dense-fp32", "dense-bf16"),
                       "dense_fp8_over_fp32": sp("dense-fp32", "dense-fp8"),
                       "rbf_bf16_over_fp32": sp("rbf-fp32", "rbf-bf16"),
                       "vjp_bf16_over_fp32": sp("rbf-vjp", "rbf-vjp-bf16"),
                       "note": "ms per step of the plain FP32 form over the precision form, same input"}
    # the same dense products by cuBLAS SGEMM, for the scale of the plain form
    cb = cublas_fp32_dense_ms(dict(WORKLOADS["dense-fp32"]))
    res["cublas_fp32_dense"] = {"ms_per_step": cb, "over_library_fp32": res["dense-fp32"]["ms_per_step"] / cb,
                                "dense_bf16_speedup_over_it": cb / res["dense-bf16"]["ms_per_step"],
                                "note": "cuBLAS SGEMM (TF32 off) on the dense-fp32 products and shapes, "
                                        "a yardstick, not a product path"}
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="csr-sparse-sign", choices=sorted(WORKLOADS))
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-residuals", action="store_true", help="skip the residual-pass timing")
    ap.add_argument("--no-accuracy", action="store_true",
                    help="skip the parity checks against FP64 (sketches, singular values, adjoint)")
    ap.add_argument("--cpu-budget", type=float, default=12.0)
    ap.add_argument("--clock-lead", type=float, default=1.0, help="seconds of load before the timed steps")
    ap.add_argument("--clock-tail", type=float, default=0.3, help="seconds of load after the timed steps")
    ap.add_argument("--rows", type=int, default=0,
                    help="rows per GPU instead of the workload's (small cases for profiling)")
    ap.add_argument("--no-secondary", action="store_true",
                    help="measure only the headline workload (the default run on one GPU also measures the "
                         "dense, RBF and adjoint configurations after it)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    cfg = dict(WORKLOADS[args.workload])
    if args.rows > 0:
        cfg["m"] = args.rows
    if args.impl == "reference":
        run_reference(args, cfg)
        return
    peaks, kind = load_peaks()
    out = run_vjp(args, cfg, peaks, kind) if cfg.get("vjp") else run_gpu(args, cfg, peaks, kind)
    if out is None:
        return
    if (int(os.environ.get("WORLD_SIZE", "1")) == 1 and args.workload == "csr-sparse-sign" and args.rows == 0
            and not args.no_secondary):
        out["secondary"] = run_secondary(args, peaks, kind)
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
