#!/usr/bin/env python
"""Benchmark of the B200 multifrontal numeric phase.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]
                    [--parts all|main]

One step = one numeric factorization plus one solve of the workload's system
(or batch of systems), inputs resident in HBM.  The headline workload is the
3D 7-point Laplacian on a 64^3 grid (n = 262,144) in FP64: ``value`` is its
factor GFLOP/s.  With the default ``--parts all`` the same line also carries
every other part of the metric, each measured the same way (warm-up, K timed
steps with L2 flushed between them, device events, max over ranks):

  fp32ir      the same Laplacian, FP32 factor + FP64 refinement, and its
              speed-up over the FP64 line (factor + solve)
  diffusion80 3D variable-coefficient diffusion 80^3, FP32 + refinement and FP64
  elasticity40  Q1 hex elasticity 40^3 elements, 64 right-hand sides, both precisions
  batch2000   2,000 uneven 2D systems: systems/s, algorithmic bytes / time
              against HBM bandwidth, end to end, both precisions
  lap2d100    2D 5-point Laplacian 100^2

Every part reports its backward error and, on one GPU, its forward error
against the oracle's FP64 solution of the same system.  ``--gpus N`` runs N
ranks (it launches torchrun itself when not started under it): single-system
parts run as N independent replicas (that path does not shard); the batch is
sharded by system over the ranks (mfdag/sharding.py, no data-path collective).

``--impl reference`` times the reference's CPU numeric phase, restated in C
(oracle/), with all host threads and the system BLAS, on the headline workload.
"""
from __future__ import annotations

import argparse
import json
import os
import socket
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "multifrontal-dag_b200"))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from mfdag import problems as P  # noqa: E402

METRIC = "factor GFLOP/s & solve time @ bwd err<=1e-12: FP64 vs mixed+IR; batched solves/s"

WORKLOADS = {
    "lap3d64": dict(desc="3D 7-point Laplacian 64^3 (n=262,144), x* ~ U[-1,1] seed 1", make=lambda: P.laplace3d(64, 1),
                    precision=0, max_zero=1000),
    "lap3d64_fp32ir": dict(desc="3D 7-point Laplacian 64^3, FP32 factor + FP64 refinement",
                           make=lambda: P.laplace3d(64, 1), precision=1, max_zero=1000),
    "lap3d40": dict(desc="3D 7-point Laplacian 40^3 (n=64,000), small case for profiling captures",
                    make=lambda: P.laplace3d(40, 1), precision=0, max_zero=1000),
    "lap3d40_fp32ir": dict(desc="3D 7-point Laplacian 40^3 (n=64,000), FP32 factor + FP64 refinement, small case for profiling",
                           make=lambda: P.laplace3d(40, 1), precision=1, max_zero=1000),
    "lap2d100": dict(desc="2D 5-point Laplacian 100x100 (n=10,000), x* ~ U[-1,1] seed 0",
                     make=lambda: P.laplace2d(100, 0), precision=0, max_zero=10),
    "diff3d80": dict(desc="3D variable-coefficient diffusion 80^3 (n=512,000), FP32 factor + FP64 refinement",
                     make=lambda: P.diffusion3d(80, 2), precision=1, max_zero=1000),
    "diff3d80_fp64": dict(desc="3D variable-coefficient diffusion 80^3 (n=512,000), FP64",
                          make=lambda: P.diffusion3d(80, 2), precision=0, max_zero=1000),
    "elast40": dict(desc="3D Q1 hex elasticity 40^3 elements, 3 dof/node, x=0 clamped (n=201,720), 64 RHS, FP64",
                    make=lambda: P.elasticity3d(40, 4, 64), precision=0, max_zero=1000),
    "elast40_fp32ir": dict(desc="3D Q1 hex elasticity 40^3 elements (n=201,720), 64 RHS, FP32 factor + FP64 refinement",
                           make=lambda: P.elasticity3d(40, 4, 64), precision=1, max_zero=1000),
    "batch2000": dict(desc="2,000 shifted 2D 5-point Laplacians, sides ~ randint[16,128], shift ~ U[0,0.1], seed 3, FP64",
                      make=lambda: BatchProblem(P.laplace2d_batch(2000, 3)), precision=0, max_zero=100, batch=True),
    "batch200": dict(desc="200 shifted 2D 5-point Laplacians (the first 200 of the 2,000-system batch), small case for profiling",
                     make=lambda: BatchProblem(P.laplace2d_batch(2000, 3)[:200]), precision=0, max_zero=100, batch=True),
    "batch2000_fp32ir": dict(desc="2,000 shifted 2D 5-point Laplacians (seed 3), FP32 factor + FP64 refinement",
                             make=lambda: BatchProblem(P.laplace2d_batch(2000, 3)), precision=1, max_zero=100,
                             batch=True),
}

# the extra parts of the default line: key -> (FP64 workload, FP32 + refinement workload)
EXTRA_PARTS = [
    ("fp32ir", None, "lap3d64_fp32ir"),
    ("diffusion80", "diff3d80_fp64", "diff3d80"),
    ("elasticity40", "elast40", "elast40_fp32ir"),
    ("batch2000", "batch2000", "batch2000_fp32ir"),
    ("lap2d100", "lap2d100", None),
]


class BatchProblem:
    """Many independent systems solved as one handle: values and right-hand
    sides concatenated in system order."""

    def __init__(self, systems):
        self.systems = systems
        self.count = len(systems)
        self.n = int(sum(p.n for p in systems))
        self.val = np.concatenate([p.val for p in systems])
        self.rhs = np.concatenate([p.rhs for p in systems])
        self.offsets = np.concatenate([[0], np.cumsum([p.n for p in systems])]).astype(np.int64)

    @property
    def nnz(self) -> int:
        return int(self.val.size)

    def analyze(self, H, **opts):
        return H.Solver.analyze_batch([(p.n, p.col, p.row, p.order) for p in self.systems], **opts)

    def backward_error(self, x) -> float:
        worst, off = 0.0, 0
        for p in self.systems:
            worst = max(worst, P.backward_error(p.n, p.col, p.row, p.val, x[off:off + p.n], p.rhs))
            off += p.n
        return worst


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def rel_err(x, xo) -> float:
    return float(np.abs(np.asarray(x) - np.asarray(xo)).max() / max(np.abs(np.asarray(xo)).max(), 1e-300))


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = os.path.join("/tmp", f"mfd_clocks_{os.getpid()}_{time.monotonic_ns()}.csv")

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.device)], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        try:
            rows = [ln.split(",") for ln in open(self.path).read().strip().splitlines() if ln.strip()]
        except Exception:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            if len(r) < 9:
                continue
            for nm, v in zip(names, r[5:9]):
                if v.strip().lower() in ("active", "1"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def measured_peaks() -> dict:
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


def fp64_gemm_peak(torch, device) -> float:
    """cuBLAS FP64 GEMM throughput on this GPU (TFLOP/s), best of 5 (8192^3)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=device)
    b = torch.randn(n, n, dtype=torch.float64, device=device)
    torch.matmul(a, b)
    torch.cuda.synchronize(device)
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = max(best, 2 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


def ncu_traffic(workload: str, kernel: str, alg_bytes_per_launch: float):
    """DRAM bytes per launch: the committed ncu ratio (DRAM bytes per
    algorithmic byte, profiles/ncu_traffic.json) times this run's average
    algorithmic bytes per launch; None without a capture for the kernel."""
    try:
        d = json.load(open(os.path.join(ROOT, "profiles", "ncu_traffic.json")))
        e = d.get(workload, {}).get(kernel)
        if not e:
            return None
        return {"bytes_per_launch": round(e["dram_per_alg_byte"] * alg_bytes_per_launch),
                "dram_per_alg_byte": e["dram_per_alg_byte"], "source": e["source"]}
    except Exception:
        return None


def algorithmic_bytes(H, s, nsys: int, w: int, nrhs: int) -> dict:
    """Algorithmic bytes of one factorization and one solve (the byte model
    of the path): A values and indices (12 per entry), each front written once
    (w n_f (n_f+1)/2), each update matrix written once and read once (2 w
    nr_f (nr_f+1)/2), the relative map (4 nr_f); a solve reads every factor
    entry once (w nnz(L) per sweep, two sweeps) plus the vectors."""
    st = s.stats()
    fb, snr = 12.0 * st.nnz_a, 0.0
    for k in range(nsys):
        nc = np.diff(s.symbolic(H.SYM_NODE_PTR, k)).astype(np.float64)
        nr = np.diff(s.symbolic(H.SYM_LPTR, k)).astype(np.float64)
        nf = nc + nr
        fb += float((w * (nf * (nf + 1) / 2 + nr * (nr + 1)) + 4.0 * nr).sum())
        snr += float(nr.sum())
    sb = nrhs * (2.0 * w * st.nonzero + 8.0 * (4.0 * st.n + 2.0 * snr))
    return {"factor": fb, "solve": sb}


# ---------------------------------------------------------------------------
# CPU baseline: the oracle (restatement of the reference's numeric phase)
# ---------------------------------------------------------------------------
def cpu_reference(prob, max_zero, steps, threads, nb=192, nrhs_sample=1, warmup=0):
    """Oracle factorization under the reference's StarPU task DAG (one task
    per tile operation, OpenMP tasks with the StarPU access modes as depend
    clauses, sequential BLAS per task) on ``threads`` host threads, and solves;
    with several right-hand sides the first ``nrhs_sample`` are timed (the
    reference solves one vector per call) and all of them are returned."""
    from oracle import oracle as O
    blas = O.use_system_blas(True)
    o = O.Oracle.analyze(prob.n, prob.col, prob.row, nb=nb, max_zero=max_zero, order_perm=prob.order)
    cost = o.cost()
    multi = prob.rhs.ndim == 2
    k = min(nrhs_sample, prob.rhs.shape[1]) if multi else 1
    ft, st = [], []
    for it in range(warmup + steps):
        t0 = time.perf_counter()
        info = o.factorize(prob.val, nthreads=threads, schedule="dag")
        t1 = time.perf_counter()
        xs = [o.solve(prob.rhs[:, j] if multi else prob.rhs) for j in range(k)]
        t2 = time.perf_counter()
        assert info == 0
        if it >= warmup:
            ft.append(t1 - t0)
            st.append(t2 - t1)
    if multi and k < prob.rhs.shape[1]:
        X = o.solve_many(prob.rhs, nthreads=threads)
    else:
        X = np.stack(xs, axis=1) if multi else xs[0]
    bwd = 0.0
    for j in range(k):
        b = prob.rhs[:, j] if multi else prob.rhs
        bwd = max(bwd, P.backward_error(prob.n, prob.col, prob.row, prob.val, X[:, j] if multi else X, b))
    return {"cost": cost, "factor_s": ft, "solve_s": st, "bwd": bwd, "blas": blas, "nb": nb, "rhs_timed": k, "x": X}


def cpu_reference_batch(bp, max_zero, threads, sample, nb=128):
    """Oracle over a sample of the batch's systems, one system per host thread
    (each system factored single-threaded, as independent jobs would be)."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle import oracle as O
    blas = O.use_system_blas(True)
    systems = bp.systems[:sample]
    handles = [O.Oracle.analyze(p.n, p.col, p.row, nb=nb, max_zero=max_zero, order_perm=p.order) for p in systems]
    cost = sum(o.cost() for o in handles)

    def job(i):
        o, p = handles[i], systems[i]
        info = o.factorize(p.val, nthreads=1)
        x = o.solve(p.rhs)
        return info, P.backward_error(p.n, p.col, p.row, p.val, x, p.rhs), x

    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=threads) as ex:
        res = list(ex.map(job, range(len(systems))))
    dt = time.perf_counter() - t0
    assert all(r[0] == 0 for r in res)
    return {"systems": len(systems), "seconds": dt, "systems_per_s": len(systems) / dt, "cost": cost,
            "bwd": max(r[1] for r in res), "blas": blas, "nb": nb, "x": [r[2] for r in res]}


def run_reference_arm(args, wl, prob):
    """The reference's CPU numeric phase (restated in C, oracle/) on this
    workload with all host threads; one untimed warm-up step, then at most 5
    timed steps, one full factorization + solve each (a batch: the first 200
    systems per step)."""
    threads = os.cpu_count() or 1
    steps = max(1, min(args.steps, 5))
    warm = 1 if args.warmup > 0 else 0
    t0 = time.time()
    batch = bool(wl.get("batch"))
    base = {"impl": "reference", "metric": METRIC, "n_gpus": args.gpus, "steps": steps, "warmup": warm,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic"}
    if batch:
        for _ in range(warm):
            cpu_reference_batch(prob, wl["max_zero"], threads, sample=200)
        rs = [cpu_reference_batch(prob, wl["max_zero"], threads, sample=200) for _ in range(steps)]
        secs = statistics.mean(r["seconds"] for r in rs)
        value = rs[0]["systems"] / secs
        unit = "systems/s"
        sample = (f"factor + solve of the first {rs[0]['systems']} of {prob.count} systems per step, one system per "
                  f"thread, {'OpenBLAS' if rs[0]['blas'] else 'C loops'} tiles nb={rs[0]['nb']}")
        extra = {"ms_per_step": round(1e3 * secs, 3), "bwd_err": max(r["bwd"] for r in rs)}
        cfg = {"workload": wl["desc"], "systems": prob.count, "max_zero": wl["max_zero"], "nb": rs[0]["nb"]}
    else:
        r = cpu_reference(prob, wl["max_zero"], steps, threads, warmup=warm)
        fs = statistics.mean(r["factor_s"])
        value = r["cost"] / fs / 1e9
        unit = "GFLOP/s"
        sample = (f"full numeric factorization + solve of one RHS per step, the StarPU task DAG as OpenMP tasks "
                  f"over {threads} threads, sequential {'OpenBLAS' if r['blas'] else 'C loops'} per tile task, "
                  f"tiles nb={r['nb']}")
        extra = {"ms_per_step": round(1e3 * (fs + statistics.mean(r["solve_s"])), 3),
                 "solve_ms": round(1e3 * statistics.mean(r["solve_s"]), 3), "bwd_err": r["bwd"]}
        cfg = {"workload": wl["desc"], "max_zero": wl["max_zero"], "nb": r["nb"], "n": prob.n, "nnz": prob.nnz,
               "cost_flops": r["cost"], "ordering": "geometric nested dissection"}
    line = dict(base, value=round(value, 3), unit=unit, config=cfg,
                cpu_baseline={"value": round(value, 3), "unit": unit, "cores": threads, "kind": "port",
                              "sample": sample},
                e2e={"value": round(value, 3), "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                wall_s=round(time.time() - t0, 1), **extra)
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
class Ctx:
    def __init__(self, world, rank, device, torch, dist):
        self.world, self.rank, self.device, self.torch, self.dist = world, rank, device, torch, dist
        self.dev = f"cuda:{device}"

    def max_over_ranks(self, vals):
        t = self.torch.tensor([float(v) for v in vals], dtype=self.torch.float64, device=self.dev)
        if self.world > 1:
            self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return [float(v) for v in t.tolist()]

    def barrier(self):
        if self.world > 1:
            self.dist.barrier()


def measure(ctx: Ctx, name: str, args, *, headline: bool, oracle_x=None):
    """One workload on this rank's GPU: setup, warm-up, K timed steps (device
    events, L2 flushed between steps), end to end through the C ABI with host
    buffers, and (headline only) the per-kernel profile.  Returns the part's
    results; the forward error needs the oracle's solution (``oracle_x`` or the
    CPU baseline leg run here)."""
    from mfdag import hppllt as H
    torch, device, dev = ctx.torch, ctx.device, ctx.dev
    wl = WORKLOADS[name]
    prob = wl["make"]()
    batch = bool(wl.get("batch"))
    total_systems = prob.count if batch else 1
    full = prob
    if batch and ctx.world > 1:
        # the batch shards by system (no data-path collective): LPT by estimated cost
        from mfdag import sharding
        costs = [sharding.system_cost(p.n, p.col, p.row, p.order, wl["max_zero"]) for p in prob.systems]
        mine = sharding.shard_lpt(costs, ctx.world)[ctx.rank]
        prob = BatchProblem([prob.systems[i] for i in mine])
    nrhs = 1 if prob.rhs.ndim == 1 else int(prob.rhs.shape[1])
    opts = dict(max_zero=wl["max_zero"], nb=10, precision=wl["precision"], device=device)
    t0 = time.perf_counter()
    s = prob.analyze(H, **opts) if batch else H.Solver.analyze(prob.n, prob.col, prob.row, prob.order, **opts)
    t_setup = time.perf_counter() - t0
    st = s.stats()
    cost = int(st.cost)
    rhs_cm = np.ascontiguousarray(prob.rhs.T) if nrhs > 1 else prob.rhs      # column-major (n, nrhs)
    a_dev = torch.from_numpy(prob.val).to(dev)
    b_dev = torch.from_numpy(rhs_cm).to(dev)
    x_dev = torch.empty_like(b_dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)   # 256 MiB > L2

    def step():
        info = s.factorize(a_dev)
        assert info == 0, info
        f_ms = s.stats().factor_ms
        x_dev.copy_(b_dev)
        torch.cuda.synchronize(device)
        rep, rc = s.solve(x_dev, nrhs=nrhs)
        assert rc == 0, rc
        return f_ms, rep.time_ms, rep.backward_error, rep.iterations

    for _ in range(max(3, args.warmup)):
        step()
    fms, sms, bwds, its = [], [], [], []
    ctx.barrier()
    torch.cuda.synchronize(device)
    with ClockSampler(device) as clk:
        w0 = time.perf_counter()
        for _ in range(args.steps):
            flush.fill_(1.0)
            f_ms, s_ms, bwd, it = step()
            fms.append(f_ms); sms.append(s_ms); bwds.append(bwd); its.append(it)
        torch.cuda.synchronize(device)
        wall = time.perf_counter() - w0
    ctx.barrier()
    clocks = clk.summary()
    f_max, s_max, wall_max, setup_max = ctx.max_over_ranks(
        [statistics.mean(fms), statistics.mean(sms), wall, t_setup])
    gflops = ctx.world * cost / (f_max * 1e-3) / 1e9
    if batch:
        unit, value = "systems/s", total_systems / ((f_max + s_max) * 1e-3)
    else:
        unit, value = "GFLOP/s", gflops
    st = s.stats()
    launches = args.steps * (int(st.launches_factor) + int(st.launches_solve) * max(1, max(its) if its else 1))
    x_last = x_dev.cpu().numpy()
    x_last = x_last.T if nrhs > 1 else x_last
    host_bwd = prob.backward_error(x_last) if batch else P.backward_error(prob.n, prob.col, prob.row, prob.val,
                                                                          x_last[:, 0] if nrhs > 1 else x_last,
                                                                          prob.rhs[:, 0] if nrhs > 1 else prob.rhs)

    # ---- end to end through the C ABI with host buffers (pinned) ----
    a_pin = torch.from_numpy(prob.val).pin_memory()
    b_host = torch.from_numpy(rhs_cm.copy()).pin_memory()
    e2e_t = []
    for k in range(args.steps + 1):
        x_host = b_host.clone()
        t0 = time.perf_counter()
        info = s.factorize(a_pin)
        rep, rc = s.solve(x_host, nrhs=nrhs)
        t1 = time.perf_counter()
        assert info == 0 and rc == 0
        if k > 0:
            e2e_t.append(t1 - t0)
    e2e_s = ctx.max_over_ranks([statistics.mean(e2e_t)])[0]
    e2e_value = total_systems / e2e_s if batch else ctx.world * cost / e2e_s / 1e9
    h2d = int(8 * prob.nnz + 8 * prob.n * nrhs)
    e2e = {"value": round(e2e_value, 3), "unit": unit, "h2d_bytes_per_step": h2d,
           "d2h_bytes_per_step": int(8 * prob.n * nrhs + 4), "ms_per_step": round(1e3 * e2e_s, 3),
           "what": "mfd_factorize(pinned host A) + mfd_solve(pinned host b), wall clock"}

    res = {"name": name, "workload": wl["desc"], "precision": "fp64" if wl["precision"] == 0 else "fp32+fp64ir",
           "value": round(value, 3), "unit": unit, "factor_ms": round(f_max, 3), "factor_gflops": round(gflops, 3),
           "solve_ms": round(s_max, 3), "ms_per_step": round(f_max + s_max, 3), "bwd_err": max(bwds),
           "bwd_err_host": host_bwd, "ir_iterations": max(its) if its else 0,
           "wall_ms_per_step": round(1e3 * wall_max / args.steps, 3), "setup_s": round(setup_max, 2),
           "clocks": clocks, "e2e": e2e, "gpu_launches": launches, "nrhs": nrhs,
           "config": {"workload": wl["desc"], "name": name, "n": prob.n, "nnz_lower": prob.nnz, "nrhs": nrhs,
                      "fronts": int(st.num_front), "levels": int(st.num_level), "max_front": int(st.max_front),
                      "cost_flops": cost, "nnz_L": int(st.nonzero), "nb": 10, "max_zero": wl["max_zero"]}}
    if batch:
        res["systems"] = total_systems
        res["config"]["systems"] = total_systems
        w = 8 if wl["precision"] == 0 else 4
        ab = algorithmic_bytes(H, s, prob.count, w, nrhs)
        peak = float(measured_peaks().get("hbm_gbs", 6650.0))
        gbs = (ab["factor"] + ab["solve"]) / ((f_max + s_max) * 1e-3) / 1e9 * ctx.world
        res["hbm"] = {"achieved_gbs": round(gbs, 1), "peak_gbs": peak, "frac": round(gbs / peak, 4),
                      "factor_gbs": round(ab["factor"] / (f_max * 1e-3) / 1e9 * ctx.world, 1),
                      "alg_bytes_factor": ab["factor"], "alg_bytes_solve": ab["solve"],
                      "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in measured_peaks() else "fallback"}

    # ---- roofline of the dominant kernel (per-launch events, graphs off) ----
    if headline and not args.no_profile:
        nprof = max(1, min(args.steps, 3))
        s.set_profiling(True)
        for _ in range(nprof):
            step()
        prof = s.profile()
        s.set_profiling(False)
        fact_classes = ["small_front", "zero", "assemble", "extend_add", "panel", "trsm", "update"]
        dom = max(fact_classes, key=lambda k: prof[k]["ms"])
        d = prof[dom]
        peaks = measured_peaks()
        per_launch_ms = d["ms"] / max(1, d["launches"])
        if dom in ("update", "trsm") and wl["precision"] == 0:
            peak = fp64_gemm_peak(torch, device)
            roof = {"kernel": dom, "bound": "tensor", "achieved": round(d["flops"] / (d["ms"] * 1e-3) / 1e12, 3),
                    "peak": round(peak, 3), "unit": "TFLOP/s",
                    "peak_source": "cuBLAS FP64 GEMM 8192^3 measured in this run (MEASURED_PEAKS.json has no FP64 figure)"}
        elif dom in ("update", "trsm"):
            # the FP32 update issues TF32 MMAs (three per product in the split form): its pipe peaks at half
            # the BF16 rate; achieved counts the algorithmic flops once
            bf = float(peaks.get("bf16_tflops_sustained", peaks.get("bf16_tflops", 1400.0)))
            roof = {"kernel": dom, "bound": "tensor", "achieved": round(d["flops"] / (d["ms"] * 1e-3) / 1e12, 3),
                    "peak": round(bf / 2, 1), "unit": "TFLOP/s", "mma_flops_per_alg_flop": 3,
                    "peak_source": "TF32 = MEASURED_PEAKS.json bf16 sustained / 2 (dense TF32:BF16 rate)"}
        else:
            peak = float(peaks.get("hbm_gbs", 6650.0))
            roof = {"kernel": dom, "bound": "hbm", "achieved": round(d["bytes"] / (d["ms"] * 1e-3) / 1e9, 1),
                    "peak": peak, "unit": "GB/s",
                    "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks else "fallback 6650 GB/s"}
        roof["frac"] = round(roof["achieved"] / roof["peak"], 4)
        tr = ncu_traffic(name, dom, d["bytes"] / max(1, d["launches"]))
        roof["traffic"] = tr["bytes_per_launch"] if tr else None
        roof["traffic_source"] = tr if tr else "no ncu capture committed for this kernel and workload"
        roof["launches_per_step"] = d["launches"] // nprof
        roof["avg_launch_ms"] = round(per_launch_ms, 4)
        roof["algorithmic_per_launch"] = (d["flops"] if roof["bound"] == "tensor" else d["bytes"]) / max(1, d["launches"])
        roof["share_of_factor"] = round(d["ms"] / max(1e-9, sum(prof[k]["ms"] for k in fact_classes)), 3)
        res["roofline"] = roof
        res["kernel_profile_ms_per_step"] = {k: round(v["ms"] / nprof, 3) for k, v in prof.items() if v["launches"]}

    # ---- CPU baseline (rank 0, one GPU) and forward error against the oracle ----
    fwd = None
    if ctx.rank == 0 and ctx.world == 1 and args.cpu_baseline == "auto":
        threads = os.cpu_count() or 1
        try:
            if batch:
                r = cpu_reference_batch(full, wl["max_zero"], threads, sample=200)
                fwd = max(rel_err(x_last[full.offsets[i]:full.offsets[i + 1]], xo) for i, xo in enumerate(r["x"]))
                if headline:
                    res["cpu_baseline"] = {
                        "value": round(r["systems_per_s"], 3), "unit": "systems/s", "cores": threads, "kind": "port",
                        "sample": f"factor + solve of the first {r['systems']} of the {full.count} systems, one "
                                  f"system per thread (oracle, {'OpenBLAS' if r['blas'] else 'C loops'} tiles "
                                  f"nb={r['nb']}), {r['seconds']:.1f} s", "bwd_err": r["bwd"]}
                else:
                    res["cpu_systems_per_s"] = round(r["systems_per_s"], 3)
                res["fwd_err_sample"] = f"first {r['systems']} systems"
            else:
                if oracle_x is None:
                    r = cpu_reference(prob, wl["max_zero"], 1, threads, nrhs_sample=min(nrhs, 2))
                    oracle_x = r["x"]
                    fs = r["factor_s"][0]
                    cpu = {"value": round(r["cost"] / fs / 1e9, 3), "unit": "GFLOP/s", "cores": threads,
                           "kind": "port",
                           "sample": f"one full numeric factorization of the same workload (oracle, StarPU task "
                                     f"DAG as OpenMP tasks, sequential {'OpenBLAS' if r['blas'] else 'C loops'} per "
                                     f"tile task, tiles nb={r['nb']}), "
                                     f"{fs:.1f} s" + (f"; solve of {r['rhs_timed']} of {nrhs} RHS, scaled"
                                                      if nrhs > 1 else ""),
                           "solve_ms": round(1e3 * r["solve_s"][0] * nrhs / r["rhs_timed"], 2), "bwd_err": r["bwd"]}
                    if headline:
                        res["cpu_baseline"] = cpu
                    else:
                        res["cpu_gflops"] = cpu["value"]
                if nrhs > 1:
                    fwd = max(rel_err(x_last[:, j], oracle_x[:, j]) for j in range(nrhs))
                else:
                    fwd = rel_err(x_last, oracle_x)
        except Exception as e:  # noqa: BLE001
            res["cpu_baseline_error"] = str(e)
    res["fwd_err_vs_oracle"] = fwd
    res["_oracle_x"] = oracle_x if not batch else None
    s.close()
    del a_dev, b_dev, x_dev, flush
    torch.cuda.empty_cache()
    return res


def part_summary(r: dict, keys=("value", "unit", "factor_ms", "factor_gflops", "solve_ms", "ms_per_step", "bwd_err",
                                "fwd_err_vs_oracle", "ir_iterations", "setup_s", "e2e", "clocks", "gpu_launches",
                                "hbm", "systems", "cpu_gflops", "cpu_systems_per_s", "fwd_err_sample")) -> dict:
    out = {"workload": r["workload"], "precision": r["precision"]}
    for k in keys:
        if k in r and r[k] is not None:
            out[k] = r[k]
    return out


def free_port() -> int:
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="lap3d64", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--parts", default="all", choices=["all", "main"],
                    help="all: the headline line also carries every other configuration; main: headline only")
    ap.add_argument("--cpu-baseline", default="auto", choices=["auto", "skip"])
    ap.add_argument("--no-profile", action="store_true")
    args = ap.parse_args()

    if "WORLD_SIZE" not in os.environ and args.gpus > 1:
        # not under torchrun: launch one rank per GPU ourselves
        cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
               "--master-addr", "127.0.0.1", "--master-port", str(free_port()), os.path.abspath(__file__)]
        cmd += sys.argv[1:]
        sys.exit(subprocess.run(cmd).returncode)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != args.gpus:
        log(f"bench.py: --gpus {args.gpus} but WORLD_SIZE={world}; launch one rank per GPU "
            f"(torchrun --nproc-per-node {args.gpus}) or pass --gpus {world}")
        sys.exit(2)
    wl = WORKLOADS[args.workload]
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))

    if args.impl == "reference":
        if rank == 0:
            run_reference_arm(args, wl, wl["make"]())
        if world > 1:
            dist.destroy_process_group()
        return

    torch.cuda.set_device(local)
    ctx = Ctx(world, rank, local, torch, dist)
    main_r = measure(ctx, args.workload, args, headline=True)
    parts = {}
    if args.parts == "all" and args.workload == "lap3d64":
        for key, w64, w32 in EXTRA_PARTS:
            entry = {}
            ox = main_r["_oracle_x"] if key == "fp32ir" else None     # the same system as the headline
            for tag, w in (("fp64", w64), ("fp32ir", w32)):
                if w is None:
                    continue
                r = measure(ctx, w, args, headline=False, oracle_x=ox)
                entry[tag] = part_summary(r)
                if not WORKLOADS[w].get("batch"):
                    ox = r["_oracle_x"]                                # reused by the other precision
            if key == "fp32ir":
                entry = entry["fp32ir"]
                entry["speedup_vs_fp64"] = round(main_r["ms_per_step"] / entry["ms_per_step"], 3)
                entry["factor_speedup_vs_fp64"] = round(main_r["factor_ms"] / entry["factor_ms"], 3)
            elif "fp64" in entry and "fp32ir" in entry:
                entry["fp32ir_speedup"] = round(entry["fp64"]["ms_per_step"] / entry["fp32ir"]["ms_per_step"], 3)
            parts[key] = entry

    if rank == 0:
        cfg = dict(main_r["config"])
        cfg.update({"ordering": "geometric nested dissection",
                    "l2": "flushed (256 MiB write) between timed steps; working set > L2",
                    "parallelism": (f"systems sharded over {world} GPU(s) by estimated cost, no collective"
                                    if WORKLOADS[args.workload].get("batch")
                                    else f"{world} independent replica(s); the batch part sharded by system")})
        batch = bool(wl.get("batch"))
        line = {
            "metric": METRIC, "value": main_r["value"], "unit": main_r["unit"], "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": main_r["ms_per_step"], "higher_is_better": True,
            "scaling": "strong" if batch else "weak", "vs_baseline": None,
            "dtype": "f64" if wl["precision"] == 0 else "f32+f64ir",
            "data": "synthetic", "config": cfg,
        }
        for k in ("factor_ms", "factor_gflops", "solve_ms", "bwd_err", "bwd_err_host", "fwd_err_vs_oracle",
                  "ir_iterations", "wall_ms_per_step", "setup_s", "clocks", "e2e", "gpu_launches", "roofline",
                  "cpu_baseline", "hbm", "kernel_profile_ms_per_step", "cpu_baseline_error"):
            if k in main_r:
                line[k] = main_r[k]
        if parts:
            line["parts"] = parts
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
