#!/usr/bin/env python
"""Benchmark of the B200 multifrontal numeric phase.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]

One step = one numeric factorization plus one solve of the workload's system
(or batch of systems), inputs resident in HBM.  The default workload is the 3D
7-point Laplacian on a 64^3 grid (n = 262,144) in FP64, the single-GPU
configuration the headline metric (factor GFLOP/s) is quoted on.  Under
torchrun every rank runs an independent replica of a single-system workload (that
path does not shard); a batch workload is sharded by system across the ranks
(mfdag/sharding.py, no collective on the data path).  ``value`` is the job
aggregate and timing is the max over ranks.

``--impl reference`` times the reference's CPU numeric phase, restated in C
(oracle/), with all host threads and the system BLAS, on the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
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


class BatchProblem:
    """Many independent systems solved as one handle: values and right-hand
    sides concatenated in system order."""

    def __init__(self, systems):
        self.systems = systems
        self.count = len(systems)
        self.n = int(sum(p.n for p in systems))
        self.val = np.concatenate([p.val for p in systems])
        self.rhs = np.concatenate([p.rhs for p in systems])

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
        self.path = os.path.join("/tmp", f"mfd_clocks_{os.getpid()}.csv")

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


# ---------------------------------------------------------------------------
# CPU baseline: the oracle (restatement of the reference's numeric phase)
# ---------------------------------------------------------------------------
def cpu_reference(prob, max_zero, steps, threads, nb=128, nrhs_sample=1):
    """Oracle factorization (tree-level parallel over ``threads``) and solves;
    with several right-hand sides the first ``nrhs_sample`` are solved (the
    reference solves one vector per call)."""
    from oracle import oracle as O
    blas = O.use_system_blas(True)
    o = O.Oracle.analyze(prob.n, prob.col, prob.row, nb=nb, max_zero=max_zero, order_perm=prob.order)
    cost = o.cost()
    multi = prob.rhs.ndim == 2
    k = min(nrhs_sample, prob.rhs.shape[1]) if multi else 1
    ft, st = [], []
    bwd = 0.0
    for _ in range(steps):
        t0 = time.perf_counter()
        info = o.factorize(prob.val, nthreads=threads)
        t1 = time.perf_counter()
        xs = [o.solve(prob.rhs[:, j] if multi else prob.rhs) for j in range(k)]
        t2 = time.perf_counter()
        assert info == 0
        ft.append(t1 - t0)
        st.append(t2 - t1)
    for j, x in enumerate(xs):
        b = prob.rhs[:, j] if multi else prob.rhs
        bwd = max(bwd, P.backward_error(prob.n, prob.col, prob.row, prob.val, x, b))
    return {"cost": cost, "factor_s": ft, "solve_s": st, "bwd": bwd, "blas": blas, "nb": nb, "rhs_timed": k}


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
        return info, P.backward_error(p.n, p.col, p.row, p.val, x, p.rhs)

    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=threads) as ex:
        res = list(ex.map(job, range(len(systems))))
    dt = time.perf_counter() - t0
    assert all(r[0] == 0 for r in res)
    return {"systems": len(systems), "seconds": dt, "systems_per_s": len(systems) / dt, "cost": cost,
            "bwd": max(r[1] for r in res), "blas": blas, "nb": nb}


def run_reference_arm(args, wl, prob):
    """The reference's CPU numeric phase (restated in C, oracle/) on this
    workload with all host threads; at most 5 timed steps, one full
    factorization + solve each (a batch: the first 200 systems per step)."""
    threads = os.cpu_count() or 1
    steps = max(1, min(args.steps, 5))
    t0 = time.time()
    batch = bool(wl.get("batch"))
    base = {"impl": "reference", "metric": METRIC, "n_gpus": args.gpus, "steps": steps, "warmup": 0,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic"}
    if batch:
        rs = [cpu_reference_batch(prob, wl["max_zero"], threads, sample=200) for _ in range(steps)]
        secs = statistics.mean(r["seconds"] for r in rs)
        value = rs[0]["systems"] / secs
        unit = "systems/s"
        sample = (f"factor + solve of the first {rs[0]['systems']} of {prob.count} systems per step, one system per "
                  f"thread, {'OpenBLAS' if rs[0]['blas'] else 'C loops'} tiles nb={rs[0]['nb']}")
        extra = {"ms_per_step": round(1e3 * secs, 3), "bwd_err": max(r["bwd"] for r in rs)}
        cfg = {"workload": wl["desc"], "systems": prob.count, "max_zero": wl["max_zero"], "nb": rs[0]["nb"]}
    else:
        r = cpu_reference(prob, wl["max_zero"], steps, threads)
        fs = statistics.mean(r["factor_s"])
        value = r["cost"] / fs / 1e9
        unit = "GFLOP/s"
        sample = (f"full numeric factorization + solve of one RHS per step, tree-level parallel over {threads} "
                  f"threads, {'OpenBLAS' if r['blas'] else 'C loops'} tiles nb={r['nb']}")
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
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="lap3d64", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-baseline", default="auto", choices=["auto", "skip"])
    ap.add_argument("--no-profile", action="store_true")
    args = ap.parse_args()
    wl = WORKLOADS[args.workload]

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
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

    from mfdag import hppllt as H
    device = local
    torch.cuda.set_device(device)
    dev = f"cuda:{device}"
    prob = wl["make"]()
    batch = bool(wl.get("batch"))
    total_systems = prob.count if batch else 1
    if batch and world > 1:
        # the batch shards by system (no data-path collective): LPT by estimated cost
        from mfdag import sharding
        costs = [sharding.system_cost(p.n, p.col, p.row, p.order, wl["max_zero"]) for p in prob.systems]
        mine = sharding.shard_lpt(costs, world)[rank]
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
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(device)
    with ClockSampler(device) as clk:
        w0 = time.perf_counter()
        for _ in range(args.steps):
            flush.fill_(1.0)
            f_ms, s_ms, bwd, it = step()
            fms.append(f_ms); sms.append(s_ms); bwds.append(bwd); its.append(it)
        torch.cuda.synchronize(device)
        wall = time.perf_counter() - w0
    if world > 1:
        dist.barrier()
    clocks = clk.summary()
    f_mean, s_mean = statistics.mean(fms), statistics.mean(sms)
    tvec = torch.tensor([f_mean, s_mean, wall], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(tvec, op=dist.ReduceOp.MAX)
    f_max, s_max, wall_max = (float(v) for v in tvec.tolist())
    gflops = world * cost / (f_max * 1e-3) / 1e9
    if batch:
        unit, value = "systems/s", total_systems / ((f_max + s_max) * 1e-3)
    else:
        unit, value = "GFLOP/s", gflops
    st = s.stats()
    launches = args.steps * (int(st.launches_factor) + int(st.launches_solve) * max(1, max(its) if its else 1))
    # host-side check of the last solution
    x_last = x_dev.cpu().numpy()
    x_last = x_last.T if nrhs > 1 else x_last
    if batch:
        host_bwd = prob.backward_error(x_last)
    else:
        host_bwd = P.backward_error(prob.n, prob.col, prob.row, prob.val, x_last, prob.rhs)

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
    e2e_tv = torch.tensor([statistics.mean(e2e_t)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(e2e_tv, op=dist.ReduceOp.MAX)
    e2e_s = float(e2e_tv.item())
    e2e_value = total_systems / e2e_s if batch else world * cost / e2e_s / 1e9

    # ---- roofline of the dominant kernel (per-launch events, graphs off) ----
    roof = None
    prof = None
    nprof = max(1, min(args.steps, 3))
    if not args.no_profile:
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
            peak = float(peaks.get("bf16_tflops_sustained", peaks.get("bf16_tflops", 1400.0)))
            roof = {"kernel": dom, "bound": "tensor", "achieved": round(d["flops"] / (d["ms"] * 1e-3) / 1e12, 3),
                    "peak": peak, "unit": "TFLOP/s", "peak_source": "MEASURED_PEAKS.json bf16 (sustained)"}
        else:
            peak = float(peaks.get("hbm_gbs", 6650.0))
            roof = {"kernel": dom, "bound": "hbm", "achieved": round(d["bytes"] / (d["ms"] * 1e-3) / 1e9, 1),
                    "peak": peak, "unit": "GB/s",
                    "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks else "fallback 6650 GB/s"}
        roof["frac"] = round(roof["achieved"] / roof["peak"], 4)
        tr = ncu_traffic(args.workload, dom, d["bytes"] / max(1, d["launches"]))
        roof["traffic"] = tr["bytes_per_launch"] if tr else None
        roof["traffic_source"] = tr if tr else "no ncu capture committed for this kernel and workload"
        roof["launches_per_step"] = d["launches"] // nprof
        roof["avg_launch_ms"] = round(per_launch_ms, 4)
        roof["algorithmic_per_launch"] = (d["flops"] if roof["bound"] == "tensor" else d["bytes"]) / max(1, d["launches"])
        roof["share_of_factor"] = round(d["ms"] / max(1e-9, sum(prof[k]["ms"] for k in fact_classes)), 3)

    # ---- CPU baseline (rank 0, N = 1) ----
    cpu = None
    if rank == 0 and world == 1 and args.cpu_baseline == "auto":
        threads = os.cpu_count() or 1
        try:
            if batch:
                r = cpu_reference_batch(prob, wl["max_zero"], threads, sample=200)
                cpu = {"value": round(r["systems_per_s"], 3), "unit": "systems/s", "cores": threads, "kind": "port",
                       "sample": f"factor + solve of the first {r['systems']} of the {prob.count} systems, one system "
                                 f"per thread (oracle, {'OpenBLAS' if r['blas'] else 'C loops'} tiles nb={r['nb']}), "
                                 f"{r['seconds']:.1f} s", "bwd_err": r["bwd"]}
            else:
                r = cpu_reference(prob, wl["max_zero"], 1, threads, nrhs_sample=min(nrhs, 2))
                fs = r["factor_s"][0]
                cpu = {"value": round(r["cost"] / fs / 1e9, 3), "unit": "GFLOP/s", "cores": threads, "kind": "port",
                       "sample": f"one full numeric factorization of the same workload (oracle, tree-level parallel, "
                                 f"{'OpenBLAS' if r['blas'] else 'C loops'} tiles nb={r['nb']}), {fs:.1f} s"
                                 + (f"; solve of {r['rhs_timed']} of {nrhs} RHS, scaled" if nrhs > 1 else ""),
                       "solve_ms": round(1e3 * r["solve_s"][0] * nrhs / r["rhs_timed"], 2), "bwd_err": r["bwd"]}
        except Exception as e:  # noqa: BLE001
            cpu = {"value": None, "unit": unit, "cores": threads, "kind": "port", "sample": f"failed: {e}"}

    if rank == 0:
        cfg = {"workload": wl["desc"], "name": args.workload, "n": prob.n, "nnz_lower": prob.nnz, "nrhs": nrhs,
               "fronts": int(st.num_front), "levels": int(st.num_level), "max_front": int(st.max_front),
               "cost_flops": cost, "nnz_L": int(st.nonzero), "nb": 10, "max_zero": wl["max_zero"],
               "ordering": "geometric nested dissection",
               "l2": "flushed (256 MiB write) between timed steps; working set > L2",
               "parallelism": (f"systems sharded over {world} GPU(s) by estimated cost, no collective" if batch
                               else f"{world} independent replica(s)")}
        if batch:
            cfg["systems"] = total_systems
        h2d = int(8 * prob.nnz + 8 * prob.n * nrhs)
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": unit, "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": round(f_max + s_max, 3), "higher_is_better": True,
            "scaling": "strong" if batch else "weak", "vs_baseline": None,
            "dtype": "f64" if wl["precision"] == 0 else "f32+f64ir",
            "data": "synthetic", "config": cfg,
            "factor_ms": round(f_max, 3), "factor_gflops": round(gflops, 3), "solve_ms": round(s_max, 3),
            "bwd_err": max(bwds), "bwd_err_host": host_bwd,
            "ir_iterations": max(its) if its else 0, "wall_ms_per_step": round(1e3 * wall_max / args.steps, 3),
            "setup_s": round(t_setup, 2),
            "clocks": clocks,
            "e2e": {"value": round(e2e_value, 3), "unit": unit, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": int(8 * prob.n * nrhs + 4), "ms_per_step": round(1e3 * e2e_s, 3),
                    "what": "mfd_factorize(pinned host A) + mfd_solve(pinned host b), wall clock"},
            "gpu_launches": launches,
            "roofline": roof,
            "cpu_baseline": cpu,
        }
        if prof is not None:
            line["kernel_profile_ms_per_step"] = {k: round(v["ms"] / nprof, 3) for k, v in prof.items() if v["launches"]}
        print(json.dumps(line), flush=True)
    s.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
