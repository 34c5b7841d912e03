"""Benchmark of the pull PageRank hot path (one JSON line on rank 0).

Workload (default): plain FP32 PageRank pull on a seeded R-MAT graph of
scale 22, edge factor 16 (a,b,c = 0.57,0.19,0.19; self loops and duplicates
removed; uint32 ids), damping 0.85, run to epsilon 1e-6 (iteration cap 100).
A step is one complete solve: init, pull passes until no vertex changes by
>= epsilon, normalisation.  The metric is GTEPS = edges x passes / time.

  value  device time of K solves, graph resident in HBM (CUDA events on the
         library stream); inputs (ids: 4 bytes x E > 126 MB L2) exceed L2.
  e2e    the same metric through the C ABI entry ag_pagerank_pull_ex with the
         graph in page-locked host memory: upload (H2D), plan, solve, ranks
         back (D2H) inside the timed region, host clock.
  roofline  algorithmic bytes of one pull pass (4E + 24N) / average pass time.
  cpu_baseline  the CPU oracle (restatement of the reference OpenMP pull) on a
         bounded number of passes of the same graph, all host threads.

--impl reference times that CPU restatement alone, as the reference arm.
--gpus N (torchrun): every rank solves its own graph (seed + rank), no data
exchange; value = all ranks' edges x passes / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "PR-pull GTEPS & % HBM roofline; time-to-1e-6: BF16/batched/warm vs plain, 1 GPU"
UNIT = "GTEPS"
SEED = 27491095


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--scale", type=int, default=22)
    p.add_argument("--edge-factor", type=int, default=16)
    p.add_argument("--epsilon", type=float, default=1e-6)
    p.add_argument("--iterations", type=int, default=300)
    p.add_argument("--precision", type=int, default=0)
    p.add_argument("--e2e-steps", type=int, default=3)
    p.add_argument("--cpu-seconds", type=float, default=12.0)
    p.add_argument("--no-cpu", action="store_true")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def reduce_time_work(seconds_or_ms: float, work: float, device=None):
    """Max of the timed region and sum of the work over all ranks (the
    whole-job rate is sum(work) / max(time)).  Identity without a process
    group."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(seconds_or_ms), float(work)
    t = torch.tensor([float(seconds_or_ms)], dtype=torch.float64, device=device)
    w = torch.tensor([float(work)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(w, op=dist.ReduceOp.SUM)
    return float(t.item()), float(w.item())


def workload_config(a, world):
    return {
        "workload": f"PageRank pull FP32, RMAT scale {a.scale} edge factor {a.edge_factor} "
                    f"(a,b,c=0.57,0.19,0.19, dedup, no self loops), d=0.85, eps={a.epsilon:g}, cap {a.iterations}",
        "graph": f"rmat{a.scale}_ef{a.edge_factor}",
        "epsilon": a.epsilon,
        "iteration_cap": a.iterations,
        "precision": ["fp32", "bf16", "fp16"][a.precision],
        "l2": "inputs larger than L2 (neighbour ids 4E bytes > 126 MB)",
        "parallelism": f"replicas{world}" if world > 1 else "single",
    }


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index: int):
        self.proc = None
        self.path = Path("/tmp") / f"ag_clocks_{os.getpid()}.csv"
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        self.path.unlink(missing_ok=True)
        if not sm:
            return None
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": max(mx), "samples": len(sm), "reasons": sorted(reasons)}


def peak_hbm():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def cpu_sample(oracle, g, a, seconds):
    """Time the CPU oracle (all host threads) on whole passes of the same
    graph, about `seconds` of work."""
    args = (g.in_edges_idx(), g.in_degree(), g.in_neighbours(), g.out_degree())
    one = oracle.pagerank_pull(*args, iterations=1, epsilon=a.epsilon)
    t1 = float(one["seconds"][0])
    k = int(max(1, min(a.iterations, seconds / max(t1, 1e-6))))
    res = oracle.pagerank_pull(*args, iterations=k, epsilon=a.epsilon)
    t = float(res["seconds"].sum())
    passes = int(res["passes"])
    return {
        "value": g.num_edges * passes / t / 1e9,
        "unit": UNIT,
        "cores": oracle.max_threads(),
        "kind": "port",
        "sample": f"{passes} PageRank-pull passes of the same RMAT s{a.scale} graph "
                  f"({t:.1f} s), per-pass timers as in pageRank.c:1025,1071",
        "seconds_per_pass": t / passes,
    }


def run_reference(a):
    rank, world, local = dist_env()
    if rank != 0:
        return
    import accelgraph_b200 as ag
    import oracle
    g = ag.Graph.rmat(a.scale, a.edge_factor, seed=SEED)
    args = (g.in_edges_idx(), g.in_degree(), g.in_neighbours(), g.out_degree())
    one = oracle.pagerank_pull(*args, iterations=1, epsilon=a.epsilon)
    t1 = float(one["seconds"][0])
    budget = min(10.0, 150.0 / max(1, a.steps + a.warmup))
    per_step = int(max(1, min(a.iterations, budget / max(t1, 1e-6))))
    for _ in range(a.warmup):
        oracle.pagerank_pull(*args, iterations=per_step, epsilon=a.epsilon)
    tot_t, tot_p = 0.0, 0
    for _ in range(a.steps):
        t0 = time.perf_counter()
        r = oracle.pagerank_pull(*args, iterations=per_step, epsilon=a.epsilon)
        tot_t += time.perf_counter() - t0
        tot_p += int(r["passes"])
    value = g.num_edges * tot_p / tot_t / 1e9
    cores = oracle.max_threads()
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": 1e3 * tot_t / a.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(a, 1),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{per_step} passes per step of the C/OpenMP restatement of "
                                   f"pageRankPullGraphCSR on RMAT s{a.scale} ef{a.edge_factor}"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "num_vertices": g.num_vertices, "num_edges": g.num_edges,
    }
    print(json.dumps(line), flush=True)


def run_b200(a):
    import numpy as np
    import torch

    rank, world, local = dist_env()
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    import accelgraph_b200 as ag
    ag.check(ag.lib.ag_init(local), "ag_init")
    stream = torch.cuda.ExternalStream(ag.lib.ag_stream(), device=torch.device("cuda", local))

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    seed = SEED + rank
    g = ag.Graph.rmat(a.scale, a.edge_factor, seed=seed, flags=ag.AG_BUILD_DEDUPE | ag.AG_BUILD_PINNED)
    N, E = g.num_vertices, g.num_edges
    dg = ag.DeviceGraph(g)
    info = dg.info()

    # -------- device-resident solves (value)
    for _ in range(a.warmup):
        dg.launch(a.iterations, a.epsilon, precision=a.precision)
    ranks_w, res_w, _ = dg.fetch()
    barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(a.steps):
        dg.launch(a.iterations, a.epsilon, precision=a.precision)
    ev1.record(stream)
    ev1.synchronize()
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    ranks, res, hist = dg.fetch(history=a.iterations)
    passes = int(res.passes)
    edges_all = E * passes * a.steps
    t_max, edges_all = reduce_time_work(ms, edges_all, device="cuda")
    value = edges_all / (t_max * 1e-3) / 1e9

    # -------- roofline of the pull pass
    alg_bytes = 4 * E + 24 * N
    if a.precision:
        alg_bytes = 4 * E + 20 * N
    pass_s = (ms * 1e-3) / (a.steps * max(passes, 1))
    peak, peak_kind = peak_hbm()
    dev_pass = np.diff(np.concatenate([[0.0], np.cumsum(hist["seconds"])]))
    achieved = alg_bytes / pass_s / 1e9
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": None, "peak_kind": peak_kind, "kernel": "ag_pull_kernel<PR,fp32,fast>",
            "bytes_per_pass": alg_bytes, "pass_us": pass_s * 1e6,
            "pass_us_device_timer_median": float(np.median(dev_pass[1:]) * 1e6) if len(dev_pass) > 1 else None}
    traffic_file = ROOT / "profiles" / "traffic.json"
    if traffic_file.exists():
        try:
            tr = json.loads(traffic_file.read_text())
            key = f"rmat{a.scale}_ef{a.edge_factor}"
            if key in tr:
                roof["traffic"] = tr[key]["dram_bytes_per_pass"]
        except Exception:
            pass

    # -------- end to end through the C ABI (host buffers, pinned)
    args = ag.default_arguments(a.iterations, a.epsilon)
    opts = ag.make_opts(precision=a.precision, quiet=True)
    out = C.POINTER(ag.PageRankStats)()
    ag.check(ag.lib.ag_pagerank_pull_ex(C.byref(args), g.ptr, C.byref(opts), C.byref(out)), "e2e warmup")
    ag.lib.freePageRankStats(out)
    barrier()
    t0 = time.perf_counter()
    e2e_passes = 0
    for _ in range(a.e2e_steps):
        ag.check(ag.lib.ag_pagerank_pull_ex(C.byref(args), g.ptr, C.byref(opts), C.byref(out)), "e2e")
        e2e_passes += int(out.contents.iterations) + (1 if out.contents.iterations < a.iterations else 0)
        ag.lib.freePageRankStats(out)
    torch.cuda.synchronize()
    e2e_t = time.perf_counter() - t0
    e2e_t, e2e_edges = reduce_time_work(e2e_t, float(E * e2e_passes), device="cuda")
    e4 = ((E + 3) & ~3) + 4
    h2d = 4 * e4 + 4 * (N + 1) + 4 * N + 16 * info.num_tasks
    d2h = 4 * N
    e2e = {"value": e2e_edges / e2e_t / 1e9, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
           "ms_per_step": 1e3 * e2e_t / a.e2e_steps, "api": "ag_pagerank_pull_ex (pageRankPullGraphCSR semantics)"}

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        import oracle
        cpu = cpu_sample(oracle, g, a, a.cpu_seconds)

    launches = a.steps * (passes + 2)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": t_max / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic", "config": workload_config(a, world),
        "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk, "gpu_launches": launches,
        "passes_per_solve": passes, "iterations": int(res.iterations), "converged": int(res.converged),
        "num_vertices": N, "num_edges": E, "tasks": info.num_tasks, "grid": info.grid,
        "hub_rows": info.num_hub_rows,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    dg.release()
    if world > 1:
        torch.distributed.destroy_process_group()


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    else:
        run_b200(a)


if __name__ == "__main__":
    main()
