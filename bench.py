"""Benchmark of the pull PageRank hot path (one JSON line on rank 0).

Workload (default): PageRank pull on a seeded R-MAT graph of scale 24, edge
factor 16 (a,b,c = 0.57,0.19,0.19; self loops and duplicates removed; uint32
ids; 16,777,216 vertices, about 2.6e8 in-edges), damping 0.85, run to epsilon
1e-6 (iteration cap 300), in EXACT order: every row is summed in the reference
loop's stream order, so ranks, per-pass active counts and the iteration count
are the reference's bit for bit.  A step is one complete solve: init, pull
passes until no vertex changes by >= epsilon, normalisation.  The metric is
GTEPS = edges x passes / time.

  value  device time of K solves, graph resident in HBM (CUDA events on the
         library stream); inputs (ids: 4 bytes x E > 126 MB L2) exceed L2.
  e2e    the same metric through the C ABI entry ag_pagerank_pull_ex with the
         graph in page-locked host memory: upload (H2D), plan, solve, ranks
         back (D2H) inside the timed region, host clock.
  roofline  algorithmic bytes of one pull pass (4E + 24N) / average pass
         time; traffic from the committed ncu summary of the same kernel and
         graph, named in traffic_source.
  parity  the CPU oracle solved on the same graph: iteration counts, per-pass
         active counts, bit-exactness and relative L1 of the ranks; relative L1
         against the FP64 fixpoint (GPU FP64 kernels).
  cpu_baseline  that oracle solve (restatement of the reference OpenMP pull,
         all host threads), timed.

--order fast sums rows of more than 32 in-edges in a fixed tree order (ranks
within 1e-5 relative L1, iteration count not guaranteed equal).
--impl reference times the CPU restatement alone, as the reference arm, on a
graph built by the oracle's own generator (the product library is not loaded).
--gpus N (torchrun): by default every rank solves its own graph (seed + rank),
no data exchange, value = all ranks' edges x passes / max-over-ranks time
(weak scaling); --mode rows splits one graph by rows across the ranks with
an all-gather of contributions per pass (strong scaling).
--workload selects the other forms (SpMV, precision, PPR, many graphs, warm
start); each prints its own JSON line.
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
    p.add_argument("--scale", type=int, default=24)
    p.add_argument("--edge-factor", type=int, default=16)
    p.add_argument("--epsilon", type=float, default=1e-6)
    p.add_argument("--iterations", type=int, default=300)
    p.add_argument("--precision", type=int, default=0)
    p.add_argument("--order", default="exact", choices=["fast", "exact"],
                   help="pagerank: summation order (exact = the reference loop's, bit for bit)")
    p.add_argument("--e2e-steps", type=int, default=3)
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--workload", default="pagerank",
                   choices=["pagerank", "spmv", "precision", "ppr", "multigraph", "warmstart", "gather-probe",
                            "data-driven", "fixed-point", "push"],
                   help="pagerank: the headline line (driver contract); the others measure the other forms")
    p.add_argument("--graphs", type=int, default=256, help="multigraph: number of graphs")
    p.add_argument("--train-graphs", type=int, default=200, help="warmstart: training graphs")
    p.add_argument("--k", type=int, default=64, help="ppr: sources")
    p.add_argument("--mode", default="replicas", choices=["replicas", "rows"],
                   help="N > 1: independent graphs per rank (replicas) or one graph split by rows (rows)")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def profiled_traffic(scale: int, edge_factor: int, order: str):
    """DRAM bytes (read + write) of one pull pass of this kernel and graph from
    the committed ncu summary profiles/ag_pull_kernel_<order>_rmat<scale>.md
    (row `dram__bytes_read.sum + write | R + W MB`), with the file it came
    from; (None, None) without one."""
    import re
    name = f"profiles/ag_pull_kernel_{order}_rmat{scale}.md"
    f = ROOT / name
    if edge_factor != 16 or not f.exists():
        return None, None
    m = re.search(r"\|\s*dram__bytes_read\.sum \+ write\s*\|\s*([0-9.]+) \+ ([0-9.]+) MB", f.read_text())
    if not m:
        return None, None
    return (float(m.group(1)) + float(m.group(2))) * 1e6, name


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
    order = ("EXACT order (stream-order row sums, bit-identical to the reference loop)" if a.order == "exact"
             else "FAST order (rows over 32 in-edges summed in a fixed tree)")
    return {
        "workload": f"PageRank pull FP32, {order}, RMAT scale {a.scale} edge factor {a.edge_factor} "
                    f"(a,b,c=0.57,0.19,0.19, dedup, no self loops), d=0.85, eps={a.epsilon:g}, cap {a.iterations}",
        "graph": f"rmat{a.scale}_ef{a.edge_factor}",
        "epsilon": a.epsilon,
        "iteration_cap": a.iterations,
        "precision": ["fp32", "bf16", "fp16"][a.precision],
        "order": a.order,
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


def oracle_solve(oracle, arrays, a):
    """The CPU oracle's complete solve of the same graph (all host threads),
    timed: the reported CPU baseline and the parity reference."""
    in_idx, in_deg, in_nb, out_deg = arrays
    t0 = time.perf_counter()
    ref = oracle.pagerank_pull(in_idx, in_deg, in_nb, out_deg, iterations=a.iterations, epsilon=a.epsilon)
    ref["wall_s"] = time.perf_counter() - t0
    return ref


def cpu_baseline(ref, num_edges, a, oracle):
    t = float(ref["seconds"].sum())
    passes = int(ref["passes"])
    return {
        "value": num_edges * passes / t / 1e9,
        "unit": UNIT,
        "cores": oracle.max_threads(),
        "kind": "port",
        "sample": f"one complete solve ({passes} passes to eps {a.epsilon:g}, {t:.1f} s) of the same RMAT "
                  f"s{a.scale} graph by the C/OpenMP restatement of pageRankPullGraphCSR, per-pass timers "
                  f"as in pageRank.c:1025,1071",
        "seconds_per_pass": t / passes,
    }


def run_reference(a):
    """The reference arm: the oracle (C/OpenMP restatement of the reference's
    pull) on all host threads, on a graph built by the oracle's own
    generator; the product library is not loaded."""
    rank, world, local = dist_env()
    if rank != 0:
        return
    import oracle
    gr = oracle.rmat_inverse(a.scale, a.edge_factor, SEED)
    args = (gr["in_idx"], gr["in_deg"], gr["in_nb"], gr["out_deg"])
    E = gr["num_edges"]
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
    value = E * tot_p / tot_t / 1e9
    cores = oracle.max_threads()
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": 1e3 * tot_t / a.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(a, 1),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"up to {per_step} passes per step (a step stops at epsilon) of the C/OpenMP "
                                   f"restatement of pageRankPullGraphCSR on RMAT s{a.scale} ef{a.edge_factor}"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "num_vertices": 1 << a.scale, "num_edges": E,
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
    order = ag.AG_ORDER_EXACT if a.order == "exact" else ag.AG_ORDER_FAST
    for _ in range(a.warmup):
        dg.launch(a.iterations, a.epsilon, precision=a.precision, order=order)
    ranks_w, res_w, _ = dg.fetch()
    barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(a.steps):
        dg.launch(a.iterations, a.epsilon, precision=a.precision, order=order)
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
            "traffic": None, "peak_kind": peak_kind, "kernel": "ag_pull_kernel<PR,fp32,%s>" % a.order,
            "bytes_per_pass": alg_bytes, "pass_us": pass_s * 1e6,
            "pass_us_device_timer_median": float(np.median(dev_pass[1:]) * 1e6) if len(dev_pass) > 1 else None}
    if a.precision == 0:
        roof["traffic"], roof["traffic_source"] = profiled_traffic(a.scale, a.edge_factor, a.order)

    # -------- end to end through the C ABI (host buffers, pinned)
    args = ag.default_arguments(a.iterations, a.epsilon)
    opts = ag.make_opts(precision=a.precision, order=order, quiet=True)
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
    # copied per step: in-neighbour ids (E rounded to 4, plus 4), row starts,
    # out-degrees; the work lists are planned on the device
    h2d = 4 * e4 + 4 * (N + 1) + 4 * N
    d2h = 4 * N
    e2e = {"value": e2e_edges / e2e_t / 1e9, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
           "ms_per_step": 1e3 * e2e_t / a.e2e_steps, "api": "ag_pagerank_pull_ex (pageRankPullGraphCSR semantics)"}

    # -------- CPU oracle on the same graph: baseline and parity
    cpu = parity = None
    if rank == 0 and world == 1 and not a.no_cpu:
        import oracle
        ref = oracle_solve(oracle, (g.in_edges_idx(), g.in_degree(), g.in_neighbours(), g.out_degree()), a)
        cpu = cpu_baseline(ref, E, a, oracle)
        r64, p64 = dg.pagerank_f64(5000, 1e-13)
        ra = ranks.astype(np.float64)
        dref = np.abs(ra - ref["ranks"])
        n_hist = min(len(hist["active"]), len(ref["active"]))
        parity = {
            "iterations": int(res.iterations), "iterations_oracle": int(ref["iterations"]),
            "passes": passes, "passes_oracle": int(ref["passes"]),
            "active_per_pass_equal": bool(passes == int(ref["passes"]) and
                                          np.array_equal(hist["active"][:n_hist], ref["active"][:n_hist])),
            "ranks_bit_exact": bool(np.array_equal(ranks.view(np.uint32), ref["ranks"].view(np.uint32))),
            "rel_l1_vs_oracle": float(dref.sum() / np.abs(ref["ranks"]).sum()),
            "max_abs_vs_oracle": float(dref.max()),
            "rel_l1_vs_fp64": float(np.abs(ra - r64).sum() / np.abs(r64).sum()),
            "max_abs_vs_fp64": float(np.abs(ra - r64).max()),
            "oracle_rel_l1_vs_fp64": float(np.abs(ref["ranks"] - r64).sum() / np.abs(r64).sum()),
            "fp64_passes": int(p64),
            "oracle": "C/OpenMP restatement of pageRankPullGraphCSR (pageRank.c:942-1109), same graph",
        }

    launches = a.steps * (passes + 2)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": t_max / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic", "config": workload_config(a, world),
        "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "parity": parity, "clocks": clk,
        "gpu_launches": launches,
        "passes_per_solve": passes, "iterations": int(res.iterations), "converged": int(res.converged),
        "num_vertices": N, "num_edges": E, "tasks": info.num_tasks, "grid": info.grid,
        "hub_rows": info.num_hub_rows,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    dg.release()
    if world > 1:
        torch.distributed.destroy_process_group()


# ---------------------------------------------------------------- forms
def _gpu_setup():
    import torch
    import accelgraph_b200 as ag
    torch.cuda.set_device(0)
    ag.check(ag.lib.ag_init(0), "ag_init")
    return ag


def _rel(a, b):
    import numpy as np
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300)), float(np.abs(a - b).max())


def run_spmv(a):
    """SpMV pull, FP32 weights and x uniform in [0,1), one multiply per edge."""
    import torch
    ag = _gpu_setup()
    g = ag.Graph.rmat(a.scale, a.edge_factor, seed=SEED, flags=ag.AG_BUILD_DEDUPE | ag.AG_BUILD_WEIGHTS)
    N, E = g.num_vertices, g.num_edges
    dg = ag.DeviceGraph(g, weights=True)
    x = torch.empty(N, dtype=torch.float32, device="cuda")
    y = torch.empty(N, dtype=torch.float32, device="cuda")
    xh = __import__("numpy").empty(N, "float32")
    ag.lib.ag_fill_uniform(xh.ctypes.data_as(ag.f32p), N, SEED + 1)
    x.copy_(torch.from_numpy(xh))
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(ag.lib.ag_stream(), device=torch.device("cuda", 0))
    import numpy as np
    import oracle
    yo = oracle.spmv_pull(g.in_edges_idx(), g.in_degree(), g.in_neighbours(), g.in_weights(), xh)
    peak, kind = peak_hbm()
    alg = 8 * E + 12 * N
    out = {"workload": f"spmv pull FP32 weighted, RMAT s{a.scale} ef{a.edge_factor}", "N": N, "E": E}
    # FAST: rows over 32 in-edges in a fixed tree; EXACT: stream order, the
    # reference's bits (what SPMVPullGraphCSR runs)
    for name, mode in (("fast", 0), ("exact", ag.AG_SPMV_EXACT)):
        for _ in range(a.warmup):
            ag.check(ag.lib.ag_spmv_pull_device(dg.h, x.data_ptr(), y.data_ptr(), mode), "spmv")
        ag.lib.ag_synchronize(0.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(a.steps * 10):
            ag.check(ag.lib.ag_spmv_pull_device(dg.h, x.data_ptr(), y.data_ptr(), mode), "spmv")
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / (a.steps * 10)
        yh = y.cpu().numpy()
        rl, mx = _rel(yh, yo)
        out[name] = {"ms_per_product": ms, "gteps": E / ms / 1e6,
                     "roofline": {"bytes": alg, "achieved_gbs": alg / ms / 1e6, "peak": peak,
                                  "frac": alg / ms / 1e6 / peak, "peak_kind": kind},
                     "rel_l1_vs_oracle": rl, "max_abs_vs_oracle": mx,
                     "bit_exact_vs_oracle": bool(np.array_equal(yh.view(np.uint32), yo.view(np.uint32)))}
    print(json.dumps(out), flush=True)


def run_precision(a):
    """Time to epsilon and error against the FP64 GPU oracle: FP32 plain vs the
    BF16 and FP16 contribution forms (switching to FP32 storage)."""
    import numpy as np
    ag = _gpu_setup()
    g = ag.Graph.rmat(a.scale, a.edge_factor, seed=SEED)
    N, E = g.num_vertices, g.num_edges
    dg = ag.DeviceGraph(g)
    r64, p64 = dg.pagerank_f64(5000, 1e-13)
    out = {"workload": f"PageRank pull to eps {a.epsilon:g}, RMAT s{a.scale} ef{a.edge_factor}", "N": N, "E": E,
           "fp64_passes": p64}
    peak, kind = peak_hbm()
    for name, prec in (("fp32", 0), ("bf16", 1), ("fp16", 2)):
        dg.launch(a.iterations, a.epsilon, precision=prec)
        dg.fetch()
        best = None
        for _ in range(max(1, a.steps)):
            r, res, hist = dg.pagerank(a.iterations, a.epsilon, precision=prec, history=a.iterations)
            if best is None or res.device_ms < best[1].device_ms:
                best = (r, res, hist)
        r, res, hist = best
        rl, mx = _rel(r, r64)
        alg = 4 * E + (24 if prec == 0 else 20) * N
        # per-pass device timer: the passes that read 16-bit contributions and
        # those after the switch to FP32 (the first pass includes the init)
        sec = hist["seconds"] * 1e6
        sw = res.switch_pass if prec else 0
        low = sec[1:sw] if sw > 1 else sec[:0]
        high = sec[max(sw, 1):]
        out[name] = {"device_ms_to_eps": res.device_ms, "passes": res.passes, "iterations": res.iterations,
                     "switch_pass": res.switch_pass, "rel_l1_vs_fp64": rl, "max_abs_vs_fp64": mx,
                     "pass_us": res.device_ms * 1e3 / res.passes,
                     "pass_us_median_16bit": float(np.median(low)) if len(low) else None,
                     "pass_us_median_fp32": float(np.median(high)) if len(high) else None,
                     "roofline_frac": alg / (res.device_ms * 1e-3 / res.passes) / 1e9 / peak}
    out["speedup_vs_fp32"] = {k: out["fp32"]["device_ms_to_eps"] / out[k]["device_ms_to_eps"]
                              for k in ("bf16", "fp16")}
    print(json.dumps(out), flush=True)


def run_ppr(a):
    """k personalized PageRanks as one SpMM per pass (Erdos-Renyi, avg degree
    16) vs solving the same graph's plain PageRank once per source."""
    import numpy as np
    ag = _gpu_setup()
    n = 1 << a.scale
    g = ag.Graph.er(n, 16, seed=SEED)
    N, E = g.num_vertices, g.num_edges
    dg = ag.DeviceGraph(g)
    rng = np.random.default_rng(SEED + 1000)
    src = rng.choice(N, size=a.k, replace=False).astype(np.uint32)
    dg.ppr(src[:2], iterations=3, epsilon=a.epsilon, want_ranks=False)
    _, res = dg.ppr(src, iterations=a.iterations, epsilon=a.epsilon, want_ranks=False)
    dg.launch(a.iterations, a.epsilon)
    dg.fetch()
    _, res1, _ = dg.pagerank(a.iterations, a.epsilon)
    peak, kind = peak_hbm()
    alg = 4 * E + 8 * N + 16 * a.k * N
    # the contribution matrix (N x 256 bytes) is far larger than L2, so every
    # in-edge's 256-byte row gather comes from HBM
    moved = 4 * E + 8 * N + 256 * E + 12 * 64 * N
    print(json.dumps({"workload": f"personalized PageRank, k={a.k} sources, ER n=2^{a.scale} avg degree 16",
                      "N": N, "E": E, "ppr_passes": res.passes, "ppr_device_ms": res.device_ms,
                      "ppr_ms_per_pass": res.device_ms / max(res.passes, 1),
                      "gteps_all_sources": a.k * E * res.passes / res.device_ms / 1e6,
                      "per_source_ms": res.device_ms / a.k,
                      "plain_single_ms": res1.device_ms, "plain_single_passes": res1.passes,
                      "speedup_per_source_vs_plain": res1.device_ms / (res.device_ms / a.k),
                      "roofline_model_frac": alg / (res.device_ms * 1e-3 / res.passes) / 1e9 / peak,
                      "gathered_row_bytes_per_pass": 256 * E,
                      "hbm_bytes_per_pass_with_row_gathers": moved,
                      "hbm_frac_with_row_gathers": moved / (res.device_ms * 1e-3 / res.passes) / 1e9 / peak,
                      "peak_gbs": peak, "peak_kind": kind}), flush=True)


def run_multigraph(a):
    """Many uneven R-MAT graphs in one launch vs one launch per graph."""
    import numpy as np
    ag = _gpu_setup()
    rng = np.random.default_rng(SEED + 2)
    gs = []
    for i in range(a.graphs):
        gs.append(ag.Graph.rmat(int(rng.integers(10, 17)), int(rng.integers(8, 33)), seed=SEED + 10 + i))
    E = sum(g.num_edges for g in gs)
    mg = ag.MultiGraph(gs)
    best, us = mg.autotune(passes=6)
    mg.pagerank(a.iterations, a.epsilon)
    parts, info = mg.pagerank(a.iterations, a.epsilon)
    one_ms = info["device_ms"]
    seq_ms = 0.0
    seq_passes = 0
    for g in gs:
        dg = ag.DeviceGraph(g)
        dg.pagerank(a.iterations, a.epsilon)
        _, res, _ = dg.pagerank(a.iterations, a.epsilon)
        seq_ms += res.device_ms
        seq_passes += res.passes
        dg.release()
    print(json.dumps({"workload": f"{a.graphs} R-MAT graphs, scale U[10,16], edge factor U[8,32], eps {a.epsilon:g}",
                      "total_edges": E, "union_device_ms": one_ms, "union_passes": int(info["passes"].max()),
                      "sequential_device_ms": seq_ms, "speedup": seq_ms / one_ms,
                      "edge_passes": int(sum(g.num_edges * int(p) for g, p in zip(gs, info["passes"]))),
                      "gteps_union": sum(g.num_edges * int(p) for g, p in zip(gs, info["passes"])) / one_ms / 1e6,
                      "all_converged": bool(info["converged"].all()),
                      "tiles": {"task_edges": best.task_edges, "hub_chunk": best.hub_chunk}}), flush=True)


def run_warmstart(a):
    """Train the warm-start MLP on this GPU's PageRank results of seeded
    graphs (scales 14-18), evaluate on a held-out RMAT graph: passes and time
    to epsilon from the prediction against the uniform start, the prediction's
    cost split into features and MLP (SIMT and tensor-core), the pass saving
    its accuracy allows at most, and the warm start combined with the
    data-driven pull and with BF16 contributions."""
    import math
    import time
    import numpy as np
    import torch
    ag = _gpu_setup()
    from accelgraph_b200 import warmstart as ws
    t0 = time.perf_counter()
    specs = ws.training_graph_specs(count=a.train_graphs, scales=(14, 18), seed=SEED)
    X, T = ws.build_training_set(specs, per_graph=4096)
    t_data = time.perf_counter() - t0
    m = ws.MLP(seed=1)
    _, loss0 = m.gradients(X, T)
    t1 = time.perf_counter()
    loss = m.train(X, T, epochs=60, batch=4096, lr=2e-3)
    t_train = time.perf_counter() - t1
    g = ag.Graph.rmat(a.scale, a.edge_factor, seed=9999)
    dg = ag.DeviceGraph(g)
    ws.compare(dg, m, a.iterations, a.epsilon)
    c = ws.compare(dg, m, a.iterations, a.epsilon)
    r64, _ = dg.pagerank_f64(5000, 1e-13)
    eu = _rel(c["ranks_uniform"], r64)
    ew = _rel(c["ranks_warm"], r64)
    ei = _rel(c["init"] / g.num_vertices, r64)
    e0 = _rel(np.full(g.num_vertices, (1.0 - 0.85) / g.num_vertices, np.float32), r64)

    # the prediction's parts, timed on the library stream
    stream = torch.cuda.ExternalStream(ag.lib.ag_stream(), device=torch.device("cuda", 0))

    def timed(fn, reps=5):
        fn()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(reps):
            fn()
        ev1.record(stream)
        ev1.synchronize()
        return ev0.elapsed_time(ev1) / reps

    n = g.num_vertices
    Xf = torch.empty((n, 8), dtype=torch.float32, device="cuda")
    Yf = torch.empty(n, dtype=torch.float32, device="cuda")
    t_feat = timed(lambda: ag.check(ag.lib.ag_features(dg.h, Xf.data_ptr()), "ag_features"))
    t_simt = timed(lambda: ag.check(ag.lib.ag_mlp_forward(m.h, Xf.data_ptr(), n, Yf.data_ptr()), "forward"))
    t_tc = timed(lambda: ag.check(ag.lib.ag_mlp_predict(m.h, Xf.data_ptr(), n, Yf.data_ptr()), "predict"))
    mlp_flops = 2.0 * (8 * 64 + 64 * 64 + 64) * n

    # what a warm start can give: each pass costs the same whatever the start,
    # so halving the time to eps means skipping half the passes.  The measured
    # saving per e-fold of start error (passes saved / ln(e_uniform / e_pred))
    # extrapolates to the start error that would skip half of them; the
    # asymptotic rate (the error shrinks by the damping factor per pass) asks
    # for far more.  `free` is the speed-up if the prediction cost nothing.
    t_u = c["uniform"]["device_ms"]
    half = c["uniform"]["passes"] / 2.0
    saved = c["uniform"]["passes"] - c["warm"]["passes"]
    gain = math.log(e0[0] / max(ei[0], 1e-300))
    slope = saved / gain if gain > 0 else 0.0
    need = e0[0] * math.exp(-half / slope) if slope > 0 else 0.0
    need_asym = e0[0] * 0.85 ** half
    free = t_u / c["warm"]["device_ms"]

    # combined forms from the same prediction
    init = torch.from_numpy(c["init"]).cuda()
    comb = {}
    for name, kw in (("warm_dd", {"data_driven": True}), ("warm_bf16", {"precision": ag.AG_PREC_BF16}),
                     ("dd", {"data_driven": True, "init": False}), ("bf16", {"precision": ag.AG_PREC_BF16,
                                                                            "init": False})):
        use_init = kw.pop("init", True)
        r, res, _ = dg.pagerank(a.iterations, a.epsilon, init_ranks=init if use_init else None, **kw)
        r, res, _ = dg.pagerank(a.iterations, a.epsilon, init_ranks=init if use_init else None, **kw)
        ms = res.device_ms + (c["warm"]["predict_ms"] if use_init else 0.0)
        comb[name] = {"passes": res.passes, "ms_to_eps": ms, "speedup_vs_uniform_fp32": t_u / ms,
                      "rel_l1_vs_fp64": _rel(r, r64)[0]}
    print(json.dumps({"workload": f"learned warm start, eval RMAT s{a.scale} ef{a.edge_factor} (seed 9999), "
                                  f"trained on {a.train_graphs} graphs s14-18", "N": g.num_vertices,
                      "E": g.num_edges, "train_samples": int(X.shape[0]), "loss_initial": loss0,
                      "loss_final": loss, "data_s": t_data, "train_s": t_train,
                      "uniform": c["uniform"], "warm": c["warm"],
                      "speedup_time_to_eps": c["uniform"]["device_ms"] / (c["warm"]["device_ms"] +
                                                                          c["warm"]["predict_ms"]),
                      "predict_breakdown_ms": {"features": t_feat, "mlp_simt_fp32": t_simt,
                                               "mlp_tensor_core": t_tc,
                                               "mlp_tensor_core_tflops": mlp_flops / (t_tc * 1e-3) / 1e12,
                                               "mlp_simt_tflops": mlp_flops / (t_simt * 1e-3) / 1e12},
                      "bound": {"rel_l1_uniform_start": e0[0], "rel_l1_prediction": ei[0],
                                "passes_saved_measured": c["uniform"]["passes"] - c["warm"]["passes"],
                                "passes_to_skip_for_2x": half,
                                "passes_saved_per_efold_of_start_error": slope,
                                "start_rel_l1_needed_for_2x": need,
                                "start_rel_l1_needed_for_2x_at_damping_rate": need_asym,
                                "speedup_with_a_free_prediction": free},
                      "combined": comb,
                      "rel_l1_vs_fp64": {"uniform": eu[0], "warm": ew[0], "prediction_alone": ei[0]}}),
          flush=True)


def run_data_driven(a):
    """Data-driven (worklist) pull, the reference's pushpull 6, against the
    topology-driven pull on the same graph: time to epsilon on the device,
    passes, accuracy against the FP64 fixpoint, and the CPU oracle of the
    worklist pull (all host threads) on the same graph."""
    import time
    import oracle
    ag = _gpu_setup()
    g = ag.Graph.rmat(a.scale, a.edge_factor, seed=SEED)
    N, E = g.num_vertices, g.num_edges
    dg = ag.DeviceGraph(g)
    r64, _ = dg.pagerank_f64(5000, 1e-13)
    out = {"workload": f"data-driven PageRank pull to eps {a.epsilon:g}, RMAT s{a.scale} ef{a.edge_factor}",
           "N": N, "E": E}
    for name, dd in (("topology", False), ("data_driven", True)):
        dg.pagerank(a.iterations, a.epsilon, data_driven=dd)
        best = None
        for _ in range(max(1, a.steps)):
            r, res, _ = dg.pagerank(a.iterations, a.epsilon, data_driven=dd)
            if best is None or res.device_ms < best[1].device_ms:
                best = (r, res)
        r, res = best
        rl, mx = _rel(r, r64)
        out[name] = {"device_ms_to_eps": res.device_ms, "passes": res.passes, "iterations": res.iterations,
                     "rel_l1_vs_fp64": rl, "max_abs_vs_fp64": mx}
    out["speedup_vs_topology"] = out["topology"]["device_ms_to_eps"] / out["data_driven"]["device_ms_to_eps"]
    t0 = time.perf_counter()
    ref = oracle.pagerank_dd(g.in_edges_idx(), g.in_degree(), g.in_neighbours(), g.out_edges_idx(),
                             g.out_degree(), g.out_neighbours(), a.iterations, a.epsilon)
    out["cpu_oracle"] = {"seconds_to_eps": time.perf_counter() - t0, "iterations": ref["iterations"],
                         "threads": oracle.lib.oracle_max_threads()}
    print(json.dumps(out), flush=True)


def run_fixed_point(a):
    """The reference's integer pulls against the FP32 pull on the same graph:
    64/32/16/8-bit fixed point (pushpull 2, 9, 10, 11) and 32/16/8-bit
    quantised (pushpull 4, 12, 13).  Per form: time to epsilon on the device,
    passes, pass time against the HBM roofline, accuracy against the FP64
    fixpoint, and the CPU oracle of the same form."""
    import time
    import oracle
    ag = _gpu_setup()
    g = ag.Graph.rmat(a.scale, a.edge_factor, seed=SEED)
    N, E = g.num_vertices, g.num_edges
    dg = ag.DeviceGraph(g)
    r64, _ = dg.pagerank_f64(5000, 1e-13)
    peak, kind = peak_hbm()
    out = {"workload": f"integer PageRank pulls to eps {a.epsilon:g}, RMAT s{a.scale} ef{a.edge_factor}",
           "N": N, "E": E, "peak_gbs": peak, "peak_kind": kind,
           "bytes_per_pass": "fixed W: 4E + (16 + 2 W/8) N; quantised W: 4E + (24 + 2 W/8) N "
                             "(pull 4E + (20 + W/8) N, quantiser 4N + W/8 N); FP32: 4E + 24N"}
    forms = (("fp32", ag.AG_PREC_FP32), ("fixed64", ag.AG_PREC_FIXED64), ("fixed32", ag.AG_PREC_FIXED32),
             ("fixed16", ag.AG_PREC_FIXED16), ("fixed8", ag.AG_PREC_FIXED8), ("quant32", ag.AG_PREC_QUANT32),
             ("quant16", ag.AG_PREC_QUANT16), ("quant8", ag.AG_PREC_QUANT8))
    for name, prec in forms:
        quant, width = ag.NARROW_FORM.get(prec, (False, 64 if prec == ag.AG_PREC_FIXED64 else 32))
        cb = width // 8
        dg.pagerank(a.iterations, a.epsilon, precision=prec)
        best = None
        for _ in range(max(1, a.steps)):
            r, res, _ = dg.pagerank(a.iterations, a.epsilon, precision=prec)
            if best is None or res.device_ms < best[1].device_ms:
                best = (r, res)
        r, res = best
        rl, mx = _rel(r, r64)
        alg = 4 * E + ((24 + 2 * cb) if quant else (16 + 2 * cb)) * N
        pass_s = res.device_ms * 1e-3 / max(res.passes, 1)
        out[name] = {"device_ms_to_eps": res.device_ms, "passes": res.passes, "iterations": res.iterations,
                     "converged": res.converged, "pass_us": pass_s * 1e6,
                     "roofline_frac": alg / pass_s / 1e9 / peak, "rel_l1_vs_fp64": rl, "max_abs_vs_fp64": mx}
        if name != "fp32":
            out[name]["time_vs_fp32"] = out["fp32"]["device_ms_to_eps"] / res.device_ms
            t0 = time.perf_counter()
            if prec == ag.AG_PREC_FIXED64:
                ref = oracle.pagerank_fixed64(g.in_edges_idx(), g.in_degree(), g.in_neighbours(), g.out_degree(),
                                              a.iterations, a.epsilon)
            else:
                ref = oracle.pagerank_narrow(quant, width, g.in_edges_idx(), g.in_degree(), g.in_neighbours(),
                                             g.out_degree(), a.iterations, a.epsilon)
            out[name]["cpu_oracle"] = {"seconds_to_eps": time.perf_counter() - t0, "iterations": ref["iterations"],
                                       "threads": oracle.lib.oracle_max_threads(),
                                       "bit_identical": bool(ref["iterations"] == res.iterations and
                                                             (ref["ranks"].view("u4") == r.view("u4")).all())}
    print(json.dumps(out), flush=True)


def run_push(a):
    """The reference's push and residual forms against the FP32 pull on the
    same graph: push (pushpull 1), 64-bit fixed-point push (3), 32-bit
    quantised push (5), data-driven push (7) and pull-push (8).  Per form: time
    to epsilon on the device (or to the iteration cap), passes, time per pass,
    accuracy against the FP64 fixpoint, and the single-thread CPU oracle of
    the same form timed on a bounded sample of its iterations."""
    import time
    import oracle
    ag = _gpu_setup()
    g = ag.Graph.rmat(a.scale, a.edge_factor, seed=SEED)
    N, E = g.num_vertices, g.num_edges
    dg = ag.DeviceGraph(g)
    r64, _ = dg.pagerank_f64(5000, 1e-13)
    out = {"workload": f"push-direction and residual PageRank to eps {a.epsilon:g}, RMAT s{a.scale} ef{a.edge_factor}",
           "N": N, "E": E, "bytes_per_pass": "push: 8E (edge list) + 4E of gathered contributions (mostly "
           "repeats of one source) + N(12..28); residual: 4E + 8E for worklist sources"}
    forms = (("pull_fp32", dict()), ("push_fp32", dict(direction=ag.AG_DIR_PUSH)),
             ("push_fixed64", dict(direction=ag.AG_DIR_PUSH, precision=ag.AG_PREC_FIXED64)),
             ("push_quant32", dict(direction=ag.AG_DIR_PUSH, precision=ag.AG_PREC_QUANT32)),
             ("push_dd", dict(direction=ag.AG_DIR_PUSH, data_driven=True)),
             ("pull_push_dd", dict(direction=ag.AG_DIR_PULL_PUSH, data_driven=True)))
    t_build = time.perf_counter()
    dg.pagerank(1, a.epsilon, direction=ag.AG_DIR_PUSH)  # builds the forward edge list once
    out["forward_list_build_s"] = time.perf_counter() - t_build
    for name, kw in forms:
        dg.pagerank(a.iterations, a.epsilon, **kw)
        best = None
        for _ in range(max(1, a.steps)):
            r, res, _ = dg.pagerank(a.iterations, a.epsilon, **kw)
            if best is None or res.device_ms < best[1].device_ms:
                best = (r, res)
        r, res = best
        rl, mx = _rel(r, r64)
        out[name] = {"device_ms_to_eps": res.device_ms, "passes": res.passes, "iterations": res.iterations,
                     "converged": res.converged, "pass_us": res.device_ms * 1e3 / max(res.passes, 1),
                     "rel_l1_vs_fp64": rl, "max_abs_vs_fp64": mx}
        if name != "pull_fp32":
            out[name]["time_vs_pull"] = out["pull_fp32"]["device_ms_to_eps"] / res.device_ms
    sample = 3
    for name, fn in (("push_fp32", lambda: oracle.pagerank_push(0, g.out_edges_idx(), g.out_degree(),
                                                                 g.out_neighbours(), sample, a.epsilon)),
                     ("push_dd", lambda: oracle.pagerank_residual(False, g.in_edges_idx(), g.in_degree(),
                                                                  g.in_neighbours(), g.out_edges_idx(),
                                                                  g.out_degree(), g.out_neighbours(), sample,
                                                                  a.epsilon))):
        t0 = time.perf_counter()
        fn()
        out[name]["cpu_oracle"] = {"seconds_per_iteration": (time.perf_counter() - t0) / sample, "threads": 1,
                                   "sample": f"first {sample} iterations"}
    print(json.dumps(out), flush=True)


def run_rows(a):
    """One graph split by rows over all ranks (NCCL all-gather per pass);
    strong scaling: the whole job solves one graph."""
    import datetime
    import numpy as np
    import torch
    import torch.distributed as dist
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    import accelgraph_b200 as ag
    from accelgraph_b200 import distributed as agd
    ag.check(ag.lib.ag_init(local), "ag_init")
    g = ag.Graph.rmat(a.scale, a.edge_factor, seed=SEED)
    exact = a.order == "exact"
    # the rows are uploaded once; each step is one partitioned solve
    part = agd.RowPartition(g)
    for _ in range(max(1, a.warmup)):
        part.solve(a.iterations, a.epsilon, exact)
    dist.barrier()
    torch.cuda.synchronize()
    stream = part.stream
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    passes = 0
    for _ in range(a.steps):
        _, p_, _, _ = part.solve(a.iterations, a.epsilon, exact)
        passes += p_
    ev1.record(stream)
    ev1.synchronize()
    torch.cuda.synchronize()
    dist.barrier()
    t, _ = reduce_time_work(ev0.elapsed_time(ev1) * 1e-3, 0.0, device="cuda")
    part.release()
    value = g.num_edges * passes / t / 1e9
    if rank == 0:
        print(json.dumps({"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
                          "warmup": a.warmup, "ms_per_step": 1e3 * t / a.steps, "higher_is_better": True,
                          "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                          "config": dict(workload_config(a, world), parallelism=f"rows{world}"),
                          "passes_per_solve": passes // a.steps,
                          "timing": "CUDA events around the solves (rows uploaded once), max over ranks"}),
              flush=True)
    dist.destroy_process_group()


def run_gather_probe(a):
    """Random 4-byte gather rates of this device: tests/probe/gather_probe.cu,
    a measuring aid outside the library, built here into its own
    libgather_probe.so (sm_100a) when missing or older than its source."""
    import numpy as np
    import torch
    torch.cuda.set_device(0)
    src = ROOT / "tests" / "probe" / "gather_probe.cu"
    lib = src.with_name("libgather_probe.so")
    if not lib.exists() or lib.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "-shared",
                        "-Xcompiler", "-fPIC", "-o", str(lib), str(src)], check=True)
    probe = C.CDLL(str(lib))
    probe.gather_probe_rates.argtypes = [C.POINTER(C.c_double)]
    r = np.zeros(6)
    rc = probe.gather_probe_rates(r.ctypes.data_as(C.POINTER(C.c_double)))
    if rc != 0:
        raise RuntimeError(f"gather_probe_rates: CUDA error {rc}")
    names = ["shared_64KB", "global_L1_256KB", "global_L2_64MB", "global_HBM_256MB", "texture_L2_64MB",
             "cluster_shared_8x160KB"]
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    print(json.dumps({"workload": "random 4-byte gathers, 1024 threads/SM, 8 in flight per thread",
                      "gathers_per_s": dict(zip(names, r.tolist())),
                      "per_clock_per_sm_at_1.9GHz": dict(zip(names, (r / sms / 1.9e9).round(3).tolist()))}),
          flush=True)


def main():
    a = parse()
    if a.impl != "reference" and a.workload == "pagerank" and a.mode == "rows":
        run_rows(a)
        return
    if a.impl == "reference":
        run_reference(a)
    elif a.workload == "pagerank":
        run_b200(a)
    else:
        {"spmv": run_spmv, "precision": run_precision, "ppr": run_ppr, "multigraph": run_multigraph,
         "warmstart": run_warmstart, "gather-probe": run_gather_probe,
         "data-driven": run_data_driven, "fixed-point": run_fixed_point, "push": run_push}[a.workload](a)


if __name__ == "__main__":
    main()
