#!/usr/bin/env python
"""Benchmark of the B200 clustering hot path: pLeiden+ edges/s.

Workload: pLeiden+ (leiden_part<plus=true> then improvement passes until the
objective stops rising, i.e. ``-ex_iters -1``) with the weighted-modularity
objective on a seeded degree-corrected SBM: n = 4,194,304, power-law degrees
(exponent 2.5, min 5, mean 20), power-law community sizes (exponent 1.5, 50 to
5,000), mu = 0.4, FP32 edge weights uniform in [0.5, 1.5).  Synthetic data
stand in for the reference's external graph collection.

One step = one full clustering run (run_clustering in app/cluster_main.cpp:116)
from a fresh cluster_data on the graph already resident in HBM.  The metric is
undirected input edges / clustering time (the reference's "Cluster time"
span).  ``e2e`` repeats the step through the public C ABI from host buffers:
CSR upload, graph + objective construction, clustering and label download.

``--impl reference`` times the CPU restatement of the reference algorithm
(the reference itself needs Kokkos, which is unavailable) on a bounded sample of
the same workload with all host threads.

Multi-GPU (torchrun): the path does not shard; every rank clusters its own
replica and ``value`` is the edges of all replicas over the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Leiden edges/s at equal modularity: batched+learned vs plain, same B200"
UNIT = "edges/s"
WORKLOAD = ("pLeiden+ until stable (ex_iters=-1), WMod, DC-SBM n=4,194,304, deg exp 2.5 min 5 mean 20, "
            "communities exp 1.5 on [50,5000], mu=0.4, FP32 weights U[0.5,1.5), int64 offsets")
DOMINANT_FAMILIES = ("select_warp", "select_block", "select_huge", "afterburner_warp", "own_weights", "contract",
                     "leiden_refine", "filter")
# sub-phases reported beside the families (not candidates for the roofline line)
SUB_PHASES = ("contract_prep", "contract_hash", "contract_place", "contract_place_big", "host_alloc")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=4194304, help="DC-SBM vertex count (default: the named workload)")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--cpu-sample-n", type=int, default=262144)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--batched-learned", type=int, default=0, metavar="K",
                    help="also time a population of K seeds run concurrently (pggc_batch_run) with the learned "
                         "move filter, trained first on logs of plain runs of smaller graphs")
    ap.add_argument("--recall", type=float, default=0.98,
                    help="--batched-learned: recall on the training logs that sets the filter threshold")
    ap.add_argument("--by-level", action="store_true",
                    help="profiled run also splits each kernel family by multilevel level (adds 'by_level')")
    ap.add_argument("--ex-iters", type=int, default=-1,
                    help="pLeiden+ passes after the first (-1: until the objective stops rising)")
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


# ---------------------------------------------------------------------------
# clocks sampler (nvidia-smi during the timed region)
# ---------------------------------------------------------------------------
class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        loaded = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU baseline / reference arm (the oracle port of the reference algorithm)
# ---------------------------------------------------------------------------
def cpu_run(sample_n: int, seed: int, steps: int, warmup: int):
    from oracle import oracle as O
    from pennsylvaniagpugraphclustering_b200 import graphgen as gg
    g = gg.dcsbm(sample_n, seed)
    og = O.Graph(g.rowptr, g.col, g.w, objective=O.OBJ_WMOD)
    times = []
    q = None
    for it in range(warmup + steps):
        cd = O.ClusterData(og, O.OBJ_WMOD, 1.0)
        t0 = time.perf_counter()
        labels, st = O.run_clustering(og, cd, method=O.METHOD_LEIDEN_PLUS, ex_iters=-1, seed=seed)
        dt = time.perf_counter() - t0
        if it >= warmup:
            times.append(dt)
        q = st.objective
    sec = statistics.mean(times)
    return {"value": g.m / sec, "unit": UNIT, "cores": int(O.lib().orc_num_threads()), "kind": "port",
            "ms_per_run": sec * 1000.0,
            "sample": f"DC-SBM n={sample_n} (m={g.m}) with the workload's parameters, seed {seed}; "
                      f"pLeiden+ until stable; {steps} timed runs, mean {sec:.3f} s; modularity {q:.6f}"}


def reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    res = cpu_run(args.cpu_sample_n, args.seed, args.steps, args.warmup)
    line = {"impl": "reference", "metric": METRIC, "value": res["value"], "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["ms_per_run"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "sample_n": args.cpu_sample_n},
            "cpu_baseline": res,
            "e2e": {"value": res["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "CPU restatement of the reference algorithm (oracle port); the reference needs Kokkos, "
                    "which is not installed"}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_for(family):
    """Per-launch DRAM bytes from the committed ncu capture summary, if any."""
    try:
        with open(os.path.join(ROOT, "profiles", "dram_traffic.json")) as f:
            return json.load(f).get(family)
    except Exception:
        return None


def ours(args):
    import torch
    import pennsylvaniagpugraphclustering_b200 as pg
    from pennsylvaniagpugraphclustering_b200 import _lib, graphgen as gg

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    g = gg.dcsbm(args.n, args.seed)
    m = g.m
    mem = pg.memory_store(local)
    stream = torch.cuda.ExternalStream(mem.stream(), device=torch.device("cuda", local))
    wg = pg.weighted_graph(mem, g.rowptr, g.col, g.w, objective=pg.OBJ_WMOD)
    labels = torch.empty(g.n, dtype=torch.int32, device=f"cuda:{local}")

    def step(seed):
        cd = pg.get_objective(mem, wg, pg.OBJ_WMOD, 1.0)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        _, st = pg.run_clustering(mem, wg, cd, method=pg.METHOD_LEIDEN_PLUS, ex_iters=args.ex_iters, seed=seed,
                                  out=labels)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        cd.close()
        return ms, st

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()

    for w in range(args.warmup):
        step(args.seed + rank)
    lib = _lib.lib()
    clocks = ClockSampler(local)
    barrier()
    clocks.start()
    l0 = lib.pggc_launch_count()
    times, stats = [], None
    for s in range(args.steps):
        ms, stats = step(args.seed + rank)
        times.append(ms)
    launches = lib.pggc_launch_count() - l0
    barrier()
    clk = clocks.stop()
    # one more, untimed run with per-family CUDA events and device byte
    # counters on: the kernel breakdown and the roofline figures
    _lib.check(lib.pggc_profile_reset(mem.handle))
    _lib.check(lib.pggc_profile_enable(mem.handle, 2 if args.by_level else 1))
    step(args.seed + rank)
    _lib.check(lib.pggc_profile_enable(mem.handle, 0))
    fam = {}

    def read_family(f):
        n_l, t_ms, by = (_lib.ctypes.c_int64(), _lib.ctypes.c_double(), _lib.ctypes.c_double())
        _lib.check(lib.pggc_profile_read(mem.handle, f.encode(), _lib.ctypes.byref(n_l), _lib.ctypes.byref(t_ms),
                                         _lib.ctypes.byref(by)))
        return n_l.value, t_ms.value, by.value

    for f in DOMINANT_FAMILIES + SUB_PHASES:
        fam[f] = read_family(f)
    by_level = None
    if args.by_level:
        need = _lib.ctypes.c_int64()
        _lib.check(lib.pggc_profile_names(mem.handle, None, 0, _lib.ctypes.byref(need)))
        buf = _lib.ctypes.create_string_buffer(need.value)
        _lib.check(lib.pggc_profile_names(mem.handle, buf, need.value, None))
        by_level = {}
        for name in buf.value.decode().split("\n"):
            if "@" in name:
                f, lv = name.split("@", 1)
                n_l, t_ms, _ = read_family(name)
                by_level.setdefault(f, {})[lv] = {"launches": n_l, "ms": round(t_ms, 3)}
    q_labels = labels.cpu().numpy()
    q, _ = pg.verify_objective(mem, wg, q_labels, pg.OBJ_WMOD)

    # e2e: host buffers through the public API, copies inside the timed region
    e2e_steps = args.e2e_steps if args.e2e_steps is not None else max(1, min(args.steps, 2))
    e2e_steps = max(0, e2e_steps)
    e2e_ms = []
    host_labels = np.empty(g.n, np.int32)
    for s in range(e2e_steps):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        g2 = pg.weighted_graph(mem, g.rowptr, g.col, g.w, objective=pg.OBJ_WMOD)
        cd2 = pg.get_objective(mem, g2, pg.OBJ_WMOD, 1.0)
        pg.run_clustering(mem, g2, cd2, method=pg.METHOD_LEIDEN_PLUS, ex_iters=args.ex_iters,
                          seed=args.seed + rank, out=host_labels)
        e1.record(stream)
        e1.synchronize()
        e2e_ms.append(e0.elapsed_time(e1))
        cd2.close()
        g2.close()
    h2d = g.rowptr.nbytes + g.col.nbytes + g.w.nbytes
    d2h = host_labels.nbytes

    ms_step = statistics.mean(times)
    ms_e2e = statistics.mean(e2e_ms) if e2e_ms else float("nan")
    if world > 1:
        from pennsylvaniagpugraphclustering_b200 import replicas
        ms_step, ms_e2e = replicas.max_over_ranks([ms_step, ms_e2e], device=f"cuda:{local}")
    value = world * m / (ms_step / 1000.0)
    e2e_value = world * m / (ms_e2e / 1000.0)

    # roofline for the dominant instrumented kernel
    dom = max((f for f in DOMINANT_FAMILIES if fam[f][2] > 0), key=lambda f: fam[f][1], default=None)
    peak, peak_kind = peaks()
    roof = None
    if dom is not None:
        nl, tms, by = fam[dom]
        achieved = by / (tms / 1000.0) / 1e9
        tr = traffic_for(dom)
        roof = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": peak_kind,
                "traffic": tr, "algorithmic_bytes_per_launch": by / max(nl, 1),
                "avg_launch_ms": tms / max(nl, 1), "launches": nl}
    if rank != 0:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    bl = None
    if args.batched_learned > 0:
        bl = batched_learned(args, pg, mem, wg, m, q)
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_run(args.cpu_sample_n, args.seed, 1, 0)
        except Exception as ex:  # report, never fail the line
            cpu = {"value": None, "unit": UNIT, "cores": None, "kind": "port", "sample": f"failed: {ex}"}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded DC-SBM)",
        "config": {"workload": WORKLOAD, "n": g.n, "m_undirected": m, "nnz": g.nnz, "seed": args.seed,
                   "parallelism": f"replicas x{world}", "l2": "inputs larger than L2 (graph CSR ~0.7 GB)",
                   "modularity": q, "levels": stats["levels"], "passes": stats["passes"],
                   "sweeps": stats["sweeps"], "labels": stats["label_count"]},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "ms_per_step": ms_e2e, "ms_each": e2e_ms},
        "roofline": roof,
        "kernel_families": {f: {"launches": v[0], "ms": v[1], "alg_bytes": v[2]} for f, v in fam.items()},
        "cpu_baseline": cpu,
        "clocks": clk,
        "gpu_launches": int(launches),
        "ms_each": [round(t, 1) for t in times],
    }
    if bl is not None:
        line["batched_learned"] = bl
    if by_level is not None:
        line["by_level"] = by_level
        line["passes_profile"] = {f: {"launches": v[0], "ms": v[1]} for f, v in
                                  ((f, read_family(f)) for f in ("pass_first", "pass_improve"))}
    print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def batched_learned(args, pg, mem, wg, m, q_plain):
    """Population of K seeds on the workload graph, concurrently on K streams,
    with the learned move filter trained on logs of plain runs of 262,144-vertex
    DC-SBMs (seeds 101-104, one pass each)."""
    from pennsylvaniagpugraphclustering_b200 import graphgen as gg, move_filter as MF
    t0 = time.perf_counter()
    xs, ys = [], []
    for s in (1, 2, 3, 4):
        h = gg.dcsbm(262144, 100 + s)
        g2 = pg.weighted_graph(mem, h.rowptr, h.col, h.w, objective=pg.OBJ_WMOD)
        MF.log_start(mem, capacity=2_000_000, sample_rate=0.25, seed=s)
        cd = pg.get_objective(mem, g2, pg.OBJ_WMOD, 1.0)
        pg.run_clustering(mem, g2, cd, method=pg.METHOD_LEIDEN_PLUS, ex_iters=0, seed=s)
        x, y, _ = MF.log_stop(mem, 2_000_000)
        xs.append(x)
        ys.append(y)
        cd.close()
        g2.close()
    x = np.concatenate(xs)
    y = np.concatenate(ys)
    pos_w = float(min(20.0, (len(y) - y.sum()) / max(y.sum(), 1.0)))
    params, losses = MF.train(mem, MF.init_params(1), x, y, epochs=6, batch=4096, lr=3e-3, pos_weight=pos_w)
    thr = MF.threshold_for_recall(mem, params, x, y, recall=args.recall)
    train_s = time.perf_counter() - t0
    K = args.batched_learned

    def jobs_for(k):
        return [dict(graph=wg, objective=pg.OBJ_WMOD, method=pg.METHOD_LEIDEN_PLUS, ex_iters=args.ex_iters,
                      seed=args.seed + j) for j in range(k)]

    def timed(k, learned):
        if learned:
            MF.enable(mem, params, thr)
        try:
            # warm-up of the worker streams and their scratch: one cheap pass per job
            warm = [dict(j, ex_iters=0) for j in jobs_for(k)]
            pg.batch_run(mem, warm, streams=k)
            MF.stats(mem, reset=True)
            t1 = time.perf_counter()
            res = pg.batch_run(mem, jobs_for(k), streams=k)
            dt = time.perf_counter() - t1
            ev, sk = MF.stats(mem)
        finally:
            MF.disable(mem)
        qs = [st["objective"] for _, st in res]
        return {"value": k * m / dt, "seconds": dt, "modularity_mean": statistics.mean(qs),
                "modularity_min": min(qs), "passes_mean": statistics.mean(st["passes"] for _, st in res),
                "sweeps_mean": statistics.mean(st["sweeps"] for _, st in res),
                "filter_skipped_frac": (sk / max(ev + sk, 1)) if learned else 0.0}

    out = {"unit": UNIT, "population": K, "streams": K, "recall": args.recall, "plain_modularity": q_plain,
           "train_rows": int(len(y)), "train_seconds": train_s, "final_train_loss": float(losses[-1]),
           "threshold_logit": thr, "timing": "host wall clock around pggc_batch_run (all streams joined)"}
    out["learned_1"] = timed(1, True)
    out["batched_plain"] = timed(K, False)
    bl = timed(K, True)
    out.update(bl)
    return out


def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
    else:
        ours(args)


if __name__ == "__main__":
    main()
