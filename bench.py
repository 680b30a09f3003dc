#!/usr/bin/env python
"""Benchmark of the B200 clustering hot path: Leiden edges/s, batched+learned vs plain.

Workload: pLeiden+ (leiden_part<plus=true> then improvement passes until the
objective stops rising, i.e. ``-ex_iters -1``) with the weighted-modularity
objective on a seeded degree-corrected SBM: n = 4,194,304, power-law degrees
(exponent 2.5, min 5, mean 20), power-law community sizes (exponent 1.5, 50 to
5,000), mu = 0.4, ~41.9 M undirected edges, FP32 edge weights uniform in
[0.5, 1.5).  Synthetic data stand in for the reference's external graph
collection.

One step = one full clustering run (run_clustering in app/cluster_main.cpp:116)
of one member of a population of seeds, from a fresh cluster_data on the graph
already resident in HBM.  The metric is undirected input edges / clustering
time (the reference's "Cluster time" span), at equal modularity:

* ``value``: the K timed steps run as ONE batch (``pggc_batch_run``, P worker
  streams) with the learned move filter on, its judge included -- the
  batched+learned configuration.  Time = CUDA events on the context stream,
  which the batch's workers are ordered against.
* ``plain``: the same seeds (all K by default, up to a wall-clock budget)
  run one after another, no filter, one stream; ``ratio_vs_plain`` = value / plain edges/s, with both
  modularities (mean over the seeds) and the criterion "ratio >= 1.5 at
  modularity within 0.001".  The number of improvement passes until the
  objective stops rising differs by up to +-30 % between seeds, so the two
  arms run the same population.
* ``e2e``: a batch of P members through the public C ABI from host buffers:
  CSR upload, graph + objective construction, clustering and label download.

The filter is trained before the warm-up (untimed) on move / no-move labels
logged from plain first passes of the three named workloads' generators at
seeds 1-8 (planted SBM n = 65,536, the DC-SBM at n = 262,144, R-MAT scale 18):
by default the label is the select step's decision (it proposes a move or
not), the threshold keeps 99.5 % of the proposals, and the filter gates the
sweeps of the coarse levels (>= 1), where they are latency-bound.

``--impl reference`` times the CPU restatement of the reference algorithm
(the reference itself needs Kokkos, which is unavailable) on a bounded sample of
the same workload (a 262,144-vertex DC-SBM with the same parameters) with all
host threads; our line reports the GPU on that same sample beside it.

Multi-GPU (torchrun): the path does not shard; every rank clusters its own
population and ``value`` is the edges of all ranks over the slowest rank's time.
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
WORKLOAD = ("pLeiden+ until stable (ex_iters=-1), WMod, DC-SBM n=4,194,304, deg exp 2.5 min 5 mean 20 "
            "(~41.9M undirected edges), communities exp 1.5 on [50,5000], mu=0.4, FP32 weights U[0.5,1.5), "
            "int64 offsets; population of seeds run as one batch with the learned move filter")
TARGET_RATIO = 1.5
Q_TOLERANCE = 0.001
DOMINANT_FAMILIES = ("select_warp", "select_block", "select_huge", "afterburner_warp", "own_weights", "contract",
                     "leiden_refine", "filter")
# sub-phases reported beside the families (not candidates for the roofline line)
SUB_PHASES = ("contract_prep", "contract_hash", "contract_place", "contract_place_big", "host_alloc", "lm_compact",
              "lm_roundtrip", "lm_newids", "lm_moves", "lm_copy")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=12, help="timed clustering runs (population members)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=4194304, help="DC-SBM vertex count (default: the named workload)")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--streams", type=int, default=6, help="worker streams of the batch (population width)")
    ap.add_argument("--plain-runs", type=int, default=-1,
                    help="plain runs for the ratio (the first seeds of the population, no filter, one stream; "
                         "-1: every seed of the population, so both arms run the same seeds, stopping after "
                         "--plain-budget seconds once two runs are done)")
    ap.add_argument("--plain-budget", type=float, default=150.0,
                    help="wall-clock bound of the plain arm when --plain-runs is -1")
    ap.add_argument("--no-filter", action="store_true", help="batched plain runs (no learned filter)")
    ap.add_argument("--recall", type=float, default=0.995,
                    help="recall on the training logs that sets the filter's logit threshold")
    ap.add_argument("--filter-label", default="candidate", choices=["candidate", "moved"],
                    help="training label: the select step proposes a move (candidate) or the vertex moves")
    ap.add_argument("--filter-min-level", type=int, default=1,
                    help="the filter gates sweeps at multilevel levels >= this (0: the input graph too)")
    ap.add_argument("--cpu-sample-n", type=int, default=262144)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=None, help="e2e batch size (default: --streams)")
    ap.add_argument("--eval-ex-iters", type=int, default=8,
                    help="filter-eval workload: improvement passes after the first (-1: until stable)")
    ap.add_argument("--by-level", action="store_true",
                    help="profiled run also splits each kernel family by multilevel level (adds 'by_level')")
    ap.add_argument("--ex-iters", type=int, default=-1,
                    help="pLeiden+ passes after the first (-1: until the objective stops rising)")
    ap.add_argument("--workload", default="dcsbm4m",
                    choices=["dcsbm4m", "rmat24", "sbm65k", "sbm-population", "filter-eval", "profile-case"],
                    help="dcsbm4m: the headline line (batched+learned vs plain pLeiden+); rmat24: plain pLouvain "
                         "on R-MAT scale 24 (contraction stress); sbm65k: plain pLouvain on the planted SBM; "
                         "sbm-population: 256 uneven SBMs, batched (autotuned) vs sequential pLeiden+; "
                         "filter-eval: the trained filter against plain pLeiden+ on unseen seed 99 graphs "
                         "(R-MAT scale 25, DC-SBM n=16,777,216 at mu=0.5)")
    ap.add_argument("--population", type=int, default=256, help="sbm-population: number of graphs")
    ap.add_argument("--rmat-scale", type=int, default=24)
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
    g = gg.dcsbm(sample_n, seed, mean_deg=gg.DCSBM_4M_MEAN_DEG)
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
            "modularity": q, "n": sample_n, "m": g.m,
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
            "config": {"workload": WORKLOAD, "sample_n": args.cpu_sample_n, "sample_m": res.get("m"),
                       "reference_runs": "plain pLeiden+ until stable (the reference has no batching and no "
                                         "learned filter) on the sample graph, seed " + str(args.seed)},
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




def train_filter(pg, mem, recall, label="candidate"):
    """Train the learned move filter on move / no-move labels logged from
    plain first passes of the named workloads' generators at seeds 1-8
    (planted SBM n = 65,536; the DC-SBM at n = 262,144; R-MAT scale 18);
    returns (params, threshold, info).  label "candidate": 1 when the select
    step proposes a move for the vertex; "moved": 1 when it moves."""
    from pennsylvaniagpugraphclustering_b200 import graphgen as gg, move_filter as MF
    t0 = time.perf_counter()
    xs, ys = [], []
    cap = 2_000_000  # above any one run's sampled rows: a full log would keep a race-dependent subset
    truncated = 0
    MF.log_label(mem, label)
    for s in range(1, 9):
        for kind in ("sbm", "dcsbm", "rmat"):
            if kind == "sbm":
                h, obj, w = gg.planted_sbm_65k(s), pg.OBJ_MOD, None
            elif kind == "dcsbm":
                h = gg.dcsbm(262144, s, mean_deg=gg.DCSBM_4M_MEAN_DEG)
                obj, w = pg.OBJ_WMOD, h.w
            else:
                h, obj, w = gg.rmat(18, 16, 0.57, 0.19, 0.19, s), pg.OBJ_MOD, None
            g2 = pg.weighted_graph(mem, h.rowptr, h.col, w, objective=obj)
            MF.log_start(mem, capacity=cap, sample_rate=0.1, seed=s)
            cd = pg.get_objective(mem, g2, obj, 1.0)
            method = pg.METHOD_LOUVAIN if kind != "dcsbm" else pg.METHOD_LEIDEN_PLUS
            pg.run_clustering(mem, g2, cd, method=method, ex_iters=0, seed=s)
            x, y, rows = MF.log_stop(mem, cap)
            truncated += max(0, rows - cap)
            xs.append(x)
            ys.append(y)
            cd.close()
            g2.close()
    MF.log_label(mem, "moved")
    x = np.concatenate(xs)
    y = np.concatenate(ys)
    # the log's row order depends on which warp appended first; a canonical
    # order (features, then label) makes the minibatches, and so the trained
    # network and its threshold, the same on every run
    order = np.lexsort(np.concatenate([y[None, :], x.T[::-1]], axis=0))
    x, y = x[order], y[order]
    pos_w = float(min(20.0, (len(y) - y.sum()) / max(y.sum(), 1.0)))
    params, losses = MF.train(mem, MF.init_params(1), x, y, epochs=6, batch=4096, lr=3e-3, pos_weight=pos_w)
    thr = MF.threshold_for_recall(mem, params, x, y, recall=recall)
    skip = float(np.mean(MF.infer(mem, params, x) < thr))
    return params, thr, {"train_rows": int(len(y)), "positive_rows": int(y.sum()), "final_loss": float(losses[-1]),
                         "threshold_logit": thr, "recall": recall, "label": label, "rows_dropped": truncated,
                         "train_rows_below_threshold": skip, "train_seconds": time.perf_counter() - t0,
                         "sources": "first passes of planted SBM 65,536, DC-SBM 262,144 and R-MAT 18, seeds 1-8"}


def ours(args):
    import torch
    import pennsylvaniagpugraphclustering_b200 as pg
    from pennsylvaniagpugraphclustering_b200 import _lib, graphgen as gg, move_filter as MF

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    g = gg.dcsbm(args.n, args.seed, mean_deg=gg.DCSBM_4M_MEAN_DEG)
    m = g.m
    mem = pg.memory_store(local)
    stream = torch.cuda.ExternalStream(mem.stream(), device=torch.device("cuda", local))
    wg = pg.weighted_graph(mem, g.rowptr, g.col, g.w, objective=pg.OBJ_WMOD)
    lib = _lib.lib()
    learned = not args.no_filter
    K = max(1, args.steps)
    P = max(1, min(args.streams, K))
    seeds = [args.seed + rank * 1000 + j for j in range(K)]

    filt_info = None
    params = thr = None
    if learned:
        params, thr, filt_info = train_filter(pg, mem, args.recall, args.filter_label)
        filt_info["min_level"] = args.filter_min_level
        MF.scope(mem, -1, args.filter_min_level)

    def jobs(sds, ex=args.ex_iters):
        return [dict(graph=wg, objective=pg.OBJ_WMOD, method=pg.METHOD_LEIDEN_PLUS, ex_iters=ex, seed=sd)
                for sd in sds]

    def timed(fn):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1), out

    def batch(sds, streams):
        if learned:
            MF.enable(mem, params, thr)
        try:
            return pg.batch_run(mem, jobs(sds), streams=streams)
        finally:
            if learned:
                MF.disable(mem)

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()

    # warm-up: W runs through the batch path (worker streams, pools, scratch)
    if args.warmup > 0:
        batch([args.seed + 500 + j for j in range(args.warmup)], min(P, args.warmup))
    clocks = ClockSampler(local)
    barrier()
    clocks.start()
    l0 = lib.pggc_launch_count()
    if learned:
        MF.stats(mem, reset=True)
    ms_batch, res = timed(lambda: batch(seeds, P))
    launches = lib.pggc_launch_count() - l0
    barrier()
    clk = clocks.stop()
    ev, sk = MF.stats(mem) if learned else (0, 0)
    q_batch = [st["objective"] for _, st in res]

    # plain: the first R seeds, no filter, one after another on one stream
    R = K if args.plain_runs < 0 else max(0, min(args.plain_runs, K))
    plain_ms, plain_q, plain_passes = [], [], []
    t_plain = time.perf_counter()
    for sd in seeds[:R]:
        if args.plain_runs < 0 and len(plain_ms) >= 2 and time.perf_counter() - t_plain > args.plain_budget:
            R = len(plain_ms)
            break
        cd = pg.get_objective(mem, wg, pg.OBJ_WMOD, 1.0)
        ms, (_, st) = timed(lambda: pg.run_clustering(mem, wg, cd, method=pg.METHOD_LEIDEN_PLUS,
                                                        ex_iters=args.ex_iters, seed=sd))
        plain_ms.append(ms)
        plain_q.append(st["objective"])
        plain_passes.append(st["passes"])
        cd.close()

    # one more learned run on the context stream with per-family CUDA events
    # and device byte counters: the kernel breakdown and the roofline figures
    _lib.check(lib.pggc_profile_reset(mem.handle))
    _lib.check(lib.pggc_profile_enable(mem.handle, 2 if args.by_level else 1))
    labels = torch.empty(g.n, dtype=torch.int32, device=f"cuda:{local}")
    if learned:
        MF.enable(mem, params, thr)
    try:
        cd = pg.get_objective(mem, wg, pg.OBJ_WMOD, 1.0)
        pg.run_clustering(mem, wg, cd, method=pg.METHOD_LEIDEN_PLUS, ex_iters=args.ex_iters, seed=seeds[0],
                          out=labels)
        cd.close()
    finally:
        if learned:
            MF.disable(mem)
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
    q_verify, _ = pg.verify_objective(mem, wg, labels.cpu().numpy(), pg.OBJ_WMOD)

    # e2e: host buffers through the public API (CSR upload, graph and objective
    # construction, a batch of E members, label download) inside the timed region
    E = args.e2e_steps if args.e2e_steps is not None else P
    E = max(0, E)
    e2e_ms = float("nan")
    if E > 0:
        # the host CSR in pinned (page-locked) buffers, as a caller streaming
        # graphs would hold it; pinning is outside the timed region
        h_rowptr, h_col, h_w = (torch.from_numpy(a).pin_memory() for a in (g.rowptr, g.col, g.w))

        def e2e_once():
            g2 = pg.weighted_graph(mem, h_rowptr, h_col, h_w, objective=pg.OBJ_WMOD)
            if learned:
                MF.enable(mem, params, thr)
            try:
                out = pg.batch_run(mem, [dict(graph=g2, objective=pg.OBJ_WMOD, method=pg.METHOD_LEIDEN_PLUS,
                                              ex_iters=args.ex_iters, seed=sd) for sd in seeds[:E]],
                                   streams=min(P, E))
            finally:
                if learned:
                    MF.disable(mem)
            g2.close()
            return out
        e2e_ms, _ = timed(e2e_once)
    h2d = g.rowptr.nbytes + g.col.nbytes + g.w.nbytes
    d2h = 4 * g.n * E

    ms_step = ms_batch / K
    ms_plain = statistics.mean(plain_ms) if plain_ms else float("nan")
    if world > 1:
        from pennsylvaniagpugraphclustering_b200 import replicas
        ms_step, ms_e2e_run, ms_plain = replicas.max_over_ranks([ms_step, e2e_ms / max(E, 1), ms_plain],
                                                                device=f"cuda:{local}")
    else:
        ms_e2e_run = e2e_ms / max(E, 1)
    value = world * m / (ms_step / 1000.0)
    e2e_value = world * m / (ms_e2e_run / 1000.0)
    plain_value = world * m / (ms_plain / 1000.0) if plain_ms else None

    # roofline for the dominant instrumented kernel family
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
    cpu = None
    same_sample = None
    if world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_run(args.cpu_sample_n, args.seed, 1, 0)
            # the GPU on the same sample graph and seed: like-for-like speed,
            # identical modularity (the two paths share one arithmetic)
            h = gg.dcsbm(args.cpu_sample_n, args.seed, mean_deg=gg.DCSBM_4M_MEAN_DEG)
            g3 = pg.weighted_graph(mem, h.rowptr, h.col, h.w, objective=pg.OBJ_WMOD)
            t3 = []
            for _ in range(3):
                cd = pg.get_objective(mem, g3, pg.OBJ_WMOD, 1.0)
                ms3, (_, st3) = timed(lambda: pg.run_clustering(mem, g3, cd, method=pg.METHOD_LEIDEN_PLUS,
                                                                  ex_iters=-1, seed=args.seed))
                t3.append(ms3)
                cd.close()
            g3.close()
            gpu_v = h.m / (min(t3) / 1000.0)
            same_sample = {"n": args.cpu_sample_n, "m": h.m, "gpu_plain_edges_per_s": gpu_v,
                           "cpu_edges_per_s": cpu["value"], "gpu_over_cpu": gpu_v / cpu["value"],
                           "gpu_modularity": st3["objective"], "cpu_modularity": cpu["modularity"],
                           "identical_modularity": st3["objective"] == cpu["modularity"]}
        except Exception as ex:  # report, never fail the line
            cpu = {"value": None, "unit": UNIT, "cores": None, "kind": "port", "sample": f"failed: {ex}"}
    q_mean = statistics.mean(q_batch[:R]) if R else statistics.mean(q_batch)
    plain_q_mean = statistics.mean(plain_q) if plain_q else None
    dq = (q_mean - plain_q_mean) if plain_q_mean is not None else None
    ratio = value / plain_value if plain_value else None
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded DC-SBM)",
        "config": {"workload": WORKLOAD, "n": g.n, "m_undirected": m, "nnz": g.nnz, "seeds": [seeds[0], seeds[-1]],
                   "parallelism": f"replicas x{world}; batch of {K} runs on {P} streams per GPU",
                   "learned_filter": learned, "l2": "inputs larger than L2 (graph CSR ~0.7 GB)",
                   "modularity_mean": statistics.mean(q_batch), "modularity_min": min(q_batch),
                   "passes_mean": statistics.mean(st["passes"] for _, st in res),
                   "exact_passes_mean": statistics.mean(st["exact_passes"] for _, st in res),
                   "fallbacks": int(sum(st["fell_back"] for _, st in res)),
                   "sweeps_mean": statistics.mean(st["sweeps"] for _, st in res),
                   "labels_mean": statistics.mean(st["label_count"] for _, st in res),
                   "filter_skipped_frac": sk / max(ev + sk, 1) if learned else 0.0},
        "plain": {"value": plain_value, "unit": UNIT, "runs": R, "ms_per_run": ms_plain,
                  "modularity_mean": plain_q_mean, "passes_mean": statistics.mean(plain_passes) if R else None,
                  "seeds": seeds[:R]},
        "ratio_vs_plain": ratio,
        "modularity_delta_vs_plain": dq,
        "criterion": {"ratio_min": TARGET_RATIO, "modularity_tolerance": Q_TOLERANCE,
                      "met": bool(ratio is not None and ratio >= TARGET_RATIO and dq is not None and dq >= -Q_TOLERANCE)},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d / max(E, 1)),
                "d2h_bytes_per_step": int(d2h / max(E, 1)), "ms_per_step": ms_e2e_run, "batch": E,
                "note": "CSR uploaded once per batch of E runs (bytes per step = upload / E)"},
        "roofline": roof,
        "kernel_families": {f: {"launches": v[0], "ms": v[1], "alg_bytes": v[2]} for f, v in fam.items()},
        "profiled_run_verify_modularity": q_verify,
        "cpu_baseline": cpu,
        "same_sample": same_sample,
        "clocks": clk,
        "gpu_launches": int(launches),
        "filter": filt_info,
    }
    if by_level is not None:
        line["by_level"] = by_level
        line["passes_profile"] = {f: {"launches": v[0], "ms": v[1]} for f, v in
                                  ((f, read_family(f)) for f in ("pass_first", "pass_improve"))}
    print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def _families(lib, _lib, mem):
    fam = {}
    for f in DOMINANT_FAMILIES + SUB_PHASES:
        n_l, t_ms, by = (_lib.ctypes.c_int64(), _lib.ctypes.c_double(), _lib.ctypes.c_double())
        _lib.check(lib.pggc_profile_read(mem.handle, f.encode(), _lib.ctypes.byref(n_l), _lib.ctypes.byref(t_ms),
                                         _lib.ctypes.byref(by)))
        fam[f] = (n_l.value, t_ms.value, by.value)
    return fam


def _roofline(fam):
    dom = max((f for f in DOMINANT_FAMILIES if fam[f][2] > 0), key=lambda f: fam[f][1], default=None)
    if dom is None:
        return None
    peak, peak_kind = peaks()
    nl, tms, by = fam[dom]
    achieved = by / (tms / 1000.0) / 1e9
    return {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic_for(dom),
            "algorithmic_bytes_per_launch": by / max(nl, 1), "avg_launch_ms": tms / max(nl, 1), "launches": nl}


def plain_workload(args):
    """One named workload, plain method, single stream: R-MAT scale 24 pLouvain
    (the contraction stress: hub rows above 15,000 edges, large hash merges) or
    the planted SBM n = 65,536 pLouvain.  K timed runs with CUDA events, a
    profiled run for the kernel families and the roofline, an e2e run from host
    buffers, and the oracle port on the CPU (the SBM in full; R-MAT at scale
    20, same generator parameters)."""
    import torch
    import pennsylvaniagpugraphclustering_b200 as pg
    from pennsylvaniagpugraphclustering_b200 import _lib, graphgen as gg
    torch.cuda.set_device(0)
    if args.workload == "rmat24":
        g = gg.rmat(args.rmat_scale, 16, 0.57, 0.19, 0.19, args.seed)
        desc = (f"plain pLouvain (ex_iters=0), Mod, R-MAT scale {args.rmat_scale} edge factor 16 a=0.57 b=c=0.19 "
                f"d=0.05, symmetrised, deduplicated, no self-loops, unit weights, int64 offsets")
        cpu_graph = lambda: gg.rmat(min(20, args.rmat_scale), 16, 0.57, 0.19, 0.19, args.seed)
    else:
        g = gg.planted_sbm_65k(args.seed)
        desc = ("plain pLouvain (ex_iters=0), Mod, planted-partition SBM n=65,536 in 64 blocks of 1,024, expected "
                "degrees 16/4, unit weights")
        cpu_graph = lambda: g
    mem = pg.memory_store(0)
    stream = torch.cuda.ExternalStream(mem.stream(), device=torch.device("cuda", 0))
    lib = _lib.lib()
    wg = pg.weighted_graph(mem, g.rowptr, g.col, None, objective=pg.OBJ_MOD)
    labels = torch.empty(max(g.n, 1), dtype=torch.int32, device="cuda:0")

    def run():
        cd = pg.get_objective(mem, wg, pg.OBJ_MOD, 1.0)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        _, st = pg.run_clustering(mem, wg, cd, method=pg.METHOD_LOUVAIN, ex_iters=0, seed=args.seed, out=labels)
        e1.record(stream)
        e1.synchronize()
        cd.close()
        return e0.elapsed_time(e1), st

    for _ in range(args.warmup):
        run()
    clocks = ClockSampler(0)
    clocks.start()
    l0 = lib.pggc_launch_count()
    times, st = [], None
    for _ in range(max(1, args.steps)):
        ms, st = run()
        times.append(ms)
    launches = lib.pggc_launch_count() - l0
    clk = clocks.stop()
    _lib.check(lib.pggc_profile_reset(mem.handle))
    _lib.check(lib.pggc_profile_enable(mem.handle, 1))
    run()
    _lib.check(lib.pggc_profile_enable(mem.handle, 0))
    fam = _families(lib, _lib, mem)
    q, _ = pg.verify_objective(mem, wg, labels[:g.n].cpu().numpy(), pg.OBJ_MOD)
    # e2e from pinned host buffers (pinned outside the timed region)
    host = torch.empty(g.n, dtype=torch.int32).pin_memory()
    h_rowptr, h_col = torch.from_numpy(g.rowptr).pin_memory(), torch.from_numpy(g.col).pin_memory()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    g2 = pg.weighted_graph(mem, h_rowptr, h_col, None, objective=pg.OBJ_MOD)
    cd2 = pg.get_objective(mem, g2, pg.OBJ_MOD, 1.0)
    pg.run_clustering(mem, g2, cd2, method=pg.METHOD_LOUVAIN, ex_iters=0, seed=args.seed, out=host)
    e1.record(stream)
    e1.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    cd2.close()
    g2.close()
    ms = statistics.mean(times)
    cpu = None
    if not args.no_cpu_baseline:
        from oracle import oracle as O
        h = cpu_graph()
        og = O.Graph(h.rowptr, h.col, None, objective=O.OBJ_MOD)
        cdo = O.ClusterData(og, O.OBJ_MOD, 1.0)
        t0 = time.perf_counter()
        _, so = O.run_clustering(og, cdo, method=O.METHOD_LOUVAIN, ex_iters=0, seed=args.seed)
        dt = time.perf_counter() - t0
        cpu = {"value": h.m / dt, "unit": UNIT, "cores": int(O.lib().orc_num_threads()), "kind": "port",
               "modularity": so.objective,
               "sample": f"{'the same graph' if h is g else f'R-MAT scale {min(20, args.rmat_scale)}'} "
                         f"(n={h.n}, m={h.m}); one pLouvain run, {dt:.3f} s; modularity {so.objective:.6f}"}
    line = {"metric": f"Louvain edges/s ({args.workload})", "value": g.m / (ms / 1000.0), "unit": UNIT,
            "n_gpus": 1, "steps": len(times), "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
            "config": {"workload": desc, "n": g.n, "m_undirected": g.m, "nnz": g.nnz,
                       "max_degree": int(np.diff(g.rowptr).max()), "modularity": st["objective"],
                       "verify_modularity": q, "levels": st["levels"], "labels": st["label_count"],
                       "l2": "inputs larger than L2" if g.nnz * 4 > 126e6 else "inputs smaller than L2"},
            "e2e": {"value": g.m / (e2e_ms / 1000.0), "unit": UNIT,
                    "h2d_bytes_per_step": int(g.rowptr.nbytes + g.col.nbytes), "d2h_bytes_per_step": int(host.nbytes),
                    "ms_per_step": e2e_ms},
            "roofline": _roofline(fam),
            "kernel_families": {f: {"launches": v[0], "ms": v[1], "alg_bytes": v[2]} for f, v in fam.items()},
            "cpu_baseline": cpu, "clocks": clk, "gpu_launches": int(launches),
            "ms_each": [round(t, 2) for t in times]}
    print(json.dumps(line), flush=True)


def population(args):
    """The batched workload's uneven-size population: `--population` planted
    SBMs (n log-uniform in [1,000, 200,000], 8-512 blocks, expected degrees
    12 / 3, unit weights), one pLeiden+ pass each.  Sequential runs on one
    stream against one batch with the autotuned width and kernel knobs (the
    autotuner runs first on every 8th graph)."""
    import torch
    import pennsylvaniagpugraphclustering_b200 as pg
    from pennsylvaniagpugraphclustering_b200 import _lib, graphgen as gg
    torch.cuda.set_device(0)
    t0 = time.perf_counter()
    pop = gg.sbm_population(args.population, args.seed)
    gen_s = time.perf_counter() - t0
    mem = pg.memory_store(0)
    stream = torch.cuda.ExternalStream(mem.stream(), device=torch.device("cuda", 0))
    graphs = [pg.weighted_graph(mem, h.rowptr, h.col, None, objective=pg.OBJ_MOD) for h in pop]
    m_total = sum(h.m for h in pop)
    jobs = [dict(graph=g, objective=pg.OBJ_MOD, method=pg.METHOD_LEIDEN_PLUS, ex_iters=0, seed=k + 1)
            for k, g in enumerate(graphs)]

    def timed(fn):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1), out

    def sequential():
        res = []
        for j in jobs:
            cd = pg.get_objective(mem, j["graph"], pg.OBJ_MOD, 1.0)
            res.append(pg.run_clustering(mem, j["graph"], cd, method=pg.METHOD_LEIDEN_PLUS, ex_iters=0,
                                         seed=j["seed"])[1])
            cd.close()
        return res

    sequential()  # warm-up (per-graph caches, pools)
    ms_seq, seq = timed(sequential)
    best, trials = pg.batch_autotune(mem, jobs[::8])
    pg.batch_run(mem, jobs, streams=0)  # warm-up at the tuned width
    ms_bat, bat = timed(lambda: pg.batch_run(mem, jobs, streams=0))
    same = all(a["objective"] == b["objective"] for a, (_, b) in zip(seq, bat))
    default_knobs = {"thread_max_deg": 32, "warp_max_deg": 127, "load_factor": 0.5}
    pg.tune_set(mem, streams=best["streams"], **default_knobs)
    ms_def, _ = timed(lambda: pg.batch_run(mem, jobs, streams=0))
    line = {"metric": "Leiden edges/s, batched vs sequential (uneven SBM population)",
            "value": m_total / (ms_bat / 1000.0), "unit": UNIT, "n_gpus": 1, "steps": len(jobs), "warmup": 1,
            "ms_per_step": ms_bat / len(jobs), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "int64", "data": "synthetic",
            "config": {"workload": f"{len(pop)} planted SBMs, n log-uniform in [1000, 200000], 8-512 blocks, "
                                   f"expected degrees 12/3, unit weights, Mod, one pLeiden+ pass each",
                       "vertices_total": int(sum(h.n for h in pop)), "m_total": int(m_total),
                       "generator_seconds": gen_s},
            "sequential": {"value": m_total / (ms_seq / 1000.0), "ms": ms_seq},
            "batched": {"value": m_total / (ms_bat / 1000.0), "ms": ms_bat, "tuned": best},
            "batched_default_knobs": {"value": m_total / (ms_def / 1000.0), "ms": ms_def},
            "batched_over_sequential": ms_seq / ms_bat, "identical_objectives": same,
            "autotune_trials": trials}
    print(json.dumps(line), flush=True)


def filter_eval(args):
    """The learned filter on unseen graphs (seed 99): a DC-SBM with
    n = 16,777,216 at mu = 0.5 (WMod, FP32 weights) and R-MAT scale 25 (Mod),
    pLeiden+ with --eval-ex-iters improvement passes (until stable takes
    minutes per run at these sizes), one run plain and one with the filter
    (and its judge), one stream, CUDA events.  The filter is trained as for the
    headline line."""
    import torch
    import pennsylvaniagpugraphclustering_b200 as pg
    from pennsylvaniagpugraphclustering_b200 import graphgen as gg, move_filter as MF
    torch.cuda.set_device(0)
    mem = pg.memory_store(0)
    stream = torch.cuda.ExternalStream(mem.stream(), device=torch.device("cuda", 0))
    params, thr, info = train_filter(pg, mem, args.recall, args.filter_label)
    MF.scope(mem, -1, args.filter_min_level)
    out = {"metric": "Leiden edges/s, learned filter vs plain on unseen seed-99 graphs", "unit": UNIT,
           "filter": dict(info, min_level=args.filter_min_level), "graphs": {}}
    out["ex_iters"] = args.eval_ex_iters
    for name in ("dcsbm16m", "rmat25"):
        t0 = time.perf_counter()
        if name == "rmat25":
            h = gg.rmat(25, 16, 0.57, 0.19, 0.19, 99)
            obj, w = pg.OBJ_MOD, None
        else:
            h = gg.dcsbm(16777216, 99, mean_deg=gg.DCSBM_4M_MEAN_DEG, mu=0.5)
            obj, w = pg.OBJ_WMOD, h.w
        gen_s = time.perf_counter() - t0
        g = pg.weighted_graph(mem, h.rowptr, h.col, w, objective=obj)
        rec = {"n": h.n, "m_undirected": h.m, "objective": "Mod" if obj == pg.OBJ_MOD else "WMod",
               "generator_seconds": gen_s}
        for mode in ("plain", "learned"):
            if mode == "learned":
                MF.enable(mem, params, thr)
                MF.stats(mem, reset=True)
            try:
                cd = pg.get_objective(mem, g, obj, 1.0)
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                lab, st = pg.run_clustering(mem, g, cd, method=pg.METHOD_LEIDEN_PLUS, ex_iters=args.eval_ex_iters,
                                            seed=99)
                e1.record(stream)
                e1.synchronize()
                ms = e0.elapsed_time(e1)
                ev, sk = MF.stats(mem) if mode == "learned" else (0, 0)
            finally:
                if mode == "learned":
                    MF.disable(mem)
            q, _ = pg.verify_objective(mem, g, lab, obj)
            rec[mode] = {"edges_per_s": h.m / (ms / 1000.0), "seconds": ms / 1000.0, "modularity": st["objective"],
                         "verify_modularity": q, "passes": st["passes"], "filtered_passes": st["filtered_passes"],
                         "exact_passes": st["exact_passes"], "judge_gain": st["judge_gain"],
                         "fell_back": st["fell_back"], "filter_skipped_frac": sk / max(ev + sk, 1)}
            cd.close()
        rec["speedup"] = rec["learned"]["edges_per_s"] / rec["plain"]["edges_per_s"]
        rec["modularity_delta"] = rec["learned"]["modularity"] - rec["plain"]["modularity"]
        out["graphs"][name] = rec
        g.close()
        del h
        print(json.dumps({name: rec}), file=sys.stderr, flush=True)
    print(json.dumps(out), flush=True)


def profile_case(args):
    """The small case for profiler captures: one pLeiden+ pass (ex_iters = 0)
    on the DC-SBM n = 1,048,576 with the workload's parameters (21 M directed
    edges, ~1 GB on the device, inputs above L2), the library's family
    counters on; prints the contraction family's launches, time and
    algorithmic bytes.  Not a bench line."""
    import ctypes
    import pennsylvaniagpugraphclustering_b200 as pg
    from pennsylvaniagpugraphclustering_b200 import _lib, graphgen as gg
    g = gg.dcsbm(1048576, 1, mean_deg=gg.DCSBM_4M_MEAN_DEG)
    mem = pg.memory_store(0)
    wg = pg.weighted_graph(mem, g.rowptr, g.col, g.w, objective=pg.OBJ_WMOD)
    cd = pg.get_objective(mem, wg, pg.OBJ_WMOD, 1.0)
    lib = _lib.lib()
    _lib.check(lib.pggc_profile_enable(mem.handle, 1))
    _, st = pg.run_clustering(mem, wg, cd, method=pg.METHOD_LEIDEN_PLUS, ex_iters=0, seed=1)
    _lib.check(lib.pggc_profile_enable(mem.handle, 0))
    n_l, t_ms, by = ctypes.c_int64(), ctypes.c_double(), ctypes.c_double()
    _lib.check(lib.pggc_profile_read(mem.handle, b"contract", ctypes.byref(n_l), ctypes.byref(t_ms),
                                     ctypes.byref(by)))
    print(json.dumps({"case": "pLeiden+ first pass, DC-SBM n=1,048,576", "n": g.n, "nnz": g.nnz,
                      "levels": st["levels"], "objective": st["objective"], "contractions": n_l.value,
                      "contract_ms": t_ms.value, "contract_algorithmic_bytes": by.value}))


def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
    elif args.workload == "dcsbm4m":
        ours(args)
    elif args.workload == "sbm-population":
        population(args)
    elif args.workload == "filter-eval":
        filter_eval(args)
    elif args.workload == "profile-case":
        profile_case(args)
    else:
        plain_workload(args)


if __name__ == "__main__":
    main()
