#!/usr/bin/env python
"""GCUPS of the Smith-Waterman hot path on B200.

Workload (the configuration the metric is quoted on): protein, affine gap,
batched uneven lengths -- 200 queries (log-normal, median 350 aa, 100-1000)
against 2,000 targets (50-2,000 aa), BLOSUM62, gap open -11 / extension -1,
10% of pairs sharing a planted 150-aa domain at 40% identity: 400,000 pairs,
all-vs-all, full path (score sweep, starting points, traceback walk, hits).
Synthetic, seeded (pypaswas_b200.workloads.config2).

One "step" = one pw_align over all 400,000 pairs with the sequences resident
in HBM.  `e2e` repeats the step through the public driver
(SmithWatermanB200.align_sequences) from host sequence records, host<->device
copies and Hit construction included.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun (N > 1) every rank aligns its own replica of the workload
(pairs are independent; no collective on the data path): weak scaling.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

import numpy as np  # noqa: E402

# algorithmic operations per cell (add and max counted separately) of the
# recurrences: linear/affine, score only / with direction classification
# the trimmer workload's end-to-end leg builds Python Hit objects: it runs on
# the first reads only (the bench line names the sample)
E2E_READS = 200_000

OPS_PER_CELL = {("linear", "score"): 5, ("linear", "dirs"): 8, ("affine", "score"): 10, ("affine", "dirs"): 14}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", type=int, choices=[1, 2, 3, 4], default=2,
                    help="workload: 1 DNA reads x adapters, 2 protein batched (the metric's configuration), "
                         "3 long DNA pairs, 4 trimmer reads x adapters")
    ap.add_argument("--reads", type=int, default=10_000_000, help="config 4: number of reads")
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="target length of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--targets", type=int, default=0,
                    help="use only every k-th target so that N targets remain (small cases for ncu captures; "
                         "the bench line then names the reduced workload)")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (ncu captures)")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain one-pair-per-launch leg")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving leg")
    ap.add_argument("--no-chain", action="store_true", help="16-bit sweep without chained strips (comparison)")
    ap.add_argument("--tune", action="append", default=[], metavar="KEY=VALUE",
                    help="engine tuning knob (chain_min, grid_share), e.g. --tune chain_min=250; "
                         "without chain_min the autotuner picks it during the warm-up")
    ap.add_argument("--serve-seconds", type=float, default=6.0, help="length of each arrival stream of the serving leg")
    ap.add_argument("--serve-loads", default="0.3,0.5,0.6,0.7", help="offered loads (fractions of batched peak) swept")
    return ap.parse_args()


def workload(args):
    from pypaswas_b200 import workloads
    if args.config == 1:
        return workloads.config1()
    if args.config == 3:
        return workloads.config3()
    if args.config == 4:
        return workloads.config4(n_reads=args.reads)
    w = workloads.config2()
    if args.targets and args.targets < len(w.targets):
        step = len(w.targets) // args.targets
        w = workloads.Workload("%s, sample: every %d-th target (%d targets)" % (w.name, step, args.targets),
                               w.queries, w.targets[::step][:args.targets], w.settings)
    return w


def reduce_max(x):
    """Max of a float over the ranks of the default process group (identity
    without one): the job's time is its slowest rank's."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_gcups(cells_per_rank, steps, seconds, world):
    """Weak scaling: every rank aligns its own replica; GCUPS of the whole job."""
    return world * cells_per_rank * steps / seconds / 1e9


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), \
        int(os.environ.get("LOCAL_RANK", "0"))


class ClockSampler(object):
    """nvidia-smi clock / throttle samples while the timed region runs."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.lines = []
        self.t0 = 0.0

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.QUERY,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def mark(self):
        """Start of the timed region: later samples only."""
        self.t0 = time.time()

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ts, ln in self.lines:
            if ts < self.t0:
                continue
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def load_peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def load_traffic():
    """DRAM bytes per launch of the dominant kernel from the committed ncu summary."""
    try:
        with open(os.path.join(REPO, "profiles", "traffic.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def engine_for(workload, device):
    from pypaswas_b200 import _native, scores
    from pypaswas_b200.smith_waterman import configure_engine, id_keys
    score = scores.make_score(workload.settings)
    e = _native.Engine(device)
    configure_engine(e, score, workload.settings)
    if workload.queries is None:  # packed reads (trimmer workload): read ids never equal target ids
        n, L = workload.reads.shape
        e.set_queries_packed(workload.reads, np.arange(n + 1, dtype=np.int64) * L, np.arange(n, dtype=np.int32))
        e.set_targets([s for _, s in workload.targets], np.arange(len(workload.targets), dtype=np.int32) + n)
    else:
        qk, tk = id_keys([i for i, _ in workload.queries], [i for i, _ in workload.targets])
        e.set_queries([s for _, s in workload.queries], qk)
        e.set_targets([s for _, s in workload.targets], tk)
    if workload.pairs is not None:
        e.set_pairs([p[0] for p in workload.pairs], [p[1] for p in workload.pairs])
    return e, score


def cpu_baseline(workload, score, seconds, processes=1):
    """The oracle (CPU restatement of the reference path) on a bounded sample of
    the workload: queries x targets taken evenly from the length-sorted lists
    (or, with explicit pairs, the first pairs).  The sample is sized for about
    `seconds` of work: a first run at an estimated rate calibrates a second,
    larger one if the first was much shorter."""
    rate = 24e6 * max(1, processes)  # cells/s first estimate of the oracle
    r = None
    for _ in range(3):
        r = _cpu_sample(workload, score, seconds * rate, processes)
        if r["seconds"] >= 0.4 * seconds or r["full"]:
            break
        rate = r["cells"] / max(r["seconds"], 1e-3)
    return {k: v for k, v in r.items() if k not in ("cells", "full")}


def _cpu_sample(workload, score, budget_cells, processes):
    import multiprocessing as mp
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle
    oracle.build()
    q_all = [s.decode() for _, s in workload.queries]
    t_all = [s.decode() for _, s in workload.targets]
    args = _oracle_args(score, workload.settings)
    if workload.pairs is not None:
        jobs, cells = [], 0
        for qi, ti in workload.pairs:
            if cells and cells + len(q_all[qi]) * len(t_all[ti]) > budget_cells:
                break
            jobs.append((args, [q_all[qi]], [t_all[ti]]))
            cells += len(q_all[qi]) * len(t_all[ti])
        full = len(jobs) == len(workload.pairs)
        sample = "the first %d explicit pairs (%d cells) of the same workload, full path" % (len(jobs), cells)
    else:
        # targets first (up to all of them) against 10 queries, then more queries
        nq = min(len(q_all), 10)
        q10 = sum(map(len, q_all[::max(1, len(q_all) // nq)][:nq]))
        t_avg = sum(map(len, t_all)) / max(1, len(t_all))
        nt = min(len(t_all), max(1, int(budget_cells / (q10 * t_avg))))
        ts = t_all[::max(1, len(t_all) // nt)][:nt]
        q_avg = sum(map(len, q_all)) / max(1, len(q_all))
        nq = min(len(q_all), max(nq, int(budget_cells / (q_avg * sum(map(len, ts))))))
        qs = q_all[::max(1, len(q_all) // nq)][:nq]
        cells = sum(map(len, qs)) * sum(map(len, ts))
        jobs = [(args, qs, ts[i::processes]) for i in range(max(1, processes))]
        jobs = [j for j in jobs if j[2]]
        full = len(qs) == len(q_all) and len(ts) == len(t_all)
        sample = "%d queries x %d targets (%d cells) of the same workload, full path" % (len(qs), len(ts), cells)
    t0 = time.time()
    if processes <= 1:
        for j in jobs:
            _oracle_chunk(j)
    else:
        ctx = mp.get_context("spawn")
        with ctx.Pool(processes) as pool:
            pool.map(_oracle_chunk, jobs)
    dt = time.time() - t0
    return {"value": cells / dt / 1e9, "unit": "GCUPS", "cores": processes, "kind": "port", "sample": sample,
            "seconds": dt, "cells": cells, "full": full}


def _oracle_args(score, settings):
    gap, ext, affine, ll, mn = score.kernel_constants()
    return (score.matrix_array(), score.char_offset_code(), float(gap), float(ext), bool(affine), float(ll),
            float(mn), float(score.highest_score), float(settings.filter_factor), float(settings.minimum_score))


def _oracle_chunk(job):
    args, qs, ts = job
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle
    m, off, gap, ext, affine, ll, mn, hi, ff, host_min = args
    p = oracle.OracleParams(m, off, gap, ext, affine, ll, mn)
    pos = np.array([[np.float32(hi * min(len(q), len(t)) * ff) for q in qs] for t in ts], np.float32)
    return len(oracle.run(p, qs, ts, pos, host_min)["hits"])


def run_reference(args, workload_fn):
    rank, world, local = dist_env()
    if rank != 0:
        return 0
    w = workload_fn()
    from pypaswas_b200 import scores
    score = scores.make_score(w.settings)
    procs = os.cpu_count() or 1
    steps = []
    # each step a bounded sample: the whole run stays near two minutes
    per_step = max(1.0, min(args.cpu_seconds, 20.0, 120.0 / max(1, args.warmup + args.steps)))
    for i in range(args.warmup + args.steps):
        r = cpu_baseline(w if w.queries is not None else w.head(200000), score, per_step, processes=procs)
        if i >= args.warmup:
            steps.append(r)
    v = float(np.median([s["value"] for s in steps]))
    line = {"impl": "reference", "metric": "GCUPS", "value": v, "unit": "GCUPS", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": w.name,
                       "pairs": len(w.pairs) if w.pairs is not None else w.n_queries * len(w.targets)},
            "cpu_baseline": {"value": v, "unit": "GCUPS", "cores": procs, "kind": "port",
                             "sample": steps[0]["sample"]},
            "e2e": {"value": v, "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "CPU restatement of the reference path (oracle/paswas_oracle.c) over all host cores"}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    from pypaswas_b200 import workloads
    if args.impl == "reference":
        return run_reference(args, lambda: workload(args))
    rank, world, local = dist_env()
    import torch
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    torch.cuda.set_device(local)
    w = workload(args)
    e, score = engine_for(w, local)
    cells = w.cells
    affine = score.gap_extension is not None
    mode = "affine" if affine else "linear"
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # > L2 (126 MB)

    chain = not args.no_chain
    from pypaswas_b200 import _native
    knobs = {"chain_min": _native.PW_TUNE_CHAIN_MIN, "grid_share": _native.PW_TUNE_GRID_SHARE,
             "segment": _native.PW_TUNE_SEGMENT, "dual": _native.PW_TUNE_DUAL, "cand_slot": _native.PW_TUNE_CAND_SLOT}
    tuning = {}
    for kv in args.tune:
        key, val = kv.split("=")
        e.set_tuning(knobs[key], int(val))
        tuning[key] = int(val)
    if "chain_min" not in tuning and chain and w.pairs is None:
        from pypaswas_b200.autotune import autotune
        tuning["autotune"] = autotune(e)  # untimed: score sweeps on this workload
    sampler = ClockSampler(local)
    sampler.start()  # started before the warm-up: nvidia-smi is up when timing begins
    for _ in range(args.warmup):
        e.align(chain=chain)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    sampler.mark()  # samples before this point are dropped
    times, infos = [], []
    for _ in range(args.steps):
        flush.zero_()  # between timed iterations: L2 flushed
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        info = e.align(chain=chain)  # synchronous: returns when the step's device work is done
        b.record()
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b))
        infos.append(info.as_dict())
    clocks = sampler.stop()
    t_ms = reduce_max(float(sum(times)))
    step_stats = {"min": float(min(times)), "median": float(np.median(times)), "max": float(max(times)),
                  "all": [round(float(t), 3) for t in times],
                  "call_ms": [round(float(i["total_ms"]), 3) for i in infos],
                  "phase_ms": {k: [round(float(i[k]), 2) for i in infos] for k in
                               ("score_ms", "trace_ms", "walk_ms", "setup_ms", "finish_ms")}}
    value = whole_job_gcups(cells, args.steps, t_ms * 1e-3, world)
    n_pairs = len(w.pairs) if w.pairs is not None else w.n_queries * len(w.targets)
    ms_per_step = t_ms / args.steps

    # roofline of the dominant kernel (integer-ALU bound: DPX add-max issue rate)
    last = infos[-1]
    trace_ms = sum(i["trace_kernel_ms"] for i in infos)
    score_ms = sum(i["score_kernel_ms"] for i in infos)
    if trace_ms >= score_ms:
        wp, tp = last["warp_pairs"], last["traced_pairs"]
        which = "band_kernel, one pair per warp" if wp >= tp else (
            "sweep_kernel phase 2" if wp == 0 else "sweep_kernel phase 2 + band_kernel")
        dom, dom_ms, dom_launch = "direction sweep (%s)" % which, trace_ms, sum(
            i["trace_launches"] for i in infos)
        ops = sum(i["traced_cells"] for i in infos) * OPS_PER_CELL[(mode, "dirs")]
    else:
        dom, dom_ms, dom_launch = "score sweep (score16_chain_kernel, 16x2 lanes)" if _sixteen_bit(e, w) else \
            ("score sweep (band_kernel, bands chained across warps)" if e.last_info.score_path == 2 else
             "score sweep (sweep_kernel phase 1)"), score_ms, sum(
            i["score_launches"] for i in infos)
        ops = cells * OPS_PER_CELL[(mode, "score")] * args.steps
    peak32, peak16, _ = e.measure_int_peak()
    lanes16 = "score" in dom and _sixteen_bit(e, w)
    peak_ops = peak16 if lanes16 else peak32
    achieved = ops / (dom_ms * 1e-3) / 1e12
    traffic = load_traffic().get("direction_sweep_bytes_per_launch" if "direction" in dom else
                                 "score_sweep_bytes_per_launch")

    # end to end through the public driver, host records in, hits out
    e2e_w = w if w.queries is not None else w.head(E2E_READS)
    e2e_value, h2d, d2h = None, 0, 0
    if not args.no_e2e:
        if world > 1:
            torch.distributed.barrier()
        dt, h2d, d2h = _e2e(e2e_w, args.steps, local)
        dt = reduce_max(dt)  # whole job: every rank's replica, the slowest rank's time
        e2e_value = whole_job_gcups(e2e_w.cells, args.steps, dt, world)

    out = {"metric": "GCUPS", "value": value, "unit": "GCUPS", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms_per_step, "step_ms": step_stats,
           "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "int32", "data": "synthetic",
           "config": {"workload": "%s (%d pairs, full path)" % (w.name, n_pairs),
                      "pairs": n_pairs,
                      "cells_per_step": cells, "traced_pairs": last["traced_pairs"],
                      "cand_overflow_pairs": last["cand_overflow_pairs"],
                      "starting_points": last["starting_points"], "hits": last["hits"],
                      "score_lanes": "targets" if last["orientation"] else "queries",
                      "trace_lanes": "targets" if last["trace_orientation"] else "queries",
                      "minimum_score": w.settings.minimum_score, "lower_limit_score": w.settings.lower_limit_score,
                      "filter_factor": w.settings.filter_factor,
                      "l2": "flushed between steps (256 MiB write); each step also writes >1e11 B of cell codes",
                      "parallelism": "replica per GPU" if world > 1 else "single GPU",
                      "tuning": tuning},
           "phases_ms": {"score": last["score_ms"], "trace": last["trace_ms"], "walk": last["walk_ms"],
                         "score_kernels": last["score_kernel_ms"], "trace_kernels": last["trace_kernel_ms"],
                         "host_setup": last["setup_ms"], "host_finish": last["finish_ms"], "call": last["total_ms"]},
           "gpu_launches": int(sum(i["kernel_launches"] for i in infos)),
           "clocks": clocks,
           "roofline": {"bound": "int_alu", "kernel": dom, "achieved": achieved,
                        "peak": peak_ops / 1e12, "unit": "Tops/s", "frac": achieved / (peak_ops / 1e12),
                        "peak_source": "measured in this run: DPX add-max issue probe (pw_measure_int_peak), "
                                       + ("16x2 form" if lanes16 else "32-bit form"),
                        "ops_per_cell": OPS_PER_CELL[(mode, "dirs" if "direction" in dom else "score")],
                        "launches": dom_launch, "avg_launch_ms": dom_ms / max(1, dom_launch),
                        "traffic": traffic,
                        "hbm_gbs_measured": load_peaks().get("hbm_gbs")},
           "e2e": {"value": e2e_value, "unit": "GCUPS", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                   "workload": e2e_w.name}}
    if not args.no_plain and w.pairs is None:
        out["plain"] = plain_vs_batched(w if w.queries is not None else w.head(64), local, value)
    if not args.no_serve and rank == 0 and args.config == 2:
        out["serve"] = serve_leg(local, args.serve_seconds, [float(x) for x in args.serve_loads.split(",")])
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(w if w.queries is not None else w.head(20000), score, args.cpu_seconds,
                                           processes=1)
    if rank == 0:
        print(json.dumps(out), flush=True)
    e.close()
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


def plain_vs_batched(w, device, batched_value, n_q=8, n_t=64):
    """GCUPS of the plain form -- one (query, target) pair per kernel launch,
    the shape of the reference's per-pair kernel calls -- on an evenly spaced
    sample of the workload, next to the batched engine on the same sample.
    Both run the full path (score, starting points, walk)."""
    import torch
    from pypaswas_b200 import workloads
    qs = w.queries[::max(1, len(w.queries) // n_q)][:n_q]
    ts = w.targets[::max(1, len(w.targets) // n_t)][:n_t]
    sample = workloads.Workload(w.name + " sample", qs, ts, w.settings)
    e, _ = engine_for(sample, device)
    out = {}
    for label, plain in (("batched", False), ("plain", True)):
        e.align(plain=plain)  # warm-up
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        info = e.align(plain=plain)
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b)
        out[label] = {"value": sample.cells / (ms * 1e-3) / 1e9, "ms": ms, "launches": int(info.kernel_launches),
                      "hits": int(info.hits)}
    e.close()
    return {"value": out["plain"]["value"], "unit": "GCUPS",
            "sample": "%d queries x %d targets (%d pairs, %d cells), evenly spaced in length order"
                      % (len(qs), len(ts), len(qs) * len(ts), sample.cells),
            "launches": out["plain"]["launches"], "batched_same_sample": out["batched"]["value"],
            "batched_over_plain": batched_value / out["plain"]["value"],
            "hits_equal": out["plain"]["hits"] == out["batched"]["hits"]}


def serve_leg(device, seconds, loads, workers=2, max_batch=32):
    """Serving configuration: a resident database of 100,000 protein sequences
    (log-normal lengths, median 300, 50-1,500 aa), Poisson arrivals of single
    queries (log-normal, median 300, max 5,000 aa), 70% top-10 by pair maximum
    and 30% full affine traceback (BLOSUM62, -11/-1).  First the batched peak:
    64 requests submitted at once; then, for each offered load (a fraction of
    that peak), an arrival stream of `seconds`, reporting p50/p99 latency and
    the GCUPS served."""
    from pypaswas_b200 import serving, workloads
    st = workloads.Settings(**workloads.C5_SETTINGS)
    db = workloads.protein_database()
    srv = serving.Server(st, device=device, workers=workers, max_batch=max_batch)
    sweep = []
    try:
        srv.load_db(db)
        serving.run_arrivals(srv, workloads.query_stream(seed=8, n=16, rate_hz=1e9))
        peak = serving.run_arrivals(srv, workloads.query_stream(seed=7, n=64, rate_hz=1e9))
        probe = workloads.query_stream(seed=9, n=4000, rate_hz=1.0)
        mean_cells = float(np.mean([len(q[2]) for q in probe])) * srv.db_residues
        for k, load in enumerate(loads):
            rate = load * peak["gcups"] * 1e9 / mean_cells
            stream = workloads.query_stream(seed=60 + k, n=max(20, int(rate * seconds)), rate_hz=rate)
            rep = serving.run_arrivals(srv, stream)
            sweep.append({"offered_load": load, "offered_rps": rep["offered_rps"], "gcups": rep["gcups"],
                          "fraction_of_peak": rep["gcups"] / peak["gcups"], "p50_ms": rep["p50_ms"],
                          "p99_ms": rep["p99_ms"], "max_ms": rep["max_ms"], "p99_top_ms": rep["p99_top_ms"],
                          "p99_traceback_ms": rep["p99_traceback_ms"], "requests": rep["requests"],
                          "mean_batch": rep["mean_batch"], "workers_used": rep["workers_used"],
                          "peak_reserved_bytes": rep["peak_reserved_bytes"]})
    finally:
        srv.close()
    return {"db": "%d sequences, %d residues, resident" % (len(db), srv.db_residues),
            "workers": workers, "max_batch": max_batch, "batched_peak_gcups": peak["gcups"],
            "seconds_per_rate": seconds, "sweep": sweep}


def _sixteen_bit(engine, w):
    """The score sweep ran on 16-bit lanes (integer scores; see pw_score16.cuh)."""
    return engine.last_info is not None and engine.last_info.score_launches > 0 and \
        engine.last_info.score_path == 0 and engine.last_info.overflow_pairs == 0 and _integer_scores(w)


def _integer_scores(w):
    from pypaswas_b200 import scores
    m = scores.make_score(w.settings).matrix_array()
    return bool(np.all(np.floor(m) == m) and np.all(np.abs(m) <= 127))


def _e2e(w, steps, device):
    """Public driver path: Aligner.process on host records -> HitList.  With
    explicit pairs (long DNA), one process() call per query against its
    targets, as the reference would be run once per pair."""
    import torch
    from pypaswas_b200.formatters import TrimmerFormatter
    from pypaswas_b200.programs import Aligner, Trimmer
    from pypaswas_b200.records import SeqRecord
    trimmer = getattr(w.settings, "program", "aligner") == "trimmer"
    queries = [SeqRecord(s, i) for i, s in w.queries]
    targets = [SeqRecord(s, i) for i, s in w.targets]
    if w.pairs is None:
        calls = [(queries, targets)]
    else:
        per_q = {}
        for qi, ti in w.pairs:
            per_q.setdefault(qi, []).append(targets[ti])
        calls = [([queries[qi]], ts) for qi, ts in sorted(per_q.items())]
    aligner = (Trimmer if trimmer else Aligner)(None, None, w.settings, device=device)
    for qs, ts in calls[:2]:
        aligner.process(qs, ts, None)  # warm-up
    torch.cuda.synchronize()
    h2d = d2h = 0
    t0 = time.perf_counter()
    for _ in range(steps):
        h2d = d2h = 0
        for qs, ts in calls:
            hl = aligner.process(qs, ts, None)
            if trimmer:
                TrimmerFormatter(None, hl, None).lines()  # the program's trimmedFasta records
            h2d += int(aligner.smith_waterman.last_h2d_bytes)
            d2h += int(aligner.smith_waterman.last_d2h_bytes)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    return dt, h2d, d2h


if __name__ == "__main__":
    sys.exit(main())
