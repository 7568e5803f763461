#!/usr/bin/env python
"""GCUPS of the Smith-Waterman hot path on B200.

Headline workload (the configuration the metric is quoted on): protein, affine
gap, batched uneven lengths -- 200 queries (log-normal, median 350 aa,
100-1000) against 2,000 targets (50-2,000 aa), BLOSUM62, gap open -11 /
extension -1, 10% of pairs sharing a planted 150-aa domain at 40% identity:
400,000 pairs, all-vs-all, full path (score sweep, starting points, traceback
walk, hits).  Synthetic, seeded (pypaswas_b200.workloads.config2).

The same JSON line carries one record per further configuration under
"configs": DNA reads x adapters (C1), long DNA pairs (C3) and the trimmer's
10 M reads (C4), each with the same legs.

Legs of every configuration:
  value     one step = one pw_align over the whole workload, sequences
            resident in HBM, the score sweep's work list rebuilt every step
            (PW_FLAG_REPLAN); CUDA events around each step, L2 flushed between
            steps
  e2e       the same metric through the public driver API with host records:
            Aligner.process -> HitList (for the trimmer: FASTA text -> native
            reader -> Trimmer.trimmed_fasta -> text), inputs alternating between
            two seeded sets of the same
            shape so that every step copies and prepares its inputs anew; the
            bytes are the engine's own count of its host<->device copies
  plain     the unbatched form (one pair per launch) against the batched
            engine on the same sample
  parity    the engine against the oracle on the CPU baseline's sample
  roofline  the dominant kernel's algorithmic ops per second against the DPX
            issue peak measured in the same run
  cpu_baseline  the oracle on one host core over a bounded sample

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun (N > 1) every rank aligns its own replica of the headline
workload (pairs are independent; no collective on the data path): weak
scaling; the further configurations and the serving leg run at N = 1 only.
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
OPS_PER_CELL = {("linear", "score"): 5, ("linear", "dirs"): 8, ("affine", "score"): 10, ("affine", "dirs"): 14}
# the trimmer workload's end-to-end leg aligns this many reads per step
E2E_READS = 2_000_000
NAMES = {1: "C1", 2: "C2", 3: "C3", 4: "C4"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", type=int, choices=[1, 2, 3, 4], default=2,
                    help="headline workload: 1 DNA reads x adapters, 2 protein batched (the metric's "
                         "configuration), 3 long DNA pairs, 4 trimmer reads x adapters")
    ap.add_argument("--also", default="auto",
                    help="further configurations in the same line, e.g. 1,3,4; 'auto' = the other three when the "
                         "headline is config 2, 'none' = headline only")
    ap.add_argument("--reads", type=int, default=10_000_000, help="config 4: number of reads")
    ap.add_argument("--pairs", type=int, default=64,
                    help="config 3: number of long pairs, each aligned with the target and its reverse complement "
                         "(small cases for ncu captures)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="length of the headline's CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--targets", type=int, default=0,
                    help="config 2: use only every k-th target so that N targets remain (small cases for ncu "
                         "captures; the bench line then names the reduced workload)")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (ncu captures)")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain one-pair-per-launch leg")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving leg")
    ap.add_argument("--no-chain", action="store_true", help="16-bit sweep without chained strips (comparison)")
    ap.add_argument("--plan-cached", action="store_true",
                    help="keep the score sweep's work list between steps (inputs unchanged)")
    ap.add_argument("--tune", action="append", default=[], metavar="KEY=VALUE",
                    help="engine tuning knob (chain_min, grid_share, segment, dual, cand_slot, lanes, trace_store, tile_trace, wait_ns), e.g. "
                         "--tune chain_min=250; without chain_min the autotuner picks it during the warm-up")
    ap.add_argument("--serve-seconds", type=float, default=20.0, help="length of each arrival stream of the serving leg")
    ap.add_argument("--serve-loads", default="0.5,0.7", help="offered loads (fractions of batched peak) swept")
    ap.add_argument("--serve-streams", type=int, default=3,
                    help="arrival streams per offered load (different seeds); the report gives the median p99")
    ap.add_argument("--serve-workers", type=int, default=2)
    ap.add_argument("--serve-max-batch", type=int, default=6)
    ap.add_argument("--serve-max-residues", type=int, default=0,
                    help="query residues per serving batch (0: no limit)")
    ap.add_argument("--serve-policy", type=int, default=1, help="0 arrival order, 1 shortest first with aging")
    return ap.parse_args()


def workload(cfg, args, seed=None):
    """The configuration's workload; `seed` draws another set of the same shape."""
    from pypaswas_b200 import workloads
    kw = {} if seed is None else {"seed": seed}
    if cfg == 1:
        return workloads.config1(**kw)
    if cfg == 3:
        return workloads.config3(n_pairs=args.pairs, **kw)
    if cfg == 4:
        return workloads.config4(n_reads=args.reads, **kw)
    w = workloads.config2(**kw)
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
        self.t1 = None

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
        self.t1 = None

    def mark_end(self):
        """End of the timed region: samples after it are not counted."""
        self.t1 = time.time()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ts, ln in list(self.lines):
            if ts < self.t0 or (self.t1 is not None and ts > self.t1):
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
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()


def load_peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def load_traffic():
    """DRAM bytes per launch of dominant kernels from the committed ncu summaries."""
    try:
        with open(os.path.join(REPO, "profiles", "traffic.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def engine_for(w, device):
    from pypaswas_b200 import _native, scores
    from pypaswas_b200.smith_waterman import configure_engine, id_keys
    score = scores.make_score(w.settings)
    e = _native.Engine(device)
    configure_engine(e, score, w.settings)
    if w.queries is None:  # packed reads (trimmer workload): read ids never equal target ids
        n, L = w.reads.shape
        e.set_queries_packed(w.reads, np.arange(n + 1, dtype=np.int64) * L, np.arange(n, dtype=np.int32))
        e.set_targets([s for _, s in w.targets], np.arange(len(w.targets), dtype=np.int32) + n)
    else:
        qk, tk = id_keys([i for i, _ in w.queries], [i for i, _ in w.targets])
        e.set_queries([s for _, s in w.queries], qk)
        e.set_targets([s for _, s in w.targets], tk)
    if w.pairs is not None:
        e.set_pairs([p[0] for p in w.pairs], [p[1] for p in w.pairs])
    return e, score


def _mode(score):
    return "affine" if score.gap_extension is not None else "linear"


# ------------------------------------------------------------------ device step
def device_steps(e, steps, warmup, replan, chain, flush, sampler=None, world=1):
    """`steps` timed pw_align calls after `warmup` untimed ones: CUDA events
    around each call (which returns when its device work is done), L2 flushed
    before each.  Returns (per-step ms, per-step run infos)."""
    import torch
    for _ in range(warmup):
        e.align(chain=chain, replan=replan)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    if sampler is not None:
        sampler.mark()
    times, infos = [], []
    for _ in range(steps):
        flush.zero_()  # between timed iterations: L2 flushed
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        info = e.align(chain=chain, replan=replan)
        b.record()
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b))
        infos.append(info.as_dict())
    if sampler is not None:
        sampler.mark_end()
    return times, infos


def roofline(e, w, score, infos, steps):
    """The dominant kernel (score or direction sweep) against the DPX issue
    peak measured now: algorithmic ops / its summed launch time."""
    mode = _mode(score)
    last = infos[-1]
    trace_ms = sum(i["trace_kernel_ms"] for i in infos)
    score_ms = sum(i["score_kernel_ms"] for i in infos)
    sixteen = last["score_path"] == 0 and last["overflow_pairs"] == 0 and last["score_launches"] > 0
    if trace_ms >= score_ms:
        wp, tp = last["warp_pairs"], last["traced_pairs"]
        which = "band_kernel, one pair per warp" if wp >= tp else (
            "sweep_kernel phase 2" if wp == 0 else "sweep_kernel phase 2 + band_kernel")
        dom, dom_ms, launches = "direction sweep (%s)" % which, trace_ms, sum(i["trace_launches"] for i in infos)
        ops = sum(i["traced_cells"] for i in infos) * OPS_PER_CELL[(mode, "dirs")]
        per_cell = OPS_PER_CELL[(mode, "dirs")]
        lanes16 = False
    else:
        dom = {0: "score sweep (score16_chain_kernel / score16_kernel, 16x2 lanes)",
               1: "score sweep (sweep_kernel phase 1, 32-bit lanes)",
               2: "score sweep (band_kernel, bands chained across warps)"}.get(last["score_path"], "score sweep")
        if last["score_path"] == 2 and last.get("tile_pairs"):
            dom = "score sweep (band_kernel, bands chained across warps, keeping the tile form's checkpoints)"
        if last["score_path"] == 2 and 2 * last.get("paired_cells", 0) >= last["cells"]:
            # most cells on the 16x2 band sweep: its DPX issue peak is the 16x2 one
            dom = ("score sweep (band16_kernel: a pair and its reverse-complement pair in 16-bit halves, bands "
                   "chained across warps, keeping the tile form's checkpoints)")
            sixteen = True
        dom_ms, launches = score_ms, sum(i["score_launches"] for i in infos)
        ops = w.cells * OPS_PER_CELL[(mode, "score")] * steps
        per_cell = OPS_PER_CELL[(mode, "score")]
        lanes16 = sixteen
    peak32, peak16, _ = e.measure_int_peak()
    peak = peak16 if lanes16 else peak32
    if dom.startswith("direction") and last.get("trace_store"):
        # the H-storing direction sweep: the score recurrence plus a 2-byte
        # store per cell; its roof is the HBM write of those bytes
        ops = sum(i["traced_cells"] for i in infos) * OPS_PER_CELL[(mode, "score")]
        per_cell = OPS_PER_CELL[(mode, "score")]
        written = sum(i["traced_cells"] for i in infos) * 2
        peaks = load_peaks()
        hbm = peaks.get("hbm_gbs")
        src = "measured (MEASURED_PEAKS.json hbm_gbs)" if hbm else "fallback 6,650 GB/s (no MEASURED_PEAKS.json)"
        hbm = float(hbm or 6650.0)
        gbs = written / (dom_ms * 1e-3) / 1e9
        alu = ops / (dom_ms * 1e-3) / 1e12
        return {"bound": "hbm", "kernel": dom + ", 16-bit H stored per cell", "achieved": gbs, "peak": hbm,
                "unit": "GB/s", "frac": gbs / hbm, "peak_source": src, "bytes_per_cell": 2,
                "alu": {"achieved": alu, "peak": peak / 1e12, "unit": "Tops/s", "frac": alu / (peak / 1e12),
                        "ops_per_cell": per_cell},
                "launches": launches, "avg_launch_ms": dom_ms / max(1, launches)}
    achieved = ops / (dom_ms * 1e-3) / 1e12
    return {"bound": "int_alu", "kernel": dom, "achieved": achieved, "peak": peak / 1e12, "unit": "Tops/s",
            "frac": achieved / (peak / 1e12),
            "peak_source": "measured in this run: DPX add-max issue probe (pw_measure_int_peak), "
                           + ("16x2 form" if lanes16 else "32-bit form"),
            "ops_per_cell": per_cell, "launches": launches, "avg_launch_ms": dom_ms / max(1, launches)}


# ------------------------------------------------------------------ end to end
def _records(w):
    from pypaswas_b200.records import SeqRecord
    if w.queries is None:
        qs = [SeqRecord(w.reads[i].tobytes(), w.read_ids[i]) for i in range(len(w.read_ids))]
    else:
        qs = [SeqRecord(s, i) for i, s in w.queries]
    return qs, [SeqRecord(s, i) for i, s in w.targets]


def _e2e_calls(w):
    """(queries, targets, explicit pairs or None) per public-API call: one
    Aligner.process call for all-vs-all, one Aligner.process_pairs call with
    explicit pairs."""
    qs, ts = _records(w)
    return [(qs, ts, w.pairs)]


def _fasta_bytes(w):
    """The trimmer workload as the two FASTA files a user hands the program:
    (reads, adapters) as bytes."""
    n = w.reads.shape[0]
    lines = []
    for i in range(n):
        lines.append(b">" + str(w.read_ids[i]).encode())
        lines.append(w.reads[i].tobytes())
    reads = b"\n".join(lines) + b"\n"
    adapters = b"".join(b">%s\n%s\n" % (i.encode(), s) for i, s in w.targets if not i.endswith("_RC"))
    return reads, adapters


def e2e_leg(ws, steps, device, trimmer):
    """The public driver API with host inputs; step k runs input set
    ws[k % len(ws)] (two sets: every step's inputs are new to the engine).
    Aligner: records -> Aligner.process -> HitList.  Trimmer: FASTA text ->
    native reader (reads sorted, adapters with their reverse complements)
    -> Trimmer.trimmed_fasta -> trimmedFasta text.
    Returns (cells, seconds, h2d bytes per step, d2h bytes per step, reuse bits seen)."""
    import torch
    from pypaswas_b200 import readers, scores
    from pypaswas_b200.programs import Aligner, Trimmer
    st = ws[0].settings
    sets = [(_fasta_bytes(w) if trimmer else _e2e_calls(w), w.cells) for w in ws]
    prog = (Trimmer if trimmer else Aligner)(None, None, st, device=device)
    sw = prog.smith_waterman
    score = scores.make_score(st)
    timing = []

    def step(calls):
        h2d = d2h = 0
        reuse = 0
        if trimmer:
            t0 = time.perf_counter()
            q = readers.read_query_records(st, calls[0])
            t = readers.read_target_records(st, score, calls[1])
            t1 = time.perf_counter()
            prog.trimmed_fasta(q, t)  # the program's output text, natively
            timing.append({"read_ms": (t1 - t0) * 1e3, "align_and_format_ms": (time.perf_counter() - t1) * 1e3,
                           "engine_ms": float(sw.last_info.total_ms)})
            return sw.last_h2d_bytes, sw.last_d2h_bytes, int(sw.last_info.reuse)
        for qs, ts, pairs in calls:
            if pairs is None:
                prog.process(qs, ts, None)  # HitList of Hit objects
            else:
                prog.process_pairs(qs, ts, pairs)
            h2d += sw.last_h2d_bytes
            d2h += sw.last_d2h_bytes
            reuse |= int(sw.last_info.reuse)
            timing.append(dict(sw.last_timing))
        return h2d, d2h, reuse

    try:
        for k in range(2):
            step(sets[k % len(sets)][0])  # warm-up
        torch.cuda.synchronize()
        h2d = d2h = reuse = 0
        cells = 0
        t0 = time.perf_counter()
        for k in range(steps):
            calls, c = sets[k % len(sets)]
            a, b, r = step(calls)
            h2d += a
            d2h += b
            reuse |= r
            cells += c
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
    finally:
        sw.close()
    parts = {k: float(np.median([t[k] for t in timing[-steps:]])) for k in timing[0]} if timing else {}
    return cells, dt, h2d // steps, d2h // steps, reuse, parts


# ------------------------------------------------------------------ plain form
def plain_leg(w, device, n_q, n_t):
    """GCUPS of the plain form -- one (query, target) pair per launch, the
    shape of the reference's per-pair kernel calls -- against the batched
    engine on the same sample; both the full path (score, starting points,
    walk).  Explicit pairs: the first n_q queries' pairs."""
    import torch
    from pypaswas_b200 import workloads
    if w.pairs is not None:
        sample = w.head(n_q)
        desc = "%d explicit pairs (%d cells)" % (len(sample.pairs), sample.cells)
    else:
        qs = w.queries[::max(1, len(w.queries) // n_q)][:n_q]
        ts = w.targets[::max(1, len(w.targets) // n_t)][:n_t]
        sample = workloads.Workload(w.name + " sample", qs, ts, w.settings)
        desc = "%d queries x %d targets (%d pairs, %d cells), evenly spaced in length order" % (
            len(qs), len(ts), len(qs) * len(ts), sample.cells)
    e, _ = engine_for(sample, device)
    out = {}
    try:
        for label, plain in (("batched", False), ("plain", True)):
            e.align(plain=plain)  # warm-up
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            info = e.align(plain=plain)
            b.record()
            torch.cuda.synchronize()
            ms = a.elapsed_time(b)
            pm = e.pair_max()
            hits, sb = e.hits()
            out[label] = {"value": sample.cells / (ms * 1e-3) / 1e9, "ms": ms, "launches": int(info.kernel_launches),
                          "hits": hits, "sb": sb, "pm": pm, "score_path": int(info.score_path)}
    finally:
        e.close()
    p, bt = out["plain"], out["batched"]
    return {"value": p["value"], "unit": "GCUPS", "sample": desc, "launches": p["launches"],
            "score_path": p["score_path"], "batched_same_sample": bt["value"],
            "batched_over_plain": bt["value"] / p["value"],
            "hits_equal": bool(np.array_equal(p["hits"], bt["hits"]) and p["sb"] == bt["sb"]),
            "pair_max_equal": bool(np.array_equal(p["pm"], bt["pm"]))}


# ------------------------------------------------------------------ CPU oracle
def _oracle_args(score, settings):
    gap, ext, affine, ll, mn = score.kernel_constants()
    return (score.matrix_array(), score.char_offset_code(), float(gap), float(ext), bool(affine), float(ll),
            float(mn), float(score.highest_score), float(settings.filter_factor), float(settings.minimum_score))


def _oracle_chunk(job):
    """The oracle's full path on queries x targets: (pair maxima, hits)."""
    args, qs, ts = job
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle
    m, off, gap, ext, affine, ll, mn, hi, ff, host_min = args
    p = oracle.OracleParams(m, off, gap, ext, affine, ll, mn)
    pos = np.array([[np.float32(hi * min(len(q), len(t)) * ff) for q in qs] for t in ts], np.float32)
    o = oracle.run(p, qs, ts, pos, host_min)
    return o["pair_max"], o["hits"]


def cpu_sample_spec(w, budget_cells):
    """A bounded sample of the workload: explicit pairs, smallest first, or
    queries x targets taken evenly from the length-sorted lists.  Returns
    (jobs as [(query strings, target strings)], index map, cells, full, text)."""
    q_all = [s.decode() for _, s in w.queries] if w.queries is not None else None
    t_all = [s.decode() for _, s in w.targets]
    if w.pairs is not None:
        order = sorted(w.pairs, key=lambda p: len(q_all[p[0]]) * len(t_all[p[1]]))
        jobs, idx, cells = [], [], 0
        for qi, ti in order:
            c = len(q_all[qi]) * len(t_all[ti])
            if cells and cells + c > budget_cells:
                break
            jobs.append(([q_all[qi]], [t_all[ti]]))
            idx.append(([qi], [ti]))
            cells += c
        return jobs, idx, cells, len(jobs) == len(w.pairs), \
            "the %d smallest explicit pairs (%d cells) of the same workload, full path" % (len(jobs), cells)
    if q_all is None:  # packed reads: the first reads only
        n = min(int(w.reads.shape[0]), 20000)
        q_all = [w.reads[i].tobytes().decode() for i in range(n)]
    nq = min(len(q_all), 10)
    q_step = max(1, len(q_all) // nq)
    q10 = sum(map(len, q_all[::q_step][:nq]))
    t_avg = sum(map(len, t_all)) / max(1, len(t_all))
    nt = min(len(t_all), max(1, int(budget_cells / (q10 * t_avg))))
    ti = list(range(0, len(t_all), max(1, len(t_all) // nt)))[:nt]
    q_avg = sum(map(len, q_all)) / max(1, len(q_all))
    nq = min(len(q_all), max(nq, int(budget_cells / (q_avg * sum(len(t_all[i]) for i in ti)))))
    qi = list(range(0, len(q_all), max(1, len(q_all) // nq)))[:nq]
    qs, ts = [q_all[i] for i in qi], [t_all[i] for i in ti]
    cells = sum(map(len, qs)) * sum(map(len, ts))
    full = len(qs) == (w.n_queries if w.queries is not None else -1) and len(ts) == len(t_all)
    return [(qs, ts)], [(qi, ti)], cells, full, \
        "%d queries x %d targets (%d cells) of the same workload, full path" % (len(qs), len(ts), cells)


def cpu_baseline(w, score, seconds, processes=1):
    """The oracle (CPU restatement of the reference path) on a bounded sample
    sized for about `seconds`: a first run at an estimated rate calibrates a
    second, larger one if the first was much shorter.  Returns (baseline
    record, sample jobs, index map, oracle results per job)."""
    import multiprocessing as mp
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle
    oracle.build()
    args = _oracle_args(score, w.settings)
    rate = 24e6 * max(1, processes)  # cells/s first estimate of the oracle
    for _ in range(3):
        jobs, idx, cells, full, text = cpu_sample_spec(w, seconds * rate)
        work = []
        for qs, ts in jobs:  # split each job's targets over the processes
            for k in range(max(1, processes)):
                if ts[k::processes]:
                    work.append((args, qs, ts[k::processes]))
        t0 = time.time()
        if processes <= 1:
            res = [_oracle_chunk(j) for j in work]
        else:
            with mp.get_context("spawn").Pool(processes) as pool:
                res = pool.map(_oracle_chunk, work)
        dt = time.time() - t0
        if dt >= 0.4 * seconds or full:
            break
        rate = cells / max(dt, 1e-3)
    rec = {"value": cells / dt / 1e9, "unit": "GCUPS", "cores": processes, "kind": "port", "sample": text,
           "seconds": dt}
    return rec, jobs, idx, (res if processes <= 1 else None)


def engine_hits(qs, ts, score, settings, device):
    """The engine on query x target strings, ids all distinct (the oracle's
    default keys): (pair maxima [nq, nt], hits as the oracle reports them)."""
    from pypaswas_b200 import _native
    from pypaswas_b200.smith_waterman import configure_engine
    e = _native.Engine(device)
    try:
        configure_engine(e, score, settings)
        e.set_queries([q.encode() for q in qs], np.arange(len(qs), dtype=np.int32))
        e.set_targets([t.encode() for t in ts], np.arange(len(ts), dtype=np.int32) + len(qs))
        e.align()
        pm = e.pair_max()
        hits, sb = e.hits()
    finally:
        e.close()
    out = []
    for h in hits:
        n, o = int(h["n_cols"]), int(h["str_offset"])
        out.append({"query": int(h["query"]), "target": int(h["target"]), "s_start": int(h["s_start"]),
                    "s_end": int(h["s_end"]), "t_start": int(h["t_start"]), "t_end": int(h["t_end"]),
                    "score": float(h["score"]), "matches": int(h["matches"]), "mismatches": int(h["mismatches"]),
                    "sequence_match": sb[o:o + n].decode("latin-1"), "alignment": sb[o + n:o + 2 * n].decode("latin-1"),
                    "target_match": sb[o + 2 * n:o + 3 * n].decode("latin-1")})
    return pm, out


def parity_leg(w, jobs, idx, oracle_res, device):
    """The engine on the CPU baseline's sample against the oracle's results
    for it: pair maxima and every hit (coordinates, score, counts, strings)."""
    from pypaswas_b200 import scores
    score = scores.make_score(w.settings)
    pairs = hits_n = 0
    pm_eq = hits_eq = True
    for (qs, ts), (qi, ti), (o_pm, o_hits) in zip(jobs, idx, oracle_res):
        pm, hits = engine_hits(qs, ts, score, w.settings, device)
        pairs += len(qs) * len(ts)
        hits_n += len(o_hits)
        pm_eq = pm_eq and bool(np.array_equal(pm, o_pm))
        hits_eq = hits_eq and hits == o_hits
    return {"sample": "the CPU baseline's sample", "pairs": pairs, "oracle_hits": hits_n,
            "pair_max_equal": pm_eq, "hits_equal": hits_eq}


# ------------------------------------------------------------------ serving
def serve_leg(device, seconds, loads, workers=2, max_batch=32, policy=1, streams=3, age_ms=25, max_residues=0):
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
        srv.tune(_native_const("PW_SERVE_TUNE_POLICY"), policy)
        srv.tune(_native_const("PW_SERVE_TUNE_AGE_MS"), age_ms)
        srv.tune(_native_const("PW_SERVE_TUNE_MAX_RESIDUES"), max_residues)
        serving.run_arrivals(srv, workloads.query_stream(seed=8, n=16, rate_hz=1e9))
        peak = serving.run_arrivals(srv, workloads.query_stream(seed=7, n=64, rate_hz=1e9))
        probe = workloads.query_stream(seed=9, n=4000, rate_hz=1.0)
        mean_cells = float(np.mean([len(q[2]) for q in probe])) * srv.db_residues
        for k, load in enumerate(loads):
            rate = load * peak["gcups"] * 1e9 / mean_cells
            reps = []
            for j in range(max(1, streams)):
                stream = workloads.query_stream(seed=60 + k + 100 * j, n=max(20, int(rate * seconds)), rate_hz=rate)
                reps.append(serving.run_arrivals(srv, stream))
            med = lambda key: float(np.median([r[key] for r in reps]))
            sweep.append({"offered_load": load, "offered_rps": med("offered_rps"), "gcups": med("gcups"),
                          "fraction_of_peak": med("gcups") / peak["gcups"], "p50_ms": med("p50_ms"),
                          "p99_ms": med("p99_ms"), "p99_ms_streams": [round(r["p99_ms"], 2) for r in reps],
                          "max_ms": max(r["max_ms"] for r in reps), "p99_top_ms": med("p99_top_ms"),
                          "p99_traceback_ms": med("p99_traceback_ms"), "p99_queue_ms": med("p99_queue_ms"),
                          "p99_run_ms": med("p99_run_ms"), "mean_run_ms": med("mean_run_ms"),
                          "requests": sum(r["requests"] for r in reps), "mean_batch": med("mean_batch"),
                          "workers_used": max(r["workers_used"] for r in reps),
                          "peak_reserved_bytes": max(r["peak_reserved_bytes"] for r in reps)})
    finally:
        srv.close()
    return {"db": "%d sequences, %d residues, resident" % (len(db), srv.db_residues),
            "workers": workers, "max_batch": max_batch, "max_residues": max_residues,
            "policy": ["arrival order", "shortest first"][policy],
            "batched_peak_gcups": peak["gcups"], "seconds_per_stream": seconds, "streams_per_load": streams,
            "sweep": sweep}


def _native_const(name):
    from pypaswas_b200 import _native
    return getattr(_native, name)


# ------------------------------------------------------------------ one config
def run_config(cfg, args, device, world, flush, sampler, headline):
    """Every leg of one configuration; returns its record."""
    from pypaswas_b200 import _native
    w = workload(cfg, args)
    e, score = engine_for(w, device)
    chain = not args.no_chain
    knobs = {"chain_min": _native.PW_TUNE_CHAIN_MIN, "grid_share": _native.PW_TUNE_GRID_SHARE,
             "segment": _native.PW_TUNE_SEGMENT, "dual": _native.PW_TUNE_DUAL, "cand_slot": _native.PW_TUNE_CAND_SLOT,
             "lanes": _native.PW_TUNE_LANES, "trace_store": _native.PW_TUNE_TRACE_STORE,
             "tile_trace": _native.PW_TUNE_TILE_TRACE, "wait_ns": _native.PW_TUNE_WAIT_NS}
    tuning = {}
    for kv in args.tune:
        key, val = kv.split("=")
        e.set_tuning(knobs[key], int(val))
        tuning[key] = int(val)
    if "chain_min" not in tuning and chain and w.pairs is None:
        from pypaswas_b200.autotune import autotune
        tuning["autotune"] = autotune(e)  # untimed: score sweeps on this workload
    replan = not args.plan_cached
    times, infos = device_steps(e, args.steps, args.warmup, replan, chain, flush, sampler if headline else None,
                                world)
    t_ms = reduce_max(float(sum(times))) if headline else float(sum(times))
    value = whole_job_gcups(w.cells, args.steps, t_ms * 1e-3, world if headline else 1)
    last = infos[-1]
    n_pairs = len(w.pairs) if w.pairs is not None else w.n_queries * len(w.targets)
    rec = {"metric": "GCUPS", "value": value, "unit": "GCUPS", "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": t_ms / args.steps,
           "step_ms": {"min": float(min(times)), "median": float(np.median(times)), "max": float(max(times)),
                       "all": [round(float(t), 3) for t in times]},
           "dtype": "int32", "data": "synthetic",
           "config": {"workload": "%s (%d pairs, full path)" % (w.name, n_pairs), "pairs": n_pairs,
                      "cells_per_step": w.cells, "traced_pairs": last["traced_pairs"],
                      "cand_overflow_pairs": last["cand_overflow_pairs"],
                      "starting_points": last["starting_points"], "hits": last["hits"],
                      "memory_waves": last["waves"],
                      "trace_store": "16-bit H per cell" if last.get("trace_store") else "4-bit cell codes",
                      "tile_form_pairs": int(last.get("tile_pairs", 0)),
                      "score_lanes": "targets" if last["orientation"] else "queries",
                      "trace_lanes": "targets" if last["trace_orientation"] else "queries",
                      "minimum_score": w.settings.minimum_score,
                      "lower_limit_score": w.settings.lower_limit_score,
                      "filter_factor": w.settings.filter_factor,
                      "l2": "flushed between steps (256 MiB write)",
                      "step": "sequences resident in HBM; the score sweep's work list "
                              + ("kept from the previous step" if not replan else "rebuilt every step")
                              + " (reuse bits seen: %d)" % int(np.bitwise_or.reduce([i["reuse"] for i in infos])),
                      "tuning": tuning},
           "phases_ms": {k: [round(float(i[k]), 2) for i in infos] for k in
                         ("score_ms", "trace_ms", "walk_ms", "setup_ms", "finish_ms", "total_ms")},
           "gpu_launches": int(sum(i["kernel_launches"] for i in infos))}
    rec["roofline"] = roofline(e, w, score, infos, args.steps)
    traffic = load_traffic().get("%s_%s" % (NAMES[cfg], "direction" if "direction" in rec["roofline"]["kernel"]
                                             else "score"))
    rec["roofline"]["traffic"] = traffic
    rec["roofline"]["hbm_gbs_measured"] = load_peaks().get("hbm_gbs")
    e.close()
    # end to end through the public API, fresh inputs every step
    if not args.no_e2e:
        if cfg == 4:
            ws = [workload(4, argparse.Namespace(**dict(vars(args), reads=E2E_READS)), seed=s) for s in (4, 14)]
        else:
            ws = [w, workload(cfg, args, seed={1: 11, 2: 12, 3: 13}[cfg])]
        if world > 1 and headline:
            import torch
            torch.distributed.barrier()
        steps_e2e = args.steps if headline else max(3, min(args.steps, 5))
        cells, dt, h2d, d2h, reuse, parts = e2e_leg(ws, steps_e2e, device, trimmer=cfg == 4)
        if headline:
            dt = reduce_max(dt)
        rec["e2e"] = {"value": whole_job_gcups(cells / steps_e2e, steps_e2e, dt, world if headline else 1),
                      "unit": "GCUPS", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                      "steps": steps_e2e, "ms_per_step": dt * 1e3 / steps_e2e,
                      "api": "FASTA text -> readers (native) -> Trimmer.trimmed_fasta -> trimmedFasta text"
                             if cfg == 4 else
                             ("Aligner.process_pairs (records, explicit pairs -> HitList)" if w.pairs is not None
                              else "Aligner.process (records -> HitList)"),
                      "host_ms_median": parts,
                      "inputs": "two seeded input sets of the same shape, alternating: every step copies and "
                                "prepares its inputs and rebuilds its plan (reuse bits seen: %d)" % reuse,
                      "workload": ws[0].name}
    return w, score, rec


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    rank, world, local = dist_env()
    import torch
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    torch.cuda.set_device(local)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # > L2 (126 MB)
    sampler = ClockSampler(local)
    sampler.start()  # started before the warm-up: nvidia-smi is up when timing begins
    try:
        w, score, out = run_config(args.config, args, local, world, flush, sampler, headline=True)
        out.update({"n_gpus": world, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                    "clocks": sampler.summary()})
        out["config"]["parallelism"] = "replica per GPU" if world > 1 else "single GPU"
        n_plain = {1: (8, 100), 2: (8, 64), 3: (16, 0), 4: (64, 48)}
        if not args.no_plain:
            out["plain"] = plain_leg(w if w.queries is not None else w.head(64), local, *n_plain[args.config])
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            rec, jobs, idx, res = cpu_baseline(w, score, args.cpu_seconds, processes=1)
            out["cpu_baseline"] = rec
            out["parity"] = parity_leg(w, jobs, idx, res, local)
        also = ([c for c in (1, 3, 4) if args.config == 2] if args.also == "auto" else
                [] if args.also == "none" else [int(c) for c in args.also.split(",") if c.strip()])
        if world == 1 and also:
            out["configs"] = {}
            for c in also:
                wc, sc, rec = run_config(c, args, local, 1, flush, sampler, headline=False)
                if not args.no_plain:
                    rec["plain"] = plain_leg(wc if wc.queries is not None else wc.head(64), local, *n_plain[c])
                if not args.no_cpu_baseline:
                    b, jobs, idx, res = cpu_baseline(wc, sc, max(5.0, args.cpu_seconds / 2), processes=1)
                    rec["cpu_baseline"] = b
                    rec["parity"] = parity_leg(wc, jobs, idx, res, local)
                out["configs"][NAMES[c]] = rec
                del wc
        if not args.no_serve and rank == 0 and world == 1 and args.config == 2:
            out["serve"] = serve_leg(local, args.serve_seconds, [float(x) for x in args.serve_loads.split(",")],
                                     workers=args.serve_workers, max_batch=args.serve_max_batch,
                                     policy=args.serve_policy, streams=args.serve_streams,
                                     max_residues=args.serve_max_residues)
    finally:
        sampler.stop()
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


# ------------------------------------------------------------------ reference arm
def run_reference(args):
    """The reference path's CPU implementation (the oracle port) over all host
    cores, each step a bounded sample of the headline workload."""
    rank, world, local = dist_env()
    if rank != 0:
        return 0
    w = workload(args.config, args)
    from pypaswas_b200 import scores
    score = scores.make_score(w.settings)
    procs = os.cpu_count() or 1
    steps = []
    # each step a bounded sample: the whole run stays near two minutes
    per_step = max(1.0, min(args.cpu_seconds, 20.0, 120.0 / max(1, args.warmup + args.steps)))
    for i in range(args.warmup + args.steps):
        rec = cpu_baseline(w, score, per_step, processes=procs)[0]
        if i >= args.warmup:
            steps.append(rec)
    v = float(np.median([s["value"] for s in steps]))
    kernels = reference_kernels(args.config, procs)
    line = {"impl": "reference", "metric": "GCUPS", "value": v, "unit": "GCUPS", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": w.name,
                       "pairs": len(w.pairs) if w.pairs is not None else w.n_queries * len(w.targets)},
            "cpu_baseline": {"value": v, "unit": "GCUPS", "cores": procs, "kind": "port",
                             "sample": steps[0]["sample"]},
            "e2e": {"value": v, "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "reference_kernels": kernels,
            "note": "value: the CPU restatement of the reference path (oracle/paswas_oracle.c) over all host cores, "
                    "the faster of the two CPU timings here; reference_kernels: the reference's own OpenCL CPU "
                    "kernels under a work-item emulation (oracle/ref), once, on a fixed sample"}
    print(json.dumps(line), flush=True)
    return 0


def reference_kernels(cfg, threads):
    """The reference's own OpenCL CPU kernels (oracle/ref/ocl_cpu_arm.py) on
    the configuration's fixed sample, when they were built; else why not."""
    sys.path.insert(0, os.path.join(REPO, "oracle", "ref"))
    try:
        import ocl_cpu_arm
    except ImportError as exc:
        return {"unavailable": str(exc)}
    if not ocl_cpu_arm.available(cfg):
        return {"unavailable": "kernels not built (built where the reference tree is present)"}
    r = ocl_cpu_arm.time_sample(cfg, threads)
    return {"value": r["value"], "unit": "GCUPS", "cores": r["threads"], "kind": "reference",
            "sample": r["sample"], "seconds": r["seconds"], "starting_points": r["starting_points"],
            "execution": "work-groups over host threads, work-items as fibers switched at barriers"}


if __name__ == "__main__":
    sys.exit(main())
