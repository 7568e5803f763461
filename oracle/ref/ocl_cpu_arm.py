"""The reference's own CPU path as a timed baseline: pyPaSWAS's OpenCL CPU
kernels (pyPaSWAS/Core/ocl/default_main_cpu.cl, template-expanded by its own
PaSWAS.CPUcode) compiled as host C++ by build_ref.py, driven by the reference
host driver's launch loops (SmithWaterman._calculate_score / _traceback_host,
SmithWaterman.py:591-655, with SmithWatermanCPU's launch shapes,
SmithWatermanOcl.py:459-511) and its buffer set-up (SmithWatermanCPU.
_init_normal_memory, SmithWatermanOcl.py:360-411), work-groups spread over all
host cores.

TEST INFRASTRUCTURE / BASELINE ONLY: bench.py's reference arm times it; the
engine never uses it.

The kernels are template constants of their batch shape (N_SEQUENCES,
N_TARGETS, X, Y), so each batch of a fixed sample of every benchmark
configuration is compiled here, where the reference tree is present
(`python oracle/ref/ocl_cpu_arm.py --build`, run by __graft_entry__.build());
the shapes and library names go to oracle/_ref/ocl_cpu_manifest.json, which
travels with the libraries.  Timing needs neither the reference tree nor the
template code.

Batches follow the reference's own batching: queries and targets sorted by
length (longest first), queries padded to a multiple of 8 with '\\0' up to the
longest query of the batch, targets in blocks, each padded to its longest
(SWSeq.extentToFillGPU, SmithWaterman.set_targets).  Cells are counted
unpadded, as the reference's GCUPS formula does (SmithWaterman.py:546-547).
What is timed per batch: the buffer set-up, the score sweep and the traceback
kernel launches; the reference's Python host walk is not (it would only slow
the baseline down).  Affine gaps follow the OpenCL CPU kernels' own semantics
(the gap opens with gapScore, not gapScore + gapExtension as in the CUDA
kernels), so affine scores may differ from the CUDA path; the work is the same.
"""
import ctypes
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
OUT_DIR = os.path.join(os.path.dirname(HERE), "_ref")
MANIFEST = os.path.join(OUT_DIR, "ocl_cpu_manifest.json")
if REPO not in sys.path:
    sys.path.insert(0, REPO)

SHARED = 8          # SHARED_X = SHARED_Y of the CPU device (SmithWatermanOcl)
WORKGROUP = 2       # SHARED / WORKLOAD (4)


def _pad8(n):
    return max(8, (n + 7) // 8 * 8)


def sample_batches(cfg):
    """The fixed sample of configuration `cfg` as the reference would batch
    it: [(query strings, target strings)] plus the workload's settings dict
    and a description."""
    from pypaswas_b200 import workloads as W
    if cfg == 3:
        w = W.config3()
        n = len(w.queries)
        sizes = sorted(range(n), key=lambda i: len(w.queries[i][1]) * len(w.targets[i][1]))
        i = sizes[0]
        q = [w.queries[i][1].decode()]
        t = sorted([w.targets[i][1].decode(), w.targets[i + n][1].decode()], key=len, reverse=True)
        return [(q, t)], dict(W.C3_SETTINGS), "the smallest long pair against its target and the target's RC"
    if cfg == 4:
        w = W.config4(n_reads=96)
        q = [w.reads[i].tobytes().decode() for i in range(96)]
        t = sorted([s.decode() for _, s in w.targets], key=len, reverse=True)
        return [(q, t)], dict(W.C4_SETTINGS), "96 reads x the 48 adapters (+RC)"
    if cfg == 1:
        w, nq, nt, block, settings = W.config1(), 24, None, 50, W.C1_SETTINGS
    else:
        w, nq, nt, block, settings = W.config2(), 4, 64, 16, W.C2_SETTINGS
    qs = sorted([s.decode() for _, s in w.queries], key=len, reverse=True)
    ts = sorted([s.decode() for _, s in w.targets], key=len, reverse=True)
    qs = qs[::max(1, len(qs) // nq)][:nq]
    if nt:
        ts = ts[::max(1, len(ts) // nt)][:nt]
    batches = [(qs, ts[k:k + block]) for k in range(0, len(ts), block)]
    desc = "%d queries x %d targets (evenly spaced in length order), target blocks of %d" % (len(qs), len(ts), block)
    return batches, dict(settings), desc


def _cells(batches):
    return sum(len(q) * len(t) for qs, ts in batches for q in qs for t in ts)


def build_all(configs=(1, 2, 3, 4)):
    """Compiles the kernels of every batch shape (here, with the reference
    tree) and writes the manifest."""
    sys.path.insert(0, HERE)
    import logging
    import build_ref
    import ref_driver as R
    from concurrent.futures import ThreadPoolExecutor
    manifest = {}
    jobs = []
    for cfg in configs:
        batches, settings, desc = sample_batches(cfg)
        st = R.Settings(**settings)
        score = R.make_score(st, logging.getLogger("ocl_cpu_arm"))
        entry = {"sample": desc, "cells": _cells(batches), "affine": score.gap_extension is not None,
                 "highest": float(score.highest_score), "filter_factor": float(st.filter_factor), "batches": []}
        for qs, ts in batches:
            X, Y = _pad8(max(map(len, qs))), _pad8(max(map(len, ts)))
            b = {"nq": len(qs), "nt": len(ts), "X": X, "Y": Y, "so": None}
            entry["batches"].append(b)
            jobs.append((b, score, len(qs), len(ts), X, Y))
        manifest[str(cfg)] = entry
    with ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as pool:
        paths = list(pool.map(lambda j: build_ref.build(j[1], j[2], j[3], j[4], j[5], "ocl_cpu"), jobs))
    for (b, *_), path in zip(jobs, paths):
        b["so"] = os.path.basename(path)
    os.makedirs(OUT_DIR, exist_ok=True)
    with open(MANIFEST + ".tmp", "w") as f:
        json.dump(manifest, f, indent=1)
    os.replace(MANIFEST + ".tmp", MANIFEST)
    return manifest


def available(cfg):
    """Whether the kernels of configuration `cfg` were built."""
    try:
        with open(MANIFEST) as f:
            entry = json.load(f).get(str(cfg))
    except (OSError, ValueError):
        return False
    return entry is not None and all(os.path.exists(os.path.join(OUT_DIR, b["so"])) for b in entry["batches"])


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


def run_batch(lib, qs, ts, X, Y, affine, highest, filter_factor, nthreads):
    """One batch through the reference's CPU kernels; returns (pair maxima
    [nq, nt], number of starting points)."""
    nq, nt = len(qs), len(ts)
    seq = np.zeros(nq * X, dtype=np.uint8)
    for i, q in enumerate(qs):
        seq[i * X:i * X + len(q)] = np.frombuffer(q.upper().encode(), dtype=np.uint8)
    tgt = np.zeros(nt * Y, dtype=np.uint8)
    for i, t in enumerate(ts):
        tgt[i * Y:i * Y + len(t)] = np.frombuffer(t.upper().encode(), dtype=np.uint8)
    cells = nq * nt * (X + 1) * (Y + 1)
    m = np.zeros(cells, dtype=np.float32)
    mi = np.full(cells if affine else 1, -1e10, dtype=np.float32)
    mj = np.full(cells if affine else 1, -1e10, dtype=np.float32)
    xd, yd = X // SHARED, Y // SHARED
    gmax = np.zeros(nq * nt * xd * yd * WORKGROUP * WORKGROUP, dtype=np.float32)
    gdir = np.zeros(nq * nt * X * Y, dtype=np.uint8)
    inc = np.zeros(1, dtype=np.uint32)
    sp = np.zeros(36 * nq * nt * 1000, dtype=np.uint8)
    mps = np.array([np.float32(highest * min(len(q), len(t)) * filter_factor) for t in ts for q in qs],
                   dtype=np.float32)
    sem = np.zeros(nq * nt * X * Y, dtype=np.int32)
    lib.emu_run_cpu_path(_p(m), _p(mi), _p(mj), _p(seq), _p(tgt), _p(gmax), _p(gdir), _p(inc), _p(sp), _p(mps),
                         _p(sem), ctypes.c_int(int(affine)), ctypes.c_int(int(nthreads)))
    pm = gmax.reshape(nq, nt, xd, yd, WORKGROUP, WORKGROUP)[:, :, -1, -1, -1, -1].copy()
    return pm, int(inc[0])


_libs = {}


def _lib(name):
    if name not in _libs:
        lib = ctypes.CDLL(os.path.join(OUT_DIR, name))
        lib.emu_run_cpu_path.restype = None
        _libs[name] = lib
    return _libs[name]


def time_sample(cfg, nthreads=None):
    """Runs configuration `cfg`'s sample once; returns {value GCUPS, seconds,
    cells, sample, starting_points}."""
    with open(MANIFEST) as f:
        entry = json.load(f)[str(cfg)]
    batches, _, _ = sample_batches(cfg)
    nthreads = nthreads or os.cpu_count() or 1
    t0 = time.time()
    starts = 0
    for (qs, ts), b in zip(batches, entry["batches"]):
        _, n = run_batch(_lib(b["so"]), qs, ts, b["X"], b["Y"], entry["affine"], entry["highest"],
                         entry["filter_factor"], nthreads)
        starts += n
    dt = time.time() - t0
    return {"value": entry["cells"] / dt / 1e9, "seconds": dt, "cells": entry["cells"], "sample": entry["sample"],
            "starting_points": starts, "threads": nthreads}


if __name__ == "__main__":
    if "--build" in sys.argv:
        m = build_all()
        print(json.dumps({k: (v["sample"], len(v["batches"])) for k, v in m.items()}))
    for c in (1, 2, 3, 4):
        if "--time" in sys.argv and available(c):
            print(c, time_sample(c))
