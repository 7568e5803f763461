"""The serving loop (pw_server_* in include/paswas_b200.h) from Python.

A Server keeps a protein or DNA database resident on the device and answers
single-query requests with continuous batching: requests that arrive while
other batches are on the GPU are batched together as soon as a worker (an
engine with its own CUDA stream) frees up, and batches of different workers
overlap on the device.  Two request kinds, as in the serving configuration:

* top hits (score only): the `top_k` database entries with the highest pair
  maximum (the reference's per-pair maxScore), ties broken by lower index;
* traceback: the full path -- starting points and the walk of
  SmithWaterman._print_alignments -- returning the query's hits in the order
  the reference appends them to its HitList.

Latency is measured inside the server, from submit to result.  `run_arrivals`
replays a timed arrival stream (Poisson in the benchmark) and reports p50/p99
latency beside the GCUPS the server sustained.
"""
import ctypes
import threading
import time

import numpy as np

from . import _native
from .exceptions import CudaException, HardwareException, InvalidOptionException
from .scores import make_score
from .smith_waterman import _filter_factor


class Server(object):
    def __init__(self, settings, score=None, device=0, workers=2, max_batch=16, direction_budget=0, lib=None):
        self.lib = lib if lib is not None else _native.load_library()
        self.settings = settings
        self.score = score if score is not None else make_score(settings)
        h = ctypes.c_void_p()
        rc = self.lib.pw_server_create(int(device), int(workers), int(max_batch), int(direction_budget),
                                       ctypes.byref(h))
        if rc != _native.PW_OK:
            raise HardwareException("pw_server_create failed (%d)" % rc)
        self.handle = h
        gap, ext, affine, ll, mn = self.score.kernel_constants()
        m = np.ascontiguousarray(self.score.matrix_array(), dtype=np.float32)
        self._check(self.lib.pw_server_set_scoring(self.handle, _native._ptr(m), int(m.shape[0]),
                                                   int(self.score.char_offset_code()), float(gap), float(ext),
                                                   int(bool(affine)), float(ll), float(mn),
                                                   float(settings.minimum_score), float(self.score.highest_score),
                                                   float(_filter_factor(settings))), "pw_server_set_scoring")
        self.db_ids = []
        self.db_residues = 0

    def _check(self, rc, what):
        if rc == _native.PW_OK:
            return
        msg = self.lib.pw_server_last_error(self.handle) if self.handle else b""
        msg = "%s failed (%d): %s" % (what, rc, (msg or b"").decode())
        if rc == _native.PW_ERR_ARG:
            raise InvalidOptionException(msg)
        if rc == _native.PW_ERR_DEVICE:
            raise HardwareException(msg)
        raise CudaException(msg)

    def load_db(self, records):
        """records: [(id, upper-case byte string)]; resident until close()."""
        seqs = [s for _, s in records]
        buf, off = _native.pack_sequences(seqs)
        keys = np.arange(len(seqs), dtype=np.int32)
        self._check(self.lib.pw_server_load_db(self.handle, _native._ptr(buf), _native._ptr(off), len(seqs),
                                               _native._ptr(keys)), "pw_server_load_db")
        self.db_ids = [i for i, _ in records]
        self.db_residues = int(off[-1])

    def submit(self, seq, traceback=False, top_k=10):
        """Queues one query (bytes); returns its ticket at once."""
        a = np.frombuffer(seq, dtype=np.uint8)
        t = ctypes.c_int64()
        mode = _native.PW_SERVE_TRACEBACK if traceback else _native.PW_SERVE_TOP
        self._check(self.lib.pw_server_submit(self.handle, _native._ptr(a), len(a), mode, int(top_k),
                                              ctypes.byref(t)), "pw_server_submit")
        return t.value

    def wait(self, ticket, timeout_ms=-1):
        """Blocks until the request is done; returns its pw_request_info as a dict."""
        info = _native.PwRequestInfo()
        rc = self.lib.pw_server_wait(self.handle, int(ticket), int(timeout_ms), ctypes.byref(info))
        self._check(rc, "pw_server_wait")
        return info.as_dict()

    def result(self, ticket, release=True):
        """Waits and returns {"info", "top": [(db index, score)]} or {"info", "hits": [...]}."""
        info = self.wait(ticket)
        out = {"info": info}
        n = int(info["n_hits"])
        if info["mode"] == _native.PW_SERVE_TOP:
            tg = np.zeros(max(n, 1), np.int32)
            sc = np.zeros(max(n, 1), np.float32)
            self._check(self.lib.pw_server_top_hits(self.handle, int(ticket), _native._ptr(tg), _native._ptr(sc),
                                                    n), "pw_server_top_hits")
            out["top"] = [(int(tg[j]), float(sc[j])) for j in range(n)]
        else:
            hits = np.zeros(max(n, 1), dtype=_native.HIT_DTYPE)
            nb = int(info["string_bytes"])
            sb = np.zeros(max(nb, 1), np.uint8)
            self._check(self.lib.pw_server_hits(self.handle, int(ticket), _native._ptr(hits), n, _native._ptr(sb),
                                                nb), "pw_server_hits")
            out["hits"] = _decode_hits(hits[:n], sb[:nb].tobytes())
        if release:
            self._check(self.lib.pw_server_release(self.handle, int(ticket)), "pw_server_release")
        return out

    def tune(self, key, value):
        """pw_set_tuning on every worker engine (e.g. _native.PW_TUNE_GRID_SHARE)."""
        self._check(self.lib.pw_server_tune(self.handle, int(key), int(value)), "pw_server_tune")

    def stats(self):
        st = _native.PwServerStats()
        self._check(self.lib.pw_server_stats(self.handle, ctypes.byref(st)), "pw_server_stats")
        return st.as_dict()

    def close(self):
        if getattr(self, "handle", None):
            self.lib.pw_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _decode_hits(hits, sb):
    out = []
    for h in hits:
        n, o = int(h["n_cols"]), int(h["str_offset"])
        out.append({"target": int(h["target"]), "s_start": int(h["s_start"]), "s_end": int(h["s_end"]),
                    "t_start": int(h["t_start"]), "t_end": int(h["t_end"]), "score": float(h["score"]),
                    "matches": int(h["matches"]), "mismatches": int(h["mismatches"]),
                    "sequence_match": sb[o:o + n].decode("latin-1"),
                    "alignment": sb[o + n:o + 2 * n].decode("latin-1"),
                    "target_match": sb[o + 2 * n:o + 3 * n].decode("latin-1")})
    return out


def percentile(values, q):
    """Nearest-rank percentile (q in 0..100) of a non-empty sequence."""
    v = sorted(values)
    k = max(0, min(len(v) - 1, int(np.ceil(q / 100.0 * len(v))) - 1))
    return float(v[k])


def run_arrivals(server, stream, keep_results=False):
    """Submits each (arrival_s, id, sequence, traceback) of `stream` at its
    arrival time (relative to the start) and collects every result.

    Returns a report: latency p50/p99 (all, top-hits, traceback), GCUPS over
    the window from the first submit to the last result, offered and served
    request rates, mean batch size."""
    tickets = [None] * len(stream)
    t0 = time.perf_counter()

    def feeder():
        for k, (at, _, seq, tb) in enumerate(stream):
            d = at - (time.perf_counter() - t0)
            if d > 0:
                time.sleep(d)
            tickets[k] = server.submit(seq, traceback=tb)

    th = threading.Thread(target=feeder)
    th.start()
    infos, results = [], []
    for k in range(len(stream)):
        while tickets[k] is None:
            time.sleep(0.0005)
        r = server.result(tickets[k])
        infos.append(r["info"])
        if keep_results:
            results.append(r)
    th.join()
    wall = time.perf_counter() - t0
    lat = [i["latency_ms"] for i in infos]
    lat_top = [i["latency_ms"] for i in infos if i["mode"] == _native.PW_SERVE_TOP]
    lat_tb = [i["latency_ms"] for i in infos if i["mode"] == _native.PW_SERVE_TRACEBACK]
    cells = sum(i["cells"] for i in infos)
    span = stream[-1][0] if stream else 0.0
    rep = {"requests": len(stream), "wall_s": wall, "cells": cells, "gcups": cells / wall / 1e9,
           "p50_ms": percentile(lat, 50), "p99_ms": percentile(lat, 99), "max_ms": max(lat),
           "p50_top_ms": percentile(lat_top, 50) if lat_top else None,
           "p99_top_ms": percentile(lat_top, 99) if lat_top else None,
           "p50_traceback_ms": percentile(lat_tb, 50) if lat_tb else None,
           "p99_traceback_ms": percentile(lat_tb, 99) if lat_tb else None,
           "offered_rps": len(stream) / span if span > 0 else None, "served_rps": len(stream) / wall,
           "mean_batch": float(np.mean([i["batch_queries"] for i in infos])),
           "p99_queue_ms": percentile([i["queue_ms"] for i in infos], 99),
           "p99_run_ms": percentile([i["run_ms"] for i in infos], 99),
           "mean_run_ms": float(np.mean([i["run_ms"] for i in infos])),
           "workers_used": len(set(i["worker"] for i in infos)),
           "peak_reserved_bytes": server.stats()["peak_reserved_bytes"]}
    if keep_results:
        rep["results"] = results
    return rep
