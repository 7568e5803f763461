"""The serving loop on the GPU: continuous batching must not change results.

Each request's result -- top hits by pair maximum, or the walk's hits -- must
equal that of a lone engine run of the same query against the database, both
when the request is served alone and when it is served in a mix of requests
that arrive together, are batched together and overlap on the device
(bit-exact: same targets, scores, coordinates and alignment strings)."""
import numpy as np
import pytest

from pypaswas_b200 import _native, scores, serving, workloads
from pypaswas_b200.smith_waterman import configure_engine

pytestmark = pytest.mark.gpu

SETTINGS = dict(workloads.C5_SETTINGS, filter_factor="0.05", minimum_score="25")


def _requests(db, n, seed):
    """Query stream with a database fragment planted in every other query, so
    that traceback requests have hits."""
    rng = np.random.default_rng(seed)
    stream = workloads.query_stream(seed=seed, n=n, median=200.0, max_len=900, rate_hz=2000.0,
                                    traceback_fraction=0.5)
    out = []
    for k, (at, rid, seq, tb) in enumerate(stream):
        if k % 2 == 0:
            src = db[int(rng.integers(0, len(db)))][1]
            a = int(rng.integers(0, max(1, len(src) - 60)))
            frag = bytearray(src[a:a + 60])
            for j in range(len(frag)):
                if rng.random() < 0.2:
                    frag[j] = workloads.AMINO[int(rng.integers(0, 20))]
            p = int(rng.integers(0, len(seq) + 1))
            seq = seq[:p] + bytes(frag) + seq[p:]
        out.append((at, rid, seq, tb))
    return out


def _direct(db, settings, req, top_k=10):
    """The same request as one lone pw_align of the query against the database."""
    score = scores.make_score(settings)
    e = _native.Engine(0)
    try:
        configure_engine(e, score, settings)
        e.set_targets([s for _, s in db], np.arange(len(db), dtype=np.int32))
        e.set_queries([req[2]], np.array([-1], np.int32))
        if req[3]:
            e.align()
            hits, sb = e.hits()
            return {"hits": serving._decode_hits(hits, sb)}
        e.align(score_only=True)
        row = e.pair_max()[0]
        idx = sorted(range(len(row)), key=lambda t: (-row[t], t))[:top_k]
        return {"top": [(int(t), float(row[t])) for t in idx]}
    finally:
        e.close()


def _served(db, settings, reqs, workers, max_batch, burst, budget=0):
    st = workloads.Settings(**settings)
    srv = serving.Server(st, workers=workers, max_batch=max_batch, direction_budget=budget)
    try:
        srv.load_db(db)
        if burst:
            tickets = [srv.submit(r[2], traceback=r[3]) for r in reqs]
            res = [srv.result(t) for t in tickets]
        else:
            res = [srv.result(srv.submit(r[2], traceback=r[3])) for r in reqs]
        return res, srv.stats()
    finally:
        srv.close()


def _strip(r):
    return {k: v for k, v in r.items() if k != "info"}


def test_results_same_alone_and_in_the_mix():
    db = workloads.protein_database(seed=21, n_seqs=1500)
    st = workloads.Settings(**SETTINGS)
    reqs = _requests(db, 24, seed=22)
    direct = [_direct(db, st, r) for r in reqs]
    alone, _ = _served(db, SETTINGS, reqs, workers=1, max_batch=1, burst=False)
    mixed, stats = _served(db, SETTINGS, reqs, workers=2, max_batch=8, burst=True)
    assert [_strip(r) for r in alone] == direct
    assert [_strip(r) for r in mixed] == direct
    assert sum(len(d.get("hits", [])) for d in direct) > 0
    assert max(r["info"]["batch_queries"] for r in mixed) > 1     # requests were batched together
    assert max(r["info"]["batch_queries"] for r in alone) == 1
    assert stats["completed"] == len(reqs)


def test_direction_memory_admission_keeps_reservations_within_budget():
    db = workloads.protein_database(seed=23, n_seqs=800)
    reqs = [r[:3] + (True,) for r in _requests(db, 10, seed=24)]
    budget = 4 << 20
    st = workloads.Settings(**SETTINGS)
    res, stats = _served(db, SETTINGS, reqs, workers=3, max_batch=4, burst=True, budget=budget)
    assert stats["peak_reserved_bytes"] <= budget
    assert all(r["info"]["reserved_bytes"] <= budget for r in res)
    assert [_strip(r) for r in res] == [_direct(db, st, r) for r in reqs]


def test_residue_cap_limits_batches_and_keeps_results():
    """PW_SERVE_TUNE_MAX_RESIDUES: a burst of requests is batched only while
    the batch's query residues stay within the cap (a longer request runs
    alone); results equal lone runs."""
    db = workloads.protein_database(seed=26, n_seqs=1200)
    st = workloads.Settings(**SETTINGS)
    reqs = _requests(db, 16, seed=27)
    cap = 500
    srv = serving.Server(st, workers=1, max_batch=16)
    try:
        srv.load_db(db)
        srv.tune(_native.PW_SERVE_TUNE_MAX_RESIDUES, cap)
        tickets = [srv.submit(r[2], traceback=r[3]) for r in reqs]
        res = [srv.result(t) for t in tickets]
    finally:
        srv.close()
    assert [_strip(r) for r in res] == [_direct(db, st, r) for r in reqs]
    lens = [len(r[2]) for r in reqs]
    # a request longer than the cap always runs alone; batches of several existed
    assert all(r["info"]["batch_queries"] == 1 for r, n in zip(res, lens) if n > cap)
    assert max(r["info"]["batch_queries"] for r in res) > 1
    assert max(r["info"]["batch_queries"] for r in res) <= cap // min(lens)


def test_arrival_stream_report():
    db = workloads.protein_database(seed=25, n_seqs=2000)
    st = workloads.Settings(**SETTINGS)
    srv = serving.Server(st, workers=2, max_batch=8)
    try:
        srv.load_db(db)
        stream = workloads.query_stream(seed=26, n=60, rate_hz=300.0)
        rep = serving.run_arrivals(srv, stream)
    finally:
        srv.close()
    assert rep["requests"] == 60
    assert 0 < rep["p50_ms"] <= rep["p99_ms"] <= rep["max_ms"]
    assert rep["gcups"] > 0
