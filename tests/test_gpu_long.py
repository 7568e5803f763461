"""Long DNA pairs at the benchmark's own lengths: the two smallest pairs of the
long-DNA workload (64 pairs of 10-50 kb with a shared 2-20 kb region at 85%
identity, each query against its target and the target's reverse complement;
here 14.9 x 14.2 kb and 11.3 x 21.2 kb), through explicit pairs on the band
sweep, against the oracle pair by pair: pair maxima, every hit with its
strings, in the tile form and with stored cell codes.  The trace memory is
capped so that the traced pairs run in separate memory waves."""
import multiprocessing as mp

import numpy as np
import pytest

import cases
from engine_helpers import configure, decode_hits
from pypaswas_b200 import _native, scores, workloads

pytestmark = pytest.mark.gpu

PAIR_INDICES = (27, 53)  # the two pairs with the fewest cells (2.1e8 and 2.4e8)


def _oracle_pair(job):
    import oracle
    params, q, t, pos, minimum = job
    p = oracle.OracleParams(*params)
    o = oracle.run(p, [q], [t], pos, minimum)
    return o["pair_max"][0, 0], o["hits"]


def test_long_dna_pairs_at_full_length_bit_exact_over_memory_waves(engine_lib, oracle_mod):
    w = workloads.config3()
    score = scores.make_score(w.settings)
    n = len(w.queries)
    q = [w.queries[i][1].decode() for i in PAIR_INDICES]
    t = [w.targets[i][1].decode() for i in PAIR_INDICES] + [w.targets[i + n][1].decode() for i in PAIR_INDICES]
    pairs = [(0, 0), (0, 2), (1, 1), (1, 3)]  # forward and reverse-complement target of each query
    assert min(len(s) for s in q + t) >= 10000
    gap, ext, affine, ll, mn = score.kernel_constants()
    params = (score.matrix_array(), score.char_offset_code(), gap, ext, affine, ll, mn)
    jobs = [(params, q[a], t[b], cases.pos_scores(score, w.settings, [q[a]], [t[b]]), float(w.settings.minimum_score))
            for a, b in pairs]
    # the oracle in fresh processes (spawned: this process already uses the GPU)
    with mp.get_context("spawn").Pool(len(jobs)) as pool:
        ref = pool.map(_oracle_pair, jobs)
    traced = [k for k, (m, _) in enumerate(ref) if m >= float(w.settings.minimum_score)]
    # the tile form (checkpoints and mark bits, ~0.17 bytes a cell) and the
    # stored cell codes (~0.63 bytes a cell), one traced pair per wave each
    for tile, limit in ((0, 48 << 20), (1, 250 << 20)):
        e = _native.Engine(0, lib=engine_lib)
        try:
            configure(e, score, w.settings)
            e.set_queries([s.encode() for s in q], np.arange(len(q)))
            e.set_targets([s.encode() for s in t], np.arange(len(t)) + len(q))
            e.set_pairs([a for a, _ in pairs], [b for _, b in pairs])
            e.set_tuning(_native.PW_TUNE_TILE_TRACE, tile)
            e.set_wave_limit(limit)
            info = e.align()
            pm = e.pair_max()
            got = decode_hits(*e.hits())
        finally:
            e.close()
        assert info.score_path == 2
        assert len(traced) >= 2 and info.waves >= 2
        assert (info.tile_pairs > 0) == (tile == 0)
        by_pair = {}
        for h in got:
            by_pair.setdefault((h["query"], h["target"]), []).append(h)
        for (a, b), (m, hits) in zip(pairs, ref):
            assert pm[a, b] == m
            want = [dict(h, query=a, target=b) for h in hits]
            assert by_pair.get((a, b), []) == want
        # the planted regions are found, 2 kb or longer
        assert all(max(h["s_end"] - h["s_start"] for h in by_pair[(a, a)]) >= 1500 for a in (0, 1))
