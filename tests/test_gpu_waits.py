"""Bounded device waits run out without faulting the GPU.

Chained strips and bands wait for their predecessor's progress flag with a
bounded wait (PW_TUNE_WAIT_NS).  PW_TUNE_STALL_TEST makes the next chained
launch re-point one queue entry at a flag that nothing ever sets, so its wait
must run out: the warp gives up, raises the launch's abort flag, every other
waiting warp gives up too, and pw_align returns PW_ERR_KERNEL with a message
(mapped to CudaException, as the reference maps its kernel failures,
SmithWaterman.py:609-613).  The engine stays usable: the next pw_align on the
same engine is bit-exact against the oracle."""
import numpy as np
import pytest

import cases
from engine_helpers import configure, decode_hits
from pypaswas_b200 import _native, scores
from pypaswas_b200.exceptions import CudaException

pytestmark = pytest.mark.gpu


def _long_protein_case(seed, n_q=320, n_t=6, t_len=(400, 600)):
    """Enough queries that the inter-sequence score sweep runs (not the band
    sweep of a few long sequences), targets of 13-19 strips."""
    rng = np.random.default_rng(seed)
    draw = lambda n: "".join(cases.PROTEIN[i] for i in rng.integers(0, 20, n))
    targets = [draw(int(rng.integers(*t_len))) for _ in range(n_t)]
    queries = []
    for _ in range(n_q):
        s = draw(int(rng.integers(40, 150)))
        tt = targets[int(rng.integers(0, n_t))]
        cut = int(rng.integers(0, len(tt) - 80))
        p = int(rng.integers(0, len(s) + 1))
        queries.append(s[:p] + cases.mutate(rng, tt[cut:cut + 80], cases.PROTEIN, 0.2, 1) + s[p:])
    st = cases.Settings(matrix_name="BLOSUM62", gap_score="-11", gap_extension="-1", minimum_score="40")
    return queries, targets, scores.make_score(st), st


def _oracle(oracle_mod, q, t, score, st):
    return oracle_mod.run(cases.oracle_params(oracle_mod, score), q, t, cases.pos_scores(score, st, q, t),
                          float(st.minimum_score))


def _engine(lib, q, t, score, st):
    e = _native.Engine(0, lib=lib)
    configure(e, score, st)
    e.set_queries([s.encode() for s in q], np.arange(len(q)))
    e.set_targets([s.encode() for s in t], np.arange(len(t)) + len(q))
    return e


def test_chained_score_sweep_wait_runs_out_and_engine_recovers(engine_lib, oracle_mod):
    q, t, score, st = _long_protein_case(5)
    o = _oracle(oracle_mod, q, t, score, st)
    e = _engine(engine_lib, q, t, score, st)
    try:
        e.set_tuning(_native.PW_TUNE_CHAIN_MIN, 1)  # chain every multi-strip item
        first = e.align()
        assert first.score_path == 0 and first.score_launches > 0
        e.set_tuning(_native.PW_TUNE_WAIT_NS, 5_000_000)  # 5 ms
        e.set_tuning(_native.PW_TUNE_STALL_TEST, 1)
        with pytest.raises(CudaException, match="waited too long"):
            e.align()
        e.set_tuning(_native.PW_TUNE_WAIT_NS, 0)
        e.align()
        np.testing.assert_array_equal(e.pair_max(), o["pair_max"])
        assert decode_hits(*e.hits()) == o["hits"]
    finally:
        e.close()


def test_band_sweep_wait_runs_out_and_engine_recovers(engine_lib, oracle_mod):
    # explicit pairs with targets over 256 rows: bands chained across warps
    rng = np.random.default_rng(8)
    motif = "".join(cases.DNA[i] for i in rng.integers(0, 4, 400))
    q = ["".join(cases.DNA[i] for i in rng.integers(0, 4, 300)) + cases.mutate(rng, motif, cases.DNA, 0.05, 2)
         for _ in range(3)]
    t = [motif + "".join(cases.DNA[i] for i in rng.integers(0, 4, 700)) for _ in range(2)]
    st = cases.Settings(minimum_score="30")
    score = scores.make_score(st)
    pairs = [(0, 0), (1, 1), (2, 0)]
    e = _engine(engine_lib, q, t, score, st)
    try:
        e.set_pairs([a for a, _ in pairs], [b for _, b in pairs])
        e.set_tuning(_native.PW_TUNE_WAIT_NS, 5_000_000)
        e.set_tuning(_native.PW_TUNE_STALL_TEST, 1)
        with pytest.raises(CudaException, match="waited too long"):
            e.align()
        e.set_tuning(_native.PW_TUNE_WAIT_NS, 0)
        info = e.align()
        assert info.score_path == 2
        got = decode_hits(*e.hits())
        pm = e.pair_max()
    finally:
        e.close()
    for a, b in pairs:
        o = _oracle(oracle_mod, [q[a]], [t[b]], score, st)
        assert pm[a, b] == o["pair_max"][0, 0]
        assert [h for h in got if (h["query"], h["target"]) == (a, b)] == \
            [dict(h, query=a, target=b) for h in o["hits"]]
