"""The two forms of the linear direction sweep give the same hits.

With linear integer scoring whose traced maxima stay below 2^15 the engine
stores every traced cell's 16-bit H and derives the direction codes on read
(pw_run_info.trace_store = 1); PW_TUNE_TRACE_STORE = 1 keeps the 4-bit cell
codes.  Both forms, on the strip sweep (both lane orientations), the one-warp
band sweep, explicit long pairs and several memory waves, must give the
oracle's hits bit for bit; affine scoring and maxima of 2^15 or more keep the
codes."""
import numpy as np
import pytest

import cases
from engine_helpers import run_engine
from pypaswas_b200 import _native

pytestmark = pytest.mark.gpu

CODES = {_native.PW_TUNE_TRACE_STORE: 1}


def _oracle(oracle_mod, queries, targets, score, settings):
    p = cases.oracle_params(oracle_mod, score)
    pos = cases.pos_scores(score, settings, queries, targets)
    return oracle_mod.run(p, queries, targets, pos, float(settings.minimum_score), None, None)


def _linear(seed, **kw):
    rng = np.random.default_rng(seed)
    while True:
        q, t, score, st = cases.make_case(int(rng.integers(0, 1 << 30)), "dna", **kw)
        if st.gap_extension == "0":
            return q, t, score, st


def _both_forms(engine_lib, oracle_mod, queries, targets, score, st, want_store, **align_kw):
    o = _oracle(oracle_mod, queries, targets, score, st)
    pm_h, hits_h, info_h, _ = run_engine(engine_lib, queries, targets, score, st, **align_kw)
    pm_c, hits_c, info_c, _ = run_engine(engine_lib, queries, targets, score, st, tuning=CODES, **align_kw)
    if info_h.traced_pairs:
        assert info_h.trace_store == want_store
    assert info_c.trace_store == 0
    np.testing.assert_array_equal(pm_h, o["pair_max"])
    np.testing.assert_array_equal(pm_c, o["pair_max"])
    assert hits_h == o["hits"]
    assert hits_c == o["hits"]
    return info_h


@pytest.mark.parametrize("seed", range(8))
def test_random_cases_forms_agree(engine_lib, oracle_mod, seed):
    """Small random cases (their few traced pairs go to the band sweep, which
    keeps the codes): the engine's choice and the codes agree."""
    queries, targets, score, st = _linear(300 + seed)
    _both_forms(engine_lib, oracle_mod, queries, targets, score, st, 0)


@pytest.mark.parametrize("shape", [(600, 40), (40, 600)])
def test_both_lane_orientations(engine_lib, oracle_mod, shape):
    """Many short queries against few targets and the reverse: the direction
    sweep runs with targets or with queries as strips."""
    rng = np.random.default_rng(sum(shape))
    nq, nt = shape
    motif = "".join(rng.choice(list("ACGT"), size=30))
    queries = ["".join(rng.choice(list("ACGT"), size=int(rng.integers(10, 60)))) + motif[: int(rng.integers(8, 30))]
               for _ in range(nq)]
    targets = [motif[int(rng.integers(0, 10)):] + "".join(rng.choice(list("ACGT"), size=int(rng.integers(1, 40))))
               for _ in range(nt)]
    st = cases.Settings(minimum_score="6", lower_limit_score="0.5")
    score = cases.scores.make_score(st)
    _both_forms(engine_lib, oracle_mod, queries, targets, score, st, 1)


def test_band_sweep_forms_agree(engine_lib, oracle_mod):
    """Targets longer than one register strip: one pair per warp, 256-row
    bands chained across warps.  Alone they keep the codes (their long walks
    read one code a step); next to a majority of strip-sweep cells they store
    H as well, in the band layout."""
    rng = np.random.default_rng(41)
    motif = "".join(rng.choice(list("ACGT"), size=700))
    queries = [cases.mutate(rng, motif[k * 50:k * 50 + 400], "ACGT", 0.1, 3) for k in range(5)]
    targets = [motif, "".join(rng.choice(list("ACGT"), size=900))]
    st = cases.Settings(minimum_score="20", lower_limit_score="0.9")
    score = cases.scores.make_score(st)
    _both_forms(engine_lib, oracle_mod, queries, targets, score, st, 0)
    # the H store forced on the band sweep (PW_TUNE_TRACE_STORE = 2)
    o = _oracle(oracle_mod, queries, targets, score, st)
    pm, hits, info, _ = run_engine(engine_lib, queries, targets, score, st,
                                   tuning={_native.PW_TUNE_TRACE_STORE: 2})
    assert info.trace_store == 1 and info.warp_pairs == info.traced_pairs
    np.testing.assert_array_equal(pm, o["pair_max"])
    assert hits == o["hits"]
    # 600 reads against 10 short adapters (strip sweep, > 32 traced pairs per
    # SM) and one target of two bands (band sweep, fewer cells), all pairs
    # traced
    ad = ["".join(rng.choice(list("ACGT"), size=int(rng.integers(24, 40)))) for _ in range(10)]
    queries = ["".join(rng.choice(list("ACGT"), size=int(rng.integers(20, 50)))) + ad[i % 10][:20]
               for i in range(600)]
    targets = ad + ["".join(rng.choice(list("ACGT"), size=250)) + ad[0]]
    st = cases.Settings(minimum_score="1", lower_limit_score="0.5", filter_factor="0.0")
    score = cases.scores.make_score(st)
    info = _both_forms(engine_lib, oracle_mod, queries, targets, score, st, 1)
    assert 0 < info.warp_pairs < info.traced_pairs


def test_memory_waves_forms_agree(engine_lib, oracle_mod):
    """The same hits when the cells of one call are split into waves."""
    seed = 77
    while True:  # a case with several hits
        queries, targets, score, st = _linear(seed, max_queries=40, max_tlen=260)
        o = _oracle(oracle_mod, queries, targets, score, st)
        if len(o["hits"]) >= 4:
            break
        seed += 1
    from engine_helpers import configure, decode_hits
    # long pairs in the tile form (a few KB each) and with stored codes
    for tile, limit in ((0, 8 << 10), (1, 64 << 10)):
        e = _native.Engine(0, lib=engine_lib)
        try:
            configure(e, score, st)
            e.set_queries([q.encode() for q in queries], np.arange(len(queries)))
            e.set_targets([t.encode() for t in targets], np.arange(len(targets)) + len(queries))
            e.set_tuning(_native.PW_TUNE_TILE_TRACE, tile)
            e.set_wave_limit(limit)
            info = e.align()
            assert info.waves > 1
            assert decode_hits(*e.hits()) == o["hits"]
        finally:
            e.close()


def test_affine_and_large_maxima_keep_codes(engine_lib, oracle_mod):
    rng = np.random.default_rng(5)
    while True:
        queries, targets, score, st = cases.make_case(int(rng.integers(0, 1 << 30)), "dna")
        if st.gap_extension != "0":
            break
    info = _both_forms(engine_lib, oracle_mod, queries, targets, score, st, 0)
    assert info.trace_store == 0
    # scores of 100 a match: maxima above 2^15 on 400-nt identical segments
    seg = "".join(rng.choice(list("ACGT"), size=400))
    queries = [seg, seg[:380] + "A" * 20]
    targets = [seg]
    st = cases.Settings(match_score="100", mismatch_score="-300", gap_score="-500", minimum_score="10")
    score = cases.scores.make_score(st)
    info = _both_forms(engine_lib, oracle_mod, queries, targets, score, st, 0)
    assert info.trace_store == 0
