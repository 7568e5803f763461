"""The tile form of the long-pair traceback against the stored cell codes and
the oracle.

Long pairs of linear integer scoring take the tile form by default
(pw_run_info.tile_pairs > 0): a checkpoint sweep keeps band rows and tile
columns of H, and collect, walk and the column operations recompute
256 x 128-cell tiles of codes where they need them.  PW_TUNE_TILE_TRACE = 1
keeps the band direction sweep's stored codes.  Both must give the oracle's
maxima, starting points and hits bit for bit: many tiles and bands, many
candidates and walks that stop on one another's cells, candidate slots that
overflow, memory waves, the starting-point cap, same-id pairs, and strip
pairs in the same wave."""
import numpy as np
import pytest

import cases
from engine_helpers import configure, decode_hits, run_engine
from pypaswas_b200 import _native, scores

pytestmark = pytest.mark.gpu

CODES = {_native.PW_TUNE_TILE_TRACE: 1}


def _oracle(oracle_mod, queries, targets, score, settings, q_keys=None, t_keys=None):
    p = cases.oracle_params(oracle_mod, score)
    pos = cases.pos_scores(score, settings, queries, targets)
    return oracle_mod.run(p, queries, targets, pos, float(settings.minimum_score), q_keys, t_keys)


def _long_case(seed, n_pairs=6, alphabet="ACGT", rate=0.1):
    """Queries and targets of 300-2,000 residues sharing mutated segments
    (several per pair, so that walks meet), plus unrelated ones."""
    rng = np.random.default_rng(seed)
    draw = lambda n: "".join(alphabet[i] for i in rng.integers(0, len(alphabet), n))
    queries, targets = [], []
    for _ in range(n_pairs):
        lq, lt = int(rng.integers(300, 2000)), int(rng.integers(300, 2000))
        q, t = draw(lq), draw(lt)
        for _ in range(int(rng.integers(1, 4))):
            n = int(rng.integers(40, min(lq, lt) // 2))
            a, b = int(rng.integers(0, lq - n)), int(rng.integers(0, lt - n))
            seg = cases.mutate(rng, q[a:a + n], alphabet, rate, 2)
            t = t[:b] + seg + t[b + len(seg):]
            t = t[:lt]
        queries.append(q)
        targets.append(t)
    return queries, targets


def _both(engine_lib, oracle_mod, queries, targets, st, q_keys=None, t_keys=None, **kw):
    score = scores.make_score(st)
    o = _oracle(oracle_mod, queries, targets, score, st, q_keys, t_keys)
    pm_t, hits_t, info_t, _ = run_engine(engine_lib, queries, targets, score, st, q_keys, t_keys, **kw)
    tuning = dict(kw.pop("tuning", None) or {})
    tuning.update(CODES)
    pm_c, hits_c, info_c, _ = run_engine(engine_lib, queries, targets, score, st, q_keys, t_keys, tuning=tuning,
                                         **kw)
    assert info_t.tile_pairs > 0 and info_t.tile_pairs == info_t.warp_pairs
    assert info_c.tile_pairs == 0
    np.testing.assert_array_equal(pm_t, o["pair_max"])
    np.testing.assert_array_equal(pm_c, o["pair_max"])
    assert hits_c == o["hits"]
    assert hits_t == o["hits"]
    return o, info_t


@pytest.mark.parametrize("seed", range(4))
def test_tile_form_matches_codes_and_oracle(engine_lib, oracle_mod, seed):
    queries, targets = _long_case(500 + seed)
    st = cases.Settings(minimum_score="15", lower_limit_score="0.4", filter_factor="0.05")
    o, info = _both(engine_lib, oracle_mod, queries, targets, st)
    assert len(o["hits"]) >= 3


def test_tile_form_many_candidates_and_slot_overflow(engine_lib, oracle_mod):
    """Low thresholds: hundreds of candidates a pair, covering chains across
    tiles, walks that end on earlier walks' cells; slots of 4 candidates
    overflow and the checkpoint sweep runs again."""
    queries, targets = _long_case(77, n_pairs=4, rate=0.05)
    st = cases.Settings(minimum_score="8", lower_limit_score="0.1", filter_factor="0.01")
    o, info = _both(engine_lib, oracle_mod, queries, targets, st)
    assert len(o["hits"]) >= 20
    o, info = _both(engine_lib, oracle_mod, queries, targets, st, tuning={_native.PW_TUNE_CAND_SLOT: 4})
    assert info.cand_overflow_pairs > 0


def test_tile_form_waves_cap_and_same_ids(engine_lib, oracle_mod):
    queries, targets = _long_case(91, n_pairs=5)
    st = cases.Settings(minimum_score="12", lower_limit_score="0.3", filter_factor="0.05")
    score = scores.make_score(st)
    # several memory waves
    o = _oracle(oracle_mod, queries, targets, score, st)
    e = _native.Engine(0, lib=engine_lib)
    try:
        configure(e, score, st)
        e.set_queries([q.encode() for q in queries], np.arange(len(queries)))
        e.set_targets([t.encode() for t in targets], np.arange(len(targets)) + len(queries))
        e.set_wave_limit(256 << 10)
        info = e.align()
        assert info.waves > 1 and info.tile_pairs > 0
        assert decode_hits(*e.hits()) == o["hits"]
        # the starting-point cap (one wave): the first starts in emission order are walked
        e.set_wave_limit(0)
        cap = max(1, int(info.starting_points) // 3)
        o_cap = oracle_mod.run(cases.oracle_params(oracle_mod, score), queries, targets,
                               cases.pos_scores(score, st, queries, targets), float(st.minimum_score),
                               start_cap=cap)
        info = e.align(start_cap=cap)
        assert info.truncated
        assert decode_hits(*e.hits()) == o_cap["hits"]
    finally:
        e.close()
    # same ids: those pairs are walked by nobody
    keys = np.arange(len(queries))
    _both(engine_lib, oracle_mod, queries, targets, st, q_keys=keys, t_keys=keys.copy())


def test_tile_form_next_to_strip_pairs(engine_lib, oracle_mod):
    """Short targets (strip sweep, H store) and long ones (tile form) traced in
    the same wave."""
    rng = np.random.default_rng(13)
    queries, targets = _long_case(13, n_pairs=2)
    # 2,600 reads against 10 short adapters: enough traced pairs per SM for the strip sweep
    ad = ["".join(rng.choice(list("ACGT"), size=int(rng.integers(24, 40)))) for _ in range(10)]
    queries += ["".join(rng.choice(list("ACGT"), size=int(rng.integers(20, 50)))) + ad[i % 10][:20]
                for i in range(2600)]
    targets += ad
    st = cases.Settings(minimum_score="6", lower_limit_score="0.5", filter_factor="0.05")
    o, info = _both(engine_lib, oracle_mod, queries, targets, st)
    assert 0 < info.warp_pairs < info.traced_pairs


def _pairs_run(engine_lib, queries, targets, pairs, st, tuning=None):
    score = scores.make_score(st)
    e = _native.Engine(0, lib=engine_lib)
    try:
        configure(e, score, st)
        e.set_queries([q.encode() for q in queries], np.arange(len(queries)))
        e.set_targets([t.encode() for t in targets], np.arange(len(targets)) + len(queries))
        for k, v in (tuning or {}).items():
            e.set_tuning(k, v)
        e.set_pairs([a for a, _ in pairs], [b for _, b in pairs])
        info = e.align()
        return e.pair_max(), decode_hits(*e.hits()), info
    finally:
        e.close()


def _oracle_pairs(oracle_mod, queries, targets, pairs, st):
    score = scores.make_score(st)
    p = cases.oracle_params(oracle_mod, score)
    hits, maxima = [], {}
    for qi, ti in pairs:
        pos = cases.pos_scores(score, st, [queries[qi]], [targets[ti]])
        o = oracle_mod.run(p, [queries[qi]], [targets[ti]], pos, float(st.minimum_score))
        maxima[(qi, ti)] = float(o["pair_max"][0, 0])
        hits += [dict(h, query=qi, target=ti) for h in o["hits"]]
    return maxima, hits


@pytest.mark.parametrize("big", [False, True])
def test_pairs_two_at_a_time_on_16x2_lanes(engine_lib, oracle_mod, big):
    """Explicit pairs that share their query and their target's length (a pair
    and its reverse-complement target) are swept two at a time in 16-bit
    halves; with scores whose maxima pass 32767 - highest, those pairs are
    swept again on 32-bit lanes (pw_run_info.overflow_pairs).  Maxima and hits
    equal the oracle's pair by pair, and the 32-bit form's."""
    rng = np.random.default_rng(61 + big)
    comp = {"A": "T", "C": "G", "G": "C", "T": "A"}
    queries, targets, pairs = [], [], []
    for k in range(3):
        lq, lt = int(rng.integers(800, 1200)), int(rng.integers(800, 1200))
        q = "".join(rng.choice(list("ACGT"), size=lq))
        t = "".join(rng.choice(list("ACGT"), size=lt))
        n = min(lq, lt) // 2
        a, b = int(rng.integers(0, lq - n)), int(rng.integers(0, lt - n))
        # big scores: exact copies of 400-600 residues reach 40,000-60,000
        seg = q[a:a + n] if big else cases.mutate(rng, q[a:a + n], "ACGT", 0.05, 1)
        t = t[:b] + seg + t[b + n:]
        t = t[:lt]
        queries.append(q)
        targets += [t, "".join(comp[c] for c in reversed(t))]
        pairs += [(k, 2 * k), (k, 2 * k + 1)]
    pairs.append((0, 3))  # a pair without a partner of its target length
    if big:
        # int8 scores (the integer sweeps' range) whose maxima pass 2^15
        st = cases.Settings(match_score="100", mismatch_score="-100", gap_score="-120", minimum_score="10",
                            lower_limit_score="0.5", filter_factor="0.01")
    else:
        st = cases.Settings(minimum_score="20", lower_limit_score="0.5", filter_factor="0.01")
    maxima, hits = _oracle_pairs(oracle_mod, queries, targets, pairs, st)
    pm, got, info = _pairs_run(engine_lib, queries, targets, pairs, st)
    pm32, got32, info32 = _pairs_run(engine_lib, queries, targets, pairs, st, {_native.PW_TUNE_LANES: 32})
    for (qi, ti), m in maxima.items():
        assert pm[qi, ti] == m and pm32[qi, ti] == m
    key = lambda h: (h["query"], h["target"], h["s_end"], h["t_end"])
    assert sorted(got, key=key) == sorted(hits, key=key)
    assert got == got32
    assert len(hits) >= 3
    assert (info.overflow_pairs > 0) == big
