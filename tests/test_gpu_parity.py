"""Engine (CUDA, through the C ABI) against the CPU oracle on seeded cases.

Bit-exact: pair maxima, every hit's coordinates, score, match counts and the
three alignment strings, in HitList order."""
import numpy as np
import pytest

import cases
from engine_helpers import configure, run_engine

pytestmark = pytest.mark.gpu

KINDS = ["dna", "protein", "dna_ambiguous", "dna_float"]


def _oracle(oracle_mod, queries, targets, score, settings, q_keys=None, t_keys=None):
    p = cases.oracle_params(oracle_mod, score)
    pos = cases.pos_scores(score, settings, queries, targets)
    return oracle_mod.run(p, queries, targets, pos, float(settings.minimum_score), q_keys, t_keys)


@pytest.mark.parametrize("seed", range(24))
def test_random_cases_bit_exact(engine_lib, oracle_mod, seed):
    kind = KINDS[seed % len(KINDS)]
    queries, targets, score, st = cases.make_case(1000 + seed, kind)
    o = _oracle(oracle_mod, queries, targets, score, st)
    pm, hits, info, launches = run_engine(engine_lib, queries, targets, score, st)
    assert launches > 0
    np.testing.assert_array_equal(pm, o["pair_max"])
    assert hits == o["hits"]


def test_same_id_pairs_are_skipped(engine_lib, oracle_mod):
    queries, targets, score, st = cases.make_case(77, "dna")
    q_keys = np.arange(len(queries))
    t_keys = np.array([0] + [len(queries) + i for i in range(1, len(targets))])  # target 0 shares query 0's id
    o = _oracle(oracle_mod, queries, targets, score, st, q_keys, t_keys)
    pm, hits, _, _ = run_engine(engine_lib, queries, targets, score, st, q_keys, t_keys)
    assert hits == o["hits"]
    assert not any(h["query"] == 0 and h["target"] == 0 for h in hits)


def test_score_only_matches_full_run(engine_lib, oracle_mod):
    queries, targets, score, st = cases.make_case(5, "protein")
    pm, hits, info, _ = run_engine(engine_lib, queries, targets, score, st, score_only=True)
    assert hits == []
    np.testing.assert_array_equal(pm, oracle_mod.pair_max(cases.oracle_params(oracle_mod, score), queries, targets))


def test_run_is_deterministic(engine_lib):
    queries, targets, score, st = cases.make_case(11, "dna")
    a = run_engine(engine_lib, queries, targets, score, st)
    b = run_engine(engine_lib, queries, targets, score, st)
    np.testing.assert_array_equal(a[0], b[0])
    assert a[1] == b[1]


def test_edge_lengths(engine_lib, oracle_mod):
    # single residues, lengths around strip and lane-group boundaries
    rng = np.random.default_rng(3)
    lens_q = [1, 2, 3, 4, 5, 7, 8, 9, 15, 16, 17, 31, 32, 33, 63, 64, 65]
    lens_t = [1, 4, 16, 17, 32, 33, 64, 65, 97]
    q = ["".join("ACGT"[i] for i in rng.integers(0, 4, n)) for n in lens_q]
    t = ["".join("ACGT"[i] for i in rng.integers(0, 4, n)) for n in lens_t]
    t[3] = q[-1][:17]
    for aff in ("0", "-1"):
        st = cases.Settings(minimum_score="2", lower_limit_score="0.5", gap_extension=aff)
        from pypaswas_b200 import scores
        score = scores.make_score(st)
        o = _oracle(oracle_mod, q, t, score, st)
        pm, hits, _, _ = run_engine(engine_lib, q, t, score, st)
        np.testing.assert_array_equal(pm, o["pair_max"])
        assert hits == o["hits"]


def test_many_pairs_pair_max(engine_lib, oracle_mod):
    # 600 x 40 pairs: several warps per target and all strip classes
    rng = np.random.default_rng(9)
    q = ["".join("ACGT"[i] for i in rng.integers(0, 4, int(rng.integers(1, 160)))) for _ in range(600)]
    t = ["".join("ACGT"[i] for i in rng.integers(0, 4, int(rng.integers(1, 120)))) for _ in range(40)]
    for aff in ("0", "-1"):
        st = cases.Settings(minimum_score="9", gap_extension=aff)
        from pypaswas_b200 import scores
        score = scores.make_score(st)
        o = _oracle(oracle_mod, q, t, score, st)
        pm, hits, _, _ = run_engine(engine_lib, q, t, score, st)
        np.testing.assert_array_equal(pm, o["pair_max"])
        assert hits == o["hits"]


def test_sixteen_bit_overflow_is_recomputed(engine_lib, oracle_mod):
    # match score 120 over 290-400 identical residues: maxima above the 16-bit
    # limit (32640), so these pairs must come from the 32-bit recompute
    from pypaswas_b200 import scores
    rng = np.random.default_rng(12)
    base = "".join("ACGT"[i] for i in rng.integers(0, 4, 400))
    q = [base, base[:330] + "A" * 20, "".join("ACGT"[i] for i in rng.integers(0, 4, 90))]
    t = [base, base[40:]]
    st = cases.Settings(match_score="120", mismatch_score="-3", minimum_score="50")
    score = scores.make_score(st)
    o = _oracle(oracle_mod, q, t, score, st)
    pm, hits, info, _ = run_engine(engine_lib, q, t, score, st)
    assert info.overflow_pairs >= 4
    np.testing.assert_array_equal(pm, o["pair_max"])
    assert hits == o["hits"]


@pytest.mark.parametrize("shape", [(600, 40), (40, 600), (97, 97)])
def test_lane_orientations_and_32_bit_sweep_agree(engine_lib, oracle_mod, shape):
    rng = np.random.default_rng(sum(shape))
    nq, nt = shape
    q = ["".join(cases.PROTEIN[i] for i in rng.integers(0, 20, int(rng.integers(1, 150)))) for _ in range(nq)]
    t = ["".join(cases.PROTEIN[i] for i in rng.integers(0, 20, int(rng.integers(1, 150)))) for _ in range(nt)]
    from pypaswas_b200 import scores
    for aff in ("0", "-1"):
        st = cases.Settings(matrix_name="BLOSUM62", gap_score="-11", gap_extension=aff, minimum_score="40")
        score = scores.make_score(st)
        pm16 = run_engine(engine_lib, q, t, score, st, score_only=True)[0]
        pm32 = run_engine(engine_lib, q, t, score, st, score_only=True, int32=True)[0]
        np.testing.assert_array_equal(pm16, pm32)
        np.testing.assert_array_equal(pm16, oracle_mod.pair_max(cases.oracle_params(oracle_mod, score), q, t))


@pytest.mark.parametrize("kind", ["dna", "protein"])
def test_long_targets_one_warp_per_pair(engine_lib, oracle_mod, kind):
    # targets longer than 64 are swept one pair per warp in 256-row bands:
    # lengths around the band edges, planted segments long enough that some
    # pairs find more candidates than their first slot holds
    from pypaswas_b200 import _native, scores
    rng = np.random.default_rng(31 if kind == "dna" else 32)
    alphabet = cases.DNA if kind == "dna" else cases.PROTEIN
    draw = lambda n: "".join(alphabet[i] for i in rng.integers(0, len(alphabet), n))
    targets = [draw(n) for n in (65, 200, 255, 256, 257, 300, 511, 513, 700)]
    queries = [draw(n) for n in (1, 2, 31, 32, 33, 90)]
    for _ in range(24):
        t = targets[int(rng.integers(0, len(targets)))]
        cut = int(rng.integers(0, len(t) // 2))
        s = draw(int(rng.integers(0, 60)))
        p = int(rng.integers(0, len(s) + 1))
        queries.append(s[:p] + cases.mutate(rng, t[cut:cut + int(rng.integers(20, 400))], alphabet, 0.05, 1) + s[p:])
    for aff in ("0", "-1"):
        kw = dict(minimum_score="10", lower_limit_score="0.5", filter_factor="0.1", gap_extension=aff)
        if kind == "protein":
            kw.update(matrix_name="BLOSUM62", gap_score="-11")
        st = cases.Settings(**kw)
        score = scores.make_score(st)
        o = _oracle(oracle_mod, queries, targets, score, st)
        pm, hits, info, _ = run_engine(engine_lib, queries, targets, score, st)
        assert info.warp_pairs > 0
        np.testing.assert_array_equal(pm, o["pair_max"])
        assert hits == o["hits"]
        # slots of 4 candidates: pairs outgrow them and are swept again
        pm, hits, info, _ = run_engine(engine_lib, queries, targets, score, st,
                                       tuning={_native.PW_TUNE_CAND_SLOT: 4})
        assert info.warp_pairs > 0 and info.cand_overflow_pairs > 0
        np.testing.assert_array_equal(pm, o["pair_max"])
        assert hits == o["hits"]


@pytest.mark.parametrize("aff", ["0", "-1"])
def test_many_short_targets_strip_direction_sweep(engine_lib, oracle_mod, aff):
    # enough traced pairs with short targets (<= 64) to fill every SM with a
    # warp: these stay on the per-lane strip sweep
    from pypaswas_b200 import scores
    rng = np.random.default_rng(41 if aff == "0" else 42)
    draw = lambda n: "".join("ACGT"[i] for i in rng.integers(0, 4, n))
    targets = [draw(int(n)) for n in rng.integers(8, 65, 12)]
    queries = []
    for _ in range(640):
        s = draw(int(rng.integers(10, 150)))
        t = targets[int(rng.integers(0, len(targets)))]
        p = int(rng.integers(0, len(s) + 1))
        queries.append(s[:p] + cases.mutate(rng, t, "ACGT", 0.1, 1) + s[p:])
    st = cases.Settings(minimum_score="5", lower_limit_score="0.9", filter_factor="0.0", gap_extension=aff)
    score = scores.make_score(st)
    o = _oracle(oracle_mod, queries, targets, score, st)
    pm, hits, info, _ = run_engine(engine_lib, queries, targets, score, st)
    assert info.traced_pairs >= 148 * 32 and info.warp_pairs == 0
    np.testing.assert_array_equal(pm, o["pair_max"])
    assert hits == o["hits"]
    # slots of 2 candidates: the strip items of pairs that outgrow them are swept again
    from pypaswas_b200 import _native
    pm, hits, info, _ = run_engine(engine_lib, queries, targets, score, st, tuning={_native.PW_TUNE_CAND_SLOT: 2})
    assert info.cand_overflow_pairs > 0
    np.testing.assert_array_equal(pm, o["pair_max"])
    assert hits == o["hits"]


@pytest.mark.parametrize("kind", ["dna", "protein", "protein_linear"])
@pytest.mark.parametrize("chain_min,segment", [(0, 0), (1, 0), (1, 37)])
def test_chained_strips_match_one_warp_items_and_oracle(engine_lib, oracle_mod, kind, chain_min, segment):
    """Multi-strip items cut into chained strips (the default share, and with
    chain_min 1 nearly every multi-strip item; segment 37 splits the queue
    into launches of 37 entries, so chains cross launches) give the same pair
    maxima as the one-warp items and the oracle, in both lane orientations."""
    from pypaswas_b200 import _native, scores
    rng = np.random.default_rng({"dna": 5, "protein": 6, "protein_linear": 7}[kind] * 10 + chain_min)
    alphabet = cases.DNA if kind == "dna" else cases.PROTEIN
    for nq, nt in ((14, 40), (40, 14)):
        q = ["".join(alphabet[i] for i in rng.integers(0, len(alphabet), int(n)))
             for n in rng.integers(33, 300, nq)]
        t = ["".join(alphabet[i] for i in rng.integers(0, len(alphabet), int(n)))
             for n in rng.integers(20, 260, nt)]
        q[0] = t[0][10:120] + q[0]  # a shared segment
        st = cases.Settings(gap_extension="-1" if kind in ("dna", "protein") else "0", minimum_score="5",
                            **({} if kind == "dna" else dict(matrix_name="BLOSUM62", gap_score="-11")))
        score = scores.make_score(st)
        ref = oracle_mod.pair_max(cases.oracle_params(oracle_mod, score), q, t)
        e = _native.Engine(0, lib=engine_lib)
        try:
            configure(e, score, st)
            e.set_queries([s.encode() for s in q], np.arange(nq))
            e.set_targets([s.encode() for s in t], np.arange(nt) + nq)
            e.set_tuning(_native.PW_TUNE_CHAIN_MIN, chain_min)
            e.set_tuning(_native.PW_TUNE_SEGMENT, segment)
            e.align(score_only=True)
            chained = e.pair_max()
            e.align(score_only=True, chain=False)
            single = e.pair_max()
        finally:
            e.close()
        np.testing.assert_array_equal(chained, ref)
        np.testing.assert_array_equal(single, ref)


@pytest.mark.parametrize("kind", ["dna", "protein", "protein_linear"])
@pytest.mark.parametrize("shape", [(1, 150), (3, 97), (14, 40), (40, 14)])
@pytest.mark.parametrize("chain_min", [0, 1])
def test_dual_lane_sweep_matches_oracle(engine_lib, oracle_mod, kind, shape, chain_min):
    """The dual-lane form of the 16-bit sweep (one strip against two lane
    sequences per lane; forced on with PW_TUNE_DUAL 1) gives the oracle's pair
    maxima and hits: single-strip and multi-strip lengths, lane groups cut
    short (97 and 150 lanes leave the second group partly empty), chained and
    one-warp items.  The automatic choice picks it for a single query."""
    from pypaswas_b200 import _native, scores
    rng = np.random.default_rng({"dna": 8, "protein": 9, "protein_linear": 10}[kind] * 100 + sum(shape) + chain_min)
    alphabet = cases.DNA if kind == "dna" else cases.PROTEIN
    nq, nt = shape
    q = ["".join(alphabet[i] for i in rng.integers(0, len(alphabet), int(n))) for n in rng.integers(5, 300, nq)]
    t = ["".join(alphabet[i] for i in rng.integers(0, len(alphabet), int(n))) for n in rng.integers(5, 260, nt)]
    q[0] = t[0][:100] + q[0]  # a shared segment
    st = cases.Settings(gap_extension="-1" if kind in ("dna", "protein") else "0", minimum_score="20",
                        **({} if kind == "dna" else dict(matrix_name="BLOSUM62", gap_score="-11")))
    score = scores.make_score(st)
    o = _oracle(oracle_mod, q, t, score, st)
    tuning = {_native.PW_TUNE_DUAL: 1, _native.PW_TUNE_CHAIN_MIN: chain_min}
    pm, hits, info, _ = run_engine(engine_lib, q, t, score, st, tuning=tuning)
    assert info.dual_lanes == 1 and info.score_path == 0
    np.testing.assert_array_equal(pm, o["pair_max"])
    assert hits == o["hits"]
    if nq == 1 and chain_min == 0:
        pm_auto, _, info_auto, _ = run_engine(engine_lib, q, t, score, st, score_only=True)
        assert info_auto.dual_lanes == 1
        np.testing.assert_array_equal(pm_auto, o["pair_max"])


def _oracle_pairs(oracle_mod, queries, targets, pairs, score, st):
    """Oracle hits and maxima of explicit pairs, one pair at a time."""
    p = cases.oracle_params(oracle_mod, score)
    hits, maxima = {}, {}
    for qi, ti in pairs:
        q, t = queries[qi], targets[ti]
        pos = cases.pos_scores(score, st, [q], [t])
        o = oracle_mod.run(p, [q], [t], pos, float(st.minimum_score))
        maxima[(qi, ti)] = float(o["pair_max"][0, 0])
        hits[(qi, ti)] = [dict(h, query=qi, target=ti) for h in o["hits"]]
    return hits, maxima


@pytest.mark.parametrize("affine", ["0", "-1"])
def test_pair_list_long_pairs_bands_chained(engine_lib, oracle_mod, affine):
    """Explicit pairs, long ones swept band by band on different warps (score
    and direction sweeps), against the oracle pair by pair."""
    from pypaswas_b200 import _native, scores
    rng = np.random.default_rng(42 if affine == "0" else 43)

    def rs(n):
        return "".join("ACGT"[i] for i in rng.integers(0, 4, n))
    queries, targets = [], []
    for lq, lt in ((2600, 2200), (700, 1900), (1800, 300), (40, 1200), (900, 900), (257, 513)):
        shared = rs(min(lq, lt) // 2)
        mut = "".join(c if rng.random() > 0.12 else "ACGT"[int(rng.integers(0, 4))] for c in shared)
        a = int(rng.integers(0, lq - len(shared) + 1))
        b = int(rng.integers(0, lt - len(shared) + 1))
        q = rs(lq)
        t = rs(lt)
        queries.append(q[:a] + shared + q[a + len(shared):])
        targets.append(t[:b] + mut + t[b + len(mut):])
    pairs = [(k, k) for k in range(len(queries))] + [(0, 1), (3, 0)]
    st = cases.Settings(gap_extension=affine, minimum_score="20", lower_limit_score="0.9", filter_factor="0.02")
    score = scores.make_score(st)
    ref_hits, ref_max = _oracle_pairs(oracle_mod, queries, targets, pairs, score, st)
    e = _native.Engine(0, lib=engine_lib)
    try:
        configure(e, score, st)
        e.set_queries([s.encode() for s in queries], np.arange(len(queries)))
        e.set_targets([s.encode() for s in targets], np.arange(len(targets)) + len(queries))
        e.set_pairs([p[0] for p in pairs], [p[1] for p in pairs])
        info = e.align()
        pm = e.pair_max()
        from engine_helpers import decode_hits
        got = decode_hits(*e.hits())
    finally:
        e.close()
    assert info.pairs == len(pairs)
    for (qi, ti), m in ref_max.items():
        assert pm[qi, ti] == m
    listed = set(pairs)
    assert all(pm[i, j] == -1.0 for i in range(len(queries)) for j in range(len(targets)) if (i, j) not in listed)
    by_pair = {}
    for h in got:
        by_pair.setdefault((h["query"], h["target"]), []).append(h)
    assert {k: v for k, v in by_pair.items()} == {k: v for k, v in ref_hits.items() if v}
    assert sum(len(v) for v in ref_hits.values()) >= 4


@pytest.mark.parametrize("seed", range(3))
def test_query_trace_mask_keeps_the_traced_queries_hits(engine_lib, oracle_mod, seed):
    """pw_set_query_trace: masked-out queries keep their pair maxima and give
    no hits; the others give exactly their hits of the unmasked run, in the
    same order.  pw_set_queries clears the mask."""
    from engine_helpers import configure, decode_hits
    from pypaswas_b200 import _native
    queries, targets, score, st = cases.make_case(500 + seed, ["dna", "protein", "dna"][seed])
    o = _oracle(oracle_mod, queries, targets, score, st)
    mask = np.arange(len(queries)) % 2 == 0
    e = _native.Engine(0, lib=engine_lib)
    try:
        configure(e, score, st)
        e.set_queries([q.encode() for q in queries], np.arange(len(queries)))
        e.set_targets([t.encode() for t in targets], np.arange(len(targets)) + len(queries))
        e.set_query_trace(mask)
        e.align()
        np.testing.assert_array_equal(e.pair_max(), o["pair_max"])
        assert decode_hits(*e.hits()) == [h for h in o["hits"] if mask[h["query"]]]
        e.set_queries([q.encode() for q in queries], np.arange(len(queries)))
        e.align()
        assert decode_hits(*e.hits()) == o["hits"]
    finally:
        e.close()
