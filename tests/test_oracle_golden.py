"""The oracle against the reference's own outputs (golden fixtures).

Pins the CPU restatement (oracle/paswas_oracle.c): pair maxima, starting points
(set and emission order per pair) and every walked hit must equal what the
reference's kernels and host walk produced."""
import numpy as np
import pytest

import cases
import golden_util as G
from pypaswas_b200 import scores
from pypaswas_b200.exceptions import CudaException
from pypaswas_b200.hits import Hit
from pypaswas_b200.records import SeqRecord

NAMES = [n for n in G.names()]


def _run_oracle(oracle_mod, fx):
    st = G.FixtureSettings(fx)
    score = scores.make_score(st)
    q = [s for _, s in fx["queries"]]
    t = [s for _, s in fx["targets"]]
    ids = {}
    qk = [ids.setdefault(i, len(ids)) for i, _ in fx["queries"]]
    tk = [ids.setdefault(i, len(ids)) for i, _ in fx["targets"]]
    pos = cases.pos_scores(score, st, q, t)
    cap = 100 * len(q) * len(t)
    return oracle_mod.run(cases.oracle_params(oracle_mod, score), q, t, pos, float(st.minimum_score), qk, tk,
                          start_cap=cap), score


@pytest.mark.parametrize("name", NAMES)
def test_scoring_model_matches_reference(name):
    fx = G.load(name)
    if "matrix" not in fx:
        pytest.skip("fixture records an exception")
    score = scores.make_score(G.FixtureSettings(fx))
    np.testing.assert_array_equal(score.matrix_array(), np.array(fx["matrix"], dtype=np.float32))
    assert score.char_offset_code() == fx["char_offset"]
    assert float(score.highest_score) == fx["highest_score"]


@pytest.mark.parametrize("name", NAMES)
def test_oracle_matches_reference(oracle_mod, name):
    fx = G.load(name)
    o, score = _run_oracle(oracle_mod, fx)
    qid = [i for i, _ in fx["queries"]]
    tid = [i for i, _ in fx["targets"]]
    if "exception" in fx:
        # the reference raised while building a Hit: the oracle's walk yields the
        # same one-column hit, which Hit rejects the same way
        with pytest.raises(CudaException):
            for h in o["hits"]:
                Hit(None, SeqRecord(fx["queries"][h["query"]][1], qid[h["query"]]),
                    SeqRecord(fx["targets"][h["target"]][1], tid[h["target"]]),
                    (h["s_start"], h["s_end"]), (h["t_start"], h["t_end"]))
        return
    # pair maxima
    ref_pm = G.global_pair_max(fx)
    known = ~np.isnan(ref_pm)
    np.testing.assert_array_equal(o["pair_max"][known], ref_pm[known].astype(np.float32))
    # starting points: per pair, same cells in the same emission order
    ref_starts = G.starts_by_pair(fx)
    mine = {}
    for s in o["starts"]:
        mine.setdefault((int(s["sequence"]), int(s["target"])), []).append(
            (int(s["block_x"]) * 8 + int(s["value_x"]), int(s["block_y"]) * 8 + int(s["value_y"]), float(s["score"])))
    assert mine == ref_starts
    # hits: per (query id, target id), same hits in the same order
    got = [{"seq_id": qid[h["query"]], "target_id": tid[h["target"]],
            "seq_location": [h["s_start"], h["s_end"]], "target_location": [h["t_start"], h["t_end"]],
            "score": h["score"], "matches": h["matches"], "mismatches": h["mismatches"],
            "sequence_match": h["sequence_match"], "alignment": h["alignment"],
            "target_match": h["target_match"]} for h in o["hits"]]
    keys = ["seq_id", "target_id", "seq_location", "target_location", "score", "matches", "mismatches",
            "sequence_match", "alignment", "target_match"]
    ref = G.hits_by_pair([{k: h[k] for k in keys} for h in fx["hits"]])
    assert G.hits_by_pair(got) == ref
    if len(fx["batches"]) == 1:
        # one batch: the whole HitList order is the walk order
        assert got == [{k: h[k] for k in keys} for h in fx["hits"]]


def test_genbank_case_reproduces_reference_expected_output():
    fx = G.load("genbank_basic")
    exp = fx["reference_expected_fields"]
    h = fx["hits"][0]
    assert [h["seq_id"], h["target_id"]] == exp[:2]
    assert h["seq_location"] + h["target_location"] == [int(v) for v in exp[2:6]]
    assert h["score"] == float(exp[6]) and h["matches"] == int(exp[7]) and h["mismatches"] == int(exp[8])
    assert len(h["alignment"]) == int(exp[10])
    assert abs(h["score"] / len(h["alignment"]) - float(exp[11])) < 1e-9


@pytest.mark.parametrize("name", NAMES)
def test_reference_emits_starting_points_in_launch_order(name):
    """Within a batch the reference's kernels, run one launch and one block
    after another, emit starting points by block anti-diagonal descending,
    block x descending, target, query, cell anti-diagonal descending, row --
    the order pw_get_starting_points reports."""
    fx = G.load(name)
    for b in fx.get("batches", []):
        keys = [(-(u[2] + u[3]), -u[2], u[1], u[0], -(u[4] + u[5]), u[5]) for u in b["starts_u32"]]
        assert keys == sorted(keys)


def test_oracle_start_cap_walks_the_first_starts_in_emission_order(oracle_mod):
    """With more starting points than the cap, the host reads the first cap of
    the device buffer (emission order, SmithWaterman.py:683-687) and walks
    those by ascending score: every capped hit ends on one of them, and a cap
    at the full count changes nothing."""
    rng = np.random.default_rng(3)
    seqs = ["".join("ACGT"[i] for i in rng.integers(0, 4, int(rng.integers(60, 200)))) for _ in range(6)]
    queries = seqs[:3] + [s[10:90] for s in seqs[3:]]
    targets = seqs[3:] + [s[5:80] for s in seqs[:3]]
    st = cases.Settings(minimum_score="6", lower_limit_score="0.3", filter_factor="0.05")
    score = scores.make_score(st)
    p = cases.oracle_params(oracle_mod, score)
    pos = cases.pos_scores(score, st, queries, targets)
    full = oracle_mod.run(p, queries, targets, pos, float(st.minimum_score))
    starts = full["starts"]
    assert len(starts) > 20
    emit = sorted(range(len(starts)), key=lambda k: (
        -(int(starts[k]["block_x"]) + int(starts[k]["block_y"])), -int(starts[k]["block_x"]),
        int(starts[k]["target"]), int(starts[k]["sequence"]),
        -(int(starts[k]["value_x"]) + int(starts[k]["value_y"])), int(starts[k]["value_y"])))
    assert oracle_mod.run(p, queries, targets, pos, float(st.minimum_score), start_cap=len(starts))["hits"] == \
        full["hits"]
    for cap in (1, len(starts) // 4, len(starts) // 2):
        first = {(int(starts[k]["sequence"]), int(starts[k]["target"]),
                  int(starts[k]["block_x"]) * 8 + int(starts[k]["value_x"]),
                  int(starts[k]["block_y"]) * 8 + int(starts[k]["value_y"])) for k in emit[:cap]}
        got = oracle_mod.run(p, queries, targets, pos, float(st.minimum_score), start_cap=cap)["hits"]
        assert all((h["query"], h["target"], h["s_end"], h["t_end"]) in first for h in got)
        assert len(got) <= cap
