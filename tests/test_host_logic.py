"""Host-side semantics that need no GPU: Hit validation and ratios, HitList
de-duplication, id keys, records and reverse complements."""
import numpy as np
import pytest

from pypaswas_b200.exceptions import CudaException, InvalidOptionException
from pypaswas_b200.hits import Hit, HitList
from pypaswas_b200.records import SeqRecord, complement_records, sort_records
from pypaswas_b200.smith_waterman import id_keys
from pypaswas_b200 import scores, workloads


def _hit(s, t, sl, tl, score=10.0, aln="||||"):
    h = Hit(None, s, t, sl, tl)
    h.set_alignment(aln)
    h.set_scores(score, 4, 0)
    return h


def test_hit_location_rules():
    s, t = SeqRecord("ACGTACGT", "q"), SeqRecord("ACGT", "t")
    _hit(s, t, (0, 3), (0, 3))
    for bad in [(3, 3), (4, 3), (0, 8), (-1, 2)]:
        with pytest.raises(CudaException):
            Hit(None, s, t, bad, (0, 3))
    with pytest.raises(CudaException):
        Hit(None, s, t, (0, 3), (0, 4))


def test_hit_ratios():
    s, t = SeqRecord("ACGTACGT", "q"), SeqRecord("ACGTAC", "t")
    h = _hit(s, t, (1, 4), (0, 3), score=8.0)
    assert h.relative_score == 8.0 / 6
    assert h.query_identity == 4 / 4.0
    assert h.query_coverage == 4 / 8.0
    assert h.base_score == 8.0 / 4
    with pytest.raises(CudaException):
        h.set_scores(-1.0, 1, 1)
    with pytest.raises(CudaException):
        h.set_scores(1.0, 1.5, 1)


def test_hitlist_keeps_best_per_start_and_end():
    s, t = SeqRecord("A" * 20, "q"), SeqRecord("A" * 20, "t")
    hl = HitList()
    a = _hit(s, t, (0, 5), (0, 5), 5.0)
    b = _hit(s, t, (0, 7), (0, 7), 7.0)  # same start, better
    c = _hit(s, t, (1, 7), (1, 7), 3.0)  # same end as b, worse: rejected
    d = _hit(s, t, (2, 7), (2, 7), 9.0)  # same end as b, better: replaces b
    for h in (a, b, c, d):
        hl.append(h)
    assert list(hl.real_hits.values()) == [d]
    assert hl.hits[("q", "t", 0, 0)] is b


def test_id_keys_equal_exactly_for_equal_ids():
    qk, tk = id_keys(["a", "b", "a"], ["b", "c"])
    assert qk[0] == qk[2] and qk[1] == tk[0] and len({qk[0], qk[1], tk[1]}) == 3


def test_records_and_reverse_complement():
    r = SeqRecord(b"acgtNKM", "x")
    assert str(r.seq) == "ACGTNKM" and r.original_length == 7
    rc = complement_records([r])
    assert [x.id for x in rc] == ["x", "x_RC"] and str(rc[1].seq) == "KMNACGT"
    assert [len(x) for x in sort_records([SeqRecord("A", "1"), SeqRecord("AAA", "2")])] == [3, 1]
    assert workloads.reverse_complement(b"ACGTU") == b"AACGT"


def test_scores_highest_and_errors():
    st = workloads.Settings(matrix_name="BLOSUM62")
    assert scores.make_score(st).highest_score == 4  # max(max(matrix)): the 'A' row
    assert scores.make_score(workloads.Settings(matrix_name="BLOSUM80")).highest_score == 7
    with pytest.raises(InvalidOptionException):
        scores.make_score(workloads.Settings(matrix_name="PAM250"))
    with pytest.raises(InvalidOptionException):
        scores.make_score(workloads.Settings(matrix_name="CUSTOM"))
    b = scores.make_score(workloads.Settings(matrix_name="BASIC", match_score="2", mismatch_score="-1"))
    m = b.matrix_array()
    assert m.shape == (255, 255) and m[5, 5] == 2 and m[5, 6] == -1 and b.char_offset_code() == 1
    ir = scores.make_score(workloads.Settings(matrix_name="IRYS", match_score="3", mismatch_score="-0.5"))
    assert ir.matrix_array().shape == (62, 62) and ir.matrix_array()[0, 3] == np.float32(-1.5)


def test_kernel_constants_follow_compiled_literals():
    st = workloads.Settings(gap_score="-5", gap_extension="0", lower_limit_score="0.1", minimum_score="15.3")
    gap, ext, affine, ll, mn = scores.make_score(st).kernel_constants()
    assert not affine and gap == np.float32(-5.0) and ext == 0
    assert ll == np.float32(0.1) and mn == np.float32(15.3)


def test_serving_percentile_is_nearest_rank():
    from pypaswas_b200.serving import percentile
    v = list(range(1, 101))
    assert percentile(v, 50) == 50 and percentile(v, 99) == 99 and percentile(v, 100) == 100
    assert percentile([7.0], 99) == 7.0
    assert percentile([3, 1, 2], 50) == 2


def test_autotune_keeps_the_fastest_candidate():
    from pypaswas_b200 import _native
    from pypaswas_b200.autotune import autotune

    class Info(object):
        def __init__(self, ms, path):
            self.total_ms = ms
            self.score_path = path

    class FakeEngine(object):
        """Score-phase time (plan and sweep) as a function of lane width, 16x2 form and chaining."""
        chain_cost = {250: 9.0, 500: 7.5, 1000: 8.0, 2000: 7.5}

        def __init__(self):
            self.tune = {}

        def set_tuning(self, key, value):
            self.tune[key] = value

        def align(self, score_only=False, replan=False):
            assert score_only and replan
            if self.tune.get(_native.PW_TUNE_LANES, 0) == 32:
                return Info(20.0, 1)
            t = self.chain_cost[self.tune.get(_native.PW_TUNE_CHAIN_MIN, 500)]
            t += {0: 0.0, 1: 0.5, 2: -0.25}[self.tune.get(_native.PW_TUNE_DUAL, 0)]
            return Info(t, 0)

    e = FakeEngine()
    r = autotune(e)
    assert r["lanes"] == 16 and e.tune[_native.PW_TUNE_LANES] == 0
    assert r["dual"] == "strip pairs" and e.tune[_native.PW_TUNE_DUAL] == 2
    assert r["chain_min"] == 500  # ties go to the smaller value
    assert e.tune[_native.PW_TUNE_CHAIN_MIN] == 500
    assert r["score_phase_ms"] == {k: v - 0.25 for k, v in FakeEngine.chain_cost.items()}


def test_fast_hit_building_matches_hitlist_append_and_checked_path():
    """SmithWaterman hit building: the vectorised path with HitList.append
    inlined gives the same HitList (keys, replacement rule, Hit fields) as
    appending through HitList.append, and as the validating constructor path."""
    import logging
    import numpy as np
    from pypaswas_b200 import _native
    from pypaswas_b200.hits import HitList
    from pypaswas_b200.records import SeqRecord
    from pypaswas_b200.smith_waterman import SmithWatermanB200
    import cases

    class PlainList(HitList):  # a subclass takes the generic append path
        pass

    rng = np.random.default_rng(7)
    seqs = [SeqRecord("".join("ACGT"[i] for i in rng.integers(0, 4, 60)), "q%d" % i) for i in range(5)]
    tgts = [SeqRecord("".join("ACGT"[i] for i in rng.integers(0, 4, 50)), "t%d" % i) for i in range(4)]
    rows = []
    for _ in range(300):
        q, t = int(rng.integers(0, 5)), int(rng.integers(0, 4))
        s0, t0 = int(rng.integers(0, 20)), int(rng.integers(0, 20))
        n = int(rng.integers(2, 25))
        s1, t1 = min(s0 + n, 59), min(t0 + n, 49)
        rows.append((q, t, s0, s1, t0, t1, float(rng.integers(5, 40)), n))
    rows += rows[:40]  # repeated keys: equal scores are rejected, higher ones replace
    hits = np.zeros(len(rows), dtype=_native.HIT_DTYPE)
    text, off = [], 0
    for k, (q, t, s0, s1, t0, t1, sc, n) in enumerate(rows):
        hits[k] = 0
        for name, v in (("query", q), ("target", t), ("s_start", s0), ("s_end", s1), ("t_start", t0),
                        ("t_end", t1), ("score", sc), ("matches", n // 2), ("mismatches", n - n // 2),
                        ("n_cols", n), ("str_offset", off)):
            hits[k][name] = v
        text.append("A" * n + "|" * n + "C" * n)
        off += 3 * n
    strbuf = "".join(text).encode("latin-1")
    st = cases.Settings(relative_score="0.1", query_identity="0.2", query_coverage="0", base_score="0")
    sw = SmithWatermanB200.__new__(SmithWatermanB200)
    sw.logger = logging.getLogger("test")
    sw.settings = st

    def run(hl):
        sw._build_hits(hits, strbuf, seqs, tgts, hl)
        return hl

    def view(hl):
        out = {}
        for name in ("hits", "real_hits"):
            d = getattr(hl, name)
            out[name] = {k: tuple(sorted((a, v) for a, v in h.__dict__.items() if a != "logger")) for k, h in d.items()}
        return out

    fast, generic = run(HitList(sw.logger)), run(PlainList(sw.logger))
    assert len(fast.hits) > 50
    assert view(fast) == view(generic)
    checked = HitList(sw.logger)
    s0 = hits["s_start"].astype(np.int64)
    sw._build_hits_checked(hits, strbuf.decode("latin-1"), seqs, tgts, checked, s0, hits["s_end"].astype(np.int64),
                           hits["t_start"].astype(np.int64), hits["t_end"].astype(np.int64))
    assert view(fast) == view(checked)
