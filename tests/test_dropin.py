"""The drop-in boundary at both ends, on the CPU.

Score in: SmithWatermanB200 configures the engine from the public attributes
of whatever Score object the reference's CLI built (pypaswasall.py:126-144),
so its kernel constants must equal this package's own Score's.

Hits out: the Hit objects the driver builds from engine records
(SmithWatermanB200._build_hits) must print through the formatters --
this package's and, where the reference tree is importable, the reference's own
DefaultFormatter / TrimmerFormatter / SamFormatter / FASTA (Formatters.py:3-186)
-- to the exact text the reference wrote for the golden fixtures.
"""
import logging
import os

import numpy as np
import pytest

import golden_util as G
from pypaswas_b200 import _native, scores
from pypaswas_b200.formatters import DefaultFormatter, FastaFormatter, SamFormatter, TrimmerFormatter, formatter_for
from pypaswas_b200.hits import HitList
from pypaswas_b200.records import SeqRecord
from pypaswas_b200.smith_waterman import SmithWatermanB200, configure_engine

NAMES = [n for n in G.names() if "exception" not in G.load(n)]
LOG = logging.getLogger("dropin")
LOG.setLevel(logging.WARNING)


def _reference():
    """oracle/ref/ref_driver (the reference's own modules behind stand-ins),
    or None where the reference tree is absent."""
    root = os.environ.get("PASWAS_REFERENCE_ROOT", "/root/reference")
    if not os.path.isdir(os.path.join(root, "pyPaSWAS")):
        return None
    import sys
    here = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "ref")
    if here not in sys.path:
        sys.path.insert(0, here)
    import ref_driver
    return ref_driver


needs_reference = pytest.mark.skipif(_reference() is None, reason="reference tree not present")


class _RecordingEngine(object):
    """Stands in for _native.Engine: keeps what set_scoring receives."""

    def set_scoring(self, *args):
        self.args = args


def _scoring_args(score, settings):
    e = _RecordingEngine()
    configure_engine(e, score, settings)
    m, rest = e.args[0], e.args[1:]
    return np.asarray(m, dtype=np.float32), tuple(float(v) for v in rest)


@needs_reference
@pytest.mark.parametrize("name", G.names())
def test_reference_score_object_configures_the_engine_identically(name):
    R = _reference()
    fx = G.load(name)
    ref_settings = R.Settings(**fx["settings"])
    ref_score = R.make_score(ref_settings, LOG)
    st = G.FixtureSettings(fx)
    ours = scores.make_score(st)
    m_ref, a_ref = _scoring_args(ref_score, ref_settings)
    m_our, a_our = _scoring_args(ours, st)
    np.testing.assert_array_equal(m_ref, m_our)
    assert a_ref == a_our
    if "matrix" in fx:
        np.testing.assert_array_equal(m_ref, np.array(fx["matrix"], dtype=np.float32))


def _engine_records(fx):
    """The fixture's HitList as the engine hands hits to the driver:
    pw_hit records in HitList order, their strings, and the record lists."""
    q_index = {i: k for k, (i, _) in enumerate(fx["queries"])}
    t_index = {i: k for k, (i, _) in enumerate(fx["targets"])}
    hits = np.zeros(len(fx["hits"]), dtype=_native.HIT_DTYPE)
    text = []
    off = 0
    for k, h in enumerate(fx["hits"]):
        n = len(h["alignment"])
        hits[k] = (q_index[h["seq_id"]], t_index[h["target_id"]], h["seq_location"][0], h["seq_location"][1],
                   h["target_location"][0], h["target_location"][1], h["score"], h["matches"], h["mismatches"],
                   n, off)
        text += [h["sequence_match"], h["alignment"], h["target_match"]]
        off += 3 * n
    queries = [SeqRecord(s, i) for i, s in fx["queries"]]
    targets = [SeqRecord(s, i) for i, s in fx["targets"]]
    return hits, "".join(text).encode("latin-1"), queries, targets


def _driver_hitlist(fx):
    """HitList built by the driver's own Hit construction path."""
    sw = SmithWatermanB200.__new__(SmithWatermanB200)
    sw.logger = LOG
    sw.settings = G.FixtureSettings(fx)
    hits, strbuf, queries, targets = _engine_records(fx)
    hl = HitList(LOG)
    sw._build_hits(hits, strbuf, queries, targets, hl)
    return hl


def _text(formatter_cls, hl, tmp_path):
    path = str(tmp_path / "out")
    formatter_cls(LOG, hl, path).print_results()
    with open(path) as f:
        return f.read()


@pytest.mark.parametrize("name", NAMES)
def test_driver_hits_replay_the_reference_hitlist(name):
    fx = G.load(name)
    hl = _driver_hitlist(fx)
    got = [(h.get_seq_id(), h.get_target_id(), list(h.seq_location), list(h.target_location), h.score)
           for h in hl.real_hits.values()]
    want = [(h["seq_id"], h["target_id"], h["seq_location"], h["target_location"], h["score"]) for h in fx["hits"]]
    assert got == want


@pytest.mark.parametrize("name", NAMES)
def test_own_formatters_write_the_reference_files(name, tmp_path):
    fx = G.load(name)
    assert _text(DefaultFormatter, _driver_hitlist(fx), tmp_path) == "".join(t + "\n" for t in fx["txt"])
    assert _text(TrimmerFormatter, _driver_hitlist(fx), tmp_path) == "".join(t + "\n" for t in fx["trimmed"])
    assert _text(FastaFormatter, _driver_hitlist(fx), tmp_path) == fx["fasta_text"]
    assert _text(SamFormatter, _driver_hitlist(fx), tmp_path) == fx["sam_text"]


@needs_reference
@pytest.mark.parametrize("name", NAMES)
def test_reference_formatters_print_driver_hits(name, tmp_path):
    R = _reference()
    fx = G.load(name)
    F = R.Formatters
    assert _text(F.DefaultFormatter, _driver_hitlist(fx), tmp_path) == "".join(t + "\n" for t in fx["txt"])
    assert _text(F.TrimmerFormatter, _driver_hitlist(fx), tmp_path) == "".join(t + "\n" for t in fx["trimmed"])
    assert _text(F.FASTA, _driver_hitlist(fx), tmp_path) == fx["fasta_text"]
    assert _text(F.SamFormatter, _driver_hitlist(fx), tmp_path) == fx["sam_text"]


def test_sam_line_of_reverse_complement_hit_mirrors_clips_and_position():
    from pypaswas_b200.hits import Hit
    q = SeqRecord("AACCGGTTAC", "read1")
    t = SeqRecord("TTGGCCAAGGTT", "adapter_RC")
    h = Hit(None, q, t, (2, 6), (3, 7))
    h.set_sequence_match("CCG-GT")
    h.set_alignment("||| ||")
    h.set_target_match("CCGAGT")
    h.set_scores(4.0, 5, 0)
    fields = h.get_sam_line().split("\t")
    # FLAG 16, POS counted from the target's end, SEQ reverse-complemented,
    # CIGAR: leading clip len-end-1 (always written), runs over the reversed
    # strings, trailing clip = seq start
    assert fields[:6] == ["read1", "16", "adapter", str(12 - 7), "255", "3S2=1D3=2S"]
    assert fields[9] == "GTAACCGGTT"
    assert h.alignment == "|| |||" and h.sequence_match == "TG-GCC"  # reversed in place, as the reference does


def test_formatter_for_names_every_output_format():
    from pypaswas_b200.exceptions import InvalidOptionException
    assert formatter_for("sam") is SamFormatter and formatter_for("TXT") is DefaultFormatter
    assert formatter_for("trimmedFasta") is TrimmerFormatter and formatter_for("FASTA") is FastaFormatter
    with pytest.raises(InvalidOptionException):
        formatter_for("graphml")


def _hit_state(hl):
    def rec(h):
        d = dict(vars(h))
        d["sequence_info"] = id(d["sequence_info"])
        d["target_info"] = id(d["target_info"])
        return tuple(sorted(d.items(), key=lambda kv: kv[0]))
    return ([(k, rec(h)) for k, h in hl.hits.items()], [(k, rec(h)) for k, h in hl.real_hits.items()])


@pytest.mark.parametrize("seed", range(6))
def test_native_hit_builder_equals_the_interpreter_path(seed):
    """csrc/hitbuild.c builds the same Hit objects and HitList dicts (keys,
    order, replacement rule, filter) as the Python loop, on records whose
    start and end keys collide with different scores."""
    rng = np.random.default_rng(seed)
    queries = [SeqRecord("ACGT" * int(rng.integers(20, 40)), "q%d" % (i % 5)) for i in range(9)]
    targets = [SeqRecord("TTGCA" * int(rng.integers(10, 30)), "t%d" % (i % 4)) for i in range(7)]
    queries[2].start_position = 3
    n = 600
    hits = np.zeros(n, dtype=_native.HIT_DTYPE)
    text = []
    off = 0
    for k in range(n):
        q, t = int(rng.integers(0, 9)), int(rng.integers(0, 7))
        lq = len(queries[q].seq) - queries[q].start_position
        lt = len(targets[t].seq)
        s0 = int(rng.integers(0, 4))
        t0 = int(rng.integers(0, 4))
        ncol = int(rng.integers(2, 12))
        s1 = min(s0 + ncol - 1 + int(rng.integers(0, 2)), lq - 1)
        t1 = min(t0 + ncol - 1, lt - 1)
        hits[k] = (q, t, s0, s1, t0, t1, float(rng.integers(1, 30)), int(rng.integers(0, ncol)),
                   int(rng.integers(0, 3)), ncol, off)
        for _ in range(3):
            text.append("".join("ACGT|. -"[i] for i in rng.integers(0, 8, ncol)))
        off += 3 * ncol
    strbuf = "".join(text).encode("latin-1")
    st = G.FixtureSettings(G.load("dna_linear_0"))
    st.relative_score, st.query_identity = "0.1", "0.2"  # the filter drops some
    sw = SmithWatermanB200.__new__(SmithWatermanB200)
    sw.logger, sw.settings = None, st
    native, python = HitList(None), HitList(None)
    sw._build_hits(hits, strbuf, queries, targets, native)
    sp = np.array([r.start_position for r in queries], np.int64)
    tp = np.zeros(len(targets), np.int64)
    ql = np.array([r.original_length for r in queries], np.int64)
    tl = np.array([r.original_length for r in targets], np.int64)
    sw._build_hits_python(hits, strbuf, queries, targets, python, sp, tp, ql, tl)
    assert 0 < len(native.real_hits) < n
    assert _hit_state(native) == _hit_state(python)


@pytest.mark.parametrize("name", NAMES)
def test_native_sam_writes_the_reference_file(name):
    """pw_sam_records on the engine records of each fixture writes the SAM
    file the reference wrote (SamFormatter over the reference's HitList)."""
    from pypaswas_b200.formatters import sam_records
    fx = G.load(name)
    hits, strbuf, queries, targets = _engine_records(fx)
    assert sam_records(hits, strbuf, queries, targets, G.FixtureSettings(fx)) == fx["sam_text"]
