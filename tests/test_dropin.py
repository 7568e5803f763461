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
