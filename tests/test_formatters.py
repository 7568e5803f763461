"""TXT and trimmedFasta output against the reference's own formatter output
(golden fixtures: Formatters.DefaultFormatter / TrimmerFormatter lines)."""
import pytest

import golden_util as G
from pypaswas_b200.formatters import DefaultFormatter, TrimmerFormatter
from pypaswas_b200.hits import Hit, HitList
from pypaswas_b200.records import SeqRecord

NAMES = [n for n in G.names() if "exception" not in G.load(n)]


def _hitlist(fx):
    seqs = {i: s for i, s in fx["queries"]}
    tgts = {i: s for i, s in fx["targets"]}
    hl = HitList(None)
    for k, h in enumerate(fx["hits"]):
        hit = Hit(None, SeqRecord(seqs[h["seq_id"]], h["seq_id"]), SeqRecord(tgts[h["target_id"]], h["target_id"]),
                  tuple(h["seq_location"]), tuple(h["target_location"]))
        hit.set_sequence_match(h["sequence_match"])
        hit.set_alignment(h["alignment"])
        hit.set_target_match(h["target_match"])
        hit.set_scores(h["score"], h["matches"], h["mismatches"])
        hl.real_hits[k] = hit  # insertion order of the reference's HitList
    return hl


@pytest.mark.parametrize("name", NAMES)
def test_txt_lines_match_reference(name):
    fx = G.load(name)
    assert DefaultFormatter(None, _hitlist(fx), None).lines() == fx["txt"]


@pytest.mark.parametrize("name", NAMES)
def test_trimmed_fasta_lines_match_reference(name):
    fx = G.load(name)
    assert TrimmerFormatter(None, _hitlist(fx), None).lines() == fx["trimmed"]


def test_trimmed_record_cuts_target_span_from_query():
    q = SeqRecord("AAAACCCCGGGG", "read7")
    t = SeqRecord("TTTTTTTTTT", "adapter3_RC")
    h = Hit(None, q, t, (2, 8), (3, 6))
    h.set_sequence_match("ACCC")
    h.set_alignment("||||")
    h.set_target_match("ACCC")
    h.set_scores(4.0, 4, 0)
    hl = HitList(None)
    hl.real_hits[0] = h
    assert TrimmerFormatter(None, hl, None).lines() == [">adapter3 read7\nAAACGGGG"]
