"""The full driver on the GPU (Aligner / Trimmer -> SmithWatermanB200 -> C ABI)
against the reference's own outputs: every field of every Hit, HitList order."""
import pytest

import golden_util as G
from pypaswas_b200.exceptions import CudaException
from pypaswas_b200.formatters import DefaultFormatter, TrimmerFormatter
from pypaswas_b200.programs import Aligner, Trimmer
from pypaswas_b200.records import SeqRecord

pytestmark = pytest.mark.gpu

FIELDS = ["seq_id", "target_id", "seq_location", "target_location", "score", "matches", "mismatches",
          "sequence_match", "alignment", "target_match", "relative_score", "query_identity", "query_coverage",
          "base_score"]


def _record(h):
    return {"seq_id": h.get_seq_id(), "target_id": h.get_target_id(), "seq_location": list(h.seq_location),
            "target_location": list(h.target_location), "score": h.score, "matches": h.matches,
            "mismatches": h.mismatches, "sequence_match": h.sequence_match, "alignment": h.alignment,
            "target_match": h.target_match, "relative_score": h.relative_score,
            "query_identity": h.query_identity, "query_coverage": h.query_coverage, "base_score": h.base_score}


@pytest.mark.parametrize("name", G.names())
def test_driver_matches_reference(engine_lib, name):
    fx = G.load(name)
    st = G.FixtureSettings(fx)
    queries = [SeqRecord(s, i) for i, s in fx["queries"]]
    targets = [SeqRecord(s, i) for i, s in fx["targets"]]
    prog = (Trimmer if fx["program"] == "trimmer" else Aligner)(None, None, st)
    try:
        if "exception" in fx:
            with pytest.raises(CudaException):
                prog.process(queries, targets, None)
            return
        hl = prog.process(queries, targets, None)
        got = [_record(h) for h in hl.real_hits.values()]
        ref = [{k: h[k] for k in FIELDS} for h in fx["hits"]]
        assert G.hits_by_pair(got) == G.hits_by_pair(ref)
        if len(fx["batches"]) == 1:
            assert got == ref
        # the program's text output, byte for byte (with several reference
        # batches, hits of equal ids and score may be listed in another order)
        txt, trimmed = DefaultFormatter(None, hl, None).lines(), TrimmerFormatter(None, hl, None).lines()
        if len(fx["batches"]) == 1:
            assert txt == fx["txt"] and trimmed == fx["trimmed"]
        else:
            assert sorted(txt) == sorted(fx["txt"]) and sorted(trimmed) == sorted(fx["trimmed"])
    finally:
        prog.smith_waterman.close()
