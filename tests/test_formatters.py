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


def _synthetic_trimmer_hits(seed, n=400):
    import numpy as np
    from pypaswas_b200 import _native
    from pypaswas_b200.records import SeqRecord
    rng = np.random.default_rng(seed)
    seqs = [SeqRecord("".join("acgtACGT"[i] for i in rng.integers(0, 8, int(rng.integers(40, 90)))),
                      "read%d" % (i % 7)) for i in range(12)]  # repeated ids
    seqs[3].id = "réad-ü"  # non-ASCII id
    for r in seqs[:4]:
        r.start_position = 5
    tgts = [SeqRecord("".join("ACGT"[i] for i in rng.integers(0, 4, int(rng.integers(20, 45)))),
                      "adapter%d%s" % (i // 2, "_RC" if i % 2 else "")) for i in range(6)]
    rows = []
    for _ in range(n):
        q, t = int(rng.integers(0, len(seqs))), int(rng.integers(0, len(tgts)))
        lq, lt = len(seqs[q].seq), len(tgts[t].seq)
        s0 = int(rng.integers(0, lq - 17))  # room for the start position of 5
        t0 = int(rng.integers(0, lt - 12))
        k = int(rng.integers(2, 10))
        rows.append((q, t, s0, s0 + k, t0, t0 + k, float(rng.integers(3, 12)), k))
    rows += rows[: n // 5]
    rows += [(q, t, s0, s1, t0, t1, sc + 1.0, k) for (q, t, s0, s1, t0, t1, sc, k) in rows[: n // 10]]
    hits = np.zeros(len(rows), dtype=_native.HIT_DTYPE)
    text, off = [], 0
    for i, (q, t, s0, s1, t0, t1, sc, k) in enumerate(rows):
        for name, v in (("query", q), ("target", t), ("s_start", s0), ("s_end", s1), ("t_start", t0),
                        ("t_end", t1), ("score", sc), ("matches", k // 2), ("mismatches", k - k // 2),
                        ("n_cols", k), ("str_offset", off)):
            hits[i][name] = v
        text.append("A" * k + "|" * k + "C" * k)
        off += 3 * k
    return hits, "".join(text).encode("latin-1"), seqs, tgts


def test_native_trimmed_fasta_matches_hitlist_and_formatter(engine_lib):
    """formatters.trimmed_fasta (pw_trimmed_fasta) writes exactly the bytes of
    the driver's HitList (filter, de-duplication, dict order) printed by
    TrimmerFormatter: repeated ids, _RC targets, start positions, a non-ASCII
    id, trimming coordinates past the query's end."""
    import logging
    import cases
    from pypaswas_b200.formatters import TrimmerFormatter, trimmed_fasta
    from pypaswas_b200.hits import HitList
    from pypaswas_b200.smith_waterman import SmithWatermanB200
    for seed, thr in ((1, ("0", "0", "0", "0")), (2, ("0.1", "0.3", "0.05", "0.5"))):
        hits, strbuf, seqs, tgts = _synthetic_trimmer_hits(seed)
        st = cases.Settings(relative_score=thr[0], query_identity=thr[1], query_coverage=thr[2],
                            base_score=thr[3])
        sw = SmithWatermanB200.__new__(SmithWatermanB200)
        sw.logger = logging.getLogger("test")
        sw.settings = st
        hl = HitList(sw.logger)
        sw._build_hits(hits, strbuf, seqs, tgts, hl)
        expect = "".join(line + "\n" for line in TrimmerFormatter(None, hl, None).lines())
        assert len(hl.real_hits) > 20
        assert trimmed_fasta(hits, seqs, tgts, st, lib=engine_lib) == expect


def test_native_trimmed_fasta_rejects_an_invalid_location(engine_lib):
    import pytest
    import cases
    from pypaswas_b200.exceptions import CudaException
    from pypaswas_b200.formatters import trimmed_fasta
    hits, strbuf, seqs, tgts = _synthetic_trimmer_hits(3, n=20)
    hits[5]["s_end"] = hits[5]["s_start"]  # a one-column hit: start == end
    st = cases.Settings(relative_score="0", query_identity="0", query_coverage="0", base_score="0")
    with pytest.raises(CudaException):
        trimmed_fasta(hits, seqs, tgts, st, lib=engine_lib)
    hits, strbuf, seqs, tgts = _synthetic_trimmer_hits(3, n=20)
    hits[2]["query"] = len(seqs)  # no such query record
    with pytest.raises(CudaException):
        trimmed_fasta(hits, seqs, tgts, st, lib=engine_lib)


def test_native_txt_records_match_default_formatter(engine_lib):
    """formatters.txt_records (pw_txt_records) writes exactly what
    DefaultFormatter.print_results writes for the driver's HitList, Python's
    float repr of the ratios included (fractional scores, long and short
    ratios, an exponent-form value)."""
    import logging
    import cases
    from pypaswas_b200.formatters import DefaultFormatter, txt_records
    from pypaswas_b200.hits import HitList
    from pypaswas_b200.smith_waterman import SmithWatermanB200
    for seed in (4, 5):
        hits, strbuf, seqs, tgts = _synthetic_trimmer_hits(seed)
        hits["score"] = hits["score"] + (seed - 4) * 0.25  # fractional fp32 scores
        hits["score"][0] = 1e-5  # a ratio printed in exponent form
        st = cases.Settings(relative_score="0", query_identity="0", query_coverage="0", base_score="0")
        sw = SmithWatermanB200.__new__(SmithWatermanB200)
        sw.logger = logging.getLogger("test")
        sw.settings = st
        hl = HitList(sw.logger)
        sw._build_hits(hits, strbuf, seqs, tgts, hl)
        expect = "".join(line + "\n" for line in DefaultFormatter(None, hl, None).lines())
        assert len(hl.real_hits) > 20
        assert txt_records(hits, strbuf, seqs, tgts, st, lib=engine_lib) == expect


def test_native_txt_float_repr_over_many_magnitudes(engine_lib):
    """The scores and ratios of the TXT records printed natively equal
    Python's repr across fp32 magnitudes from 1e-38 to 1e38 (the exponent
    and fixed forms, the boundaries at 1e-4 and 1e16)."""
    import logging
    import numpy as np
    import cases
    from pypaswas_b200.formatters import DefaultFormatter, txt_records
    from pypaswas_b200.hits import HitList
    from pypaswas_b200.smith_waterman import SmithWatermanB200
    hits, strbuf, seqs, tgts = _synthetic_trimmer_hits(6, n=300)
    rng = np.random.default_rng(6)
    special = [0.0, 1e-4, 9.999e-5, 1e-5, 1e15, 1e16, 1e17, 0.1, 0.5, 1.0, 2.0 ** 24, 3.4e38, 1.2e-38, 123456.78]
    vals = np.concatenate([special, 10.0 ** rng.uniform(-38, 38, len(hits) - len(special))]).astype(np.float32)
    hits["score"] = vals[: len(hits)]
    st = cases.Settings(relative_score="0", query_identity="0", query_coverage="0", base_score="0")
    sw = SmithWatermanB200.__new__(SmithWatermanB200)
    sw.logger = logging.getLogger("test")
    sw.settings = st
    hl = HitList(sw.logger)
    sw._build_hits(hits, strbuf, seqs, tgts, hl)
    expect = "".join(line + "\n" for line in DefaultFormatter(None, hl, None).lines())
    assert len(hl.real_hits) > 100
    assert txt_records(hits, strbuf, seqs, tgts, st, lib=engine_lib) == expect


def test_native_formatter_retries_with_the_exact_size(engine_lib, monkeypatch):
    """A short output estimate costs a second call, not a wrong result."""
    import cases
    from pypaswas_b200 import formatters
    hits, strbuf, seqs, tgts = _synthetic_trimmer_hits(8, n=50)
    st = cases.Settings(relative_score="0", query_identity="0", query_coverage="0", base_score="0")
    full = formatters.trimmed_fasta(hits, seqs, tgts, st, lib=engine_lib)
    real = formatters._call_twice
    monkeypatch.setattr(formatters, "_call_twice", lambda fn, head, tail, estimate: real(fn, head, tail, 1))
    assert formatters.trimmed_fasta(hits, seqs, tgts, st, lib=engine_lib) == full
    assert formatters.txt_records(hits, strbuf, seqs, tgts, st, lib=engine_lib)


def test_native_formatter_sizes_first_when_the_estimate_cannot_be_allocated(engine_lib, monkeypatch):
    """An estimate the host cannot allocate turns into a size pass (null
    buffer) and one call at the exact size."""
    import cases
    import numpy as np
    from pypaswas_b200 import formatters
    hits, strbuf, seqs, tgts = _synthetic_trimmer_hits(9, n=50)
    st = cases.Settings(relative_score="0", query_identity="0", query_coverage="0", base_score="0")
    full = formatters.trimmed_fasta(hits, seqs, tgts, st, lib=engine_lib)
    real_empty, real_call, sizes = np.empty, formatters._call_twice, []

    def empty(n, dtype=None):
        sizes.append(n)
        if len(sizes) == 1:
            raise MemoryError("planted")
        return real_empty(n, dtype=dtype)

    def call(*a):  # the plant covers the formatter call alone
        monkeypatch.setattr(np, "empty", empty)
        try:
            return real_call(*a)
        finally:
            monkeypatch.setattr(np, "empty", real_empty)
    monkeypatch.setattr(formatters, "_call_twice", call)
    assert formatters.trimmed_fasta(hits, seqs, tgts, st, lib=engine_lib) == full
    assert len(sizes) == 2 and sizes[1] == len(full.encode())


def test_native_formatter_id_ranks_follow_python_order():
    """The id ranks given to the native formatters order ids as Python's
    sorted() does: mixed case, digits, non-ASCII, prefixes, whitespace, and
    integer ids."""
    import cases
    from pypaswas_b200.formatters import _record_arrays
    from pypaswas_b200.records import SeqRecord
    st = cases.Settings(relative_score="0", query_identity="0", query_coverage="0", base_score="0")
    for ids in (["b", "B", "a10", "a9", "a", "ä", "Z", "a", "é", "ab", "a b", "a\t"],
                ["r%d" % i for i in (10, 2, 33, 2, 1)], [5, 3, 10, 3, -1]):
        recs = [SeqRecord("ACGT", i) for i in ids]
        q, _, _, _ = _record_arrays(recs, recs, st, False)
        order = {v: k for k, v in enumerate(sorted(set(ids)))}
        assert q[0].tolist() == [order[v] for v in ids]


def test_native_sam_records_match_sam_formatter(engine_lib):
    """formatters.sam_records (pw_sam_records) writes exactly what
    SamFormatter.print_results writes for the driver's HitList: @SQ lines in
    the formatter's dict order (ids that strip to the same key, one without
    the suffix), RC flags and mirrored CIGARs, reverse-complemented SEQ,
    soft clips with start positions, mixed match / mismatch / gap runs, the
    float fields in Python's repr."""
    import logging
    import numpy as np
    import cases
    from pypaswas_b200.formatters import SamFormatter, sam_records
    from pypaswas_b200.hits import HitList
    from pypaswas_b200.smith_waterman import SmithWatermanB200
    for seed in (6, 7, 8):
        hits, strbuf, seqs, tgts = _synthetic_trimmer_hits(seed)
        rng = np.random.default_rng(seed)
        seqs[5].id = "read5_RC"
        seqs[6].id = "readRC"
        tgts[4].id = "adapter1zRC"  # strips to the key of adapter1_RC
        tgts[5].id = "adapter1"
        # alignment strings with runs of matches, mismatches and both gap kinds
        text = bytearray(strbuf)
        for h in hits:
            k, o = int(h["n_cols"]), int(h["str_offset"])
            kinds = rng.integers(0, 4, size=k)
            text[o:o + k] = b"".join(b"-" if c == 2 else b"ACGT"[int(rng.integers(0, 4))].to_bytes(1, "little")
                                     for c in kinds)
            text[o + k:o + 2 * k] = b"".join(b"|" if c == 0 else b"." if c == 1 else b" " for c in kinds)
            text[o + 2 * k:o + 3 * k] = b"".join(b"-" if c == 3 else b"G" for c in kinds)
        strbuf = bytes(text)
        hits["score"] = hits["score"] + (seed - 6) * 0.5
        st = cases.Settings(relative_score="0", query_identity="0", query_coverage="0", base_score="0")
        sw = SmithWatermanB200.__new__(SmithWatermanB200)
        sw.logger = logging.getLogger("test")
        sw.settings = st
        hl = HitList(sw.logger)
        sw._build_hits(hits, strbuf, seqs, tgts, hl)
        expect = "".join(line + "\n" for line in SamFormatter(None, hl, None).lines())
        assert len(hl.real_hits) > 20 and "\t16\t" in expect
        assert sam_records(hits, strbuf, seqs, tgts, st, lib=engine_lib) == expect
