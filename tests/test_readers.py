"""The native FASTA / FASTQ reader (pw_records_*, pypaswas_b200/readers.py)
against the record preparation of the reference (Readers.py:30-118 with
Biopython's parsers, pypaswasall.py:98-124), on the CPU."""
import numpy as np
import pytest

from pypaswas_b200 import _native, readers, scores, workloads
from pypaswas_b200.exceptions import InvalidOptionException, ReaderException

FASTA = (b"; a comment line before the first record is skipped\n"
         b">read1 first read, description\n"
         b"acgtN\r\n"
         b"AC GT  \n"
         b"\n"
         b">read2\n"
         b"TTTT\n"
         b">\n"
         b"GGG\n"
         b">  spaced_title here\n"
         b"A\n"
         b">empty\n"
         b">long\n" + b"ACGT" * 10 + b"\n")


def _as_list(rs):
    return [(i, rs.seq(k)) for k, i in enumerate(rs.ids)]


def test_fasta_titles_sequences_and_case():
    rs = readers.read_records(FASTA, "fasta", 0, None, 0, _native.PW_RECORDS_AS_READ, False)
    assert _as_list(rs) == [("read1", "ACGTNACGT"), ("read2", "TTTT"), ("", "GGG"), ("spaced_title", "A"),
                            ("empty", ""), ("long", "ACGT" * 10)]


def test_limit_length_keeps_nonempty_records_up_to_the_limit():
    rs = readers.read_records(FASTA, "fasta", 0, None, 9, _native.PW_RECORDS_AS_READ, False)
    assert [i for i in rs.ids] == ["read1", "read2", "", "spaced_title"]
    assert rs.dropped == 2  # the empty record and the 40-long one


def test_start_end_slice_before_the_filter():
    rs = readers.read_records(FASTA, "fasta", 1, 3, 100, _native.PW_RECORDS_AS_READ, False)
    assert rs.ids == ["read2", ""]
    with pytest.raises(ReaderException):
        readers.read_records(FASTA, "fasta", 6, 9, 100, _native.PW_RECORDS_AS_READ, False)
    # a slice whose records are all filtered out is not an error (Readers.py:105-114)
    rs = readers.read_records(FASTA, "fasta", 4, 5, 100, _native.PW_RECORDS_AS_READ, False)
    assert len(rs) == 0 and rs.dropped == 1
    with pytest.raises(ReaderException):  # islice(it, 2, 1) selects nothing
        readers.read_records(FASTA, "fasta", 2, 1, 100, _native.PW_RECORDS_AS_READ, False)


def test_targets_get_reverse_complements_and_a_stable_length_sort():
    data = b">a\nACGTT\n>b\nGGC\n>c\nAAAAA\n>d\nKMRYSWN\n"
    rs = readers.read_records(data, "fasta", 0, None, 100, _native.PW_RECORDS_APPEND_RC, True)
    rc = lambda s: workloads.reverse_complement(s.encode()).decode()
    want = [("a", "ACGTT"), ("b", "GGC"), ("c", "AAAAA"), ("d", "KMRYSWN")]
    want = want + [(i + "_RC", rc(s)) for i, s in want]
    want = sorted(want, key=lambda r: len(r[1]), reverse=True)  # Python's sort: stable
    assert _as_list(rs) == want


def test_reverse_and_rc_only_transforms():
    data = b">x\nACGG\n>y\nTTA\n"
    rs = readers.read_records(data, "fasta", 0, None, 100, _native.PW_RECORDS_APPEND_REVERSED, False)
    assert _as_list(rs) == [("x", "ACGG"), ("y", "TTA"), ("x_RC", "GGCA"), ("y_RC", "ATT")]
    rs = readers.read_records(data, "fasta", 0, None, 100, _native.PW_RECORDS_RC_ONLY, False)
    assert _as_list(rs) == [("x_RC", "CCGT"), ("y_RC", "TAA")]


def test_fastq_records_multiline_and_errors():
    data = (b"@r1 desc\nACGT\nAC\n+\nIIII\nII\n"
            b"@r2\r\nggtt\r\n+r2\r\n@@@@\r\n"
            b"\n")
    rs = readers.read_records(data, "fastq", 0, None, 0, _native.PW_RECORDS_AS_READ, False)
    assert _as_list(rs) == [("r1", "ACGTAC"), ("r2", "GGTT")]
    with pytest.raises(InvalidOptionException):
        readers.read_records(b"@r\nACGT\n+\nII\n", "fastq", 0, None, 0, 0, False)
    with pytest.raises(InvalidOptionException):
        readers.read_records(b"r\nACGT\n+\nIIII\n", "fastq", 0, None, 0, 0, False)
    with pytest.raises(InvalidOptionException):
        readers.read_records(FASTA, "genbank", 0, None, 0, 0, False)


def test_files_and_the_cli_chain(tmp_path):
    p = tmp_path / "t.fa"
    p.write_bytes(b">t1\nACGTACGT\n>t2\nACG\n")
    st = workloads.Settings(limit_length="100")
    score = scores.make_score(st)
    rs = readers.read_target_records(st, score, str(p))
    assert rs.ids == ["t1", "t1_RC", "t2", "t2_RC"]
    st.matrix_name = "BLOSUM62"
    rs = readers.read_target_records(st, scores.make_score(st), str(p))
    assert rs.ids == ["t1", "t2"]
    q = readers.read_query_records(st, str(p))
    assert [r.id for r in q.records()] == ["t1", "t2"] and str(q.records()[0].seq) == "ACGTACGT"
    with pytest.raises(InvalidOptionException):
        readers.read_records(str(tmp_path / "missing.fa"))


def test_native_reader_interface_matches_the_packed_chain(tmp_path):
    rng = np.random.default_rng(3)
    lines = []
    for k in range(50):
        lines.append(">s%d x" % k)
        s = "".join("acgtACGT"[i] for i in rng.integers(0, 8, int(rng.integers(1, 40))))
        lines.append(s)
    p = tmp_path / "r.fa"
    p.write_text("\n".join(lines) + "\n")
    r = readers.NativeReader(None, str(p), "fasta", 30)
    r.read_records(5, 45)
    r.complement_records()
    r.sort_records()
    got = [(x.id, str(x.seq)) for x in r.get_records()]
    want = readers.read_records(str(p), "fasta", 5, 45, 30, _native.PW_RECORDS_APPEND_RC, True)
    assert got == _as_list(want)


def test_native_id_ranks_follow_python_string_order():
    """pw_id_ranks: dense ranks in Python's str order (ASCII ids: prefixes
    first, equal ids share a rank), across the threaded sort-and-merge."""
    from pypaswas_b200.formatters import _native_ranks
    rng = np.random.default_rng(5)
    alphabet = np.array(list("ab_Z09.-"))
    for n in (0, 1, 7, 40000):
        ids = ["".join(rng.choice(alphabet, size=int(rng.integers(0, 6)))) for _ in range(n)]
        blob = np.frombuffer("".join(ids).encode() or b"\0", dtype=np.uint8)[:sum(map(len, ids))]
        off = np.zeros(n + 1, dtype=np.int64)
        np.cumsum([len(i) for i in ids], out=off[1:])
        got = _native_ranks(blob, off)
        order = {v: k for k, v in enumerate(sorted(set(ids)))}
        assert got.tolist() == [order[v] for v in ids]


def test_parallel_fasta_pieces_equal_one_piece():
    """A FASTA input large enough to be parsed in pieces on host threads
    gives the records a sequential parse gives (pieces start at '>' lines;
    junk before the first record, blank and wrapped lines, CRLF)."""
    rng = np.random.default_rng(9)
    parts = [b"junk line\n\n"]
    want = []
    letters = np.array(list("ACGTacgtN"))
    for i in range(60000):
        seq = "".join(letters[rng.integers(0, 9, size=int(rng.integers(1, 400)))])
        wrapped = "\n".join(seq[k:k + 60] for k in range(0, len(seq), 60))
        eol = "\r\n" if i % 7 == 0 else "\n"
        parts.append((">r%d desc %d%s%s%s" % (i, i, eol, wrapped.replace("\n", eol), eol)).encode())
        if i % 11 == 0:
            parts.append(b"\n")
        want.append(("r%d" % i, seq.upper()))
    data = b"".join(parts)
    assert len(data) > (1 << 23)  # several pieces
    rs = readers.read_records(data, "fasta", 0, None, 0, _native.PW_RECORDS_AS_READ, False)
    assert len(rs) == len(want)
    assert rs.ids == [w[0] for w in want]
    assert [rs.seq(k) for k in range(len(rs))] == [w[1] for w in want]
