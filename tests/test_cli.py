"""The command-line driver (pypaswas_b200.cli), restating pypaswasall.py's
Pypaswas.run: options and defaults on the CPU; on the GPU, whole runs on the
golden fixtures' inputs written as FASTA files, whose output files must equal
the reference's (TXT, SAM, trimmedFasta), through the object path, the native
path and the chunked loop."""
import pytest

import golden_util as G
from pypaswas_b200 import cli, scores
from pypaswas_b200.exceptions import InvalidOptionException

LONG = {dest: long_ for _, long_, dest, _, _ in cli._OPTIONS}


def test_defaults_follow_the_reference_configuration():
    st, args = cli.parse_cli(["q.fa", "t.fa"])
    assert args == ["q.fa", "t.fa"]
    assert (st.gap_score, st.match_score, st.mismatch_score, st.matrix_name, st.minimum_score) == \
        ("-5", "5", "-3", "DNA-RNA", "30")
    assert (st.query_step, st.sequence_step, st.limit_length, st.out_format, st.loglevel) == \
        ("1000000", "100000000", "100000", "TXT", "DEBUG")
    with pytest.raises(InvalidOptionException):
        cli.parse_cli(["only_one.fa"])


def test_config_file_overrides_settings_it_names(tmp_path):
    cfg = tmp_path / "run.cfg"
    cfg.write_text("[Aligner]\ngap_score=-7\nhighest_score=9\n[Filter]\nbase_score=\n")
    st, _ = cli.parse_cli(["-G", "-3", "--base_score", "1.5", "-c", str(cfg), "a", "b"])
    assert st.gap_score == "-7"      # the file wins over the command line
    assert st.base_score == "1.5"    # empty values are ignored
    assert not hasattr(st, "highest_score")


def _write_fasta(path, records):
    with open(path, "w") as f:
        for i, s in records:
            f.write(">%s\n%s\n" % (i, s))


def _chunk_ids(tmp_path, argv, n_q=7, n_t=5):
    q = [("q%d" % k, "ACGT" * (k + 1)) for k in range(n_q)]
    t = [("t%d" % k, "ACG" * (k + 2)) for k in range(n_t)]
    _write_fasta(tmp_path / "q.fa", q)
    _write_fasta(tmp_path / "t.fa", t)
    p = cli.Pypaswas()
    p.settings, p.arguments = cli.parse_cli(argv + [str(tmp_path / "q.fa"), str(tmp_path / "t.fa")])
    p.score = scores.make_score(p.settings)
    return [(sorted(a.ids), sorted(b.ids)) for a, b in p._chunks()]


def test_chunk_loop_walks_query_and_target_steps(tmp_path):
    chunks = _chunk_ids(tmp_path, ["--query_step", "3", "--sequence_step", "2", "-M", "BLOSUM62"])
    # queries [0,3) [3,6) [6,9).  The target loop ends after a chunk that
    # holds no more records than its end index (pypaswasall.py:234-237): with
    # 2-record steps and no reverse complements that is the first chunk
    assert [c[0] for c in chunks] == [["q0", "q1", "q2"], ["q3", "q4", "q5"], ["q6"]]
    assert all(c[1] == ["t0", "t1"] for c in chunks)
    chunks = _chunk_ids(tmp_path, ["--query_step", "4", "--sequence_step", "4", "--start_target", "1",
                                   "--end_target", "9", "-M", "BLOSUM62"])
    # targets [1,5): 4 records <= 5, the loop ends there too
    assert chunks == [(["q0", "q1", "q2", "q3"], ["t1", "t2", "t3", "t4"]),
                      (["q4", "q5", "q6"], ["t1", "t2", "t3", "t4"])]
    # a start index without an end index: the end is clamped to 0
    # (pypaswasall.py:194-196), the slice is empty and nothing is processed
    assert _chunk_ids(tmp_path, ["--start_target", "1", "-M", "BLOSUM62"]) == []


def test_chunk_loop_with_reverse_complements_and_end_indices(tmp_path):
    chunks = _chunk_ids(tmp_path, ["--sequence_step", "2", "--start_query", "1", "--end_query", "3",
                                   "--end_target", "4"])
    # DNA targets carry their reverse complements: 4 records read per 2-record step
    assert [c[1] for c in chunks] == [["t0", "t0_RC", "t1", "t1_RC"], ["t2", "t2_RC", "t3", "t3_RC"]]
    assert all(c[0] == ["q1", "q2"] for c in chunks)


# ------------------------------------------------------------------ GPU runs
NAMES = [n for n in G.names() if "exception" not in G.load(n) and G.load(n)["hits"]]


def _inputs(tmp_path, fx):
    _write_fasta(tmp_path / "q.fa", fx["queries"])
    _write_fasta(tmp_path / "t.fa", [(i, s) for i, s in fx["targets"] if not i.endswith("_RC")])
    return [str(tmp_path / "q.fa"), str(tmp_path / "t.fa")]


def _argv(fx, out, fmt, extra=()):
    argv = []
    for k, v in fx["settings"].items():
        argv += [LONG[k], str(v)]
    if fx["program"] == "trimmer":
        argv += ["-p", "trimmer"]
    return argv + ["-o", out, "--outputformat", fmt, "--limit_length", "0"] + list(extra)


def _same(text, want, fx):
    if len(fx["batches"]) == 1:
        return text == want
    return sorted(text.split("\n")) == sorted(want.split("\n"))


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_cli_output_files_equal_the_reference(engine_lib, tmp_path, name):
    fx = G.load(name)
    files = _inputs(tmp_path, fx)
    want = {"TXT": "".join(t + "\n" for t in fx["txt"]), "SAM": fx["sam_text"],
            "trimmedFasta": "".join(t + "\n" for t in fx["trimmed"])}
    runs = [("TXT", ["--loglevel", "ERROR"], True),
            ("TXT", ["--loglevel", "INFO", "-L", str(tmp_path / "log")], False),
            ("SAM", ["--loglevel", "ERROR"], True),
            ("SAM", ["--loglevel", "INFO", "-L", str(tmp_path / "log_sam")], False),
            # query chunks of 3 records (the target chunk covers the whole file)
            ("TXT", ["--loglevel", "ERROR", "--query_step", "3"], True)]
    if fx["program"] == "trimmer":
        runs.append(("trimmedFasta", ["--loglevel", "ERROR"], True))
    for k, (fmt, extra, native) in enumerate(runs):
        out = str(tmp_path / ("out_%d" % k))
        p = cli.Pypaswas()
        p.run(_argv(fx, out, fmt, extra) + files)
        assert p.native_output == native
        with open(out) as f:
            assert _same(f.read(), want[fmt], fx), (fmt, extra)
