"""Generates the golden fixtures in tests/golden/*.json from the REFERENCE itself.

Run in a container that has the read-only reference tree (default
/root/reference, override with PASWAS_REFERENCE_ROOT):

    python tests/golden/make_golden.py

Each fixture is produced by the reference's own code: its CUDA kernels
(pyPaSWAS/Core/cuda/default_main.cu, template-expanded by its own PaSWAS.py and
compiled for the CPU by oracle/ref/build_ref.py) driven by its unmodified
Python host code (Programs.Aligner/Trimmer.process -> SmithWaterman
.align_sequences -> _print_alignments -> Hit / HitList), see
oracle/ref/ref_driver.py for the stand-ins it needs (Bio.Seq, pycuda, NumPy 2).

A fixture records the inputs exactly as the program received them (after the
CLI's reverse-complement and length sort), the settings, the scoring matrix and
highest_score the reference built, and its results: the HitList in insertion
order, the TXT formatter line of every hit, the trimmedFasta lines, the whole
FASTA and SAM files the reference's formatters write, and the raw device results of each
batch (pair maxima, starting points in emission order).  The test-suite uses
them to pin the oracle and the engine; nothing at test time reads the
reference tree.
"""
import io
import json
import logging
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle", "ref"))
import ref_driver as R  # noqa: E402

LOG = logging.getLogger("golden")
LOG.setLevel(logging.WARNING)


def read_genbank(path):
    """(id, sequence) from a single-record GenBank file: VERSION and ORIGIN."""
    rid, seq, in_origin = None, [], False
    with open(path) as f:
        for line in f:
            if line.startswith("VERSION"):
                rid = line.split()[1]
            elif line.startswith("ORIGIN"):
                in_origin = True
            elif line.startswith("//"):
                in_origin = False
            elif in_origin:
                seq.extend(line.split()[1:])
    return rid, "".join(seq)


def prepare(queries, targets, dna):
    """CLI preparation: targets get reverse complements for DNA-RNA scores
    (pypaswasall.py:108-124), both lists are sorted by length, longest first."""
    q = R.make_records(queries)
    t = R.make_records(targets)
    if dna:
        t = t + [R.SWSeqRecord(R._Seq(str(r.seq.reverse_complement())), identifier=r.id + "_RC") for r in t]
    q.sort(key=lambda r: len(r.seq), reverse=True)
    t.sort(key=lambda r: len(r.seq), reverse=True)
    return q, t


def hit_record(h):
    return {"seq_id": h.get_seq_id(), "target_id": h.get_target_id(),
            "seq_location": list(h.seq_location), "target_location": list(h.target_location),
            "score": h.score, "matches": h.matches, "mismatches": h.mismatches,
            "sequence_match": h.sequence_match, "alignment": h.alignment, "target_match": h.target_match,
            "relative_score": h.relative_score, "query_identity": h.query_identity,
            "query_coverage": h.query_coverage, "base_score": h.base_score}


def txt_lines(hitlist):
    f = R.Formatters.DefaultFormatter(LOG, hitlist, os.devnull)
    return [f._format_hit(h) for h in f._get_hits()]


def trimmed_lines(hitlist):
    """Record lines of the trimmedFasta output (Formatters.TrimmerFormatter,
    Hit.get_trimmed_line), in the formatter's hit order."""
    f = R.Formatters.TrimmerFormatter(LOG, hitlist, os.devnull)
    return [h.get_trimmed_line() for h in f._get_hits()]


def formatter_text(cls, hitlist):
    """The whole file a reference formatter's print_results writes."""
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "out")
        cls(LOG, hitlist, path).print_results()
        with open(path) as f:
            return f.read()


def run_case(name, queries, targets, settings, dna, program="aligner", device_memory=8 << 30):
    q, t = prepare(queries, targets, dna)
    st = R.Settings(**settings)
    out = {"name": name, "program": program, "settings": settings, "device_memory": device_memory,
           "queries": [[r.id, str(r.seq)] for r in q], "targets": [[r.id, str(r.seq)] for r in t]}
    try:
        hl, sw = R.run_reference(q, t, st, program=program, device_memory=device_memory, logger=LOG)
    except R.CudaException as exc:
        out["exception"] = {"type": "CudaException", "message": str(exc)}
        return out
    score = sw.score
    out["matrix"] = [[float(v) for v in row] for row in score.matrix]
    out["char_offset"] = ord(score.char_offset)
    out["highest_score"] = float(score.highest_score)
    out["hits"] = [hit_record(h) for h in hl.real_hits.values()]
    out["txt"] = txt_lines(hl)
    out["trimmed"] = trimmed_lines(hl)
    out["fasta_text"] = formatter_text(R.Formatters.FASTA, hl)
    # last: get_sam_line reverses the alignment strings of RC hits in place
    out["sam_text"] = formatter_text(R.Formatters.SamFormatter, hl)
    out["batches"] = []
    for b in sw.raw_batches:
        out["batches"].append({"X": b["X"], "Y": b["Y"], "n_seq": b["n_seq"], "n_tgt": b["n_tgt"],
                               "pair_max": b["pair_max"].tolist(), "starts_u32": b["starts_u32"].tolist(),
                               "starts_f32": b["starts_f32"].tolist()})
    # batch offsets: the order of align_sequences calls (targets outer, queries inner)
    out["batch_offsets"] = sw.batch_offsets
    return out


def random_dna_case(rng, n_q, n_t, affine, qlen=(20, 120), tlen=(10, 60), alphabet="ACGT"):
    def rs(n):
        return "".join(rng.choice(list(alphabet), n))
    adapters = [rs(int(rng.integers(*tlen))) for _ in range(n_t)]
    reads = []
    for i in range(n_q):
        s = rs(int(rng.integers(*qlen)))
        if rng.random() < 0.6:
            a = list(adapters[int(rng.integers(0, n_t))])
            for j in range(len(a)):
                if rng.random() < 0.08:
                    a[j] = rng.choice(list(alphabet))
            if rng.random() < 0.3 and len(a) > 2:
                del a[int(rng.integers(0, len(a)))]
            p = int(rng.integers(0, len(s) + 1))
            s = s[:p] + "".join(a) + s[p:]
        reads.append(("read%d" % i, s))
    return reads, [("adapter%d" % i, a) for i, a in enumerate(adapters)]


def random_protein_case(rng, n_q, n_t, qlen=(30, 160), tlen=(20, 120)):
    alphabet = "ARNDCQEGHILKMFPSTWYV"

    def rs(n):
        return "".join(rng.choice(list(alphabet), n))
    domain = rs(40)
    qs, ts = [], []
    for i in range(n_q):
        s = rs(int(rng.integers(*qlen)))
        if rng.random() < 0.5:
            p = int(rng.integers(0, len(s) + 1))
            s = s[:p] + domain + s[p:]
        qs.append(("prot_q%d" % i, s))
    for i in range(n_t):
        s = rs(int(rng.integers(*tlen)))
        if rng.random() < 0.5:
            d = list(domain)
            for j in range(len(d)):
                if rng.random() < 0.4:
                    d[j] = rng.choice(list(alphabet))
            p = int(rng.integers(0, len(s) + 1))
            s = s[:p] + "".join(d) + s[p:]
        ts.append(("prot_t%d" % i, s))
    return qs, ts


RELAXED = dict(relative_score="0", base_score="0", query_identity="0", query_coverage="0")


def cases():
    rng = np.random.default_rng(20240101)
    out = []
    data = os.path.join(R.REFERENCE_ROOT, "pyPaSWAS", "Core", "test", "data")
    # the reference's own end-to-end golden test (test_pypaswasall.py:65-86)
    gq, gt = read_genbank(os.path.join(data, "query_genbank.gb")), read_genbank(os.path.join(data, "target_genbank.gb"))
    case = run_case("genbank_basic", [gq], [gt],
                    dict(match_score="1", mismatch_score="-3", gap_score="-5", any_score="1", **RELAXED), True)
    # the numbers of the reference's committed expected output
    # (test/data/reference/aligner_basic_genbank_output.txt, first line)
    with open(os.path.join(data, "reference", "aligner_basic_genbank_output.txt")) as f:
        case["reference_expected_fields"] = [v.strip() for v in f.readline().split(",")]
    out.append(case)
    for k in range(4):
        q, t = random_dna_case(rng, 12, 4, False)
        out.append(run_case("dna_linear_%d" % k, q, t,
                            dict(match_score="1", mismatch_score="-3", gap_score="-5", any_score="1",
                                 minimum_score=str([8, 10, 12, 6][k]), lower_limit_score=["1.0", "0.8", "0.5", "1.0"][k],
                                 filter_factor=["0.2", "0.1", "0.2", "0.0"][k], **RELAXED), True))
    for k in range(3):
        q, t = random_dna_case(rng, 10, 4, True)
        out.append(run_case("dna_affine_%d" % k, q, t,
                            dict(match_score="1", mismatch_score="-3", gap_score="-5", gap_extension="-1",
                                 any_score="1", minimum_score=str([8, 6, 10][k]),
                                 lower_limit_score=["1.0", "0.5", "0.9"][k], **RELAXED), True))
    q, t = random_dna_case(rng, 10, 3, False, alphabet="ACGTNKMRYSW")
    out.append(run_case("dna_ambiguity_codes", q, t,
                        dict(match_score="1", mismatch_score="-3", gap_score="-5", any_score="1", other_score="-1",
                             minimum_score="6", **RELAXED), True))
    for k in range(2):
        q, t = random_protein_case(rng, 8, 6)
        out.append(run_case("protein_affine_%d" % k, q, t,
                            dict(matrix_name="BLOSUM62", gap_score="-11", gap_extension="-1",
                                 minimum_score=str([30, 20][k]), lower_limit_score=["1.0", "0.7"][k], **RELAXED),
                            False))
    q, t = random_protein_case(rng, 8, 6)
    out.append(run_case("protein_linear_blosum80", q, t,
                        dict(matrix_name="BLOSUM80", gap_score="-5", minimum_score="25", **RELAXED), False))
    # the reference's batching: a small device memory forces several query
    # batches and target blocks (SmithWaterman.py:202-221,420-432)
    q, t = random_dna_case(rng, 24, 5, False)
    out.append(run_case("dna_multi_batch", q, t,
                        dict(match_score="1", mismatch_score="-3", gap_score="-5", any_score="1", minimum_score="8",
                             **RELAXED), True, device_memory=400000))
    # trimmer program (Programs.py:95-120)
    q, t = random_dna_case(rng, 16, 3, False, qlen=(40, 80), tlen=(12, 30))
    out.append(run_case("dna_trimmer", q, t,
                        dict(match_score="1", mismatch_score="-3", gap_score="-5", any_score="1", minimum_score="8",
                             program="trimmer", **RELAXED), True, program="trimmer"))
    # self alignment: records with equal ids are skipped (SmithWaterman.py:752-755)
    q, _ = random_dna_case(rng, 6, 2, False)
    out.append(run_case("dna_self_alignment", q, list(q),
                        dict(match_score="1", mismatch_score="-3", gap_score="-5", any_score="1", minimum_score="10",
                             **RELAXED), False))
    # a one-column alignment makes the reference raise CudaException
    # (Hit.py:64-66): a lone W-W match (11) between C-D mismatches (-3)
    out.append(run_case("one_column_hit_raises", [("q", "CCCCWCCCC")], [("t", "DDDWDDD")],
                        dict(matrix_name="BLOSUM62", gap_score="-11", minimum_score="10", filter_factor="0.0",
                             **RELAXED), False))
    return out


def main():
    for case in cases():
        path = os.path.join(HERE, case["name"] + ".json")
        with open(path, "w") as f:
            json.dump(case, f, indent=None, separators=(",", ":"))
        n = len(case.get("hits", []))
        print("%-28s hits=%-4d batches=%-3d %s" % (case["name"], n, len(case.get("batches", [])),
                                                  case.get("exception", {}).get("type", "")))


if __name__ == "__main__":
    main()
