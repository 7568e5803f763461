"""The benchmark configurations on the GPU.

Samples of each configuration are checked bit-exact against the oracle (pair
maxima, every hit, and for the trimmer the trimmedFasta text).  At full size,
where the oracle would take hours, the checks are properties that need no
oracle: the 16-bit dual-pair sweep and the 32-bit sweep give the same pair
maxima, and the batched and plain forms give the same hits."""
import numpy as np
import pytest

import cases
from engine_helpers import run_engine
from pypaswas_b200 import scores, workloads
from pypaswas_b200.formatters import DefaultFormatter, TrimmerFormatter
from pypaswas_b200.hits import Hit, HitList
from pypaswas_b200.programs import Aligner, Trimmer
from pypaswas_b200.records import SeqRecord

pytestmark = pytest.mark.gpu


def _spread(items, n):
    return items[::max(1, len(items) // n)][:n]


def _oracle(oracle_mod, q, t, score, st):
    pos = cases.pos_scores(score, st, q, t)
    return oracle_mod.run(cases.oracle_params(oracle_mod, score), q, t, pos, float(st.minimum_score))


def _bit_exact(engine_lib, oracle_mod, queries, targets, settings):
    q = [s.decode() for _, s in queries]
    t = [s.decode() for _, s in targets]
    score = scores.make_score(settings)
    o = _oracle(oracle_mod, q, t, score, settings)
    pm, hits, info, launches = run_engine(engine_lib, q, t, score, settings)
    assert launches > 0
    np.testing.assert_array_equal(pm, o["pair_max"])
    assert hits == o["hits"]
    return o


def test_config1_sample_bit_exact(engine_lib, oracle_mod):
    w = workloads.config1()
    o = _bit_exact(engine_lib, oracle_mod, _spread(w.queries, 120), w.targets, w.settings)
    assert len(o["hits"]) > 10


def test_config1_aligner_native_txt_matches_the_formatter(engine_lib):
    """Aligner.txt (engine records -> TXT bytes natively) equals
    DefaultFormatter over Aligner.process's HitList."""
    w = workloads.config1()
    qrec = [SeqRecord(s.decode(), i) for i, s in _spread(w.queries, 120)]
    trec = [SeqRecord(s.decode(), i) for i, s in w.targets]
    prog = Aligner(None, None, w.settings)
    try:
        want = "".join(line + "\n" for line in DefaultFormatter(None, prog.process(qrec, trec, None), None).lines())
        got = prog.txt(qrec, trec)
    finally:
        prog.smith_waterman.close()
    assert len(want) > 1000
    assert got == want


def test_config2_sample_bit_exact(engine_lib, oracle_mod):
    w = workloads.config2()
    o = _bit_exact(engine_lib, oracle_mod, _spread(w.queries, 8), _spread(w.targets, 48), w.settings)
    assert len(o["hits"]) > 0


def _c4_sample(n_reads):
    w = workloads.config4(n_reads=n_reads)
    reads = [(w.read_ids[i], w.reads[i].tobytes()) for i in range(n_reads)]
    return w, reads


def test_config4_sample_bit_exact_with_trimmed_fasta(engine_lib, oracle_mod):
    w, reads = _c4_sample(400)
    o = _bit_exact(engine_lib, oracle_mod, reads, w.targets, w.settings)
    assert len(o["hits"]) > 50
    # the trimmer program's output against the oracle's hits put through the
    # same HitList and formatter
    qrec = [SeqRecord(s.decode(), i) for i, s in reads]
    trec = [SeqRecord(s.decode(), i) for i, s in w.targets]
    prog = Trimmer(None, None, w.settings)
    try:
        got = TrimmerFormatter(None, prog.process(qrec, trec, None), None).lines()
    finally:
        prog.smith_waterman.close()
    hl = HitList(None)
    for h in o["hits"]:
        hit = Hit(None, qrec[h["query"]], trec[h["target"]], (h["s_start"], h["s_end"]), (h["t_start"], h["t_end"]))
        hit.set_sequence_match(h["sequence_match"])
        hit.set_alignment(h["alignment"])
        hit.set_target_match(h["target_match"])
        hit.set_scores(h["score"], h["matches"], h["mismatches"])
        if prog.smith_waterman._filter_hit(hit):
            hl.append(hit)
    assert got == TrimmerFormatter(None, hl, None).lines()
    assert len(got) > 50
    # the native output path (engine records -> trimmedFasta bytes, no Hit objects)
    prog2 = Trimmer(None, None, w.settings)
    try:
        text = prog2.trimmed_fasta(qrec, trec)
    finally:
        prog2.smith_waterman.close()
    assert text == "".join(line + "\n" for line in got)


@pytest.mark.parametrize("config", [1, 2])
def test_full_size_sixteen_and_thirty_two_bit_sweeps_agree(engine_lib, config):
    w = workloads.config1() if config == 1 else workloads.config2()
    score = scores.make_score(w.settings)
    q = [s.decode() for _, s in w.queries]
    t = [s.decode() for _, s in w.targets]
    pm16, _, info16, _ = run_engine(engine_lib, q, t, score, w.settings, score_only=True)
    pm32, _, info32, _ = run_engine(engine_lib, q, t, score, w.settings, score_only=True, int32=True)
    assert info16.score_launches > 0 and info32.score_launches > 0
    np.testing.assert_array_equal(pm16, pm32)
    assert np.all(pm16 >= 0)


def test_config4_one_million_reads_sweeps_agree(engine_lib):
    w = workloads.config4(n_reads=1_000_000)
    score = scores.make_score(w.settings)
    q = [w.reads[i].tobytes().decode() for i in range(len(w.read_ids))]
    t = [s.decode() for _, s in w.targets]
    pm16, _, _, _ = run_engine(engine_lib, q, t, score, w.settings, score_only=True)
    pm32, _, _, _ = run_engine(engine_lib, q, t, score, w.settings, score_only=True, int32=True)
    np.testing.assert_array_equal(pm16, pm32)


def test_plain_and_batched_forms_agree_on_config1_sample(engine_lib):
    w = workloads.config1()
    score = scores.make_score(w.settings)
    q = [s.decode() for _, s in _spread(w.queries, 20)]
    t = [s.decode() for _, s in w.targets]
    pm_b, hits_b, info_b, _ = run_engine(engine_lib, q, t, score, w.settings)
    pm_p, hits_p, info_p, _ = run_engine(engine_lib, q, t, score, w.settings, plain=True)
    np.testing.assert_array_equal(pm_b, pm_p)
    assert hits_b == hits_p
    assert info_p.kernel_launches >= len(q) * len(t)


def test_config3_sample_pairs_bit_exact_and_driver_agrees(engine_lib, oracle_mod):
    """Long DNA pairs (scaled down) with their reverse-complement targets:
    explicit pairs through the engine against the oracle pair by pair, and
    the driver run once per query (as the reference is run per pair) giving
    the same hits."""
    from engine_helpers import configure, decode_hits
    from pypaswas_b200 import _native
    from pypaswas_b200.programs import Aligner
    w = workloads.config3(n_pairs=3, length=(2500, 4000), shared=(800, 2000))
    score = scores.make_score(w.settings)
    q = [s.decode() for _, s in w.queries]
    t = [s.decode() for _, s in w.targets]
    ref = {}
    p = cases.oracle_params(oracle_mod, score)
    for qi, ti in w.pairs:
        o = oracle_mod.run(p, [q[qi]], [t[ti]], cases.pos_scores(score, w.settings, [q[qi]], [t[ti]]),
                           float(w.settings.minimum_score))
        ref[(qi, ti)] = [dict(h, query=qi, target=ti) for h in o["hits"]]
    e = _native.Engine(0, lib=engine_lib)
    try:
        configure(e, score, w.settings)
        e.set_queries([s.encode() for s in q], np.arange(len(q)))
        e.set_targets([s.encode() for s in t], np.arange(len(t)) + len(q))
        e.set_pairs([a for a, _ in w.pairs], [b for _, b in w.pairs])
        info = e.align()
        got = decode_hits(*e.hits())
    finally:
        e.close()
    assert info.score_path == 2
    by_pair = {}
    for h in got:
        by_pair.setdefault((h["query"], h["target"]), []).append(h)
    assert by_pair == {k: v for k, v in ref.items() if v}
    assert all(ref[(i, i)] for i in range(3))  # every planted pair is found
    # the driver, once per query against its forward and reverse-complement target
    qrec = [SeqRecord(s, i) for i, s in zip([i for i, _ in w.queries], q)]
    trec = [SeqRecord(s, i) for i, s in zip([i for i, _ in w.targets], t)]
    for qi in range(3):
        prog = Aligner(None, None, w.settings)
        try:
            hl = prog.process([qrec[qi]], [trec[qi], trec[qi + 3]], None)
        finally:
            prog.smith_waterman.close()
        assert prog.smith_waterman.last_info.score_path == 2
        got_d = sorted((h.target_info.id, h.seq_location, h.target_location, h.score, h.sequence_match)
                       for h in hl.real_hits.values())
        want = sorted((trec[r["target"]].id, (r["s_start"], r["s_end"]), (r["t_start"], r["t_end"]), r["score"],
                       r["sequence_match"]) for r in ref[(qi, qi)] + ref[(qi, qi + 3)])
        assert got_d == want
    # all pairs in one call through the public pairs API
    prog = Aligner(None, None, w.settings)
    try:
        hl = prog.process_pairs(qrec, trec, w.pairs)
    finally:
        prog.smith_waterman.close()
    got_p = sorted((h.sequence_info.id, h.target_info.id, h.seq_location, h.target_location, h.score,
                    h.sequence_match, h.alignment, h.target_match) for h in hl.real_hits.values())
    want_p = sorted((qrec[r["query"]].id, trec[r["target"]].id, (r["s_start"], r["s_end"]), (r["t_start"], r["t_end"]),
                     r["score"], r["sequence_match"], r["alignment"], r["target_match"])
                    for v in ref.values() for r in v)
    assert got_p == want_p
