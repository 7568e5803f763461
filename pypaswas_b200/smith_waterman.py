"""SmithWatermanB200: the pyPaSWAS driver interface on the B200 engine.

Public interface of pyPaSWAS/Core/SmithWaterman.py:
  set_total_work_size(size)                                  (:434-439)
  set_targets(targets, target_index, max_length=None,
              records_seqs=None, use_all_records_seqs=True) -> next index  (:370-414)
  align_sequences(records_seqs, targets, target_index) -> HitList         (:441-560)
  _filter_hit(hit)                                           (:843-848)

The reference splits the work into memory-sized batches, pads every sequence
with '\\0' to a multiple of 8 and launches one kernel per block anti-diagonal.
Here one call hands all queries and the whole target block to the engine,
which batches internally (length-binned work items, memory waves) and returns
the hits in the order the reference's walk produces them.  Hit and HitList
objects are built exactly as SmithWaterman._print_alignments builds them
(:822-838).

Queries are aligned in full.  (The reference truncates a query that is longer
than the first query of its batch, SWSeq.extentToFillGPU, which only happens
when callers pass records that are not sorted by length; its CLI always
sorts.)
"""
import logging
import math
import time

import numpy as np

from . import _native, scores
from .exceptions import InvalidOptionException
from .hits import Hit, HitList


def id_keys(query_ids, target_ids):
    """Integer keys per record, equal exactly when the ids are equal."""
    table = {}
    qk = np.array([table.setdefault(i, len(table)) for i in query_ids], dtype=np.int32)
    tk = np.array([table.setdefault(i, len(table)) for i in target_ids], dtype=np.int32)
    return qk, tk


def packed_id_keys(queries, targets):
    """id_keys of two packed record sets (pypaswas_b200.readers.RecordSet),
    without Python strings: the dense byte-order ranks of all ids together
    (pw_id_ranks) are equal exactly when the id bytes are, i.e. when the ids
    are (their UTF-8 / surrogate-escape decoding is one to one)."""
    from .formatters import _native_ranks
    blob = np.concatenate([queries.id_blob, targets.id_blob])
    off = np.concatenate([queries.id_offsets, targets.id_offsets[1:] + queries.id_offsets[-1]])
    r = _native_ranks(blob, off)
    return r[:len(queries)].astype(np.int32), r[len(queries):].astype(np.int32)


def configure_engine(engine, score, settings):
    """Scoring model and thresholds as the reference's kernels see them.
    `score` is any scoring model with the reference Score's public attributes:
    one of pypaswas_b200.scores, or the reference's own pyPaSWAS.Core.Scores
    object that pypaswasall.py:126-144 builds."""
    gap, ext, affine, ll, mn = scores.kernel_constants(score)
    engine.set_scoring(scores.matrix_array(score), scores.char_offset_code(score), gap, ext, affine, ll, mn,
                       float(settings.minimum_score), scores.highest_score(score), float(_filter_factor(settings)))


def _filter_factor(settings):
    ff = getattr(settings, "filter_factor", None)
    try:
        return float(ff) if ff else 0.7  # SmithWaterman.py:167,309-315
    except ValueError:
        raise InvalidOptionException("Filterfactor should be a float but is {0}".format(ff))


def _packed(records):
    """(residues uint8, offsets int64) of the records' upper-cased sequences.
    ASCII text goes as it is (the engine upper-cases ASCII letters in its own
    copy); other text is upper-cased here, per record where a character's
    upper case is longer."""
    seqs = [r.seq if isinstance(r.seq, str) else str(r.seq) for r in records]
    lens = np.fromiter(map(len, seqs), dtype=np.int64, count=len(seqs))
    off = np.zeros(len(seqs) + 1, dtype=np.int64)
    np.cumsum(lens, out=off[1:])
    text = "".join(seqs)
    if text.isascii():
        data = text.encode("ascii")
        return np.frombuffer(data, dtype=np.uint8) if data else np.zeros(0, np.uint8), off
    seqs = [str(s) for s in seqs]
    text = text.upper()
    if len(text) != off[-1]:  # a character whose upper case is longer: per record
        text = "".join(s.upper() for s in seqs)
        lens = np.fromiter((len(s.upper()) for s in seqs), dtype=np.int64, count=len(seqs))
        np.cumsum(lens, out=off[1:])
    data = text.encode("latin-1")
    return np.frombuffer(data, dtype=np.uint8) if data else np.zeros(0, np.uint8), off


def _hitbuild():
    """The native Hit builder (pypaswas_b200/_hitbuild*.so, csrc/hitbuild.c)."""
    try:
        from . import _hitbuild as mod
    except ImportError as exc:
        raise ImportError("pypaswas_b200._hitbuild is not built: run python -m pypaswas_b200.build") from exc
    return mod


def _logs_hits(hit_list):
    """HitList.append logs every added (INFO) and rejected (DEBUG) hit; the
    native builder is used only when neither record would be emitted."""
    lg = hit_list.logger
    if lg is None:
        return False
    enabled = getattr(lg, "isEnabledFor", None)
    return enabled is None or enabled(logging.INFO) or enabled(logging.DEBUG)


class SmithWatermanB200(object):
    """Drop-in for SmithWatermanCuda: same constructor and driver methods."""

    def __init__(self, logger, score, settings, device=None):
        self.logger = logger or logging.getLogger("pypaswas_b200")
        self.score = score
        self.settings = settings
        self.device = int(device if device is not None else (getattr(settings, "device_number", 0) or 0))
        self.filter_factor = _filter_factor(settings)
        try:
            self.mem_fill_factor = float(getattr(settings, "maximum_memory_usage", 0.8))
        except ValueError:
            raise InvalidOptionException("maximux_memory_usage is not a float")
        if self.mem_fill_factor > 1.0 or self.mem_fill_factor <= 0.0:
            raise InvalidOptionException("maximux_memory_usage is not a float between 0.0 and 1.0")
        self.gap_extension = score.gap_extension is not None
        self.engine = _native.Engine(self.device)
        configure_engine(self.engine, score, settings)
        self.number_of_targets = 0
        self.number_targets = 0
        self.total_work_size = 0
        self.total_processed = 0
        self.start_time = time.time()
        self.maximum_number_starting_points = 100  # per pair, SmithWaterman.py:144
        self.last_info = None
        self.last_h2d_bytes = 0
        self.last_d2h_bytes = 0
        self.last_timing = {}

    def set_total_work_size(self, size):
        self.total_work_size = size
        self.total_processed = 0
        self.start_time = time.time()

    def set_targets(self, targets, target_index, max_length=None, records_seqs=None, use_all_records_seqs=True):
        """Selects the next block of targets; the engine takes all remaining ones."""
        self.number_of_targets = len(targets) - target_index
        self.number_targets = self.number_of_targets
        self._block = (targets, target_index)
        return target_index + self.number_of_targets

    def _upload(self, records_seqs, targets, target_index):
        """Hands the records to the engine (copy_sequences, SmithWatermanCuda.py:176-184):
        upper-cased residues of each list concatenated, with offsets and id
        keys.  The device copy happens in the engine's next pw_align.
        Returns the target block."""
        block = targets[target_index:target_index + self.number_targets]
        qkeys, tkeys = id_keys([r.id for r in records_seqs], [r.id for r in block])
        self.engine.set_queries_packed(*_packed(records_seqs), qkeys)
        self.engine.set_targets_packed(*_packed(block), tkeys)
        return block

    def align_sequences(self, records_seqs, targets, target_index):
        """Aligns every record against the current target block; returns a HitList."""
        hitlist = HitList(self.logger)
        if self.number_targets <= 0:
            self.set_targets(targets, target_index)
        if len(records_seqs) == 0 or self.number_targets == 0:
            return hitlist
        t0 = time.time()
        block = self._upload(records_seqs, targets, target_index)
        self._align_into(records_seqs, block, hitlist, len(records_seqs) * len(block), t0)
        self._progress(records_seqs, block, t0)
        return hitlist

    def align_pairs(self, records_seqs, targets, pairs):
        """Explicit (query index, target index) pairs instead of all against
        all; returns a HitList.  The same hits as running align_sequences once
        per pair (how the reference is run on pair files), in one engine call
        whose long pairs are swept band by band across the whole GPU."""
        hitlist = HitList(self.logger)
        if len(pairs) == 0:
            return hitlist
        t0 = time.time()
        self.number_targets = len(targets)
        block = self._upload(records_seqs, targets, 0)
        self.engine.set_pairs([int(p[0]) for p in pairs], [int(p[1]) for p in pairs])
        try:
            self._align_into(records_seqs, block, hitlist, len(pairs), t0)
        finally:
            self.engine.set_pairs([], [])
        return hitlist

    def _align_into(self, records_seqs, block, hitlist, n_pairs, t0):
        """One engine call on the uploaded records; its Hits into hitlist.
        last_timing holds the call's host wall time in parts (ms): records to
        the engine, the engine call with the copy of its hit records (and of
        that, pw_align alone, and pw_align's own clock), hits to Hit objects."""
        t1 = time.time()
        info = self.engine.align(start_cap=self.maximum_number_starting_points * n_pairs)
        self.last_info = info
        if info.truncated:
            self.logger.warning("Too many hits returned. Skipping the rest. Please set lower_limit_score "
                                "higher in config.")
        t_align = time.time()
        # the engine's own host copies, turned into Hit objects before its next call
        hits, strbuf = self.engine.hits_view()
        t2 = time.time()
        self.last_h2d_bytes = int(info.h2d_bytes)  # counted by the engine, copy by copy
        self.last_d2h_bytes = int(info.d2h_bytes)
        self._build_hits(hits, strbuf, records_seqs, block, hitlist)
        self.last_timing = {"records_ms": (t1 - t0) * 1e3, "engine_ms": (t2 - t1) * 1e3,
                            "engine_call_ms": (t_align - t1) * 1e3, "engine_info_total_ms": float(info.total_ms),
                            "hits_ms": (time.time() - t2) * 1e3}

    def align_records(self, records_seqs, targets, target_index):
        """align_sequences without the Python Hit objects: the engine's hit
        records of the current target block (walk order), their alignment
        strings and the block."""
        if self.number_targets <= 0:
            self.set_targets(targets, target_index)
        if len(records_seqs) == 0 or self.number_targets == 0:
            return np.zeros(0, dtype=_native.HIT_DTYPE), b"", []
        t0 = time.time()
        block = self._upload(records_seqs, targets, target_index)
        info = self.engine.align(start_cap=self.maximum_number_starting_points * len(records_seqs) * len(block))
        self.last_info = info
        if info.truncated:
            self.logger.warning("Too many hits returned. Skipping the rest. Please set lower_limit_score "
                                "higher in config.")
        hits, strbuf = self.engine.hits()
        self.last_h2d_bytes = int(info.h2d_bytes)  # counted by the engine, copy by copy
        self.last_d2h_bytes = int(info.d2h_bytes)
        self._progress(records_seqs, block, t0)
        return hits, strbuf, block

    def align_packed(self, queries, targets, strings=True):
        """One engine call on packed record sets (pypaswas_b200.readers.RecordSet):
        all queries against all targets; returns the hit records (walk order)
        and their strings (b"" with strings=False), without Python record or
        Hit objects."""
        qk, tk = packed_id_keys(queries, targets)
        self.engine.set_queries_packed(queries.residues, queries.offsets, qk)
        self.engine.set_targets_packed(targets.residues, targets.offsets, tk)
        info = self.engine.align(start_cap=self.maximum_number_starting_points * len(queries) * len(targets))
        self.last_info = info
        if info.truncated:
            self.logger.warning("Too many hits returned. Skipping the rest. Please set lower_limit_score "
                                "higher in config.")
        self.last_h2d_bytes = int(info.h2d_bytes)
        self.last_d2h_bytes = int(info.d2h_bytes)
        return self.engine.hits(strings)

    def _build_hits(self, hits, strbuf, sequences, targets, hit_list):
        """Hit objects in walk order (SmithWaterman._print_alignments :822-838).

        Locations, ratios and the filter are evaluated for all hits at once
        (float64, the same IEEE operations as the reference's Python floats);
        when every location is valid the Hit objects are filled directly,
        otherwise each Hit is built through its validating constructor, which
        raises at the first invalid one like the reference."""
        n_hits = len(hits)
        if n_hits == 0:
            return
        sp = np.array([getattr(r, "start_position", 0) for r in sequences], dtype=np.int64)
        tp = np.array([getattr(r, "start_position", 0) for r in targets], dtype=np.int64)
        qlen = np.array([r.original_length for r in sequences], dtype=np.int64)
        tlen = np.array([r.original_length for r in targets], dtype=np.int64)
        if type(hit_list) is HitList and not _logs_hits(hit_list):
            # the same objects, built in native code (csrc/hitbuild.c); None
            # means an invalid location, reported below by the checked path
            kept = _hitbuild().build(np.ascontiguousarray(hits, dtype=_native.HIT_DTYPE), strbuf,
                                     list(sequences), list(targets), [r.id for r in sequences],
                                     [r.id for r in targets], qlen, tlen, sp, tp, self._filter_thresholds(), Hit,
                                     self.logger, hit_list.hits, hit_list.real_hits)
            if kept is not None:
                return
        self._build_hits_python(hits, strbuf, sequences, targets, hit_list, sp, tp, qlen, tlen)

    def _build_hits_python(self, hits, strbuf, sequences, targets, hit_list, sp, tp, qlen, tlen):
        """_build_hits in the interpreter: HitLists of other classes, loggers
        that record every append, and inputs with an invalid location."""
        q_col, t_col = hits["query"].astype(np.int64), hits["target"].astype(np.int64)
        s0 = hits["s_start"].astype(np.int64) + sp[q_col]
        s1 = hits["s_end"].astype(np.int64) + sp[q_col]
        t0 = hits["t_start"].astype(np.int64) + tp[t_col]
        t1 = hits["t_end"].astype(np.int64) + tp[t_col]
        ql, tl = qlen[q_col], tlen[t_col]
        valid = ((0 <= s0) & (s0 < s1) & (s1 < ql) & (0 <= t0) & (t0 < t1) & (t1 < tl)).all()
        text = bytes(strbuf).decode("latin-1")
        if not valid:
            self._build_hits_checked(hits, text, sequences, targets, hit_list, s0, s1, t0, t1)
            return
        score = hits["score"].astype(np.float64)
        mt, mm = hits["matches"].astype(np.int64), hits["mismatches"].astype(np.int64)
        nc, so = hits["n_cols"].tolist(), hits["str_offset"].tolist()
        span = (s1 - s0 + 1).astype(np.float64)
        rel = score / np.minimum(ql, tl).astype(np.float64)
        ident = mt.astype(np.float64) / span
        cov = span / ql.astype(np.float64)
        base = score / hits["n_cols"].astype(np.float64)
        thr = self._filter_thresholds()
        kidx = np.nonzero((rel >= thr[0]) & (ident >= thr[1]) & (cov >= thr[2]) & (base >= thr[3]))[0]
        for qi in set(q_col[kidx].tolist()):
            if not hasattr(sequences[qi], "distance"):
                sequences[qi].distance = 0.0
        # the kept hits' columns, one list each, walked together
        cols = [c[kidx].tolist() for c in (q_col, t_col, s0, s1, t0, t1, score, mt, mm, rel, ident, cov, base,
                                            hits["n_cols"], hits["str_offset"])]
        logger = self.logger
        new = Hit.__new__
        if type(hit_list) is not HitList:
            for qi, ti, a0, a1, b0, b1, sc, m1, m2, rl, idn, cv, bs, n, o in zip(*cols):
                h = new(Hit)
                h.__dict__ = dict(
                    logger=logger, sequence_info=sequences[qi], target_info=targets[ti],
                    seq_location=(a0, a1), target_location=(b0, b1),
                    sequence_match=text[o:o + n], alignment=text[o + n:o + 2 * n],
                    target_match=text[o + 2 * n:o + 3 * n], score=sc, matches=m1, mismatches=m2,
                    query_identity=idn, query_coverage=cv, relative_score=rl, base_score=bs,
                    distance=None, rc=False)
                hit_list.append(h)
            return
        # HitList.append inlined (same keys, same replacement rule, same log
        # records): the ids come from the record lists, the keys from the arrays
        hits_d, real = hit_list.hits, hit_list.real_hits
        get = hits_d.get
        hl_log = hit_list.logger
        enabled = getattr(hl_log, "isEnabledFor", lambda level: True)
        log_info = hl_log is not None and enabled(logging.INFO)
        log_debug = hl_log is not None and enabled(logging.DEBUG)
        qid = [r.id for r in sequences]
        tid = [r.id for r in targets]
        for qi, ti, a0, a1, b0, b1, sc, m1, m2, rl, idn, cv, bs, n, o in zip(*cols):
            sid, gid = qid[qi], tid[ti]
            h = new(Hit)
            h.__dict__ = {
                "logger": logger, "sequence_info": sequences[qi], "target_info": targets[ti],
                "seq_location": (a0, a1), "target_location": (b0, b1),
                "sequence_match": text[o:o + n], "alignment": text[o + n:o + 2 * n],
                "target_match": text[o + 2 * n:o + 3 * n], "score": sc, "matches": m1, "mismatches": m2,
                "query_identity": idn, "query_coverage": cv, "relative_score": rl,
                "base_score": bs, "distance": None, "rc": False}
            k0 = (sid, gid, a0, b0)
            k1 = (sid, gid, a1, b1)
            old0, old1 = get(k0), get(k1)
            better_end = old1 is not None and old1.score < sc
            if (old0 is None and old1 is None) or better_end or (old0 is not None and old0.score < sc):
                if better_end:
                    ok = old1.keys()[2]
                    if ok in real:
                        del real[ok]
                hits_d[k0] = h
                hits_d[k1] = h
                real[k0] = h
                if log_info:
                    hl_log.info("Added hit (query ID: %s, target ID: %s) to hitlist", sid, gid)
            elif log_debug:
                hl_log.debug("Rejected hit (query ID: %s, target ID: %s) from addition to hitlist", sid, gid)

    def _build_hits_checked(self, hits, text, sequences, targets, hit_list, s0, s1, t0, t1):
        q_col, t_col = hits["query"].tolist(), hits["target"].tolist()
        s0, s1, t0, t1 = s0.tolist(), s1.tolist(), t0.tolist(), t1.tolist()
        sc = hits["score"].tolist()
        mt, mm = hits["matches"].tolist(), hits["mismatches"].tolist()
        nc, so = hits["n_cols"].tolist(), hits["str_offset"].tolist()
        for k in range(len(q_col)):
            seq_rec, tgt_rec = sequences[q_col[k]], targets[t_col[k]]
            if not hasattr(seq_rec, "distance"):
                seq_rec.distance = 0.0
            hit = Hit(self.logger, seq_rec, tgt_rec, (s0[k], s1[k]), (t0[k], t1[k]))
            n, o = nc[k], so[k]
            hit.set_sequence_match(text[o:o + n])
            hit.set_alignment(text[o + n:o + 2 * n])
            hit.set_target_match(text[o + 2 * n:o + 3 * n])
            hit.set_scores(sc[k], mt[k], mm[k])
            if self._filter_hit(hit):
                hit_list.append(hit)

    def _filter_thresholds(self):
        s = self.settings
        return (float(s.relative_score), float(s.query_identity), float(s.query_coverage), float(s.base_score))

    def _filter_hit(self, hit):
        """SmithWaterman._filter_hit (SmithWaterman.py:843-848)."""
        thr = self._filter_thresholds()
        return (hit.relative_score >= thr[0] and hit.query_identity >= thr[1] and hit.query_coverage >= thr[2]
                and hit.base_score >= thr[3])

    def _progress(self, sequences, targets, t0):
        """GCUPS progress line of SmithWaterman.py:544-557."""
        if self.total_work_size <= 0:
            return
        t1 = time.time()
        processed = sum(len(s.seq) for s in targets) * sum(len(s.seq) for s in sequences)
        self.total_processed += processed
        duration = max(t1 - t0, 1e-9)
        total = max(t1 - self.start_time, 1e-9)
        progress = self.total_processed / float(self.total_work_size)
        self.logger.info("Duration: {:5.3f} | Performance: {:5.2f} GCUPS | Avg: {:5.2f} GCUPS | Progress: {:7.3%}"
                         .format(duration, processed / 1e9 / duration, self.total_processed / 1e9 / total,
                                 progress))

    def close(self):
        self.engine.close()
