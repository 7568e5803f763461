"""Output formatters of the aligner and trimmer programs
(pyPaSWAS/Core/Formatters.py:3-186).

Every formatter visits HitList.real_hits sorted by (query id, target id, score)
(Formatters.py:34-37; a stable sort, so equal keys keep HitList order) and
produce the reference's text byte for byte:

* DefaultFormatter ("TXT"): one comma-separated summary line per hit followed by
  the three alignment strings (Formatters.py:19-31).
* SamFormatter ("SAM"): header lines, then Hit.get_sam_line per hit
  (Formatters.py:51-106, Hit.py:222-272,338-406).
* FastaFormatter ("FASTA"): the whole query per hit (Formatters.py:152-186).
* TrimmerFormatter ("trimmedFasta"): one FASTA record per hit, the query with
  the span [target_start, target_end] cut out (Hit.get_trimmed_line,
  pyPaSWAS/Core/Hit.py:274-286, which slices the query by the hit's TARGET
  coordinates; that is the reference's behaviour and is kept).
"""
from .exceptions import CudaException


def ordered_hits(hitlist):
    return sorted(hitlist.real_hits.values(), key=lambda h: (h.get_seq_id(), h.get_target_id(), h.score))


def txt_record(hit):
    """The DefaultFormatter record of one hit (Formatters.py:19-31)."""
    n_cols = len(hit.alignment)
    gaps = n_cols - hit.matches - hit.mismatches
    q_len = hit.sequence_info.original_length
    t_len = hit.target_info.original_length
    head = ", ".join(str(v) for v in (
        hit.get_seq_id(), hit.get_target_id(), hit.seq_location[0], hit.seq_location[1], hit.target_location[0],
        hit.target_location[1], hit.score, hit.matches, hit.mismatches, gaps, n_cols, hit.score / n_cols, q_len,
        t_len, hit.score / q_len, hit.score / t_len, hit.distance))
    return "\n".join((head, hit.sequence_match, hit.alignment, hit.target_match))


def _strip_rc(identifier):
    return identifier[:-3] if identifier[-2:] == "RC" else identifier


def trimmed_record(hit):
    """The trimmedFasta record of one hit (Hit.get_trimmed_line, Hit.py:274-286)."""
    if not hit.sequence_match or not hit.target_match or not hit.alignment:
        raise CudaException("sequence_match, target_match and alignment should be set and have lengths > 0.")
    seq = str(hit.sequence_info.seq)
    t0, t1 = hit.target_location
    return "".join((">", _strip_rc(hit.get_target_id()), " ", hit.sequence_info.id, "\n", seq[:t0], seq[t1 + 1:]))


def _is_packed(records):
    """Records given as one packed set (residues, offsets, ids; see
    pypaswas_b200.readers.RecordSet) instead of a list of record objects."""
    return hasattr(records, "id_blob") and hasattr(records, "residues")


def _record_arrays(sequences, targets, settings, strip_target_rc):
    """Per-record inputs of the native formatters: id ranks in Python's
    order, lengths, start positions, id bytes, thresholds."""
    import numpy as np

    def ranks(ids):
        # Python's order of the ids: numpy's sort agrees with it for all-str
        # ids (code points; no NUL, which fixed-width strings would drop) and
        # for all-int ids; anything else takes sorted()
        if ids and ((all(type(v) is str for v in ids) and "\0" not in "".join(ids)) or
                    all(type(v) is int for v in ids)):
            arr = np.array(ids)
            if arr.dtype.kind in "Ui" and arr.ndim == 1:
                return np.unique(arr, return_inverse=True)[1].astype(np.int32).reshape(-1)
        order = {v: k for k, v in enumerate(sorted(set(ids)))}
        return np.array([order[v] for v in ids], dtype=np.int32)

    blob = _blob

    def arrays(records, strip_rc):
        if _is_packed(records):  # packed records (pypaswas_b200.readers): no per-record objects
            if not strip_rc and _ascii(records.id_blob):
                # ASCII ids: byte order is Python's string order; ranked natively
                return (_native_ranks(records.id_blob, records.id_offsets), records.lengths.astype(np.int64),
                        np.zeros(len(records), dtype=np.int64), records.id_blob, records.id_offsets)
            ids = records.ids
            b = blob([_strip_rc(i) for i in ids]) if strip_rc else (records.id_blob, records.id_offsets)
            return (ranks(ids), records.lengths.astype(np.int64), np.zeros(len(ids), dtype=np.int64)) + tuple(b)
        ids = [r.id for r in records]
        return (ranks(ids), np.array([r.original_length for r in records], dtype=np.int64),
                np.array([getattr(r, "start_position", 0) for r in records], dtype=np.int64)) + \
            blob([_strip_rc(str(i)) if strip_rc else str(i) for i in ids])

    q = arrays(sequences, False)
    t = arrays(targets, strip_target_rc)
    thr = np.array([float(settings.relative_score), float(settings.query_identity),
                    float(settings.query_coverage), float(settings.base_score)], dtype=np.float64)
    return q, t, thr, blob


def _blob(items):
    """The UTF-8 bytes of strings concatenated, with int64 offsets."""
    import numpy as np
    text = "".join(items)
    if text.isascii():
        data = text.encode("ascii")
        lens = np.fromiter(map(len, items), dtype=np.int64, count=len(items))
    else:
        enc = [x.encode("utf-8") for x in items]
        data = b"".join(enc)
        lens = np.fromiter(map(len, enc), dtype=np.int64, count=len(enc))
    off = np.zeros(len(items) + 1, dtype=np.int64)
    np.cumsum(lens, out=off[1:])
    return np.frombuffer(data or b"\0", dtype=np.uint8), off


def _ascii(blob):
    return len(blob) == 0 or int(blob.max()) < 128


def _native_ranks(blob, offsets):
    """Dense ranks of the ids blob[offsets[i]:offsets[i + 1]] in byte order
    (pw_id_ranks): Python's string order for ASCII ids."""
    import ctypes
    import numpy as np
    from . import _native
    n = len(offsets) - 1
    out = np.zeros(max(n, 0), dtype=np.int32)
    blob = np.ascontiguousarray(blob, dtype=np.uint8)
    offsets = np.ascontiguousarray(offsets, dtype=np.int64)
    vp = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    rc = _native.load_library().pw_id_ranks(vp(blob) if len(blob) else None, vp(offsets), n, vp(out))
    if rc != _native.PW_OK:
        raise CudaException("pw_id_ranks failed (%d)" % rc)
    return out


# first output buffer at most this large; a longer text takes the exact-size
# retry (the estimate is per hit, so it is near the real size unless the score
# filter drops most hits)
_ESTIMATE_CAP = 1 << 30


def _per_hit_estimate(hits, q_id_off, t_id_off, body):
    """Bytes of the records of `hits` if none were filtered out: each hit's
    own query and target id lengths plus `body` (per hit, or a scalar), capped
    at _ESTIMATE_CAP."""
    import numpy as np
    if len(hits) == 0:
        return 1
    q_ids, t_ids = np.diff(q_id_off), np.diff(t_id_off)
    # indices outside the record lists are rejected by the native call; clip them here
    qi = np.clip(hits["query"].astype(np.int64), 0, max(len(q_ids) - 1, 0))
    ti = np.clip(hits["target"].astype(np.int64), 0, max(len(t_ids) - 1, 0))
    total = int((np.sum(q_ids[qi]) if len(q_ids) else 0) + (np.sum(t_ids[ti]) if len(t_ids) else 0)
                + np.sum(body))
    return min(total, _ESTIMATE_CAP)


def _call_twice(fn, head, tail, estimate):
    """A native formatter into a buffer of `estimate` bytes, once more with
    the exact size when the estimate was short; returns the text."""
    import ctypes
    import numpy as np
    from . import _native
    n = ctypes.c_int64()
    try:
        out = np.empty(max(int(estimate), 1), dtype=np.uint8)
        rc = fn(*head, *tail, out.ctypes.data_as(ctypes.c_void_p), len(out), ctypes.byref(n))
    except MemoryError:
        # no room for the estimate: a size pass (null buffer), then the exact size
        rc = fn(*head, *tail, None, 0, ctypes.byref(n))
        rc = _native.PW_ERR_CAPACITY if rc == _native.PW_OK else rc
    if rc == _native.PW_ERR_CAPACITY:
        out = np.empty(max(n.value, 1), dtype=np.uint8)
        rc = fn(*head, *tail, out.ctypes.data_as(ctypes.c_void_p), len(out), ctypes.byref(n))
    if rc == _native.PW_ERR_ARG:
        raise CudaException("Invalid hit location in the engine's records")
    if rc != _native.PW_OK:
        raise CudaException("native formatter failed (%d)" % rc)
    return str(memoryview(out[:n.value]), "utf-8")


def txt_records(hits, strbuf, sequences, targets, settings, lib=None):
    """The TXT text (DefaultFormatter.print_results) of engine hit records and
    their strings (Engine.hits()), built in native code (pw_txt_records)."""
    import ctypes
    import numpy as np
    from . import _native
    lib = lib if lib is not None else _native.load_library()
    hits = np.ascontiguousarray(hits, dtype=_native.HIT_DTYPE)
    q, t, thr, _ = _record_arrays(sequences, targets, settings, False)
    sb = np.frombuffer(bytes(strbuf) or b"\0", dtype=np.uint8)
    vp = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    head = (vp(hits) if len(hits) else None, len(hits), len(sequences), len(targets), vp(sb), len(strbuf))
    tail = tuple(vp(a) for a in q) + tuple(vp(a) for a in t) + (vp(thr),)
    # each hit's own record: its two ids, three strings of n_cols and the numbers
    est = _per_hit_estimate(hits, q[4], t[4], 3 * hits["n_cols"].astype(np.int64) + 220)
    return _call_twice(lib.pw_txt_records, head, tail, est)


def _query_residues(sequences, what):
    """(residues, offsets) of the queries for a native formatter; ASCII only."""
    from .exceptions import InvalidOptionException
    if _is_packed(sequences):
        q_seq, q_seq_off = sequences.residues, sequences.offsets
        if len(q_seq) and int(q_seq.max()) >= 128:
            raise InvalidOptionException("%s needs ASCII sequences" % what)
        return q_seq, q_seq_off
    qseqs = [str(r.seq) for r in sequences]
    if not "".join(qseqs).isascii():
        raise InvalidOptionException("%s needs ASCII sequences" % what)
    return _blob(qseqs)


def sam_records(hits, strbuf, sequences, targets, settings, lib=None):
    """The SAM text (SamFormatter.print_results: @HD, @SQ, @PG and one line
    per hit) of engine hit records and their strings (Engine.hits()), built
    in native code (pw_sam_records)."""
    import ctypes
    import numpy as np
    from . import _native
    lib = lib if lib is not None else _native.load_library()
    hits = np.ascontiguousarray(hits, dtype=_native.HIT_DTYPE)
    q, t, thr, _ = _record_arrays(sequences, targets, settings, False)
    q_seq, q_seq_off = _query_residues(sequences, "SAM output")
    sb = np.frombuffer(bytes(strbuf) or b"\0", dtype=np.uint8)
    vp = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    head = (vp(hits) if len(hits) else None, len(hits), len(sequences), len(targets), vp(sb), len(strbuf))
    tail = tuple(vp(a) for a in q) + (vp(q_seq), vp(q_seq_off)) + tuple(vp(a) for a in t) + (vp(thr),)
    q_len = np.diff(q_seq_off)
    qi = np.clip(hits["query"].astype(np.int64), 0, max(len(q_len) - 1, 0))
    body = (2 * hits["n_cols"].astype(np.int64) + q_len[qi] + 200) if len(hits) and len(q_len) else 0
    est = _per_hit_estimate(hits, q[4], t[4], body) + 64 * (len(targets) + 2)
    return _call_twice(lib.pw_sam_records, head, tail, est)


def trimmed_fasta(hits, sequences, targets, settings, lib=None):
    """The trimmedFasta text of engine hit records (pw_get_hits order) -- the
    bytes TrimmerFormatter(...).print_results writes for the HitList that the
    driver builds from the same records, built in native code without Hit
    objects (pw_trimmed_fasta).  `sequences` / `targets` are the records the
    engine aligned (query / target indices of the hits); sequences must be
    ASCII, as DNA, RNA and protein alphabets are."""
    import ctypes
    import numpy as np
    from . import _native
    from .exceptions import InvalidOptionException
    lib = lib if lib is not None else _native.load_library()
    hits = np.ascontiguousarray(hits, dtype=_native.HIT_DTYPE)
    q, t, thr, _ = _record_arrays(sequences, targets, settings, True)
    q_seq, q_seq_off = _query_residues(sequences, "trimmed_fasta")
    vp = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    head = (vp(hits) if len(hits) else None, len(hits), len(sequences), len(targets))
    tail = tuple(vp(a) for a in q) + (vp(q_seq), vp(q_seq_off)) + tuple(vp(a) for a in t) + (vp(thr),)
    # each hit's own record: its two ids and its query's residues
    q_len = np.diff(q_seq_off)
    qi = np.clip(hits["query"].astype(np.int64), 0, max(len(q_len) - 1, 0))
    est = _per_hit_estimate(hits, q[4], t[4], q_len[qi] + 4 if len(hits) and len(q_len) else 0)
    return _call_twice(lib.pw_trimmed_fasta, head, tail, est)


class DefaultFormatter(object):
    """TXT output (Formatters.py:3-47)."""

    record = staticmethod(txt_record)

    def __init__(self, logger, hitlist, outputfile):
        self.logger = logger
        self.hitlist = hitlist
        self.outputfile = outputfile

    def lines(self):
        return [self.record(h) for h in ordered_hits(self.hitlist)]

    def print_results(self):
        with open(self.outputfile, "w") as out:
            for line in self.lines():
                out.write(line + "\n")


class TrimmerFormatter(DefaultFormatter):
    """trimmedFasta output (Formatters.py:110-150)."""

    record = staticmethod(trimmed_record)


def sam_header_and_records(hits):
    """The @SQ lines (one per target id without its RC suffix, first seen
    first) and the alignment lines of `hits` in the given order
    (SamFormatter._format_hit, Formatters.py:67-83).  Hit.get_sam_line
    reverses an RC hit's alignment strings in place, as the reference does."""
    sq = {}
    records = []
    for h in hits:
        tid = h.get_target_id()
        if tid not in sq:
            sq[tid[:-3] if tid[-2:] == "RC" else tid] = h.get_sam_sq()
        records.append(h.get_sam_line())
    return list(sq.values()), records


class SamFormatter(DefaultFormatter):
    """SAM output (Formatters.py:51-106): the @HD line, one @SQ line per
    target, the @PG line, then one alignment line per hit in the formatter's
    order (query id, target id, score)."""

    HD = "@HD\tVN:1.4\tSO:unknown"
    PG = "@PG\tID:0\tPN:paswas\tVN:3.0"

    def lines(self):
        sq, records = sam_header_and_records(ordered_hits(self.hitlist))
        return [self.HD] + sq + [self.PG] + records


class FastaFormatter(DefaultFormatter):
    """FASTA output (Formatters.py:152-186, class FASTA): the whole query of
    every hit, in the formatter's order."""

    @staticmethod
    def record(hit):
        return hit.get_full_fasta()


FORMATTERS = {"TXT": DefaultFormatter, "SAM": SamFormatter, "TRIMMEDFASTA": TrimmerFormatter,
              "FASTA": FastaFormatter}


def formatter_for(out_format):
    """Formatter class of an --outputformat value (pypaswasall.py:58-72,150-164)."""
    from .exceptions import InvalidOptionException
    key = str(out_format).upper()
    if key not in FORMATTERS:
        raise InvalidOptionException("Invalid output format {0}.".format(out_format))
    return FORMATTERS[key]
