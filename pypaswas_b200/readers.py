"""Sequence records from FASTA / FASTQ, parsed in native code.

Mirrors pyPaSWAS/Core/Readers.py (BioPythonReader, :12-118) without
Biopython: pw_records_read / pw_records_parse (csrc/reader.cpp) parse the file,
take the records [start, end) of it, drop records outside 0 < len <=
limit_length (when limit_length > 0), upper-case the residues as SWSeqRecord
does, and can append the reverse complements (or reversed copies) and sort by
length, longest first (stable), all before a single Python object exists.  The
records come back packed -- residues with offsets, ids with offsets -- which is
what the engine takes (Engine.set_queries_packed / set_targets_packed); Python
SeqRecord objects are made only on request (RecordSet.records).

read_query_records / read_target_records restate the chain of
Pypaswas._get_query_sequences / _get_target_sequences (pypaswasall.py:98-124):
queries are sorted; targets of a DNA-RNA score get their reverse complements,
of a PALINDROME score are replaced by them, of an IRYS score get reversed
copies; then they are sorted.
"""
import ctypes

import numpy as np

from . import _native
from .exceptions import InvalidOptionException, ReaderException
from .records import SeqRecord

FORMATS = {"fasta": _native.PW_FORMAT_FASTA, "fastq": _native.PW_FORMAT_FASTQ}


class RecordSet(object):
    """Records in packed form, in their final order."""

    def __init__(self, residues, offsets, id_blob, id_offsets, dropped=0):
        self.residues = residues
        self.offsets = offsets
        self.id_blob = id_blob
        self.id_offsets = id_offsets
        self.dropped = int(dropped)
        self._ids = None
        self._records = None

    def __len__(self):
        return len(self.offsets) - 1

    @property
    def lengths(self):
        return np.diff(self.offsets)

    @property
    def ids(self):
        """The record ids as str (decoded once)."""
        if self._ids is None:
            text = self.id_blob.tobytes().decode("utf-8", errors="surrogateescape")
            if len(text) == len(self.id_blob):  # ASCII: byte offsets are character offsets
                o = self.id_offsets.tolist()
                self._ids = [text[o[k]:o[k + 1]] for k in range(len(self))]
            else:
                b = self.id_blob.tobytes()
                o = self.id_offsets.tolist()
                self._ids = [b[o[k]:o[k + 1]].decode("utf-8", errors="surrogateescape") for k in range(len(self))]
        return self._ids

    def seq(self, k):
        return self.residues[self.offsets[k]:self.offsets[k + 1]].tobytes().decode("latin-1")

    def records(self):
        """SeqRecord objects (the driver's record interface), made once."""
        if self._records is None:
            text = self.residues.tobytes().decode("latin-1")
            o = self.offsets.tolist()
            self._records = [SeqRecord(text[o[k]:o[k + 1]], i) for k, i in enumerate(self.ids)]
        return self._records


def concat(sets):
    """One RecordSet of several, in order (offsets shifted)."""
    if len(sets) == 1:
        return sets[0]
    res = np.concatenate([s.residues for s in sets]) if sets else np.zeros(0, np.uint8)
    blob = np.concatenate([s.id_blob for s in sets]) if sets else np.zeros(0, np.uint8)
    off, id_off = [np.zeros(1, np.int64)], [np.zeros(1, np.int64)]
    r0 = i0 = 0
    for s in sets:
        off.append(s.offsets[1:] + r0)
        id_off.append(s.id_offsets[1:] + i0)
        r0 += int(s.offsets[-1])
        i0 += int(s.id_offsets[-1])
    out = RecordSet(res, np.concatenate(off), blob, np.concatenate(id_off), sum(s.dropped for s in sets))
    if all(s._ids is not None for s in sets):
        out._ids = [i for s in sets for i in s._ids]
    return out


def _from_handle(lib, h):
    n, nres, nid, dropped = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
    try:
        lib.pw_records_sizes(h, ctypes.byref(n), ctypes.byref(nres), ctypes.byref(nid), ctypes.byref(dropped))
        res = np.empty(max(nres.value, 1), dtype=np.uint8)
        off = np.empty(n.value + 1, dtype=np.int64)
        ids = np.empty(max(nid.value, 1), dtype=np.uint8)
        id_off = np.empty(n.value + 1, dtype=np.int64)
        lib.pw_records_copy(h, res.ctypes.data, off.ctypes.data, ids.ctypes.data, id_off.ctypes.data)
    finally:
        lib.pw_records_free(h)
    return RecordSet(res[:nres.value], off, ids[:nid.value], id_off, dropped.value)


def _format_code(filetype):
    key = str(filetype).lower()
    if key not in FORMATS:
        raise InvalidOptionException("File type {0} is not read natively (fasta, fastq)".format(filetype))
    return FORMATS[key]


def _limit(limit_length):
    try:
        return int(limit_length)
    except (TypeError, ValueError):
        raise InvalidOptionException("Limitlength should be an int but is {0}".format(limit_length))


def read_records(source, filetype="fasta", start=0, end=None, limit_length=5000, transform=0, sort=True,
                 path_label=None, lib=None):
    """Records of a FASTA / FASTQ file path, or of `source` bytes.  Raises
    ReaderException when [start, end) holds no record (Readers.py:105-106)."""
    lib = lib if lib is not None else _native.load_library()
    fmt = _format_code(filetype)
    limit = _limit(limit_length)
    err = ctypes.create_string_buffer(512)
    h = ctypes.c_void_p()
    e = -1 if end is None else int(end)
    if isinstance(source, (bytes, bytearray, memoryview)):
        buf = np.frombuffer(bytes(source), dtype=np.uint8) if not isinstance(source, bytes) else \
            np.frombuffer(source, dtype=np.uint8)
        rc = lib.pw_records_parse(buf.ctypes.data if len(buf) else None, len(buf), fmt, int(start), e, limit,
                                  int(transform), int(bool(sort)), ctypes.byref(h), err, len(err))
        label = path_label or "<bytes>"
    else:
        rc = lib.pw_records_read(str(source).encode(), fmt, int(start), e, limit, int(transform), int(bool(sort)),
                                 ctypes.byref(h), err, len(err))
        label = str(source)
    if rc != _native.PW_OK:
        raise InvalidOptionException(err.value.decode() or "reading {0} failed".format(label))
    rs = _from_handle(lib, h)
    if len(rs) == 0 and rs.dropped == 0:
        raise ReaderException("No (more) sequence data found in input file ({}), of file type {}.".format(
            label, filetype))
    return rs


def _transform_for(score):
    """Target transform of a scoring model (pypaswasall.py:113-118)."""
    st = getattr(score, "score_type", "")
    if st == "DNA_RNA":
        return _native.PW_RECORDS_APPEND_RC
    if st == "PALINDROME":
        return _native.PW_RECORDS_RC_ONLY
    if st == "IRYS":
        return _native.PW_RECORDS_APPEND_REVERSED
    return _native.PW_RECORDS_AS_READ


def read_query_records(settings, source, start=0, end=None, logger=None):
    """Pypaswas._get_query_sequences: read, limit, sort (pypaswasall.py:98-106)."""
    rs = read_records(source, getattr(settings, "filetype1", "fasta"), start, end,
                      getattr(settings, "limit_length", 5000), _native.PW_RECORDS_AS_READ, True)
    _log_dropped(logger, rs, settings)
    return rs


def read_target_records(settings, score, source, start=0, end=None, logger=None):
    """Pypaswas._get_target_sequences: read, limit, the score's transform,
    sort (pypaswasall.py:108-124)."""
    rs = read_records(source, getattr(settings, "filetype2", "fasta"), start, end,
                      getattr(settings, "limit_length", 5000), _transform_for(score), True)
    _log_dropped(logger, rs, settings)
    return rs


def _log_dropped(logger, rs, settings):
    if logger is not None and rs.dropped > 0:
        logger.info("{} sequence(s) removed with length > limit_length ({}bp)".format(
            rs.dropped, getattr(settings, "limit_length", "")))


class NativeReader(object):
    """BioPythonReader's interface (Readers.py:12-118) on the native parser:
    read_records, complement_records, complement_records_only,
    reverse_records, sort_records, get_records.  The transforms run on the
    packed records (vectorised); get_records returns SeqRecord objects."""

    def __init__(self, logger, path, filetype, limitlength=5000):
        self.logger = logger
        self.path = path
        self.filetype = filetype
        self.rc_string = "_RC"
        self.limitlength = _limit(limitlength)
        self.set = None

    def read_records(self, start=0, end=None):
        self.set = read_records(self.path, self.filetype, start, end, self.limitlength,
                                _native.PW_RECORDS_AS_READ, False)
        _log_dropped(self.logger, self.set, type("S", (), {"limit_length": self.limitlength})())

    def _append(self, residues, keep_originals):
        s = self.set
        n = len(s)
        ids = s.id_blob.tobytes()
        suffix = self.rc_string.encode()
        new_ids = b"".join(ids[s.id_offsets[k]:s.id_offsets[k + 1]] + suffix for k in range(n))
        id_lens = np.diff(s.id_offsets) + len(suffix)
        if keep_originals:
            res = np.concatenate([s.residues, residues])
            off = np.concatenate([s.offsets, s.offsets[1:] + s.offsets[-1]])
            blob = np.frombuffer(ids + new_ids, dtype=np.uint8)
            id_off = np.concatenate([s.id_offsets, np.cumsum(id_lens) + s.id_offsets[-1]])
        else:
            res, off = residues, s.offsets.copy()
            blob = np.frombuffer(new_ids, dtype=np.uint8)
            id_off = np.concatenate([[0], np.cumsum(id_lens)]).astype(np.int64)
        self.set = RecordSet(res, off, blob, id_off, s.dropped)

    def _reversed_residues(self):
        s = self.set
        lens = np.diff(s.offsets)
        rec = np.repeat(np.arange(len(s)), lens)
        pos = np.arange(len(s.residues), dtype=np.int64)
        # position p of record r reads position off[r] + off[r + 1] - 1 - p
        return s.residues[(s.offsets[:-1] + s.offsets[1:] - 1)[rec] - pos]

    def complement_records(self):
        self._append(self._rc(), True)

    def _rc(self):
        from .workloads import _COMPLEMENT
        table = np.frombuffer(_COMPLEMENT, dtype=np.uint8)
        return table[self._reversed_residues()]

    def complement_records_only(self):
        self._append(self._rc(), False)

    def reverse_records(self):
        self._append(self._reversed_residues(), True)

    def sort_records(self, reverse=True):
        s = self.set
        lens = np.diff(s.offsets)
        order = np.argsort(-lens if reverse else lens, kind="stable")
        self.set = _reorder(s, order)

    def get_records(self):
        return self.set.records()


def _reorder(s, order):
    lens = np.diff(s.offsets)[order]
    starts = s.offsets[:-1][order]
    rec = np.repeat(np.arange(len(order)), lens)
    off = np.zeros(len(order) + 1, dtype=np.int64)
    np.cumsum(lens, out=off[1:])
    res = s.residues[starts[rec] + np.arange(off[-1], dtype=np.int64) - off[:-1][rec]] if off[-1] else \
        s.residues[:0]
    id_lens = np.diff(s.id_offsets)[order]
    id_starts = s.id_offsets[:-1][order]
    irec = np.repeat(np.arange(len(order)), id_lens)
    id_off = np.zeros(len(order) + 1, dtype=np.int64)
    np.cumsum(id_lens, out=id_off[1:])
    blob = s.id_blob[id_starts[irec] + np.arange(id_off[-1], dtype=np.int64) - id_off[:-1][irec]] if id_off[-1] \
        else s.id_blob[:0]
    return RecordSet(res, off, blob, id_off, s.dropped)
